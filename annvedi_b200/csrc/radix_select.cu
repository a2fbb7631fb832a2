// Per-query radix selection: the R smallest keys of a long stream, as an unsorted set, or just the
// R-th smallest key (a bar).
//
// Used where only the set of the best R matters (the candidates an exact FP32 re-rank will sort) or
// only a bar. One CTA per query: histogram passes over the order-preserving integer image of the float
// keys (11, 11 and 10 bits) narrow down the R-th smallest key t; a final pass collects every key < t
// and, in stream order, as many keys == t as fill the set to R. Each pass reads the query's keys once
// (coalesced); histograms live in shared memory. A second rank R2 can be resolved in the same passes
// (a second histogram follows its own prefix). With kth_upper set and no set wanted, two passes
// suffice: the bar reported is the upper edge of the 22-bit bin that holds the R-th key, which is at or
// above that key and within 2^-13 of it relative to the key.
#include "common.cuh"
#include "ivf.cuh"
#include "radix_select.cuh"

namespace annb {

namespace {

__device__ __forceinline__ uint32_t ord(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unord(uint32_t t) {
    const float f = __uint_as_float((t & 0x80000000u) ? (t & 0x7fffffffu) : ~t);
    return isnan(f) ? kInf : f;
}

constexpr int kThreads = 256;
constexpr int kBins = 2048;

// The bin holding the rank-th smallest (0-based) element of the histogram, and the count of elements
// in lower bins. Whole block.
__device__ int find_bin(const int* hist, int rank, int* below, int* sScan) {
    constexpr int per = kBins / kThreads;
    int local = 0;
#pragma unroll
    for (int i = 0; i < per; ++i) local += hist[threadIdx.x * per + i];
    sScan[threadIdx.x] = local;
    __syncthreads();
    for (int off = 1; off < kThreads; off <<= 1) {
        const int v = threadIdx.x >= off ? sScan[threadIdx.x - off] : 0;
        __syncthreads();
        sScan[threadIdx.x] += v;
        __syncthreads();
    }
    const int incl = sScan[threadIdx.x];
    const int excl = incl - local;
    __shared__ int sBin, sBelow;
    if (rank >= excl && rank < incl) {
        int c = excl;
#pragma unroll
        for (int i = 0; i < per; ++i) {
            const int h = hist[threadIdx.x * per + i];
            if (rank < c + h) {
                sBin = threadIdx.x * per + i;
                sBelow = c;
                break;
            }
            c += h;
        }
    }
    __syncthreads();
    *below = sBelow;
    const int bin = sBin;
    __syncthreads();
    return bin;
}

// The bin holding the rank-th smallest (0-based) element of a kBins histogram, by a warp-shuffle block
// scan (two barriers). Whole block; every thread gets the bin. sScan: >= kThreads / 32 + 1 ints.
__device__ int find_bin_scan(const int* hist, int rank, int* sScan, int* below = nullptr) {
    constexpr int per = kBins / kThreads;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int local = 0;
#pragma unroll
    for (int i = 0; i < per; ++i) local += hist[threadIdx.x * per + i];
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) sScan[warp] = incl;
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; ++w) before += sScan[w];
    incl += before;
    const int excl = incl - local;
    if (rank >= excl && rank < incl) {
        int c = excl;
        for (int i = 0; i < per; ++i) {
            const int h = hist[threadIdx.x * per + i];
            if (rank < c + h) {
                sScan[kThreads / 32] = threadIdx.x * per + i;
                sScan[kThreads / 32 + 1] = c;  // elements in lower bins
                break;
            }
            c += h;
        }
    }
    __syncthreads();
    if (below) *below = sScan[kThreads / 32 + 1];
    return sScan[kThreads / 32];
}

__device__ __forceinline__ int lin_bin(float k, float lo, float scale) {
    const float f = (k - lo) * scale;  // NaN (0 * inf) counts as bin 0
    return !(f > 0.f) ? 0 : (f >= (float)(kBins - 1) ? kBins - 1 : (int)f);
}

// Block-wide bitonic sort of n (a power of two) (key, val) pairs in shared memory by (key, val).
__device__ void block_sort_pairs(float* key, int* val, int n) {
    for (int size = 2; size <= n; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < (n >> 1); t += kThreads) {
                const int lo = 2 * t - (t & (stride - 1));
                const int hi = lo + stride;
                const bool asc = (lo & size) == 0;
                const float kl = key[lo], kh = key[hi];
                const int vl = val[lo], vh = val[hi];
                if (asc ? pair_less(kh, vh, kl, vl) : pair_less(kl, vl, kh, vh)) {
                    key[lo] = kh;
                    key[hi] = kl;
                    val[lo] = vh;
                    val[hi] = vl;
                }
            }
            __syncthreads();
        }
    }
}

// Block-wide min and max (kThreads threads); the results are visible to every thread on return.
__device__ void block_minmax(float& lo, float& hi, float* sRed) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sRed[warp] = lo;
        sRed[32 + warp] = hi;
    }
    __syncthreads();
    lo = kInf;
    hi = -kInf;
    for (int w = 0; w < kThreads / 32; ++w) {
        lo = fminf(lo, sRed[w]);
        hi = fmaxf(hi, sRed[32 + w]);
    }
    __syncthreads();
}

constexpr int kTieCap = 256;   // pairs of a sampled set's boundary bin sorted by one warp
constexpr int kLinCap = 2048;  // keys sorted in shared memory (the final sub-bin, or a sampled bar's set)
constexpr int kSamples = 1024; // keys of the stream sampled for a bar
constexpr int kLoadBatch = 8;   // keys per thread loaded ahead of their use

// f(p, key) for every position p < len of the stream (each thread a strided share), with kLoadBatch
// loads in flight per thread.
template <typename F>
__device__ __forceinline__ void for_each_key(const float* __restrict__ kq, int64_t len, F&& f) {
    for (int64_t base = threadIdx.x; base < len; base += (int64_t)kLoadBatch * kThreads) {
        float v[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int64_t p = base + (int64_t)u * kThreads;
            v[u] = p < len ? kq[p] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int64_t p = base + (int64_t)u * kThreads;
            if (p < len) f(p, v[u]);
        }
    }
}

__global__ void __launch_bounds__(kThreads) radix_select_kernel(RadixSelectArgs a) {
    __shared__ int hist[2][kBins];
    __shared__ float sCandK[kLinCap];
    __shared__ int sCandP[kLinCap];
    __shared__ float sRed[64];
    __shared__ int sScan[kThreads];
    __shared__ int sCount, sTies;
    __shared__ float sTieK[kTieCap];
    __shared__ int sTieP[kTieCap];
    const int q = blockIdx.x;
    const int64_t off = a.offs ? a.offs[q] : (int64_t)q * a.ld;
    int64_t len = a.lens ? a.lens[q] : a.ld;
    if (a.lens32) len = min((int64_t)a.lens32[q], a.ld);
    const float* kq = a.keys + off;
    const int R = a.R;
    const int64_t orow = a.out_rows ? a.out_rows[q] : q;
    float* ok = a.out_key ? a.out_key + orow * R : nullptr;
    int* oi = a.out_id ? a.out_id + orow * R : nullptr;
    const bool two = a.out_kth2 != nullptr;
    const bool want_set = ok || oi;

    auto id_of = [&](int64_t p) -> int {
        if (a.ids) return a.ids[off + p];
        if (a.use_plan) return (int)plan_row(a.plan, q, p);
        return (int)p;
    };

    if (len <= R && (!two || len <= a.R2)) {  // everything is in the set; no bar below +inf
        for (int64_t p = threadIdx.x; p < R && want_set; p += kThreads) {
            const bool v = p < len;
            if (ok) ok[p] = v ? kq[p] : kInf;
            if (oi) oi[p] = v ? id_of(p) : kNoId;
        }
        if (threadIdx.x == 0) {
            if (a.out_kth) a.out_kth[orow] = kInf;
            if (two) a.out_kth2[orow] = kInf;
        }
        return;
    }
    if (want_set && !two && !a.kth_upper && (int64_t)R * 8 <= len && R <= 512) {
        // Sampled bar: every s-th key, the bar at the ~1.3 R / s-th smallest sample; one pass gathers
        // the keys at or below it with their positions, and if there are at least R of them (the R
        // smallest keys then all are), the set is resolved among them exactly (below).
        const int64_t sstep = max((int64_t)1, len / kSamples);
        const int ns = (int)min((int64_t)kSamples, (len + sstep - 1) / sstep);
        const int r = min(ns, (int)(((int64_t)R * 13 + 10 * sstep - 1) / (10 * sstep)) + 4);
        // the bar: the linear bin (2,048 over the samples' [min, max]) holding the r-th smallest sample;
        // the gather below keeps every key of that bin or a lower one (the same bin function), so at
        // least r samples' worth of keys pass, and few more (about half a sample per bin)
        constexpr int kPer = kSamples / kThreads;
        float sv[kPer];
        float slo = kInf, shi = -kInf;
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int i = threadIdx.x + u * kThreads;
            sv[u] = i < ns ? kq[(int64_t)i * sstep] : kInf;
            if (i < ns) {
                slo = fminf(slo, sv[u]);
                shi = fmaxf(shi, sv[u]);
            }
        }
        for (int i = threadIdx.x; i < kBins; i += kThreads) hist[0][i] = 0;
        if (threadIdx.x == 0) sCount = 0;
        block_minmax(slo, shi, sRed);  // (its barriers also publish the zeroed bins)
        const float sscale = (float)kBins / (shi - slo);
        const bool spread = shi > slo && isfinite(sscale);
        if (spread) {
#pragma unroll
            for (int u = 0; u < kPer; ++u)
                if (threadIdx.x + u * kThreads < ns) atomicAdd(&hist[0][lin_bin(sv[u], slo, sscale)], 1);
        }
        __syncthreads();
        const int bb = spread ? find_bin_scan(hist[0], r - 1, sScan) : kBins - 1;
        for_each_key(kq, len, [&](int64_t p, float kv) {
            if (lin_bin(kv, slo, sscale) <= bb || !spread) {
                const int at = atomicAdd(&sCount, 1);
                if (at < kLinCap) {
                    sCandK[at] = kv;
                    sCandP[at] = (int)p;
                }
            }
        });
        __syncthreads();
        const int cnt = sCount;
        if (cnt >= R && cnt <= kLinCap) {
            // The set (unordered) of the R smallest of the cnt gathered pairs: linear bins over their range;
            // every pair in a bin below the one holding the R-th is in, and that bin's pairs (few) are
            // sorted by (key, position) by one warp to fill the set. Equal keys throughout, or a crowded
            // boundary bin, take the full sort below.
            float clo = kInf, chi = -kInf;
            for (int e = threadIdx.x; e < cnt; e += kThreads) {
                clo = fminf(clo, sCandK[e]);
                chi = fmaxf(chi, sCandK[e]);
            }
            for (int i = threadIdx.x; i < kBins; i += kThreads) hist[1][i] = 0;
            block_minmax(clo, chi, sRed);  // its barriers also order every read of sCount before the resets
            const float csc = (float)kBins / (chi - clo);
            if (chi > clo && isfinite(csc)) {
                if (threadIdx.x == 0) {
                    sCount = 0;
                    sTies = 0;
                }
                for (int e = threadIdx.x; e < cnt; e += kThreads) atomicAdd(&hist[1][lin_bin(sCandK[e], clo, csc)], 1);
                __syncthreads();
                int below = 0;
                const int bb = find_bin_scan(hist[1], R - 1, sScan, &below);
                const int nb = hist[1][bb];
                if (nb <= kTieCap) {
                    for (int e = threadIdx.x; e < cnt; e += kThreads) {
                        const float kv = sCandK[e];
                        const int bin = lin_bin(kv, clo, csc);
                        if (bin < bb) {
                            const int slot = atomicAdd(&sCount, 1);
                            if (ok) ok[slot] = kv;
                            if (oi) oi[slot] = id_of(sCandP[e]);
                        } else if (bin == bb) {
                            const int at = atomicAdd(&sTies, 1);
                            sTieK[at] = kv;
                            sTieP[at] = sCandP[e];
                        }
                    }
                    __syncthreads();
                    if (threadIdx.x < 32) {
                        int cap2 = 32;
                        while (cap2 < nb) cap2 <<= 1;
                        for (int e = nb + threadIdx.x; e < cap2; e += 32) {
                            sTieK[e] = kInf;
                            sTieP[e] = INT_MAX;
                        }
                        __syncwarp();
                        warp_sort_smem(sTieK, sTieP, cap2);
                        for (int e = threadIdx.x; e < R - below; e += 32) {
                            if (ok) ok[below + e] = sTieK[e];
                            if (oi) oi[below + e] = id_of(sTieP[e]);
                        }
                    }
                    return;
                }
            }
            __syncthreads();
            int cap2 = 32;
            while (cap2 < cnt) cap2 <<= 1;
            for (int e = cnt + threadIdx.x; e < cap2; e += kThreads) {
                sCandK[e] = kInf;
                sCandP[e] = INT_MAX;
            }
            __syncthreads();
            block_sort_pairs(sCandK, sCandP, cap2);
            for (int e = threadIdx.x; e < R; e += kThreads) {
                if (ok) ok[e] = sCandK[e];
                if (oi) oi[e] = id_of(sCandP[e]);
            }
            return;
        }
        __syncthreads();  // too few or too many under the bar: the linear bins below
    }
    if (want_set && !two && !a.kth_upper) {
        // Linear bins over the stream's [min, max]: keys of similar magnitude spread over many bins
        // (the integer image's top bits would put them all in one, serialising the histogram).
        float lo = kInf, hi = -kInf;
        for_each_key(kq, len, [&](int64_t, float kv) {
            lo = fminf(lo, kv);
            hi = fmaxf(hi, kv);
        });
        block_minmax(lo, hi, sRed);
        const float scale1 = (float)kBins / (hi - lo);
        if (!(hi > lo) || !isfinite(scale1)) {  // all keys equal: the first R in stream order
            for (int64_t p = threadIdx.x; p < R; p += kThreads) {
                if (ok) ok[p] = kq[p];
                if (oi) oi[p] = id_of(p);
            }
            return;
        }
        for (int i = threadIdx.x; i < kBins; i += kThreads) {
            hist[0][i] = 0;
            hist[1][i] = 0;
        }
        __syncthreads();
        for_each_key(kq, len, [&](int64_t, float kv) { atomicAdd(&hist[0][lin_bin(kv, lo, scale1)], 1); });
        __syncthreads();
        int below1 = 0, below2 = 0;
        const int b1 = find_bin(hist[0], R - 1, &below1, sScan);
        const float w = (hi - lo) / (float)kBins;
        const float lo2 = lo + w * (float)b1;
        const float scale2 = (float)kBins / w;
        for_each_key(kq, len, [&](int64_t, float kv) {
            if (lin_bin(kv, lo, scale1) == b1) atomicAdd(&hist[1][lin_bin(kv, lo2, scale2)], 1);
        });
        __syncthreads();
        const int b2 = find_bin(hist[1], R - 1 - below1, &below2, sScan);
        const int ncand = hist[1][b2];
        const int fixed = below1 + below2;  // keys certainly in the set
        if (ncand <= kLinCap) {
            if (threadIdx.x == 0) {
                sCount = 0;
                sTies = 0;
            }
            __syncthreads();
            // keys below the final sub-bin go straight to the set; the final sub-bin's keys (few: the
            // sub-bin is 2^-22 of the range) are gathered with their positions and sorted below, so
            // their gathering order does not matter
            for_each_key(kq, len, [&](int64_t p, float kv) {
                const int bk = lin_bin(kv, lo, scale1);
                const int sk = bk == b1 ? lin_bin(kv, lo2, scale2) : -1;
                if (bk < b1 || (bk == b1 && sk < b2)) {
                    const int slot = atomicAdd(&sCount, 1);
                    if (ok) ok[slot] = kv;
                    if (oi) oi[slot] = id_of(p);
                } else if (bk == b1 && sk == b2) {
                    const int at = atomicAdd(&sTies, 1);
                    sCandK[at] = kv;
                    sCandP[at] = (int)p;
                }
            });
            __syncthreads();
            // the sub-bin's keys by (key, stream position); the first `need` complete the set
            if (threadIdx.x < 32) {
                int cap2 = 32;
                while (cap2 < ncand) cap2 <<= 1;
                for (int e = ncand + threadIdx.x; e < cap2; e += 32) {
                    sCandK[e] = kInf;
                    sCandP[e] = INT_MAX;
                }
                __syncwarp();
                warp_sort_smem(sCandK, sCandP, cap2);
            }
            __syncthreads();
            const int need = R - fixed;
            for (int e = threadIdx.x; e < need; e += kThreads) {
                if (ok) ok[fixed + e] = sCandK[e];
                if (oi) oi[fixed + e] = id_of(sCandP[e]);
            }
            return;
        }
        __syncthreads();  // more equal keys than the buffer holds: the exact integer radix below
    }
    const int npass = (a.kth_upper && !want_set) ? 2 : 3;
    uint32_t prefix[2] = {0, 0}, mask = 0;
    int rank[2] = {(int)min((int64_t)R, len) - 1, two ? (int)min((int64_t)a.R2, len) - 1 : 0};
    int below_total = 0;
    for (int pass = 0; pass < npass; ++pass) {
        const int sh = pass == 0 ? 21 : (pass == 1 ? 10 : 0);
        const uint32_t dmask = pass == 2 ? 0x3FFu : 0x7FFu;
        for (int i = threadIdx.x; i < kBins; i += kThreads) {
            hist[0][i] = 0;
            hist[1][i] = 0;
        }
        __syncthreads();
        for (int64_t p = threadIdx.x; p < len; p += kThreads) {
            const uint32_t o = ord(kq[p]);
            if ((o & mask) == prefix[0]) atomicAdd(&hist[0][(o >> sh) & dmask], 1);
            if (two && (o & mask) == prefix[1]) atomicAdd(&hist[1][(o >> sh) & dmask], 1);
        }
        __syncthreads();
        for (int j = 0; j < (two ? 2 : 1); ++j) {
            int below = 0;
            const int bin = find_bin(hist[j], rank[j], &below, sScan);
            rank[j] -= below;
            if (j == 0) below_total += below;
            prefix[j] |= (uint32_t)bin << sh;
        }
        mask |= dmask << sh;
    }
    const uint32_t low = npass == 2 ? 0x3FFu : 0u;  // upper edge of the last bin
    if (threadIdx.x == 0) {
        if (a.out_kth) a.out_kth[orow] = len >= R ? unord(prefix[0] | low) : kInf;
        if (two) a.out_kth2[orow] = len >= a.R2 ? unord(prefix[1] | low) : kInf;
    }
    if (!want_set) return;
    // collect: all keys < t, then keys == t in stream order (a block scan per chunk) up to R; fewer
    // than R keys: all, padded
    const uint32_t t = prefix[0];
    const int need_ties = R - below_total;
    __shared__ int sWarpTies[kThreads / 32];
    if (threadIdx.x == 0) {
        sCount = 0;
        sTies = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t base = 0; base < len; base += kThreads) {
        const int64_t p = base + threadIdx.x;
        const bool valid = p < len;
        const float kv = valid ? kq[p] : 0.f;
        const uint32_t o = ord(kv);
        const bool tie = valid && o == t;
        if (valid && o < t) {
            const int slot = atomicAdd(&sCount, 1);
            if (ok) ok[slot] = kv;
            if (oi) oi[slot] = id_of(p);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, tie);
        if (__syncthreads_or(bal != 0)) {  // uniform: some tie in this chunk
            if (lane == 0) sWarpTies[warp] = __popc(bal);
            __syncthreads();
            int before = sTies;
            for (int w = 0; w < warp; ++w) before += sWarpTies[w];
            const int rank = before + __popc(bal & ((1u << lane) - 1u));
            if (tie && rank < need_ties) {
                if (ok) ok[below_total + rank] = kv;
                if (oi) oi[below_total + rank] = id_of(p);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                int tot = 0;
                for (int w = 0; w < kThreads / 32; ++w) tot += sWarpTies[w];
                sTies += tot;
            }
            __syncthreads();
        }
    }
    for (int64_t p = len + threadIdx.x; p < R; p += kThreads) {
        if (ok) ok[p] = kInf;
        if (oi) oi[p] = kNoId;
    }
}

// ---- bars from a resident row of sampled keys ----------------------------------------------------
// One CTA per query holds its S keys in shared memory. Level 1: 2048 linear bins over [min, max]; the
// bins holding the r1-th and r2-th smallest keys are found; level 2 splits each of those bins into 2048
// linear sub-bins. The bar is the largest key of the bins at or below the chosen (bin, sub-bin): the
// binning is monotone in the key, so exactly the keys <= that bar are counted below it, at least r of
// them (a bar at or above the r-th smallest key, within a sub-bin of it).
constexpr int kBarThreads = 1024;


// rank-th smallest (0-based) bin of a histogram over kBins, kBarThreads threads.
__device__ int find_bin_bar(const int* hist, int rank, int* below, int* sScan) {
    constexpr int per = kBins / kBarThreads;
    int local = 0;
#pragma unroll
    for (int i = 0; i < per; ++i) local += hist[threadIdx.x * per + i];
    sScan[threadIdx.x] = local;
    __syncthreads();
    for (int off = 1; off < kBarThreads; off <<= 1) {
        const int v = threadIdx.x >= off ? sScan[threadIdx.x - off] : 0;
        __syncthreads();
        sScan[threadIdx.x] += v;
        __syncthreads();
    }
    const int incl = sScan[threadIdx.x];
    const int excl = incl - local;
    __shared__ int sBin, sBelow;
    if (rank >= excl && rank < incl) {
        int c = excl;
#pragma unroll
        for (int i = 0; i < per; ++i) {
            const int h = hist[threadIdx.x * per + i];
            if (rank < c + h) {
                sBin = threadIdx.x * per + i;
                sBelow = c;
                break;
            }
            c += h;
        }
    }
    __syncthreads();
    *below = sBelow;
    const int bin = sBin;
    __syncthreads();
    return bin;
}

__device__ float block_reduce(float v, bool is_max, float* sRed) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float w = __shfl_xor_sync(0xffffffffu, v, o);
        v = is_max ? fmaxf(v, w) : fminf(v, w);
    }
    if ((threadIdx.x & 31) == 0) sRed[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = sRed[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float w = __shfl_xor_sync(0xffffffffu, v, o);
            v = is_max ? fmaxf(v, w) : fminf(v, w);
        }
        if (threadIdx.x == 0) sRed[32] = v;
    }
    __syncthreads();
    const float r = sRed[32];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kBarThreads) sample_bars_kernel(const float* __restrict__ keys, int S, int r1,
                                                                  int r2, float* bar1, float* bar2) {
    extern __shared__ __align__(16) float sK[];  // [S]
    __shared__ int hist[2][kBins];
    __shared__ uint32_t smax[2][kBins];          // ordered image of the largest key per level-2 bin
    __shared__ int sScan[kBarThreads];
    __shared__ float sRed[33];
    const int q = blockIdx.x;
    const float4* src = reinterpret_cast<const float4*>(keys + (int64_t)q * S);
    float4* sK4 = reinterpret_cast<float4*>(sK);
    const int S4 = S / 4;
    float lo = kInf, hi = -kInf;
    constexpr int kLoadBatch = 8;  // loads issued before the first is used
    for (int i0 = threadIdx.x; i0 < S4; i0 += kLoadBatch * kBarThreads) {
        float4 v[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int i = i0 + u * kBarThreads;
            if (i < S4) v[u] = __ldcs(src + i);
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int i = i0 + u * kBarThreads;
            if (i < S4) {
                sK4[i] = v[u];
                lo = fminf(lo, fminf(fminf(v[u].x, v[u].y), fminf(v[u].z, v[u].w)));
                hi = fmaxf(hi, fmaxf(fmaxf(v[u].x, v[u].y), fmaxf(v[u].z, v[u].w)));
            }
        }
    }
    for (int i = threadIdx.x; i < kBins; i += kBarThreads) {
        hist[0][i] = 0;
        hist[1][i] = 0;
        smax[0][i] = 0;
        smax[1][i] = 0;
    }
    lo = block_reduce(lo, false, sRed);  // (synchronises, so the stores above are visible)
    hi = block_reduce(hi, true, sRed);
    const int rank[2] = {min(r1, S) - 1, min(r2, S) - 1};
    if (!(hi > lo) || !isfinite((float)kBins / (hi - lo))) {  // all keys equal, or a range too narrow to bin
        if (threadIdx.x == 0) {
            bar1[q] = hi;
            bar2[q] = hi;
        }
        return;
    }
    const float scale1 = (float)kBins / (hi - lo);
    for (int i = threadIdx.x; i < S4; i += kBarThreads) {
        const float4 v = sK4[i];
        atomicAdd(&hist[0][lin_bin(v.x, lo, scale1)], 1);
        atomicAdd(&hist[0][lin_bin(v.y, lo, scale1)], 1);
        atomicAdd(&hist[0][lin_bin(v.z, lo, scale1)], 1);
        atomicAdd(&hist[0][lin_bin(v.w, lo, scale1)], 1);
    }
    __syncthreads();
    int b[2], rr[2];
    for (int j = 0; j < 2; ++j) {
        int below = 0;
        b[j] = find_bin_bar(hist[0], rank[j], &below, sScan);
        rr[j] = rank[j] - below;
    }
    for (int i = threadIdx.x; i < kBins; i += kBarThreads) hist[0][i] = 0;
    __syncthreads();
    // level 2 inside each chosen bin, with the largest key of every sub-bin
    const float w = (hi - lo) / (float)kBins;
    const float lo2[2] = {lo + w * (float)b[0], lo + w * (float)b[1]};
    const float scale2 = (float)kBins / w;
    for (int i = threadIdx.x; i < S; i += kBarThreads) {
        const float k = sK[i];
        const int bk = lin_bin(k, lo, scale1);
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            if (bk == b[j]) {
                const int sb = lin_bin(k, lo2[j], scale2);
                atomicAdd(&hist[j][sb], 1);
                atomicMax(&smax[j][sb], ord(k));
            }
        }
    }
    __syncthreads();
    for (int j = 0; j < 2; ++j) {
        int below = 0;
        const int sb = find_bin_bar(hist[j], rr[j], &below, sScan);
        // keys of bins below b[j], and of sub-bins below sb, are all smaller than those of sub-bin sb
        if (threadIdx.x == 0) (j ? bar2 : bar1)[q] = unord(smax[j][sb]);
    }
}

}  // namespace

size_t sample_bars_smem(int S) { return sizeof(float) * (size_t)S; }

int launch_sample_bars(const float* keys, int S, int nq, int r1, int r2, float* bar1, float* bar2, cudaStream_t st) {
    if (nq == 0) return ANN_OK;
    ANN_CHECK_ARG(S > 0 && S % 4 == 0 && sample_bars_smem(S) <= kSampleBarsMaxSmem && r1 >= 1 && r2 >= 1,
                  "sample bars: S=%d, ranks %d, %d", S, r1, r2);
    const int smem = (int)sample_bars_smem(S);
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(sample_bars_kernel)));
    sample_bars_kernel<<<nq, kBarThreads, smem, st>>>(keys, S, r1, r2, bar1, bar2);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_radix_select(const RadixSelectArgs& a, int nq, cudaStream_t st) {
    if (nq == 0) return ANN_OK;
    ANN_CHECK_ARG(a.R >= 1 && (a.out_kth2 == nullptr || a.R2 >= 1), "radix select: R=%d, R2=%d", a.R, a.R2);
    ANN_CHECK_ARG(a.keys != nullptr && a.ld >= 0, "radix select: no keys");
    radix_select_kernel<<<nq, kThreads, 0, st>>>(a);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

// Helpers of the tensor-core search around the GEMM: survivor grouping, bar check, re-run gather and
// the row order of the BF16 base copy.
#include <numeric>

#include "common.cuh"
#include "tc_search.cuh"

namespace annb {

int64_t tc_row_mult(int64_t n) {
    if (n <= 1) return 1;
    int64_t g = std::max<int64_t>(1, (int64_t)(0.6180339887498949 * (double)n));
    while (std::gcd(g, n) != 1) ++g;
    return g % n == 0 ? 1 : g;
}

namespace {

__device__ __forceinline__ int pos_to_row(int64_t p, int64_t n, int64_t mult) {
    return (int)(((unsigned __int128)p * (uint64_t)mult) % (uint64_t)n);
}

__global__ void tc_count_kernel(TcGroupArgs g) {
    const int w = blockIdx.x;
    const int cnt = min(g.wcount[w], g.wcap);
    const int64_t base = (int64_t)w * g.wcap;
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) atomicAdd(&g.rowcnt[g.frow[base + e]], 1);
}

// One block: exclusive scan of rowcnt into offs, cursors zeroed, largest warp count.
__global__ void __launch_bounds__(1024) tc_scan_kernel(TcGroupArgs g) {
    __shared__ int64_t sPart[1024];
    __shared__ int sMax[32];
    const int per = (g.M + 1023) / 1024;
    const int r0 = threadIdx.x * per;
    int64_t local = 0;
    for (int i = 0; i < per; ++i)
        if (r0 + i < g.M) local += g.rowcnt[r0 + i];
    sPart[threadIdx.x] = local;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int64_t v = threadIdx.x >= off ? sPart[threadIdx.x - off] : 0;
        __syncthreads();
        sPart[threadIdx.x] += v;
        __syncthreads();
    }
    int64_t run = sPart[threadIdx.x] - local;
    for (int i = 0; i < per; ++i) {
        const int r = r0 + i;
        if (r < g.M) {
            g.offs[r] = run;
            g.cursor[r] = 0;
            run += g.rowcnt[r];
        }
    }
    int m = 0;
    for (int w = threadIdx.x; w < g.nwarps; w += 1024) m = max(m, g.wcount[w]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sMax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        int r = 0;
        for (int i = 0; i < 32; ++i) r = max(r, sMax[i]);
        *g.max_wcount = r;
    }
}

__global__ void tc_scatter_kernel(TcGroupArgs g) {
    const int w = blockIdx.x;
    const int cnt = min(g.wcount[w], g.wcap);
    const int64_t base = (int64_t)w * g.wcap;
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
        const int row = g.frow[base + e];
        const int64_t at = g.offs[row] + atomicAdd(&g.cursor[row], 1);
        g.gkey[at] = g.fkey[base + e];
        g.gid[at] = pos_to_row(g.fcol[base + e], g.n, g.mult);
    }
}

__global__ void tc_bar_check_kernel(const int* rowcnt, int M, int R, int* list, int* flags, const int64_t* lens,
                                    int* mark) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= M) return;
    const int64_t need = lens ? min((int64_t)R, lens[q]) : (int64_t)R;
    const bool rerun = rowcnt[q] < need;
    if (rerun) list[atomicAdd(&flags[0], 1)] = q;
    if (mark) mark[q] = rerun;
}

__global__ void tc_gather_kernel(const unsigned char* A, int row_bytes, const int* list, int nb, const float* tau,
                                 unsigned char* A2, float* tau2, const float* rfac, float* rfac2) {
    const int j = blockIdx.x;
    if (j >= nb) return;
    const int q = list[j];
    const uint4* src = reinterpret_cast<const uint4*>(A + (size_t)q * row_bytes);
    uint4* dst = reinterpret_cast<uint4*>(A2 + (size_t)j * row_bytes);
    for (int c = threadIdx.x; c < row_bytes / 16; c += blockDim.x) dst[c] = src[c];
    if (threadIdx.x == 0) {
        tau2[j] = tau[q];
        if (rfac) rfac2[j] = rfac[q];
    }
}

__global__ void tc_map_ids_kernel(int* ids, int64_t count, int64_t n, int64_t mult) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const int p = ids[i];
        if (p != kNoId) ids[i] = pos_to_row(p, n, mult);
    }
}

__global__ void tc_unpermute_kernel(const float* keys, int64_t n, int64_t mult, float* out) {
    const int q = blockIdx.y;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        out[(int64_t)q * n + pos_to_row(p, n, mult)] = keys[(int64_t)q * n + p];
}

__global__ void __launch_bounds__(1024) tc_ivf_items_kernel(const int64_t* lq_off, const int64_t* list_off, int C,
                                                            int64_t* item_off, const int64_t* list_len) {
    __shared__ int64_t sPart[1024];
    const int per = (C + 1023) / 1024;
    const int l0 = threadIdx.x * per;
    auto items = [&](int l) -> int64_t {
        const int64_t np = lq_off[l + 1] - lq_off[l];
        const int64_t nr = list_len ? list_len[l] : list_off[l + 1] - list_off[l];
        return (np == 0 || nr == 0) ? 0 : ((np + 127) / 128) * ((nr + 255) / 256);
    };
    int64_t local = 0;
    for (int i = 0; i < per; ++i)
        if (l0 + i < C) local += items(l0 + i);
    sPart[threadIdx.x] = local;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int64_t v = threadIdx.x >= off ? sPart[threadIdx.x - off] : 0;
        __syncthreads();
        sPart[threadIdx.x] += v;
        __syncthreads();
    }
    int64_t run = sPart[threadIdx.x] - local;
    for (int i = 0; i < per; ++i) {
        const int l = l0 + i;
        if (l < C) {
            item_off[l] = run;
            run += items(l);
        }
    }
    if (threadIdx.x == 1023) item_off[C] = sPart[1023];
}

// one warp per pair
__global__ void tc_ivf_pairs_kernel(const unsigned char* qrows, int row_bytes, const int32_t* pair_vals,
                                    const int32_t* pair_lists, const int64_t* n_pairs, int64_t max_pairs, int npc,
                                    const int64_t* cand_off, const int64_t* seg_pref, const int64_t* list_off,
                                    unsigned char* A, int64_t* dbase, TcIvfSampleMaps sm) {
    const int64_t np = min(*n_pairs, max_pairs);
    const int lane = threadIdx.x & 31;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < np;
         i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int32_t v = pair_vals[i];
        const int q = v / npc, j = v % npc;
        const uint4* src = reinterpret_cast<const uint4*>(qrows + (size_t)q * row_bytes);
        uint4* dst = reinterpret_cast<uint4*>(A + (size_t)i * row_bytes);
        for (int c = lane; c < row_bytes / 16; c += 32) dst[c] = src[c];
        if (lane == 0) {
            if (sm.pfac) sm.pfac[i] = sm.qfac[q];
            if (dbase) dbase[i] = cand_off[q] + seg_pref[(int64_t)q * (npc + 1) + j] - list_off[pair_lists[i]];
            if (sm.row_query) sm.row_query[i] = q;
            // the grouped epilogue adds the tile's absolute list row, as for dbase
            if (sm.sdbase) sm.sdbase[i] = sm.soff[q] + sm.sseg[(int64_t)q * npc + j] - list_off[pair_lists[i]];
        }
    }
}

// One thread per query: the sample stream of its probed lists (the first lcap[l] rows of each), the
// segment starts sseg[q][j] and its length slen[q]; the candidates' count comes from the plan.
__global__ void tc_ivf_sample_plan_kernel(IvfPlan p, const int64_t* __restrict__ lcap, int64_t* __restrict__ sseg,
                                          int64_t* __restrict__ slen) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= p.nq) return;
    const int ns = p.n_seg[q];
    int64_t run = 0;
    for (int j = 0; j < p.npc; ++j) {
        sseg[(int64_t)q * p.npc + j] = run;
        const int l = p.probes[(int64_t)q * p.npc + j];
        if (j < ns && l >= 0) run += lcap[l];
    }
    slen[q] = run;
}

// One warp per query: the int8 weights of the SQ8 tensor-core key. w_d = -2 scale_d (q_d - offset_d), so that
// sum_d code_d * w_d + sum_d (code_d scale_d)^2 = the SQ8 distance - |q - offset|^2 (a per-query constant).
// a_d = rint(w_d * 127 / max|w|) as int8 (zero past dim), qfac = max|w| / 127 (1 for an all-zero w).
__global__ void tc_sq8_query_kernel(const float* __restrict__ q, int nq, int dim, int ldq,
                                    const float* __restrict__ scale, const float* __restrict__ offset,
                                    int8_t* __restrict__ out, int ldo, float* __restrict__ qfac) {
    const int qi = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (qi >= nq) return;
    const float* qr = q + (int64_t)qi * ldq;
    float mx = 0.f;
    for (int d = lane; d < dim; d += 32) mx = fmaxf(mx, fabsf(-2.f * scale[d] * (qr[d] - offset[d])));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const float alpha = mx > 0.f ? 127.f / mx : 1.f;
    for (int d = lane; d < ldo; d += 32) {
        float v = 0.f;
        if (d < dim) v = rintf(-2.f * scale[d] * (qr[d] - offset[d]) * alpha);
        out[(int64_t)qi * ldo + d] = (int8_t)fmaxf(-127.f, fminf(127.f, v));
    }
    if (lane == 0) qfac[qi] = 1.f / alpha;
}

// One warp per row: fac[i] = (1, sum_d (code_d scale_d)^2), the row's reconstructed squared norm.
__global__ void tc_sq8_norms_kernel(const uint8_t* __restrict__ codes, int64_t n, int dim, int ldc,
                                    const float* __restrict__ scale, float2* __restrict__ fac) {
    const int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    float s = 0.f;
    for (int d = lane; d < dim; d += 32) {
        const float x = (float)codes[i * ldc + d] * scale[d];
        s = fmaf(x, x, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) fac[i] = make_float2(1.f, s);
}

// ---- warp-level exact selection (one warp per query) -----------------------------------------------
__device__ __forceinline__ uint32_t ord_key(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ord(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

// The r-th smallest (1 <= r <= n) of keys[0..n) as an ordered key, by one warp: four passes of 8-bit digits
// from the top, each counting the keys that match the digits found so far into the warp's 256-bin
// histogram `hist` (shared memory). Exact; every lane returns it.
__device__ uint32_t warp_kth_ord(const float* __restrict__ keys, int64_t n, int64_t r, int* hist) {
    const int lane = threadIdx.x & 31;
    uint32_t prefix = 0, pmask = 0;
    int64_t rem = r;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = lane; i < 256; i += 32) hist[i] = 0;
        __syncwarp();
        for (int64_t p = lane; p < n; p += 32) {
            const uint32_t o = ord_key(keys[p]);
            if ((o & pmask) == prefix) atomicAdd(&hist[(o >> shift) & 255u], 1);
        }
        __syncwarp();
        int c[8];
        int sum = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            c[j] = hist[lane * 8 + j];
            sum += c[j];
        }
        int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - sum;
        const unsigned hit = __ballot_sync(0xffffffffu, excl < rem && rem <= incl);
        const int src = __ffs(hit) - 1;
        int d = 0, before = 0;
        if (lane == src) {
            int acc = excl;
            for (int j = 0; j < 8; ++j) {
                if (acc + c[j] >= rem) {
                    d = lane * 8 + j;
                    before = acc;
                    break;
                }
                acc += c[j];
            }
        }
        d = __shfl_sync(0xffffffffu, d, src);
        before = __shfl_sync(0xffffffffu, before, src);
        rem -= before;
        prefix |= (uint32_t)d << shift;
        pmask |= 255u << shift;
        __syncwarp();
    }
    return prefix;
}

// One warp per query: bar1 / bar2 = the r1-th / r2-th smallest of the query's keys[offs[q] .. + lens[q])
// (+inf where the stream is shorter).
__global__ void __launch_bounds__(256) warp_bars_kernel(const float* __restrict__ keys, const int64_t* __restrict__ offs,
                                                        const int64_t* __restrict__ lens, int nq, int r1, int r2,
                                                        float* __restrict__ bar1, float* __restrict__ bar2) {
    __shared__ int sHist[8][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x * 8 + warp;
    if (q >= nq) return;  // the whole warp
    const float* kq = keys + offs[q];
    const int64_t n = lens[q];
    const float b1 = r1 <= n ? from_ord(warp_kth_ord(kq, n, r1, sHist[warp])) : kInf;
    const float b2 = r2 <= n ? from_ord(warp_kth_ord(kq, n, r2, sHist[warp])) : kInf;
    if (lane == 0) {
        bar1[q] = b1;
        bar2[q] = b2;
    }
}

// The digit of rank `rem` (1-based) in a 256-bin histogram and the count of keys below that digit, on
// every lane of the warp.
__device__ __forceinline__ void warp_hist_pick(const int* hist, int64_t rem, int* digit, int* before) {
    const int lane = threadIdx.x & 31;
    int c[8];
    int sum = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        c[j] = hist[lane * 8 + j];
        sum += c[j];
    }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const int excl = incl - sum;
    const unsigned hit = __ballot_sync(0xffffffffu, excl < rem && rem <= incl);
    const int src = hit ? __ffs(hit) - 1 : 31;
    int d = 255, bf = 0;
    if (lane == src && hit) {
        int acc = excl;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (acc + c[j] >= rem) {
                d = lane * 8 + j;
                bf = acc;
                break;
            }
            acc += c[j];
        }
    }
    *digit = __shfl_sync(0xffffffffu, d, src);
    *before = __shfl_sync(0xffffffffu, bf, src);
}

// Adds one to hist[digit] for every lane whose key is valid, one atomic per distinct digit of the warp.
__device__ __forceinline__ void warp_hist_add(int* hist, bool valid, uint32_t digit) {
    const uint32_t key = valid ? digit : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (valid && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[digit], __popc(peers));
}

// One 128-thread block per query: bar1 / bar2 = the r1-th / r2-th smallest of keys[offs[q] .. + lens[q]) (+inf
// where the stream is shorter), both ranks' digits found in the same four 8-bit radix passes. A stream of at most
// `staged` keys is read once into shared memory (as ordered keys) and the passes run there; a longer one is read
// from global memory by every pass.
constexpr int kBarThreads = 128;
constexpr int kBarBins = 1024;   // linear bins of the staged form
constexpr int kBarBinCap = 256;  // keys of a rank's bin picked by counting; more fall back to radix passes

// The bin of rank `rank` (1-based) in hist[0..kBarBins) and the count of keys in lower bins, by one warp (each
// lane sums 32 consecutive bins, a warp scan, then the holding lane walks its bins). Every lane returns them.
__device__ __forceinline__ void warp_bin_pick(const int* hist, int rank, int* bin, int* before) {
    const int lane = threadIdx.x & 31;
    int sum = 0;
    for (int j = 0; j < kBarBins / 32; ++j) sum += hist[lane * (kBarBins / 32) + j];
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const int excl = incl - sum;
    const unsigned hit = __ballot_sync(0xffffffffu, excl < rank && rank <= incl);
    const int src = hit ? __ffs(hit) - 1 : 31;
    int b = kBarBins - 1, bf = 0;
    if (lane == src && hit) {
        int acc = excl;
        for (int j = 0; j < kBarBins / 32; ++j) {
            const int c = hist[lane * (kBarBins / 32) + j];
            if (acc + c >= rank) {
                b = lane * (kBarBins / 32) + j;
                bf = acc;
                break;
            }
            acc += c;
        }
    }
    *bin = __shfl_sync(0xffffffffu, b, src);
    *before = __shfl_sync(0xffffffffu, bf, src);
}
__global__ void __launch_bounds__(kBarThreads) block_bars_kernel(const float* __restrict__ keys,
                                                                 const int64_t* __restrict__ offs,
                                                                 const int64_t* __restrict__ lens, int nq, int r1,
                                                                 int r2, int staged, float* __restrict__ bar1,
                                                                 float* __restrict__ bar2) {
    extern __shared__ uint32_t smem_bars[];
    __shared__ int sHist[2][256];
    __shared__ int sPick[4];  // digit and count below it, per rank
    const int q = blockIdx.x;
    if (q >= nq) return;  // the whole block
    const int warp = threadIdx.x >> 5;
    const int64_t n = lens[q];
    const float* kq = keys + offs[q];
    const bool in_smem = n <= staged;
    if (in_smem)
        for (int64_t p = threadIdx.x; p < n; p += kBarThreads) smem_bars[p] = ord_key(kq[p]);
    const bool want1 = r1 <= n, want2 = r2 <= n;  // uniform across the block
    if (in_smem && n > 0 && (want1 || want2)) {
        // Linear bins over [min, max] of the staged keys. The bin of a key is monotone in the key, so a rank's key
        // lies in the bin where the running count reaches the rank; it is picked among that bin's keys by
        // counting, exactly. A bin holding more than kBarBinCap keys leaves the rank to the radix passes below.
        __shared__ int sBin[kBarBins];
        __shared__ uint32_t sList[2][kBarBinCap];
        __shared__ int sAux[8];  // [2..5] bin and count below per rank, [6,7] list sizes
        __shared__ float sRes[2];
        if (threadIdx.x == 0) sAux[6] = sAux[7] = 0;
        for (int i = threadIdx.x; i < kBarBins; i += kBarThreads) sBin[i] = 0;
        __syncthreads();  // also orders the staging above
        uint32_t omin = 0xffffffffu, omax = 0u;
        for (int64_t p = threadIdx.x; p < n; p += kBarThreads) {
            omin = min(omin, smem_bars[p]);
            omax = max(omax, smem_bars[p]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            omin = min(omin, __shfl_xor_sync(0xffffffffu, omin, o));
            omax = max(omax, __shfl_xor_sync(0xffffffffu, omax, o));
        }
        __shared__ uint32_t sMinMax[2];
        if (threadIdx.x == 0) {
            sMinMax[0] = 0xffffffffu;
            sMinMax[1] = 0u;
        }
        __syncthreads();
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&sMinMax[0], omin);
            atomicMax(&sMinMax[1], omax);
        }
        __syncthreads();
        const float lo = from_ord(sMinMax[0]), hi = from_ord(sMinMax[1]);
        const float scale = (float)kBarBins / (hi - lo);
        if (!(hi > lo) || !isfinite(scale)) {  // every key the same (or not finite): each rank's key is lo
            if (threadIdx.x == 0 && hi == lo) {
                bar1[q] = want1 ? lo : kInf;
                bar2[q] = want2 ? lo : kInf;
            }
            if (hi == lo) return;
        } else {
            auto bin_of = [&](uint32_t o) { return min(kBarBins - 1, (int)((from_ord(o) - lo) * scale)); };
            for (int64_t p = threadIdx.x; p < n; p += kBarThreads) atomicAdd(&sBin[bin_of(smem_bars[p])], 1);
            __syncthreads();
            if (warp < 2 && (warp == 0 ? want1 : want2)) {
                int b, bf;
                warp_bin_pick(sBin, warp == 0 ? r1 : r2, &b, &bf);
                if ((threadIdx.x & 31) == 0) {
                    sAux[2 + 2 * warp] = b;
                    sAux[3 + 2 * warp] = bf;
                }
            }
            __syncthreads();
            const bool fit1 = want1 && sBin[sAux[2]] <= kBarBinCap;
            const bool fit2 = want2 && sBin[sAux[4]] <= kBarBinCap;
            if ((!want1 || fit1) && (!want2 || fit2)) {  // uniform: both ranks settle here
                for (int64_t p = threadIdx.x; p < n; p += kBarThreads) {
                    const uint32_t o = smem_bars[p];
                    const int b = bin_of(o);
                    if (want1 && b == sAux[2]) sList[0][atomicAdd(&sAux[6], 1)] = o;
                    if (want2 && b == sAux[4]) sList[1][atomicAdd(&sAux[7], 1)] = o;
                }
                __syncthreads();
                for (int r = 0; r < 2; ++r) {
                    if (r == 0 ? !want1 : !want2) continue;
                    const int cnt = sAux[6 + r];
                    const int want = (r == 0 ? r1 : r2) - sAux[3 + 2 * r] - 1;  // 0-based rank inside the bin
                    for (int t = threadIdx.x; t < cnt; t += kBarThreads) {
                        const uint32_t v = sList[r][t];
                        int below = 0, equal_before = 0;
                        for (int u = 0; u < cnt; ++u) {
                            const uint32_t w = sList[r][u];
                            below += w < v;
                            equal_before += (w == v) && (u < t);
                        }
                        if (below + equal_before == want) sRes[r] = from_ord(v);
                    }
                }
                __syncthreads();
                if (threadIdx.x == 0) {
                    bar1[q] = want1 ? sRes[0] : kInf;
                    bar2[q] = want2 ? sRes[1] : kInf;
                }
                return;
            }
        }
        __syncthreads();  // the radix passes below reuse nothing of the above but the staged keys
    }
    uint32_t p1 = 0, p2 = 0, pmask = 0;
    int64_t rem1 = r1, rem2 = r2;
    for (int shift = 24; shift >= 0 && (want1 || want2); shift -= 8) {
        for (int i = threadIdx.x; i < 512; i += kBarThreads) (&sHist[0][0])[i] = 0;
        __syncthreads();  // also orders the staging above before the first pass
        for (int64_t p0 = 0; p0 < n; p0 += kBarThreads) {  // uniform trip count: all lanes take part in the match
            const int64_t p = p0 + threadIdx.x;
            const bool ok = p < n;
            const uint32_t o = ok ? (in_smem ? smem_bars[p] : ord_key(kq[p])) : 0u;
            const uint32_t dgt = (o >> shift) & 255u;
            if (want1) warp_hist_add(sHist[0], ok && (o & pmask) == p1, dgt);
            if (want2) warp_hist_add(sHist[1], ok && (o & pmask) == p2, dgt);
        }
        __syncthreads();
        if (warp < 2 && (warp == 0 ? want1 : want2)) {
            int d, bf;
            warp_hist_pick(sHist[warp], warp == 0 ? rem1 : rem2, &d, &bf);
            if ((threadIdx.x & 31) == 0) {
                sPick[2 * warp] = d;
                sPick[2 * warp + 1] = bf;
            }
        }
        __syncthreads();
        if (want1) {
            rem1 -= sPick[1];
            p1 |= (uint32_t)sPick[0] << shift;
        }
        if (want2) {
            rem2 -= sPick[3];
            p2 |= (uint32_t)sPick[2] << shift;
        }
        pmask |= 255u << shift;
    }
    if (threadIdx.x == 0) {
        bar1[q] = want1 ? from_ord(p1) : kInf;
        bar2[q] = want2 ? from_ord(p2) : kInf;
    }
}

// One warp per query: the R smallest of the query's (key, id) buffer [q * cap, + min(count[q], cap)) as a set:
// every key below the R-th smallest, then the keys equal to it with the lowest ids; padded with
// (+inf, kNoId) when fewer. Written unordered to out_key / out_id [q * R ..].
__global__ void __launch_bounds__(256) warp_select_kernel(const float* __restrict__ keys, const int* __restrict__ ids,
                                                          const int* __restrict__ count, int cap, int nq, int R,
                                                          float* __restrict__ out_key, int* __restrict__ out_id) {
    __shared__ int sHist[8][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x * 8 + warp;
    if (q >= nq) return;
    const int64_t n = min(count[q], cap);
    const float* kq = keys + (int64_t)q * cap;
    const int* iq = ids + (int64_t)q * cap;
    float* ok = out_key + (int64_t)q * R;
    int* oi = out_id + (int64_t)q * R;
    const uint32_t T = n > R ? warp_kth_ord(kq, n, R, sHist[warp]) : 0xffffffffu;
    int w = 0;  // written so far (uniform)
    for (int64_t p0 = 0; p0 < n; p0 += 32) {  // every key below T (all of them when n <= R)
        const int64_t p = p0 + lane;
        const bool take = p < n && (n <= R || ord_key(kq[p]) < T);
        const unsigned b = __ballot_sync(0xffffffffu, take);
        if (take) {
            const int at = w + __popc(b & ((1u << lane) - 1u));
            ok[at] = kq[p];
            oi[at] = iq[p];
        }
        w += __popc(b);
    }
    int last = -1;  // then keys equal to T by increasing id
    while (n > R && w < R) {
        int best = INT_MAX;
        for (int64_t p = lane; p < n; p += 32)
            if (ord_key(kq[p]) == T && iq[p] > last) best = min(best, iq[p]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (best == INT_MAX) break;
        if (lane == 0) {
            ok[w] = from_ord(T);
            oi[w] = best;
        }
        last = best;
        ++w;
    }
    for (int e = w + lane; e < R; e += 32) {
        ok[e] = kInf;
        oi[e] = kNoId;
    }
}

// lcap[l] = ceil(size_l / div): the sampled head of list l
__global__ void tc_ivf_list_caps_kernel(const int64_t* __restrict__ list_off, int C, int div, int64_t* __restrict__ lcap) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l < C) lcap[l] = (list_off[l + 1] - list_off[l] + div - 1) / div;
}

// tauR[q] = tauS[q] for the queries marked for a re-run, else -inf (no key passes)
__global__ void tc_rerun_bars_kernel(const int* __restrict__ mark, const float* __restrict__ tauS, int nq,
                                     float* __restrict__ tauR, int* __restrict__ rcount) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    tauR[q] = mark[q] ? tauS[q] : -kInf;
    if (rcount && mark[q]) rcount[q] = 0;  // the re-run refills the query's buffer from its start
}

// offs2[j] = offs[list[j]], lens2[j] = rowcnt[list[j]] for the j < count listed rows
__global__ void tc_compact_rows_kernel(const int* __restrict__ list, const int* __restrict__ count,
                                       const int64_t* __restrict__ offs, const int* __restrict__ rowcnt,
                                       int64_t* __restrict__ offs2, int* __restrict__ lens2) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < *count) {
        offs2[j] = offs[list[j]];
        lens2[j] = rowcnt[list[j]];
    }
}

constexpr int kCoarseChunks = 16;  // dims up to 512 take the register path of the exact distances

// The coarse ranking of one query (one warp) from its keys kr [C] and their 32-key chunk minima cq [nch],
// nch = ceil(C / 32) <= 64, for npc <= 32 and dpad <= 32 kCoarseChunks (cmax > 0).
//  1. bar = the npc-th smallest chunk minimum (total order by (minimum, chunk); +inf when npc > nch): each
//     of those npc chunks holds a key <= bar, so the npc-th smallest key T is <= bar.
//  2. The window lim = bar + 2 eps + delta (the keys' certified error, as below): a centroid whose key
//     exceeds lim exceeds T + 2 eps + delta, so its exact distance exceeds those of the npc centroids of
//     smallest key, and it is not among the best npc.
//  3. Every key <= lim (found in the chunks whose minimum is <= lim) gets its exact FP32 distance, and the
//     best npc by (distance, id) are kept, lane j holding the j-th: no candidate buffer and no sort.
__device__ __forceinline__ void coarse_by_chunks(const float* __restrict__ kr, const float* __restrict__ cq, int C,
                                                 int npc, const float* __restrict__ qv,
                                                 const float* __restrict__ cent, int dpad, int dim, float cmax,
                                                 int32_t* __restrict__ pout) {
    const int lane = threadIdx.x & 31;
    const int nch = (C + 31) >> 5;
    const float a0 = lane < nch ? cq[lane] : kInf, a1 = lane + 32 < nch ? cq[lane + 32] : kInf;
    float qr[kCoarseChunks];
    float s2 = 0.f;
#pragma unroll
    for (int i = 0; i < kCoarseChunks; ++i) {
        qr[i] = lane + 32 * i < dpad ? qv[lane + 32 * i] : 0.f;
        s2 = fmaf(qr[i], qr[i], s2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    float bar = kInf;
    if (npc <= nch) {  // lane l holds chunks l and l + 32; ranks among the 64 (padding +inf, sorted last)
        int r0 = 0, r1 = 0;
#pragma unroll 8
        for (int j = 0; j < 32; ++j) {
            const float o0 = __shfl_sync(0xffffffffu, a0, j), o1 = __shfl_sync(0xffffffffu, a1, j);
            r0 += (o0 < a0 || (o0 == a0 && j < lane)) + (o1 < a0);
            r1 += (o0 <= a1) + (o1 < a1 || (o1 == a1 && j < lane));
        }
        const unsigned s0 = __ballot_sync(0xffffffffu, r0 == npc - 1);
        const unsigned s1 = __ballot_sync(0xffffffffu, r1 == npc - 1);
        const float b0 = __shfl_sync(0xffffffffu, a0, s0 ? __ffs(s0) - 1 : 0);
        const float b1 = __shfl_sync(0xffffffffu, a1, s1 ? __ffs(s1) - 1 : 0);
        bar = s0 ? b0 : (s1 ? b1 : kInf);  // no rank npc - 1 only with NaN minima: every chunk
    }
    const float qn = sqrtf(s2) * 1.0001f;
    const float acc = (float)(dim + 3) * 4.76837158e-7f;  // (dim + 3) 2^-21
    const float eps = qn * cmax * (7.8125e-3f * 1.05f + 2.1f * acc) + cmax * cmax * acc;
    const float delta = acc * (qn + cmax) * (qn + cmax);
    const float lim = bar + 2.f * eps + delta;
    float bd = kInf;  // lane j < npc: the j-th best (distance, id) so far
    int bi = kNoId;
    auto insert = [&](float d, int id) {  // warp-uniform (d, id)
        const int pos = __popc(__ballot_sync(0xffffffffu, lane < npc && pair_less(bd, bi, d, id)));
        const float ud = __shfl_up_sync(0xffffffffu, bd, 1);
        const int ui = __shfl_up_sync(0xffffffffu, bi, 1);
        if (pos < npc) {
            if (lane == pos) {
                bd = d;
                bi = id;
            } else if (lane > pos) {
                bd = ud;
                bi = ui;
            }
        }
    };
    unsigned c0m = __ballot_sync(0xffffffffu, lane < nch && !(a0 > lim));
    unsigned c1m = __ballot_sync(0xffffffffu, lane + 32 < nch && !(a1 > lim));
    while (c0m | c1m) {  // four chunks' loads in flight
        int ch[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (c0m) {
                ch[u] = __ffs(c0m) - 1;
                c0m &= c0m - 1;
            } else if (c1m) {
                ch[u] = 32 + __ffs(c1m) - 1;
                c1m &= c1m - 1;
            } else {
                ch[u] = -1;
            }
        }
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c = ch[u] * 32 + lane;
            v[u] = ch[u] >= 0 && c < C ? kr[c] : kInf;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            unsigned hit = __ballot_sync(0xffffffffu, ch[u] >= 0 && ch[u] * 32 + lane < C && v[u] <= lim);
            while (hit) {  // two centroids at a time, all their pieces loaded before use; per lane the sum
                           // runs over d = lane, lane + 32, ... as in the kernel below
                const int ca = ch[u] * 32 + __ffs(hit) - 1;
                hit &= hit - 1;
                const bool two = hit != 0;
                const int cb = two ? ch[u] * 32 + __ffs(hit) - 1 : ca;
                hit &= hit - 1;
                const float* xa = cent + (int64_t)ca * dpad;
                const float* xb = cent + (int64_t)cb * dpad;
                float va[kCoarseChunks], vb[kCoarseChunks];
#pragma unroll
                for (int i = 0; i < kCoarseChunks; ++i) {
                    const int d = lane + 32 * i;
                    va[i] = d < dpad ? xa[d] : 0.f;
                    vb[i] = d < dpad ? xb[d] : 0.f;
                }
                float accA = 0.f, accB = 0.f;
#pragma unroll
                for (int i = 0; i < kCoarseChunks; ++i) {
                    if (lane + 32 * i < dpad) {
                        const float ta = va[i] - qr[i], tb = vb[i] - qr[i];
                        accA = fmaf(ta, ta, accA);
                        accB = fmaf(tb, tb, accB);
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    accA += __shfl_xor_sync(0xffffffffu, accA, o);
                    accB += __shfl_xor_sync(0xffffffffu, accB, o);
                }
                insert(accA, ca);
                if (two) insert(accB, cb);
            }
        }
    }
    if (lane < npc) pout[lane] = bi != kNoId ? bi : 0;
}

// one warp per query; CMIN: the keys' 32-column chunk minima are given, and coarse_by_chunks ranks the query
template <bool CMIN>
__global__ void __launch_bounds__(128) tc_coarse_kernel(const float* __restrict__ keys, int64_t ldk, int nq, int C,
                                                       int npc, int m, const float* __restrict__ q,
                                                       const float* __restrict__ cent, int dpad, int32_t* probes,
                                                       float cmax, int dim, const float* __restrict__ cmin) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cap = topk_cap(m);
    float* sK = reinterpret_cast<float*>(smem_raw) + warp * 2 * cap;
    int* sI = reinterpret_cast<int*>(sK + cap);
    const int qi = blockIdx.x * 4 + warp;
    if (qi >= nq) return;
    if (CMIN) {
        coarse_by_chunks(keys + (int64_t)qi * ldk, cmin + (int64_t)qi * ((C + 31) >> 5), C, npc, q + (int64_t)qi * dpad,
                         cent, dpad, dim, cmax, probes + (int64_t)qi * npc);
        return;
    }
    WarpTopK top;
    top.init(sK, sI, m);
    const float* kr = keys + (int64_t)qi * ldk;
    // A bar that keeps the offers few: each lane's smallest key, and the m-th smallest of those 32 minima
    // (m <= 32). At least m keys lie at or below it, so the m-th smallest key does, and with it every key of
    // the best m (ties included): offering only keys <= bar gives the same best m.
    float bar = kInf;
    if (m <= 32) {
        float mn = kInf;
        for (int c0 = 0; c0 < C; c0 += 128) {
            float v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int c = c0 + 32 * u + lane;
                v[u] = c < C ? kr[c] : kInf;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) mn = fminf(mn, v[u]);
        }
        int rank = 0;  // among the lane minima, ties by lane
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const float o = __shfl_sync(0xffffffffu, mn, j);
            rank += (o < mn) || (o == mn && j < lane);
        }
        const unsigned sel = __ballot_sync(0xffffffffu, rank == m - 1);
        bar = __shfl_sync(0xffffffffu, mn, __ffs(sel) - 1);
    }
    for (int c0 = 0; c0 < C; c0 += 128) {  // four loads in flight, offered in key order
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c = c0 + 32 * u + lane;
            v[u] = c < C ? kr[c] : kInf;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c = c0 + 32 * u + lane;
            top.offer(v[u], c < C ? c : kNoId, c < C && v[u] <= bar);
        }
    }
    top.compact();
    const int cnt = top.count;  // sK / sI [0, cnt): the best m by (key, id), ascending
    const float* qv = q + (int64_t)qi * dpad;
    // The certified window. A BF16 key differs from the real key |c|^2 - 2 q.c by at most
    //   eps = |q| |c| (2^-7 * 1.05 + (dim + 3) 2^-21 * 2.1) + |c|^2 (dim + 3) 2^-21
    // (both operands rounded to 8 significant bits, relative 2^-9 each; FP32 accumulation of dim + 3 products,
    // bounded with a factor 2 to allow truncating adds). With T the npc-th smallest key, a candidate whose key
    // exceeds T + 2 eps + delta -- delta bounding the FP32 rounding of the exact distances below -- is farther
    // than the best npc candidates in FP32 as in real arithmetic, so it is never among them: only the
    // candidates inside the window get exact distances, and the result is the one over all m.
    int ncert = cnt;
    if (cmax > 0.f && cnt > npc) {
        float s2 = 0.f;
        for (int d = lane; d < dpad; d += 32) s2 = fmaf(qv[d], qv[d], s2);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        const float qn = sqrtf(s2) * 1.0001f;
        const float acc = (float)(dim + 3) * 4.76837158e-7f;  // (dim + 3) 2^-21
        const float eps = qn * cmax * (7.8125e-3f * 1.05f + 2.1f * acc) + cmax * cmax * acc;
        const float delta = acc * (qn + cmax) * (qn + cmax);
        const float lim = sK[npc - 1] + 2.f * eps + delta;
        int inside = 0;
        for (int e = lane; e < cnt; e += 32) inside += sK[e] <= lim;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) inside += __shfl_xor_sync(0xffffffffu, inside, o);
        ncert = max(npc, inside);  // sK is sorted: the window is a prefix
        __syncwarp();
    }
    // exact FP32 squared distances of the candidates in the window
    if (dpad <= 32 * kCoarseChunks) {
        // the query's pieces in registers; two centroids at a time with all their pieces loaded before
        // use; per lane the sum runs over d = lane, lane + 32, ... as in the loop below
        float qr[kCoarseChunks];
#pragma unroll
        for (int i = 0; i < kCoarseChunks; ++i) qr[i] = lane + 32 * i < dpad ? qv[lane + 32 * i] : 0.f;
        for (int e = 0; e < ncert; e += 2) {
            const bool two = e + 1 < ncert;
            const float* xa = cent + (int64_t)sI[e] * dpad;
            const float* xb = cent + (int64_t)(two ? sI[e + 1] : sI[e]) * dpad;
            float va[kCoarseChunks], vb[kCoarseChunks];
#pragma unroll
            for (int i = 0; i < kCoarseChunks; ++i) {
                const int d = lane + 32 * i;
                va[i] = d < dpad ? xa[d] : 0.f;
                vb[i] = d < dpad ? xb[d] : 0.f;
            }
            float accA = 0.f, accB = 0.f;
#pragma unroll
            for (int i = 0; i < kCoarseChunks; ++i) {
                if (lane + 32 * i < dpad) {
                    const float ta = va[i] - qr[i], tb = vb[i] - qr[i];
                    accA = fmaf(ta, ta, accA);
                    accB = fmaf(tb, tb, accB);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                accA += __shfl_xor_sync(0xffffffffu, accA, o);
                accB += __shfl_xor_sync(0xffffffffu, accB, o);
            }
            if (lane == 0) {
                sK[e] = accA;
                if (two) sK[e + 1] = accB;
            }
            __syncwarp();
        }
    }
    for (int e = 0; e < ncert && dpad > 32 * kCoarseChunks; ++e) {
        const int c = sI[e];
        const float* x = cent + (int64_t)c * dpad;
        float acc = 0.f;
        for (int d = lane; d < dpad; d += 32) {
            const float t = x[d] - qv[d];
            acc = fmaf(t, t, acc);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) sK[e] = acc;
        __syncwarp();
    }
    for (int e = ncert + lane; e < cap; e += 32) {  // outside the window (or empty): sorted last
        sK[e] = kInf;
        if (e >= cnt) sI[e] = kNoId;
    }
    __syncwarp();
    warp_sort_smem(sK, sI, cap);
    for (int j = lane; j < npc; j += 32) probes[(int64_t)qi * npc + j] = j < cnt ? sI[j] : 0;
}

}  // namespace

int launch_tc_coarse(const float* keys, int64_t ldk, int nq, int C, int npc, int margin, const float* q,
                     const float* centroids, int dpad, int32_t* probes, cudaStream_t st, float cmax, int dim,
                     const float* cmin) {
    if (nq == 0) return ANN_OK;
    const int m = std::min(C, npc + margin);
    ANN_CHECK_ARG(npc >= 1 && npc <= m && m <= 1024, "tensor-core coarse ranking: npc=%d, m=%d", npc, m);
    const size_t smem = (size_t)4 * 2 * topk_cap(m) * 4;
    const bool chunks = cmin != nullptr && C <= 64 * 32 && npc <= 32 && cmax > 0.f && dpad <= 32 * kCoarseChunks;
    auto kern = chunks ? tc_coarse_kernel<true> : tc_coarse_kernel<false>;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(kern)));
    kern<<<(unsigned)ceil_div(nq, 4), 128, smem, st>>>(keys, ldk, nq, C, npc, m, q, centroids, dpad, probes, cmax,
                                                       dim > 0 ? dim : dpad, cmin);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_ivf_items(const int64_t* lq_off, const int64_t* list_off, int C, int64_t* item_off, cudaStream_t st,
                        const int64_t* list_len) {
    ANN_CHECK_ARG(C >= 1, "tensor-core IVF: no lists");
    tc_ivf_items_kernel<<<1, 1024, 0, st>>>(lq_off, list_off, C, item_off, list_len);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

namespace {
// item_list[t] = l for every item t of list l (t < cap)
__global__ void tc_item_lists_kernel(const int64_t* __restrict__ item_off, int C, int32_t* __restrict__ item_list,
                                     int64_t cap) {
    for (int l = blockIdx.x; l < C; l += gridDim.x)
        for (int64_t t = item_off[l] + threadIdx.x; t < item_off[l + 1] && t < cap; t += blockDim.x) item_list[t] = l;
}
}  // namespace

int launch_tc_item_lists(const int64_t* item_off, int C, int32_t* item_list, int64_t cap, cudaStream_t st) {
    ANN_CHECK_ARG(C >= 1, "tensor-core IVF: no lists");
    tc_item_lists_kernel<<<(unsigned)std::min(C, 4 * kNumSMs), 128, 0, st>>>(item_off, C, item_list, cap);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_ivf_pairs(const void* qrows, int row_bytes, const int32_t* pair_vals, const int32_t* pair_lists,
                        const int64_t* n_pairs, int64_t max_pairs, int npc, const int64_t* cand_off,
                        const int64_t* seg_pref, const int64_t* list_off, void* A, int64_t* dbase, cudaStream_t st,
                        const TcIvfSampleMaps& sm) {
    if (max_pairs == 0) return ANN_OK;
    ANN_CHECK_ARG(row_bytes % 16 == 0, "tensor-core IVF: operand rows of %d bytes", row_bytes);
    ANN_CHECK_ARG((sm.pfac == nullptr) == (sm.qfac == nullptr), "tensor-core IVF: pair factors need query factors");
    const int grid = (int)std::min<int64_t>(ceil_div(max_pairs * 32, 256), 16 * kNumSMs);
    tc_ivf_pairs_kernel<<<grid, 256, 0, st>>>(static_cast<const unsigned char*>(qrows), row_bytes, pair_vals,
                                              pair_lists, n_pairs, max_pairs, npc, cand_off, seg_pref, list_off,
                                              static_cast<unsigned char*>(A), dbase, sm);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_group(const TcGroupArgs& g, cudaStream_t st) {
    if (g.M == 0) return ANN_OK;
    ANN_CHECK_ARG(g.nwarps > 0 && g.wcap > 0, "survivor grouping: no regions");
    ANN_CUDA_TRY(cudaMemsetAsync(g.rowcnt, 0, sizeof(int) * (size_t)g.M, st));
    tc_count_kernel<<<g.nwarps, 256, 0, st>>>(g);
    ANN_LAUNCH_CHECK();
    tc_scan_kernel<<<1, 1024, 0, st>>>(g);
    ANN_LAUNCH_CHECK();
    tc_scatter_kernel<<<g.nwarps, 256, 0, st>>>(g);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_bar_check(const int* rowcnt, int M, int R, int* list, int* flags, cudaStream_t st, const int64_t* lens,
                        int* mark) {
    if (M == 0) return ANN_OK;
    tc_bar_check_kernel<<<(unsigned)ceil_div(M, 256), 256, 0, st>>>(rowcnt, M, R, list, flags, lens, mark);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_ivf_sample_plan(const IvfPlan& p, const int64_t* list_off, int C, int div, int64_t* lcap, int64_t* sseg,
                              int64_t* slen, cudaStream_t st) {
    ANN_CHECK_ARG(C >= 1 && div >= 1, "IVF sample plan: %d lists, 1/%d", C, div);
    tc_ivf_list_caps_kernel<<<(unsigned)ceil_div(C, 256), 256, 0, st>>>(list_off, C, div, lcap);
    ANN_LAUNCH_CHECK();
    if (p.nq == 0) return ANN_OK;
    tc_ivf_sample_plan_kernel<<<(unsigned)ceil_div(p.nq, 128), 128, 0, st>>>(p, lcap, sseg, slen);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_sq8_query(const float* q, int nq, int dim, int ldq, const float* scale, const float* offset, int8_t* out,
                        int ldo, float* qfac, cudaStream_t st) {
    if (nq == 0) return ANN_OK;
    ANN_CHECK_ARG(ldo >= dim && ldo % 16 == 0, "SQ8 query weights: row of %d bytes for dim %d", ldo, dim);
    tc_sq8_query_kernel<<<(unsigned)ceil_div(nq, 8), 256, 0, st>>>(q, nq, dim, ldq, scale, offset, out, ldo, qfac);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_sq8_norms(const uint8_t* codes, int64_t n, int dim, int ldc, const float* scale, float2* fac,
                        cudaStream_t st) {
    if (n == 0) return ANN_OK;
    tc_sq8_norms_kernel<<<(unsigned)ceil_div(n, 8), 256, 0, st>>>(codes, n, dim, ldc, scale, fac);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

namespace {
__global__ void max_int_kernel(const int* __restrict__ v, int n, int* __restrict__ out) {
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, v[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(out, m);
}
}  // namespace

int launch_max_int(const int* v, int n, int* out, cudaStream_t st) {
    ANN_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int), st));
    if (n == 0) return ANN_OK;
    max_int_kernel<<<(unsigned)std::min<int64_t>(ceil_div(n, 256), 4 * kNumSMs), 256, 0, st>>>(v, n, out);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_warp_bars(const float* keys, const int64_t* offs, const int64_t* lens, int nq, int r1, int r2, float* bar1,
                     float* bar2, cudaStream_t st, int64_t max_len) {
    if (nq == 0) return ANN_OK;
    ANN_CHECK_ARG(r1 >= 1 && r2 >= 1, "bars: ranks %d, %d", r1, r2);
    if (max_len > 0) {  // one block per query; streams of up to 6,144 keys (24 KB) staged in shared memory
        const int staged = (int)std::min<int64_t>(max_len, 6144);
        block_bars_kernel<<<(unsigned)nq, kBarThreads, (size_t)staged * 4, st>>>(keys, offs, lens, nq, r1, r2, staged,
                                                                                bar1, bar2);
    } else {
        warp_bars_kernel<<<(unsigned)ceil_div(nq, 8), 256, 0, st>>>(keys, offs, lens, nq, r1, r2, bar1, bar2);
    }
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_warp_select(const float* keys, const int* ids, const int* count, int cap, int nq, int R, float* out_key,
                       int* out_id, cudaStream_t st) {
    if (nq == 0) return ANN_OK;
    ANN_CHECK_ARG(R >= 1 && cap >= 1, "warp select: R=%d, cap=%d", R, cap);
    warp_select_kernel<<<(unsigned)ceil_div(nq, 8), 256, 0, st>>>(keys, ids, count, cap, nq, R, out_key, out_id);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_rerun_bars(const int* mark, const float* tauS, int nq, float* tauR, cudaStream_t st, int* rcount) {
    if (nq == 0) return ANN_OK;
    tc_rerun_bars_kernel<<<(unsigned)ceil_div(nq, 256), 256, 0, st>>>(mark, tauS, nq, tauR, rcount);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_compact_rows(const int* list, const int* count, int max_count, const int64_t* offs, const int* rowcnt,
                           int64_t* offs2, int* lens2, cudaStream_t st) {
    if (max_count == 0) return ANN_OK;
    tc_compact_rows_kernel<<<(unsigned)ceil_div(max_count, 256), 256, 0, st>>>(list, count, offs, rowcnt, offs2, lens2);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_gather(const void* A, int row_bytes, const int* list, int nb, const float* tau, void* A2, float* tau2,
                     const float* rfac, float* rfac2, cudaStream_t st) {
    if (nb == 0) return ANN_OK;
    ANN_CHECK_ARG(row_bytes % 16 == 0, "gather: row of %d bytes", row_bytes);
    tc_gather_kernel<<<nb, 128, 0, st>>>(static_cast<const unsigned char*>(A), row_bytes, list, nb, tau,
                                         static_cast<unsigned char*>(A2), tau2, rfac, rfac2);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_map_ids(int* ids, int64_t count, int64_t n, int64_t mult, cudaStream_t st) {
    if (count == 0) return ANN_OK;
    const int grid = (int)std::min<int64_t>(ceil_div(count, 256), 4 * kNumSMs);
    tc_map_ids_kernel<<<grid, 256, 0, st>>>(ids, count, n, mult);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_unpermute(const float* keys, int nq, int64_t n, int64_t mult, float* out, cudaStream_t st) {
    if (nq == 0 || n == 0) return ANN_OK;
    ANN_CHECK_ARG(nq <= 65535, "unpermute: %d query rows", nq);
    dim3 grid((unsigned)std::min<int64_t>(ceil_div(n, 256), 64), (unsigned)nq);
    tc_unpermute_kernel<<<grid, 256, 0, st>>>(keys, n, mult, out);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

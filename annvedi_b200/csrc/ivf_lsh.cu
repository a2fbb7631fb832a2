// LSH bucket tables of the IVF-LSH index: per-query candidate streams in the reference's order, and the
// signatures of the table build.
//
// The candidate stream of LSHIndex::query (competitors/ivf_lsh/src/lsh_index_optimized.cpp:352-457):
// for each probed list in order, for each table: the query's signature (sign of (q - mean) . p over the
// table's B projections, :376-394), the points of the list's bucket with that signature not yet taken
// (:398-405), then, with n_probes > 0, the buckets one or two bit flips away, the flips ordered by the
// |dot| of the flipped bits (:407-446); the cap max_candidates is checked before each list, each table
// and each probed bucket, never inside a bucket; fewer than k candidates fall back to every row
// (:453-457).
//
// Two kernels, one warp per query each, no block barriers. lsh_signatures_kernel computes the query's
// signature in every table and its flip masks in probe order once (global scratch); lsh_candidates_kernel
// walks the buckets. Per probed list the walk warp walks the list's T * (1 + flips) buckets 32 at a time: each lane loads one bucket's
// bounds, a warp scan lays the 32 buckets' members out in walk order, and the members are read 32 at a
// time. A member is new if the list's visited bitmap (shared memory) does not hold it and no earlier lane
// of the same 32 holds the same row (__match_any_sync): the first occurrence in walk order wins, as in
// the reference's sequential walk. A bucket is admitted iff the count of new members before its first
// member is below the cap; the first bucket refused ends the walk.
#include <climits>

#include "common.cuh"
#include "ivf_lsh.cuh"

namespace annb {

namespace {

constexpr int kMaxWarps = 4;        // queries per CTA
constexpr int kMaxSigDots = 1024;   // T * B <= 64 * 16
constexpr unsigned kFull = 0xffffffffu;

// (score, generation index) order of the flips: the reference's sort by score, ties in the order the
// flips were generated (singles by bit rank, then pairs (i, j) with i < j)
__device__ __forceinline__ bool flip_before(float sa, int ga, float sb, int gb) {
    return sa < sb || (sa == sb && ga < gb);
}

// Per-warp shared memory (32-bit words) of the signatures kernel: q - mean [dim], dots [T * B].
struct LshSigSmem {
    int qm, dots, total;
    __host__ __device__ LshSigSmem(int dim, int T, int B) {
        qm = 0;
        dots = qm + dim;
        total = (dots + T * B + 3) & ~3;  // 16-byte aligned per warp
    }
};
// ... and of the walk: signatures [T], flip masks [T * P], visited bitmap of one list [nwords].
struct LshWarpSmem {
    int sig, pert, vis, total;
    __host__ __device__ LshWarpSmem(int T, int P, int nwords) {
        sig = 0;
        pert = sig + T;
        vis = pert + T * P;
        total = (vis + nwords + 3) & ~3;
    }
};

__global__ void __launch_bounds__(32 * kMaxWarps) lsh_signatures_kernel(LshCandArgs a, int P) {
    extern __shared__ __align__(16) uint32_t smem_w[];
    const int T = a.lsh.T, B = a.lsh.B, TB = T * B;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qi = blockIdx.x * (blockDim.x >> 5) + warp;
    if (qi >= a.nq) return;  // the whole warp; no block barrier follows
    const int dim = a.ix.dim;
    const LshSigSmem L(dim, T, B);
    uint32_t* ws = smem_w + (size_t)warp * L.total;
    float* sQm = reinterpret_cast<float*>(ws + L.qm);
    float* sDot = reinterpret_cast<float*>(ws + L.dots);
    uint32_t* sSig = a.sig + (int64_t)qi * T;
    int* sPert = a.pert + (int64_t)qi * T * P;
    const float* q = a.q + (int64_t)qi * a.ldq;
    // 1. the query's dot with every projection: sum over d ascending of (q[d] - mean[d]) * p[d], each
    // product rounded, no fused multiply-add (the restatement's order). Lane l runs four independent sums,
    // projections i0 + l + 32c; projT is [dim][T * B], so each step of the warp reads whole lines.
    for (int d = lane; d < dim; d += 32) sQm[d] = __fsub_rn(q[d], a.lsh.mean[d]);
    __syncwarp();
    for (int i0 = 0; i0 < TB; i0 += 128) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        const float* pt = a.lsh.projT + i0 + lane;
        const int nc = min(4, (TB - i0 - lane + 31) / 32);  // sums this lane owns in this round (0..4)
#pragma unroll 4
        for (int d = 0; d < dim; ++d) {
            const float qd = sQm[d];
            const float* row = pt + (int64_t)d * TB;
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (c < nc) acc[c] = __fadd_rn(acc[c], __fmul_rn(qd, row[32 * c]));
        }
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if (c < nc) sDot[i0 + lane + 32 * c] = acc[c];
    }
    __syncwarp();
    // 2. signatures and the first P flips of each table, a lane per table
    for (int t = lane; t < T; t += 32) {
        uint32_t sig = 0;
        for (int b = 0; b < B; ++b)
            if (sDot[t * B + b] > 0.f) sig |= 1u << b;
        sSig[t] = sig;
        if (P > 0) {
            // bits by (|dot|, bit) (a pair order, so the sort is exact), the first m of them
            int order[16];
            float av[16];
            for (int b = 0; b < B; ++b) {
                const float v = fabsf(sDot[t * B + b]);
                int j = b - 1;
                while (j >= 0 && (v < av[j] || (v == av[j] && b < order[j]))) {
                    av[j + 1] = av[j];
                    order[j + 1] = order[j];
                    --j;
                }
                av[j + 1] = v;
                order[j + 1] = b;
            }
            const int m = min(B, a.n_probes);
            // the P smallest flips by (score, generation index), by repeated selection
            float ps = -1.f;
            int pg = -1;
            for (int p = 0; p < P; ++p) {
                float bs = 0.f;
                int bg = INT_MAX, bmask = 0, g = 0;
                for (int i = 0; i < m; ++i, ++g) {
                    const float sc = av[i];
                    if (flip_before(ps, pg, sc, g) && (bg == INT_MAX || flip_before(sc, g, bs, bg))) {
                        bs = sc;
                        bg = g;
                        bmask = 1 << order[i];
                    }
                }
                for (int i = 0; i < m; ++i)
                    for (int j = i + 1; j < m; ++j, ++g) {
                        const float sc = __fadd_rn(av[i], av[j]);
                        if (flip_before(ps, pg, sc, g) && (bg == INT_MAX || flip_before(sc, g, bs, bg))) {
                            bs = sc;
                            bg = g;
                            bmask = (1 << order[i]) | (1 << order[j]);
                        }
                    }
                sPert[t * P + p] = bmask;
                ps = bs;
                pg = bg;
            }
        }
    }
}

__global__ void __launch_bounds__(32 * kMaxWarps) lsh_candidates_kernel(LshCandArgs a, int P, int nwords) {
    extern __shared__ __align__(16) uint32_t smem_w[];
    const int T = a.lsh.T, B = a.lsh.B;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qi = blockIdx.x * (blockDim.x >> 5) + warp;
    if (qi >= a.nq) return;  // the whole warp; no block barrier follows
    const LshWarpSmem L(T, P, nwords);
    uint32_t* ws = smem_w + (size_t)warp * L.total;
    uint32_t* sSig = ws + L.sig;
    int* sPert = reinterpret_cast<int*>(ws + L.pert);
    uint32_t* sVis = ws + L.vis;
    for (int i = lane; i < T; i += 32) sSig[i] = a.sig[(int64_t)qi * T + i];
    for (int i = lane; i < T * P; i += 32) sPert[i] = a.pert[(int64_t)qi * T * P + i];
    __syncwarp();
    // 3. the walk
    const int64_t nb = (int64_t)1 << B;
    const int per_list = T * (1 + P);
    int32_t* out = a.cand_ids + (int64_t)qi * a.ld;
    long long nc = 0;
    bool stop = false;
    for (int ci = 0; ci < a.npc && !stop; ++ci) {
        if (nc >= a.max_c) break;
        const int cid = a.probes[(int64_t)qi * a.npc + ci];
        if (cid < 0 || cid >= a.ix.C) break;
        const int64_t lstart = a.ix.list_off[cid];
        const int64_t lsize = a.ix.list_off[cid + 1] - lstart;
        const int lw = (int)min((lsize + 31) / 32, (int64_t)nwords);
        for (int w = lane; w < lw; w += 32) sVis[w] = 0;
        __syncwarp();
        for (int b0 = 0; b0 < per_list && !stop; b0 += 32) {
            const int bi = b0 + lane;
            int64_t bstart = 0;
            int blen = 0;
            if (bi < per_list) {
                const int t = bi / (1 + P), p = bi - t * (1 + P);
                const uint32_t sig = sSig[t] ^ (p ? (uint32_t)sPert[t * P + p - 1] : 0u);
                const int64_t o = ((int64_t)t * a.ix.C + cid) * nb + sig;
                bstart = a.lsh.tab_off[o];
                blen = (int)(a.lsh.tab_off[o + 1] - bstart);
            }
            int incl = blen;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += v;
            }
            const int excl = incl - blen;
            const int total = __shfl_sync(kFull, incl, 31);
            for (int m0 = 0; m0 < total && !stop; m0 += 32) {
                const int pos = m0 + lane;
                const bool valid = pos < total;
                // this member's bucket: the first lane whose inclusive end exceeds pos
                int lo = 0, hi = 31;
#pragma unroll
                for (int s = 0; s < 5; ++s) {
                    const int mid = (lo + hi) >> 1;
                    const int v = __shfl_sync(kFull, incl, mid);
                    if (v > pos)
                        hi = mid;
                    else
                        lo = mid + 1;
                }
                const int64_t jstart = __shfl_sync(kFull, bstart, lo);
                const int jexcl = __shfl_sync(kFull, excl, lo);
                int32_t row = -1 - lane;  // distinct from every row for the match below
                bool fresh = false;
                if (valid) {
                    row = a.lsh.tab_ids[jstart + (pos - jexcl)];
                    const int64_t r = (int64_t)row - lstart;
                    fresh = r >= 0 && r < lsize && r < 32 * (int64_t)nwords && !((sVis[r >> 5] >> (r & 31)) & 1u);
                }
                const unsigned same = __match_any_sync(kFull, row);
                fresh = fresh && (__ffs(same) - 1) == lane;
                const unsigned fb = __ballot_sync(kFull, fresh);
                // a bucket starting in this chunk is admitted iff the count before its first member is
                // below the cap; one that started in an earlier chunk was admitted then
                const bool admitted =
                    !valid || jexcl < m0 || nc + __popc(fb & ((1u << (jexcl - m0)) - 1u)) < a.max_c;
                const bool keep = fresh && admitted;
                const unsigned kb = __ballot_sync(kFull, keep);
                if (keep) {
                    const long long at = nc + __popc(kb & ((1u << lane) - 1u));
                    if (at < a.ld) out[at] = row;
                    const int64_t r = (int64_t)row - lstart;
                    atomicOr(&sVis[r >> 5], 1u << (r & 31));
                }
                nc += __popc(kb);
                stop = __any_sync(kFull, !admitted);
                __syncwarp();
            }
        }
    }
    if (lane == 0) {
        int64_t ncs = nc;
        if (ncs < a.k) {  // every row
            a.n_seg[qi] = -1;
            ncs = a.ix.n;
        } else {
            a.n_seg[qi] = 0;
        }
        a.n_cands[qi] = ncs;
        if (a.ndist) atomicAdd(a.ndist, (unsigned long long)ncs);
    }
}

// projT[d][i] = proj[i][d]
__global__ void lsh_transpose_kernel(const float* __restrict__ proj, int rows, int dim, int dpad,
                                     float* __restrict__ projT) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= (int64_t)rows * dim) return;
    const int d = (int)(e / rows), i = (int)(e % rows);
    projT[e] = proj[(int64_t)i * dpad + d];
}

__global__ void lsh_row_keys_kernel(IvfView ix, LshView lsh, int32_t* keys) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= (int64_t)lsh.T * ix.n) return;
    const int t = (int)(e / ix.n);
    const int64_t i = e % ix.n;
    // the row's list: the last list whose first row is <= i
    int lo = 0, hi = ix.C - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ix.list_off[mid] <= i)
            lo = mid;
        else
            hi = mid - 1;
    }
    const float* x = ix.original + i * ix.dpad;
    uint32_t sig = 0;
    for (int b = 0; b < lsh.B; ++b) {
        const float* p = lsh.proj + (int64_t)(t * lsh.B + b) * ix.dpad;
        float dot = 0.f;
        for (int d = 0; d < ix.dim; ++d) dot = __fadd_rn(dot, __fmul_rn(__fsub_rn(x[d], lsh.mean[d]), p[d]));
        if (dot > 0.f) sig |= 1u << b;
    }
    keys[e] = (int32_t)((int64_t)lo * (1 << lsh.B) + sig);
}

__global__ void lsh_mean_kernel(const float* rows, int64_t n, int dim, int dpad, float* mean) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= dpad) return;
    if (d >= dim) {
        mean[d] = 0.f;
        return;
    }
    float s = 0.f;
    for (int64_t i = 0; i < n; ++i) s = __fadd_rn(s, rows[i * dpad + d]);
    mean[d] = __fmul_rn(s, 1.f / (float)n);
}

}  // namespace

int lsh_flips_kept(int B, int n_probes) {
    if (n_probes <= 0) return 0;
    const int m = std::min(B, n_probes);
    return std::min(n_probes, m + m * (m - 1) / 2);
}

int launch_lsh_candidates(const LshCandArgs& a, cudaStream_t st) {
    if (a.nq == 0) return ANN_OK;
    ANN_CHECK_ARG(a.lsh.T >= 1 && a.lsh.T <= 64 && a.lsh.B >= 0 && a.lsh.B <= 16 && a.lsh.T * a.lsh.B <= kMaxSigDots,
                  "LSH candidates: %d tables of %d bits", a.lsh.T, a.lsh.B);
    ANN_CHECK_ARG(a.lsh.B == 0 || a.lsh.projT != nullptr, "LSH candidates: no projections");
    ANN_CHECK_ARG(a.sig != nullptr && a.pert != nullptr, "LSH candidates: no signature scratch");
    const int P = lsh_flips_kept(a.lsh.B, a.n_probes);
    const int nwords = (int)std::max<int64_t>(1, (a.largest_list + 31) / 32);
    const LshWarpSmem L(a.lsh.T, P, nwords);
    const size_t per_warp = sizeof(uint32_t) * (size_t)L.total;
    const int warps = (int)std::min<size_t>(kMaxWarps, (227 * 1024) / per_warp);
    ANN_CHECK_ARG(warps >= 1, "LSH candidates: lists of %lld rows with %d tables x %d flips need too much shared memory",
                  (long long)a.largest_list, a.lsh.T, P);
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(lsh_candidates_kernel)));
    lsh_candidates_kernel<<<(unsigned)ceil_div(a.nq, warps), 32 * warps, per_warp * warps, st>>>(a, P, nwords);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_lsh_signatures(const LshCandArgs& a, cudaStream_t st) {
    if (a.nq == 0) return ANN_OK;
    ANN_CHECK_ARG(a.lsh.T >= 1 && a.lsh.T <= 64 && a.lsh.B >= 0 && a.lsh.B <= 16 && a.lsh.T * a.lsh.B <= kMaxSigDots,
                  "LSH signatures: %d tables of %d bits", a.lsh.T, a.lsh.B);
    ANN_CHECK_ARG(a.lsh.B == 0 || a.lsh.projT != nullptr, "LSH signatures: no projections");
    ANN_CHECK_ARG(a.sig != nullptr && a.pert != nullptr, "LSH signatures: no scratch");
    const int P = lsh_flips_kept(a.lsh.B, a.n_probes);
    const LshSigSmem L(a.ix.dim, a.lsh.T, a.lsh.B);
    const size_t per_warp = sizeof(uint32_t) * (size_t)L.total;
    const int warps = (int)std::min<size_t>(kMaxWarps, (227 * 1024) / per_warp);
    ANN_CHECK_ARG(warps >= 1, "LSH signatures: dim %d with %d projections needs too much shared memory", a.ix.dim,
                  a.lsh.T * a.lsh.B);
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(lsh_signatures_kernel)));
    lsh_signatures_kernel<<<(unsigned)ceil_div(a.nq, warps), 32 * warps, per_warp * warps, st>>>(a, P);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_lsh_transpose(const float* proj, int rows, int dim, int dpad, float* projT, cudaStream_t st) {
    const int64_t total = (int64_t)rows * dim;
    if (total == 0) return ANN_OK;
    lsh_transpose_kernel<<<(unsigned)ceil_div(total, 256), 256, 0, st>>>(proj, rows, dim, dpad, projT);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_lsh_row_keys(const IvfView& ix, const LshView& lsh, int32_t* keys, cudaStream_t st) {
    const int64_t total = (int64_t)lsh.T * ix.n;
    if (total == 0) return ANN_OK;
    ANN_CHECK_ARG((int64_t)ix.C << lsh.B < INT32_MAX, "LSH build: %d lists x 2^%d buckets", ix.C, lsh.B);
    lsh_row_keys_kernel<<<(unsigned)ceil_div(total, 256), 256, 0, st>>>(ix, lsh, keys);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_lsh_mean(const float* rows, int64_t n, int dim, int dpad, float* mean, cudaStream_t st) {
    lsh_mean_kernel<<<(unsigned)ceil_div(dpad, 128), 128, 0, st>>>(rows, n, dim, dpad, mean);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

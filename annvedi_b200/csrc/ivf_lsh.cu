// LSH bucket tables of the IVF-LSH index: per-query candidate streams in the reference's order, and the
// signatures of the table build.
//
// The candidate stream of LSHIndex::query (competitors/ivf_lsh/src/lsh_index_optimized.cpp:352-457):
// for each probed list in order, for each table: the query's signature (sign of (q - mean) . p over the
// table's B projections, :376-394), the points of the list's bucket with that signature not yet taken
// (:398-405), then, with n_probes > 0, the buckets one or two bit flips away, the flips ordered by the
// |dot| of the flipped bits (:407-446); the cap max_candidates is checked before each list, each table
// and each probed bucket, never inside a bucket; fewer than k candidates fall back to every row
// (:453-457). One CTA per query: the signatures and flip orders are computed once, the buckets walked in
// order with a visited bitmap of the current list in shared memory (a bucket's members are distinct, and
// all belong to that list), each bucket's new members appended in bucket order by a block prefix sum.
#include "common.cuh"
#include "ivf_lsh.cuh"

namespace annb {

namespace {

constexpr int kThreads = 128;
constexpr int kMaxSigDots = 1024;  // T * B dots held in shared memory
constexpr int kMaxPert = 256;      // flips per table (m + m(m-1)/2, m = min(B, n_probes))

// (value, bit) order of the flip candidates: |dot| ascending, then bit
__device__ __forceinline__ bool bd_less(float va, int ba, float vb, int bb) { return va < vb || (va == vb && ba < bb); }

__global__ void __launch_bounds__(kThreads) lsh_candidates_kernel(LshCandArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int T = a.lsh.T, B = a.lsh.B;
    float* sDot = reinterpret_cast<float*>(smem_raw);                       // [T * B]
    uint32_t* sSig = reinterpret_cast<uint32_t*>(sDot + kMaxSigDots);       // [T]
    int* sPert = reinterpret_cast<int*>(sSig + 64);                         // [T][kMaxPert] flip masks
    int* sNp = sPert + 64 * kMaxPert;                                      // [T] flips per table
    uint32_t* sVis = reinterpret_cast<uint32_t*>(sNp + 64);                // visited bitmap of one list
    __shared__ int sWarp[kThreads / 32];
    __shared__ long long sNc;
    const int qi = blockIdx.x;
    const float* q = a.q + (int64_t)qi * a.ldq;
    const int dim = a.ix.dim, dpad = a.ix.dpad;
    // 1. the query's dot with every projection, the reference's order: d ascending, no fused multiply-add
    for (int i = threadIdx.x; i < T * B; i += kThreads) {
        const float* p = a.lsh.proj + (int64_t)i * dpad;
        float dot = 0.f;
        for (int d = 0; d < dim; ++d) dot = __fadd_rn(dot, __fmul_rn(__fsub_rn(q[d], a.lsh.mean[d]), p[d]));
        sDot[i] = dot;
    }
    __syncthreads();
    // 2. signatures and the flip orders, one thread per table
    for (int t = threadIdx.x; t < T; t += kThreads) {
        uint32_t sig = 0;
        for (int b = 0; b < B; ++b)
            if (sDot[t * B + b] > 0.f) sig |= 1u << b;
        sSig[t] = sig;
        int np = 0;
        if (a.n_probes > 0 && B > 0) {
            // bits by (|dot|, bit), the first m of them
            int order[32];
            for (int b = 0; b < B; ++b) order[b] = b;
            for (int i = 1; i < B; ++i) {  // insertion sort (stable)
                const int x = order[i];
                const float vx = fabsf(sDot[t * B + x]);
                int j = i - 1;
                while (j >= 0 && bd_less(vx, x, fabsf(sDot[t * B + order[j]]), order[j])) {
                    order[j + 1] = order[j];
                    --j;
                }
                order[j + 1] = x;
            }
            const int m = min(B, a.n_probes);
            float score[kMaxPert];
            int mask[kMaxPert];
            for (int i = 0; i < m; ++i) {
                score[np] = fabsf(sDot[t * B + order[i]]);
                mask[np++] = 1 << order[i];
            }
            for (int i = 0; i < m; ++i)
                for (int j = i + 1; j < m; ++j) {
                    score[np] = fabsf(sDot[t * B + order[i]]) + fabsf(sDot[t * B + order[j]]);
                    mask[np++] = (1 << order[i]) | (1 << order[j]);
                }
            // flips by score, then by the order they were generated in (stable insertion sort)
            for (int i = 1; i < np; ++i) {
                const float sx = score[i];
                const int mx = mask[i];
                int j = i - 1;
                while (j >= 0 && sx < score[j]) {
                    score[j + 1] = score[j];
                    mask[j + 1] = mask[j];
                    --j;
                }
                score[j + 1] = sx;
                mask[j + 1] = mx;
            }
            np = min(np, a.n_probes);
            for (int i = 0; i < np; ++i) sPert[t * kMaxPert + i] = mask[i];
        }
        sNp[t] = np;
    }
    if (threadIdx.x == 0) sNc = 0;
    __syncthreads();
    const int nb = 1 << B;
    int32_t* out = a.cand_ids + (int64_t)qi * a.ld;
    const int nwords = (int)((a.largest_list + 31) / 32);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // appends the bucket's members not yet visited, in bucket order
    auto take_bucket = [&](int64_t b0, int64_t b1, int64_t lstart) {
        for (int64_t base = b0; base < b1; base += kThreads) {
            const int64_t j = base + threadIdx.x;
            int32_t row = 0;
            bool fresh = false;
            if (j < b1) {
                row = a.lsh.tab_ids[j];
                const int64_t r = row - lstart;
                fresh = !((sVis[r >> 5] >> (r & 31)) & 1u);
            }
            const unsigned bal = __ballot_sync(0xffffffffu, fresh);
            if (lane == 0) sWarp[warp] = __popc(bal);
            __syncthreads();
            int before = 0, total = 0;
            for (int w = 0; w < kThreads / 32; ++w) {
                if (w < warp) before += sWarp[w];
                total += sWarp[w];
            }
            const long long nc0 = sNc;
            if (fresh) {
                const int64_t at = nc0 + before + __popc(bal & ((1u << lane) - 1u));
                if (at < a.ld) out[at] = row;
                const int64_t r = row - lstart;
                atomicOr(&sVis[r >> 5], 1u << (r & 31));
            }
            __syncthreads();
            if (threadIdx.x == 0) sNc = nc0 + total;
            __syncthreads();
        }
    };
    // 3. the walk
    for (int ci = 0; ci < a.npc; ++ci) {
        if (sNc >= a.max_c) break;
        const int cid = a.probes[(int64_t)qi * a.npc + ci];
        if (cid < 0 || cid >= a.ix.C) break;
        const int64_t lstart = a.ix.list_off[cid];
        const int64_t lsize = a.ix.list_off[cid + 1] - lstart;
        for (int w = threadIdx.x; w < (int)((lsize + 31) / 32) && w < nwords; w += kThreads) sVis[w] = 0;
        __syncthreads();
        for (int t = 0; t < T; ++t) {
            if (sNc >= a.max_c) break;
            const int64_t base = ((int64_t)t * a.ix.C + cid) * nb;
            const uint32_t sig = sSig[t];
            take_bucket(a.lsh.tab_off[base + sig], a.lsh.tab_off[base + sig + 1], lstart);
            for (int p = 0; p < sNp[t]; ++p) {
                if (sNc >= a.max_c) break;
                const uint32_t ps = sig ^ (uint32_t)sPert[t * kMaxPert + p];
                take_bucket(a.lsh.tab_off[base + ps], a.lsh.tab_off[base + ps + 1], lstart);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        int64_t nc = sNc;
        if (nc < a.k) {  // every row
            a.n_seg[qi] = -1;
            nc = a.ix.n;
        } else {
            a.n_seg[qi] = 0;
        }
        a.n_cands[qi] = nc;
        if (a.ndist) atomicAdd(a.ndist, (unsigned long long)nc);
    }
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

int launch_lsh_candidates(const LshCandArgs& a, cudaStream_t st) {
    if (a.nq == 0) return ANN_OK;
    ANN_CHECK_ARG(a.lsh.T >= 1 && a.lsh.T <= 64 && a.lsh.B >= 0 && a.lsh.B <= 16 && a.lsh.T * a.lsh.B <= kMaxSigDots,
                  "LSH candidates: %d tables of %d bits", a.lsh.T, a.lsh.B);
    const int m = std::min(a.lsh.B, a.n_probes);
    ANN_CHECK_ARG(m + m * (m - 1) / 2 <= kMaxPert, "LSH candidates: n_probes %d", a.n_probes);
    const size_t smem = sizeof(float) * kMaxSigDots + 4 * 64 + sizeof(int) * 64 * kMaxPert + sizeof(int) * 64 +
                        4 * (size_t)((a.largest_list + 31) / 32);
    ANN_CHECK_ARG(smem <= 227 * 1024, "LSH candidates: lists of %lld rows", (long long)a.largest_list);
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(lsh_candidates_kernel)));
    lsh_candidates_kernel<<<a.nq, kThreads, smem, st>>>(a);
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

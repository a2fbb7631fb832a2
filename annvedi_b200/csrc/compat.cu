// Reference-semantics linear scan: reproduces the ranking LinearIndex::query returns
// (competitors/linear/src/linear_index.cpp:27-60, 100-121), including its 64-entry early-abandon
// heap, bit for bit.
//
// The reference ranks point i by v_i, where T_i is the 64th-smallest exact distance among points
// 0..i-1 (FLT_MAX before 64 are seen): v_i = d_i when d_i < T_i, else the first checkpoint partial
// sum of compute_l2_distance (competitors/linear/src/simd.h:32-64) that reached T_i. It returns
// the k smallest (v_i, i) pairs.
//
// Pass 1 (compat_partials_kernel) is parallel: each group of 16 threads plays the 16 AVX-512
// lanes of one (query, row) pair -- lane j sums elements j, j+16, ... with an unfused multiply
// and add -- and folds the lanes in the compiled reference's order at every checkpoint (after
// 96, 192, ... elements and after the last full 16-chunk). The remainder (dim % 16) follows the
// compiled reference too: one fused 8-wide chunk folded the same way, then scalar fused steps.
// It writes the full distance D[q][i] and the checkpoint values P[q][c][i].
//
// Pass 2 (compat_threshold_kernel) is one warp per query walking the rows in order: the running
// 64-heap is replayed only at insertions (rows with D < T, which are rare once T settles), and each
// row's threshold T_i is recorded. Pass 3 (compat_values_kernel), parallel over rows, picks v_i from D,
// P and T_i. The k best (v_i, i) pairs come from the radix selection (the exact set, ties by row) and
// a sort of those k.
#include "common.cuh"
#include "compat.cuh"
#include "flat_scan.cuh"
#include "radix_select.cuh"
#include "refmath.cuh"

namespace annb {

// grid: (row blocks, query groups); block: 256 threads = 16 rows x 16 lanes.
__global__ void __launch_bounds__(256) compat_partials_kernel(CompatArgs a, int q_begin) {
    extern __shared__ float sQ[];  // [QG][dim]
    const int grp = threadIdx.x >> 4;
    const int qg0 = q_begin + blockIdx.y * kCompatQG;
    const int nqg = min(kCompatQG, a.q_end - qg0);
    for (int e = threadIdx.x; e < nqg * a.dim; e += blockDim.x) sQ[e] = a.q[(int64_t)(qg0 + e / a.dim) * a.ldq + e % a.dim];
    __syncthreads();
    const int ncp = a.ncp;
    const bool leader = (threadIdx.x & 15) == 0;
    for (int64_t r0 = (int64_t)blockIdx.x * 16; r0 < a.n; r0 += (int64_t)gridDim.x * 16) {
        const int64_t row = r0 + grp;
        const bool valid = row < a.n;
        const float* x = a.base + (valid ? row : 0) * a.ldb;
        for (int qq = 0; qq < nqg; ++qq) {
            const int64_t qi = qg0 + qq - q_begin;  // index within this chunk of queries
            float* P = a.P + (int64_t)qi * ncp * a.n + row;
            const float d = ref_l2_f32(x, sQ + qq * a.dim, a.dim, [&](int c, float v) {
                if (leader && valid) P[(int64_t)c * a.n] = v;
            });
            if (leader && valid) a.D[(int64_t)qi * a.n + row] = d;
        }
    }
}

constexpr int kCompatAhead = 8;  // 32-row steps of distances loaded ahead of the walk

__global__ void __launch_bounds__(128) compat_threshold_kernel(CompatArgs a, int q_begin) {
    constexpr int WARPS = 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qi = blockIdx.x * WARPS + warp;  // within chunk
    if (q_begin + qi >= a.q_end) return;       // the whole warp; no block barrier follows
    const int lim = a.k < 64 ? a.k : 64;
    const int64_t n = a.n;
    const float* D = a.D + (int64_t)qi * n;
    float* T = a.T + (int64_t)qi * n;
    const float inf = __int_as_float(0x7f800000);
    WarpHeap64 heap;
    heap.init(lim);
    float Tcur = 3.402823466e+38f;  // FLT_MAX until the heap holds lim distances
    float nxt[kCompatAhead];
#pragma unroll
    for (int j = 0; j < kCompatAhead; ++j) {
        const int64_t i = (int64_t)j * 32 + lane;
        nxt[j] = i < n ? D[i] : inf;
    }
    for (int64_t base = 0; base < n; base += 32 * kCompatAhead) {
        float cur[kCompatAhead];
#pragma unroll
        for (int j = 0; j < kCompatAhead; ++j) {
            cur[j] = nxt[j];
            const int64_t i = base + 32 * kCompatAhead + (int64_t)j * 32 + lane;
            nxt[j] = i < n ? D[i] : inf;
        }
#pragma unroll
        for (int j = 0; j < kCompatAhead; ++j) {
            const int64_t i = base + (int64_t)j * 32 + lane;
            const bool valid = i < n;
            const float d = cur[j];
            // rows enter the heap in row order; a row's threshold is the heap's before its own insertion
            float myT = Tcur;
            int last = -1;
            while (true) {
                const unsigned cand = __ballot_sync(0xffffffffu, valid && lane > last && d < myT);
                if (cand == 0) break;
                const int l0 = __ffs(cand) - 1;
                heap.insert(__shfl_sync(0xffffffffu, d, l0));
                Tcur = heap.worst();
                if (lane > l0) myT = Tcur;
                last = l0;
            }
            if (valid) T[i] = myT;
        }
    }
}

// v_i = d_i when d_i < T_i, else the first checkpoint value >= T_i (d_i if none), written over T_i.
__global__ void __launch_bounds__(256) compat_values_kernel(CompatArgs a, int q_count) {
    const int64_t n = a.n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)q_count * n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t qi = e / n, i = e - qi * n;
        const float d = a.D[e];
        const float t = a.T[e];
        float v = d;
        if (!(d < t)) {
            const float* P = a.P + qi * a.ncp * n + i;
            for (int c = 0; c < a.ncp; ++c) {
                const float p = P[(int64_t)c * n];
                if (p >= t) {
                    v = p;
                    break;
                }
            }
        }
        a.T[e] = v;
    }
}

int compat_num_checkpoints(int dim) { return ref_num_checkpoints(dim); }

int launch_compat(CompatArgs a, int q_begin, int q_count, cudaStream_t st) {
    ANN_CHECK_ARG(a.k >= 1 && a.k <= 512, "reference mode: k=%d outside [1, 512]", a.k);
    ANN_CHECK_ARG(a.dim >= 1 && a.dim <= 4096, "reference mode: dim=%d outside [1, 4096]", a.dim);
    if (q_count <= 0 || a.n == 0) return ANN_OK;
    a.q_end = q_begin + q_count;
    const size_t smem = sizeof(float) * kCompatQG * a.dim;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(compat_partials_kernel)));
    const int64_t rblocks = std::min<int64_t>(ceil_div(a.n, 16), kNumSMs * 8);
    dim3 g1((unsigned)rblocks, (unsigned)ceil_div(q_count, kCompatQG));
    compat_partials_kernel<<<g1, 256, smem, st>>>(a, q_begin);
    ANN_LAUNCH_CHECK();
    compat_threshold_kernel<<<(unsigned)ceil_div(q_count, 4), 128, 0, st>>>(a, q_begin);
    ANN_LAUNCH_CHECK();
    compat_values_kernel<<<(unsigned)std::min<int64_t>(ceil_div((int64_t)q_count * a.n, 256), 16 * kNumSMs), 256, 0,
                           st>>>(a, q_count);
    ANN_LAUNCH_CHECK();
    RadixSelectArgs rs{};
    rs.keys = a.T;
    rs.ld = a.n;
    rs.R = a.k;
    rs.out_key = a.kbuf;
    rs.out_id = a.ibuf;
    int rc = launch_radix_select(rs, q_count, st);
    if (rc) return rc;
    return launch_sort_topk(a.kbuf, a.ibuf, q_count, a.k, 0, a.out_ids ? a.out_ids + (int64_t)q_begin * a.k : nullptr,
                            a.out_dists ? a.out_dists + (int64_t)q_begin * a.k : nullptr, st);
}

}  // namespace annb

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
// Pass 2 (compat_select_kernel) is one warp per query walking the rows in order: the running
// 64-heap is replayed only at insertions (rows with D < T, which are rare once T settles), each
// row's T_i is known exactly, v_i is picked from P, and the warp keeps the k best (v_i, i) pairs.
#include "common.cuh"
#include "compat.cuh"
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

__global__ void __launch_bounds__(128) compat_select_kernel(CompatArgs a, int q_begin) {
    constexpr int WARPS = 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int cap = topk_cap(a.k);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* sKey = reinterpret_cast<float*>(smem_raw) + warp * cap;
    int* sId = reinterpret_cast<int*>(reinterpret_cast<float*>(smem_raw) + WARPS * cap) + warp * cap;
    const int qi = blockIdx.x * WARPS + warp;  // within chunk
    if (q_begin + qi >= a.q_end) return;
    const int k = a.k;
    WarpTopK top;
    top.init(sKey, sId, k);
    ref_replay(a.D + (int64_t)qi * a.n, a.P + (int64_t)qi * a.ncp * a.n, a.n, a.ncp, 0, a.n, k < 64 ? k : 64,
               [&](int64_t i, float v, bool valid) { top.offer(v, (int)i, valid); });
    top.compact();
    const int cnt = top.count;
    const int64_t qo = q_begin + qi;
    for (int e = lane; e < k; e += 32) {
        const bool ok = e < cnt;
        if (a.out_ids) a.out_ids[qo * k + e] = ok ? (int64_t)sId[e] : -1;
        if (a.out_dists) a.out_dists[qo * k + e] = ok ? sKey[e] : kInf;
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
    const unsigned g2 = (unsigned)ceil_div(q_count, 4);
    const size_t smem2 = (size_t)4 * topk_cap(a.k) * 8;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(compat_select_kernel)));
    compat_select_kernel<<<g2, 128, smem2, st>>>(a, q_begin);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

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

namespace annb {

__device__ __forceinline__ float fold16(float lane_val) {
    // lanes j and j+8, then the halving fold of the 8 partial sums (simd.h:21-28 as compiled)
    float t = __fadd_rn(lane_val, __shfl_xor_sync(0xffffffffu, lane_val, 8));
    float a = __fadd_rn(t, __shfl_xor_sync(0xffffffffu, t, 4));
    float b = __fadd_rn(a, __shfl_xor_sync(0xffffffffu, a, 2));
    return __fadd_rn(b, __shfl_xor_sync(0xffffffffu, b, 1));
}

// grid: (row blocks, query groups); block: 256 threads = 16 rows x 16 lanes.
__global__ void __launch_bounds__(256) compat_partials_kernel(CompatArgs a, int q_begin) {
    extern __shared__ float sQ[];  // [QG][dim]
    const int lane = threadIdx.x & 15;
    const int grp = threadIdx.x >> 4;
    const int qg0 = q_begin + blockIdx.y * kCompatQG;
    const int nqg = min(kCompatQG, a.q_end - qg0);
    for (int e = threadIdx.x; e < nqg * a.dim; e += blockDim.x) sQ[e] = a.q[(int64_t)(qg0 + e / a.dim) * a.ldq + e % a.dim];
    __syncthreads();
    const int full16 = a.dim / 16;
    const int rem = a.dim - full16 * 16;
    const int ncp = a.ncp;
    for (int64_t r0 = (int64_t)blockIdx.x * 16; r0 < a.n; r0 += (int64_t)gridDim.x * 16) {
        const int64_t row = r0 + grp;
        const bool valid = row < a.n;
        const float* x = a.base + (valid ? row : 0) * a.ldb;
        for (int qq = 0; qq < nqg; ++qq) {
            const float* q = sQ + qq * a.dim;
            const int64_t qi = qg0 + qq - q_begin;  // index within this chunk of queries
            float acc = 0.f;
            int cp = 0;
            for (int c = 0; c < full16; ++c) {
                const float diff = __fsub_rn(x[c * 16 + lane], q[c * 16 + lane]);
                acc = __fadd_rn(acc, __fmul_rn(diff, diff));
                if (c % 6 == 5) {  // i % 96 == 80 at chunk start i = 16c
                    const float p = fold16(acc);
                    if (lane == 0 && valid) a.P[((int64_t)qi * ncp + cp) * a.n + row] = p;
                    ++cp;
                }
            }
            float sum = fold16(acc);  // the final check after the vector loop
            if (lane == 0 && valid) {
                a.P[((int64_t)qi * ncp + (ncp - 1)) * a.n + row] = sum;
                int i = full16 * 16;
                if (rem >= 8) {
                    float t[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const float diff = __fsub_rn(x[i + j], q[i + j]);
                        t[j] = __fmul_rn(diff, diff);
                    }
                    const float a0 = __fadd_rn(t[0], t[4]), a1 = __fadd_rn(t[1], t[5]);
                    const float a2 = __fadd_rn(t[2], t[6]), a3 = __fadd_rn(t[3], t[7]);
                    sum = __fadd_rn(sum, __fadd_rn(__fadd_rn(a0, a2), __fadd_rn(a1, a3)));
                    i += 8;
                }
                for (; i < a.dim; ++i) {
                    const float diff = __fsub_rn(x[i], q[i]);
                    sum = __fmaf_rn(diff, diff, sum);
                }
                a.D[(int64_t)qi * a.n + row] = sum;
            }
        }
    }
}

// The reference's sorted worst-last heap of `lim` values (linear_index.cpp:50-58), held by one
// warp: lane l owns slots l and l+32. Only values matter (they set the threshold).
struct WarpHeap64 {
    float lo, hi;  // slots lane and lane+32
    int lim;

    __device__ void init(int lim_) {
        lim = lim_;
        lo = FLT_MAX;
        hi = FLT_MAX;
    }
    __device__ float worst() const {
        const int s = lim - 1;
        const float v = s < 32 ? lo : hi;
        return __shfl_sync(0xffffffffu, v, s & 31);
    }
    // Insert v (caller guarantees v < worst()).
    __device__ void insert(float v) {
        const int lane = threadIdx.x & 31;
        const int pos = __popc(__ballot_sync(0xffffffffu, lane < lim - 1 && lo <= v)) +
                        __popc(__ballot_sync(0xffffffffu, lane + 32 < lim - 1 && hi <= v));
        const float up_lo = __shfl_up_sync(0xffffffffu, lo, 1);
        const float lo31 = __shfl_sync(0xffffffffu, lo, 31);
        const float up_hi = __shfl_up_sync(0xffffffffu, hi, 1);
        const float prev_lo = up_lo;                       // slot lane-1 (lane > 0)
        const float prev_hi = lane == 0 ? lo31 : up_hi;    // slot lane+31
        const int s_lo = lane, s_hi = lane + 32;
        float nlo = lo, nhi = hi;
        if (s_lo < lim) nlo = s_lo < pos ? lo : (s_lo == pos ? v : prev_lo);
        if (s_hi < lim) nhi = s_hi < pos ? hi : (s_hi == pos ? v : prev_hi);
        lo = nlo;
        hi = nhi;
    }
};

__global__ void __launch_bounds__(128) compat_select_kernel(CompatArgs a, int q_begin) {
    constexpr int WARPS = 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int cap = topk_cap(a.k);
    float* sKey = reinterpret_cast<float*>(smem_raw) + (threadIdx.x >> 5) * cap;
    int* sId = reinterpret_cast<int*>(reinterpret_cast<float*>(smem_raw) + WARPS * cap) + (threadIdx.x >> 5) * cap;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qi = blockIdx.x * WARPS + warp;  // within chunk
    if (q_begin + qi >= a.q_end) return;
    const int k = a.k;
    WarpHeap64 heap;
    heap.init(k < 64 ? k : 64);
    WarpTopK top;
    top.init(sKey, sId, k);
    const float* D = a.D + (int64_t)qi * a.n;
    const float* P = a.P + (int64_t)qi * a.ncp * a.n;
    float T = FLT_MAX;
    float d_next = lane < a.n ? D[lane] : kInf;
    for (int64_t r0 = 0; r0 < a.n; r0 += 32) {
        const int64_t row = r0 + lane;
        const bool valid = row < a.n;
        const float d = d_next;
        d_next = (row + 32 < a.n) ? D[row + 32] : kInf;
        float myT = T;
        int last = -1;
        while (true) {
            const unsigned cand = __ballot_sync(0xffffffffu, valid && lane > last && d < myT);
            if (cand == 0) break;
            const int l0 = __ffs(cand) - 1;
            const float v0 = __shfl_sync(0xffffffffu, d, l0);
            heap.insert(v0);
            T = heap.worst();
            if (lane > l0) myT = T;
            last = l0;
        }
        float v = d;
        if (valid && !(d < myT)) {
            for (int c = 0; c < a.ncp; ++c) {
                const float p = P[(int64_t)c * a.n + row];
                if (p >= myT) {
                    v = p;
                    break;
                }
            }
        }
        top.offer(v, (int)row, valid);
    }
    top.compact();
    const int cnt = top.count;
    const int64_t qo = q_begin + qi;
    for (int e = lane; e < k; e += 32) {
        const bool ok = e < cnt;
        if (a.out_ids) a.out_ids[qo * k + e] = ok ? (int64_t)sId[e] : -1;
        if (a.out_dists) a.out_dists[qo * k + e] = ok ? sKey[e] : kInf;
    }
}

int compat_num_checkpoints(int dim) { return dim / 16 / 6 + 1; }

int launch_compat(CompatArgs a, int q_begin, int q_count, cudaStream_t st) {
    ANN_CHECK_ARG(a.k >= 1 && a.k <= 512, "reference mode: k=%d outside [1, 512]", a.k);
    ANN_CHECK_ARG(a.dim >= 1 && a.dim <= 4096, "reference mode: dim=%d outside [1, 4096]", a.dim);
    if (q_count <= 0 || a.n == 0) return ANN_OK;
    a.q_end = q_begin + q_count;
    const size_t smem = sizeof(float) * kCompatQG * a.dim;
    ANN_CUDA_TRY(cudaFuncSetAttribute(compat_partials_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t rblocks = std::min<int64_t>(ceil_div(a.n, 16), kNumSMs * 8);
    dim3 g1((unsigned)rblocks, (unsigned)ceil_div(q_count, kCompatQG));
    compat_partials_kernel<<<g1, 256, smem, st>>>(a, q_begin);
    ANN_LAUNCH_CHECK();
    const unsigned g2 = (unsigned)ceil_div(q_count, 4);
    const size_t smem2 = (size_t)4 * topk_cap(a.k) * 8;
    ANN_CUDA_TRY(cudaFuncSetAttribute(compat_select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
    compat_select_kernel<<<g2, 128, smem2, st>>>(a, q_begin);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

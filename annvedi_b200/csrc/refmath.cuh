// The reference's distance arithmetic, reproduced bit for bit by a group of 16 threads.
//
// compute_l2_distance and compute_l2_distance_quantized (competitors/ivf_lsh/src/simd.h:32-64,
// 118-154; the AVX-512 build the reference is compiled to with -O3 -ffast-math) keep 16 lane sums:
// lane j adds elements j, j+16, j+32, ... For FP32 each step is an unfused multiply then add; for
// SQ8 it is a fused (code*scale - q_shifted) followed by a fused square-add. At every checkpoint
// (after 96, 192, ... elements, simd.h:45) and after the last full 16-chunk the lanes are folded:
// lanes j and j+8 first, then the compiled reference's halving fold of the 8 sums. Leftover
// elements (dim % 16) follow the compiled code: for FP32 one fused 8-wide chunk folded the same way
// and then scalar fused steps; for SQ8 scalar fused steps.
//
// Here thread j of a 16-thread group plays lane j; folds use shuffles inside the group, so every
// lane of the group ends with the same value.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace annb {

__device__ __forceinline__ float ref_fold16(float lane_val) {
    float t = __fadd_rn(lane_val, __shfl_xor_sync(0xffffffffu, lane_val, 8));
    float a = __fadd_rn(t, __shfl_xor_sync(0xffffffffu, t, 4));
    float b = __fadd_rn(a, __shfl_xor_sync(0xffffffffu, a, 2));
    return __fadd_rn(b, __shfl_xor_sync(0xffffffffu, b, 1));
}

// Number of checkpoint values (checkpoints + the final fold) for `dim`.
__host__ __device__ inline int ref_num_checkpoints(int dim) { return dim / 16 / 6 + 1; }

// FP32 distance between x and q (both `dim` floats), computed by the calling 16-thread group.
// Calls emit(c, value) for checkpoint c = 0..ref_num_checkpoints(dim)-1 (the last is the final
// fold before the remainder). Returns the full distance in every lane of the group. All 32 lanes of
// the warp must call it together (both halves run a group each).
template <class Emit>
__device__ __forceinline__ float ref_l2_f32(const float* __restrict__ x, const float* __restrict__ q, int dim,
                                            Emit&& emit) {
    const int lane = threadIdx.x & 15;
    const int full16 = dim >> 4;
    float acc = 0.f;
    int cp = 0;
    for (int c = 0; c < full16; ++c) {
        const float diff = __fsub_rn(x[c * 16 + lane], q[c * 16 + lane]);
        acc = __fadd_rn(acc, __fmul_rn(diff, diff));
        if (c % 6 == 5) emit(cp++, ref_fold16(acc));
    }
    float sum = ref_fold16(acc);
    emit(cp, sum);
    if (lane == 0) {
        int i = full16 * 16;
        if (dim - i >= 8) {
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
        for (; i < dim; ++i) {
            const float diff = __fsub_rn(x[i], q[i]);
            sum = __fmaf_rn(diff, diff, sum);
        }
    }
    return __shfl_sync(0xffffffffu, sum, 0, 16);
}

// SQ8 distance sum_d (code[d]*scale[d] - qs[d])^2, the reference's arithmetic.
template <class Emit>
__device__ __forceinline__ float ref_l2_sq8(const uint8_t* __restrict__ code, const float* __restrict__ qs,
                                            const float* __restrict__ scale, int dim, Emit&& emit) {
    const int lane = threadIdx.x & 15;
    const int full16 = dim >> 4;
    float acc = 0.f;
    int cp = 0;
    for (int c = 0; c < full16; ++c) {
        const int d = c * 16 + lane;
        const float diff = __fmaf_rn((float)code[d], scale[d], -qs[d]);
        acc = __fmaf_rn(diff, diff, acc);
        if (c % 6 == 5) emit(cp++, ref_fold16(acc));
    }
    float sum = ref_fold16(acc);
    emit(cp, sum);
    if (lane == 0) {
        for (int i = full16 * 16; i < dim; ++i) {
            const float diff = __fmaf_rn((float)code[i], scale[i], -qs[i]);
            sum = __fmaf_rn(diff, diff, sum);
        }
    }
    return __shfl_sync(0xffffffffu, sum, 0, 16);
}

struct NoEmit {
    __device__ __forceinline__ void operator()(int, float) const {}
};

// The reference's sorted worst-last heap of `lim` (<= 64) values (linear_index.cpp:50-58,
// lsh_index_optimized.cpp:112-120), held by one warp: lane l owns slots l and l+32. Only the
// values matter: they set the early-abandon threshold.
struct WarpHeap64 {
    float lo, hi;
    int lim;

    __device__ void init(int lim_) {
        lim = lim_;
        lo = 3.402823466e+38f;  // FLT_MAX, the reference's empty slot
        hi = 3.402823466e+38f;
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
        const float prev_hi = lane == 0 ? lo31 : up_hi;
        const int s_lo = lane, s_hi = lane + 32;
        float nlo = lo, nhi = hi;
        if (s_lo < lim) nlo = s_lo < pos ? lo : (s_lo == pos ? v : up_lo);
        if (s_hi < lim) nhi = s_hi < pos ? hi : (s_hi == pos ? v : prev_hi);
        lo = nlo;
        hi = nhi;
    }
};

// One warp replays the reference's early-abandon scan over values D[0..len) (full distances) with
// checkpoint values P[c*stride + i] (c < ncp): returns through `out(i, v_i)` the value the
// reference ranks position i by -- D[i] when it beats the running 64th-best, else the first
// checkpoint value reaching it. `lim` = min(k, 64).
template <class Out>
__device__ void ref_replay(const float* __restrict__ D, const float* __restrict__ P, int64_t stride, int ncp,
                           int64_t begin, int64_t end, int lim, Out&& out) {
    const int lane = threadIdx.x & 31;
    WarpHeap64 heap;
    heap.init(lim);
    float T = 3.402823466e+38f;
    float d_next = begin + lane < end ? D[begin + lane] : __int_as_float(0x7f800000);
    for (int64_t r0 = begin; r0 < end; r0 += 32) {
        const int64_t i = r0 + lane;
        const bool valid = i < end;
        const float d = d_next;
        d_next = (i + 32 < end) ? D[i + 32] : __int_as_float(0x7f800000);
        float myT = T;
        int last = -1;
        while (true) {
            const unsigned cand = __ballot_sync(0xffffffffu, valid && lane > last && d < myT);
            if (cand == 0) break;
            const int l0 = __ffs(cand) - 1;
            heap.insert(__shfl_sync(0xffffffffu, d, l0));
            T = heap.worst();
            if (lane > l0) myT = T;
            last = l0;
        }
        float v = d;
        if (valid && !(d < myT)) {
            for (int c = 0; c < ncp; ++c) {
                const float p = P[(int64_t)c * stride + i];
                if (p >= myT) {
                    v = p;
                    break;
                }
            }
        }
        out(i, v, valid);
    }
}

}  // namespace annb

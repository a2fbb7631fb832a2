// Shared helpers for the annvedi_b200 kernels and the C ABI: error reporting, (key, id) pair
// ordering, warp-level bitonic sorting and the small per-warp top-k buffer used by every
// selection step.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cfloat>
#include <climits>
#include <cstdio>
#include <mutex>
#include <set>
#include <string>
#include <utility>

#include "../../include/annvedi_b200.h"

namespace annb {

// Raises a kernel's dynamic shared-memory limit to the device's opt-in maximum, once per (kernel,
// device). Launches of any size up to that limit then need no attribute call, so concurrent host
// threads never change a kernel's attributes while another thread launches it.
inline cudaError_t smem_optin(const void* func) {
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (done.count({func, dev})) return cudaSuccess;
    cudaFuncAttributes fa;
    if ((e = cudaFuncGetAttributes(&fa, func)) != cudaSuccess) return e;
    int optin = 0;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes)) !=
        cudaSuccess)
        return e;
    done.insert({func, dev});
    return cudaSuccess;
}

// ---------------------------------------------------------------------------------------------
// Host-side error state: the last failing call's message, per host thread.
// ---------------------------------------------------------------------------------------------
void set_error(const char* fmt, ...);
void clear_error();

#define ANN_CUDA_TRY(expr)                                                                        \
    do {                                                                                          \
        cudaError_t _e = (expr);                                                                  \
        if (_e != cudaSuccess) {                                                                  \
            ::annb::set_error("CUDA error %s (%s) at %s:%d", cudaGetErrorName(_e),                \
                              cudaGetErrorString(_e), __FILE__, __LINE__);                        \
            return ANN_ERR_CUDA;                                                                  \
        }                                                                                         \
    } while (0)

#define ANN_CHECK_ARG(cond, ...)                                                                  \
    do {                                                                                          \
        if (!(cond)) {                                                                            \
            ::annb::set_error(__VA_ARGS__);                                                       \
            return ANN_ERR_INVALID;                                                               \
        }                                                                                         \
    } while (0)

// Counts every kernel launch (ann_kernel_launches) and checks the launch itself; asynchronous
// faults surface at the next synchronising call.
void count_launch();
#define ANN_LAUNCH_CHECK()            \
    do {                              \
        ::annb::count_launch();       \
        ANN_CUDA_TRY(cudaGetLastError()); \
    } while (0)

constexpr int kWarp = 32;
constexpr int kNumSMs = 148;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
__host__ __device__ inline int pow2_ceil(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// ---------------------------------------------------------------------------------------------
// (key, id) pairs ordered by key, ties by lower id -- the order of std::pair<float,int> used by
// LinearIndex::query's partial_sort (competitors/linear/src/linear_index.cpp:111).
// Empty slots hold (+inf, INT_MAX).
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ bool pair_less(float ka, int ia, float kb, int ib) {
    return ka < kb || (ka == kb && ia < ib);
}

constexpr float kInf = __builtin_huge_valf();
constexpr int kNoId = INT_MAX;

// Bitonic sort, by one warp, of `cap` (key, id) pairs in shared memory (cap a power of two),
// ascending in pair order. Loop-based so one instance serves every buffer size.
__device__ __forceinline__ void warp_sort_smem(float* key, int* id, int cap) {
    const int lane = threadIdx.x & 31;
    for (int size = 2; size <= cap; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < (cap >> 1); t += 32) {
                const int lo = 2 * t - (t & (stride - 1));
                const int hi = lo + stride;
                const bool asc = (lo & size) == 0;
                const float kl = key[lo], kh = key[hi];
                const int il = id[lo], ih = id[hi];
                const bool sw = asc ? pair_less(kh, ih, kl, il) : pair_less(kl, il, kh, ih);
                if (sw) {
                    key[lo] = kh;
                    key[hi] = kl;
                    id[lo] = ih;
                    id[hi] = il;
                }
            }
            __syncwarp();
        }
    }
}

// Sorts a buffer holding `count` valid pairs (count <= cap) after padding the rest with empty
// slots, and keeps the best k. Returns the number kept; the bar is then key[k-1], id[k-1] when
// k pairs are kept. Warp-collective.
__device__ __forceinline__ int warp_compact_smem(float* key, int* id, int count, int cap, int k) {
    const int lane = threadIdx.x & 31;
    if (count > cap) count = cap;
    for (int e = count + lane; e < cap; e += 32) {
        key[e] = kInf;
        id[e] = kNoId;
    }
    __syncwarp();
    warp_sort_smem(key, id, cap);
    return count < k ? count : k;
}

// Buffer capacity for keeping the best k: twice the next power of two, at least 64.
__host__ __device__ inline int topk_cap(int k) {
    int p = 32;
    while (p < k) p <<= 1;
    return 2 * p;
}

// A per-warp candidate buffer in shared memory of `cap` pairs (topk_cap(k)). It keeps the best k
// pairs seen so far once compacted; (tau, tau_id) is the k-th best pair -- the bar a new pair
// must beat -- and (+inf, INT_MAX) until k pairs are held.
struct WarpTopK {
    float* key;  // [cap] shared
    int* id;     // [cap] shared
    int cap;
    int k;
    int count;   // warp-uniform
    float tau;
    int tau_id;

    __device__ void init(float* k_smem, int* i_smem, int k_) {
        key = k_smem;
        id = i_smem;
        k = k_;
        cap = topk_cap(k_);
        count = 0;
        tau = kInf;
        tau_id = kNoId;
    }

    // Sort the buffer, keep the first k pairs and update the bar. Warp-collective.
    __device__ void compact() {
        count = warp_compact_smem(key, id, count, cap, k);
        if (count == k) {
            tau = key[k - 1];
            tau_id = id[k - 1];
        }
        __syncwarp();
    }

    // Offer one pair per lane (pred false = nothing). Pairs that do not beat the bar are dropped;
    // the buffer is compacted when it would overflow. Warp-collective.
    __device__ void offer(float kv, int iv, bool pred) {
        const int lane = threadIdx.x & 31;
        bool want = pred && pair_less(kv, iv, tau, tau_id);
        unsigned m = __ballot_sync(0xffffffffu, want);
        if (m == 0) return;
        if (count + __popc(m) > cap) {
            compact();
            want = want && pair_less(kv, iv, tau, tau_id);
            m = __ballot_sync(0xffffffffu, want);
            if (m == 0) return;
        }
        const int pos = count + __popc(m & ((1u << lane) - 1u));
        if (want) {
            key[pos] = kv;
            id[pos] = iv;
        }
        count += __popc(m);
        __syncwarp();
    }
};

}  // namespace annb

// The reference's GPU quantized-filter contestant (competitors/gpu_filter/src/gpu_filter.cu) served by B200
// kernels behind its own C ABI (include/annvedi_gpu_filter.h).
//
// The reference, per query: one thread per row sums (code * scale - qshift)^2 over dim-major SQ8 codes
// (:52-63), a CUB radix sort orders all N (key, row) pairs, the first R row ids come back to the host,
// and the host re-ranks them in FP32 from the borrowed train array and partial-sorts (distance, id)
// pairs (:135-176). Here, per query:
//   gf_scan_kernel     the same key with the same FMA chain per row (8 rows per thread, one 64-bit load
//                      of 8 codes per dimension, 16 dimensions' loads in flight, scale and q - offset
//                      staged in shared memory) -- HBM-bound, N * dim code bytes per query;
//   selection          the R rows with the smallest (key, row) -- the rows the reference's stable
//                      ascending sort puts first -- in two stages: radix selection (radix_select.cu)
//                      of each of up to 64 row segments' R smallest as a set (ties to the lower row),
//                      in parallel, then the R smallest (key, row) of their union by one block
//                      (gf_union_select_kernel: an exact radix selection of the R-th key, then one of
//                      the cut among the rows that share it); one segment when the base is small or R
//                      is above the top-k kernel's bound;
//   gf_rerank_kernel   each candidate's FP32 squared distance from a device copy of train, with the
//                      reference's host arithmetic (v = p - q, acc = acc + v * v, no fused multiply-add);
//   gf_topk_kernel     the best k (distance, id) pairs in ascending order, as 64-bit keys
//                      (distance bits << 32 | id) bitonic-sorted in shared memory, chunk by chunk with
//                      the running best k kept in front.
// Only the query (dim floats) goes in and the k ids come out.
//
// Build (gf_create): exact per-dimension min / max (ivf_build.cu), the scale and offset formed on the host
// with the reference's expressions (:103-117), then gf_encode_kernel quantises with a true division and
// round-half-even (lrintf, :119-127) into the dim-major layout the scan reads.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/annvedi_gpu_filter.h"
#include "common.cuh"
#include "ivf.cuh"
#include "radix_select.cuh"
#include "runtime.cuh"

namespace annb {
namespace {

constexpr int kGfMaxDim = 4096;  // the reference's __constant__ arrays bound dim (:49-50, :80-83)
constexpr int kGfMaxK = 4096;
constexpr int kGfSortCap = 8192;  // 64-bit keys in the top-k kernel's shared buffer (64 KB)
constexpr int kGfMaxSeg = 64;     // row segments of the first selection stage
constexpr int64_t kGfSegRows = 32768;  // rows per segment, at least

__global__ void gf_encode_kernel(const float* __restrict__ x, int64_t n, int dim, int64_t npad,
                                 const float* __restrict__ scale, const float* __restrict__ offset,
                                 uint8_t* __restrict__ codes) {
    // one thread per (dimension d, row i), rows fastest: the stores of a warp are 32 consecutive bytes
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npad * dim) return;
    const int d = (int)(t / npad);
    const int64_t i = t - (int64_t)d * npad;
    int c = 0;
    if (i < n) {
        const int v = __float2int_rn(__fdiv_rn(__fsub_rn(x[i * dim + d], offset[d]), scale[d]));
        c = max(0, min(255, v));
    }
    codes[t] = (uint8_t)c;
}

// The code byte `sel` of w as a float, exactly: its bits placed in the mantissa of 2^23 (byte permute),
// then 2^23 subtracted -- two full-rate instructions where an integer-to-float conversion runs at a quarter.
// byte sel of w as a float: its bits under the exponent of 2^23, then 2^23 taken off (exact)
__device__ __forceinline__ float gf_byte_bits(uint32_t w, uint32_t sel) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u | sel));
}
// rows i (byte i of c.x) and 4 + i (byte i of c.y) as the pair a[i], with packed FP32 instructions: each
// half rounds as its scalar form (x - 2^23, fma(x, s, nq), fma(v, v, a)), so the keys are those of the
// scalar chain, at 2.5 instructions a code byte instead of 4
__device__ __forceinline__ void gf_acc8(uint2 c, float s, float nq, float2 (&a)[4]) {
    const float2 s2 = make_float2(s, s), n2 = make_float2(nq, nq), m2 = make_float2(-8388608.0f, -8388608.0f);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 x = __fadd2_rn(make_float2(gf_byte_bits(c.x, i), gf_byte_bits(c.y, i)), m2);
        const float2 v = __ffma2_rn(x, s2, n2);
        a[i] = __ffma2_rn(v, v, a[i]);
    }
}

// dist[i] = sum_d fma(code[d][i], scale[d], -(q[d] - offset[d]))^2, accumulated with fma in dimension
// order; thread t takes rows 8t .. 8t + 7 (npad a multiple of 16; rows past n get keys nobody reads): one
// 8-byte load of their codes per dimension, sixteen dimensions' loads to a batch (eight 128-thread CTAs a
// multiprocessor leave the registers for them; the small CTAs spread the rows evenly over the SMs).
constexpr int kGfScanBatch = 16;
__global__ void __launch_bounds__(128, 8) gf_scan_kernel(const uint8_t* __restrict__ codes, int64_t npad, int dim,
                                                      const float* __restrict__ scale,
                                                      const float* __restrict__ offset,
                                                      const float* __restrict__ q, float* __restrict__ dist) {
    extern __shared__ float2 gf_sn[];  // [dim] (scale, -(q - offset))
    for (int d = threadIdx.x; d < dim; d += blockDim.x) gf_sn[d] = make_float2(scale[d], -__fsub_rn(q[d], offset[d]));
    __syncthreads();
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t octs = npad >> 3;
    if (t >= octs) return;
    const uint2* col = reinterpret_cast<const uint2*>(codes) + t;
    float2 a[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    int d0 = 0;
    for (; d0 + kGfScanBatch <= dim; d0 += kGfScanBatch) {
        uint2 c[kGfScanBatch];
#pragma unroll
        for (int g = 0; g < kGfScanBatch; ++g) c[g] = __ldcs(col + (int64_t)(d0 + g) * octs);
#pragma unroll
        for (int g = 0; g < kGfScanBatch; ++g) gf_acc8(c[g], gf_sn[d0 + g].x, gf_sn[d0 + g].y, a);
    }
    for (; d0 < dim; ++d0) gf_acc8(col[(int64_t)d0 * octs], gf_sn[d0].x, gf_sn[d0].y, a);
    float4* o = reinterpret_cast<float4*>(dist) + 2 * t;
    o[0] = make_float4(a[0].x, a[1].x, a[2].x, a[3].x);
    o[1] = make_float4(a[0].y, a[1].y, a[2].y, a[3].y);
}

// One warp per candidate (two per CTA): the warp brings the candidate's row into shared memory with
// coalesced loads, then one lane applies the reference's host re-rank arithmetic (a rounded product,
// then a rounded sum, in dimension order); the distance and the row id go out as one ordered 64-bit key.
constexpr int kGfRerankWarps = 2;
__global__ void __launch_bounds__(32 * kGfRerankWarps) gf_rerank_kernel(const float* __restrict__ base, int64_t n,
                                                                        int dim, const float* __restrict__ q,
                                                                        const int* __restrict__ cand, int r,
                                                                        unsigned long long* __restrict__ keys) {
    extern __shared__ float gf_rs[];  // [dim] query, then [kGfRerankWarps][dim] rows
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = threadIdx.x; d < dim; d += blockDim.x) gf_rs[d] = q[d];
    const int j = blockIdx.x * kGfRerankWarps + warp;
    const int id = j < r ? cand[j] : -1;
    const bool ok = j < r && id >= 0 && (int64_t)id < n;
    float* row = gf_rs + dim + warp * dim;
    if (ok) {
        const float* p = base + (int64_t)id * dim;
        for (int d = lane; d < dim; d += 32) row[d] = p[d];
    }
    __syncthreads();
    if (j >= r || lane != 0) return;
    if (!ok) {
        keys[j] = ~0ull;
        return;
    }
    float acc = 0.f;
#pragma unroll 8
    for (int d = 0; d < dim; ++d) {
        const float v = __fsub_rn(row[d], gf_rs[d]);
        acc = __fadd_rn(acc, __fmul_rn(v, v));
    }
    keys[j] = ((unsigned long long)__float_as_uint(acc) << 32) | (unsigned)id;
}

// ---- the union's R smallest (key, row), by one block ----------------------------------------------------
constexpr int kGfUnionThreads = 1024;
__device__ __forceinline__ uint32_t gf_ord(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Entry j of the segments' selected sets (segment j / R, its R entries in any order): its ordered key and
// its row, or valid = false for padding.
struct GfUnion {
    const float* selk;
    const int* selp;
    const int64_t* offs;
    int R, total;
    __device__ __forceinline__ bool at(int j, uint32_t* key, uint32_t* row) const {
        const int p = selp[j];
        const float kv = selk[j];
        if (p < 0 || p == kNoId || !(kv < kInf)) return false;
        *key = gf_ord(kv);
        *row = (uint32_t)(offs[j / R] + p);
        return true;
    }
};

// The rank-th smallest (1 <= rank <= count) of the values v(j) of the entries j with sel(j), over four 8-bit
// passes of a block histogram (warp-aggregated shared atomics). Every thread returns it.
template <typename Val>
__device__ uint32_t gf_block_select(const GfUnion& u, Val val, int64_t rank, int* hist, int* pick) {
    uint32_t prefix = 0, pmask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        for (int j0 = 0; j0 < u.total; j0 += blockDim.x) {  // uniform trip count: whole warps match
            const int j = j0 + threadIdx.x;
            uint32_t v = 0;
            const bool ok = j < u.total && val(j, &v) && (v & pmask) == prefix;
            const uint32_t dgt = (v >> shift) & 255u;
            const unsigned peers = __match_any_sync(0xffffffffu, ok ? dgt : 0xffffffffu);
            if (ok && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[dgt], __popc(peers));
        }
        __syncthreads();
        if (threadIdx.x < 32) {  // the digit holding rank, and the count below it
            const int lane = threadIdx.x;
            int c[8], sum = 0;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                c[i] = hist[lane * 8 + i];
                sum += c[i];
            }
            int incl = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int excl = incl - sum;
            if (excl < rank && rank <= incl) {
                int acc = excl;
                for (int i = 0; i < 8; ++i) {
                    if (acc + c[i] >= rank) {
                        pick[0] = lane * 8 + i;
                        pick[1] = acc;
                        break;
                    }
                    acc += c[i];
                }
            }
        }
        __syncthreads();
        prefix |= (uint32_t)pick[0] << shift;
        rank -= pick[1];
        pmask |= 255u << shift;
        __syncthreads();  // pick is rewritten by the next pass
    }
    return prefix;
}

// out[0 .. min(R, valid)) = the rows of the R smallest (key, row) of the union, in no particular order (the
// re-rank reads them as a set): the keys below the R-th smallest key, then the rows with that key below the
// cut among them, found by a second selection over the tie rows (rows are distinct, so the cut is exact).
// Entries past the valid count are -1. One block.
__global__ void __launch_bounds__(kGfUnionThreads) gf_union_select_kernel(GfUnion u, int* __restrict__ out) {
    __shared__ int hist[256];
    __shared__ int pick[2];
    __shared__ int sCount[3];  // valid entries, written below, written ties
    if (threadIdx.x == 0) sCount[0] = sCount[1] = sCount[2] = 0;
    __syncthreads();
    int nv = 0;
    for (int j = threadIdx.x; j < u.total; j += blockDim.x) {
        uint32_t k, r;
        nv += u.at(j, &k, &r);
    }
    atomicAdd(&sCount[0], nv);
    __syncthreads();
    const int valid = sCount[0];
    const int R = min(u.R, valid);
    if (R == 0) {
        for (int j = threadIdx.x; j < u.R; j += blockDim.x) out[j] = -1;
        return;
    }
    const uint32_t T = gf_block_select(u, [&](int j, uint32_t* v) {
        uint32_t r;
        return u.at(j, v, &r);
    }, R, hist, pick);
    // keys below T all belong; count them while writing
    for (int j = threadIdx.x; j < u.total; j += blockDim.x) {
        uint32_t k, r;
        if (u.at(j, &k, &r) && k < T) out[atomicAdd(&sCount[1], 1)] = (int)r;
    }
    __syncthreads();
    const int below = sCount[1];
    const int need = R - below;  // >= 1: T itself is the R-th key
    const uint32_t Trow = gf_block_select(u, [&](int j, uint32_t* v) {
        uint32_t k;
        return u.at(j, &k, v) && k == T;
    }, need, hist, pick);
    for (int j = threadIdx.x; j < u.total; j += blockDim.x) {
        uint32_t k, r;
        if (u.at(j, &k, &r) && k == T && r <= Trow) out[below + atomicAdd(&sCount[2], 1)] = (int)r;
    }
    for (int j = R + threadIdx.x; j < u.R; j += blockDim.x) out[j] = -1;
}

// The k smallest of r 64-bit keys, ascending, into out (the low 32 bits: row ids). P (a power of two,
// <= kGfSortCap) keys sit in shared memory: the running best k in front, then the next P - k keys;
// each round bitonic-sorts all P. P is the smallest power of two >= min(r + k, Pmax), Pmax the keys the
// launch's shared memory holds.
template <typename OutT>
__global__ void __launch_bounds__(512) gf_topk_kernel(const unsigned long long* __restrict__ keys, int r, int k,
                                                      int Pmax, OutT* __restrict__ out) {
    extern __shared__ unsigned long long gf_buf[];
    int P = 64;
    while (P < min(r + k, Pmax)) P <<= 1;
    const int C = P - k;
    for (int i = threadIdx.x; i < k; i += blockDim.x) gf_buf[i] = ~0ull;
    for (int b0 = 0; b0 < r; b0 += C) {
        for (int i = threadIdx.x; i < C; i += blockDim.x) gf_buf[k + i] = b0 + i < r ? keys[b0 + i] : ~0ull;
        __syncthreads();
        for (int size = 2; size <= P; size <<= 1) {
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int t = threadIdx.x; t < (P >> 1); t += blockDim.x) {
                    const int i = 2 * t - (t & (stride - 1));
                    const int j = i + stride;
                    const unsigned long long a = gf_buf[i], b = gf_buf[j];
                    if ((a > b) == ((i & size) == 0)) {
                        gf_buf[i] = b;
                        gf_buf[j] = a;
                    }
                }
                __syncthreads();
            }
        }
    }
    for (int i = threadIdx.x; i < k; i += blockDim.x) out[i] = (OutT)(unsigned)(gf_buf[i] & 0xffffffffull);
}

}  // namespace
}  // namespace annb

using namespace annb;

struct gf_handle {
    int64_t n = 0, npad = 0;
    int dim = 0, device = 0;
    cudaStream_t st = nullptr;
    uint8_t* codes = nullptr;  // [dim][npad], dim-major
    float* base = nullptr;     // [n][dim] FP32 copy of train (the re-rank's rows)
    float* scale = nullptr;    // [dim]
    float* offset = nullptr;   // [dim]
    float* q = nullptr;        // [dim]
    float* dist = nullptr;     // [npad]
    float* selk = nullptr;     // [rcap]
    int* seli = nullptr;       // [rcap]
    int* uni = nullptr;        // [rcap] the union's R rows (several segments)
    unsigned long long* keys = nullptr;  // [rcap]
    long long* out = nullptr;  // [kGfMaxK]
    int64_t* segs = nullptr;   // [2][kGfMaxSeg] segment starts and lengths (fixed by n)
    int nseg = 1;              // first-stage segments when R <= kGfMaxK
    float* hq = nullptr;       // pinned staging: the query
    long long* hout = nullptr; // pinned staging: the ids
    int64_t rcap = 0;
    // gf_query's launches and copies for a (k, r), captured once and replayed as one graph
    struct Graph {
        int k, r;
        cudaGraphExec_t exec;  // null: capture failed for this (k, r); the launches run one by one
    };
    std::vector<Graph> graphs;
    std::atomic<long long> ndist{0};
    std::mutex mu;
};

namespace {

void gf_drop_graphs(gf_handle* h) {
    for (auto& gr : h->graphs)
        if (gr.exec) cudaGraphExecDestroy(gr.exec);
    h->graphs.clear();
}

void gf_release(gf_handle* h) {
    DeviceGuard g(h->device);
    gf_drop_graphs(h);
    for (void* p : {(void*)h->codes, (void*)h->base, (void*)h->scale, (void*)h->offset, (void*)h->q, (void*)h->dist,
                    (void*)h->selk, (void*)h->seli, (void*)h->keys, (void*)h->out, (void*)h->segs,
                    (void*)h->uni})
        if (p) cudaFree(p);
    if (h->hq) cudaFreeHost(h->hq);
    if (h->hout) cudaFreeHost(h->hout);
    if (h->st) cudaStreamDestroy(h->st);
}

int gf_build(gf_handle* h, const float* train) {
    const int64_t n = h->n;
    const int dim = h->dim;
    ANN_CUDA_TRY(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    ANN_CUDA_TRY(cudaMalloc(&h->base, sizeof(float) * (size_t)n * dim));
    ANN_CUDA_TRY(cudaMalloc(&h->codes, (size_t)h->npad * dim));
    ANN_CUDA_TRY(cudaMalloc(&h->scale, sizeof(float) * dim));
    ANN_CUDA_TRY(cudaMalloc(&h->offset, sizeof(float) * dim));
    ANN_CUDA_TRY(cudaMalloc(&h->q, sizeof(float) * dim));
    ANN_CUDA_TRY(cudaMalloc(&h->dist, sizeof(float) * (size_t)h->npad));
    ANN_CUDA_TRY(cudaMalloc(&h->out, sizeof(long long) * kGfMaxK));
    ANN_CUDA_TRY(cudaMalloc(&h->segs, sizeof(int64_t) * 2 * kGfMaxSeg));
    ANN_CUDA_TRY(cudaHostAlloc(&h->hq, sizeof(float) * dim, cudaHostAllocDefault));
    ANN_CUDA_TRY(cudaHostAlloc(&h->hout, sizeof(long long) * kGfMaxK, cudaHostAllocDefault));
    // first-stage segments: about kGfSegRows rows each, at most kGfMaxSeg
    h->nseg = (int)std::clamp<int64_t>(n / kGfSegRows, 1, kGfMaxSeg);
    std::vector<int64_t> seg(2 * kGfMaxSeg, 0);
    const int64_t L = ceil_div(n, h->nseg);
    for (int s2 = 0; s2 < h->nseg; ++s2) {
        seg[s2] = s2 * L;
        seg[kGfMaxSeg + s2] = std::max<int64_t>(0, std::min(n, (s2 + 1) * L) - s2 * L);
    }
    ANN_CUDA_TRY(cudaMemcpyAsync(h->segs, seg.data(), sizeof(int64_t) * 2 * kGfMaxSeg, cudaMemcpyHostToDevice, h->st));
    ANN_CUDA_TRY(cudaMemcpyAsync(h->base, train, sizeof(float) * (size_t)n * dim, cudaMemcpyHostToDevice, h->st));
    // exact per-dimension minimum and maximum, then the reference's scale and offset (host FP32)
    float *mn = nullptr, *mx = nullptr;
    ANN_CUDA_TRY(cudaMalloc(&mn, sizeof(float) * dim * 2));
    mx = mn + dim;
    int rc = launch_sq8_minmax(h->base, n, dim, dim, mn, mx, h->st);
    std::vector<float> hmn(dim), hmx(dim), sc(dim), off(dim);
    if (rc == ANN_OK) {
        cudaError_t e = cudaMemcpyAsync(hmn.data(), mn, sizeof(float) * dim, cudaMemcpyDeviceToHost, h->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hmx.data(), mx, sizeof(float) * dim, cudaMemcpyDeviceToHost, h->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
        if (e != cudaSuccess) {
            set_error("CUDA error %s (%s) at %s:%d", cudaGetErrorName(e), cudaGetErrorString(e), __FILE__, __LINE__);
            rc = ANN_ERR_CUDA;
        }
    }
    cudaFree(mn);
    if (rc) return rc;
    for (int d = 0; d < dim; ++d) {
        const float range = hmx[d] - hmn[d];
        sc[d] = range > 1e-8f ? range / 255.0f : 1.0f;
        off[d] = hmn[d];
    }
    ANN_CUDA_TRY(cudaMemcpyAsync(h->scale, sc.data(), sizeof(float) * dim, cudaMemcpyHostToDevice, h->st));
    ANN_CUDA_TRY(cudaMemcpyAsync(h->offset, off.data(), sizeof(float) * dim, cudaMemcpyHostToDevice, h->st));
    const int64_t total = h->npad * dim;
    gf_encode_kernel<<<(unsigned)ceil_div(total, 256), 256, 0, h->st>>>(h->base, n, dim, h->npad, h->scale,
                                                                         h->offset, h->codes);
    ANN_LAUNCH_CHECK();
    ANN_CUDA_TRY(cudaStreamSynchronize(h->st));  // sc / off (host) feed the copies above
    return ANN_OK;
}

int gf_reserve(gf_handle* h, int64_t r) {
    if (r <= h->rcap) return ANN_OK;
    gf_drop_graphs(h);  // the graphs hold the old buffers' addresses
    if (h->selk) cudaFree(h->selk);
    if (h->seli) cudaFree(h->seli);
    if (h->keys) cudaFree(h->keys);
    if (h->uni) cudaFree(h->uni);
    h->uni = nullptr;
    h->selk = nullptr;
    h->seli = nullptr;
    h->keys = nullptr;
    h->rcap = 0;
    ANN_CUDA_TRY(cudaMalloc(&h->selk, sizeof(float) * (size_t)r));
    ANN_CUDA_TRY(cudaMalloc(&h->seli, sizeof(int) * (size_t)r));
    ANN_CUDA_TRY(cudaMalloc(&h->keys, sizeof(unsigned long long) * (size_t)r));
    ANN_CUDA_TRY(cudaMalloc(&h->uni, sizeof(int) * (size_t)r));
    h->rcap = r;
    return ANN_OK;
}

// keys [r] (or the near set, see gf_topk_kernel) -> the k smallest, ascending; shared memory for
// min(r + k, kGfSortCap) keys rounded up to a power of two.
template <typename OutT>
int launch_gf_topk(const unsigned long long* keys, int64_t r, int k, OutT* out, cudaStream_t st) {
    int Pmax = 64;
    while (Pmax < std::min<int64_t>(r + k, kGfSortCap)) Pmax <<= 1;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(gf_topk_kernel<OutT>)));
    gf_topk_kernel<OutT><<<1, 512, sizeof(unsigned long long) * Pmax, st>>>(keys, (int)r, k, Pmax, out);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// The launches and copies of one query on h->st (query from h->hq in, ids to h->hout out), no sync.
int gf_enqueue(gf_handle* h, int k, int r, int nseg) {
    const int64_t n = h->n;
    const int dim = h->dim;
    cudaStream_t st = h->st;
    int rc;
    ANN_CUDA_TRY(cudaMemcpyAsync(h->q, h->hq, sizeof(float) * dim, cudaMemcpyHostToDevice, st));
    gf_scan_kernel<<<(unsigned)ceil_div(h->npad >> 3, 128), 128, sizeof(float) * 2 * dim, st>>>(
        h->codes, h->npad, dim, h->scale, h->offset, h->q, h->dist);
    ANN_LAUNCH_CHECK();
    RadixSelectArgs sa{};
    sa.keys = h->dist;
    sa.ld = n;
    sa.R = r;
    sa.out_key = h->selk;
    sa.out_id = h->seli;
    if (nseg > 1) {
        sa.offs = h->segs;
        sa.lens = h->segs + kGfMaxSeg;
    }
    if ((rc = launch_radix_select(sa, nseg, st))) return rc;
    if (nseg > 1) {  // the union's R smallest (key, row), as row ids in the first R entries of the union
        GfUnion u{h->selk, h->seli, h->segs, r, nseg * r};
        gf_union_select_kernel<<<1, kGfUnionThreads, 0, st>>>(u, h->uni);
        ANN_LAUNCH_CHECK();
    }
    const int* cand = nseg > 1 ? h->uni : h->seli;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(gf_rerank_kernel)));
    gf_rerank_kernel<<<(unsigned)ceil_div(r, kGfRerankWarps), 32 * kGfRerankWarps,
                       sizeof(float) * dim * (1 + kGfRerankWarps), st>>>(h->base, n, dim, h->q, cand, r, h->keys);
    ANN_LAUNCH_CHECK();
    if ((rc = launch_gf_topk<long long>(h->keys, r, k, h->out, st))) return rc;
    ANN_CUDA_TRY(cudaMemcpyAsync(h->hout, h->out, sizeof(long long) * k, cudaMemcpyDeviceToHost, st));
    return ANN_OK;
}

// The first query of a (k, r) runs its launches one by one and then records them into a graph (no work
// runs while recording); later queries of that (k, r) replay the graph: one launch instead of about ten
// calls. The graphs read the query from, and write the ids to, the handle's pinned staging buffers.
int gf_search(gf_handle* h, const float* q, int k, int r, long long* out_ids) {
    cudaStream_t st = h->st;
    // one segment when R exceeds the top-k kernel's bound (the second stage keeps R keys in front of each
    // sorted round)
    const int nseg = r <= kGfMaxK ? h->nseg : 1;
    int rc = gf_reserve(h, (int64_t)nseg * r);
    if (rc) return rc;
    std::memcpy(h->hq, q, sizeof(float) * h->dim);
    gf_handle::Graph* gr = nullptr;
    for (auto& x : h->graphs)
        if (x.k == k && x.r == r) gr = &x;
    if (gr && gr->exec) {
        ANN_CUDA_TRY(cudaGraphLaunch(gr->exec, st));
    } else if ((rc = gf_enqueue(h, k, r, nseg))) {
        return rc;
    }
    ANN_CUDA_TRY(cudaStreamSynchronize(st));
    std::memcpy(out_ids, h->hout, sizeof(long long) * k);
    if (!gr && h->graphs.size() < 16) {  // record this (k, r) once
        gf_handle::Graph x{k, r, nullptr};
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const int erc = gf_enqueue(h, k, r, nseg);
            const cudaError_t e = cudaStreamEndCapture(st, &graph);
            if (erc == ANN_OK && e == cudaSuccess && graph &&
                cudaGraphInstantiate(&x.exec, graph, 0) != cudaSuccess)
                x.exec = nullptr;
            if (graph) cudaGraphDestroy(graph);
        }
        cudaGetLastError();  // a failed recording leaves the launches one by one for this (k, r)
        clear_error();
        h->graphs.push_back(x);
    }
    return ANN_OK;
}

}  // namespace

extern "C" {

const char* gf_last_error(void) { return ann_last_error(); }

void* gf_create(const float* train, long n, long dim) {
    clear_error();
    if (dim > kGfMaxDim) {
        set_error("dim %ld > 4096 unsupported", dim);
        return nullptr;
    }
    if (!train || n <= 0 || n >= INT32_MAX || dim <= 0) {
        set_error("gf_create: train=%p n=%ld dim=%ld", (const void*)train, n, dim);
        return nullptr;
    }
    int ndev = 0;
    const cudaError_t derr = cudaGetDeviceCount(&ndev);
    if (derr != cudaSuccess || ndev == 0) {
        set_error("no CUDA device visible (%s)", derr == cudaSuccess ? "0 devices" : cudaGetErrorString(derr));
        return nullptr;
    }
    gf_handle* h = new (std::nothrow) gf_handle();
    if (!h) {
        set_error("gf_create: out of host memory");
        return nullptr;
    }
    if (cudaGetDevice(&h->device) != cudaSuccess) h->device = 0;
    h->n = n;
    h->dim = (int)dim;
    h->npad = ceil_div((int64_t)n, 16) * 16;
    if (gf_build(h, train) != ANN_OK) {
        gf_release(h);
        delete h;
        return nullptr;
    }
    return h;
}

int gf_query(void* handle, const float* q, int k, int r, long long* out_ids) {
    clear_error();
    gf_handle* h = static_cast<gf_handle*>(handle);
    if (!h || !q || (k > 0 && !out_ids) || k < 0) {
        set_error("gf_query: handle=%p q=%p k=%d out_ids=%p", handle, (const void*)q, k, (void*)out_ids);
        return -1;
    }
    if (k > kGfMaxK) {
        set_error("gf_query: k=%d > %d unsupported", k, kGfMaxK);
        return -1;
    }
    if (r < k) r = k;
    if (r > h->n) r = (int)h->n;
    const int out_k = std::min(k, r);
    if (out_k <= 0) {  // nothing to return; the reference still counts its r distances
        h->ndist += r;
        return out_k;
    }
    std::lock_guard<std::mutex> lk(h->mu);
    DeviceGuard g(h->device);
    if (!g.ok) {
        set_error("gf_query: cannot select device %d", h->device);
        return -1;
    }
    if (gf_search(h, q, out_k, r, out_ids) != ANN_OK) return -1;
    h->ndist += r;
    return out_k;
}

long long gf_ndist(void* handle) { return handle ? static_cast<gf_handle*>(handle)->ndist.load() : 0; }

void gf_free(void* handle) {
    gf_handle* h = static_cast<gf_handle*>(handle);
    if (!h) return;
    gf_release(h);
    delete h;
}

}  // extern "C"

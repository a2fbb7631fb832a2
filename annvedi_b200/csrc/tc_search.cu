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

__global__ void tc_bar_check_kernel(const int* rowcnt, int M, int R, int* list, int* flags) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < M && rowcnt[q] < R) list[atomicAdd(&flags[0], 1)] = q;
}

__global__ void tc_gather_kernel(const __nv_bfloat16* A, int kpad, const int* list, int nb, const float* tau,
                                 __nv_bfloat16* A2, float* tau2) {
    const int j = blockIdx.x;
    if (j >= nb) return;
    const int q = list[j];
    const uint4* src = reinterpret_cast<const uint4*>(A + (size_t)q * kpad);
    uint4* dst = reinterpret_cast<uint4*>(A2 + (size_t)j * kpad);
    for (int c = threadIdx.x; c < kpad / 8; c += blockDim.x) dst[c] = src[c];
    if (threadIdx.x == 0) tau2[j] = tau[q];
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

}  // namespace

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

int launch_tc_bar_check(const int* rowcnt, int M, int R, int* list, int* flags, cudaStream_t st) {
    if (M == 0) return ANN_OK;
    tc_bar_check_kernel<<<(unsigned)ceil_div(M, 256), 256, 0, st>>>(rowcnt, M, R, list, flags);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_gather(const __nv_bfloat16* A, int kpad, const int* list, int nb, const float* tau, __nv_bfloat16* A2,
                     float* tau2, cudaStream_t st) {
    if (nb == 0) return ANN_OK;
    ANN_CHECK_ARG(kpad % 8 == 0, "gather: kpad %d", kpad);
    tc_gather_kernel<<<nb, 128, 0, st>>>(A, kpad, list, nb, tau, A2, tau2);
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

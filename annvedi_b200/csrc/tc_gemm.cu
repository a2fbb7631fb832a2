// BF16 distance GEMM on the 5th-generation tensor cores (tcgen05 + TMA + TMEM) for sm_100a.
//
// keys[m][n] = f(sum_k A[m][k] * B[n][k]) with A = queries [M, K] and B = base rows [N, K], both BF16
// row-major (K-major for the MMA), FP32 accumulation; f gives the ranking key: for squared L2,
// |b_n|^2 - 2 a.b (+ |a_m|^2) from FP32 norms; for inner product, -a.b (smaller is better).
//
// Structure (one CTA per SM, persistent over 128 x 256 output tiles, query tiles fastest so a base
// tile is fetched from HBM once and reused from L2 by the query tiles that follow it):
//   warp 0    TMA producer: 128x64 A and 256x64 B boxes (128-byte swizzle) into a 4-stage ring,
//             mbarrier expect-tx completion; no multicast;
//   warp 1    allocates 512 TMEM columns (two 128 x 256 FP32 accumulators) and, from one thread,
//             issues tcgen05.mma (kind::f16, BF16 in, FP32 out, M = 128, N = 256, K = 16 per
//             instruction, 4 per stage); tcgen05.commit frees each stage and publishes each tile;
//   warps 2-5 epilogue: tcgen05.ld 32 columns at a time from the warp's 32 TMEM lanes, apply f,
//             store the keys, release the accumulator.
// Every mbarrier wait is bounded (about 2 s); a timeout raises a device flag and the CTA winds down.
#include <cuda.h>

#include "common.cuh"
#include "tc_gemm.cuh"

namespace annb {

namespace {

constexpr int kBM = 128, kBN = 256, kBK = 64, kStages = 4;
constexpr int kABytes = kBM * kBK * 2;  // 16 KB
constexpr int kBBytes = kBN * kBK * 2;  // 32 KB
constexpr int kTmemCols = 512;

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t n) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(su32(b)), "r"(parity)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity, int* err) {
    if (bar_try(b, parity)) return true;
    const uint64_t t0 = gtimer();
    while (!bar_try(b, parity))
        if (gtimer() - t0 > 2000000000ull) {
            if (err) atomicExch(err, 2);
            return false;
        }
    return true;
}
__device__ __forceinline__ void bar_arrive(uint64_t* b) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ void bar_expect(uint64_t* b, uint32_t bytes) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(su32(b)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, int c0, int c1, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            su32(dst)),
        "l"(tm), "r"(c0), "r"(c1), "r"(su32(bar))
        : "memory");
}
// Shared-memory matrix descriptor for a K-major tile in the 128-byte swizzle layout (rows of 128 B,
// 8-row groups 1024 B apart): start address >> 4, leading offset 1 (unused with swizzle), stride
// offset 1024 >> 4, descriptor version 1, layout type 2 (128-byte swizzle).
__device__ __forceinline__ uint64_t sw128_desc(const void* p) {
    const uint64_t addr = (su32(p) >> 4) & 0x3FFFull;
    return addr | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}
// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N = 256, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
        "l"(ad), "l"(bd), "r"(kIdesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
        "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(192, 1) tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA,
                                                         const __grid_constant__ CUtensorMap tmB, TcGemmArgs a) {
    extern __shared__ unsigned char smem_raw[];
    // 1024-byte alignment for the swizzled tiles
    unsigned char* smem = smem_raw + ((1024 - (su32(smem_raw) & 1023)) & 1023);
    unsigned char* sA = smem;
    unsigned char* sB = smem + kStages * kABytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + kStages * kBBytes);
    uint64_t* empty = full + kStages;
    uint64_t* tfull = empty + kStages;
    uint64_t* tempty = tfull + 2;
    uint64_t* done = tempty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = (int)ceil_div(a.M, kBM), nt = (int)ceil_div(a.N, kBN), kt = a.K / kBK;
    const int64_t tiles = (int64_t)mt * nt;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            bar_init(&full[s], 1);
            bar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            bar_init(&tfull[b], 1);
            bar_init(&tempty[b], 128);
        }
        bar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {  // TMA producer
            int64_t it = 0;
            bool ok = true;
            for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                const int m0 = (int)(t % mt) * kBM, n0 = (int)(t / mt) * kBN;
                for (int kb = 0; kb < kt; ++kb, ++it) {
                    const int s = (int)(it % kStages);
                    const uint32_t ph = (uint32_t)((it / kStages) & 1);
                    if (!(ok = bar_wait(&empty[s], ph ^ 1u, a.err))) break;
                    bar_expect(&full[s], kABytes + kBBytes);
                    tma_load_2d(sA + s * kABytes, &tmA, kb * kBK, m0, &full[s]);
                    tma_load_2d(sB + s * kBBytes, &tmB, kb * kBK, n0, &full[s]);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            int64_t it = 0, acc = 0;
            bool ok = true;
            for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++acc) {
                const int b = (int)(acc & 1);
                const uint32_t aph = (uint32_t)((acc >> 1) & 1);
                if (!(ok = bar_wait(&tempty[b], aph ^ 1u, a.err))) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(b * kBN);
                for (int kb = 0; kb < kt; ++kb, ++it) {
                    const int s = (int)(it % kStages);
                    const uint32_t ph = (uint32_t)((it / kStages) & 1);
                    if (!(ok = bar_wait(&full[s], ph, a.err))) break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                    for (int k16 = 0; k16 < kBK / 16; ++k16)
                        mma_bf16(d, sw128_desc(sA + s * kABytes + k16 * 32), sw128_desc(sB + s * kBBytes + k16 * 32),
                                 (kb | k16) ? 1u : 0u);
                    mma_commit(&empty[s]);
                }
                mma_commit(&tfull[b]);
            }
            // every MMA issued has completed before TMEM is released
            mma_commit(done);
            bar_wait(done, 0, nullptr);
        }
    } else {  // epilogue warps 2..5: TMEM lanes 32 * (warp % 4) ...
        const int lane_base = 32 * (warp & 3);
        int64_t acc = 0;
        for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x, ++acc) {
            const int b = (int)(acc & 1);
            if (!bar_wait(&tfull[b], (uint32_t)((acc >> 1) & 1), a.err)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int m0 = (int)(t % mt) * kBM, n0 = (int)(t / mt) * kBN;
            const int m = m0 + lane_base + lane;
            const float an = (a.normA && m < a.M) ? a.normA[m] : 0.f;
            for (int c = 0; c < kBN / 32; ++c) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)lane_base << 16) + (uint32_t)(b * kBN + c * 32), v);
                const int nb = n0 + c * 32;
                if (m < a.M) {
                    float* orow = a.out + (int64_t)m * a.ldo;
#pragma unroll
                    for (int j = 0; j < 32; j += 4) {
                        float4 o;
                        float* op = &o.x;
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int n = nb + j + u;
                            const float dot = v[j + u];
                            float key;
                            if (a.metric == ANN_METRIC_L2)
                                key = (n < a.N ? a.normB[n] : 0.f) - 2.f * dot + an;
                            else
                                key = -dot;
                            op[u] = n < a.N ? key : kInf;
                        }
                        if (nb + j + 3 < a.N)
                            *reinterpret_cast<float4*>(orow + nb + j) = o;
                        else
                            for (int u = 0; u < 4; ++u)
                                if (nb + j + u < a.N) orow[nb + j + u] = op[u];
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            bar_arrive(&tempty[b]);
        }
    }
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

int make_map(CUtensorMap* tm, const void* base, int64_t rows, int cols, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("cuTensorMapEncodeTiled is not available from the driver");
        return ANN_ERR_CUDA;
    }
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d) for a [%lld, %d] bf16 matrix", (int)r, (long long)rows, cols);
        return ANN_ERR_CUDA;
    }
    return ANN_OK;
}

}  // namespace

size_t tc_gemm_smem() { return (size_t)kStages * (kABytes + kBBytes) + 1024 + 256; }

int launch_tc_gemm(const __nv_bfloat16* A, const __nv_bfloat16* B, const TcGemmArgs& a, cudaStream_t st) {
    ANN_CHECK_ARG(a.K % kBK == 0 && a.K > 0, "tensor-core scan: K=%d not a positive multiple of %d", a.K, kBK);
    ANN_CHECK_ARG((reinterpret_cast<uintptr_t>(A) & 15) == 0 && (reinterpret_cast<uintptr_t>(B) & 15) == 0,
                  "tensor-core scan: operands must be 16-byte aligned");
    ANN_CHECK_ARG(a.metric == ANN_METRIC_IP || a.normB != nullptr, "tensor-core scan: L2 keys need base norms");
    if (a.M == 0 || a.N == 0) return ANN_OK;
    CUtensorMap tmA, tmB;
    int rc = make_map(&tmA, A, a.M, a.K, kBM);
    if (rc) return rc;
    rc = make_map(&tmB, B, a.N, a.K, kBN);
    if (rc) return rc;
    const size_t smem = tc_gemm_smem();
    ANN_CUDA_TRY(cudaFuncSetAttribute(tc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t tiles = ceil_div(a.M, kBM) * ceil_div(a.N, kBN);
    const int grid = (int)std::min<int64_t>(tiles, kNumSMs);
    tc_gemm_kernel<<<grid, 192, smem, st>>>(tmA, tmB, a);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// FP32 [rows, ld] (first `cols` columns) -> BF16 [rows, kpad] zero-padded, plus optional FP32 row norms
// of the converted values' sources (exact squared norms of the FP32 rows).
__global__ void to_bf16_kernel(const float* __restrict__ x, int64_t rows, int cols, int64_t ld, __nv_bfloat16* out,
                               int kpad, float* norms) {
    const int64_t r = blockIdx.x * (int64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    float s = 0.f;
    for (int c = lane; c < kpad; c += 32) {
        const float v = c < cols ? x[r * ld + c] : 0.f;
        out[r * kpad + c] = __float2bfloat16_rn(v);
        s = fmaf(v, v, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (norms && lane == 0) norms[r] = s;
}

int launch_to_bf16(const float* x, int64_t rows, int cols, int64_t ld, __nv_bfloat16* out, int kpad, float* norms,
                   cudaStream_t st) {
    if (rows == 0) return ANN_OK;
    to_bf16_kernel<<<(unsigned)ceil_div(rows, 8), 256, 0, st>>>(x, rows, cols, ld, out, kpad, norms);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

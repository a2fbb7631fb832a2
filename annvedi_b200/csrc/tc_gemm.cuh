// Launch interface of the tcgen05 BF16 distance GEMM (tc_gemm.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace annb {

struct TcGemmArgs {
    int M, N, K;           // A [M, K], B [N, K] BF16 row-major; K a multiple of 64
    const float* normA;    // [M] squared norms of A rows (L2; optional)
    const float* normB;    // [N] squared norms of B rows (L2)
    int metric;            // ANN_METRIC_L2: |b|^2 - 2 a.b (+ |a|^2); ANN_METRIC_IP: -a.b
    float* out;            // [M, ldo] keys (smaller is better)
    int64_t ldo;
    int* err;              // device flag set if a bounded wait gives up
};

size_t tc_gemm_smem();
int launch_tc_gemm(const __nv_bfloat16* A, const __nv_bfloat16* B, const TcGemmArgs& a, cudaStream_t st);
int launch_to_bf16(const float* x, int64_t rows, int cols, int64_t ld, __nv_bfloat16* out, int kpad, float* norms,
                   cudaStream_t st);

}  // namespace annb

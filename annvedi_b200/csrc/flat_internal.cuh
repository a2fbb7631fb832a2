// The flat index handle, shared by the C ABI translation units.
#pragma once
#include <atomic>

#include <cuda_bf16.h>

#include "common.cuh"
#include "runtime.cuh"

struct ann_flat {
    int device = 0;
    int64_t n = 0;
    int dim = 0;
    int dpad = 0;
    int metric = ANN_METRIC_L2;
    float* base = nullptr;  // [n, dpad]
    std::atomic<int64_t> ndist{0};
    ann_workspace ws;       // default workspace
    annb::StageProfiler prof;     // stage 0: scan kernel(s); stage 1: merge / selection
    __nv_bfloat16* base_bf16 = nullptr;  // [n, kpad] BF16 operand form for the tensor-core scan (built on first use)
    int64_t row_mult = 1;                // position p of base_bf16 holds row (p * row_mult) mod n
    int kpad = 0;                        // operand columns: dim plus the key columns, rounded up to 64
    int query_tile = 0;                  // the exact scan's queries per CTA (0: chosen by the batch size)
    int* d_err = nullptr;                // device flag of bounded waits
    int tc_kind = 0;                     // element kind of the tensor-core search (0 BF16, 1 E4M3)
    uint8_t* base_e4m3 = nullptr;        // [n, kpad8] E4M3 operand form, Weyl order, built on first use
    float2* fac_e4m3 = nullptr;          // [n] its per-row key factors
    int kpad8 = 0;                       // dim rounded up to 32
};

namespace annb {
// Number of row splits (and rows per split) for an exact scan of n rows by nq queries in tiles of bq.
// ctas_per_sm: resident CTAs per SM of the scan form used (one wave = kNumSMs * ctas_per_sm CTAs).
int flat_choose_nsplit(int64_t n, int nq, int bq, int64_t* rows_per_split, int ctas_per_sm = 1);
}  // namespace annb

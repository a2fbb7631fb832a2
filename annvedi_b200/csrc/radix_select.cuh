// Launch interface of the per-query radix selection (radix_select.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ivf.cuh"

namespace annb {

struct RadixSelectArgs {
    const float* keys;      // query q's stream: keys[offs[q] + p] (or keys[q * ld + p]), p < len
    int64_t ld;             // row stride when offs is null; also the upper bound of len
    const int64_t* offs;    // optional
    const int64_t* lens;    // optional int64 lengths
    const int* lens32;      // optional int32 lengths (clamped to ld)
    const int* ids;         // optional explicit ids (ids[offs[q] + p]); else plan rows; else p
    IvfPlan plan;           // ids from the candidate-stream plan when use_plan is set
    int use_plan;
    int R;
    float* out_key;         // [nq, R] the set (unsorted), padded with +inf / kNoId
    int* out_id;            // [nq, R]
    float* out_kth;         // [nq] the R-th smallest key (+inf if fewer), optional
    const int* out_rows = nullptr;  // optional: query q writes output row out_rows[q]
    int R2 = 0;                     // optional second rank, reported only as its key
    float* out_kth2 = nullptr;      // [nq] the R2-th smallest key (+inf if fewer)
    int kth_upper = 0;              // bars only: report the upper edge of the key's 22-bit bin (two passes)
};

int launch_radix_select(const RadixSelectArgs& a, int nq, cudaStream_t st);

// Bars from rows of S sampled keys (keys[q * S + i], S a multiple of 4, the row resident in shared
// memory): bar1[q] / bar2[q] at or above the r1-th / r2-th smallest key of row q, within 2^-22 of the
// row's key range above it.
constexpr size_t kSampleBarsMaxSmem = 160 * 1024;
size_t sample_bars_smem(int S);
int launch_sample_bars(const float* keys, int S, int nq, int r1, int r2, float* bar1, float* bar2, cudaStream_t st);

}  // namespace annb

// Launch interface of the batched, list-major SQ8 pass (ivf_batched.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ivf.cuh"

namespace annb {

constexpr int64_t kItemRows = 2048;  // list rows per work item

struct IvfBatchArgs {
    IvfView ix;
    IvfPlan plan;
    const int32_t* pair_vals;   // (q * npc + j) of each probe, grouped by list
    const int32_t* pair_lists;  // the list of each pair (C past the valid pairs)
    const int64_t* lq_off;      // [C + 1] first pair of each list
    const int64_t* item_off;    // [C + 1] first work item of each list
    const int64_t* total_items; // device scalar (item_off[C])
    const int64_t* cand_off;    // [nq + 1] first candidate-stream slot of each query in D
    unsigned* counter;          // work-item counter (zeroed by batched_prepare)
    const float* qs;            // [nq, dpad] q - offset
    float* D;                   // [sum of n_cands] SQ8 distances in stream order
};

// Scratch of batched_prepare for nq queries x npc probes over C lists (CUB temp sizes returned).
size_t batched_scratch_bytes(int nq, int npc, int C, size_t* sort_tmp, size_t* scan_tmp);
// Groups the plan's probes by list, counts work items and candidate offsets; host_totals[0..2] =
// {work items, total candidates, fallback flag}. Synchronises the stream.
// With sync = false the totals are copied to host_totals (which must then be page-locked) without waiting: they
// are valid after the caller's next synchronisation of st.
int batched_prepare(const IvfQueryArgs& a, void* scratch, size_t sort_tmp, size_t scan_tmp, IvfBatchArgs* out,
                    int64_t* host_totals, cudaStream_t st, bool sync = true);
int launch_batched(const IvfBatchArgs& b, const float* qdev, float* qs, float* D, cudaStream_t st);

}  // namespace annb

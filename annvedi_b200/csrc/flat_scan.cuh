// Launch interfaces of the exact FP32 scan (flat_scan.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace annb {

struct FlatScanArgs {
    const float* base;       // [n, dpad] FP32, zero-padded rows
    int64_t n;
    int dpad;                // multiple of 32
    const float* q;          // [nq, dpad] FP32, zero-padded
    int nq;
    int metric;              // ANN_METRIC_L2 / ANN_METRIC_IP
    int k;                   // 1..512
    int64_t rows_per_split;
    int nsplit;
    float* out_key;          // [nq, nsplit, k] scratch
    int* out_id;             // [nq, nsplit, k] scratch
    int cap;                 // per-query buffer capacity (set by launch_flat_scan)
    // optional scratch of 2 ceil(nq / 2) dpad floats: with 32-query tiles of squared L2, launch_flat_scan writes
    // the queries there as interleaved negated pairs and the scan takes two queries a packed FP32
    // instruction, each half rounding as the scalar form (the same distances)
    float* qpair = nullptr;
};

struct MergeArgs {
    const float* in_key;     // [nq, nsplit, kin] sorted per split, (+inf, INT_MAX) padded
    const int* in_id;
    int nq;
    int nsplit;
    int kin;
    int k;
    int negate;              // 1: output -key (inner-product scores)
    int64_t* out_ids;        // [nq, k], -1 where fewer than k exist
    float* out_dists;        // [nq, k] or nullptr
    int* out_id32 = nullptr;   // [nq, k] raw ids (INT_MAX where fewer than k exist), optional
    float* out_key32 = nullptr; // [nq, k] raw keys (+inf where fewer), optional
};

// Pipeline depth of the query tiles of 1..8 queries (HBM-bound: four 36 KB stages keep enough bytes
// in flight with one CTA per SM).
constexpr int kSmallTileStages = 4;

int flat_scan_bq(int nq);
// Tiles of 1, 2 or 4 queries run the register-streaming form (several CTAs per SM, as the occupancy
// calculator allows); the others the shared-memory pipeline (one CTA per SM).
bool flat_stream_eligible(int bq, int k, int dpad);
int flat_scan_ctas_per_sm(int bq, int k, int dpad, int metric);
int flat_scan_max_bq(int k);
int launch_flat_scan(const FlatScanArgs& a, int bq, cudaStream_t st);
int launch_merge_splits(const MergeArgs& a, cudaStream_t st);
// Sorts per-query sets of k pairs by (key, id) into the final top-k (see flat_scan.cu).
int launch_sort_topk(const float* keys, const int* ids, int nq, int k, int negate, int64_t* out_ids, float* out_dists,
                     cudaStream_t st);
int launch_pad_rows(const float* src, int64_t n, int dim, int64_t ld, float* dst, int dpad, cudaStream_t st);

// Best k of `parts` per-shard top-k lists per query: d / ids [nq, parts, k], each part sorted by (key, id)
// (key = distance, or -score when ip), ids < 0 empty, parts in increasing id ranges. out [nq, k].
int launch_merge_parts(const float* d, const int64_t* ids, int nq, int parts, int k, int ip, int64_t* out_ids,
                       float* out_d, cudaStream_t st);

}  // namespace annb

// Launch interfaces of the IVF-SQ8 kernels (ivf.cu, ivf_build.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace annb {

// Device view of an IVF-SQ8 index (n_tables = 1, n_bits = 0 inverted lists).
struct IvfView {
    int64_t n;
    int dim;
    int dpad;                  // FP32 row stride (floats), multiple of 32
    int dpad8;                 // SQ8 row stride (bytes), multiple of 16
    int C;                     // lists
    const float* centroids;    // [C, dpad]
    const float* original;     // [n, dpad] rows in list order
    const uint8_t* codes;      // [n, dpad8] rows in list order
    const float* scale;        // [dpad], zero past dim
    const float* offset;       // [dpad], zero past dim
    const int32_t* r2o;        // [n] list-order row -> original id
    const int64_t* list_off;   // [C + 1]
};

// Per-query candidate streams: the probed lists, in probe order, concatenated. Position p of
// query q maps to a list-order row through the segments (or p itself when the query fell back to
// scanning every row because its lists held fewer than k points).
struct IvfPlan {
    int nq;
    int npc;                   // probes per query (columns of probes / seg arrays)
    const int32_t* probes;     // [nq, npc] list ids, best first
    int64_t* seg_start;        // [nq, npc]
    int64_t* seg_pref;         // [nq, npc + 1]
    int32_t* n_seg;            // [nq] lists used; -1 = all rows
    int64_t* n_cands;          // [nq]
    const int32_t* cand_ids = nullptr;  // [nq, cand_ld] explicit streams (LSH buckets) instead of whole lists
    int64_t cand_ld = 0;
};

// Position p of query q's candidate stream -> list-order row.
__device__ __forceinline__ int64_t plan_row(const IvfPlan& p, int q, int64_t pos) {
    const int ns = p.n_seg[q];
    if (ns < 0) return pos;
    if (p.cand_ids) return p.cand_ids[(int64_t)q * p.cand_ld + pos];
    const int64_t* pref = p.seg_pref + (int64_t)q * (p.npc + 1);
    int lo = 0, hi = ns - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pref[mid] <= pos)
            lo = mid;
        else
            hi = mid - 1;
    }
    return p.seg_start[(int64_t)q * p.npc + lo] + (pos - pref[lo]);
}

struct IvfQueryArgs {
    IvfView ix;
    IvfPlan plan;
    const float* q;            // [nq, ldq]
    int64_t ldq;
    int k;
    int R;                     // candidates kept for the FP32 re-rank
    int64_t max_cands;         // cap on the candidate stream (INT64_MAX = none)
    int no_fallback;           // a shard of the lists: a stream short of k stays as it is (no every-row scan)
    int nsplit;                // CTAs per query in the exact SQ8 scan
    int num_threads;           // reference mode: the reference ThreadPool size
    int ncp;                   // reference mode: SQ8 checkpoints
    int64_t L;                 // reference mode: stride of the per-query position arrays
    float* keyR;               // [nq, nsplit, R] or [nq, R]
    int* idR;
    float* D;                  // reference mode [nq, L]
    float* P;                  // reference mode [nq, ncp, L]
    float* V;                  // reference mode [nq, L]
    unsigned long long* ndist; // device counter of candidates scanned (get_n_distances)
    int* err;                  // device flag: a bounded wait gave up
    int metric;                // re-rank metric: ANN_METRIC_L2 (default) or ANN_METRIC_IP
    int64_t* out_ids;          // [nq, k]
    float* out_dists;          // [nq, k]
    const int32_t* qorder;     // re-rank: CTA b takes query qorder[b] (NULL: query b)
};

int launch_ivf_plan(const IvfQueryArgs& a, cudaStream_t st);
int launch_ivf_sq8_scan(const IvfQueryArgs& a, cudaStream_t st);
// SQ8 keys of whole candidate streams, D[q * ld + p] (the scan's arithmetic, no selection).
int launch_ivf_sq8_dists(const IvfQueryArgs& a, float* D, int64_t ld, cudaStream_t st);
int launch_ivf_ref_sq8(const IvfQueryArgs& a, int64_t Lmax, cudaStream_t st);
int launch_select_topk(const float* keys, int64_t ld_keys, const int64_t* lens, int nq, int kout,
                       const IvfPlan* plan, float* out_key, int* out_id, cudaStream_t st,
                       const int64_t* offs = nullptr, bool set_only = false);
int launch_ivf_rerank(const IvfQueryArgs& a, const float* keyR, const int* idR, int reference, cudaStream_t st);
int launch_ref_centroid_dists(const IvfView& ix, const float* q, int64_t ldq, int nq, float* Dc, cudaStream_t st);

// Build helpers (ivf_build.cu).
int launch_sq8_minmax(const float* x, int64_t n, int dim, int ld, float* mn, float* mx, cudaStream_t st);
int launch_sq8_params(const float* mn, const float* mx, int dim, int dpad, float* scale, float* offset,
                      cudaStream_t st);
int launch_sq8_encode(const float* x, int64_t n, int dim, int ld, const float* scale, const float* offset,
                      uint8_t* codes, int dpad8, cudaStream_t st);
int launch_gather_rows(const float* src, int64_t n, int ld_src, const int32_t* rows, float* dst, int ld_dst,
                       cudaStream_t st);
int launch_list_offsets(const int32_t* sorted_assign, int64_t n, int C, int64_t* off, cudaStream_t st);
int launch_iota(int32_t* v, int64_t n, cudaStream_t st);                 // v[i] = i
// Every query whose stream is every row (n_seg < 0) becomes an empty stream: n_seg = n_cands = 0.
int launch_clear_every_row(const IvfPlan& plan, cudaStream_t st);
// order[0..nq) = the queries grouped by their first probed list (probes[q * npc], in [0, C)), so that
// neighbouring re-rank CTAs gather rows of the same lists; one CTA, C <= kQueryOrderMaxLists.
constexpr int kQueryOrderMaxLists = 32768;
int launch_query_order(const int32_t* probes, int npc, int nq, int C, int32_t* order, cudaStream_t st);
int launch_add_offset(int64_t* v, int64_t n, int64_t add, cudaStream_t st);  // v[i] += add
// k-means of the reference (ivf_build.cu): certification of the fast two nearest centroids, the
// reference arithmetic for the queued near-ties, and the ThreadPool-chunk-ordered update.
int launch_kmeans_certify(const float* key2, const int* id2, int64_t n, float margin, int32_t* assign, int32_t* amb,
                          int* amb_count, cudaStream_t st);
int launch_kmeans_ref_assign(const float* x, int ldx, int dim, const float* cent, int ldc, int C, const int32_t* amb,
                             const int* amb_count, int32_t* assign, cudaStream_t st);
int launch_kmeans_update(const float* x, int ldx, int dim, const int32_t* order, const int64_t* off, int C,
                         float* centroids, int ldc, const int32_t* reseed_rows, int64_t n, int num_threads,
                         cudaStream_t st);

}  // namespace annb

// Helpers of the tensor-core search around the GEMM (tc_search.cu): grouping filter survivors into
// per-query streams, the bar check and re-run gather, and the row order of the BF16 base copy.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ivf.cuh"

namespace annb {

// The BF16 base copy stores row (p * mult) mod n at position p (a Weyl sequence with mult ~ 0.618 n,
// coprime to n): any 256 consecutive positions cover the rows evenly, so a strided sample of whole
// tiles is an even sample of the base whatever order the rows came in.
int64_t tc_row_mult(int64_t n);

struct TcGroupArgs {
    // filter survivors: warp w holds entries [w * wcap, w * wcap + min(wcount[w], wcap))
    const float* fkey;
    const int* fcol;
    const int* frow;
    const int* wcount;
    int nwarps;
    int wcap;
    int M;            // rows (queries) of the filter launch
    int64_t n;        // base rows, for the position -> row map
    int64_t mult;     // tc_row_mult(n)
    // outputs
    int* rowcnt;      // [M] survivors per row
    int64_t* offs;    // [M] start of row m's stream in gkey / gid
    int* cursor;      // [M] scratch
    float* gkey;      // [nwarps * wcap]
    int* gid;         // [nwarps * wcap] base row ids
    int* max_wcount;  // [1] largest wcount (an overflow if > wcap)
};
int launch_tc_group(const TcGroupArgs& g, cudaStream_t st);

// Rows with fewer than R survivors -- fewer than min(R, lens[row]) where lens is given -- go to list (count in
// flags[0]); mark[row], if given, is 1 for them and 0 for the others.
int launch_tc_bar_check(const int* rowcnt, int M, int R, int* list, int* flags, cudaStream_t st,
                        const int64_t* lens = nullptr, int* mark = nullptr);
// A2[j] = A[list[j]] (rows of row_bytes), tau2[j] = tau[list[j]] and, if given, rfac2[j] = rfac[list[j]].
int launch_tc_gather(const void* A, int row_bytes, const int* list, int nb, const float* tau, void* A2, float* tau2,
                     const float* rfac, float* rfac2, cudaStream_t st);
// ids[i] (positions of the BF16 copy) -> base rows, in place; kNoId stays.
int launch_tc_map_ids(int* ids, int64_t count, int64_t n, int64_t mult, cudaStream_t st);
// out[q][row(p)] = keys[q][p] for a [nq, n] key matrix in position order.
int launch_tc_unpermute(const float* keys, int nq, int64_t n, int64_t mult, float* out, cudaStream_t st);

// IVF batches on the tensor cores (a list-major grouping of (query, list) pairs, ivf_batched.cu):
// items per list = ceil(pairs / 128) x ceil(rows / 256), exclusively scanned into item_off[0..C]
// (item_off[C] = all items). One block.
// With list_len, list l counts list_len[l] rows (a capped head of each list) instead of its size.
int launch_tc_ivf_items(const int64_t* lq_off, const int64_t* list_off, int C, int64_t* item_off, cudaStream_t st,
                        const int64_t* list_len = nullptr);
// item_list[t] = the list of work item t (item_off [C + 1] from launch_tc_ivf_items), for t < cap.
int launch_tc_item_lists(const int64_t* item_off, int C, int32_t* item_list, int64_t cap, cudaStream_t st);
// Work items of a grouped batch at most: (pairs / 128 + C) x (largest list / 256 + 1).
inline int64_t tc_items_bound(int64_t pairs, int C, int64_t largest) { return (pairs / 128 + C) * (largest / 256 + 1); }
// For each valid pair i (< lq_off[C]; pairs grouped by list, pair_vals = q * npc + j, pair_lists = the
// list): A[i] = qb[q] (kpad BF16 columns) and dbase[i] = cand_off[q] + seg_pref[q][j] - list_off[list],
// the stream position of the list's row 0 in the candidate array.
// Optional maps of the sampled form: row_query[i] = q; sdbase[i] = soff[q] + sseg[q][j] - list_off[list]
// (the sample-stream position of the list's row 0, as dbase is for the candidate stream).
// With qfac / pfac (the int8 form), pfac[i] = qfac[q].
struct TcIvfSampleMaps {
    int32_t* row_query = nullptr;
    const int64_t* soff = nullptr;
    const int64_t* sseg = nullptr;  // [nq, npc]
    int64_t* sdbase = nullptr;
    const float* qfac = nullptr;
    float* pfac = nullptr;
};
// qrows: the queries' operand rows of row_bytes each (BF16 kpad columns, or int8 weights); A: the pairs' rows.
int launch_tc_ivf_pairs(const void* qrows, int row_bytes, const int32_t* pair_vals, const int32_t* pair_lists,
                        const int64_t* n_pairs, int64_t max_pairs, int npc, const int64_t* cand_off,
                        const int64_t* seg_pref, const int64_t* list_off, void* A, int64_t* dbase, cudaStream_t st,
                        const TcIvfSampleMaps& sm = TcIvfSampleMaps{});
// SQ8 codes on the tensor cores (kind::i8): the int8 query weights rint(-2 scale_d (q_d - offset_d) * 127 / max)
// [nq, ldo] (zero past dim) with their factor qfac = max / 127, and per row fac = (1, sum_d (code_d scale_d)^2);
// the key fac.y + qfac * sum_d code_d a_d is the SQ8 distance less |q - offset|^2, up to the weights' rounding.
int launch_tc_sq8_query(const float* q, int nq, int dim, int ldq, const float* scale, const float* offset, int8_t* out,
                        int ldo, float* qfac, cudaStream_t st);
int launch_tc_sq8_norms(const uint8_t* codes, int64_t n, int dim, int ldc, const float* scale, float2* fac,
                        cudaStream_t st);
// The sampled heads of the lists, lcap[l] = ceil(size_l / div), and each query's sample stream over its
// probed lists: segment starts sseg [nq, npc] and length slen [nq].
int launch_tc_ivf_sample_plan(const IvfPlan& p, const int64_t* list_off, int C, int div, int64_t* lcap, int64_t* sseg,
                              int64_t* slen, cudaStream_t st);
// tauR[q] = mark[q] ? tauS[q] : -inf; with rcount, the marked queries' counts are reset to 0.
int launch_tc_rerun_bars(const int* mark, const float* tauS, int nq, float* tauR, cudaStream_t st,
                         int* rcount = nullptr);
// *out = max(0, v[0..n)) (out zeroed first).
int launch_max_int(const int* v, int n, int* out, cudaStream_t st);
// One warp per query: bar1 / bar2 = the r1-th / r2-th smallest key of keys[offs[q] .. + lens[q]) (exact; +inf
// where the stream is shorter).
// With max_len > 0 (a bound of the lens[q]) one block works on each query and streams of up to
// min(max_len, 6144) keys are staged in shared memory.
int launch_warp_bars(const float* keys, const int64_t* offs, const int64_t* lens, int nq, int r1, int r2, float* bar1,
                     float* bar2, cudaStream_t st, int64_t max_len = 0);
// One warp per query: the R smallest (key, id) of the buffer [q * cap, + min(count[q], cap)) as a set (the keys
// below the R-th smallest, then those equal to it by increasing id), padded with (+inf, kNoId), unordered.
int launch_warp_select(const float* keys, const int* ids, const int* count, int cap, int nq, int R, float* out_key,
                       int* out_id, cudaStream_t st);
// offs2[j] = offs[list[j]], lens2[j] = rowcnt[list[j]] for j < *count (<= max_count).
int launch_tc_compact_rows(const int* list, const int* count, int max_count, const int64_t* offs, const int* rowcnt,
                           int64_t* offs2, int* lens2, cudaStream_t st);

// Coarse ranking of the tensor-core IVF form from BF16 keys [nq, C] (ldk per row): per query, the best
// m = min(C, npc + margin) centroids by key, their exact FP32 squared distances (FP32 queries and
// centroids, row stride dpad), and the best npc of those by (distance, id) into probes [nq, npc],
// best first. With cmax > 0 (the largest centroid norm; dim the vectors' dimension) only the candidates whose
// key lies within the keys' certified error window of the npc-th key get exact distances: the others cannot
// be among the best npc, so the result is the same. cmin (optional): the keys' 32-column chunk minima
// [nq, ceil(C / 32)] (TcGemmArgs::out_cmin); with C <= 2,048 and m <= 32, only the chunks at or below a bar
// taken from them are read, with the same result.
int launch_tc_coarse(const float* keys, int64_t ldk, int nq, int C, int npc, int margin, const float* q,
                     const float* centroids, int dpad, int32_t* probes, cudaStream_t st, float cmax = 0.f,
                     int dim = 0, const float* cmin = nullptr);

}  // namespace annb

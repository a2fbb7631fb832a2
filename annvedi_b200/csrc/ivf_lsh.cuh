// LSH bucket tables of the IVF-LSH index (n_bits > 0, or several tables): candidate streams and the
// table build (ivf_lsh.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ivf.cuh"

namespace annb {

struct LshView {
    int T, B;                 // tables, bits per signature (B = 0: one bucket per list)
    const float* proj;        // [T * B, dpad] projections (zero past dim)
    const float* projT;       // [dim, T * B] the same, transposed (the query signatures read it)
    const float* mean;        // [dpad] mean of the rows (zero past dim)
    const int64_t* tab_off;   // [T * C * 2^B + 1]: bucket (t, c, sig) holds tab_ids[off .. off')
    const int32_t* tab_ids;   // [T * n] list-order row ids, ascending within a bucket
};

struct LshCandArgs {
    IvfView ix;
    LshView lsh;
    const int32_t* probes;  // [nq, npc] probed lists, best first
    int npc;
    const float* q;         // [nq, ldq] FP32 queries
    int64_t ldq;
    int nq, k, n_probes;
    int64_t max_c;          // candidate cap (INT64_MAX: none)
    int64_t ld;             // row stride of cand_ids (>= the longest possible stream)
    int64_t largest_list;   // rows of the largest list (visited bitmap size)
    int32_t* cand_ids;      // [nq, ld] the candidate stream (list-order rows)
    int64_t* n_cands;       // [nq]
    int32_t* n_seg;         // [nq] 0, or -1 when the query falls back to every row
    unsigned long long* ndist;  // distance counter (+= n_cands)
    uint32_t* sig;          // [nq, T] the query's signature per table (written by launch_lsh_signatures)
    int* pert;              // [nq, T, P] its flip masks in probe order, P = lsh_flips_kept(B, n_probes)
};

// The query's signatures and multiprobe flips (lsh_index_optimized.cpp:376-394, 407-426), one warp per
// query, into a.sig / a.pert.
int launch_lsh_signatures(const LshCandArgs& a, cudaStream_t st);
// LSHIndex::query's candidate stream (competitors/ivf_lsh/src/lsh_index_optimized.cpp:352-457) from the
// signatures above, one warp per query.
int launch_lsh_candidates(const LshCandArgs& a, cudaStream_t st);
// Flips probed per table: min(n_probes, m + m(m-1)/2), m = min(B, n_probes) (:407-426).
int lsh_flips_kept(int B, int n_probes);
// projT [dim, rows] from proj [rows, dpad].
int launch_lsh_transpose(const float* proj, int rows, int dim, int dpad, float* projT, cudaStream_t st);

// Signature of every list-order row in every table (the bucket build of IVFLSHIndex::fit, :260-283):
// key[t * n + i] = cluster_of(i) * 2^B + sig_t(i).
int launch_lsh_row_keys(const IvfView& ix, const LshView& lsh, int32_t* keys, cudaStream_t st);
// One thread per dimension: mean[d] = (sum over rows in list order, FP32) * (1 / n) (:176-184).
int launch_lsh_mean(const float* rows, int64_t n, int dim, int dpad, float* mean, cudaStream_t st);

}  // namespace annb

// Launch interface of the reference-semantics linear scan (compat.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace annb {

constexpr int kCompatQG = 8;  // queries per pass-1 block (kept in shared memory)

struct CompatArgs {
    const float* base;  // [n, ldb] FP32
    int64_t n;
    int dim;
    int64_t ldb;
    const float* q;     // [nq, ldq] FP32
    int64_t ldq;
    int q_end;          // set by launch_compat
    int k;
    int ncp;            // compat_num_checkpoints(dim)
    float* D;           // [chunk, n] scratch: full distances
    float* P;           // [chunk, ncp, n] scratch: checkpoint values
    float* T;           // [chunk, n] scratch: each row's heap threshold, then its ranking value
    float* kbuf;        // [chunk, k] scratch: the selected values
    int* ibuf;          // [chunk, k] scratch: their rows
    int64_t* out_ids;   // [nq, k]
    float* out_dists;   // [nq, k] ranking values, or nullptr
};

int compat_num_checkpoints(int dim);
// Runs queries [q_begin, q_begin + q_count) using D/P scratch sized for q_count queries.
int launch_compat(CompatArgs a, int q_begin, int q_count, cudaStream_t st);

}  // namespace annb

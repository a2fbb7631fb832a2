/*
 * annvedi_b200 -- C ABI of the B200 (sm_100a) search kernels for ANNvedi's data-parallel path.
 *
 * Plain C: opaque handles, pointers and sizes; no C++ or framework types cross this boundary, so
 * a ctypes/cffi, cgo, JNI or N-API host can bind it directly. Every function returns ANN_OK (0) or
 * a negative status; ann_last_error() then describes the failure (per host thread).
 *
 * Memory: `mem` = ANN_MEM_HOST means the data / query / output pointers are host memory and the
 * call is synchronous (it stages through pinned buffers and returns once results are written).
 * ANN_MEM_DEVICE means they are device pointers on the index's device and the call is
 * asynchronous on `stream` (a cudaStream_t; NULL = the legacy default stream).
 *
 * Workspaces: scratch device memory for queries lives in an ann_workspace. Calls that run
 * concurrently (on different streams) must use different workspaces; passing NULL uses the
 * index's own workspace. Workspaces grow on demand (stream-ordered allocation on `stream`).
 */
#ifndef ANNVEDI_B200_H
#define ANNVEDI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define ANN_OK 0
#define ANN_ERR_INVALID (-1)     /* bad argument (shape, k, null pointer, ...) */
#define ANN_ERR_CUDA (-2)        /* CUDA runtime error */
#define ANN_ERR_STATE (-3)       /* index not fitted */
#define ANN_ERR_NOMEM (-4)       /* allocation failed or admission refused */
#define ANN_ERR_TIMEOUT (-5)     /* a bounded device wait gave up */
#define ANN_ERR_UNSUPPORTED (-6) /* a size or mode this build does not handle */

/* metrics */
#define ANN_METRIC_L2 0 /* squared Euclidean distance, smaller is better */
#define ANN_METRIC_IP 1 /* inner product, larger is better */

/* search semantics */
#define ANN_MODE_EXACT 0     /* the true top-k by (distance, id) */
#define ANN_MODE_REFERENCE 1 /* the reference's ranking, incl. its 64-entry early-abandon heap */

/* where caller pointers live */
#define ANN_MEM_HOST 0
#define ANN_MEM_DEVICE 1

typedef struct ann_flat ann_flat;
typedef struct ann_workspace ann_workspace;

/* Library version string ("annvedi_b200 <major>.<minor> sm_100a"). */
const char* ann_version(void);

/* Message for the last failing call on this host thread ("" if none). Mirrors gf_last_error
 * (competitors/gpu_filter/src/gpu_filter.cu:77). */
const char* ann_last_error(void);

/* Number of kernels this library has launched in this process (all devices, all threads). */
int64_t ann_kernel_launches(void);

/* ---- workspaces -------------------------------------------------------------------------- */
int ann_workspace_create(ann_workspace** out, int device);
int ann_workspace_destroy(ann_workspace* ws);
/* Bytes of device scratch currently reserved. */
int64_t ann_workspace_bytes(const ann_workspace* ws);

/* ---- flat (linear) index -------------------------------------------------------------------
 * Replaces linear_ann_cpp.LinearIndex (competitors/linear/src/linear_index.cpp:62-131):
 *   LinearIndex() / fit(float32[N, d]) / query(float32[d], k) -> int64[k] /
 *   total_distances_count(). */

/* LinearIndex() (linear_index.cpp:71). */
int ann_flat_create(ann_flat** out, int device);
int ann_flat_destroy(ann_flat* h);

/* LinearIndex::fit (linear_index.cpp:73-88): copies `n` rows of `dim` floats (row stride `ld`
 * floats, ld >= dim) into the index's device memory. metric: ANN_METRIC_L2 or ANN_METRIC_IP. */
int ann_flat_fit(ann_flat* h, const float* data, int64_t n, int32_t dim, int64_t ld, int32_t metric, int32_t mem,
                 void* stream);

/* LinearIndex::query (linear_index.cpp:90-121), batched: `nq` queries of `dim` floats (row
 * stride `ldq`). Writes out_ids[nq][k'] (int64, -1 padded) and, if out_dists is not NULL, the
 * ranking values out_dists[nq][k'] (squared L2, or inner product for ANN_METRIC_IP), with
 * k' = min(k, n) as the reference clips k to n (linear_index.cpp:110). ANN_MODE_REFERENCE
 * reproduces the reference's own ranking (L2 only); ANN_MODE_EXACT returns the true top-k.
 * Adds n per query to the distance counter (linear_index.cpp:108). */
int ann_flat_query(ann_flat* h, ann_workspace* ws, const float* queries, int32_t nq, int64_t ldq, int32_t k,
                   int32_t mode, int32_t mem, int64_t* out_ids, float* out_dists, void* stream);

/* Per-stage timing with CUDA events recorded on the query's stream, in the spirit of the
 * reference's get_profile_results (competitors/ivf_lsh/src/lsh_index_optimized.cpp:535-548).
 * ann_flat_profile synchronises pending events and writes
 * out[0] = total scan-kernel ms, out[1] = total merge/selection ms, out[2] = scan launches,
 * out[3] = profiled query calls. Reset clears them. */
int ann_flat_set_profiling(ann_flat* h, int32_t enable);
int ann_flat_profile(ann_flat* h, double* out4);
int ann_flat_reset_profile(ann_flat* h);

/* LinearIndex::total_distances_count (linear_index.cpp:123). */
int64_t ann_flat_total_distances(const ann_flat* h);
int32_t ann_flat_dim(const ann_flat* h);
int64_t ann_flat_size(const ann_flat* h);

#ifdef __cplusplus
}
#endif
#endif /* ANNVEDI_B200_H */

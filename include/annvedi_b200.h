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
 * index's own workspace. A workspace grows on demand; growing drains the device first.
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
#define ANN_MODE_TC 2        /* IVF: candidates ranked by BF16 tensor-core keys, then the exact FP32 re-rank */
#define ANN_MODE_TC_SQ8 3    /* IVF: candidates ranked by tensor-core keys over the SQ8 codes themselves (int8
                                query weights x uint8 codes, int32 accumulation), then the exact FP32 re-rank */
/* IVF query flag, or'ed into the mode (no counterpart in the reference): the index holds one rank's share of
 * the lists (list sharding), so a query whose probed lists hold fewer than k of its rows returns what they
 * hold instead of scanning every row; the caller applies the every-row rule to the whole index. */
#define ANN_QUERY_SHARD 0x100

/* where caller pointers live */
#define ANN_MEM_HOST 0
#define ANN_MEM_DEVICE 1

typedef struct ann_flat ann_flat;
typedef struct ann_ivf ann_ivf;
typedef struct ann_workspace ann_workspace;

/* Library version string ("annvedi_b200 <major>.<minor> sm_100a"). */
const char* ann_version(void);

/* The code the loaded library runs on `device` (no counterpart in the reference): out2 = {binary
 * version, PTX version} of its kernels as cudaFuncGetAttributes reports them (100 = sm_100a machine
 * code). Needs a visible device. */
int ann_kernel_arch(int device, int32_t* out2);

/* Self-test of the tensor-core GEMM's bounded waits (no counterpart in the reference; the failure
 * path of its error status, gf_last_error at competitors/gpu_filter/src/gpu_filter.cu:27-47): one small
 * GEMM on `device` whose producer issues no copies and whose waits give up after `wait_ns`
 * (1e3..2e9). Every waiting warp gives up, sets the device flag and leaves; TMEM is released and the
 * context stays usable. flag_out = the flag the kernel left (2: a wait gave up). */
int ann_tc_wait_selftest(int device, int64_t wait_ns, int32_t* flag_out);

/* Message for the last failing call on this host thread ("" if none). Mirrors gf_last_error
 * (competitors/gpu_filter/src/gpu_filter.cu:77). */
const char* ann_last_error(void);

/* Number of kernels this library has launched in this process (all devices, all threads). */
int64_t ann_kernel_launches(void);

/* ---- workspaces -------------------------------------------------------------------------- */
int ann_workspace_create(ann_workspace** out, int device);
int ann_workspace_destroy(ann_workspace* ws);
/* Bytes of device scratch currently reserved (both of the workspace's device arenas). */
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
/* All stage totals of the flat index: out[0] scan ms, out[1] merge ms; for ann_flat_query_tc out[2]
 * sample pass and bars ms, out[3] filter pass (or full key matrix) ms, out[4] grouping, selections and
 * re-runs ms, out[5] exact re-rank ms; out[6] scan launches, out[7] tensor-core GEMM launches, out[8]
 * filter passes (each timed alone in out[3]), out[9] profiled calls. */
int ann_flat_profile_stages(ann_flat* h, double* out10);

/* Tensor-core form of ann_flat_query (no counterpart in the reference; the reference's only fast scan
 * is its CPU loop): keys for every (query, row) from a BF16 tcgen05 GEMM with FP32 accumulation
 * (|x|^2 - 2 x.q for L2, -x.q for inner product; the base is copied to BF16 once, on first use), the
 * best R = max(k, refine_r > 0 ? refine_r : 4k) rows per query by that key, then their exact FP32
 * distances (or inner products) re-ranked to the final k. Same outputs and counter as ann_flat_query. */
int ann_flat_query_tc(ann_flat* h, ann_workspace* ws, const float* queries, int32_t nq, int64_t ldq, int32_t k,
                      int32_t refine_r, int32_t mem, int64_t* out_ids, float* out_dists, void* stream);

/* Element kind of the tensor-core search (no counterpart in the reference): ANN_TC_BF16 (default) or
 * ANN_TC_E4M3 -- FP8 operands with a scale per vector (s = max|x| / 448), FP32 accumulation, the key
 * |x|^2 - 2 s_x s_q acc (or -s_x s_q acc for inner product) formed in the GEMM's epilogue; twice the tensor
 * rate of BF16 and half the bytes, with a coarser key that a deeper re-rank (refine_r) wins back. The
 * operand copy of a kind is built on its first query. */
#define ANN_TC_BF16 0
#define ANN_TC_E4M3 1
int ann_flat_set_tc_precision(ann_flat* h, int32_t precision);

/* Options of the exact scan (no counterpart in the reference):
 *   ANN_FLAT_OPT_QUERY_TILE: queries per CTA of the exact scan's staged form -- 8, 16 or 32 queries share
 *     each staged row chunk; 0 (the default) picks by the batch size (batches of up to 4 queries then stream
 *     the rows instead, whose sums run in another order). Among 8, 16 and 32 the results are identical (every
 *     tile sums a pair's terms in the same order and the splits merge by (distance, id)); the tile changes
 *     speed only, and autotune.tune_flat_tile picks it by timing. */
#define ANN_FLAT_OPT_QUERY_TILE 1
int ann_flat_set_option(ann_flat* h, int32_t option, int64_t value);

/* Diagnostic: the tensor-core key matrix out_keys[nq][n] (device pointers; synchronous). */
int ann_flat_scores_tc(ann_flat* h, const float* queries, int32_t nq, int64_t ldq, float* out_keys, void* stream);

/* Reads and clears the index's device error flag (ANN_ERR_TIMEOUT if a bounded device wait gave up). */
int ann_flat_device_status(ann_flat* h);

/* Merge of per-shard results (row or list sharding over ranks: each rank searches its share, maps its
 * ids to global ids, and the ranks' lists are all-gathered): dists / ids [nq, parts, k] device arrays,
 * each part as the search returns it (ids < 0 empty, global ids below 2^31; squared L2 distances, or
 * inner-product scores when metric = ANN_METRIC_IP); out_ids / out_dists [nq, k] (out_dists may be NULL)
 * get the best k by (distance, id), ties by the lower id whatever part holds it. Asynchronous on
 * `stream`. No counterpart in the reference, whose indexes live in one process (the exchange step of a
 * sharded linear_index or IVF index). */
int ann_merge_topk(const float* dists, const int64_t* ids, int32_t nq, int32_t parts, int32_t k, int32_t metric,
                   int64_t* out_ids, float* out_dists, void* stream);

/* The r smallest keys of each of nq device rows keys[q * ld + p], p < lens[q] (ld when lens is NULL),
 * by (key, position): out_keys / out_pos [nq, r] device arrays, padded with +inf / INT32_MAX where a
 * row holds fewer than r keys. The set is exact; its order is unspecified. This is the selection of the
 * tensor-core forms (the best R candidates before the exact re-rank); the reference partially sorts
 * its candidate pairs for the same purpose (lsh_index_optimized.cpp:471-480). Asynchronous on `stream`. */
int ann_select_smallest(const float* keys, int64_t ld, const int64_t* lens, int32_t nq, int32_t r, float* out_keys,
                        int32_t* out_pos, void* stream);

/* Exact-mode ann_flat_query for callers that cannot let a library allocate device memory (an
 * application that owns every device allocation through its own pool, or a serving thread that must
 * not call cudaMalloc/cudaFree because they can synchronise the device). No counterpart in the
 * reference. Queries and outputs are device pointers on the index's device (ANN_MEM_DEVICE); the
 * call runs asynchronously on `stream`. Its scratch is a fixed 16 MiB array compiled into the library
 * (held on every device that loads it until exit); batches needing more scratch are rejected with
 * ANN_ERR_INVALID. The first call on a device resolves the array's device address (make that call
 * before any stream capture). All calls share the array: calls that overlap on the GPU race. Adds n
 * per query to the distance counter, as ann_flat_query does. */
int ann_flat_query_noalloc(ann_flat* h, const float* queries, int32_t nq, int64_t ldq, int32_t k,
                           int64_t* out_ids, float* out_dists, void* stream);

/* LinearIndex::total_distances_count (linear_index.cpp:123). */
int64_t ann_flat_total_distances(const ann_flat* h);
int32_t ann_flat_dim(const ann_flat* h);
int64_t ann_flat_size(const ann_flat* h);

/* ---- IVF-SQ8 index ------------------------------------------------------------------------
 * Replaces ivf_lsh_cpp.LSHIndex (competitors/ivf_lsh/src/lsh_index_optimized.cpp:124-667) with
 * n_tables = 1, n_bits = 0: inverted lists of per-dimension SQ8 codes and an FP32 re-rank. */

/* LSHIndex() (lsh_index_optimized.cpp:126). */
int ann_ivf_create(ann_ivf** out, int device);
int ann_ivf_destroy(ann_ivf* h);

/* LSHIndex::fit (lsh_index_optimized.cpp:128-292) on the GPU: `n_clusters` lists (clamped to n).
 * Centroids: `centroids` [n_clusters, dim] if not NULL, else the reference's k-means (run_kmeans,
 * :551-616) for `kmeans_iters` rounds (the reference runs 15): seeds from std::shuffle with
 * std::mt19937(1337), assignment by the reference's distance arithmetic, sums per ThreadPool chunk
 * of `num_threads` (<= 0: this host's hardware concurrency, as the reference sizes its pool, :140).
 * With the same thread count the centroids and lists are bit-identical to the reference's fit.
 * Lists: `assign` [n] if not NULL, else the nearest centroid (the last k-means assignment when
 * iterating). Rows are reordered list by list and SQ8-encoded with per-dimension scale/offset
 * exactly as the reference computes them. `data`, `centroids` and `assign` live where `mem` says. */
int ann_ivf_fit(ann_ivf* h, const float* data, int64_t n, int32_t dim, int64_t ld, int32_t n_clusters,
                const float* centroids, const int32_t* assign, int32_t kmeans_iters, int32_t num_threads,
                int32_t mem, void* stream);

/* Imports an index state in the reference's layout (all host pointers, rows in list order):
 * centroids [C, dim], original [n, dim] FP32, codes [n, dim] uint8, scale / offset [dim],
 * r2o [n] list-order row -> original id, list_offsets [C + 1]. The parity path: the reference
 * (through a state export) and this index then answer queries over the same lists. */
int ann_ivf_import(ann_ivf* h, int64_t n, int32_t dim, int32_t n_clusters, const float* centroids,
                   const float* original, const uint8_t* codes, const float* scale, const float* offset,
                   const int32_t* r2o, const int64_t* list_offsets);

/* Copies the state out to host arrays of the same shapes (NULL skips an array). */
int ann_ivf_export(ann_ivf* h, float* centroids, float* original, uint8_t* codes, float* scale, float* offset,
                   int32_t* r2o, int64_t* list_offsets);

/* out4 = {n, dim, n_clusters, largest list}. */
int ann_ivf_info(const ann_ivf* h, int64_t* out4);

/* LSH bucket tables of IVFLSHIndex (lsh_index_optimized.cpp:216-283): n_tables tables of 2^n_bits
 * buckets per list; bucket (t, c, sig) holds table_ids[table_offsets[(t*C + c)*2^n_bits + sig] ..] (list-
 * order rows, ascending), signatures the signs of (x - mean) . p over the table's n_bits projections.
 * Queries then walk the buckets as LSHIndex::query does (:352-457), n_probes multiprobe flips included.
 * import: the reference's arrays (after ann_ivf_import); build: the reference's projections (mt19937(42),
 * N(0,1), Gram-Schmidt per table) and tables from the fitted lists; export: out2 = {n_tables, n_bits},
 * then the arrays (NULL skips one). */
int ann_ivf_import_tables(ann_ivf* h, int32_t n_tables, int32_t n_bits, const float* projections, const float* mean,
                          const int64_t* table_offsets, const int32_t* table_ids);
int ann_ivf_build_tables(ann_ivf* h, int32_t n_tables, int32_t n_bits, void* stream);
int ann_ivf_export_tables(ann_ivf* h, int32_t* out2, float* projections, float* mean, int64_t* table_offsets,
                          int32_t* table_ids);

/* LSHIndex::query (lsh_index_optimized.cpp:304-516), batched over `nq` queries:
 * lists ranked by centroid distance, the first `n_probe_clusters` probed whole, in order, until the
 * candidate stream reaches `max_candidates` (-1: the reference's max(2000, 4 * refine target);
 * 0: no cap); a query whose probed lists hold fewer than k points scans every row; SQ8 distances
 * over the stream; the best R = max(k, refine_r > 0 ? refine_r : 4k) re-ranked with exact FP32
 * distances; the best k returned as original ids (-1 padded) with their squared distances.
 * ANN_MODE_REFERENCE reproduces the reference's own ranking, including the 64-entry early-abandon
 * heap of each of `num_threads` ThreadPool chunks (<= 0: this host's hardware concurrency, as the
 * reference sizes its pool); ANN_MODE_EXACT ranks by full SQ8 distances; ANN_MODE_TC ranks the same
 * candidate streams by BF16 tcgen05 keys of the FP32 rows (|x|^2 - 2 x.q, FP32 accumulate), the lists
 * scored list-major as grouped GEMMs (no counterpart in the reference; whole lists only). With
 * bucket tables (ann_ivf_import_tables / ann_ivf_build_tables) the candidate streams are the buckets'
 * and `n_probes` flips widen each table's probe. Adds each query's candidate count to the distance counter (:459-460). */
int ann_ivf_query(ann_ivf* h, ann_workspace* ws, const float* queries, int32_t nq, int64_t ldq, int32_t k,
                  int32_t n_probes, int32_t n_probe_clusters, int32_t refine_r, int64_t max_candidates, int32_t mode,
                  int32_t num_threads, int32_t mem, int64_t* out_ids, float* out_dists, void* stream);

/* Reads and clears the index's device error flag: ANN_ERR_TIMEOUT if a kernel's bounded wait gave up
 * since the last check (its queries' results are invalid), else ANN_OK. Synchronous; host-memory
 * queries check it themselves. No counterpart in the reference (its waits are host condition
 * variables, src/thread_pool.h:119-122). */
int ann_ivf_device_status(ann_ivf* h);

/* LSHIndex::total_distances_count / reset_distances_count (lsh_index_optimized.cpp:518-524). */
int64_t ann_ivf_total_distances(ann_ivf* h);
int ann_ivf_reset_distances(ann_ivf* h);

/* LSHIndex::get_profile_results / reset_profile_results (lsh_index_optimized.cpp:526-548), timed
 * with CUDA events on the query stream while profiling is on: out8 = {coarse ranking ms, LSH
 * signature ms, candidate plan / bucket walk ms, SQ8 (or BF16) key ms, best-R selection ms, FP32
 * re-rank + top-k ms, profiled calls, queries}. Totals, not averages. */
int ann_ivf_set_profiling(ann_ivf* h, int32_t enable);
int ann_ivf_profile(ann_ivf* h, double* out8);
/* Query options of an index (no counterpart in the reference, whose query takes its settings as
 * arguments); none of them changes results:
 *   ANN_IVF_OPT_SAMPLE_DIV: the tensor-core forms' sampled bars score the first ceil(size / value) rows of
 *     each probed list (2..64, default 8); the bars only prune.
 *   ANN_IVF_OPT_SAMPLED_MIN: batches of at least this many queries take the sampled path (default 256). */
#define ANN_IVF_OPT_SAMPLE_DIV 2
#define ANN_IVF_OPT_SAMPLED_MIN 3
int ann_ivf_set_option(ann_ivf* h, int32_t option, int64_t value);

/* Single-kernel times of the same profiled calls (CUDA events around each launch, on the query stream):
 * out8 = {list-keys kernel ms (the grouped tensor-core GEMM of the list rows, or the SQ8 batched
 * kernel), sampled-bar kernel ms, best-R selection kernel ms, FP32 re-rank kernel ms, then the launch
 * count of each}. Totals; cleared by ann_ivf_reset_profile. No counterpart in the reference. */
int ann_ivf_kernel_profile(ann_ivf* h, double* out8);
int ann_ivf_reset_profile(ann_ivf* h);

#ifdef __cplusplus
}
#endif
#endif /* ANNVEDI_B200_H */

/* The reference's GPU quantized-filter contestant, as a drop-in C ABI served by this library's B200 kernels.
 *
 * The five entry points have the names, signatures, argument meaning and return conventions of the
 * reference's libgpufilter.so (competitors/gpu_filter/src/gpu_filter.cu:77-190), which its ctypes wrapper
 * (competitors/gpu_filter/algorithm.py:6-16) binds; loading libannvedi_b200.so under that name serves the
 * wrapper unchanged. Results: the same ids as the reference for the same inputs (the same SQ8 codes, the same
 * FMA chain per row for the filter key, the first R rows by (key, row id), the same FP32 re-rank arithmetic,
 * the top k by (distance, id)), with the scan, selection and re-rank on the GPU.
 */
#ifndef ANNVEDI_GPU_FILTER_H
#define ANNVEDI_GPU_FILTER_H

#ifdef __cplusplus
extern "C" {
#endif

/* Message for the last failing gf_* call on this host thread ("" if none).
 * Replaces gf_last_error (gpu_filter.cu:77). */
const char* gf_last_error(void);

/* Per-dimension SQ8 of train [n, dim] (row-major FP32): scale = (max - min) / 255 (1 when the range is
 * <= 1e-8), offset = min, code = clamp(rint((x - offset) / scale), 0, 255); the codes (dim-major) and an
 * FP32 copy of train go to the current device. NULL on error (dim > 4096, no device, bad arguments), with
 * the message in gf_last_error. The reference borrows train for the handle's lifetime; this one copies it,
 * so the caller may release it. Replaces gf_create (gpu_filter.cu:79-133). */
void* gf_create(const float* train, long n, long dim);

/* Top-k ids of query q [dim] (host FP32) into out_ids [k] (host int64): r is raised to k and capped at n;
 * every row's SQ8 key sum_d (code * scale - (q - offset))^2 (one FMA chain in dimension order), the r rows
 * with the smallest (key, id), their exact FP32 squared distances, the best min(k, r) by (distance, id) in
 * ascending order. Returns min(k, r), or -1 on error. Adds r to the distance count. One call at a time per
 * handle (calls are serialised). Replaces gf_query (gpu_filter.cu:135-176); k <= 4096. */
int gf_query(void* handle, const float* q, int k, int r, long long* out_ids);

/* Full-precision distances computed so far (r per query). Replaces gf_ndist (gpu_filter.cu:178). */
long long gf_ndist(void* handle);

/* Releases the handle and its device memory (NULL is a no-op). Replaces gf_free (gpu_filter.cu:180-190). */
void gf_free(void* handle);

#ifdef __cplusplus
}
#endif

#endif /* ANNVEDI_GPU_FILTER_H */

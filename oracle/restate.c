/*
 * CPU restatement of ANNvedi's search path: the oracle for the GPU kernels.
 *
 * ORACLE INFRASTRUCTURE. Only tests/, the smoke check and bench.py's CPU-baseline leg load this
 * library, and only to check or time against; no product code path calls it.
 *
 * Every function restates a reference function, cited by file:line (paths inside the reference
 * project). The reference is compiled with -O3 -ffast-math (setup.py:10); under those flags the
 * compiler fuses `sum + diff*diff` into a fused multiply-add and fixes one order for the
 * 8-float horizontal add. This file is compiled with -ffp-contract=off and spells both out
 * (fmaf, explicit parenthesisation) so its results are bit-identical to the compiled reference;
 * tests/test_oracle.py pins that against the reference's own compute_l2_distance.
 *
 * `isa` selects the reference build's code path: 16 = AVX-512 (simd.h:33-64), 8 = AVX2
 * (simd.h:65-100), 1 = scalar (simd.h:101-114).
 */
#define _GNU_SOURCE
#include <float.h>
#include <pthread.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/*
 * Arithmetic of the compiled reference (-O3 -ffast-math, GCC 13, x86-64-v4 / x86-64-v3), pinned
 * bit-for-bit against the reference's own compute_l2_distance / compute_l2_distance_quantized by
 * tests/test_oracle.py:
 *   - FP32 lanes accumulate as sum = sum + diff*diff, NOT fused (the _mm512_add_ps/_mm512_mul_ps
 *     intrinsics are kept separate);
 *   - the 8-float horizontal add (simd.h:21-28, :87-89) is a halving fold
 *     ((t0+t4)+(t2+t6)) + ((t1+t5)+(t3+t7));
 *   - the scalar remainder loop for dim % lanes != 0 (simd.h:58-62, :94-98) is vectorised by the
 *     compiler: one half-width chunk of fused squares folded the same way and added to the sum,
 *     then fused scalar steps;
 *   - the SQ8 body uses explicit fmsub/fmadd intrinsics (fused) and its remainder is scalar fused.
 */
static inline float fold8(const float *t) {
    float a0 = t[0] + t[4], a1 = t[1] + t[5], a2 = t[2] + t[6], a3 = t[3] + t[7];
    return (a0 + a2) + (a1 + a3);
}

static inline float fold4(const float *t) { return (t[0] + t[2]) + (t[1] + t[3]); }

static inline float lanes_reduce(const float *lane, int isa) {
    float t[8];
    if (isa == 16) {
        for (int j = 0; j < 8; ++j) t[j] = lane[j] + lane[j + 8];
    } else {
        for (int j = 0; j < 8; ++j) t[j] = lane[j];
    }
    return fold8(t);
}

/* compute_l2_distance, competitors/ivf_lsh/src/simd.h:32-115 (same text in competitors/linear). */
float orc_l2(const float *a, const float *b, int dim, float threshold, int isa) {
    if (isa == 1) {
        float sum = 0.0f;
        for (int i = 0; i < dim; ++i) {
            float diff = a[i] - b[i];
            sum = fmaf(diff, diff, sum);
            if (i % 16 == 15 && sum >= threshold) return sum;
        }
        return sum;
    }
    float lane[16] = {0};
    const int w = isa; /* 16 or 8 lanes */
    const int chk = (w == 16) ? 80 : 88;
    int i = 0;
    for (; i + w - 1 < dim; i += w) {
        for (int j = 0; j < w; ++j) {
            float diff = a[i + j] - b[i + j];
            float sq = diff * diff;
            lane[j] = lane[j] + sq;
        }
        if (i % 96 == chk) {
            float s = lanes_reduce(lane, w);
            if (s >= threshold) return s;
        }
    }
    float sum = lanes_reduce(lane, w);
    if (sum >= threshold) return sum;
    const int half = w / 2;
    if (dim - i >= half) {
        float t[8];
        for (int j = 0; j < half; ++j) {
            float diff = a[i + j] - b[i + j];
            t[j] = diff * diff;
        }
        sum = sum + (half == 8 ? fold8(t) : fold4(t));
        i += half;
    }
    for (; i < dim; ++i) {
        float diff = a[i] - b[i];
        sum = fmaf(diff, diff, sum);
    }
    return sum;
}

/* compute_l2_distance_quantized, competitors/ivf_lsh/src/simd.h:118-211. */
float orc_l2_sq8(const uint8_t *a, const float *qs, int dim, const float *scale, float threshold, int isa) {
    if (isa == 1) {
        float sum = 0.0f;
        for (int i = 0; i < dim; ++i) {
            float diff = fmaf((float)a[i], scale[i], -qs[i]);
            sum = fmaf(diff, diff, sum);
            if (i % 16 == 15 && sum >= threshold) return sum;
        }
        return sum;
    }
    float lane[16] = {0};
    const int w = isa;
    const int chk = (w == 16) ? 80 : 88;
    int i = 0;
    for (; i + w - 1 < dim; i += w) {
        for (int j = 0; j < w; ++j) {
            float diff = fmaf((float)a[i + j], scale[i + j], -qs[i + j]);
            lane[j] = fmaf(diff, diff, lane[j]);
        }
        if (i % 96 == chk) {
            float s = lanes_reduce(lane, w);
            if (s >= threshold) return s;
        }
    }
    float sum = lanes_reduce(lane, w);
    if (sum >= threshold) return sum;
    for (; i < dim; ++i) {
        float diff = fmaf((float)a[i], scale[i], -qs[i]);
        sum = fmaf(diff, diff, sum);
    }
    return sum;
}

typedef struct {
    float v;
    int32_t id;
} pair_t;

static int cmp_pair(const void *x, const void *y) {
    const pair_t *a = (const pair_t *)x, *b = (const pair_t *)y;
    if (a->v < b->v) return -1;
    if (a->v > b->v) return 1;
    return (a->id > b->id) - (a->id < b->id);
}

/* Sorted insert into a worst-last heap of `lim` entries, as in linear_worker
 * (competitors/linear/src/linear_index.cpp:50-58) and lsh_worker
 * (competitors/ivf_lsh/src/lsh_index_optimized.cpp:112-120). */
static inline void heap_insert(pair_t *h, int lim, float v, int32_t id) {
    int pos = lim - 1;
    while (pos > 0 && v < h[pos - 1].v) {
        h[pos] = h[pos - 1];
        --pos;
    }
    h[pos].v = v;
    h[pos].id = id;
}

/* linear_worker over [0, n): the value each point is ranked by
 * (competitors/linear/src/linear_index.cpp:27-60). vals[i] is the exact squared distance when it
 * beats the current 64th-best, else the first checkpoint partial sum that reached it. */
void orc_linear_values(const float *data, int64_t n, int dim, int64_t ld, const float *q, int k, int isa,
                       float *vals) {
    pair_t heap[64];
    int lim = k < 64 ? k : 64;
    for (int j = 0; j < lim; ++j) {
        heap[j].v = FLT_MAX;
        heap[j].id = -1;
    }
    for (int64_t i = 0; i < n; ++i) {
        float thr = heap[lim - 1].v;
        float v = orc_l2(data + i * ld, q, dim, thr, isa);
        vals[i] = v;
        if (v < thr) heap_insert(heap, lim, v, (int32_t)i);
    }
}

/* LinearIndex::query (competitors/linear/src/linear_index.cpp:90-121): values as above, then
 * partial_sort of (value, id) pairs and the first k ids. Returns the number written. */
int orc_linear_query(const float *data, int64_t n, int dim, int64_t ld, const float *q, int k, int isa,
                     int64_t *out_ids, float *out_vals) {
    float *vals = (float *)malloc(sizeof(float) * (size_t)n);
    pair_t *p = (pair_t *)malloc(sizeof(pair_t) * (size_t)n);
    if (!vals || !p) {
        free(vals);
        free(p);
        return -1;
    }
    orc_linear_values(data, n, dim, ld, q, k, isa, vals);
    for (int64_t i = 0; i < n; ++i) {
        p[i].v = vals[i];
        p[i].id = (int32_t)i;
    }
    if (k > n) k = (int)n;
    qsort(p, (size_t)n, sizeof(pair_t), cmp_pair);
    for (int i = 0; i < k; ++i) {
        out_ids[i] = p[i].id;
        if (out_vals) out_vals[i] = p[i].v;
    }
    free(vals);
    free(p);
    return k;
}

/* Batched form of the above over many queries, parallel over queries with plain pthreads
 * (each query is serial, exactly as the reference runs it). */
typedef struct {
    const float *data, *qs;
    int64_t n, ld;
    int dim, nq, k, isa, tid, nt, bad;
    int64_t *out_ids;
    float *out_vals;
} lin_job_t;

static void *lin_job(void *arg) {
    lin_job_t *j = (lin_job_t *)arg;
    for (int i = j->tid; i < j->nq; i += j->nt)
        if (orc_linear_query(j->data, j->n, j->dim, j->ld, j->qs + (int64_t)i * j->dim, j->k, j->isa,
                             j->out_ids + (int64_t)i * j->k, j->out_vals ? j->out_vals + (int64_t)i * j->k : NULL) < 0)
            j->bad = 1;
    return NULL;
}

int orc_linear_query_batch(const float *data, int64_t n, int dim, int64_t ld, const float *qs, int nq, int k,
                           int isa, int64_t *out_ids, float *out_vals) {
    enum { MAXT = 64 };
    long nt = sysconf(_SC_NPROCESSORS_ONLN);
    if (nt < 1) nt = 1;
    if (nt > MAXT) nt = MAXT;
    if (nt > nq) nt = nq > 0 ? nq : 1;
    pthread_t th[MAXT];
    lin_job_t jobs[MAXT];
    int bad = 0;
    for (int t = 0; t < nt; ++t) {
        lin_job_t j = {data, qs, n, ld, dim, nq, k, isa, t, (int)nt, 0, out_ids, out_vals};
        jobs[t] = j;
        if (pthread_create(&th[t], NULL, lin_job, &jobs[t]) != 0) {
            lin_job(&jobs[t]);
            th[t] = 0;
        }
    }
    for (int t = 0; t < nt; ++t) {
        if (th[t]) pthread_join(th[t], NULL);
        bad |= jobs[t].bad;
    }
    return bad ? -1 : 0;
}

/* ThreadPool::run_parallel chunking (src/thread_pool.h:93-124): chunk c of `t` covers
 * [start_c, end_c), the first n % t chunks one element longer. */
static void chunk_bounds(int64_t n, int t, int c, int64_t *s, int64_t *e) {
    int64_t base = n / t, rem = n % t;
    *s = c * base + (c < rem ? c : rem);
    *e = *s + base + (c < rem ? 1 : 0);
}

/* lsh_worker (competitors/ivf_lsh/src/lsh_index_optimized.cpp:86-122) over one chunk. */
static void sq8_chunk(const int32_t *cand, int64_t s, int64_t e, const uint8_t *codes, int dim, const float *qs,
                      const float *scale, int k, int isa, pair_t *dists) {
    pair_t heap[64];
    int lim = k < 64 ? k : 64;
    for (int j = 0; j < lim; ++j) {
        heap[j].v = FLT_MAX;
        heap[j].id = -1;
    }
    for (int64_t i = s; i < e; ++i) {
        int32_t idx = cand[i];
        float thr = heap[lim - 1].v;
        float v = orc_l2_sq8(codes + (int64_t)idx * dim, qs, dim, scale, thr, isa);
        dists[i].v = v;
        dists[i].id = idx;
        if (v < thr) heap_insert(heap, lim, v, idx);
    }
}

static int cmp_first(const void *x, const void *y) {
    const pair_t *a = (const pair_t *)x, *b = (const pair_t *)y;
    if (a->v < b->v) return -1;
    if (a->v > b->v) return 1;
    return (a->id > b->id) - (a->id < b->id); /* the reference leaves this order unspecified */
}

typedef struct {
    int64_t i;
    float s;
    int b1, b2;
} pert_t;

static int cmp_pert(const void *x, const void *y) {
    const pert_t *a = (const pert_t *)x, *b = (const pert_t *)y;
    if (a->s < b->s) return -1;
    if (a->s > b->s) return 1;
    return (a->i > b->i) - (a->i < b->i);
}

typedef struct {
    float v;
    int b;
} bd_t;
static int cmp_bd(const void *x, const void *y) {
    const bd_t *a = (const bd_t *)x, *b = (const bd_t *)y;
    if (a->v < b->v) return -1;
    if (a->v > b->v) return 1;
    return (a->b > b->b) - (a->b < b->b);
}

/*
 * IVFLSHIndex::query (competitors/ivf_lsh/src/lsh_index_optimized.cpp:304-516) over an index
 * state laid out as the reference keeps it:
 *   centroids [C, dim]; codes [N, dim] (cluster-contiguous order); original [N, dim]; scale,
 *   offset, mean [dim]; r2o [N] (reordered -> original id); projections [T*B, dim];
 *   table_off [T*C*2^B + 1] / table_ids: bucket (t, c, sig) holds ids table_ids[off..off').
 * `num_threads` is the reference ThreadPool size (hardware_concurrency() on the reference host).
 * `max_cands` < 0 uses the reference cap max(2000, 4*target_refine) (:357-358); 0 lifts it.
 * Writes k ids (original numbering, -1 padded) and their exact distances; returns n_cands
 * (the amount added to get_n_distances, :459-460), or -1 on allocation failure.
 */
int64_t orc_ivf_query(int64_t N, int dim, int C, int T, int B, const float *centroids, const uint8_t *codes,
                      const float *original, const float *scale, const float *offset, const float *mean,
                      const int32_t *r2o, const float *projections, const int64_t *table_off,
                      const int32_t *table_ids, const float *q, int k, int n_probes, int n_probe_clusters,
                      int refine_r, int num_threads, int isa, int64_t max_cands_override, int64_t *out_ids,
                      float *out_dists) {
    float *qs = (float *)malloc(sizeof(float) * dim);
    pair_t *cd = (pair_t *)malloc(sizeof(pair_t) * (size_t)C);
    uint8_t *visited = (uint8_t *)calloc((size_t)N, 1);
    int32_t *cand = (int32_t *)malloc(sizeof(int32_t) * (size_t)(N > 0 ? N : 1));
    float *dots = (float *)malloc(sizeof(float) * (B > 0 ? B : 1));
    bd_t *bd = (bd_t *)malloc(sizeof(bd_t) * (B > 0 ? B : 1));
    pert_t *pert = (pert_t *)malloc(sizeof(pert_t) * (size_t)(B + B * (B - 1) / 2 + 1));
    pair_t *dists = NULL;
    int64_t nc = 0;
    int64_t ret = -1;
    if (!qs || !cd || !visited || !cand || !dots || !bd || !pert) goto done;
    for (int d = 0; d < dim; ++d) qs[d] = q[d] - offset[d];
    for (int c = 0; c < C; ++c) {
        cd[c].v = orc_l2(q, centroids + (int64_t)c * dim, dim, FLT_MAX, isa);
        cd[c].id = c;
    }
    int active = n_probe_clusters < C ? n_probe_clusters : C;
    qsort(cd, (size_t)C, sizeof(pair_t), cmp_pair);
    int target_refine = refine_r > 0 ? refine_r : 4 * k;
    int64_t max_c = 4 * (int64_t)target_refine;
    if (max_c < 2000) max_c = 2000;
    if (max_cands_override == 0) max_c = INT64_MAX;
    else if (max_cands_override > 0) max_c = max_cands_override;
    const int nb = 1 << B;
    for (int ci = 0; ci < active; ++ci) {
        if (nc >= max_c) break;
        int cid = cd[ci].id;
        for (int t = 0; t < T; ++t) {
            if (nc >= max_c) break;
            uint32_t sig = 0;
            for (int b = 0; b < B; ++b) {
                const float *pr = projections + (int64_t)(t * B + b) * dim;
                float dot = 0.0f;
                for (int d = 0; d < dim; ++d) dot += (q[d] - mean[d]) * pr[d];
                dots[b] = dot;
                bd[b].v = fabsf(dot);
                bd[b].b = b;
                if (dot > 0.0f) sig |= (1u << b);
            }
            int64_t base = ((int64_t)t * C + cid) * nb;
            for (int64_t j = table_off[base + sig]; j < table_off[base + sig + 1]; ++j) {
                int32_t idx = table_ids[j];
                if (!visited[idx]) {
                    visited[idx] = 1;
                    cand[nc++] = idx;
                }
            }
            if (n_probes > 0) {
                qsort(bd, (size_t)B, sizeof(bd_t), cmp_bd);
                int m = B < n_probes ? B : n_probes, np = 0;
                for (int i = 0; i < m; ++i) {
                    pert[np].i = np;
                    pert[np].s = bd[i].v;
                    pert[np].b1 = bd[i].b;
                    pert[np].b2 = -1;
                    ++np;
                }
                for (int i = 0; i < m; ++i)
                    for (int j = i + 1; j < m; ++j) {
                        pert[np].i = np;
                        pert[np].s = bd[i].v + bd[j].v;
                        pert[np].b1 = bd[i].b;
                        pert[np].b2 = bd[j].b;
                        ++np;
                    }
                qsort(pert, (size_t)np, sizeof(pert_t), cmp_pert);
                int pc = n_probes < np ? n_probes : np;
                for (int p = 0; p < pc; ++p) {
                    if (nc >= max_c) break;
                    uint32_t ps = sig ^ (1u << pert[p].b1);
                    if (pert[p].b2 != -1) ps ^= (1u << pert[p].b2);
                    for (int64_t j = table_off[base + ps]; j < table_off[base + ps + 1]; ++j) {
                        int32_t idx = table_ids[j];
                        if (!visited[idx]) {
                            visited[idx] = 1;
                            cand[nc++] = idx;
                        }
                    }
                }
            }
        }
    }
    if (nc < k) {
        nc = N;
        for (int64_t i = 0; i < N; ++i) cand[i] = (int32_t)i;
    }
    dists = (pair_t *)malloc(sizeof(pair_t) * (size_t)(nc > 0 ? nc : 1));
    if (!dists) goto done;
    if (num_threads > 0 && nc >= 2 * (int64_t)num_threads) {
        for (int c = 0; c < num_threads; ++c) {
            int64_t s, e;
            chunk_bounds(nc, num_threads, c, &s, &e);
            sq8_chunk(cand, s, e, codes, dim, qs, scale, k, isa, dists);
        }
    } else {
        sq8_chunk(cand, 0, nc, codes, dim, qs, scale, k, isa, dists);
    }
    int tr = refine_r > 0 ? refine_r : 4 * k;
    if (tr < k) tr = k;
    int64_t ar = tr < nc ? tr : nc;
    qsort(dists, (size_t)nc, sizeof(pair_t), cmp_first);
    for (int64_t i = 0; i < ar; ++i) {
        int32_t idx = dists[i].id;
        dists[i].v = orc_l2(original + (int64_t)idx * dim, q, dim, FLT_MAX, isa);
    }
    qsort(dists, (size_t)ar, sizeof(pair_t), cmp_first);
    int64_t sk = k < ar ? k : ar;
    for (int i = 0; i < k; ++i) {
        if (i < sk) {
            out_ids[i] = r2o[dists[i].id];
            if (out_dists) out_dists[i] = dists[i].v;
        } else {
            out_ids[i] = -1;
            if (out_dists) out_dists[i] = FLT_MAX;
        }
    }
    ret = nc;
done:
    free(qs);
    free(cd);
    free(visited);
    free(cand);
    free(dots);
    free(bd);
    free(pert);
    free(dists);
    return ret;
}

/* Per-dimension SQ8 training and encoding (lsh_index_optimized.cpp:187-214): scale = range/255,
 * offset = min (1 and 0 when the range is <= 1e-8); code = clamp(round((x - offset)/scale)),
 * round-half-away-from-zero as std::round. Under -ffast-math the compiled reference turns the
 * division by the constant 255 into a multiplication by its float reciprocal; the division by
 * scale stays a true division (both pinned by test against the reference's exported state). */
void orc_sq8_train(const float *x, int64_t n, int dim, float *scale, float *offset) {
    for (int d = 0; d < dim; ++d) {
        float mn = FLT_MAX, mx = -FLT_MAX;
        for (int64_t i = 0; i < n; ++i) {
            float v = x[i * dim + d];
            if (v < mn) mn = v;
            if (v > mx) mx = v;
        }
        if (mx - mn > 1e-8f) {
            scale[d] = (mx - mn) * (1.0f / 255.0f);
            offset[d] = mn;
        } else {
            scale[d] = 1.0f;
            offset[d] = 0.0f;
        }
    }
}

void orc_sq8_encode(const float *x, int64_t n, int dim, const float *scale, const float *offset, uint8_t *codes) {
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < dim; ++d) {
            int qv = (int)roundf((x[i * dim + d] - offset[d]) / scale[d]);
            codes[i * dim + d] = (uint8_t)(qv < 0 ? 0 : (qv > 255 ? 255 : qv));
        }
}

/* ---------------------------------------------------------------------------------------------
 * The GPU quantized-filter contestant (competitors/gpu_filter/src/gpu_filter.cu), restated.
 * Its host code is compiled by nvcc with -O3 and no -ffast-math (Dockerfile:17-19), so divisions
 * stay true divisions and the host re-rank's `acc += v * v` is an unfused multiply and add; its
 * device key is an explicit fmaf chain (:57-60).
 * --------------------------------------------------------------------------------------------- */

/* Per-dimension SQ8 (gpu_filter.cu:100-117): min / max as std::min / std::max keep them, scale =
 * (max - min) / 255 (a true division) when the range is > 1e-8, else 1; offset = min either way. */
void orc_gf_train(const float *x, int64_t n, int dim, float *scale, float *offset) {
    for (int d = 0; d < dim; ++d) {
        float mn = 3.4e38f, mx = -3.4e38f;
        for (int64_t i = 0; i < n; ++i) {
            const float v = x[i * dim + d];
            mn = (v < mn) ? v : mn;
            mx = (mx < v) ? v : mx;
        }
        scale[d] = (mx - mn > 1e-8f) ? (mx - mn) / 255.0f : 1.0f;
        offset[d] = mn;
    }
}

/* code = clamp(lrintf((x - offset) / scale), 0, 255) (gpu_filter.cu:119-127), row-major [n, dim]. */
void orc_gf_encode(const float *x, int64_t n, int dim, const float *scale, const float *offset, uint8_t *codes) {
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < dim; ++d) {
            const int qv = (int)lrintf((x[i * dim + d] - offset[d]) / scale[d]);
            codes[i * dim + d] = (uint8_t)(qv < 0 ? 0 : (qv > 255 ? 255 : qv));
        }
}

typedef struct {
    float key;
    int32_t id;
} gf_pair_t;

static int cmp_gf_pair(const void *x, const void *y) {
    const gf_pair_t *a = (const gf_pair_t *)x, *b = (const gf_pair_t *)y;
    if (a->key < b->key) return -1;
    if (b->key < a->key) return 1;
    return (a->id > b->id) - (a->id < b->id);
}

/* gf_query (gpu_filter.cu:135-176): r raised to k and capped at n; every row's key
 * sum_d fmaf(code, scale, -(q - offset))^2 by an fmaf chain in dimension order (:52-63); the first r
 * rows of the stable ascending sort by key (:155-157), i.e. by (key, row); their FP32 squared
 * distances v = x - q, acc += v * v (:163-171); the best min(k, r) by (distance, id) (:173-175).
 * Returns min(k, r); adds r to *ndist. */
int orc_gf_query(const float *x, const uint8_t *codes, int64_t n, int dim, const float *scale,
                 const float *offset, const float *q, int k, int r, int64_t *out_ids, int64_t *ndist) {
    if (r < k) r = k;
    if (r > n) r = (int)n;
    float *qshift = (float *)malloc(sizeof(float) * (size_t)dim);
    gf_pair_t *keys = (gf_pair_t *)malloc(sizeof(gf_pair_t) * (size_t)(n > 0 ? n : 1));
    gf_pair_t *exact = (gf_pair_t *)malloc(sizeof(gf_pair_t) * (size_t)(r > 0 ? r : 1));
    for (int d = 0; d < dim; ++d) qshift[d] = q[d] - offset[d];
    for (int64_t i = 0; i < n; ++i) {
        float acc = 0.0f;
        for (int d = 0; d < dim; ++d) {
            const float v = fmaf((float)codes[i * dim + d], scale[d], -qshift[d]);
            acc = fmaf(v, v, acc);
        }
        keys[i].key = acc;
        keys[i].id = (int32_t)i;
    }
    qsort(keys, (size_t)n, sizeof(gf_pair_t), cmp_gf_pair);
    for (int j = 0; j < r; ++j) {
        const float *p = x + (int64_t)keys[j].id * dim;
        float acc = 0.0f;
        for (int d = 0; d < dim; ++d) {
            const float v = p[d] - q[d];
            acc += v * v;
        }
        exact[j].key = acc;
        exact[j].id = keys[j].id;
    }
    qsort(exact, (size_t)r, sizeof(gf_pair_t), cmp_gf_pair);
    const int out_k = k < r ? k : r;
    for (int j = 0; j < out_k; ++j) out_ids[j] = exact[j].id;
    if (ndist) *ndist += r;
    free(qshift);
    free(keys);
    free(exact);
    return out_k;
}

// C ABI of the IVF-SQ8 index: the B200 form of ivf_lsh_cpp.LSHIndex
// (competitors/ivf_lsh/src/lsh_index_optimized.cpp:124-667) for n_tables = 1, n_bits = 0.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <mutex>
#include <numeric>
#include <random>
#include <thread>
#include <vector>

#include "common.cuh"
#include "flat_scan.cuh"
#include "ivf.cuh"
#include "ivf_batched.cuh"
#include "ivf_lsh.cuh"
#include "radix_select.cuh"
#include "refmath.cuh"
#include "runtime.cuh"
#include "tc_gemm.cuh"
#include "tc_search.cuh"

using namespace annb;

struct ann_ivf {
    int device = 0;
    int64_t n = 0;
    int dim = 0, dpad = 0, dpad8 = 0, C = 0;
    float* centroids = nullptr;   // [C, dpad]
    float* original = nullptr;    // [n, dpad]
    uint8_t* codes = nullptr;     // [n, dpad8]
    float* scale = nullptr;       // [dpad]
    float* offset = nullptr;      // [dpad]
    int32_t* r2o = nullptr;       // [n]
    int64_t* list_off = nullptr;  // [C + 1]
    unsigned long long* d_ndist = nullptr;
    int* d_err = nullptr;             // set by a kernel whose bounded wait gave up
    std::vector<int64_t> h_list_off;
    std::vector<int64_t> sizes_desc;  // list sizes, largest first (bounds for planning)
    ann_workspace ws;
    StageProfiler prof;  // 0: coarse ranking, 1: plan, 2: SQ8 pass (+ merge), 3: re-rank
    // LSH bucket tables (n_bits > 0, or several tables); T = 1, B = 0 is the plain inverted-list index
    int T = 1, B = 0;
    float* proj = nullptr;        // [T * B, dpad]
    float* projT = nullptr;       // [dim, T * B]
    float* lsh_mean = nullptr;    // [dpad]
    int64_t* tab_off = nullptr;   // [T * C * 2^B + 1]
    int32_t* tab_ids = nullptr;   // [T * n]
    bool lsh() const { return tab_off != nullptr && (B > 0 || T > 1); }
    LshView lsh_view() const { return LshView{T, B, proj, projT, lsh_mean, tab_off, tab_ids}; }
    __nv_bfloat16* base_bf16 = nullptr;  // [n, kpad] BF16 operand form of the list-ordered rows (tensor-core form)
    __nv_bfloat16* cent_bf16 = nullptr;  // [C, kpad] BF16 operand form of the centroids
    float2* sq8_fac = nullptr;           // [n] (1, reconstructed |x|^2) of the SQ8 rows (codes on the tensor cores)
    int kpad = 0;
    float cent_norm_max = 0.f;           // the largest centroid norm (the coarse ranking's key error bound)
    std::mutex tc_mu;
    int64_t query_count = 0;
    // query options (ann_ivf_set_option)
    int sample_div = 8;             // the sampled bars score the first ceil(size / sample_div) rows of a list
    int sampled_min_queries = 256;  // batches from this size take the sampled tensor-core path

    IvfView view() const {
        IvfView v;
        v.n = n;
        v.dim = dim;
        v.dpad = dpad;
        v.dpad8 = dpad8;
        v.C = C;
        v.centroids = centroids;
        v.original = original;
        v.codes = codes;
        v.scale = scale;
        v.offset = offset;
        v.r2o = r2o;
        v.list_off = list_off;
        return v;
    }
};

static void ivf_free_state(ann_ivf* h) {
    for (void* p : {(void*)h->centroids, (void*)h->original, (void*)h->codes, (void*)h->scale, (void*)h->offset,
                    (void*)h->r2o, (void*)h->list_off, (void*)h->base_bf16, (void*)h->cent_bf16, (void*)h->proj,
                    (void*)h->projT, (void*)h->lsh_mean, (void*)h->tab_off, (void*)h->tab_ids, (void*)h->sq8_fac})
        if (p) cudaFree(p);
    h->base_bf16 = nullptr;
    h->cent_bf16 = nullptr;
    h->cent_norm_max = 0.f;
    h->sq8_fac = nullptr;
    h->proj = h->projT = h->lsh_mean = nullptr;
    h->tab_off = nullptr;
    h->tab_ids = nullptr;
    h->T = 1;
    h->B = 0;
    h->kpad = 0;
    h->centroids = nullptr;
    h->original = nullptr;
    h->codes = nullptr;
    h->scale = h->offset = nullptr;
    h->r2o = nullptr;
    h->list_off = nullptr;
    h->n = 0;
}

template <typename T>
static int dmalloc(T** p, size_t count) {
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * std::max<size_t>(count, 1));
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        set_error("cannot allocate %zu bytes of device memory (%s)", sizeof(T) * count, cudaGetErrorString(e));
        return ANN_ERR_NOMEM;
    }
    return ANN_OK;
}

// Host-side list bookkeeping after the device list offsets are final.
static int ivf_finish_lists(ann_ivf* h, cudaStream_t st) {
    h->h_list_off.resize(h->C + 1);
    ANN_CUDA_TRY(cudaMemcpyAsync(h->h_list_off.data(), h->list_off, sizeof(int64_t) * (h->C + 1),
                                 cudaMemcpyDeviceToHost, st));
    ANN_CUDA_TRY(cudaStreamSynchronize(st));
    h->sizes_desc.resize(h->C);
    for (int c = 0; c < h->C; ++c) h->sizes_desc[c] = h->h_list_off[c + 1] - h->h_list_off[c];
    std::sort(h->sizes_desc.begin(), h->sizes_desc.end(), std::greater<int64_t>());
    if (!h->d_ndist) {
        int rc = dmalloc(&h->d_ndist, 1);
        if (rc) return rc;
        ANN_CUDA_TRY(cudaMemsetAsync(h->d_ndist, 0, sizeof(unsigned long long), st));
    }
    if (!h->d_err) {
        int rc = dmalloc(&h->d_err, 1);
        if (rc) return rc;
        ANN_CUDA_TRY(cudaMemsetAsync(h->d_err, 0, sizeof(int), st));
    }
    return ANN_OK;
}

// Nearest centroid of every row (exact FP32 scan, k = 1): assign[i] in [0, C).
// Nearest centroid of every row, as the reference's kmeans_assign_worker picks it (first minimum of
// compute_l2_distance, lsh_index_optimized.cpp:32-47): the exact FP32 scan's two nearest per row,
// certified by the rounding bound of both arithmetics, the near-ties redone in the reference's.
static int assign_rows(const float* x, int64_t n, int dim, int dpad, const float* cent, int C, int32_t* assign,
                       ann_workspace* ws, cudaStream_t st) {
    const int bq = 32;
    const int nq_chunk = 1 << 20;
    // relative error of a computed squared distance: the scan's FMA chain over dpad terms, and the
    // reference's 16 lane sums of dim/16 terms, folds and remainder; margin covers both with room
    const double u = 1.0 / 16777216.0;
    const double e_fast = (dpad + 4) * u, e_ref = (dim / 16 + 24) * u;
    const float margin = (float)(1.0 + 4.0 * (e_fast + e_ref));
    const int k = C >= 2 ? 2 : 1;
    for (int64_t r0 = 0; r0 < n; r0 += nq_chunk) {
        const int nq = (int)std::min<int64_t>(nq_chunk, n - r0);
        Sizer sz;
        sz.take<float>((size_t)nq * k);
        sz.take<int>((size_t)nq * k);
        sz.take<float>((size_t)nq * 2);
        sz.take<int>((size_t)nq * 2);
        sz.take<int32_t>((size_t)nq);
        sz.take<int>(1);
        int rc = ws_reserve_device(ws, sz.bytes());
        if (rc) return rc;
        Carver cv(ws->dev);
        float* sk = cv.take<float>((size_t)nq * k);
        int* si = cv.take<int>((size_t)nq * k);
        float* k2 = cv.take<float>((size_t)nq * 2);
        int* i2 = cv.take<int>((size_t)nq * 2);
        int32_t* amb = cv.take<int32_t>((size_t)nq);
        int* amb_count = cv.take<int>(1);
        if (k == 1) {  // one centroid: every row is in list 0
            ANN_CUDA_TRY(cudaMemsetAsync(assign + r0, 0, sizeof(int32_t) * nq, st));
            continue;
        }
        FlatScanArgs a{cent, C, dpad, x + r0 * dpad, nq, ANN_METRIC_L2, k, (int64_t)C, 1, sk, si};
        rc = launch_flat_scan(a, bq, st);
        if (rc) return rc;
        MergeArgs m{sk, si, nq, 1, k, 2, 0, nullptr, nullptr};
        m.out_id32 = i2;
        m.out_key32 = k2;
        rc = launch_merge_splits(m, st);
        if (rc) return rc;
        ANN_CUDA_TRY(cudaMemsetAsync(amb_count, 0, sizeof(int), st));
        rc = launch_kmeans_certify(k2, i2, nq, margin, assign + r0, amb, amb_count, st);
        if (rc) return rc;
        rc = launch_kmeans_ref_assign(x + r0 * dpad, dpad, dim, cent, dpad, C, amb, amb_count, assign + r0, st);
        if (rc) return rc;
    }
    return ANN_OK;
}

extern "C" {

int ann_ivf_create(ann_ivf** out, int device) {
    clear_error();
    ANN_CHECK_ARG(out != nullptr, "ann_ivf_create: out is NULL");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("no CUDA device visible (%s)", e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
        return ANN_ERR_CUDA;
    }
    ANN_CHECK_ARG(device >= 0 && device < ndev, "ann_ivf_create: device %d not in [0, %d)", device, ndev);
    ann_ivf* h = new (std::nothrow) ann_ivf();
    if (!h) {
        set_error("ann_ivf_create: out of host memory");
        return ANN_ERR_NOMEM;
    }
    h->device = device;
    h->ws.device = device;
    *out = h;
    return ANN_OK;
}

int ann_ivf_destroy(ann_ivf* h) {
    if (!h) return ANN_OK;
    {
        DeviceGuard g(h->device);
        ivf_free_state(h);
        if (h->d_ndist) cudaFree(h->d_ndist);
        if (h->d_err) cudaFree(h->d_err);
        if (h->ws.dev) cudaFree(h->ws.dev);
        if (h->ws.big) cudaFree(h->ws.big);
        if (h->ws.pinned) cudaFreeHost(h->ws.pinned);
        h->ws.pinned = nullptr;
        h->ws.dev = nullptr;
        h->ws.big = nullptr;
    }
    delete h;
    return ANN_OK;
}

int ann_ivf_fit(ann_ivf* h, const float* data, int64_t n, int32_t dim, int64_t ld, int32_t n_clusters,
                const float* centroids, const int32_t* assign, int32_t kmeans_iters, int32_t num_threads, int32_t mem,
                void* stream) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr, "ann_ivf_fit: null index");
    ANN_CHECK_ARG(n >= 1 && dim >= 1 && data, "ann_ivf_fit: need a non-empty 2-D array");
    ANN_CHECK_ARG(n < INT32_MAX, "ann_ivf_fit: n=%lld exceeds 32-bit ids", (long long)n);
    ANN_CHECK_ARG(ld >= dim, "ann_ivf_fit: row stride < dim");
    ANN_CHECK_ARG(n_clusters >= 1, "ann_ivf_fit: n_clusters=%d < 1", n_clusters);
    ANN_CHECK_ARG(kmeans_iters >= 0, "ann_ivf_fit: kmeans_iters < 0");
    DeviceGuard g(h->device);
    // the reference sizes its ThreadPool, and with it the k-means chunks, from hardware_concurrency() (:140)
    const int fit_threads = num_threads > 0 ? num_threads : (int)std::max(1u, std::thread::hardware_concurrency());
    cudaStream_t st = as_stream(stream);
    // the reference clamps too (:137); given centroids are kept as they are (lists may be empty)
    const int C = centroids ? n_clusters : (int)std::min<int64_t>(n_clusters, n);
    const int dpad = (int)ceil_div(dim, 32) * 32;
    const int dpad8 = (int)ceil_div(dim, 128) * 128;  // 16 threads x (multiple of 8) code bytes per row
    ANN_CUDA_TRY(cudaDeviceSynchronize());
    ivf_free_state(h);
    const cudaMemcpyKind kind = mem == ANN_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;

    float* X = nullptr;  // [n, dpad] input rows
    int32_t* a_raw = nullptr;
    int32_t* a_sorted = nullptr;
    int32_t* idx = nullptr;
    int32_t* order = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    float* mn = nullptr;
    float* mx = nullptr;
    int32_t* seed_rows = nullptr;
    int rc = ANN_OK;
#define FIT_TRY(x)          \
    do {                    \
        rc = (x);           \
        if (rc) goto fail;  \
    } while (0)
#define FIT_CUDA(x)                                                                                      \
    do {                                                                                                 \
        cudaError_t _e = (x);                                                                            \
        if (_e != cudaSuccess) {                                                                         \
            set_error("CUDA error %s at %s:%d", cudaGetErrorString(_e), __FILE__, __LINE__);             \
            rc = ANN_ERR_CUDA;                                                                           \
            goto fail;                                                                                   \
        }                                                                                                \
    } while (0)
    {
        FIT_TRY(dmalloc(&X, (size_t)n * dpad));
        FIT_TRY(dmalloc(&h->centroids, (size_t)C * dpad));
        FIT_TRY(dmalloc(&a_raw, n));
        FIT_TRY(dmalloc(&a_sorted, n));
        FIT_TRY(dmalloc(&idx, n));
        FIT_TRY(dmalloc(&order, n));
        FIT_TRY(dmalloc(&h->list_off, C + 1));
        FIT_CUDA(cudaMemsetAsync(X, 0, sizeof(float) * (size_t)n * dpad, st));
        FIT_CUDA(cudaMemcpy2DAsync(X, sizeof(float) * dpad, data, sizeof(float) * ld, sizeof(float) * dim, n, kind, st));
        FIT_CUDA(cudaMemsetAsync(h->centroids, 0, sizeof(float) * (size_t)C * dpad, st));
        // rand_indices of run_kmeans: std::shuffle(iota(n), std::mt19937(1337)) (:553-555), the same
        // libstdc++ algorithm the reference runs. Row rand_indices[c] seeds list c (:557-561); row
        // rand_indices[(c * 37) % n] reseeds it whenever it ends an update empty (:608-613).
        {
            std::vector<int32_t> perm((size_t)n);
            std::iota(perm.begin(), perm.end(), 0);
            std::shuffle(perm.begin(), perm.end(), std::mt19937(1337));
            std::vector<int32_t> seeds(2 * (size_t)C);
            for (int c = 0; c < C; ++c) {
                seeds[c] = perm[(size_t)(c % n)];
                seeds[(size_t)C + c] = perm[(size_t)(((int64_t)c * 37) % n)];
            }
            FIT_TRY(dmalloc(&seed_rows, 2 * (size_t)C));
            FIT_CUDA(cudaMemcpyAsync(seed_rows, seeds.data(), sizeof(int32_t) * 2 * C, cudaMemcpyHostToDevice, st));
            FIT_CUDA(cudaStreamSynchronize(st));
        }
        if (centroids) {
            FIT_CUDA(cudaMemcpy2DAsync(h->centroids, sizeof(float) * dpad, centroids, sizeof(float) * dim,
                                       sizeof(float) * dim, C, kind, st));
        } else {
            FIT_TRY(launch_gather_rows(X, C, dpad, seed_rows, h->centroids, dpad, st));
        }
        // iota for the sort values
        {
            std::vector<int32_t> io((size_t)n);
            for (int64_t i = 0; i < n; ++i) io[i] = (int32_t)i;
            FIT_CUDA(cudaMemcpyAsync(idx, io.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
            FIT_CUDA(cudaStreamSynchronize(st));
        }
        FIT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, a_raw, a_sorted, idx, order, (int)n, 0, 32, st));
        FIT_CUDA(cudaMalloc(&tmp, tmp_bytes));
        const bool given_assign = assign != nullptr;
        const int iters = (centroids || given_assign) ? 0 : kmeans_iters;
        for (int it = 0; it < iters; ++it) {
            FIT_TRY(assign_rows(X, n, dim, dpad, h->centroids, C, a_raw, &h->ws, st));
            FIT_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, a_raw, a_sorted, idx, order, (int)n, 0, 32, st));
            FIT_TRY(launch_list_offsets(a_sorted, n, C, h->list_off, st));
            FIT_TRY(launch_kmeans_update(X, dpad, dim, order, h->list_off, C, h->centroids, dpad, seed_rows + C, n,
                                         fit_threads, st));
        }
        // the lists: given assignment, else nearest to the current centroids (the last k-means
        // assignment when iterating, as the reference's lists come from its last assign step)
        if (given_assign) {
            FIT_CUDA(cudaMemcpyAsync(a_raw, assign, sizeof(int32_t) * n, kind, st));
        } else if (iters == 0) {
            FIT_TRY(assign_rows(X, n, dim, dpad, h->centroids, C, a_raw, &h->ws, st));
        }
        FIT_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, a_raw, a_sorted, idx, order, (int)n, 0, 32, st));
        FIT_TRY(launch_list_offsets(a_sorted, n, C, h->list_off, st));
        // reorder rows, SQ8 train / encode over the reordered rows
        FIT_TRY(dmalloc(&h->original, (size_t)n * dpad));
        FIT_TRY(dmalloc(&h->codes, (size_t)n * dpad8));
        FIT_TRY(dmalloc(&h->scale, dpad));
        FIT_TRY(dmalloc(&h->offset, dpad));
        FIT_TRY(dmalloc(&mn, dpad));
        FIT_TRY(dmalloc(&mx, dpad));
        FIT_TRY(launch_gather_rows(X, n, dpad, order, h->original, dpad, st));
        FIT_TRY(launch_sq8_minmax(h->original, n, dim, dpad, mn, mx, st));
        FIT_TRY(launch_sq8_params(mn, mx, dim, dpad, h->scale, h->offset, st));
        FIT_TRY(launch_sq8_encode(h->original, n, dim, dpad, h->scale, h->offset, h->codes, dpad8, st));
        h->r2o = order;
        order = nullptr;
        h->n = n;
        h->dim = dim;
        h->dpad = dpad;
        h->dpad8 = dpad8;
        h->C = C;
        FIT_TRY(ivf_finish_lists(h, st));
        FIT_CUDA(cudaStreamSynchronize(st));
    }
fail:
    for (void* p : {(void*)X, (void*)a_raw, (void*)a_sorted, (void*)idx, (void*)order, tmp, (void*)mn, (void*)mx,
                    (void*)seed_rows})
        if (p) cudaFree(p);
    if (rc) ivf_free_state(h);
    return rc;
#undef FIT_TRY
#undef FIT_CUDA
}

int ann_ivf_import(ann_ivf* h, int64_t n, int32_t dim, int32_t n_clusters, const float* centroids,
                   const float* original, const uint8_t* codes, const float* scale, const float* offset,
                   const int32_t* r2o, const int64_t* list_offsets) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr, "ann_ivf_import: null index");
    ANN_CHECK_ARG(n >= 1 && dim >= 1 && n_clusters >= 1, "ann_ivf_import: empty state");
    ANN_CHECK_ARG(centroids && original && codes && scale && offset && r2o && list_offsets,
                  "ann_ivf_import: null array");
    ANN_CHECK_ARG(list_offsets[0] == 0 && list_offsets[n_clusters] == n, "ann_ivf_import: list offsets do not span n");
    for (int c = 0; c < n_clusters; ++c)
        ANN_CHECK_ARG(list_offsets[c + 1] >= list_offsets[c], "ann_ivf_import: list offsets not sorted");
    DeviceGuard g(h->device);
    ANN_CUDA_TRY(cudaDeviceSynchronize());
    ivf_free_state(h);
    const int dpad = (int)ceil_div(dim, 32) * 32;
    const int dpad8 = (int)ceil_div(dim, 128) * 128;
    int rc = ANN_OK;
    if ((rc = dmalloc(&h->centroids, (size_t)n_clusters * dpad)) || (rc = dmalloc(&h->original, (size_t)n * dpad)) ||
        (rc = dmalloc(&h->codes, (size_t)n * dpad8)) || (rc = dmalloc(&h->scale, dpad)) ||
        (rc = dmalloc(&h->offset, dpad)) || (rc = dmalloc(&h->r2o, n)) || (rc = dmalloc(&h->list_off, n_clusters + 1))) {
        ivf_free_state(h);
        return rc;
    }
    cudaStream_t st = nullptr;
    ANN_CUDA_TRY(cudaMemset(h->centroids, 0, sizeof(float) * (size_t)n_clusters * dpad));
    ANN_CUDA_TRY(cudaMemset(h->original, 0, sizeof(float) * (size_t)n * dpad));
    ANN_CUDA_TRY(cudaMemset(h->codes, 0, (size_t)n * dpad8));
    ANN_CUDA_TRY(cudaMemset(h->scale, 0, sizeof(float) * dpad));
    ANN_CUDA_TRY(cudaMemset(h->offset, 0, sizeof(float) * dpad));
    ANN_CUDA_TRY(cudaMemcpy2D(h->centroids, sizeof(float) * dpad, centroids, sizeof(float) * dim, sizeof(float) * dim,
                              n_clusters, cudaMemcpyHostToDevice));
    ANN_CUDA_TRY(cudaMemcpy2D(h->original, sizeof(float) * dpad, original, sizeof(float) * dim, sizeof(float) * dim, n,
                              cudaMemcpyHostToDevice));
    ANN_CUDA_TRY(cudaMemcpy2D(h->codes, dpad8, codes, dim, dim, n, cudaMemcpyHostToDevice));
    ANN_CUDA_TRY(cudaMemcpy(h->scale, scale, sizeof(float) * dim, cudaMemcpyHostToDevice));
    ANN_CUDA_TRY(cudaMemcpy(h->offset, offset, sizeof(float) * dim, cudaMemcpyHostToDevice));
    ANN_CUDA_TRY(cudaMemcpy(h->r2o, r2o, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
    ANN_CUDA_TRY(cudaMemcpy(h->list_off, list_offsets, sizeof(int64_t) * (n_clusters + 1), cudaMemcpyHostToDevice));
    h->n = n;
    h->dim = dim;
    h->dpad = dpad;
    h->dpad8 = dpad8;
    h->C = n_clusters;
    return ivf_finish_lists(h, st);
}

int ann_ivf_export(ann_ivf* h, float* centroids, float* original, uint8_t* codes, float* scale, float* offset,
                   int32_t* r2o, int64_t* list_offsets) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr, "ann_ivf_export: null index");
    if (h->n == 0) {
        set_error("index not fitted");
        return ANN_ERR_STATE;
    }
    DeviceGuard g(h->device);
    const int dim = h->dim;
    if (centroids)
        ANN_CUDA_TRY(cudaMemcpy2D(centroids, sizeof(float) * dim, h->centroids, sizeof(float) * h->dpad,
                                  sizeof(float) * dim, h->C, cudaMemcpyDeviceToHost));
    if (original)
        ANN_CUDA_TRY(cudaMemcpy2D(original, sizeof(float) * dim, h->original, sizeof(float) * h->dpad,
                                  sizeof(float) * dim, h->n, cudaMemcpyDeviceToHost));
    if (codes) ANN_CUDA_TRY(cudaMemcpy2D(codes, dim, h->codes, h->dpad8, dim, h->n, cudaMemcpyDeviceToHost));
    if (scale) ANN_CUDA_TRY(cudaMemcpy(scale, h->scale, sizeof(float) * dim, cudaMemcpyDeviceToHost));
    if (offset) ANN_CUDA_TRY(cudaMemcpy(offset, h->offset, sizeof(float) * dim, cudaMemcpyDeviceToHost));
    if (r2o) ANN_CUDA_TRY(cudaMemcpy(r2o, h->r2o, sizeof(int32_t) * h->n, cudaMemcpyDeviceToHost));
    if (list_offsets)
        ANN_CUDA_TRY(cudaMemcpy(list_offsets, h->list_off, sizeof(int64_t) * (h->C + 1), cudaMemcpyDeviceToHost));
    return ANN_OK;
}

int ann_ivf_info(const ann_ivf* h, int64_t* out4) {
    ANN_CHECK_ARG(h != nullptr && out4 != nullptr, "ann_ivf_info: null argument");
    out4[0] = h->n;
    out4[1] = h->dim;
    out4[2] = h->C;
    out4[3] = h->sizes_desc.empty() ? 0 : h->sizes_desc[0];
    return ANN_OK;
}

static void lsh_free(ann_ivf* h) {
    for (void* p : {(void*)h->proj, (void*)h->projT, (void*)h->lsh_mean, (void*)h->tab_off, (void*)h->tab_ids})
        if (p) cudaFree(p);
    h->proj = h->projT = h->lsh_mean = nullptr;
    h->tab_off = nullptr;
    h->tab_ids = nullptr;
    h->T = 1;
    h->B = 0;
}

static int lsh_alloc(ann_ivf* h, int T, int B) {
    const int64_t nbk = (int64_t)T * h->C * ((int64_t)1 << B);
    cudaError_t e = cudaSuccess;
    e = cudaMalloc(&h->proj, sizeof(float) * (size_t)std::max(1, T * B) * h->dpad);
    if (e == cudaSuccess) e = cudaMalloc(&h->projT, sizeof(float) * (size_t)std::max(1, T * B) * h->dim);
    if (e == cudaSuccess) e = cudaMalloc(&h->lsh_mean, sizeof(float) * h->dpad);
    if (e == cudaSuccess) e = cudaMalloc(&h->tab_off, sizeof(int64_t) * (size_t)(nbk + 1));
    if (e == cudaSuccess) e = cudaMalloc(&h->tab_ids, sizeof(int32_t) * (size_t)std::max<int64_t>(1, T * h->n));
    if (e != cudaSuccess) {
        cudaGetLastError();
        lsh_free(h);
        set_error("LSH tables: cannot allocate (%s)", cudaGetErrorString(e));
        return ANN_ERR_NOMEM;
    }
    h->T = T;
    h->B = B;
    return ANN_OK;
}

int ann_ivf_import_tables(ann_ivf* h, int32_t n_tables, int32_t n_bits, const float* projections, const float* mean,
                          const int64_t* table_offsets, const int32_t* table_ids) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr && h->n > 0, "ann_ivf_import_tables: index not imported");
    ANN_CHECK_ARG(n_tables >= 1 && n_tables <= 64 && n_bits >= 0 && n_bits <= 16,
                  "ann_ivf_import_tables: %d tables of %d bits", n_tables, n_bits);
    ANN_CHECK_ARG(table_offsets && table_ids && mean && (n_bits == 0 || projections), "ann_ivf_import_tables: null");
    {
        // every bucket (t, c, sig) a range of table t's n ids, in order, each a row of list c
        const int64_t nbl = (int64_t)1 << n_bits;
        ANN_CHECK_ARG(table_offsets[0] == 0, "ann_ivf_import_tables: table offsets do not start at 0");
        for (int t = 0; t < n_tables; ++t)
            for (int64_t c = 0; c < h->C; ++c) {
                const int64_t lo = h->h_list_off[c], hi = h->h_list_off[c + 1];
                for (int64_t sg = 0; sg < nbl; ++sg) {
                    const int64_t bkt = ((int64_t)t * h->C + c) * nbl + sg;
                    const int64_t b0 = table_offsets[bkt], b1 = table_offsets[bkt + 1];
                    ANN_CHECK_ARG(b0 <= b1 && b0 >= (int64_t)t * h->n && b1 <= (int64_t)(t + 1) * h->n,
                                  "ann_ivf_import_tables: bucket %lld has offsets [%lld, %lld)", (long long)bkt,
                                  (long long)b0, (long long)b1);
                    for (int64_t j = b0; j < b1; ++j)
                        ANN_CHECK_ARG(table_ids[j] >= lo && table_ids[j] < hi,
                                      "ann_ivf_import_tables: bucket %lld holds row %d outside its list",
                                      (long long)bkt, table_ids[j]);
                }
            }
        ANN_CHECK_ARG(table_offsets[(int64_t)n_tables * h->C * nbl] == (int64_t)n_tables * h->n,
                      "ann_ivf_import_tables: table offsets do not span n per table");
    }
    DeviceGuard g(h->device);
    lsh_free(h);
    int rc = lsh_alloc(h, n_tables, n_bits);
    if (rc) return rc;
    const int dim = h->dim;
    const int64_t nbk = (int64_t)n_tables * h->C * ((int64_t)1 << n_bits);
    ANN_CUDA_TRY(cudaMemset(h->proj, 0, sizeof(float) * (size_t)std::max(1, n_tables * n_bits) * h->dpad));
    ANN_CUDA_TRY(cudaMemset(h->lsh_mean, 0, sizeof(float) * h->dpad));
    if (n_bits > 0)
        ANN_CUDA_TRY(cudaMemcpy2D(h->proj, sizeof(float) * h->dpad, projections, sizeof(float) * dim,
                                  sizeof(float) * dim, (size_t)n_tables * n_bits, cudaMemcpyHostToDevice));
    ANN_CUDA_TRY(cudaMemcpy(h->lsh_mean, mean, sizeof(float) * dim, cudaMemcpyHostToDevice));
    ANN_CUDA_TRY(cudaMemcpy(h->tab_off, table_offsets, sizeof(int64_t) * (size_t)(nbk + 1), cudaMemcpyHostToDevice));
    ANN_CUDA_TRY(cudaMemcpy(h->tab_ids, table_ids, sizeof(int32_t) * (size_t)n_tables * h->n, cudaMemcpyHostToDevice));
    if ((rc = launch_lsh_transpose(h->proj, n_tables * n_bits, dim, h->dpad, h->projT, nullptr))) return rc;
    ANN_CUDA_TRY(cudaDeviceSynchronize());
    return ANN_OK;
}

int ann_ivf_export_tables(ann_ivf* h, int32_t* out2, float* projections, float* mean, int64_t* table_offsets,
                          int32_t* table_ids) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr, "ann_ivf_export_tables: null index");
    DeviceGuard g(h->device);
    if (out2) {
        out2[0] = h->tab_off ? h->T : 1;
        out2[1] = h->tab_off ? h->B : 0;
    }
    if (!h->tab_off) return ANN_OK;
    const int dim = h->dim;
    const int64_t nbk = (int64_t)h->T * h->C * ((int64_t)1 << h->B);
    if (projections && h->B > 0)
        ANN_CUDA_TRY(cudaMemcpy2D(projections, sizeof(float) * dim, h->proj, sizeof(float) * h->dpad,
                                  sizeof(float) * dim, (size_t)h->T * h->B, cudaMemcpyDeviceToHost));
    if (mean) ANN_CUDA_TRY(cudaMemcpy(mean, h->lsh_mean, sizeof(float) * dim, cudaMemcpyDeviceToHost));
    if (table_offsets)
        ANN_CUDA_TRY(cudaMemcpy(table_offsets, h->tab_off, sizeof(int64_t) * (size_t)(nbk + 1), cudaMemcpyDeviceToHost));
    if (table_ids)
        ANN_CUDA_TRY(cudaMemcpy(table_ids, h->tab_ids, sizeof(int32_t) * (size_t)h->T * h->n, cudaMemcpyDeviceToHost));
    return ANN_OK;
}

int ann_ivf_build_tables(ann_ivf* h, int32_t n_tables, int32_t n_bits, void* stream) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr && h->n > 0, "ann_ivf_build_tables: index not fitted");
    ANN_CHECK_ARG(n_tables >= 1 && n_tables <= 64 && n_bits >= 0 && n_bits <= 16,
                  "ann_ivf_build_tables: %d tables of %d bits", n_tables, n_bits);
    DeviceGuard g(h->device);
    cudaStream_t st = as_stream(stream);
    lsh_free(h);
    int rc = lsh_alloc(h, n_tables, n_bits);
    if (rc) return rc;
    const int dim = h->dim, T = n_tables, B = n_bits;
    // projections: mt19937(42), N(0, 1) floats, row by row (:216-225); Gram-Schmidt within each table
    // when B <= dim (:228-257), in FP32 in the reference's loop order
    std::vector<float> proj((size_t)T * B * dim);
    {
        std::mt19937 gen(42);
        std::normal_distribution<float> dist(0.0f, 1.0f);
        for (auto& v : proj) v = dist(gen);
        if (B <= dim)
            for (int t = 0; t < T; ++t)
                for (int b = 0; b < B; ++b) {
                    float* pi = proj.data() + (size_t)(t * B + b) * dim;
                    for (int bp = 0; bp < b; ++bp) {
                        const float* pp = proj.data() + (size_t)(t * B + bp) * dim;
                        float dot = 0.f;
                        for (int d = 0; d < dim; ++d) dot += pi[d] * pp[d];
                        for (int d = 0; d < dim; ++d) pi[d] -= dot * pp[d];
                    }
                    float nrm = 0.f;
                    for (int d = 0; d < dim; ++d) nrm += pi[d] * pi[d];
                    nrm = std::sqrt(nrm);
                    if (nrm > 1e-8f)
                        for (int d = 0; d < dim; ++d) pi[d] /= nrm;
                }
    }
    ANN_CUDA_TRY(cudaMemsetAsync(h->proj, 0, sizeof(float) * (size_t)std::max(1, T * B) * h->dpad, st));
    if (B > 0)
        ANN_CUDA_TRY(cudaMemcpy2DAsync(h->proj, sizeof(float) * h->dpad, proj.data(), sizeof(float) * dim,
                                       sizeof(float) * dim, (size_t)T * B, cudaMemcpyHostToDevice, st));
    if ((rc = launch_lsh_transpose(h->proj, T * B, dim, h->dpad, h->projT, st))) return rc;
    if ((rc = launch_lsh_mean(h->original, h->n, dim, h->dpad, h->lsh_mean, st))) return rc;
    // bucket keys (list, signature) of every row per table, stably sorted: members ascend by row
    const int64_t n = h->n;
    const int nb = 1 << B;
    int32_t *keys = nullptr, *kout = nullptr, *vin = nullptr;
    void* tmp = nullptr;
    size_t tb = 0;
    int end_bit = 1;
    while (((int64_t)1 << end_bit) <= (int64_t)h->C * nb) ++end_bit;
    ANN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, (int32_t*)nullptr, (int32_t*)nullptr, (int32_t*)nullptr,
                                                 (int32_t*)nullptr, (int)n, 0, end_bit, st));
    cudaError_t e = cudaMalloc(&keys, sizeof(int32_t) * (size_t)T * n);
    if (e == cudaSuccess) e = cudaMalloc(&kout, sizeof(int32_t) * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&vin, sizeof(int32_t) * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tb);
    if (e != cudaSuccess) {
        cudaGetLastError();
        for (void* p : {(void*)keys, (void*)kout, (void*)vin, tmp})
            if (p) cudaFree(p);
        set_error("LSH build: cannot allocate scratch (%s)", cudaGetErrorString(e));
        return ANN_ERR_NOMEM;
    }
    rc = launch_lsh_row_keys(h->view(), h->lsh_view(), keys, st);
    if (!rc) rc = launch_iota(vin, n, st);
    for (int t = 0; t < T && !rc; ++t) {
        size_t tb2 = tb;
        cudaError_t e2 = cub::DeviceRadixSort::SortPairs(tmp, tb2, keys + (size_t)t * n, kout, vin,
                                                         h->tab_ids + (size_t)t * n, (int)n, 0, end_bit, st);
        if (e2 != cudaSuccess) {
            set_error("LSH build: sort failed (%s)", cudaGetErrorString(e2));
            rc = ANN_ERR_CUDA;
            break;
        }
        rc = launch_list_offsets(kout, n, h->C * nb, h->tab_off + (size_t)t * h->C * nb, st);
        if (!rc && t > 0) rc = launch_add_offset(h->tab_off + (size_t)t * h->C * nb, (int64_t)h->C * nb + 1,
                                                 (int64_t)t * n, st);
    }
    cudaError_t e3 = cudaStreamSynchronize(st);
    for (void* p : {(void*)keys, (void*)kout, (void*)vin, tmp}) cudaFree(p);
    if (rc) return rc;
    ANN_CUDA_TRY(e3);
    return ANN_OK;
}

}  // extern "C"

namespace {

// Exact-mode SQ8 pass: batches of at least kBatchedMinQueries queries run list-major (ivf_batched.cu),
// smaller ones query by query (ivf.cu).
constexpr int kBatchedMinQueries = 32;
constexpr int kQueryOrderMinBatch = 256;  // smaller batches have no shared candidates worth grouping
constexpr int kEveryRowMinSplit = 8;      // exact batches split fewer ways redo every-row queries apart

struct IvfQueryCfg {
    int k, npc, R, nsplit, num_threads, bqc, nsplit_c, ncp;
    int64_t max_c, ub, rps_c;
    bool ref, coarse_flat, batched, tc, lsh;
    bool i8;          // the tensor-core form over the SQ8 codes (int8 x uint8 MMA) instead of BF16 rows
    bool shard;       // ANN_QUERY_SHARD: streams short of k are not widened to every row
    bool fallback;    // a query's stream can fall short of k points and become every row
    bool lsh_keys;    // exact LSH batch: SQ8 keys of the whole streams, then selection
    int64_t ub_cand;  // longest explicit candidate stream (LSH buckets; a fallback to every row needs none)
    int n_probes;
    size_t sort_tmp, scan_tmp, bscratch;
};

// Operand forms of the tensor-core forms, built once: BF16 centroids (the coarse ranking of both), and the BF16
// list-ordered rows (ANN_MODE_TC) or the SQ8 rows' reconstructed norms (ANN_MODE_TC_SQ8, whose B operand is the
// codes themselves).
static int ivf_ensure_tc(ann_ivf* h, bool i8, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(h->tc_mu);
    const int kpad = tc_kpad(h->dim, ANN_METRIC_L2);
    int rc = ANN_OK;
    if (!h->cent_bf16) {
        __nv_bfloat16* cb = nullptr;
        if (cudaMalloc(&cb, sizeof(__nv_bfloat16) * (size_t)h->C * kpad) != cudaSuccess) {
            cudaGetLastError();
            set_error("tensor-core IVF: cannot allocate the BF16 centroids");
            return ANN_ERR_NOMEM;
        }
        if ((rc = launch_tc_operand(h->centroids, h->C, h->dim, h->dpad, cb, kpad, kTcBase, ANN_METRIC_L2, 0, st))) {
            cudaFree(cb);
            return rc;
        }
        ANN_CUDA_TRY(cudaStreamSynchronize(st));
        // the largest centroid norm, from a host copy of the (small) centroid table
        std::vector<float> hc((size_t)h->C * h->dpad);
        const cudaError_t ce = cudaMemcpy(hc.data(), h->centroids, sizeof(float) * hc.size(), cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) {
            cudaFree(cb);
            set_error("tensor-core IVF: %s", cudaGetErrorString(ce));
            return ANN_ERR_CUDA;
        }
        double mx = 0.0;
        for (int c = 0; c < h->C; ++c) {
            double s2 = 0.0;
            for (int d = 0; d < h->dim; ++d) s2 += (double)hc[(size_t)c * h->dpad + d] * hc[(size_t)c * h->dpad + d];
            mx = std::max(mx, s2);
        }
        h->cent_norm_max = (float)(std::sqrt(mx) * (1.0 + 1e-6));
        h->cent_bf16 = cb;
        h->kpad = kpad;
    }
    if (!i8 && !h->base_bf16) {
        __nv_bfloat16* b = nullptr;
        const cudaError_t e = cudaMalloc(&b, sizeof(__nv_bfloat16) * (size_t)h->n * kpad);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error("tensor-core IVF: cannot allocate the BF16 copy of the lists (%s)", cudaGetErrorString(e));
            return ANN_ERR_NOMEM;
        }
        if ((rc = launch_tc_operand(h->original, h->n, h->dim, h->dpad, b, kpad, kTcBase, ANN_METRIC_L2, 0, st))) {
            cudaFree(b);
            return rc;
        }
        ANN_CUDA_TRY(cudaStreamSynchronize(st));
        h->base_bf16 = b;
    }
    if (i8 && !h->sq8_fac) {
        float2* f = nullptr;
        if (cudaMalloc(&f, sizeof(float2) * (size_t)h->n) != cudaSuccess) {
            cudaGetLastError();
            set_error("tensor-core IVF: cannot allocate the SQ8 row norms");
            return ANN_ERR_NOMEM;
        }
        if ((rc = launch_tc_sq8_norms(h->codes, h->n, h->dim, h->dpad8, h->scale, f, st))) {
            cudaFree(f);
            return rc;
        }
        ANN_CUDA_TRY(cudaStreamSynchronize(st));
        h->sq8_fac = f;
    }
    return ANN_OK;
}

// Operand rows of the pairs: BF16 (kpad columns) or int8 weights (dpad8 bytes).
static int64_t tc_pair_row_bytes(const ann_ivf* h) {
    return std::max<int64_t>(2 * (int64_t)tc_kpad(h->dim, ANN_METRIC_L2), h->dpad8);
}

// Bytes of scratch one device-side query call of nq queries needs (mirrors the carving below).
static size_t ivf_scratch(const ann_ivf* h, const IvfQueryCfg& c, int nq) {
    Sizer sz;
    sz.take<int32_t>((size_t)nq * c.npc);
    sz.take<int64_t>((size_t)nq * c.npc);
    sz.take<int64_t>((size_t)nq * (c.npc + 1));
    sz.take<int32_t>((size_t)nq);
    sz.take<int64_t>((size_t)nq);
    if (c.coarse_flat) {
        sz.take<float>((size_t)nq * c.nsplit_c * c.npc);
        sz.take<int>((size_t)nq * c.nsplit_c * c.npc);
    } else {
        sz.take<float>((size_t)nq * h->C);
        sz.take<float>((size_t)nq * c.npc);
    }
    sz.take<float>((size_t)nq * c.nsplit * c.R);
    sz.take<int>((size_t)nq * c.nsplit * c.R);
    sz.take<float>((size_t)nq * c.R);
    sz.take<int>((size_t)nq * c.R);
    if (c.ref) sz.take<float>((size_t)nq * c.ub * (c.ncp + 2));
    if (c.batched) {
        sz.take<float>((size_t)nq * h->dpad);
        sz.take<char>(c.bscratch);
    }
    const int lsh_p = c.lsh ? lsh_flips_kept(h->B, c.n_probes) : 0;
    if (c.lsh) {
        sz.take<int32_t>((size_t)nq * c.ub_cand);
        sz.take<uint32_t>((size_t)nq * h->T);
        sz.take<int>((size_t)nq * h->T * std::max(1, lsh_p));
    }
    if (c.lsh_keys) sz.take<float>((size_t)nq * c.ub_cand);
    if (c.tc) {
        sz.take<float>((size_t)nq * h->C);  // BF16 coarse keys
        sz.take<float>((size_t)nq * ceil_div(h->C, 32));  // their 32-centroid chunk minima
        sz.take<__nv_bfloat16>((size_t)nq * h->kpad);
        sz.take<unsigned char>((size_t)nq * c.npc * tc_pair_row_bytes(h));
        sz.take<int8_t>((size_t)nq * h->dpad8);  // int8 query weights and factors (ANN_MODE_TC_SQ8)
        sz.take<float>((size_t)nq);
        sz.take<float>((size_t)nq * c.npc);
        sz.take<int64_t>((size_t)nq * c.npc);
        sz.take<int64_t>((size_t)h->C + 1);
        sz.take<int4>((size_t)tc_items_bound((int64_t)nq * c.npc, (int)h->C, h->sizes_desc[0]));
    }
    sz.take<int32_t>((size_t)nq);  // re-rank query order
    sz.take<int64_t>(1);           // an every-row stream: its length
    sz.take<int32_t>(1);           // and its segment flag
    return sz.off;
}

// IVF on the tensor cores with sampled bars (large batches). Every probed list's head -- its first
// ceil(size / div) rows (div = the sample_div option, 8 by default), an even sample since rows are in
// ascending original id inside a list -- is scored by a first grouped GEMM into each query's sample
// stream. Per query, the fast bar is the rF-th smallest sampled key (rF = ceil(3 R / div): about 3 R keys
// of the whole stream pass it) and the safe bar the R-th (at or above the stream's R-th key), both exact
// (the bars kernel). The grouped GEMM over all rows then appends only the keys at or below the fast bar to
// the query's own buffer (kRowCapFactor R slots); a query left with fewer than min(R, its candidates)
// survivors is redone under its safe bar. Each query ends with the exact best R keys of its stream
// (warp_select_kernel: the keys below the R-th, then equal ones by increasing row), as the key-stream path
// selects them, without writing the stream. Returns with *done = false (and no output) when a query's
// buffer overflowed.
struct TcOperands {
    const void* qrows;     // the queries' operand rows
    int row_bytes;
    const void* B;         // the list-ordered base operand
    int K;                 // operand columns (elements)
    int kind;
    const float2* col_fac;  // per base row (int8 form)
    const float* qfac;      // per query (int8 form)
    float* pfac;            // per pair, filled with the pairs (int8 form)
};
static TcOperands tc_operands(const ann_ivf* h, const IvfQueryCfg& c, const __nv_bfloat16* qb, const int8_t* q8,
                              const float* qfac, float* pfac) {
    if (c.i8) return TcOperands{q8, h->dpad8, h->codes, h->dpad8, kTcI8, h->sq8_fac, qfac, pfac};
    return TcOperands{qb, 2 * h->kpad, h->base_bf16, h->kpad, kTcBF16, nullptr, nullptr, nullptr};
}

// Kernel timer slots of the IVF query (ann_ivf_kernel_profile): the list-keys kernel (the grouped GEMM,
// or the SQ8 batched kernel), the sampled bars, the best-R selection and the exact re-rank.
constexpr int kKernKeys = 0, kKernBars = 1, kKernSelect = 2, kKernRerank = 3;
constexpr int kRowCapFactor = 16;

static int ivf_tc_sampled(ann_ivf* h, ann_workspace* ws, const IvfQueryCfg& c, const IvfQueryArgs& a,
                          const IvfBatchArgs& b, const TcOperands& op, unsigned char* Apk, int64_t* titem,
                          int4* titem_desc, int64_t items_cap, float* keyR, int* idR, int prec, bool* done,
                          cudaStream_t st) {
    *done = false;
    const int nq = a.plan.nq, npc = c.npc, C = (int)h->C, R = c.R;
    const int64_t max_pairs = (int64_t)nq * npc;
    const int64_t largest = h->sizes_desc.empty() ? 1 : h->sizes_desc[0];
    const int div = h->sample_div;
    const int64_t head_max = ceil_div(largest, div);
    const int64_t s_bound = (int64_t)nq * npc * head_max;  // sample keys at most
    const int64_t scap = tc_items_bound(max_pairs, C, head_max);
    const int rF = (int)std::min<int64_t>(R, std::max<int64_t>(1, ceil_div(3 * (int64_t)R, div)));
    const int cap = kRowCapFactor * R;
    size_t scan_tmp = 0;
    ANN_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, (int64_t*)nullptr, (int64_t*)nullptr, nq + 1, st));
    Sizer sz;
    sz.take<int64_t>((size_t)C);                 // list heads
    sz.take<int64_t>((size_t)max_pairs);         // sseg
    sz.take<int64_t>((size_t)nq + 1);            // slen
    sz.take<int64_t>((size_t)nq + 1);            // soff
    sz.take<char>(scan_tmp);
    sz.take<int64_t>((size_t)C + 1);             // sample items
    sz.take<int4>((size_t)scap);
    sz.take<int64_t>((size_t)max_pairs);         // sdbase
    sz.take<int32_t>((size_t)max_pairs);         // row -> query
    sz.take<float>((size_t)s_bound);             // sample keys
    for (int i = 0; i < 3; ++i) sz.take<float>((size_t)nq);  // fast, safe, re-run bars
    sz.take<float>((size_t)nq * cap);            // survivors per query: key, list row
    sz.take<int>((size_t)nq * cap);
    for (int i = 0; i < 3; ++i) sz.take<int>((size_t)nq);    // counts, re-run list, marks
    sz.take<int>(4);                             // flags
    int rc = ws_reserve_big(ws, sz.bytes());
    if (rc) return rc;
    Carver cv(ws->big);
    int64_t* lcap = cv.take<int64_t>((size_t)C);
    int64_t* sseg = cv.take<int64_t>((size_t)max_pairs);
    int64_t* slen = cv.take<int64_t>((size_t)nq + 1);
    int64_t* soff = cv.take<int64_t>((size_t)nq + 1);
    void* stmp = cv.take<char>(scan_tmp);
    int64_t* sitem = cv.take<int64_t>((size_t)C + 1);
    int4* sitem_desc = cv.take<int4>((size_t)scap);
    int64_t* sdbase = cv.take<int64_t>((size_t)max_pairs);
    int32_t* rowq = cv.take<int32_t>((size_t)max_pairs);
    float* SK = cv.take<float>((size_t)s_bound);
    float* tauF = cv.take<float>((size_t)nq);
    float* tauS = cv.take<float>((size_t)nq);
    float* tauR = cv.take<float>((size_t)nq);
    float* skey = cv.take<float>((size_t)nq * cap);
    int* srow = cv.take<int>((size_t)nq * cap);
    int* scount = cv.take<int>((size_t)nq);
    int* list = cv.take<int>((size_t)nq);
    int* mark = cv.take<int>((size_t)nq);
    int* flags = cv.take<int>(4);

    // sample streams: heads of the probed lists, each query's stream offsets
    if ((rc = launch_tc_ivf_sample_plan(a.plan, h->list_off, C, div, lcap, sseg, slen, st))) return rc;
    ANN_CUDA_TRY(cudaMemsetAsync(slen + nq, 0, sizeof(int64_t), st));
    size_t tb = scan_tmp;
    ANN_CUDA_TRY(cub::DeviceScan::ExclusiveSum(stmp, tb, slen, soff, nq + 1, st));
    TcIvfSampleMaps maps;
    maps.row_query = rowq;
    maps.soff = soff;
    maps.sseg = sseg;
    maps.sdbase = sdbase;
    maps.qfac = op.qfac;
    maps.pfac = op.pfac;
    if ((rc = launch_tc_ivf_pairs(op.qrows, op.row_bytes, b.pair_vals, b.pair_lists, b.lq_off + C, max_pairs, npc,
                                  b.cand_off, a.plan.seg_pref, h->list_off, Apk, nullptr, st, maps)))
        return rc;
    // 1. sample pass: keys of the list heads into the sample streams; the two bars per query
    if ((rc = launch_tc_ivf_items(b.lq_off, h->list_off, C, sitem, st, lcap))) return rc;
    if ((rc = launch_tc_item_descs(sitem, C, b.lq_off, h->list_off, lcap, sitem_desc, scap, st))) return rc;
    TcGemmArgs gs{(int)max_pairs, (int)h->n, op.K, nullptr, SK, 0, h->d_err};
    gs.kind = op.kind;
    gs.col_fac = op.col_fac;
    gs.row_fac = op.pfac;
    gs.g_item_off = sitem;
    gs.g_a_off = b.lq_off;
    gs.g_b_off = h->list_off;
    gs.g_b_len = lcap;
    gs.g_dbase = sdbase;
    gs.g_total = sitem + C;
    gs.g_lists = C;
    gs.g_item_desc = sitem_desc;
    if ((rc = launch_tc_gemm(Apk, op.B, gs, st))) return rc;
    int kt = h->prof.kbegin(st);
    if ((rc = launch_warp_bars(SK, soff, slen, nq, rF, R, tauF, tauS, st, (int64_t)npc * head_max))) return rc;
    h->prof.kend(kt, kKernBars, st);
    // 2. filter pass over every row of the probed lists into the queries' buffers
    if ((rc = launch_tc_ivf_items(b.lq_off, h->list_off, C, titem, st))) return rc;
    if ((rc = launch_tc_item_descs(titem, C, b.lq_off, h->list_off, nullptr, titem_desc, items_cap, st))) return rc;
    auto filter = [&](const float* tau, const int* skip_if_zero) -> int {
        TcGemmArgs g{(int)max_pairs, (int)h->n, op.K, nullptr, nullptr, 0, h->d_err};
        g.skip_if_zero = skip_if_zero;
        g.kind = op.kind;
        g.col_fac = op.col_fac;
        g.row_fac = op.pfac;
        g.g_item_off = titem;
        g.g_a_off = b.lq_off;
        g.g_b_off = h->list_off;
        g.g_total = titem + C;
        g.g_lists = C;
        g.g_item_desc = titem_desc;
        g.g_row_query = rowq;
        g.tau = tau;
        g.fkey = skey;
        g.fcol = srow;
        g.row_cap = cap;
        g.rcount = scount;
        const int k0 = skip_if_zero ? -1 : h->prof.kbegin(st);  // the timer sees the first pass only
        const int r = launch_tc_gemm(Apk, op.B, g, st);
        h->prof.kend(k0, kKernKeys, st);
        return r;
    };
    ANN_CUDA_TRY(cudaMemsetAsync(scount, 0, sizeof(int) * (size_t)nq, st));
    if ((rc = filter(tauF, nullptr))) return rc;
    h->prof.mark(prec, st);
    ANN_CUDA_TRY(cudaMemsetAsync(flags, 0, sizeof(int), st));
    if ((rc = launch_tc_bar_check(scount, nq, R, list, flags, st, a.plan.n_cands, mark))) return rc;
    // queries short of survivors: again under their safe bars (their buffers refilled), the rest under -inf;
    // the pass returns at once on the device when no query is short (flags[0] == 0), with no host round trip
    if ((rc = launch_tc_rerun_bars(mark, tauS, nq, tauR, st, scount))) return rc;
    if ((rc = filter(tauR, flags))) return rc;
    if (prec >= 0) h->prof.tc_launches += 1;
    // a query with more survivors than its buffer holds: the caller takes the key-stream path
    if ((rc = launch_max_int(scount, nq, flags + 1, st))) return rc;
    int most = 0;
    ANN_CUDA_TRY(cudaMemcpyAsync(&most, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    ANN_CUDA_TRY(cudaStreamSynchronize(st));
    if (most > cap) return ANN_OK;
    kt = h->prof.kbegin(st);
    if ((rc = launch_warp_select(skey, srow, scount, cap, nq, R, keyR, idR, st))) return rc;
    h->prof.kend(kt, kKernSelect, st);
    if (prec >= 0) h->prof.tc_launches += 2;
    *done = true;
    return ANN_OK;
}

// All stages for nq device-resident padded queries; scratch carved from `base`.
static int ivf_query_device(ann_ivf* h, ann_workspace* ws, const IvfQueryCfg& c, char* base, const float* qdev,
                            int nq, int64_t* ids_dev, float* dists_dev, cudaStream_t st) {
    Carver cv(base);
    int32_t* probes = cv.take<int32_t>((size_t)nq * c.npc);
    int64_t* seg_start = cv.take<int64_t>((size_t)nq * c.npc);
    int64_t* seg_pref = cv.take<int64_t>((size_t)nq * (c.npc + 1));
    int32_t* n_seg = cv.take<int32_t>((size_t)nq);
    int64_t* n_cands = cv.take<int64_t>((size_t)nq);
    float *ckey = nullptr, *Dc = nullptr, *pkey = nullptr;
    int* cid = nullptr;
    if (c.coarse_flat) {
        ckey = cv.take<float>((size_t)nq * c.nsplit_c * c.npc);
        cid = cv.take<int>((size_t)nq * c.nsplit_c * c.npc);
    } else {
        Dc = cv.take<float>((size_t)nq * h->C);
        pkey = cv.take<float>((size_t)nq * c.npc);
    }
    float* keyS = cv.take<float>((size_t)nq * c.nsplit * c.R);
    int* idS = cv.take<int>((size_t)nq * c.nsplit * c.R);
    float* keyR = cv.take<float>((size_t)nq * c.R);
    int* idR = cv.take<int>((size_t)nq * c.R);
    float* DP = c.ref ? cv.take<float>((size_t)nq * c.ub * (c.ncp + 2)) : nullptr;
    float* qs = c.batched ? cv.take<float>((size_t)nq * h->dpad) : nullptr;
    void* bscratch = c.batched ? cv.take<char>(c.bscratch) : nullptr;
    const int lsh_p = c.lsh ? lsh_flips_kept(h->B, c.n_probes) : 0;
    int32_t* cand = c.lsh ? cv.take<int32_t>((size_t)nq * c.ub_cand) : nullptr;
    uint32_t* lsig = c.lsh ? cv.take<uint32_t>((size_t)nq * h->T) : nullptr;
    int* lpert = c.lsh ? cv.take<int>((size_t)nq * h->T * std::max(1, lsh_p)) : nullptr;
    float* lkeys = c.lsh_keys ? cv.take<float>((size_t)nq * c.ub_cand) : nullptr;
    float* ckeys = c.tc ? cv.take<float>((size_t)nq * h->C) : nullptr;
    float* ckmin = c.tc ? cv.take<float>((size_t)nq * ceil_div(h->C, 32)) : nullptr;
    __nv_bfloat16* qb = c.tc ? cv.take<__nv_bfloat16>((size_t)nq * h->kpad) : nullptr;
    unsigned char* Apk = c.tc ? cv.take<unsigned char>((size_t)nq * c.npc * tc_pair_row_bytes(h)) : nullptr;
    int8_t* q8 = c.tc ? cv.take<int8_t>((size_t)nq * h->dpad8) : nullptr;
    float* qfac = c.tc ? cv.take<float>((size_t)nq) : nullptr;
    float* pfac = c.tc ? cv.take<float>((size_t)nq * c.npc) : nullptr;
    int64_t* dbase = c.tc ? cv.take<int64_t>((size_t)nq * c.npc) : nullptr;
    int64_t* titem = c.tc ? cv.take<int64_t>((size_t)h->C + 1) : nullptr;
    const int64_t items_cap = c.tc ? tc_items_bound((int64_t)nq * c.npc, (int)h->C, h->sizes_desc[0]) : 0;
    int4* titem_desc = c.tc ? cv.take<int4>((size_t)items_cap) : nullptr;
    int32_t* qorder = cv.take<int32_t>((size_t)nq);
    int64_t* every_len = cv.take<int64_t>(1);
    int32_t* every_seg = cv.take<int32_t>(1);

    IvfQueryArgs a{};
    a.ix = h->view();
    a.plan.nq = nq;
    a.plan.npc = c.npc;
    a.plan.probes = probes;
    a.plan.seg_start = seg_start;
    a.plan.seg_pref = seg_pref;
    a.plan.n_seg = n_seg;
    a.plan.n_cands = n_cands;
    a.q = qdev;
    a.ldq = h->dpad;
    a.k = c.k;
    a.R = c.R;
    a.max_cands = c.max_c;
    a.no_fallback = c.shard ? 1 : 0;
    a.nsplit = c.nsplit;
    a.num_threads = c.num_threads;
    a.ndist = h->d_ndist;
    a.err = h->d_err;
    a.out_ids = ids_dev;
    a.out_dists = dists_dev;

    int rc;
    const int prec = h->prof.begin(st);
    // 1. coarse ranking
    if (c.tc) {
        // BF16 keys to every centroid, then the exact FP32 order of the best npc + 16
        if ((rc = launch_tc_operand(qdev, nq, h->dim, h->dpad, qb, h->kpad, kTcQuery, ANN_METRIC_L2, 0, st))) return rc;
        TcGemmArgs ca{nq, h->C, h->kpad, nullptr, ckeys, h->C, h->d_err};
        ca.out_cmin = ckmin;  // and each query's 32-centroid chunk minima, which let the ranking skip chunks
        if ((rc = launch_tc_gemm(qb, h->cent_bf16, ca, st))) return rc;
        if ((rc = launch_tc_coarse(ckeys, h->C, nq, h->C, c.npc, 16, qdev, h->centroids, h->dpad, probes, st,
                                   h->cent_norm_max, h->dim, ckmin)))
            return rc;
        if (c.i8 && (rc = launch_tc_sq8_query(qdev, nq, h->dim, h->dpad, h->scale, h->offset, q8, h->dpad8, qfac, st)))
            return rc;
    } else if (c.coarse_flat) {
        FlatScanArgs fa{h->centroids, h->C, h->dpad, qdev, nq, ANN_METRIC_L2, c.npc, c.rps_c, c.nsplit_c, ckey, cid};
        if ((rc = launch_flat_scan(fa, c.bqc, st))) return rc;
        MergeArgs m{ckey, cid, nq, c.nsplit_c, c.npc, c.npc, 0, nullptr, nullptr};
        m.out_id32 = probes;
        if ((rc = launch_merge_splits(m, st))) return rc;
    } else {
        if ((rc = launch_ref_centroid_dists(a.ix, qdev, h->dpad, nq, Dc, st))) return rc;
        if ((rc = launch_select_topk(Dc, h->C, nullptr, nq, c.npc, nullptr, pkey, probes, st))) return rc;
    }
    h->prof.mark(prec, st);
    // 2. plan: whole lists, or the LSH buckets' explicit streams (signatures first, their own stage)
    LshCandArgs la{};
    if (c.lsh) {
        la.ix = a.ix;
        la.lsh = h->lsh_view();
        la.q = qdev;
        la.ldq = h->dpad;
        la.nq = nq;
        la.n_probes = c.n_probes;
        la.sig = lsig;
        la.pert = lpert;
        if ((rc = launch_lsh_signatures(la, st))) return rc;
    }
    h->prof.mark(prec, st);
    if (c.lsh) {
        la.probes = probes;
        la.npc = c.npc;
        la.k = c.k;
        la.max_c = c.max_c;
        la.ld = c.ub_cand;
        la.largest_list = h->sizes_desc.empty() ? 1 : h->sizes_desc[0];
        la.cand_ids = cand;
        la.n_cands = n_cands;
        la.n_seg = n_seg;
        la.ndist = h->d_ndist;
        if ((rc = launch_lsh_candidates(la, st))) return rc;
        a.plan.cand_ids = cand;
        a.plan.cand_ld = c.ub_cand;
    } else if ((rc = launch_ivf_plan(a, st))) {
        return rc;
    }
    h->prof.mark(prec, st);
    // The queries whose stream is every row (fewer than k candidates, :453-457): in reference mode they do
    // not fit the per-query scratch of L = ub positions, and in a large exact batch one CTA would scan all
    // n rows. The main pass sees them as empty streams; each is redone below on its own, split over the
    // whole GPU. (Small exact batches already split every query that widely and skip the host read.)
    std::vector<int> every_row;
    auto take_every_row = [&]() -> int {
        std::vector<int32_t> ns(nq);
        ANN_CUDA_TRY(cudaMemcpyAsync(ns.data(), n_seg, sizeof(int32_t) * (size_t)nq, cudaMemcpyDeviceToHost, st));
        ANN_CUDA_TRY(cudaStreamSynchronize(st));
        for (int i = 0; i < nq; ++i)
            if (ns[i] < 0) every_row.push_back(i);
        if (!every_row.empty()) {
            int r = launch_clear_every_row(a.plan, st);
            if (r) return r;
            const int64_t len = h->n;
            const int32_t seg = -1;
            ANN_CUDA_TRY(cudaMemcpyAsync(every_len, &len, sizeof(len), cudaMemcpyHostToDevice, st));
            ANN_CUDA_TRY(cudaMemcpyAsync(every_seg, &seg, sizeof(seg), cudaMemcpyHostToDevice, st));
            ANN_CUDA_TRY(cudaStreamSynchronize(st));  // the host values above live on this frame
        }
        return ANN_OK;
    };
    const bool every_row_apart = c.fallback && (c.ref || c.nsplit < kEveryRowMinSplit);
    // batched passes learn of every-row queries from the batch set-up's own host read (below), so the common
    // case takes no extra round trip here
    if (every_row_apart && !(c.batched && !c.ref) && (rc = take_every_row())) return rc;
    // 3. SQ8 pass -> best R per query
    bool done = false;
    if (!c.ref && c.batched) {
        IvfBatchArgs b{};
        int64_t tot_local[3] = {0, 0, 0};
        int64_t* tot = tot_local;
        // The sampled path needs none of the set-up's totals to run: they land in page-locked words and are read
        // after its own synchronisation (a batch with every-row queries, rare, is then set up again and redone).
        const bool sampled = c.tc && nq >= h->sampled_min_queries;
        if (sampled && (rc = ws_pinned(ws, &tot))) return rc;
        tot[0] = tot[1] = tot[2] = 0;
        auto run_sampled = [&](bool* ok) -> int {
            return ivf_tc_sampled(h, ws, c, a, b, tc_operands(h, c, qb, q8, qfac, pfac), Apk, titem, titem_desc,
                                  items_cap, keyR, idR, prec, ok, st);
        };
        bool sampled_done = false;
        if ((rc = batched_prepare(a, bscratch, c.sort_tmp, c.scan_tmp, &b, tot, st, !sampled))) return rc;
        if (sampled && (rc = run_sampled(&sampled_done))) return rc;  // synchronises st: tot is current
        if (tot[2] != 0) sampled_done = false;
        if (tot[2] != 0 && every_row_apart) {  // every-row queries: set apart, then the batch set up again
            if ((rc = take_every_row())) return rc;
            if ((rc = batched_prepare(a, bscratch, c.sort_tmp, c.scan_tmp, &b, tot, st))) return rc;
            if (tot[2] == 0 && sampled && (rc = run_sampled(&sampled_done))) return rc;
        }
        done = sampled_done;
        if (tot[2] == 0 && !sampled_done) {  // no query fell back to scanning every row
            if ((rc = ws_reserve_big(ws, sizeof(float) * (size_t)std::max<int64_t>(tot[1], 1)))) return rc;
            float* D = reinterpret_cast<float*>(ws->big);
            if (c.tc) {
                // BF16 keys of every (pair, list row) from grouped tcgen05 GEMMs, the best R of each
                // query's stream by radix selection
                const TcOperands op = tc_operands(h, c, qb, q8, qfac, pfac);
                const int64_t max_pairs = (int64_t)nq * c.npc;
                TcIvfSampleMaps maps;
                maps.qfac = op.qfac;
                maps.pfac = op.pfac;
                if ((rc = launch_tc_ivf_pairs(op.qrows, op.row_bytes, b.pair_vals, b.pair_lists, b.lq_off + h->C,
                                              max_pairs, c.npc, b.cand_off, a.plan.seg_pref, h->list_off, Apk, dbase,
                                              st, maps)))
                    return rc;
                if ((rc = launch_tc_ivf_items(b.lq_off, h->list_off, h->C, titem, st))) return rc;
                if ((rc = launch_tc_item_descs(titem, (int)h->C, b.lq_off, h->list_off, nullptr, titem_desc, items_cap,
                                               st)))
                    return rc;
                TcGemmArgs g{(int)max_pairs, (int)h->n, op.K, nullptr, D, 0, h->d_err};
                g.kind = op.kind;
                g.col_fac = op.col_fac;
                g.row_fac = op.pfac;
                g.g_item_off = titem;
                g.g_a_off = b.lq_off;
                g.g_b_off = h->list_off;
                g.g_dbase = dbase;
                g.g_total = titem + h->C;
                g.g_lists = h->C;
                g.g_item_desc = titem_desc;
                const int kg = h->prof.kbegin(st);
                if ((rc = launch_tc_gemm(Apk, op.B, g, st))) return rc;
                h->prof.kend(kg, kKernKeys, st);
                h->prof.mark(prec, st);
                RadixSelectArgs rs{};
                rs.keys = D;
                rs.offs = b.cand_off;
                rs.lens = n_cands;
                rs.plan = a.plan;
                rs.use_plan = 1;
                rs.R = c.R;
                rs.out_key = keyR;
                rs.out_id = idR;
                const int ks = h->prof.kbegin(st);
                if ((rc = launch_radix_select(rs, nq, st))) return rc;
                h->prof.kend(ks, kKernSelect, st);
            } else {
                const int kb = h->prof.kbegin(st);
                if ((rc = launch_batched(b, qdev, qs, D, st))) return rc;
                h->prof.kend(kb, kKernKeys, st);
                h->prof.mark(prec, st);
                // the best R of each stream as a set (ties by stream position); the re-rank orders them
                RadixSelectArgs rs{};
                rs.keys = D;
                rs.offs = b.cand_off;
                rs.lens = n_cands;
                rs.plan = a.plan;
                rs.use_plan = 1;
                rs.R = c.R;
                rs.out_key = keyR;
                rs.out_id = idR;
                const int ks = h->prof.kbegin(st);
                if ((rc = launch_radix_select(rs, nq, st))) return rc;
                h->prof.kend(ks, kKernSelect, st);
            }
            done = true;
        }
    }
    if (!done && c.lsh_keys) {
        if ((rc = launch_ivf_sq8_dists(a, lkeys, c.ub_cand, st))) return rc;
        h->prof.mark(prec, st);
        if ((rc = launch_select_topk(lkeys, c.ub_cand, n_cands, nq, c.R, &a.plan, keyR, idR, st, nullptr, true))) return rc;
        done = true;
    }
    if (done) {
    } else if (!c.ref) {
        a.keyR = keyS;
        a.idR = idS;
        if ((rc = launch_ivf_sq8_scan(a, st))) return rc;  // keys and each split's best R in one kernel
        h->prof.mark(prec, st);
        if (c.nsplit > 1) {
            MergeArgs m{keyS, idS, nq, c.nsplit, c.R, c.R, 0, nullptr, nullptr};
            m.out_id32 = idR;
            m.out_key32 = keyR;
            if ((rc = launch_merge_splits(m, st))) return rc;
        } else {
            keyR = keyS;
            idR = idS;
        }
    } else {
        a.L = c.ub;
        a.ncp = c.ncp;
        a.D = DP;
        a.V = DP + (size_t)nq * c.ub;
        a.P = DP + (size_t)2 * nq * c.ub;
        if ((rc = launch_ivf_ref_sq8(a, c.ub, st))) return rc;
        h->prof.mark(prec, st);
        if ((rc = launch_select_topk(a.V, c.ub, n_cands, nq, c.R, &a.plan, keyR, idR, st, nullptr, true))) return rc;
    }
    h->prof.mark(prec, st);
    // 4. FP32 re-rank and the final top-k; batches run their queries grouped by first probed list, so that
    // CTAs resident together gather rows of the same lists (shared candidates come from L2)
    if (!c.ref && nq >= kQueryOrderMinBatch && h->C <= kQueryOrderMaxLists) {
        if ((rc = launch_query_order(probes, c.npc, nq, (int)h->C, qorder, st))) return rc;
        a.qorder = qorder;
    }
    const int kr = h->prof.kbegin(st);
    if ((rc = launch_ivf_rerank(a, keyR, idR, c.ref ? 1 : 0, st))) return rc;
    h->prof.kend(kr, kKernRerank, st);
    if (!every_row.empty()) {
        const int64_t L = h->n;
        const int nsp = (int)std::min<int64_t>(2 * kNumSMs, std::max<int64_t>(1, ceil_div(L, 2048)));
        const size_t need = c.ref ? sizeof(float) * (size_t)L * (c.ncp + 2) : (size_t)8 * nsp * c.R;
        if ((rc = ws_reserve_big(ws, need))) return rc;
        float* big = reinterpret_cast<float*>(ws->big);
        for (int q : every_row) {
            IvfQueryArgs b = a;
            b.qorder = nullptr;
            b.plan.nq = 1;
            b.plan.probes = probes + (size_t)q * c.npc;
            b.plan.seg_start = seg_start + (size_t)q * c.npc;
            b.plan.seg_pref = seg_pref + (size_t)q * (c.npc + 1);
            b.plan.n_seg = every_seg;
            b.plan.n_cands = every_len;
            b.plan.cand_ids = nullptr;
            b.q = qdev + (size_t)q * h->dpad;
            b.out_ids = ids_dev + (size_t)q * c.k;
            b.out_dists = dists_dev ? dists_dev + (size_t)q * c.k : nullptr;
            float* kq = keyR + (size_t)q * c.R;
            int* iq = idR + (size_t)q * c.R;
            if (c.ref) {
                b.L = L;
                b.D = big;
                b.V = big + L;
                b.P = big + 2 * L;
                if ((rc = launch_ivf_ref_sq8(b, L, st))) return rc;
                if ((rc = launch_select_topk(b.V, L, b.plan.n_cands, 1, c.R, &b.plan, kq, iq, st, nullptr, true))) return rc;
            } else {
                b.nsplit = nsp;
                b.keyR = big;
                b.idR = reinterpret_cast<int*>(big + (size_t)nsp * c.R);
                if ((rc = launch_ivf_sq8_scan(b, st))) return rc;
                MergeArgs m{b.keyR, b.idR, 1, nsp, c.R, c.R, 0, nullptr, nullptr};
                m.out_id32 = iq;
                m.out_key32 = kq;
                if ((rc = launch_merge_splits(m, st))) return rc;
            }
            if ((rc = launch_ivf_rerank(b, kq, iq, c.ref ? 1 : 0, st))) return rc;
        }
    }
    h->prof.mark(prec, st);
    return ANN_OK;
}

}  // namespace

extern "C" {

int ann_ivf_query(ann_ivf* h, ann_workspace* ws, const float* queries, int32_t nq, int64_t ldq, int32_t k,
                  int32_t n_probes, int32_t n_probe_clusters, int32_t refine_r, int64_t max_candidates, int32_t mode,
                  int32_t num_threads, int32_t mem, int64_t* out_ids, float* out_dists, void* stream) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr, "ann_ivf_query: null index");
    if (h->n == 0) {
        set_error("index not fitted");
        return ANN_ERR_STATE;
    }
    ANN_CHECK_ARG(nq >= 0 && k >= 1, "ann_ivf_query: nq=%d, k=%d", nq, k);
    ANN_CHECK_ARG(ldq >= h->dim, "ann_ivf_query: query stride < dim");
    const bool shard = (mode & ANN_QUERY_SHARD) != 0;
    mode &= ~ANN_QUERY_SHARD;
    ANN_CHECK_ARG(!shard || mode != ANN_MODE_REFERENCE, "ann_ivf_query: a shard of the lists has no reference semantics");
    ANN_CHECK_ARG(mode == ANN_MODE_EXACT || mode == ANN_MODE_REFERENCE || mode == ANN_MODE_TC || mode == ANN_MODE_TC_SQ8,
                  "ann_ivf_query: unknown mode %d", mode);
    ANN_CHECK_ARG(nq == 0 || (queries && out_ids), "ann_ivf_query: null pointer");
    ANN_CHECK_ARG(k <= 1024, "ann_ivf_query: k=%d > 1024", k);
    ANN_CHECK_ARG(n_probes >= 0, "ann_ivf_query: n_probes=%d < 0", n_probes);
    if (nq == 0) return ANN_OK;
    if (!ws) ws = &h->ws;
    DeviceGuard g(h->device);
    cudaStream_t st = as_stream(stream);

    IvfQueryCfg c{};
    int rc0 = ANN_OK;
    c.ref = mode == ANN_MODE_REFERENCE;
    c.tc = mode == ANN_MODE_TC || mode == ANN_MODE_TC_SQ8;
    c.i8 = mode == ANN_MODE_TC_SQ8;
    c.shard = shard;
    c.k = k;
    c.npc = std::max(1, std::min(n_probe_clusters, h->C));  // active_clusters (:332)
    // R = max(k, refine_r > 0 ? refine_r : 4k) (:472-474); cap max(2000, 4 * target) (:357-358)
    const int target = refine_r > 0 ? refine_r : 4 * k;
    c.R = std::max(k, target);
    c.max_c = max_candidates;
    if (c.max_c < 0) c.max_c = std::max<int64_t>(2000, 4 * (int64_t)target);
    if (c.max_c == 0) c.max_c = INT64_MAX;
    c.num_threads = num_threads > 0 ? num_threads : (int)std::max(1u, std::thread::hardware_concurrency());
    if (c.ref) ANN_CHECK_ARG(c.R <= 8192, "reference mode: refine count %d > 8192", c.R);
    if (!c.ref && c.R > 1024) {
        set_error("ann_ivf_query: refine count %d > 1024 in exact mode", c.R);
        return ANN_ERR_UNSUPPORTED;
    }
    // longest possible candidate stream: the npc largest lists up to the cap; every row when a
    // query's lists could hold fewer than k points (the reference then scans all rows, :453-457)
    // (a list is added while the stream is below the cap, so a capped stream ends below
    // cap - 1 + the largest list)
    int64_t ub = 0, smallest = 0;
    for (int j = 0; j < c.npc; ++j) ub += h->sizes_desc[j];
    if (c.max_c != INT64_MAX) ub = std::min(ub, c.max_c - 1 + h->sizes_desc[0]);
    for (int j = 0; j < c.npc; ++j) smallest += h->sizes_desc[h->C - 1 - j];
    c.lsh = h->lsh();
    c.n_probes = c.lsh ? n_probes : 0;
    // an LSH stream can fall short of k however large its lists; reference-mode scratch is sized for the
    // capped streams and a query that scans every row is redone on its own (ivf_query_device)
    c.fallback = !c.shard && (c.lsh || smallest < k);
    if (c.shard && c.lsh) {
        set_error("ann_ivf_query: a shard of the lists is searched without LSH bucket tables");
        return ANN_ERR_UNSUPPORTED;
    }
    c.ub_cand = std::max<int64_t>(ub, 1);
    c.ub = c.ub_cand;
    if (c.lsh && c.tc) {
        set_error("ann_ivf_query: the tensor-core form scores whole lists; LSH bucket tables use the SQ8 forms");
        return ANN_ERR_UNSUPPORTED;
    }
    c.ncp = ref_num_checkpoints(h->dim);
    c.coarse_flat = !c.ref && c.npc <= 512;
    c.batched = !c.ref && !c.lsh && (c.tc || nq >= kBatchedMinQueries);
    if (c.tc && (rc0 = ivf_ensure_tc(h, c.i8, st))) return rc0;
    const int dpad = h->dpad;
    const bool host = mem == ANN_MEM_HOST;

    // queries per device call: bounded scratch in reference mode
    int qc = nq;
    if (c.ref || c.lsh) {
        const bool keys = c.lsh && !c.ref && nq >= 64;  // the lsh_keys path, decided below
        const size_t per_q = (c.ref ? sizeof(float) * (size_t)c.ub * (c.ncp + 2) : 0) +
                             (c.lsh ? sizeof(int32_t) * (size_t)c.ub_cand : 0) +
                             (keys ? sizeof(float) * (size_t)c.ub_cand : 0) + 4096;
        qc = (int)std::max<size_t>(1, std::min<size_t>(nq, ((size_t)2 << 30) / per_q));
    }
    c.nsplit = c.ref ? 1 : (int)std::max<int64_t>(1, std::min<int64_t>(64, ceil_div(2 * kNumSMs, qc)));
    c.lsh_keys = c.lsh && !c.ref && c.nsplit < kEveryRowMinSplit;
    c.bqc = std::min(flat_scan_bq(qc), flat_scan_max_bq(c.npc));
    {
        const int n_qt = (int)ceil_div(qc, c.bqc);
        c.nsplit_c = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(kNumSMs, n_qt), ceil_div(h->C, 512)));
        c.rps_c = ceil_div(ceil_div(h->C, c.nsplit_c), 256) * 256;
        c.nsplit_c = (int)ceil_div(h->C, c.rps_c);
    }
    if (c.batched) c.bscratch = batched_scratch_bytes(qc, c.npc, h->C, &c.sort_tmp, &c.scan_tmp);
    Sizer head;
    head.take<float>((size_t)nq * dpad);
    if (host) {
        head.take<int64_t>((size_t)nq * k);
        head.take<float>((size_t)nq * k);
    }
    const size_t head_bytes = (head.off + 255) / 256 * 256;
    int rc = ws_reserve_device(ws, head_bytes + ivf_scratch(h, c, qc) + 512);
    if (rc) return rc;
    Carver cv(ws->dev);
    float* qdev = cv.take<float>((size_t)nq * dpad);
    int64_t* ids_dev = out_ids;
    float* dists_dev = out_dists;
    if (host) {
        ids_dev = cv.take<int64_t>((size_t)nq * k);
        dists_dev = cv.take<float>((size_t)nq * k);
    }
    char* scratch = ws->dev + head_bytes;
    const float* qrows = qdev;  // the queries in the padded layout the kernels read (read only)
    if (host) {
        if ((rc = queries_in(qdev, dpad, queries, ldq, nq, h->dim, st))) return rc;
    } else if (h->dim == dpad && ldq == dpad && (reinterpret_cast<uintptr_t>(queries) & 15) == 0) {
        qrows = queries;  // already in that layout: no copy
    } else {
        rc = launch_pad_rows(queries, nq, h->dim, ldq, qdev, dpad, st);
        if (rc) return rc;
    }
    for (int q0 = 0; q0 < nq; q0 += qc) {
        const int nc = std::min(qc, nq - q0);
        rc = ivf_query_device(h, ws, c, scratch, qrows + (size_t)q0 * dpad, nc, ids_dev + (size_t)q0 * k,
                              dists_dev ? dists_dev + (size_t)q0 * k : nullptr, st);
        if (rc) return rc;
    }
    h->query_count += nq;
    if (host) {
        ANN_CUDA_TRY(cudaMemcpyAsync(out_ids, ids_dev, sizeof(int64_t) * (size_t)nq * k, cudaMemcpyDeviceToHost, st));
        if (out_dists)
            ANN_CUDA_TRY(cudaMemcpyAsync(out_dists, dists_dev, sizeof(float) * (size_t)nq * k, cudaMemcpyDeviceToHost, st));
        ANN_CUDA_TRY(cudaStreamSynchronize(st));
        return ann_ivf_device_status(h);
    }
    return ANN_OK;
}

int ann_ivf_device_status(ann_ivf* h) {
    ANN_CHECK_ARG(h != nullptr, "null index");
    if (!h->d_err) return ANN_OK;
    DeviceGuard g(h->device);
    int v = 0;
    ANN_CUDA_TRY(cudaMemcpy(&v, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (v) {
        ANN_CUDA_TRY(cudaMemset(h->d_err, 0, sizeof(int)));
        set_error("a device-side wait gave up after its time limit; the results of the affected queries are invalid");
        return ANN_ERR_TIMEOUT;
    }
    return ANN_OK;
}

int64_t ann_ivf_total_distances(ann_ivf* h) {
    if (!h || !h->d_ndist) return 0;
    DeviceGuard g(h->device);
    unsigned long long v = 0;
    if (cudaMemcpy(&v, h->d_ndist, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return (int64_t)v;
}

int ann_ivf_reset_distances(ann_ivf* h) {
    ANN_CHECK_ARG(h != nullptr, "null index");
    if (!h->d_ndist) return ANN_OK;
    DeviceGuard g(h->device);
    ANN_CUDA_TRY(cudaMemset(h->d_ndist, 0, sizeof(unsigned long long)));
    return ANN_OK;
}

int ann_ivf_set_profiling(ann_ivf* h, int32_t enable) {
    ANN_CHECK_ARG(h != nullptr, "null index");
    h->prof.enabled = enable != 0;
    return ANN_OK;
}

int ann_ivf_profile(ann_ivf* h, double* out8) {
    ANN_CHECK_ARG(h != nullptr && out8 != nullptr, "null argument");
    DeviceGuard g(h->device);
    h->prof.collect();
    for (int i = 0; i < 6; ++i) out8[i] = h->prof.total_ms[i];
    out8[6] = (double)h->prof.calls;
    out8[7] = (double)h->query_count;
    return ANN_OK;
}

int ann_ivf_set_option(ann_ivf* h, int32_t option, int64_t value) {
    ANN_CHECK_ARG(h != nullptr, "null index");
    switch (option) {
        case ANN_IVF_OPT_SAMPLE_DIV:
            ANN_CHECK_ARG(value >= 2 && value <= 64, "sample divisor %lld (2..64)", (long long)value);
            h->sample_div = (int)value;
            return ANN_OK;
        case ANN_IVF_OPT_SAMPLED_MIN:
            ANN_CHECK_ARG(value >= 1 && value <= INT32_MAX, "sampled-path batch size %lld", (long long)value);
            h->sampled_min_queries = (int)value;
            return ANN_OK;
        default:
            set_error("ann_ivf_set_option: unknown option %d", option);
            return ANN_ERR_INVALID;
    }
}

int ann_ivf_kernel_profile(ann_ivf* h, double* out8) {
    ANN_CHECK_ARG(h != nullptr && out8 != nullptr, "null argument");
    DeviceGuard g(h->device);
    h->prof.collect();
    for (int i = 0; i < StageProfiler::kKernels; ++i) {
        out8[i] = h->prof.kern_ms[i];
        out8[4 + i] = (double)h->prof.kern_launches[i];
    }
    return ANN_OK;
}

int ann_ivf_reset_profile(ann_ivf* h) {
    ANN_CHECK_ARG(h != nullptr, "null index");
    DeviceGuard g(h->device);
    h->prof.reset();
    h->query_count = 0;
    return ANN_OK;
}

}  // extern "C"

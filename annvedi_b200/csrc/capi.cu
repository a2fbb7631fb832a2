// C ABI: error state, workspaces and the flat (linear) index.
//
// The flat index mirrors linear_ann_cpp.LinearIndex (competitors/linear/src/linear_index.cpp:
// 62-131): fit copies the base into memory the index owns (linear_index.cpp:82 copies into a
// std::vector; here the copy lands in HBM as zero-padded rows), query returns int64 ids and adds
// n to the cumulative distance counter per query (linear_index.cpp:108, 123).
#include <cstdarg>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <vector>

#include "common.cuh"
#include "compat.cuh"
#include "flat_scan.cuh"
#include "runtime.cuh"
#include "flat_internal.cuh"
#include "ivf.cuh"
#include "tc_gemm.cuh"

namespace annb {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
void clear_error() { g_err[0] = 0; }

static std::atomic<int64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int ws_reserve_device(ann_workspace* ws, size_t bytes) {
    std::lock_guard<std::mutex> lk(ws->mu);
    if (ws->dev_cap >= bytes) return ANN_OK;
    size_t cap = std::max(bytes, ws->dev_cap + ws->dev_cap / 2);
    if (ws->dev) {
        ANN_CUDA_TRY(cudaDeviceSynchronize());
        ANN_CUDA_TRY(cudaFree(ws->dev));
        ws->dev = nullptr;
        ws->dev_cap = 0;
    }
    cudaError_t e = cudaMalloc(&ws->dev, cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        e = cudaMalloc(&ws->dev, bytes);
        cap = bytes;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        ws->dev = nullptr;
        set_error("workspace: cannot allocate %zu bytes of device scratch (%s)", bytes, cudaGetErrorString(e));
        return ANN_ERR_NOMEM;
    }
    ws->dev_cap = cap;
    return ANN_OK;
}

int ws_reserve_big(ann_workspace* ws, size_t bytes) {
    std::lock_guard<std::mutex> lk(ws->mu);
    if (ws->big_cap >= bytes) return ANN_OK;
    size_t cap = std::max(bytes, ws->big_cap + ws->big_cap / 4);
    if (ws->big) {
        ANN_CUDA_TRY(cudaDeviceSynchronize());
        ANN_CUDA_TRY(cudaFree(ws->big));
        ws->big = nullptr;
        ws->big_cap = 0;
    }
    cudaError_t e = cudaMalloc(&ws->big, cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        e = cudaMalloc(&ws->big, bytes);
        cap = bytes;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        ws->big = nullptr;
        set_error("workspace: cannot allocate %zu bytes of device scratch (%s)", bytes, cudaGetErrorString(e));
        return ANN_ERR_NOMEM;
    }
    ws->big_cap = cap;
    return ANN_OK;
}

int ws_reserve_host(ann_workspace* ws, size_t bytes) {
    std::lock_guard<std::mutex> lk(ws->mu);
    if (ws->host_cap >= bytes) return ANN_OK;
    size_t cap = std::max(bytes, ws->host_cap + ws->host_cap / 2);
    if (ws->host) {
        ANN_CUDA_TRY(cudaDeviceSynchronize());
        ANN_CUDA_TRY(cudaFreeHost(ws->host));
        ws->host = nullptr;
        ws->host_cap = 0;
    }
    cudaError_t e = cudaMallocHost(&ws->host, cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("workspace: cannot allocate %zu bytes of pinned host memory (%s)", cap, cudaGetErrorString(e));
        return ANN_ERR_NOMEM;
    }
    ws->host_cap = cap;
    return ANN_OK;
}

}  // namespace annb

using namespace annb;


extern "C" {

const char* ann_version(void) { return "annvedi_b200 0.1 sm_100a"; }
const char* ann_last_error(void) { return g_err; }
int64_t ann_kernel_launches(void) { return g_launches.load(); }

int ann_workspace_create(ann_workspace** out, int device) {
    ANN_CHECK_ARG(out != nullptr, "ann_workspace_create: out is NULL");
    ann_workspace* ws = new (std::nothrow) ann_workspace();
    if (!ws) {
        set_error("ann_workspace_create: out of host memory");
        return ANN_ERR_NOMEM;
    }
    ws->device = device;
    *out = ws;
    return ANN_OK;
}

static void ws_release(ann_workspace* ws) {
    DeviceGuard g(ws->device);
    if (ws->dev) cudaFree(ws->dev);
    if (ws->host) cudaFreeHost(ws->host);
    if (ws->big) cudaFree(ws->big);
    ws->dev = nullptr;
    ws->host = nullptr;
    ws->big = nullptr;
    ws->dev_cap = ws->host_cap = ws->big_cap = 0;
}

int ann_workspace_destroy(ann_workspace* ws) {
    if (!ws) return ANN_OK;
    ws_release(ws);
    delete ws;
    return ANN_OK;
}

int64_t ann_workspace_bytes(const ann_workspace* ws) { return ws ? (int64_t)ws->dev_cap : 0; }

int ann_flat_create(ann_flat** out, int device) {
    clear_error();
    ANN_CHECK_ARG(out != nullptr, "ann_flat_create: out is NULL");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("no CUDA device visible (%s)", e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
        return ANN_ERR_CUDA;
    }
    ANN_CHECK_ARG(device >= 0 && device < ndev, "ann_flat_create: device %d not in [0, %d)", device, ndev);
    ann_flat* h = new (std::nothrow) ann_flat();
    if (!h) {
        set_error("ann_flat_create: out of host memory");
        return ANN_ERR_NOMEM;
    }
    h->device = device;
    h->ws.device = device;
    *out = h;
    return ANN_OK;
}

int ann_flat_destroy(ann_flat* h) {
    if (!h) return ANN_OK;
    {
        DeviceGuard g(h->device);
        if (h->base) cudaFree(h->base);
        if (h->base_bf16) cudaFree(h->base_bf16);
        if (h->norms) cudaFree(h->norms);
        if (h->d_err) cudaFree(h->d_err);
    }
    ws_release(&h->ws);
    delete h;
    return ANN_OK;
}

int ann_flat_fit(ann_flat* h, const float* data, int64_t n, int32_t dim, int64_t ld, int32_t metric, int32_t mem,
                 void* stream) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr, "ann_flat_fit: null index");
    ANN_CHECK_ARG(n >= 1 && dim >= 1, "ann_flat_fit: need a non-empty 2-D array, got [%lld, %d]", (long long)n, dim);
    ANN_CHECK_ARG(n < INT32_MAX, "ann_flat_fit: n=%lld exceeds 32-bit ids", (long long)n);
    ANN_CHECK_ARG(ld >= dim, "ann_flat_fit: row stride %lld < dim %d", (long long)ld, dim);
    ANN_CHECK_ARG(metric == ANN_METRIC_L2 || metric == ANN_METRIC_IP, "ann_flat_fit: unknown metric %d", metric);
    ANN_CHECK_ARG(data != nullptr, "ann_flat_fit: data is NULL");
    DeviceGuard g(h->device);
    cudaStream_t st = as_stream(stream);
    const int dpad = (int)ceil_div(dim, 32) * 32;
    if (h->base) {
        ANN_CUDA_TRY(cudaDeviceSynchronize());
        ANN_CUDA_TRY(cudaFree(h->base));
        h->base = nullptr;
    }
    if (h->base_bf16) {
        ANN_CUDA_TRY(cudaFree(h->base_bf16));
        h->base_bf16 = nullptr;
    }
    if (h->norms) {
        ANN_CUDA_TRY(cudaFree(h->norms));
        h->norms = nullptr;
    }
    const size_t bytes = sizeof(float) * (size_t)n * dpad;
    cudaError_t e = cudaMalloc(&h->base, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        h->base = nullptr;
        h->n = 0;
        set_error("ann_flat_fit: cannot allocate %zu bytes for the base (%s)", bytes, cudaGetErrorString(e));
        return ANN_ERR_NOMEM;
    }
    if (dpad != dim) ANN_CUDA_TRY(cudaMemsetAsync(h->base, 0, bytes, st));
    ANN_CUDA_TRY(cudaMemcpy2DAsync(h->base, sizeof(float) * dpad, data, sizeof(float) * ld, sizeof(float) * dim, n,
                                   mem == ANN_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st));
    if (mem == ANN_MEM_HOST) ANN_CUDA_TRY(cudaStreamSynchronize(st));
    h->n = n;
    h->dim = dim;
    h->dpad = dpad;
    h->metric = metric;
    return ANN_OK;
}

}  // extern "C"

// Number of row splits for an exact scan of n rows by nq queries in tiles of bq.
int annb::flat_choose_nsplit(int64_t n, int nq, int bq, int64_t* rows_per_split) {
    const int n_qtiles = (int)ceil_div(nq, bq);
    const int ctas_per_sm = bq <= 8 ? 2 : 1;
    const int64_t target = (int64_t)kNumSMs * ctas_per_sm;
    int64_t nsplit = ceil_div(target, n_qtiles);
    const int64_t tile = 256;
    const int64_t max_split = std::max<int64_t>(1, ceil_div(n, 2 * tile));
    nsplit = std::max<int64_t>(1, std::min(nsplit, max_split));
    int64_t rps = ceil_div(ceil_div(n, nsplit), tile) * tile;
    nsplit = ceil_div(n, rps);
    *rows_per_split = rps;
    return (int)nsplit;
}

extern "C" {

int ann_flat_query(ann_flat* h, ann_workspace* ws, const float* queries, int32_t nq, int64_t ldq, int32_t k,
                   int32_t mode, int32_t mem, int64_t* out_ids, float* out_dists, void* stream) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr, "ann_flat_query: null index");
    if (h->base == nullptr || h->n == 0) {
        set_error("index not fitted");
        return ANN_ERR_STATE;
    }
    ANN_CHECK_ARG(nq >= 0, "ann_flat_query: nq=%d < 0", nq);
    ANN_CHECK_ARG(k >= 1, "ann_flat_query: k=%d < 1", k);
    ANN_CHECK_ARG(ldq >= h->dim, "ann_flat_query: query stride %lld < dim %d", (long long)ldq, h->dim);
    ANN_CHECK_ARG(mode == ANN_MODE_EXACT || mode == ANN_MODE_REFERENCE, "ann_flat_query: unknown mode %d", mode);
    ANN_CHECK_ARG(mode == ANN_MODE_EXACT || h->metric == ANN_METRIC_L2,
                  "ann_flat_query: the reference ranking is defined for squared L2 only");
    ANN_CHECK_ARG(nq == 0 || (queries != nullptr && out_ids != nullptr), "ann_flat_query: null pointer");
    if (nq == 0) return ANN_OK;
    const int kk = (int)std::min<int64_t>(k, h->n);
    if (kk > 512) {
        set_error("ann_flat_query: k=%d > 512 is not supported by the fused selection", kk);
        return ANN_ERR_UNSUPPORTED;
    }
    if (!ws) ws = &h->ws;
    DeviceGuard g(h->device);
    cudaStream_t st = as_stream(stream);
    const int dpad = h->dpad;
    const bool host = mem == ANN_MEM_HOST;
    const bool need_pad = host || (mode == ANN_MODE_EXACT && (ldq != dpad || (reinterpret_cast<uintptr_t>(queries) & 15)));

    // ---- plan the scratch: [padded queries][device outputs][search scratch] ----
    int bq = 0, nsplit = 0, qc = 0, ncp = 0;
    int64_t rps = 0;
    Sizer sz;
    if (need_pad) sz.take<float>((size_t)nq * dpad);
    if (host) {
        sz.take<int64_t>((size_t)nq * kk);
        sz.take<float>((size_t)nq * kk);
    }
    if (mode == ANN_MODE_EXACT) {
        bq = std::min(flat_scan_bq(nq), flat_scan_max_bq(kk));
        nsplit = flat_choose_nsplit(h->n, nq, bq, &rps);
        sz.take<float>((size_t)nq * nsplit * kk);
        sz.take<int>((size_t)nq * nsplit * kk);
    } else {
        ncp = compat_num_checkpoints(h->dim);
        const size_t per_q = sizeof(float) * (size_t)h->n * (ncp + 1);
        const size_t budget = (size_t)1 << 30;
        qc = (int)std::max<size_t>(1, std::min<size_t>((size_t)nq, budget / per_q));
        sz.take<float>((size_t)qc * h->n);
        sz.take<float>((size_t)qc * h->n * ncp);
    }
    int rc = ws_reserve_device(ws, sz.bytes());
    if (rc) return rc;
    Carver cv(ws->dev);
    float* qdev = const_cast<float*>(queries);
    int64_t ldq_dev = ldq;
    if (need_pad) {
        qdev = cv.take<float>((size_t)nq * dpad);
        ldq_dev = dpad;
    }
    int64_t* ids_dev = out_ids;
    float* dists_dev = out_dists;
    if (host) {
        ids_dev = cv.take<int64_t>((size_t)nq * kk);
        dists_dev = cv.take<float>((size_t)nq * kk);
    }

    // ---- queries in ----
    if (host) {
        const size_t qbytes = sizeof(float) * (size_t)nq * dpad;
        rc = ws_reserve_host(ws, std::max(qbytes, (sizeof(int64_t) + sizeof(float)) * (size_t)nq * kk));
        if (rc) return rc;
        float* hq = reinterpret_cast<float*>(ws->host);
        for (int i = 0; i < nq; ++i) {
            std::memcpy(hq + (size_t)i * dpad, queries + (size_t)i * ldq, sizeof(float) * h->dim);
            if (dpad > h->dim) std::memset(hq + (size_t)i * dpad + h->dim, 0, sizeof(float) * (dpad - h->dim));
        }
        ANN_CUDA_TRY(cudaMemcpyAsync(qdev, hq, qbytes, cudaMemcpyHostToDevice, st));
    } else if (need_pad) {
        rc = launch_pad_rows(queries, nq, h->dim, ldq, qdev, dpad, st);
        if (rc) return rc;
    }

    // ---- search ----
    const int prec = h->prof.begin(st);
    if (mode == ANN_MODE_EXACT) {
        float* skey = cv.take<float>((size_t)nq * nsplit * kk);
        int* sid = cv.take<int>((size_t)nq * nsplit * kk);
        FlatScanArgs a{h->base, h->n, dpad, qdev, nq, h->metric, kk, rps, nsplit, skey, sid};
        rc = launch_flat_scan(a, bq, st);
        if (rc) return rc;
        h->prof.mark(prec, st);
        MergeArgs m{skey, sid, nq, nsplit, kk, kk, h->metric == ANN_METRIC_IP ? 1 : 0, ids_dev, dists_dev};
        rc = launch_merge_splits(m, st);
        if (rc) return rc;
        h->prof.mark(prec, st);
        if (prec >= 0) h->prof.launches += 1;
    } else {
        CompatArgs a{};
        a.base = h->base;
        a.n = h->n;
        a.dim = h->dim;
        a.ldb = dpad;
        a.q = qdev;
        a.ldq = ldq_dev;
        a.k = kk;
        a.ncp = ncp;
        a.D = cv.take<float>((size_t)qc * h->n);
        a.P = cv.take<float>((size_t)qc * h->n * ncp);
        a.out_ids = ids_dev;
        a.out_dists = dists_dev;
        for (int q0 = 0; q0 < nq; q0 += qc) {
            rc = launch_compat(a, q0, std::min(qc, nq - q0), st);
            if (rc) return rc;
        }
    }
    h->ndist.fetch_add(h->n * (int64_t)nq);

    // ---- results out ----
    if (host) {
        int64_t* hid = reinterpret_cast<int64_t*>(ws->host);
        float* hd = reinterpret_cast<float*>(ws->host + sizeof(int64_t) * (size_t)nq * kk);
        ANN_CUDA_TRY(cudaMemcpyAsync(hid, ids_dev, sizeof(int64_t) * (size_t)nq * kk, cudaMemcpyDeviceToHost, st));
        if (out_dists)
            ANN_CUDA_TRY(cudaMemcpyAsync(hd, dists_dev, sizeof(float) * (size_t)nq * kk, cudaMemcpyDeviceToHost, st));
        ANN_CUDA_TRY(cudaStreamSynchronize(st));
        std::memcpy(out_ids, hid, sizeof(int64_t) * (size_t)nq * kk);
        if (out_dists) std::memcpy(out_dists, hd, sizeof(float) * (size_t)nq * kk);
    }
    return ANN_OK;
}

int ann_flat_set_profiling(ann_flat* h, int32_t enable) {
    ANN_CHECK_ARG(h != nullptr, "null index");
    h->prof.enabled = enable != 0;
    return ANN_OK;
}

int ann_flat_profile(ann_flat* h, double* out4) {
    ANN_CHECK_ARG(h != nullptr && out4 != nullptr, "null argument");
    DeviceGuard g(h->device);
    h->prof.collect();
    out4[0] = h->prof.total_ms[0];
    out4[1] = h->prof.total_ms[1];
    out4[2] = (double)h->prof.launches;
    out4[3] = (double)h->prof.calls;
    return ANN_OK;
}

int ann_flat_reset_profile(ann_flat* h) {
    ANN_CHECK_ARG(h != nullptr, "null index");
    DeviceGuard g(h->device);
    h->prof.reset();
    return ANN_OK;
}

// BF16 copy of the base (and FP32 row norms) for the tensor-core scan, built once.
static int flat_ensure_bf16(ann_flat* h, cudaStream_t st) {
    if (h->base_bf16) return ANN_OK;
    const int kpad = (int)ceil_div(h->dim, 64) * 64;
    __nv_bfloat16* b = nullptr;
    float* nr = nullptr;
    int* err = nullptr;
    cudaError_t e = cudaMalloc(&b, sizeof(__nv_bfloat16) * (size_t)h->n * kpad);
    if (e == cudaSuccess) e = cudaMalloc(&nr, sizeof(float) * (size_t)h->n);
    if (e == cudaSuccess && !h->d_err) e = cudaMalloc(&err, sizeof(int));
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (b) cudaFree(b);
        if (nr) cudaFree(nr);
        if (err) cudaFree(err);
        set_error("tensor-core scan: cannot allocate the BF16 copy of the base (%s)", cudaGetErrorString(e));
        return ANN_ERR_NOMEM;
    }
    if (err) {
        ANN_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
        h->d_err = err;
    }
    int rc = launch_to_bf16(h->base, h->n, h->dim, h->dpad, b, kpad, nr, st);
    if (rc) return rc;
    ANN_CUDA_TRY(cudaStreamSynchronize(st));
    h->base_bf16 = b;
    h->norms = nr;
    h->kpad = kpad;
    return ANN_OK;
}

static int flat_check_err(ann_flat* h) {
    int v = 0;
    if (!h->d_err) return ANN_OK;
    ANN_CUDA_TRY(cudaMemcpy(&v, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (v) {
        ANN_CUDA_TRY(cudaMemset(h->d_err, 0, sizeof(int)));
        set_error("a device-side wait gave up after its time limit; the results are invalid");
        return ANN_ERR_TIMEOUT;
    }
    return ANN_OK;
}

int ann_flat_scores_tc(ann_flat* h, const float* queries, int32_t nq, int64_t ldq, float* out_keys, void* stream) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr && h->base != nullptr, "ann_flat_scores_tc: index not fitted");
    ANN_CHECK_ARG(nq >= 0 && ldq >= h->dim && (nq == 0 || (queries && out_keys)), "ann_flat_scores_tc: bad arguments");
    if (nq == 0) return ANN_OK;
    DeviceGuard g(h->device);
    cudaStream_t st = as_stream(stream);
    int rc = flat_ensure_bf16(h, st);
    if (rc) return rc;
    Sizer sz;
    sz.take<__nv_bfloat16>((size_t)nq * h->kpad);
    rc = ws_reserve_device(&h->ws, sz.bytes());
    if (rc) return rc;
    Carver cv(h->ws.dev);
    __nv_bfloat16* qb = cv.take<__nv_bfloat16>((size_t)nq * h->kpad);
    if ((rc = launch_to_bf16(queries, nq, h->dim, ldq, qb, h->kpad, nullptr, st))) return rc;
    TcGemmArgs a{nq, (int)h->n, h->kpad, nullptr, h->norms, h->metric, out_keys, h->n, h->d_err};
    if ((rc = launch_tc_gemm(qb, h->base_bf16, a, st))) return rc;
    ANN_CUDA_TRY(cudaStreamSynchronize(st));
    return flat_check_err(h);
}

int ann_flat_query_tc(ann_flat* h, ann_workspace* ws, const float* queries, int32_t nq, int64_t ldq, int32_t k,
                      int32_t refine_r, int32_t mem, int64_t* out_ids, float* out_dists, void* stream) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr, "ann_flat_query_tc: null index");
    if (h->base == nullptr || h->n == 0) {
        set_error("index not fitted");
        return ANN_ERR_STATE;
    }
    ANN_CHECK_ARG(nq >= 0 && k >= 1, "ann_flat_query_tc: nq=%d, k=%d", nq, k);
    ANN_CHECK_ARG(ldq >= h->dim, "ann_flat_query_tc: query stride < dim");
    ANN_CHECK_ARG(nq == 0 || (queries && out_ids), "ann_flat_query_tc: null pointer");
    if (nq == 0) return ANN_OK;
    const int kk = (int)std::min<int64_t>(k, h->n);
    const int R = (int)std::min<int64_t>(std::max(kk, refine_r > 0 ? refine_r : 4 * kk), h->n);
    ANN_CHECK_ARG(kk <= 1024 && R <= 8192, "ann_flat_query_tc: k=%d, refine %d too large", kk, R);
    if (!ws) ws = &h->ws;
    DeviceGuard g(h->device);
    cudaStream_t st = as_stream(stream);
    int rc = flat_ensure_bf16(h, st);
    if (rc) return rc;
    const int dpad = h->dpad, kpad = h->kpad;
    const bool host = mem == ANN_MEM_HOST;
    // key matrix chunk: queries per pass bounded by ~4 GB of FP32 keys
    const size_t budget = (size_t)4 << 30;
    int qc = (int)std::max<int64_t>(128, (int64_t)(budget / (sizeof(float) * (size_t)h->n)) / 128 * 128);
    qc = std::min(qc, nq);
    Sizer sz;
    sz.take<float>((size_t)nq * dpad);
    sz.take<__nv_bfloat16>((size_t)nq * kpad);
    sz.take<float>((size_t)nq * R);
    sz.take<int>((size_t)nq * R);
    if (host) {
        sz.take<int64_t>((size_t)nq * kk);
        sz.take<float>((size_t)nq * kk);
    }
    if ((rc = ws_reserve_device(ws, sz.bytes()))) return rc;
    if ((rc = ws_reserve_big(ws, sizeof(float) * (size_t)qc * h->n))) return rc;
    Carver cv(ws->dev);
    float* qdev = cv.take<float>((size_t)nq * dpad);
    __nv_bfloat16* qb = cv.take<__nv_bfloat16>((size_t)nq * kpad);
    float* keyR = cv.take<float>((size_t)nq * R);
    int* idR = cv.take<int>((size_t)nq * R);
    int64_t* ids_dev = out_ids;
    float* dists_dev = out_dists;
    if (host) {
        ids_dev = cv.take<int64_t>((size_t)nq * kk);
        dists_dev = cv.take<float>((size_t)nq * kk);
        if ((rc = ws_reserve_host(ws, std::max(sizeof(float) * (size_t)nq * dpad, (sizeof(int64_t) + 4) * (size_t)nq * kk))))
            return rc;
        float* hq = reinterpret_cast<float*>(ws->host);
        for (int i = 0; i < nq; ++i) {
            std::memcpy(hq + (size_t)i * dpad, queries + (size_t)i * ldq, sizeof(float) * h->dim);
            if (dpad > h->dim) std::memset(hq + (size_t)i * dpad + h->dim, 0, sizeof(float) * (dpad - h->dim));
        }
        ANN_CUDA_TRY(cudaMemcpyAsync(qdev, hq, sizeof(float) * (size_t)nq * dpad, cudaMemcpyHostToDevice, st));
    } else {
        if ((rc = launch_pad_rows(queries, nq, h->dim, ldq, qdev, dpad, st))) return rc;
    }
    if ((rc = launch_to_bf16(qdev, nq, h->dim, dpad, qb, kpad, nullptr, st))) return rc;
    float* keys = reinterpret_cast<float*>(ws->big);
    const int prec = h->prof.begin(st);
    for (int q0 = 0; q0 < nq; q0 += qc) {
        const int nc = std::min(qc, nq - q0);
        TcGemmArgs a{nc, (int)h->n, kpad, nullptr, h->norms, h->metric, keys, h->n, h->d_err};
        if ((rc = launch_tc_gemm(qb + (size_t)q0 * kpad, h->base_bf16, a, st))) return rc;
        if ((rc = launch_select_topk(keys, h->n, nullptr, nc, R, nullptr, keyR + (size_t)q0 * R, idR + (size_t)q0 * R, st)))
            return rc;
    }
    h->prof.mark(prec, st);
    IvfQueryArgs ra{};
    ra.ix.n = h->n;
    ra.ix.dim = h->dim;
    ra.ix.dpad = dpad;
    ra.ix.original = h->base;
    ra.ix.r2o = nullptr;
    ra.plan.nq = nq;
    ra.q = qdev;
    ra.ldq = dpad;
    ra.k = kk;
    ra.R = R;
    ra.metric = h->metric;
    ra.out_ids = ids_dev;
    ra.out_dists = dists_dev;
    if ((rc = launch_ivf_rerank(ra, keyR, idR, 0, st))) return rc;
    h->prof.mark(prec, st);
    if (prec >= 0) h->prof.launches += 1;
    h->ndist.fetch_add(h->n * (int64_t)nq);
    if (host) {
        int64_t* hid = reinterpret_cast<int64_t*>(ws->host);
        float* hd = reinterpret_cast<float*>(ws->host + sizeof(int64_t) * (size_t)nq * kk);
        ANN_CUDA_TRY(cudaMemcpyAsync(hid, ids_dev, sizeof(int64_t) * (size_t)nq * kk, cudaMemcpyDeviceToHost, st));
        if (out_dists)
            ANN_CUDA_TRY(cudaMemcpyAsync(hd, dists_dev, sizeof(float) * (size_t)nq * kk, cudaMemcpyDeviceToHost, st));
        ANN_CUDA_TRY(cudaStreamSynchronize(st));
        std::memcpy(out_ids, hid, sizeof(int64_t) * (size_t)nq * kk);
        if (out_dists) std::memcpy(out_dists, hd, sizeof(float) * (size_t)nq * kk);
        return flat_check_err(h);
    }
    return ANN_OK;
}

int ann_flat_device_status(ann_flat* h) {
    ANN_CHECK_ARG(h != nullptr, "null index");
    DeviceGuard g(h->device);
    return flat_check_err(h);
}

int64_t ann_flat_total_distances(const ann_flat* h) { return h ? h->ndist.load() : 0; }
int32_t ann_flat_dim(const ann_flat* h) { return h ? h->dim : 0; }
int64_t ann_flat_size(const ann_flat* h) { return h ? h->n : 0; }

}  // extern "C"

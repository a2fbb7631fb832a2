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
#include "tc_search.cuh"
#include "radix_select.cuh"

namespace annb {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
void clear_error() { g_err[0] = 0; }

int queries_in(float* dev, int64_t dpad, const float* host, int64_t ld, int64_t rows, int cols, cudaStream_t st) {
    if (rows == 0) return ANN_OK;
    ANN_CUDA_TRY(cudaMemcpy2DAsync(dev, sizeof(float) * dpad, host, sizeof(float) * ld, sizeof(float) * cols, rows,
                                   cudaMemcpyHostToDevice, st));
    if (dpad > cols)
        ANN_CUDA_TRY(cudaMemset2DAsync(dev + cols, sizeof(float) * dpad, 0, sizeof(float) * (dpad - cols), rows, st));
    return ANN_OK;
}

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

int ws_pinned(ann_workspace* ws, int64_t** out) {
    std::lock_guard<std::mutex> lk(ws->mu);
    if (!ws->pinned) {
        void* p = nullptr;
        const cudaError_t e = cudaHostAlloc(&p, 8 * sizeof(int64_t), cudaHostAllocDefault);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error("workspace: cannot allocate page-locked host words (%s)", cudaGetErrorString(e));
            return ANN_ERR_NOMEM;
        }
        ws->pinned = static_cast<int64_t*>(p);
    }
    *out = ws->pinned;
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

}  // namespace annb

using namespace annb;


// An empty kernel compiled with the library's flags: its attributes are the library's code form.
__global__ void arch_probe_kernel() {}

extern "C" {

const char* ann_version(void) { return "annvedi_b200 0.1 sm_100a"; }

int ann_tc_wait_selftest(int device, int64_t wait_ns, int32_t* flag_out) {
    clear_error();
    ANN_CHECK_ARG(flag_out != nullptr, "ann_tc_wait_selftest: flag_out is NULL");
    ANN_CHECK_ARG(wait_ns >= 1000 && wait_ns <= 2000000000LL, "ann_tc_wait_selftest: wait_ns=%lld outside [1e3, 2e9]",
                  (long long)wait_ns);
    DeviceGuard g(device);
    if (!g.ok) {
        cudaGetLastError();
        set_error("ann_tc_wait_selftest: device %d not usable", device);
        return ANN_ERR_CUDA;
    }
    int flag = -1;
    const int rc = tc_wait_selftest((uint64_t)wait_ns, &flag);
    *flag_out = flag;
    return rc;
}

int ann_kernel_arch(int device, int32_t* out2) {
    clear_error();
    ANN_CHECK_ARG(out2 != nullptr, "ann_kernel_arch: out2 is NULL");
    DeviceGuard g(device);
    if (!g.ok) {
        cudaGetLastError();
        set_error("ann_kernel_arch: device %d not usable", device);
        return ANN_ERR_CUDA;
    }
    cudaFuncAttributes fa{};
    ANN_CUDA_TRY(cudaFuncGetAttributes(&fa, arch_probe_kernel));
    out2[0] = fa.binaryVersion;
    out2[1] = fa.ptxVersion;
    return ANN_OK;
}
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
    if (ws->big) cudaFree(ws->big);
    if (ws->pinned) cudaFreeHost(ws->pinned);
    ws->pinned = nullptr;
    ws->dev = nullptr;
    ws->big = nullptr;
    ws->dev_cap = ws->big_cap = 0;
}

int ann_workspace_destroy(ann_workspace* ws) {
    if (!ws) return ANN_OK;
    ws_release(ws);
    delete ws;
    return ANN_OK;
}

int64_t ann_workspace_bytes(const ann_workspace* ws) { return ws ? (int64_t)(ws->dev_cap + ws->big_cap) : 0; }

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
        if (h->base_e4m3) cudaFree(h->base_e4m3);
        if (h->fac_e4m3) cudaFree(h->fac_e4m3);
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
    if (h->base_e4m3) {
        ANN_CUDA_TRY(cudaFree(h->base_e4m3));
        ANN_CUDA_TRY(cudaFree(h->fac_e4m3));
        h->base_e4m3 = nullptr;
        h->fac_e4m3 = nullptr;
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
int annb::flat_choose_nsplit(int64_t n, int nq, int bq, int64_t* rows_per_split, int ctas_per_sm) {
    // Choose the splits per query tile so that (query tiles x splits) fills whole waves of
    // kNumSMs * ctas_per_sm CTAs, with a small charge per split for the merge.
    const int64_t wave = (int64_t)kNumSMs * std::max(1, ctas_per_sm);
    const int64_t n_qtiles = ceil_div(nq, bq);
    const int64_t tile = 256;
    const int64_t max_split = std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 2 * tile), 4 * wave));
    int64_t best_s = 1;
    double best = 1e300;
    for (int64_t s = 1; s <= max_split; ++s) {
        const int64_t ctas = n_qtiles * s;
        const int64_t waves = ceil_div(ctas, wave);
        const double cost = (double)waves * wave / (double)ctas * (1.0 + 0.002 * (double)s);
        if (cost < best - 1e-12) {
            best = cost;
            best_s = s;
        }
    }
    int64_t rps = ceil_div(ceil_div(n, best_s), tile) * tile;
    const int64_t nsplit = ceil_div(n, rps);
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
    bool radix_merge = false;
    if (mode == ANN_MODE_EXACT) {
        bq = std::min(h->query_tile > 0 ? h->query_tile : flat_scan_bq(nq), flat_scan_max_bq(kk));
        nsplit = flat_choose_nsplit(h->n, nq, bq, &rps, flat_scan_ctas_per_sm(bq, kk, dpad, h->metric));
        sz.take<float>((size_t)nq * nsplit * kk);
        sz.take<int>((size_t)nq * nsplit * kk);
        sz.take<float>((size_t)(nq + 1) / 2 * 2 * dpad);  // the paired query tile
        // many splits per query: select the k best with the radix selection, then sort them
        radix_merge = nsplit >= 16;
        if (radix_merge) {
            sz.take<float>((size_t)nq * kk);
            sz.take<int>((size_t)nq * kk);
        }
    } else {
        ncp = compat_num_checkpoints(h->dim);
        const size_t per_q = sizeof(float) * (size_t)h->n * (ncp + 2) + (size_t)8 * kk;
        const size_t budget = (size_t)1 << 30;
        qc = (int)std::max<size_t>(1, std::min<size_t>((size_t)nq, budget / per_q));
        sz.take<float>((size_t)qc * h->n);
        sz.take<float>((size_t)qc * h->n * ncp);
        sz.take<float>((size_t)qc * h->n);
        sz.take<float>((size_t)qc * kk);
        sz.take<int>((size_t)qc * kk);
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
        if ((rc = queries_in(qdev, dpad, queries, ldq, nq, h->dim, st))) return rc;
    } else if (need_pad) {
        rc = launch_pad_rows(queries, nq, h->dim, ldq, qdev, dpad, st);
        if (rc) return rc;
    }

    // ---- search ----
    const int prec = h->prof.begin(st);
    if (mode == ANN_MODE_EXACT) {
        float* skey = cv.take<float>((size_t)nq * nsplit * kk);
        int* sid = cv.take<int>((size_t)nq * nsplit * kk);
        float* qpair = cv.take<float>((size_t)(nq + 1) / 2 * 2 * dpad);
        FlatScanArgs a{h->base, h->n, dpad, qdev, nq, h->metric, kk, rps, nsplit, skey, sid};
        a.qpair = qpair;
        rc = launch_flat_scan(a, bq, st);
        if (rc) return rc;
        h->prof.mark(prec, st);
        if (radix_merge) {
            float* mkey = cv.take<float>((size_t)nq * kk);
            int* mid = cv.take<int>((size_t)nq * kk);
            RadixSelectArgs rs{};
            rs.keys = skey;
            rs.ld = (int64_t)nsplit * kk;
            rs.ids = sid;
            rs.R = kk;
            rs.out_key = mkey;
            rs.out_id = mid;
            if ((rc = launch_radix_select(rs, nq, st))) return rc;
            rc = launch_sort_topk(mkey, mid, nq, kk, h->metric == ANN_METRIC_IP ? 1 : 0, ids_dev, dists_dev, st);
        } else {
            MergeArgs m{skey, sid, nq, nsplit, kk, kk, h->metric == ANN_METRIC_IP ? 1 : 0, ids_dev, dists_dev};
            rc = launch_merge_splits(m, st);
        }
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
        a.T = cv.take<float>((size_t)qc * h->n);
        a.kbuf = cv.take<float>((size_t)qc * kk);
        a.ibuf = cv.take<int>((size_t)qc * kk);
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
        ANN_CUDA_TRY(cudaMemcpyAsync(out_ids, ids_dev, sizeof(int64_t) * (size_t)nq * kk, cudaMemcpyDeviceToHost, st));
        if (out_dists)
            ANN_CUDA_TRY(cudaMemcpyAsync(out_dists, dists_dev, sizeof(float) * (size_t)nq * kk, cudaMemcpyDeviceToHost, st));
        ANN_CUDA_TRY(cudaStreamSynchronize(st));
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

int ann_flat_profile_stages(ann_flat* h, double* out10) {
    ANN_CHECK_ARG(h != nullptr && out10 != nullptr, "null argument");
    DeviceGuard g(h->device);
    h->prof.collect();
    for (int i = 0; i < 6; ++i) out10[i] = h->prof.total_ms[i];
    out10[6] = (double)h->prof.launches;
    out10[7] = (double)h->prof.tc_launches;
    out10[8] = (double)h->prof.filter_launches;
    out10[9] = (double)h->prof.calls;
    return ANN_OK;
}

int ann_flat_reset_profile(ann_flat* h) {
    ANN_CHECK_ARG(h != nullptr, "null index");
    DeviceGuard g(h->device);
    h->prof.reset();
    return ANN_OK;
}

// BF16 operand form of the base for the tensor-core scan (key columns included, rows in the Weyl
// order of tc_row_mult), built once.
static int flat_ensure_bf16(ann_flat* h, cudaStream_t st) {
    if (h->base_bf16) return ANN_OK;
    const int kpad = tc_kpad(h->dim, h->metric);
    __nv_bfloat16* b = nullptr;
    int* err = nullptr;
    cudaError_t e = cudaMalloc(&b, sizeof(__nv_bfloat16) * (size_t)h->n * kpad);
    if (e == cudaSuccess && !h->d_err) e = cudaMalloc(&err, sizeof(int));
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (b) cudaFree(b);
        if (err) cudaFree(err);
        set_error("tensor-core scan: cannot allocate the BF16 copy of the base (%s)", cudaGetErrorString(e));
        return ANN_ERR_NOMEM;
    }
    if (err) {
        ANN_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
        h->d_err = err;
    }
    const int64_t mult = tc_row_mult(h->n);
    int rc = launch_tc_operand(h->base, h->n, h->dim, h->dpad, b, kpad, kTcBase, h->metric, mult, st);
    if (rc) return rc;
    ANN_CUDA_TRY(cudaStreamSynchronize(st));
    h->base_bf16 = b;
    h->row_mult = mult;
    h->kpad = kpad;
    return ANN_OK;
}

// E4M3 operand form of the base (per-row scales, same Weyl order), built once.
static int flat_ensure_e4m3(ann_flat* h, cudaStream_t st) {
    if (h->base_e4m3) return ANN_OK;
    int rc = flat_ensure_bf16(h, st);  // the row order and the error flag
    if (rc) return rc;
    const int kpad8 = (int)ceil_div(h->dim, 32) * 32;
    uint8_t* b = nullptr;
    float2* f = nullptr;
    cudaError_t e = cudaMalloc(&b, (size_t)h->n * kpad8);
    if (e == cudaSuccess) e = cudaMalloc(&f, sizeof(float2) * (size_t)h->n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (b) cudaFree(b);
        set_error("tensor-core scan: cannot allocate the E4M3 copy of the base (%s)", cudaGetErrorString(e));
        return ANN_ERR_NOMEM;
    }
    rc = launch_tc_operand_e4m3(h->base, h->n, h->dim, h->dpad, b, kpad8, kTcBase, h->metric, h->row_mult, nullptr, f,
                                st);
    if (rc) {
        cudaFree(b);
        cudaFree(f);
        return rc;
    }
    ANN_CUDA_TRY(cudaStreamSynchronize(st));
    h->base_e4m3 = b;
    h->fac_e4m3 = f;
    h->kpad8 = kpad8;
    return ANN_OK;
}

// The tensor-core operands of the index's current element kind.
struct FlatTc {
    int kind, kpad;
    size_t es;  // bytes per element
    const void* base;
    const float2* cfac;
};
static int flat_ensure_tc(ann_flat* h, cudaStream_t st, FlatTc* t) {
    int rc = h->tc_kind == kTcE4M3 ? flat_ensure_e4m3(h, st) : flat_ensure_bf16(h, st);
    if (rc) return rc;
    t->kind = h->tc_kind;
    t->kpad = t->kind == kTcE4M3 ? h->kpad8 : h->kpad;
    t->es = t->kind == kTcE4M3 ? 1 : 2;
    t->base = t->kind == kTcE4M3 ? (const void*)h->base_e4m3 : (const void*)h->base_bf16;
    t->cfac = t->kind == kTcE4M3 ? h->fac_e4m3 : nullptr;
    return ANN_OK;
}
// Queries to the operand form: E4M3 rows with their scales into rfac, or BF16 rows.
static int flat_tc_queries(const ann_flat* h, const FlatTc& t, const float* q, int nq, int64_t ldq, void* out,
                           float* rfac, cudaStream_t st) {
    if (t.kind == kTcE4M3)
        return launch_tc_operand_e4m3(q, nq, h->dim, ldq, static_cast<uint8_t*>(out), t.kpad, kTcQuery, h->metric, 0,
                                      rfac, nullptr, st);
    return launch_tc_operand(q, nq, h->dim, ldq, static_cast<__nv_bfloat16*>(out), t.kpad, kTcQuery, h->metric, 0, st);
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
    FlatTc t;
    int rc = flat_ensure_tc(h, st, &t);
    if (rc) return rc;
    Sizer sz;
    sz.take<unsigned char>((size_t)nq * t.kpad * t.es);
    sz.take<float>((size_t)nq);
    if ((rc = ws_reserve_device(&h->ws, sz.bytes()))) return rc;
    if ((rc = ws_reserve_big(&h->ws, sizeof(float) * (size_t)nq * h->n))) return rc;
    Carver cv(h->ws.dev);
    unsigned char* qb = cv.take<unsigned char>((size_t)nq * t.kpad * t.es);
    float* rfac = cv.take<float>((size_t)nq);
    float* tmp = reinterpret_cast<float*>(h->ws.big);
    if ((rc = flat_tc_queries(h, t, queries, nq, ldq, qb, rfac, st))) return rc;
    TcGemmArgs a{nq, (int)h->n, t.kpad, nullptr, tmp, h->n, h->d_err};
    a.kind = t.kind;
    a.col_fac = t.cfac;
    a.row_fac = t.kind == kTcE4M3 ? rfac : nullptr;
    if ((rc = launch_tc_gemm(qb, t.base, a, st))) return rc;
    if ((rc = launch_tc_unpermute(tmp, nq, h->n, h->row_mult, out_keys, st))) return rc;
    ANN_CUDA_TRY(cudaStreamSynchronize(st));
    return flat_check_err(h);
}

int ann_flat_set_option(ann_flat* h, int32_t option, int64_t value) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr, "ann_flat_set_option: null index");
    switch (option) {
        case ANN_FLAT_OPT_QUERY_TILE:
            ANN_CHECK_ARG(value == 0 || value == 8 || value == 16 || value == 32,
                          "ann_flat_set_option: query tile %lld (0, 8, 16 or 32)", (long long)value);
            h->query_tile = (int)value;
            return ANN_OK;
        default:
            set_error("ann_flat_set_option: unknown option %d", option);
            return ANN_ERR_INVALID;
    }
}

int ann_flat_set_tc_precision(ann_flat* h, int32_t precision) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr, "ann_flat_set_tc_precision: null index");
    ANN_CHECK_ARG(precision == ANN_TC_BF16 || precision == ANN_TC_E4M3, "ann_flat_set_tc_precision: %d", precision);
    h->tc_kind = precision == ANN_TC_E4M3 ? kTcE4M3 : kTcBF16;
    return ANN_OK;
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
    FlatTc t;
    int rc = flat_ensure_tc(h, st, &t);
    if (rc) return rc;
    const int dpad = h->dpad, kpad = t.kpad;
    const size_t rowb = (size_t)kpad * t.es;  // bytes of an operand row
    const bool e4 = t.kind == kTcE4M3;
    const bool host = mem == ANN_MEM_HOST;
    Sizer sz;
    sz.take<float>((size_t)nq * dpad);
    sz.take<unsigned char>((size_t)nq * rowb);
    sz.take<float>((size_t)nq);
    sz.take<float>((size_t)nq * R);
    sz.take<int>((size_t)nq * R);
    if (host) {
        sz.take<int64_t>((size_t)nq * kk);
        sz.take<float>((size_t)nq * kk);
    }
    if ((rc = ws_reserve_device(ws, sz.bytes()))) return rc;
    Carver cv(ws->dev);
    float* qdev = cv.take<float>((size_t)nq * dpad);
    unsigned char* qb = cv.take<unsigned char>((size_t)nq * rowb);
    float* rfac = cv.take<float>((size_t)nq);
    float* keyR = cv.take<float>((size_t)nq * R);
    int* idR = cv.take<int>((size_t)nq * R);
    int64_t* ids_dev = out_ids;
    float* dists_dev = out_dists;
    if (host) {
        ids_dev = cv.take<int64_t>((size_t)nq * kk);
        dists_dev = cv.take<float>((size_t)nq * kk);
        if ((rc = queries_in(qdev, dpad, queries, ldq, nq, h->dim, st))) return rc;
    } else {
        if ((rc = launch_pad_rows(queries, nq, h->dim, ldq, qdev, dpad, st))) return rc;
    }
    if ((rc = flat_tc_queries(h, t, qdev, nq, dpad, qb, rfac, st))) return rc;
    // Sampled bars: keys over a strided sample of S positions of the BF16 copy (an even sample of the
    // base, by its row order) give each query two bars. The safe bar, its R-th best sampled key, is at
    // or above its R-th best key over all rows (about n * R / S keys pass it). The fast bar, its rF-th
    // best sampled key with rF ~ 3 R S / n, lets about 3 R keys pass. The full pass keeps the keys
    // under the fast bar; a query with fewer than R survivors (the count is exact) is re-run under its
    // safe bar, so every query ends with its best R keys among its survivors. Small bases, or a
    // survivor overflow, use the full key matrix.
    const int64_t n = h->n;
    const int64_t full_tiles = n / 256;
    const int64_t want_tiles = std::max<int64_t>(128, ceil_div(16 * (int64_t)R, 256));
    const bool sampled = full_tiles >= 4 * want_tiles;
    const int stride = sampled ? (int)(full_tiles / want_tiles) : 1;
    const int64_t S = sampled ? (full_tiles / stride) * 256 : 0;
    const int rF = sampled ? (int)std::min<int64_t>(R, std::max<int64_t>(1, ceil_div(3 * (int64_t)R * S, n))) : 0;
    constexpr int kRerunBatch = 128;
    // queries per chunk: ~2 GB of sampled keys, or ~4 GB of full key matrix
    const int64_t qfull64 = std::max<int64_t>(128, ((int64_t)4 << 30) / (int64_t)(sizeof(float) * n) / 128 * 128);
    const int qfull = (int)std::min<int64_t>(qfull64, 65535);
    const int qmax = sampled ? (int)std::clamp<int64_t>(((int64_t)2 << 30) / (4 * S) / 128 * 128, 128, 8192) : qfull;
    const int nchunks = (int)ceil_div(nq, qmax);
    const int qc = (int)std::min<int64_t>(qmax, ceil_div(ceil_div(nq, nchunks), 128) * 128);
    for (int q0 = 0; q0 < nq; q0 += qc) {
        const int nc = std::min(qc, nq - q0);
        const unsigned char* qbc = qb + (size_t)q0 * rowb;
        const float* rfc = e4 ? rfac + q0 : nullptr;
        float* keyRc = keyR + (size_t)q0 * R;
        int* idRc = idR + (size_t)q0 * R;
        bool done = false;
        if (sampled) {
            const int nwarps = tc_filter_warps(nc, (int)n);
            const int64_t main_total = ceil_div((int64_t)nc * rF * n, S);
            const int64_t rerun_total = ceil_div((int64_t)std::min(nc, kRerunBatch) * R * n, S);
            const int64_t wcap64 = 4 * ceil_div(std::max(main_total, rerun_total), nwarps) + 1024;
            const int wcap = (int)std::min<int64_t>(wcap64, INT32_MAX / std::max(1, nwarps));
            const size_t ent = (size_t)nwarps * wcap;
            Sizer s2;
            s2.take<float>((size_t)nc * S);            // sample keys
            s2.take<float>(ent);                       // survivors: key, column, row
            s2.take<int>(ent);
            s2.take<int>(ent);
            s2.take<float>(ent);                       // grouped: key, id
            s2.take<int>(ent);
            s2.take<int>((size_t)nwarps);              // warp counts
            for (int i = 0; i < 3; ++i) s2.take<float>((size_t)nc);  // fast, safe, gathered bars
            for (int i = 0; i < 3; ++i) s2.take<int>((size_t)nc);    // row counts, cursors, re-run list
            s2.take<int64_t>((size_t)nc);              // stream offsets
            s2.take<int>(4);                           // flags
            s2.take<unsigned char>((size_t)kRerunBatch * rowb);
            s2.take<float>((size_t)kRerunBatch);
            if ((rc = ws_reserve_big(ws, s2.bytes()))) return rc;
            Carver cb(ws->big);
            float* kA = cb.take<float>((size_t)nc * S);
            float* fkey = cb.take<float>(ent);
            int* fcol = cb.take<int>(ent);
            int* frow = cb.take<int>(ent);
            float* gkey = cb.take<float>(ent);
            int* gid = cb.take<int>(ent);
            int* wcnt = cb.take<int>((size_t)nwarps);
            float* tauF = cb.take<float>((size_t)nc);
            float* tauS = cb.take<float>((size_t)nc);
            float* tau2 = cb.take<float>((size_t)nc);
            int* rowcnt = cb.take<int>((size_t)nc);
            int* cursor = cb.take<int>((size_t)nc);
            int* list = cb.take<int>((size_t)nc);
            int64_t* offs = cb.take<int64_t>((size_t)nc);
            int* flags = cb.take<int>(4);
            unsigned char* A2 = cb.take<unsigned char>((size_t)kRerunBatch * rowb);
            float* rfac2 = cb.take<float>((size_t)kRerunBatch);

            // stages 2: sample pass and bars, 3: filter pass, 4: grouping, selections and re-runs
            const int prec = h->prof.begin(st, 2);
            TcGemmArgs sa{nc, (int)S, kpad, nullptr, kA, S, h->d_err};
            sa.b_tile_stride = stride;
            sa.b_rows = n;
            sa.kind = t.kind;
            sa.col_fac = t.cfac;
            sa.row_fac = rfc;
            if ((rc = launch_tc_gemm(qbc, t.base, sa, st))) return rc;
            if (sample_bars_smem((int)S) <= kSampleBarsMaxSmem) {
                if ((rc = launch_sample_bars(kA, (int)S, nc, rF, R, tauF, tauS, st))) return rc;
            } else {
                RadixSelectArgs bar{};
                bar.keys = kA;
                bar.ld = S;
                bar.R = rF;
                bar.out_kth = tauF;
                bar.R2 = R;
                bar.out_kth2 = tauS;
                bar.kth_upper = 1;
                if ((rc = launch_radix_select(bar, nc, st))) return rc;
            }
            h->prof.mark(prec, st);
            auto filter = [&](const void* A, int M, const float* tau, const float* rf) -> int {
                TcGemmArgs fa{M, (int)n, kpad, nullptr, nullptr, n, h->d_err};
                fa.kind = t.kind;
                fa.col_fac = t.cfac;
                fa.row_fac = rf;
                fa.tau = tau;
                fa.fkey = fkey;
                fa.fcol = fcol;
                fa.frow = frow;
                fa.wcount = wcnt;
                fa.wcap = wcap;
                int r = launch_tc_gemm(A, t.base, fa, st);
                if (r) return r;
                TcGroupArgs ga{fkey, fcol, frow, wcnt, tc_filter_warps(M, (int)n), wcap, M, n, h->row_mult,
                               rowcnt, offs, cursor, gkey, gid, flags + 1};
                return launch_tc_group(ga, st);
            };
            if ((rc = filter(qbc, nc, tauF, rfc))) return rc;
            h->prof.mark(prec, st);
            if (prec >= 0) h->prof.filter_launches += 1;
            ANN_CUDA_TRY(cudaMemsetAsync(flags, 0, sizeof(int), st));
            if ((rc = launch_tc_bar_check(rowcnt, nc, R, list, flags, st))) return rc;
            int hf[2] = {0, 0};  // re-runs, largest warp count
            ANN_CUDA_TRY(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
            ANN_CUDA_TRY(cudaStreamSynchronize(st));
            int ngemm = 2;
            if (hf[1] <= wcap) {
                RadixSelectArgs sv{};
                sv.keys = gkey;
                sv.ld = (int64_t)ent;
                sv.offs = offs;
                sv.lens32 = rowcnt;
                sv.ids = gid;
                sv.R = R;
                sv.out_key = keyRc;
                sv.out_id = idRc;
                if ((rc = launch_radix_select(sv, nc, st))) return rc;
                done = true;
                for (int j0 = 0; j0 < hf[0] && done; j0 += kRerunBatch) {
                    const int nb = std::min(kRerunBatch, hf[0] - j0);
                    if ((rc = launch_tc_gather(qbc, (int)rowb, list + j0, nb, tauS, A2, tau2, rfc, rfac2, st)))
                        return rc;
                    if ((rc = filter(A2, nb, tau2, e4 ? rfac2 : nullptr))) return rc;
                    ++ngemm;
                    int hmax = 0;
                    ANN_CUDA_TRY(cudaMemcpyAsync(&hmax, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
                    ANN_CUDA_TRY(cudaStreamSynchronize(st));
                    if (hmax > wcap) {
                        done = false;
                        break;
                    }
                    RadixSelectArgs sv2 = sv;
                    sv2.out_rows = list + j0;
                    if ((rc = launch_radix_select(sv2, nb, st))) return rc;
                }
            }
            h->prof.mark(prec, st);
            if (prec >= 0) h->prof.tc_launches += ngemm;
        }
        for (int f0 = 0; !done && f0 < nc; f0 += qfull) {  // the full key matrix, qfull queries at a time
            const int nf = std::min(qfull, nc - f0);
            if ((rc = ws_reserve_big(ws, sizeof(float) * (size_t)nf * n))) return rc;
            float* keys = reinterpret_cast<float*>(ws->big);
            const int prec = h->prof.begin(st, 3);  // stage 3: the full key matrix, 4: its selection
            TcGemmArgs a{nf, (int)n, kpad, nullptr, keys, n, h->d_err};
            a.kind = t.kind;
            a.col_fac = t.cfac;
            a.row_fac = e4 ? rfc + f0 : nullptr;
            if ((rc = launch_tc_gemm(qbc + (size_t)f0 * rowb, t.base, a, st))) return rc;
            h->prof.mark(prec, st);
            RadixSelectArgs fs{};
            fs.keys = keys;
            fs.ld = n;
            fs.R = R;
            fs.out_key = keyRc + (size_t)f0 * R;
            fs.out_id = idRc + (size_t)f0 * R;
            if ((rc = launch_radix_select(fs, nf, st))) return rc;
            if ((rc = launch_tc_map_ids(fs.out_id, (int64_t)nf * R, n, h->row_mult, st))) return rc;
            h->prof.mark(prec, st);
            if (prec >= 0) h->prof.tc_launches += 1;
        }
    }
    const int prec = h->prof.begin(st, 5);  // stage 5: re-rank
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
    h->ndist.fetch_add(h->n * (int64_t)nq);
    if (host) {
        ANN_CUDA_TRY(cudaMemcpyAsync(out_ids, ids_dev, sizeof(int64_t) * (size_t)nq * kk, cudaMemcpyDeviceToHost, st));
        if (out_dists)
            ANN_CUDA_TRY(cudaMemcpyAsync(out_dists, dists_dev, sizeof(float) * (size_t)nq * kk, cudaMemcpyDeviceToHost, st));
        ANN_CUDA_TRY(cudaStreamSynchronize(st));
        return flat_check_err(h);
    }
    return ANN_OK;
}

int ann_flat_device_status(ann_flat* h) {
    ANN_CHECK_ARG(h != nullptr, "null index");
    DeviceGuard g(h->device);
    return flat_check_err(h);
}

int ann_merge_topk(const float* dists, const int64_t* ids, int32_t nq, int32_t parts, int32_t k, int32_t metric,
                   int64_t* out_ids, float* out_dists, void* stream) {
    clear_error();
    ANN_CHECK_ARG(nq >= 0 && (nq == 0 || (dists && ids && out_ids)), "ann_merge_topk: null pointer");
    ANN_CHECK_ARG(metric == ANN_METRIC_L2 || metric == ANN_METRIC_IP, "ann_merge_topk: metric %d", metric);
    return launch_merge_parts(dists, ids, nq, parts, k, metric == ANN_METRIC_IP ? 1 : 0, out_ids, out_dists,
                              as_stream(stream));
}

int ann_select_smallest(const float* keys, int64_t ld, const int64_t* lens, int32_t nq, int32_t r, float* out_keys,
                        int32_t* out_pos, void* stream) {
    clear_error();
    ANN_CHECK_ARG(nq >= 0 && r >= 1 && ld >= 0 && ld < INT32_MAX, "ann_select_smallest: nq=%d r=%d ld=%lld", nq, r,
                  (long long)ld);
    ANN_CHECK_ARG(nq == 0 || (keys && out_keys && out_pos), "ann_select_smallest: null pointer");
    RadixSelectArgs a{};
    a.keys = keys;
    a.ld = ld;
    a.lens = lens;
    a.R = r;
    a.out_key = out_keys;
    a.out_id = out_pos;
    return launch_radix_select(a, nq, as_stream(stream));
}

int64_t ann_flat_total_distances(const ann_flat* h) { return h ? h->ndist.load() : 0; }
int32_t ann_flat_dim(const ann_flat* h) { return h ? h->dim : 0; }
int64_t ann_flat_size(const ann_flat* h) { return h ? h->n : 0; }

}  // extern "C"

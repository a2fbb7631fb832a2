// Exact flat search that allocates no memory of its own.
//
// Some callers cannot let a library allocate device memory: a host application that hands out every
// byte of device memory from its own pool and forbids third-party allocations, or a latency-critical
// serving thread that must never call cudaMalloc / cudaFree, because those calls can synchronise the
// whole device and take unbounded time. ann_flat_query allocates its scratch (a workspace that grows
// on demand); this entry point instead takes its scratch from one fixed array compiled into the
// library, so a call performs no allocation at all. The caller still provides the query and output
// buffers (device memory it owns).
//
// The scratch is a file-scope __device__ array of kNoAllocScratchBytes (16 MiB). Every GPU that loads
// this library keeps that much memory reserved until the process exits. All calls on a device share
// it and it keeps whatever the last call wrote; nothing in it must start at zero, because each call
// writes every scratch element it reads first. Calls whose work overlaps on the GPU (different
// streams, or different host threads) therefore overwrite each other's scratch: they must not overlap.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "flat_internal.cuh"
#include "flat_scan.cuh"
#include "runtime.cuh"

using namespace annb;

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Host code cannot use g_noalloc_scratch's name as a device address: on the host it names a host-side
// shadow. Its device address is looked up once per device, with that device current.
std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

int scratch_address(int device, void** out) {
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (device < 0 || device >= kMaxDevices) {
        set_error("ann_flat_query_noalloc: device %d outside [0, %d)", device, kMaxDevices);
        return ANN_ERR_INVALID;
    }
    if (!g_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            set_error("ann_flat_query_noalloc: cannot resolve the scratch array on device %d (%s)", device,
                      cudaGetErrorString(e));
            return ANN_ERR_CUDA;
        }
        g_addr[device] = p;
    }
    *out = g_addr[device];
    return ANN_OK;
}

}  // namespace

extern "C" int ann_flat_query_noalloc(ann_flat* h, const float* queries, int32_t nq, int64_t ldq, int32_t k,
                                      int64_t* out_ids, float* out_dists, void* stream) {
    clear_error();
    ANN_CHECK_ARG(h != nullptr, "ann_flat_query_noalloc: null index");
    if (h->base == nullptr || h->n == 0) {
        set_error("index not fitted");
        return ANN_ERR_STATE;
    }
    ANN_CHECK_ARG(nq >= 0, "ann_flat_query_noalloc: nq=%d < 0", nq);
    ANN_CHECK_ARG(k >= 1, "ann_flat_query_noalloc: k=%d < 1", k);
    ANN_CHECK_ARG(ldq >= h->dim, "ann_flat_query_noalloc: query stride %lld < dim %d", (long long)ldq, h->dim);
    ANN_CHECK_ARG(nq == 0 || (queries != nullptr && out_ids != nullptr), "ann_flat_query_noalloc: null pointer");
    if (nq == 0) return ANN_OK;
    const int kk = (int)std::min<int64_t>(k, h->n);
    if (kk > 512) {
        set_error("ann_flat_query_noalloc: k=%d > 512 is not supported by the fused selection", kk);
        return ANN_ERR_UNSUPPORTED;
    }
    DeviceGuard g(h->device);
    cudaStream_t st = as_stream(stream);
    void* base = nullptr;
    int rc = scratch_address(h->device, &base);
    if (rc) return rc;

    // Plan: padded queries (unless usable as they are) and the per-split top-k lists, shrinking the
    // number of splits until they fit the fixed array.
    const int dpad = h->dpad;
    const bool need_pad = ldq != dpad || (reinterpret_cast<uintptr_t>(queries) & 15);
    const int bq = std::min(flat_scan_bq(nq), flat_scan_max_bq(kk));
    int64_t rps = 0;
    int nsplit = flat_choose_nsplit(h->n, nq, bq, &rps);
    auto bytes_for = [&](int ns) {
        Sizer sz;
        if (need_pad) sz.take<float>((size_t)nq * dpad);
        sz.take<float>((size_t)nq * ns * kk);
        sz.take<int>((size_t)nq * ns * kk);
        return sz.bytes();
    };
    while (bytes_for(nsplit) > kNoAllocScratchBytes && nsplit > 1) {
        nsplit = std::max(1, nsplit / 2);
        rps = ceil_div(ceil_div(h->n, nsplit), 256) * 256;
        nsplit = (int)ceil_div(h->n, rps);
    }
    if (bytes_for(nsplit) > kNoAllocScratchBytes) {
        set_error("ann_flat_query_noalloc: nq=%d, k=%d, dim=%d need %zu bytes of scratch; the fixed scratch "
                  "holds %zu bytes (split the batch)", nq, kk, h->dim, bytes_for(nsplit), kNoAllocScratchBytes);
        return ANN_ERR_INVALID;
    }
    Carver cv(base);
    const float* qdev = queries;
    if (need_pad) {
        float* qp = cv.take<float>((size_t)nq * dpad);
        rc = launch_pad_rows(queries, nq, h->dim, ldq, qp, dpad, st);
        if (rc) return rc;
        qdev = qp;
    }
    float* skey = cv.take<float>((size_t)nq * nsplit * kk);
    int* sid = cv.take<int>((size_t)nq * nsplit * kk);
    FlatScanArgs a{h->base, h->n, dpad, qdev, nq, h->metric, kk, rps, nsplit, skey, sid};
    rc = launch_flat_scan(a, bq, st);
    if (rc) return rc;
    MergeArgs m{skey, sid, nq, nsplit, kk, kk, h->metric == ANN_METRIC_IP ? 1 : 0, out_ids, out_dists};
    rc = launch_merge_splits(m, st);
    if (rc) return rc;
    h->ndist.fetch_add(h->n * (int64_t)nq);
    return ANN_OK;
}

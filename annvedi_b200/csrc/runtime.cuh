// Host runtime pieces shared by the C ABI entry points: device guard, workspaces (device scratch
// arena + pinned host staging) and a bump allocator over them.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <vector>

#include "common.cuh"

struct ann_workspace {
    int device = 0;
    char* dev = nullptr;
    size_t dev_cap = 0;
    char* big = nullptr;   // second device arena for large per-batch buffers sized after planning
    size_t big_cap = 0;
    int64_t* pinned = nullptr;  // page-locked host words for totals read after a later synchronisation
    std::mutex mu;         // serialises growth; concurrent calls must still use separate workspaces
};

namespace annb {

// Makes `device` current for the scope and restores the previous device afterwards.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != device) ok = cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// Grows the workspace's device arena to at least `bytes` (drains the device first, since the old
// block may be in use by earlier asynchronous work).
int ws_reserve_device(ann_workspace* ws, size_t bytes);
int ws_reserve_big(ann_workspace* ws, size_t bytes);
// The workspace's page-locked host words (at least 8), allocated on first use.
int ws_pinned(ann_workspace* ws, int64_t** out);

// Stage timer: records CUDA events around consecutive stages of a call on its stream; totals are
// accumulated lazily (collect() synchronises on the recorded events). A call's first stage index is
// chosen at begin(), so different call kinds report into different slots of one table.
struct StageProfiler {
    static constexpr int kStages = 6;
    static constexpr size_t kMaxPending = 1024;
    bool enabled = false;
    struct Rec {
        cudaEvent_t ev[kStages + 1];
        int first;
        int nstage;
    };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    double total_ms[kStages] = {0, 0, 0, 0, 0, 0};
    // Kernel timers: events around single launches (the largest kernels of a call), by slot.
    static constexpr int kKernels = 4;
    struct KRec {
        cudaEvent_t a, b;
        int slot;
    };
    std::vector<KRec> kpending;
    double kern_ms[kKernels] = {0, 0, 0, 0};
    int64_t kern_launches[kKernels] = {0, 0, 0, 0};
    int64_t launches = 0;     // exact-scan launches
    int64_t tc_launches = 0;  // tensor-core GEMM launches
    int64_t filter_launches = 0;  // tensor-core filter passes timed alone
    int64_t calls = 0;
    std::mutex mu;

    cudaEvent_t get_event() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    // begin(): returns a record index; mark(rec) closes the next stage, starting at first_stage
    int begin(cudaStream_t st, int first_stage = 0) {
        if (!enabled) return -1;
        std::lock_guard<std::mutex> lk(mu);
        if (pending.size() >= kMaxPending) collect_locked();  // bounded record list for long runs
        Rec r{};
        r.first = first_stage;
        r.nstage = 0;
        r.ev[0] = get_event();
        cudaEventRecord(r.ev[0], st);
        pending.push_back(r);
        return (int)pending.size() - 1;
    }
    void mark(int rec, cudaStream_t st) {
        if (rec < 0) return;
        std::lock_guard<std::mutex> lk(mu);
        if (rec >= (int)pending.size()) return;
        Rec& r = pending[rec];
        if (r.first + r.nstage >= kStages) return;
        r.ev[++r.nstage] = get_event();
        cudaEventRecord(r.ev[r.nstage], st);
    }
    // kbegin() before a launch, kend(rec, slot) after it: the launch's time goes to kern_ms[slot].
    int kbegin(cudaStream_t st) {
        if (!enabled) return -1;
        std::lock_guard<std::mutex> lk(mu);
        if (kpending.size() >= kMaxPending) collect_kernels_locked();  // the stage records stay open
        KRec r{get_event(), nullptr, -1};
        cudaEventRecord(r.a, st);
        kpending.push_back(r);
        return (int)kpending.size() - 1;
    }
    void kend(int rec, int slot, cudaStream_t st) {
        if (rec < 0 || slot < 0 || slot >= kKernels) return;
        std::lock_guard<std::mutex> lk(mu);
        if (rec >= (int)kpending.size() || kpending[rec].b != nullptr) return;
        KRec& r = kpending[rec];
        r.b = get_event();
        r.slot = slot;
        cudaEventRecord(r.b, st);
    }
    void collect() {
        std::lock_guard<std::mutex> lk(mu);
        collect_locked();
    }
    void collect_locked() {
        collect_kernels_locked();
        collect_stages_locked();
    }
    void collect_kernels_locked() {
        for (KRec& r : kpending) {
            if (r.b != nullptr) {
                cudaEventSynchronize(r.b);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, r.a, r.b);
                kern_ms[r.slot] += ms;
                kern_launches[r.slot] += 1;
                pool.push_back(r.b);
            }
            pool.push_back(r.a);
        }
        kpending.clear();
    }
    void collect_stages_locked() {
        for (Rec& r : pending) {
            for (int s = 0; s < r.nstage; ++s) {
                cudaEventSynchronize(r.ev[s + 1]);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, r.ev[s], r.ev[s + 1]);
                total_ms[r.first + s] += ms;
            }
            for (int s = 0; s <= r.nstage; ++s) pool.push_back(r.ev[s]);
            calls += 1;
        }
        pending.clear();
    }
    void reset() {
        collect();
        std::lock_guard<std::mutex> lk(mu);
        for (double& t : total_ms) t = 0;
        for (int i = 0; i < kKernels; ++i) {
            kern_ms[i] = 0;
            kern_launches[i] = 0;
        }
        launches = 0;
        tc_launches = 0;
        filter_launches = 0;
        calls = 0;
    }
    ~StageProfiler() {
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
        for (Rec& r : pending)
            for (int s = 0; s <= r.nstage; ++s) cudaEventDestroy(r.ev[s]);
        for (KRec& r : kpending) {
            cudaEventDestroy(r.a);
            if (r.b) cudaEventDestroy(r.b);
        }
    }
};

// Carves aligned sub-buffers out of a base pointer.
struct Carver {
    char* base;
    size_t off = 0;
    explicit Carver(void* b) : base(static_cast<char*>(b)) {}
    template <typename T>
    T* take(size_t count, size_t align = 256) {
        off = (off + align - 1) / align * align;
        T* p = reinterpret_cast<T*>(base + off);
        off += count * sizeof(T);
        return p;
    }
    // bytes needed for the same sequence of takes when base is null
};

// Size calculator mirroring Carver.
struct Sizer {
    size_t off = 0;
    template <typename T>
    void take(size_t count, size_t align = 256) {
        off = (off + align - 1) / align * align;
        off += count * sizeof(T);
    }
    size_t bytes() const { return off + 256; }
};

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Queries and results of calls with host buffers move straight between the caller's memory and the device
// (the driver stages pageable memory itself; a copy through the library's own pinned buffer measured slower).
// queries_in: rows of `cols` floats (host stride ld) into dev rows of stride dpad, columns past cols zeroed.
int queries_in(float* dev, int64_t dpad, const float* host, int64_t ld, int64_t rows, int cols, cudaStream_t st);

}  // namespace annb

// Batched, list-major SQ8 pass of the exact-mode IVF query: the batch's (query, probed list) pairs
// grouped by list, scored in one persistent launch.
//
// A query batch probes each list from many queries at once (queries are drawn in proportion to list
// size, so the big lists are shared by hundreds of queries). Scanning query by query decodes every
// code once per query; here a work item is (list, up to 32 of the queries probing it, a range of up to
// kItemRows of its rows): the rows stream through shared memory in tiles of 256 rows x 32 dimensions,
// are decoded once (the exact integer of each code, FP32) and scored against the item's queries with a
// register-tiled micro-kernel (8 queries x 4 rows per thread, two fused multiply-adds per element
// pair). Each distance lands at its position in its query's candidate stream (the positions the plan
// assigns, lsh_index_optimized.cpp:372-405 order), so a per-query selection and the FP32 re-rank
// follow unchanged. Items are taken from a global counter by a persistent grid (uneven list lengths and
// query counts balance dynamically).
//
// The SQ8 distance is the per-query scan kernel's arithmetic (ivf.cu), so a query's keys do not depend
// on the batch it came in: diff_d = fma(code_d, scale_d, -(q_d - offset_d)), the squares summed by fused
// multiply-adds in dimension order separately over the two halves of the padded code row, then
// low + high. The FP32 re-rank that follows decides the final order.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "ivf.cuh"
#include "ivf_batched.cuh"
#include "runtime.cuh"

namespace annb {

namespace {

constexpr int kBQ = 32, kTQ = 8, kTR = 4;
constexpr int kThreads = 256;
constexpr int kWQ = kBQ / kTQ;       // 4 query groups
constexpr int kWR = kThreads / kWQ;  // 64 row groups
constexpr int kBR = kWR * kTR;       // 256 rows per tile
constexpr int kKC = 32;              // dimensions per step
constexpr int kPitch = kKC + 4;      // floats

__device__ __forceinline__ void cp16(void* smem, const void* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// pairs (list, q*npc + j) for every probed list of every query; unused slots get list id C (sorted last)
__global__ void pairs_kernel(IvfPlan p, int C, int32_t* keys, int32_t* vals, int* fallback) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= (int64_t)p.nq * p.npc) return;
    const int q = (int)(e / p.npc), j = (int)(e % p.npc);
    const int ns = p.n_seg[q];
    if (ns < 0 && j == 0) atomicExch(fallback, 1);
    keys[e] = (j < ns) ? p.probes[e] : C;
    vals[e] = (int32_t)e;
}

// items per list: ceil(queries / 32) * ceil(rows / kItemRows)
__global__ void items_kernel(const int64_t* lq_off, const int64_t* list_off, int C, int64_t* items) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l > C) return;
    if (l == C) {
        items[l] = 0;
        return;
    }
    const int64_t nq = lq_off[l + 1] - lq_off[l];
    const int64_t nr = list_off[l + 1] - list_off[l];
    items[l] = (nq == 0 || nr == 0) ? 0 : ceil_div(nq, kBQ) * ceil_div(nr, kItemRows);
}

// qs = q - offset (zero past dim), the shifted query the SQ8 distance compares against
__global__ void shift_queries_kernel(const float* q, int nq, int dpad, int dim, const float* offset, float* qs) {
    const int64_t total = (int64_t)nq * dpad;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int d = (int)(e % dpad);
        qs[e] = d < dim ? __fsub_rn(q[e], offset[d]) : 0.f;
    }
}

__global__ void __launch_bounds__(kThreads, 2) ivf_batched_kernel(IvfBatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int dpad = a.ix.dpad, dpad8 = a.ix.dpad8;
    float* sQ = reinterpret_cast<float*>(smem_raw);                 // [kBQ][dpad] shifted queries
    float* sX = sQ + (size_t)kBQ * dpad;                             // [kBR][kPitch] decoded rows
    float* sScale = sX + (size_t)kBR * kPitch;                       // [dpad]
    unsigned char* sRaw = reinterpret_cast<unsigned char*>(sScale + dpad);  // [2][kBR][kKC] codes
    int64_t* sBase = reinterpret_cast<int64_t*>(sRaw + 2 * kBR * kKC);     // [kBQ] D position of row 0
    int* sItem = reinterpret_cast<int*>(sBase + kBQ);

    const int tid = threadIdx.x;
    const int tq = tid / kWR, tr = tid % kWR;
    for (int d = tid; d < dpad; d += kThreads) sScale[d] = a.ix.scale[d];
    const int nkc = dpad8 / kKC;  // code chunks (>= dpad / kKC; extra chunks hold zero codes and scale)
    const int half_kc = nkc / 2;  // first chunk of the high half of the padded code row (dpad8 / 2)

    while (true) {
        __syncthreads();
        if (tid == 0) sItem[0] = (int)atomicAdd(a.counter, 1u);
        __syncthreads();
        const int64_t item = sItem[0];
        if (item >= a.total_items[0]) break;
        // item -> (list, query tile, row range)
        int lo = 0, hi = a.ix.C - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.item_off[mid] <= item)
                lo = mid;
            else
                hi = mid - 1;
        }
        const int l = lo;
        const int64_t local = item - a.item_off[l];
        const int64_t nrange = ceil_div(a.ix.list_off[l + 1] - a.ix.list_off[l], kItemRows);
        const int64_t qt = local / nrange, rr = local % nrange;
        const int64_t q0 = a.lq_off[l] + qt * kBQ;
        const int nqi = (int)min((int64_t)kBQ, a.lq_off[l + 1] - q0);
        const int64_t lstart = a.ix.list_off[l];
        const int64_t r_begin = lstart + rr * kItemRows;
        const int64_t r_end = min(a.ix.list_off[l + 1], r_begin + kItemRows);
        // the item's queries: shifted query rows and the stream position of this list's row 0
        for (int e = tid; e < kBQ * (dpad / 4); e += kThreads) {
            const int qq = e / (dpad / 4), piece = e % (dpad / 4);
            const bool ok = qq < nqi;
            const int32_t v = ok ? a.pair_vals[q0 + qq] : 0;
            const int qi = v / a.plan.npc;
            cp16(sQ + (size_t)qq * dpad + piece * 4, a.qs + (int64_t)qi * dpad + piece * 4, ok);
        }
        cp_commit();
        if (tid < kBQ) {
            int64_t base = 0;
            if (tid < nqi) {
                const int32_t v = a.pair_vals[q0 + tid];
                const int qi = v / a.plan.npc, j = v % a.plan.npc;
                base = a.cand_off[qi] + a.plan.seg_pref[(int64_t)qi * (a.plan.npc + 1) + j] - lstart;
            }
            sBase[tid] = base;
        }
        const int64_t ntiles = ceil_div(r_end - r_begin, kBR);
        const int64_t nsteps = ntiles * nkc;
        auto issue = [&](int64_t step) {
            if (step < nsteps) {
                const int64_t t = step / nkc;
                const int kc = (int)(step % nkc);
                unsigned char* dst = sRaw + (size_t)(step & 1) * kBR * kKC;
                for (int c = tid; c < kBR * 2; c += kThreads) {  // 256 rows x 2 pieces of 16 codes
                    const int r = c >> 1, piece = c & 1;
                    const int64_t row = r_begin + t * kBR + r;
                    const bool ok = row < r_end;
                    cp16(dst + r * kKC + piece * 16, a.ix.codes + (ok ? row : r_begin) * dpad8 + kc * kKC + piece * 16, ok);
                }
            }
            cp_commit();
        };
        issue(0);
        float acc[kTQ][kTR], lowh[kTQ][kTR];
#pragma unroll
        for (int j = 0; j < kTQ; ++j)
#pragma unroll
            for (int i = 0; i < kTR; ++i) acc[j][i] = lowh[j][i] = 0.f;
        for (int64_t step = 0; step < nsteps; ++step) {
            cp_wait0();
            __syncthreads();  // raw codes of this step (and the queries) landed; last step's reads are done
            issue(step + 1);
            const int kc = (int)(step % nkc);
            // decode 256 rows x 32 codes: code * scale, exact integer from the byte first
            {
                const unsigned char* raw = sRaw + (size_t)(step & 1) * kBR * kKC;
                for (int e = tid; e < kBR * (kKC / 4); e += kThreads) {
                    const int r = e / (kKC / 4), w4 = e % (kKC / 4);
                    const uint32_t w = *reinterpret_cast<const uint32_t*>(raw + r * kKC + w4 * 4);
                    const int d0 = kc * kKC + w4 * 4;
                    float4 v;
                    (void)d0;
                    v.x = __fsub_rn(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u)), 8388608.f);
                    v.y = __fsub_rn(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7541u)), 8388608.f);
                    v.z = __fsub_rn(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7542u)), 8388608.f);
                    v.w = __fsub_rn(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7543u)), 8388608.f);
                    *reinterpret_cast<float4*>(sX + r * kPitch + w4 * 4) = v;
                }
            }
            __syncthreads();
            if (kc == half_kc) {  // the high half starts: keep the low half's sums apart
#pragma unroll
                for (int j = 0; j < kTQ; ++j)
#pragma unroll
                    for (int i = 0; i < kTR; ++i) {
                        lowh[j][i] = acc[j][i];
                        acc[j][i] = 0.f;
                    }
            }
            if (kc * kKC < dpad) {
                const float* qbase = sQ + kc * kKC;
#pragma unroll
                for (int kk = 0; kk < kKC; kk += 4) {
                    float4 xv[kTR], qv[kTQ];
                    const float4 sc = *reinterpret_cast<const float4*>(sScale + kc * kKC + kk);
#pragma unroll
                    for (int i = 0; i < kTR; ++i) xv[i] = *reinterpret_cast<const float4*>(sX + (tr + i * kWR) * kPitch + kk);
#pragma unroll
                    for (int j = 0; j < kTQ; ++j)
                        qv[j] = *reinterpret_cast<const float4*>(qbase + (size_t)(tq * kTQ + j) * dpad + kk);
#pragma unroll
                    for (int j = 0; j < kTQ; ++j)
#pragma unroll
                        for (int i = 0; i < kTR; ++i) {
                            const float d0 = __fmaf_rn(xv[i].x, sc.x, -qv[j].x);
                            const float d1 = __fmaf_rn(xv[i].y, sc.y, -qv[j].y);
                            const float d2 = __fmaf_rn(xv[i].z, sc.z, -qv[j].z);
                            const float d3 = __fmaf_rn(xv[i].w, sc.w, -qv[j].w);
                            acc[j][i] = __fmaf_rn(d0, d0, acc[j][i]);
                            acc[j][i] = __fmaf_rn(d1, d1, acc[j][i]);
                            acc[j][i] = __fmaf_rn(d2, d2, acc[j][i]);
                            acc[j][i] = __fmaf_rn(d3, d3, acc[j][i]);
                        }
                }
            }
            if (kc == nkc - 1) {
                const int64_t t = step / nkc;
#pragma unroll
                for (int j = 0; j < kTQ; ++j) {
                    const int qq = tq * kTQ + j;
#pragma unroll
                    for (int i = 0; i < kTR; ++i) {
                        const int64_t row = r_begin + t * kBR + tr + i * kWR;
                        if (qq < nqi && row < r_end) a.D[sBase[qq] + row] = __fadd_rn(lowh[j][i], acc[j][i]);
                        acc[j][i] = 0.f;
                        lowh[j][i] = 0.f;
                    }
                }
            }
        }
        cp_wait0();
    }
}

}  // namespace

size_t batched_scratch_bytes(int nq, int npc, int C, size_t* sort_tmp, size_t* scan_tmp) {
    const int n = nq * npc;
    size_t b1 = 0, b2 = 0, b3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b1, (int32_t*)nullptr, (int32_t*)nullptr, (int32_t*)nullptr,
                                    (int32_t*)nullptr, n);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, (int64_t*)nullptr, (int64_t*)nullptr, C + 1);
    cub::DeviceScan::ExclusiveSum(nullptr, b3, (int64_t*)nullptr, (int64_t*)nullptr, nq + 1);
    *sort_tmp = b1;
    *scan_tmp = std::max(b2, b3);
    Sizer sz;
    sz.take<int32_t>(n);      // keys in
    sz.take<int32_t>(n);      // keys out
    sz.take<int32_t>(n);      // vals in
    sz.take<int32_t>(n);      // vals out
    sz.take<char>(b1);
    sz.take<char>(*scan_tmp);
    sz.take<int64_t>(C + 1);  // lq_off
    sz.take<int64_t>(C + 1);  // items per list
    sz.take<int64_t>(C + 1);  // item_off
    sz.take<int64_t>(nq + 1); // n_cands + trailing 0
    sz.take<int64_t>(nq + 1); // cand_off
    sz.take<float>((size_t)nq * 0 + 1);
    sz.take<int>(4);          // fallback flag, counter
    return sz.bytes();
}

int batched_prepare(const IvfQueryArgs& a, void* scratch, size_t sort_tmp, size_t scan_tmp, IvfBatchArgs* out,
                    int64_t* host_totals, cudaStream_t st, bool sync) {
    const int nq = a.plan.nq, npc = a.plan.npc, C = a.ix.C;
    const int n = nq * npc;
    Carver cv(scratch);
    int32_t* kin = cv.take<int32_t>(n);
    int32_t* kout = cv.take<int32_t>(n);
    int32_t* vin = cv.take<int32_t>(n);
    int32_t* vout = cv.take<int32_t>(n);
    void* stmp = cv.take<char>(sort_tmp);
    void* ctmp = cv.take<char>(scan_tmp);
    int64_t* lq_off = cv.take<int64_t>(C + 1);
    int64_t* items = cv.take<int64_t>(C + 1);
    int64_t* item_off = cv.take<int64_t>(C + 1);
    int64_t* ncand = cv.take<int64_t>(nq + 1);
    int64_t* cand_off = cv.take<int64_t>(nq + 1);
    cv.take<float>(1);
    int* flags = cv.take<int>(4);  // [0] fallback, [1] counter
    ANN_CUDA_TRY(cudaMemsetAsync(flags, 0, sizeof(int) * 4, st));
    pairs_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(a.plan, C, kin, vin, flags);
    ANN_LAUNCH_CHECK();
    int end_bit = 1;
    while ((1 << end_bit) <= C) ++end_bit;
    size_t tb = sort_tmp;
    ANN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(stmp, tb, kin, kout, vin, vout, n, 0, end_bit, st));
    int rc = launch_list_offsets(kout, n, C, lq_off, st);
    if (rc) return rc;
    items_kernel<<<(unsigned)ceil_div(C + 1, 128), 128, 0, st>>>(lq_off, a.ix.list_off, C, items);
    ANN_LAUNCH_CHECK();
    size_t sb = scan_tmp;
    ANN_CUDA_TRY(cub::DeviceScan::ExclusiveSum(ctmp, sb, items, item_off, C + 1, st));
    ANN_CUDA_TRY(cudaMemcpyAsync(ncand, a.plan.n_cands, sizeof(int64_t) * nq, cudaMemcpyDeviceToDevice, st));
    ANN_CUDA_TRY(cudaMemsetAsync(ncand + nq, 0, sizeof(int64_t), st));
    sb = scan_tmp;
    ANN_CUDA_TRY(cub::DeviceScan::ExclusiveSum(ctmp, sb, ncand, cand_off, nq + 1, st));
    // totals to the host: items, candidates, fallback
    ANN_CUDA_TRY(cudaMemcpyAsync(host_totals, item_off + C, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    ANN_CUDA_TRY(cudaMemcpyAsync(host_totals + 1, cand_off + nq, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    ANN_CUDA_TRY(cudaMemcpyAsync(host_totals + 2, flags, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (sync) ANN_CUDA_TRY(cudaStreamSynchronize(st));
    IvfBatchArgs b{};
    b.ix = a.ix;
    b.plan = a.plan;
    b.pair_vals = vout;
    b.pair_lists = kout;
    b.lq_off = lq_off;
    b.item_off = item_off;
    b.total_items = item_off + C;
    b.cand_off = cand_off;
    b.counter = reinterpret_cast<unsigned*>(flags + 1);
    *out = b;
    return ANN_OK;
}

int launch_batched(const IvfBatchArgs& b, const float* qdev, float* qs, float* D, cudaStream_t st) {
    IvfBatchArgs a = b;
    a.D = D;
    a.qs = qs;
    const int nq = a.plan.nq;
    shift_queries_kernel<<<(unsigned)std::min<int64_t>(ceil_div((int64_t)nq * a.ix.dpad, 256), kNumSMs * 16), 256, 0,
                           st>>>(qdev, nq, a.ix.dpad, a.ix.dim, a.ix.offset, qs);
    ANN_LAUNCH_CHECK();
    const size_t smem = sizeof(float) * ((size_t)kBQ * a.ix.dpad + (size_t)kBR * kPitch + a.ix.dpad) +
                        (size_t)2 * kBR * kKC + sizeof(int64_t) * kBQ + 16;
    ANN_CHECK_ARG(smem <= 227 * 1024, "batched SQ8 pass: dim %d needs %zu bytes of shared memory", a.ix.dim, smem);
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(ivf_batched_kernel)));
    int per_sm = 0;
    ANN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ivf_batched_kernel, kThreads, smem));
    const int grid = kNumSMs * std::max(1, per_sm);
    ivf_batched_kernel<<<grid, kThreads, smem, st>>>(a);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

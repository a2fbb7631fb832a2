// IVF-SQ8 query kernels: the B200 form of IVFLSHIndex::query
// (competitors/ivf_lsh/src/lsh_index_optimized.cpp:304-516) for n_tables = 1, n_bits = 0, i.e.
// inverted lists of per-dimension SQ8 codes with an FP32 re-rank.
//
// Pipeline per query batch (one launch per stage, every query of the batch in each launch):
//   1. coarse ranking of the lists (exact FP32 scan of the centroids, or -- reference mode -- the
//      reference's arithmetic and pair order, :326-333);
//   2. plan: the probed lists in order, whole lists only, until the candidate cap is reached
//      (:352-378); a query whose lists hold fewer than k points scans every row (:453-457);
//      the candidate count is added to get_n_distances (:459-460);
//   3. SQ8 pass over the candidate stream (:462-469):
//        exact mode   -- one fused kernel streams the codes through shared memory (cp.async), decodes
//                        them in registers and keeps the best R (SQ8 distance, row) pairs per query;
//        reference mode -- the reference's SQ8 arithmetic with its checkpoints, then one warp per
//                        ThreadPool chunk replays the chunk's 64-entry early-abandon heap
//                        (lsh_worker, :86-122) and the best R ranking values are selected;
//   4. FP32 re-rank of the R candidates against the original rows and the final top-k
//      (:471-512), ids mapped back to original numbering.
//
// Layout in HBM: codes [n, dpad8] uint8 and original rows [n, dpad] FP32, both in list order, so a
// list is one contiguous byte range; per-dimension scale/offset zero-padded past dim.
#include "common.cuh"
#include "ivf.cuh"
#include "refmath.cuh"

namespace annb {

__device__ __forceinline__ void cp_async16_ivf(void* smem, const void* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int sz = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit_ivf() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all_ivf() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ---- 2. plan ---------------------------------------------------------------------------------
__global__ void ivf_plan_kernel(IvfQueryArgs a) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.plan.nq) return;
    const IvfPlan& p = a.plan;
    const int32_t* probes = p.probes + (int64_t)q * p.npc;
    int64_t* pref = p.seg_pref + (int64_t)q * (p.npc + 1);
    int64_t* start = p.seg_start + (int64_t)q * p.npc;
    int64_t cands = 0;
    int j = 0;
    for (; j < p.npc; ++j) {
        if (cands >= a.max_cands) break;
        const int cid = probes[j];
        if (cid < 0 || cid >= a.ix.C) break;
        const int64_t s = a.ix.list_off[cid], e = a.ix.list_off[cid + 1];
        start[j] = s;
        pref[j] = cands;
        cands += e - s;
    }
    pref[j] = cands;
    if (cands < a.k && !a.no_fallback) {
        p.n_seg[q] = -1;
        cands = a.ix.n;
    } else {
        p.n_seg[q] = j;
    }
    p.n_cands[q] = cands;
    if (a.ndist) atomicAdd(a.ndist, (unsigned long long)cands);
}

int launch_ivf_plan(const IvfQueryArgs& a, cudaStream_t st) {
    if (a.plan.nq == 0) return ANN_OK;
    ivf_plan_kernel<<<(unsigned)ceil_div(a.plan.nq, 128), 128, 0, st>>>(a);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// ---- 3a. exact-mode SQ8 scan with fused top-R -------------------------------------------------
constexpr int kSq8Tile = 128;  // candidate rows per shared-memory tile (2 threads per row)

__device__ __forceinline__ float u8_to_f32(uint32_t word, int byte) {
    // 0x4B000000 | byte is the float 2^23 + byte; subtracting 2^23 is exact
    return __fsub_rn(__uint_as_float(__byte_perm(word, 0x4B000000u, 0x7540u | byte)), 8388608.f);
}

__global__ void __launch_bounds__(256) ivf_sq8_scan_kernel(IvfQueryArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int dpad8 = a.ix.dpad8;
    const int pitch = dpad8 + 16;  // 16-byte pad: row r starts 4r words later, conflict-free
    const int cap = topk_cap(a.R);
    unsigned char* sCodes = smem_raw;                                   // [2][Tile][pitch]
    float* sQs = reinterpret_cast<float*>(sCodes + 2 * kSq8Tile * pitch);  // [dpad8]
    float* sSc = sQs + dpad8;                                           // [dpad8]
    float* sKey = sSc + dpad8;                                          // [cap]
    int* sId = reinterpret_cast<int*>(sKey + cap);                      // [cap]
    int* sMisc = sId + cap;                                             // cnt, tau_id
    float* sTau = reinterpret_cast<float*>(sMisc + 2);

    const int tid = threadIdx.x;
    const int q = blockIdx.x;
    const int s = blockIdx.y;
    const int R = a.R;
    const int64_t L = a.plan.n_cands[q];
    const int64_t ps = L * s / a.nsplit, pe = L * (s + 1) / a.nsplit;
    const float* qv = a.q + (int64_t)q * a.ldq;
    for (int d = tid; d < dpad8; d += 256) {
        sQs[d] = d < a.ix.dim ? __fsub_rn(qv[d], a.ix.offset[d]) : 0.f;
        sSc[d] = d < a.ix.dim ? a.ix.scale[d] : 0.f;
    }
    if (tid == 0) {
        sMisc[0] = 0;
        sMisc[1] = kNoId;
        sTau[0] = kInf;
    }

    const int r = tid >> 1, h = tid & 1;  // row within tile, half of the dimensions
    const int half = dpad8 >> 1;          // bytes per half (multiple of 16)
    const int64_t ntiles = pe > ps ? ceil_div(pe - ps, kSq8Tile) : 0;
    int64_t row_next = -1;  // row of this thread's position in the tile being loaded

    auto issue = [&](int64_t t) {
        if (t < ntiles) {
            const int buf = (int)(t & 1);
            const int64_t p = ps + t * kSq8Tile + r;
            const bool ok = p < pe;
            const int64_t row = ok ? plan_row(a.plan, q, p) : -1;
            row_next = row;
            const unsigned char* src = a.ix.codes + (ok ? row : 0) * dpad8 + h * half;
            unsigned char* dst = sCodes + ((size_t)buf * kSq8Tile + r) * pitch + h * half;
            for (int b = 0; b < half; b += 16) cp_async16_ivf(dst + b, src + b, ok);
        }
        cp_async_commit_ivf();
    };

    issue(0);
    for (int64_t t = 0; t < ntiles; ++t) {
        cp_async_wait_all_ivf();
        __syncthreads();
        const int64_t row = row_next;
        issue(t + 1);
        const int buf = (int)(t & 1);
        const unsigned char* row_codes = sCodes + ((size_t)buf * kSq8Tile + r) * pitch + h * half;
        const float* qs = sQs + h * half;
        const float* sc = sSc + h * half;
        float acc = 0.f;
        for (int b = 0; b < half; b += 16) {
            const uint4 c = *reinterpret_cast<const uint4*>(row_codes + b);
            const uint32_t w[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
            for (int wi = 0; wi < 4; ++wi) {
                const float4 s4 = *reinterpret_cast<const float4*>(sc + b + wi * 4);
                const float4 q4 = *reinterpret_cast<const float4*>(qs + b + wi * 4);
                const float d0 = __fmaf_rn(u8_to_f32(w[wi], 0), s4.x, -q4.x);
                const float d1 = __fmaf_rn(u8_to_f32(w[wi], 1), s4.y, -q4.y);
                const float d2 = __fmaf_rn(u8_to_f32(w[wi], 2), s4.z, -q4.z);
                const float d3 = __fmaf_rn(u8_to_f32(w[wi], 3), s4.w, -q4.w);
                acc = __fmaf_rn(d0, d0, acc);
                acc = __fmaf_rn(d1, d1, acc);
                acc = __fmaf_rn(d2, d2, acc);
                acc = __fmaf_rn(d3, d3, acc);
            }
        }
        const float dist = acc + __shfl_xor_sync(0xffffffffu, acc, 1);
        bool pend = h == 0 && row >= 0;
        // offer to the query's buffer; compaction by warp 0, overflow re-offered after it
        while (true) {
            if (pend) {
                if (pair_less(dist, (int)row, sTau[0], sMisc[1])) {
                    const int slot = atomicAdd(&sMisc[0], 1);
                    if (slot < cap) {
                        sKey[slot] = dist;
                        sId[slot] = (int)row;
                        pend = false;
                    }
                } else {
                    pend = false;
                }
            }
            const int overflow = __syncthreads_or(pend);
            if (tid < 32 && sMisc[0] >= cap / 2) {
                const int kept = warp_compact_smem(sKey, sId, sMisc[0], cap, R);
                if (tid == 0) {
                    sMisc[0] = kept;
                    if (kept == R) {
                        sTau[0] = sKey[R - 1];
                        sMisc[1] = sId[R - 1];
                    }
                }
            }
            __syncthreads();
            if (!overflow) break;
        }
    }
    cp_async_wait_all_ivf();
    __syncthreads();
    if (tid < 32) {
        const int kept = warp_compact_smem(sKey, sId, sMisc[0], cap, R);
        float* ok = a.keyR + ((int64_t)q * a.nsplit + s) * R;
        int* oi = a.idR + ((int64_t)q * a.nsplit + s) * R;
        for (int e = tid; e < R; e += 32) {
            ok[e] = e < kept ? sKey[e] : kInf;
            oi[e] = e < kept ? sId[e] : kNoId;
        }
    }
}

static size_t sq8_scan_smem(int dpad8, int R) {
    return (size_t)2 * kSq8Tile * (dpad8 + 16) + (size_t)2 * dpad8 * 4 + (size_t)topk_cap(R) * 8 + 16;
}

int launch_ivf_sq8_scan(const IvfQueryArgs& a, cudaStream_t st) {
    if (a.plan.nq == 0) return ANN_OK;
    ANN_CHECK_ARG(a.ix.dpad8 % 32 == 0, "sq8 scan: code stride %d not a multiple of 32", a.ix.dpad8);
    const size_t smem = sq8_scan_smem(a.ix.dpad8, a.R);
    if (smem > 227 * 1024) {
        set_error("sq8 scan: R=%d with dim %d needs %zu bytes of shared memory", a.R, a.ix.dim, smem);
        return ANN_ERR_UNSUPPORTED;
    }
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(ivf_sq8_scan_kernel)));
    dim3 grid(a.plan.nq, a.nsplit);
    ivf_sq8_scan_kernel<<<grid, 256, smem, st>>>(a);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// ---- 3a'. exact-mode SQ8 keys of whole candidate streams --------------------------------------------
// D[q * ld + p] = the SQ8 distance of position p of query q's stream, for p < min(n_cands[q], ld): the
// arithmetic of ivf_sq8_scan_kernel (two threads per row, each a fused multiply-add chain over its half of
// the bytes in order, then the halves added), so either kernel gives a candidate the same key. grid:
// (queries, tile slices); a tile is 128 positions; each thread's twelve 16-byte loads (dim 384) are
// independent, so many are in flight.
constexpr int kDistGroup = 6;  // 16-byte chunks in flight per thread (dim 384: two groups per half row)

__global__ void __launch_bounds__(256) ivf_sq8_dists_kernel(IvfQueryArgs a, float* __restrict__ D, int64_t ld) {
    extern __shared__ __align__(16) float sh_qs[];  // qs [dpad8], scale [dpad8]
    const int dpad8 = a.ix.dpad8;
    float* sQs = sh_qs;
    float* sSc = sh_qs + dpad8;
    const int q = blockIdx.x, tid = threadIdx.x;
    const float* qv = a.q + (int64_t)q * a.ldq;
    for (int d = tid; d < dpad8; d += 256) {
        sQs[d] = d < a.ix.dim ? __fsub_rn(qv[d], a.ix.offset[d]) : 0.f;
        sSc[d] = d < a.ix.dim ? a.ix.scale[d] : 0.f;
    }
    __syncthreads();
    const int64_t L = min(a.plan.n_cands[q], ld);
    const int r = tid >> 1, h = tid & 1;
    const int half = dpad8 >> 1;
    const float* qs = sQs + h * half;
    const float* sc = sSc + h * half;
    float* Dq = D + (int64_t)q * ld;
    for (int64_t p0 = (int64_t)blockIdx.y * kSq8Tile; p0 < L; p0 += (int64_t)gridDim.y * kSq8Tile) {
        const int64_t p = p0 + r;
        const bool valid = p < L;
        const int64_t row = valid ? plan_row(a.plan, q, p) : 0;
        const uint4* src = reinterpret_cast<const uint4*>(a.ix.codes + row * dpad8 + h * half);
        float acc = 0.f;
        // chunks of 16 bytes, loaded kDistGroup at a time so that they are in flight together
        for (int b0 = 0; valid && b0 < half; b0 += 16 * kDistGroup) {
            uint4 cw[kDistGroup];
#pragma unroll
            for (int i = 0; i < kDistGroup; ++i)
                if (b0 + 16 * i < half) cw[i] = src[(b0 >> 4) + i];
#pragma unroll
            for (int i = 0; i < kDistGroup; ++i) {
                if (b0 + 16 * i >= half) break;
                const int b = b0 + 16 * i;
                const uint32_t w[4] = {cw[i].x, cw[i].y, cw[i].z, cw[i].w};
#pragma unroll
                for (int wi = 0; wi < 4; ++wi) {
                    const float4 s4 = *reinterpret_cast<const float4*>(sc + b + wi * 4);
                    const float4 q4 = *reinterpret_cast<const float4*>(qs + b + wi * 4);
                    const float d0 = __fmaf_rn(u8_to_f32(w[wi], 0), s4.x, -q4.x);
                    const float d1 = __fmaf_rn(u8_to_f32(w[wi], 1), s4.y, -q4.y);
                    const float d2 = __fmaf_rn(u8_to_f32(w[wi], 2), s4.z, -q4.z);
                    const float d3 = __fmaf_rn(u8_to_f32(w[wi], 3), s4.w, -q4.w);
                    acc = __fmaf_rn(d0, d0, acc);
                    acc = __fmaf_rn(d1, d1, acc);
                    acc = __fmaf_rn(d2, d2, acc);
                    acc = __fmaf_rn(d3, d3, acc);
                }
            }
        }
        const float other = __shfl_xor_sync(0xffffffffu, acc, 1);  // every lane runs each trip of the loop
        if (valid && h == 0) Dq[p] = acc + other;
    }
}

int launch_ivf_sq8_dists(const IvfQueryArgs& a, float* D, int64_t ld, cudaStream_t st) {
    if (a.plan.nq == 0) return ANN_OK;
    ANN_CHECK_ARG(a.ix.dpad8 % 32 == 0, "sq8 keys: code stride %d not a multiple of 32", a.ix.dpad8);
    const size_t smem = sizeof(float) * 2 * a.ix.dpad8;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(ivf_sq8_dists_kernel)));
    const int slices = (int)std::min<int64_t>(8, std::max<int64_t>(1, ceil_div(ld, kSq8Tile)));
    ivf_sq8_dists_kernel<<<dim3(a.plan.nq, slices), 256, smem, st>>>(a, D, ld);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// ---- 3b. reference-mode SQ8 pass ----------------------------------------------------------------
// grid: (queries, position blocks); block: 16 groups of 16 lanes, one candidate per group.
__global__ void __launch_bounds__(256) ivf_ref_sq8_kernel(IvfQueryArgs a) {
    extern __shared__ float sh[];  // qs [dim], scale [dim]
    const int q = blockIdx.x;
    const int dim = a.ix.dim;
    float* sQs = sh;
    float* sSc = sh + dim;
    const float* qv = a.q + (int64_t)q * a.ldq;
    for (int d = threadIdx.x; d < dim; d += blockDim.x) {
        sQs[d] = __fsub_rn(qv[d], a.ix.offset[d]);  // q_shifted (lsh_index_optimized.cpp:320-323)
        sSc[d] = a.ix.scale[d];
    }
    __syncthreads();
    const int64_t L = min(a.plan.n_cands[q], a.L);  // a longer stream (every row) is redone on its own
    const int grp = threadIdx.x >> 4;
    const bool leader = (threadIdx.x & 15) == 0;
    float* D = a.D + (int64_t)q * a.L;
    float* P = a.P + (int64_t)q * a.ncp * a.L;
    for (int64_t p0 = (int64_t)blockIdx.y * 16; p0 < L; p0 += (int64_t)gridDim.y * 16) {
        const int64_t p = p0 + grp;
        const bool valid = p < L;
        const int64_t row = valid ? plan_row(a.plan, q, p) : 0;
        const float d = ref_l2_sq8(a.ix.codes + row * a.ix.dpad8, sQs, sSc, dim, [&](int c, float v) {
            if (leader && valid) P[(int64_t)c * a.L + p] = v;
        });
        if (leader && valid) D[p] = d;
    }
}

// One warp per ThreadPool chunk (src/thread_pool.h:93-124): chunk c of T covers
// [c*(L/T) + min(c, L%T), ...), the first L%T chunks one longer; T = 1 when L < 2*num_threads
// (lsh_index_optimized.cpp:465-469).
__global__ void __launch_bounds__(1024) ivf_ref_replay_kernel(IvfQueryArgs a) {
    const int q = blockIdx.x;
    const int warp = threadIdx.x >> 5;
    const int64_t L = min(a.plan.n_cands[q], a.L);
    const int T = (a.num_threads > 0 && L >= 2 * (int64_t)a.num_threads) ? a.num_threads : 1;
    const int lim = a.k < 64 ? a.k : 64;
    float* V = a.V + (int64_t)q * a.L;
    for (int c = warp; c < T; c += blockDim.x >> 5) {
        const int64_t base = L / T, rem = L % T;
        const int64_t b = c * base + (c < rem ? c : rem);
        const int64_t e = b + base + (c < rem ? 1 : 0);
        ref_replay(a.D + (int64_t)q * a.L, a.P + (int64_t)q * a.ncp * a.L, a.L, a.ncp, b, e, lim,
                   [&](int64_t i, float v, bool valid) {
                       if (valid) V[i] = v;
                   });
    }
}

int launch_ivf_ref_sq8(const IvfQueryArgs& a, int64_t Lmax, cudaStream_t st) {
    if (a.plan.nq == 0 || Lmax == 0) return ANN_OK;
    const size_t smem = sizeof(float) * 2 * a.ix.dim;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(ivf_ref_sq8_kernel)));
    const int64_t blocks = std::min<int64_t>(ceil_div(Lmax, 16), 4096);
    dim3 g1(a.plan.nq, (unsigned)blocks);
    ivf_ref_sq8_kernel<<<g1, 256, smem, st>>>(a);
    ANN_LAUNCH_CHECK();
    // one warp per ThreadPool chunk (up to 32 in a block; more chunks loop)
    const int rwarps = std::max(1, std::min(32, a.num_threads > 0 ? a.num_threads : 1));
    ivf_ref_replay_kernel<<<a.plan.nq, 32 * rwarps, 0, st>>>(a);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// ---- generic per-query top-k selection over a dense key array -----------------------------------
constexpr int kSelBins = 1024;  // set-only selection: linear bins (4 per thread of a 256-thread block)
constexpr int kSelTie = 256;    // boundary-bin pairs sorted by one warp

// keys[q * ld + p] (keys[offs[q] + p] when offs is given) for p < lens[q] (at most ld without offs; ld when
// lens is null);
// id = plan_row(q, p) when a plan is
// given, else p. Keeps the best kout (key, id) pairs, sorted, padded with (+inf, INT_MAX); with set_only
// the same pairs in no particular order.
__global__ void __launch_bounds__(256) select_topk_kernel(const float* __restrict__ keys, int64_t ld,
                                                          const int64_t* __restrict__ offs,
                                                          const int64_t* __restrict__ lens, int kout,
                                                          IvfPlan plan, int use_plan, float* out_key,
                                                          int* out_id, int set_only) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warps = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cap = topk_cap(kout);
    float* sKey = reinterpret_cast<float*>(smem_raw);
    int* sId = reinterpret_cast<int*>(sKey + warps * cap);
    const int q = blockIdx.x;
    const int64_t len = lens ? (offs || ld <= 0 ? lens[q] : min(lens[q], ld)) : ld;
    const float* kq = keys + (offs ? offs[q] : (int64_t)q * ld);
    auto id_at = [&](int64_t p) { return (int)(use_plan ? plan_row(plan, q, p) : p); };
    if (set_only && blockDim.x == kSelBins / 4 && len > kout) {
        // The set only (unordered): kSelBins linear bins over the stream's keys find the bin holding the
        // kout-th; every pair in a lower bin is in, and the boundary bin's pairs (few) are sorted by (key, id)
        // by one warp -- the set the sorted path keeps, ties by id. Equal keys throughout, or a crowded
        // boundary bin, take the sorted path below.
        int* sHist = reinterpret_cast<int*>(smem_raw);                      // [kSelBins]
        float* sBK = reinterpret_cast<float*>(sHist + kSelBins);             // [kSelTie]
        int* sBI = reinterpret_cast<int*>(sBK + kSelTie);                    // [kSelTie]
        __shared__ float sRf[64];
        __shared__ int sRi[40];
        float lo = kInf, hi = -kInf;
        for (int64_t p = threadIdx.x; p < len; p += blockDim.x) {
            const float kv = kq[p];
            lo = fminf(lo, kv);
            hi = fmaxf(hi, kv);
        }
        for (int i = threadIdx.x; i < kSelBins; i += blockDim.x) sHist[i] = 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            sRf[warp] = lo;
            sRf[32 + warp] = hi;
        }
        if (threadIdx.x == 0) {
            sRi[32] = 0;  // slots of the lower bins
            sRi[33] = 0;  // boundary pairs
        }
        __syncthreads();
        lo = kInf;
        hi = -kInf;
        for (int w = 0; w < warps; ++w) {
            lo = fminf(lo, sRf[w]);
            hi = fmaxf(hi, sRf[32 + w]);
        }
        const float sc = (float)kSelBins / (hi - lo);
        if (hi > lo && isfinite(sc)) {  // uniform
            auto bin_of = [&](float kv) {
                const float f = (kv - lo) * sc;
                return !(f > 0.f) ? 0 : (f >= (float)(kSelBins - 1) ? kSelBins - 1 : (int)f);
            };
            for (int64_t p = threadIdx.x; p < len; p += blockDim.x) atomicAdd(&sHist[bin_of(kq[p])], 1);
            __syncthreads();
            // the bin holding rank kout - 1: kSelBins / blockDim bins per thread, a warp-shuffle scan
            constexpr int per = 4;
            int own = 0;
#pragma unroll
            for (int i = 0; i < per; ++i) own += sHist[threadIdx.x * per + i];
            int incl = own;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            if (lane == 31) sRi[warp] = incl;
            __syncthreads();
            for (int w = 0; w < warp; ++w) incl += sRi[w];
            const int excl = incl - own;
            if (kout - 1 >= excl && kout - 1 < incl) {
                int c = excl;
                for (int i = 0; i < per; ++i) {
                    const int h = sHist[threadIdx.x * per + i];
                    if (kout - 1 < c + h) {
                        sRi[34] = threadIdx.x * per + i;
                        sRi[35] = c;
                        sRi[36] = h;
                        break;
                    }
                    c += h;
                }
            }
            __syncthreads();
            const int bb = sRi[34], below = sRi[35], nb = sRi[36];
            if (nb <= kSelTie) {
                for (int64_t p = threadIdx.x; p < len; p += blockDim.x) {
                    const float kv = kq[p];
                    const int bin = bin_of(kv);
                    if (bin < bb) {
                        const int slot = atomicAdd(&sRi[32], 1);
                        out_key[(int64_t)q * kout + slot] = kv;
                        out_id[(int64_t)q * kout + slot] = id_at(p);
                    } else if (bin == bb) {
                        const int at = atomicAdd(&sRi[33], 1);
                        sBK[at] = kv;
                        sBI[at] = id_at(p);
                    }
                }
                __syncthreads();
                if (warp == 0) {
                    int cap2 = 32;
                    while (cap2 < nb) cap2 <<= 1;
                    for (int e = nb + lane; e < cap2; e += 32) {
                        sBK[e] = kInf;
                        sBI[e] = kNoId;
                    }
                    __syncwarp();
                    warp_sort_smem(sBK, sBI, cap2);
                    for (int e = lane; e < kout - below; e += 32) {
                        out_key[(int64_t)q * kout + below + e] = sBK[e];
                        out_id[(int64_t)q * kout + below + e] = sBI[e];
                    }
                }
                return;
            }
        }
        __syncthreads();  // the sorted path reuses the shared memory
    }
    WarpTopK top;
    top.init(sKey + warp * cap, sId + warp * cap, kout);
    for (int64_t base = (int64_t)warp * 32; base < len; base += (int64_t)warps * 32) {
        const int64_t p = base + lane;
        const bool ok = p < len;
        const float kv = ok ? kq[p] : kInf;
        const int iv = ok ? id_at(p) : kNoId;
        top.offer(kv, iv, ok);
    }
    top.compact();
    __syncthreads();
    if (warp == 0) {
        for (int w = 1; w < warps; ++w)
            for (int e0 = 0; e0 < kout; e0 += 32) {
                const int e = e0 + lane;
                const bool ok = e < kout && sId[w * cap + e] != kNoId;
                top.offer(ok ? sKey[w * cap + e] : kInf, ok ? sId[w * cap + e] : kNoId, ok);
            }
        top.compact();
        for (int e = lane; e < kout; e += 32) {
            const bool ok = e < top.count;
            out_key[(int64_t)q * kout + e] = ok ? sKey[e] : kInf;
            out_id[(int64_t)q * kout + e] = ok ? sId[e] : kNoId;
        }
    }
}

int launch_select_topk(const float* keys, int64_t ld, const int64_t* lens, int nq, int kout, const IvfPlan* plan,
                       float* out_key, int* out_id, cudaStream_t st, const int64_t* offs, bool set_only) {
    if (nq == 0) return ANN_OK;
    ANN_CHECK_ARG(kout >= 1 && kout <= 8192, "select: k=%d outside [1, 8192]", kout);
    const size_t per_warp = (size_t)topk_cap(kout) * 8;
    int warps = (int)std::max<size_t>(1, std::min<size_t>(8, (96 * 1024) / per_warp));
    size_t smem = per_warp * warps;
    if (set_only) smem = std::max(smem, sizeof(int) * kSelBins + (size_t)8 * kSelTie);
    ANN_CHECK_ARG(smem <= 227 * 1024, "select: k=%d needs too much shared memory", kout);
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(select_topk_kernel)));
    IvfPlan p{};
    if (plan) p = *plan;
    select_topk_kernel<<<nq, warps * 32, smem, st>>>(keys, ld, offs, lens, kout, p, plan ? 1 : 0, out_key, out_id,
                                                      set_only ? 1 : 0);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// ---- 4. FP32 re-rank and final top-k -------------------------------------------------------------
constexpr int kRerankRankMax = 1024;  // R up to this: the final top-k by block-wide ranks
constexpr int kRerankBins = 256;      // bins of the distances that narrow the ranking down

// Sum of v over the block (every thread gets it); scratch: >= blockDim.x / 32 floats of shared memory, free
// for the caller's use again after the call.
__device__ __forceinline__ int block_sum_int(int v, float* scratch) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    int* s = reinterpret_cast<int*>(scratch);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
    return t;
}
// One CTA per query: exact distances of its R candidates to the original rows (the reference's
// arithmetic in reference mode, lsh_index_optimized.cpp:481-486), then the best k by (distance, row)
// and the mapping back to original ids (:503-512).
template <bool REF>
__global__ void __launch_bounds__(256, 5) ivf_rerank_kernel(IvfQueryArgs a, const float* __restrict__ keyR,
                                                          const int* __restrict__ idR) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int R = a.R, k = a.k;
    const int cap = topk_cap(k);
    const int dpad = a.ix.dpad;
    float* sQ = reinterpret_cast<float*>(smem_raw);   // [dpad]
    float* sD = sQ + dpad;                            // [R]
    int* sRow = reinterpret_cast<int*>(sD + R);       // [R]
    float* sKey = reinterpret_cast<float*>(sRow + R); // [cap]
    int* sId = reinterpret_cast<int*>(sKey + cap);    // [cap]
    const int q = a.qorder ? a.qorder[blockIdx.x] : blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float* qv = a.q + (int64_t)q * a.ldq;
    for (int d = threadIdx.x; d < dpad; d += blockDim.x) sQ[d] = d < a.ix.dim ? qv[d] : 0.f;
    for (int e = threadIdx.x; e < R; e += blockDim.x) sRow[e] = idR[(int64_t)q * R + e];
    __syncthreads();
    if (REF) {
        // two candidates per warp, one per 16-lane group
        for (int e0 = warp * 2; e0 < R; e0 += 16) {
            const int e = e0 + (lane >> 4);
            const int row = e < R ? sRow[e] : kNoId;
            const bool ok = row != kNoId;
            const float* x = a.ix.original + (int64_t)(ok ? row : 0) * dpad;
            const float d = ref_l2_f32(x, sQ, a.ix.dim, NoEmit{});
            if ((lane & 15) == 0 && e < R) sD[e] = ok ? d : kInf;
        }
    } else if (dpad <= 512) {
        // two rows per warp step; each lane's (up to four) 16-byte pieces of both rows are loaded before they
        // are used, so eight loads per lane are in flight. Per lane the sum runs over d in the same order as
        // below, so the distances are the same.
        for (int e0 = warp; e0 < R; e0 += 16) {
            const int e1 = e0 + 8;
            const int rowA = sRow[e0];
            const int rowB = e1 < R ? sRow[e1] : kNoId;
            const bool okA = rowA != kNoId, okB = rowB != kNoId;
            const float* pa = a.ix.original + (int64_t)(okA ? rowA : 0) * dpad;
            const float* pb = a.ix.original + (int64_t)(okB ? rowB : 0) * dpad;
            float4 xa[4], xb[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int d = lane * 4 + 128 * i;
                xa[i] = make_float4(0.f, 0.f, 0.f, 0.f);
                xb[i] = xa[i];
                if (d < dpad) {
                    if (okA) xa[i] = *reinterpret_cast<const float4*>(pa + d);
                    if (okB) xb[i] = *reinterpret_cast<const float4*>(pb + d);
                }
            }
            float accA = 0.f, accB = 0.f;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int d = lane * 4 + 128 * i;
                if (d < dpad) {
                    const float4 q4 = *reinterpret_cast<const float4*>(sQ + d);
                    if (a.metric == ANN_METRIC_IP) {
                        accA = fmaf(xa[i].x, q4.x, accA);
                        accA = fmaf(xa[i].y, q4.y, accA);
                        accA = fmaf(xa[i].z, q4.z, accA);
                        accA = fmaf(xa[i].w, q4.w, accA);
                        accB = fmaf(xb[i].x, q4.x, accB);
                        accB = fmaf(xb[i].y, q4.y, accB);
                        accB = fmaf(xb[i].z, q4.z, accB);
                        accB = fmaf(xb[i].w, q4.w, accB);
                    } else {
                        float t0 = xa[i].x - q4.x, t1 = xa[i].y - q4.y, t2 = xa[i].z - q4.z, t3 = xa[i].w - q4.w;
                        accA = fmaf(t0, t0, accA);
                        accA = fmaf(t1, t1, accA);
                        accA = fmaf(t2, t2, accA);
                        accA = fmaf(t3, t3, accA);
                        t0 = xb[i].x - q4.x, t1 = xb[i].y - q4.y, t2 = xb[i].z - q4.z, t3 = xb[i].w - q4.w;
                        accB = fmaf(t0, t0, accB);
                        accB = fmaf(t1, t1, accB);
                        accB = fmaf(t2, t2, accB);
                        accB = fmaf(t3, t3, accB);
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                accA += __shfl_xor_sync(0xffffffffu, accA, o);
                accB += __shfl_xor_sync(0xffffffffu, accB, o);
            }
            if (lane == 0) {
                sD[e0] = okA ? (a.metric == ANN_METRIC_IP ? -accA : accA) : kInf;
                if (e1 < R) sD[e1] = okB ? (a.metric == ANN_METRIC_IP ? -accB : accB) : kInf;
            }
        }
    } else {
        for (int e = warp; e < R; e += 8) {
            const int row = sRow[e];
            float acc = 0.f;
            if (row != kNoId) {
                const float* x = a.ix.original + (int64_t)row * dpad;
                for (int d = lane * 4; d < dpad; d += 128) {
                    const float4 xv = *reinterpret_cast<const float4*>(x + d);
                    const float4 q4 = *reinterpret_cast<const float4*>(sQ + d);
                    if (a.metric == ANN_METRIC_IP) {
                        acc = fmaf(xv.x, q4.x, acc);
                        acc = fmaf(xv.y, q4.y, acc);
                        acc = fmaf(xv.z, q4.z, acc);
                        acc = fmaf(xv.w, q4.w, acc);
                    } else {
                        const float d0 = xv.x - q4.x, d1 = xv.y - q4.y, d2 = xv.z - q4.z, d3 = xv.w - q4.w;
                        acc = fmaf(d0, d0, acc);
                        acc = fmaf(d1, d1, acc);
                        acc = fmaf(d2, d2, acc);
                        acc = fmaf(d3, d3, acc);
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) sD[e] = row != kNoId ? (a.metric == ANN_METRIC_IP ? -acc : acc) : kInf;
        }
    }
    __syncthreads();
    const float kEmpty = a.metric == ANN_METRIC_IP ? -kInf : kInf;
    if (R <= kRerankRankMax) {
        // The best k in order, every warp working: entries are ranked by (distance, row) (the rows are
        // distinct, so the ranks are) and an entry of rank < k goes to out[rank]. Ranking every entry
        // against all R costs R^2 comparisons; first, 256 linear bins over the valid distances find the bin
        // holding the k-th, and only the entries of that bin or lower (about k) are ranked, among themselves.
        __shared__ int sHist[kRerankBins];
        __shared__ float sRedF[2 * 32];
        __shared__ int sRedI[32 + 3];
        {
            float lo = kInf, hi = -kInf;
            int nv = 0;
            for (int e = threadIdx.x; e < R; e += blockDim.x)
                if (sRow[e] != kNoId) {
                    lo = fminf(lo, sD[e]);
                    hi = fmaxf(hi, sD[e]);
                    ++nv;
                }
            for (int i = threadIdx.x; i < kRerankBins; i += blockDim.x) sHist[i] = 0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
                nv += __shfl_xor_sync(0xffffffffu, nv, o);
            }
            const int nw = (int)(blockDim.x >> 5);
            if (lane == 0) {
                sRedF[warp] = lo;
                sRedF[32 + warp] = hi;
                sRedI[warp] = nv;
            }
            if (threadIdx.x == 0) sRedI[32] = 0;  // list length
            __syncthreads();
            lo = kInf;
            hi = -kInf;
            nv = 0;
            for (int w = 0; w < nw; ++w) {
                lo = fminf(lo, sRedF[w]);
                hi = fmaxf(hi, sRedF[32 + w]);
                nv += sRedI[w];
            }
            const float sc = (float)kRerankBins / (hi - lo);
            if (nv > k && hi > lo && isfinite(sc)) {  // uniform across the block
                auto bin_of = [&](float d) {
                    const float f = (d - lo) * sc;
                    return !(f > 0.f) ? 0 : (f >= (float)(kRerankBins - 1) ? kRerankBins - 1 : (int)f);
                };
                for (int e = threadIdx.x; e < R; e += blockDim.x)
                    if (sRow[e] != kNoId) atomicAdd(&sHist[bin_of(sD[e])], 1);
                __syncthreads();
                // the bin holding rank k - 1: one bin per thread, a warp-shuffle scan
                int incl = 0, own = 0;
                for (int b = threadIdx.x; b < kRerankBins; b += blockDim.x) own = sHist[b];
                incl = own;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                if (lane == 31) sRedI[warp] = incl;
                __syncthreads();
                for (int w = 0; w < warp; ++w) incl += sRedI[w];
                if (threadIdx.x < kRerankBins && k - 1 >= incl - own && k - 1 < incl) {
                    sRedI[33] = threadIdx.x;
                    sRedI[34] = incl;  // entries in this bin or lower
                }
                __syncthreads();
                const int bb = sRedI[33], m = sRedI[34];
                if (m <= topk_cap(k)) {
                    for (int e = threadIdx.x; e < R; e += blockDim.x)
                        if (sRow[e] != kNoId && bin_of(sD[e]) <= bb) {
                            const int slot = atomicAdd(&sRedI[32], 1);
                            sKey[slot] = sD[e];
                            sId[slot] = sRow[e];
                        }
                    __syncthreads();
                    for (int e = threadIdx.x; e < m; e += blockDim.x) {
                        const float key = sKey[e];
                        const int row = sId[e];
                        int rank = 0;
                        for (int j = 0; j < m; ++j) rank += pair_less(sKey[j], sId[j], key, row);
                        if (rank < k) {
                            a.out_ids[(int64_t)q * k + rank] = (int64_t)(a.ix.r2o ? a.ix.r2o[row] : row);
                            if (a.out_dists) a.out_dists[(int64_t)q * k + rank] = a.metric == ANN_METRIC_IP ? -key : key;
                        }
                    }
                    return;  // nv > k: all k slots written
                }
            }
            __syncthreads();
        }
        int nvalid = 0;
        for (int e = threadIdx.x; e < R; e += blockDim.x) {
            const int row = sRow[e];
            if (row == kNoId) continue;
            ++nvalid;
            const float key = sD[e];
            int rank = 0;
            for (int j = 0; j < R; ++j) rank += pair_less(sD[j], sRow[j], key, row);
            if (rank < k) {
                a.out_ids[(int64_t)q * k + rank] = (int64_t)(a.ix.r2o ? a.ix.r2o[row] : row);
                if (a.out_dists) a.out_dists[(int64_t)q * k + rank] = a.metric == ANN_METRIC_IP ? -key : key;
            }
        }
        nvalid = block_sum_int(nvalid, sKey);
        for (int e = nvalid + threadIdx.x; e < k; e += blockDim.x) {
            a.out_ids[(int64_t)q * k + e] = -1;
            if (a.out_dists) a.out_dists[(int64_t)q * k + e] = kEmpty;
        }
        return;
    }
    if (warp == 0) {
        WarpTopK top;
        top.init(sKey, sId, k);
        for (int e0 = 0; e0 < R; e0 += 32) {
            const int e = e0 + lane;
            const bool ok = e < R && sRow[e] != kNoId;
            top.offer(ok ? sD[e] : kInf, ok ? sRow[e] : kNoId, ok);
        }
        top.compact();
        for (int e = lane; e < k; e += 32) {
            const bool ok = e < top.count;
            a.out_ids[(int64_t)q * k + e] = ok ? (int64_t)(a.ix.r2o ? a.ix.r2o[sId[e]] : sId[e]) : -1;
            if (a.out_dists)
                a.out_dists[(int64_t)q * k + e] =
                    ok ? (a.metric == ANN_METRIC_IP ? -sKey[e] : sKey[e]) : kEmpty;
        }
    }
}

int launch_ivf_rerank(const IvfQueryArgs& a, const float* keyR, const int* idR, int reference, cudaStream_t st) {
    if (a.plan.nq == 0) return ANN_OK;
    const size_t smem = sizeof(float) * a.ix.dpad + (size_t)a.R * 8 + (size_t)topk_cap(a.k) * 8;
    ANN_CHECK_ARG(smem <= 227 * 1024, "re-rank: R=%d, k=%d need too much shared memory", a.R, a.k);
    if (reference) {
        ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(ivf_rerank_kernel<true>)));
        ivf_rerank_kernel<true><<<a.plan.nq, 256, smem, st>>>(a, keyR, idR);
    } else {
        ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(ivf_rerank_kernel<false>)));
        ivf_rerank_kernel<false><<<a.plan.nq, 256, smem, st>>>(a, keyR, idR);
    }
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

__global__ void clear_every_row_kernel(IvfPlan plan) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < plan.nq && plan.n_seg[q] < 0) {
        plan.n_seg[q] = 0;
        plan.n_cands[q] = 0;
    }
}

int launch_clear_every_row(const IvfPlan& plan, cudaStream_t st) {
    if (plan.nq == 0) return ANN_OK;
    clear_every_row_kernel<<<(unsigned)ceil_div(plan.nq, 256), 256, 0, st>>>(plan);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// Counting sort of the queries by first probed list, in one CTA: counts in shared memory, an
// exclusive scan, then each query placed at its list's cursor. The order inside a list follows the
// shared-memory atomics (the re-rank's results do not depend on it).
__global__ void __launch_bounds__(1024) query_order_kernel(const int32_t* __restrict__ probes, int npc, int nq, int C,
                                                           int32_t* __restrict__ order) {
    extern __shared__ int sCnt[];  // [C]
    __shared__ int sWarp[32];
    for (int c = threadIdx.x; c < C; c += blockDim.x) sCnt[c] = 0;
    __syncthreads();
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        const int c = probes[(int64_t)q * npc];
        if (c >= 0 && c < C) atomicAdd(&sCnt[c], 1);
    }
    __syncthreads();
    // exclusive scan of sCnt: each thread a contiguous run of lists
    const int per = (C + blockDim.x - 1) / blockDim.x;
    const int c0 = threadIdx.x * per, c1 = min(C, c0 + per);
    int run = 0;
    for (int c = c0; c < c1; ++c) run += sCnt[c];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane == 31) sWarp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (int)(blockDim.x >> 5) ? sWarp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += v;
        }
        sWarp[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    int acc = inc - run + (warp > 0 ? sWarp[warp - 1] : 0);
    for (int c = c0; c < c1; ++c) {
        const int v = sCnt[c];
        sCnt[c] = acc;
        acc += v;
    }
    __syncthreads();
    // queries without a valid first list go last, in order
    const int n_valid = sWarp[(blockDim.x >> 5) - 1];
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        const int c = probes[(int64_t)q * npc];
        if (c >= 0 && c < C) order[atomicAdd(&sCnt[c], 1)] = q;
    }
    if (n_valid < nq && threadIdx.x == 0) {
        int pos = n_valid;
        for (int q = 0; q < nq; ++q) {
            const int c = probes[(int64_t)q * npc];
            if (!(c >= 0 && c < C)) order[pos++] = q;
        }
    }
}

int launch_query_order(const int32_t* probes, int npc, int nq, int C, int32_t* order, cudaStream_t st) {
    ANN_CHECK_ARG(C >= 1 && C <= kQueryOrderMaxLists && npc >= 1, "query order: %d lists", C);
    if (nq == 0) return ANN_OK;
    const size_t smem = sizeof(int) * (size_t)C;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(query_order_kernel)));
    query_order_kernel<<<1, 1024, smem, st>>>(probes, npc, nq, C, order);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// ---- 1b. reference-mode coarse ranking ----------------------------------------------------------
// Dc[q][c] = compute_l2_distance(q, centroid_c) with the reference's arithmetic (:326-331).
__global__ void __launch_bounds__(256) ref_centroid_kernel(IvfView ix, const float* __restrict__ q, int64_t ldq,
                                                           float* __restrict__ Dc) {
    extern __shared__ float sQ[];
    const int qi = blockIdx.x;
    for (int d = threadIdx.x; d < ix.dim; d += blockDim.x) sQ[d] = q[(int64_t)qi * ldq + d];
    __syncthreads();
    const int grp = threadIdx.x >> 4;
    for (int c0 = blockIdx.y * 16; c0 < ix.C; c0 += gridDim.y * 16) {
        const int c = c0 + grp;
        const bool ok = c < ix.C;
        const float d = ref_l2_f32(sQ, ix.centroids + (int64_t)(ok ? c : 0) * ix.dpad, ix.dim, NoEmit{});
        if (ok && (threadIdx.x & 15) == 0) Dc[(int64_t)qi * ix.C + c] = d;
    }
}

int launch_ref_centroid_dists(const IvfView& ix, const float* q, int64_t ldq, int nq, float* Dc, cudaStream_t st) {
    if (nq == 0) return ANN_OK;
    const size_t smem = sizeof(float) * ix.dim;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(ref_centroid_kernel)));
    dim3 g(nq, (unsigned)std::min<int64_t>(ceil_div(ix.C, 16), 64));
    ref_centroid_kernel<<<g, 256, smem, st>>>(ix, q, ldq, Dc);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

// Exact FP32 brute-force scan with fused top-k: the B200 form of the reference's linear scan
// (LinearIndex::query, competitors/linear/src/linear_index.cpp:90-121, distance kernel
// competitors/linear/src/simd.h:32-115) in its exact semantics: the true top-k by
// (squared L2 distance, id), or by (-inner product, id).
//
// Layout: base rows [n, dpad] FP32 in HBM, dpad = dim rounded up to 32 floats with zero padding
// (zeros add nothing to either metric). Grid = (query tiles of BQ) x (row splits). Each CTA
// streams its split's rows through a cp.async shared-memory pipeline in KC=32-float chunks,
// keeps its BQ queries' chunks beside them, and computes a BQ x BR distance tile per thread
// micro-tile (TQ queries x TR rows, direct sum of (x - q)^2). After each row tile, distances that
// beat a query's current k-th best are appended to that query's shared-memory buffer, which one
// warp sorts and truncates to k when it fills. Each CTA writes its split's top-k; a merge kernel
// reduces the splits to the final top-k per query.
//
// Roofline: one pass over the base per query tile: N*dpad*4 bytes, 2*N*dpad FP32 instructions
// per query (sub + fma for L2; 1 fma for IP). HBM-bound below ~11 queries per tile, FP32-bound
// above.
#include "common.cuh"
#include "flat_scan.cuh"

namespace annb {

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int sz = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// One warp sorts a query's shared-memory buffer (`*count` entries, at most cap) and keeps the
// best k, updating the bar (tau, tau_id) once k entries are held.
__device__ __forceinline__ void smem_compact(float* key, int* id, int* count, float* tau, int* tau_id, int cap, int k) {
    const int kept = warp_compact_smem(key, id, *count, cap, k);
    if ((threadIdx.x & 31) == 0) {
        *count = kept;
        if (kept == k) {
            *tau = key[k - 1];
            *tau_id = id[k - 1];
        }
    }
    __syncwarp();
}

template <int BQ, int TQ, int TR, int STAGES, int METRIC>
struct ScanCfg {
    static constexpr int THREADS = 256;
    static constexpr int WQ = BQ / TQ;
    static constexpr int WR = THREADS / WQ;
    static constexpr int BR = WR * TR;
    static constexpr int KC = 32;
    static constexpr int PITCH = KC + 4;  // floats; 16-byte pad keeps 128-bit row reads conflict-free
    static constexpr size_t SX = (size_t)BR * PITCH;  // floats per stage
    static constexpr size_t SQ = (size_t)BQ * PITCH;
    static constexpr size_t PIPE = sizeof(float) * STAGES * (SX + SQ);
    static size_t smem(int cap) { return PIPE + (size_t)BQ * cap * 8 + (size_t)BQ * 16; }
    static_assert(WR >= 32, "a warp must share one query group so query reads broadcast");
    static_assert(BQ % TQ == 0 && THREADS % WQ == 0, "bad tile");
};

// PQ: the query tile comes from FlatScanArgs::qpair (query pairs interleaved element by element, negated for
// L2), staged per chunk as BQ / 2 rows of 2 KC floats; thread query pairs (2 jj, 2 jj + 1) share each x element
// through packed FP32 instructions (x - q as x + (-q), then fma, per half exactly the scalar steps)
template <int BQ, int TQ, int TR, int STAGES, int METRIC, bool PQ>
__global__ void __launch_bounds__(256) flat_scan_kernel(FlatScanArgs a) {
    using C = ScanCfg<BQ, TQ, TR, STAGES, METRIC>;
    static_assert(!PQ || TQ % 2 == 0, "query pairs");
    constexpr int PITCHQ = 2 * C::KC + 4;  // paired query tile: floats per pair row
    constexpr int TQ2 = TQ / 2 > 0 ? TQ / 2 : 1;
    static_assert(!PQ || (BQ / 2) * PITCHQ <= (int)C::SQ, "paired query tile fits the query stage");
    const int cap = a.cap;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sX = reinterpret_cast<float*>(smem_raw);
    float* sQ = sX + STAGES * C::SX;
    float* sKey = sQ + STAGES * C::SQ;
    int* sId = reinterpret_cast<int*>(sKey + BQ * cap);
    int* sCnt = sId + BQ * cap;
    float* sTau = reinterpret_cast<float*>(sCnt + BQ);
    int* sTauId = reinterpret_cast<int*>(sTau + BQ);

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int tq = tid / C::WR;
    const int tr = tid % C::WR;
    const int q0 = blockIdx.x * BQ;
    const int split = blockIdx.y;
    const int64_t row_begin = (int64_t)split * a.rows_per_split;
    int64_t row_end = row_begin + a.rows_per_split;
    if (row_end > a.n) row_end = a.n;
    const int k = a.k;

    for (int i = tid; i < BQ; i += C::THREADS) {
        sCnt[i] = 0;
        sTau[i] = kInf;
        sTauId[i] = kNoId;
    }

    const int nkc = a.dpad / C::KC;
    const int64_t ntiles = row_end > row_begin ? ceil_div(row_end - row_begin, C::BR) : 0;
    const int64_t nsteps = ntiles * nkc;

    auto issue = [&](int64_t step) {
        if (step < nsteps) {
            const int buf = (int)(step % STAGES);
            const int64_t t = step / nkc;
            const int kc = (int)(step % nkc);
            const int64_t r0 = row_begin + t * C::BR;
            float* dx = sX + buf * C::SX;
            // BR rows x 8 16-byte pieces
#pragma unroll
            for (int c = tid; c < C::BR * 8; c += C::THREADS) {
                const int r = c >> 3, piece = c & 7;
                const int64_t row = r0 + r;
                const bool ok = row < row_end;
                const float* src = a.base + (ok ? row : row_begin) * (int64_t)a.dpad + kc * C::KC + piece * 4;
                cp_async16(dx + r * C::PITCH + piece * 4, src, ok);
            }
            float* dq = sQ + buf * C::SQ;
            if constexpr (PQ) {
                for (int c = tid; c < (BQ / 2) * 16; c += C::THREADS) {  // pair rows x 16 16-byte pieces
                    const int pp = c >> 4, piece = c & 15;
                    const int64_t pr = q0 / 2 + pp;
                    const bool ok = 2 * pr < a.nq;
                    const float* src = a.qpair + ((ok ? pr : 0) * a.dpad + kc * C::KC) * 2 + piece * 4;
                    cp_async16(dq + pp * PITCHQ + piece * 4, src, ok);
                }
            } else {
                for (int c = tid; c < BQ * 8; c += C::THREADS) {
                    const int qq = c >> 3, piece = c & 7;
                    const bool ok = (q0 + qq) < a.nq;
                    const float* src = a.q + (int64_t)(ok ? q0 + qq : 0) * a.dpad + kc * C::KC + piece * 4;
                    cp_async16(dq + qq * C::PITCH + piece * 4, src, ok);
                }
            }
        }
        cp_async_commit();
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) issue(s);

    float acc[TQ][TR];
#pragma unroll
    for (int j = 0; j < TQ; ++j)
#pragma unroll
        for (int i = 0; i < TR; ++i) acc[j][i] = 0.f;
    float2 acc2[TQ2][TR];  // PQ: queries (2 jj, 2 jj + 1) of row i
#pragma unroll
    for (int jj = 0; jj < TQ2; ++jj)
#pragma unroll
        for (int i = 0; i < TR; ++i) acc2[jj][i] = make_float2(0.f, 0.f);

    for (int64_t step = 0; step < nsteps; ++step) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        issue(step + STAGES - 1);
        const int buf = (int)(step % STAGES);
        const float* xs = sX + buf * C::SX;
        const float* qs = sQ + buf * C::SQ;
#pragma unroll
        for (int kk = 0; kk < C::KC && PQ; kk += 4) {
            float4 xv[TR], qa[TQ2], qb[TQ2];
#pragma unroll
            for (int i = 0; i < TR; ++i) xv[i] = *reinterpret_cast<const float4*>(xs + (tr + i * C::WR) * C::PITCH + kk);
#pragma unroll
            for (int jj = 0; jj < TQ2; ++jj) {  // (A kk, B kk, A kk+1, B kk+1), (A kk+2, B kk+2, A kk+3, B kk+3)
                const float* qp = qs + (tq * (TQ / 2) + jj) * PITCHQ + 2 * kk;
                qa[jj] = *reinterpret_cast<const float4*>(qp);
                qb[jj] = *reinterpret_cast<const float4*>(qp + 4);
            }
#pragma unroll
            for (int jj = 0; jj < TQ2; ++jj)
#pragma unroll
                for (int i = 0; i < TR; ++i) {
                    const float2 q0v = make_float2(qa[jj].x, qa[jj].y), q1v = make_float2(qa[jj].z, qa[jj].w);
                    const float2 q2v = make_float2(qb[jj].x, qb[jj].y), q3v = make_float2(qb[jj].z, qb[jj].w);
                    if (METRIC == ANN_METRIC_L2) {  // the pairs hold -q: x + (-q) is x - q
                        const float2 d0 = __fadd2_rn(make_float2(xv[i].x, xv[i].x), q0v);
                        const float2 d1 = __fadd2_rn(make_float2(xv[i].y, xv[i].y), q1v);
                        const float2 d2 = __fadd2_rn(make_float2(xv[i].z, xv[i].z), q2v);
                        const float2 d3 = __fadd2_rn(make_float2(xv[i].w, xv[i].w), q3v);
                        acc2[jj][i] = __ffma2_rn(d0, d0, acc2[jj][i]);
                        acc2[jj][i] = __ffma2_rn(d1, d1, acc2[jj][i]);
                        acc2[jj][i] = __ffma2_rn(d2, d2, acc2[jj][i]);
                        acc2[jj][i] = __ffma2_rn(d3, d3, acc2[jj][i]);
                    } else {
                        acc2[jj][i] = __ffma2_rn(make_float2(xv[i].x, xv[i].x), q0v, acc2[jj][i]);
                        acc2[jj][i] = __ffma2_rn(make_float2(xv[i].y, xv[i].y), q1v, acc2[jj][i]);
                        acc2[jj][i] = __ffma2_rn(make_float2(xv[i].z, xv[i].z), q2v, acc2[jj][i]);
                        acc2[jj][i] = __ffma2_rn(make_float2(xv[i].w, xv[i].w), q3v, acc2[jj][i]);
                    }
                }
        }
#pragma unroll
        for (int kk = 0; kk < C::KC && !PQ; kk += 4) {
            float4 xv[TR], qv[TQ];
#pragma unroll
            for (int i = 0; i < TR; ++i) xv[i] = *reinterpret_cast<const float4*>(xs + (tr + i * C::WR) * C::PITCH + kk);
#pragma unroll
            for (int j = 0; j < TQ; ++j) qv[j] = *reinterpret_cast<const float4*>(qs + (tq * TQ + j) * C::PITCH + kk);
#pragma unroll
            for (int j = 0; j < TQ; ++j)
#pragma unroll
                for (int i = 0; i < TR; ++i) {
                    if (METRIC == ANN_METRIC_L2) {
                        float d0 = xv[i].x - qv[j].x, d1 = xv[i].y - qv[j].y;
                        float d2 = xv[i].z - qv[j].z, d3 = xv[i].w - qv[j].w;
                        acc[j][i] = fmaf(d0, d0, acc[j][i]);
                        acc[j][i] = fmaf(d1, d1, acc[j][i]);
                        acc[j][i] = fmaf(d2, d2, acc[j][i]);
                        acc[j][i] = fmaf(d3, d3, acc[j][i]);
                    } else {
                        acc[j][i] = fmaf(xv[i].x, qv[j].x, acc[j][i]);
                        acc[j][i] = fmaf(xv[i].y, qv[j].y, acc[j][i]);
                        acc[j][i] = fmaf(xv[i].z, qv[j].z, acc[j][i]);
                        acc[j][i] = fmaf(xv[i].w, qv[j].w, acc[j][i]);
                    }
                }
        }

        if ((int)(step % nkc) == nkc - 1) {
            // ---- epilogue for row tile t: offer distances to the per-query buffers ----
            const int64_t r0 = row_begin + (step / nkc) * C::BR;
            uint32_t pend = 0;
#pragma unroll
            for (int j = 0; j < TQ; ++j)
#pragma unroll
                for (int i = 0; i < TR; ++i) {
                    const int64_t row = r0 + tr + i * C::WR;
                    if (row < row_end && q0 + tq * TQ + j < a.nq) pend |= 1u << (j * TR + i);
                }
            while (true) {
#pragma unroll
                for (int j = 0; j < TQ; ++j) {
                    const int ql = tq * TQ + j;
#pragma unroll
                    for (int i = 0; i < TR; ++i) {
                        const uint32_t bit = 1u << (j * TR + i);
                        if (pend & bit) {
                            const int row = (int)(r0 + tr + i * C::WR);
                            const float av = PQ ? ((j & 1) ? acc2[j >> 1][i].y : acc2[j >> 1][i].x) : acc[j][i];
                            const float key = METRIC == ANN_METRIC_L2 ? av : -av;
                            if (pair_less(key, row, sTau[ql], sTauId[ql])) {
                                const int slot = atomicAdd(&sCnt[ql], 1);
                                if (slot < cap) {
                                    sKey[ql * cap + slot] = key;
                                    sId[ql * cap + slot] = row;
                                    pend &= ~bit;
                                }
                            } else {
                                pend &= ~bit;
                            }
                        }
                    }
                }
                const int overflow = __syncthreads_or(pend != 0);
                for (int ql = warp; ql < BQ; ql += C::THREADS / 32) {
                    if (sCnt[ql] >= cap / 2)
                        smem_compact(sKey + ql * cap, sId + ql * cap, &sCnt[ql], &sTau[ql], &sTauId[ql], cap, k);
                }
                __syncthreads();
                if (!overflow) break;
            }
#pragma unroll
            for (int j = 0; j < TQ; ++j)
#pragma unroll
                for (int i = 0; i < TR; ++i) acc[j][i] = 0.f;
#pragma unroll
            for (int jj = 0; jj < TQ2; ++jj)
#pragma unroll
                for (int i = 0; i < TR; ++i) acc2[jj][i] = make_float2(0.f, 0.f);
        }
    }
    cp_async_wait<0>();
    __syncthreads();

    // ---- final: each query's split top-k, sorted, padded with (+inf, INT_MAX) ----
    for (int ql = warp; ql < BQ; ql += C::THREADS / 32) {
        const int qi = q0 + ql;
        if (qi >= a.nq) continue;
        smem_compact(sKey + ql * cap, sId + ql * cap, &sCnt[ql], &sTau[ql], &sTauId[ql], cap, k);
        const int cnt = sCnt[ql];
        float* ok = a.out_key + ((int64_t)qi * a.nsplit + split) * k;
        int* oi = a.out_id + ((int64_t)qi * a.nsplit + split) * k;
        for (int e = threadIdx.x & 31; e < k; e += 32) {
            ok[e] = e < cnt ? sKey[ql * cap + e] : kInf;
            oi[e] = e < cnt ? sId[ql * cap + e] : kNoId;
        }
    }
}

// Merge kernel: one CTA (8 warps) per query reduces nsplit sorted lists of kin pairs to the
// final top-k. Each warp keeps a private top-k over a strided share of the lists; warp 0 then
// merges the eight.
__global__ void __launch_bounds__(256) merge_splits_kernel(MergeArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int cap = topk_cap(a.k);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* sKey = reinterpret_cast<float*>(smem_raw);
    int* sId = reinterpret_cast<int*>(sKey + 8 * cap);
    const int qi = blockIdx.x;
    const int k = a.k;
    WarpTopK top;
    top.init(sKey + warp * cap, sId + warp * cap, k);
    const int64_t total = (int64_t)a.nsplit * a.kin;
    const float* ik = a.in_key + (int64_t)qi * total;
    const int* ii = a.in_id + (int64_t)qi * total;
    for (int64_t base = (int64_t)warp * 32; base < total; base += 8 * 32) {
        const int64_t e = base + lane;
        float kv = kInf;
        int iv = kNoId;
        if (e < total) {
            kv = ik[e];
            iv = ii[e];
        }
        top.offer(kv, iv, e < total && iv != kNoId);
    }
    top.compact();
    __syncthreads();
    if (warp == 0) {
        for (int w = 1; w < 8; ++w) {
            for (int e0 = 0; e0 < k; e0 += 32) {
                const int e = e0 + lane;
                const bool ok = e < k;
                const float kv = ok ? sKey[w * cap + e] : kInf;
                const int iv = ok ? sId[w * cap + e] : kNoId;
                top.offer(kv, iv, ok && iv != kNoId);
            }
        }
        top.compact();
        const int cnt = top.count;
        for (int e = lane; e < k; e += 32) {
            const bool ok = e < cnt;
            const float kv = ok ? sKey[e] : kInf;
            const int iv = ok ? sId[e] : kNoId;
            if (a.out_ids) a.out_ids[(int64_t)qi * k + e] = ok ? (int64_t)iv : -1;
            if (a.out_dists) a.out_dists[(int64_t)qi * k + e] = ok ? (a.negate ? -kv : kv) : (a.negate ? -kInf : kInf);
            if (a.out_id32) a.out_id32[(int64_t)qi * k + e] = ok ? iv : kNoId;
            if (a.out_key32) a.out_key32[(int64_t)qi * k + e] = ok ? kv : kInf;
        }
    }
}

// One warp per query sorts its set of k (key, id) pairs (any order, kNoId padding) by (key, id) and
// writes the final top-k: int64 ids (-1 for padding) and distances (negated back for inner product).
__global__ void sort_topk_kernel(const float* __restrict__ keys, const int* __restrict__ ids, int nq, int k, int negate,
                                 int64_t* out_ids, float* out_dists) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int cap = topk_cap(k);
    float* sKey = reinterpret_cast<float*>(smem_raw);
    int* sId = reinterpret_cast<int*>(sKey + cap);
    const int q = blockIdx.x;
    const int lane = threadIdx.x;
    for (int e = lane; e < cap; e += 32) {
        const bool ok = e < k && ids[(int64_t)q * k + e] != kNoId;
        sKey[e] = ok ? keys[(int64_t)q * k + e] : kInf;
        sId[e] = ok ? ids[(int64_t)q * k + e] : kNoId;
    }
    __syncwarp();
    warp_sort_smem(sKey, sId, cap);
    for (int e = lane; e < k; e += 32) {
        const bool ok = sId[e] != kNoId;
        if (out_ids) out_ids[(int64_t)q * k + e] = ok ? (int64_t)sId[e] : -1;
        if (out_dists) out_dists[(int64_t)q * k + e] = ok ? (negate ? -sKey[e] : sKey[e]) : (negate ? -kInf : kInf);
    }
}

int launch_sort_topk(const float* keys, const int* ids, int nq, int k, int negate, int64_t* out_ids, float* out_dists,
                     cudaStream_t st) {
    if (nq == 0) return ANN_OK;
    ANN_CHECK_ARG(k >= 1 && k <= 1024, "sort top-k: k=%d outside [1, 1024]", k);
    const size_t smem = (size_t)topk_cap(k) * 8;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(sort_topk_kernel)));
    sort_topk_kernel<<<nq, 32, smem, st>>>(keys, ids, nq, k, negate, out_ids, out_dists);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// Copies rows [n, dim] (row stride ld floats) into [n, dpad] with zero padding.
__global__ void pad_rows_kernel(const float* __restrict__ src, int64_t n, int dim, int64_t ld, float* __restrict__ dst,
                                int dpad) {
    const int64_t total = n * dpad;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / dpad;
        const int c = (int)(e % dpad);
        dst[e] = c < dim ? src[r * ld + c] : 0.f;
    }
}

int launch_pad_rows(const float* src, int64_t n, int dim, int64_t ld, float* dst, int dpad, cudaStream_t st) {
    if (n == 0) return ANN_OK;
    const int64_t total = n * dpad;
    int blocks = (int)std::min<int64_t>(ceil_div(total, 256), kNumSMs * 16);
    pad_rows_kernel<<<blocks, 256, 0, st>>>(src, n, dim, ld, dst, dpad);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// ---------------------------------------------------------------------------------------------
// Streaming form for 1, 2 or 4 queries per CTA, where the scan is HBM-bound: no shared-memory
// staging of the base. Each warp reads 4 rows at a time, 8 lanes per row, each lane a 16-byte piece
// of every 128-byte stretch of its row (coalesced 128-byte reads), straight into registers; the 8
// lanes combine their partial sums with three shuffles. The queries sit in shared memory (read as
// broadcasts). Every warp keeps its own top-k per query (WarpTopK, no block barriers while
// scanning); at the end one warp per query merges the eight warps' lists into the split's top-k.
// ---------------------------------------------------------------------------------------------
constexpr int kStreamWarps = 8;
constexpr int kStreamBatch = 12;  // 16-byte loads in flight per lane (a 384-float row in one batch)

template <int BQ, int METRIC>
__global__ void __launch_bounds__(32 * kStreamWarps) flat_stream_kernel(FlatScanArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int dpad = a.dpad, cap = a.cap, k = a.k;
    float* sQ = reinterpret_cast<float*>(smem_raw);                 // [BQ][dpad]
    float* bufK = sQ + BQ * dpad;                                   // [warps][BQ][cap]
    int* bufI = reinterpret_cast<int*>(bufK + kStreamWarps * BQ * cap);
    int* sCount = bufI + kStreamWarps * BQ * cap;                   // [warps][BQ]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int oct = lane >> 3, o = lane & 7;
    const int q0 = blockIdx.x * BQ;
    const int split = blockIdx.y;
    const int64_t row_begin = (int64_t)split * a.rows_per_split;
    const int64_t row_end = min(row_begin + a.rows_per_split, a.n);
    for (int i = threadIdx.x; i < BQ * dpad; i += blockDim.x) {
        const int qi = i / dpad;
        sQ[i] = q0 + qi < a.nq ? a.q[(int64_t)(q0 + qi) * dpad + (i - qi * dpad)] : 0.f;
    }
    __syncthreads();
    WarpTopK top[BQ];
#pragma unroll
    for (int qi = 0; qi < BQ; ++qi) top[qi].init(bufK + (warp * BQ + qi) * cap, bufI + (warp * BQ + qi) * cap, k);
    const int nj = dpad / 32;
    for (int64_t r0 = row_begin + warp * 4; r0 < row_end; r0 += 4 * kStreamWarps) {
        const int64_t row = r0 + oct;
        const bool valid = row < row_end;
        const float4* x = reinterpret_cast<const float4*>(a.base + (valid ? row : row_begin) * (int64_t)dpad) + o;
        const float4* qv4 = reinterpret_cast<const float4*>(sQ) + o;
        float acc[BQ];
#pragma unroll
        for (int qi = 0; qi < BQ; ++qi) acc[qi] = 0.f;
        for (int j0 = 0; j0 < nj; j0 += kStreamBatch) {
            // every load of the batch is issued before the first is used
            float4 xb[kStreamBatch];
#pragma unroll
            for (int u = 0; u < kStreamBatch; ++u)
                if (j0 + u < nj) xb[u] = __ldcs(x + 8 * (j0 + u));
#pragma unroll
            for (int u = 0; u < kStreamBatch; ++u) {
            if (j0 + u >= nj) break;
            const int j = j0 + u;
            const float4 xv = xb[u];
#pragma unroll
            for (int qi = 0; qi < BQ; ++qi) {
                const float4 qv = qv4[qi * (dpad / 4) + 8 * j];
                if (METRIC == ANN_METRIC_L2) {
                    const float d0 = xv.x - qv.x, d1 = xv.y - qv.y, d2 = xv.z - qv.z, d3 = xv.w - qv.w;
                    acc[qi] = fmaf(d0, d0, acc[qi]);
                    acc[qi] = fmaf(d1, d1, acc[qi]);
                    acc[qi] = fmaf(d2, d2, acc[qi]);
                    acc[qi] = fmaf(d3, d3, acc[qi]);
                } else {
                    acc[qi] = fmaf(xv.x, qv.x, acc[qi]);
                    acc[qi] = fmaf(xv.y, qv.y, acc[qi]);
                    acc[qi] = fmaf(xv.z, qv.z, acc[qi]);
                    acc[qi] = fmaf(xv.w, qv.w, acc[qi]);
                }
            }
            }
        }
        float key = kInf;
#pragma unroll
        for (int qi = 0; qi < BQ; ++qi) {
            float v = acc[qi];
            v += __shfl_xor_sync(0xffffffffu, v, 1);
            v += __shfl_xor_sync(0xffffffffu, v, 2);
            v += __shfl_xor_sync(0xffffffffu, v, 4);
            if (o == qi) key = METRIC == ANN_METRIC_L2 ? v : -v;
        }
#pragma unroll
        for (int qi = 0; qi < BQ; ++qi) top[qi].offer(key, (int)row, valid && o == qi && q0 + qi < a.nq);
    }
#pragma unroll
    for (int qi = 0; qi < BQ; ++qi) {
        top[qi].compact();
        if (lane == 0) sCount[warp * BQ + qi] = top[qi].count;
    }
    __syncthreads();
    // warp qi merges query qi's lists from the other warps into its own
#pragma unroll
    for (int qi = 0; qi < BQ; ++qi) {
        if (warp != qi || q0 + qi >= a.nq) continue;
        for (int w = 0; w < kStreamWarps; ++w) {
            if (w == warp) continue;
            const int cnt = sCount[w * BQ + qi];
            const float* wk = bufK + (w * BQ + qi) * cap;
            const int* wi = bufI + (w * BQ + qi) * cap;
            for (int e0 = 0; e0 < cnt; e0 += 32) {
                const int e = e0 + lane;
                const bool ok = e < cnt;
                top[qi].offer(ok ? wk[e] : kInf, ok ? wi[e] : kNoId, ok);
            }
        }
        top[qi].compact();
        const int cnt = top[qi].count;
        float* okey = a.out_key + ((int64_t)(q0 + qi) * a.nsplit + split) * k;
        int* oid = a.out_id + ((int64_t)(q0 + qi) * a.nsplit + split) * k;
        for (int e = lane; e < k; e += 32) {
            okey[e] = e < cnt ? top[qi].key[e] : kInf;
            oid[e] = e < cnt ? top[qi].id[e] : kNoId;
        }
    }
}

static size_t stream_smem(int bq, int dpad, int cap) {
    return sizeof(float) * (size_t)bq * dpad + (size_t)kStreamWarps * bq * cap * 8 + sizeof(int) * kStreamWarps * bq;
}

bool flat_stream_eligible(int bq, int k, int dpad) {
    return (bq == 1 || bq == 2 || bq == 4) && stream_smem(bq, dpad, topk_cap(k)) <= 100 * 1024;
}

template <int BQ, int METRIC>
static int stream_occupancy(int dpad, int cap) {
    auto kern = flat_stream_kernel<BQ, METRIC>;
    const size_t smem = stream_smem(BQ, dpad, cap);
    if (smem_optin(reinterpret_cast<const void*>(kern)) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    int nb = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 32 * kStreamWarps, smem) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return std::max(1, nb);
}

int flat_scan_ctas_per_sm(int bq, int k, int dpad, int metric) {
    if (!flat_stream_eligible(bq, k, dpad)) return 1;
    const int cap = topk_cap(k);
    const bool l2 = metric == ANN_METRIC_L2;
    switch (bq) {
    case 1: return l2 ? stream_occupancy<1, ANN_METRIC_L2>(dpad, cap) : stream_occupancy<1, ANN_METRIC_IP>(dpad, cap);
    case 2: return l2 ? stream_occupancy<2, ANN_METRIC_L2>(dpad, cap) : stream_occupancy<2, ANN_METRIC_IP>(dpad, cap);
    default: return l2 ? stream_occupancy<4, ANN_METRIC_L2>(dpad, cap) : stream_occupancy<4, ANN_METRIC_IP>(dpad, cap);
    }
}

template <int BQ, int METRIC>
static int launch_stream_t(const FlatScanArgs& a, int n_qtiles, cudaStream_t st) {
    auto kern = flat_stream_kernel<BQ, METRIC>;
    const size_t smem = stream_smem(BQ, a.dpad, a.cap);
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(kern)));
    dim3 grid(n_qtiles, a.nsplit);
    kern<<<grid, 32 * kStreamWarps, smem, st>>>(a);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

template <int METRIC>
static int dispatch_stream(const FlatScanArgs& a, int bq, int n_qtiles, cudaStream_t st) {
    switch (bq) {
    case 1: return launch_stream_t<1, METRIC>(a, n_qtiles, st);
    case 2: return launch_stream_t<2, METRIC>(a, n_qtiles, st);
    default: return launch_stream_t<4, METRIC>(a, n_qtiles, st);
    }
}

// ---------------------------------------------------------------------------------------------
// Host-side launch selection.
// ---------------------------------------------------------------------------------------------
template <int BQ, int TQ, int TR, int STAGES, int METRIC, bool PQ = false>
static int launch_scan_t(FlatScanArgs a, int n_qtiles, cudaStream_t st) {
    using C = ScanCfg<BQ, TQ, TR, STAGES, METRIC>;
    auto kern = flat_scan_kernel<BQ, TQ, TR, STAGES, METRIC, PQ>;
    const size_t smem = C::smem(a.cap);
    ANN_CHECK_ARG(smem <= 227 * 1024, "flat scan: %zu bytes of shared memory for k=%d", smem, a.k);
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(kern)));
    dim3 grid(n_qtiles, a.nsplit);
    kern<<<grid, C::THREADS, smem, st>>>(a);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// Largest query tile whose per-query top-k buffers still fit in shared memory.
int flat_scan_max_bq(int k) { return k <= 128 ? 32 : (k <= 256 ? 16 : 8); }

int flat_scan_bq(int nq) {
    if (nq <= 1) return 1;
    if (nq <= 2) return 2;
    if (nq <= 4) return 4;
    if (nq <= 8) return 8;
    if (nq <= 64) return 16;
    return 32;
}

template <int METRIC>
static int dispatch_bq(const FlatScanArgs& a, int bq, int n_qtiles, cudaStream_t st) {
    switch (bq) {
    case 1: return launch_scan_t<1, 1, 1, kSmallTileStages, METRIC>(a, n_qtiles, st);
    case 2: return launch_scan_t<2, 2, 1, kSmallTileStages, METRIC>(a, n_qtiles, st);
    case 4: return launch_scan_t<4, 4, 1, kSmallTileStages, METRIC>(a, n_qtiles, st);
    case 8: return launch_scan_t<8, 8, 1, kSmallTileStages, METRIC>(a, n_qtiles, st);
    case 16: return launch_scan_t<16, 8, 2, 3, METRIC>(a, n_qtiles, st);
    default:
        // the paired query tile where ptxas keeps it spill-free: 32-query tiles of squared L2
        if constexpr (METRIC == ANN_METRIC_L2) {
            if (a.qpair) return launch_scan_t<32, 8, 4, 3, METRIC, true>(a, n_qtiles, st);
        }
        return launch_scan_t<32, 8, 4, 3, METRIC>(a, n_qtiles, st);
    }
}

// qpair[(p dpad + d) 2 + h] = s q[2 p + h][d] (s = -1 for L2, +1 for inner products; 0 past nq)
__global__ void flat_pair_queries_kernel(const float* __restrict__ q, int nq, int dpad, float s,
                                         float* __restrict__ qpair) {
    const int64_t total = (int64_t)((nq + 1) / 2) * dpad * 2;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int h = (int)(e & 1);
        const int64_t pd = e >> 1;
        const int64_t p = pd / dpad;
        const int d = (int)(pd % dpad);
        const int64_t qi = 2 * p + h;
        qpair[e] = qi < nq ? s * q[qi * dpad + d] : 0.f;
    }
}

int launch_flat_scan(const FlatScanArgs& a0, int bq, cudaStream_t st) {
    ANN_CHECK_ARG(a0.k >= 1 && a0.k <= 512, "flat scan: k=%d outside [1, 512]", a0.k);
    ANN_CHECK_ARG(a0.dpad % 32 == 0, "flat scan: padded dim %d not a multiple of 32", a0.dpad);
    FlatScanArgs a = a0;
    a.cap = topk_cap(a.k);
    if (bq > flat_scan_max_bq(a.k)) bq = flat_scan_max_bq(a.k);
    const int n_qtiles = (int)ceil_div(a.nq, bq);
    if (flat_stream_eligible(bq, a.k, a.dpad)) {
        if (a.metric == ANN_METRIC_L2) return dispatch_stream<ANN_METRIC_L2>(a, bq, n_qtiles, st);
        return dispatch_stream<ANN_METRIC_IP>(a, bq, n_qtiles, st);
    }
    if (a.qpair && bq >= 32 && a.metric == ANN_METRIC_L2 && a.nq > 0) {  // the paired query tile
        const int64_t total = (int64_t)((a.nq + 1) / 2) * a.dpad * 2;
        flat_pair_queries_kernel<<<(unsigned)std::min<int64_t>(ceil_div(total, 256), 8 * kNumSMs), 256, 0, st>>>(
            a.q, a.nq, a.dpad, a.metric == ANN_METRIC_L2 ? -1.f : 1.f, a.qpair);
        ANN_LAUNCH_CHECK();
    } else {
        a.qpair = nullptr;
    }
    if (a.metric == ANN_METRIC_L2) return dispatch_bq<ANN_METRIC_L2>(a, bq, n_qtiles, st);
    return dispatch_bq<ANN_METRIC_IP>(a, bq, n_qtiles, st);
}

int launch_merge_splits(const MergeArgs& a, cudaStream_t st) {
    ANN_CHECK_ARG(a.k >= 1 && a.k <= 1024, "merge: k=%d outside [1, 1024]", a.k);
    if (a.nq == 0) return ANN_OK;
    const size_t smem = (size_t)8 * topk_cap(a.k) * 8;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(merge_splits_kernel)));
    merge_splits_kernel<<<a.nq, 256, smem, st>>>(a);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// ---- merge of per-shard top-k lists --------------------------------------------------------------------
// One warp per query: the parts' k pairs each (sorted by (key, id), id < 0 = empty) offered as (key, slot)
// with slot = part * k + position, the best k kept, slots mapped back to the parts' int64 ids. Parts hold
// increasing id ranges, so (key, slot) order is (key, id) order.
__global__ void __launch_bounds__(128) merge_parts_kernel(const float* __restrict__ d, const int64_t* __restrict__ ids,
                                                          int nq, int parts, int k, int ip, int64_t* __restrict__ out_ids,
                                                          float* __restrict__ out_d) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x * (blockDim.x >> 5) + warp;
    if (q >= nq) return;  // the whole warp; no block barrier follows
    const int cap = topk_cap(k);
    float* key = reinterpret_cast<float*>(smem_raw) + (size_t)warp * 2 * cap;
    int* slot = reinterpret_cast<int*>(key + cap);
    WarpTopK top;
    top.init(key, slot, k);
    const int64_t total = (int64_t)parts * k;
    const float* dq = d + (int64_t)q * total;
    const int64_t* iq = ids + (int64_t)q * total;
    for (int64_t e0 = 0; e0 < total; e0 += 32) {
        const int64_t e = e0 + lane;
        const bool ok = e < total && iq[e] >= 0;
        const float kv = ok ? (ip ? -dq[e] : dq[e]) : kInf;
        top.offer(kv, ok ? (int)iq[e] : kNoId, ok);  // ties by the lower id, whatever part holds it
    }
    top.compact();
    for (int e = lane; e < k; e += 32) {
        const bool ok = e < top.count;
        out_ids[(int64_t)q * k + e] = ok ? slot[e] : -1;
        if (out_d) out_d[(int64_t)q * k + e] = ok ? (ip ? -key[e] : key[e]) : (ip ? -kInf : kInf);
    }
}

int launch_merge_parts(const float* d, const int64_t* ids, int nq, int parts, int k, int ip, int64_t* out_ids,
                       float* out_d, cudaStream_t st) {
    ANN_CHECK_ARG(k >= 1 && k <= 1024 && parts >= 1 && (int64_t)parts * k < INT32_MAX,
                  "merge: %d parts of k=%d", parts, k);
    if (nq == 0) return ANN_OK;
    const size_t smem = (size_t)4 * topk_cap(k) * 8;
    ANN_CUDA_TRY(smem_optin(reinterpret_cast<const void*>(merge_parts_kernel)));
    merge_parts_kernel<<<(unsigned)ceil_div(nq, 4), 128, smem, st>>>(d, ids, nq, parts, k, ip, out_ids, out_d);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

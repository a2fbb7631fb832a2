// BF16 distance GEMM on the 5th-generation tensor cores (tcgen05 + TMA + TMEM) for sm_100a.
//
// keys[m][n] = sum_k A[m][k] * B[n][k] with A = queries [M, K] and B = base rows [N, K], both BF16
// row-major (K-major for the MMA), FP32 accumulation. The operands carry the key (tc_gemm.cuh): for
// squared L2 three extra columns add |b|^2 split into BF16 pieces against a query side scaled by -2,
// so the accumulator holds |b|^2 - 2 a.b and the epilogue does no arithmetic per key.
//
// Structure (one CTA per SM, persistent over 128 x 256 output tiles, query tiles fastest so a base
// tile is fetched from HBM once and reused from L2 by the query tiles that follow it):
//   warp 0    TMA producer: 128x64 A and 256x64 B boxes (128-byte swizzle) into a 4-stage ring,
//             mbarrier expect-tx completion; no multicast;
//   warp 1    allocates 512 TMEM columns (two 128 x 256 FP32 accumulators) and, from one thread,
//             issues tcgen05.mma (kind::f16, BF16 in, FP32 out, M = 128, N = 256, K = 16 per
//             instruction, 4 per stage); tcgen05.commit frees each stage and publishes each tile;
//   warps 2.. epilogue: 8 warps, two per TMEM lane quarter (warp w reads lanes 32 * (w % 4)), each
//             taking half of the 256 columns, for the key-matrix and grouped forms; 16 warps, four
//             per quarter taking 64 columns each, for the filter form, whose per-key test and
//             survivor compaction are bound by issue latency at two warps per scheduler.
//             tcgen05.ld 2 x 32 columns per wait, then either store the keys (transposed through
//             shared memory into coalesced rows) or, in filter mode, one test per key against the
//             row's bar (the sign bit of a packed FP32 difference, gathered by funnel shifts);
//             survivors go to the warp's own region at slots from a warp prefix sum (no atomics,
//             nothing waits on memory).
// Every mbarrier wait is bounded (about 2 s); a timeout raises a device flag and the CTA winds down.
#include <cuda.h>
#include <cuda_fp8.h>

#include "common.cuh"
#include "tc_gemm.cuh"

namespace annb {

namespace {

// A k-block is one 128-byte row per operand row: 64 BF16 or 128 E4M3 elements.
constexpr int kBM = 128, kBN = 256, kBK = 64;
constexpr int kRowBytes = 128;
constexpr int kABytes = kBM * kRowBytes;  // 16 KB
constexpr int kBBytes = kBN * kRowBytes;  // 32 KB
template <int KIND>
struct KindOf {
    static constexpr int kBlockK = KIND == kTcBF16 ? 64 : 128;  // elements per k-block
    static constexpr int kMmaK = KIND == kTcBF16 ? 16 : 32;     // elements per MMA
};
constexpr int kTmemCols = 512;

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// 4 bytes from global src to shared dst, asynchronously (zeros when !valid: no bytes are read)
__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(su32(dst)), "l"(src), "r"(valid ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t n) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(su32(b)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// try_wait that may suspend the thread for up to 0.1 ms (woken early when the phase completes), so a
// waiting warp takes few issue slots from the epilogue warps that share its scheduler
__device__ __forceinline__ bool bar_try_sleep(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity), "r"(100000u)
        : "memory");
    return ok != 0;
}
// Waits for the phase; gives up after `limit_ns` (2 s when 0), sets *err = 2 and returns false.
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity, int* err, uint64_t limit_ns = 0) {
    if (bar_try(b, parity)) return true;
    const uint64_t limit = limit_ns ? limit_ns : 2000000000ull;
    const uint64_t t0 = gtimer();
    while (!bar_try_sleep(b, parity))
        if (gtimer() - t0 > limit) {
            if (err) atomicExch(err, 2);
            return false;
        }
    return true;
}
__device__ __forceinline__ void bar_arrive(uint64_t* b) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ void bar_expect(uint64_t* b, uint32_t bytes) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(su32(b)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, int c0, int c1, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            su32(dst)),
        "l"(tm), "r"(c0), "r"(c1), "r"(su32(bar))
        : "memory");
}
// Shared-memory matrix descriptor for a K-major tile in the 128-byte swizzle layout (rows of 128 B,
// 8-row groups 1024 B apart): start address >> 4, leading offset 1 (unused with swizzle), stride
// offset 1024 >> 4, descriptor version 1, layout type 2 (128-byte swizzle).
__device__ __forceinline__ uint64_t sw128_desc(const void* p) {
    const uint64_t addr = (su32(p) >> 4) & 0x3FFFull;
    return addr | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}
// Instruction descriptors: FP32 accumulator (bits 4-5 = 1), A and B K-major, N = 256 (bits 17-22 = N / 8),
// M = 128 (bits 24-28 = M / 16); A and B types in bits 7-9 and 10-12: BF16 = 1 under kind::f16, E4M3 = 0
// under kind::f8f6f4.
constexpr uint32_t kIdescShape = (1u << 4) | ((uint32_t)(kBN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
constexpr uint32_t kIdescBF16 = kIdescShape | (1u << 7) | (1u << 10);
constexpr uint32_t kIdescE4M3 = kIdescShape;
// kind::i8: S32 accumulator (bits 4-5 = 2), A signed (bits 7-9 = 1), B unsigned (bits 10-12 = 0)
constexpr uint32_t kIdescI8 = (2u << 4) | ((uint32_t)(kBN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24) | (1u << 7);

// One MMA of the 32 bytes of K that follow each descriptor's start: 16 BF16 or 32 E4M3 elements.
template <int KIND>
__device__ __forceinline__ void mma_issue(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t accumulate) {
    if (KIND == kTcBF16)
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
            "l"(ad), "l"(bd), "r"(kIdescBF16), "r"(accumulate)
            : "memory");
    else if (KIND == kTcE4M3)
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
            "l"(ad), "l"(bd), "r"(kIdescE4M3), "r"(accumulate)
            : "memory");
    else
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
            "l"(ad), "l"(bd), "r"(kIdescI8), "r"(accumulate)
            : "memory");
}
// An accumulator read from TMEM as a float: FP32 bits, or (kind::i8) an int32 converted (exact below 2^24).
template <int KIND>
__device__ __forceinline__ float acc_value(uint32_t r) {
    return KIND == kTcI8 ? __int2float_rn((int)r) : __uint_as_float(r);
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}
// tcgen05.ld of 32 consecutive columns of the warp's 32 lanes; the registers are valid only after
// tmem_wait (which names them, so no use is scheduled before the wait).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
        "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait(uint32_t (&r)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                   "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                   "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
}
// Orders a second register set after the wait already issued for the first.
__device__ __forceinline__ void tmem_after_wait(uint32_t (&r)[32]) {
    asm volatile(""
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                   "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                   "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
}

// A grouped-mode work item: A rows [a0, a0 + am), B rows [b0, b0 + bn).
struct GroupTile {
    int64_t a0, b0;
    int am, bn;
};
__device__ __forceinline__ GroupTile tile_of_desc(int4 d) { return GroupTile{d.x, d.y, d.z, d.w}; }
__device__ __forceinline__ GroupTile group_tile(const TcGemmArgs& a, int64_t t) {
    if (a.g_item_desc) return tile_of_desc(a.g_item_desc[t]);
    int lo = 0, hi = a.g_lists - 1;
    if (a.g_item_list) {
        lo = a.g_item_list[t];  // one load, where a search would chain a dozen
    } else {
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.g_item_off[mid] <= t)
                lo = mid;
            else
                hi = mid - 1;
        }
    }
    const int64_t np = a.g_a_off[lo + 1] - a.g_a_off[lo];
    const int64_t nr = a.g_b_len ? a.g_b_len[lo] : a.g_b_off[lo + 1] - a.g_b_off[lo];
    const int64_t npt = (np + kBM - 1) / kBM;
    const int64_t local = t - a.g_item_off[lo];
    const int64_t g = local % npt, rt = local / npt;
    GroupTile gt;
    gt.a0 = a.g_a_off[lo] + g * kBM;
    gt.b0 = a.g_b_off[lo] + rt * kBN;
    gt.am = (int)min((int64_t)kBM, np - g * kBM);
    gt.bn = (int)min((int64_t)kBN, nr - rt * kBN);
    return gt;
}

// Epilogue warps of the key-matrix and grouped forms, and of the filter form; threads and shared memory
// (4 stages, 1 KB alignment slack, barriers, a per-warp area: a 32 x 33 transpose area, or in the filter
// form only its column factors, x and y) follow.
constexpr int kStages = 4;
constexpr int kKeyEpi = 8, kFilterEpi = 16;
constexpr int epi_threads(int epi) { return 64 + 32 * epi; }
constexpr int epi_area_floats(int epi) { return epi == kFilterEpi ? 2 * (kBN / (epi / 4)) : 32 * 33; }
constexpr size_t epi_smem(int epi) {
    return (size_t)kStages * (kABytes + kBBytes) + 1024 + 256 + (size_t)epi * epi_area_floats(epi) * 4;
}
static_assert(epi_smem(kKeyEpi) <= 232448 && epi_smem(kFilterEpi) <= 232448, "shared memory per CTA");

template <int KIND, int EPI>
__global__ void __launch_bounds__(epi_threads(EPI), 1) tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA,
                                                                     const __grid_constant__ CUtensorMap tmB,
                                                                     TcGemmArgs a) {
    constexpr int kCols = kBN / (EPI / 4);  // columns of a tile per epilogue warp
    constexpr bool kFilterOnly = EPI == kFilterEpi;
    if (a.skip_if_zero && *a.skip_if_zero == 0) return;  // every thread reads the same flag
    extern __shared__ unsigned char smem_raw[];
    // 1024-byte alignment for the swizzled tiles
    unsigned char* smem = smem_raw + ((1024 - (su32(smem_raw) & 1023)) & 1023);
    unsigned char* sA = smem;
    unsigned char* sB = smem + kStages * kABytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + kStages * kBBytes);
    uint64_t* empty = full + kStages;
    uint64_t* tfull = empty + kStages;
    uint64_t* tempty = tfull + 2;
    uint64_t* done = tempty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    float* sT = reinterpret_cast<float*>(smem + kStages * (kABytes + kBBytes) + 256);  // [EPI warps][area]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int kBlockK = KindOf<KIND>::kBlockK, kMmaK = KindOf<KIND>::kMmaK;
    const int mt = (int)ceil_div(a.M, kBM), nt = (int)ceil_div(a.N, kBN), kt = (int)ceil_div(a.K, kBlockK);
    const int k16_last = (a.K - (kt - 1) * kBlockK) / kMmaK;  // MMAs of the last k-block
    const bool grouped = a.g_item_off != nullptr;
    const int64_t tiles = grouped ? *a.g_total : (int64_t)mt * nt;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            bar_init(&full[s], 1);
            bar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            bar_init(&tfull[b], 1);
            bar_init(&tempty[b], 32 * EPI);
        }
        bar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // TMA producer (with test_no_loads it issues nothing, so that the other roles' bounded waits
        // run out with no copy in flight: the self-test of the timeout path)
        if (lane == 0 && !a.test_no_loads) {
            int64_t it = 0;
            bool ok = true;
            // with item descriptors, the next item's is loaded while this one's copies are issued
            const bool pre = grouped && a.g_item_desc != nullptr;
            int4 dnext = pre && (int64_t)blockIdx.x < tiles ? a.g_item_desc[blockIdx.x] : make_int4(0, 0, 0, 0);
            for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                int64_t arow, brow;
                if (pre) {
                    const int4 d = dnext;
                    if (t + gridDim.x < tiles) dnext = a.g_item_desc[t + gridDim.x];
                    arow = d.x;
                    brow = d.y;
                } else if (grouped) {
                    const GroupTile gt = group_tile(a, t);
                    arow = gt.a0;
                    brow = gt.b0;
                } else {
                    arow = (t % mt) * kBM;
                    brow = (t / mt) * kBN * a.b_tile_stride;
                }
                for (int kb = 0; kb < kt; ++kb, ++it) {
                    const int s = (int)(it % kStages);
                    const uint32_t ph = (uint32_t)((it / kStages) & 1);
                    if (!(ok = bar_wait(&empty[s], ph ^ 1u, a.err, a.wait_ns))) break;
                    bar_expect(&full[s], kABytes + kBBytes);
                    tma_load_2d(sA + s * kABytes, &tmA, kb * kBlockK, (int)arow, &full[s]);
                    tma_load_2d(sB + s * kBBytes, &tmB, kb * kBlockK, (int)brow, &full[s]);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            int64_t it = 0, acc = 0;
            bool ok = true;
            for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++acc) {
                const int b = (int)(acc & 1);
                const uint32_t aph = (uint32_t)((acc >> 1) & 1);
                if (!(ok = bar_wait(&tempty[b], aph ^ 1u, a.err, a.wait_ns))) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(b * kBN);
                for (int kb = 0; kb < kt; ++kb, ++it) {
                    const int s = (int)(it % kStages);
                    const uint32_t ph = (uint32_t)((it / kStages) & 1);
                    if (!(ok = bar_wait(&full[s], ph, a.err, a.wait_ns))) break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    // the last k-block's box runs past K (zero fill); its zero columns are not multiplied
                    const int n16 = kb == kt - 1 ? k16_last : kBlockK / kMmaK;
#pragma unroll
                    for (int k16 = 0; k16 < kBlockK / kMmaK; ++k16)
                        if (k16 < n16)
                            mma_issue<KIND>(d, sw128_desc(sA + s * kABytes + k16 * 32),
                                            sw128_desc(sB + s * kBBytes + k16 * 32), (kb | k16) ? 1u : 0u);
                    mma_commit(&empty[s]);
                }
                mma_commit(&tfull[b]);
            }
            // every MMA issued has completed before TMEM is released
            mma_commit(done);
            bar_wait(done, 0, nullptr);
        }
    } else {  // epilogue warps 2..9
        const int lane_base = 32 * (warp & 3);
        const int ew = warp - 2;
        const int col0 = kCols * (ew >> 2);  // this warp's share of the tile's columns
        float* tw = sT + ew * epi_area_floats(EPI);
        const int64_t wbase = ((int64_t)blockIdx.x * EPI + ew) * a.wcap;
        int wcount = 0;  // survivors met by this warp (uniform across the warp)
        int64_t acc = 0;
        for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x, ++acc) {
            const int b = (int)(acc & 1);
            // the tile's rows and columns, and the per-row values the filter needs, read before the wait for
            // the accumulator, so that their loads overlap the tile's MMAs: a dense tile, or a grouped one (a
            // list's pairs and rows; rows and columns past them belong to the next list and are masked like
            // rows past M)
            const int m0 = (int)(t % mt) * kBM, n0 = (int)(t / mt) * kBN;
            const int m = m0 + lane_base + lane;
            const GroupTile gt = grouped ? group_tile(a, t) : GroupTile{0, 0, 0, 0};
            int rq = m;                         // the row recorded for a survivor (grouped: its query)
            int64_t arow = m;                   // the A row (per-row factors)
            bool mvalid = m < a.M;
            int64_t cbase = n0;                 // recorded column of the tile's first column
            int ncols = a.N - n0;               // valid columns of the tile from its first
            if (grouped) {
                const int ml = lane_base + lane;
                mvalid = ml < gt.am;
                arow = gt.a0 + ml;
                rq = mvalid ? (a.g_row_query ? a.g_row_query[gt.a0 + ml] : (int)(gt.a0 + ml)) : 0;
                cbase = gt.b0;
                ncols = gt.bn;
            }
            const float an = (a.normA && mvalid) ? a.normA[arow] : 0.f;
            const float rfac = (a.row_fac && mvalid) ? a.row_fac[arow] : 1.f;
            // rows past M or past a grouped item's pairs get a NaN bar, which no key passes (not even a -inf
            // key, which a -inf bar would let through)
            const float tau = (a.tau && mvalid) ? a.tau[rq] : __int_as_float(0x7fffffff);
            // filter mode with scaled operands: the warp's kCols column factors, copied here (asynchronously,
            // so that they land while the MMAs run) into its (otherwise unused) transpose buffer as two arrays
            // (x then y), so that the factors of two adjacent columns load as one float2 broadcast; zeros past
            // the valid columns
            const bool staged = a.col_fac != nullptr && (kFilterOnly || a.out == nullptr);
            float* sfx = tw;
            float* sfy = tw + kCols;
            if (staged) {
                __syncwarp();  // every lane is done with the last tile's factors
#pragma unroll
                for (int i = 0; i < kCols / 32; ++i) {
                    const int lcol = col0 + 32 * i + lane;  // column within the tile
                    const int col = n0 + lcol;
                    const int64_t nrow = grouped ? cbase + lcol : (int64_t)(col / kBN) * kBN * a.b_tile_stride + col % kBN;
                    const bool in = lcol < ncols;
                    const float* src = reinterpret_cast<const float*>(a.col_fac + (in ? nrow : 0));
                    cp_async4(sfx + 32 * i + lane, src, in);
                    cp_async4(sfy + 32 * i + lane, src + 1, in);
                }
            }
            // every lane waits; the warp leaves together if any lane gave up, so that no lane is left
            // behind at a warp-wide instruction
            const bool got = bar_wait(&tfull[b], (uint32_t)((acc >> 1) & 1), a.err, a.wait_ns);
            if (!__all_sync(0xffffffffu, got)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (!kFilterOnly && grouped) {  // keys of pair a0 + row, list rows b0 + column, to their stream positions
                const int ml = lane_base + lane;
                // the stream position of list row b0 for each of the warp's 32 pairs (lane r holds row r's)
                const int64_t dst_lane = (ml < gt.am ? a.g_dbase[gt.a0 + ml] : 0) + gt.b0;
                const int rows = min(32, gt.am - lane_base);  // valid pairs of this warp
                const float grf = (a.row_fac && ml < gt.am) ? a.row_fac[gt.a0 + ml] : 1.f;
                const uint32_t tb = tmem + ((uint32_t)lane_base << 16) + (uint32_t)(b * kBN + col0);
#pragma unroll 1
                for (int c = 0; c < kCols; c += 64) {
                    uint32_t r0[32], r1[32];
                    __syncwarp();  // tcgen05.ld is .sync.aligned: the whole warp, converged
                    tmem_ld32(tb + (uint32_t)c, r0);
                    tmem_ld32(tb + (uint32_t)(c + 32), r1);
                    tmem_wait(r0);
                    tmem_after_wait(r1);
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int cb = col0 + c + 32 * h;
                        if (rows <= 0 || cb >= gt.bn) continue;  // uniform across the warp
                        const bool cok = cb + lane < gt.bn;
                        // transpose through shared memory: each store writes 32 consecutive keys of one pair
                        if (a.col_fac) {  // scaled operands: the column factors of the 32 columns by shuffles
                            const float2 f = cok ? a.col_fac[gt.b0 + cb + lane] : make_float2(0.f, 0.f);
#pragma unroll
                            for (int u = 0; u < 32; ++u)
                                tw[lane * 33 + u] = fmaf(__shfl_sync(0xffffffffu, f.x, u),
                                                         grf * acc_value<KIND>(h ? r1[u] : r0[u]),
                                                         __shfl_sync(0xffffffffu, f.y, u));
                        } else {
#pragma unroll
                            for (int u = 0; u < 32; ++u) tw[lane * 33 + u] = acc_value<KIND>(h ? r1[u] : r0[u]);
                        }
                        __syncwarp();
                        for (int r = 0; r < rows; ++r) {
                            const int64_t dr = __shfl_sync(0xffffffffu, dst_lane, r);
                            if (cok) a.out[dr + cb + lane] = tw[r * 33 + lane];
                        }
                        __syncwarp();
                    }
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                bar_arrive(&tempty[b]);
                continue;
            }
            const float tau_up = nextafterf(tau, kInf);
            const float2 ntau2 = make_float2(-tau_up, -tau_up);
            const uint32_t tbase = tmem + ((uint32_t)lane_base << 16) + (uint32_t)(b * kBN + col0);
            if (staged) {
                asm volatile("cp.async.wait_all;" ::: "memory");
                __syncwarp();
            }
            const bool has_an = a.normA != nullptr;  // uniform
            const bool rowbuf = a.row_cap > 0 && (kFilterOnly || a.out == nullptr);
            // filter keys of the 32 columns from col0 + c + 32 h (raw accumulators r): the row norm, the
            // scale factors, NaN past the tile's valid columns
            auto half_keys = [&](const uint32_t (&r)[32], int h, int c, float (&v)[32]) {
#pragma unroll
                for (int u = 0; u < 32; ++u) v[u] = acc_value<KIND>(r[u]) + (has_an ? an : 0.f);
                if (staged) {
                    const float2 r2 = make_float2(rfac, rfac);
#pragma unroll
                    for (int u = 0; u < 32; u += 4) {
                        const float4 fx = *reinterpret_cast<const float4*>(sfx + c + 32 * h + u);
                        const float4 fy = *reinterpret_cast<const float4*>(sfy + c + 32 * h + u);
                        const float2 t0 = __fmul2_rn(r2, make_float2(v[u], v[u + 1]));
                        const float2 t1 = __fmul2_rn(r2, make_float2(v[u + 2], v[u + 3]));
                        const float2 k0 = __ffma2_rn(make_float2(fx.x, fx.y), t0, make_float2(fy.x, fy.y));
                        const float2 k1 = __ffma2_rn(make_float2(fx.z, fx.w), t1, make_float2(fy.z, fy.w));
                        v[u] = k0.x;
                        v[u + 1] = k0.y;
                        v[u + 2] = k1.x;
                        v[u + 3] = k1.y;
                    }
                }
                const int lb = col0 + c + 32 * h;
                if (lb + 32 > ncols) {
#pragma unroll
                    for (int u = 0; u < 32; ++u)
                        if (lb + u >= ncols) v[u] = __int_as_float(0x7fffffff);
                }
            };
            // bit u set when v[u] passes the bar: v[u] <= tau exactly when v[u] - tau_up < 0 (tau_up the next
            // float above tau: a difference of two distinct floats is never +0, equal ones give +0, a NaN key
            // gives the positive default NaN), so the sign bits of packed differences, shifted in by funnel
            // shifts in four independent 8-key chains, form the mask
            auto half_mask = [&](const float (&v)[32]) -> uint32_t {
                uint32_t mq[4] = {0u, 0u, 0u, 0u};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
#pragma unroll
                    for (int u = 7; u >= 1; u -= 2) {
                        const float2 d = __fadd2_rn(make_float2(v[8 * j + u - 1], v[8 * j + u]), ntau2);
                        mq[j] = __funnelshift_l(__float_as_uint(d.y), mq[j], 1);
                        mq[j] = __funnelshift_l(__float_as_uint(d.x), mq[j], 1);
                    }
                }
                return (mq[0] | (mq[1] << 8)) | ((mq[2] << 16) | (mq[3] << 24));
            };
            // the survivors (mask mm) of keys v, columns col + u, into the row's buffer from slot sl
            auto put_row = [&](const float (&v)[32], uint32_t mm, int sl, int64_t rbase, int64_t col) {
                while (mm) {
                    const int u = __ffs(mm) - 1;
                    mm &= mm - 1;
                    if (sl < a.row_cap) {
                        // v[u] for a run-time u: a five-level select tree on u's bits
                        float s16[16], s8[8], s4[4], s2[2];
#pragma unroll
                        for (int z = 0; z < 16; ++z) s16[z] = (u & 16) ? v[z + 16] : v[z];
#pragma unroll
                        for (int z = 0; z < 8; ++z) s8[z] = (u & 8) ? s16[z + 8] : s16[z];
#pragma unroll
                        for (int z = 0; z < 4; ++z) s4[z] = (u & 4) ? s8[z + 4] : s8[z];
#pragma unroll
                        for (int z = 0; z < 2; ++z) s2[z] = (u & 2) ? s4[z + 2] : s4[z];
                        a.fkey[rbase + sl] = (u & 1) ? s2[1] : s2[0];
                        a.fcol[rbase + sl] = (int)(col + u);
                    }
                    ++sl;
                }
            };
#pragma unroll 1
            for (int c = 0; c < kCols; c += 64) {
                // per-row buffers: the survivors of the 64 columns under one atomic, so that the lane waits
                // for one round trip per 64 columns; one 32-column half in registers at a time (the first
                // half's keys are loaded and made again for their stores)
                if (rowbuf) {
                    uint32_t r[32];
                    float v[32];
                    __syncwarp();  // .sync.aligned loads after the divergent survivor stores of the last step
                    tmem_ld32(tbase + (uint32_t)c, r);
                    tmem_wait(r);
                    half_keys(r, 0, c, v);
                    const uint32_t ma = half_mask(v);
                    tmem_ld32(tbase + (uint32_t)(c + 32), r);
                    tmem_wait(r);
                    half_keys(r, 1, c, v);
                    const uint32_t mb = half_mask(v);
                    const int na = __popc(ma);
                    const int slot = (ma | mb) ? atomicAdd(&a.rcount[rq], na + __popc(mb)) : 0;
                    const int64_t rbase = (int64_t)rq * a.row_cap;
                    put_row(v, mb, slot + na, rbase, cbase + col0 + c + 32);
                    if (__any_sync(0xffffffffu, ma != 0u)) {  // uniform: the warp reloads the first half
                        __syncwarp();  // converged for the .sync.aligned load after the divergent stores
                        tmem_ld32(tbase + (uint32_t)c, r);
                        tmem_wait(r);
                        half_keys(r, 0, c, v);
                        put_row(v, ma, slot, rbase, cbase + col0 + c);
                    }
                    continue;
                }
                uint32_t r0[32], r1[32];
                __syncwarp();  // .sync.aligned loads after the divergent survivor stores of the last chunk
                tmem_ld32(tbase + (uint32_t)c, r0);
                tmem_ld32(tbase + (uint32_t)(c + 32), r1);
                tmem_wait(r0);
                tmem_after_wait(r1);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    float v[32];
                    if (has_an) {
#pragma unroll
                        for (int u = 0; u < 32; ++u) v[u] = acc_value<KIND>(h ? r1[u] : r0[u]) + an;
                    } else {
#pragma unroll
                        for (int u = 0; u < 32; ++u) v[u] = acc_value<KIND>(h ? r1[u] : r0[u]);
                    }
                    const int nb = n0 + col0 + c + 32 * h;  // output column of v[0]
                    const int lb = col0 + c + 32 * h;       // its column within the tile
                    if (staged) {  // scaled operands: key = f.y + f.x * (row scale * accumulator), two at a time
                        const float2 r2 = make_float2(rfac, rfac);
#pragma unroll
                        for (int u = 0; u < 32; u += 4) {
                            const float4 fx = *reinterpret_cast<const float4*>(sfx + c + 32 * h + u);
                            const float4 fy = *reinterpret_cast<const float4*>(sfy + c + 32 * h + u);
                            const float2 t0 = __fmul2_rn(r2, make_float2(v[u], v[u + 1]));
                            const float2 t1 = __fmul2_rn(r2, make_float2(v[u + 2], v[u + 3]));
                            const float2 k0 = __ffma2_rn(make_float2(fx.x, fx.y), t0, make_float2(fy.x, fy.y));
                            const float2 k1 = __ffma2_rn(make_float2(fx.z, fx.w), t1, make_float2(fy.z, fy.w));
                            v[u] = k0.x;
                            v[u + 1] = k0.y;
                            v[u + 2] = k1.x;
                            v[u + 3] = k1.y;
                        }
                    } else if (!kFilterOnly && a.col_fac) {
                        const int col = nb + lane;  // output column -> base row (strided sample of 256-row tiles)
                        const int64_t nrow = (int64_t)(col / kBN) * kBN * a.b_tile_stride + col % kBN;
                        const float2 f = col < a.N ? a.col_fac[nrow] : make_float2(0.f, 0.f);
#pragma unroll
                        for (int u = 0; u < 32; ++u)
                            v[u] = fmaf(__shfl_sync(0xffffffffu, f.x, u), rfac * v[u], __shfl_sync(0xffffffffu, f.y, u));
                    }
                    if (lb + 32 > ncols) {  // ragged last tile: columns past it pass no bar (NaN) and are not stored
#pragma unroll
                        for (int u = 0; u < 32; ++u)
                            if (lb + u >= ncols) v[u] = __int_as_float(0x7fffffff);
                    }
                    if (!kFilterOnly && a.out) {
                        if (a.out_cmin && m < a.M && nb < a.N) {  // the chunk's minimum (NaN columns past N ignored)
                            float mn = v[0];
#pragma unroll
                            for (int u = 1; u < 32; ++u) mn = fminf(mn, v[u]);
                            a.out_cmin[(int64_t)m * ((a.N + 31) / 32) + nb / 32] = mn;
                        }
                        // transpose through shared memory so each store covers 32 consecutive columns
#pragma unroll
                        for (int u = 0; u < 32; ++u) tw[lane * 33 + u] = v[u];
                        __syncwarp();
                        for (int r = 0; r < 32; ++r) {
                            const int mr = m0 + lane_base + r;
                            if (mr < a.M && nb + lane < a.N) a.out[(int64_t)mr * a.ldo + nb + lane] = tw[r * 33 + lane];
                        }
                        __syncwarp();
                    } else {
                        uint32_t msk = half_mask(v);
                        if (__any_sync(0xffffffffu, msk != 0)) {
                            const int cnt = __popc(msk);
                            int incl = cnt;
#pragma unroll
                            for (int o = 1; o < 32; o <<= 1) {
                                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                                if (lane >= o) incl += y;
                            }
                            int slot = wcount + incl - cnt;
                            wcount += __shfl_sync(0xffffffffu, incl, 31);
                            while (msk) {
                                const int u = __ffs(msk) - 1;
                                msk &= msk - 1;
                                if (slot < a.wcap) {
                                    // v[u] for a run-time u: a five-level select tree on u's bits
                                    float s16[16], s8[8], s4[4], s2[2];
#pragma unroll
                                    for (int z = 0; z < 16; ++z) s16[z] = (u & 16) ? v[z + 16] : v[z];
#pragma unroll
                                    for (int z = 0; z < 8; ++z) s8[z] = (u & 8) ? s16[z + 8] : s16[z];
#pragma unroll
                                    for (int z = 0; z < 4; ++z) s4[z] = (u & 4) ? s8[z + 4] : s8[z];
#pragma unroll
                                    for (int z = 0; z < 2; ++z) s2[z] = (u & 2) ? s4[z + 2] : s4[z];
                                    const float kv = (u & 1) ? s2[1] : s2[0];
                                    a.fkey[wbase + slot] = kv;
                                    a.fcol[wbase + slot] = (int)(cbase + lb + u);
                                    a.frow[wbase + slot] = rq;
                                }
                                ++slot;
                            }
                        }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            bar_arrive(&tempty[b]);
        }
        if (a.wcount && lane == 0) a.wcount[(int64_t)blockIdx.x * EPI + ew] = wcount;
    }
    __syncthreads();
    if (warp == 1) {
        __syncwarp();  // lane 0 issued the MMAs alone: the warp meets again before the .sync.aligned dealloc
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

int make_map(CUtensorMap* tm, const void* base, int64_t rows, int cols, int box_rows, int kind) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("cuTensorMapEncodeTiled is not available from the driver");
        return ANN_ERR_CUDA;
    }
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const int esize = kind == kTcBF16 ? 2 : 1;
    const cuuint64_t strides[1] = {(cuuint64_t)cols * esize};
    const cuuint32_t box[2] = {(cuuint32_t)(kRowBytes / esize), (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(tm, kind == kTcBF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8, 2,
                          const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d) for a [%lld, %d] matrix", (int)r, (long long)rows, cols);
        return ANN_ERR_CUDA;
    }
    return ANN_OK;
}

}  // namespace

size_t tc_gemm_smem() { return std::max(epi_smem(kKeyEpi), epi_smem(kFilterEpi)); }

int tc_kpad(int dim, int metric) { return (int)ceil_div(dim + (metric == ANN_METRIC_L2 ? 3 : 0), 16) * 16; }

static int tc_grid(int M, int N) { return (int)std::min<int64_t>(ceil_div(M, kBM) * ceil_div(N, kBN), kNumSMs); }
int tc_filter_warps(int M, int N) { return tc_grid(M, N) * kFilterEpi; }
int tc_grouped_filter_warps() { return kNumSMs * kFilterEpi; }

template <int KIND, int EPI>
static cudaError_t run_tc_gemm(const CUtensorMap& tmA, const CUtensorMap& tmB, const TcGemmArgs& a, int grid,
                               cudaStream_t st) {
    const cudaError_t e = smem_optin(reinterpret_cast<const void*>(tc_gemm_kernel<KIND, EPI>));
    if (e != cudaSuccess) return e;
    tc_gemm_kernel<KIND, EPI><<<grid, epi_threads(EPI), epi_smem(EPI), st>>>(tmA, tmB, a);
    return cudaSuccess;
}

int launch_tc_gemm(const void* A, const void* B, const TcGemmArgs& a, cudaStream_t st) {
    const int step = a.kind == kTcBF16 ? 16 : 32;
    ANN_CHECK_ARG(a.kind == kTcBF16 || a.kind == kTcE4M3 || a.kind == kTcI8, "tensor-core scan: element kind %d",
                  a.kind);
    ANN_CHECK_ARG(a.K % step == 0 && a.K > 0, "tensor-core scan: K=%d not a positive multiple of %d", a.K, step);
    ANN_CHECK_ARG(a.kind == kTcBF16 || (a.col_fac && a.row_fac && (a.g_item_off == nullptr || a.kind == kTcI8)),
                  "tensor-core scan: E4M3 / I8 operands need their scale factors (E4M3: no grouping)");
    ANN_CHECK_ARG((reinterpret_cast<uintptr_t>(A) & 15) == 0 && (reinterpret_cast<uintptr_t>(B) & 15) == 0,
                  "tensor-core scan: operands must be 16-byte aligned");
    ANN_CHECK_ARG(a.out != nullptr || (a.tau && a.fkey && a.fcol &&
                                       ((a.frow && a.wcount && a.wcap > 0) || (a.row_cap > 0 && a.rcount))),
                  "tensor-core scan: neither an output matrix nor a filter");
    ANN_CHECK_ARG(a.g_item_off == nullptr ||
                      (a.g_a_off && a.g_b_off && a.g_total && a.g_lists > 0 &&
                       ((a.out && a.g_dbase && a.tau == nullptr) || (a.out == nullptr && a.tau && a.g_row_query))),
                  "tensor-core scan: incomplete grouping");
    ANN_CHECK_ARG(a.b_tile_stride >= 1, "tensor-core scan: bad sample stride");
    ANN_CHECK_ARG(a.out_cmin == nullptr || (a.out && a.g_item_off == nullptr && a.b_tile_stride == 1),
                  "tensor-core scan: chunk minima need the dense key-matrix mode");
    if (a.M == 0 || a.N == 0) return ANN_OK;
    const int64_t b_rows = a.b_rows > 0 ? a.b_rows : a.N;
    // the last sampled tile must start inside B
    ANN_CHECK_ARG(a.g_item_off != nullptr || (ceil_div(a.N, kBN) - 1) * kBN * (int64_t)a.b_tile_stride < b_rows,
                  "tensor-core scan: sample runs past the base");
    CUtensorMap tmA, tmB;
    int rc = make_map(&tmA, A, a.M, a.K, kBM, a.kind);
    if (rc) return rc;
    rc = make_map(&tmB, B, b_rows, a.K, kBN, a.kind);
    if (rc) return rc;
    const int grid = a.g_item_off ? kNumSMs : tc_grid(a.M, a.N);  // grouped: persistent over the items
    const bool filter = a.out == nullptr;
    cudaError_t e;
    if (a.kind == kTcBF16)
        e = filter ? run_tc_gemm<kTcBF16, kFilterEpi>(tmA, tmB, a, grid, st)
                   : run_tc_gemm<kTcBF16, kKeyEpi>(tmA, tmB, a, grid, st);
    else if (a.kind == kTcE4M3)
        e = filter ? run_tc_gemm<kTcE4M3, kFilterEpi>(tmA, tmB, a, grid, st)
                   : run_tc_gemm<kTcE4M3, kKeyEpi>(tmA, tmB, a, grid, st);
    else
        e = filter ? run_tc_gemm<kTcI8, kFilterEpi>(tmA, tmB, a, grid, st)
                   : run_tc_gemm<kTcI8, kKeyEpi>(tmA, tmB, a, grid, st);
    ANN_CUDA_TRY(e);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

namespace {
// desc[t] for the items of list l = blockIdx.x (strided): the tile group_tile would derive for item t.
__global__ void tc_item_descs_kernel(const int64_t* __restrict__ item_off, int C, const int64_t* __restrict__ a_off,
                                     const int64_t* __restrict__ b_off, const int64_t* __restrict__ b_len,
                                     int4* __restrict__ desc, int64_t cap) {
    for (int l = blockIdx.x; l < C; l += gridDim.x) {
        const int64_t np = a_off[l + 1] - a_off[l];
        const int64_t nr = b_len ? b_len[l] : b_off[l + 1] - b_off[l];
        const int64_t npt = (np + kBM - 1) / kBM;
        for (int64_t t = item_off[l] + threadIdx.x; t < item_off[l + 1] && t < cap; t += blockDim.x) {
            const int64_t local = t - item_off[l];
            const int64_t g = local % npt, rt = local / npt;
            desc[t] = make_int4((int)(a_off[l] + g * kBM), (int)(b_off[l] + rt * kBN),
                                (int)min((int64_t)kBM, np - g * kBM), (int)min((int64_t)kBN, nr - rt * kBN));
        }
    }
}
}  // namespace

int launch_tc_item_descs(const int64_t* item_off, int C, const int64_t* a_off, const int64_t* b_off,
                         const int64_t* b_len, int4* desc, int64_t cap, cudaStream_t st) {
    ANN_CHECK_ARG(C >= 1, "tensor-core grouping: no lists");
    tc_item_descs_kernel<<<(unsigned)std::min(C, 4 * kNumSMs), 128, 0, st>>>(item_off, C, a_off, b_off, b_len, desc,
                                                                             cap);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int tc_wait_selftest(uint64_t wait_ns, int* flag_out) {
    // A [128, 64] and B [256, 64] BF16 (zeros), keys [128, 256], the flag
    const size_t a_bytes = (size_t)kBM * 64 * 2, b_bytes = (size_t)kBN * 64 * 2, o_bytes = (size_t)kBM * kBN * 4;
    char* buf = nullptr;
    ANN_CUDA_TRY(cudaMalloc(&buf, a_bytes + b_bytes + o_bytes + 256));
    int rc = ANN_OK;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemsetAsync(buf, 0, a_bytes + b_bytes + o_bytes + 256, st);
    if (e == cudaSuccess) {
        int* flag = reinterpret_cast<int*>(buf + a_bytes + b_bytes + o_bytes);
        TcGemmArgs a{kBM, kBN, 64, nullptr, reinterpret_cast<float*>(buf + a_bytes + b_bytes), kBN, flag};
        a.wait_ns = wait_ns;
        a.test_no_loads = 1;
        rc = launch_tc_gemm(buf, buf + a_bytes, a, st);
        if (rc == ANN_OK) e = cudaMemcpyAsync(flag_out, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (rc == ANN_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (st) cudaStreamDestroy(st);
    cudaFree(buf);
    if (rc) return rc;
    ANN_CUDA_TRY(e);
    return ANN_OK;
}

// One warp per output row: the BF16 operand form (tc_gemm.cuh) of an FP32 row. The squared norm is the
// FP32 sum of the row's FP32 squares; its three BF16 pieces are hi = bf16(s), mid = bf16(s - hi) and
// lo = bf16(s - hi - mid), each difference exact in FP32.
__global__ void tc_operand_kernel(const float* __restrict__ x, int64_t rows, int cols, int64_t ld, __nv_bfloat16* out,
                                  int kpad, float scale, int base_l2, int query_l2, int64_t row_mult) {
    const int64_t p = blockIdx.x * (int64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (p >= rows) return;
    const int64_t r = row_mult > 0 ? (int64_t)(((unsigned __int128)p * (uint64_t)row_mult) % (uint64_t)rows) : p;
    float s = 0.f;
    for (int c = lane; c < kpad; c += 32) {
        const float v = c < cols ? x[r * ld + c] : 0.f;
        s = fmaf(v, v, s);
        float o = v * scale;
        if (query_l2 && c >= cols && c < cols + 3) o = 1.f;
        out[p * kpad + c] = __float2bfloat16_rn(o);
    }
    if (!base_l2) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        const __nv_bfloat16 hi = __float2bfloat16_rn(s);
        const float r1 = s - __bfloat162float(hi);
        const __nv_bfloat16 mid = __float2bfloat16_rn(r1);
        const float r2 = r1 - __bfloat162float(mid);
        out[p * kpad + cols] = hi;
        out[p * kpad + cols + 1] = mid;
        out[p * kpad + cols + 2] = __float2bfloat16_rn(r2);
    }
}

// One warp per output row: the E4M3 operand form of an FP32 row with its own scale s = max|x| / 448
// (1 for a zero row): out = e4m3(x / s), saturating; fac = s for a query row; for a base row
// fac = (-2 s, |x|^2) under L2 and (-s, 0) under inner product, the key's per-column factors.
__global__ void tc_operand_e4m3_kernel(const float* __restrict__ x, int64_t rows, int cols, int64_t ld, uint8_t* out,
                                       int kpad, int base, int l2, int64_t row_mult, float* qfac, float2* bfac) {
    const int64_t p = blockIdx.x * (int64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (p >= rows) return;
    const int64_t r = row_mult > 0 ? (int64_t)(((unsigned __int128)p * (uint64_t)row_mult) % (uint64_t)rows) : p;
    float mx = 0.f, ss = 0.f;
    for (int c = lane; c < cols; c += 32) {
        const float v = x[r * ld + c];
        mx = fmaxf(mx, fabsf(v));
        ss = fmaf(v, v, ss);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        ss += __shfl_xor_sync(0xffffffffu, ss, o);
    }
    const float sc = mx > 0.f ? mx / 448.f : 1.f;
    const float inv = 1.f / sc;
    for (int c = lane; c < kpad; c += 32) {
        const float v = c < cols ? x[r * ld + c] * inv : 0.f;
        out[p * kpad + c] = (uint8_t)__nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
    }
    if (lane == 0) {
        if (base)
            bfac[p] = l2 ? make_float2(-2.f * sc, ss) : make_float2(-sc, 0.f);
        else
            qfac[p] = sc;
    }
}

int launch_tc_operand_e4m3(const float* x, int64_t rows, int cols, int64_t ld, uint8_t* out, int kpad, int role,
                           int metric, int64_t row_mult, float* qfac, float2* bfac, cudaStream_t st) {
    ANN_CHECK_ARG(kpad >= cols && kpad % 32 == 0, "E4M3 operand: kpad %d", kpad);
    ANN_CHECK_ARG(role == kTcBase ? bfac != nullptr : (qfac != nullptr && row_mult == 0), "E4M3 operand: factors");
    if (rows == 0) return ANN_OK;
    tc_operand_e4m3_kernel<<<(unsigned)ceil_div(rows, 8), 256, 0, st>>>(x, rows, cols, ld, out, kpad,
                                                                         role == kTcBase ? 1 : 0,
                                                                         metric == ANN_METRIC_L2 ? 1 : 0, row_mult,
                                                                         qfac, bfac);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_tc_operand(const float* x, int64_t rows, int cols, int64_t ld, __nv_bfloat16* out, int kpad, int role,
                      int metric, int64_t row_mult, cudaStream_t st) {
    ANN_CHECK_ARG(kpad >= tc_kpad(cols, metric) && kpad % 16 == 0, "tensor-core operand: kpad %d too small", kpad);
    ANN_CHECK_ARG(row_mult == 0 || role == kTcBase, "tensor-core operand: only the base is reordered");
    if (rows == 0) return ANN_OK;
    const bool l2 = metric == ANN_METRIC_L2;
    const float scale = role == kTcBase ? 1.f : (l2 ? -2.f : -1.f);
    tc_operand_kernel<<<(unsigned)ceil_div(rows, 8), 256, 0, st>>>(x, rows, cols, ld, out, kpad, scale,
                                                                    (l2 && role == kTcBase) ? 1 : 0,
                                                                    (l2 && role == kTcQuery) ? 1 : 0, row_mult);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

// Launch interface of the tcgen05 BF16 distance GEMM (tc_gemm.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace annb {

// The GEMM output is the ranking key itself: the operands carry it (launch_tc_operand).
//   L2: base row [bf16(b), hi, mid, lo] with hi + mid + lo = |b|^2 (FP32, split into three BF16),
//       query row [bf16(-2a), 1, 1, 1]  ->  sum = |b|^2 - 2 a.b
//   IP: base row [bf16(b)], query row [bf16(-a)]  ->  sum = -a.b
// Smaller keys are better in both metrics.
// kTcI8: A int8, B uint8 (tcgen05.mma.kind::i8, exact int32 accumulation): the SQ8 codes of an IVF index as
// they are stored, against an int8 query weight; the key is col_fac[n].y + col_fac[n].x * row_fac[m] * acc.
enum TcKind { kTcBF16 = 0, kTcE4M3 = 1, kTcI8 = 2 };

struct TcGemmArgs {
    int M, N, K;           // A [M, K], B [N, K] BF16 row-major; K a multiple of 16
    const float* normA;    // [M] optional per-row addend (|a|^2 turns the L2 key into the squared distance)
    float* out;            // [M, ldo] keys; null in filter mode
    int64_t ldo;
    int* err;              // device flag set (to 2) if a bounded wait gives up
    int b_tile_stride = 1; // B rows of output tile j start at row j * 256 * b_tile_stride (a strided sample)
    int64_t b_rows = 0;    // rows of the B matrix when sampling (0: N)
    // Filter mode (out == null): keys <= tau[m] are appended, as (key, column, row m), to the region of
    // the epilogue warp that met them: warp w of the grid owns entries [w * wcap, (w + 1) * wcap) of
    // fkey / fcol / frow, and wcount[w] receives its count (which may exceed wcap: the caller checks).
    const float* tau = nullptr;
    float* fkey = nullptr;
    int* fcol = nullptr;
    int* frow = nullptr;
    int* wcount = nullptr;
    int wcap = 0;
    // Grouped mode (g_item_off != null): work item t of a list-major grouping (an IVF batch). List l owns
    // the A rows [g_row_off[l], + g_row_len[l] or up to g_row_off[l+1]) -- its list-ordered base rows, the
    // M side -- and the B rows [g_pair_off[l], g_pair_off[l+1]) -- its (query, list) pairs, the N side; its
    // items are ceil(pairs / 256) x ceil(rows / 128) tiles, pair tiles fastest, numbered from
    // g_item_off[l]; *g_total items in all (read on the device); the MMA runs N = the tile's pairs
    // rounded up to 16. Keys (out != null): the key of pair i and list row r goes to out[g_dbase[i] + r].
    // Filter (out == null): pair i belongs to query g_row_query[i]; a key at or below tau[that query] goes
    // to fkey / fcol [query * row_cap + slot] (fcol = the list row) at slot = atomicAdd(&rcount[query], ..)
    // -- one atomic per warp and column -- and nothing is written at slots past row_cap (rcount may exceed
    // it: the caller checks). With scaled operands, col_fac is per list row and row_fac per pair.
    const int64_t* g_item_off = nullptr;
    const int64_t* g_pair_off = nullptr;
    const int64_t* g_row_off = nullptr;
    const int64_t* g_row_len = nullptr;
    const int64_t* g_dbase = nullptr;
    const int64_t* g_total = nullptr;
    int g_lists = 0;
    const int32_t* g_item_list = nullptr;  // optional: the list of each item (else a search of g_item_off)
    const int32_t* g_row_query = nullptr;
    int row_cap = 0;
    int* rcount = nullptr;
    // Element kind of A and B. E4M3 and I8 operands carry factors per row: the key is
    // col_fac[n].y + col_fac[n].x * row_fac[m] * accumulator for the dense key-matrix and filter modes (n the
    // B row, m the A row); in the grouped mode (I8) col_fac is per list row and row_fac per pair.
    int kind = kTcBF16;
    const float2* col_fac = nullptr;
    const float* row_fac = nullptr;
    // Bounded waits: every mbarrier wait gives up after wait_ns (0: 2 s), sets *err = 2 and the CTA
    // winds down (remaining copies and MMAs drained, TMEM released). test_no_loads (self-test only):
    // the producer issues no copies, so the waits run out with nothing in flight.
    uint64_t wait_ns = 0;
    int test_no_loads = 0;
};

enum TcRole { kTcBase = 0, kTcQuery = 1 };

// Columns of the BF16 operands for vectors of `dim` FP32 values: the key columns included, rounded up
// to the 16-column MMA step (the 64-column TMA boxes of the last k-block read zeros past it).
int tc_kpad(int dim, int metric);
// Epilogue warps of a filter launch over M x N keys (the size of the wcount array).
int tc_filter_warps(int M, int N);
// ... and of a grouped filter launch (persistent over the work items).
int tc_grouped_filter_warps();
size_t tc_gemm_smem();
int launch_tc_gemm(const void* A, const void* B, const TcGemmArgs& a, cudaStream_t st);
// Runs one small GEMM whose producer issues no copies, with every wait limited to wait_ns, and returns the
// device flag it left (2: a bounded wait gave up, as it must); the flag is cleared afterwards.
int tc_wait_selftest(uint64_t wait_ns, int* flag_out);
// FP32 rows -> E4M3 [rows, kpad] (kpad >= cols, a multiple of 32) with a per-row scale: a query row's
// scale into qfac[row]; a base row's key factors into bfac[row] (row_mult as for launch_tc_operand).
int launch_tc_operand_e4m3(const float* x, int64_t rows, int cols, int64_t ld, uint8_t* out, int kpad, int role,
                           int metric, int64_t row_mult, float* qfac, float2* bfac, cudaStream_t st);
// FP32 [rows, ld] (first `cols` columns) -> the BF16 operand form of `role` for `metric`, [rows, kpad].
// With row_mult > 0 (base only), output row p holds input row (p * row_mult) mod rows.
int launch_tc_operand(const float* x, int64_t rows, int cols, int64_t ld, __nv_bfloat16* out, int kpad, int role,
                      int metric, int64_t row_mult, cudaStream_t st);

}  // namespace annb

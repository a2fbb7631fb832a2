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
    // Filter mode, per-row buffers (row_cap > 0; the grouped form, rows = queries): a survivor of row r goes
    // to fkey / fcol [r * row_cap + slot] at slot = atomicAdd(&rcount[r], n) -- one atomic per lane per 32
    // columns, n its survivors there -- and nothing is written at slots past row_cap (rcount[r] may exceed
    // it: the caller checks).
    int row_cap = 0;
    int* rcount = nullptr;
    // Grouped mode (g_item_off != null; out receives the keys): tile t is work item t of a list-major
    // grouping (an IVF batch). List l owns A rows [g_a_off[l], g_a_off[l+1]) (its (query, list) pairs)
    // and B rows [g_b_off[l], g_b_off[l+1]) (its rows); its items are ceil(pairs/128) x ceil(rows/256)
    // tiles, pair tiles fastest, numbered from g_item_off[l]; *g_total items in all (read on the
    // device). The key of pair i and list row r goes to out[g_dbase[i] + r].
    const int64_t* g_item_off = nullptr;
    const int64_t* g_a_off = nullptr;
    const int64_t* g_b_off = nullptr;
    const int64_t* g_dbase = nullptr;
    const int64_t* g_total = nullptr;
    int g_lists = 0;
    const int32_t* g_item_list = nullptr;  // optional: the list of each item (else a search of g_item_off)
    // optional, in place of the two above: item t's tile as (first A row, first B row, A rows, B rows), one
    // 16-byte load (launch_tc_item_descs); the roles read the next item's ahead of its use
    const int4* g_item_desc = nullptr;
    const int64_t* g_b_len = nullptr;      // optional: rows of list l taken (else g_b_off[l+1] - g_b_off[l])
    // Grouped filter mode (grouped, out == null): A row i belongs to query g_row_query[i]; its bar is
    // tau[g_row_query[i]], and a survivor is recorded as (key, list row g_b_off[l] + r, that query).
    const int32_t* g_row_query = nullptr;
    // Element kind of A and B. E4M3 and I8 operands carry factors per row: the key is
    // col_fac[n].y + col_fac[n].x * row_fac[m] * accumulator (key-matrix and filter modes; I8 also grouped,
    // with n the absolute B row and m the A row).
    int kind = kTcBF16;
    const float2* col_fac = nullptr;  // per B row, indexed like B's rows
    const float* row_fac = nullptr;   // per A row
    // Bounded waits: every mbarrier wait gives up after wait_ns (0: 2 s), sets *err = 2 and the CTA
    // winds down (remaining copies and MMAs drained, TMEM released). test_no_loads (self-test only):
    // the producer issues no copies, so the waits run out with nothing in flight.
    uint64_t wait_ns = 0;
    int test_no_loads = 0;
    // Key-matrix mode (dense, out given): if out_cmin is given, it also receives the minimum key of each row's
    // 32-column chunks, out_cmin[m * ceil(N / 32) + n / 32], so that a reader can skip chunks.
    float* out_cmin = nullptr;
    // If given and *skip_if_zero == 0 (read on the device), the launch does nothing: a pass whose need is
    // known only on the device, without a host round trip.
    const int* skip_if_zero = nullptr;
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
// The grouped mode's item descriptors (TcGemmArgs::g_item_desc) for items [0, min(item_off[C], cap)): list l's
// items from item_off[l] (launch_tc_ivf_items), its A rows [a_off[l], a_off[l+1]) and B rows from b_off[l]
// (b_len[l] of them when given, else to b_off[l+1]).
int launch_tc_item_descs(const int64_t* item_off, int C, const int64_t* a_off, const int64_t* b_off,
                         const int64_t* b_len, int4* desc, int64_t cap, cudaStream_t st);
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

// IVF-SQ8 index build on the GPU: the B200 form of IVFLSHIndex::fit
// (competitors/ivf_lsh/src/lsh_index_optimized.cpp:128-214, 551-616) for n_tables = 1, n_bits = 0.
//
// * k-means, the reference's run_kmeans (:551-616) reproduced bit for bit for a given ThreadPool
//   size T (the reference sizes its pool from hardware_concurrency(), :140):
//   - assignment (:32-47): each row goes to the first centroid with the smallest
//     compute_l2_distance. The exact FP32 scan (flat_scan.cu) finds each row's two nearest
//     centroids; when the second is farther than the first by more than the two arithmetics'
//     combined rounding bound, the first is also the reference's choice (kmeans_certify_kernel).
//     The remaining rows -- near-ties -- are recomputed against every centroid with the
//     reference's own arithmetic (refmath.cuh), first minimum kept (kmeans_ref_assign_kernel).
//   - update (:60-73, :594-613): per list, each ThreadPool chunk's rows summed in row order from
//     0.0f, the chunk sums added in chunk order from 0.0f, then multiplied by the float reciprocal
//     of the count (the compiled reference's form of the division); an empty list takes row
//     rand_indices[(c * 37) % n] (kmeans_update_kernel).
// * reorder: rows grouped list by list, ascending original id inside a list (:155-173).
// * per-dimension SQ8 (:187-214), bit-identical to the reference: exact min/max, scale =
//   (max - min) * (1/255) -- the compiled reference multiplies by the float reciprocal -- or 1
//   when the range is <= 1e-8, offset = min (or 0), code = clamp(round((x - offset) / scale)) with
//   a true division and round-half-away-from-zero.
#include "common.cuh"
#include "ivf.cuh"
#include "refmath.cuh"

namespace annb {

__device__ __forceinline__ unsigned ordered_bits(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ordered(unsigned o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

__global__ void minmax_init_kernel(unsigned* mn, unsigned* mx, int dim) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d < dim) {
        mn[d] = 0xffffffffu;
        mx[d] = 0u;
    }
}

// grid: (dim blocks of 128, row chunks)
__global__ void minmax_kernel(const float* __restrict__ x, int64_t n, int dim, int ld, unsigned* mn, unsigned* mx) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= dim) return;
    const int64_t chunk = ceil_div(n, gridDim.y);
    const int64_t r0 = (int64_t)blockIdx.y * chunk;
    const int64_t r1 = min(n, r0 + chunk);
    float lo = kInf, hi = -kInf;
    for (int64_t r = r0; r < r1; ++r) {
        const float v = x[r * ld + d];
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
    }
    if (r0 < r1) {
        atomicMin(&mn[d], ordered_bits(lo));
        atomicMax(&mx[d], ordered_bits(hi));
    }
}

__global__ void minmax_finish_kernel(unsigned* mn, unsigned* mx, int dim) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d < dim) {
        reinterpret_cast<float*>(mn)[d] = from_ordered(mn[d]);
        reinterpret_cast<float*>(mx)[d] = from_ordered(mx[d]);
    }
}

int launch_sq8_minmax(const float* x, int64_t n, int dim, int ld, float* mn, float* mx, cudaStream_t st) {
    unsigned* umn = reinterpret_cast<unsigned*>(mn);
    unsigned* umx = reinterpret_cast<unsigned*>(mx);
    const unsigned gd = (unsigned)ceil_div(dim, 128);
    minmax_init_kernel<<<gd, 128, 0, st>>>(umn, umx, dim);
    ANN_LAUNCH_CHECK();
    const unsigned chunks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(1024, ceil_div(n, 256)));
    minmax_kernel<<<dim3(gd, chunks), 128, 0, st>>>(x, n, dim, ld, umn, umx);
    ANN_LAUNCH_CHECK();
    minmax_finish_kernel<<<gd, 128, 0, st>>>(umn, umx, dim);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

__global__ void sq8_params_kernel(const float* mn, const float* mx, int dim, int dpad, float* scale, float* offset) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= dpad) return;
    if (d >= dim) {
        scale[d] = 0.f;
        offset[d] = 0.f;
        return;
    }
    const float range = __fsub_rn(mx[d], mn[d]);
    if (range > 1e-8f) {
        scale[d] = __fmul_rn(range, 1.0f / 255.0f);
        offset[d] = mn[d];
    } else {
        scale[d] = 1.0f;
        offset[d] = 0.0f;
    }
}

int launch_sq8_params(const float* mn, const float* mx, int dim, int dpad, float* scale, float* offset,
                      cudaStream_t st) {
    sq8_params_kernel<<<(unsigned)ceil_div(dpad, 128), 128, 0, st>>>(mn, mx, dim, dpad, scale, offset);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

__global__ void sq8_encode_kernel(const float* __restrict__ x, int64_t n, int dim, int ld,
                                  const float* __restrict__ scale, const float* __restrict__ offset,
                                  uint8_t* __restrict__ codes, int dpad8) {
    const int64_t total = n * dpad8;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / dpad8;
        const int d = (int)(e % dpad8);
        uint8_t c = 0;
        if (d < dim) {
            const float v = __fdiv_rn(__fsub_rn(x[r * ld + d], offset[d]), scale[d]);
            const int qv = (int)roundf(v);
            c = (uint8_t)(qv < 0 ? 0 : (qv > 255 ? 255 : qv));
        }
        codes[e] = c;
    }
}

int launch_sq8_encode(const float* x, int64_t n, int dim, int ld, const float* scale, const float* offset,
                      uint8_t* codes, int dpad8, cudaStream_t st) {
    if (n == 0) return ANN_OK;
    const int blocks = (int)std::min<int64_t>(ceil_div(n * dpad8, 256), kNumSMs * 32);
    sq8_encode_kernel<<<blocks, 256, 0, st>>>(x, n, dim, ld, scale, offset, codes, dpad8);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// dst row i = src row rows[i] (ld floats each; ld_src == ld_dst assumed by callers padding both)
__global__ void gather_rows_kernel(const float* __restrict__ src, int64_t n, int ld_src,
                                   const int32_t* __restrict__ rows, float* __restrict__ dst, int ld_dst) {
    const int64_t total = n * ld_dst;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / ld_dst;
        const int c = (int)(e % ld_dst);
        dst[e] = c < ld_src ? src[(int64_t)rows[i] * ld_src + c] : 0.f;
    }
}

int launch_gather_rows(const float* src, int64_t n, int ld_src, const int32_t* rows, float* dst, int ld_dst,
                       cudaStream_t st) {
    if (n == 0) return ANN_OK;
    const int blocks = (int)std::min<int64_t>(ceil_div(n * ld_dst, 256), kNumSMs * 32);
    gather_rows_kernel<<<blocks, 256, 0, st>>>(src, n, ld_src, rows, dst, ld_dst);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// off[c] = first position of list c in the sorted assignment (lower bound), off[C] = n.
__global__ void list_offsets_kernel(const int32_t* __restrict__ a, int64_t n, int C, int64_t* off) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > C) return;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] < c)
            lo = mid + 1;
        else
            hi = mid;
    }
    off[c] = lo;
}

__global__ void iota_kernel(int32_t* v, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = (int32_t)i;
}

__global__ void add_offset_kernel(int64_t* v, int64_t n, int64_t add) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] += add;
}

int launch_iota(int32_t* v, int64_t n, cudaStream_t st) {
    if (n == 0) return ANN_OK;
    iota_kernel<<<(unsigned)std::min<int64_t>(ceil_div(n, 256), 16 * kNumSMs), 256, 0, st>>>(v, n);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_add_offset(int64_t* v, int64_t n, int64_t add, cudaStream_t st) {
    if (n == 0) return ANN_OK;
    add_offset_kernel<<<(unsigned)std::min<int64_t>(ceil_div(n, 256), 16 * kNumSMs), 256, 0, st>>>(v, n, add);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_list_offsets(const int32_t* sorted_assign, int64_t n, int C, int64_t* off, cudaStream_t st) {
    list_offsets_kernel<<<(unsigned)ceil_div(C + 1, 128), 128, 0, st>>>(sorted_assign, n, C, off);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

// ---- k-means -----------------------------------------------------------------------------------

// Rows whose second-nearest centroid (fast FP32 scan) is farther than the nearest by a factor above
// `margin` take the nearest; the rest are queued for the reference arithmetic. margin bounds the
// ratio that the rounding of both arithmetics can hide (sums of non-negative squares: each value is
// within a relative (terms + a few) * 2^-24 of the true distance). Keys under 1e-30 (possible
// underflow) are always queued.
__global__ void kmeans_certify_kernel(const float* __restrict__ key2, const int* __restrict__ id2, int64_t n,
                                      float margin, int32_t* __restrict__ assign, int32_t* __restrict__ amb,
                                      int* __restrict__ amb_count) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float k0 = key2[2 * i], k1 = key2[2 * i + 1];
        const int c0 = id2[2 * i], c1 = id2[2 * i + 1];
        const bool single = c1 == INT_MAX && c0 != INT_MAX;  // one centroid only
        const bool clear = k1 > 1e-30f && k1 > k0 * margin && c0 != INT_MAX;
        if (single || clear)
            assign[i] = c0;
        else
            amb[atomicAdd(amb_count, 1)] = (int32_t)i;
    }
}

// One warp per queued row: its two 16-thread groups evaluate centroids c = g, g + 2, ... with the
// reference's compute_l2_distance (refmath.cuh); the smallest distance wins, the lower centroid on
// equal distances (the reference's strict `<` from FLT_MAX keeps the first minimum; a row whose
// distances are all >= FLT_MAX stays at centroid 0).
__global__ void __launch_bounds__(256) kmeans_ref_assign_kernel(const float* __restrict__ x, int ldx, int dim,
                                                                const float* __restrict__ cent, int ldc, int C,
                                                                const int32_t* __restrict__ amb,
                                                                const int* __restrict__ amb_count,
                                                                int32_t* __restrict__ assign) {
    const int wpb = blockDim.x >> 5;
    const int warp = blockIdx.x * wpb + (threadIdx.x >> 5);
    const int nwarps = gridDim.x * wpb;
    const int g = (threadIdx.x >> 4) & 1;
    const int cnt = *amb_count;
    for (int p = warp; p < cnt; p += nwarps) {
        const int64_t i = amb[p];
        const float* xr = x + i * ldx;
        float best = FLT_MAX;
        int bc = INT_MAX;
        for (int c0 = 0; c0 < C; c0 += 2) {
            const int c = c0 + g;
            const bool ok = c < C;
            const float d = ref_l2_f32(xr, cent + (int64_t)(ok ? c : c0) * ldc, dim, NoEmit{});
            if (ok && d < best) {
                best = d;
                bc = c;
            }
        }
        const float ob = __shfl_xor_sync(0xffffffffu, best, 16);
        const int oc = __shfl_xor_sync(0xffffffffu, bc, 16);
        if (ob < best || (ob == best && oc < bc)) {
            best = ob;
            bc = oc;
        }
        if ((threadIdx.x & 31) == 0) assign[i] = bc == INT_MAX ? 0 : bc;
    }
}

// One CTA per list, thread d on component d: the list's rows (order[off[c]..off[c+1]), ascending
// ids) are summed per ThreadPool chunk -- chunk t of `active` covers [t*q + min(t, r), ...) with
// q = n / active, r = n % active (src/thread_pool.h:93-124) -- and the chunk sums are added in
// chunk order; chunks without rows of the list add 0.0f, which changes nothing. Then the sum times
// the float reciprocal of the count; an empty list copies row reseed_rows[c].
__global__ void kmeans_update_kernel(const float* __restrict__ x, int ldx, int dim, const int32_t* __restrict__ order,
                                     const int64_t* __restrict__ off, float* __restrict__ cent, int ldc,
                                     const int32_t* __restrict__ reseed_rows, int64_t q, int64_t r) {
    const int c = blockIdx.x;
    const int64_t b = off[c], e = off[c + 1];
    const int64_t big = r * (q + 1);  // rows of the chunks one element longer
    for (int d = threadIdx.x; d < dim; d += blockDim.x) {
        if (e == b) {
            cent[(int64_t)c * ldc + d] = x[(int64_t)reseed_rows[c] * ldx + d];
            continue;
        }
        float acc = 0.f, s = 0.f;
        int64_t bound = -1;  // first row past the current chunk
        constexpr int U = 8;
        for (int64_t i0 = b; i0 < e; i0 += U) {
            int32_t rows[U];
            float v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) rows[u] = i0 + u < e ? order[i0 + u] : -1;
#pragma unroll
            for (int u = 0; u < U; ++u) v[u] = rows[u] >= 0 ? x[(int64_t)rows[u] * ldx + d] : 0.f;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (rows[u] < 0) break;
                if (rows[u] >= bound) {  // a new chunk starts: fold the finished one in
                    acc = __fadd_rn(acc, s);
                    s = 0.f;
                    const int64_t rr = rows[u];
                    const int64_t t = rr < big ? rr / (q + 1) : r + (rr - big) / q;
                    bound = (t + 1) * q + min(t + 1, r);
                }
                s = __fadd_rn(s, v[u]);
            }
        }
        acc = __fadd_rn(acc, s);
        const float rc = __fdiv_rn(1.0f, (float)(e - b));
        cent[(int64_t)c * ldc + d] = __fmul_rn(acc, rc);
    }
}

int launch_kmeans_certify(const float* key2, const int* id2, int64_t n, float margin, int32_t* assign, int32_t* amb,
                          int* amb_count, cudaStream_t st) {
    if (n == 0) return ANN_OK;
    const int blocks = (int)std::min<int64_t>(ceil_div(n, 256), kNumSMs * 8);
    kmeans_certify_kernel<<<blocks, 256, 0, st>>>(key2, id2, n, margin, assign, amb, amb_count);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_kmeans_ref_assign(const float* x, int ldx, int dim, const float* cent, int ldc, int C, const int32_t* amb,
                             const int* amb_count, int32_t* assign, cudaStream_t st) {
    kmeans_ref_assign_kernel<<<kNumSMs * 4, 256, 0, st>>>(x, ldx, dim, cent, ldc, C, amb, amb_count, assign);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

int launch_kmeans_update(const float* x, int ldx, int dim, const int32_t* order, const int64_t* off, int C,
                         float* centroids, int ldc, const int32_t* reseed_rows, int64_t n, int num_threads,
                         cudaStream_t st) {
    ANN_CHECK_ARG(num_threads >= 1 && n >= 1, "k-means update: %d threads over %lld rows", num_threads, (long long)n);
    const int64_t active = std::min<int64_t>(num_threads, n);  // run_parallel's actual_threads
    const int threads = (int)std::min<int64_t>(1024, ceil_div(dim, 32) * 32);
    kmeans_update_kernel<<<C, threads, 0, st>>>(x, ldx, dim, order, off, centroids, ldc, reseed_rows, n / active,
                                                n % active);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

// IVF-SQ8 index build on the GPU: the B200 form of IVFLSHIndex::fit
// (competitors/ivf_lsh/src/lsh_index_optimized.cpp:128-214, 551-616) for n_tables = 1, n_bits = 0.
//
// * k-means: the assignment step is the exact FP32 scan with k = 1 (flat_scan.cu, ties to the
//   lower centroid as the reference's strict `<` keeps the first minimum, :38-44); the update is a
//   per-list sum in a fixed order (rows sorted by list with a stable radix sort), so results do not
//   depend on thread scheduling -- unlike the reference, whose per-thread partial sums make its
//   centroids depend on the host's core count (:61-73, 594-601). Empty lists are reseeded.
// * reorder: rows grouped list by list, ascending original id inside a list (:155-173).
// * per-dimension SQ8 (:187-214), bit-identical to the reference: exact min/max, scale =
//   (max - min) * (1/255) -- the compiled reference multiplies by the float reciprocal -- or 1
//   when the range is <= 1e-8, offset = min (or 0), code = clamp(round((x - offset) / scale)) with
//   a true division and round-half-away-from-zero.
#include "common.cuh"
#include "ivf.cuh"

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

// One CTA per list: centroid = mean of its rows in ascending order (rows order[off[c]..off[c+1]));
// an empty list takes fallback_rows[c] (the reference reseeds from a fixed point, :609-613).
__global__ void centroid_update_kernel(const float* __restrict__ x, int ld, int dim, const int32_t* __restrict__ order,
                                       const int64_t* __restrict__ off, float* __restrict__ cent, int ldc,
                                       const float* __restrict__ fallback) {
    const int c = blockIdx.x;
    const int64_t b = off[c], e = off[c + 1];
    for (int d = threadIdx.x; d < dim; d += blockDim.x) {
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
        int64_t i = b;
        for (; i + 4 <= e; i += 4) {
            s0 += x[(int64_t)order[i] * ld + d];
            s1 += x[(int64_t)order[i + 1] * ld + d];
            s2 += x[(int64_t)order[i + 2] * ld + d];
            s3 += x[(int64_t)order[i + 3] * ld + d];
        }
        for (; i < e; ++i) s0 += x[(int64_t)order[i] * ld + d];
        const float s = (s0 + s1) + (s2 + s3);
        cent[(int64_t)c * ldc + d] = e > b ? s / (float)(e - b) : fallback[(int64_t)c * ld + d];
    }
}

int launch_centroid_update(const float* x, int ld, int dim, const int32_t* order, const int64_t* off, int C,
                           float* centroids, int ldc, const float* fallback_rows, cudaStream_t st) {
    centroid_update_kernel<<<C, 128, 0, st>>>(x, ld, dim, order, off, centroids, ldc, fallback_rows);
    ANN_LAUNCH_CHECK();
    return ANN_OK;
}

}  // namespace annb

/*
 * CPU restatement of the reference's k-means (IVFLSHIndex::run_kmeans,
 * competitors/ivf_lsh/src/lsh_index_optimized.cpp:551-616, with its workers :32-73).
 *
 * ORACLE INFRASTRUCTURE. Only tests/ load this code (through oracle/refmod.py), and only as the
 * checker; no product code path calls it.
 *
 * It is C++ rather than C for one reason: the initial centroids and the empty-list reseeds come
 * from std::shuffle(iota, std::mt19937(1337)) (:553-555), whose draw sequence is libstdc++'s
 * (std::mt19937 is fully specified, std::shuffle and uniform_int_distribution are not). Calling the
 * same library is the restatement. Everything else is written out step by step and compiled
 * without -ffast-math (see oracle/Makefile), so each rounding is the one written here:
 *
 *   assignment  every row to the first centroid with the smallest compute_l2_distance (:32-47),
 *               the reference's compiled arithmetic restated by orc_l2 (restate.c);
 *   update      ThreadPool chunk c of T (src/thread_pool.h:93-124; chunk c runs as thread_id c,
 *               :43-45) sums its rows per list, component by component, in row order starting
 *               from 0.0f (:60-73); the lists' sums are the chunk sums added in chunk order
 *               t = 0..T-1 starting from 0.0f (:594-601); a list's centroid is that sum divided by
 *               its count (:603-607), which the compiled reference (-ffast-math) computes as a
 *               multiplication by the float reciprocal of the count (pinned by tests/test_oracle.py
 *               against the reference's own fit: a true division differs in the last bit); an empty
 *               list takes row rand_indices[(c*37) % n] (:608-613).
 */
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <thread>
#include <vector>

extern "C" float orc_l2(const float *a, const float *b, int dim, float threshold, int isa);

extern "C" {

/* rand_indices of run_kmeans (:553-555): a permutation of [0, n). */
void orc_kmeans_order(int64_t n, int32_t *out) {
    std::vector<int> v((size_t)n);
    std::iota(v.begin(), v.end(), 0);
    std::shuffle(v.begin(), v.end(), std::mt19937(1337));
    std::copy(v.begin(), v.end(), out);
}

/* kmeans_assign_worker (:32-47) over rows [s, e). */
static void assign_range(const float *x, int64_t s, int64_t e, int dim, const float *cent, int C, int isa,
                         int32_t *assign) {
    for (int64_t i = s; i < e; ++i) {
        const float *pt = x + i * dim;
        float best = FLT_MAX;
        int bc = 0;
        for (int c = 0; c < C; ++c) {
            const float d = orc_l2(pt, cent + (int64_t)c * dim, dim, FLT_MAX, isa);
            if (d < best) {
                best = d;
                bc = c;
            }
        }
        assign[i] = bc;
    }
}

/*
 * run_kmeans: `iters` rounds of assign + update over x [n, dim] with C lists and a ThreadPool of
 * `num_threads`. Writes the final centroids [C, dim] and the last round's assignment [n] (the
 * lists the reference's fit builds, :150-173). `workers` only speeds up the assignment (each row is
 * independent, so the result does not depend on it).
 */
int orc_kmeans(const float *x, int64_t n, int dim, int C, int iters, int num_threads, int isa, int workers,
               float *cent, int32_t *assign) {
    if (n < 1 || dim < 1 || C < 1 || C > n || num_threads < 1) return -1;
    std::vector<int32_t> order((size_t)n);
    orc_kmeans_order(n, order.data());
    for (int c = 0; c < C; ++c)
        std::memcpy(cent + (int64_t)c * dim, x + (int64_t)order[(size_t)(c % n)] * dim, sizeof(float) * dim);
    std::fill(assign, assign + n, 0);
    const int T = num_threads;
    const int active = (int)std::min<int64_t>(T, n);  // run_parallel's actual_threads
    const int64_t chunk = n / active, rem = n % active;
    std::vector<float> local((size_t)T * C * dim);
    std::vector<int> lcount((size_t)T * C);
    std::vector<float> sums((size_t)C * dim);
    std::vector<int> counts(C);
    if (workers < 1) workers = 1;
    for (int it = 0; it < iters; ++it) {
        {
            std::vector<std::thread> th;
            const int64_t per = (n + workers - 1) / workers;
            for (int w = 0; w < workers; ++w) {
                const int64_t s = w * per, e = std::min<int64_t>(n, s + per);
                if (s < e) th.emplace_back(assign_range, x, s, e, dim, cent, C, isa, assign);
            }
            for (auto &t : th) t.join();
        }
        std::fill(local.begin(), local.end(), 0.0f);
        std::fill(lcount.begin(), lcount.end(), 0);
        int64_t start = 0;
        for (int t = 0; t < active; ++t) {  // chunk t runs with thread_id t
            const int64_t end = start + chunk + (t < rem ? 1 : 0);
            float *my = local.data() + (size_t)t * C * dim;
            int *mc = lcount.data() + (size_t)t * C;
            for (int64_t i = start; i < end; ++i) {
                const int c = assign[i];
                mc[c]++;
                for (int d = 0; d < dim; ++d) my[(size_t)c * dim + d] = my[(size_t)c * dim + d] + x[i * dim + d];
            }
            start = end;
        }
        std::fill(sums.begin(), sums.end(), 0.0f);
        std::fill(counts.begin(), counts.end(), 0);
        for (int t = 0; t < T; ++t)
            for (int c = 0; c < C; ++c) {
                counts[c] += lcount[(size_t)t * C + c];
                for (int d = 0; d < dim; ++d)
                    sums[(size_t)c * dim + d] = sums[(size_t)c * dim + d] + local[((size_t)t * C + c) * dim + d];
            }
        for (int c = 0; c < C; ++c) {
            if (counts[c] > 0) {
                const float rc = 1.0f / (float)counts[c];
                for (int d = 0; d < dim; ++d) cent[(int64_t)c * dim + d] = sums[(size_t)c * dim + d] * rc;
            } else {
                const int64_t r = order[(size_t)(((int64_t)c * 37) % n)];
                std::memcpy(cent + (int64_t)c * dim, x + r * dim, sizeof(float) * dim);
            }
        }
    }
    return 0;
}

}  // extern "C"

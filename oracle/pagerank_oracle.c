/*
 * ORACLE — test infrastructure only.
 *
 * A plain-C restatement of the reference's PageRank arithmetic, used by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg to CHECK
 * RESULTS (and as the timed CPU port of the reference's OpenMP path).  The
 * product path (eggpu_b200/) never links, loads or calls anything here.
 *
 * Functions and the reference code each one restates (paths are relative to
 * the reference project root):
 *
 *   orc_build_inbound      gpu_easygraph/functions/centrality/pagerank.cu:286-347
 *                          (build_inbound_from_csr: weight sanitising, FP64
 *                          out-weight sums, in-degree count, exclusive scan,
 *                          stable scatter by ascending source, dangling mask)
 *   orc_inbound_values     pagerank.cu:343 (alpha-scaled FP32 in_val)
 *   orc_pagerank_push      easygraph/functions/centrality/pagerank.py:75-139
 *                          (_pagerank_power_iteration: FP64 push loop, dangling
 *                          test out_sum <= 1e-15, uniform dangling mass, L1 stop
 *                          rule err < tol*n, one final normalisation), extended
 *                          with an optional teleport (personalisation) vector
 *   orc_pagerank_pull      the same maths as orc_pagerank_push evaluated as a
 *                          pull over the inbound CSR (bit-identical additions
 *                          per destination; OpenMP over destinations)
 *   orc_cpu_pagerank_omp   cpp_easygraph/functions/pagerank/pagerank.cpp:21-122
 *                          (_pagerank: OpenMP push with atomic adds; returns
 *                          the unnormalised vector like the reference)
 *
 * Parity pins: tests/golden/ holds vectors produced by the reference itself
 * (its Python power iteration and its compiled build_inbound_from_csr); the
 * oracle tests check every function above against them.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_BAD_ARG 8
#define ORC_NO_MEM 1

/* pagerank.cu:282-284 */
static int valid_endpoint(int32_t x, int32_t n) { return 0 <= x && x < n; }

/* pagerank.cu:305-312 and :330-340: each row's [begin, end) is clipped to
 * [0, m] and an inverted range becomes empty. */
static void row_range(const int32_t* V, int32_t u, int64_t m, int64_t* b, int64_t* e) {
    int64_t begin = V[u], end = V[u + 1];
    if (begin < 0) begin = 0;
    if (end > m) end = m;
    if (begin > end) begin = end;
    *b = begin;
    *e = end;
}

/* Final normalisation sum.  pagerank.py:134 uses Python's built-in sum(),
 * which since CPython 3.12 adds floats with Neumaier's compensated
 * (improved Kahan-Babuska) summation; restated here so the oracle's
 * normalised ranks match the reference bit for bit. */
static double neumaier_sum(const double* x, int32_t n) {
    double s = 0.0, c = 0.0;
    for (int32_t i = 0; i < n; ++i) {
        double t = s + x[i];
        if (fabs(s) >= fabs(x[i])) c += (s - t) + x[i];
        else c += (x[i] - t) + s;
        s = t;
    }
    if (c != 0.0 && isfinite(c)) s += c;
    return s;
}

/* pagerank.cu:311-312: non-finite or negative weights count as zero. */
static double sanitize(double w) { return (!isfinite(w) || w < 0.0) ? 0.0 : w; }

/*
 * Restates build_inbound_from_csr (pagerank.cu:286-347).  Outputs:
 *   in_row[n+1], in_col[nnz]   inbound CSR, rows = destinations, entries in
 *                              ascending source order (stable scatter :328-346)
 *   in_w[nnz] (nullable)       the sanitised FP64 edge weight of each entry
 *   dangling01[n]              1 where the FP64 out-weight sum is <= 0 (:324-326)
 *   out_weight_sum[n]          FP64 sums, accumulated in row order (:314)
 * Returns nnz (count of valid entries) through *out_nnz.
 */
int orc_build_inbound(const int32_t* V, const int32_t* E, const double* W, int32_t n, int64_t m,
                      int32_t* in_row, int32_t* in_col, double* in_w, int32_t* dangling01,
                      double* out_weight_sum, int64_t* out_nnz) {
    if (n < 0 || m < 0) return ORC_BAD_ARG;
    int32_t* indeg = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    int32_t* cur = (int32_t*)malloc(((size_t)n + 1) * sizeof(int32_t));
    if (!indeg || !cur) { free(indeg); free(cur); return ORC_NO_MEM; }
    for (int32_t u = 0; u < n; ++u) out_weight_sum[u] = 0.0;
    for (int32_t u = 0; u < n; ++u) {
        int64_t b, e;
        row_range(V, u, m, &b, &e);
        for (int64_t p = b; p < e; ++p) {
            int32_t v = E[p];
            if (!valid_endpoint(v, n)) continue;
            double w = W ? sanitize(W[p]) : 1.0;
            out_weight_sum[u] += w;
            indeg[v] += 1;
        }
    }
    in_row[0] = 0;
    for (int32_t i = 0; i < n; ++i) in_row[i + 1] = in_row[i] + indeg[i];
    for (int32_t u = 0; u < n; ++u) dangling01[u] = out_weight_sum[u] <= 0.0 ? 1 : 0;
    memcpy(cur, in_row, ((size_t)n + 1) * sizeof(int32_t));
    for (int32_t u = 0; u < n; ++u) {
        int64_t b, e;
        row_range(V, u, m, &b, &e);
        for (int64_t p = b; p < e; ++p) {
            int32_t v = E[p];
            if (!valid_endpoint(v, n)) continue;
            int32_t pos = cur[v]++;
            in_col[pos] = u;
            if (in_w) in_w[pos] = W ? sanitize(W[p]) : 1.0;
        }
    }
    *out_nnz = n > 0 ? in_row[n] : 0;
    free(indeg);
    free(cur);
    return ORC_OK;
}

/* pagerank.cu:343: in_val = (float)(alpha * (w / denom)), or 0 when denom <= 0. */
void orc_inbound_values(const int32_t* in_col, const double* in_w, const double* out_weight_sum,
                        int64_t nnz, double alpha, float* in_val) {
    for (int64_t i = 0; i < nnz; ++i) {
        double denom = out_weight_sum[in_col[i]];
        in_val[i] = denom > 0.0 ? (float)(alpha * (in_w[i] / denom)) : 0.0f;
    }
}

/*
 * Restates _pagerank_power_iteration (pagerank.py:75-139) on an out-edge CSR.
 *   W == NULL            unit weights (pagerank.py:104-107)
 *   sanitize != 0        weights cleaned like the GPU preparation (pagerank.cu:311)
 *   dangling_eps         a source is dangling when out_sum <= dangling_eps
 *                        (pagerank.py:118 uses 1e-15)
 *   teleport (nullable)  personalisation: the (1-alpha)/n term becomes
 *                        (1-alpha)*teleport[i]; dangling mass stays uniform
 * Returns the normalised ranks in out[n] (pagerank.py:134-139), the number
 * of sweeps run and the last L1 residual.
 */
int orc_pagerank_push(const int32_t* V, const int32_t* E, const double* W, int32_t n, int64_t m,
                      int32_t sanitize_w, double dangling_eps, double alpha, int32_t max_iter,
                      double tol, const double* teleport, double* out, int32_t* iters,
                      double* residual) {
    (void)m; /* rows come from V; m is the caller's size of E and W */
    if (n <= 0) { *iters = 0; *residual = 0.0; return ORC_OK; }
    if (max_iter < 1) max_iter = 1; /* pagerank.py:47-49 */
    if (tol < 0.0) tol = 0.0;       /* pagerank.py:51-52 */
    double* out_sums = (double*)calloc((size_t)n, sizeof(double));
    double* pr = (double*)malloc((size_t)n * sizeof(double));
    double* new_pr = (double*)malloc((size_t)n * sizeof(double));
    if (!out_sums || !pr || !new_pr) { free(out_sums); free(pr); free(new_pr); return ORC_NO_MEM; }
    int64_t edges = 0;
    for (int32_t u = 0; u < n; ++u) {
        for (int64_t p = V[u]; p < V[u + 1]; ++p) {
            double w = W ? (sanitize_w ? sanitize(W[p]) : W[p]) : 1.0;
            out_sums[u] += w;
            ++edges;
        }
    }
    if (edges == 0) { /* pagerank.py:96-98 */
        for (int32_t i = 0; i < n; ++i) out[i] = 1.0 / n;
        *iters = 0; *residual = 0.0;
        free(out_sums); free(pr); free(new_pr);
        return ORC_OK;
    }
    for (int32_t i = 0; i < n; ++i) pr[i] = 1.0 / n;
    int32_t it = 0;
    double err = 0.0;
    for (it = 0; it < max_iter; ++it) {
        for (int32_t i = 0; i < n; ++i) new_pr[i] = 0.0;
        double dangling_sum = 0.0;
        for (int32_t i = 0; i < n; ++i) {
            if (out_sums[i] <= dangling_eps) { dangling_sum += pr[i]; continue; }
            double base = alpha * pr[i] / out_sums[i];
            for (int64_t p = V[i]; p < V[i + 1]; ++p) {
                double w = W ? (sanitize_w ? sanitize(W[p]) : W[p]) : 1.0;
                new_pr[E[p]] += base * w;
            }
        }
        double jump = (1.0 - alpha) / n + alpha * dangling_sum / n;
        double dmass = alpha * dangling_sum / n;
        err = 0.0;
        for (int32_t i = 0; i < n; ++i) {
            double val = teleport ? new_pr[i] + (1.0 - alpha) * teleport[i] + dmass : new_pr[i] + jump;
            err += fabs(val - pr[i]);
            pr[i] = val;
        }
        if (err < tol * n) { ++it; break; }
    }
    double norm = neumaier_sum(pr, n);
    if (norm <= 0.0) {
        for (int32_t i = 0; i < n; ++i) out[i] = 1.0 / n;
    } else {
        double inv = 1.0 / norm;
        for (int32_t i = 0; i < n; ++i) out[i] = pr[i] * inv;
    }
    *iters = it;
    *residual = err;
    free(out_sums); free(pr); free(new_pr);
    return ORC_OK;
}

/*
 * The same arithmetic as orc_pagerank_push, evaluated as a pull over the
 * inbound CSR from orc_build_inbound (entries in ascending source order, so
 * each destination sees the same sequence of FP64 additions as the push loop).
 * out_weight_sum / in_w come from orc_build_inbound (sanitised weights); the
 * dangling test is out_weight_sum <= dangling_eps.  The residual is summed in
 * vertex order like pagerank.py:127-130.  OpenMP parallel over destinations.
 * Optionally returns the unnormalised final iterate and the previous one.
 */
int orc_pagerank_pull(const int32_t* in_row, const int32_t* in_col, const double* in_w,
                      const double* out_weight_sum, int32_t n, double dangling_eps, double alpha,
                      int32_t max_iter, double tol, const double* teleport, double* out,
                      int32_t* iters, double* residual, int32_t nthreads) {
    if (n <= 0) { *iters = 0; *residual = 0.0; return ORC_OK; }
    if (max_iter < 1) max_iter = 1;
    if (tol < 0.0) tol = 0.0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    if (in_row[n] == 0) {
        for (int32_t i = 0; i < n; ++i) out[i] = 1.0 / n;
        *iters = 0; *residual = 0.0;
        return ORC_OK;
    }
    double* pr = (double*)malloc((size_t)n * sizeof(double));
    double* base = (double*)malloc((size_t)n * sizeof(double));
    double* nxt = (double*)malloc((size_t)n * sizeof(double));
    if (!pr || !base || !nxt) { free(pr); free(base); free(nxt); return ORC_NO_MEM; }
    for (int32_t i = 0; i < n; ++i) pr[i] = 1.0 / n;
    int32_t it;
    double err = 0.0;
    for (it = 0; it < max_iter; ++it) {
        double dangling_sum = 0.0;
        for (int32_t i = 0; i < n; ++i) {
            if (out_weight_sum[i] <= dangling_eps) { dangling_sum += pr[i]; base[i] = 0.0; }
            else base[i] = alpha * pr[i] / out_weight_sum[i];
        }
#pragma omp parallel for schedule(dynamic, 1024)
        for (int32_t v = 0; v < n; ++v) {
            double acc = 0.0;
            for (int32_t k = in_row[v]; k < in_row[v + 1]; ++k) {
                int32_t u = in_col[k];
                if (out_weight_sum[u] <= dangling_eps) continue;
                acc += base[u] * (in_w ? in_w[k] : 1.0);
            }
            nxt[v] = acc;
        }
        double jump = (1.0 - alpha) / n + alpha * dangling_sum / n;
        double dmass = alpha * dangling_sum / n;
        err = 0.0;
        for (int32_t i = 0; i < n; ++i) {
            double val = teleport ? nxt[i] + (1.0 - alpha) * teleport[i] + dmass : nxt[i] + jump;
            err += fabs(val - pr[i]);
            pr[i] = val;
        }
        if (err < tol * n) { ++it; break; }
    }
    double norm = neumaier_sum(pr, n);
    if (norm <= 0.0) {
        for (int32_t i = 0; i < n; ++i) out[i] = 1.0 / n;
    } else {
        double inv = 1.0 / norm;
        for (int32_t i = 0; i < n; ++i) out[i] = pr[i] * inv;
    }
    *iters = it;
    *residual = err;
    free(pr); free(base); free(nxt);
    return ORC_OK;
}

/*
 * Port of the reference's OpenMP CPU PageRank (_pagerank,
 * cpp_easygraph/functions/pagerank/pagerank.cpp:21-122), over an out-edge
 * CSR instead of the reference's linked-list graph (the traversal order of
 * a source's edges does not matter: every contribution is an atomic add).
 *   weighted logic only when W is given and some weight differs from 1
 *   (:52-67); dangling = outdeg == 0, or out-weight < 1e-15 when weighted
 *   (:76); push with `omp atomic` (:82-102); jump (:105); stop when the
 *   L1 diff < threshold*N (:115).  Writes the unnormalised ranks (the
 *   reference returns them as a list, :119-121) and the sweep count.
 */
int orc_cpu_pagerank_omp(const int32_t* V, const int32_t* E, const double* W, int32_t n,
                         double alpha, int32_t max_iter, double threshold, double* out,
                         int32_t* sweeps, int32_t nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    if (n <= 0) { *sweeps = 0; return ORC_OK; }
    double* outw = (double*)calloc((size_t)n, sizeof(double));
    double* old_pr = (double*)malloc((size_t)n * sizeof(double));
    double* new_pr = (double*)calloc((size_t)n, sizeof(double));
    if (!outw || !old_pr || !new_pr) { free(outw); free(old_pr); free(new_pr); return ORC_NO_MEM; }
    int weighted = 0;
    if (W) {
#pragma omp parallel for reduction(| : weighted)
        for (int32_t i = 0; i < n; ++i) {
            double s = 0.0;
            for (int64_t p = V[i]; p < V[i + 1]; ++p) {
                s += W[p];
                if (fabs(W[p] - 1.0) > 1e-9) weighted = 1;
            }
            outw[i] = s;
        }
    }
    for (int32_t i = 0; i < n; ++i) old_pr[i] = 1.0 / n;
    int32_t cnt = 0, performed = 0;
    while (cnt < max_iter) {
        double dangling_sum = 0.0;
#pragma omp parallel for reduction(+ : dangling_sum)
        for (int32_t i = 0; i < n; ++i) {
            int is_dangling = weighted ? (outw[i] < 1e-15) : (V[i + 1] == V[i]);
            if (is_dangling) dangling_sum += old_pr[i];
        }
#pragma omp parallel for schedule(dynamic, 128)
        for (int32_t i = 0; i < n; ++i) {
            int64_t deg = V[i + 1] - V[i];
            if (weighted ? (outw[i] < 1e-15) : (deg == 0)) continue;
            double out_val = (old_pr[i] / (weighted ? outw[i] : (double)deg)) * alpha;
            for (int64_t p = V[i]; p < V[i + 1]; ++p) {
                double add = weighted ? out_val * W[p] : out_val;
#pragma omp atomic
                new_pr[E[p]] += add;
            }
        }
        double diff_sum = 0.0;
        double jump = (1.0 - alpha) / n + (dangling_sum / n) * alpha;
#pragma omp parallel for reduction(+ : diff_sum)
        for (int32_t i = 0; i < n; ++i) {
            double fin = new_pr[i] + jump;
            diff_sum += fabs(fin - old_pr[i]);
            old_pr[i] = fin;
            new_pr[i] = 0.0;
        }
        if (diff_sum < threshold * n) { ++performed; break; }
        cnt++;
        ++performed;
    }
    memcpy(out, old_pr, (size_t)n * sizeof(double));
    *sweeps = performed;
    free(outw); free(old_pr); free(new_pr);
    return ORC_OK;
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/*
 * nmf_oracle.c -- CPU restatement of the reference NMF iteration loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA library
 * is compared against (parity tests, smoke(), and the CPU-baseline leg of
 * bench.py).  Nothing in the shipped library links, loads or calls it.
 *
 * It restates, in plain C, the f64 algorithms of omicverse/rust-NMF
 * `rust/src/lib.rs` (cited per function below): same loop structure, same
 * summation order (forward / reverse exactly as cited), no FMA contraction
 * (build with -ffp-contract=off), and OpenMP over H columns / W rows the way
 * the reference uses rayon.  Every output element is reduced sequentially by
 * one thread, so results do not depend on the thread count.
 *
 * Third-party arithmetic that the reference delegates to `matrixmultiply
 * 0.3.10` through `ndarray 0.16.1` (rust/Cargo.lock:86-88, 105-107) -- the
 * HALS/dnmf products W^T V and V H^T (lib.rs:514, 536) and the dense WH used
 * by the objectives (lib.rs:57) -- is restated as a plain forward-order dot
 * product.  matrixmultiply's own blocking order is not pinned by any
 * reference test, so HALS/dnmf/objective parity is a tolerance, not bits.
 *
 * Pinned against the reference's recorded outputs in
 * examples/tutorial_quickstart.ipynb (see tests/golden/).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Method ids: same numbering as include/nmfcu.h. */
enum { ORC_BRUNET = 0, ORC_LEE = 1, ORC_HALS = 4, ORC_EHALS = 5, ORC_DNMF = 6 };
enum { ORC_STOP_MAX_ITER = 0, ORC_STOP_STATIONARY = 1 };

typedef int64_t i64;

/* transpose_owned, lib.rs:28-38: a (m x n) -> a_t (n x m). */
static double *transpose(const double *a, i64 m, i64 n) {
    double *t = (double *)malloc(sizeof(double) * (size_t)(m * n > 0 ? m * n : 1));
    for (i64 i = 0; i < m; i++)
        for (i64 j = 0; j < n; j++) t[j * m + i] = a[i * n + j];
    return t;
}

static void set_threads(int nt) {
#ifdef _OPENMP
    if (nt > 0) omp_set_num_threads(nt);
#else
    (void)nt;
#endif
}

/* ------------------------------------------------------------------------ */
/* Brunet / KL multiplicative updates                                        */
/* ------------------------------------------------------------------------ */

/* divergence_update_h_inner, lib.rs:74-115.  v_t is p x n, w is n x r,
 * w_t is r x n, h is r x p, sum_w has r entries.  Writes hp (r x p). */
static void div_update_h_inner(i64 n, i64 p, i64 r, const double *v_t, const double *w,
                               const double *w_t, const double *h, const double *sum_w,
                               double *hp) {
#pragma omp parallel
    {
        double *h_col = (double *)malloc(sizeof(double) * (size_t)(r > 0 ? r : 1));
        double *wh_col = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(static)
        for (i64 j = 0; j < p; j++) {
            for (i64 k = 0; k < r; k++) h_col[k] = h[k * p + j];
            for (i64 u = 0; u < n; u++) {
                double wh = 0.0;
                for (i64 k = 0; k < r; k++) wh += w[u * r + k] * h_col[k];
                wh_col[u] = (wh != 0.0) ? v_t[j * n + u] / wh : 0.0;
            }
            for (i64 i = 0; i < r; i++) {
                double tmp = 0.0;
                for (i64 u = 0; u < n; u++) tmp += w_t[i * n + u] * wh_col[u];
                hp[i * p + j] = h_col[i] * tmp / sum_w[i];
            }
        }
        free(h_col);
        free(wh_col);
    }
}

/* Column sums of W in forward order, lib.rs:1563-1568 / 132-139. */
static void col_sums(i64 n, i64 r, const double *w, double *sum_w) {
    for (i64 k = 0; k < r; k++) {
        double s = 0.0;
        for (i64 u = 0; u < n; u++) s += w[u * r + k];
        sum_w[k] = s;
    }
}

/* divergence_update_w_impl, lib.rs:151-204.  Writes wp (n x r). */
static void div_update_w(i64 n, i64 p, i64 r, const double *v, const double *w,
                         const double *h, double *wp) {
    double *sum_h = (double *)malloc(sizeof(double) * (size_t)(r > 0 ? r : 1));
    for (i64 k = 0; k < r; k++) {
        double s = 0.0;
        for (i64 u = 0; u < p; u++) s += h[k * p + u];
        sum_h[k] = s;
    }
    double *h_t = transpose(h, r, p); /* p x r, lib.rs:175-180 */
#pragma omp parallel
    {
        double *wh_row = (double *)malloc(sizeof(double) * (size_t)(p > 0 ? p : 1));
#pragma omp for schedule(static)
        for (i64 i = 0; i < n; i++) {
            for (i64 u = 0; u < p; u++) {
                double wh = 0.0;
                for (i64 k = 0; k < r; k++) wh += w[i * r + k] * h_t[u * r + k];
                wh_row[u] = (wh != 0.0) ? v[i * p + u] / wh : 0.0;
            }
            for (i64 j = 0; j < r; j++) {
                double tmp = 0.0;
                for (i64 u = 0; u < p; u++) tmp += h[j * p + u] * wh_row[u];
                wp[i * r + j] = w[i * r + j] * tmp / sum_h[j];
            }
        }
        free(wh_row);
    }
    free(h_t);
    free(sum_h);
}

/* ------------------------------------------------------------------------ */
/* Lee / Frobenius multiplicative updates                                    */
/* ------------------------------------------------------------------------ */

/* W^T W with reverse-u order from w_t, lib.rs:1622-1631 and 264-273. */
static void wtw_rev(i64 n, i64 r, const double *w_t, double *wtw) {
    for (i64 i = 0; i < r; i++)
        for (i64 j = 0; j < r; j++) {
            double s = 0.0;
            for (i64 u = n - 1; u >= 0; u--) s += w_t[i * n + u] * w_t[j * n + u];
            wtw[i * r + j] = s;
        }
}

/* euclidean_update_h_inner, lib.rs:213-245. */
static void euc_update_h_inner(i64 n, i64 p, i64 r, const double *v_t, const double *w_t,
                               const double *h, const double *wtw, double eps, double *hp) {
#pragma omp parallel for schedule(static)
    for (i64 j = 0; j < p; j++) {
        for (i64 i = 0; i < r; i++) {
            double numer = 0.0;
            for (i64 u = n - 1; u >= 0; u--) numer += w_t[i * n + u] * v_t[j * n + u];
            double den = 0.0;
            for (i64 l = r - 1; l >= 0; l--) den += wtw[i * r + l] * h[l * p + j];
            double temp = h[i * p + j] * numer;
            hp[i * p + j] = (temp > eps ? temp : eps) / (den + eps);
        }
    }
}

/* euclidean_update_w_impl, lib.rs:281-322. */
static void euc_update_w(i64 n, i64 p, i64 r, const double *v, const double *w,
                         const double *h, double eps, double *wp) {
    double *hht = (double *)malloc(sizeof(double) * (size_t)(r * r > 0 ? r * r : 1));
    for (i64 j = 0; j < r; j++)
        for (i64 i = 0; i < r; i++) {
            double s = 0.0;
            for (i64 u = p - 1; u >= 0; u--) s += h[j * p + u] * h[i * p + u];
            hht[i * r + j] = s;
        }
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; i++) {
        for (i64 j = 0; j < r; j++) {
            double numer = 0.0;
            for (i64 u = p - 1; u >= 0; u--) numer += v[i * p + u] * h[j * p + u];
            double den = 0.0;
            for (i64 l = r - 1; l >= 0; l--) den += w[i * r + l] * hht[l * r + j];
            double temp = w[i * r + j] * numer;
            wp[i * r + j] = (temp < eps ? eps : temp) / (den + eps);
        }
    }
    free(hht);
}

/* ------------------------------------------------------------------------ */
/* HALS / dnmf                                                               */
/* ------------------------------------------------------------------------ */

/* Rust f64::max: returns the non-NaN operand if one is NaN. */
static double rmax(double a, double b) {
    if (isnan(a)) return b;
    if (isnan(b)) return a;
    return a > b ? a : b;
}

/* compute_wtv, lib.rs:493-519 (matrixmultiply restated as forward dots).
 * v_t is p x n, w_t is r x n; writes wtv (r x p). */
static void compute_wtv(i64 n, i64 p, i64 r, const double *w_t, const double *v_t, double *wtv) {
#pragma omp parallel for schedule(static)
    for (i64 j = 0; j < p; j++)
        for (i64 k = 0; k < r; k++) {
            double s = 0.0;
            for (i64 u = 0; u < n; u++) s += w_t[k * n + u] * v_t[j * n + u];
            wtv[k * p + j] = s;
        }
}

/* compute_vht, lib.rs:522-540; writes vht (n x r). */
static void compute_vht(i64 n, i64 p, i64 r, const double *v, const double *h, double *vht) {
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; i++)
        for (i64 k = 0; k < r; k++) {
            double s = 0.0;
            for (i64 u = 0; u < p; u++) s += v[i * p + u] * h[k * p + u];
            vht[i * r + k] = s;
        }
}

/* compute_wtw_from_wt, lib.rs:543-560 (forward order). */
static void wtw_fwd(i64 n, i64 r, const double *w_t, double *wtw) {
    for (i64 k = 0; k < r; k++)
        for (i64 j = 0; j < r; j++) {
            double s = 0.0;
            for (i64 i = 0; i < n; i++) s += w_t[k * n + i] * w_t[j * n + i];
            wtw[k * r + j] = s;
        }
}

/* compute_hht, lib.rs:563-579 (forward order). */
static void hht_fwd(i64 p, i64 r, const double *h, double *hht) {
    for (i64 k = 0; k < r; k++)
        for (i64 j = 0; j < r; j++) {
            double s = 0.0;
            for (i64 u = 0; u < p; u++) s += h[k * p + u] * h[j * p + u];
            hht[k * r + j] = s;
        }
}

/* hals_update_h (lib.rs:582-608) when lambda = gamma = 0 and the plain
 * max(wtw_kk, eps) denominator; hals_update_h_reg (lib.rs:1068-1092) with
 * reg != 0.  The two differ only in `wtv - lambda` and `wtw_kk + gamma`;
 * with lambda = gamma = 0 the reg form is bitwise the plain form
 * (x - 0.0 == x, x + 0.0 == x for every non-NaN, non -0.0 x). */
static void hals_update_h(i64 p, i64 r, double *h, const double *wtv, const double *wtw,
                          double lambda, double gamma, int reg, double eps) {
#pragma omp parallel
    {
        double *hc = (double *)malloc(sizeof(double) * (size_t)(r > 0 ? r : 1));
#pragma omp for schedule(static)
        for (i64 u = 0; u < p; u++) {
            for (i64 k = 0; k < r; k++) hc[k] = h[k * p + u];
            for (i64 k = 0; k < r; k++) {
                double s = reg ? wtv[k * p + u] - lambda : wtv[k * p + u];
                for (i64 j = 0; j < r; j++)
                    if (j != k) s -= wtw[k * r + j] * hc[j];
                double d = reg ? rmax(wtw[k * r + k] + gamma, eps) : rmax(wtw[k * r + k], eps);
                double val = s / d;
                hc[k] = val > eps ? val : eps;
            }
            for (i64 k = 0; k < r; k++) h[k * p + u] = hc[k];
        }
        free(hc);
    }
}

/* hals_update_w (lib.rs:611-635) / hals_update_w_reg (lib.rs:1095-1119). */
static void hals_update_w(i64 n, i64 r, double *w, const double *vht, const double *hht,
                          double lambda, double gamma, int reg, double eps) {
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; i++) {
        double *wr = w + i * r;
        for (i64 k = 0; k < r; k++) {
            double s = reg ? vht[i * r + k] - lambda : vht[i * r + k];
            for (i64 j = 0; j < r; j++)
                if (j != k) s -= hht[k * r + j] * wr[j];
            double d = reg ? rmax(hht[k * r + k] + gamma, eps) : rmax(hht[k * r + k], eps);
            double val = s / d;
            wr[k] = val > eps ? val : eps;
        }
    }
}

/* extract_diagonal, lib.rs:808-824: unit-norm W columns / H rows; d[k]. */
static void extract_diagonal(i64 n, i64 p, i64 r, double *w, double *h, double *d) {
    for (i64 k = 0; k < r; k++) {
        double nw = 0.0, nh = 0.0;
        for (i64 i = 0; i < n; i++) nw += w[i * r + k] * w[i * r + k];
        for (i64 j = 0; j < p; j++) nh += h[k * p + j] * h[k * p + j];
        nw = sqrt(nw);
        nh = sqrt(nh);
        double dk = nw * nh;
        if (nw > 0.0)
            for (i64 i = 0; i < n; i++) w[i * r + k] /= nw;
        if (nh > 0.0)
            for (i64 j = 0; j < p; j++) h[k * p + j] /= nh;
        d[k] = dk;
    }
}

/* ------------------------------------------------------------------------ */
/* Objectives and stopping                                                   */
/* ------------------------------------------------------------------------ */

/* wh_dense (lib.rs:43-61) element, restated as a forward dot. */
static inline double wh_at(i64 p, i64 r, const double *w, const double *h, i64 i, i64 j) {
    double s = 0.0;
    for (i64 k = 0; k < r; k++) s += w[i * r + k] * h[k * p + j];
    return s;
}

/* kl_divergence, lib.rs:1410-1431 (j outer, i inner, one running sum). */
double orc_kl_divergence(i64 n, i64 p, i64 r, const double *v, const double *w, const double *h) {
    double s = 0.0;
    for (i64 j = 0; j < p; j++)
        for (i64 i = 0; i < n; i++) {
            double vv = v[i * p + j];
            double ww = wh_at(p, r, w, h, i, j);
            if (vv > 0.0) {
                if (ww > 0.0) s += vv * log(vv / ww) - vv + ww;
            } else {
                s += ww;
            }
        }
    return s;
}

/* euclidean_distance, lib.rs:1434-1445: 0.5 * sum((V - WH)^2). */
double orc_euclidean_distance(i64 n, i64 p, i64 r, const double *v, const double *w,
                              const double *h) {
    double s = 0.0;
    for (i64 j = 0; j < p; j++)
        for (i64 i = 0; i < n; i++) {
            double d = v[i * p + j] - wh_at(p, r, w, h, i, j);
            s += d * d;
        }
    return 0.5 * s;
}

/* StationaryStop, lib.rs:1336-1401. */
typedef struct {
    i64 check_interval, check_niter;
    double threshold, last_max, last_min;
    i64 n_collected;
} stationary_t;

static void st_reset(stationary_t *s) {
    s->last_max = -INFINITY;
    s->last_min = INFINITY;
    s->n_collected = 0;
}
static void st_record(stationary_t *s, double v) {
    if (v > s->last_max) s->last_max = v;
    if (v < s->last_min) s->last_min = v;
    s->n_collected++;
}
static int st_should_stop(stationary_t *s, i64 i, double dev) {
    if (isnan(dev)) return 1;
    if (i == 0) {
        st_reset(s);
        st_record(s, dev);
        return 0;
    }
    if (s->n_collected == 0) {
        /* `i % check_interval` panics in the reference when check_interval
         * is 0; it is only evaluated once the window is empty. */
        if (s->check_interval == 0) return -1;
        if (i % s->check_interval != 0) return 0;
    }
    st_record(s, dev);
    if (s->n_collected == s->check_niter + 1) {
        double crit = fabs(s->last_max - s->last_min) / (double)s->check_niter;
        if (crit <= s->threshold) return 1;
        st_reset(s);
    }
    return 0;
}

/* pmax_inplace, lib.rs:1452-1458. */
static void pmax_inplace(double *x, i64 len, double eps) {
    for (i64 i = 0; i < len; i++)
        if (x[i] < eps) x[i] = eps;
}

/* col_rescale, lib.rs:1461-1470. */
static void col_rescale(i64 n, i64 r, double *w) {
    for (i64 j = 0; j < r; j++) {
        double s = 0.0;
        for (i64 i = 0; i < n; i++) s += w[i * r + j];
        if (s > 0.0)
            for (i64 i = 0; i < n; i++) w[i * r + j] /= s;
    }
}

/* ------------------------------------------------------------------------ */
/* Public oracle entry points                                                */
/* ------------------------------------------------------------------------ */

/* Single-step updates: py_divergence_update_{h,w} / py_euclidean_update_{h,w}
 * (lib.rs:1849-1907 -> divergence_update_h_impl :120-144,
 * divergence_update_w_impl :151-204, euclidean_update_h_impl :249-276,
 * euclidean_update_w_impl :281-322). */
void orc_update_h_brunet(i64 n, i64 p, i64 r, const double *v, const double *w, const double *h,
                         double *hp, int nt) {
    set_threads(nt);
    double *sum_w = (double *)malloc(sizeof(double) * (size_t)(r > 0 ? r : 1));
    col_sums(n, r, w, sum_w);
    double *v_t = transpose(v, n, p);
    double *w_t = transpose(w, n, r);
    div_update_h_inner(n, p, r, v_t, w, w_t, h, sum_w, hp);
    free(v_t);
    free(w_t);
    free(sum_w);
}

void orc_update_w_brunet(i64 n, i64 p, i64 r, const double *v, const double *w, const double *h,
                         double *wp, int nt) {
    set_threads(nt);
    div_update_w(n, p, r, v, w, h, wp);
}

void orc_update_h_lee(i64 n, i64 p, i64 r, const double *v, const double *w, const double *h,
                      double eps, double *hp, int nt) {
    set_threads(nt);
    double *v_t = transpose(v, n, p);
    double *w_t = transpose(w, n, r);
    double *wtw = (double *)malloc(sizeof(double) * (size_t)(r * r > 0 ? r * r : 1));
    wtw_rev(n, r, w_t, wtw);
    euc_update_h_inner(n, p, r, v_t, w_t, h, wtw, eps, hp);
    free(wtw);
    free(v_t);
    free(w_t);
}

void orc_update_w_lee(i64 n, i64 p, i64 r, const double *v, const double *w, const double *h,
                      double eps, double *wp, int nt) {
    set_threads(nt);
    euc_update_w(n, p, r, v, w, h, eps, wp);
}

/*
 * orc_nmf_run: the full loop for brunet / lee / hals / ehals / dnmf.
 *   nmf_run_brunet lib.rs:1529-1586, nmf_run_lee :1589-1647,
 *   nmf_run_hals :638-688, nmf_run_ehals :711-786, nmf_run_dnmf :827-906.
 * W (n x r) and H (r x p) hold W0/H0 on entry and the result on exit.
 * dev must hold max_iter + 1 doubles.  Returns 0, or -1 for an unknown
 * method, -2 when the stationary stop evaluates `i % 0` (the reference
 * panics there, lib.rs:1388).
 */
int orc_nmf_run(int method, i64 n, i64 p, i64 r, const double *v, double *w, double *h,
                i64 max_iter, double eps, int rescale, double sparsity_h, double sparsity_w,
                double smoothness_h, double smoothness_w, int stop, double stationary_th,
                i64 check_interval, i64 check_niter, double *dev, i64 *n_dev, i64 *n_iter,
                int nt) {
    if (method != ORC_BRUNET && method != ORC_LEE && method != ORC_HALS && method != ORC_EHALS &&
        method != ORC_DNMF)
        return -1;
    set_threads(nt);
    stationary_t st = {check_interval, check_niter, stationary_th, -INFINITY, INFINITY, 0};
    i64 nd = 0;
    const int kl = (method == ORC_BRUNET);
    const int stat = (stop == ORC_STOP_STATIONARY);
    const double beps = DBL_EPSILON; /* lib.rs:1539 */

    double *v_t = transpose(v, n, p); /* lib.rs:1546 / 1606 / 652 / 844 */
    double *tmp_h = (double *)malloc(sizeof(double) * (size_t)(r * p > 0 ? r * p : 1));
    double *tmp_w = (double *)malloc(sizeof(double) * (size_t)(n * r > 0 ? n * r : 1));
    double *sq = (double *)malloc(sizeof(double) * (size_t)(r * r > 0 ? r * r : 1));
    double *sq2 = (double *)malloc(sizeof(double) * (size_t)(r * r > 0 ? r * r : 1));
    double *sum_w = (double *)malloc(sizeof(double) * (size_t)(r > 0 ? r : 1));
    double *dg = (double *)malloc(sizeof(double) * (size_t)(r > 0 ? r : 1));
    double *wtv = (method == ORC_HALS || method == ORC_EHALS || method == ORC_DNMF)
                      ? (double *)malloc(sizeof(double) * (size_t)(r * p > 0 ? r * p : 1))
                      : NULL;
    double *vht = (method == ORC_HALS || method == ORC_EHALS || method == ORC_DNMF)
                      ? (double *)malloc(sizeof(double) * (size_t)(n * r > 0 ? n * r : 1))
                      : NULL;
    /* ehals: the previous iterate, initially the start (lib.rs:743-744). */
    double *w_prev = NULL, *h_prev = NULL;
    if (method == ORC_EHALS) {
        w_prev = (double *)malloc(sizeof(double) * (size_t)(n * r > 0 ? n * r : 1));
        h_prev = (double *)malloc(sizeof(double) * (size_t)(r * p > 0 ? r * p : 1));
        memcpy(w_prev, w, sizeof(double) * (size_t)(n * r));
        memcpy(h_prev, h, sizeof(double) * (size_t)(r * p));
    }

    i64 iter = 0;
    int done = 0, status = 0;
    if (stat) {
        double d = kl ? orc_kl_divergence(n, p, r, v, w, h) : orc_euclidean_distance(n, p, r, v, w, h);
        dev[nd++] = d;
        if (st_should_stop(&st, 0, d) != 0) done = 1;
    }
    while (!done && iter < max_iter) {
        iter++;
        double *w_t = transpose(w, n, r);
        if (method == ORC_BRUNET) {
            col_sums(n, r, w, sum_w);
            div_update_h_inner(n, p, r, v_t, w, w_t, h, sum_w, tmp_h);
            memcpy(h, tmp_h, sizeof(double) * (size_t)(r * p));
            div_update_w(n, p, r, v, w, h, tmp_w);
            memcpy(w, tmp_w, sizeof(double) * (size_t)(n * r));
            if (iter % 10 == 0) {
                pmax_inplace(h, r * p, beps);
                pmax_inplace(w, n * r, beps);
            }
        } else if (method == ORC_LEE) {
            wtw_rev(n, r, w_t, sq);
            euc_update_h_inner(n, p, r, v_t, w_t, h, sq, eps, tmp_h);
            memcpy(h, tmp_h, sizeof(double) * (size_t)(r * p));
            euc_update_w(n, p, r, v, w, h, eps, tmp_w);
            memcpy(w, tmp_w, sizeof(double) * (size_t)(n * r));
            if (rescale) col_rescale(n, r, w);
        } else {
            const int reg = (method == ORC_DNMF);
            if (method == ORC_EHALS) {
                /* x <- max(eps, x + 0.5 (x - prev)); prev <- old x (lib.rs:755-767) */
                for (i64 t = 0; t < n * r; t++) {
                    const double x = w[t], ext = x + 0.5 * (x - w_prev[t]);
                    w[t] = ext > eps ? ext : eps;
                    w_prev[t] = x;
                }
                for (i64 t = 0; t < r * p; t++) {
                    const double x = h[t], ext = x + 0.5 * (x - h_prev[t]);
                    h[t] = ext > eps ? ext : eps;
                    h_prev[t] = x;
                }
                free(w_t);
                w_t = transpose(w, n, r);
            }
            compute_wtv(n, p, r, w_t, v_t, wtv);
            wtw_fwd(n, r, w_t, sq);
            hals_update_h(p, r, h, wtv, sq, sparsity_h, smoothness_h, reg, eps);
            compute_vht(n, p, r, v, h, vht);
            hht_fwd(p, r, h, sq2);
            hals_update_w(n, r, w, vht, sq2, sparsity_w, smoothness_w, reg, eps);
            if (reg) {
                extract_diagonal(n, p, r, w, h, dg);
                for (i64 k = 0; k < r; k++)
                    for (i64 j = 0; j < p; j++) h[k * p + j] *= dg[k];
            }
        }
        free(w_t);
        if (stat) {
            double d = kl ? orc_kl_divergence(n, p, r, v, w, h)
                          : orc_euclidean_distance(n, p, r, v, w, h);
            dev[nd++] = d;
            int rc = st_should_stop(&st, iter, d);
            if (rc < 0) {
                status = -2;
                break;
            }
            if (rc) break;
        }
    }
    /* dnmf stopped at iteration 0 extracts the diagonal before returning
     * (lib.rs:852-855). */
    if (method == ORC_DNMF && stat && iter == 0 && done) extract_diagonal(n, p, r, w, h, dg);

    *n_dev = nd;
    *n_iter = iter;
    free(v_t);
    free(tmp_h);
    free(tmp_w);
    free(sq);
    free(sq2);
    free(sum_w);
    free(dg);
    free(wtv);
    free(vht);
    free(w_prev);
    free(h_prev);
    return status;
}

/* ------------------------------------------------------------------------ */
/* nsNMF and offset                                                          */
/* ------------------------------------------------------------------------ */

/* smoothing_matrix, lib.rs:458-466: S = (1 - theta) I + (theta / r) 1 1^T. */
static void smoothing(i64 r, double theta, double *s) {
    const double off = theta / (double)r;
    for (i64 i = 0; i < r; i++)
        for (i64 j = 0; j < r; j++) s[i * r + j] = (i == j) ? (1.0 - theta) + off : off;
}

/* c = a (m x k) * b (k x q), forward dots (ndarray `dot`, lib.rs:1811 and
 * :1819, restated). */
static void mul_rs(i64 m, i64 k, i64 q, const double *a, const double *b, double *c) {
    for (i64 i = 0; i < m; i++)
        for (i64 j = 0; j < q; j++) {
            double acc = 0.0;
            for (i64 l = 0; l < k; l++) acc += a[i * k + l] * b[l * q + j];
            c[i * q + j] = acc;
        }
}

/*
 * orc_nmf_run_nsnmf: nmf_run_nsnmf, lib.rs:1762-1830.  Each iteration: the
 * KL H update with W S in place of W, the KL W update with S H in place of H,
 * then col_rescale(W); objective KL(V, (W S) H).  No clamp.
 */
int orc_nmf_run_nsnmf(i64 n, i64 p, i64 r, const double *v, double *w, double *h, i64 max_iter,
                      double theta, int stop, double stationary_th, i64 check_interval,
                      i64 check_niter, double *dev, i64 *n_dev, i64 *n_iter, int nt) {
    set_threads(nt);
    stationary_t st = {check_interval, check_niter, stationary_th, -INFINITY, INFINITY, 0};
    const int stat = (stop == ORC_STOP_STATIONARY);
    const size_t rr = (size_t)(r * r > 0 ? r * r : 1);
    const size_t nr = (size_t)(n * r > 0 ? n * r : 1), rp = (size_t)(r * p > 0 ? r * p : 1);
    double *S = (double *)malloc(sizeof(double) * rr);
    double *ws = (double *)malloc(sizeof(double) * nr);
    double *sh = (double *)malloc(sizeof(double) * rp);
    double *tmp_h = (double *)malloc(sizeof(double) * rp);
    double *tmp_w = (double *)malloc(sizeof(double) * nr);
    double *sum_ws = (double *)malloc(sizeof(double) * (size_t)(r > 0 ? r : 1));
    smoothing(r, theta, S);
    double *v_t = transpose(v, n, p);
    i64 nd = 0, iter = 0;
    int done = 0, status = 0;
    if (stat) {
        mul_rs(n, r, r, w, S, ws);
        double d = orc_kl_divergence(n, p, r, v, ws, h);
        dev[nd++] = d;
        if (st_should_stop(&st, 0, d) != 0) done = 1;
    }
    while (!done && iter < max_iter) {
        iter++;
        mul_rs(n, r, r, w, S, ws);
        double *ws_t = transpose(ws, n, r);
        col_sums(n, r, ws, sum_ws);
        div_update_h_inner(n, p, r, v_t, ws, ws_t, h, sum_ws, tmp_h);
        memcpy(h, tmp_h, sizeof(double) * (size_t)(r * p));
        free(ws_t);
        mul_rs(r, r, p, S, h, sh);
        div_update_w(n, p, r, v, w, sh, tmp_w);
        memcpy(w, tmp_w, sizeof(double) * (size_t)(n * r));
        col_rescale(n, r, w);
        if (stat) {
            mul_rs(n, r, r, w, S, ws);
            double d = orc_kl_divergence(n, p, r, v, ws, h);
            dev[nd++] = d;
            int rc = st_should_stop(&st, iter, d);
            if (rc < 0) {
                status = -2;
                break;
            }
            if (rc) break;
        }
    }
    *n_dev = nd;
    *n_iter = iter;
    free(S);
    free(ws);
    free(sh);
    free(tmp_h);
    free(tmp_w);
    free(sum_ws);
    free(v_t);
    return status;
}

/* euclidean_distance of V against W H + off 1^T (lib.rs:1688-1694,
 * :1745-1752): 0.5 * sum((V - WH - off)^2), j outer. */
double orc_euclidean_distance_offset(i64 n, i64 p, i64 r, const double *v, const double *w,
                                     const double *h, const double *off) {
    double s = 0.0;
    for (i64 j = 0; j < p; j++)
        for (i64 i = 0; i < n; i++) {
            double d = v[i * p + j] - (wh_at(p, r, w, h, i, j) + off[i]);
            s += d * d;
        }
    return 0.5 * s;
}

/*
 * orc_nmf_run_offset: nmf_run_offset, lib.rs:1650-1760.  off (n) holds the
 * starting offsets on entry (rowMeans(V) by default, computed by the caller)
 * and the result on exit.  Per iteration: the Frobenius H update with
 * W^T off added to its denominator (offset_update_h_inner :330-361), the W
 * update with off[i] rowSums(H)[j] added (offset_update_w_impl :398-450), then
 * off_i <- off_i max(rowSums(V)_i, eps) / (rowSums(W H + off)_i + eps).
 */
int orc_nmf_run_offset(i64 n, i64 p, i64 r, const double *v, double *w, double *h, double *off,
                       i64 max_iter, double eps, int stop, double stationary_th,
                       i64 check_interval, i64 check_niter, double *dev, i64 *n_dev,
                       i64 *n_iter, int nt) {
    set_threads(nt);
    stationary_t st = {check_interval, check_niter, stationary_th, -INFINITY, INFINITY, 0};
    const int stat = (stop == ORC_STOP_STATIONARY);
    const size_t rr = (size_t)(r * r > 0 ? r * r : 1);
    const size_t nr = (size_t)(n * r > 0 ? n * r : 1), rp = (size_t)(r * p > 0 ? r * p : 1);
    double *wtw = (double *)malloc(sizeof(double) * rr);
    double *hht = (double *)malloc(sizeof(double) * rr);
    double *addon = (double *)malloc(sizeof(double) * (size_t)(r > 0 ? r : 1));
    double *rsh = (double *)malloc(sizeof(double) * (size_t)(r > 0 ? r : 1));
    double *hp = (double *)malloc(sizeof(double) * rp);
    double *wp = (double *)malloc(sizeof(double) * nr);
    double *v_t = transpose(v, n, p);
    i64 nd = 0, iter = 0;
    int done = 0, status = 0;
    if (stat) {
        double d = orc_euclidean_distance_offset(n, p, r, v, w, h, off);
        dev[nd++] = d;
        if (st_should_stop(&st, 0, d) != 0) done = 1;
    }
    while (!done && iter < max_iter) {
        iter++;
        double *w_t = transpose(w, n, r);
        wtw_rev(n, r, w_t, wtw);
        for (i64 i = 0; i < r; i++) {
            double a = 0.0;
            for (i64 u = n - 1; u >= 0; u--) a += w_t[i * n + u] * off[u];
            addon[i] = a;
        }
#pragma omp parallel for schedule(static)
        for (i64 j = 0; j < p; j++)
            for (i64 i = 0; i < r; i++) {
                double numer = 0.0;
                for (i64 u = n - 1; u >= 0; u--) numer += w_t[i * n + u] * v_t[j * n + u];
                double den = 0.0;
                for (i64 l = r - 1; l >= 0; l--) den += wtw[i * r + l] * h[l * p + j];
                den += addon[i];
                double temp = h[i * p + j] * numer;
                hp[i * p + j] = (temp > eps ? temp : eps) / (den + eps);
            }
        memcpy(h, hp, sizeof(double) * (size_t)(r * p));
        free(w_t);
        for (i64 j = 0; j < r; j++)
            for (i64 i = 0; i < r; i++) {
                double a = 0.0;
                for (i64 u = p - 1; u >= 0; u--) a += h[j * p + u] * h[i * p + u];
                hht[i * r + j] = a;
            }
        for (i64 i = 0; i < r; i++) {
            double a = 0.0;
            for (i64 u = p - 1; u >= 0; u--) a += h[i * p + u];
            rsh[i] = a;
        }
#pragma omp parallel for schedule(static)
        for (i64 i = 0; i < n; i++)
            for (i64 j = 0; j < r; j++) {
                double numer = 0.0;
                for (i64 u = p - 1; u >= 0; u--) numer += v[i * p + u] * h[j * p + u];
                double den = 0.0;
                for (i64 l = r - 1; l >= 0; l--) den += w[i * r + l] * hht[l * r + j];
                den += off[i] * rsh[j];
                double temp = w[i * r + j] * numer;
                wp[i * r + j] = (temp < eps ? eps : temp) / (den + eps);
            }
        memcpy(w, wp, sizeof(double) * (size_t)(n * r));
#pragma omp parallel for schedule(static)
        for (i64 i = 0; i < n; i++) {
            double rs_v = 0.0, rs_whpo = 0.0;
            for (i64 j = 0; j < p; j++) {
                rs_v += v[i * p + j];
                rs_whpo += wh_at(p, r, w, h, i, j) + off[i];
            }
            const double num = rs_v > eps ? rs_v : eps;
            off[i] = off[i] * num / (rs_whpo + eps);
        }
        if (stat) {
            double d = orc_euclidean_distance_offset(n, p, r, v, w, h, off);
            dev[nd++] = d;
            int rc = st_should_stop(&st, iter, d);
            if (rc < 0) {
                status = -2;
                break;
            }
            if (rc) break;
        }
    }
    *n_dev = nd;
    *n_iter = iter;
    free(wtw);
    free(hht);
    free(addon);
    free(rsh);
    free(hp);
    free(wp);
    free(v_t);
    return status;
}

/* 0.5 sum ((V - W H) o S)^2, rows outer (lib.rs:962-975 / 1024-1035). */
double orc_weighted_distance(i64 n, i64 p, i64 r, const double *v, const double *weight,
                             const double *w, const double *h) {
    double s = 0.0;
    for (i64 u = 0; u < n; u++)
        for (i64 j = 0; j < p; j++) {
            const double d = (v[u * p + j] - wh_at(p, r, w, h, u, j)) * weight[u * p + j];
            s += d * d;
        }
    return 0.5 * s;
}

/* est o S for the current W, H (wh_dense then elementwise_mul, lib.rs:980-981). */
static void est_weighted(i64 n, i64 p, i64 r, const double *w, const double *h,
                         const double *weight, double *out) {
#pragma omp parallel for schedule(static)
    for (i64 u = 0; u < n; u++)
        for (i64 j = 0; j < p; j++) out[u * p + j] = wh_at(p, r, w, h, u, j) * weight[u * p + j];
}

/*
 * orc_nmf_run_lsnmf: nmf_run_lsnmf, lib.rs:945-1043 (weighted Frobenius).
 * Per iteration: H <- max(eps, H o W^T(V o S)) / (W^T((W H) o S) + eps), then
 * W <- max(eps, W o (V o S) H^T) / (((W H) o S) H^T + eps) with the new H.
 */
int orc_nmf_run_lsnmf(i64 n, i64 p, i64 r, const double *v, const double *weight, double *w,
                      double *h, i64 max_iter, double eps, int stop, double stationary_th,
                      i64 check_interval, i64 check_niter, double *dev, i64 *n_dev,
                      i64 *n_iter, int nt) {
    set_threads(nt);
    stationary_t st = {check_interval, check_niter, stationary_th, -INFINITY, INFINITY, 0};
    const int stat = (stop == ORC_STOP_STATIONARY);
    const size_t np = (size_t)(n * p > 0 ? n * p : 1);
    const size_t nr = (size_t)(n * r > 0 ? n * r : 1), rp = (size_t)(r * p > 0 ? r * p : 1);
    double *v_w = (double *)malloc(sizeof(double) * np);
    double *est_w = (double *)malloc(sizeof(double) * np);
    double *num = (double *)malloc(sizeof(double) * (rp > nr ? rp : nr));
    double *den = (double *)malloc(sizeof(double) * (rp > nr ? rp : nr));
    for (i64 t = 0; t < n * p; t++) v_w[t] = v[t] * weight[t];
    double *v_w_t = transpose(v_w, n, p);
    i64 nd = 0, iter = 0;
    int done = 0, status = 0;
    if (stat) {
        const double d = orc_weighted_distance(n, p, r, v, weight, w, h);
        dev[nd++] = d;
        if (st_should_stop(&st, 0, d) != 0) done = 1;
    }
    while (!done && iter < max_iter) {
        iter++;
        est_weighted(n, p, r, w, h, weight, est_w);
        double *est_w_t = transpose(est_w, n, p);
        double *w_t = transpose(w, n, r);
        compute_wtv(n, p, r, w_t, v_w_t, num);
        compute_wtv(n, p, r, w_t, est_w_t, den);
        for (i64 k = 0; k < r; k++)
            for (i64 u = 0; u < p; u++) {
                const double temp = h[k * p + u] * num[k * p + u];
                h[k * p + u] = (temp > eps ? temp : eps) / (den[k * p + u] + eps);
            }
        free(est_w_t);
        free(w_t);
        est_weighted(n, p, r, w, h, weight, est_w);
        compute_vht(n, p, r, v_w, h, num);
        compute_vht(n, p, r, est_w, h, den);
        for (i64 u = 0; u < n; u++)
            for (i64 k = 0; k < r; k++) {
                const double temp = w[u * r + k] * num[u * r + k];
                w[u * r + k] = (temp > eps ? temp : eps) / (den[u * r + k] + eps);
            }
        if (stat) {
            const double d = orc_weighted_distance(n, p, r, v, weight, w, h);
            dev[nd++] = d;
            int rc = st_should_stop(&st, iter, d);
            if (rc < 0) {
                status = -2;
                break;
            }
            if (rc) break;
        }
    }
    *n_dev = nd;
    *n_iter = iter;
    free(v_w);
    free(v_w_t);
    free(est_w);
    free(num);
    free(den);
    return status;
}

/* ------------------------------------------------------------------------ */
/* Kim-Park sparse NMF (snmf/r, snmf/l): ANLS with FCNNLS                    */
/* ------------------------------------------------------------------------ */

/* Cholesky factor in place (lower triangle of the m x m row-major a), in
 * the order of fcnnls.rs:19-41; 0 when a pivot is not positive. */
static int chol_inplace(double *a, int m) {
    for (int j = 0; j < m; j++) {
        double s = a[j * m + j];
        for (int q = 0; q < j; q++) s -= a[j * m + q] * a[j * m + q];
        if (s <= 0.0) return 0;
        const double l = sqrt(s);
        a[j * m + j] = l;
        for (int i = j + 1; i < m; i++) {
            double t = a[i * m + j];
            for (int q = 0; q < j; q++) t -= a[i * m + q] * a[j * m + q];
            a[i * m + j] = t / l;
        }
    }
    return 1;
}

/* L L^T x = b in place (fcnnls.rs:44-60). */
static void chol_solve(const double *l, int m, double *b) {
    for (int i = 0; i < m; i++) {
        double s = b[i];
        for (int q = 0; q < i; q++) s -= l[i * m + q] * b[q];
        b[i] = s / l[i * m + i];
    }
    for (int i = m - 1; i >= 0; i--) {
        double s = b[i];
        for (int q = i + 1; q < m; q++) s -= l[q * m + i] * b[q];
        b[i] = s / l[i * m + i];
    }
}

/* Solve a x = b (m x m), falling back as pseudoinv_solve does
 * (fcnnls.rs:62-90): while the Cholesky fails, add eps to the diagonal
 * (eps = 1e-12, then x10 each try, accumulating); zeros once eps > 1e6.
 * work holds 2 m^2 doubles. */
static void spd_solve(const double *a, int m, double *b, double *work) {
    double *f = work, *areg = work + m * m;
    memcpy(f, a, sizeof(double) * (size_t)(m * m));
    if (chol_inplace(f, m)) {
        chol_solve(f, m, b);
        return;
    }
    memcpy(areg, a, sizeof(double) * (size_t)(m * m));
    double eps = 1e-12;
    for (;;) {
        memcpy(f, areg, sizeof(double) * (size_t)(m * m));
        if (chol_inplace(f, m)) {
            chol_solve(f, m, b);
            return;
        }
        for (int i = 0; i < m; i++) areg[i * m + i] += eps;
        eps *= 10.0;
        if (eps > 1e6) {
            for (int i = 0; i < m; i++) b[i] = 0.0;
            return;
        }
    }
}

/* One column of cssls (fcnnls.rs:93-290): the least-squares solution on the
 * passive variables (pset, bit i = variable i), zero elsewhere.  ctc is
 * l x l; rhs_i = cta[i * cs + j * js]; k receives l values. */
static void cssls_col(int l, const double *ctc, const double *cta, i64 cs, i64 js, int j,
                      unsigned pset, double *k, double *work) {
    int act[32], m = 0;
    for (int i = 0; i < l; i++) {
        k[i] = 0.0;
        if (pset >> i & 1u) act[m++] = i;
    }
    if (m == 0) return;
    double *g = work, *b = work + 32 * 32, *w2 = b + 32;
    for (int a = 0; a < m; a++) {
        for (int c = 0; c < m; c++) g[a * m + c] = ctc[act[a] * l + act[c]];
        b[a] = cta[act[a] * cs + (i64)j * js];
    }
    spd_solve(g, m, b, w2);
    for (int a = 0; a < m; a++) k[act[a]] = b[a];
}

/*
 * orc_fcnnls: fcnnls (fcnnls.rs:297-470) on precomputed normal equations:
 * ctc (l x l, row-major), cta (l x P, element (i, j) at cta[i * cs + j * js]),
 * eps; K (l x P, element (i, j) at K[j * l + i]).  Restated step by step,
 * including its control flow: one iteration counter (cap 3 l) for all
 * columns; the inner loop's set of columns recomputed over all P columns as
 * "any value < eps" (which counts the zeros of inactive variables); a column
 * of that set without a passive variable below eps takes the step with
 * alpha = inf, as the reference does.  l <= 32.
 */
void orc_fcnnls(int l, i64 P, const double *ctc, const double *cta, i64 cs, i64 js, double eps,
                double *K) {
    const int max_iter = 3 * l;
    int iter = 0;
    unsigned *pset = (unsigned *)calloc((size_t)(P > 0 ? P : 1), sizeof(unsigned));
    unsigned char *fset = (unsigned char *)calloc((size_t)(P > 0 ? P : 1), 1);
    unsigned char *hset = (unsigned char *)calloc((size_t)(P > 0 ? P : 1), 1);
    double *D = (double *)malloc(sizeof(double) * (size_t)(P * l > 0 ? P * l : 1));
    double work[32 * 32 + 32 + 2 * 32 * 32];
    /* Unconstrained start: cssls with every variable passive. */
    const unsigned all = (l == 32) ? 0xffffffffu : ((1u << l) - 1u);
    i64 nf = 0;
    for (i64 j = 0; j < P; j++) {
        double *kj = K + j * l;
        cssls_col(l, ctc, cta, cs, js, (int)j, all, kj, work);
        unsigned ps = 0;
        for (int i = 0; i < l; i++) {
            if (kj[i] > 0.0) ps |= 1u << i;
            else kj[i] = 0.0;
        }
        pset[j] = ps;
        memcpy(D + j * l, kj, sizeof(double) * (size_t)l);
        fset[j] = (ps != all);
        nf += fset[j];
    }
    while (nf > 0) {
        i64 nh = 0;
        for (i64 j = 0; j < P; j++) {
            hset[j] = 0;
            if (!fset[j]) continue;
            cssls_col(l, ctc, cta, cs, js, (int)j, pset[j], K + j * l, work);
        }
        for (i64 j = 0; j < P; j++) {
            if (!fset[j]) continue;
            for (int i = 0; i < l; i++)
                if (K[j * l + i] < eps) {
                    hset[j] = 1;
                    break;
                }
            nh += hset[j];
        }
        while (nh > 0 && iter < max_iter) {
            iter++;
            int any_ij = 0;
            for (i64 j = 0; j < P && !any_ij; j++)
                if (hset[j])
                    for (int i = 0; i < l; i++)
                        if ((pset[j] >> i & 1u) && K[j * l + i] < eps) {
                            any_ij = 1;
                            break;
                        }
            if (!any_ij) break;
            for (i64 j = 0; j < P; j++) {
                if (!hset[j]) continue;
                double *dj = D + j * l;
                const double *kj = K + j * l;
                double amin = INFINITY;
                int imin = 0;
                for (int i = 0; i < l; i++) {
                    double a = INFINITY;
                    if ((pset[j] >> i & 1u) && kj[i] < eps) {
                        const double den = dj[i] - kj[i];
                        if (den != 0.0) a = dj[i] / den;
                    }
                    if (a < amin) {
                        amin = a;
                        imin = i;
                    }
                }
                for (int i = 0; i < l; i++) dj[i] -= amin * (dj[i] - kj[i]);
                dj[imin] = 0.0;
                pset[j] &= ~(1u << imin);
            }
            for (i64 j = 0; j < P; j++)
                if (hset[j]) cssls_col(l, ctc, cta, cs, js, (int)j, pset[j], K + j * l, work);
            nh = 0;
            for (i64 j = 0; j < P; j++) {
                hset[j] = 0;
                for (int i = 0; i < l; i++)
                    if (K[j * l + i] < eps) {
                        hset[j] = 1;
                        break;
                    }
                nh += hset[j];
            }
        }
        nf = 0;
        for (i64 j = 0; j < P; j++) {
            if (!fset[j]) continue;
            const double *kj = K + j * l;
            double best = -INFINITY;
            int ib = 0;
            for (int i = 0; i < l; i++) {
                if (pset[j] >> i & 1u) continue;
                double w = cta[i * cs + j * js];
                double s = 0.0;
                for (int q = 0; q < l; q++) s += ctc[i * l + q] * kj[q];
                w -= s;
                if (w > best) {
                    best = w;
                    ib = i;
                }
            }
            fset[j] = 0;
            if (best > eps) {
                pset[j] |= 1u << ib;
                memcpy(D + j * l, kj, sizeof(double) * (size_t)l);
                fset[j] = 1;
                nf++;
            }
        }
        if (iter >= max_iter) break;
    }
    free(pset);
    free(fset);
    free(hset);
    free(D);
}

/* Test hook: the Cholesky factor of an m x m matrix, in place; 0 on failure. */
int orc_cholesky(int m, double *a) { return chol_inplace(a, m); }

/* col_l2_normalize (lib.rs:1203-1213). */
static void col_l2_normalize(i64 m, i64 k, double *w) {
    for (i64 j = 0; j < k; j++) {
        double s = 0.0;
        for (i64 i = 0; i < m; i++) s += w[i * k + j] * w[i * k + j];
        const double nrm = sqrt(s);
        if (nrm > 0.0)
            for (i64 i = 0; i < m; i++) w[i * k + j] /= nrm;
    }
}

/*
 * orc_nmf_run_snmf: nmf_run_snmf_kim_park (lib.rs:1216-1320).  snmf/r
 * (is_left 0) works on A = V (n x p) with W (n x k), H (k x p); snmf/l on
 * A = V^T with the roles swapped.  Per iteration: H from FCNNLS on
 * [W; sqrt(beta) 1^T] against [A; 0], then W^T from FCNNLS on [H^T; eta I]
 * against [A^T; 0]; eta < 0 means max(A); beta floors at 1e-30.  Records
 * 0.5 ||A - W H||^2 every iteration (dev: max_iter doubles); runs max_iter
 * iterations.  w, h hold the user's W0 / H0 on entry and W / H on exit.
 */
int orc_nmf_run_snmf(int is_left, i64 n, i64 p, i64 k, const double *v, double *w, double *h,
                     i64 max_iter, double eta, double beta, double eps, double *dev, int nt) {
    set_threads(nt);
    if (k > 32) return -1;
    /* Internal problem: A (m x q), Wi (m x k), Hi (k x q). */
    const i64 m = is_left ? p : n, q = is_left ? n : p;
    double *A = is_left ? transpose(v, n, p) : (double *)malloc(sizeof(double) * (size_t)(n * p > 0 ? n * p : 1));
    if (!is_left) memcpy(A, v, sizeof(double) * (size_t)(n * p));
    double *Wi = is_left ? transpose(h, k, p) : (double *)malloc(sizeof(double) * (size_t)(m * k > 0 ? m * k : 1));
    double *Hi = is_left ? transpose(w, n, k) : (double *)malloc(sizeof(double) * (size_t)(k * q > 0 ? k * q : 1));
    if (!is_left) {
        memcpy(Wi, w, sizeof(double) * (size_t)(m * k));
        memcpy(Hi, h, sizeof(double) * (size_t)(k * q));
    }
    double eta_eff = eta;
    if (eta < 0.0) {
        eta_eff = 0.0;
        for (i64 t = 0; t < m * q; t++) eta_eff = (A[t] > eta_eff) ? A[t] : eta_eff;
    }
    const double beta_eff = beta > 1e-30 ? beta : 1e-30;
    const double sb = sqrt(beta_eff);
    col_l2_normalize(m, k, Wi);
    double ctc[32 * 32];
    double *cta = (double *)malloc(sizeof(double) * (size_t)(k * (m > q ? m : q) + 1));
    double *K = (double *)malloc(sizeof(double) * (size_t)(k * (m > q ? m : q) + 1));
    for (i64 it = 0; it < max_iter; it++) {
        /* H: x = [Wi; sb 1^T] ((m + 1) x k), y = [A; 0]. */
        for (i64 a = 0; a < k; a++)
            for (i64 c = 0; c < k; c++) {
                double s = 0.0;
                for (i64 r = 0; r < m; r++) s += Wi[r * k + a] * Wi[r * k + c];
                s += sb * sb;
                ctc[a * k + c] = s;
            }
#pragma omp parallel for schedule(static)
        for (i64 a = 0; a < k; a++)
            for (i64 j = 0; j < q; j++) {
                double s = 0.0;
                for (i64 r = 0; r < m; r++) s += Wi[r * k + a] * A[r * q + j];
                cta[a * q + j] = s;
            }
        orc_fcnnls((int)k, q, ctc, cta, q, 1, eps, K);
        for (i64 a = 0; a < k; a++)
            for (i64 j = 0; j < q; j++) Hi[a * q + j] = K[j * k + a];
        /* W: x = [Hi^T; eta I] ((q + k) x k), y = [A^T; 0]. */
        for (i64 a = 0; a < k; a++)
            for (i64 c = 0; c < k; c++) {
                double s = 0.0;
                for (i64 r = 0; r < q; r++) s += Hi[a * q + r] * Hi[c * q + r];
                if (a == c) s += eta_eff * eta_eff;
                ctc[a * k + c] = s;
            }
#pragma omp parallel for schedule(static)
        for (i64 a = 0; a < k; a++)
            for (i64 i = 0; i < m; i++) {
                double s = 0.0;
                for (i64 r = 0; r < q; r++) s += Hi[a * q + r] * A[i * q + r];
                cta[a * m + i] = s;
            }
        orc_fcnnls((int)k, m, ctc, cta, m, 1, eps, K);
        for (i64 i = 0; i < m; i++)
            for (i64 a = 0; a < k; a++) Wi[i * k + a] = K[i * k + a];
        double s = 0.0;
        for (i64 i = 0; i < m; i++)
            for (i64 j = 0; j < q; j++) {
                double r = 0.0;
                for (i64 a = 0; a < k; a++) r += Wi[i * k + a] * Hi[a * q + j];
                const double d = A[i * q + j] - r;
                s += d * d;
            }
        dev[it] = 0.5 * s;
    }
    if (is_left) {  /* user W = Hi^T (n x k), user H = Wi^T (k x p) */
        for (i64 i = 0; i < n; i++)
            for (i64 a = 0; a < k; a++) w[i * k + a] = Hi[a * n + i];
        for (i64 a = 0; a < k; a++)
            for (i64 j = 0; j < p; j++) h[a * p + j] = Wi[j * k + a];
    } else {
        memcpy(w, Wi, sizeof(double) * (size_t)(n * k));
        memcpy(h, Hi, sizeof(double) * (size_t)(k * p));
    }
    free(A);
    free(Wi);
    free(Hi);
    free(cta);
    free(K);
    return 0;
}

/* Build identification so the Python side can tell a stale build apart. */
int orc_version(void) { return 4; }

// fcnnls.cuh -- the FCNNLS solves of the Kim-Park sparse NMF (snmf/r,
// snmf/l; nmf_run_snmf_kim_park lib.rs:1216-1320 over fcnnls.rs:297-470),
// one thread a column.
//
// Each column j solves min ||y_j - X k_j|| s.t. k_j >= 0 from the normal
// equations shared by all columns: ctc (l x l, l <= 32) and its right-hand
// side cta_j (element i at cta[i * cs + j * js]).  The state of a column is
// its solution K (l values), the step vector D, the passive set (bit i =
// variable i) and two flags (F: in the outer set, H: in the inner set).
// The kernels are the steps of fcnnls.rs restated one for one; the host runs
// its loops, with the one iteration counter the reference keeps for all
// columns and its tests for empty sets (a device counter each).
#pragma once

#include <cmath>
#include <cstdint>

#include "kernels.cuh"

namespace nmfcu {

constexpr int kFcMax = 32;  // largest rank

// Cholesky factor of the m x m row-major a, in place (fcnnls.rs:19-41).
__device__ inline bool fc_chol(double *a, int m) {
    for (int j = 0; j < m; j++) {
        double s = a[j * m + j];
        for (int q = 0; q < j; q++) s -= a[j * m + q] * a[j * m + q];
        if (s <= 0.0) return false;
        const double l = sqrt(s);
        a[j * m + j] = l;
        for (int i = j + 1; i < m; i++) {
            double t = a[i * m + j];
            for (int q = 0; q < j; q++) t -= a[i * m + q] * a[j * m + q];
            a[i * m + j] = t / l;
        }
    }
    return true;
}
__device__ inline void fc_chol_solve(const double *l, int m, double *b) {
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

// The least-squares solution of column j on its passive variables, zero
// elsewhere (cssls, fcnnls.rs:93-290): the passive sub-Gram's Cholesky, or,
// when that fails, the regularised retries of pseudoinv_solve
// (fcnnls.rs:62-90: eps = 1e-12 added to the diagonal, x10 a retry,
// accumulating; zeros once eps > 1e6).
__device__ inline void fc_cssls(int l, const double *__restrict__ ctc,
                                const double *__restrict__ cta, int64_t cs, int64_t js, int64_t j,
                                unsigned pset, double *k) {
    int act[kFcMax];
    int m = 0;
    for (int i = 0; i < l; i++) {
        k[i] = 0.0;
        if (pset >> i & 1u) act[m++] = i;
    }
    if (m == 0) return;
    // The (regularised) sub-Gram is the passive rows and columns of ctc with
    // the diagonal dreg; each try rebuilds it in f and factors it in place
    // (one m x m array a thread).
    double f[kFcMax * kFcMax], b[kFcMax], rhs[kFcMax], dreg[kFcMax];
    for (int a = 0; a < m; a++) {
        rhs[a] = cta[act[a] * cs + j * js];
        dreg[a] = ctc[act[a] * l + act[a]];
    }
    double eps = 1e-12;
    bool first = true;
    for (int tries = 0; tries < 64; tries++) {
        for (int a = 0; a < m; a++)
            for (int c = 0; c < m; c++)
                f[a * m + c] = (a == c) ? dreg[a] : ctc[act[a] * l + act[c]];
        if (fc_chol(f, m)) {
            for (int a = 0; a < m; a++) b[a] = rhs[a];
            fc_chol_solve(f, m, b);
            for (int a = 0; a < m; a++) k[act[a]] = b[a];
            return;
        }
        if (!first) {
            for (int a = 0; a < m; a++) dreg[a] += eps;
            eps *= 10.0;
            if (eps > 1e6) return;  // zeros
        }
        first = false;
    }
}

struct FcState {
    double *K;         // P x l (column j's values at K[j * l + i])
    double *D;         // P x l
    unsigned *pset;    // P
    uint8_t *fflag;    // P
    uint8_t *hflag;    // P
    int *count;        // a device counter
};

// Start: all variables passive, then K > 0 passive (fcnnls.rs:316-341).
__global__ void fc_start(int l, int64_t P, const double *__restrict__ ctc,
                         const double *__restrict__ cta, int64_t cs, int64_t js, FcState s) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= P) return;
    const unsigned all = (l == 32) ? 0xffffffffu : ((1u << l) - 1u);
    double *k = s.K + j * l;
    fc_cssls(l, ctc, cta, cs, js, j, all, k);
    unsigned ps = 0;
    for (int i = 0; i < l; i++) {
        if (k[i] > 0.0) ps |= 1u << i;
        else k[i] = 0.0;
        s.D[j * l + i] = k[i];
    }
    s.pset[j] = ps;
    s.fflag[j] = (ps != all);
    if (ps != all) atomicAdd(s.count, 1);
}

// cssls on the columns whose flag (F or H) is set.
__global__ void fc_solve(int l, int64_t P, const double *__restrict__ ctc,
                         const double *__restrict__ cta, int64_t cs, int64_t js, FcState s,
                         const uint8_t *__restrict__ flag) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= P || !flag[j]) return;
    fc_cssls(l, ctc, cta, cs, js, j, s.pset[j], s.K + j * l);
}

// H = F columns with a value below eps (from_fset = 1), or all columns with
// a value below eps (fcnnls.rs:343-348 and 414-416); counts H.
__global__ void fc_hset(int l, int64_t P, double eps, FcState s, int from_fset) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= P) return;
    uint8_t h = 0;
    if (!from_fset || s.fflag[j]) {
        const double *k = s.K + j * l;
        for (int i = 0; i < l; i++)
            if (k[i] < eps) {
                h = 1;
                break;
            }
    }
    s.hflag[j] = h;
    if (h) atomicAdd(s.count, 1);
}

// Counts the H columns with a passive variable below eps (fcnnls.rs:358-367).
__global__ void fc_any_ij(int l, int64_t P, double eps, FcState s) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= P || !s.hflag[j]) return;
    const double *k = s.K + j * l;
    for (int i = 0; i < l; i++)
        if ((s.pset[j] >> i & 1u) && k[i] < eps) {
            atomicAdd(s.count, 1);
            return;
        }
}

// The inner step on the H columns (fcnnls.rs:368-404): the smallest step
// alpha over the passive variables below eps (inf when there is none, as in
// the reference), D <- D - alpha (D - K), and that variable leaves the set.
__global__ void fc_step(int l, int64_t P, double eps, FcState s) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= P || !s.hflag[j]) return;
    double *d = s.D + j * l;
    const double *k = s.K + j * l;
    const unsigned ps = s.pset[j];
    double amin = INFINITY;
    int imin = 0;
    for (int i = 0; i < l; i++) {
        double a = INFINITY;
        if ((ps >> i & 1u) && k[i] < eps) {
            const double den = d[i] - k[i];
            if (den != 0.0) a = d[i] / den;
        }
        if (a < amin) {
            amin = a;
            imin = i;
        }
    }
    for (int i = 0; i < l; i++) d[i] -= amin * (d[i] - k[i]);
    d[imin] = 0.0;
    s.pset[j] = ps & ~(1u << imin);
}

// The outer step's end on the F columns (fcnnls.rs:419-444): the largest
// gradient cta - ctc K over the active variables; above eps it becomes
// passive, D <- K, and the column stays in F.  Counts the new F.
__global__ void fc_tail(int l, int64_t P, const double *__restrict__ ctc,
                        const double *__restrict__ cta, int64_t cs, int64_t js, double eps,
                        FcState s) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= P || !s.fflag[j]) return;
    const double *k = s.K + j * l;
    const unsigned ps = s.pset[j];
    double best = -INFINITY;
    int ib = 0;
    for (int i = 0; i < l; i++) {
        if (ps >> i & 1u) continue;
        double sum = 0.0;
        for (int q = 0; q < l; q++) sum += ctc[i * l + q] * k[q];
        const double w = cta[i * cs + j * js] - sum;
        if (w > best) {
            best = w;
            ib = i;
        }
    }
    if (best > eps) {
        s.pset[j] = ps | (1u << ib);
        for (int i = 0; i < l; i++) s.D[j * l + i] = k[i];
        s.fflag[j] = 1;
        atomicAdd(s.count, 1);
    } else {
        s.fflag[j] = 0;
    }
}

// ctc (l x l) = G (RP x RP, the Gram) + add_all everywhere + add_diag on the
// diagonal: [W; sqrt(beta) 1^T]^T [W; sqrt(beta) 1^T] (add_all = beta') or
// [H^T; eta I]^T [H^T; eta I] (add_diag = eta^2).
__global__ void fc_normal(const double *__restrict__ G, int RP, int l, double add_all,
                          double add_diag, double *__restrict__ ctc) {
    const int t = threadIdx.x;
    if (t >= l * l) return;
    const int a = t / l, c = t - a * l;
    double v = G[a * RP + c] + add_all;
    if (a == c) v += add_diag;
    ctc[t] = v;
}

// K (P x l) -> the factor: H rows (l x P, pitch P; to_rows = 1) or W rows
// (P x RP; to_rows = 0).
__global__ void fc_scatter(const double *__restrict__ K, int l, int64_t P, int RP, int to_rows,
                           double *__restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P * l) return;
    const int64_t j = t / l;
    const int i = (int)(t - j * l);
    if (to_rows)
        out[(int64_t)i * P + j] = K[t];
    else
        out[j * RP + i] = K[t];
}

// L2-normalise the l columns of X (rows x RP) (col_l2_normalize,
// lib.rs:1203-1213), or the l rows of X (l x cols, pitch cols) when rows_mode.
__global__ void fc_normalize(double *__restrict__ X, int64_t len, int l, int RP, int rows_mode) {
    const int c = blockIdx.x;
    if (c >= l) return;
    __shared__ double red[256];
    double s = 0.0;
    for (int64_t t = threadIdx.x; t < len; t += 256) {
        const double x = rows_mode ? X[(int64_t)c * len + t] : X[t * RP + c];
        s += x * x;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const double nrm = sqrt(red[0]);
    if (!(nrm > 0.0)) return;
    for (int64_t t = threadIdx.x; t < len; t += 256) {
        double &x = rows_mode ? X[(int64_t)c * len + t] : X[t * RP + c];
        x /= nrm;
    }
}

// max(0, max of V) over the n x p matrix (pitch ld), into out (one block).
__global__ void fc_vmax(const double *__restrict__ V, int64_t ld, int n, int p,
                        double *__restrict__ out) {
    __shared__ double red[256];
    double m = 0.0;
    for (int64_t t = threadIdx.x; t < (int64_t)n * p; t += 256) {
        const int64_t i = t / p;
        const double v = V[i * ld + (t - i * p)];
        m = (v > m) ? v : m;
    }
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
            red[threadIdx.x] = red[threadIdx.x + o] > red[threadIdx.x] ? red[threadIdx.x + o]
                                                                         : red[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0];
}

}  // namespace nmfcu

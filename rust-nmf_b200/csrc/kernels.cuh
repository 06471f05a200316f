// kernels.cuh -- device code of the B200 NMF engine.
//
// One iteration of every built method is two streaming passes over V plus
// small O(r^2 (n + p)) work:
//
//   H step  (reduce over the n rows of V, one output column per thread):
//     plain : A[k][j] = sum_u W[u][k] V[u][j]                 lee, hals, dnmf
//     ratio : A[k][j] = sum_u W[u][k] V[u][j] / (W H)[u][j]    brunet (WH never stored)
//   W step  (reduce over the p columns of V, one output row per thread):
//     plain : B[i][k] = sum_j V[i][j] H'[k][j]
//     ratio : B[i][k] = sum_j H'[k][j] V[i][j] / (W H')[i][j]
//
// followed by a per-column (H) / per-row (W) epilogue that applies the
// method's update exactly as the reference writes it (multiplicative update
// or a Gauss-Seidel sweep).  Partial sums are written per split and summed
// in a fixed order, so every result is bit-reproducible run to run.
//
// Layouts (device): V row-major n x p with leading dimension ldv; W n x RP
// and H RP x p f64 with the rank padded to the compile-time bucket RP by
// zero columns / rows (a zero pad contributes exact zeros to every sum).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nmfcu {

// Method ids, same values as include/nmfcu.h.
enum : int { M_BRUNET = 0, M_LEE = 1, M_OFFSET = 2, M_NSNMF = 3, M_HALS = 4, M_EHALS = 5,
             M_DNMF = 6, M_LSNMF = 7 };
// Not a method: the epilogues store the contraction itself (the products of
// the randomized range finder behind the NNDSVD start).
constexpr int M_PRODUCT = 100;

// Device-side state of the stationary stop (lib.rs:1336-1401) and of the
// run: written by single-thread kernels, read by every kernel of an
// iteration so that the iterations after a stop do no work.
struct RunState {
    double last_max;
    double last_min;
    long long n_collected;
    long long n_iter;  // iteration at which the stop fired
    int stopped;       // 1 once the loop has stopped
    int error;         // 1: `iter % check_interval` with check_interval == 0
    int timeout;       // a bounded mbarrier wait gave up (stream.cuh codes)
    unsigned gram_ticket;  // blocks of the running Gram launch that are done
};

// Fixed constants of the streaming kernels.
constexpr int kThreads = 256;
constexpr int kWarps = 8;

__device__ __forceinline__ bool run_stopped(const RunState *st) {
    return st != nullptr && st->stopped != 0;
}

// ---------------------------------------------------------------------------
// Arithmetic helpers
// ---------------------------------------------------------------------------

// x / y for the ratio V / (WH), y != 0.  f64: x (1 / y) with the reciprocal
// from the hardware approximation (rcp.approx.ftz.f64) refined by two
// Newton-Raphson steps r <- r + r (1 - y r), each of which doubles the
// correct bits, so the quotient is within about an ulp of the IEEE one (the
// tests hold the loop to 1e-10 of the oracle's IEEE divisions); |y| outside
// [2^-1000, 2^1000] and NaN take the IEEE division.  f32: the fast
// reciprocal-multiply form (the FP32 form is tolerance-checked).
__device__ __forceinline__ double ratio_div(double x, double y) {
    const double a = fabs(y);
    if (!(a > 0x1p-1000 && a < 0x1p1000)) return x / y;
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(y));
    double e = fma(-y, r, 1.0);
    r = fma(r, e, r);
    e = fma(-y, r, 1.0);
    r = fma(r, e, r);
    return x * r;
}
__device__ __forceinline__ float ratio_div(float x, float y) { return __fdividef(x, y); }

// Epilogue arithmetic without FMA contraction, so that the update formulas
// round exactly as the reference's scalar Rust code does.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// ---------------------------------------------------------------------------
// H-step contraction: reduce over rows [u0, u1) for 32 columns per CTA.
// grid (ceil(p/32), S), block (32, 8).  part is [S][RP][p] f64.
// ---------------------------------------------------------------------------
template <typename TV, typename TA, int RP, bool RATIO>
__global__ void __launch_bounds__(kThreads)
    hstep_contract(const TV *__restrict__ V, int64_t ldv, int n, int p,
                   const double *__restrict__ W, const double *__restrict__ H,
                   int rows_per_split, double *__restrict__ part, const RunState *st) {
    if (run_stopped(st)) return;
    // Rows of W staged per chunk; in f32 the per-chunk f32 sums are flushed
    // into f64 accumulators once per chunk.
    constexpr int CH = (sizeof(TA) == 8) ? 64 : 256;
    constexpr int SBUF = (CH * RP * (int)sizeof(TA) > 4 * RP * 32 * 8)
                             ? CH * RP
                             : (4 * RP * 32 * 8) / (int)sizeof(TA);
    __shared__ __align__(16) TA sbuf[SBUF];

    const int lane = threadIdx.x;
    const int warp = threadIdx.y;
    const int tid = warp * 32 + lane;
    const int j = blockIdx.x * 32 + lane;
    const bool colok = j < p;
    const int u0 = blockIdx.y * rows_per_split;
    const int u1 = min(n, u0 + rows_per_split);

    double acc[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) acc[k] = 0.0;
    TA hcol[RATIO ? RP : 1];
    if constexpr (RATIO) {
#pragma unroll
        for (int k = 0; k < RP; k++) hcol[k] = colok ? (TA)H[(int64_t)k * p + j] : (TA)0;
    }

    // f64: accf is the accumulator.  f32: accf holds one chunk's sums and is
    // flushed into the f64 acc after every chunk.
    TA accf[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) accf[k] = (TA)0;

    for (int base = u0; base < u1; base += CH) {
        const int rows = min(CH, u1 - base);
        __syncthreads();
        const double *wsrc = W + (int64_t)base * RP;
        for (int t = tid; t < CH * RP; t += kThreads)
            sbuf[t] = (t < rows * RP) ? (TA)wsrc[t] : (TA)0;
        __syncthreads();

        // Each warp takes rows warp, warp + 8, ...; 4 rows per step so four
        // independent V loads are in flight before the arithmetic.
        for (int rr = warp; rr < rows; rr += 4 * kWarps) {
            TA v[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int row = rr + q * kWarps;
                v[q] = (colok && row < rows) ? (TA)V[(int64_t)(base + row) * ldv + j] : (TA)0;
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int row = rr + q * kWarps;
                if (row < rows) {
                    const TA *wr = sbuf + row * RP;
                    if constexpr (RATIO) {
                        TA wh = (TA)0;
#pragma unroll
                        for (int k = 0; k < RP; k++) wh = fma(wr[k], hcol[k], wh);
                        const TA qv = (wh != (TA)0) ? ratio_div(v[q], wh) : (TA)0;
#pragma unroll
                        for (int k = 0; k < RP; k++) accf[k] = fma(wr[k], qv, accf[k]);
                    } else {
#pragma unroll
                        for (int k = 0; k < RP; k++) accf[k] = fma(wr[k], v[q], accf[k]);
                    }
                }
            }
        }
        if constexpr (sizeof(TA) == 4) {
#pragma unroll
            for (int k = 0; k < RP; k++) {
                acc[k] += (double)accf[k];
                accf[k] = (TA)0;
            }
        }
    }
    if constexpr (sizeof(TA) == 8) {
#pragma unroll
        for (int k = 0; k < RP; k++) acc[k] = (double)accf[k];
    }

    // CTA reduction over the 8 warps in a fixed tree order (deterministic).
    // sbuf holds CH * RP >= 4 * 32 * RP * 8 / sizeof(TA) elements, enough for
    // 4 * 32 * RP doubles in both precisions.
    double *red = reinterpret_cast<double *>(sbuf);
#pragma unroll
    for (int level = 4; level >= 1; level >>= 1) {
        __syncthreads();
        if (warp >= level && warp < 2 * level) {
#pragma unroll
            for (int k = 0; k < RP; k++) red[((warp - level) * RP + k) * 32 + lane] = acc[k];
        }
        __syncthreads();
        if (warp < level) {
#pragma unroll
            for (int k = 0; k < RP; k++) acc[k] += red[(warp * RP + k) * 32 + lane];
        }
    }
    if (warp == 0 && colok) {
        double *dst = part + (int64_t)blockIdx.y * RP * p + j;
#pragma unroll
        for (int k = 0; k < RP; k++) dst[(int64_t)k * p] = acc[k];
    }
}

// ---------------------------------------------------------------------------
// Row-owned V pass: one thread per row of V, V tiles staged through shared
// memory so that a warp's global loads are row-contiguous.
//   MODE 0 (plain)  : part[i][k] += V[i][j] H[k][j]
//   MODE 1 (ratio)  : part[i][k] += H[k][j] V[i][j] / (W H)[i][j]
//   MODE 2 (KL)     : obj += kl term of (V, W H)   (lib.rs:1418-1427)
//   MODE 3 (Frob)   : obj += (V - W H)^2           (lib.rs:1440-1441)
// grid (ceil(n/256), S2), block 256.  part is [S2][n][RP] (modes 0, 1);
// obj is one f64 per CTA (modes 2, 3), indexed blockIdx.y * gridDim.x + x.
// ---------------------------------------------------------------------------
template <typename TV, typename TA, int RP, int MODE>
__global__ void __launch_bounds__(kThreads)
    rowpass(const TV *__restrict__ V, int64_t ldv, int n, int p, const double *__restrict__ W,
            const double *__restrict__ H, int cols_per_split, double *__restrict__ part,
            double *__restrict__ obj, const RunState *st, const double *__restrict__ roff = nullptr) {
    if (run_stopped(st)) return;
    constexpr int TC = (sizeof(TV) == 8) ? 16 : 32;  // 128 B of a V row per tile
    __shared__ TV sV[kThreads][TC + 1];
    __shared__ __align__(16) TA sH[TC][RP];

    const int tid = threadIdx.x;
    const int row0 = blockIdx.x * kThreads;
    const int i = row0 + tid;
    const bool rowok = i < n;
    const int c0 = blockIdx.y * cols_per_split;
    const int c1 = min(p, c0 + cols_per_split);

    constexpr bool NEED_W = (MODE != 0);
    TA wrow[NEED_W ? RP : 1];
    if constexpr (NEED_W) {
#pragma unroll
        for (int k = 0; k < RP; k++) wrow[k] = rowok ? (TA)W[(int64_t)i * RP + k] : (TA)0;
    }
    double acc[MODE <= 1 ? RP : 1];
#pragma unroll
    for (int k = 0; k < (MODE <= 1 ? RP : 1); k++) acc[k] = 0.0;
    double objacc = 0.0;
    // offset method: the row's offset is part of the estimate (lib.rs:1746-1752)
    const double ro = (MODE == 3 && roff != nullptr && rowok) ? roff[i] : 0.0;

    constexpr int NA = (MODE <= 1) ? RP : 1;
    TA accf[NA];  // f64: the accumulator; f32: one tile's sums
#pragma unroll
    for (int k = 0; k < NA; k++) accf[k] = (TA)0;

    for (int c = c0; c < c1; c += TC) {
        __syncthreads();
        for (int e = tid; e < kThreads * TC; e += kThreads) {
            const int rr = e / TC, cc = e - rr * TC;
            const int gi = row0 + rr, gc = c + cc;
            sV[rr][cc] = (gi < n && gc < c1) ? V[(int64_t)gi * ldv + gc] : (TV)0;
        }
        for (int e = tid; e < TC * RP; e += kThreads) {
            const int k = e / TC, cc = e - k * TC;
            const int gc = c + cc;
            sH[cc][k] = (gc < c1) ? (TA)H[(int64_t)k * p + gc] : (TA)0;
        }
        __syncthreads();
        const int ncols = min(TC, c1 - c);
#pragma unroll 4
        for (int cc = 0; cc < ncols; cc++) {
            const TA v = (TA)sV[tid][cc];
            const TA *hr = sH[cc];
            if constexpr (MODE == 0) {
#pragma unroll
                for (int k = 0; k < RP; k++) accf[k] = fma(v, hr[k], accf[k]);
            } else {
                TA wh = (TA)0;
#pragma unroll
                for (int k = 0; k < RP; k++) wh = fma(wrow[k], hr[k], wh);
                if constexpr (MODE == 1) {
                    const TA q = (wh != (TA)0) ? ratio_div(v, wh) : (TA)0;
#pragma unroll
                    for (int k = 0; k < RP; k++) accf[k] = fma(hr[k], q, accf[k]);
                } else if constexpr (MODE == 2) {
                    const double vv = (double)v, ww = (double)wh;
                    if (vv > 0.0) {
                        if (ww > 0.0) objacc += vv * log(vv / ww) - vv + ww;
                    } else {
                        objacc += ww;
                    }
                } else {
                    const double d = (double)v - ((double)wh + ro);
                    objacc += d * d;
                }
            }
        }
        if constexpr (MODE <= 1 && sizeof(TA) == 4) {
#pragma unroll
            for (int k = 0; k < RP; k++) {
                acc[k] += (double)accf[k];
                accf[k] = (TA)0;
            }
        }
    }

    if constexpr (MODE <= 1) {
        if constexpr (sizeof(TA) == 8) {
#pragma unroll
            for (int k = 0; k < RP; k++) acc[k] = (double)accf[k];
        }
        if (rowok) {
            double *dst = part + ((int64_t)blockIdx.y * n + i) * RP;
#pragma unroll
            for (int k = 0; k < RP; k++) dst[k] = acc[k];
        }
    } else {
        // Block reduction of the objective in a fixed order.
        __shared__ double red[kThreads];
        red[tid] = rowok ? objacc : 0.0;
        __syncthreads();
        for (int s = kThreads / 2; s > 0; s >>= 1) {
            if (tid < s) red[tid] += red[tid + s];
            __syncthreads();
        }
        if (tid == 0) obj[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = red[0];
    }
}

// ---------------------------------------------------------------------------
// nsNMF and offset helpers
// ---------------------------------------------------------------------------
// Smoothing matrix entry S[k][j] = (1 - theta) I + (theta / r) (lib.rs:458-466).
__device__ __forceinline__ double smooth_at(int k, int j, int r, double theta) {
    const double off = theta / (double)r;
    return (k == j) ? (1.0 - theta) + off : off;
}
// out = X S for X (rows x RP, row-major; columns >= r zero), forward k
// (W S of nmf_run_nsnmf, lib.rs:1811).
template <int RP>
__global__ void __launch_bounds__(kThreads)
    ns_right_s(const double *__restrict__ X, int rows, int r, double theta,
               double *__restrict__ out, const RunState *st) {
    if (run_stopped(st)) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= rows) return;
    double x[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) x[k] = X[(size_t)i * RP + k];
#pragma unroll
    for (int j = 0; j < RP; j++) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < RP; k++)
            if (k < r && j < r) acc = add(acc, mul(x[k], smooth_at(k, j, r, theta)));
        out[(size_t)i * RP + j] = acc;
    }
}
// out = S H for H (RP x p; rows >= r zero), forward l (S H, lib.rs:1819).
template <int RP>
__global__ void __launch_bounds__(kThreads)
    ns_left_s(const double *__restrict__ H, int p, int r, double theta, double *__restrict__ out,
              const RunState *st) {
    if (run_stopped(st)) return;
    const int j = blockIdx.x * kThreads + threadIdx.x;
    if (j >= p) return;
    double h[RP];
#pragma unroll
    for (int l = 0; l < RP; l++) h[l] = H[(size_t)l * p + j];
#pragma unroll
    for (int k = 0; k < RP; k++) {
        double acc = 0.0;
#pragma unroll
        for (int l = 0; l < RP; l++)
            if (k < r && l < r) acc = add(acc, mul(smooth_at(k, l, r, theta), h[l]));
        out[(size_t)k * p + j] = acc;
    }
}
// addon[k] = sum_u W[u][k] off[u] (den_addon, lib.rs:1705-1709); one block a
// component, a fixed-order tree over the rows.
template <int RP>
__global__ void __launch_bounds__(kThreads)
    off_addon(const double *__restrict__ W, int n, int r, const double *__restrict__ off,
              double *__restrict__ addon, const RunState *st) {
    if (run_stopped(st)) return;
    const int k = blockIdx.x;
    __shared__ double red[kThreads];
    double acc = 0.0;
    if (k < r)
        for (int u = threadIdx.x; u < n; u += kThreads) acc = add(acc, mul(W[(size_t)u * RP + k], off[u]));
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) addon[k] = (k < r) ? red[0] : 0.0;
}
// lsNMF objective partials (lib.rs:1024-1035): sum_ij (Vs_ij - (W H)_ij S_ij)^2
// with Vs = V o S precomputed, i.e. ((V - W H) o S)^2.  Block b takes rows
// b, b + nblocks, ... one warp a row (lanes over columns in a fixed order, a
// xor butterfly), and writes its sum to part[b].
template <int RP>
__global__ void __launch_bounds__(kThreads)
    ls_objective(const double *__restrict__ Vs, const double *__restrict__ S, int64_t ld, int n,
                 int p, const double *__restrict__ W, const double *__restrict__ H,
                 double *__restrict__ part, const RunState *st) {
    if (run_stopped(st)) return;
    constexpr int kWarps = kThreads / 32;
    __shared__ double red[kWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int i = blockIdx.x * kWarps + warp; i < n; i += gridDim.x * kWarps) {
        double w[RP];
#pragma unroll
        for (int k = 0; k < RP; k++) w[k] = W[(size_t)i * RP + k];
        for (int j = lane; j < p; j += 32) {
            double wh = 0.0;
#pragma unroll
            for (int k = 0; k < RP; k++) wh = fma(w[k], H[(size_t)k * p + j], wh);
            const double d = Vs[(size_t)i * ld + j] - wh * S[(size_t)i * ld + j];
            acc = fma(d, d, acc);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < kWarps; q++) s += red[q];
        part[blockIdx.x] = s;
    }
}
// Vs <- V o S in place (the weighted target of lsNMF, lib.rs:961).
static __global__ void mul_weight(double *__restrict__ V, const double *__restrict__ S,
                                  int64_t ld, int n, int p) {
    const int64_t total = (int64_t)n * p;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / p, at = i * ld + (t - i * p);
        V[at] = mul(V[at], S[at]);
    }
}

// E-HALS extrapolation (nmf_run_ehals, lib.rs:755-767) of the first `cols`
// entries of each of `rows` rows (leading dimension ld):
//   x <- max(eps, x + beta (x - prev)),  prev <- the old x.
static __global__ void ehals_extrapolate(double *__restrict__ X, double *__restrict__ prev,
                                         int64_t rows, int ld, int cols, double beta, double eps,
                                         const RunState *st) {
    if (run_stopped(st)) return;
    const int64_t total = rows * cols;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / cols;
        const int64_t at = i * ld + (t - i * cols);
        const double x = X[at];
        const double ext = add(x, mul(beta, sub(x, prev[at])));
        X[at] = ext > eps ? ext : eps;
        prev[at] = x;
    }
}

// Row sums of V (one warp a row, fixed-order lanes + butterfly).
static __global__ void __launch_bounds__(kThreads)
    v_row_sums(const double *__restrict__ V, int64_t ldv, int n, int p, double *__restrict__ out) {
    const int i = (int)(((size_t)blockIdx.x * kThreads + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    double acc = 0.0;
    for (int j = lane; j < p; j += 32) acc += V[(size_t)i * ldv + j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[i] = acc;
}
// Default offset: rowMeans(V) (lib.rs:1667-1679).
static __global__ void off_init(const double *__restrict__ rsv, int n, int p,
                                double *__restrict__ off) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) off[i] = rsv[i] / (double)p;
}
// off_i <- off_i max(rowSums(V)_i, eps) / (rowSums(W H + off)_i + eps)
// (lib.rs:1729-1742), with rowSums(W H)_i = sum_k W[i][k] rowSums(H)_k.
template <int RP>
__global__ void __launch_bounds__(kThreads)
    off_update(const double *__restrict__ W, int n, int r, const double *__restrict__ rsh,
               const double *__restrict__ rsv, int p, double eps, double *__restrict__ off,
               const RunState *st) {
    if (run_stopped(st)) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < RP; k++)
        if (k < r) s = add(s, mul(W[(size_t)i * RP + k], rsh[k]));
    const double o = off[i];
    const double rsw = add(s, mul((double)p, o));
    const double num = rsv[i] > eps ? rsv[i] : eps;
    off[i] = mul(o, num) / add(rsw, eps);
}

// ---------------------------------------------------------------------------
// Epilogues.  Parameters shared by the H and W epilogues.
// ---------------------------------------------------------------------------
struct EpiParams {
    int method;
    int r;
    double eps;
    double lambda;  // dnmf L1 (sparsity)
    double gamma;   // dnmf L2 (smoothness)
    const double *G;    // RP x RP Gram (W^T W for H, H H^T for W)
    const double *sums; // colsum(W) for the brunet H step, rowsum(H) for the W step
    const double *addon = nullptr;  // offset, H step: (W^T off)[k] added to the denominator
    const double *roff = nullptr;   // offset, W step: the row offsets off[i]
    // lsNMF: the numerator contraction (W^T (V o S) as RP x p for the H step,
    // (V o S) H^T as n x RP for the W step); the pass supplies the denominator.
    const double *aux = nullptr;
};

// Per-column H update from the reduced contraction num[] (old column hc[]).
//   lee    : euclidean_update_h_inner  lib.rs:227-241
//   brunet : divergence_update_h_inner lib.rs:105-111
//   hals   : hals_update_h             lib.rs:595-605
//   dnmf   : hals_update_h_reg         lib.rs:1079-1089
template <int RP>
__device__ __forceinline__ void h_update(const EpiParams &e, const double *num, double *hc,
                                         const double *ax = nullptr) {
    const int r = e.r;
    if (e.method == M_LSNMF) {
        // nmf_run_lsnmf lib.rs:990-999: max(eps, H numer) / (denom + eps)
#pragma unroll
        for (int i = 0; i < RP; i++)
            if (i < r) {
                const double temp = mul(hc[i], ax[i]);
                hc[i] = (temp > e.eps ? temp : e.eps) / add(num[i], e.eps);
            }
    } else if (e.method == M_PRODUCT) {
#pragma unroll
        for (int i = 0; i < RP; i++)
            if (i < r) hc[i] = num[i];
    } else if (e.method == M_LEE || e.method == M_OFFSET) {
        // offset (offset_update_h_inner, lib.rs:330-361): + (W^T off)[i]
        double out[RP];
#pragma unroll
        for (int i = 0; i < RP; i++) {
            if (i < r) {
                double den = 0.0;
#pragma unroll
                for (int l = RP - 1; l >= 0; l--)
                    if (l < r) den = add(den, mul(e.G[i * RP + l], hc[l]));
                if (e.addon) den = add(den, e.addon[i]);
                const double temp = mul(hc[i], num[i]);
                out[i] = (temp > e.eps ? temp : e.eps) / add(den, e.eps);
            }
        }
#pragma unroll
        for (int i = 0; i < RP; i++)
            if (i < r) hc[i] = out[i];
    } else if (e.method == M_BRUNET || e.method == M_NSNMF) {
#pragma unroll
        for (int i = 0; i < RP; i++)
            if (i < r) hc[i] = mul(hc[i], num[i]) / e.sums[i];
    } else {
        const bool reg = (e.method == M_DNMF);
#pragma unroll
        for (int k = 0; k < RP; k++) {
            if (k < r) {
                double s = reg ? sub(num[k], e.lambda) : num[k];
#pragma unroll
                for (int jj = 0; jj < RP; jj++)
                    if (jj < r && jj != k) s = sub(s, mul(e.G[k * RP + jj], hc[jj]));
                const double d = reg ? fmax(add(e.G[k * RP + k], e.gamma), e.eps)
                                     : fmax(e.G[k * RP + k], e.eps);
                const double val = s / d;
                hc[k] = val > e.eps ? val : e.eps;
            }
        }
    }
}

// Per-row W update from the reduced contraction num[] (old row wr[]).
//   lee    : euclidean_update_w_impl lib.rs:307-318
//   brunet : divergence_update_w_impl lib.rs:194-200
//   hals   : hals_update_w           lib.rs:622-632
//   dnmf   : hals_update_w_reg       lib.rs:1106-1116
// ro: the row's offset (offset method; lib.rs:441-446), else unused.
template <int RP>
__device__ __forceinline__ void w_update(const EpiParams &e, const double *num, double *wr,
                                         double ro = 0.0, const double *ax = nullptr) {
    const int r = e.r;
    if (e.method == M_LSNMF) {
        // nmf_run_lsnmf lib.rs:1011-1018
#pragma unroll
        for (int j = 0; j < RP; j++)
            if (j < r) {
                const double temp = mul(wr[j], ax[j]);
                wr[j] = (temp > e.eps ? temp : e.eps) / add(num[j], e.eps);
            }
    } else if (e.method == M_PRODUCT) {
#pragma unroll
        for (int j = 0; j < RP; j++)
            if (j < r) wr[j] = num[j];
    } else if (e.method == M_LEE || e.method == M_OFFSET) {
        double out[RP];
#pragma unroll
        for (int j = 0; j < RP; j++) {
            if (j < r) {
                double den = 0.0;
#pragma unroll
                for (int l = RP - 1; l >= 0; l--)
                    if (l < r) den = add(den, mul(wr[l], e.G[l * RP + j]));
                if (e.method == M_OFFSET) den = add(den, mul(ro, e.sums[j]));
                const double temp = mul(wr[j], num[j]);
                out[j] = (temp < e.eps ? e.eps : temp) / add(den, e.eps);
            }
        }
#pragma unroll
        for (int j = 0; j < RP; j++)
            if (j < r) wr[j] = out[j];
    } else if (e.method == M_BRUNET || e.method == M_NSNMF) {
#pragma unroll
        for (int j = 0; j < RP; j++)
            if (j < r) wr[j] = mul(wr[j], num[j]) / e.sums[j];
    } else {
        const bool reg = (e.method == M_DNMF);
#pragma unroll
        for (int k = 0; k < RP; k++) {
            if (k < r) {
                double s = reg ? sub(num[k], e.lambda) : num[k];
#pragma unroll
                for (int jj = 0; jj < RP; jj++)
                    if (jj < r && jj != k) s = sub(s, mul(e.G[k * RP + jj], wr[jj]));
                const double d = reg ? fmax(add(e.G[k * RP + k], e.gamma), e.eps)
                                     : fmax(e.G[k * RP + k], e.eps);
                const double val = s / d;
                wr[k] = val > e.eps ? val : e.eps;
            }
        }
    }
}

// Whether w_update's new W[i][j] depends on row i's old values and num only
// through column j's own formula (every method but the sequential HALS /
// dnmf sweeps), so that its columns can be computed by different threads.
__device__ __forceinline__ bool w_update_by_column(int method) {
    return method == M_LEE || method == M_OFFSET || method == M_BRUNET ||
           method == M_NSNMF || method == M_LSNMF || method == M_PRODUCT;
}
// Column j (< e.r) of w_update for those methods, with the same operations
// in the same order (so the same bits).  numj = num[j], wrj = wr[j].
template <int RP>
__device__ __forceinline__ double w_update_column(const EpiParams &e, double numj, double wrj,
                                                  const double (&wr)[RP], int j,
                                                  double ro = 0.0,
                                                  const double *ax = nullptr) {
    if (e.method == M_LSNMF) {
        const double temp = mul(wrj, ax[j]);
        return (temp > e.eps ? temp : e.eps) / add(numj, e.eps);
    }
    if (e.method == M_PRODUCT) return numj;
    if (e.method == M_LEE || e.method == M_OFFSET) {
        double den = 0.0;
#pragma unroll
        for (int l = RP - 1; l >= 0; l--)
            if (l < e.r) den = add(den, mul(wr[l], e.G[l * RP + j]));
        if (e.method == M_OFFSET) den = add(den, mul(ro, e.sums[j]));
        const double temp = mul(wrj, numj);
        return (temp < e.eps ? e.eps : temp) / add(den, e.eps);
    }
    return mul(wrj, numj) / e.sums[j];  // M_BRUNET, M_NSNMF
}

// H epilogue: one thread per column; sums the S split partials in order.
template <int RP>
__global__ void __launch_bounds__(kThreads)
    h_epilogue(double *__restrict__ H, int p, const double *__restrict__ part, int S,
               EpiParams e, const RunState *st) {
    if (run_stopped(st)) return;
    const int j = blockIdx.x * kThreads + threadIdx.x;
    if (j >= p) return;
    double num[RP], hc[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) {
        double s = 0.0;
        for (int sp = 0; sp < S; sp++) s += part[((int64_t)sp * RP + k) * p + j];
        num[k] = s;
        hc[k] = H[(int64_t)k * p + j];
    }
    h_update<RP>(e, num, hc);
#pragma unroll
    for (int k = 0; k < RP; k++)
        if (k < e.r) H[(int64_t)k * p + j] = hc[k];
}

// W epilogue: one thread per row.
template <int RP>
__global__ void __launch_bounds__(kThreads)
    w_epilogue(double *__restrict__ W, int n, const double *__restrict__ part, int S,
               EpiParams e, const RunState *st) {
    if (run_stopped(st)) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    double num[RP], wr[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) {
        double s = 0.0;
        for (int sp = 0; sp < S; sp++) s += part[((int64_t)sp * n + i) * RP + k];
        num[k] = s;
        wr[k] = W[(int64_t)i * RP + k];
    }
    w_update<RP>(e, num, wr, e.roff ? e.roff[i] : 0.0);
#pragma unroll
    for (int k = 0; k < RP; k++)
        if (k < e.r) W[(int64_t)i * RP + k] = wr[k];
}

// ---------------------------------------------------------------------------
// Gram matrices and sums (two-stage, fixed order).
// ---------------------------------------------------------------------------

// The second stage inside the first stage's launch: each block publishes
// its partials and takes a ticket; the block that takes the last ticket sums
// the B = gridDim.x partials in block order (the sums gram_finalize forms,
// bit for bit) and resets the ticket for the next launch.  No block waits
// on another.  G == nullptr leaves the partials for the caller (lee's and
// nsNMF's col_rescale read them).
template <int RP>
__device__ __forceinline__ void gram_finish_last(const double *pg, const double *ps, double *G,
                                                 double *sums, unsigned *ticket) {
    if (G == nullptr) return;
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int tid = threadIdx.x;
    const int B = (int)gridDim.x;
    double g = 0.0;
    for (int b = 0; b < B; b++) g += __ldcg(&pg[(int64_t)b * RP * RP + tid]);
    G[tid] = g;
    if (tid < RP) {
        double t = 0.0;
        for (int b = 0; b < B; b++) t += __ldcg(&ps[(int64_t)b * RP + tid]);
        sums[tid] = t;
    }
    if (tid == 0) *ticket = 0u;
}

// W^T W and colsum(W) partials over a row range, and with G given the
// finished Gram and sums (gram_finish_last).  block RP*RP threads.
template <int RP>
__global__ void gram_w_partial(const double *__restrict__ W, int n, int rows_per_block,
                               double *__restrict__ pg, double *__restrict__ ps,
                               const RunState *st, double *G = nullptr, double *sums = nullptr,
                               unsigned *ticket = nullptr) {
    if (run_stopped(st)) return;
    constexpr int CH = 64;
    __shared__ double sW[CH][RP];
    const int tid = threadIdx.x;
    const int k = tid / RP, l = tid % RP;
    const int u0 = blockIdx.x * rows_per_block;
    const int u1 = min(n, u0 + rows_per_block);
    double g = 0.0, s = 0.0;
    for (int base = u0; base < u1; base += CH) {
        const int rows = min(CH, u1 - base);
        __syncthreads();
        for (int t = tid; t < CH * RP; t += RP * RP)
            (&sW[0][0])[t] = (t < rows * RP) ? W[(int64_t)base * RP + t] : 0.0;
        __syncthreads();
        for (int u = 0; u < rows; u++) {
            g = fma(sW[u][k], sW[u][l], g);
            if (tid < RP) s += sW[u][tid];
        }
    }
    pg[(int64_t)blockIdx.x * RP * RP + tid] = g;
    if (tid < RP) ps[(int64_t)blockIdx.x * RP + tid] = s;
    gram_finish_last<RP>(pg, ps, G, sums, ticket);
}

// H H^T and rowsum(H) partials over a column range, and with G given the
// finished Gram and sums.  block RP*RP threads.
template <int RP>
__global__ void gram_h_partial(const double *__restrict__ H, int p, int cols_per_block,
                               double *__restrict__ pg, double *__restrict__ ps,
                               const RunState *st, double *G = nullptr, double *sums = nullptr,
                               unsigned *ticket = nullptr) {
    if (run_stopped(st)) return;
    constexpr int CC = 64;
    __shared__ double sH[RP][CC + 1];
    const int tid = threadIdx.x;
    const int k = tid / RP, l = tid % RP;
    const int c0 = blockIdx.x * cols_per_block;
    const int c1 = min(p, c0 + cols_per_block);
    double g = 0.0, s = 0.0;
    for (int base = c0; base < c1; base += CC) {
        const int cols = min(CC, c1 - base);
        __syncthreads();
        for (int t = tid; t < RP * CC; t += RP * RP) {
            const int kk = t / CC, cc = t % CC;
            sH[kk][cc] = (cc < cols) ? H[(int64_t)kk * p + base + cc] : 0.0;
        }
        __syncthreads();
        for (int c = 0; c < cols; c++) {
            g = fma(sH[k][c], sH[l][c], g);
            if (tid < RP) s += sH[tid][c];
        }
    }
    pg[(int64_t)blockIdx.x * RP * RP + tid] = g;
    if (tid < RP) ps[(int64_t)blockIdx.x * RP + tid] = s;
    gram_finish_last<RP>(pg, ps, G, sums, ticket);
}

// Sum B partial Grams / sums in block order.  block RP*RP threads.
template <int RP>
__global__ void gram_finalize(const double *__restrict__ pg, const double *__restrict__ ps,
                              int B, double *__restrict__ G, double *__restrict__ sums,
                              const RunState *st) {
    if (run_stopped(st)) return;
    const int tid = threadIdx.x;
    double g = 0.0;
    for (int b = 0; b < B; b++) g += pg[(int64_t)b * RP * RP + tid];
    G[tid] = g;
    if (tid < RP) {
        double s = 0.0;
        for (int b = 0; b < B; b++) s += ps[(int64_t)b * RP + tid];
        sums[tid] = s;
    }
}

// lee's col_rescale (lib.rs:1461-1470): every block re-sums the colsum
// partials in the same order, then divides its rows.  W[:, k] /= s_k when
// s_k > 0.
template <int RP>
__global__ void col_rescale(double *__restrict__ W, int n, int r, const double *__restrict__ ps,
                            int B, const RunState *st) {
    if (run_stopped(st)) return;
    __shared__ double s[RP];
    if (threadIdx.x < RP) {
        double a = 0.0;
        for (int b = 0; b < B; b++) a += ps[(int64_t)b * RP + threadIdx.x];
        s[threadIdx.x] = a;
    }
    __syncthreads();
    const int64_t total = (int64_t)n * RP;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % RP);
        if (k < r && s[k] > 0.0) W[t] = W[t] / s[k];
    }
}

// dnmf's extract_diagonal (lib.rs:808-824) followed by H *= d (lib.rs:880-884).
// Gw / Gh are the Grams of the current W and H; their diagonals are the
// squared norms of W's columns and H's rows.
template <int RP>
__global__ void dnmf_rescale(double *__restrict__ W, double *__restrict__ H, int n, int p, int r,
                             const double *__restrict__ Gw, const double *__restrict__ Gh,
                             const RunState *st) {
    if (run_stopped(st)) return;
    __shared__ double nw[RP], nh[RP], dk[RP];
    if (threadIdx.x < RP) {
        const int k = threadIdx.x;
        const double a = sqrt(Gw[k * RP + k]);
        const double b = sqrt(Gh[k * RP + k]);
        nw[k] = a;
        nh[k] = b;
        dk[k] = a * b;
    }
    __syncthreads();
    const int64_t tw = (int64_t)n * RP;
    const int64_t th = (int64_t)r * p;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tw; t += stride) {
        const int k = (int)(t % RP);
        if (k < r && nw[k] > 0.0) W[t] = W[t] / nw[k];
    }
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < th; t += stride) {
        const int k = (int)(t / p);
        double h = H[t];
        if (nh[k] > 0.0) h = h / nh[k];
        H[t] = h * dk[k];
    }
}

// brunet's every-10-iterations clamp (pmax_inplace, lib.rs:1452-1458):
// x < eps -> eps (NaN stays NaN), on the r real columns / rows only.
template <int RP>
__global__ void clamp_wh(double *__restrict__ W, double *__restrict__ H, int n, int p, int r,
                         double eps, const RunState *st) {
    if (run_stopped(st)) return;
    const int64_t tw = (int64_t)n * RP;
    const int64_t th = (int64_t)r * p;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tw; t += stride) {
        const int k = (int)(t % RP);
        if (k < r && W[t] < eps) W[t] = eps;
    }
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < th; t += stride)
        if (H[t] < eps) H[t] = eps;
}

// ---------------------------------------------------------------------------
// Objective finalisation + stationary stop (one block).
// ---------------------------------------------------------------------------
struct StopParams {
    int stationary;       // 1: run StationaryStop::should_stop
    long long iter;       // 0 for the initial objective
    long long check_interval;
    long long check_niter;
    double threshold;
    double scale;         // 0.5 for the Frobenius objective, 1 for KL
};

// Sum of B partials in objective_finalize's order, into out[0] (a column
// shard's objective term, before the sum over shards).
static __global__ void sum_partials(const double *__restrict__ part, int B,
                                    double *__restrict__ out) {
    __shared__ double red[kThreads];
    const int tid = threadIdx.x;
    double a = 0.0;
    for (int b = tid; b < B; b += kThreads) a += part[b];
    red[tid] = a;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (tid < s) red[tid] += red[tid + s];
        __syncthreads();
    }
    if (tid == 0) out[0] = red[0];
}

// W update from a dense contraction num (n x RP) summed over column shards:
// one thread a row, the update of w_update.
template <int RP>
__global__ void __launch_bounds__(kThreads)
    w_apply_dense(double *__restrict__ W, int n, const double *__restrict__ num, EpiParams e,
                  const RunState *st) {
    if (run_stopped(st)) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    double nm[RP], wr[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) {
        nm[k] = num[(size_t)i * RP + k];
        wr[k] = W[(size_t)i * RP + k];
    }
    w_update<RP>(e, nm, wr);
#pragma unroll
    for (int k = 0; k < RP; k++)
        if (k < e.r) W[(size_t)i * RP + k] = wr[k];
}

static __global__ void objective_finalize(const double *__restrict__ part, int B, double *__restrict__ dev,
                                   StopParams sp, RunState *st) {
    if (st->stopped) return;
    __shared__ double red[kThreads];
    const int tid = threadIdx.x;
    double a = 0.0;
    for (int b = tid; b < B; b += kThreads) a += part[b];
    red[tid] = a;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (tid < s) red[tid] += red[tid + s];
        __syncthreads();
    }
    if (tid != 0) return;
    const double d = red[0] * sp.scale;
    if (dev) dev[sp.iter] = d;
    if (!sp.stationary) return;
    // StationaryStop::should_stop, lib.rs:1378-1400.
    bool stop = false;
    if (isnan(d)) {
        stop = true;
    } else if (sp.iter == 0) {
        st->last_max = d;  // reset() then record(d)
        st->last_min = d;
        st->n_collected = 1;
    } else {
        bool sample = true;
        if (st->n_collected == 0) {
            if (sp.check_interval == 0) {
                st->error = 1;  // the reference panics on `i % 0`
                stop = true;
                sample = false;
            } else if (sp.iter % sp.check_interval != 0) {
                sample = false;
            }
        }
        if (sample) {
            if (d > st->last_max) st->last_max = d;
            if (d < st->last_min) st->last_min = d;
            st->n_collected += 1;
            if (st->n_collected == sp.check_niter + 1) {
                const double crit = fabs(st->last_max - st->last_min) / (double)sp.check_niter;
                if (crit <= sp.threshold) {
                    stop = true;
                } else {
                    st->last_max = -INFINITY;
                    st->last_min = INFINITY;
                    st->n_collected = 0;
                }
            }
        }
    }
    if (stop) {
        st->stopped = 1;
        st->n_iter = sp.iter;
    }
}

// ---------------------------------------------------------------------------
// Layout helpers.
// ---------------------------------------------------------------------------

// H (RP x p f64) -> H^T (p x rps, type TH), zero past the first r entries.
template <typename TH>
__global__ void h_transpose(const double *__restrict__ H, TH *__restrict__ Ht, int p, int r,
                            int rps) {
    const int64_t total = (int64_t)p * rps;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / rps;
        const int k = (int)(t - j * rps);
        Ht[t] = (k < r) ? (TH)H[(int64_t)k * p + j] : (TH)0;
    }
}

static __global__ void convert_f64_f32(const double *__restrict__ src, int64_t lds, float *__restrict__ dst,
                                int64_t ldd, int n, int p) {
    const int64_t total = (int64_t)n * p;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / p, j = t - i * p;
        dst[i * ldd + j] = (float)src[i * lds + j];
    }
}

}  // namespace nmfcu

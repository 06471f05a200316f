// wide.cu -- the FP64 loop for ranks above the streaming passes' largest
// bucket (NMFCU_MAX_RANK = 32): lee, brunet, hals and dnmf at any rank up to
// NMFCU_MAX_WIDE_RANK.  The reference has no rank limit (nmf_run_lee
// rust/src/lib.rs:1589-1647, nmf_run_brunet :1529-1586, nmf_run_hals
// :638-688, nmf_run_dnmf :827-906).
//
// The V contractions are the FP64 tensor-core streaming passes run in rank
// chunks of at most 32 (nmfcu_internal::v_product_locked, one pass over V a
// chunk):
//   lee / hals / dnmf   W^T V and V H'^T  -> the H and W numerators
//   brunet              the ratio Q = V / (W H) (0 where W H is 0,
//                       lib.rs:89-97 / 181-189) is written out by a tiled
//                       kernel, then W^T Q and Q H'^T by the same passes.
// Everything rank-dependent (Grams, updates, rescaling, objective) runs in
// the kernels below with the rank as a run-time value: one thread per column
// of H / row of W for the updates, in the operation order of the dense
// engine's epilogues (kernels.cuh h_update / w_update), which follow the
// reference term by term.  The stop state is the context's run state, so
// every pass and kernel of an iteration after a stationary stop does no work.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <string>
#include <vector>

#include "../../include/nmfcu.h"
#include "internal.h"
#include "kernels.cuh"

using nmfcu_internal::fail;

namespace {

using nmfcu::RunState;
using nmfcu::add;
using nmfcu::mul;
using nmfcu::sub;
constexpr int kT = 256;

// Context scratch slots of this file.
constexpr int kSlotQ = 24;    // brunet: the ratio V / (W H), n x ldq
constexpr int kSlotBuf = 25;  // factors, contractions, Grams, partials

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }
inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// ---------------------------------------------------------------------------
// Grams: G[k][l] = sum_u X(u, k) X(u, l) and sums[k] = sum_u X(u, k) for
// X(u, k) = X[u * sr + k * sc] (W: sr = r, sc = 1; H^T: sr = 1, sc = p).
// Stage 1: block (b, g) adds rows [b * rpb, (b + 1) * rpb) for pairs
// g * kT * kPPT + i * kT + t, pair = k * (r + 1) + l (l == r: the sum);
// rows staged kRowsChunk at a time.  Stage 2 adds the blocks in order.
// ---------------------------------------------------------------------------
constexpr int kPPT = 8;
constexpr int kRowsChunk = 16;  // 16 x 256 f64 = 32 KB of staging at the largest rank

__global__ void __launch_bounds__(kT)
    wide_gram_partial(const double *__restrict__ X, int64_t m, int r, int64_t sr, int64_t sc,
                      int64_t rpb, double *__restrict__ part, const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    extern __shared__ double chunk[];  // [kRowsChunk][r]
    const int npairs = r * (r + 1);
    const int64_t u0 = blockIdx.x * rpb, u1 = min(m, u0 + rpb);
    int pk[kPPT], pl[kPPT];
    double acc[kPPT];
#pragma unroll
    for (int i = 0; i < kPPT; i++) {
        const int pr = (blockIdx.y * kPPT + i) * kT + threadIdx.x;
        pk[i] = pr < npairs ? pr / (r + 1) : -1;
        pl[i] = pr < npairs ? pr - pk[i] * (r + 1) : 0;
        acc[i] = 0.0;
    }
    for (int64_t c0 = u0; c0 < u1; c0 += kRowsChunk) {
        const int nr = (int)min((int64_t)kRowsChunk, u1 - c0);
        __syncthreads();
        for (int e = threadIdx.x; e < nr * r; e += kT) {
            const int uu = e / r, k = e - uu * r;
            chunk[e] = X[(c0 + uu) * sr + (int64_t)k * sc];
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kPPT; i++) {
            if (pk[i] < 0) continue;
            double a = acc[i];
            if (pl[i] == r) {
                for (int uu = 0; uu < nr; uu++) a += chunk[uu * r + pk[i]];
            } else {
                for (int uu = 0; uu < nr; uu++) a += chunk[uu * r + pk[i]] * chunk[uu * r + pl[i]];
            }
            acc[i] = a;
        }
    }
#pragma unroll
    for (int i = 0; i < kPPT; i++)
        if (pk[i] >= 0) part[(int64_t)blockIdx.x * npairs + pk[i] * (r + 1) + pl[i]] = acc[i];
}

__global__ void wide_gram_final(const double *__restrict__ part, int B, int r,
                                double *__restrict__ G, double *__restrict__ sums,
                                const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    const int npairs = r * (r + 1);
    const int pr = blockIdx.x * kT + threadIdx.x;
    if (pr >= npairs) return;
    double a = 0.0;
    for (int b = 0; b < B; b++) a += part[(int64_t)b * npairs + pr];
    const int k = pr / (r + 1), l = pr - k * (r + 1);
    if (l == r)
        sums[k] = a;
    else
        G[k * r + l] = a;
}

// Ht (p x r) = H (r x p)^T through 32 x 32 shared-memory tiles.
__global__ void wide_transpose(const double *__restrict__ H, int r, int64_t p,
                               double *__restrict__ Ht, const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    __shared__ double t[32][33];
    const int64_t j0 = (int64_t)blockIdx.x * 32;
    const int k0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int k = k0 + y;
        const int64_t j = j0 + threadIdx.x;
        if (k < r && j < p) t[y][threadIdx.x] = H[(int64_t)k * p + j];
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int64_t j = j0 + y;
        const int k = k0 + threadIdx.x;
        if (k < r && j < p) Ht[j * r + k] = t[threadIdx.x][y];
    }
}

// ---------------------------------------------------------------------------
// W H in 64 x 64 tiles (16 x 16 threads, 4 x 4 outputs a thread, the rank
// in chunks of 16 through shared memory), and what each use makes of it:
//   MODE 0  Q[i][j] = V[i][j] / (W H)[i][j], 0 where W H is 0 (brunet's ratio)
//   MODE 1  per-block partial of the KL objective (kl_divergence lib.rs:1418-1427)
//   MODE 2  per-block partial of sum (V - W H)^2 (euclidean_distance :1440-1441)
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(kT)
    wide_wh(const double *__restrict__ V, int64_t ldv, const double *__restrict__ W,
            const double *__restrict__ H, int n, int64_t p, int r, double *__restrict__ Q,
            int64_t ldq, double *__restrict__ part, const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    __shared__ double sW[64][17];
    __shared__ double sH[16][64];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int i0 = blockIdx.y * 64;
    const int64_t j0 = (int64_t)blockIdx.x * 64;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
    for (int k0 = 0; k0 < r; k0 += 16) {
        __syncthreads();
        for (int e = threadIdx.x; e < 64 * 16; e += kT) {
            const int ii = e >> 4, kk = e & 15;
            const int i = i0 + ii, k = k0 + kk;
            sW[ii][kk] = (i < n && k < r) ? W[(int64_t)i * r + k] : 0.0;
            const int kh = e >> 6, jj = e & 63;
            const int64_t j = j0 + jj;
            sH[kh][jj] = (k0 + kh < r && j < p) ? H[(int64_t)(k0 + kh) * p + j] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; kk++) {
            double w[4], h[4];
#pragma unroll
            for (int a = 0; a < 4; a++) w[a] = sW[ty + 16 * a][kk];
#pragma unroll
            for (int b = 0; b < 4; b++) h[b] = sH[kk][tx + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 4; b++) acc[a][b] = fma(w[a], h[b], acc[a][b]);
        }
    }
    double term = 0.0;
#pragma unroll
    for (int a = 0; a < 4; a++) {
        const int i = i0 + ty + 16 * a;
        if (i >= n) continue;
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int64_t j = j0 + tx + 16 * b;
            if (j >= p) continue;
            const double v = V[(int64_t)i * ldv + j];
            const double wh = acc[a][b];
            if (MODE == 0) {
                Q[(int64_t)i * ldq + j] = (wh != 0.0) ? v / wh : 0.0;
            } else if (MODE == 1) {
                if (v > 0.0) {
                    if (wh > 0.0) term = add(term, add(sub(mul(v, log(v / wh)), v), wh));
                } else {
                    term = add(term, wh);
                }
            } else {
                const double d = sub(v, wh);
                term = add(term, mul(d, d));
            }
        }
    }
    if (MODE != 0) {
        __shared__ double red[kT];
        red[threadIdx.x] = term;
        __syncthreads();
        for (int s = kT / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = red[0];
    }
}

// ---------------------------------------------------------------------------
// Updates, one thread per column of H / row of W, in the dense epilogues'
// operation order (kernels.cuh h_update / w_update).
// ---------------------------------------------------------------------------
struct WideEpi {
    int method;
    int r;
    double eps, lambda, gamma;
    const double *G;     // r x r
    const double *sums;  // r
};

// H (r x p); num: p x r (num[j * r + k]); lee writes Hn, the others H.
__global__ void __launch_bounds__(kT)
    wide_h_update(double *__restrict__ H, double *__restrict__ Hn, int64_t p,
                  const double *__restrict__ num, WideEpi e, const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    const int64_t j = (int64_t)blockIdx.x * kT + threadIdx.x;
    if (j >= p) return;
    const int r = e.r;
    const double *nj = num + j * r;
    if (e.method == nmfcu::M_LEE) {
        // euclidean_update_h_inner lib.rs:227-241
        for (int i = 0; i < r; i++) {
            double den = 0.0;
            for (int l = r - 1; l >= 0; l--) den = add(den, mul(e.G[i * r + l], H[(int64_t)l * p + j]));
            const double temp = mul(H[(int64_t)i * p + j], nj[i]);
            Hn[(int64_t)i * p + j] = (temp > e.eps ? temp : e.eps) / add(den, e.eps);
        }
    } else if (e.method == nmfcu::M_BRUNET) {
        // divergence_update_h_inner lib.rs:105-111
        for (int i = 0; i < r; i++) {
            double &h = H[(int64_t)i * p + j];
            h = mul(h, nj[i]) / e.sums[i];
        }
    } else {
        // hals_update_h lib.rs:595-605; hals_update_h_reg lib.rs:1079-1089
        const bool reg = (e.method == nmfcu::M_DNMF);
        for (int k = 0; k < r; k++) {
            double s = reg ? sub(nj[k], e.lambda) : nj[k];
            for (int jj = 0; jj < r; jj++)
                if (jj != k) s = sub(s, mul(e.G[k * r + jj], H[(int64_t)jj * p + j]));
            const double d = reg ? fmax(add(e.G[k * r + k], e.gamma), e.eps) : fmax(e.G[k * r + k], e.eps);
            const double val = s / d;
            H[(int64_t)k * p + j] = val > e.eps ? val : e.eps;
        }
    }
}

// W (n x r); num: n x r; lee writes Wn, the others W.
__global__ void __launch_bounds__(kT)
    wide_w_update(double *__restrict__ W, double *__restrict__ Wn, int n,
                  const double *__restrict__ num, WideEpi e, const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    const int i = blockIdx.x * kT + threadIdx.x;
    if (i >= n) return;
    const int r = e.r;
    double *wr = W + (int64_t)i * r;
    const double *ni = num + (int64_t)i * r;
    if (e.method == nmfcu::M_LEE) {
        // euclidean_update_w_impl lib.rs:307-318
        for (int j = 0; j < r; j++) {
            double den = 0.0;
            for (int l = r - 1; l >= 0; l--) den = add(den, mul(wr[l], e.G[l * r + j]));
            const double temp = mul(wr[j], ni[j]);
            Wn[(int64_t)i * r + j] = (temp < e.eps ? e.eps : temp) / add(den, e.eps);
        }
    } else if (e.method == nmfcu::M_BRUNET) {
        // divergence_update_w_impl lib.rs:194-200
        for (int j = 0; j < r; j++) wr[j] = mul(wr[j], ni[j]) / e.sums[j];
    } else {
        // hals_update_w lib.rs:622-632; hals_update_w_reg lib.rs:1106-1116
        const bool reg = (e.method == nmfcu::M_DNMF);
        for (int k = 0; k < r; k++) {
            double s = reg ? sub(ni[k], e.lambda) : ni[k];
            for (int jj = 0; jj < r; jj++)
                if (jj != k) s = sub(s, mul(e.G[k * r + jj], wr[jj]));
            const double d = reg ? fmax(add(e.G[k * r + k], e.gamma), e.eps) : fmax(e.G[k * r + k], e.eps);
            const double val = s / d;
            wr[k] = val > e.eps ? val : e.eps;
        }
    }
}

// lee's col_rescale (lib.rs:1461-1470): W[:, k] /= colsum_k when > 0.
__global__ void wide_col_rescale(double *__restrict__ W, int64_t n, int r,
                                 const double *__restrict__ sums, const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    const int64_t total = n * r;
    for (int64_t t = blockIdx.x * (int64_t)kT + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * kT) {
        const double s = sums[t % r];
        if (s > 0.0) W[t] = W[t] / s;
    }
}

// brunet's every-10-iterations clamp (pmax_inplace, lib.rs:1452-1458).
__global__ void wide_clamp(double *__restrict__ W, int64_t nw, double *__restrict__ H, int64_t nh,
                           double eps, const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    const int64_t stride = (int64_t)gridDim.x * kT;
    for (int64_t t = blockIdx.x * (int64_t)kT + threadIdx.x; t < nw; t += stride)
        if (W[t] < eps) W[t] = eps;
    for (int64_t t = blockIdx.x * (int64_t)kT + threadIdx.x; t < nh; t += stride)
        if (H[t] < eps) H[t] = eps;
}

// dnmf's extract_diagonal (lib.rs:808-824) and H *= d (lib.rs:880-884), as
// kernels.cuh dnmf_rescale.
__global__ void wide_dnmf_rescale(double *__restrict__ W, int64_t n, double *__restrict__ H,
                                  int64_t p, int r, const double *__restrict__ Gw,
                                  const double *__restrict__ Gh, const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    const int64_t stride = (int64_t)gridDim.x * kT;
    for (int64_t t = blockIdx.x * (int64_t)kT + threadIdx.x; t < n * r; t += stride) {
        const int k = (int)(t % r);
        const double a = sqrt(Gw[k * r + k]);
        if (a > 0.0) W[t] = W[t] / a;
    }
    for (int64_t t = blockIdx.x * (int64_t)kT + threadIdx.x; t < (int64_t)r * p; t += stride) {
        const int k = (int)(t / p);
        const double a = sqrt(Gw[k * r + k]), b = sqrt(Gh[k * r + k]);
        double h = H[t];
        if (b > 0.0) h = h / b;
        H[t] = h * (a * b);
    }
}

// ---------------------------------------------------------------------------
// Host loop
// ---------------------------------------------------------------------------

struct Bufs {
    double *W, *H, *Ht, *NW, *NH, *Wn, *Hn, *part, *Gw, *sw, *Gh, *sh, *Gw2, *sw2, *opart;
    double *Q;
    int64_t ldq;
    int Bw, Bh, gy;
    int64_t rpw, rph;
    int gx_obj, gy_obj;
};

struct Loop {
    nmfcu_context *c;
    const nmfcu_options *o;
    int64_t n, p;
    int r;
    const double *V;
    int64_t ldv;
    Bufs b;
    RunState *st;
    double *dev;
    cudaStream_t s;

    nmfcu_status gram(const double *X, int64_t m, int64_t sr, int64_t sc, int B, int64_t rpb,
                      double *G, double *sums) {
        nmfcu_internal::TimedScope sc_(c, s, NMFCU_KCLASS_OTHER, 2);
        const size_t sm = sizeof(double) * kRowsChunk * r;
        wide_gram_partial<<<dim3(B, b.gy), kT, sm, s>>>(X, m, r, sr, sc, rpb, b.part, st);
        wide_gram_final<<<cdiv((int64_t)r * (r + 1), kT), kT, 0, s>>>(b.part, B, r, G, sums, st);
        NMFCU_CUDA_TRY(cudaGetLastError());
        return NMFCU_OK;
    }
    nmfcu_status gram_w(double *G, double *sums) { return gram(b.W, n, r, 1, b.Bw, b.rpw, G, sums); }
    nmfcu_status gram_h(double *G, double *sums) { return gram(b.H, p, 1, p, b.Bh, b.rph, G, sums); }
    void transpose() {
        nmfcu_internal::TimedScope sc_(c, s, NMFCU_KCLASS_OTHER);
        wide_transpose<<<dim3(cdiv(p, 32), cdiv(r, 32)), dim3(32, 8), 0, s>>>(b.H, r, p, b.Ht, st);
    }
    void ratio() {
        nmfcu_internal::TimedScope sc_(c, s, NMFCU_KCLASS_OTHER);
        wide_wh<0><<<dim3(b.gx_obj, b.gy_obj), kT, 0, s>>>(V, ldv, b.W, b.H, (int)n, p, r, b.Q,
                                                          b.ldq, nullptr, st);
    }
    WideEpi epi(const double *G, const double *sums, bool hside) const {
        WideEpi e;
        e.method = o->method;
        e.r = r;
        e.eps = o->eps;
        e.lambda = hside ? o->sparsity_h : o->sparsity_w;
        e.gamma = hside ? o->smoothness_h : o->smoothness_w;
        e.G = G;
        e.sums = sums;
        return e;
    }
    // The H step: numerator p x r (V^T W, or Q^T W for brunet), then the update.
    nmfcu_status h_step(const WideEpi &e) {
        const bool kl = o->method == NMFCU_BRUNET;
        if (kl) ratio();
        // (the passes time themselves as H-step launches)
        NMFCU_TRY(nmfcu_internal::v_product_locked(c, 1, n, p, r, kl ? b.Q : V, kl ? b.ldq : ldv,
                                                   b.W, r, b.NH, r, s, false, false));
        nmfcu_internal::TimedScope sc_(c, s, NMFCU_KCLASS_OTHER);
        wide_h_update<<<std::max(1u, cdiv(p, kT)), kT, 0, s>>>(b.H, b.Hn, p, b.NH, e, st);
        if (o->method == NMFCU_LEE)
            NMFCU_CUDA_TRY(cudaMemcpyAsync(b.H, b.Hn, sizeof(double) * (size_t)r * p,
                                           cudaMemcpyDeviceToDevice, s));
        return NMFCU_OK;
    }
    // The W step: numerator n x r (V H'^T, or Q H'^T for brunet), then the update.
    nmfcu_status w_step(const WideEpi &e) {
        const bool kl = o->method == NMFCU_BRUNET;
        if (kl) ratio();
        transpose();
        // (the passes time themselves as W-step launches)
        NMFCU_TRY(nmfcu_internal::v_product_locked(c, 0, n, p, r, kl ? b.Q : V, kl ? b.ldq : ldv,
                                                   b.Ht, r, b.NW, r, s, false, false));
        nmfcu_internal::TimedScope sc_(c, s, NMFCU_KCLASS_OTHER);
        wide_w_update<<<std::max(1u, cdiv(n, kT)), kT, 0, s>>>(b.W, b.Wn, (int)n, b.NW, e, st);
        if (o->method == NMFCU_LEE)
            NMFCU_CUDA_TRY(cudaMemcpyAsync(b.W, b.Wn, sizeof(double) * (size_t)n * r,
                                           cudaMemcpyDeviceToDevice, s));
        return NMFCU_OK;
    }
    nmfcu_status objective(long long iter) {
        const bool kl = o->method == NMFCU_BRUNET;
        {
            nmfcu_internal::TimedScope sc_(c, s, NMFCU_KCLASS_OBJECTIVE);
            if (kl)
                wide_wh<1><<<dim3(b.gx_obj, b.gy_obj), kT, 0, s>>>(V, ldv, b.W, b.H, (int)n, p, r,
                                                                  nullptr, 0, b.opart, st);
            else
                wide_wh<2><<<dim3(b.gx_obj, b.gy_obj), kT, 0, s>>>(V, ldv, b.W, b.H, (int)n, p, r,
                                                                  nullptr, 0, b.opart, st);
        }
        nmfcu::StopParams sp;
        sp.stationary = 1;
        sp.iter = iter;
        sp.check_interval = o->check_interval;
        sp.check_niter = o->check_niter;
        sp.threshold = o->stationary_th;
        sp.scale = kl ? 1.0 : 0.5;
        nmfcu_internal::TimedScope sc_(c, s, NMFCU_KCLASS_OTHER);
        nmfcu::objective_finalize<<<1, nmfcu::kThreads, 0, s>>>(
            b.opart, b.gx_obj * b.gy_obj, dev, sp, st);
        NMFCU_CUDA_TRY(cudaGetLastError());
        return NMFCU_OK;
    }
    nmfcu_status iteration(long long it) {
        switch (o->method) {
            case NMFCU_BRUNET:
                // nmf_run_brunet lib.rs:1558-1575
                NMFCU_TRY(gram_w(b.Gw, b.sw));
                NMFCU_TRY(h_step(epi(b.Gw, b.sw, true)));
                NMFCU_TRY(gram_h(b.Gh, b.sh));
                NMFCU_TRY(w_step(epi(b.Gh, b.sh, false)));
                if (it % 10 == 0) {
                    nmfcu_internal::TimedScope sc_(c, s, NMFCU_KCLASS_OTHER);
                    wide_clamp<<<std::min(4096u, std::max(1u, cdiv(std::max(n, p) * r, kT))), kT, 0, s>>>(
                        b.W, n * r, b.H, (int64_t)r * p, DBL_EPSILON, st);
                }
                break;
            case NMFCU_LEE:
                // nmf_run_lee lib.rs:1618-1636
                NMFCU_TRY(gram_w(b.Gw, b.sw));
                NMFCU_TRY(h_step(epi(b.Gw, b.sw, true)));
                NMFCU_TRY(gram_h(b.Gh, b.sh));
                NMFCU_TRY(w_step(epi(b.Gh, b.sh, false)));
                if (o->rescale) {
                    NMFCU_TRY(gram_w(b.Gw2, b.sw2));
                    nmfcu_internal::TimedScope sc_(c, s, NMFCU_KCLASS_OTHER);
                    wide_col_rescale<<<std::min(4096u, std::max(1u, cdiv(n * r, kT))), kT, 0, s>>>(
                        b.W, n, r, b.sw2, st);
                }
                break;
            default:
                // nmf_run_hals lib.rs:667-676; nmf_run_dnmf lib.rs:862-884
                NMFCU_TRY(gram_w(b.Gw, b.sw));
                NMFCU_TRY(h_step(epi(b.Gw, b.sw, true)));
                NMFCU_TRY(gram_h(b.Gh, b.sh));
                NMFCU_TRY(w_step(epi(b.Gh, b.sh, false)));
                if (o->method == NMFCU_DNMF) {
                    NMFCU_TRY(gram_w(b.Gw2, b.sw2));
                    nmfcu_internal::TimedScope sc_(c, s, NMFCU_KCLASS_OTHER);
                    wide_dnmf_rescale<<<std::min(4096u, std::max(1u, cdiv(std::max(n, p) * r, kT))), kT, 0, s>>>(
                        b.W, n, b.H, p, r, b.Gw2, b.Gh, st);
                }
                break;
        }
        NMFCU_CUDA_TRY(cudaGetLastError());
        return NMFCU_OK;
    }
};

nmfcu_status make_bufs(nmfcu_context *c, const nmfcu_options *o, int64_t n, int64_t p, int r,
                       Bufs &b) {
    const int sms = nmfcu_internal::context_sms(c);
    b.Bw = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sms));
    b.rpw = std::max<int64_t>(1, (n + b.Bw - 1) / b.Bw);
    b.Bh = (int)std::max<int64_t>(1, std::min<int64_t>((p + 255) / 256, sms));
    b.rph = std::max<int64_t>(1, (p + b.Bh - 1) / b.Bh);
    b.gy = (int)cdiv((int64_t)r * (r + 1), (int64_t)kT * kPPT);
    b.gx_obj = (int)std::max<int64_t>(1, (p + 63) / 64);
    b.gy_obj = (int)std::max<int64_t>(1, (n + 63) / 64);
    const int npairs = r * (r + 1);
    const size_t d = sizeof(double);
    const size_t nr = (size_t)n * r, pr = (size_t)p * r;
    const std::vector<size_t> sizes = {
        d * nr, d * pr, d * pr, d * nr, d * pr, d * nr, d * pr,
        d * (size_t)std::max(b.Bw, b.Bh) * npairs,
        d * r * r, d * r, d * r * r, d * r, d * r * r, d * r,
        d * (size_t)b.gx_obj * b.gy_obj};
    size_t total = 0;
    for (size_t z : sizes) total += align256(std::max<size_t>(z, 1));
    void *base = nullptr;
    NMFCU_TRY(nmfcu_internal::context_buffer(c, kSlotBuf, total, &base));
    double **dst[] = {&b.W, &b.H, &b.Ht, &b.NW, &b.NH, &b.Wn, &b.Hn, &b.part, &b.Gw, &b.sw,
                      &b.Gh, &b.sh, &b.Gw2, &b.sw2, &b.opart};
    char *q = static_cast<char *>(base);
    for (size_t i = 0; i < sizes.size(); i++) {
        *dst[i] = reinterpret_cast<double *>(q);
        q += align256(std::max<size_t>(sizes[i], 1));
    }
    b.Q = nullptr;
    b.ldq = std::max<int64_t>(16, (p + 15) / 16 * 16);
    if (o->method == NMFCU_BRUNET) {
        void *pq = nullptr;
        NMFCU_TRY(nmfcu_internal::context_buffer(c, kSlotQ, d * (size_t)n * b.ldq, &pq));
        b.Q = static_cast<double *>(pq);
    }
    return NMFCU_OK;
}

}  // namespace

namespace nmfcu_internal {

// The option checks for a rank above NMFCU_MAX_RANK.
nmfcu_status wide_validate(const nmfcu_options *o, int64_t n, int64_t p, int64_t r) {
    if (!o) return fail(NMFCU_ERR_INVALID_ARG, "options pointer is NULL");
    if (r > NMFCU_MAX_WIDE_RANK)
        return fail(NMFCU_ERR_UNSUPPORTED, "rank " + std::to_string(r) +
                                               " exceeds the largest supported rank (" +
                                               std::to_string(NMFCU_MAX_WIDE_RANK) + ")");
    if (o->method != NMFCU_LEE && o->method != NMFCU_BRUNET && o->method != NMFCU_HALS &&
        o->method != NMFCU_DNMF)
        return fail(NMFCU_ERR_UNSUPPORTED,
                    "ranks above " + std::to_string(NMFCU_MAX_RANK) +
                        " run lee, brunet, hals and dnmf");
    if (o->precision != NMFCU_PREC_FP64)
        return fail(NMFCU_ERR_UNSUPPORTED,
                    "ranks above " + std::to_string(NMFCU_MAX_RANK) + " run in FP64 only");
    return validate_options_rank(o, n, p, r, NMFCU_MAX_WIDE_RANK);
}

// The loop at a rank above NMFCU_MAX_RANK, V f64 n x p (pitch ldv, a
// 16-byte aligned base and pitch) on the device.  W0 (n x r) and H0 (r x p)
// are read with `in_kind`, W and H written with `out_kind` (host or device
// copies; they may alias W0 / H0); d_dev: device deviances (or NULL).  The
// caller holds the context's mutex with its device current and has checked
// the options (wide_validate).
nmfcu_status wide_run(nmfcu_context *c, const nmfcu_options *o, int64_t n, int64_t p, int64_t r,
                      const double *V, int64_t ldv, const double *W0, const double *H0,
                      double *W, double *H, cudaMemcpyKind in_kind, cudaMemcpyKind out_kind,
                      double *d_dev, cudaStream_t s, int64_t *n_dev, int64_t *n_iter) {
    const bool stat = o->stop == NMFCU_STOP_STATIONARY;
    // The passes' workspace (and the run state) for the largest chunk.
    NMFCU_TRY(context_prepare(c, n, p));
    RunState *st = static_cast<RunState *>(context_state(c));
    Bufs b;
    NMFCU_TRY(make_bufs(c, o, n, p, (int)r, b));
    NMFCU_CUDA_TRY(cudaMemcpyAsync(b.W, W0, sizeof(double) * (size_t)(n * r), in_kind, s));
    NMFCU_CUDA_TRY(cudaMemcpyAsync(b.H, H0, sizeof(double) * (size_t)(r * p), in_kind, s));
    NMFCU_CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(RunState), s));
    Loop L{c, o, n, p, (int)r, V, ldv, b, st, d_dev, s};
    if (stat) NMFCU_TRY(L.objective(0));
    for (long long it = 1; it <= o->max_iter; it++) {
        NMFCU_TRY(L.iteration(it));
        if (stat) NMFCU_TRY(L.objective(it));
    }
    NMFCU_CUDA_TRY(cudaMemcpyAsync(W, b.W, sizeof(double) * (size_t)(n * r), out_kind, s));
    NMFCU_CUDA_TRY(cudaMemcpyAsync(H, b.H, sizeof(double) * (size_t)(r * p), out_kind, s));
    RunState hs;
    NMFCU_CUDA_TRY(cudaMemcpyAsync(&hs, st, sizeof(RunState), cudaMemcpyDeviceToHost, s));
    NMFCU_CUDA_TRY(cudaStreamSynchronize(s));
    drain_timing(c);
    if (hs.timeout != 0)
        return fail(NMFCU_ERR_TIMEOUT, "a streaming kernel gave up waiting for its copies (code " +
                                           std::to_string(hs.timeout) + ")");
    if (hs.error == 1)
        return fail(NMFCU_ERR_INVALID_ARG,
                    "check_interval must be > 0 (the stationary stop evaluates iter % check_interval)");
    const int64_t iters = hs.stopped ? hs.n_iter : o->max_iter;
    *n_iter = iters;
    *n_dev = stat ? iters + 1 : 0;
    return NMFCU_OK;
}

}  // namespace nmfcu_internal

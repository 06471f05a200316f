// sparse.cu -- the NMF loop on a sparse V given in compressed sparse row
// (CSR) form: lee, brunet, hals and dnmf in FP64, the same updates as the
// dense engine (rust/src/lib.rs nmf_run_lee :1589-1647, nmf_run_brunet
// :1529-1586, nmf_run_hals :638-688, nmf_run_dnmf :827-906).
//
// Single-cell matrices are mostly zeros (AnnData keeps them as CSR); the
// reference densifies V before its loop (python/nmf_rs/__init__.py:495).
// Every V term of the updates is zero at an unstored entry:
//   lee / hals / dnmf  W^T V and V H^T are sums over the stored entries;
//   brunet             V / (W H) is 0 where V is 0 (lib.rs:89-97, 181-189),
//                      so W H is formed only at the stored entries;
// the denominators (W^T W, H H^T, colsum(W), rowsum(H)) do not involve V.
// The objectives split into a stored-entry pass plus closed forms:
//   KL   sum_stored,v>0 [v ln(v/wh) - v + wh] + (sum_all wh - sum_stored,v>0 wh),
//        sum_all wh = sum_k colsum(W)_k rowsum(H)_k     (lib.rs:1410-1431)
//   Fro  sum_stored [(v - wh)^2 - wh^2] + ||W H||^2,
//        ||W H||^2 = sum_kl (W^T W)_kl (H H^T)_kl        (lib.rs:1434-1445)
//
// Passes (one warp a line, lanes across its stored entries, a fixed
// butterfly reduction, so results are bit-reproducible run to run):
//   W pass  rows of the CSR:     out[i][k] = sum_t f(v_t) H^T[j_t][k]
//   H pass  columns of a CSC copy made once a run (a stable radix sort of
//           the column indices, so each column lists its rows in order):
//                                out[k][j] = sum_t f(v_t) W[i_t][k]
// with f(v) = v, or v / (W H)_ij for brunet (0 where W H is 0).  The outputs
// have the layouts of the dense engine's one-split epilogue partials, so its
// update epilogues (h_epilogue / w_epilogue), Grams, rescaling, clamp and
// stationary stop run unchanged.  Bytes per pass: nnz x 12 (value + index)
// plus the factor rows gathered from L2 (W: n x RP, H^T: p x RP f64).
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <string>
#include <vector>

#include "../../include/nmfcu.h"
#include "internal.h"
#include "kernels.cuh"

using nmfcu_internal::fail;

namespace {

using nmfcu::RunState;
using nmfcu::EpiParams;
constexpr int kT = nmfcu::kThreads;  // 256

// Context scratch slots of this file.
constexpr int kSlotCsr = 18;    // host entry: the uploaded CSR
constexpr int kSlotCsc = 19;    // the CSC copy
constexpr int kSlotSort = 20;   // the radix sort's buffers (CSC build only)
constexpr int kSlotFac = 21;    // padded W, H, H^T and the two contractions
constexpr int kSlotSmall = 22;  // Grams, sums, objective partials, state, deviances
constexpr int kSlotCheck = 23;  // validation flags of the device entry

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }
inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

int bucket_for(int64_t r) {
    static const int b[] = {2, 4, 6, 8, 10, 12, 14, 16, 20, 24, 28, 32};
    for (int v : b)
        if (r <= v) return v;
    return -1;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// rows_of[t] = the row of stored entry t.
__global__ void csr_rows_of(const int64_t *__restrict__ indptr, int n, int32_t *__restrict__ rows) {
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)(((int64_t)gridDim.x * blockDim.x) >> 5);
    for (int i = gw; i < n; i += nw)
        for (int64_t t = indptr[i] + lane; t < indptr[i + 1]; t += 32) rows[t] = i;
}

__global__ void iota32(int32_t *__restrict__ x, int64_t nnz) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnz;
         t += (int64_t)gridDim.x * blockDim.x)
        x[t] = (int32_t)t;
}

// The CSC copy from the sorted column keys and the permutation of the sort.
__global__ void csc_gather(const int32_t *__restrict__ perm, const int32_t *__restrict__ rows_of,
                           const double *__restrict__ data, int32_t *__restrict__ rows,
                           double *__restrict__ vals, int64_t nnz) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnz;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t src = perm[t];
        rows[t] = rows_of[src];
        vals[t] = data[src];
    }
}

// colptr[c] = first position of column c in the sorted keys (empty columns
// included); thread t = nnz closes the columns after the last key.
__global__ void csc_colptr(const int32_t *__restrict__ keys, int64_t nnz, int p,
                           int64_t *__restrict__ colptr) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t <= nnz;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int prev = (t == 0) ? -1 : keys[t - 1];
        const int cur = (t == nnz) ? p : keys[t];
        for (int c = prev + 1; c <= cur; c++) colptr[c] = t;
    }
}

// Checks a device CSR: indptr[0] == 0, non-decreasing, indptr[n] == nnz, and
// every column index in [0, p).  flags[0] = 1 on a bad indptr, flags[1] = 1
// on a bad index (flags cleared by the caller).
__global__ void csr_check(const int64_t *__restrict__ indptr, int n, const int32_t *__restrict__ idx,
                          int64_t nnz, int p, int *__restrict__ flags) {
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = tid; i <= n; i += stride) {
        const int64_t v = indptr[i];
        if ((i == 0 && v != 0) || (i == n && v != nnz) || v < 0 || v > nnz ||
            (i > 0 && indptr[i - 1] > v))
            flags[0] = 1;
    }
    for (int64_t t = tid; t < nnz; t += stride) {
        const int32_t j = idx[t];
        if (j < 0 || j >= p) flags[1] = 1;
    }
}

// The contraction over the stored entries of each line (a CSR row for the W
// pass, a CSC column for the H pass), one warp a line:
//   out[m][k] = sum_t f(v_t) F[x_t][k],  f(v) = v, or v / (sum_k G[m][k] F[x_t][k])
// (0 where that is 0) when RATIO.  G: the line's own factor rows (lines x
// RP), F: the rows the stored entries index.  OUT_KM writes out[k * ldo + m]
// (the H epilogue's [RP][p] layout), else out[m * RP + k].
template <int RP, bool RATIO, bool OUT_KM>
__global__ void __launch_bounds__(kT)
    sparse_pass(const int64_t *__restrict__ ptr, const int32_t *__restrict__ idx,
                const double *__restrict__ val, int lines, int64_t ldo,
                const double *__restrict__ G, const double *__restrict__ F,
                double *__restrict__ out, const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)(((int64_t)gridDim.x * blockDim.x) >> 5);
    for (int m = gw; m < lines; m += nw) {
        double g[RATIO ? RP : 1];
        if (RATIO) {
            const double2 *g2 = reinterpret_cast<const double2 *>(G + (int64_t)m * RP);
#pragma unroll
            for (int k = 0; k < RP / 2; k++) {
                const double2 x = g2[k];
                g[2 * k] = x.x;
                g[2 * k + 1] = x.y;
            }
        }
        double acc[RP];
#pragma unroll
        for (int k = 0; k < RP; k++) acc[k] = 0.0;
        const int64_t t1 = ptr[m + 1];
        for (int64_t t = ptr[m] + lane; t < t1; t += 32) {
            const int x = idx[t];
            const double v = val[t];
            const double2 *f2 = reinterpret_cast<const double2 *>(F + (int64_t)x * RP);
            double f[RP];
#pragma unroll
            for (int k = 0; k < RP / 2; k++) {
                const double2 y = __ldg(f2 + k);
                f[2 * k] = y.x;
                f[2 * k + 1] = y.y;
            }
            double q = v;
            if (RATIO) {
                double wh = 0.0;
#pragma unroll
                for (int k = 0; k < RP; k++) wh = fma(g[k], f[k], wh);
                q = (wh != 0.0) ? nmfcu::ratio_div(v, wh) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < RP; k++) acc[k] = fma(q, f[k], acc[k]);
        }
        double mine = 0.0;
#pragma unroll
        for (int k = 0; k < RP; k++) {
            double a = acc[k];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
            if (lane == k) mine = a;
        }
        if (lane < RP) {
            if (OUT_KM)
                out[(int64_t)lane * ldo + m] = mine;
            else
                out[(int64_t)m * RP + lane] = mine;
        }
    }
}

// Stored-entry part of the objective, one warp a CSR row; per block two
// partials: part[2 b] the stored terms, part[2 b + 1] (KL) the sum of W H
// over the stored entries with v > 0.
template <int RP, bool KL>
__global__ void __launch_bounds__(kT)
    sparse_objective(const int64_t *__restrict__ ptr, const int32_t *__restrict__ idx,
                     const double *__restrict__ val, int n, const double *__restrict__ W,
                     const double *__restrict__ Ht, double *__restrict__ part,
                     const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gw = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)(((int64_t)gridDim.x * blockDim.x) >> 5);
    double a = 0.0, b = 0.0;
    for (int i = gw; i < n; i += nw) {
        double w[RP];
        const double2 *w2 = reinterpret_cast<const double2 *>(W + (int64_t)i * RP);
#pragma unroll
        for (int k = 0; k < RP / 2; k++) {
            const double2 x = w2[k];
            w[2 * k] = x.x;
            w[2 * k + 1] = x.y;
        }
        const int64_t t1 = ptr[i + 1];
        for (int64_t t = ptr[i] + lane; t < t1; t += 32) {
            const double2 *h2 = reinterpret_cast<const double2 *>(Ht + (int64_t)idx[t] * RP);
            double wh = 0.0;
#pragma unroll
            for (int k = 0; k < RP / 2; k++) {
                const double2 y = __ldg(h2 + k);
                wh = fma(w[2 * k], y.x, wh);
                wh = fma(w[2 * k + 1], y.y, wh);
            }
            const double v = val[t];
            if (KL) {
                if (v > 0.0) {
                    if (wh > 0.0) a += v * log(v / wh) - v + wh;
                    b += wh;
                }
            } else {
                const double d = v - wh;
                a += d * d - wh * wh;
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, off);
        b += __shfl_xor_sync(0xffffffffu, b, off);
    }
    __shared__ double ra[kT / 32], rb[kT / 32];
    if (lane == 0) {
        ra[warp] = a;
        rb[warp] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0.0, sb = 0.0;
        for (int w = 0; w < kT / 32; w++) {
            sa += ra[w];
            sb += rb[w];
        }
        part[2 * blockIdx.x] = sa;
        part[2 * blockIdx.x + 1] = sb;
    }
}

// obj[0] = the objective before its scale: the stored-entry partials (in
// block order) plus the closed-form part over all entries.
template <int RP, bool KL>
__global__ void sparse_objective_combine(const double *__restrict__ part, int B, int r,
                                         const double *__restrict__ Gw, const double *__restrict__ sw,
                                         const double *__restrict__ Gh, const double *__restrict__ sh,
                                         double *__restrict__ obj, const RunState *st) {
    if (nmfcu::run_stopped(st)) return;
    __shared__ double ra[kT], rb[kT];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < B; i += kT) {
        a += part[2 * i];
        b += part[2 * i + 1];
    }
    ra[threadIdx.x] = a;
    rb[threadIdx.x] = b;
    __syncthreads();
    for (int s = kT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            ra[threadIdx.x] += ra[threadIdx.x + s];
            rb[threadIdx.x] += rb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    double dense = 0.0;
    if (KL) {
        for (int k = 0; k < r; k++) dense += sw[k] * sh[k];  // sum of W H over all entries
        obj[0] = ra[0] + (dense - rb[0]);
    } else {
        for (int k = 0; k < r; k++)
            for (int l = 0; l < r; l++) dense += Gw[k * RP + l] * Gh[k * RP + l];  // ||W H||^2
        obj[0] = ra[0] + dense;
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

// Device views of one run.
struct SparseV {
    const int64_t *rptr;   // CSR
    const int32_t *ridx;
    const double *rval;
    int64_t *cptr;         // CSC copy
    int32_t *cidx;
    double *cval;
    int64_t nnz;
};

struct Work {
    double *W, *H, *Ht, *numW, *numH;          // padded factors, contractions
    double *pg, *ps, *Gw, *sw, *Gh, *sh, *Gw2, *sw2;
    double *opart, *obj, *dev;
    RunState *st;
    int Bw, rows_per_gram, Bh, cols_per_gram, Bo;
};

// Carves `sizes` (bytes) out of one context slot, 256-byte aligned.
nmfcu_status carve(nmfcu_context *c, int slot, const std::vector<size_t> &sizes,
                   std::vector<void *> &out) {
    size_t total = 0;
    for (size_t b : sizes) total += align256(std::max<size_t>(b, 1));
    void *base = nullptr;
    NMFCU_TRY(nmfcu_internal::context_buffer(c, slot, total, &base));
    out.clear();
    char *p = static_cast<char *>(base);
    for (size_t b : sizes) {
        out.push_back(p);
        p += align256(std::max<size_t>(b, 1));
    }
    return NMFCU_OK;
}

// The CSC copy of the CSR (stable radix sort of the column indices).
nmfcu_status build_csc(nmfcu_context *c, int64_t n, int64_t p, SparseV &sv, cudaStream_t s) {
    const int64_t nnz = sv.nnz;
    int bits = 1;
    while (bits < 31 && ((int64_t)1 << bits) < p) bits++;
    size_t temp = 0;
    NMFCU_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp, (const int32_t *)nullptr,
                                                   (int32_t *)nullptr, (const int32_t *)nullptr,
                                                   (int32_t *)nullptr, (int)std::max<int64_t>(nnz, 1),
                                                   0, bits, s));
    std::vector<void *> b;
    const size_t i4 = sizeof(int32_t) * (size_t)nnz;
    NMFCU_TRY(carve(c, kSlotSort, {i4, i4, i4, i4, temp}, b));
    int32_t *keys_out = static_cast<int32_t *>(b[0]);
    int32_t *perm_in = static_cast<int32_t *>(b[1]);
    int32_t *perm = static_cast<int32_t *>(b[2]);
    int32_t *rows_of = static_cast<int32_t *>(b[3]);
    std::vector<void *> cb;
    NMFCU_TRY(carve(c, kSlotCsc, {sizeof(int64_t) * (size_t)(p + 1), i4, sizeof(double) * (size_t)nnz}, cb));
    sv.cptr = static_cast<int64_t *>(cb[0]);
    sv.cidx = static_cast<int32_t *>(cb[1]);
    sv.cval = static_cast<double *>(cb[2]);
    const int sms = nmfcu_internal::context_sms(c);
    const unsigned gb = std::max(1u, std::min<unsigned>(cdiv(std::max<int64_t>(nnz, 1), kT), (unsigned)sms * 16));
    nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_OTHER, 5);
    if (nnz > 0) {
        iota32<<<gb, kT, 0, s>>>(perm_in, nnz);
        NMFCU_CUDA_TRY(cub::DeviceRadixSort::SortPairs(b[4], temp, sv.ridx, keys_out, perm_in, perm,
                                                       (int)nnz, 0, bits, s));
        if (n > 0)
            csr_rows_of<<<std::max(1u, std::min<unsigned>(cdiv(n, kT / 32), (unsigned)sms * 16)), kT, 0, s>>>(
                sv.rptr, (int)n, rows_of);
        csc_gather<<<gb, kT, 0, s>>>(perm, rows_of, sv.rval, sv.cidx, sv.cval, nnz);
    }
    csc_colptr<<<std::max(1u, std::min<unsigned>(cdiv(nnz + 1, kT), (unsigned)sms * 16)), kT, 0, s>>>(
        keys_out, nnz, (int)p, sv.cptr);
    NMFCU_CUDA_TRY(cudaGetLastError());
    return NMFCU_OK;
}

unsigned line_grid(int64_t lines, int sms) {
    return std::max(1u, std::min<unsigned>(cdiv(lines, kT / 32), (unsigned)sms * 8));
}

template <int RP>
struct Loop {
    nmfcu_context *c;
    const nmfcu_options *o;
    int n, p, r;
    SparseV sv;
    Work w;
    cudaStream_t s;
    int sms;

    void transpose_h() {
        if (p <= 0) return;
        nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_OTHER);
        const unsigned blocks =
            std::max(1u, std::min<unsigned>(cdiv((int64_t)p * RP, kT), 4096u));
        nmfcu::h_transpose<double><<<blocks, kT, 0, s>>>(w.H, w.Ht, p, r, RP);
    }
    void gram_w(double *G, double *sums) {
        nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_OTHER, 2);
        nmfcu::gram_w_partial<RP><<<w.Bw, RP * RP, 0, s>>>(w.W, n, w.rows_per_gram, w.pg, w.ps, w.st);
        nmfcu::gram_finalize<RP><<<1, RP * RP, 0, s>>>(w.pg, w.ps, w.Bw, G, sums, w.st);
    }
    void gram_h(double *G, double *sums) {
        nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_OTHER, 2);
        nmfcu::gram_h_partial<RP><<<w.Bh, RP * RP, 0, s>>>(w.H, p, w.cols_per_gram, w.pg, w.ps, w.st);
        nmfcu::gram_finalize<RP><<<1, RP * RP, 0, s>>>(w.pg, w.ps, w.Bh, G, sums, w.st);
    }
    EpiParams epi(const double *G, const double *sums, bool hside) const {
        EpiParams e;
        e.method = o->method;
        e.r = r;
        e.eps = o->eps;
        e.lambda = hside ? o->sparsity_h : o->sparsity_w;
        e.gamma = hside ? o->smoothness_h : o->smoothness_w;
        e.G = G;
        e.sums = sums;
        return e;
    }
    void h_step(bool ratio, const EpiParams &e) {
        if (ratio) transpose_h();
        {
            nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_HSTEP);
            const unsigned g = line_grid(p, sms);
            if (ratio)
                sparse_pass<RP, true, true><<<g, kT, 0, s>>>(sv.cptr, sv.cidx, sv.cval, p, p, w.Ht,
                                                             w.W, w.numH, w.st);
            else
                sparse_pass<RP, false, true><<<g, kT, 0, s>>>(sv.cptr, sv.cidx, sv.cval, p, p,
                                                              nullptr, w.W, w.numH, w.st);
        }
        nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_OTHER);
        nmfcu::h_epilogue<RP><<<std::max(1u, cdiv(p, kT)), kT, 0, s>>>(w.H, p, w.numH, 1, e, w.st);
    }
    void w_step(bool ratio, const EpiParams &e) {
        transpose_h();
        {
            nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_WSTEP);
            const unsigned g = line_grid(n, sms);
            if (ratio)
                sparse_pass<RP, true, false><<<g, kT, 0, s>>>(sv.rptr, sv.ridx, sv.rval, n, 0, w.W,
                                                              w.Ht, w.numW, w.st);
            else
                sparse_pass<RP, false, false><<<g, kT, 0, s>>>(sv.rptr, sv.ridx, sv.rval, n, 0,
                                                               nullptr, w.Ht, w.numW, w.st);
        }
        nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_OTHER);
        nmfcu::w_epilogue<RP><<<std::max(1u, cdiv(n, kT)), kT, 0, s>>>(w.W, n, w.numW, 1, e, w.st);
    }
    void objective(long long iter) {
        const bool kl = (o->method == NMFCU_BRUNET);
        gram_w(w.Gw2, w.sw2);
        gram_h(w.Gh, w.sh);
        transpose_h();
        {
            nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_OBJECTIVE, 2);
            if (kl) {
                sparse_objective<RP, true><<<w.Bo, kT, 0, s>>>(sv.rptr, sv.ridx, sv.rval, n, w.W,
                                                               w.Ht, w.opart, w.st);
                sparse_objective_combine<RP, true><<<1, kT, 0, s>>>(w.opart, w.Bo, r, w.Gw2, w.sw2,
                                                                    w.Gh, w.sh, w.obj, w.st);
            } else {
                sparse_objective<RP, false><<<w.Bo, kT, 0, s>>>(sv.rptr, sv.ridx, sv.rval, n, w.W,
                                                                w.Ht, w.opart, w.st);
                sparse_objective_combine<RP, false><<<1, kT, 0, s>>>(w.opart, w.Bo, r, w.Gw2,
                                                                     w.sw2, w.Gh, w.sh, w.obj, w.st);
            }
        }
        nmfcu::StopParams sp;
        sp.stationary = 1;
        sp.iter = iter;
        sp.check_interval = o->check_interval;
        sp.check_niter = o->check_niter;
        sp.threshold = o->stationary_th;
        sp.scale = kl ? 1.0 : 0.5;
        nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_OTHER);
        nmfcu::objective_finalize<<<1, kT, 0, s>>>(w.obj, 1, w.dev, sp, w.st);
    }
    void iteration(long long it) {
        switch (o->method) {
            case NMFCU_BRUNET:
                // nmf_run_brunet lib.rs:1558-1575
                gram_w(w.Gw, w.sw);
                h_step(true, epi(w.Gw, w.sw, true));
                gram_h(w.Gh, w.sh);
                w_step(true, epi(w.Gh, w.sh, false));
                if (it % 10 == 0) {
                    nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_OTHER);
                    const int64_t m = std::max<int64_t>((int64_t)n * RP, (int64_t)r * p);
                    nmfcu::clamp_wh<RP><<<std::max(1u, std::min<unsigned>(cdiv(m, kT), 1184u)), kT, 0, s>>>(
                        w.W, w.H, n, p, r, DBL_EPSILON, w.st);
                }
                break;
            case NMFCU_LEE:
                // nmf_run_lee lib.rs:1618-1636
                gram_w(w.Gw, w.sw);
                h_step(false, epi(w.Gw, w.sw, true));
                gram_h(w.Gh, w.sh);
                w_step(false, epi(w.Gh, w.sh, false));
                if (o->rescale && n > 0) {
                    nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_OTHER, 2);
                    nmfcu::gram_w_partial<RP><<<w.Bw, RP * RP, 0, s>>>(w.W, n, w.rows_per_gram,
                                                                       w.pg, w.ps, w.st);
                    nmfcu::col_rescale<RP><<<std::min<unsigned>(cdiv((int64_t)n * RP, kT), 1184u), kT, 0, s>>>(
                        w.W, n, r, w.ps, w.Bw, w.st);
                }
                break;
            default:
                // nmf_run_hals lib.rs:667-676; nmf_run_dnmf lib.rs:862-884
                gram_w(w.Gw, w.sw);
                h_step(false, epi(w.Gw, w.sw, true));
                gram_h(w.Gh, w.sh);
                w_step(false, epi(w.Gh, w.sh, false));
                if (o->method == NMFCU_DNMF) {
                    gram_w(w.Gw2, w.sw2);
                    nmfcu_internal::TimedScope sc(c, s, NMFCU_KCLASS_OTHER);
                    const int64_t m = std::max<int64_t>((int64_t)n * RP, (int64_t)r * p);
                    nmfcu::dnmf_rescale<RP><<<std::max(1u, std::min<unsigned>(cdiv(m, kT), 1184u)), kT, 0, s>>>(
                        w.W, w.H, n, p, r, w.Gw2, w.Gh, w.st);
                }
                break;
        }
    }
};

// Workspace of a run: padded factors and contractions (slot kSlotFac), the
// small buffers (slot kSlotSmall).
nmfcu_status make_work(nmfcu_context *c, int64_t n, int64_t p, int RP, int64_t max_iter,
                       Work &w) {
    const int sms = nmfcu_internal::context_sms(c);
    std::vector<void *> b;
    const size_t d = sizeof(double);
    NMFCU_TRY(carve(c, kSlotFac, {d * n * RP, d * RP * p, d * p * RP, d * n * RP, d * RP * p}, b));
    w.W = static_cast<double *>(b[0]);
    w.H = static_cast<double *>(b[1]);
    w.Ht = static_cast<double *>(b[2]);
    w.numW = static_cast<double *>(b[3]);
    w.numH = static_cast<double *>(b[4]);
    w.Bw = (int)std::max<int64_t>(1, std::min<int64_t>((n + 63) / 64, sms));
    w.rows_per_gram = (int)std::max<int64_t>(1, (n + w.Bw - 1) / w.Bw);
    w.Bh = (int)std::max<int64_t>(1, std::min<int64_t>((p + 63) / 64, sms));
    w.cols_per_gram = (int)std::max<int64_t>(1, (p + w.Bh - 1) / w.Bh);
    w.Bo = (int)line_grid(n, sms);
    const int B = std::max(w.Bw, w.Bh);
    const size_t g = d * RP * RP, v = d * RP;
    NMFCU_TRY(carve(c, kSlotSmall,
                    {d * B * RP * RP, d * B * RP, g, v, g, v, g, v, d * 2 * w.Bo, d * 8,
                     sizeof(RunState), d * (size_t)(max_iter + 1)},
                    b));
    w.pg = static_cast<double *>(b[0]);
    w.ps = static_cast<double *>(b[1]);
    w.Gw = static_cast<double *>(b[2]);
    w.sw = static_cast<double *>(b[3]);
    w.Gh = static_cast<double *>(b[4]);
    w.sh = static_cast<double *>(b[5]);
    w.Gw2 = static_cast<double *>(b[6]);
    w.sw2 = static_cast<double *>(b[7]);
    w.opart = static_cast<double *>(b[8]);
    w.obj = static_cast<double *>(b[9]);
    w.st = static_cast<RunState *>(b[10]);
    w.dev = static_cast<double *>(b[11]);
    return NMFCU_OK;
}

template <int RP>
nmfcu_status run_loop_t(nmfcu_context *c, const nmfcu_options *o, int64_t n, int64_t p, int64_t r,
                        SparseV sv, Work w, cudaStream_t s, bool stat, int64_t *n_dev,
                        int64_t *n_iter) {
    Loop<RP> L{c, o, (int)n, (int)p, (int)r, sv, w, s, nmfcu_internal::context_sms(c)};
    NMFCU_CUDA_TRY(cudaMemsetAsync(w.st, 0, sizeof(RunState), s));
    if (stat) L.objective(0);
    for (long long it = 1; it <= o->max_iter; it++) {
        L.iteration(it);
        if (stat) L.objective(it);
    }
    NMFCU_CUDA_TRY(cudaGetLastError());
    RunState hs;
    NMFCU_CUDA_TRY(cudaMemcpyAsync(&hs, w.st, sizeof(RunState), cudaMemcpyDeviceToHost, s));
    NMFCU_CUDA_TRY(cudaStreamSynchronize(s));
    nmfcu_internal::drain_timing(c);
    if (hs.error == 1)
        return fail(NMFCU_ERR_INVALID_ARG,
                    "check_interval must be > 0 (the stationary stop evaluates iter % check_interval)");
    const int64_t iters = hs.stopped ? hs.n_iter : o->max_iter;
    *n_iter = iters;
    *n_dev = stat ? iters + 1 : 0;
    return NMFCU_OK;
}

nmfcu_status run_loop(int RP, nmfcu_context *c, const nmfcu_options *o, int64_t n, int64_t p,
                      int64_t r, const SparseV &sv, const Work &w, cudaStream_t s, bool stat,
                      int64_t *n_dev, int64_t *n_iter) {
    switch (RP) {
#define NMFCU_SPARSE_CASE(R) \
    case R: return run_loop_t<R>(c, o, n, p, r, sv, w, s, stat, n_dev, n_iter);
        NMFCU_SPARSE_CASE(2)
        NMFCU_SPARSE_CASE(4)
        NMFCU_SPARSE_CASE(6)
        NMFCU_SPARSE_CASE(8)
        NMFCU_SPARSE_CASE(10)
        NMFCU_SPARSE_CASE(12)
        NMFCU_SPARSE_CASE(14)
        NMFCU_SPARSE_CASE(16)
        NMFCU_SPARSE_CASE(20)
        NMFCU_SPARSE_CASE(24)
        NMFCU_SPARSE_CASE(28)
        NMFCU_SPARSE_CASE(32)
#undef NMFCU_SPARSE_CASE
        default: return fail(NMFCU_ERR_UNSUPPORTED, "rank bucket");
    }
}

nmfcu_status validate_csr_options(const nmfcu_options *o, int64_t n, int64_t p, int64_t r,
                                  int64_t nnz) {
    NMFCU_TRY(nmfcu_internal::validate_options(o, n, p, r));
    if (o->method != NMFCU_LEE && o->method != NMFCU_BRUNET && o->method != NMFCU_HALS &&
        o->method != NMFCU_DNMF)
        return fail(NMFCU_ERR_UNSUPPORTED,
                    "a sparse (CSR) V runs lee, brunet, hals and dnmf; densify V for the others");
    if (o->precision != NMFCU_PREC_FP64)
        return fail(NMFCU_ERR_UNSUPPORTED, "a sparse (CSR) V runs in FP64 only");
    if (nnz < 0) return fail(NMFCU_ERR_INVALID_ARG, "nnz must be >= 0");
    if (nnz > INT32_MAX)
        return fail(NMFCU_ERR_UNSUPPORTED, "nnz must fit in 31 bits (2147483647 stored entries)");
    return NMFCU_OK;
}

// Upload of the padded factors (W n x r -> n x RP, H r x p -> RP x p).
nmfcu_status put_factors(const Work &w, int64_t n, int64_t p, int64_t r, int RP, const double *W,
                         const double *H, cudaMemcpyKind kind, cudaStream_t s) {
    NMFCU_CUDA_TRY(cudaMemsetAsync(w.W, 0, sizeof(double) * (size_t)n * RP, s));
    NMFCU_CUDA_TRY(cudaMemsetAsync(w.H, 0, sizeof(double) * (size_t)RP * p, s));
    if (n > 0)
        NMFCU_CUDA_TRY(cudaMemcpy2DAsync(w.W, RP * sizeof(double), W, r * sizeof(double),
                                         r * sizeof(double), n, kind, s));
    if (p > 0) NMFCU_CUDA_TRY(cudaMemcpyAsync(w.H, H, sizeof(double) * (size_t)r * p, kind, s));
    return NMFCU_OK;
}
nmfcu_status get_factors(const Work &w, int64_t n, int64_t p, int64_t r, int RP, double *W,
                         double *H, cudaMemcpyKind kind, cudaStream_t s) {
    if (n > 0)
        NMFCU_CUDA_TRY(cudaMemcpy2DAsync(W, r * sizeof(double), w.W, RP * sizeof(double),
                                         r * sizeof(double), n, kind, s));
    if (p > 0) NMFCU_CUDA_TRY(cudaMemcpyAsync(H, w.H, sizeof(double) * (size_t)r * p, kind, s));
    return NMFCU_OK;
}

// The loop on a CSR already on the device; factors in/out through W, H
// (host or device per `kind`), deviances to `dev_out` (host or device).
nmfcu_status run_csr(nmfcu_context *c, const nmfcu_options *o, int64_t n, int64_t p, int64_t r,
                     SparseV sv, const double *W0, const double *H0, double *W, double *H,
                     double *dev_out, cudaMemcpyKind in_kind, cudaMemcpyKind out_kind,
                     cudaStream_t s, int64_t *n_dev, int64_t *n_iter) {
    const int RP = bucket_for(r);
    const bool stat = o->stop == NMFCU_STOP_STATIONARY;
    NMFCU_TRY(build_csc(c, n, p, sv, s));
    Work w;
    NMFCU_TRY(make_work(c, n, p, RP, o->max_iter, w));
    NMFCU_TRY(put_factors(w, n, p, r, RP, W0, H0, in_kind, s));
    int64_t nd = 0, ni = 0;
    NMFCU_TRY(run_loop(RP, c, o, n, p, r, sv, w, s, stat, &nd, &ni));
    NMFCU_TRY(get_factors(w, n, p, r, RP, W, H, out_kind, s));
    if (stat && nd > 0 && dev_out)
        NMFCU_CUDA_TRY(cudaMemcpyAsync(dev_out, w.dev, sizeof(double) * (size_t)nd,
                                       out_kind == cudaMemcpyDeviceToHost ? cudaMemcpyDeviceToHost
                                                                          : cudaMemcpyDeviceToDevice,
                                       s));
    NMFCU_CUDA_TRY(cudaStreamSynchronize(s));
    *n_dev = nd;
    *n_iter = ni;
    return NMFCU_OK;
}

}  // namespace

extern "C" {

nmfcu_status nmfcu_run_csr(const nmfcu_options *opt, int64_t n, int64_t p, int64_t r, int64_t nnz,
                           const int64_t *indptr, const int32_t *indices, const double *data,
                           const double *W0, const double *H0, double *W, double *H,
                           double *deviances, int64_t deviances_cap, int64_t *n_deviances,
                           int64_t *n_iter) {
    NMFCU_TRY(validate_csr_options(opt, n, p, r, nnz));
    if (!indptr || (nnz > 0 && (!indices || !data)) || !W0 || !H0 || !W || !H || !n_deviances ||
        !n_iter)
        return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    const bool stat = opt->stop == NMFCU_STOP_STATIONARY;
    if (stat && (!deviances || deviances_cap < opt->max_iter + 1))
        return fail(NMFCU_ERR_INVALID_ARG, "deviances must hold max_iter + 1 values");
    // The CSR's structure, on the host (the kernels index with it).
    if (indptr[0] != 0 || indptr[n] != nnz)
        return fail(NMFCU_ERR_INVALID_ARG, "indptr must start at 0 and end at nnz");
    for (int64_t i = 0; i < n; i++)
        if (indptr[i + 1] < indptr[i])
            return fail(NMFCU_ERR_INVALID_ARG, "indptr must be non-decreasing");
    for (int64_t t = 0; t < nnz; t++)
        if (indices[t] < 0 || indices[t] >= p)
            return fail(NMFCU_ERR_INVALID_ARG,
                        "column index " + std::to_string(indices[t]) + " outside [0, p)");
    nmfcu_context *c = nullptr;
    NMFCU_TRY(nmfcu_internal::default_context(opt->device, &c));
    std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(c));
    nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(c));
    cudaStream_t s = nmfcu_internal::context_stream(c);
    std::vector<void *> b;
    NMFCU_TRY(carve(c, kSlotCsr,
                    {sizeof(int64_t) * (size_t)(n + 1), sizeof(int32_t) * (size_t)nnz,
                     sizeof(double) * (size_t)nnz},
                    b));
    NMFCU_CUDA_TRY(cudaMemcpyAsync(b[0], indptr, sizeof(int64_t) * (size_t)(n + 1),
                                   cudaMemcpyHostToDevice, s));
    if (nnz > 0) {
        NMFCU_CUDA_TRY(cudaMemcpyAsync(b[1], indices, sizeof(int32_t) * (size_t)nnz,
                                       cudaMemcpyHostToDevice, s));
        NMFCU_CUDA_TRY(cudaMemcpyAsync(b[2], data, sizeof(double) * (size_t)nnz,
                                       cudaMemcpyHostToDevice, s));
    }
    SparseV sv{static_cast<const int64_t *>(b[0]), static_cast<const int32_t *>(b[1]),
               static_cast<const double *>(b[2]), nullptr, nullptr, nullptr, nnz};
    return run_csr(c, opt, n, p, r, sv, W0, H0, W, H, deviances, cudaMemcpyHostToDevice,
                   cudaMemcpyDeviceToHost, s, n_deviances, n_iter);
}

nmfcu_status nmfcu_run_csr_device(nmfcu_context *ctx, const nmfcu_options *opt, int64_t n,
                                  int64_t p, int64_t r, int64_t nnz, const int64_t *d_indptr,
                                  const int32_t *d_indices, const double *d_data, double *dW,
                                  double *dH, double *d_dev, int64_t *n_deviances,
                                  int64_t *n_iter, void *stream) {
    if (!ctx) return fail(NMFCU_ERR_INVALID_ARG, "context is NULL");
    NMFCU_TRY(validate_csr_options(opt, n, p, r, nnz));
    if (!d_indptr || (nnz > 0 && (!d_indices || !d_data)) || !dW || !dH || !n_deviances ||
        !n_iter)
        return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(ctx));
    nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(ctx));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The CSR's structure is checked on the device before any kernel
    // indexes with it.
    void *fl = nullptr;
    NMFCU_TRY(nmfcu_internal::context_buffer(ctx, kSlotCheck, 2 * sizeof(int), &fl));
    NMFCU_CUDA_TRY(cudaMemsetAsync(fl, 0, 2 * sizeof(int), s));
    {
        nmfcu_internal::TimedScope sc(ctx, s, NMFCU_KCLASS_OTHER);
        const int sms = nmfcu_internal::context_sms(ctx);
        csr_check<<<std::max(1u, std::min<unsigned>(cdiv(std::max(n + 1, nnz), kT), (unsigned)sms * 8)), kT, 0, s>>>(
            d_indptr, (int)n, d_indices, nnz, (int)p, static_cast<int *>(fl));
    }
    int hf[2] = {0, 0};
    NMFCU_CUDA_TRY(cudaMemcpyAsync(hf, fl, sizeof(hf), cudaMemcpyDeviceToHost, s));
    NMFCU_CUDA_TRY(cudaStreamSynchronize(s));
    if (hf[0])
        return fail(NMFCU_ERR_INVALID_ARG,
                    "indptr must start at 0, be non-decreasing and end at nnz");
    if (hf[1]) return fail(NMFCU_ERR_INVALID_ARG, "a column index lies outside [0, p)");
    SparseV sv{d_indptr, d_indices, d_data, nullptr, nullptr, nullptr, nnz};
    return run_csr(ctx, opt, n, p, r, sv, dW, dH, dW, dH, d_dev, cudaMemcpyDeviceToDevice,
                   cudaMemcpyDeviceToDevice, s, n_deviances, n_iter);
}

}  // extern "C"

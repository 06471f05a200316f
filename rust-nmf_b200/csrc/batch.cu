// batch.cu -- many brunet (KL) solves on one shared V in one stream of
// graph-launched kernels: random restarts and a rank sweep, the consensus
// workflow that the reference runs as a serial Python loop of nmf() calls
// (examples/build_scaling_notebook.py:157-208).
//
// Layout: the factors of all solves are stacked -- W_all is n x R_total with
// solve s in columns [off_s, off_s + r_s), H_all is R_total x p with solve s
// in rows [off_s, off_s + r_s).  Solves of one rank form a class; a CTA
// takes NS solves of a class and one tile of V, so each V element it loads
// serves NS solves (V itself stays L2-resident across the classes).  Each
// CTA owns its outputs completely (all rows of a column tile in the H step,
// all columns of a row tile in the W step), so the update epilogue is fused
// and no partial sums leave the CTA.
//
// One iteration is exactly nmf_run_brunet's (rust/src/lib.rs:1558-1575):
// colsum(W) -> H update -> rowsum(H') -> W update -> every 10th iteration
// clamp both factors at DBL_EPSILON.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "../../include/nmfcu.h"
#include "internal.h"

using nmfcu_internal::fail;

namespace {

constexpr int kMaxBatchRank = 16;  // largest rank of a batched solve
constexpr int kRowChunk = 64;      // W rows staged per chunk (H step)

__device__ __forceinline__ double bdiv(double x, double y) { return x / y; }
__device__ __forceinline__ float bdiv(float x, float y) { return __fdividef(x, y); }

// Solves of rank R per CTA: enough that each V load serves ~32 (f32) or
// ~16 (f64) rank components.
template <typename T, int R>
struct BCfg {
    static constexpr int kComponents = sizeof(T) == 4 ? 32 : 16;
    static constexpr int NS = kComponents / R > 0 ? kComponents / R : 1;
};

// H update of a group of NS rank-R solves for 256 columns.
//   off[g * NS + i]: first stacked index of the group's i-th solve (or -1).
template <typename T, int R>
__global__ void __launch_bounds__(256)
    batch_hstep(const T *__restrict__ V, int64_t ldv, int n, int p, const T *__restrict__ W,
                int ldw, T *__restrict__ H, const T *__restrict__ sumW,
                const int *__restrict__ off) {
    constexpr int NS = BCfg<T, R>::NS;
    __shared__ T sW[kRowChunk][NS * R];
    const int j = blockIdx.x * 256 + threadIdx.x;
    const bool colok = j < p;
    const int *goff = off + blockIdx.y * NS;
    int o[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) o[s] = goff[s];
    T hcol[NS][R], acc[NS][R];
#pragma unroll
    for (int s = 0; s < NS; s++)
#pragma unroll
        for (int k = 0; k < R; k++) {
            hcol[s][k] = (colok && o[s] >= 0) ? H[(size_t)(o[s] + k) * p + j] : (T)0;
            acc[s][k] = (T)0;
        }
    for (int base = 0; base < n; base += kRowChunk) {
        const int rows = min(kRowChunk, n - base);
        __syncthreads();
        for (int e = threadIdx.x; e < kRowChunk * NS * R; e += 256) {
            const int rr = e / (NS * R), c = e - rr * (NS * R);
            const int s = c / R, k = c - s * R;
            sW[rr][c] = (rr < rows && o[s] >= 0) ? W[(size_t)(base + rr) * ldw + o[s] + k] : (T)0;
        }
        __syncthreads();
        for (int rr = 0; rr < rows; rr += 4) {
            T v[4];
#pragma unroll
            for (int q = 0; q < 4; q++)
                v[q] = (colok && rr + q < rows) ? V[(size_t)(base + rr + q) * ldv + j] : (T)0;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (rr + q >= rows) break;
                const T *wr = sW[rr + q];
#pragma unroll
                for (int s = 0; s < NS; s++) {
                    T wh = (T)0;
#pragma unroll
                    for (int k = 0; k < R; k++) wh = fma(wr[s * R + k], hcol[s][k], wh);
                    const T qv = (wh != (T)0) ? bdiv(v[q], wh) : (T)0;
#pragma unroll
                    for (int k = 0; k < R; k++) acc[s][k] = fma(wr[s * R + k], qv, acc[s][k]);
                }
            }
        }
    }
    if (!colok) return;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        if (o[s] < 0) continue;
#pragma unroll
        for (int k = 0; k < R; k++)  // h * tmp / sum_w (lib.rs:110)
            H[(size_t)(o[s] + k) * p + j] = (hcol[s][k] * acc[s][k]) / sumW[o[s] + k];
    }
}

// W update of a group of NS rank-R solves for 256 rows.
template <typename T, int R>
__global__ void __launch_bounds__(256)
    batch_wstep(const T *__restrict__ V, int64_t ldv, int n, int p, T *__restrict__ W, int ldw,
                const T *__restrict__ H, const T *__restrict__ sumH, const int *__restrict__ off) {
    constexpr int NS = BCfg<T, R>::NS;
    constexpr int kColChunk = 128 / (int)sizeof(T);  // V columns staged per chunk
    __shared__ T sV[256][kColChunk + 1];
    __shared__ T sH[kColChunk][NS * R];
    const int row0 = blockIdx.x * 256;
    const int i = row0 + threadIdx.x;
    const bool rowok = i < n;
    const int *goff = off + blockIdx.y * NS;
    int o[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) o[s] = goff[s];
    T wrow[NS][R], acc[NS][R];
#pragma unroll
    for (int s = 0; s < NS; s++)
#pragma unroll
        for (int k = 0; k < R; k++) {
            wrow[s][k] = (rowok && o[s] >= 0) ? W[(size_t)i * ldw + o[s] + k] : (T)0;
            acc[s][k] = (T)0;
        }
    for (int c0 = 0; c0 < p; c0 += kColChunk) {
        const int cols = min(kColChunk, p - c0);
        __syncthreads();
        for (int e = threadIdx.x; e < 256 * kColChunk; e += 256) {
            const int rr = e / kColChunk, cc = e - rr * kColChunk;
            const int gi = row0 + rr;
            sV[rr][cc] = (gi < n && cc < cols) ? V[(size_t)gi * ldv + c0 + cc] : (T)0;
        }
        for (int e = threadIdx.x; e < kColChunk * NS * R; e += 256) {
            const int c = e / kColChunk, cc = e - c * kColChunk;
            const int s = c / R, k = c - s * R;
            sH[cc][c] = (cc < cols && o[s] >= 0) ? H[(size_t)(o[s] + k) * p + c0 + cc] : (T)0;
        }
        __syncthreads();
        for (int cc = 0; cc < cols; cc++) {
            const T v = sV[threadIdx.x][cc];
            const T *hc = sH[cc];
#pragma unroll
            for (int s = 0; s < NS; s++) {
                T wh = (T)0;
#pragma unroll
                for (int k = 0; k < R; k++) wh = fma(wrow[s][k], hc[s * R + k], wh);
                const T qv = (wh != (T)0) ? bdiv(v, wh) : (T)0;
#pragma unroll
                for (int k = 0; k < R; k++) acc[s][k] = fma(hc[s * R + k], qv, acc[s][k]);
            }
        }
    }
    if (!rowok) return;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        if (o[s] < 0) continue;
#pragma unroll
        for (int k = 0; k < R; k++)  // w * tmp / sum_h (lib.rs:199)
            W[(size_t)i * ldw + o[s] + k] = (wrow[s][k] * acc[s][k]) / sumH[o[s] + k];
    }
}

// Column sums of W_all (one thread per stacked column, rows in forward
// order as lib.rs:1563-1568) and row sums of H_all (one warp per row).
template <typename T>
__global__ void batch_colsum(const T *__restrict__ W, int n, int ldw, int rtot, T *__restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= rtot) return;
    T s = (T)0;
    for (int u = 0; u < n; u++) s += W[(size_t)u * ldw + c];
    out[c] = s;
}
template <typename T>
__global__ void batch_rowsum(const T *__restrict__ H, int p, int rtot, T *__restrict__ out) {
    const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= rtot) return;
    T s = (T)0;
    for (int j = lane; j < p; j += 32) s += H[(size_t)row * p + j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[row] = s;
}

// pmax_inplace (lib.rs:1452-1458) on both stacked factors.
template <typename T>
__global__ void batch_clamp(T *__restrict__ W, int64_t nw, T *__restrict__ H, int64_t nh, T eps) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nw; t += stride)
        if (W[t] < eps) W[t] = eps;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nh; t += stride)
        if (H[t] < eps) H[t] = eps;
}

template <typename A, typename B>
__global__ void convert(const A *__restrict__ src, B *__restrict__ dst, int64_t count) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += stride)
        dst[t] = (B)src[t];
}
template <typename A, typename B>
__global__ void convert_2d(const A *__restrict__ src, int64_t lds, B *__restrict__ dst, int64_t ldd,
                           int rows, int cols) {
    const int64_t total = (int64_t)rows * cols;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        const int64_t i = t / cols, j = t - i * cols;
        dst[i * ldd + j] = (B)src[i * lds + j];
    }
}

// Consensus: labels[s][j] = argmax_k H_s[k][j] (first maximum, as numpy's
// argmax in connectivity_matrix, examples/build_scaling_notebook.py:121-124).
template <typename T>
__global__ void batch_labels(const T *__restrict__ H, int p, const int *__restrict__ off,
                             const int *__restrict__ rk, int nsel, unsigned char *__restrict__ lab) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (j >= p || s >= nsel) return;
    const T *h = H + (size_t)off[s] * p + j;
    int best = 0;
    T bv = h[0];
    for (int k = 1; k < rk[s]; k++) {
        const T x = h[(size_t)k * p];
        if (x > bv) {
            bv = x;
            best = k;
        }
    }
    lab[(size_t)j * nsel + s] = (unsigned char)best;
}

// consensus[j1][j2] = (1 / nsel) * #{s : label_s(j1) == label_s(j2)};
// labels are stored column-major over solves (lab[j * nsel + s]).
__global__ void batch_consensus(const unsigned char *__restrict__ lab, int p, int nsel,
                                float *__restrict__ out) {
    const int j1 = blockIdx.y * 16 + (threadIdx.x >> 4);
    const int j2 = blockIdx.x * 16 + (threadIdx.x & 15);
    if (j1 >= p || j2 >= p) return;
    const unsigned char *a = lab + (size_t)j1 * nsel;
    const unsigned char *b = lab + (size_t)j2 * nsel;
    int same = 0;
    for (int s = 0; s < nsel; s++) same += (a[s] == b[s]);
    out[(size_t)j1 * p + j2] = (float)same / (float)nsel;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct RankClass {
    int R;
    int groups;     // CTAs along the solve dimension
    int off_index;  // first entry of this class in the group-offset table
};

template <typename T>
int ns_for(int R) {
    switch (R) {
#define NS_CASE(r) case r: return BCfg<T, r>::NS;
        NS_CASE(1) NS_CASE(2) NS_CASE(3) NS_CASE(4) NS_CASE(5) NS_CASE(6) NS_CASE(7) NS_CASE(8)
        NS_CASE(9) NS_CASE(10) NS_CASE(11) NS_CASE(12) NS_CASE(13) NS_CASE(14) NS_CASE(15) NS_CASE(16)
#undef NS_CASE
    }
    return 1;
}

template <typename T>
void launch_class(bool hside, const RankClass &rc, const T *V, int64_t ldv, int n, int p, T *W,
                  int ldw, T *H, const T *sums, const int *off, cudaStream_t s) {
    const dim3 grid(hside ? (p + 255) / 256 : (n + 255) / 256, rc.groups);
    const int *o = off + rc.off_index;
    switch (rc.R) {
#define CLS_CASE(r)                                                                        \
    case r:                                                                                \
        if (hside)                                                                         \
            batch_hstep<T, r><<<grid, 256, 0, s>>>(V, ldv, n, p, W, ldw, H, sums, o);      \
        else                                                                               \
            batch_wstep<T, r><<<grid, 256, 0, s>>>(V, ldv, n, p, W, ldw, H, sums, o);      \
        break;
        CLS_CASE(1) CLS_CASE(2) CLS_CASE(3) CLS_CASE(4) CLS_CASE(5) CLS_CASE(6) CLS_CASE(7)
        CLS_CASE(8) CLS_CASE(9) CLS_CASE(10) CLS_CASE(11) CLS_CASE(12) CLS_CASE(13) CLS_CASE(14)
        CLS_CASE(15) CLS_CASE(16)
#undef CLS_CASE
    }
}

struct BatchPlan {
    int rtot = 0;
    std::vector<int> offsets;      // per solve, stacked index
    std::vector<RankClass> classes;
    std::vector<int> group_off;    // per class, groups * NS entries (-1 padded)
};

template <typename T>
BatchPlan plan_batch(int nsolves, const int32_t *ranks) {
    BatchPlan bp;
    bp.offsets.resize(nsolves);
    std::map<int, std::vector<int>> by_rank;
    for (int s = 0; s < nsolves; s++) {
        bp.offsets[s] = bp.rtot;
        bp.rtot += ranks[s];
        by_rank[ranks[s]].push_back(s);
    }
    for (auto &kv : by_rank) {
        RankClass rc;
        rc.R = kv.first;
        const int ns = ns_for<T>(rc.R);
        rc.groups = (int)((kv.second.size() + ns - 1) / ns);
        rc.off_index = (int)bp.group_off.size();
        for (int g = 0; g < rc.groups; g++)
            for (int i = 0; i < ns; i++) {
                const size_t idx = (size_t)g * ns + i;
                bp.group_off.push_back(idx < kv.second.size() ? bp.offsets[kv.second[idx]] : -1);
            }
        bp.classes.push_back(rc);
    }
    return bp;
}

// Enqueue iterations [it0, it1] of the batched brunet loop.
template <typename T>
void enqueue_batch_iters(long long it0, long long it1, const BatchPlan &bp, const T *V,
                         int64_t ldv, int n, int p, T *W, T *H, T *sw, T *sh, const int *doff,
                         cudaStream_t s, int64_t *launches) {
    const int rtot = bp.rtot;
    for (long long it = it0; it <= it1; it++) {
        batch_colsum<T><<<(rtot + 127) / 128, 128, 0, s>>>(W, n, rtot, rtot, sw);
        for (const auto &rc : bp.classes)
            launch_class<T>(true, rc, V, ldv, n, p, W, rtot, H, sw, doff, s);
        batch_rowsum<T><<<(rtot + 7) / 8, 256, 0, s>>>(H, p, rtot, sh);
        for (const auto &rc : bp.classes)
            launch_class<T>(false, rc, V, ldv, n, p, W, rtot, H, sh, doff, s);
        *launches += 2 + 2 * (int64_t)bp.classes.size();
        if (it % 10 == 0) {
            batch_clamp<T><<<592, 256, 0, s>>>(W, (int64_t)n * rtot, H, (int64_t)rtot * p,
                                               (T)DBL_EPSILON);
            *launches += 1;
        }
    }
}

template <typename T>
nmfcu_status run_batch_t(nmfcu_context *c, int64_t max_iter, int n, int p, const T *V,
                         int64_t ldv, int nsolves, const int32_t *ranks, T *W, T *H,
                         cudaStream_t s) {
    const BatchPlan bp = plan_batch<T>(nsolves, ranks);
    void *p_off = nullptr, *p_sw = nullptr, *p_sh = nullptr;
    NMFCU_TRY(nmfcu_internal::context_buffer(
        c, 0, sizeof(int) * std::max<size_t>(bp.group_off.size(), 1), &p_off));
    NMFCU_TRY(nmfcu_internal::context_buffer(c, 1, sizeof(T) * (size_t)bp.rtot, &p_sw));
    NMFCU_TRY(nmfcu_internal::context_buffer(c, 2, sizeof(T) * (size_t)bp.rtot, &p_sh));
    int *doff = static_cast<int *>(p_off);
    T *sw = static_cast<T *>(p_sw), *sh = static_cast<T *>(p_sh);
    NMFCU_CUDA_TRY(cudaMemcpyAsync(doff, bp.group_off.data(), sizeof(int) * bp.group_off.size(),
                                   cudaMemcpyHostToDevice, s));
    // The pageable copy above is staged before cudaMemcpyAsync returns, so
    // the plan may go out of scope; the kernels below read doff in order.
    int64_t launches = 0;
    // The loop in blocks of 10 iterations (the clamp period), captured once
    // as a CUDA graph and replayed; the remainder is launched directly.
    const long long blocks = max_iter / 10;
    if (blocks > 0) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaStream_t cs = nullptr;
        cudaEvent_t ready = nullptr;
        NMFCU_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaError_t e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(ready, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, ready, 0);
        if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            int64_t cap_launches = 0;
            enqueue_batch_iters<T>(1, 10, bp, V, ldv, n, p, W, H, sw, sh, doff, cs, &cap_launches);
            e = cudaStreamEndCapture(cs, &graph);
            if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
            for (long long b = 0; e == cudaSuccess && b < blocks; b++) {
                e = cudaGraphLaunch(exec, cs);
                launches += cap_launches;
            }
        }
        if (e == cudaSuccess) e = cudaEventRecord(ready, cs);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ready, 0);
        cudaStreamSynchronize(cs);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        if (ready) cudaEventDestroy(ready);
        if (e != cudaSuccess) return nmfcu_internal::cuda_fail(e, "batched iteration graph");
    }
    enqueue_batch_iters<T>(blocks * 10 + 1, max_iter, bp, V, ldv, n, p, W, H, sw, sh, doff, s,
                           &launches);
    NMFCU_CUDA_TRY(cudaGetLastError());
    nmfcu_internal::count_launches(c, launches);
    return NMFCU_OK;
}

nmfcu_status validate_batch(int32_t method, int32_t precision, int64_t max_iter, int64_t n,
                            int64_t p, int32_t nsolves, const int32_t *ranks) {
    if (method != NMFCU_BRUNET)
        return fail(NMFCU_ERR_UNSUPPORTED, "batched solves are built for brunet only");
    if (precision != NMFCU_PREC_FP64 && precision != NMFCU_PREC_FP32)
        return fail(NMFCU_ERR_INVALID_ARG, "unknown precision id");
    if (max_iter < 0) return fail(NMFCU_ERR_INVALID_ARG, "max_iter must be >= 0");
    if (n < 1 || p < 1 || n > INT32_MAX || p > INT32_MAX)
        return fail(NMFCU_ERR_INVALID_ARG, "n and p must be in [1, 2^31)");
    if (nsolves < 1 || !ranks) return fail(NMFCU_ERR_INVALID_ARG, "need at least one solve");
    int64_t rtot = 0;
    for (int s = 0; s < nsolves; s++) {
        if (ranks[s] < 1 || ranks[s] > kMaxBatchRank)
            return fail(NMFCU_ERR_UNSUPPORTED, "batched ranks must be in [1, 16]");
        rtot += ranks[s];
    }
    if (rtot > INT32_MAX) return fail(NMFCU_ERR_INVALID_ARG, "sum of ranks must fit in 32 bits");
    return NMFCU_OK;
}

}  // namespace

extern "C" {

nmfcu_status nmfcu_run_batch_device(nmfcu_context *ctx, int32_t method, int32_t precision,
                                    int64_t max_iter, int64_t n, int64_t p, const double *dV,
                                    int64_t ldv, int32_t nsolves, const int32_t *ranks,
                                    double *dW, double *dH, void *stream) {
    if (!ctx) return fail(NMFCU_ERR_INVALID_ARG, "NULL context");
    NMFCU_TRY(validate_batch(method, precision, max_iter, n, p, nsolves, ranks));
    if (!dV || !dW || !dH) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    if (ldv < p) return fail(NMFCU_ERR_INVALID_ARG, "ldv must be >= p");
    std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(ctx));
    nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(ctx));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int64_t rtot = 0;
    for (int i = 0; i < nsolves; i++) rtot += ranks[i];
    const int ni = (int)n, pi = (int)p;
    if (precision == NMFCU_PREC_FP64) {
        NMFCU_TRY(run_batch_t<double>(ctx, max_iter, ni, pi, dV, ldv, nsolves, ranks, dW, dH, s));
    } else {
        // f32 copies of V and of the stacked factors (context slots 3..5).
        void *v32 = nullptr, *w32 = nullptr, *h32 = nullptr;
        NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 3, sizeof(float) * (size_t)n * p, &v32));
        NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 4, sizeof(float) * (size_t)n * rtot, &w32));
        NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 5, sizeof(float) * (size_t)rtot * p, &h32));
        convert_2d<double, float><<<1184, 256, 0, s>>>(dV, ldv, (float *)v32, p, ni, pi);
        convert<double, float><<<1184, 256, 0, s>>>(dW, (float *)w32, n * rtot);
        convert<double, float><<<1184, 256, 0, s>>>(dH, (float *)h32, rtot * p);
        NMFCU_TRY(run_batch_t<float>(ctx, max_iter, ni, pi, (const float *)v32, p, nsolves, ranks,
                                     (float *)w32, (float *)h32, s));
        convert<float, double><<<1184, 256, 0, s>>>((const float *)w32, dW, n * rtot);
        convert<float, double><<<1184, 256, 0, s>>>((const float *)h32, dH, rtot * p);
        nmfcu_internal::count_launches(ctx, 5);
    }
    NMFCU_CUDA_TRY(cudaGetLastError());
    NMFCU_CUDA_TRY(cudaStreamSynchronize(s));
    return NMFCU_OK;
}

nmfcu_status nmfcu_run_batch(int32_t method, int32_t precision, int64_t max_iter, int64_t n,
                             int64_t p, const double *V, int32_t nsolves, const int32_t *ranks,
                             const double *W0, const double *H0, double *W, double *H,
                             int32_t device) {
    NMFCU_TRY(validate_batch(method, precision, max_iter, n, p, nsolves, ranks));
    if (!V || !W0 || !H0 || !W || !H) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    nmfcu_context *c = nullptr;
    NMFCU_TRY(nmfcu_internal::default_context(device, &c));
    int64_t rtot = 0;
    for (int i = 0; i < nsolves; i++) rtot += ranks[i];
    void *dv = nullptr, *dw = nullptr, *dh = nullptr;
    {
        std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(c));
        nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(c));
        NMFCU_TRY(nmfcu_internal::context_buffer(c, 6, sizeof(double) * (size_t)n * p, &dv));
        NMFCU_TRY(nmfcu_internal::context_buffer(c, 7, sizeof(double) * (size_t)n * rtot, &dw));
        NMFCU_TRY(nmfcu_internal::context_buffer(c, 8, sizeof(double) * (size_t)rtot * p, &dh));
        cudaStream_t s = nmfcu_internal::context_stream(c);
        NMFCU_CUDA_TRY(cudaMemcpyAsync(dv, V, sizeof(double) * n * p, cudaMemcpyHostToDevice, s));
        NMFCU_CUDA_TRY(cudaMemcpyAsync(dw, W0, sizeof(double) * n * rtot, cudaMemcpyHostToDevice, s));
        NMFCU_CUDA_TRY(cudaMemcpyAsync(dh, H0, sizeof(double) * rtot * p, cudaMemcpyHostToDevice, s));
    }
    NMFCU_TRY(nmfcu_run_batch_device(c, method, precision, max_iter, n, p, (const double *)dv, p,
                                     nsolves, ranks, (double *)dw, (double *)dh,
                                     nmfcu_internal::context_stream(c)));
    std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(c));
    nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(c));
    cudaStream_t s = nmfcu_internal::context_stream(c);
    NMFCU_CUDA_TRY(cudaMemcpyAsync(W, dw, sizeof(double) * n * rtot, cudaMemcpyDeviceToHost, s));
    NMFCU_CUDA_TRY(cudaMemcpyAsync(H, dh, sizeof(double) * rtot * p, cudaMemcpyDeviceToHost, s));
    NMFCU_CUDA_TRY(cudaStreamSynchronize(s));
    return NMFCU_OK;
}

nmfcu_status nmfcu_consensus_device(nmfcu_context *ctx, int64_t p, int32_t nsolves,
                                    const int32_t *ranks, const double *dH, int32_t nsel,
                                    const int32_t *sel, float *d_out, void *stream) {
    if (!ctx) return fail(NMFCU_ERR_INVALID_ARG, "NULL context");
    if (p < 1 || p > 65535 * 16 || nsolves < 1 || !ranks || !dH || !d_out)
        return fail(NMFCU_ERR_INVALID_ARG, "bad consensus arguments");
    if (nsel < 1 || nsel > 65535 || !sel)
        return fail(NMFCU_ERR_INVALID_ARG, "need 1..65535 selected solves");
    std::vector<int> off(nsolves), so(nsel), sr(nsel);
    int64_t acc = 0;
    for (int s = 0; s < nsolves; s++) {
        if (ranks[s] < 1 || ranks[s] > 255)
            return fail(NMFCU_ERR_INVALID_ARG, "ranks must be in [1, 255]");
        if (acc > INT32_MAX - 255) return fail(NMFCU_ERR_INVALID_ARG, "too many stacked rows");
        off[s] = (int)acc;
        acc += ranks[s];
    }
    for (int i = 0; i < nsel; i++) {
        if (sel[i] < 0 || sel[i] >= nsolves)
            return fail(NMFCU_ERR_INVALID_ARG, "selected solve out of range");
        so[i] = off[sel[i]];
        sr[i] = ranks[sel[i]];
    }
    std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(ctx));
    nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(ctx));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void *pso = nullptr, *psr = nullptr, *plab = nullptr;
    NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 9, sizeof(int) * nsel, &pso));
    NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 10, sizeof(int) * nsel, &psr));
    NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 11, (size_t)p * nsel, &plab));
    NMFCU_CUDA_TRY(cudaMemcpyAsync(pso, so.data(), sizeof(int) * nsel, cudaMemcpyHostToDevice, s));
    NMFCU_CUDA_TRY(cudaMemcpyAsync(psr, sr.data(), sizeof(int) * nsel, cudaMemcpyHostToDevice, s));
    const dim3 lg((unsigned)((p + 255) / 256), (unsigned)nsel);
    batch_labels<double><<<lg, 256, 0, s>>>(dH, (int)p, (const int *)pso, (const int *)psr, nsel,
                                            (unsigned char *)plab);
    const dim3 cg((unsigned)((p + 15) / 16), (unsigned)((p + 15) / 16));
    batch_consensus<<<cg, 256, 0, s>>>((const unsigned char *)plab, (int)p, nsel, d_out);
    NMFCU_CUDA_TRY(cudaGetLastError());
    nmfcu_internal::count_launches(ctx, 2);
    NMFCU_CUDA_TRY(cudaStreamSynchronize(s));
    return NMFCU_OK;
}

}  // extern "C"

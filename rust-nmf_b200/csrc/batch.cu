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
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/nmfcu.h"
#include "internal.h"

using nmfcu_internal::fail;

namespace {

constexpr int kMaxBatchRank = 16;  // largest rank of a batched solve
constexpr int kThreads = 128;      // threads per CTA
constexpr int kRowChunk = 64;      // W rows staged per chunk (H step)
constexpr int kPrefetch = 4;       // V rows in flight per thread (H step)
constexpr int kColChunk = 16;      // V columns staged per chunk (W step)

// Per element type: a thread owns CPT adjacent columns (H step) or rows
// (W step) of V, held in one "lane pack" P.  f32 packs two (float2, one
// FFMA2 updates both), so a W value times an H pair, or an H value times a
// W pair, is one instruction and the per-element ratio is computed for two
// elements at once; f64 owns one (DFMA).  kComponents bounds the rank
// components (sum of the ranks of the solves) a CTA carries.
template <typename T>
struct BTraits;
template <>
struct BTraits<float> {
    using P = float2;
    static constexpr int CPT = 2;
    static constexpr int kComponents = 16;
};
template <>
struct BTraits<double> {
    using P = double;
    static constexpr int CPT = 1;
    static constexpr int kComponents = 16;
};

template <typename T, int R>
struct BCfg {
    static constexpr int NS = BTraits<T>::kComponents / R > 0 ? BTraits<T>::kComponents / R : 1;
    static constexpr int ROW = NS * R;  // staged values per W row / H column
};
constexpr int kMaxRow = 16;             // >= ROW for every (T, R)
template <typename T>
constexpr int kTile = kThreads * BTraits<T>::CPT;  // columns / rows per CTA

__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ double pfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float2 pdup(float x) { return make_float2(x, x); }
__device__ __forceinline__ double pdup(double x) { return x; }
__device__ __forceinline__ void pzero(float2 &x) { x = make_float2(0.f, 0.f); }
__device__ __forceinline__ void pzero(double &x) { x = 0.0; }
__device__ __forceinline__ float &plane(float2 &a, int c) { return c ? a.y : a.x; }
__device__ __forceinline__ double &plane(double &a, int) { return a; }

// The brunet ratio V / (WH), 0 where WH == 0 (lib.rs:93-99).  f32 uses the
// hardware reciprocal approximation (rcp.approx.ftz.f32, about 1 ulp).
__device__ __forceinline__ float ratio1(float v, float wh) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(wh));
    return (wh != 0.f) ? v * r : 0.f;
}
__device__ __forceinline__ float2 ratio(float2 v, float2 wh) {
    return make_float2(ratio1(v.x, wh.x), ratio1(v.y, wh.y));
}
// f64: v * (1 / wh) with the reciprocal from the hardware approximation
// (rcp.approx.ftz.f64) refined by two Newton-Raphson steps
// y <- y + y (1 - wh y), each of which doubles the number of correct bits;
// the quotient is then within about an ulp of the IEEE one.  |wh| outside
// [2^-1000, 2^1000] (and NaN) takes the exact division.
__device__ __forceinline__ double ratio(double v, double wh) {
    if (wh == 0.0) return 0.0;
    const double a = fabs(wh);
    if (!(a > 0x1p-1000 && a < 0x1p1000)) return v / wh;
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(wh));
    double e = fma(-wh, y, 1.0);
    y = fma(y, e, y);
    e = fma(-wh, y, 1.0);
    y = fma(y, e, y);
    return v * y;
}

// Shared memory of one CTA (the larger of the two steps' layouts).  W
// values (H step) and H values (W step) are stored duplicated across the
// lane pack, so one load feeds both lanes.
template <typename T>
struct BSmem {
    using P = typename BTraits<T>::P;
    union {
        P hW[kRowChunk][kMaxRow];                 // H step: W rows of the group
        struct {
            T Vt[kColChunk][kTile<T> + 2];        // W step: V tile, transposed
            P Hc[kColChunk][kMaxRow];             // W step: H columns of the group
        } w;
    };
    int off[BTraits<T>::kComponents];             // stacked offset per solve (-1: none)
};

// One unit of a step: NS solves of rank R (offsets at goff[0..NS)) on one
// tile of kTile columns (H step) or rows (W step).
struct BItem {
    int R;
    int goff;  // index of the first offset in the group-offset table
    int tile;
    int pad;
};

// H update of one item (divergence_update_h_inner, lib.rs:74-115, per solve):
//   H[k][j] <- H[k][j] * (sum_i W[i][k] V[i][j] / (WH)[i][j]) / sum_i W[i][k]
// A thread owns CPT adjacent columns; W rows are staged in shared memory
// (zero beyond n), V rows stream from L2 a few rows ahead.  V's leading
// dimension must make a CPT-column load aligned, and V must be zero in
// columns [p, round_up(p, CPT)).
template <typename T, int R>
__device__ __forceinline__ void hstep_item(BSmem<T> &sm, const T *__restrict__ V, int64_t ldv,
                                           int n, int p, const T *__restrict__ W, int ldw,
                                           T *__restrict__ H, const T *__restrict__ sumW,
                                           const int *__restrict__ goff, int tile) {
    using C = BCfg<T, R>;
    using P = typename BTraits<T>::P;
    constexpr int CPT = BTraits<T>::CPT;
    constexpr int NS = C::NS, ROW = C::ROW;
    constexpr int WPT = (kRowChunk * ROW + kThreads - 1) / kThreads;  // staged W values per thread
    static_assert(ROW <= kMaxRow && NS <= BTraits<T>::kComponents, "staging row too long");
    static_assert(kRowChunk % kPrefetch == 0, "row chunk must hold whole prefetch groups");
    if (threadIdx.x < NS) sm.off[threadIdx.x] = goff[threadIdx.x];
    __syncthreads();
    const int j0 = tile * kTile<T> + threadIdx.x * CPT;
    const bool colok = j0 < p;
    P h[NS][R], acc[NS][R];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const int o = sm.off[s];
#pragma unroll
        for (int k = 0; k < R; k++) {
#pragma unroll
            for (int c = 0; c < CPT; c++)
                plane(h[s][k], c) = (o >= 0 && j0 + c < p) ? H[(size_t)(o + k) * p + j0 + c] : (T)0;
            pzero(acc[s][k]);
        }
    }
    // W values of the next row chunk, loaded while the current one is used.
    T wpre[WPT];
    auto load_w = [&](int base) {
        const int rows = min(kRowChunk, n - base);
#pragma unroll
        for (int t = 0; t < WPT; t++) {
            const int e = t * kThreads + threadIdx.x;
            const int rr = e / ROW, c = e - rr * ROW;
            const int s = c / R, k = c - s * R;
            const int o = (e < kRowChunk * ROW) ? sm.off[s] : -1;
            wpre[t] = (rr < rows && o >= 0) ? W[(size_t)(base + rr) * ldw + o + k] : (T)0;
        }
    };
    load_w(0);
    for (int base = 0; base < n; base += kRowChunk) {
        const int rows = min(kRowChunk, n - base);
        __syncthreads();
#pragma unroll
        for (int t = 0; t < WPT; t++) {
            const int e = t * kThreads + threadIdx.x;
            if (e < kRowChunk * ROW) sm.hW[e / ROW][e % ROW] = pdup(wpre[t]);
        }
        __syncthreads();
        if (base + kRowChunk < n) load_w(base + kRowChunk);
        const P *vp = reinterpret_cast<const P *>(V + (size_t)base * ldv + j0);
        const int64_t ldp = ldv / CPT;
        P vb[kPrefetch];
#pragma unroll
        for (int q = 0; q < kPrefetch; q++) {
            if (colok && q < rows) vb[q] = vp[q * ldp];
            else pzero(vb[q]);
        }
        for (int r0 = 0; r0 < rows; r0 += kPrefetch) {
            P vn[kPrefetch];
#pragma unroll
            for (int q = 0; q < kPrefetch; q++) {
                const int rr = r0 + kPrefetch + q;
                if (colok && rr < rows) vn[q] = vp[rr * ldp];
                else pzero(vn[q]);
            }
            // Rows past the chunk's end read zero W rows and v = 0: no-ops.
#pragma unroll
            for (int q = 0; q < kPrefetch; q++) {
                const P *wr = sm.hW[r0 + q];
#pragma unroll
                for (int s = 0; s < NS; s++) {
                    P d;
                    pzero(d);
#pragma unroll
                    for (int k = 0; k < R; k++) d = pfma(wr[s * R + k], h[s][k], d);
                    const P qq = ratio(vb[q], d);
#pragma unroll
                    for (int k = 0; k < R; k++) acc[s][k] = pfma(wr[s * R + k], qq, acc[s][k]);
                }
            }
#pragma unroll
            for (int q = 0; q < kPrefetch; q++) vb[q] = vn[q];
        }
    }
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const int o = sm.off[s];
        if (o < 0) continue;
#pragma unroll
        for (int k = 0; k < R; k++)
#pragma unroll
            for (int c = 0; c < CPT; c++)
                if (j0 + c < p)  // h * tmp / sum_w (lib.rs:110)
                    H[(size_t)(o + k) * p + j0 + c] =
                        (plane(h[s][k], c) * plane(acc[s][k], c)) / sumW[o + k];
    }
}

// W update of one item (divergence_update_w_impl, lib.rs:151-204, per solve):
//   W[i][k] <- W[i][k] * (sum_j H[k][j] V[i][j] / (WH)[i][j]) / sum_j H[k][j]
// A thread owns CPT adjacent rows; V tiles are staged transposed (one
// aligned load gives a thread its rows of one column) and H columns are
// staged, both loaded a chunk ahead into registers.
template <typename T, int R>
__device__ __forceinline__ void wstep_item(BSmem<T> &sm, const T *__restrict__ V, int64_t ldv,
                                           int n, int p, T *__restrict__ W, int ldw,
                                           const T *__restrict__ H, const T *__restrict__ sumH,
                                           const int *__restrict__ goff, int tile) {
    using C = BCfg<T, R>;
    using P = typename BTraits<T>::P;
    constexpr int CPT = BTraits<T>::CPT;
    constexpr int NS = C::NS, ROW = C::ROW;
    constexpr int CC = kColChunk;
    constexpr int TILE = kTile<T>;
    constexpr int VPT = TILE * CC / kThreads;                    // staged V values per thread
    constexpr int HPT = (CC * ROW + kThreads - 1) / kThreads;    // staged H values per thread
    static_assert(ROW <= kMaxRow && NS <= BTraits<T>::kComponents, "staging row too long");
    static_assert(kThreads % CC == 0, "V staging maps a thread to one column");
    if (threadIdx.x < NS) sm.off[threadIdx.x] = goff[threadIdx.x];
    __syncthreads();
    const int row0 = tile * TILE;
    const int i0 = row0 + threadIdx.x * CPT;
    P w[NS][R], acc[NS][R];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const int o = sm.off[s];
#pragma unroll
        for (int k = 0; k < R; k++) {
#pragma unroll
            for (int c = 0; c < CPT; c++)
                plane(w[s][k], c) = (o >= 0 && i0 + c < n) ? W[(size_t)(i0 + c) * ldw + o + k] : (T)0;
            pzero(acc[s][k]);
        }
    }
    // Thread t stages column t % CC of rows t / CC + v * (kThreads / CC).
    const int vcol = threadIdx.x % CC, vrow = threadIdx.x / CC;
    T vpre[VPT], hpre[HPT];
    auto load_chunk = [&](int c0) {
        const int cols = min(CC, p - c0);
#pragma unroll
        for (int v = 0; v < VPT; v++) {
            const int gi = row0 + vrow + v * (kThreads / CC);
            vpre[v] = (gi < n && vcol < cols) ? V[(size_t)gi * ldv + c0 + vcol] : (T)0;
        }
#pragma unroll
        for (int t = 0; t < HPT; t++) {
            const int e = t * kThreads + threadIdx.x;
            const int c = e / CC, cc = e - c * CC;
            const int s = c / R, k = c - s * R;
            const int o = (e < CC * ROW) ? sm.off[s] : -1;
            hpre[t] = (cc < cols && o >= 0) ? H[(size_t)(o + k) * p + c0 + cc] : (T)0;
        }
    };
    load_chunk(0);
    for (int c0 = 0; c0 < p; c0 += CC) {
        __syncthreads();
#pragma unroll
        for (int v = 0; v < VPT; v++) sm.w.Vt[vcol][vrow + v * (kThreads / CC)] = vpre[v];
#pragma unroll
        for (int t = 0; t < HPT; t++) {
            const int e = t * kThreads + threadIdx.x;
            if (e < CC * ROW) sm.w.Hc[e % CC][e / CC] = pdup(hpre[t]);
        }
        __syncthreads();
        if (c0 + CC < p) load_chunk(c0 + CC);
        // Columns past p hold V = 0 and H = 0: no-ops.
#pragma unroll 2
        for (int cc = 0; cc < CC; cc++) {
            const P v = *reinterpret_cast<const P *>(&sm.w.Vt[cc][threadIdx.x * CPT]);
            const P *hc = sm.w.Hc[cc];
#pragma unroll
            for (int s = 0; s < NS; s++) {
                P d;
                pzero(d);
#pragma unroll
                for (int k = 0; k < R; k++) d = pfma(w[s][k], hc[s * R + k], d);
                const P qq = ratio(v, d);
#pragma unroll
                for (int k = 0; k < R; k++) acc[s][k] = pfma(hc[s * R + k], qq, acc[s][k]);
            }
        }
    }
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const int o = sm.off[s];
        if (o < 0) continue;
#pragma unroll
        for (int k = 0; k < R; k++)
#pragma unroll
            for (int c = 0; c < CPT; c++)
                if (i0 + c < n)  // w * tmp / sum_h (lib.rs:199)
                    W[(size_t)(i0 + c) * ldw + o + k] =
                        (plane(w[s][k], c) * plane(acc[s][k], c)) / sumH[o + k];
    }
}

#define BATCH_RANK_CASES(X) \
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

// One launch per step for every rank class: CTA b runs item b.  The
// register caps (measured best among 2..4 resident CTAs per SM) keep the
// H step at 3 (f32) / 2 (f64) and the W step at 3 CTAs per SM.
template <typename T>
constexpr int kMinBlocksH = sizeof(T) == 4 ? 3 : 2;
template <typename T>
constexpr int kMinBlocksW = sizeof(T) == 4 ? 3 : 3;

template <typename T>
__global__ void __launch_bounds__(kThreads, kMinBlocksH<T>)
    batch_hstep(const T *__restrict__ V, int64_t ldv, int n, int p, const T *__restrict__ W, int ldw,
                T *__restrict__ H, const T *__restrict__ sumW, const int *__restrict__ off,
                const BItem *__restrict__ items) {
    __shared__ __align__(16) BSmem<T> sm;
    const BItem it = items[blockIdx.x];
    switch (it.R) {
#define H_CASE(r) \
    case r: hstep_item<T, r>(sm, V, ldv, n, p, W, ldw, H, sumW, off + it.goff, it.tile); break;
        BATCH_RANK_CASES(H_CASE)
#undef H_CASE
    }
}
template <typename T>
__global__ void __launch_bounds__(kThreads, kMinBlocksW<T>)
    batch_wstep(const T *__restrict__ V, int64_t ldv, int n, int p, T *__restrict__ W, int ldw,
                const T *__restrict__ H, const T *__restrict__ sumH, const int *__restrict__ off,
                const BItem *__restrict__ items) {
    __shared__ __align__(16) BSmem<T> sm;
    const BItem it = items[blockIdx.x];
    switch (it.R) {
#define W_CASE(r) \
    case r: wstep_item<T, r>(sm, V, ldv, n, p, W, ldw, H, sumH, off + it.goff, it.tile); break;
        BATCH_RANK_CASES(W_CASE)
#undef W_CASE
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
template <typename T>
int ns_for(int R) {
    switch (R) {
#define NS_CASE(r) case r: return BCfg<T, r>::NS;
        BATCH_RANK_CASES(NS_CASE)
#undef NS_CASE
    }
    return 1;
}

struct BatchPlan {
    int rtot = 0;
    std::vector<int> group_off;  // per group, NS offsets (-1 padded)
    std::vector<BItem> hitems, witems;
};

// Solves of one rank form a class; a class is cut into groups of NS solves;
// every (group, tile) pair is one CTA of the step's launch.
template <typename T>
BatchPlan plan_batch(int n, int p, int nsolves, const int32_t *ranks) {
    BatchPlan bp;
    std::vector<int> offsets(nsolves);
    std::map<int, std::vector<int>> by_rank;
    for (int s = 0; s < nsolves; s++) {
        offsets[s] = bp.rtot;
        bp.rtot += ranks[s];
        by_rank[ranks[s]].push_back(s);
    }
    const int htiles = (p + kTile<T> - 1) / kTile<T>, wtiles = (n + kTile<T> - 1) / kTile<T>;
    // Larger ranks first: their CTAs are the longest, so they start first.
    for (auto it = by_rank.rbegin(); it != by_rank.rend(); ++it) {
        const int R = it->first;
        const auto &members = it->second;
        const int ns = ns_for<T>(R);
        const int groups = (int)((members.size() + ns - 1) / ns);
        for (int g = 0; g < groups; g++) {
            const int at = (int)bp.group_off.size();
            for (int i = 0; i < ns; i++) {
                const size_t idx = (size_t)g * ns + i;
                bp.group_off.push_back(idx < members.size() ? offsets[members[idx]] : -1);
            }
            for (int t = 0; t < htiles; t++) bp.hitems.push_back({R, at, t, 0});
            for (int t = 0; t < wtiles; t++) bp.witems.push_back({R, at, t, 0});
        }
    }
    return bp;
}

struct BatchDev {
    const int *off;
    const BItem *hitems, *witems;
    int nh, nw;
};

// Enqueue iterations [it0, it1] of the batched brunet loop.
template <typename T>
void enqueue_batch_iters(long long it0, long long it1, const BatchPlan &bp, const BatchDev &d,
                         const T *V, int64_t ldv, int n, int p, T *W, T *H, T *sw, T *sh,
                         cudaStream_t s, int64_t *launches) {
    const int rtot = bp.rtot;
    for (long long it = it0; it <= it1; it++) {
        batch_colsum<T><<<(rtot + 127) / 128, 128, 0, s>>>(W, n, rtot, rtot, sw);
        batch_hstep<T><<<d.nh, kThreads, 0, s>>>(V, ldv, n, p, W, rtot, H, sw, d.off, d.hitems);
        batch_rowsum<T><<<(rtot + 7) / 8, 256, 0, s>>>(H, p, rtot, sh);
        batch_wstep<T><<<d.nw, kThreads, 0, s>>>(V, ldv, n, p, W, rtot, H, sh, d.off, d.witems);
        *launches += 4;
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
    const BatchPlan bp = plan_batch<T>(n, p, nsolves, ranks);
    // One upload: group offsets, then H items, then W items (16-byte aligned).
    const size_t off_bytes = (sizeof(int) * bp.group_off.size() + 15) / 16 * 16;
    const size_t item_bytes = sizeof(BItem) * (bp.hitems.size() + bp.witems.size());
    std::vector<unsigned char> table(off_bytes + item_bytes, 0);
    std::memcpy(table.data(), bp.group_off.data(), sizeof(int) * bp.group_off.size());
    std::memcpy(table.data() + off_bytes, bp.hitems.data(), sizeof(BItem) * bp.hitems.size());
    std::memcpy(table.data() + off_bytes + sizeof(BItem) * bp.hitems.size(), bp.witems.data(),
                sizeof(BItem) * bp.witems.size());
    void *p_tab = nullptr, *p_sw = nullptr, *p_sh = nullptr;
    NMFCU_TRY(nmfcu_internal::context_buffer(c, 0, table.size(), &p_tab));
    NMFCU_TRY(nmfcu_internal::context_buffer(c, 1, sizeof(T) * (size_t)bp.rtot, &p_sw));
    NMFCU_TRY(nmfcu_internal::context_buffer(c, 2, sizeof(T) * (size_t)bp.rtot, &p_sh));
    T *sw = static_cast<T *>(p_sw), *sh = static_cast<T *>(p_sh);
    // A pageable host source is staged before cudaMemcpyAsync returns, so the
    // table may go out of scope; the kernels below read it in stream order.
    NMFCU_CUDA_TRY(cudaMemcpyAsync(p_tab, table.data(), table.size(), cudaMemcpyHostToDevice, s));
    BatchDev d;
    d.off = static_cast<const int *>(p_tab);
    d.hitems = reinterpret_cast<const BItem *>(static_cast<unsigned char *>(p_tab) + off_bytes);
    d.witems = d.hitems + bp.hitems.size();
    d.nh = (int)bp.hitems.size();
    d.nw = (int)bp.witems.size();
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
            enqueue_batch_iters<T>(1, 10, bp, d, V, ldv, n, p, W, H, sw, sh, cs, &cap_launches);
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
    enqueue_batch_iters<T>(blocks * 10 + 1, max_iter, bp, d, V, ldv, n, p, W, H, sw, sh, s,
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
        // The f32 V's leading dimension is a multiple of 4 with the pad
        // columns zero (the H step loads column pairs, aligned).
        const int64_t ld32 = (p + 3) / 4 * 4;
        NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 3, sizeof(float) * (size_t)n * ld32, &v32));
        NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 4, sizeof(float) * (size_t)n * rtot, &w32));
        NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 5, sizeof(float) * (size_t)rtot * p, &h32));
        if (ld32 > p) NMFCU_CUDA_TRY(cudaMemsetAsync(v32, 0, sizeof(float) * (size_t)n * ld32, s));
        convert_2d<double, float><<<1184, 256, 0, s>>>(dV, ldv, (float *)v32, ld32, ni, pi);
        convert<double, float><<<1184, 256, 0, s>>>(dW, (float *)w32, n * rtot);
        convert<double, float><<<1184, 256, 0, s>>>(dH, (float *)h32, rtot * p);
        NMFCU_TRY(run_batch_t<float>(ctx, max_iter, ni, pi, (const float *)v32, ld32, nsolves, ranks,
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

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

// Per element type: a thread owns CPT adjacent columns (H step) or rows
// (W step) of V, held in one "lane pack" P.  f32 packs four as two float2
// halves (one FFMA2 updates each half), so a staged factor value times an
// H (or W) pack is two instructions that share the value's register pair;
// the staged factor sits in shared memory as a duplicated pair (SV), so
// one 128-bit load brings two values for eight columns' worth of FFMA2.
// f64 owns one column (DFMA).
struct F4 {
    float2 a, b;  // columns 0, 1 and 2, 3
};
template <typename T>
struct BTraits;
template <>
struct BTraits<float> {
    using P = F4;
    using SV = float2;  // a staged value in shared memory
    static constexpr int CPT = 4;
};
template <>
struct BTraits<double> {
    using P = double;
    using SV = double;
    static constexpr int CPT = 1;
};

// Kernel shapes the autotuner chooses from (run_batch_t): `comp` bounds the
// rank components (sum of the ranks of the solves) a CTA carries -- so a CTA
// takes comp / R solves of rank R and each V element it loads serves them
// all -- and `min_blocks` is the CTAs a multiprocessor keeps resident (the
// register cap of __launch_bounds__).  Shape 0 is the one measured best at
// the consensus shape during development; a shape changes which solves share
// a CTA, never the arithmetic of a solve, so every shape gives the same bits.
template <typename T>
struct BShapes;
template <>
struct BShapes<float> {
    static constexpr int kN = 3;
    static constexpr int comp[kN] = {6, 4, 8};
    static constexpr int min_blocks[kN] = {4, 4, 4};  // ranks 1..8; 9..16: min_blocks_for
};
template <>
struct BShapes<double> {
    static constexpr int kN = 3;
    static constexpr int comp[kN] = {8, 4, 12};
    static constexpr int min_blocks[kN] = {5, 6, 4};
};
constexpr int kShapesMax = 3;

template <typename T, int R, int COMP>
struct BCfg {
    static constexpr int NS = COMP / R > 0 ? COMP / R : 1;
    static constexpr int ROW = NS * R;  // staged values per W row / H column
};
constexpr int kMaxRow = 16;             // >= ROW for every (T, R, COMP)
template <typename T>
constexpr int kTile = kThreads * BTraits<T>::CPT;  // columns / rows per CTA

// A staged value (SV) times a pack plus a pack.
__device__ __forceinline__ F4 pfma(float2 s, F4 b, F4 c) {
    return F4{__ffma2_rn(s, b.a, c.a), __ffma2_rn(s, b.b, c.b)};
}
__device__ __forceinline__ double pfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float2 sdup(float x) { return make_float2(x, x); }
__device__ __forceinline__ double sdup(double x) { return x; }
__device__ __forceinline__ void pzero(F4 &x) {
    x.a = make_float2(0.f, 0.f);
    x.b = make_float2(0.f, 0.f);
}
__device__ __forceinline__ void pzero(double &x) { x = 0.0; }
__device__ __forceinline__ float &plane(F4 &a, int c) {
    return c == 0 ? a.a.x : c == 1 ? a.a.y : c == 2 ? a.b.x : a.b.y;
}
__device__ __forceinline__ double &plane(double &a, int) { return a; }

// The brunet ratio V / (WH), 0 where WH == 0 (lib.rs:93-99).  f32 uses the
// hardware reciprocal approximation (rcp.approx.ftz.f32, about 1 ulp); for a
// pack of four columns the reciprocals are taken one by one and the
// products v * (1 / wh) as two packed f32x2 multiplies.
__device__ __forceinline__ float rcp1(float wh) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(wh));
    return r;
}
__device__ __forceinline__ F4 ratio(F4 v, F4 wh) {
    const float2 qa = __fmul2_rn(v.a, make_float2(rcp1(wh.a.x), rcp1(wh.a.y)));
    const float2 qb = __fmul2_rn(v.b, make_float2(rcp1(wh.b.x), rcp1(wh.b.y)));
    return F4{make_float2(wh.a.x != 0.f ? qa.x : 0.f, wh.a.y != 0.f ? qa.y : 0.f),
              make_float2(wh.b.x != 0.f ? qb.x : 0.f, wh.b.y != 0.f ? qb.y : 0.f)};
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

// One multiplicative update, written once for both steps.  The step
// streams a matrix A (rows x cols) whose columns are the outputs: A = V for
// the H step (columns = cells), A = V^T for the W step (columns = genes).
// For each output column j and solve s it forms
//   acc[k] = sum_r S[r][k] * A[r][j] / (sum_k' S[r][k'] X[k'][j])
// and writes X[k][j] <- X[k][j] * acc[k] / norm[k], where S is the staged
// factor (W for the H step, H^T for the W step) and X the updated one.
// This is divergence_update_h_inner (lib.rs:74-115) for the H step and
// divergence_update_w_impl (lib.rs:151-204) for the W step, per solve.
template <typename T>
struct MuArgs {
    const T *A;          // rows x cols, leading dimension lda
    int64_t lda;
    int rows, cols;
    const T *S;          // staged factor: S(r, c) = S[r * s_row + c * s_col]
    int64_t s_row, s_col;
    T *X;                // updated factor: X(c, j) = X[c * x_comp + j * x_col]
    int64_t x_comp, x_col;
    const T *norm;       // per stacked component
};

// Shared memory of one CTA: the staged factor's rows, duplicated across the
// lane pack (one load feeds both lanes); rows padded so that the transposing
// stores of the W step spread over the banks and rows stay 16-B aligned.
template <typename T>
struct BSmem {
    using SV = typename BTraits<T>::SV;
    SV S[kRowChunk][kMaxRow + 2];
    int off[kMaxRow];  // stacked offset per solve (-1: none)
};

// One unit of a step: NS solves of rank R (offsets at goff[0..NS)) on one
// tile of kTile output columns.
struct BItem {
    int R;
    int goff;  // index of the first offset in the group-offset table
    int tile;
    int pad;
};

// A thread owns CPT adjacent output columns; the staged factor's rows are
// staged in shared memory a chunk ahead (zero beyond `rows`), A streams from
// L2 a few rows ahead.  A's leading dimension must make a CPT-column load
// aligned, and A must be zero in columns [cols, round_up(cols, CPT)).
// kComponentFast: the staged factor is contiguous along components (W in
// the H step) -- staging loads walk components; otherwise (H^T) they walk rows.
template <typename T, int R, int COMP, bool kComponentFast>
__device__ __forceinline__ void mu_item(BSmem<T> &sm, const MuArgs<T> &a,
                                        const int *__restrict__ goff, int tile) {
    using C = BCfg<T, R, COMP>;
    using P = typename BTraits<T>::P;
    constexpr int CPT = BTraits<T>::CPT;
    constexpr int NS = C::NS, ROW = C::ROW;
    constexpr int SPT = (kRowChunk * ROW + kThreads - 1) / kThreads;  // staged values per thread
    static_assert(ROW <= kMaxRow && NS <= kMaxRow, "staging row too long");
    static_assert(kRowChunk % kPrefetch == 0, "row chunk must hold whole prefetch groups");
    if (threadIdx.x < NS) sm.off[threadIdx.x] = goff[threadIdx.x];
    __syncthreads();
    const int rows = a.rows, cols = a.cols;
    const int j0 = tile * kTile<T> + threadIdx.x * CPT;
    const bool colok = j0 < cols;
    P x[NS][R], acc[NS][R];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const int o = sm.off[s];
#pragma unroll
        for (int k = 0; k < R; k++) {
#pragma unroll
            for (int c = 0; c < CPT; c++)
                plane(x[s][k], c) = (o >= 0 && j0 + c < cols)
                                        ? a.X[(size_t)(o + k) * a.x_comp + (size_t)(j0 + c) * a.x_col]
                                        : (T)0;
            pzero(acc[s][k]);
        }
    }
    // Staged values of the next row chunk, loaded while the current one is used.
    T spre[SPT];
    auto stage_index = [&](int e, int &rr, int &c) {
        if (kComponentFast) {
            rr = e / ROW;
            c = e - rr * ROW;
        } else {
            c = e / kRowChunk;
            rr = e - c * kRowChunk;
        }
    };
    auto load_s = [&](int base) {
        const int nr = min(kRowChunk, rows - base);
#pragma unroll
        for (int t = 0; t < SPT; t++) {
            const int e = t * kThreads + threadIdx.x;
            int rr, c;
            stage_index(e, rr, c);
            const int s = c / R, k = c - s * R;
            const int o = (e < kRowChunk * ROW) ? sm.off[s] : -1;
            spre[t] = (rr < nr && o >= 0)
                          ? a.S[(size_t)(base + rr) * a.s_row + (size_t)(o + k) * a.s_col]
                          : (T)0;
        }
    };
    load_s(0);
    const int64_t ldp = a.lda / CPT;
    for (int base = 0; base < rows; base += kRowChunk) {
        const int nr = min(kRowChunk, rows - base);
        __syncthreads();
#pragma unroll
        for (int t = 0; t < SPT; t++) {
            const int e = t * kThreads + threadIdx.x;
            int rr, c;
            stage_index(e, rr, c);
            if (e < kRowChunk * ROW) sm.S[rr][c] = sdup(spre[t]);
        }
        __syncthreads();
        if (base + kRowChunk < rows) load_s(base + kRowChunk);
        const P *ap = reinterpret_cast<const P *>(a.A + (size_t)base * a.lda + j0);
        P vb[kPrefetch];
#pragma unroll
        for (int q = 0; q < kPrefetch; q++) {
            if (colok && q < nr) vb[q] = ap[q * ldp];
            else pzero(vb[q]);
        }
        for (int r0 = 0; r0 < nr; r0 += kPrefetch) {
            P vn[kPrefetch];
#pragma unroll
            for (int q = 0; q < kPrefetch; q++) {
                const int rr = r0 + kPrefetch + q;
                if (colok && rr < nr) vn[q] = ap[rr * ldp];
                else pzero(vn[q]);
            }
            // Rows past the chunk's end read zero staged rows and a = 0: no-ops.
#pragma unroll
            for (int q = 0; q < kPrefetch; q++) {
                const typename BTraits<T>::SV *sr = sm.S[r0 + q];
#pragma unroll
                for (int s = 0; s < NS; s++) {
                    P d;
                    pzero(d);
#pragma unroll
                    for (int k = 0; k < R; k++) d = pfma(sr[s * R + k], x[s][k], d);
                    const P qq = ratio(vb[q], d);
#pragma unroll
                    for (int k = 0; k < R; k++) acc[s][k] = pfma(sr[s * R + k], qq, acc[s][k]);
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
                if (j0 + c < cols)  // x * tmp / sum (lib.rs:110, :199)
                    a.X[(size_t)(o + k) * a.x_comp + (size_t)(j0 + c) * a.x_col] =
                        (plane(x[s][k], c) * plane(acc[s][k], c)) / a.norm[o + k];
    }
}

#define BATCH_RANK_CASES(X) \
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

// Rank buckets: ranks 1..8, 9..10 and 11..16 run as separate kernels, so
// the register budget of one bucket is not set by another's largest rank.
// Within a bucket one launch covers every rank class: CTA b runs item b.
constexpr int kBuckets = 3;
constexpr int kBucketHi[kBuckets] = {8, 10, kMaxBatchRank};  // largest rank of each
template <int B>
struct BBucket {
    static constexpr int kLo = B == 0 ? 1 : kBucketHi[B - 1] + 1;
    static constexpr int kHi = kBucketHi[B];
};
constexpr int bucket_of(int R) { return R <= kBucketHi[0] ? 0 : R <= kBucketHi[1] ? 1 : 2; }

// CTAs a multiprocessor keeps resident (the register cap) for a bucket and
// shape.  f32 carries four columns a thread, x and acc holding 8 R
// registers of packs: ranks 1..8 keep four CTAs (128 registers), 9..10
// three (168), 11..16 two (255).
template <typename T, int B, int SHAPE>
constexpr int min_blocks_for() {
    if constexpr (sizeof(T) == 4) return B == 0 ? 4 : B == 1 ? 3 : 2;
    return BShapes<T>::min_blocks[SHAPE];
}

template <typename T, int B, int SHAPE, bool kComponentFast>
__global__ void __launch_bounds__(kThreads, (min_blocks_for<T, B, SHAPE>()))
    batch_mu(MuArgs<T> a, const int *__restrict__ off, const BItem *__restrict__ items) {
    __shared__ __align__(16) BSmem<T> sm;
    const BItem it = items[blockIdx.x];
    constexpr int COMP = BShapes<T>::comp[SHAPE];
    switch (it.R) {
#define MU_CASE(r)                                                                     \
    case r:                                                                            \
        if constexpr (r >= BBucket<B>::kLo && r <= BBucket<B>::kHi)                    \
            mu_item<T, r, COMP, kComponentFast>(sm, a, off + it.goff, it.tile);        \
        break;
        BATCH_RANK_CASES(MU_CASE)
#undef MU_CASE
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

// dst (cols x ldd) = src (rows x cols, leading dimension lds) transposed,
// through 32 x 32 shared-memory tiles; dst columns [rows, ldd) are zeroed.
template <typename A, typename B>
__global__ void transpose_2d(const A *__restrict__ src, int64_t lds, B *__restrict__ dst,
                             int64_t ldd, int rows, int cols) {
    __shared__ B tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
    for (int y = ty; y < 32; y += 8) {
        const int r = r0 + y, c = c0 + tx;
        tile[y][tx] = (r < rows && c < cols) ? (B)src[(size_t)r * lds + c] : (B)0;
    }
    __syncthreads();
    for (int y = ty; y < 32; y += 8) {
        const int c = c0 + y, r = r0 + tx;
        if (c < cols && r < ldd) dst[(size_t)c * ldd + r] = tile[tx][y];
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
// Solves of rank R a CTA of shape `comp` carries (BCfg::NS).
int ns_for(int R, int comp) { return comp / R > 0 ? comp / R : 1; }

struct BatchPlan {
    int rtot = 0;
    std::vector<int> group_off;           // per group, NS offsets (-1 padded)
    std::vector<BItem> hitems, witems;    // bucket 0 items, then bucket 1, then 2
    int nh[kBuckets] = {}, nw[kBuckets] = {};  // items per bucket
};

// Solves of one rank form a class; a class is cut into groups of NS solves;
// every (group, tile) pair is one CTA of its bucket's launch.
template <typename T>
BatchPlan plan_batch(int n, int p, int nsolves, const int32_t *ranks, int comp) {
    BatchPlan bp;
    std::vector<int> offsets(nsolves);
    std::map<int, std::vector<int>> by_rank;
    for (int s = 0; s < nsolves; s++) {
        offsets[s] = bp.rtot;
        bp.rtot += ranks[s];
        by_rank[ranks[s]].push_back(s);
    }
    const int htiles = (p + kTile<T> - 1) / kTile<T>, wtiles = (n + kTile<T> - 1) / kTile<T>;
    for (int b = 0; b < kBuckets; b++) {
        // Larger ranks first: their CTAs are the longest, so they start first.
        for (auto it = by_rank.rbegin(); it != by_rank.rend(); ++it) {
            const int R = it->first;
            if (bucket_of(R) != b) continue;
            const auto &members = it->second;
            const int ns = ns_for(R, comp);
            const int groups = (int)((members.size() + ns - 1) / ns);
            for (int g = 0; g < groups; g++) {
                const int at = (int)bp.group_off.size();
                for (int i = 0; i < ns; i++) {
                    const size_t idx = (size_t)g * ns + i;
                    bp.group_off.push_back(idx < members.size() ? offsets[members[idx]] : -1);
                }
                for (int t = 0; t < htiles; t++) bp.hitems.push_back({R, at, t, 0});
                for (int t = 0; t < wtiles; t++) bp.witems.push_back({R, at, t, 0});
                bp.nh[b] += htiles;
                bp.nw[b] += wtiles;
            }
        }
    }
    return bp;
}

struct BatchDev {
    const int *off;
    const BItem *hitems, *witems;
};

template <typename T>
struct BatchSteps {
    MuArgs<T> h, w;  // the H step streams V, the W step streams V^T
};

// One step's launches, one per bucket with items (bucket b's items follow
// those of the buckets before it).
template <typename T, int SHAPE, bool kComponentFast>
void launch_buckets(const MuArgs<T> &a, const int *off, const BItem *items,
                    const int (&count)[kBuckets], cudaStream_t s, int64_t *launches) {
    static_assert(kBuckets == 3, "one launch per bucket");
    const BItem *at = items;
    if (count[0]) batch_mu<T, 0, SHAPE, kComponentFast><<<count[0], kThreads, 0, s>>>(a, off, at);
    at += count[0];
    if (count[1]) batch_mu<T, 1, SHAPE, kComponentFast><<<count[1], kThreads, 0, s>>>(a, off, at);
    at += count[1];
    if (count[2]) batch_mu<T, 2, SHAPE, kComponentFast><<<count[2], kThreads, 0, s>>>(a, off, at);
    *launches += (count[0] > 0) + (count[1] > 0) + (count[2] > 0);
}

// Enqueue iterations [it0, it1] of the batched brunet loop with shape SHAPE.
template <typename T, int SHAPE>
void enqueue_batch_iters_s(long long it0, long long it1, const BatchPlan &bp, const BatchDev &d,
                           const BatchSteps<T> &st, int n, int p, T *W, T *H, T *sw, T *sh,
                           cudaStream_t s, int64_t *launches) {
    const int rtot = bp.rtot;
    for (long long it = it0; it <= it1; it++) {
        batch_colsum<T><<<(rtot + 127) / 128, 128, 0, s>>>(W, n, rtot, rtot, sw);
        launch_buckets<T, SHAPE, true>(st.h, d.off, d.hitems, bp.nh, s, launches);
        batch_rowsum<T><<<(rtot + 7) / 8, 256, 0, s>>>(H, p, rtot, sh);
        launch_buckets<T, SHAPE, false>(st.w, d.off, d.witems, bp.nw, s, launches);
        *launches += 2;
        if (it % 10 == 0) {
            batch_clamp<T><<<592, 256, 0, s>>>(W, (int64_t)n * rtot, H, (int64_t)rtot * p,
                                               (T)DBL_EPSILON);
            *launches += 1;
        }
    }
}

template <typename T>
void enqueue_batch_iters(int shape, long long it0, long long it1, const BatchPlan &bp,
                         const BatchDev &d, const BatchSteps<T> &st, int n, int p, T *W, T *H,
                         T *sw, T *sh, cudaStream_t s, int64_t *launches) {
    static_assert(BShapes<T>::kN == 3, "one case per shape");
    switch (shape) {
        case 1:
            enqueue_batch_iters_s<T, 1>(it0, it1, bp, d, st, n, p, W, H, sw, sh, s, launches);
            break;
        case 2:
            enqueue_batch_iters_s<T, 2>(it0, it1, bp, d, st, n, p, W, H, sw, sh, s, launches);
            break;
        default:
            enqueue_batch_iters_s<T, 0>(it0, it1, bp, d, st, n, p, W, H, sw, sh, s, launches);
    }
}

// The autotuner's state, process-wide: the shape chosen per problem
// signature, a forced shape (nmfcu_batch_set_shape) and the last one used.
std::mutex g_shape_mu;
std::map<std::string, int> g_shape_cache;
int g_forced_shape = NMFCU_BATCH_SHAPE_AUTO;
int g_last_shape = -1;
constexpr long long kTuneMinIters = 20;  // shorter runs take shape 0 untimed
constexpr int kTuneIters = 3;            // timed iterations per candidate shape

std::string shape_key(int device, size_t es, int n, int p, int nsolves, const int32_t *ranks) {
    int hist[kMaxBatchRank + 1] = {0};
    for (int s = 0; s < nsolves; s++) hist[ranks[s]]++;
    std::string k = std::to_string(device) + "/" + std::to_string(es) + "/" + std::to_string(n) +
                    "x" + std::to_string(p);
    for (int r = 1; r <= kMaxBatchRank; r++) k += "," + std::to_string(hist[r]);
    return k;
}

// Uploads a plan's group offsets and items (context slot 0) and points `d`
// at them.
nmfcu_status upload_plan(nmfcu_context *c, const BatchPlan &bp, cudaStream_t s, BatchDev *d) {
    // One upload: group offsets, then H items, then W items (16-byte aligned).
    const size_t off_bytes = (sizeof(int) * bp.group_off.size() + 15) / 16 * 16;
    const size_t item_bytes = sizeof(BItem) * (bp.hitems.size() + bp.witems.size());
    std::vector<unsigned char> table(off_bytes + item_bytes, 0);
    std::memcpy(table.data(), bp.group_off.data(), sizeof(int) * bp.group_off.size());
    std::memcpy(table.data() + off_bytes, bp.hitems.data(), sizeof(BItem) * bp.hitems.size());
    std::memcpy(table.data() + off_bytes + sizeof(BItem) * bp.hitems.size(), bp.witems.data(),
                sizeof(BItem) * bp.witems.size());
    void *p_tab = nullptr;
    NMFCU_TRY(nmfcu_internal::context_buffer(c, 0, table.size(), &p_tab));
    // A pageable host source is staged before cudaMemcpyAsync returns, so the
    // table may go out of scope; the kernels read it in stream order.
    NMFCU_CUDA_TRY(cudaMemcpyAsync(p_tab, table.data(), table.size(), cudaMemcpyHostToDevice, s));
    d->off = static_cast<const int *>(p_tab);
    d->hitems = reinterpret_cast<const BItem *>(static_cast<unsigned char *>(p_tab) + off_bytes);
    d->witems = d->hitems + bp.hitems.size();
    return NMFCU_OK;
}

// The shape for this problem: the forced one, the cached choice, or the
// fastest of the candidates timed over kTuneIters iterations (after one
// untimed) on copies of the starting factors (context slots 16, 17), so
// that the caller's run itself is unchanged.  Blocks until the timing ends.
template <typename T>
nmfcu_status pick_shape(nmfcu_context *c, int64_t max_iter, int n, int p, const T *V,
                        int64_t ldv, const T *Vt, int64_t ldvt, int nsolves,
                        const int32_t *ranks, const T *W, const T *H, T *sw, T *sh,
                        cudaStream_t s, int64_t *launches, int *shape) {
    const std::string key = shape_key(nmfcu_internal::context_device(c), sizeof(T), n, p,
                                      nsolves, ranks);
    {
        std::lock_guard<std::mutex> lk(g_shape_mu);
        if (g_forced_shape >= 0) {
            *shape = g_forced_shape;
            return NMFCU_OK;
        }
        auto it = g_shape_cache.find(key);
        if (it != g_shape_cache.end()) {
            *shape = it->second;
            return NMFCU_OK;
        }
    }
    *shape = 0;
    if (max_iter < kTuneMinIters) return NMFCU_OK;
    int64_t rtot = 0;
    for (int i = 0; i < nsolves; i++) rtot += ranks[i];
    void *p_w = nullptr, *p_h = nullptr;
    NMFCU_TRY(nmfcu_internal::context_buffer(c, 16, sizeof(T) * (size_t)n * rtot, &p_w));
    NMFCU_TRY(nmfcu_internal::context_buffer(c, 17, sizeof(T) * (size_t)rtot * p, &p_h));
    T *W2 = static_cast<T *>(p_w), *H2 = static_cast<T *>(p_h);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    NMFCU_CUDA_TRY(cudaEventCreate(&e0));
    cudaError_t ce = cudaEventCreate(&e1);
    float best = 0.f;
    for (int v = 0; ce == cudaSuccess && v < BShapes<T>::kN; v++) {
        const BatchPlan bp = plan_batch<T>(n, p, nsolves, ranks, BShapes<T>::comp[v]);
        BatchDev d;
        const nmfcu_status ps = upload_plan(c, bp, s, &d);
        if (ps != NMFCU_OK) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return ps;
        }
        ce = cudaMemcpyAsync(W2, W, sizeof(T) * (size_t)n * rtot, cudaMemcpyDeviceToDevice, s);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(H2, H, sizeof(T) * (size_t)rtot * p, cudaMemcpyDeviceToDevice, s);
        if (ce != cudaSuccess) break;
        BatchSteps<T> st;
        st.h = MuArgs<T>{V, ldv, n, p, W2, (int64_t)bp.rtot, 1, H2, (int64_t)p, 1, sw};
        st.w = MuArgs<T>{Vt, ldvt, p, n, H2, 1, (int64_t)p, W2, 1, (int64_t)bp.rtot, sh};
        enqueue_batch_iters<T>(v, 1, 1, bp, d, st, n, p, W2, H2, sw, sh, s, launches);
        ce = cudaEventRecord(e0, s);
        if (ce != cudaSuccess) break;
        enqueue_batch_iters<T>(v, 2, 1 + kTuneIters, bp, d, st, n, p, W2, H2, sw, sh, s,
                               launches);
        ce = cudaEventRecord(e1, s);
        if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
        if (ce == cudaSuccess && (v == 0 || ms < best)) {
            best = ms;
            *shape = v;
        }
    }
    cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (ce != cudaSuccess) return nmfcu_internal::cuda_fail(ce, "batched shape timing");
    std::lock_guard<std::mutex> lk(g_shape_mu);
    g_shape_cache[key] = *shape;
    return NMFCU_OK;
}

// V (n x p, leading dimension ldv; for f32 zero in columns [p, ldv) with
// ldv a multiple of 4) is streamed by the H step; the W step streams V^T,
// built here once per call in context slot 12 (zero-padded the same way).
template <typename T>
nmfcu_status run_batch_t(nmfcu_context *c, int64_t max_iter, int n, int p, const T *V,
                         int64_t ldv, int nsolves, const int32_t *ranks, T *W, T *H,
                         cudaStream_t s) {
    int64_t rtot = 0;
    for (int i = 0; i < nsolves; i++) rtot += ranks[i];
    void *p_sw = nullptr, *p_sh = nullptr, *p_vt = nullptr;
    NMFCU_TRY(nmfcu_internal::context_buffer(c, 1, sizeof(T) * (size_t)rtot, &p_sw));
    NMFCU_TRY(nmfcu_internal::context_buffer(c, 2, sizeof(T) * (size_t)rtot, &p_sh));
    const int64_t ldvt = sizeof(T) == 4 ? ((int64_t)n + 3) / 4 * 4 : (int64_t)n;
    NMFCU_TRY(nmfcu_internal::context_buffer(c, 12, sizeof(T) * (size_t)p * ldvt, &p_vt));
    T *sw = static_cast<T *>(p_sw), *sh = static_cast<T *>(p_sh), *Vt = static_cast<T *>(p_vt);
    {
        const dim3 tg((unsigned)((p + 31) / 32), (unsigned)((ldvt + 31) / 32));
        transpose_2d<T, T><<<tg, 256, 0, s>>>(V, ldv, Vt, ldvt, n, p);
    }
    int64_t launches = 1;
    int shape = 0;
    NMFCU_TRY(pick_shape<T>(c, max_iter, n, p, V, ldv, Vt, ldvt, nsolves, ranks, W, H, sw, sh, s,
                            &launches, &shape));
    {
        std::lock_guard<std::mutex> lk(g_shape_mu);
        g_last_shape = shape;
    }
    const BatchPlan bp = plan_batch<T>(n, p, nsolves, ranks, BShapes<T>::comp[shape]);
    BatchDev d;
    NMFCU_TRY(upload_plan(c, bp, s, &d));
    BatchSteps<T> st;
    st.h = MuArgs<T>{V, ldv, n, p, W, (int64_t)bp.rtot, 1, H, (int64_t)p, 1, sw};
    st.w = MuArgs<T>{Vt, ldvt, p, n, H, 1, (int64_t)p, W, 1, (int64_t)bp.rtot, sh};
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
            enqueue_batch_iters<T>(shape, 1, 10, bp, d, st, n, p, W, H, sw, sh, cs,
                                   &cap_launches);
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
    enqueue_batch_iters<T>(shape, blocks * 10 + 1, max_iter, bp, d, st, n, p, W, H, sw, sh, s,
                           &launches);
    NMFCU_CUDA_TRY(cudaGetLastError());
    nmfcu_internal::count_launches(c, launches);
    return NMFCU_OK;
}

nmfcu_status validate_batch(int32_t method, int32_t precision, int64_t max_iter, int64_t n,
                            int64_t p, int32_t nsolves, const int32_t *ranks) {
    if (method != NMFCU_BRUNET)
        return fail(NMFCU_ERR_UNSUPPORTED, "batched solves are built for brunet only");
    // BF16X3 runs brunet (whose ratio is formed per element) as FP32, as the
    // single solve does.
    if (precision != NMFCU_PREC_FP64 && precision != NMFCU_PREC_FP32 &&
        precision != NMFCU_PREC_BF16X3)
        return fail(NMFCU_ERR_INVALID_ARG, "unknown precision id");
    if (max_iter < 0) return fail(NMFCU_ERR_INVALID_ARG, "max_iter must be >= 0");
    if (n < 1 || p < 1 || n > INT32_MAX || p > INT32_MAX)
        return fail(NMFCU_ERR_INVALID_ARG, "n and p must be in [1, 2^31)");
    if (nsolves < 1 || !ranks) return fail(NMFCU_ERR_INVALID_ARG, "need at least one solve");
    int64_t rtot = 0;
    for (int s = 0; s < nsolves; s++) {
        if (ranks[s] < 1 || ranks[s] > NMFCU_MAX_WIDE_RANK)
            return fail(NMFCU_ERR_UNSUPPORTED,
                        "batched ranks must be in [1, " + std::to_string(NMFCU_MAX_WIDE_RANK) + "]");
        rtot += ranks[s];
    }
    if (rtot > INT32_MAX) return fail(NMFCU_ERR_INVALID_ARG, "sum of ranks must fit in 32 bits");
    return NMFCU_OK;
}

}  // namespace

extern "C" {

nmfcu_status nmfcu_batch_set_shape(int32_t shape) {
    if (shape != NMFCU_BATCH_SHAPE_AUTO && (shape < 0 || shape >= kShapesMax))
        return fail(NMFCU_ERR_INVALID_ARG, "shape must be NMFCU_BATCH_SHAPE_AUTO or 0..count-1");
    std::lock_guard<std::mutex> lk(g_shape_mu);
    g_forced_shape = shape;
    return NMFCU_OK;
}

int32_t nmfcu_batch_shape_count(void) { return kShapesMax; }

int32_t nmfcu_batch_last_shape(void) {
    std::lock_guard<std::mutex> lk(g_shape_mu);
    return g_last_shape;
}

}  // extern "C"

namespace {

// The batched kernels on solves of ranks 1..kMaxBatchRank (checked).
nmfcu_status run_batch_narrow(nmfcu_context *ctx, int32_t precision, int64_t max_iter, int64_t n,
                              int64_t p, const double *dV, int64_t ldv, int32_t nsolves,
                              const int32_t *ranks, double *dW, double *dH, void *stream) {
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

// A batch with solves above kMaxBatchRank: the others run through the
// batched kernels on compacted copies of their stacked factors (context
// slots 20, 21); each wide solve runs alone through the single-solve engine
// in FP64 (ranks above 32 run only there) on a compact copy of its W
// (slot 22) and its rows of H in place.  Results are copied back into the
// stacked arrays.
nmfcu_status run_batch_mixed(nmfcu_context *ctx, int32_t precision, int64_t max_iter, int64_t n,
                             int64_t p, const double *dV, int64_t ldv, int32_t nsolves,
                             const int32_t *ranks, double *dW, double *dH, void *stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::vector<int64_t> off(nsolves);
    std::vector<int32_t> nranks;
    std::vector<int> nidx, widx;
    int64_t rtot = 0, rtot_n = 0, rmax_w = 0;
    for (int i = 0; i < nsolves; i++) {
        off[i] = rtot;
        rtot += ranks[i];
        if (ranks[i] <= kMaxBatchRank) {
            nidx.push_back(i);
            nranks.push_back(ranks[i]);
            rtot_n += ranks[i];
        } else {
            widx.push_back(i);
            rmax_w = std::max<int64_t>(rmax_w, ranks[i]);
        }
    }
    const size_t d8 = sizeof(double);
    void *wn = nullptr, *hn = nullptr, *ws = nullptr;
    // Copies of solve i's W columns between the stacked W (pitch rtot) and a
    // compact buffer (pitch `pitch`, first column `col`), either way.
    auto w_copy = [&](int i, double *buf, int64_t pitch, int64_t col, bool to_buf) {
        const size_t width = d8 * (size_t)ranks[i];
        if (to_buf)
            return cudaMemcpy2DAsync(buf + col, d8 * pitch, dW + off[i], d8 * rtot, width,
                                     (size_t)n, cudaMemcpyDeviceToDevice, s);
        return cudaMemcpy2DAsync(dW + off[i], d8 * rtot, buf + col, d8 * pitch, width, (size_t)n,
                                 cudaMemcpyDeviceToDevice, s);
    };
    if (!nidx.empty()) {
        {
            std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(ctx));
            nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(ctx));
            NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 20, d8 * (size_t)(n * rtot_n), &wn));
            NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 21, d8 * (size_t)(rtot_n * p), &hn));
            int64_t o = 0;
            for (int i : nidx) {
                NMFCU_CUDA_TRY(w_copy(i, (double *)wn, rtot_n, o, true));
                NMFCU_CUDA_TRY(cudaMemcpyAsync((double *)hn + o * p, dH + off[i] * p,
                                               d8 * (size_t)(ranks[i] * p),
                                               cudaMemcpyDeviceToDevice, s));
                o += ranks[i];
            }
        }
        NMFCU_TRY(run_batch_narrow(ctx, precision, max_iter, n, p, dV, ldv, (int32_t)nidx.size(),
                                   nranks.data(), (double *)wn, (double *)hn, stream));
        std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(ctx));
        nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(ctx));
        int64_t o = 0;
        for (int i : nidx) {
            NMFCU_CUDA_TRY(w_copy(i, (double *)wn, rtot_n, o, false));
            NMFCU_CUDA_TRY(cudaMemcpyAsync(dH + off[i] * p, (double *)hn + o * p,
                                           d8 * (size_t)(ranks[i] * p), cudaMemcpyDeviceToDevice,
                                           s));
            o += ranks[i];
        }
    }
    nmfcu_options opt;
    nmfcu_options_default(&opt);
    opt.method = NMFCU_BRUNET;
    opt.stop = NMFCU_STOP_MAX_ITER;
    opt.max_iter = max_iter;
    opt.precision = NMFCU_PREC_FP64;
    opt.device = nmfcu_internal::context_device(ctx);
    for (int i : widx) {
        {
            std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(ctx));
            nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(ctx));
            NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 22, d8 * (size_t)(n * rmax_w), &ws));
            NMFCU_CUDA_TRY(w_copy(i, (double *)ws, ranks[i], 0, true));
        }
        int64_t ndev = 0, nit = 0;
        NMFCU_TRY(nmfcu_run_device(ctx, &opt, n, p, ranks[i], dV, NMFCU_F64, ldv, nullptr, 0,
                                   (double *)ws, dH + off[i] * p, nullptr, &ndev, &nit, stream));
        std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(ctx));
        nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(ctx));
        NMFCU_CUDA_TRY(w_copy(i, (double *)ws, ranks[i], 0, false));
    }
    NMFCU_CUDA_TRY(cudaStreamSynchronize(s));
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
    for (int i = 0; i < nsolves; i++)
        if (ranks[i] > kMaxBatchRank)
            return run_batch_mixed(ctx, precision, max_iter, n, p, dV, ldv, nsolves, ranks, dW,
                                   dH, stream);
    return run_batch_narrow(ctx, precision, max_iter, n, p, dV, ldv, nsolves, ranks, dW, dH,
                            stream);
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

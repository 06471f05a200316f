// stream.cuh -- the two V-streaming passes of an NMF iteration, fed by TMA.
//
// Each pass is one kernel with one CTA (8 or 16 warps) per SM.  V tiles (and
// the W rows / H^T columns that pair with them) arrive by
// cp.async.bulk.tensor into a ring of shared-memory stages, each guarded by a
// "full" mbarrier; all warps do the FMAs out of shared memory, so no LSU
// instruction waits on HBM.  A stage is refilled by the last warp to finish
// with it (a per-stage arrival counter in shared memory), so no warp ever
// blocks waiting to refill and the ring keeps STAGES - 1 units in flight.
// (A separate producer warp would put an extra warp on one SM sub-partition
// and cap every thread below the registers the FMA loops need.)
//
// Work split ("stream-K"): a tile is TCOLS columns x one segment of at most
// 2048 rows (H pass), or TROWS rows x one segment of at most 2048 columns (W
// pass); a unit is one stage of one tile.  The U units of all tiles are dealt
// out in equal contiguous ranges, so every CTA streams the same number of
// bytes whatever the tile count.  A CTA writes a partial sum for every tile
// its range touches (at most `slots` of them), and the epilogue adds the
// partials of an output row / column over segments and CTAs in a fixed
// order: deterministic, no atomics.  Segments bound every f32 running sum to
// 2048 terms; all sums across segments and CTAs are f64.
//
//   H pass  A[k][j] = sum_u W[u][k] V[u][j]              (lee, hals, dnmf)
//           A[k][j] = sum_u W[u][k] V[u][j] / (WH)[u][j]   (brunet)
//     thread = CPT adjacent columns, all rows; W rows broadcast from smem.
//     f32 products use the packed FFMA2 (two k at a time).
//   W pass  B[i][k] = sum_j V[i][j] H[k][j]
//           B[i][k] = sum_j H[k][j] V[i][j] / (WH)[i][j]
//     thread = RT rows, all columns; V rows read from a 128B-swizzled tile,
//     H^T columns broadcast from smem.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "kernels.cuh"

namespace nmfcu {

// Iterations of mbarrier.try_wait before a wait is declared failed.  Each
// try_wait may itself suspend briefly, so this bounds a wait to well under a
// few seconds; a kernel that gives up records it in RunState::timeout.
constexpr uint32_t kSpinLimit = 1u << 22;
enum : int { TIMEOUT_FULL = 1 };

// ---------------------------------------------------------------------------
// PTX wrappers (mbarrier, TMA)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase of parity `parity` to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (uint32_t i = 0; i < kSpinLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
// The same with an L2 cache policy (createpolicy) for the loaded lines.
__device__ __forceinline__ void tma_load_2d_hint(void *dst, const CUtensorMap *map, uint64_t *bar,
                                                 int x, int y, uint64_t policy) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void record_timeout(RunState *st, int code) {
    if (st) atomicCAS(&st->timeout, 0, code);
}

// ---------------------------------------------------------------------------
// Stream-K bookkeeping
// ---------------------------------------------------------------------------
struct StreamK {
    long long U;  // units in all tiles
    int G;        // CTAs (G <= U, so no CTA is empty)
    int UPT;      // units per tile (= per segment)
    int slots;    // partial slots per CTA
    int nseg;     // segments per major tile (tile t = major * nseg + segment)
    // 0: one partial per (CTA, tile).  1: one per (CTA, major tile) -- the
    // pass adds a CTA's segments of a major tile in f64 before writing it,
    // and `slots` counts major tiles.
    int fold;
    // Units of a major tile that carry data: a prefix of its nseg * UPT (the
    // rest pad its last segment).  A CTA that meets a major tile only in
    // its padding may write no partial for it.
    int valid;
    __host__ __device__ __forceinline__ long long start(int b) const {
        return (long long)b * U / G;
    }
    // Units of a major tile.
    __host__ __device__ __forceinline__ long long major_units() const {
        return (long long)nseg * UPT;
    }
};

// CTAs [lo, hi] whose unit range meets units [a, e) (a < e <= U).
__device__ __forceinline__ void sk_range_units(const StreamK &sk, long long a, long long e,
                                               int *lo, int *hi) {
    int l = 0, h = sk.G - 1;
    while (l < h) {  // first b with start(b + 1) > a
        const int m = (l + h) >> 1;
        if (sk.start(m + 1) > a) h = m; else l = m + 1;
    }
    *lo = l;
    l = 0;
    h = sk.G - 1;
    while (l < h) {  // last b with start(b) < e
        const int m = (l + h + 1) >> 1;
        if (sk.start(m) < e) l = m; else h = m - 1;
    }
    *hi = l;
}

// CTAs [lo, hi] whose unit range meets tile t.
__device__ __forceinline__ void sk_range(const StreamK &sk, int t, int *lo, int *hi) {
    const long long a = (long long)t * sk.UPT;
    sk_range_units(sk, a, min(a + sk.UPT, sk.U), lo, hi);
}

// CTAs [lo, hi] whose unit range meets the units of major tile m that carry
// data (folded partials).
__device__ __forceinline__ void sk_range_major(const StreamK &sk, int m, int *lo, int *hi) {
    const long long a = (long long)m * sk.major_units();
    sk_range_units(sk, a, min(a + (long long)sk.valid, sk.U), lo, hi);
}

// Slot of major tile m in CTA b's folded partials.
__device__ __forceinline__ int fold_slot(const StreamK &sk, int b, int m) {
    return m - (int)(sk.start(b) / sk.major_units());
}

// Slot of tile t among the partials of a CTA whose first tile is tile0, and
// whether the write adds to it: with folded partials a later segment of the
// major tile written last adds to that slot.  Flushes come in tile order;
// `last` is the major tile of the previous flush (-1 before the first).
__device__ __forceinline__ size_t partial_slot(const StreamK &sk, int t, int tile0, int &last,
                                               bool &add) {
    if (!sk.fold) {
        add = false;
        return (size_t)(t - tile0);
    }
    const int m = t / sk.nseg;
    add = (m == last);
    last = m;
    return (size_t)(m - tile0 / sk.nseg);
}
// Write (or, folding, add) one partial value.  Only the thread that wrote
// an element adds to it later, so no other thread's write intervenes.
__device__ __forceinline__ void put_partial(double *d, double v, bool add) {
    *d = add ? *d + v : v;
}

// Position of a unit in the tile order, advanced one unit at a time so that
// the loops do no integer division (a runtime 64-bit division per unit costs
// more than the arithmetic of a small unit).
struct UnitCursor {
    int t;       // tile = major * nseg + seg
    int within;  // unit within the tile (segment)
    int major;   // column tile (H pass) / row tile (W pass)
    int seg;     // segment within the major tile
    __device__ __forceinline__ void init(const StreamK &sk, long long u) {
        t = (int)(u / sk.UPT);
        within = (int)(u - (long long)t * sk.UPT);
        major = t / sk.nseg;
        seg = t - major * sk.nseg;
    }
    __device__ __forceinline__ void next(const StreamK &sk) {
        if (++within == sk.UPT) {
            within = 0;
            ++t;
            if (++seg == sk.nseg) {
                seg = 0;
                ++major;
            }
        }
    }
    // Unit index along the major tile (row block / column block).
    __device__ __forceinline__ int along(const StreamK &sk) const { return seg * sk.UPT + within; }
};

// Orders this thread's earlier generic-proxy shared-memory accesses before
// its later async-proxy (TMA) writes to shared memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// End of a warp's work on stage `s`: count the warp in; the last of `warps`
// to arrive resets the counter and refills the stage with the unit `next`
// (if `has_next`).  Called by one lane per warp after __syncwarp().
template <int STAGE_BYTES, int TX_BYTES, typename Issue>
__device__ __forceinline__ void release_stage(unsigned char *smem, uint64_t *full, int *arrivals,
                                              int s, int warps, bool has_next,
                                              const UnitCursor &next, Issue &&issue) {
    __threadfence_block();  // this warp's reads of the stage before the count
    if (atomicAdd(&arrivals[s], 1) == warps - 1) {
        __threadfence_block();  // every warp's reads before the refill
        arrivals[s] = 0;
        if (has_next) {
            fence_proxy_async_smem();
            mbar_expect_tx(&full[s], TX_BYTES);
            issue(smem + s * STAGE_BYTES, &full[s], next);
        }
    }
}

template <typename T, int RP>
struct RankPad {
    // W rows / H^T rows padded to 16 bytes (the TMA inner-box granule).
    static constexpr int RPS = ((RP * (int)sizeof(T) + 15) / 16 * 16) / (int)sizeof(T);
};

// Vector load of N consecutive T from shared memory (16 / 8 / 4 B aligned).
template <typename T, int N>
__device__ __forceinline__ void lds_vec(T (&dst)[N], const T *src) {
    if constexpr (sizeof(T) * N == 16) {
        const float4 x = *reinterpret_cast<const float4 *>(src);
        const T *y = reinterpret_cast<const T *>(&x);
#pragma unroll
        for (int i = 0; i < N; i++) dst[i] = y[i];
    } else if constexpr (sizeof(T) * N == 8) {
        const float2 x = *reinterpret_cast<const float2 *>(src);
        const T *y = reinterpret_cast<const T *>(&x);
#pragma unroll
        for (int i = 0; i < N; i++) dst[i] = y[i];
    } else {
#pragma unroll
        for (int i = 0; i < N; i++) dst[i] = src[i];
    }
}

// N consecutive values from shared memory into registers, in vectors of up to
// 16 bytes; ALIGN is the byte alignment the caller guarantees for `src`.
template <typename T, int N, int ALIGN = 16>
__device__ __forceinline__ void lds_row(T (&dst)[N], const T *src) {
    constexpr int VB = ALIGN >= 16 ? 16 : (ALIGN >= 8 ? 8 : (int)sizeof(T));
    constexpr int V = VB / (int)sizeof(T) > 0 ? VB / (int)sizeof(T) : 1;
#pragma unroll
    for (int k0 = 0; k0 < N; k0 += V) {
        T tmp[V];
        lds_vec<T, V>(tmp, src + k0);
#pragma unroll
        for (int i = 0; i < V; i++)
            if (k0 + i < N) dst[k0 + i] = tmp[i];
    }
}

// Byte alignment of an offset of `elems` T within a 16-byte aligned row.
template <typename T>
__host__ __device__ constexpr int align_of_offset(int elems) {
    return (elems * (int)sizeof(T)) % 16 == 0 ? 16 : ((elems * (int)sizeof(T)) % 8 == 0 ? 8 : 4);
}

// acc[k] += a[k] * x for k < RP.  f32: packed FFMA2 on pairs of k (RP is
// even); f64: one DFMA per k.
template <int RP>
__device__ __forceinline__ void axpy(float (&acc)[RP], const float (&a)[RP], float x) {
    const float2 xx = make_float2(x, x);
#pragma unroll
    for (int k = 0; k + 1 < RP; k += 2) {
        const float2 r = __ffma2_rn(make_float2(a[k], a[k + 1]), xx,
                                    make_float2(acc[k], acc[k + 1]));
        acc[k] = r.x;
        acc[k + 1] = r.y;
    }
    if constexpr (RP % 2 == 1) acc[RP - 1] = fmaf(a[RP - 1], x, acc[RP - 1]);
}
template <int RP>
__device__ __forceinline__ void axpy(double (&acc)[RP], const double (&a)[RP], double x) {
#pragma unroll
    for (int k = 0; k < RP; k++) acc[k] = fma(a[k], x, acc[k]);
}

// sum_k a[k] * b[k].  f32: two packed partial sums, added at the end.
template <int RP>
__device__ __forceinline__ float dot(const float (&a)[RP], const float (&b)[RP]) {
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k + 1 < RP; k += 2)
        s = __ffma2_rn(make_float2(a[k], a[k + 1]), make_float2(b[k], b[k + 1]), s);
    if constexpr (RP % 2 == 1) s.x = fmaf(a[RP - 1], b[RP - 1], s.x);
    return s.x + s.y;
}
template <int RP>
__device__ __forceinline__ double dot(const double (&a)[RP], const double (&b)[RP]) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < RP; k++) s = fma(a[k], b[k], s);
    return s;
}

// Register blocking.  The rank range is split in KS = 2 halves across the
// two half-warps (lanes 0-15 take k < RP/2, lanes 16-31 the rest), so that a
// thread can own several columns (H pass) or rows (W pass) and reuse every
// shared-memory load for several FMAs.  Where a pass needs a full dot
// product over k (the brunet ratio), the two halves are added with one
// shfl_xor(16).
constexpr int KS = 2;

// Warp count from the 32-bit registers a thread's live arrays take: 16 warps
// (128 registers a thread) when the estimate leaves room for addressing and
// loop state, else 8 (255 registers).  `limit` is the estimate that still
// compiled without spills at 128 registers (80; 64 for the f64 ratio
// kernels, whose IEEE divide sequence needs more).
__host__ __device__ constexpr int warps_for(int regs, int limit) {
    return regs <= limit ? 16 : 8;
}
template <typename T, bool RATIO>
__host__ __device__ constexpr int reg_limit() {
    return (sizeof(T) == 8 && RATIO) ? 64 : 80;
}

// Rows / columns a segment may span (bounds every f32 running sum).
constexpr int kSegSpan = 2048;
// Units a segment may span in the f64 passes: unbounded, so that a tile is
// one segment and its running sums stay in registers until the tile ends.
constexpr int kSegNone = 1 << 30;

// ---------------------------------------------------------------------------
// H pass
// ---------------------------------------------------------------------------
template <typename T, int RP, bool RATIO>
struct HCfg {
    static constexpr int W32 = (int)sizeof(T) / 4;  // 32-bit registers per T
    static constexpr int KB = RP / KS;               // k per thread
    static constexpr int LPK = 32 / KS;              // lanes per k-half
    // Columns per thread: more where one column's arithmetic is cheap; two in
    // the f32 ratio pass, whose per-column chain (dot, exchange, reciprocal,
    // axpy) needs a second independent chain to hide its latency.
    static constexpr int CPT = RATIO ? (sizeof(T) == 4 ? 2 : 1) : (sizeof(T) == 4 ? 4 : 2);
    static constexpr int REGS = W32 * (CPT * KB * (RATIO ? 2 : 1) + KB + CPT);
    static constexpr int kWarps = warps_for(REGS, reg_limit<T, RATIO>());
    static constexpr int TCOLS = LPK * CPT * kWarps;
    static constexpr int BOXC = TCOLS < 256 ? TCOLS : 256;
    static constexpr int NBOX = TCOLS / BOXC;
    static constexpr int BROWS = 8;
    static constexpr int SEGU = sizeof(T) == 8 ? kSegNone : kSegSpan / BROWS;  // max units per segment
    static constexpr int RPS = RankPad<T, RP>::RPS;
    static constexpr int KALIGN = align_of_offset<T>(KB);
    static constexpr int VBYTES = BROWS * TCOLS * (int)sizeof(T);
    static constexpr int WBYTES = BROWS * RPS * (int)sizeof(T);
    static constexpr int STAGE = (VBYTES + WBYTES + 1023) / 1024 * 1024;
    static constexpr int STAGES_FIT = (220 * 1024) / STAGE;
    static constexpr int STAGES = STAGES_FIT > 10 ? 10 : STAGES_FIT;
    static constexpr int SMEM = STAGES * STAGE + 2 * STAGES * 8 + 1024;
    static_assert(RP % KS == 0, "rank buckets are even");
    static_assert(STAGES >= 3, "a ring needs stages in flight");
};

// RATIO: each V element enters as v / (W H)_ij (0 where W H is 0); with
// WEIGHTED as v (W H)_ij instead (lsNMF's denominator, V holding the weights).
template <typename T, int RP, bool RATIO, bool WEIGHTED = false>
__global__ void __launch_bounds__(HCfg<T, RP, RATIO>::kWarps * 32, 1)
    hpass(const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmW,
          const double *__restrict__ H, int n, int p, StreamK sk, double *__restrict__ part,
          RunState *st) {
    using C = HCfg<T, RP, RATIO>;
    constexpr int CPT = C::CPT, KB = C::KB;
    if (run_stopped(st)) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024 B alignment for the boxes, by offsetting the shared array itself so
    // that every access stays a shared-memory (LDS) access.
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + C::STAGES * C::STAGE);
    int *arrivals = reinterpret_cast<int *>(full + C::STAGES);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer = (threadIdx.x == 0);
    const int b = blockIdx.x;
    const long long u0 = sk.start(b), u1 = sk.start(b + 1);
    const long long nunits = u1 - u0;

    // Loads of one unit: the V boxes of its columns and rows, and its W rows.
    auto issue = [&](unsigned char *stg, uint64_t *bar, const UnitCursor &c) {
        const int rb = c.along(sk);
#pragma unroll
        for (int q = 0; q < C::NBOX; q++)
            tma_load_2d(stg + q * C::BROWS * C::BOXC * (int)sizeof(T), &tmV, bar,
                        c.major * C::TCOLS + q * C::BOXC, rb * C::BROWS);
        tma_load_2d(stg + C::VBYTES, &tmW, bar, 0, rb * C::BROWS);
    };
    // `ahead`: the unit STAGES after the one being consumed (lane 0 of each
    // warp keeps one, for the refill it may have to issue).
    UnitCursor ahead;
    ahead.init(sk, u0);
    if (producer) {
        for (int s = 0; s < C::STAGES; s++) {
            mbar_init(&full[s], 1);
            arrivals[s] = 0;
        }
        fence_mbar_init();
        for (int j = 0; j < C::STAGES; j++) {
            if (j < nunits) {
                mbar_expect_tx(&full[j], C::VBYTES + C::WBYTES);
                issue(smem + j * C::STAGE, &full[j], ahead);
            }
            ahead.next(sk);
        }
    } else {
        for (int j = 0; j < C::STAGES; j++) ahead.next(sk);
    }
    __syncthreads();

    const int kh = lane / C::LPK, cl = lane % C::LPK;
    const int k0 = kh * KB;                                // this thread's k range
    const int colw = (warp * C::LPK + cl) * CPT;           // first column within the tile
    const int box = colw / C::BOXC, boff = colw % C::BOXC;
    T acc[CPT][KB];
    T hcol[RATIO ? CPT : 1][RATIO ? KB : 1];
    int cur = -1;
    UnitCursor uc;
    uc.init(sk, u0);
    const int tile0 = uc.t;
    int flast = -1;  // major tile of the last flush
    int s = 0, rnd = 0;
    bool ok = true;

    auto flush = [&](int t) {
        bool add;
        const size_t slot = partial_slot(sk, t, tile0, flast, add);
        double *dst = part + ((size_t)b * sk.slots + slot) * RP * C::TCOLS + colw;
#pragma unroll
        for (int k = 0; k < KB; k++)
#pragma unroll
            for (int c = 0; c < CPT; c++)
                put_partial(&dst[(size_t)(k0 + k) * C::TCOLS + c], (double)acc[c][k], add);
    };

    int cur_major = -1;
    for (long long i = 0; i < nunits; ++i) {
        const int t = uc.t;
        if (t != cur) {
            if (cur >= 0) flush(cur);
            cur = t;
#pragma unroll
            for (int c = 0; c < CPT; c++)
#pragma unroll
                for (int k = 0; k < KB; k++) acc[c][k] = (T)0;
            if constexpr (RATIO) {
                if (uc.major != cur_major) {
                    cur_major = uc.major;
#pragma unroll
                    for (int c = 0; c < CPT; c++) {
                        const int j = uc.major * C::TCOLS + colw + c;
#pragma unroll
                        for (int k = 0; k < KB; k++)
                            hcol[c][k] = (j < p) ? (T)H[(size_t)(k0 + k) * p + j] : (T)0;
                    }
                }
            }
        }
        if (!mbar_wait(&full[s], (uint32_t)(rnd & 1))) {
            record_timeout(st, TIMEOUT_FULL);
            ok = false;
            break;
        }
        const unsigned char *stg = smem + s * C::STAGE;
        const T *sv = reinterpret_cast<const T *>(stg) + box * C::BROWS * C::BOXC + boff;
        const T *sw = reinterpret_cast<const T *>(stg + C::VBYTES) + k0;
#pragma unroll 2
        for (int r = 0; r < C::BROWS; r++) {
            T v[CPT];
            lds_vec<T, CPT>(v, sv + r * C::BOXC);
            T w[KB];
            lds_row<T, KB, C::KALIGN>(w, sw + r * C::RPS);
#pragma unroll
            for (int c = 0; c < CPT; c++) {
                if constexpr (RATIO) {
                    T wh = dot<KB>(w, hcol[c]);
                    wh += __shfl_xor_sync(0xffffffffu, wh, C::LPK);  // the other k-half
                    T q;
                    if constexpr (WEIGHTED)
                        q = v[c] * wh;
                    else
                        q = (wh != (T)0) ? ratio_div(v[c], wh) : (T)0;
                    axpy<KB>(acc[c], w, q);
                } else {
                    axpy<KB>(acc[c], w, v[c]);
                }
            }
        }
        __syncwarp();
        if (lane == 0)
            release_stage<C::STAGE, C::VBYTES + C::WBYTES>(smem, full, arrivals, s, C::kWarps,
                                                           i + C::STAGES < nunits, ahead, issue);
        ahead.next(sk);
        if (++s == C::STAGES) {
            s = 0;
            ++rnd;
        }
        uc.next(sk);
    }
    if (ok && cur >= 0) flush(cur);
}

// ---------------------------------------------------------------------------
// W pass
// ---------------------------------------------------------------------------
template <typename T, int RP, bool RATIO>
struct WCfg {
    static constexpr int W32 = (int)sizeof(T) / 4;
    static constexpr int KB = RP / KS;
    static constexpr int LPK = 32 / KS;
    // Rows per thread: more where one row's arithmetic is cheap.
    static constexpr int RT = RATIO ? (sizeof(T) == 4 ? 2 : 1) : (sizeof(T) == 4 ? 4 : 2);
    static constexpr int REGS = W32 * (RT * KB * (RATIO ? 2 : 1) + KB + 2 * RT);
    static constexpr int kWarps = warps_for(REGS, reg_limit<T, RATIO>());
    static constexpr int TROWS = LPK * RT * kWarps;       // rows per tile
    static constexpr int BOXR = TROWS < 256 ? TROWS : 256;  // rows per V box
    static constexpr int NBOX = TROWS / BOXR;
    // Bytes of a row per unit: a 32 KB stage, at most one 128 B swizzle span.
    static constexpr int ROWB = 32768 / TROWS < 128 ? 32768 / TROWS : 128;
    static constexpr int BCOLS = ROWB / (int)sizeof(T);   // columns per unit
    static constexpr int CHUNKS = ROWB / 16;              // 16 B chunks per row
    static constexpr int SEGU = sizeof(T) == 8 ? kSegNone : kSegSpan / BCOLS;  // max units per segment
    // TMA swizzle of span ROWB: logical chunk c of row r sits at physical
    // chunk c ^ ((r * ROWB >> 7) & (CHUNKS - 1)).
    static constexpr int RPS = RankPad<T, RP>::RPS;
    static constexpr int KALIGN = align_of_offset<T>(KB);
    static constexpr int VBYTES = TROWS * ROWB;
    static constexpr int HBYTES = BCOLS * RPS * (int)sizeof(T);
    static constexpr int STAGE = (VBYTES + HBYTES + 1023) / 1024 * 1024;
    static constexpr int STAGES_FIT = (220 * 1024) / STAGE;
    static constexpr int STAGES = STAGES_FIT > 8 ? 8 : STAGES_FIT;
    static constexpr int SMEM = STAGES * STAGE + 2 * STAGES * 8 + 1024;
    static_assert(STAGES >= 3, "a ring needs stages in flight");
    static_assert(ROWB == 32 || ROWB == 64 || ROWB == 128, "swizzle span");
    static_assert(TROWS % BOXR == 0, "whole boxes");
};

template <typename T, int RP, bool RATIO, bool WEIGHTED = false>
__global__ void __launch_bounds__(WCfg<T, RP, RATIO>::kWarps * 32, 1)
    wpass(const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmH,
          const double *__restrict__ W, int n, int p, StreamK sk, double *__restrict__ part,
          RunState *st) {
    using C = WCfg<T, RP, RATIO>;
    constexpr int RT = C::RT, KB = C::KB;
    constexpr int VEC = 16 / (int)sizeof(T);  // columns per 16-byte chunk
    if (run_stopped(st)) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + C::STAGES * C::STAGE);
    int *arrivals = reinterpret_cast<int *>(full + C::STAGES);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer = (threadIdx.x == 0);
    const int b = blockIdx.x;
    const long long u0 = sk.start(b), u1 = sk.start(b + 1);
    const long long nunits = u1 - u0;

    // Loads of one unit: NBOX boxes of BOXR rows x BCOLS columns of V
    // (swizzled) and the matching BCOLS rows of H^T.
    auto issue = [&](unsigned char *stg, uint64_t *bar, const UnitCursor &c) {
        const int cb = c.along(sk);
#pragma unroll
        for (int q = 0; q < C::NBOX; q++)
            tma_load_2d(stg + q * C::BOXR * C::ROWB, &tmV, bar, cb * C::BCOLS,
                        c.major * C::TROWS + q * C::BOXR);
        tma_load_2d(stg + C::VBYTES, &tmH, bar, 0, cb * C::BCOLS);
    };
    // `ahead`: the unit STAGES after the one being consumed (lane 0 of each
    // warp keeps one, for the refill it may have to issue).
    UnitCursor ahead;
    ahead.init(sk, u0);
    if (producer) {
        for (int s = 0; s < C::STAGES; s++) {
            mbar_init(&full[s], 1);
            arrivals[s] = 0;
        }
        fence_mbar_init();
        for (int j = 0; j < C::STAGES; j++) {
            if (j < nunits) {
                mbar_expect_tx(&full[j], C::VBYTES + C::HBYTES);
                issue(smem + j * C::STAGE, &full[j], ahead);
            }
            ahead.next(sk);
        }
    } else {
        for (int j = 0; j < C::STAGES; j++) ahead.next(sk);
    }
    __syncthreads();

    const int kh = lane / C::LPK, rl = lane % C::LPK;
    const int k0 = kh * KB;
    // Rows of this thread within the tile: a warp owns LPK * RT consecutive
    // rows; lane rl takes rows rl, rl + LPK, ... (a half-warp's loads touch
    // LPK distinct rows, the other half-warp reads the same rows).
    int rows[RT];
    int swz[RT];
#pragma unroll
    for (int q = 0; q < RT; q++) {
        rows[q] = warp * C::LPK * RT + q * C::LPK + rl;
        swz[q] = ((rows[q] * C::ROWB) >> 7) & (C::CHUNKS - 1);
    }
    T acc[RT][KB];
    T wrow[RATIO ? RT : 1][RATIO ? KB : 1];
    int cur = -1;
    UnitCursor uc;
    uc.init(sk, u0);
    const int tile0 = uc.t;
    int flast = -1;  // major tile of the last flush
    int s = 0, rnd = 0;
    bool ok = true;

    auto flush = [&](int t) {
        bool add;
        const size_t slot = partial_slot(sk, t, tile0, flast, add);
        double *dst = part + ((size_t)b * sk.slots + slot) * C::TROWS * RP + k0;
#pragma unroll
        for (int q = 0; q < RT; q++)
#pragma unroll
            for (int k = 0; k < KB; k++)
                put_partial(&dst[(size_t)rows[q] * RP + k], (double)acc[q][k], add);
    };

    int cur_major = -1;
    for (long long i = 0; i < nunits; ++i) {
        const int t = uc.t;
        if (t != cur) {
            if (cur >= 0) flush(cur);
            cur = t;
#pragma unroll
            for (int q = 0; q < RT; q++)
#pragma unroll
                for (int k = 0; k < KB; k++) acc[q][k] = (T)0;
            if constexpr (RATIO) {
                if (uc.major != cur_major) {
                    cur_major = uc.major;
#pragma unroll
                    for (int q = 0; q < RT; q++) {
                        const int row = uc.major * C::TROWS + rows[q];
#pragma unroll
                        for (int k = 0; k < KB; k++)
                            wrow[q][k] = (row < n) ? (T)W[(size_t)row * RP + k0 + k] : (T)0;
                    }
                }
            }
        }
        if (!mbar_wait(&full[s], (uint32_t)(rnd & 1))) {
            record_timeout(st, TIMEOUT_FULL);
            ok = false;
            break;
        }
        const unsigned char *stg = smem + s * C::STAGE;
        const T *sh = reinterpret_cast<const T *>(stg + C::VBYTES) + k0;
#pragma unroll
        for (int ci = 0; ci < C::CHUNKS; ci++) {
            T v[RT][VEC];
#pragma unroll
            for (int q = 0; q < RT; q++)
                lds_vec<T, VEC>(v[q], reinterpret_cast<const T *>(
                                          stg + rows[q] * C::ROWB + ((ci ^ swz[q]) << 4)));
#pragma unroll
            for (int e = 0; e < VEC; e++) {
                T hc[KB];
                lds_row<T, KB, C::KALIGN>(hc, sh + (ci * VEC + e) * C::RPS);
#pragma unroll
                for (int q = 0; q < RT; q++) {
                    if constexpr (RATIO) {
                        T wh = dot<KB>(wrow[q], hc);
                        wh += __shfl_xor_sync(0xffffffffu, wh, C::LPK);  // the other k-half
                        T qv;
                        if constexpr (WEIGHTED)
                            qv = v[q][e] * wh;
                        else
                            qv = (wh != (T)0) ? ratio_div(v[q][e], wh) : (T)0;
                        axpy<KB>(acc[q], hc, qv);
                    } else {
                        axpy<KB>(acc[q], hc, v[q][e]);
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0)
            release_stage<C::STAGE, C::VBYTES + C::HBYTES>(smem, full, arrivals, s, C::kWarps,
                                                           i + C::STAGES < nunits, ahead, issue);
        ahead.next(sk);
        if (++s == C::STAGES) {
            s = 0;
            ++rnd;
        }
        uc.next(sk);
    }
    if (ok && cur >= 0) flush(cur);
}

// ---------------------------------------------------------------------------
// FP64 plain passes on the FP64 tensor cores (lee / hals / dnmf / offset,
// the lsNMF numerators and the NNDSVD products in the plain method)
// ---------------------------------------------------------------------------
// mma.sync.m8n8k4 with f64 operands: D (8 x 8) += A (8 x 4) B (4 x 8), one
// A and one B element and two D elements a thread (A[g][q], B[q][g],
// D[g][2q + e] with g = lane / 4, q = lane % 4).  One instruction does 256
// FMAs, where the CUDA-core passes issue one DFMA (and its operand loads)
// per 32; the ring, stream-K split and partial layouts are the CUDA-core
// passes' own, so the epilogues are shared.  The asm has no side effects
// beyond its operands (not volatile), so independent MMAs may be scheduled
// across one another; each accumulator's chain keeps its order.
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

// H pass: A[k][j] = sum_u W[u][k] V[u][j] with M = k (rank tiles of 8), N = j
// (4 column tiles of 8 a warp), K = u (4 rows a k-step, 4 k-steps a unit of
// 16 rows, so that a stage's wait and release serve 4 k-steps).
template <int RP>
struct DHCfg {
    static constexpr int MT = (RP + 7) / 8;
    // 16 warps of at most 128 registers; ranks above 24 (four rank tiles of
    // accumulators) take 8 warps and their 255 registers.
    static constexpr int kWarps = MT >= 4 ? 8 : 16;
    static constexpr int NT = 4;
    static constexpr int WCOLS = NT * 8;
    static constexpr int TCOLS = kWarps * WCOLS;  // 512 columns a tile
    static constexpr int BOXC = 256;
    static constexpr int NBOX = TCOLS / BOXC;
    static constexpr int BROWS = 16;
    static constexpr int SEGU = kSegNone;  // f64 sums: one segment a tile
    static constexpr int RPS = RankPad<double, RP>::RPS;
    static constexpr int VBYTES = BROWS * TCOLS * 8;
    static constexpr int WBYTES = BROWS * RPS * 8;
    static constexpr int STAGE = (VBYTES + WBYTES + 1023) / 1024 * 1024;
    static constexpr int STAGES_FIT = (220 * 1024) / STAGE;
    static constexpr int STAGES = STAGES_FIT > 10 ? 10 : STAGES_FIT;
    static constexpr int SMEM = STAGES * STAGE + 2 * STAGES * 8 + 1024;
    static_assert(WCOLS <= BOXC && BOXC % WCOLS == 0, "a warp's columns lie in one box");
    static_assert(STAGES >= 3, "a ring needs stages in flight");
};

template <int RP>
__global__ void __launch_bounds__(DHCfg<RP>::kWarps * 32, 1)
    hpass_dmma(const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmW,
               int n, int p, StreamK sk, double *__restrict__ part, RunState *st) {
    using C = DHCfg<RP>;
    if (run_stopped(st)) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + C::STAGES * C::STAGE);
    int *arrivals = reinterpret_cast<int *>(full + C::STAGES);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer = (threadIdx.x == 0);
    const int b = blockIdx.x;
    const long long u0 = sk.start(b), u1 = sk.start(b + 1);
    const long long nunits = u1 - u0;

    auto issue = [&](unsigned char *stg, uint64_t *bar, const UnitCursor &c) {
        const int rb = c.along(sk);
#pragma unroll
        for (int q = 0; q < C::NBOX; q++)
            tma_load_2d(stg + q * C::BROWS * C::BOXC * 8, &tmV, bar,
                        c.major * C::TCOLS + q * C::BOXC, rb * C::BROWS);
        tma_load_2d(stg + C::VBYTES, &tmW, bar, 0, rb * C::BROWS);
    };
    UnitCursor ahead;
    ahead.init(sk, u0);
    if (producer) {
        for (int s = 0; s < C::STAGES; s++) {
            mbar_init(&full[s], 1);
            arrivals[s] = 0;
        }
        fence_mbar_init();
        for (int j = 0; j < C::STAGES; j++) {
            if (j < nunits) {
                mbar_expect_tx(&full[j], C::VBYTES + C::WBYTES);
                issue(smem + j * C::STAGE, &full[j], ahead);
            }
            ahead.next(sk);
        }
    } else {
        for (int j = 0; j < C::STAGES; j++) ahead.next(sk);
    }
    __syncthreads();

    const int g = lane >> 2, q4 = lane & 3;
    const int wc0 = warp * C::WCOLS;  // this warp's first column in the tile
    const int vbox = wc0 / C::BOXC, voff = wc0 % C::BOXC;
    double acc[C::MT][C::NT][2];
    int cur = -1;
    UnitCursor uc;
    uc.init(sk, u0);
    const int tile0 = uc.t;
    int flast = -1;  // major tile of the last flush
    int s = 0, rnd = 0;
    bool ok = true;

    auto flush = [&](int t) {
        bool add;
        const size_t slot = partial_slot(sk, t, tile0, flast, add);
        double *dst = part + ((size_t)b * sk.slots + slot) * RP * C::TCOLS;
#pragma unroll
        for (int mt = 0; mt < C::MT; mt++) {
            const int k = mt * 8 + g;
            if (k < RP) {
#pragma unroll
                for (int nt = 0; nt < C::NT; nt++) {
                    double *d = dst + (size_t)k * C::TCOLS + wc0 + nt * 8 + 2 * q4;
                    put_partial(&d[0], acc[mt][nt][0], add);
                    put_partial(&d[1], acc[mt][nt][1], add);
                }
            }
        }
    };

    for (long long i = 0; i < nunits; ++i) {
        const int t = uc.t;
        if (t != cur) {
            if (cur >= 0) flush(cur);
            cur = t;
#pragma unroll
            for (int mt = 0; mt < C::MT; mt++)
#pragma unroll
                for (int nt = 0; nt < C::NT; nt++) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
        }
        if (!mbar_wait(&full[s], (uint32_t)(rnd & 1))) {
            record_timeout(st, TIMEOUT_FULL);
            ok = false;
            break;
        }
        const unsigned char *stg = smem + s * C::STAGE;
        const double *sv =
            reinterpret_cast<const double *>(stg) + vbox * C::BROWS * C::BOXC + voff + g;
        const double *sw = reinterpret_cast<const double *>(stg + C::VBYTES);
#pragma unroll
        for (int ks = 0; ks < C::BROWS / 4; ks++) {
            const int r = ks * 4 + q4;
            double a[C::MT], bv[C::NT];
#pragma unroll
            for (int mt = 0; mt < C::MT; mt++) {
                const int k = mt * 8 + g;
                a[mt] = (k < RP) ? sw[r * C::RPS + k] : 0.0;
            }
#pragma unroll
            for (int nt = 0; nt < C::NT; nt++) bv[nt] = sv[r * C::BOXC + nt * 8];
#pragma unroll
            for (int mt = 0; mt < C::MT; mt++)
#pragma unroll
                for (int nt = 0; nt < C::NT; nt++) dmma_8x8x4(acc[mt][nt], a[mt], bv[nt]);
        }
        __syncwarp();
        if (lane == 0)
            release_stage<C::STAGE, C::VBYTES + C::WBYTES>(smem, full, arrivals, s, C::kWarps,
                                                           i + C::STAGES < nunits, ahead, issue);
        ahead.next(sk);
        if (++s == C::STAGES) {
            s = 0;
            ++rnd;
        }
        uc.next(sk);
    }
    if (ok && cur >= 0) flush(cur);
}

// W pass: B[i][k] = sum_j V[i][j] H[k][j] with M = i (4 row tiles of 8 a
// warp), N = k (rank tiles of 8), K = j (4 columns a k-step, 4 k-steps a
// unit of 16 columns read from a 128B-swizzled V box).
template <int RP>
struct DWCfg {
    static constexpr int NT = (RP + 7) / 8;
    static constexpr int kWarps = NT >= 4 ? 8 : 16;
    static constexpr int MW = 4;
    static constexpr int WROWS = MW * 8;
    static constexpr int TROWS = kWarps * WROWS;  // 512 rows a tile
    static constexpr int BOXR = 256;
    static constexpr int NBOX = TROWS / BOXR;
    static constexpr int ROWB = 128;  // one 128-byte swizzle span of a row a unit
    static constexpr int BCOLS = ROWB / 8;
    static constexpr int SEGU = kSegNone;  // f64 sums: one segment a tile
    static constexpr int RPS = RankPad<double, RP>::RPS;
    static constexpr int VBYTES = TROWS * ROWB;
    static constexpr int HBYTES = BCOLS * RPS * 8;
    static constexpr int STAGE = (VBYTES + HBYTES + 1023) / 1024 * 1024;
    static constexpr int STAGES_FIT = (220 * 1024) / STAGE;
    static constexpr int STAGES = STAGES_FIT > 8 ? 8 : STAGES_FIT;
    static constexpr int SMEM = STAGES * STAGE + 2 * STAGES * 8 + 1024;
    static_assert(STAGES >= 3, "a ring needs stages in flight");
    static_assert(TROWS % BOXR == 0 && BOXR % 8 == 0, "whole boxes of whole swizzle groups");
};

template <int RP>
__global__ void __launch_bounds__(DWCfg<RP>::kWarps * 32, 1)
    wpass_dmma(const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmH,
               int n, int p, StreamK sk, double *__restrict__ part, RunState *st) {
    using C = DWCfg<RP>;
    if (run_stopped(st)) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + C::STAGES * C::STAGE);
    int *arrivals = reinterpret_cast<int *>(full + C::STAGES);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer = (threadIdx.x == 0);
    const int b = blockIdx.x;
    const long long u0 = sk.start(b), u1 = sk.start(b + 1);
    const long long nunits = u1 - u0;

    auto issue = [&](unsigned char *stg, uint64_t *bar, const UnitCursor &c) {
        const int cb = c.along(sk);
#pragma unroll
        for (int q = 0; q < C::NBOX; q++)
            tma_load_2d(stg + q * C::BOXR * C::ROWB, &tmV, bar, cb * C::BCOLS,
                        c.major * C::TROWS + q * C::BOXR);
        tma_load_2d(stg + C::VBYTES, &tmH, bar, 0, cb * C::BCOLS);
    };
    UnitCursor ahead;
    ahead.init(sk, u0);
    if (producer) {
        for (int s = 0; s < C::STAGES; s++) {
            mbar_init(&full[s], 1);
            arrivals[s] = 0;
        }
        fence_mbar_init();
        for (int j = 0; j < C::STAGES; j++) {
            if (j < nunits) {
                mbar_expect_tx(&full[j], C::VBYTES + C::HBYTES);
                issue(smem + j * C::STAGE, &full[j], ahead);
            }
            ahead.next(sk);
        }
    } else {
        for (int j = 0; j < C::STAGES; j++) ahead.next(sk);
    }
    __syncthreads();

    const int g = lane >> 2, q4 = lane & 3;
    // Row of A fragment mw: warp * 32 + mw * 8 + g (its swizzle key is g, the
    // row mod 8); its byte offset within the stage, before the chunk.
    const int rbase = warp * C::WROWS + g;
    double acc[C::MW][C::NT][2];
    int cur = -1;
    UnitCursor uc;
    uc.init(sk, u0);
    const int tile0 = uc.t;
    int flast = -1;  // major tile of the last flush
    int s = 0, rnd = 0;
    bool ok = true;

    auto flush = [&](int t) {
        bool add;
        const size_t slot = partial_slot(sk, t, tile0, flast, add);
        double *dst = part + ((size_t)b * sk.slots + slot) * C::TROWS * RP;
#pragma unroll
        for (int mw = 0; mw < C::MW; mw++) {
            const int row = rbase + mw * 8;
#pragma unroll
            for (int nt = 0; nt < C::NT; nt++) {
                const int k = nt * 8 + 2 * q4;
                if (k < RP) {  // RP is even: k + 1 < RP too
                    double *d = dst + (size_t)row * RP + k;
                    put_partial(&d[0], acc[mw][nt][0], add);
                    put_partial(&d[1], acc[mw][nt][1], add);
                }
            }
        }
    };

    for (long long i = 0; i < nunits; ++i) {
        const int t = uc.t;
        if (t != cur) {
            if (cur >= 0) flush(cur);
            cur = t;
#pragma unroll
            for (int mw = 0; mw < C::MW; mw++)
#pragma unroll
                for (int nt = 0; nt < C::NT; nt++) acc[mw][nt][0] = acc[mw][nt][1] = 0.0;
        }
        if (!mbar_wait(&full[s], (uint32_t)(rnd & 1))) {
            record_timeout(st, TIMEOUT_FULL);
            ok = false;
            break;
        }
        const unsigned char *stg = smem + s * C::STAGE;
        const double *sh = reinterpret_cast<const double *>(stg + C::VBYTES);
#pragma unroll
        for (int ks = 0; ks < C::BCOLS / 4; ks++) {
            const int j = ks * 4 + q4;              // column within the unit
            const int chunk = j >> 1, within = j & 1;
            double a[C::MW], bh[C::NT];
#pragma unroll
            for (int mw = 0; mw < C::MW; mw++) {
                const int row = rbase + mw * 8;     // row & 7 == g
                a[mw] = *reinterpret_cast<const double *>(
                    stg + row * C::ROWB + (((chunk ^ g) << 4) | (within << 3)));
            }
#pragma unroll
            for (int nt = 0; nt < C::NT; nt++) {
                const int k = nt * 8 + g;
                bh[nt] = (k < RP) ? sh[j * C::RPS + k] : 0.0;
            }
#pragma unroll
            for (int mw = 0; mw < C::MW; mw++)
#pragma unroll
                for (int nt = 0; nt < C::NT; nt++) dmma_8x8x4(acc[mw][nt], a[mw], bh[nt]);
        }
        __syncwarp();
        if (lane == 0)
            release_stage<C::STAGE, C::VBYTES + C::HBYTES>(smem, full, arrivals, s, C::kWarps,
                                                           i + C::STAGES < nunits, ahead, issue);
        ahead.next(sk);
        if (++s == C::STAGES) {
            s = 0;
            ++rnd;
        }
        uc.next(sk);
    }
    if (ok && cur >= 0) flush(cur);
}

// ---------------------------------------------------------------------------
// FP64 ratio passes on the FP64 tensor cores (brunet / nsNMF; lsNMF's
// weighted denominators with WEIGHTED)
// ---------------------------------------------------------------------------
// Per 8 x 8 tile of (rows i, columns j) two MMA chains:
//   1. WH: D1[g][2q + e] = sum_k (W H) over the rank (K = k in steps of 4);
//   2. the contraction, K = the tile's 8 rows (H pass) or columns (W pass)
//      taken as two k-steps (2q and 2q + 1): the B (H pass) or A (W pass)
//      operand a thread needs there is exactly its own D1[e], turned into
//      q = V / WH (0 where WH == 0, lib.rs:93-99) or q = S WH (WEIGHTED).
// Accumulators and partial layouts are the plain DMMA passes'.

// H pass: A[k][j] = sum_i W[i][k] q[i][j].  MMA 1: M = j, N = i, K = k (A = H
// columns, held in registers for the whole column tile; B = W rows).  MMA 2:
// M = k, N = j, K = i.
template <int RP>
struct DHRCfg {
    static constexpr int KST = (RP + 3) / 4;  // k-steps of the WH chain
    static constexpr int MT = (RP + 7) / 8;
    static constexpr int kWarps = MT >= 4 ? 8 : 16;
    static constexpr int NT = 2;  // column tiles of 8 a warp
    static constexpr int WCOLS = NT * 8;
    static constexpr int TCOLS = kWarps * WCOLS;
    static constexpr int BOXC = TCOLS;
    static constexpr int BROWS = 16;  // two 8-row tiles a unit
    static constexpr int SEGU = kSegNone;  // f64 sums: one segment a tile
    static constexpr int RPS = RankPad<double, RP>::RPS;
    static constexpr int VBYTES = BROWS * TCOLS * 8;
    static constexpr int WBYTES = BROWS * RPS * 8;
    static constexpr int STAGE = (VBYTES + WBYTES + 1023) / 1024 * 1024;
    static constexpr int STAGES_FIT = (220 * 1024) / STAGE;
    static constexpr int STAGES = STAGES_FIT > 10 ? 10 : STAGES_FIT;
    static constexpr int SMEM = STAGES * STAGE + 2 * STAGES * 8 + 1024;
    static_assert(BOXC <= 256, "one V box a unit");
    static_assert(STAGES >= 3, "a ring needs stages in flight");
};

template <int RP, bool WEIGHTED>
__global__ void __launch_bounds__(DHRCfg<RP>::kWarps * 32, 1)
    hpass_dmma_ratio(const __grid_constant__ CUtensorMap tmV,
                     const __grid_constant__ CUtensorMap tmW, const double *__restrict__ H, int n,
                     int p, StreamK sk, double *__restrict__ part, RunState *st) {
    using C = DHRCfg<RP>;
    if (run_stopped(st)) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + C::STAGES * C::STAGE);
    int *arrivals = reinterpret_cast<int *>(full + C::STAGES);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer = (threadIdx.x == 0);
    const int b = blockIdx.x;
    const long long u0 = sk.start(b), u1 = sk.start(b + 1);
    const long long nunits = u1 - u0;

    auto issue = [&](unsigned char *stg, uint64_t *bar, const UnitCursor &c) {
        const int rb = c.along(sk);
        tma_load_2d(stg, &tmV, bar, c.major * C::TCOLS, rb * C::BROWS);
        tma_load_2d(stg + C::VBYTES, &tmW, bar, 0, rb * C::BROWS);
    };
    UnitCursor ahead;
    ahead.init(sk, u0);
    if (producer) {
        for (int s = 0; s < C::STAGES; s++) {
            mbar_init(&full[s], 1);
            arrivals[s] = 0;
        }
        fence_mbar_init();
        for (int j = 0; j < C::STAGES; j++) {
            if (j < nunits) {
                mbar_expect_tx(&full[j], C::VBYTES + C::WBYTES);
                issue(smem + j * C::STAGE, &full[j], ahead);
            }
            ahead.next(sk);
        }
    } else {
        for (int j = 0; j < C::STAGES; j++) ahead.next(sk);
    }
    __syncthreads();

    const int g = lane >> 2, q4 = lane & 3;
    const int wc0 = warp * C::WCOLS;
    double acc[C::MT][C::NT][2];
    double hreg[C::NT][C::KST];  // MMA 1's A: H[ks * 4 + q4][column of row g]
    int cur = -1, cur_major = -1;
    UnitCursor uc;
    uc.init(sk, u0);
    const int tile0 = uc.t;
    int flast = -1;  // major tile of the last flush
    int s = 0, rnd = 0;
    bool ok = true;

    auto flush = [&](int t) {
        bool add;
        const size_t slot = partial_slot(sk, t, tile0, flast, add);
        double *dst = part + ((size_t)b * sk.slots + slot) * RP * C::TCOLS;
#pragma unroll
        for (int mt = 0; mt < C::MT; mt++) {
            const int k = mt * 8 + g;
            if (k < RP) {
#pragma unroll
                for (int nt = 0; nt < C::NT; nt++) {
                    double *d = dst + (size_t)k * C::TCOLS + wc0 + nt * 8 + 2 * q4;
                    put_partial(&d[0], acc[mt][nt][0], add);
                    put_partial(&d[1], acc[mt][nt][1], add);
                }
            }
        }
    };

    for (long long i = 0; i < nunits; ++i) {
        const int t = uc.t;
        if (t != cur) {
            if (cur >= 0) flush(cur);
            cur = t;
#pragma unroll
            for (int mt = 0; mt < C::MT; mt++)
#pragma unroll
                for (int nt = 0; nt < C::NT; nt++) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
            if (uc.major != cur_major) {
                cur_major = uc.major;
#pragma unroll
                for (int nt = 0; nt < C::NT; nt++) {
                    const int j = uc.major * C::TCOLS + wc0 + nt * 8 + g;
#pragma unroll
                    for (int ks = 0; ks < C::KST; ks++) {
                        const int k = ks * 4 + q4;
                        hreg[nt][ks] = (k < RP && j < p) ? H[(size_t)k * p + j] : 0.0;
                    }
                }
            }
        }
        if (!mbar_wait(&full[s], (uint32_t)(rnd & 1))) {
            record_timeout(st, TIMEOUT_FULL);
            ok = false;
            break;
        }
        const unsigned char *stg = smem + s * C::STAGE;
        const double *sv = reinterpret_cast<const double *>(stg) + wc0 + g;
        const double *sw = reinterpret_cast<const double *>(stg + C::VBYTES);
#pragma unroll
        for (int rt = 0; rt < C::BROWS / 8; rt++) {
            const int r0 = rt * 8;
            double b1[C::KST];  // MMA 1's B: W[r0 + g][ks * 4 + q4]
#pragma unroll
            for (int ks = 0; ks < C::KST; ks++) {
                const int k = ks * 4 + q4;
                b1[ks] = (k < RP) ? sw[(r0 + g) * C::RPS + k] : 0.0;
            }
            double a2[C::MT][2];  // MMA 2's A: W[r0 + 2 q4 + e][mt * 8 + g]
#pragma unroll
            for (int mt = 0; mt < C::MT; mt++) {
                const int k = mt * 8 + g;
#pragma unroll
                for (int e = 0; e < 2; e++)
                    a2[mt][e] = (k < RP) ? sw[(r0 + 2 * q4 + e) * C::RPS + k] : 0.0;
            }
            // The column tiles' WH chains interleaved (independent), then
            // their ratios, then MMA 2: the tensor pipe has a second chain
            // to issue while one waits.  Each accumulator sees the same
            // operations in the same order as tile by tile.
            double wh[C::NT][2];
#pragma unroll
            for (int nt = 0; nt < C::NT; nt++) wh[nt][0] = wh[nt][1] = 0.0;
#pragma unroll
            for (int ks = 0; ks < C::KST; ks++)
#pragma unroll
                for (int nt = 0; nt < C::NT; nt++) dmma_8x8x4(wh[nt], hreg[nt][ks], b1[ks]);
            double qv[C::NT][2];
#pragma unroll
            for (int nt = 0; nt < C::NT; nt++)
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const double v = sv[(r0 + 2 * q4 + e) * C::BOXC + nt * 8];
                    if constexpr (WEIGHTED)
                        qv[nt][e] = v * wh[nt][e];
                    else
                        qv[nt][e] = (wh[nt][e] != 0.0) ? ratio_div(v, wh[nt][e]) : 0.0;
                }
#pragma unroll
            for (int e = 0; e < 2; e++)
#pragma unroll
                for (int mt = 0; mt < C::MT; mt++)
#pragma unroll
                    for (int nt = 0; nt < C::NT; nt++)
                        dmma_8x8x4(acc[mt][nt], a2[mt][e], qv[nt][e]);
        }
        __syncwarp();
        if (lane == 0)
            release_stage<C::STAGE, C::VBYTES + C::WBYTES>(smem, full, arrivals, s, C::kWarps,
                                                           i + C::STAGES < nunits, ahead, issue);
        ahead.next(sk);
        if (++s == C::STAGES) {
            s = 0;
            ++rnd;
        }
        uc.next(sk);
    }
    if (ok && cur >= 0) flush(cur);
}

// W pass: B[i][k] = sum_j q[i][j] H[k][j].  MMA 1: M = i, N = j, K = k (A = W
// rows, held in registers for the whole row tile; B = H^T rows).  MMA 2:
// M = i, N = k, K = j.
template <int RP>
struct DWRCfg {
    static constexpr int KST = (RP + 3) / 4;
    static constexpr int NT = (RP + 7) / 8;
    static constexpr int kWarps = NT >= 4 ? 8 : 16;
    static constexpr int MW = 2;  // row tiles of 8 a warp
    static constexpr int WROWS = MW * 8;
    static constexpr int TROWS = kWarps * WROWS;
    static constexpr int BOXR = TROWS;
    static constexpr int ROWB = 128;
    static constexpr int BCOLS = ROWB / 8;  // two 8-column tiles a unit
    static constexpr int SEGU = kSegNone;  // f64 sums: one segment a tile
    static constexpr int RPS = RankPad<double, RP>::RPS;
    static constexpr int VBYTES = TROWS * ROWB;
    static constexpr int HBYTES = BCOLS * RPS * 8;
    static constexpr int STAGE = (VBYTES + HBYTES + 1023) / 1024 * 1024;
    static constexpr int STAGES_FIT = (220 * 1024) / STAGE;
    static constexpr int STAGES = STAGES_FIT > 8 ? 8 : STAGES_FIT;
    static constexpr int SMEM = STAGES * STAGE + 2 * STAGES * 8 + 1024;
    static_assert(BOXR <= 256 && BOXR % 8 == 0, "one V box of whole swizzle groups");
    static_assert(STAGES >= 3, "a ring needs stages in flight");
};

template <int RP, bool WEIGHTED>
__global__ void __launch_bounds__(DWRCfg<RP>::kWarps * 32, 1)
    wpass_dmma_ratio(const __grid_constant__ CUtensorMap tmV,
                     const __grid_constant__ CUtensorMap tmH, const double *__restrict__ W, int n,
                     int p, StreamK sk, double *__restrict__ part, RunState *st) {
    using C = DWRCfg<RP>;
    if (run_stopped(st)) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + C::STAGES * C::STAGE);
    int *arrivals = reinterpret_cast<int *>(full + C::STAGES);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer = (threadIdx.x == 0);
    const int b = blockIdx.x;
    const long long u0 = sk.start(b), u1 = sk.start(b + 1);
    const long long nunits = u1 - u0;

    auto issue = [&](unsigned char *stg, uint64_t *bar, const UnitCursor &c) {
        const int cb = c.along(sk);
        tma_load_2d(stg, &tmV, bar, cb * C::BCOLS, c.major * C::TROWS);
        tma_load_2d(stg + C::VBYTES, &tmH, bar, 0, cb * C::BCOLS);
    };
    UnitCursor ahead;
    ahead.init(sk, u0);
    if (producer) {
        for (int s = 0; s < C::STAGES; s++) {
            mbar_init(&full[s], 1);
            arrivals[s] = 0;
        }
        fence_mbar_init();
        for (int j = 0; j < C::STAGES; j++) {
            if (j < nunits) {
                mbar_expect_tx(&full[j], C::VBYTES + C::HBYTES);
                issue(smem + j * C::STAGE, &full[j], ahead);
            }
            ahead.next(sk);
        }
    } else {
        for (int j = 0; j < C::STAGES; j++) ahead.next(sk);
    }
    __syncthreads();

    const int g = lane >> 2, q4 = lane & 3;
    const int rbase = warp * C::WROWS + g;  // row of fragment mw: rbase + mw * 8 (row & 7 == g)
    double acc[C::MW][C::NT][2];
    double wreg[C::MW][C::KST];  // MMA 1's A: W[row][ks * 4 + q4]
    int cur = -1, cur_major = -1;
    UnitCursor uc;
    uc.init(sk, u0);
    const int tile0 = uc.t;
    int flast = -1;  // major tile of the last flush
    int s = 0, rnd = 0;
    bool ok = true;

    auto flush = [&](int t) {
        bool add;
        const size_t slot = partial_slot(sk, t, tile0, flast, add);
        double *dst = part + ((size_t)b * sk.slots + slot) * C::TROWS * RP;
#pragma unroll
        for (int mw = 0; mw < C::MW; mw++) {
            const int row = rbase + mw * 8;
#pragma unroll
            for (int nt = 0; nt < C::NT; nt++) {
                const int k = nt * 8 + 2 * q4;
                if (k < RP) {
                    double *d = dst + (size_t)row * RP + k;
                    put_partial(&d[0], acc[mw][nt][0], add);
                    put_partial(&d[1], acc[mw][nt][1], add);
                }
            }
        }
    };

    for (long long i = 0; i < nunits; ++i) {
        const int t = uc.t;
        if (t != cur) {
            if (cur >= 0) flush(cur);
            cur = t;
#pragma unroll
            for (int mw = 0; mw < C::MW; mw++)
#pragma unroll
                for (int nt = 0; nt < C::NT; nt++) acc[mw][nt][0] = acc[mw][nt][1] = 0.0;
            if (uc.major != cur_major) {
                cur_major = uc.major;
#pragma unroll
                for (int mw = 0; mw < C::MW; mw++) {
                    const int row = uc.major * C::TROWS + rbase + mw * 8;
#pragma unroll
                    for (int ks = 0; ks < C::KST; ks++) {
                        const int k = ks * 4 + q4;
                        wreg[mw][ks] = (k < RP && row < n) ? W[(size_t)row * RP + k] : 0.0;
                    }
                }
            }
        }
        if (!mbar_wait(&full[s], (uint32_t)(rnd & 1))) {
            record_timeout(st, TIMEOUT_FULL);
            ok = false;
            break;
        }
        const unsigned char *stg = smem + s * C::STAGE;
        const double *sh = reinterpret_cast<const double *>(stg + C::VBYTES);
#pragma unroll
        for (int jt = 0; jt < C::BCOLS / 8; jt++) {
            const int j0 = jt * 8;
            double b1[C::KST];  // MMA 1's B: H^T[j0 + g][ks * 4 + q4]
#pragma unroll
            for (int ks = 0; ks < C::KST; ks++) {
                const int k = ks * 4 + q4;
                b1[ks] = (k < RP) ? sh[(j0 + g) * C::RPS + k] : 0.0;
            }
            double b2[C::NT][2];  // MMA 2's B: H^T[j0 + 2 q4 + e][nt * 8 + g]
#pragma unroll
            for (int nt = 0; nt < C::NT; nt++) {
                const int k = nt * 8 + g;
#pragma unroll
                for (int e = 0; e < 2; e++)
                    b2[nt][e] = (k < RP) ? sh[(j0 + 2 * q4 + e) * C::RPS + k] : 0.0;
            }
            // V[row][j0 + 2 q4 + e], e = 0, 1: one 16-byte chunk of the row.
            const int chunk = (j0 >> 1) + q4;
            // The row tiles' WH chains interleaved, then their ratios, then
            // MMA 2 (the same operations per accumulator, in the same order).
            double wh[C::MW][2];
#pragma unroll
            for (int mw = 0; mw < C::MW; mw++) wh[mw][0] = wh[mw][1] = 0.0;
#pragma unroll
            for (int ks = 0; ks < C::KST; ks++)
#pragma unroll
                for (int mw = 0; mw < C::MW; mw++) dmma_8x8x4(wh[mw], wreg[mw][ks], b1[ks]);
            double qv[C::MW][2];
#pragma unroll
            for (int mw = 0; mw < C::MW; mw++) {
                const int row = rbase + mw * 8;
                const double2 v2 = *reinterpret_cast<const double2 *>(
                    stg + row * C::ROWB + ((chunk ^ g) << 4));
                const double vv[2] = {v2.x, v2.y};
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    if constexpr (WEIGHTED)
                        qv[mw][e] = vv[e] * wh[mw][e];
                    else
                        qv[mw][e] = (wh[mw][e] != 0.0) ? ratio_div(vv[e], wh[mw][e]) : 0.0;
                }
            }
#pragma unroll
            for (int e = 0; e < 2; e++)
#pragma unroll
                for (int nt = 0; nt < C::NT; nt++)
#pragma unroll
                    for (int mw = 0; mw < C::MW; mw++)
                        dmma_8x8x4(acc[mw][nt], qv[mw][e], b2[nt][e]);
        }
        __syncwarp();
        if (lane == 0)
            release_stage<C::STAGE, C::VBYTES + C::HBYTES>(smem, full, arrivals, s, C::kWarps,
                                                           i + C::STAGES < nunits, ahead, issue);
        ahead.next(sk);
        if (++s == C::STAGES) {
            s = 0;
            ++rnd;
        }
        uc.next(sk);
    }
    if (ok && cur >= 0) flush(cur);
}

// ---------------------------------------------------------------------------
// Epilogues for the stream-K partials
// ---------------------------------------------------------------------------

// Sum of the partials of output `c` of major tile `mt`, over its segments and
// their CTAs, in that order.  `stride_k` / `stride_row` describe the partial
// layout: element (slot base) + k * stride_k + c * stride_c.
template <int RP>
__device__ __forceinline__ void gather_partials(const double *__restrict__ part,
                                                const StreamK &sk, int mt, size_t slot_elems,
                                                size_t off, size_t stride_k, double (&num)[RP]) {
#pragma unroll
    for (int k = 0; k < RP; k++) num[k] = 0.0;
    if (sk.G <= 0) return;  // no units at all: every sum is empty
    if (sk.fold) {
        int lo, hi;
        sk_range_major(sk, mt, &lo, &hi);
        for (int b = lo; b <= hi; b++) {
            const double *src =
                part + ((size_t)b * sk.slots + fold_slot(sk, b, mt)) * slot_elems + off;
#pragma unroll
            for (int k = 0; k < RP; k++) num[k] += src[(size_t)k * stride_k];
        }
        return;
    }
    for (int seg = 0; seg < sk.nseg; seg++) {
        const int t = mt * sk.nseg + seg;
        int lo, hi;
        sk_range(sk, t, &lo, &hi);
        for (int b = lo; b <= hi; b++) {
            const int slot = t - (int)(sk.start(b) / sk.UPT);
            const double *src = part + ((size_t)b * sk.slots + slot) * slot_elems + off;
#pragma unroll
            for (int k = 0; k < RP; k++) num[k] += src[(size_t)k * stride_k];
        }
    }
}

// One thread per column: sum the partials, apply the H update, write H
// (RP x p, f64) and the copy H^T (p x RPS_T, type TH) the next W pass streams.
template <int RP, typename TH, int RPS_T>
__global__ void __launch_bounds__(kThreads)
    h_epilogue_sk(double *__restrict__ H, TH *__restrict__ Ht, int p,
                  const double *__restrict__ part, StreamK sk, int tcols, EpiParams e,
                  const RunState *st) {
    if (run_stopped(st)) return;
    const int j = blockIdx.x * kThreads + threadIdx.x;
    if (j >= p) return;
    const int ct = j / tcols, c = j - ct * tcols;
    double num[RP], hc[RP];
    gather_partials<RP>(part, sk, ct, (size_t)RP * tcols, c, tcols, num);
#pragma unroll
    for (int k = 0; k < RP; k++) hc[k] = H[(size_t)k * p + j];
    double ax[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) ax[k] = (e.aux != nullptr && k < e.r) ? e.aux[(size_t)k * p + j] : 0.0;
    h_update<RP>(e, num, hc, ax);
#pragma unroll
    for (int k = 0; k < RP; k++)
        if (k < e.r) H[(size_t)k * p + j] = hc[k];
    if (Ht == nullptr) return;  // the tensor-core passes stream their own H terms
    TH *ht = Ht + (size_t)j * RPS_T;
#pragma unroll
    for (int k = 0; k < RPS_T; k++) ht[k] = (k < e.r && k < RP) ? (TH)hc[k] : (TH)0;
}

// One warp per row: lane l adds the partials of segments l, l + 32, ...
// (each over its CTAs in order; with folded partials, of CTAs l, l + 32, ...
// of the row tile), a fixed xor butterfly adds the lanes, and
// lane 0 applies the W update -- a long row (many column segments) is
// gathered 32 segments at a time.  Deterministic.
template <int RP>
__global__ void __launch_bounds__(kThreads)
    w_epilogue_sk(double *__restrict__ W, int n, const double *__restrict__ part, StreamK sk,
                  int trows, EpiParams e, const RunState *st) {
    if (run_stopped(st)) return;
    const int i = (int)(((size_t)blockIdx.x * kThreads + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;  // uniform across the warp
    const int rt = i / trows, rl = i - rt * trows;
    double num[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) num[k] = 0.0;
    if (sk.G > 0 && sk.fold) {
        // Folded partials: lane l adds CTAs lo + l, lo + l + 32, ...
        const size_t slot_elems = (size_t)trows * RP;
        int lo, hi;
        sk_range_major(sk, rt, &lo, &hi);
        for (int b = lo + lane; b <= hi; b += 32) {
            const double *src = part + ((size_t)b * sk.slots + fold_slot(sk, b, rt)) * slot_elems +
                                (size_t)rl * RP;
#pragma unroll
            for (int k = 0; k < RP; k++) num[k] += src[k];
        }
    } else if (sk.G > 0) {
        const size_t slot_elems = (size_t)trows * RP;
        for (int seg = lane; seg < sk.nseg; seg += 32) {
            const int t = rt * sk.nseg + seg;
            int lo, hi;
            sk_range(sk, t, &lo, &hi);
            for (int b = lo; b <= hi; b++) {
                const int slot = t - (int)(sk.start(b) / sk.UPT);
                const double *src = part + ((size_t)b * sk.slots + slot) * slot_elems + (size_t)rl * RP;
#pragma unroll
                for (int k = 0; k < RP; k++) num[k] += src[k];
            }
        }
    }
#pragma unroll
    for (int k = 0; k < RP; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) num[k] += __shfl_xor_sync(0xffffffffu, num[k], o);
    // Every lane now holds the row's sums.  Methods whose columns update
    // independently take one lane a column; the HALS / dnmf sweeps, which
    // run over the columns in order, lane 0.
    double wr[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) wr[k] = W[(size_t)i * RP + k];
    const double ro = e.roff ? e.roff[i] : 0.0;
    if (w_update_by_column(e.method)) {
        if (lane >= e.r || lane >= RP) return;
        double numj = 0.0, wrj = 0.0;
#pragma unroll
        for (int k = 0; k < RP; k++)
            if (k == lane) {
                numj = num[k];
                wrj = wr[k];
            }
        const double *ax = e.aux != nullptr ? e.aux + (size_t)i * RP : nullptr;
        const double out = w_update_column<RP>(e, numj, wrj, wr, lane, ro, ax);
        // All lanes have read the row before any writes it.
        __syncwarp(__activemask());
        W[(size_t)i * RP + lane] = out;
        return;
    }
    if (lane != 0) return;
    double ax[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) ax[k] = e.aux != nullptr ? e.aux[(size_t)i * RP + k] : 0.0;
    w_update<RP>(e, num, wr, ro, ax);
#pragma unroll
    for (int k = 0; k < RP; k++)
        if (k < e.r) W[(size_t)i * RP + k] = wr[k];
}

// f32 copy of W (n x RP f64 -> n x RPS f32, zero pad) for the f32 H pass.
template <int RP, int RPS>
__global__ void w_to_f32(const double *__restrict__ W, float *__restrict__ Wf, int n,
                         const RunState *st) {
    if (run_stopped(st)) return;
    const int64_t total = (int64_t)n * RPS;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / RPS;
        const int k = (int)(t - i * RPS);
        Wf[t] = (k < RP) ? (float)W[i * RP + k] : 0.0f;
    }
}

}  // namespace nmfcu

// stream.cuh -- the two V-streaming passes of an NMF iteration, fed by TMA.
//
// Each pass is one kernel with one CTA (8 warps) per SM.  Lane 0 of warp 0
// issues cp.async.bulk.tensor loads of V tiles (and of the W rows / H^T
// columns that pair with them) into a ring of shared-memory stages guarded by
// mbarriers; all eight warps do the FMAs out of shared memory, so no LSU
// instruction ever waits on HBM.  The refill of a stage trails its
// consumption by LAG units, so the issuing lane rarely waits on the other
// warps.  (A separate producer warp would put three warps on one SM
// sub-partition and cap every thread at 168 registers.)
//
// Work split ("stream-K"): a tile is TCOLS columns x all rows (H pass) or
// TROWS rows x all columns (W pass); a unit is one stage of one tile.  The U
// units of all tiles are dealt out in equal contiguous ranges, so every CTA
// streams the same number of bytes whatever the tile count.  A CTA writes a
// partial sum for every tile its range touches (at most `slots` of them),
// and the epilogue adds the partials of a tile in CTA order: deterministic,
// no atomics.
//
//   H pass  A[k][j] = sum_u W[u][k] V[u][j]              (lee, hals, dnmf)
//           A[k][j] = sum_u W[u][k] V[u][j] / (WH)[u][j]   (brunet)
//     thread = CPT adjacent columns, all rows; W rows broadcast from smem.
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
enum : int { TIMEOUT_FULL = 1, TIMEOUT_EMPTY = 2 };

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
__device__ __forceinline__ void record_timeout(RunState *st, int code) {
    if (st) atomicCAS(&st->timeout, 0, code);
}

// Units trail: a stage is refilled for unit i + STAGES - kLag right after the
// issuing warp has consumed unit i.
constexpr int kLag = 2;

// Producer step for local unit j (0-based within this CTA's range): wait
// until the stage's previous occupant has been released by all warps, then
// arm the full barrier and issue the loads.  `issue(stage_ptr, bar, j)`
// issues the TMA copies.  Returns false on a timed-out wait.
template <int STAGES, int STAGE_BYTES, int TX_BYTES, typename Issue>
__device__ __forceinline__ bool produce(unsigned char *smem, uint64_t *full, uint64_t *empty,
                                        long long j, Issue &&issue) {
    const int s = (int)(j % STAGES);
    const long long round = j / STAGES;
    if (round > 0 && !mbar_wait(&empty[s], (uint32_t)((round - 1) & 1))) return false;
    mbar_expect_tx(&full[s], TX_BYTES);
    issue(smem + s * STAGE_BYTES, &full[s], j);
    return true;
}

// ---------------------------------------------------------------------------
// Stream-K bookkeeping
// ---------------------------------------------------------------------------
struct StreamK {
    long long U;  // units in all tiles
    int G;        // CTAs (G <= U, so no CTA is empty)
    int UPT;      // units per tile
    int slots;    // partial slots per CTA
    __host__ __device__ __forceinline__ long long start(int b) const {
        return (long long)b * U / G;
    }
};

// CTAs [lo, hi] whose unit range meets tile t.
__device__ __forceinline__ void sk_range(const StreamK &sk, int t, int *lo, int *hi) {
    const long long a = (long long)t * sk.UPT;
    const long long e = min(a + sk.UPT, sk.U);
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

// A row of RP values (RPS-padded) from shared memory into registers.
template <typename T, int RP>
__device__ __forceinline__ void lds_row(T (&dst)[RP], const T *src) {
    constexpr int V = 16 / (int)sizeof(T);
#pragma unroll
    for (int k0 = 0; k0 < RP; k0 += V) {
        T tmp[V];
        lds_vec<T, V>(tmp, src + k0);
#pragma unroll
        for (int i = 0; i < V; i++)
            if (k0 + i < RP) dst[k0 + i] = tmp[i];
    }
}

// ---------------------------------------------------------------------------
// H pass
// ---------------------------------------------------------------------------
template <typename T, int RP, bool RATIO>
struct HCfg {
    static constexpr int kWarps = 8;
    static constexpr int CPT = (sizeof(T) == 8 && RATIO) ? 1 : 2;  // columns per thread
    static constexpr int TCOLS = 32 * CPT * kWarps;
    static constexpr int BOXC = TCOLS < 256 ? TCOLS : 256;
    static constexpr int NBOX = TCOLS / BOXC;
    static constexpr int BROWS = 8;
    static constexpr int RPS = RankPad<T, RP>::RPS;
    static constexpr int VBYTES = BROWS * TCOLS * (int)sizeof(T);
    static constexpr int WBYTES = BROWS * RPS * (int)sizeof(T);
    static constexpr int STAGE = (VBYTES + WBYTES + 1023) / 1024 * 1024;
    static constexpr int STAGES_FIT = (180 * 1024) / STAGE;
    static constexpr int STAGES = STAGES_FIT > 10 ? 10 : STAGES_FIT;
    static constexpr int SMEM = STAGES * STAGE + 2 * STAGES * 8 + 1024;
    static constexpr int FLUSH2 = 32;  // f32: stages per f32 partial sum
    // 32-bit registers a row needs: accumulators (+ H columns when RATIO)
    // and the row of W.
    static constexpr int REGS = (int)sizeof(T) / 4 * RP * (CPT * (RATIO ? 2 : 1) + 1);
    // f32: the running total of the per-FLUSH2 partial sums is f64 when it
    // fits the register budget, f32 otherwise.
    static constexpr bool TOTAL64 = sizeof(T) == 8 || REGS + 2 * CPT * RP <= 160;
    using Total = typename std::conditional<TOTAL64, double, float>::type;
    static constexpr int UNROLL = (REGS + (int)sizeof(T) / 4 * RP <= 150) ? 2 : 1;
    static_assert(STAGES >= kLag + 2, "the refill lag needs more stages");
};

template <typename T, int RP, bool RATIO>
__global__ void __launch_bounds__(256, 1)
    hpass(const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmW,
          const double *__restrict__ H, int n, int p, StreamK sk, double *__restrict__ part,
          RunState *st) {
    using C = HCfg<T, RP, RATIO>;
    using Total = typename C::Total;
    constexpr int CPT = C::CPT;
    if (run_stopped(st)) return;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + C::STAGES * C::STAGE);
    uint64_t *empty = full + C::STAGES;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer = (threadIdx.x == 0);
    const int b = blockIdx.x;
    const long long u0 = sk.start(b), u1 = sk.start(b + 1);
    const long long nunits = u1 - u0;

    // Loads of local unit j: the V boxes of its tile and rows, and its W rows.
    auto issue = [&](unsigned char *stg, uint64_t *bar, long long j) {
        const long long u = u0 + j;
        const int t = (int)(u / sk.UPT), rb = (int)(u % sk.UPT);
#pragma unroll
        for (int q = 0; q < C::NBOX; q++)
            tma_load_2d(stg + q * C::BROWS * C::BOXC * (int)sizeof(T), &tmV, bar,
                        t * C::TCOLS + q * C::BOXC, rb * C::BROWS);
        tma_load_2d(stg + C::VBYTES, &tmW, bar, 0, rb * C::BROWS);
    };
    if (producer) {
        for (int s = 0; s < C::STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], C::kWarps);
        }
        fence_mbar_init();
        for (long long j = 0; j < nunits && j < C::STAGES; j++)
            produce<C::STAGES, C::STAGE, C::VBYTES + C::WBYTES>(smem, full, empty, j, issue);
    }
    __syncthreads();

    const int colw = warp * 32 * CPT + lane * CPT;  // column within the tile
    const int box = colw / C::BOXC, boff = colw % C::BOXC;
    T acc[CPT][RP];
    Total acc2[CPT][RP];  // f32: running total of the FLUSH2-stage partial sums
    T hcol[RATIO ? CPT : 1][RATIO ? RP : 1];
    int cur = -1, cnt = 0;
    const int tile0 = (int)(u0 / sk.UPT);
    bool ok = true;

    auto flush = [&](int t) {
        double *dst = part + ((size_t)b * sk.slots + (t - tile0)) * RP * C::TCOLS + colw;
#pragma unroll
        for (int k = 0; k < RP; k++)
#pragma unroll
            for (int c = 0; c < CPT; c++)
                dst[(size_t)k * C::TCOLS + c] =
                    (sizeof(T) == 4) ? (double)acc2[c][k] + (double)acc[c][k] : (double)acc[c][k];
    };

    for (long long i = 0; i < nunits; ++i) {
        const long long u = u0 + i;
        const int t = (int)(u / sk.UPT);
        if (t != cur) {
            if (cur >= 0) flush(cur);
            cur = t;
            cnt = 0;
#pragma unroll
            for (int c = 0; c < CPT; c++)
#pragma unroll
                for (int k = 0; k < RP; k++) {
                    acc[c][k] = (T)0;
                    acc2[c][k] = (Total)0;
                }
            if constexpr (RATIO) {
#pragma unroll
                for (int c = 0; c < CPT; c++) {
                    const int j = t * C::TCOLS + colw + c;
#pragma unroll
                    for (int k = 0; k < RP; k++)
                        hcol[c][k] = (j < p) ? (T)H[(size_t)k * p + j] : (T)0;
                }
            }
        }
        const int s = (int)(i % C::STAGES);
        if (!mbar_wait(&full[s], (uint32_t)((i / C::STAGES) & 1))) {
            record_timeout(st, TIMEOUT_FULL);
            ok = false;
            break;
        }
        const unsigned char *stg = smem + s * C::STAGE;
        const T *sv = reinterpret_cast<const T *>(stg) + box * C::BROWS * C::BOXC + boff;
        const T *sw = reinterpret_cast<const T *>(stg + C::VBYTES);
#pragma unroll(C::UNROLL)
        for (int r = 0; r < C::BROWS; r++) {
            T v[CPT];
            lds_vec<T, CPT>(v, sv + r * C::BOXC);
            T w[RP];
            lds_row<T, RP>(w, sw + r * C::RPS);
            if constexpr (RATIO) {
#pragma unroll
                for (int c = 0; c < CPT; c++) {
                    T wh = (T)0;
#pragma unroll
                    for (int k = 0; k < RP; k++) wh = fma(w[k], hcol[c][k], wh);
                    const T q = (wh != (T)0) ? ratio_div(v[c], wh) : (T)0;
#pragma unroll
                    for (int k = 0; k < RP; k++) acc[c][k] = fma(w[k], q, acc[c][k]);
                }
            } else {
#pragma unroll
                for (int c = 0; c < CPT; c++)
#pragma unroll
                    for (int k = 0; k < RP; k++) acc[c][k] = fma(w[k], v[c], acc[c][k]);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (producer && i >= kLag && i - kLag + C::STAGES < nunits) {
            if (!produce<C::STAGES, C::STAGE, C::VBYTES + C::WBYTES>(
                    smem, full, empty, i - kLag + C::STAGES, issue)) {
                record_timeout(st, TIMEOUT_EMPTY);
                ok = false;
                break;
            }
        }
        if constexpr (sizeof(T) == 4) {
            if (++cnt == C::FLUSH2) {
                cnt = 0;
#pragma unroll
                for (int c = 0; c < CPT; c++)
#pragma unroll
                    for (int k = 0; k < RP; k++) {
                        acc2[c][k] += (Total)acc[c][k];
                        acc[c][k] = (T)0;
                    }
            }
        }
    }
    if (ok && cur >= 0) flush(cur);
}

// ---------------------------------------------------------------------------
// W pass
// ---------------------------------------------------------------------------
template <typename T, int RP, bool RATIO>
struct WCfg {
    static constexpr int kWarps = 8;
    static constexpr int RT = (sizeof(T) == 4) ? 2 : 1;  // rows per thread
    static constexpr int TROWS = 256 * RT;
    static constexpr int BCOLS = 16;                       // columns per unit
    static constexpr int ROWB = BCOLS * (int)sizeof(T);    // bytes of a row per unit
    static constexpr int CHUNKS = ROWB / 16;               // 16 B chunks per row
    // TMA swizzle matching the row: 128 B (f64) or 64 B (f32).  Physical chunk
    // of logical chunk c in row r: c ^ ((r * ROWB >> 7) & (CHUNKS - 1)).
    static constexpr int RPS = RankPad<T, RP>::RPS;
    static constexpr int VBYTES = TROWS * ROWB;
    static constexpr int HBYTES = BCOLS * RPS * (int)sizeof(T);
    static constexpr int STAGE = (VBYTES + HBYTES + 1023) / 1024 * 1024;
    static constexpr int STAGES_FIT = (200 * 1024) / STAGE;
    static constexpr int STAGES = STAGES_FIT > 8 ? 8 : STAGES_FIT;
    static constexpr int SMEM = STAGES * STAGE + 2 * STAGES * 8 + 1024;
    static constexpr int FLUSH2 = 32;
    // 32-bit registers: accumulators (+ W rows when RATIO) and one H column.
    static constexpr int REGS = (int)sizeof(T) / 4 * RP * (RT * (RATIO ? 2 : 1) + 1);
    static constexpr bool TOTAL64 = sizeof(T) == 8 || REGS + 2 * RT * RP <= 160;
    using Total = typename std::conditional<TOTAL64, double, float>::type;
    static constexpr int UNROLL = (REGS + (int)sizeof(T) / 4 * RP <= 150) ? 2 : 1;
    static_assert(STAGES >= kLag + 2, "the refill lag needs more stages");
};

template <typename T, int RP, bool RATIO>
__global__ void __launch_bounds__(256, 1)
    wpass(const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmH,
          const double *__restrict__ W, int n, int p, StreamK sk, double *__restrict__ part,
          RunState *st) {
    using C = WCfg<T, RP, RATIO>;
    using Total = typename C::Total;
    constexpr int RT = C::RT;
    constexpr int VEC = 16 / (int)sizeof(T);  // columns per 16-byte chunk
    if (run_stopped(st)) return;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + C::STAGES * C::STAGE);
    uint64_t *empty = full + C::STAGES;
    const int lane = threadIdx.x & 31;
    const bool producer = (threadIdx.x == 0);
    const int b = blockIdx.x;
    const long long u0 = sk.start(b), u1 = sk.start(b + 1);
    const long long nunits = u1 - u0;

    // Loads of local unit j: RT boxes of 256 rows x BCOLS columns of V
    // (swizzled) and the matching BCOLS rows of H^T.
    auto issue = [&](unsigned char *stg, uint64_t *bar, long long j) {
        const long long u = u0 + j;
        const int t = (int)(u / sk.UPT), cb = (int)(u % sk.UPT);
#pragma unroll
        for (int q = 0; q < RT; q++)
            tma_load_2d(stg + q * 256 * C::ROWB, &tmV, bar, cb * C::BCOLS, t * C::TROWS + q * 256);
        tma_load_2d(stg + C::VBYTES, &tmH, bar, 0, cb * C::BCOLS);
    };
    if (producer) {
        for (int s = 0; s < C::STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], C::kWarps);
        }
        fence_mbar_init();
        for (long long j = 0; j < nunits && j < C::STAGES; j++)
            produce<C::STAGES, C::STAGE, C::VBYTES + C::HBYTES>(smem, full, empty, j, issue);
    }
    __syncthreads();

    const int tid = threadIdx.x;  // rows tid + 256 q of the tile
    T acc[RT][RP];
    Total acc2[RT][RP];
    T wrow[RATIO ? RT : 1][RATIO ? RP : 1];
    int cur = -1, cnt = 0;
    const int tile0 = (int)(u0 / sk.UPT);
    bool ok = true;

    auto flush = [&](int t) {
        double *dst = part + ((size_t)b * sk.slots + (t - tile0)) * C::TROWS * RP;
#pragma unroll
        for (int q = 0; q < RT; q++)
#pragma unroll
            for (int k = 0; k < RP; k++)
                dst[(size_t)(tid + 256 * q) * RP + k] =
                    (sizeof(T) == 4) ? (double)acc2[q][k] + (double)acc[q][k] : (double)acc[q][k];
    };

    for (long long i = 0; i < nunits; ++i) {
        const long long u = u0 + i;
        const int t = (int)(u / sk.UPT);
        if (t != cur) {
            if (cur >= 0) flush(cur);
            cur = t;
            cnt = 0;
#pragma unroll
            for (int q = 0; q < RT; q++)
#pragma unroll
                for (int k = 0; k < RP; k++) {
                    acc[q][k] = (T)0;
                    acc2[q][k] = (Total)0;
                }
            if constexpr (RATIO) {
#pragma unroll
                for (int q = 0; q < RT; q++) {
                    const int row = t * C::TROWS + tid + 256 * q;
#pragma unroll
                    for (int k = 0; k < RP; k++)
                        wrow[q][k] = (row < n) ? (T)W[(size_t)row * RP + k] : (T)0;
                }
            }
        }
        const int s = (int)(i % C::STAGES);
        if (!mbar_wait(&full[s], (uint32_t)((i / C::STAGES) & 1))) {
            record_timeout(st, TIMEOUT_FULL);
            ok = false;
            break;
        }
        const unsigned char *stg = smem + s * C::STAGE;
        const T *sh = reinterpret_cast<const T *>(stg + C::VBYTES);
        // Swizzle phase of this thread's row (same for every box: boxes start
        // on 16 KB boundaries).
        const int sw = ((tid * C::ROWB) >> 7) & (C::CHUNKS - 1);
#pragma unroll(C::UNROLL)
        for (int ci = 0; ci < C::CHUNKS; ci++) {
            T v[RT][VEC];
#pragma unroll
            for (int q = 0; q < RT; q++)
                lds_vec<T, VEC>(v[q], reinterpret_cast<const T *>(
                                          stg + q * 256 * C::ROWB + tid * C::ROWB + ((ci ^ sw) << 4)));
#pragma unroll
            for (int e = 0; e < VEC; e++) {
                T hc[RP];
                lds_row<T, RP>(hc, sh + (ci * VEC + e) * C::RPS);
#pragma unroll
                for (int q = 0; q < RT; q++) {
                    if constexpr (RATIO) {
                        T wh = (T)0;
#pragma unroll
                        for (int k = 0; k < RP; k++) wh = fma(wrow[q][k], hc[k], wh);
                        const T qv = (wh != (T)0) ? ratio_div(v[q][e], wh) : (T)0;
#pragma unroll
                        for (int k = 0; k < RP; k++) acc[q][k] = fma(hc[k], qv, acc[q][k]);
                    } else {
#pragma unroll
                        for (int k = 0; k < RP; k++) acc[q][k] = fma(v[q][e], hc[k], acc[q][k]);
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (producer && i >= kLag && i - kLag + C::STAGES < nunits) {
            if (!produce<C::STAGES, C::STAGE, C::VBYTES + C::HBYTES>(
                    smem, full, empty, i - kLag + C::STAGES, issue)) {
                record_timeout(st, TIMEOUT_EMPTY);
                ok = false;
                break;
            }
        }
        if constexpr (sizeof(T) == 4) {
            if (++cnt == C::FLUSH2) {
                cnt = 0;
#pragma unroll
                for (int q = 0; q < RT; q++)
#pragma unroll
                    for (int k = 0; k < RP; k++) {
                        acc2[q][k] += (Total)acc[q][k];
                        acc[q][k] = (T)0;
                    }
            }
        }
    }
    if (ok && cur >= 0) flush(cur);
}

// ---------------------------------------------------------------------------
// Epilogues for the stream-K partials
// ---------------------------------------------------------------------------

// One thread per column: sum the tile's partials in CTA order, apply the H
// update, write H (RP x p, f64) and the copy H^T (p x RPS_T, type TH) that
// the next W pass streams.
template <int RP, typename TH, int RPS_T>
__global__ void __launch_bounds__(kThreads)
    h_epilogue_sk(double *__restrict__ H, TH *__restrict__ Ht, int p,
                  const double *__restrict__ part, StreamK sk, int tcols, EpiParams e,
                  const RunState *st) {
    if (run_stopped(st)) return;
    const int j = blockIdx.x * kThreads + threadIdx.x;
    if (j >= p) return;
    const int t = j / tcols, c = j - t * tcols;
    int lo = 0, hi = -1;  // no units at all (n == 0): every sum is empty
    if (sk.G > 0) sk_range(sk, t, &lo, &hi);
    double num[RP], hc[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) {
        num[k] = 0.0;
        hc[k] = H[(size_t)k * p + j];
    }
    for (int b = lo; b <= hi; b++) {
        const int slot = t - (int)(sk.start(b) / sk.UPT);
        const double *src = part + ((size_t)b * sk.slots + slot) * RP * tcols + c;
#pragma unroll
        for (int k = 0; k < RP; k++) num[k] += src[(size_t)k * tcols];
    }
    h_update<RP>(e, num, hc);
#pragma unroll
    for (int k = 0; k < RP; k++)
        if (k < e.r) H[(size_t)k * p + j] = hc[k];
    TH *ht = Ht + (size_t)j * RPS_T;
#pragma unroll
    for (int k = 0; k < RPS_T; k++) ht[k] = (k < e.r && k < RP) ? (TH)hc[k] : (TH)0;
}

// One thread per row: sum the tile's partials in CTA order, apply the W update.
template <int RP>
__global__ void __launch_bounds__(kThreads)
    w_epilogue_sk(double *__restrict__ W, int n, const double *__restrict__ part, StreamK sk,
                  int trows, EpiParams e, const RunState *st) {
    if (run_stopped(st)) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const int t = i / trows, rl = i - t * trows;
    int lo = 0, hi = -1;  // no units at all (p == 0): every sum is empty
    if (sk.G > 0) sk_range(sk, t, &lo, &hi);
    double num[RP], wr[RP];
#pragma unroll
    for (int k = 0; k < RP; k++) {
        num[k] = 0.0;
        wr[k] = W[(size_t)i * RP + k];
    }
    for (int b = lo; b <= hi; b++) {
        const int slot = t - (int)(sk.start(b) / sk.UPT);
        const double *src = part + (((size_t)b * sk.slots + slot) * trows + rl) * RP;
#pragma unroll
        for (int k = 0; k < RP; k++) num[k] += src[k];
    }
    w_update<RP>(e, num, wr);
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

// tc.cuh -- the two V passes of lee / hals / dnmf on the tensor cores
// (tcgen05), for the split-bf16 precision form.
//
// V is held as two bf16 arrays, Vh = bf16(V) and Vl = bf16(V - Vh) (4 bytes
// an element, like an f32 V), the factor of the pass as three bf16 terms
// (Fh + Fm + Fl ~ F to about 2^-24).  A pass computes, per tile of 128
// outputs, D = A * B^T with A the V tile and B the factor, as five bf16
// products accumulated in f32 in tensor memory:
//   Vh Fh + Vh Fm + Vl Fh + Vh Fl + Vl Fm
// (Vl Fl, ~2^-24 relative, is dropped).  The three factor terms sit in
// shared memory as one stacked operand [Fh; Fm; Fl], so a K step is two MMAs
// -- Vh x [Fh; Fm; Fl] (N = 3 RPN) and Vl x [Fh; Fm] (N = 2 RPN) -- into one
// accumulator of 3 RPN columns whose three column groups the epilogue adds;
// each V tile is read from shared memory twice per K step, not five times.
//
//   W pass  D[i][k] = sum_j V[i][j] H[k][j]     A = V tile, K-major (rows of V)
//   H pass  D[j][k] = sum_i V[i][j] W[i][k]     A = V^T tile, K-major (rows of a
//                                               transposed split copy made once a
//                                               run), or the V tile read MN-major
// Both passes then walk each A row 128 bytes at a time, so consecutive units
// of a CTA stay in the same DRAM pages.
//
// One CTA per SM, six warps: warp 0 issues the TMA loads of a ring of
// shared-memory stages, warp 1 owns the tensor memory and issues the MMAs
// (one thread), warps 2..5 move finished accumulators from tensor memory to
// the stream-K partial buffer.  Work is split stream-K exactly like the
// CUDA-core passes (stream.cuh): a unit is 64 streamed elements of one tile,
// a segment of at most 32 units bounds every f32 sum to 2048 terms, the
// epilogue warps add a CTA's segments of one tile in f64, and each CTA
// writes one f64 partial per tile it touches (folded stream-K partials), in
// the layout the CUDA-core epilogues read (H: [RP][128], W: [128][RP]).  Two
// accumulators let the MMAs of the next segment run while the previous one
// is drained.  Every wait is bounded; a CTA that gives up records a timeout
// in RunState, waits (bounded) for its own loads and MMAs, frees its tensor
// memory and returns.
#pragma once

#include <cuda_bf16.h>

#include "stream.cuh"

namespace nmfcu {
namespace tc {

constexpr int kM = 128;         // outputs per tile (MMA M)
constexpr int kKC = 64;         // streamed elements per unit (a 128-B bf16 row)
constexpr int kStages = 5;
constexpr int kWarps = 6;       // 0 TMA, 1 MMA + TMEM, 2..5 epilogue
constexpr int kThreadsTC = kWarps * 32;
constexpr int kTmemCols = 256;  // two accumulators of up to 96 columns (at 0, 128)
constexpr int kSegUnits = 32;   // units per segment: 2048 terms per f32 sum

template <int RPN>
struct TcCfg {
    static_assert(RPN == 16 || RPN == 32, "MMA N (padded rank) must be 16 or 32");
    static constexpr int A_PART = kM * kKC * 2;     // one bf16 V tile (hi or lo)
    static constexpr int B_PART = RPN * kKC * 2;    // one bf16 term of the factor
    static constexpr int STAGE = 2 * A_PART + 3 * B_PART;
    static_assert(A_PART % 1024 == 0 && B_PART % 1024 == 0, "swizzle atoms need 1 KB alignment");
};

struct TcBars {
    uint64_t full[kStages];
    uint64_t empty[kStages];
    uint64_t accf[2];   // accumulator a holds a finished segment (MMA commit)
    uint64_t acce[2];   // accumulator a has been read (128 epilogue arrivals)
    uint64_t drain;     // all MMAs of this CTA finished (abort path)
    uint32_t tmem_base;
    int abort;
};

template <int RPN>
constexpr int tc_smem_bytes() {
    return kStages * TcCfg<RPN>::STAGE + (int)sizeof(TcBars) + 1024;  // + alignment slack
}

// ---------------------------------------------------------------------------
// tcgen05 / descriptor helpers
// ---------------------------------------------------------------------------

// Shared-memory matrix descriptor of a 128-B-swizzled bf16 tile.
//   K-major  (rows of 64 K-elements): SBO = 1024 B between 8-row groups.
//   MN-major (rows of 64 M/N-elements, one per K): LBO = byte distance between
//            64-wide M/N blocks, SBO = 1024 B between 8-K groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;  // 128-byte swizzle
    return d;
}

// Instruction descriptor: bf16 x bf16 -> f32, M = 128, N = RPN, B K-major.
template <int N, bool A_MN_MAJOR>
__host__ __device__ constexpr uint32_t instr_desc() {
    static_assert(N % 16 == 0 && N >= 16 && N <= 256, "MMA N for M = 128");
    return (1u << 4)                        // D format f32
           | (1u << 7)                      // A format bf16
           | (1u << 10)                     // B format bf16
           | ((A_MN_MAJOR ? 1u : 0u) << 15) // A major
           | ((uint32_t)(N >> 3) << 17)     // N / 8
           | ((uint32_t)(kM >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t *holder, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(holder)),
                 "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                     uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrive on `bar` once every tcgen05 operation this thread issued so far is done.
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
// 16 consecutive f32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---------------------------------------------------------------------------
// The pass
// ---------------------------------------------------------------------------
//   tmAh/tmAl  A hi / lo (bf16), 128-B swizzle; box {64, 128} when A is read
//              K-major, {64, 64} when read MN-major
//   tmB[3]     factor terms (bf16, RPN rows x K), box {64, RPN}, 128-B swizzle
//   kext       streamed extent (columns of V for the W pass, rows for the H pass)
// A_MN: A is read MN-major (the V tile for the H pass, no transposed copy);
// OUT_KM: partials in the H epilogue's [RP][128] layout (else [128][RP]).
template <int RPN, bool A_MN, bool OUT_KM>
__global__ void __launch_bounds__(kThreadsTC, 1)
    tc_pass(const __grid_constant__ CUtensorMap tmAh, const __grid_constant__ CUtensorMap tmAl,
            const __grid_constant__ CUtensorMap tmBh, const __grid_constant__ CUtensorMap tmBm,
            const __grid_constant__ CUtensorMap tmBl, int kext, int RP, StreamK sk,
            double *__restrict__ part, RunState *st) {
    using C = TcCfg<RPN>;
    extern __shared__ unsigned char tc_smem_raw[];
    if (run_stopped(st)) return;
    // 1 KB-aligned base for the swizzle atoms (offset, not a pointer cast,
    // keeps the accesses in the shared address space).
    const uint32_t raw = smem_u32(tc_smem_raw);
    unsigned char *smem = tc_smem_raw + ((1024 - (raw & 1023)) & 1023);
    TcBars &bars = *reinterpret_cast<TcBars *>(smem + kStages * C::STAGE);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x;
    const long long u0 = sk.start(b), u1 = sk.start(b + 1);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&bars.full[s], 1);
            mbar_init(&bars.empty[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&bars.accf[a], 1);
            mbar_init(&bars.acce[a], 4 * 32);
        }
        mbar_init(&bars.drain, 1);
        bars.abort = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(&bars.tmem_base, kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = bars.tmem_base;
    volatile int *abort_flag = &bars.abort;
    auto give_up = [&]() {
        *abort_flag = 1;
        record_timeout(st, TIMEOUT_FULL);
    };

    if (warp == 0 && lane == 0) {
        // ---- TMA producer -------------------------------------------------
        int s = 0;
        uint32_t ph = 0;
        int issued[kStages] = {0};
        const uint64_t pol_v = l2_evict_first_policy(), pol_f = l2_evict_last_policy();
        UnitCursor cur;
        cur.init(sk, u0);
        for (long long u = u0; u < u1; ++u, cur.next(sk)) {
            if (*abort_flag) break;
            const int kc = cur.along(sk);
            if ((long long)kc * kKC >= kext) continue;  // past the streamed extent
            if (!mbar_wait(&bars.empty[s], ph ^ 1)) {
                give_up();
                break;
            }
            unsigned char *base = smem + s * C::STAGE;
            mbar_expect_tx(&bars.full[s], C::STAGE);
            // V is streamed once (evict first); the factor terms are re-read by
            // every tile (evict last).
            if (A_MN) {
                const int x = cur.major * kM, y = kc * kKC;
                tma_load_2d_hint(base, &tmAh, &bars.full[s], x, y, pol_v);
                tma_load_2d_hint(base + C::A_PART / 2, &tmAh, &bars.full[s], x + 64, y, pol_v);
                tma_load_2d_hint(base + C::A_PART, &tmAl, &bars.full[s], x, y, pol_v);
                tma_load_2d_hint(base + C::A_PART + C::A_PART / 2, &tmAl, &bars.full[s], x + 64, y,
                                 pol_v);
            } else {
                const int x = kc * kKC, y = cur.major * kM;
                tma_load_2d_hint(base, &tmAh, &bars.full[s], x, y, pol_v);
                tma_load_2d_hint(base + C::A_PART, &tmAl, &bars.full[s], x, y, pol_v);
            }
            unsigned char *bb = base + 2 * C::A_PART;
            tma_load_2d_hint(bb, &tmBh, &bars.full[s], kc * kKC, 0, pol_f);
            tma_load_2d_hint(bb + C::B_PART, &tmBm, &bars.full[s], kc * kKC, 0, pol_f);
            tma_load_2d_hint(bb + 2 * C::B_PART, &tmBl, &bars.full[s], kc * kKC, 0, pol_f);
            issued[s]++;
            if (++s == kStages) {
                s = 0;
                ph ^= 1;
            }
        }
        if (*abort_flag) {
            // Let this CTA's own loads land before the CTA exits.
            for (int i = 0; i < kStages; i++)
                if (issued[i] > 0) mbar_wait(&bars.full[i], (uint32_t)((issued[i] - 1) & 1));
        }
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer ---------------------------------------------------
        constexpr uint32_t idesc3 = instr_desc<3 * RPN, A_MN>();  // Vh x [Fh; Fm; Fl]
        constexpr uint32_t idesc2 = instr_desc<2 * RPN, A_MN>();  // Vl x [Fh; Fm]
        int s = 0;
        uint32_t ph = 0;
        int acc = 0;
        uint32_t aph[2] = {0, 0};
        UnitCursor cur;
        cur.init(sk, u0);
        long long u = u0;
        while (u < u1 && !*abort_flag) {
            const int t = cur.t;
            if (!mbar_wait(&bars.acce[acc], aph[acc] ^ 1)) {
                give_up();
                break;
            }
            aph[acc] ^= 1;
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(acc * 128);
            uint32_t accumulate = 0;
            for (; u < u1 && cur.t == t; ++u, cur.next(sk)) {
                const int kc = cur.along(sk);
                if ((long long)kc * kKC >= kext) continue;
                if (!mbar_wait(&bars.full[s], ph)) {
                    give_up();
                    break;
                }
                tc_fence_after();
                const uint32_t base = smem_u32(smem + s * C::STAGE);
                const uint32_t ah = base, al = base + C::A_PART, bs = base + 2 * C::A_PART;
#pragma unroll
                for (int ks = 0; ks < kKC / 16; ks++) {
                    // K step of 16 elements: 32 B into a K-major row, 2 swizzle
                    // atoms (2 KB) down an MN-major tile.
                    const uint32_t ka = A_MN ? (uint32_t)ks * 2048u : (uint32_t)ks * 32u;
                    const uint32_t lbo_a = A_MN ? (uint32_t)(C::A_PART / 2) : 16u;
                    const uint64_t dah = smem_desc(ah + ka, lbo_a, 1024);
                    const uint64_t dal = smem_desc(al + ka, lbo_a, 1024);
                    const uint64_t dbs = smem_desc(bs + (uint32_t)ks * 32u, 16, 1024);
                    umma(d, dah, dbs, idesc3, accumulate);
                    umma(d, dal, dbs, idesc2, 1);
                    accumulate = 1;
                }
                umma_commit(&bars.empty[s]);  // the stage is free once these MMAs are done
                if (++s == kStages) {
                    s = 0;
                    ph ^= 1;
                }
            }
            if (*abort_flag) break;
            umma_commit(&bars.accf[acc]);
            acc ^= 1;
        }
        if (*abort_flag) {
            umma_commit(&bars.drain);
            mbar_wait(&bars.drain, 0);
        }
    } else if (warp >= 2) {
        // ---- epilogue: tensor memory -> f64 partials -----------------------
        const int q = warp & 3;           // lane quarter this warp may read
        const int row = q * 32 + lane;    // output index within the tile
        const uint32_t lane_off = (uint32_t)(q * 32) << 16;
        int acc = 0;
        uint32_t fph[2] = {0, 0};
        UnitCursor cur;
        cur.init(sk, u0);
        long long u = u0;
        const int major0 = cur.major;
        // The segments of one major tile are added here in f64, in segment
        // order, and written once per (CTA, major tile) when the next unit
        // starts another major tile or the CTA's range ends.
        double sum[RPN];
#pragma unroll
        for (int i = 0; i < RPN; i++) sum[i] = 0.0;
        while (u < u1) {
            const int t = cur.t, m = cur.major;
            bool any = false;
            for (; u < u1 && cur.t == t; ++u, cur.next(sk))
                if ((long long)cur.along(sk) * kKC < kext) any = true;
            if (!mbar_wait(&bars.accf[acc], fph[acc])) {
                give_up();
                break;
            }
            fph[acc] ^= 1;
            tc_fence_after();
            float v[RPN];
            if (any) {
                // Column groups [0, RPN), [RPN, 2 RPN), [2 RPN, 3 RPN): the
                // products with Fh, Fm and Fl; their sum is the result.
#pragma unroll
                for (int c0 = 0; c0 < RPN; c0 += 16) {
                    float x0[16], x1[16], x2[16];
                    const uint32_t ta = tmem + lane_off + (uint32_t)(acc * 128 + c0);
                    tmem_ld16(ta, x0);
                    tmem_ld16(ta + RPN, x1);
                    tmem_ld16(ta + 2 * RPN, x2);
                    tmem_wait_ld();
#pragma unroll
                    for (int i = 0; i < 16; i++) v[c0 + i] = x0[i] + x1[i] + x2[i];
                }
            } else {
#pragma unroll
                for (int i = 0; i < RPN; i++) v[i] = 0.f;
            }
            tc_fence_before();
            mbar_arrive(&bars.acce[acc]);
#pragma unroll
            for (int k = 0; k < RPN; k++) sum[k] += (double)v[k];
            if (u >= u1 || cur.major != m) {
                double *dst =
                    part + ((size_t)b * sk.slots + (size_t)(m - major0)) * (size_t)kM * RP;
#pragma unroll
                for (int k = 0; k < RPN; k++) {
                    if (k < RP) {
                        if (OUT_KM)
                            dst[(size_t)k * kM + row] = sum[k];
                        else
                            dst[(size_t)row * RP + k] = sum[k];
                    }
                    sum[k] = 0.0;
                }
            }
            acc ^= 1;
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) {
        __syncwarp();
        tmem_dealloc(tmem, kTmemCols);
    }
}

// Split kernels.  V (f64, n x p, leading dimension ldv) -> Vh, Vl (bf16,
// n x ldb) and Vth, Vtl (bf16 V^T, p x ldbt), zero in the pad columns.
__global__ void split_v_both(const double *__restrict__ V, int64_t ldv,
                             __nv_bfloat16 *__restrict__ Vh, __nv_bfloat16 *__restrict__ Vl,
                             int64_t ldb, __nv_bfloat16 *__restrict__ Vth,
                             __nv_bfloat16 *__restrict__ Vtl, int64_t ldbt, int n, int p);
// F (f64, logically R x K with F(k, x) = F[k * fk + x * fx]) -> three bf16
// terms, each RPN x ldk (rows k >= R and columns x >= K zero).
__global__ void split_factor(const double *__restrict__ F, int64_t fk, int64_t fx, int R, int K,
                             __nv_bfloat16 *__restrict__ out, int RPN, int64_t ldk,
                             const RunState *st);

}  // namespace tc
}  // namespace nmfcu

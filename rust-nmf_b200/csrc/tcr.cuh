// tcr.cuh -- brunet's two V passes on the tensor cores (tcgen05), for the
// split-bf16 precision form.
//
// The KL multiplicative update contracts the element-wise ratio V / (W H)
// with a factor (rust/src/lib.rs:74-115 divergence_update_h_inner, 151-204
// divergence_update_w_impl; the loop nmf_run_brunet, 1529-1586):
//   H pass  N[j][k] = sum_i W[i][k] V[i][j] / (W H)[i][j]
//   W pass  N[i][k] = sum_j H[k][j] V[i][j] / (W H)[i][j]
// Per tile of 128 outputs (columns j for the H pass, rows i for the W pass)
// and chunk of 64 streamed elements (rows i, columns j) the pass runs two
// MMAs with the element-wise step between them, like the FP64 ratio passes:
//   MMA1  WH[o][e] = sum_k T[o][k] F[e][k]      T: the tile's factor rows,
//                                               F: the chunk's factor rows
//   ratio Q[o][e]  = V[o][e] / WH[o][e]         (0 where WH is 0), f32, on
//                                               the CUDA cores, split into
//                                               bf16 hi + lo in shared memory
//   MMA2  N[o][k] += sum_e Q[o][e] F[e][k]      accumulated over a segment;
//                                               F read from MMA1's tile of it,
//                                               as an MN-major operand
// so W H is never written out.  V is read once, as f32 (4 bytes an element);
// the factors are L2-resident.  Factor operands are three bf16 terms each
// (Fh + Fm + Fl ~ F to about 2^-24); MMA1 keeps the six products down to
// 2^-16 x 2^-8 (Th[Fh;Fm;Fl], Tm[Fh;Fm], Tl Fh as N = 192 / 128 / 64 into
// one accumulator of three column groups), MMA2 the five of the split-bf16
// lee passes (Qh [Fh;Fm;Fl] + Ql [Fh;Fm], N = 96 / 64).
//
// One CTA per SM, twenty warps: warp 0 loads V into a ring of its own (a
// slot is refilled as soon as the ratio step has read it), warp 1 the factor
// terms (L2-resident), warp 2 owns the tensor memory and issues MMA1 of each
// chunk as soon as a WH accumulator is free, warp 3 issues MMA2 behind the
// ratio step (two issuers, so that MMA1 of later chunks never waits on a
// contraction), warps 4..19 read WH from tensor memory, form Q and drain the
// contraction: warp w reads TMEM lanes 32 (w mod 4) .. +31, and the four
// warps of a lane quarter take 16 of the chunk's 64 elements each.  Tensor memory:
// two WH accumulators (3 x 64 columns at 0 and 192), one contraction
// accumulator (3 x 32 columns at 384).  The stream-K split, the 2048-term
// segments of every f32 sum and the folded f64 partials (one per CTA and
// tile, layout H: [RP][128], W: [128][RP]) are those of the split-bf16 lee
// passes, so the CUDA-core brunet epilogues apply unchanged.  Every wait is
// bounded; a CTA that gives up records a timeout, lets its own loads and
// MMAs finish, frees its tensor memory and returns.
#pragma once

#include "tc.cuh"

namespace nmfcu {
namespace tcr {

constexpr int kM = 128;        // outputs per tile (TMEM lanes, MMA M)
constexpr int kC = 64;         // streamed elements per chunk (one stream-K unit)
constexpr int kR = 32;         // padded rank: MMA1's K, MMA2's N per factor term
constexpr int kVStages = 4;   // V ring: freed as soon as the ratio step has read V
constexpr int kFStages = 3;   // factor ring: freed when the chunk's MMA2 is done
// Warp roles: V producer, factor producer, MMA1 issuer (and the tensor
// memory's owner), MMA2 issuer, then the epilogue warps.
constexpr int kVProdWarp = 0, kFProdWarp = 1, kMma1Warp = 2, kMma2Warp = 3, kEpiWarp0 = 4;
constexpr int kEpiWarps = 16;
constexpr int kParts = kEpiWarps / 4;       // epilogue warps per TMEM lane quarter
constexpr int kPartElems = kC / kParts;    // chunk elements per epilogue warp
constexpr int kPartRanks = kR / kParts;    // contraction ranks per epilogue warp
constexpr int kWarps = kEpiWarp0 + kEpiWarps;
constexpr int kThreads = kWarps * 32;
constexpr int kSegUnits = 32;  // chunks per segment: 2048 terms per f32 sum
constexpr int kTmemCols = 512;
constexpr uint32_t kD1 = 0;    // WH accumulators at columns 0 and 192
constexpr uint32_t kD1Cols = 192;
constexpr uint32_t kD2 = 384;  // contraction accumulator (96 columns)

// Shared memory, from a 1 KB-aligned base.
constexpr int V_BYTES = kC * kM * 4;      // the f32 V chunk (one V ring slot)
// One factor term of a chunk: 64 rows x 32 k, 64-B swizzle.  MMA1 reads it
// K-major (B = F, K = k); MMA2 reads the same tile MN-major (B[k][e], N = k
// along a row, K = e down the rows), the three terms one 32-wide N block
// apart.
constexpr int F1_TERM = kC * kR * 2;
constexpr int F_SLOT = 3 * F1_TERM;       // one factor ring slot: the three terms
constexpr int T_TERM = kM * kR * 2;       // MMA1's A term: 128 rows x 32 k, 64-B swizzle
constexpr int Q_PLANE = kM * kC * 2;      // Q hi or lo: 128 x 64, 128-B swizzle
constexpr int OFF_F = kVStages * V_BYTES;
constexpr int OFF_T = OFF_F + kFStages * F_SLOT;
constexpr int OFF_Q = OFF_T + 3 * T_TERM;
constexpr int OFF_BARS = OFF_Q + 2 * Q_PLANE;
static_assert(V_BYTES % 1024 == 0 && F_SLOT % 1024 == 0 && OFF_F % 1024 == 0 &&
                  OFF_T % 1024 == 0 && OFF_Q % 1024 == 0 && T_TERM % 1024 == 0 &&
                  Q_PLANE % 1024 == 0 && F1_TERM % 512 == 0,
              "swizzle atoms need their alignment");

struct Bars {
    uint64_t vfull[kVStages];   // V slot loaded (TMA bytes)
    uint64_t vempty[kVStages];  // V slot read (one arrival per epilogue warp)
    uint64_t ffull[kFStages];   // factor slot loaded (TMA bytes)
    uint64_t fempty[kFStages];  // factor slot free (MMA2 of its chunk done)
    uint64_t tfull, tempty;   // the tile operand loaded / free (last MMA1 of its tile done)
    uint64_t d1full[2];       // WH accumulator b written (MMA1 commit)
    uint64_t d1empty[2];      // WH accumulator b read (one arrival per epilogue warp)
    uint64_t qfull, qempty;   // Q written (epilogue warps) / read (MMA2 commit)
    uint64_t d2full, d2empty; // a segment's contraction done / drained (epilogue warps)
    uint64_t drain[2];        // every MMA of an issuer done (abort path)
    uint32_t tmem_base;
    int abort;
};
constexpr int SMEM = OFF_BARS + (int)sizeof(Bars) + 1024;  // + alignment slack
static_assert(SMEM <= 232448, "shared memory per CTA");

// K-major shared-memory descriptor, 64-byte swizzle (rows of 32 bf16): 8-row
// groups 512 bytes apart.
__device__ __forceinline__ uint64_t desc_sw64(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;               // leading byte offset (unused when swizzled)
    d |= (uint64_t)(512 >> 4) << 32;      // stride byte offset
    d |= (uint64_t)1 << 46;               // descriptor version (sm_100)
    d |= (uint64_t)4 << 61;               // 64-byte swizzle
    return d;
}
// MN-major, 64-byte swizzle: rows of 32 MN elements, one per K; 32-wide MN
// blocks `lbo` bytes apart, 8-K groups 512 bytes apart.
__device__ __forceinline__ uint64_t desc_sw64_mn(uint32_t addr, uint32_t lbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)(512 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)4 << 61;
    return d;
}
// Instruction descriptor as tc::instr_desc, with B read MN-major.
template <int N>
__host__ __device__ constexpr uint32_t instr_desc_bmn() {
    return tc::instr_desc<N, false>() | (1u << 16);
}
// K-major, 128-byte swizzle (rows of 64 bf16): 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr) {
    return tc::smem_desc(addr, 16, 1024);
}

// 8 consecutive 32-bit columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7])
        : "r"(taddr));
}

// Bounded wait that lets the thread sleep: each try suspends it until the
// phase completes or 1 us has passed, so waiting warps leave their issue
// slots to the working ones; at most 2^21 tries (about 2 s).
__device__ __forceinline__ bool mbar_sleep_wait(uint64_t *bar, uint32_t parity) {
    for (uint32_t i = 0; i < (1u << 21); ++i) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
            " selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity), "r"(1000u)
            : "memory");
        if (ok) return true;
    }
    return false;
}
// Bounded wait taken by a whole warp, with one outcome for all its lanes (the
// epilogue warps arrive once a warp, after a __syncwarp).
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity) {
    return __all_sync(0xffffffffu, mbar_sleep_wait(bar, parity)) != 0;
}

// Walks the valid chunks of a CTA's stream-K range in order (units past the
// streamed extent, which pad the last segment of a tile, are skipped).
struct ChunkWalker {
    UnitCursor cur;
    long long u, u1;
    bool ok;
    __device__ __forceinline__ void skip(const StreamK &sk, int kext) {
        while (u < u1 && (long long)cur.along(sk) * kC >= kext) {
            ++u;
            cur.next(sk);
        }
        ok = u < u1;
    }
    __device__ __forceinline__ void init(const StreamK &sk, long long u0, long long end, int kext) {
        cur.init(sk, u0);
        u = u0;
        u1 = end;
        skip(sk, kext);
    }
    __device__ __forceinline__ void advance(const StreamK &sk, int kext) {
        ++u;
        cur.next(sk);
        skip(sk, kext);
    }
};

// Position of one valid chunk in its tile and segment.
struct ChunkInfo {
    int t, major, along;
    bool first_seg, last_seg, last_tile;
};

// The chunk under `w`, given the tile-segment of the chunk before it (-1 for
// none); advances `w` past it.
__device__ __forceinline__ ChunkInfo take(ChunkWalker &w, const StreamK &sk, int kext,
                                          int prev_t) {
    ChunkInfo ci;
    ci.t = w.cur.t;
    ci.major = w.cur.major;
    ci.along = w.cur.along(sk);
    ci.first_seg = (ci.t != prev_t);
    w.advance(sk, kext);
    ci.last_seg = !w.ok || w.cur.t != ci.t;
    ci.last_tile = !w.ok || w.cur.major != ci.major;
    return ci;
}

// HPASS: tile = 128 columns of V, chunk = 64 rows; else tile = 128 rows,
// chunk = 64 columns.
//   tmV   the f32 V: HPASS box {128, 64}, no swizzle; else box {32, 128},
//         128-B swizzle (two boxes a chunk)
//   tmT   the tile factor's terms as [3][xpadT][32] bf16, box {32, 128}, 64-B swizzle
//   tmF1  the chunk factor's terms as [3][xpadF][32] bf16, box {32, 64}, 64-B swizzle
//   kext  streamed extent (n for the H pass, p for the W pass)
template <bool HPASS>
__global__ void __launch_bounds__(kThreads, 1)
    tcr_pass(const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmT,
             const __grid_constant__ CUtensorMap tmF1,
             int xpadT, int xpadF, int kext, int RP, StreamK sk, double *__restrict__ part,
             RunState *st) {
    extern __shared__ unsigned char tcr_smem_raw[];
    if (run_stopped(st)) return;
    const uint32_t raw = smem_u32(tcr_smem_raw);
    unsigned char *smem = tcr_smem_raw + ((1024 - (raw & 1023)) & 1023);
    Bars &bars = *reinterpret_cast<Bars *>(smem + OFF_BARS);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x;
    const long long u0 = sk.start(b), u1 = sk.start(b + 1);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kVStages; s++) {
            mbar_init(&bars.vfull[s], 1);
            mbar_init(&bars.vempty[s], kEpiWarps);
        }
        for (int s = 0; s < kFStages; s++) {
            mbar_init(&bars.ffull[s], 1);
            mbar_init(&bars.fempty[s], 1);
        }
        mbar_init(&bars.tfull, 1);
        mbar_init(&bars.tempty, 1);
        for (int a = 0; a < 2; a++) {
            mbar_init(&bars.d1full[a], 1);
            mbar_init(&bars.d1empty[a], kEpiWarps);
        }
        mbar_init(&bars.qfull, kEpiWarps);
        mbar_init(&bars.qempty, 1);
        mbar_init(&bars.d2full, 1);
        mbar_init(&bars.d2empty, kEpiWarps);
        mbar_init(&bars.drain[0], 1);
        mbar_init(&bars.drain[1], 1);
        bars.abort = 0;
        fence_mbar_init();
    }
    if (warp == kMma1Warp) {
        tc::tmem_alloc(&bars.tmem_base, kTmemCols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = bars.tmem_base;
    volatile int *abort_flag = &bars.abort;
    auto give_up = [&]() {
        *abort_flag = 1;
        record_timeout(st, TIMEOUT_FULL);
    };

    if (warp == kVProdWarp && lane == 0) {
        // ---- TMA producer of V ----------------------------------------------
        const uint64_t pol_v = l2_evict_first_policy();
        ChunkWalker w;
        w.init(sk, u0, u1, kext);
        int issued[kVStages] = {0};
        long long ci = 0;
        while (w.ok && !*abort_flag) {
            const int major = w.cur.major, along = w.cur.along(sk);
            const int s = (int)(ci % kVStages);
            if (!mbar_sleep_wait(&bars.vempty[s], (uint32_t)(((ci / kVStages) & 1) ^ 1))) {
                give_up();
                break;
            }
            unsigned char *base = smem + s * V_BYTES;
            mbar_expect_tx(&bars.vfull[s], V_BYTES);
            if (HPASS) {
                tma_load_2d_hint(base, &tmV, &bars.vfull[s], major * kM, along * kC, pol_v);
            } else {
                tma_load_2d_hint(base, &tmV, &bars.vfull[s], along * kC, major * kM, pol_v);
                tma_load_2d_hint(base + V_BYTES / 2, &tmV, &bars.vfull[s], along * kC + kC / 2,
                                 major * kM, pol_v);
            }
            issued[s]++;
            ++ci;
            w.advance(sk, kext);
        }
        if (*abort_flag) {
            // Let this thread's own loads land before the CTA exits.
            for (int i = 0; i < kVStages; i++)
                if (issued[i] > 0) mbar_sleep_wait(&bars.vfull[i], (uint32_t)((issued[i] - 1) & 1));
        }
    } else if (warp == kFProdWarp && lane == 0) {
        // ---- TMA producer of the factor terms (L2-resident) ------------------
        const uint64_t pol_f = l2_evict_last_policy();
        ChunkWalker w;
        w.init(sk, u0, u1, kext);
        int issued[kFStages] = {0};
        int tloads = 0, cur_major = -1;
        long long ci = 0;
        while (w.ok && !*abort_flag) {
            const int major = w.cur.major, along = w.cur.along(sk);
            if (major != cur_major) {
                // The tile operand is reloaded once the last MMA1 of the
                // previous tile has read it.
                if (tloads > 0 && !mbar_sleep_wait(&bars.tempty, (uint32_t)((tloads - 1) & 1))) {
                    give_up();
                    break;
                }
                mbar_expect_tx(&bars.tfull, 3 * T_TERM);
                for (int q = 0; q < 3; q++)
                    tma_load_2d_hint(smem + OFF_T + q * T_TERM, &tmT, &bars.tfull, 0,
                                     q * xpadT + major * kM, pol_f);
                ++tloads;
                cur_major = major;
            }
            const int s = (int)(ci % kFStages);
            if (!mbar_sleep_wait(&bars.fempty[s], (uint32_t)(((ci / kFStages) & 1) ^ 1))) {
                give_up();
                break;
            }
            unsigned char *base = smem + OFF_F + s * F_SLOT;
            mbar_expect_tx(&bars.ffull[s], F_SLOT);
            for (int q = 0; q < 3; q++)
                tma_load_2d_hint(base + q * F1_TERM, &tmF1, &bars.ffull[s], 0,
                                 q * xpadF + along * kC, pol_f);
            issued[s]++;
            ++ci;
            w.advance(sk, kext);
        }
        if (*abort_flag) {
            for (int i = 0; i < kFStages; i++)
                if (issued[i] > 0) mbar_sleep_wait(&bars.ffull[i], (uint32_t)((issued[i] - 1) & 1));
            if (tloads > 0) mbar_sleep_wait(&bars.tfull, (uint32_t)((tloads - 1) & 1));
        }
    } else if ((warp == kMma1Warp || warp == kMma2Warp) && lane == 0) {
        // ---- MMA issuers ------------------------------------------------------
        // MMA1 (W H of a chunk) runs ahead, held back only by free WH
        // accumulators and landed factor terms; MMA2 (the contraction)
        // follows the ratio step.  Each commit covers its own thread's MMAs.
        constexpr uint32_t id192 = tc::instr_desc<192, false>();
        constexpr uint32_t id128 = tc::instr_desc<128, false>();
        constexpr uint32_t id64 = tc::instr_desc<64, false>();
        constexpr uint32_t id96m = instr_desc_bmn<96>();  // MMA2: B = F MN-major
        constexpr uint32_t id64m = instr_desc_bmn<64>();
        const uint32_t sbase = smem_u32(smem);
        const bool first = (warp == kMma1Warp);
        ChunkWalker w;
        w.init(sk, u0, u1, kext);
        long long ci = 0;
        int tcount = 0, segs = 0, prev_t = -1, prev_major = -1;
        bool ok = true;
        while (w.ok && !*abort_flag) {
            const ChunkInfo c = take(w, sk, kext, prev_t);
            prev_t = c.t;
            const int s = (int)(ci % kFStages);
            const uint32_t fB = sbase + OFF_F + s * F_SLOT;
            if (first) {
                // MMA1 of chunk ci into WH accumulator ci & 1.
                if (!mbar_sleep_wait(&bars.ffull[s], (uint32_t)((ci / kFStages) & 1))) {
                    ok = false;
                    break;
                }
                if (c.major != prev_major) {
                    if (!mbar_sleep_wait(&bars.tfull, (uint32_t)(tcount & 1))) {
                        ok = false;
                        break;
                    }
                    ++tcount;
                    prev_major = c.major;
                }
                const int db = (int)(ci & 1);
                if (!mbar_sleep_wait(&bars.d1empty[db], (uint32_t)(((ci >> 1) & 1) ^ 1))) {
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t d = tmem + kD1 + (uint32_t)db * kD1Cols;
                const uint32_t tA = sbase + OFF_T;
#pragma unroll
                for (int ks = 0; ks < kR / 16; ks++) {
                    const uint32_t ko = (uint32_t)ks * 32u;  // 16 bf16 along a 64-byte row
                    const uint64_t bdesc = desc_sw64(fB + ko);
                    tc::umma(d, desc_sw64(tA + ko), bdesc, id192, ks > 0 ? 1u : 0u);
                    tc::umma(d, desc_sw64(tA + T_TERM + ko), bdesc, id128, 1u);
                    tc::umma(d, desc_sw64(tA + 2 * T_TERM + ko), bdesc, id64, 1u);
                }
                tc::umma_commit(&bars.d1full[db]);
                if (c.last_tile) tc::umma_commit(&bars.tempty);
            } else {
                // MMA2 of chunk ci into the contraction accumulator.  The
                // factor slot landed before MMA1 of this chunk, which the
                // ratio step waited for.
                if (c.first_seg && segs > 0 &&
                    !mbar_sleep_wait(&bars.d2empty, (uint32_t)((segs - 1) & 1))) {
                    ok = false;
                    break;
                }
                if (!mbar_sleep_wait(&bars.qfull, (uint32_t)(ci & 1))) {
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t qh = sbase + OFF_Q, ql = qh + Q_PLANE;
#pragma unroll
                for (int ks = 0; ks < kC / 16; ks++) {
                    // K step: 16 bf16 along a Q row; 16 rows (1 KB) down F.
                    const uint64_t bdesc = desc_sw64_mn(fB + (uint32_t)ks * 1024u, F1_TERM);
                    tc::umma(tmem + kD2, desc_sw128(qh + (uint32_t)ks * 32u), bdesc, id96m,
                             (c.first_seg && ks == 0) ? 0u : 1u);
                    tc::umma(tmem + kD2, desc_sw128(ql + (uint32_t)ks * 32u), bdesc, id64m, 1u);
                }
                tc::umma_commit(&bars.qempty);
                tc::umma_commit(&bars.fempty[s]);
                if (c.last_seg) {
                    tc::umma_commit(&bars.d2full);
                    ++segs;
                }
            }
            ++ci;
        }
        if (!ok) give_up();
        if (*abort_flag) {
            uint64_t *dr = first ? &bars.drain[0] : &bars.drain[1];
            tc::umma_commit(dr);
            mbar_sleep_wait(dr, 0);
        }
    } else if (warp >= kEpiWarp0) {
        // ---- epilogue: WH -> Q, and the contraction -> f64 partials --------
        const int q = warp & 3;                  // lane quarter this warp may read
        const int pw = (warp - kEpiWarp0) >> 2;  // its share of the chunk / the ranks
        const int e0 = pw * kPartElems;        // first chunk element of this warp
        const int o = q * 32 + lane;             // output (TMEM lane) within the tile
        const uint32_t lane_off = (uint32_t)(q * 32) << 16;
        unsigned char *qrow0 = smem + OFF_Q + o * 128;  // this output's Q row (hi plane)
        ChunkWalker w;
        w.init(sk, u0, u1, kext);
        const int major0 = (int)(u0 / sk.major_units());
        long long ci = 0;
        int segs = 0, prev_t = -1;
        double sum[kPartRanks];
#pragma unroll
        for (int i = 0; i < kPartRanks; i++) sum[i] = 0.0;
        while (w.ok && !*abort_flag) {
            const ChunkInfo c = take(w, sk, kext, prev_t);
            prev_t = c.t;
            const int s = (int)(ci % kVStages), db = (int)(ci & 1);
            // V first: its slot is refilled as soon as every epilogue thread
            // has read its 16 values.
            if (!warp_wait(&bars.vfull[s], (uint32_t)((ci / kVStages) & 1))) {
                give_up();
                break;
            }
            const unsigned char *vs = smem + s * V_BYTES;
            uint32_t packh[kPartElems / 2], packl[kPartElems / 2];  // Q hi / lo, bf16 pairs
            {
                // Elements e0 .. e0 + 15 of the chunk.
                float v[16];
                if (HPASS) {
                    const float *vf = reinterpret_cast<const float *>(vs);
#pragma unroll
                    for (int i = 0; i < 16; i++) v[i] = vf[(e0 + i) * kM + o];
                } else {
                    // Box e0 / 32 holds columns (e0 / 32) * 32 .. +31 of rows
                    // 0..127, 16-byte chunk ch of row o at (ch ^ (o & 7)).
                    const unsigned char *row = vs + (e0 >> 5) * (V_BYTES / 2) + o * 128;
#pragma unroll
                    for (int c4 = 0; c4 < 4; c4++) {
                        const int ch = ((e0 & 31) >> 2) + c4;
                        const float4 x =
                            *reinterpret_cast<const float4 *>(row + ((ch ^ (o & 7)) << 4));
                        v[4 * c4] = x.x;
                        v[4 * c4 + 1] = x.y;
                        v[4 * c4 + 2] = x.z;
                        v[4 * c4 + 3] = x.w;
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&bars.vempty[s]);
                // W H as the sum of the three column groups.
                if (!warp_wait(&bars.d1full[db], (uint32_t)((ci >> 1) & 1))) {
                    give_up();
                    break;
                }
                tc::tc_fence_after();
                float g0[16], g1[16], g2[16];
                const uint32_t ta =
                    tmem + lane_off + kD1 + (uint32_t)db * kD1Cols + (uint32_t)e0;
                tc::tmem_ld16(ta, g0);
                tc::tmem_ld16(ta + 64, g1);
                tc::tmem_ld16(ta + 128, g2);
                tc::tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; i += 2) {
                    float qv[2];
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const float wh = g0[i + e] + g1[i + e] + g2[i + e];
                        qv[e] = (wh != 0.f) ? ratio_div(v[i + e], wh) : 0.f;
                    }
                    const __nv_bfloat162 hi = __floats2bfloat162_rn(qv[0], qv[1]);
                    const float2 hf = __bfloat1622float2(hi);
                    const __nv_bfloat162 lo = __floats2bfloat162_rn(qv[0] - hf.x, qv[1] - hf.y);
                    packh[i / 2] = *reinterpret_cast<const uint32_t *>(&hi);
                    packl[i / 2] = *reinterpret_cast<const uint32_t *>(&lo);
                }
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars.d1empty[db]);
            // Q of the previous chunk must have been read by its MMA2.
            if (!warp_wait(&bars.qempty, (uint32_t)((ci & 1) ^ 1))) {
                give_up();
                break;
            }
            unsigned char *qrow = qrow0;
#pragma unroll
            for (int c2 = 0; c2 < 2; c2++) {
                const int kc = (e0 >> 3) + c2;  // 16-byte chunk of the 128-byte Q row
                const int pos = (kc ^ (o & 7)) << 4;
                *reinterpret_cast<uint4 *>(qrow + pos) =
                    make_uint4(packh[4 * c2], packh[4 * c2 + 1], packh[4 * c2 + 2],
                               packh[4 * c2 + 3]);
                *reinterpret_cast<uint4 *>(qrow + Q_PLANE + pos) =
                    make_uint4(packl[4 * c2], packl[4 * c2 + 1], packl[4 * c2 + 2],
                               packl[4 * c2 + 3]);
            }
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars.qfull);
            if (c.last_seg) {
                if (!warp_wait(&bars.d2full, (uint32_t)(segs & 1))) {
                    give_up();
                    break;
                }
                tc::tc_fence_after();
                // Ranks pw * 8 .. +7 of the three groups (the products with
                // Fh, Fm, Fl); their sum is the contraction.
                uint32_t x0[8], x1[8], x2[8];
                const uint32_t ta = tmem + lane_off + kD2 + (uint32_t)(pw * kPartRanks);
                tmem_ld8(ta, x0);
                tmem_ld8(ta + kR, x1);
                tmem_ld8(ta + 2 * kR, x2);
                tc::tmem_wait_ld();
                tc::tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bars.d2empty);
#pragma unroll
                for (int i = 0; i < kPartRanks; i++)
                    sum[i] += (double)(__uint_as_float(x0[i]) + __uint_as_float(x1[i]) +
                                       __uint_as_float(x2[i]));
                ++segs;
            }
            if (c.last_tile) {
                double *dst = part + ((size_t)b * sk.slots + (size_t)(c.major - major0)) *
                                         (size_t)kM * RP;
#pragma unroll
                for (int i = 0; i < kPartRanks; i++) {
                    const int k = pw * kPartRanks + i;
                    if (k < RP) {
                        if (HPASS)
                            dst[(size_t)k * kM + o] = sum[i];
                        else
                            dst[(size_t)o * RP + k] = sum[i];
                    }
                    sum[i] = 0.0;
                }
            }
            ++ci;
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    if (warp == kMma1Warp) {
        __syncwarp();
        tc::tmem_dealloc(tmem, kTmemCols);
    }
}

// The factor F (f64, logically R x K with F(k, x) = F[k * fk + x * fx]) as
// three bf16 terms in both layouts the passes read: kx = [3][RPN][ldk]
// (k-rows, as the split-bf16 lee passes) and xk = [3][xpad][32] (x-rows);
// zero outside k < R, x < K.  Either output may be null.
__global__ void split_factor_both(const double *__restrict__ F, int64_t fk, int64_t fx, int R,
                                  int K, __nv_bfloat16 *__restrict__ kx, int RPN, int64_t ldk,
                                  __nv_bfloat16 *__restrict__ xk, int64_t xpad,
                                  const RunState *st);

}  // namespace tcr
}  // namespace nmfcu

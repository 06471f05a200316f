// tcr.cuh -- brunet's two V passes on the tensor cores (tcgen05), for the
// split-bf16 precision form.
//
// The KL multiplicative update contracts the element-wise ratio V / (W H)
// with a factor (rust/src/lib.rs:74-115 divergence_update_h_inner, 151-204
// divergence_update_w_impl; the loop nmf_run_brunet, 1529-1586):
//   H pass  N[j][k] = sum_i W[i][k] V[i][j] / (W H)[i][j]
//   W pass  N[i][k] = sum_j H[k][j] V[i][j] / (W H)[i][j]
// Per tile of 128 outputs (columns j for the H pass, rows i for the W pass)
// and unit of 128 streamed elements (rows i, columns j) the pass runs two
// MMAs with the element-wise step between them, like the FP64 ratio passes:
//   MMA1  WH[o][e] = sum_k T[o][k] F[e][k]      T: the tile's factor rows,
//                                               F: the unit's factor rows
//   ratio Q[o][e]  = V[o][e] / WH[o][e]         (0 where WH is 0), f32, on
//                                               the CUDA cores, split into
//                                               bf16 hi + lo
//   MMA2  N[o][k] += sum_e Q[o][e] F[e][k]      accumulated over a segment
// so W H is never written out.  V is read once, as f32 (4 bytes an element);
// the factors are L2-resident.  Factor operands are three bf16 terms each
// (Fh + Fm + Fl ~ F to about 2^-24).
//
// A tcgen05 MMA (M = 128, K = 16) costs about the same issue time for any N
// up to 128, so the pass is shaped to issue few, wide MMAs: a 128-element
// unit makes MMA1 N = 128 (12 MMAs a unit: six term products x two 16-rank
// K steps), MMA2 is 8 K steps x 2 (Qh, Ql) with N = 96 / 64.
//
// Tensor memory carries everything that is not streamed, so shared memory
// holds only the two rings (V and the unit factor F) and its bandwidth goes
// to the streams:
//   * T, the tile operand of MMA1, sits in tensor memory for the whole tile
//     (MMA1 reads A from tensor memory): its three terms, 16 columns each.
//   * MMA1 adds the six products Th Fh, Th Fm, Th Fl, Tm Fh, Tm Fm, Tl Fh
//     (products down to 2^-16 x 2^-8) into ONE 128-column accumulator per
//     unit, so the ratio step reads one value an element.
//   * The ratio step writes Q back over the W H it has just read, as bf16
//     pairs: for unit elements 16g .. 16g + 15 the hi terms fill columns
//     16g .. 16g + 7 and the lo terms 16g + 8 .. 16g + 15 of the same
//     buffer, and MMA2 reads them as its A operand (K step g: Qh at 16g, Ql
//     at 16g + 8).  Each epilogue warp reads and rewrites only its own 32
//     columns.  MMA2 contracts Qh [Fh; Fm; Fl] + Ql [Fh; Fm] (N = 96 / 64,
//     B = F read MN-major) into a segment accumulator of three column groups.
//   * Two W H / Q buffers (a buffer is freed by the MMA2 that read its Q),
//     two segment accumulators (drained one unit late, so MMA2 of the next
//     segment never waits on the drain).
//
// One CTA per SM, twenty warps: warp 0 loads V by TMA into a ring of
// half-unit slots (a slot is refilled as soon as the ratio step has read
// it), warp 1 copies the unit factor terms with plain asynchronous copies,
// warp 2 owns the tensor memory and issues MMA1 as soon as a buffer is free,
// warp 3 issues MMA2 behind the ratio step, warps 4..19 form Q and drain the
// contraction: warp w reads tensor-memory lanes 32 (w mod 4) .. +31 and the
// four warps of a lane quarter take 32 of the unit's 128 elements each
// (three of them also write the quarter's rows of T when a tile starts).
// The stream-K split folds a CTA's segments (16 units: 2048 terms per f32
// sum) of one tile in f64 into one partial per CTA and tile (layout H:
// [RP][128], W: [128][RP]), the layout of the split-bf16 lee passes, so the
// CUDA-core brunet epilogues apply unchanged.  Every wait is bounded; a CTA
// that gives up records a timeout, lets its own loads and MMAs finish, frees
// its tensor memory and returns.
#pragma once

#include "tc.cuh"

namespace nmfcu {
namespace tcr {

constexpr int kM = 128;        // outputs per tile (TMEM lanes, MMA M)
constexpr int kU = 128;        // streamed elements per unit (one stream-K unit; MMA1's N)
constexpr int kC = 64;         // streamed elements per V ring slot (half a unit)
constexpr int kR = 32;         // padded rank: MMA1's K, MMA2's N per factor term
constexpr int kVStages = 4;    // V ring (half units): freed as soon as the ratio step has read V
constexpr int kFStages = 3;    // factor ring (units): freed when the unit's MMA2 is done
constexpr int kNB = 2;         // W H / Q buffers (units) in tensor memory
// Warp roles: V producer, factor producer, MMA1 issuer (and the tensor
// memory's owner), MMA2 issuer, then the epilogue warps.
constexpr int kVProdWarp = 0, kFProdWarp = 1, kMma1Warp = 2, kMma2Warp = 3, kEpiWarp0 = 4;
constexpr int kEpiWarps = 16;
constexpr int kParts = kEpiWarps / 4;       // epilogue warps per TMEM lane quarter
constexpr int kPartElems = kU / kParts;    // unit elements per epilogue warp (32)
constexpr int kPartRanks = kR / kParts;    // contraction ranks per epilogue warp
constexpr int kTWarps = 3;                 // warps of a lane quarter that write T
constexpr int kWarps = kEpiWarp0 + kEpiWarps;
constexpr int kThreads = kWarps * 32;
constexpr int kSegUnits = 16;  // units per segment: 2048 terms per f32 sum
static_assert(kPartElems == 32 && kVStages == 4,
              "a warp's share of a unit is two 16-element MMA2 K steps of one V slot");

// Tensor-memory columns.
constexpr int kTmemCols = 512;
constexpr uint32_t kQCols = kU;          // one W H / Q buffer
constexpr uint32_t kTOff = kNB * kQCols;  // T: three terms of 16 columns
constexpr uint32_t kTCols = 3 * (kR / 2);
constexpr uint32_t kD2Off = 320;          // two segment accumulators of 96 columns
constexpr uint32_t kD2Cols = 3 * kR;
static_assert(kTOff + kTCols <= kD2Off && kD2Off + 2 * kD2Cols <= (uint32_t)kTmemCols,
              "tensor memory budget");

// Shared memory, from a 1 KB-aligned base.
constexpr int V_BYTES = kC * kM * 4;      // half a unit of f32 V (one V ring slot)
// One factor term of a unit: 128 rows x 32 k, 64-B swizzle.  MMA1 reads it
// K-major (B = F, K = k); MMA2 reads the same tile MN-major (B[k][e], N = k
// along a row, K = e down the rows), the three terms one 32-wide N block
// apart.
constexpr int F1_TERM = kU * kR * 2;
constexpr int F_SLOT = 3 * F1_TERM;       // one factor ring slot: the three terms
constexpr int kFPieces = F_SLOT / 16;      // 16-byte copies a factor slot takes
constexpr int kFLag = 1;                   // factor slots in flight before one is announced
static_assert(kFPieces % 32 == 0 && kFLag < kFStages, "factor producer shape");
constexpr int OFF_F = kVStages * V_BYTES;
constexpr int OFF_BARS = OFF_F + kFStages * F_SLOT;
static_assert(V_BYTES % 1024 == 0 && F_SLOT % 1024 == 0 && OFF_F % 1024 == 0 &&
                  F1_TERM % 512 == 0,
              "swizzle atoms need their alignment");

struct Bars {
    uint64_t vfull[kVStages];   // V slot loaded (TMA bytes)
    uint64_t vempty[kVStages];  // V slot read (one arrival per epilogue warp that reads it)
    uint64_t ffull[kFStages];   // factor slot landed (one arrival by the factor producer)
    uint64_t fempty[kFStages];  // factor slot free (MMA2 of its unit done)
    uint64_t tfull, tempty;     // T written (T-writing warps) / free (last MMA1 of its tile done)
    uint64_t d1full[kNB];       // W H of buffer b written (MMA1 commit)
    uint64_t qfull[kNB];        // Q of buffer b written (one arrival per epilogue warp)
    uint64_t qempty[kNB];       // buffer b free again (MMA2 commit)
    uint64_t d2full[2], d2empty[2];  // a segment's contraction done / drained
    uint64_t drain[2];          // every MMA of an issuer done (abort path)
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

// MMA with A read from tensor memory (rows in lanes, two bf16 K elements a
// 32-bit column) and B from a shared-memory descriptor.
__device__ __forceinline__ void umma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b,
                                        uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

// 8 consecutive 32-bit columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7])
        : "r"(taddr));
}
// Writes 16 consecutive 32-bit columns of this thread's lane and waits until
// the writes are done.
__device__ __forceinline__ void tmem_st16_wait(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
        "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
        "r"(r[15])
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// 16-byte asynchronous copy global -> shared (L2 only), and its groups.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// 1 / y to about 1 ulp (approximate reciprocal, subnormals flushed).
__device__ __forceinline__ float rcp_approx(float y) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(y));
    return r;
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

// Slot and phase parity of a ring of N slots, advanced one use at a time.
template <int N>
struct RingPos {
    int slot = 0;
    uint32_t par = 0;
    __device__ __forceinline__ void next() {
        if (++slot == N) {
            slot = 0;
            par ^= 1u;
        }
    }
};

// Walks the valid units of a CTA's stream-K range in order (units past the
// streamed extent, which pad the last segment of a tile, are skipped).
struct ChunkWalker {
    UnitCursor cur;
    long long u, u1;
    bool ok;
    __device__ __forceinline__ void skip(const StreamK &sk, int kext) {
        while (u < u1 && (long long)cur.along(sk) * kU >= kext) {
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

// Position of one valid unit in its tile and segment.
struct ChunkInfo {
    int t, major, along;
    bool first_seg, last_seg, last_tile;
};

// The unit under `w`, given the tile-segment of the unit before it (-1 for
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

// HPASS: tile = 128 columns of V, unit = 128 rows; else tile = 128 rows,
// unit = 128 columns.
//   tmV   the f32 V: HPASS box {128, 64}, no swizzle; else box {32, 128},
//         128-B swizzle (two boxes a V slot)
//   xT    the tile factor's terms as [3][xpadT][32] bf16 (rows of 64 bytes)
//   xF    the unit factor's terms as [3][xpadF][32] bf16 (rows of 64 bytes)
//   kext  streamed extent (n for the H pass, p for the W pass)
template <bool HPASS>
__global__ void __launch_bounds__(kThreads, 1)
    tcr_pass(const __grid_constant__ CUtensorMap tmV, const __nv_bfloat16 *__restrict__ xT,
             const __nv_bfloat16 *__restrict__ xF,
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
            mbar_init(&bars.vempty[s], kEpiWarps / 2);
        }
        for (int s = 0; s < kFStages; s++) {
            mbar_init(&bars.ffull[s], 1);
            mbar_init(&bars.fempty[s], 1);
        }
        mbar_init(&bars.tfull, 4 * kTWarps);
        mbar_init(&bars.tempty, 1);
        for (int a = 0; a < kNB; a++) {
            mbar_init(&bars.d1full[a], 1);
            mbar_init(&bars.qfull[a], kEpiWarps);
            mbar_init(&bars.qempty[a], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&bars.d2full[a], 1);
            mbar_init(&bars.d2empty[a], kEpiWarps);
            mbar_init(&bars.drain[a], 1);
        }
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
        RingPos<kVStages / 2> ur;  // a unit takes V slots 2 slot and 2 slot + 1
        bool okv = true;
        while (okv && w.ok && !*abort_flag) {
            const int major = w.cur.major, along = w.cur.along(sk);
            for (int h = 0; h < 2; h++) {
                const int s = 2 * ur.slot + h;
                if (!mbar_sleep_wait(&bars.vempty[s], ur.par ^ 1u)) {
                    give_up();
                    okv = false;
                    break;
                }
                unsigned char *base = smem + s * V_BYTES;
                const int e0 = along * kU + h * kC;  // first streamed element of the slot
                mbar_expect_tx(&bars.vfull[s], V_BYTES);
                if (HPASS) {
                    tma_load_2d_hint(base, &tmV, &bars.vfull[s], major * kM, e0, pol_v);
                } else {
                    tma_load_2d_hint(base, &tmV, &bars.vfull[s], e0, major * kM, pol_v);
                    tma_load_2d_hint(base + V_BYTES / 2, &tmV, &bars.vfull[s], e0 + kC / 2,
                                     major * kM, pol_v);
                }
                issued[s]++;
            }
            ur.next();
            w.advance(sk, kext);
        }
        if (*abort_flag) {
            // Let this thread's own loads land before the CTA exits.
            for (int i = 0; i < kVStages; i++)
                if (issued[i] > 0) mbar_sleep_wait(&bars.vfull[i], (uint32_t)((issued[i] - 1) & 1));
        }
    } else if (warp == kFProdWarp) {
        // ---- producer of the unit factor terms (L2-resident) ----------------
        // Plain 16-byte asynchronous copies by the whole warp, not TMA: the
        // factor slot of a unit is needed by MMA1 long before its V, and TMA
        // copies would queue behind the V stream's.  Each lane copies 48 of
        // the slot's 1536 16-byte pieces into the 64-byte-swizzled layout the
        // MMAs read (16-byte piece j of row r at r * 64 + ((j ^ (r / 2 % 4))
        // * 16)).  A slot is announced once its copies have landed, kFLag
        // units later or before the warp would wait for a free slot: wait
        // for them, order them before the tensor cores' reads (proxy fence),
        // then one arrival.
        ChunkWalker w;
        w.init(sk, u0, u1, kext);
        RingPos<kFStages> fr, sig;
        int unsig = 0;
        auto announce = [&]() {
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars.ffull[sig.slot]);
            sig.next();
            --unsig;
        };
        while (w.ok && !*abort_flag) {
            const int along = w.cur.along(sk);
            // Never hold landed-but-unannounced slots while waiting for a
            // free one: MMA1 may need them to make progress.
            if (unsig > 0 &&
                !__all_sync(0xffffffffu, mbar_try_wait(&bars.fempty[fr.slot], fr.par ^ 1u))) {
                cp_async_wait<0>();
                while (unsig > 0) announce();
            }
            if (!warp_wait(&bars.fempty[fr.slot], fr.par ^ 1u)) {
                if (lane == 0) give_up();
                break;
            }
            const uint32_t dst0 = smem_u32(smem + OFF_F + fr.slot * F_SLOT);
#pragma unroll
            for (int i = 0; i < kFPieces / 32; i++) {
                const int k = lane + 32 * i;
                const int t = k / (kU * 4), r = (k >> 2) & (kU - 1), j = k & 3;
                const __nv_bfloat16 *src =
                    xF + (((size_t)t * xpadF + (size_t)along * kU + r) * kR + j * 8);
                cp_async16(dst0 + (uint32_t)(t * F1_TERM + r * 64 + ((j ^ ((r >> 1) & 3)) << 4)),
                           src);
            }
            cp_async_commit();
            fr.next();
            ++unsig;
            if (unsig > kFLag) {
                cp_async_wait<kFLag>();
                announce();
            }
            w.advance(sk, kext);
        }
        // The remaining slots (or, after a give-up, only this warp's own
        // copies) land before the CTA exits.
        cp_async_wait<0>();
        while (unsig > 0 && !*abort_flag) announce();
    } else if ((warp == kMma1Warp || warp == kMma2Warp) && lane == 0) {
        // ---- MMA issuers ------------------------------------------------------
        // MMA1 (W H of a unit) runs ahead, held back only by free buffers,
        // the tile's T and landed factor terms; MMA2 (the contraction)
        // follows the ratio step.  Each commit covers its own thread's MMAs.
        constexpr uint32_t id128 = tc::instr_desc<kU, false>();
        constexpr uint32_t id96m = instr_desc_bmn<96>();  // MMA2: B = F MN-major
        constexpr uint32_t id64m = instr_desc_bmn<64>();
        const uint32_t sbase = smem_u32(smem);
        const bool first = (warp == kMma1Warp);
        ChunkWalker w;
        w.init(sk, u0, u1, kext);
        long long ci = 0;
        RingPos<kFStages> fr;
        RingPos<kNB> qr, qlast;
        int tiles = 0, segs = 0, prev_t = -1, prev_major = -1;
        bool ok = true;
        while (w.ok && !*abort_flag) {
            const ChunkInfo c = take(w, sk, kext, prev_t);
            prev_t = c.t;
            const int s = fr.slot;
            const int qb = qr.slot;
            const uint32_t qpar = qr.par;
            const uint32_t fB = sbase + OFF_F + s * F_SLOT;
            const uint32_t qcol = tmem + (uint32_t)qb * kQCols;
            if (first) {
                // MMA1 of unit ci into buffer qb (N = the unit's 128 elements).
                if (!mbar_sleep_wait(&bars.ffull[s], fr.par)) {
                    ok = false;
                    break;
                }
                if (c.major != prev_major) {
                    if (!mbar_sleep_wait(&bars.tfull, (uint32_t)(tiles & 1))) {
                        ok = false;
                        break;
                    }
                    ++tiles;
                    prev_major = c.major;
                }
                if (!mbar_sleep_wait(&bars.qempty[qb], qpar ^ 1u)) {
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                // Products (T term, F term): hh, hm, hl, mh, mm, lh; two K
                // steps of 16 ranks each.
                constexpr int ta[6] = {0, 0, 0, 1, 1, 2};
                constexpr int fa[6] = {0, 1, 2, 0, 1, 0};
#pragma unroll
                for (int pr = 0; pr < 6; pr++) {
#pragma unroll
                    for (int ks = 0; ks < kR / 16; ks++) {
                        const uint32_t a =
                            tmem + kTOff + (uint32_t)(ta[pr] * (kR / 2) + ks * 8);
                        const uint64_t bdesc =
                            desc_sw64(fB + (uint32_t)(fa[pr] * F1_TERM) + (uint32_t)ks * 32u);
                        umma_ts(qcol, a, bdesc, id128, (pr > 0 || ks > 0) ? 1u : 0u);
                    }
                }
                tc::umma_commit(&bars.d1full[qb]);
                if (c.last_tile) tc::umma_commit(&bars.tempty);
            } else {
                // MMA2 of unit ci into segment accumulator segs & 1.  The
                // factor slot landed before MMA1 of this unit, which the
                // ratio step waited for.
                const int x = segs & 1;
                if (c.first_seg &&
                    !mbar_sleep_wait(&bars.d2empty[x], (uint32_t)(((segs >> 1) & 1) ^ 1))) {
                    ok = false;
                    break;
                }
                if (!mbar_sleep_wait(&bars.qfull[qb], qpar)) {
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t d2 = tmem + kD2Off + (uint32_t)x * kD2Cols;
#pragma unroll
                for (int ks = 0; ks < kU / 16; ks++) {
                    // K step: unit elements 16 ks .. +15; 16 rows (1 KB) down F.
                    const uint64_t bdesc = desc_sw64_mn(fB + (uint32_t)ks * 1024u, F1_TERM);
                    umma_ts(d2, qcol + (uint32_t)ks * 16u, bdesc, id96m,
                            (c.first_seg && ks == 0) ? 0u : 1u);
                    umma_ts(d2, qcol + (uint32_t)ks * 16u + 8u, bdesc, id64m, 1u);
                }
                tc::umma_commit(&bars.qempty[qb]);
                tc::umma_commit(&bars.fempty[s]);
                if (c.last_seg) {
                    tc::umma_commit(&bars.d2full[x]);
                    ++segs;
                }
            }
            qlast = qr;
            fr.next();
            qr.next();
            ++ci;
        }
        if (!ok) give_up();
        if (!*abort_flag && ci > 0) {
            // The arrivals of this thread's last commits land before the CTA
            // exits.
            if (first) {
                mbar_sleep_wait(&bars.d1full[qlast.slot], qlast.par);
                if (tiles > 0) mbar_sleep_wait(&bars.tempty, (uint32_t)((tiles - 1) & 1));
            } else {
                mbar_sleep_wait(&bars.qempty[qlast.slot], qlast.par);
            }
        }
        if (*abort_flag) {
            uint64_t *dr = first ? &bars.drain[0] : &bars.drain[1];
            tc::umma_commit(dr);
            mbar_sleep_wait(dr, 0);
        }
    } else if (warp >= kEpiWarp0) {
        // ---- epilogue: W H -> Q in place, T, and the contraction -> partials
        const int q = warp & 3;                  // lane quarter this warp may access
        const int pw = (warp - kEpiWarp0) >> 2;  // its share of the unit / the ranks
        const int e0 = pw * kPartElems;          // first unit element of this warp
        const int vh = e0 / kC;                  // the unit's V slot (half) it reads
        const int ev = e0 - vh * kC;             // first element within that slot
        const int o = q * 32 + lane;             // output (TMEM lane) within the tile
        const uint32_t lane_off = (uint32_t)(q * 32) << 16;
        // This quarter's rows of T for the tile `major` (warps pw < 3, one
        // term each), after the last MMA1 of the previous tile.
        auto write_t = [&](int major, int tiles_done) -> bool {
            if (pw >= kTWarps) return true;
            if (tiles_done > 0 && !warp_wait(&bars.tempty, (uint32_t)((tiles_done - 1) & 1)))
                return false;
            tc::tc_fence_after();
            const uint4 *src = reinterpret_cast<const uint4 *>(
                xT + ((size_t)pw * xpadT + (size_t)major * kM + o) * kR);
            uint32_t r[16];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint4 x = __ldg(src + i);
                r[4 * i] = x.x;
                r[4 * i + 1] = x.y;
                r[4 * i + 2] = x.z;
                r[4 * i + 3] = x.w;
            }
            tmem_st16_wait(tmem + lane_off + kTOff + (uint32_t)(pw * (kR / 2)), r);
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars.tfull);
            return true;
        };
        ChunkWalker w;
        w.init(sk, u0, u1, kext);
        const int major0 = (int)(u0 / sk.major_units());
        RingPos<kVStages / 2> ur;
        RingPos<kNB> qr;
        int segs = 0, tiles = 0, prev_t = -1;
        // A finished segment waiting to be drained (one unit late).
        bool pend = false, pend_last_tile = false;
        int pend_x = 0, pend_major = 0;
        uint32_t pend_par = 0;
        double sum[kPartRanks];
#pragma unroll
        for (int i = 0; i < kPartRanks; i++) sum[i] = 0.0;
        auto drain = [&]() -> bool {
            if (!warp_wait(&bars.d2full[pend_x], pend_par)) return false;
            tc::tc_fence_after();
            // Ranks pw * 8 .. +7 of the three groups (the products with Fh,
            // Fm, Fl); their sum is the contraction.
            uint32_t x0[8], x1[8], x2[8];
            const uint32_t ta = tmem + lane_off + kD2Off + (uint32_t)pend_x * kD2Cols +
                                (uint32_t)(pw * kPartRanks);
            tmem_ld8(ta, x0);
            tmem_ld8(ta + kR, x1);
            tmem_ld8(ta + 2 * kR, x2);
            tc::tmem_wait_ld();
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars.d2empty[pend_x]);
#pragma unroll
            for (int i = 0; i < kPartRanks; i++)
                sum[i] += (double)(__uint_as_float(x0[i]) + __uint_as_float(x1[i]) +
                                   __uint_as_float(x2[i]));
            if (pend_last_tile) {
                double *dst = part + ((size_t)b * sk.slots + (size_t)(pend_major - major0)) *
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
            pend = false;
            return true;
        };
        bool ok = true;
        if (w.ok) {
            ok = write_t(w.cur.major, 0);
            tiles = 1;
        }
        while (ok && w.ok && !*abort_flag) {
            const ChunkInfo c = take(w, sk, kext, prev_t);
            prev_t = c.t;
            const int s = 2 * ur.slot + vh;
            const int qb = qr.slot;
            const uint32_t qpar = qr.par;
            // V first: its slot is refilled as soon as the eight warps that
            // read it are done.
            if (!warp_wait(&bars.vfull[s], ur.par)) {
                ok = false;
                break;
            }
            const unsigned char *vs = smem + s * V_BYTES;
            // This warp's 32 elements, 16 at a time: V, W H from tensor
            // memory, Q written over it.  The V slot is released after the
            // second group's read, W H is awaited before the first group's.
#pragma unroll 1
            for (int g = 0; g < kPartElems / 16; g++) {
                float v[16];
                if (HPASS) {
                    const float *vf = reinterpret_cast<const float *>(vs);
#pragma unroll
                    for (int i = 0; i < 16; i++) v[i] = vf[(ev + 16 * g + i) * kM + o];
                } else {
                    // Box ev / 32 holds columns (ev / 32) * 32 .. +31 of rows
                    // 0..127, 16-byte chunk ch of row o at (ch ^ (o & 7)).
                    const unsigned char *row = vs + (ev >> 5) * (V_BYTES / 2) + o * 128;
#pragma unroll
                    for (int c4 = 0; c4 < 4; c4++) {
                        const int ch = 4 * g + c4;
                        const float4 x =
                            *reinterpret_cast<const float4 *>(row + ((ch ^ (o & 7)) << 4));
                        v[4 * c4] = x.x;
                        v[4 * c4 + 1] = x.y;
                        v[4 * c4 + 2] = x.z;
                        v[4 * c4 + 3] = x.w;
                    }
                }
                if (g == kPartElems / 16 - 1) {
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&bars.vempty[s]);
                }
                if (g == 0) {
                    if (!warp_wait(&bars.d1full[qb], qpar)) {
                        ok = false;
                        break;
                    }
                    tc::tc_fence_after();
                }
                const uint32_t ta =
                    tmem + lane_off + (uint32_t)qb * kQCols + (uint32_t)(e0 + 16 * g);
                float wh[16];
                tc::tmem_ld16(ta, wh);
                tc::tmem_wait_ld();
                uint32_t qp[16];  // [0, 8): hi pairs, [8, 16): lo pairs
#pragma unroll
                for (int i = 0; i < 16; i += 2) {
                    // q = v / wh as v times an approximate reciprocal (two
                    // elements a packed multiply), 0 where wh is 0.
                    float2 qv = __fmul2_rn(make_float2(v[i], v[i + 1]),
                                           make_float2(rcp_approx(wh[i]), rcp_approx(wh[i + 1])));
                    qv.x = (wh[i] != 0.f) ? qv.x : 0.f;
                    qv.y = (wh[i + 1] != 0.f) ? qv.y : 0.f;
                    const __nv_bfloat162 hi = __float22bfloat162_rn(qv);
                    const uint32_t hb = *reinterpret_cast<const uint32_t *>(&hi);
                    const float2 hf = make_float2(__uint_as_float(hb << 16),
                                                  __uint_as_float(hb & 0xffff0000u));
                    // lo = bf16(q - hi); q - hi is exact in f32.
                    const __nv_bfloat162 lo =
                        __float22bfloat162_rn(__ffma2_rn(hf, make_float2(-1.f, -1.f), qv));
                    qp[i / 2] = hb;
                    qp[8 + i / 2] = *reinterpret_cast<const uint32_t *>(&lo);
                }
                tmem_st16_wait(ta, qp);
            }
            if (!ok) break;
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars.qfull[qb]);
            // The segment finished one unit ago (its MMA2 has had this
            // unit's ratio step to complete).
            if (pend && !drain()) {
                ok = false;
                break;
            }
            if (c.last_seg) {
                pend = true;
                pend_x = segs & 1;
                pend_par = (uint32_t)((segs >> 1) & 1);
                pend_last_tile = c.last_tile;
                pend_major = c.major;
                ++segs;
            }
            // The next tile's T, once the last MMA1 of this one is done.
            if (c.last_tile && w.ok) {
                if (!write_t(w.cur.major, tiles)) {
                    ok = false;
                    break;
                }
                ++tiles;
            }
            ur.next();
            qr.next();
        }
        if (ok && pend && !*abort_flag && !drain()) ok = false;
        if (!ok) give_up();
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

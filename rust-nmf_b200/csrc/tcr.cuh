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
// A tcgen05 MMA (M = 128, K = 16) takes about 125 cycles of tensor-pipe
// time for any N up to 128 (measured), so the pass is shaped to issue few,
// wide MMAs: a 128-element unit makes MMA1 N = 128, and the six term
// products are concatenated along K (ceil(6 r / 16) MMAs a unit: 8 at rank
// 20, not 6 x 2); MMA2 is 8 K steps x 2 (Qh, Ql) with N = round16(3 r).
//
// Tensor memory carries everything that is not streamed, so shared memory
// holds only the two TMA rings (V, and the unit factor rows):
//   * T, the tile operand of MMA1, sits in tensor memory for the whole tile
//     (MMA1 reads A from tensor memory) in the tile layout.
//   * MMA1 sums the six term products into ONE 128-column accumulator per
//     unit, so the ratio step reads one value an element.
//   * The ratio step writes Q back over the W H it has just read, as bf16
//     pairs: for unit elements 16g .. 16g + 15 the hi terms fill columns
//     16g .. 16g + 7 and the lo terms 16g + 8 .. 16g + 15 of the same
//     buffer, and MMA2 reads them as its A operand (K step g: Qh at 16g, Ql
//     at 16g + 8).  Each epilogue warp reads and rewrites only its own 32
//     columns.  MMA2 contracts Qh [Fh; Fm; Fl] + Ql [Fh; Fm; Fl] (B = the
//     unit rows read MN-major) into a segment accumulator whose columns k,
//     r + k, 2 r + k hold rank k's three terms.
//   * Two W H / Q buffers (a buffer is freed by the MMA2 that read its Q);
//     two segment accumulators at ranks up to 21 (drained one unit late, so
//     MMA2 of the next segment does not wait on the drain), one above.
//
// One CTA per SM, twenty warps: warp 0 loads V by TMA into a ring of
// half-unit slots (a slot is refilled as soon as the ratio step has read
// it), warp 1 loads the unit factor rows by TMA into a ring of their own,
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
constexpr int kMaxRank = 32;
constexpr int kVStages = 4;    // V ring (half units): freed as soon as the ratio step has read V
// Warp roles: V producer, factor producer, MMA1 issuer (and the tensor
// memory's owner), MMA2 issuer, then the epilogue warps.
constexpr int kVProdWarp = 0, kFProdWarp = 1, kMma1Warp = 2, kMma2Warp = 3, kEpiWarp0 = 4;
constexpr int kEpiWarps = 16;
constexpr int kParts = kEpiWarps / 4;          // epilogue warps per TMEM lane quarter
constexpr int kPartElems = kU / kParts;       // unit elements per epilogue warp (32)
constexpr int kPartRanks = kMaxRank / kParts;  // contraction ranks per epilogue warp
constexpr int kWarps = kEpiWarp0 + kEpiWarps;
constexpr int kThreads = kWarps * 32;
constexpr int kSegUnits = 16;  // units per segment: 2048 terms per f32 sum
static_assert(kPartElems == 32 && kVStages == 4,
              "a warp's share of a unit is two 16-element MMA2 K steps of one V slot");
constexpr int kTmemCols = 512;
constexpr int V_BYTES = kC * kM * 4;  // half a unit of f32 V (one V ring slot)
constexpr int kKBlock = 16384;        // one 64-element K block of a factor slot (128 rows x 128 B)

// The shape of the pass for a padded concatenated rank KC (128: rank <= 21,
// 192: rank <= 32).  A factor row in the pass's two layouts holds six
// blocks of `rank` bf16 each, zero-padded to KC:
//   tile layout  [Th Th Th Tm Tm Tl]   (MMA1's A, in tensor memory)
//   unit layout  [Fh Fm Fl Fh Fm Fh]   (MMA1's B and MMA2's B, in shared memory)
// so MMA1 adds the six products Th Fh, Th Fm, Th Fl, Tm Fh, Tm Fm, Tl Fh in
// ceil(6 rank / 16) K steps into one accumulator, and the first three
// blocks of the unit layout are [Fh; Fm; Fl] along MMA2's N.
template <int KC>
struct Cfg {
    static_assert(KC == 128 || KC == 192, "concatenated rank");
    static constexpr int kFStages = KC == 128 ? 3 : 2;  // factor ring (units)
    static constexpr int kNB = 2;                       // W H / Q buffers (units)
    static constexpr int kD2Buf = KC == 128 ? 2 : 1;    // segment accumulators
    static constexpr int kN2Max = KC == 128 ? 64 : 96;  // MMA2's N: round16(3 rank)
    // Tensor-memory columns: W H / Q buffers, then T, then the segment
    // accumulators.
    static constexpr uint32_t kQCols = kU;
    static constexpr uint32_t kTOff = kNB * kQCols;
    static constexpr uint32_t kTCols = KC / 2;
    static constexpr uint32_t kD2Off = kTOff + kTCols;
    static constexpr uint32_t kD2Cols = kN2Max;
    static_assert(kD2Off + kD2Buf * kD2Cols <= (uint32_t)kTmemCols, "tensor memory budget");
    // Shared memory, from a 1 KB-aligned base: the V ring, the factor ring
    // (a unit's rows in the unit layout, 128-B swizzle, K blocks of 64).
    static constexpr int F_SLOT = (KC / 64) * kKBlock;
    static constexpr int OFF_F = kVStages * V_BYTES;
    static constexpr int OFF_BARS = OFF_F + kFStages * F_SLOT;
    struct Bars {
        uint64_t vfull[kVStages];   // V slot loaded (TMA bytes)
        uint64_t vempty[kVStages];  // V slot read (one arrival per epilogue warp that reads it)
        uint64_t ffull[kFStages];   // factor slot loaded (TMA bytes)
        uint64_t fempty[kFStages];  // factor slot free (MMA2 of its unit done)
        uint64_t tfull, tempty;     // T written (epilogue warps) / free (last MMA1 of its tile done)
        uint64_t d1full[kNB];       // W H of buffer b written (MMA1 commit)
        uint64_t qfull[kNB];        // Q of buffer b written (one arrival per epilogue warp)
        uint64_t qempty[kNB];       // buffer b free again (MMA2 commit)
        uint64_t d2full[kD2Buf], d2empty[kD2Buf];  // a segment's contraction done / drained
        uint64_t drain[2];          // every MMA of an issuer done (abort path)
        uint32_t tmem_base;
        int abort;
    };
    static constexpr int SMEM = OFF_BARS + (int)sizeof(Bars) + 1024;  // + alignment slack
    static_assert(SMEM <= 232448, "shared memory per CTA");
    static_assert(V_BYTES % 1024 == 0 && F_SLOT % 1024 == 0 && OFF_F % 1024 == 0,
                  "swizzle atoms need their alignment");
};

// Instruction descriptor as tc::instr_desc, for a run-time N, with B read
// MN-major when `b_mn`.
__device__ __forceinline__ uint32_t instr_desc_rt(int n, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (b_mn ? (1u << 16) : 0u) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
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

// One 32-bit column of this thread's tensor-memory lane.
__device__ __forceinline__ uint32_t tmem_ld1(uint32_t taddr) {
    uint32_t r;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
    return r;
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
//   xT    the tile factor's rows in the tile layout (KC bf16 a row)
//   tmF   the unit factor's rows in the unit layout, box {64, 128}, 128-B swizzle
//   kext  streamed extent (n for the H pass, p for the W pass)
template <bool HPASS, int KC>
__global__ void __launch_bounds__(kThreads, 1)
    tcr_pass(const __grid_constant__ CUtensorMap tmV, const __nv_bfloat16 *__restrict__ xT,
             const __grid_constant__ CUtensorMap tmF, int kext, int rank,
             int RP, StreamK sk, double *__restrict__ part, RunState *st) {
    using C = Cfg<KC>;
    constexpr int kFStages = C::kFStages, kNB = C::kNB, kD2Buf = C::kD2Buf;
    extern __shared__ unsigned char tcr_smem_raw[];
    if (run_stopped(st)) return;
    const uint32_t raw = smem_u32(tcr_smem_raw);
    unsigned char *smem = tcr_smem_raw + ((1024 - (raw & 1023)) & 1023);
    typename C::Bars &bars = *reinterpret_cast<typename C::Bars *>(smem + C::OFF_BARS);
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
        mbar_init(&bars.tfull, kEpiWarps);
        mbar_init(&bars.tempty, 1);
        for (int a = 0; a < kNB; a++) {
            mbar_init(&bars.d1full[a], 1);
            mbar_init(&bars.qfull[a], kEpiWarps);
            mbar_init(&bars.qempty[a], 1);
        }
        for (int a = 0; a < kD2Buf; a++) {
            mbar_init(&bars.d2full[a], 1);
            mbar_init(&bars.d2empty[a], kEpiWarps);
        }
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
    } else if (warp == kFProdWarp && lane == 0) {
        // ---- TMA producer of the unit factor terms (L2-resident) ------------
        // The unit layout's rows along * 128 .. +127, one 64-column box (a K
        // block, 128-B swizzle) at a time.
        const uint64_t pol_f = l2_evict_last_policy();
        ChunkWalker w;
        w.init(sk, u0, u1, kext);
        RingPos<kFStages> fr;
        int issued[kFStages] = {0};
        while (w.ok && !*abort_flag) {
            const int along = w.cur.along(sk);
            if (!mbar_sleep_wait(&bars.fempty[fr.slot], fr.par ^ 1u)) {
                give_up();
                break;
            }
            unsigned char *base = smem + C::OFF_F + fr.slot * C::F_SLOT;
            mbar_expect_tx(&bars.ffull[fr.slot], C::F_SLOT);
            for (int kb = 0; kb < KC / 64; kb++)
                tma_load_2d_hint(base + kb * kKBlock, &tmF, &bars.ffull[fr.slot], kb * 64,
                                 along * kU, pol_f);
            issued[fr.slot]++;
            fr.next();
            w.advance(sk, kext);
        }
        if (*abort_flag) {
            // Let this thread's own loads land before the CTA exits.
            for (int i = 0; i < kFStages; i++)
                if (issued[i] > 0) mbar_sleep_wait(&bars.ffull[i], (uint32_t)((issued[i] - 1) & 1));
        }
    } else if ((warp == kMma1Warp || warp == kMma2Warp) && lane == 0) {
        // ---- MMA issuers ------------------------------------------------------
        // MMA1 (W H of a unit) runs ahead, held back only by free buffers,
        // the tile's T and landed factor terms; MMA2 (the contraction)
        // follows the ratio step.  Each commit covers its own thread's MMAs.
        constexpr uint32_t id128 = tc::instr_desc<kU, false>();
        const int nks1 = (6 * rank + 15) / 16;          // MMA1's K steps
        const int n2 = (3 * rank + 15) / 16 * 16;       // MMA2's N: [Fh; Fm; Fl]
        const uint32_t id2 = instr_desc_rt(n2, true);  // MMA2: B = F MN-major
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
            const uint32_t fB = sbase + C::OFF_F + s * C::F_SLOT;
            const uint32_t qcol = tmem + (uint32_t)qb * C::kQCols;
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
                // The six term products, concatenated along K: K step ks
                // reads T columns 8 ks .. +7 and the unit rows' elements
                // 16 ks .. +15 (K block ks / 4, 32 bytes a step within it).
                for (int ks = 0; ks < nks1; ks++) {
                    const uint64_t bdesc = tc::smem_desc(
                        fB + (uint32_t)((ks >> 2) * kKBlock + (ks & 3) * 32), 16, 1024);
                    umma_ts(qcol, tmem + C::kTOff + (uint32_t)(ks * 8), bdesc, id128,
                            ks > 0 ? 1u : 0u);
                }
                tc::umma_commit(&bars.d1full[qb]);
                if (c.last_tile) tc::umma_commit(&bars.tempty);
            } else {
                // MMA2 of unit ci into segment accumulator segs % kD2Buf.
                // The factor slot landed before MMA1 of this unit, which
                // the ratio step waited for.
                const int x = segs % kD2Buf;
                if (c.first_seg &&
                    !mbar_sleep_wait(&bars.d2empty[x], (uint32_t)(((segs / kD2Buf) & 1) ^ 1))) {
                    ok = false;
                    break;
                }
                if (!mbar_sleep_wait(&bars.qfull[qb], qpar)) {
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t d2 = tmem + C::kD2Off + (uint32_t)x * C::kD2Cols;
#pragma unroll
                for (int ks = 0; ks < kU / 16; ks++) {
                    // K step: unit elements 16 ks .. +15, 16 rows (2 KB) down
                    // the unit rows read MN-major (N blocks of 64 elements one
                    // K block apart).
                    const uint64_t bdesc = tc::smem_desc(fB + (uint32_t)ks * 2048u, kKBlock, 1024);
                    umma_ts(d2, qcol + (uint32_t)ks * 16u, bdesc, id2,
                            (c.first_seg && ks == 0) ? 0u : 1u);
                    umma_ts(d2, qcol + (uint32_t)ks * 16u + 8u, bdesc, id2, 1u);
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
        // This quarter's rows of T for the tile `major` (the tile layout, KC
        // bf16 a row: 16-column pieces pw, pw + 4, ...), after the last MMA1
        // of the previous tile.
        auto write_t = [&](int major, int tiles_done) -> bool {
            if (tiles_done > 0 && !warp_wait(&bars.tempty, (uint32_t)((tiles_done - 1) & 1)))
                return false;
            tc::tc_fence_after();
            for (int piece = pw; piece < KC / 32; piece += kParts) {
                const uint4 *src = reinterpret_cast<const uint4 *>(
                    xT + ((size_t)major * kM + o) * KC + piece * 32);
                uint32_t r[16];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const uint4 x = __ldg(src + i);
                    r[4 * i] = x.x;
                    r[4 * i + 1] = x.y;
                    r[4 * i + 2] = x.z;
                    r[4 * i + 3] = x.w;
                }
                tmem_st16_wait(tmem + lane_off + C::kTOff + (uint32_t)(piece * 16), r);
            }
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
            // Ranks pw * 8 .. +7: columns k, rank + k and 2 rank + k hold
            // the products with Fh, Fm and Fl; their sum is the contraction.
            float xs[kPartRanks];
            const uint32_t ta = tmem + lane_off + C::kD2Off + (uint32_t)pend_x * C::kD2Cols;
#pragma unroll
            for (int i = 0; i < kPartRanks; i++) {
                const int k = pw * kPartRanks + i;
                xs[i] = 0.f;
                if (k < rank) {  // the same for the whole warp
                    const uint32_t a0 = tmem_ld1(ta + (uint32_t)k);
                    const uint32_t a1 = tmem_ld1(ta + (uint32_t)(rank + k));
                    const uint32_t a2 = tmem_ld1(ta + (uint32_t)(2 * rank + k));
                    tc::tmem_wait_ld();
                    xs[i] = __uint_as_float(a0) + __uint_as_float(a1) + __uint_as_float(a2);
                }
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars.d2empty[pend_x]);
#pragma unroll
            for (int i = 0; i < kPartRanks; i++) sum[i] += (double)xs[i];
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
                    tmem + lane_off + (uint32_t)qb * C::kQCols + (uint32_t)(e0 + 16 * g);
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
                pend_x = segs % kD2Buf;
                pend_par = (uint32_t)((segs / kD2Buf) & 1);
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

}  // namespace tcr
}  // namespace nmfcu

// tcr.cuh -- brunet's two V passes on the tensor cores (tcgen05), for the
// split-bf16 precision form.
//
// The KL multiplicative update contracts the element-wise ratio V / (W H)
// with a factor (rust/src/lib.rs:1474-1519, the brunet H and W updates):
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
//   MMA2  N[o][k] += sum_e Q[o][e] F[e][k]      accumulated over a segment
// so W H is never written out.  V is read once, as f32 (4 bytes an element);
// the factors are L2-resident.  Factor operands are three bf16 terms each
// (Fh + Fm + Fl ~ F to about 2^-24); MMA1 keeps the six products down to
// 2^-16 x 2^-8 (Th[Fh;Fm;Fl], Tm[Fh;Fm], Tl Fh as N = 192 / 128 / 64 into
// one accumulator of three column groups), MMA2 the five of the split-bf16
// lee passes (Qh [Fh;Fm;Fl] + Ql [Fh;Fm], N = 96 / 64).
//
// One CTA per SM, ten warps: warp 0 issues the TMA loads, warp 1 owns the
// tensor memory and issues the MMAs (one thread; MMA1 of the next chunk is
// issued before MMA2 of the current one, so the ratio overlaps the tensor
// pipe), warps 2..9 read WH from tensor memory, form Q and drain the
// contraction: warp w reads TMEM lanes 32 (w mod 4) .. +31, and the two
// warps of a lane quarter split the chunk's 64 elements.  Tensor memory:
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
constexpr int kStages = 3;
constexpr int kEpiWarps = 8;
constexpr int kWarps = 2 + kEpiWarps;
constexpr int kThreads = kWarps * 32;
constexpr int kSegUnits = 32;  // chunks per segment: 2048 terms per f32 sum
constexpr int kTmemCols = 512;
constexpr uint32_t kD1 = 0;    // WH accumulators at columns 0 and 192
constexpr uint32_t kD1Cols = 192;
constexpr uint32_t kD2 = 384;  // contraction accumulator (96 columns)

// Shared memory, from a 1 KB-aligned base.
constexpr int V_BYTES = kC * kM * 4;      // the f32 V chunk
constexpr int F1_TERM = kC * kR * 2;      // MMA1's B term: 64 rows x 32 k, 64-B swizzle
constexpr int F2_TERM = kR * kC * 2;      // MMA2's B term: 32 k x 64, 128-B swizzle
constexpr int OFF_F1 = V_BYTES;
constexpr int OFF_F2 = OFF_F1 + 3 * F1_TERM;
constexpr int STAGE = OFF_F2 + 3 * F2_TERM;   // 56 KB
constexpr int T_TERM = kM * kR * 2;       // MMA1's A term: 128 rows x 32 k, 64-B swizzle
constexpr int Q_PLANE = kM * kC * 2;      // Q hi or lo: 128 x 64, 128-B swizzle
constexpr int OFF_T = kStages * STAGE;
constexpr int OFF_Q = OFF_T + 3 * T_TERM;
constexpr int OFF_BARS = OFF_Q + 2 * Q_PLANE;
static_assert(STAGE % 1024 == 0 && OFF_F2 % 1024 == 0 && T_TERM % 1024 == 0 &&
                  Q_PLANE % 1024 == 0 && F1_TERM % 512 == 0,
              "swizzle atoms need their alignment");

struct Bars {
    uint64_t full[kStages];   // stage loaded (TMA bytes)
    uint64_t empty[kStages];  // stage free (MMA2 of its chunk done)
    uint64_t tfull, tempty;   // the tile operand loaded / free (last MMA1 of its tile done)
    uint64_t d1full[2];       // WH accumulator b written (MMA1 commit)
    uint64_t d1empty[2];      // WH accumulator b read (256 epilogue arrivals)
    uint64_t qfull, qempty;   // Q written (256 arrivals) / read (MMA2 commit)
    uint64_t d2full, d2empty; // a segment's contraction done / drained (256 arrivals)
    uint64_t drain;           // every MMA of this CTA done (abort path)
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
// K-major, 128-byte swizzle (rows of 64 bf16): 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr) {
    return tc::smem_desc(addr, 16, 1024);
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
//   tmF2  the chunk factor's terms as [3][32][ld] bf16, box {64, 32}, 128-B swizzle
//   kext  streamed extent (n for the H pass, p for the W pass)
template <bool HPASS>
__global__ void __launch_bounds__(kThreads, 1)
    tcr_pass(const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmT,
             const __grid_constant__ CUtensorMap tmF1, const __grid_constant__ CUtensorMap tmF2,
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
        for (int s = 0; s < kStages; s++) {
            mbar_init(&bars.full[s], 1);
            mbar_init(&bars.empty[s], 1);
        }
        mbar_init(&bars.tfull, 1);
        mbar_init(&bars.tempty, 1);
        for (int a = 0; a < 2; a++) {
            mbar_init(&bars.d1full[a], 1);
            mbar_init(&bars.d1empty[a], kEpiWarps * 32);
        }
        mbar_init(&bars.qfull, kEpiWarps * 32);
        mbar_init(&bars.qempty, 1);
        mbar_init(&bars.d2full, 1);
        mbar_init(&bars.d2empty, kEpiWarps * 32);
        mbar_init(&bars.drain, 1);
        bars.abort = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
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

    if (warp == 0 && lane == 0) {
        // ---- TMA producer -------------------------------------------------
        const uint64_t pol_v = l2_evict_first_policy(), pol_f = l2_evict_last_policy();
        ChunkWalker w;
        w.init(sk, u0, u1, kext);
        int issued[kStages] = {0};
        int tloads = 0, cur_major = -1;
        long long ci = 0;
        while (w.ok && !*abort_flag) {
            const int major = w.cur.major, along = w.cur.along(sk);
            if (major != cur_major) {
                // The tile operand is reloaded once the last MMA1 of the
                // previous tile has read it.
                if (tloads > 0 && !mbar_wait(&bars.tempty, (uint32_t)((tloads - 1) & 1))) {
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
            const int s = (int)(ci % kStages);
            if (!mbar_wait(&bars.empty[s], (uint32_t)(((ci / kStages) & 1) ^ 1))) {
                give_up();
                break;
            }
            unsigned char *base = smem + s * STAGE;
            mbar_expect_tx(&bars.full[s], STAGE);
            if (HPASS) {
                tma_load_2d_hint(base, &tmV, &bars.full[s], major * kM, along * kC, pol_v);
            } else {
                tma_load_2d_hint(base, &tmV, &bars.full[s], along * kC, major * kM, pol_v);
                tma_load_2d_hint(base + V_BYTES / 2, &tmV, &bars.full[s], along * kC + kC / 2,
                                 major * kM, pol_v);
            }
            for (int q = 0; q < 3; q++) {
                tma_load_2d_hint(base + OFF_F1 + q * F1_TERM, &tmF1, &bars.full[s], 0,
                                 q * xpadF + along * kC, pol_f);
                tma_load_2d_hint(base + OFF_F2 + q * F2_TERM, &tmF2, &bars.full[s], along * kC,
                                 q * kR, pol_f);
            }
            issued[s]++;
            ++ci;
            w.advance(sk, kext);
        }
        if (*abort_flag) {
            // Let this CTA's own loads land before the CTA exits.
            for (int i = 0; i < kStages; i++)
                if (issued[i] > 0) mbar_wait(&bars.full[i], (uint32_t)((issued[i] - 1) & 1));
            if (tloads > 0) mbar_wait(&bars.tfull, (uint32_t)((tloads - 1) & 1));
        }
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer -----------------------------------------------------
        constexpr uint32_t id192 = tc::instr_desc<192, false>();
        constexpr uint32_t id128 = tc::instr_desc<128, false>();
        constexpr uint32_t id96 = tc::instr_desc<96, false>();
        constexpr uint32_t id64 = tc::instr_desc<64, false>();
        const uint32_t sbase = smem_u32(smem);
        ChunkWalker w;
        w.init(sk, u0, u1, kext);
        long long a_ci = 0, b_ci = 0;  // chunks whose MMA1 / MMA2 were issued
        int tcount = 0, segs = 0, prev_t = -1, prev_major = -1;
        ChunkInfo pend;                // chunk whose MMA2 is next
        bool have = false;
        // MMA1 of one chunk into WH accumulator (a_ci & 1).
        auto mma1 = [&](const ChunkInfo &c) -> bool {
            const int s = (int)(a_ci % kStages);
            if (!mbar_wait(&bars.full[s], (uint32_t)((a_ci / kStages) & 1))) return false;
            if (c.major != prev_major) {
                if (!mbar_wait(&bars.tfull, (uint32_t)(tcount & 1))) return false;
                ++tcount;
                prev_major = c.major;
            }
            const int db = (int)(a_ci & 1);
            if (!mbar_wait(&bars.d1empty[db], (uint32_t)(((a_ci >> 1) & 1) ^ 1))) return false;
            tc::tc_fence_after();
            const uint32_t d = tmem + kD1 + (uint32_t)db * kD1Cols;
            const uint32_t tA = sbase + OFF_T, fB = sbase + s * STAGE + OFF_F1;
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
            ++a_ci;
            return true;
        };
        // MMA2 of the pending chunk into the contraction accumulator.
        auto mma2 = [&](const ChunkInfo &c) -> bool {
            const int s = (int)(b_ci % kStages);
            if (c.first_seg && segs > 0 &&
                !mbar_wait(&bars.d2empty, (uint32_t)((segs - 1) & 1)))
                return false;
            if (!mbar_wait(&bars.qfull, (uint32_t)(b_ci & 1))) return false;
            tc::tc_fence_after();
            const uint32_t qh = sbase + OFF_Q, ql = qh + Q_PLANE;
            const uint32_t fB = sbase + s * STAGE + OFF_F2;
#pragma unroll
            for (int ks = 0; ks < kC / 16; ks++) {
                const uint32_t ko = (uint32_t)ks * 32u;
                const uint64_t bdesc = desc_sw128(fB + ko);
                tc::umma(tmem + kD2, desc_sw128(qh + ko), bdesc, id96,
                         (c.first_seg && ks == 0) ? 0u : 1u);
                tc::umma(tmem + kD2, desc_sw128(ql + ko), bdesc, id64, 1u);
            }
            tc::umma_commit(&bars.qempty);
            tc::umma_commit(&bars.empty[s]);
            if (c.last_seg) {
                tc::umma_commit(&bars.d2full);
                ++segs;
            }
            ++b_ci;
            return true;
        };
        bool ok = true;
        if (w.ok) {
            pend = take(w, sk, kext, prev_t);
            prev_t = pend.t;
            have = true;
            ok = mma1(pend);
        }
        while (ok && have && !*abort_flag) {
            ChunkInfo next;
            const bool more = w.ok;
            if (more) {
                next = take(w, sk, kext, prev_t);
                prev_t = next.t;
                if (!mma1(next)) {
                    ok = false;
                    break;
                }
            }
            if (!mma2(pend)) {
                ok = false;
                break;
            }
            have = more;
            pend = next;
        }
        if (!ok) give_up();
        if (*abort_flag) {
            tc::umma_commit(&bars.drain);
            mbar_wait(&bars.drain, 0);
        }
    } else if (warp >= 2) {
        // ---- epilogue: WH -> Q, and the contraction -> f64 partials --------
        const int q = warp & 3;                  // lane quarter this warp may read
        const int half = (warp - 2) >> 2;        // which 32 of the chunk's 64 elements
        const int o = q * 32 + lane;             // output (TMEM lane) within the tile
        const uint32_t lane_off = (uint32_t)(q * 32) << 16;
        unsigned char *qrow = smem + OFF_Q + o * 128;  // this output's Q row (hi plane)
        ChunkWalker w;
        w.init(sk, u0, u1, kext);
        const int major0 = (int)(u0 / sk.major_units());
        long long ci = 0;
        int segs = 0, prev_t = -1;
        double sum[16];
#pragma unroll
        for (int i = 0; i < 16; i++) sum[i] = 0.0;
        while (w.ok && !*abort_flag) {
            const ChunkInfo c = take(w, sk, kext, prev_t);
            prev_t = c.t;
            const int s = (int)(ci % kStages), db = (int)(ci & 1);
            if (!mbar_wait(&bars.d1full[db], (uint32_t)((ci >> 1) & 1))) {
                give_up();
                break;
            }
            tc::tc_fence_after();
            const unsigned char *vs = smem + s * STAGE;
            uint32_t packh[16], packl[16];  // Q hi / lo of this thread's 32 elements, bf16 pairs
#pragma unroll
            for (int sub = 0; sub < 2; sub++) {
                // Elements e = half * 32 + sub * 16 + i of the chunk.
                float g0[16], g1[16], g2[16];
                const uint32_t ta = tmem + lane_off + kD1 + (uint32_t)db * kD1Cols +
                                    (uint32_t)(half * 32 + sub * 16);
                tc::tmem_ld16(ta, g0);
                tc::tmem_ld16(ta + 64, g1);
                tc::tmem_ld16(ta + 128, g2);
                tc::tmem_wait_ld();
                float v[16];
                if (HPASS) {
                    const float *vf = reinterpret_cast<const float *>(vs);
#pragma unroll
                    for (int i = 0; i < 16; i++) v[i] = vf[(half * 32 + sub * 16 + i) * kM + o];
                } else {
                    // Box `half` holds columns half * 32 .. +31 of rows 0..127,
                    // 16-byte chunk c of row o at (c ^ (o & 7)).
                    const unsigned char *row = vs + half * (V_BYTES / 2) + o * 128;
#pragma unroll
                    for (int c4 = 0; c4 < 4; c4++) {
                        const int ch = sub * 4 + c4;
                        const float4 x =
                            *reinterpret_cast<const float4 *>(row + ((ch ^ (o & 7)) << 4));
                        v[4 * c4] = x.x;
                        v[4 * c4 + 1] = x.y;
                        v[4 * c4 + 2] = x.z;
                        v[4 * c4 + 3] = x.w;
                    }
                }
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
                    packh[sub * 8 + i / 2] = *reinterpret_cast<const uint32_t *>(&hi);
                    packl[sub * 8 + i / 2] = *reinterpret_cast<const uint32_t *>(&lo);
                }
            }
            tc::tc_fence_before();
            mbar_arrive(&bars.d1empty[db]);
            // Q of the previous chunk must have been read by its MMA2.
            if (!mbar_wait(&bars.qempty, (uint32_t)((ci & 1) ^ 1))) {
                give_up();
                break;
            }
#pragma unroll
            for (int c4 = 0; c4 < 4; c4++) {
                const int kc = half * 4 + c4;  // 16-byte chunk of the 128-byte Q row
                const int pos = (kc ^ (o & 7)) << 4;
                *reinterpret_cast<uint4 *>(qrow + pos) =
                    make_uint4(packh[4 * c4], packh[4 * c4 + 1], packh[4 * c4 + 2],
                               packh[4 * c4 + 3]);
                *reinterpret_cast<uint4 *>(qrow + Q_PLANE + pos) =
                    make_uint4(packl[4 * c4], packl[4 * c4 + 1], packl[4 * c4 + 2],
                               packl[4 * c4 + 3]);
            }
            fence_proxy_async_smem();
            mbar_arrive(&bars.qfull);
            if (c.last_seg) {
                if (!mbar_wait(&bars.d2full, (uint32_t)(segs & 1))) {
                    give_up();
                    break;
                }
                tc::tc_fence_after();
                // Columns half * 16 .. +15 of the three groups (k of the
                // products with Fh, Fm, Fl); their sum is the contraction.
                float x0[16], x1[16], x2[16];
                const uint32_t ta = tmem + lane_off + kD2 + (uint32_t)(half * 16);
                tc::tmem_ld16(ta, x0);
                tc::tmem_ld16(ta + kR, x1);
                tc::tmem_ld16(ta + 2 * kR, x2);
                tc::tmem_wait_ld();
                tc::tc_fence_before();
                mbar_arrive(&bars.d2empty);
#pragma unroll
                for (int i = 0; i < 16; i++) sum[i] += (double)(x0[i] + x1[i] + x2[i]);
                ++segs;
            }
            if (c.last_tile) {
                double *dst = part + ((size_t)b * sk.slots + (size_t)(c.major - major0)) *
                                         (size_t)kM * RP;
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const int k = half * 16 + i;
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
    if (warp == 1) {
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

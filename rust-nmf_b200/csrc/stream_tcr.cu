// stream_tcr.cu -- launch of brunet's tensor-core passes (tcr.cuh) and the
// split of a factor into the two concatenated bf16 term layouts they read.
#include <atomic>
#include <algorithm>

#include "launch.h"
#include "tcr.cuh"

namespace nmfcu {
namespace tcr {

constexpr int kAttrDevices = 64;  // devices whose launch attributes are cached

// Three bf16 terms of f: h = bf16(f), m = bf16(f - h), l = bf16(f - h - m).
__device__ __forceinline__ void split3(double f, __nv_bfloat16 &h, __nv_bfloat16 &m,
                                       __nv_bfloat16 &l) {
    h = __double2bfloat16(f);
    const double r1 = f - (double)__bfloat162float(h);
    m = __double2bfloat16(r1);
    l = __double2bfloat16(r1 - (double)__bfloat162float(m));
}

// F (f64, logically R x K with F(k, x) = F[k * fk + x * fx]) -> rows x of
// KC bf16 in the two layouts of tcr.cuh: element b * R + k (block b < 6,
// k < R) holds term tile_term[b] of F(k, x) in `tile` and term unit_term[b]
// in `unit`; everything else (x >= K, positions >= 6 R) is zero.  Either
// output may be null.
__global__ void split_factor_concat(const double *__restrict__ F, int64_t fk, int64_t fx, int R,
                                    int K, int KC, int64_t xpad,
                                    __nv_bfloat16 *__restrict__ tile,
                                    __nv_bfloat16 *__restrict__ unit, const RunState *st) {
    if (run_stopped(st)) return;
    const int64_t total = xpad * KC;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        const int64_t x = t / KC;
        const int p = (int)(t - x * KC);
        __nv_bfloat16 vt = __float2bfloat16(0.f), vu = vt;
        if (x < K && p < 6 * R) {
            const int blk = p / R, k = p - blk * R;
            __nv_bfloat16 th[3];
            split3(F[k * fk + x * fx], th[0], th[1], th[2]);
            // Products Th Fh, Th Fm, Th Fl, Tm Fh, Tm Fm, Tl Fh.
            constexpr int tile_term[6] = {0, 0, 0, 1, 1, 2};
            constexpr int unit_term[6] = {0, 1, 2, 0, 1, 0};
            vt = th[tile_term[blk]];
            vu = th[unit_term[blk]];
        }
        if (tile) tile[t] = vt;
        if (unit) unit[t] = vu;
    }
}

template <bool HPASS, int KC>
cudaError_t launch_one(const CUtensorMap &v, const void *t, const CUtensorMap &f1, int kext,
                       int rank, int RP, const StreamK &sk, double *part, RunState *st,
                       cudaStream_t s) {
    // The attribute lives in each device's context: set it once per device
    // and instantiation.  Serving worker threads launch these passes
    // concurrently, so the flags are atomics (a repeated set is harmless).
    static std::atomic<bool> configured[kAttrDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kAttrDevices || !configured[dev].load(std::memory_order_acquire)) {
        e = cudaFuncSetAttribute(tcr_pass<HPASS, KC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Cfg<KC>::SMEM);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < kAttrDevices) configured[dev].store(true, std::memory_order_release);
    }
    tcr_pass<HPASS, KC><<<sk.G, kThreads, Cfg<KC>::SMEM, s>>>(
        v, static_cast<const __nv_bfloat16 *>(t), f1, kext, rank, RP, sk, part, st);
    return cudaGetLastError();
}

}  // namespace tcr

int tcr_concat_rank(int rank) { return rank <= 21 ? 128 : 192; }

cudaError_t tcr_pass_launch(bool hpass, const CUtensorMap &v, const void *t,
                            const CUtensorMap &f1, int kext, int rank, int RP, const StreamK &sk,
                            double *part, RunState *st, cudaStream_t s) {
    if (sk.G <= 0) return cudaSuccess;
    if (rank < 1 || rank > tcr::kMaxRank) return cudaErrorInvalidValue;
    if (tcr_concat_rank(rank) == 128)
        return hpass ? tcr::launch_one<true, 128>(v, t, f1, kext, rank, RP, sk, part, st, s)
                     : tcr::launch_one<false, 128>(v, t, f1, kext, rank, RP, sk, part, st, s);
    return hpass ? tcr::launch_one<true, 192>(v, t, f1, kext, rank, RP, sk, part, st, s)
                 : tcr::launch_one<false, 192>(v, t, f1, kext, rank, RP, sk, part, st, s);
}

void tcr_split_factor(const double *F, int64_t fk, int64_t fx, int R, int K, int64_t xpad,
                      void *tile, void *unit, const RunState *st, int sms, cudaStream_t s) {
    const int KC = tcr_concat_rank(R);
    const int64_t work = xpad * KC;
    const unsigned blocks =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)sms * 8));
    tcr::split_factor_concat<<<blocks, 256, 0, s>>>(F, fk, fx, R, K, KC, xpad,
                                                    static_cast<__nv_bfloat16 *>(tile),
                                                    static_cast<__nv_bfloat16 *>(unit), st);
}

}  // namespace nmfcu

// stream_tcr.cu -- launch of brunet's tensor-core passes (tcr.cuh) and the
// split of a factor into the two bf16 term layouts they read.
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

__global__ void split_factor_both(const double *__restrict__ F, int64_t fk, int64_t fx, int R,
                                  int K, __nv_bfloat16 *__restrict__ kx, int RPN, int64_t ldk,
                                  __nv_bfloat16 *__restrict__ xk, int64_t xpad,
                                  const RunState *st) {
    if (run_stopped(st)) return;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (kx) {
        const int64_t plane = (int64_t)RPN * ldk;
        for (int64_t t = t0; t < plane; t += stride) {
            const int64_t k = t / ldk, x = t - k * ldk;
            const double f = (k < R && x < K) ? F[k * fk + x * fx] : 0.0;
            split3(f, kx[t], kx[plane + t], kx[2 * plane + t]);
        }
    }
    if (xk) {
        const int64_t plane = xpad * kR;
        for (int64_t t = t0; t < plane; t += stride) {
            const int64_t x = t / kR, k = t - x * kR;
            const double f = (k < R && x < K) ? F[k * fk + x * fx] : 0.0;
            split3(f, xk[t], xk[plane + t], xk[2 * plane + t]);
        }
    }
}

template <bool HPASS>
cudaError_t launch_one(const CUtensorMap &v, const void *t, const void *f1,
                       int xpadT, int xpadF, int kext, int RP, const StreamK &sk, double *part,
                       RunState *st, cudaStream_t s) {
    // The attribute lives in each device's context: set it once per device
    // and instantiation.  Serving worker threads launch these passes
    // concurrently, so the flags are atomics (a repeated set is harmless).
    static std::atomic<bool> configured[kAttrDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kAttrDevices || !configured[dev].load(std::memory_order_acquire)) {
        e = cudaFuncSetAttribute(tcr_pass<HPASS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 SMEM);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < kAttrDevices) configured[dev].store(true, std::memory_order_release);
    }
    tcr_pass<HPASS><<<sk.G, kThreads, SMEM, s>>>(v, static_cast<const __nv_bfloat16 *>(t),
                                                  static_cast<const __nv_bfloat16 *>(f1), xpadT,
                                                  xpadF, kext, RP, sk, part, st);
    return cudaGetLastError();
}

}  // namespace tcr

cudaError_t tcr_pass_launch(bool hpass, const CUtensorMap &v, const void *t, const void *f1, int xpadT, int xpadF, int kext, int RP,
                            const StreamK &sk, double *part, RunState *st, cudaStream_t s) {
    if (sk.G <= 0) return cudaSuccess;
    return hpass ? tcr::launch_one<true>(v, t, f1, xpadT, xpadF, kext, RP, sk, part, st, s)
                 : tcr::launch_one<false>(v, t, f1, xpadT, xpadF, kext, RP, sk, part, st, s);
}

void tcr_split_factor(const double *F, int64_t fk, int64_t fx, int R, int K, void *kx, int RPN,
                      int64_t ldk, void *xk, int64_t xpad, const RunState *st, int sms,
                      cudaStream_t s) {
    const int64_t work = std::max<int64_t>(kx ? (int64_t)RPN * ldk : 0, xk ? xpad * tcr::kR : 0);
    const unsigned blocks =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)sms * 8));
    tcr::split_factor_both<<<blocks, 256, 0, s>>>(F, fk, fx, R, K,
                                                  static_cast<__nv_bfloat16 *>(kx), RPN, ldk,
                                                  static_cast<__nv_bfloat16 *>(xk), xpad, st);
}

}  // namespace nmfcu

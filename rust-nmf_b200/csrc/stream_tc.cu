// stream_tc.cu -- instantiation and launch of the tensor-core passes, and
// the bf16 split kernels of the split-bf16 precision form.
#include <atomic>
#include <algorithm>

#include "launch.h"
#include "tc.cuh"

namespace nmfcu {
namespace tc {

constexpr int kAttrDevices = 64;  // devices whose launch attributes are cached

// One read of V, both split copies: V hi/lo (n x ldb) and V^T hi/lo (p x ldbt),
// through 64 x 64 tiles: 16-byte reads of V rows, 4-byte (bf16 pair) writes
// of both copies.  Grid: x over 64-column tiles up to ldb, y over 64-row
// tiles up to ldbt; zero in the pad columns of both.  V's leading dimension
// is even and its base 16-byte aligned; ldb and ldbt are multiples of 8.
__global__ void split_v_both(const double *__restrict__ V, int64_t ldv,
                             __nv_bfloat16 *__restrict__ Vh, __nv_bfloat16 *__restrict__ Vl,
                             int64_t ldb, __nv_bfloat16 *__restrict__ Vth,
                             __nv_bfloat16 *__restrict__ Vtl, int64_t ldbt, int n, int p) {
    __shared__ double tile[64][65];
    const int c0 = blockIdx.x * 64, r0 = blockIdx.y * 64;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;  // 8 warps
    const int cc = 2 * lane;
    for (int y = w; y < 64; y += 8) {
        const int r = r0 + y, c = c0 + cc;
        double a = 0.0, b = 0.0;
        if (r < n) {
            const double *src = V + (int64_t)r * ldv + c;
            if (c + 1 < p) {
                const double2 x = *reinterpret_cast<const double2 *>(src);
                a = x.x;
                b = x.y;
            } else if (c < p) {
                a = src[0];
            }
        }
        tile[y][cc] = a;
        tile[y][cc + 1] = b;
        if (r < n && c < ldb) {
            const __nv_bfloat16 ha = __double2bfloat16(a), hb = __double2bfloat16(b);
            const int64_t o = (int64_t)r * ldb + c;
            *reinterpret_cast<__nv_bfloat162 *>(Vh + o) = __halves2bfloat162(ha, hb);
            *reinterpret_cast<__nv_bfloat162 *>(Vl + o) = __halves2bfloat162(
                __double2bfloat16(a - (double)__bfloat162float(ha)),
                __double2bfloat16(b - (double)__bfloat162float(hb)));
        }
    }
    __syncthreads();
    for (int y = w; y < 64; y += 8) {
        const int c = c0 + y, r = r0 + cc;  // V^T row c, columns r, r + 1
        if (c < p && r < ldbt) {
            const double a = tile[cc][y], b = tile[cc + 1][y];
            const __nv_bfloat16 ha = __double2bfloat16(a), hb = __double2bfloat16(b);
            const int64_t o = (int64_t)c * ldbt + r;
            *reinterpret_cast<__nv_bfloat162 *>(Vth + o) = __halves2bfloat162(ha, hb);
            *reinterpret_cast<__nv_bfloat162 *>(Vtl + o) = __halves2bfloat162(
                __double2bfloat16(a - (double)__bfloat162float(ha)),
                __double2bfloat16(b - (double)__bfloat162float(hb)));
        }
    }
}

__global__ void split_factor(const double *__restrict__ F, int64_t fk, int64_t fx, int R, int K,
                             __nv_bfloat16 *__restrict__ out, int RPN, int64_t ldk,
                             const RunState *st) {
    if (run_stopped(st)) return;
    const int64_t plane = (int64_t)RPN * ldk;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < plane; t += stride) {
        const int64_t k = t / ldk, x = t - k * ldk;
        double f = 0.0;
        if (k < R && x < K) f = F[k * fk + x * fx];
        const __nv_bfloat16 h = __double2bfloat16(f);
        const double r1 = f - (double)__bfloat162float(h);
        const __nv_bfloat16 m = __double2bfloat16(r1);
        const double r2 = r1 - (double)__bfloat162float(m);
        out[t] = h;
        out[plane + t] = m;
        out[2 * plane + t] = __double2bfloat16(r2);
    }
}

template <int RPN, bool A_MN, bool OUT_KM>
cudaError_t launch_one(const CUtensorMap &ah, const CUtensorMap &al, const CUtensorMap *b3,
                       int kext, int RP, const StreamK &sk, double *part, RunState *st,
                       cudaStream_t s) {
    constexpr int smem = tc_smem_bytes<RPN>();
    // The attribute lives in each device's context: set it once per device
    // and instantiation.  Serving worker threads launch these passes
    // concurrently, so the flags are atomics (a repeated set is harmless).
    static std::atomic<bool> configured[kAttrDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kAttrDevices || !configured[dev].load(std::memory_order_acquire)) {
        e = cudaFuncSetAttribute(tc_pass<RPN, A_MN, OUT_KM>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < kAttrDevices) configured[dev].store(true, std::memory_order_release);
    }
    tc_pass<RPN, A_MN, OUT_KM><<<sk.G, kThreadsTC, smem, s>>>(ah, al, b3[0], b3[1], b3[2], kext,
                                                               RP, sk, part, st);
    return cudaGetLastError();
}

}  // namespace tc

cudaError_t tc_pass_launch(bool hpass, int RPN, const CUtensorMap &ah, const CUtensorMap &al,
                           const CUtensorMap *b3, int kext, int RP, const StreamK &sk,
                           double *part, RunState *st, cudaStream_t s) {
    if (sk.G <= 0) return cudaSuccess;
    // Both passes read A K-major; the H pass's A is the transposed split V.
    if (RPN == 16)
        return hpass ? tc::launch_one<16, false, true>(ah, al, b3, kext, RP, sk, part, st, s)
                     : tc::launch_one<16, false, false>(ah, al, b3, kext, RP, sk, part, st, s);
    return hpass ? tc::launch_one<32, false, true>(ah, al, b3, kext, RP, sk, part, st, s)
                 : tc::launch_one<32, false, false>(ah, al, b3, kext, RP, sk, part, st, s);
}

void tc_split_v(const double *V, int64_t ldv, void *Vh, void *Vl, int64_t ldb, void *Vth,
                void *Vtl, int64_t ldbt, int n, int p, cudaStream_t s) {
    const dim3 grid((unsigned)((ldb + 63) / 64), (unsigned)((ldbt + 63) / 64));
    tc::split_v_both<<<grid, 256, 0, s>>>(V, ldv, static_cast<__nv_bfloat16 *>(Vh),
                                          static_cast<__nv_bfloat16 *>(Vl), ldb,
                                          static_cast<__nv_bfloat16 *>(Vth),
                                          static_cast<__nv_bfloat16 *>(Vtl), ldbt, n, p);
}

void tc_split_factor(const double *F, int64_t fk, int64_t fx, int R, int K, void *out, int RPN,
                     int64_t ldk, const RunState *st, int sms, cudaStream_t s) {
    const int64_t plane = (int64_t)RPN * ldk;
    const unsigned blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>((plane + 255) / 256, (int64_t)sms * 8));
    tc::split_factor<<<blocks, 256, 0, s>>>(F, fk, fx, R, K, static_cast<__nv_bfloat16 *>(out),
                                            RPN, ldk, st);
}

}  // namespace nmfcu

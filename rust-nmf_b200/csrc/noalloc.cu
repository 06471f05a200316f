// noalloc.cu -- the objective (KL divergence or Frobenius distance of V
// against W H) on device pointers, with no device allocation at all.
//
// Who needs this: callers that may not call cudaMalloc while they run.
// Examples are a serving process that reserves all of its device memory up
// front and hands out slices, code running under another framework's memory
// pool (where a raw cudaMalloc bypasses the pool's accounting and can fail
// once the pool holds the free memory), and a real-time loop that cannot
// afford the implicit synchronisation a cudaMalloc/cudaFree may cause.  The
// regular entry points keep per-context scratch that grows with the problem;
// this one uses only a fixed array compiled into the library.
//
// The scratch is the per-block partial sums of the objective pass: one f64
// per 8 rows of V, in `g_noalloc_partials`.  That caps n at
// NMFCU_NOALLOC_MAX_ROWS (include/nmfcu.h); larger n is rejected.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/nmfcu.h"

namespace nmfcu_internal {
nmfcu_status fail(nmfcu_status s, const std::string &msg);
}

namespace {

constexpr int kRowsPerBlock = 8;  // one warp per row, 8 warps per block
constexpr int kPartials = NMFCU_NOALLOC_MAX_ROWS / kRowsPerBlock;

// The scratch.  Every GPU that loads the library keeps these 512 KB until the
// process exits.  Host code must not pass `g_noalloc_partials` itself to a
// kernel: on the host that name is only a stand-in, not a device address.
// The device address comes from cudaGetSymbolAddress (noalloc_scratch below).
static __device__ __align__(256) double g_noalloc_partials[kPartials];

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// One warp per row of V, lanes across its columns; W and H are the caller's
// unpadded n x r and r x p arrays.  Block b writes partials[b] (every slot
// that the finalize step reads is written by this launch, so nothing needs to
// be cleared between calls).
template <int RP, bool KL>
__global__ void __launch_bounds__(256)
    noalloc_objective_partial(const double *__restrict__ V, int64_t ldv, int n, int64_t p, int r,
                              const double *__restrict__ W, const double *__restrict__ H,
                              double *__restrict__ partials) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * kRowsPerBlock + warp;
    double acc = 0.0;
    if (i < n) {
        double w[RP];
#pragma unroll
        for (int k = 0; k < RP; k++) w[k] = (k < r) ? W[(int64_t)i * r + k] : 0.0;
        const double *vrow = V + (int64_t)i * ldv;
        // 64-bit column index: j + 32 cannot wrap for any p the entry accepts.
        for (int64_t j = lane; j < p; j += 32) {
            double wh = 0.0;
#pragma unroll
            for (int k = 0; k < RP; k++)
                if (k < r) wh = fma(w[k], H[k * p + j], wh);
            const double v = vrow[j];
            if (KL) {
                // kl_divergence term, lib.rs:1418-1427
                if (v > 0.0) {
                    if (wh > 0.0) acc = add(acc, add(sub(mul(v, log(v / wh)), v), wh));
                } else {
                    acc = add(acc, wh);
                }
            } else {
                const double d = v - wh;  // euclidean_distance term, lib.rs:1440-1441
                acc = add(acc, mul(d, d));
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    __shared__ double red[kRowsPerBlock];
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kRowsPerBlock; w++) s += red[w];
        partials[blockIdx.x] = s;
    }
}

// Sums `count` partials in a fixed order and writes scale * sum to *out.
__global__ void noalloc_objective_finalize(const double *__restrict__ partials, int count,
                                           double scale, double *__restrict__ out) {
    __shared__ double red[256];
    double a = 0.0;
    for (int b = threadIdx.x; b < count; b += 256) a += partials[b];
    red[threadIdx.x] = a;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0] * scale;
}

// Device address of the scratch, looked up with the caller's device current
// the first time a call runs in a CUDA context, and cached per (device,
// context): a caller that runs in a context of its own (cuCtxCreate) rather
// than the device's primary context gets that context's copy of the array.
std::mutex g_scratch_mu;
constexpr int kMaxDevices = 64;
struct ScratchSlot {
    void *ctx;
    double *ptr;
};
ScratchSlot g_scratch[kMaxDevices] = {};

typedef int (*CtxGetCurrentFn)(void **);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<CtxGetCurrentFn>(p);
        cudaGetLastError();
        return static_cast<CtxGetCurrentFn>(nullptr);
    }();
    return fn;
}

nmfcu_status noalloc_scratch(int device, double **out) {
    if (device < 0 || device >= kMaxDevices)
        return nmfcu_internal::fail(NMFCU_ERR_UNSUPPORTED, "device ordinal beyond 63");
    CtxGetCurrentFn get = ctx_get_current();
    void *ctx = nullptr;
    if (get) get(&ctx);
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    ScratchSlot &slot = g_scratch[device];
    if (ctx && slot.ptr && slot.ctx == ctx) {
        *out = slot.ptr;
        return NMFCU_OK;
    }
    // First call in this context (or no context is current yet: the lookup
    // makes the device's primary context current, and the context is read
    // again after it).
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_partials);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return nmfcu_internal::fail(
            NMFCU_ERR_CUDA,
            std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
    }
    if (!ctx && get) get(&ctx);
    slot.ctx = ctx;
    slot.ptr = static_cast<double *>(ptr);
    *out = slot.ptr;
    return NMFCU_OK;
}

template <int RP>
void launch_partial(bool kl, unsigned blocks, cudaStream_t s, const double *V, int64_t ldv,
                    int n, int64_t p, int r, const double *W, const double *H, double *part) {
    if (kl)
        noalloc_objective_partial<RP, true><<<blocks, 256, 0, s>>>(V, ldv, n, p, r, W, H, part);
    else
        noalloc_objective_partial<RP, false><<<blocks, 256, 0, s>>>(V, ldv, n, p, r, W, H, part);
}

}  // namespace

extern "C" nmfcu_status nmfcu_objective_noalloc(int32_t kind, int64_t n, int64_t p, int64_t r,
                                                const double *dV, int64_t ldv, const double *dW,
                                                const double *dH, double *d_out, void *stream) {
    using nmfcu_internal::fail;
    if (kind != NMFCU_OBJECTIVE_KL && kind != NMFCU_OBJECTIVE_FROBENIUS)
        return fail(NMFCU_ERR_INVALID_ARG, "kind must be NMFCU_OBJECTIVE_KL or _FROBENIUS");
    if (n < 0 || p < 0) return fail(NMFCU_ERR_INVALID_ARG, "negative matrix dimension");
    if (r < 1) return fail(NMFCU_ERR_INVALID_ARG, "rank must be >= 1");
    if (r > NMFCU_MAX_RANK)
        return fail(NMFCU_ERR_UNSUPPORTED, "rank exceeds the largest built rank (32)");
    if (n > NMFCU_NOALLOC_MAX_ROWS)
        return fail(NMFCU_ERR_INVALID_ARG,
                    "n = " + std::to_string(n) + " exceeds the no-allocation scratch limit of " +
                        std::to_string(NMFCU_NOALLOC_MAX_ROWS) +
                        " rows; use nmfcu_divergence / nmfcu_distance");
    if (p > INT32_MAX) return fail(NMFCU_ERR_UNSUPPORTED, "p must fit in 32 bits");
    if (ldv < p) return fail(NMFCU_ERR_INVALID_ARG, "ldv must be >= p");
    if (!d_out || (n > 0 && p > 0 && (!dV || !dW || !dH)))
        return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? NMFCU_ERR_NO_DEVICE
                                                                                : NMFCU_ERR_CUDA,
                    std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    }
    double *part = nullptr;
    nmfcu_status st = noalloc_scratch(device, &part);
    if (st != NMFCU_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool kl = (kind == NMFCU_OBJECTIVE_KL);
    // An empty V (n == 0 or p == 0) has objective 0: no partial block runs
    // (so NULL factor pointers are never read) and the finalize step sums
    // zero partials.
    const unsigned blocks =
        (n > 0 && p > 0) ? (unsigned)((n + kRowsPerBlock - 1) / kRowsPerBlock) : 0u;
    if (blocks > 0) {
        const int ni = (int)n, ri = (int)r;
        const int64_t pi = p;
        if (r <= 8)
            launch_partial<8>(kl, blocks, s, dV, ldv, ni, pi, ri, dW, dH, part);
        else if (r <= 16)
            launch_partial<16>(kl, blocks, s, dV, ldv, ni, pi, ri, dW, dH, part);
        else
            launch_partial<32>(kl, blocks, s, dV, ldv, ni, pi, ri, dW, dH, part);
    }
    noalloc_objective_finalize<<<1, 256, 0, s>>>(part, (int)blocks, kl ? 1.0 : 0.5, d_out);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(NMFCU_ERR_CUDA, std::string("no-alloc objective launch: ") + cudaGetErrorString(e));
    return NMFCU_OK;
}

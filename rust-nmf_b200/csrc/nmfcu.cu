// nmfcu.cu -- host driver and C ABI of the B200 NMF engine.
//
// The loop of nmf_run_{brunet,lee,hals,dnmf} (omicverse/rust-NMF
// rust/src/lib.rs:1529-1647, 638-688, 827-906) re-expressed as a sequence of
// kernels on one CUDA stream.  The host never reads device data inside the
// loop: the stationary stop runs on the device and later kernels of a
// stopped run return immediately, so one synchronisation ends a call.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "../../include/nmfcu.h"
#include "internal.h"
#include "kernels.cuh"
#include "launch.h"
#include "stream.cuh"
#include "fcnnls.cuh"

using namespace nmfcu;

// ===========================================================================
// Errors
// ===========================================================================
namespace {

thread_local std::string g_last_error;

nmfcu_status fail(nmfcu_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

nmfcu_status cuda_fail(cudaError_t e, const char *what) {
    cudaGetLastError();  // clear a non-sticky error
    const nmfcu_status s = (e == cudaErrorMemoryAllocation) ? NMFCU_ERR_OOM
                           : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
                               ? NMFCU_ERR_NO_DEVICE
                               : NMFCU_ERR_CUDA;
    return fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

// Error reporting shared with the other translation units of the library
// (C++ linkage, so the nmfcu_* export list does not pick it up).
namespace nmfcu_internal {
nmfcu_status fail(nmfcu_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}
nmfcu_status cuda_fail(cudaError_t e, const char *what) { return ::cuda_fail(e, what); }
}  // namespace nmfcu_internal

namespace {

#define CUDA_TRY(expr)                                        \
    do {                                                      \
        cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, #expr);   \
    } while (0)

#define NMF_TRY(expr)                          \
    do {                                       \
        nmfcu_status s_ = (expr);              \
        if (s_ != NMFCU_OK) return s_;         \
    } while (0)

// ===========================================================================
// Rank buckets and the small per-bucket kernels
// ===========================================================================
constexpr int kBuckets[] = {2, 4, 6, 8, 10, 12, 14, 16, 20, 24, 28, 32};

int bucket_for(int64_t r) {
    for (int b : kBuckets)
        if (r <= b) return b;
    return 0;
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }
// Blocks of a grid-stride loop over `total` elements.
inline unsigned grid_for(int64_t total) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(total, kThreads), 4096));
}
inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Grams, rescaling, clamps and the objective pass: O(r^2 (n + p)) work plus
// the objective's one read of V.
struct Ops {
    virtual ~Ops() = default;
    // mode 2 KL objective, 3 Frobenius objective (f64 V); roff: row offsets
    // added to W H (offset method) or nullptr
    virtual void objective(const double *V, int64_t ldv, int n, int p, const double *W,
                           const double *H, int mode, int S2, int cols_per_split, double *obj,
                           const RunState *st, cudaStream_t s,
                           const double *roff = nullptr) const = 0;
    // W update from a dense (summed) contraction num (n x RP)
    virtual void w_apply(double *W, int n, const double *num, const EpiParams &e,
                         const RunState *st, cudaStream_t s) const = 0;
    // lsNMF objective partials over V o S and S: one per block, nblocks blocks
    virtual void ls_objective(const double *Vs, const double *S, int64_t ld, int n, int p,
                              const double *W, const double *H, int nblocks, double *part,
                              const RunState *st, cudaStream_t s) const = 0;
    // nsNMF: out = X S (rows x RP) and out = S H (RP x p)
    virtual void ns_right(const double *X, int rows, int r, double theta, double *out,
                          const RunState *st, cudaStream_t s) const = 0;
    virtual void ns_left(const double *H, int p, int r, double theta, double *out,
                         const RunState *st, cudaStream_t s) const = 0;
    // offset: addon = W^T off; off update from rowSums(H) and rowSums(V)
    virtual void off_addon(const double *W, int n, int r, const double *off, double *addon,
                           const RunState *st, cudaStream_t s) const = 0;
    virtual void off_update(const double *W, int n, int r, const double *rsh, const double *rsv,
                            int p, double eps, double *off, const RunState *st,
                            cudaStream_t s) const = 0;
    virtual void gram_w(const double *W, int n, int B, int rows_per_block, double *pg,
                        double *ps, const RunState *st, cudaStream_t s) const = 0;
    virtual void gram_h(const double *H, int p, int B, int cols_per_block, double *pg,
                        double *ps, const RunState *st, cudaStream_t s) const = 0;
    // The same partials, and the finished Gram G and sums from the launch's
    // last block (one launch; ticket zero before and after).
    virtual void gram_w_fin(const double *W, int n, int B, int rows_per_block, double *pg,
                            double *ps, double *G, double *sums, unsigned *ticket,
                            const RunState *st, cudaStream_t s) const = 0;
    virtual void gram_h_fin(const double *H, int p, int B, int cols_per_block, double *pg,
                            double *ps, double *G, double *sums, unsigned *ticket,
                            const RunState *st, cudaStream_t s) const = 0;
    virtual void rescale(double *W, int n, int r, const double *ps, int B, const RunState *st,
                         cudaStream_t s) const = 0;
    virtual void dnmf_scale(double *W, double *H, int n, int p, int r, const double *Gw,
                            const double *Gh, const RunState *st, cudaStream_t s) const = 0;
    virtual void clamp(double *W, double *H, int n, int p, int r, double eps,
                       const RunState *st, cudaStream_t s) const = 0;
};

template <int RP>
struct OpsT final : Ops {
    void objective(const double *V, int64_t ldv, int n, int p, const double *W, const double *H,
                   int mode, int S2, int cols_per_split, double *obj, const RunState *st,
                   cudaStream_t s, const double *roff) const override {
        if (n <= 0 || S2 <= 0) return;
        dim3 grid(cdiv(n, kThreads), S2), block(kThreads);
        if (mode == 2)
            nmfcu::rowpass<double, double, RP, 2><<<grid, block, 0, s>>>(
                V, ldv, n, p, W, H, cols_per_split, nullptr, obj, st);
        else
            nmfcu::rowpass<double, double, RP, 3><<<grid, block, 0, s>>>(
                V, ldv, n, p, W, H, cols_per_split, nullptr, obj, st, roff);
    }
    void w_apply(double *W, int n, const double *num, const EpiParams &e, const RunState *st,
                 cudaStream_t s) const override {
        if (n > 0) nmfcu::w_apply_dense<RP><<<cdiv(n, kThreads), kThreads, 0, s>>>(W, n, num, e, st);
    }
    void ls_objective(const double *Vs, const double *S, int64_t ld, int n, int p,
                      const double *W, const double *H, int nblocks, double *part,
                      const RunState *st, cudaStream_t s) const override {
        if (nblocks > 0)
            nmfcu::ls_objective<RP><<<nblocks, kThreads, 0, s>>>(Vs, S, ld, n, p, W, H, part, st);
    }
    void ns_right(const double *X, int rows, int r, double theta, double *out, const RunState *st,
                  cudaStream_t s) const override {
        if (rows > 0)
            nmfcu::ns_right_s<RP><<<cdiv(rows, kThreads), kThreads, 0, s>>>(X, rows, r, theta, out, st);
    }
    void ns_left(const double *H, int p, int r, double theta, double *out, const RunState *st,
                 cudaStream_t s) const override {
        if (p > 0) nmfcu::ns_left_s<RP><<<cdiv(p, kThreads), kThreads, 0, s>>>(H, p, r, theta, out, st);
    }
    void off_addon(const double *W, int n, int r, const double *off, double *addon,
                   const RunState *st, cudaStream_t s) const override {
        nmfcu::off_addon<RP><<<RP, kThreads, 0, s>>>(W, n, r, off, addon, st);
    }
    void off_update(const double *W, int n, int r, const double *rsh, const double *rsv, int p,
                    double eps, double *off, const RunState *st, cudaStream_t s) const override {
        if (n > 0)
            nmfcu::off_update<RP><<<cdiv(n, kThreads), kThreads, 0, s>>>(W, n, r, rsh, rsv, p, eps, off, st);
    }
    void gram_w(const double *W, int n, int B, int rows_per_block, double *pg, double *ps,
                const RunState *st, cudaStream_t s) const override {
        gram_w_partial<RP><<<B, RP * RP, 0, s>>>(W, n, rows_per_block, pg, ps, st);
    }
    void gram_h(const double *H, int p, int B, int cols_per_block, double *pg, double *ps,
                const RunState *st, cudaStream_t s) const override {
        gram_h_partial<RP><<<B, RP * RP, 0, s>>>(H, p, cols_per_block, pg, ps, st);
    }
    void gram_w_fin(const double *W, int n, int B, int rows_per_block, double *pg, double *ps,
                    double *G, double *sums, unsigned *ticket, const RunState *st,
                    cudaStream_t s) const override {
        gram_w_partial<RP><<<B, RP * RP, 0, s>>>(W, n, rows_per_block, pg, ps, st, G, sums,
                                                 ticket);
    }
    void gram_h_fin(const double *H, int p, int B, int cols_per_block, double *pg, double *ps,
                    double *G, double *sums, unsigned *ticket, const RunState *st,
                    cudaStream_t s) const override {
        gram_h_partial<RP><<<B, RP * RP, 0, s>>>(H, p, cols_per_block, pg, ps, st, G, sums,
                                                 ticket);
    }
    void rescale(double *W, int n, int r, const double *ps, int B, const RunState *st,
                 cudaStream_t s) const override {
        if (n <= 0) return;
        const unsigned blocks = std::min<unsigned>(cdiv((int64_t)n * RP, kThreads), 1184u);
        col_rescale<RP><<<blocks, kThreads, 0, s>>>(W, n, r, ps, B, st);
    }
    void dnmf_scale(double *W, double *H, int n, int p, int r, const double *Gw,
                    const double *Gh, const RunState *st, cudaStream_t s) const override {
        const int64_t m = std::max<int64_t>((int64_t)n * RP, (int64_t)r * p);
        const unsigned blocks = std::max(1u, std::min<unsigned>(cdiv(m, kThreads), 1184u));
        dnmf_rescale<RP><<<blocks, kThreads, 0, s>>>(W, H, n, p, r, Gw, Gh, st);
    }
    void clamp(double *W, double *H, int n, int p, int r, double eps, const RunState *st,
               cudaStream_t s) const override {
        const int64_t m = std::max<int64_t>((int64_t)n * RP, (int64_t)r * p);
        const unsigned blocks = std::max(1u, std::min<unsigned>(cdiv(m, kThreads), 1184u));
        clamp_wh<RP><<<blocks, kThreads, 0, s>>>(W, H, n, p, r, eps, st);
    }
};

const Ops *ops_for(int rp) {
    static const OpsT<2> o2;
    static const OpsT<4> o4;
    static const OpsT<6> o6;
    static const OpsT<8> o8;
    static const OpsT<10> o10;
    static const OpsT<12> o12;
    static const OpsT<14> o14;
    static const OpsT<16> o16;
    static const OpsT<20> o20;
    static const OpsT<24> o24;
    static const OpsT<28> o28;
    static const OpsT<32> o32;
    switch (rp) {
        case 2: return &o2;
        case 4: return &o4;
        case 6: return &o6;
        case 8: return &o8;
        case 10: return &o10;
        case 12: return &o12;
        case 14: return &o14;
        case 16: return &o16;
        case 20: return &o20;
        case 24: return &o24;
        case 28: return &o28;
        case 32: return &o32;
        default: return nullptr;
    }
}

// ===========================================================================
// TMA tensor maps
// ===========================================================================
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
        cudaGetLastError();
    });
    return fn;
}

// A 2-D row-major tensor of `rows` x `cols` elements (leading dimension ld)
// read in boxes of box_rows x box_cols.
nmfcu_status encode_2d(CUtensorMap *map, const void *base, bool f32, int64_t rows, int64_t cols,
                       int64_t ld, int box_cols, int box_rows,
                       CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_NONE) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return fail(NMFCU_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const size_t es = f32 ? 4 : 8;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * es)};
    cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                     2, const_cast<void *>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(NMFCU_ERR_CUDA, "cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) +
                                        ")");
    return NMFCU_OK;
}

bool tma_layout_ok(const void *base, int64_t ld, size_t es) {
    return (reinterpret_cast<uintptr_t>(base) % 16 == 0) && ((ld * (int64_t)es) % 16 == 0);
}

// bf16 matrix (rows x cols, leading dimension ld elements) with a swizzled
// box of box_cols x box_rows (box_cols * 2 <= the swizzle span).
nmfcu_status encode_2d_bf16(CUtensorMap *map, const void *base, int64_t rows, int64_t cols,
                            int64_t ld, int box_cols, int box_rows,
                            CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_128B) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return fail(NMFCU_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
    cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(NMFCU_ERR_CUDA, "cuTensorMapEncodeTiled (bf16) failed (code " +
                                        std::to_string((int)r) + ")");
    return NMFCU_OK;
}

// ===========================================================================
// Device buffers
// ===========================================================================
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    ~DevBuf() {
        if (ptr) cudaFree(ptr);
    }
    nmfcu_status ensure(size_t want) {
        want = std::max<size_t>(want, 256);
        if (want <= bytes) return NMFCU_OK;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&ptr, want);
        if (e != cudaSuccess) {
            ptr = nullptr;
            return cuda_fail(e, "cudaMalloc");
        }
        bytes = want;
        return NMFCU_OK;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <typename T>
    T *as() const { return static_cast<T *>(ptr); }
};

// Launch geometry of the small kernels of one problem shape.
struct Plan {
    int n = 0, p = 0, r = 0, RP = 0;
    int S2 = 1, cols_per_split = 1;    // objective pass column splits
    int Bw = 1, rows_per_gram = 1;     // W Gram blocks
    int Bh = 1, cols_per_gram = 1;     // H Gram blocks
    int obj_blocks = 0;                // objective partial count
};

Plan make_plan(int64_t n, int64_t p, int64_t r, int sms) {
    Plan pl;
    pl.n = (int)n;
    pl.p = (int)p;
    pl.r = (int)r;
    pl.RP = bucket_for(r);
    const int64_t target = (int64_t)sms * 8;
    const int64_t rb = std::max<int64_t>(1, (n + kThreads - 1) / kThreads);
    int64_t S2 = std::max<int64_t>(1, (target + rb - 1) / rb);
    S2 = std::min<int64_t>(S2, std::max<int64_t>(1, p / 256));
    int64_t cps = std::max<int64_t>(32, ((p + S2 - 1) / S2 + 31) / 32 * 32);
    pl.cols_per_split = (int)cps;
    pl.S2 = (int)std::max<int64_t>(1, (p + cps - 1) / cps);
    pl.obj_blocks = (int)(((n + kThreads - 1) / kThreads) * pl.S2);
    pl.Bw = (int)std::max<int64_t>(1, std::min<int64_t>((n + 63) / 64, sms));
    pl.rows_per_gram = (int)std::max<int64_t>(1, (n + pl.Bw - 1) / pl.Bw);
    pl.Bh = (int)std::max<int64_t>(1, std::min<int64_t>((p + 63) / 64, sms));
    pl.cols_per_gram = (int)std::max<int64_t>(1, (p + pl.Bh - 1) / pl.Bh);
    return pl;
}

// Stream-K split of `majors` major tiles, each `units` units long and cut
// into segments of at most `segu` units, over at most `sms` CTAs.
StreamK plan_sk(int64_t majors, int64_t units, int64_t segu, int sms) {
    StreamK sk;
    sk.fold = 0;
    sk.nseg = (int)std::max<int64_t>(1, (units + segu - 1) / segu);
    sk.UPT = (int)std::max<int64_t>(1, (units + sk.nseg - 1) / sk.nseg);
    sk.U = (units > 0) ? majors * sk.nseg * (int64_t)sk.UPT : 0;
    sk.valid = (int)std::max<int64_t>(units, 0);
    sk.G = (int)std::min<int64_t>(sms, sk.U);
    if (sk.G <= 0) {
        sk.G = 0;
        sk.slots = 0;
        return sk;
    }
    const int64_t per = (sk.U + sk.G - 1) / sk.G;
    sk.slots = (int)((per + sk.UPT - 1) / sk.UPT + 1);
    return sk;
}

// Every pass folds its partials: one slot per major tile a CTA meets (at
// most ceil(units a CTA / units a major tile) + 1 of them).
StreamK fold_sk(StreamK sk) {
    if (sk.G <= 0) return sk;
    sk.fold = 1;
    const int64_t per = (sk.U + sk.G - 1) / sk.G, mu = (int64_t)sk.nseg * sk.UPT;
    sk.slots = (int)((per + mu - 1) / mu + 1);
    return sk;
}

StreamK plan_h(const StreamOps *so, bool ratio, int64_t n, int64_t p, int sms) {
    const int tcols = so->h_tcols(ratio);
    return fold_sk(plan_sk((p + tcols - 1) / tcols,
                           (n + so->h_brows(ratio) - 1) / so->h_brows(ratio), so->h_segu(ratio),
                           sms));
}
StreamK plan_w(const StreamOps *so, bool ratio, int64_t n, int64_t p, int sms) {
    const int trows = so->w_trows(ratio), bcols = so->w_bcols(ratio);
    return fold_sk(
        plan_sk((n + trows - 1) / trows, (p + bcols - 1) / bcols, so->w_segu(ratio), sms));
}

}  // namespace

// ===========================================================================
// Context
// ===========================================================================
struct nmfcu_context {
    int device = 0;
    int sms = 148;
    cudaStream_t own_stream = nullptr;
    std::mutex mu;

    // Workspace.
    DevBuf V64, V32, W, H, part, pg, ps, Gw, sw, Gh, sh, Gw2, sw2, obj, dev, state;
    DevBuf Wf32, Ht64, Ht32;
    DevBuf Vs, Fs;     // split-bf16 form: V hi/lo, the factor's three terms
    DevBuf Xs;         // split-bf16 brunet: W and H in the tcr tile and unit layouts
    DevBuf Wns, Hns;   // nsNMF: W S (n x RP), S H (RP x p)
    DevBuf off, rsv, addon;  // offset: row offsets, row sums of V, W^T off
    DevBuf Wprev, Hprev;     // ehals: the iterate before the last extrapolation
    DevBuf S64, NH, NW;      // lsNMF: weights (pitched like V), the numerator contractions
                             // (snmf: the FCNNLS right-hand sides)
    DevBuf fcK, fcD, fcP, fcF, fcC;  // snmf: FCNNLS solutions, steps, sets, flags, ctc + counter
    DevBuf extra[nmfcu_internal::kContextSlots];  // scratch slots of the other translation units
    RunState *h_state = nullptr;  // pinned
    int *h_count = nullptr;       // pinned: the FCNNLS set sizes

    // Timing.
    bool timing = false;
    struct Ev {
        cudaEvent_t a, b;
        int kclass;
    };
    std::vector<Ev> events;
    std::vector<cudaEvent_t> pool;
    double total_ms[NMFCU_KCLASS_COUNT] = {};
    int64_t count[NMFCU_KCLASS_COUNT] = {};
    int64_t launch_total = 0;

    ~nmfcu_context() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        for (auto &e : events) {
            cudaEventDestroy(e.a);
            cudaEventDestroy(e.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
        if (h_state) cudaFreeHost(h_state);
        if (h_count) cudaFreeHost(h_count);
        if (own_stream) cudaStreamDestroy(own_stream);
        cudaSetDevice(prev);
    }

    cudaEvent_t get_event() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }

    // Brackets the launches of one scope for the timing hooks and counts them.
    struct Scope {
        nmfcu_context *c;
        cudaStream_t s;
        int kclass;
        cudaEvent_t a = nullptr;
        Scope(nmfcu_context *c_, cudaStream_t s_, int k, int launches = 1)
            : c(c_), s(s_), kclass(k) {
            c->launch_total += launches;
            if (c->timing) {
                a = c->get_event();
                cudaEventRecord(a, s);
            }
        }
        ~Scope() {
            if (c->timing) {
                cudaEvent_t b = c->get_event();
                cudaEventRecord(b, s);
                c->events.push_back({a, b, kclass});
            }
        }
    };

    void drain_timing() {
        for (auto &e : events) {
            float ms = 0.f;
            if (cudaEventSynchronize(e.b) == cudaSuccess &&
                cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
                total_ms[e.kclass] += ms;
                count[e.kclass] += 1;
            }
            pool.push_back(e.a);
            pool.push_back(e.b);
        }
        events.clear();
    }
};

namespace {

// ===========================================================================
// Pass sets: what one V element type needs for its two streaming passes
// ===========================================================================
struct PassSet {
    const StreamOps *so = nullptr;
    bool f32 = false;
    CUtensorMap tmVh, tmVw, tmW, tmHt;
    void *Ht = nullptr;  // H^T, written by the H epilogue, streamed by the W pass
    void *Wc = nullptr;  // f32 copy of W (f32 only; f64 streams the master W)
    // Split-bf16 form (tensor-core passes): V hi/lo maps for the H pass (box
    // 64 x 64) and the W pass (box 64 x 128), and the factor terms' maps.
    bool tc = false;
    int rpn = 0;
    int64_t ldw = 0, ldh = 0;  // leading dimensions of the W / H term planes
    CUtensorMap tmVhH, tmVlH, tmVhW, tmVlW, tmFw[3], tmFh[3];  // H: V^T planes; W: V planes
    // brunet in the split-bf16 form (tensor-core ratio passes over the f32
    // V): V maps of the H and W passes, and the factors' [3][xpad][32] term
    // planes as tile (box 128 rows) and chunk (box 64 rows) operands.
    bool tcr = false;
    int64_t xpadW = 0, xpadH = 0;
    CUtensorMap tmVrH, tmVrW, tmXwU, tmXhU;  // tcr: V (f32), W / H unit layouts
};

// The split-bf16 form runs lee / offset / hals / dnmf on the tensor cores;
// brunet's and nsNMF's ratio is formed per element, so they keep the FP32
// CUDA-core passes.
bool tc_form(const nmfcu_options *o) {
    return o->precision == NMFCU_PREC_BF16X3 && o->method != NMFCU_BRUNET &&
           o->method != NMFCU_NSNMF;
}
// Element type of the main passes is f32 (FP32 form, or brunet in the split form).
bool f32_form(const nmfcu_options *o) {
    return o->precision == NMFCU_PREC_FP32 || (o->precision == NMFCU_PREC_BF16X3 && !tc_form(o));
}
// brunet and nsNMF in the split-bf16 form run their ratio passes on the
// tensor cores (tcr.cuh) over the f32 V; their element type is still f32
// (f32_form).
bool tcr_form(const nmfcu_options *o) {
    return o->precision == NMFCU_PREC_BF16X3 &&
           (o->method == NMFCU_BRUNET || o->method == NMFCU_NSNMF);
}
int64_t round8(int64_t x) { return std::max<int64_t>(8, (x + 7) / 8 * 8); }
int64_t round128(int64_t x) { return std::max<int64_t>(128, (x + 127) / 128 * 128); }
int tc_rpn(int RP) { return RP <= 16 ? 16 : 32; }
constexpr int kTcrRank = 32;  // the tensor-core ratio passes pad the rank to 32
StreamK plan_tc_h(int64_t n, int64_t p, int sms) {
    return fold_sk(
        plan_sk((p + kTcTile - 1) / kTcTile, (n + kTcUnit - 1) / kTcUnit, kTcSegUnits, sms));
}
StreamK plan_tc_w(int64_t n, int64_t p, int sms) {
    return fold_sk(
        plan_sk((n + kTcTile - 1) / kTcTile, (p + kTcUnit - 1) / kTcUnit, kTcSegUnits, sms));
}
StreamK plan_tcr_h(int64_t n, int64_t p, int sms) {
    return fold_sk(plan_sk((p + kTcTile - 1) / kTcTile, (n + kTcrUnit - 1) / kTcrUnit,
                           kTcrSegUnits, sms));
}
StreamK plan_tcr_w(int64_t n, int64_t p, int sms) {
    return fold_sk(plan_sk((n + kTcTile - 1) / kTcTile, (p + kTcrUnit - 1) / kTcrUnit,
                           kTcrSegUnits, sms));
}
size_t tc_partial_bytes(const Plan &pl, int sms) {
    const StreamK h = plan_tc_h(pl.n, pl.p, sms), w = plan_tc_w(pl.n, pl.p, sms);
    const StreamK rh = plan_tcr_h(pl.n, pl.p, sms), rw = plan_tcr_w(pl.n, pl.p, sms);
    return sizeof(double) * (size_t)pl.RP * kTcTile *
           std::max({(size_t)h.G * h.slots, (size_t)w.G * w.slots, (size_t)rh.G * rh.slots,
                     (size_t)rw.G * rw.slots});
}

// Partial-sum bytes the two passes of `so` need for this shape.
size_t pass_partial_bytes(const StreamOps *so, const Plan &pl, bool ratio, int sms) {
    const int tcols = so->h_tcols(ratio), trows = so->w_trows(ratio);
    const StreamK skh = plan_h(so, ratio, pl.n, pl.p, sms);
    const StreamK skw = plan_w(so, ratio, pl.n, pl.p, sms);
    const size_t h = (size_t)skh.G * skh.slots * pl.RP * tcols;
    const size_t w = (size_t)skw.G * skw.slots * trows * pl.RP;
    return sizeof(double) * std::max(h, w);
}

// wsrc: the f64 matrix the H pass streams as W (W itself, or W S for nsNMF).
nmfcu_status make_passset(nmfcu_context *c, const Plan &pl, bool f32, bool ratio,
                          const void *V, int64_t ldv, PassSet *ps,
                          const double *wsrc = nullptr) {
    ps->f32 = f32;
    ps->so = f32 ? stream_ops_f32(pl.RP) : stream_ops_f64(pl.RP);
    if (!ps->so) return fail(NMFCU_ERR_UNSUPPORTED, "no streaming kernels for this rank");
    const int rps = ps->so->rps();
    ps->Ht = f32 ? c->Ht32.ptr : c->Ht64.ptr;
    ps->Wc = f32 ? c->Wf32.ptr : nullptr;
    if (pl.n <= 0 || pl.p <= 0) return NMFCU_OK;  // no pass runs
    if (!tma_layout_ok(V, ldv, f32 ? 4 : 8))
        return fail(NMFCU_ERR_INVALID_ARG, "V must be 16-byte aligned with 16-byte aligned rows");
    // The W pass reads rows of w_rowb() bytes (32, 64 or 128), swizzled with the
    // same span so that a warp's row-wise reads are conflict-free.
    const int rowb = ps->so->w_rowb(ratio);
    const CUtensorMapSwizzle wsw = rowb == 32   ? CU_TENSOR_MAP_SWIZZLE_32B
                                   : rowb == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                                : CU_TENSOR_MAP_SWIZZLE_128B;
    NMF_TRY(encode_2d(&ps->tmVh, V, f32, pl.n, pl.p, ldv, ps->so->h_boxc(ratio),
                      ps->so->h_brows(ratio)));
    NMF_TRY(encode_2d(&ps->tmVw, V, f32, pl.n, pl.p, ldv, ps->so->w_bcols(ratio),
                      ps->so->w_boxr(ratio), wsw));
    if (f32)
        NMF_TRY(encode_2d(&ps->tmW, c->Wf32.ptr, true, pl.n, rps, rps, rps,
                          ps->so->h_brows(ratio)));
    else
        NMF_TRY(encode_2d(&ps->tmW, wsrc ? wsrc : c->W.as<double>(), false, pl.n, pl.RP, pl.RP,
                          pl.RP, ps->so->h_brows(ratio)));
    NMF_TRY(encode_2d(&ps->tmHt, ps->Ht, f32, pl.p, rps, rps, rps, ps->so->w_bcols(ratio)));
    return NMFCU_OK;
}

// The split-bf16 passes over the f64 V (leading dimension ldv): splits V into
// the context's hi/lo planes and encodes every tensor map.
nmfcu_status make_tc_passset(nmfcu_context *c, const Plan &pl, const double *V64, int64_t ldv,
                             cudaStream_t s, PassSet *ps) {
    ps->tc = true;
    ps->f32 = false;
    ps->so = stream_ops_f32(pl.RP);  // its epilogues read the tensor-core partials
    if (!ps->so) return fail(NMFCU_ERR_UNSUPPORTED, "no streaming kernels for this rank");
    ps->Ht = nullptr;  // no H^T copy: the W pass streams the split terms of H
    ps->Wc = nullptr;
    ps->rpn = tc_rpn(pl.RP);
    ps->ldw = round8(pl.n);
    ps->ldh = round8(pl.p);
    if (pl.n <= 0 || pl.p <= 0) return NMFCU_OK;
    // Planes: V hi, V lo (n x ldb), V^T hi, V^T lo (p x ldbt).
    const int64_t ldb = round8(pl.p), ldbt = round8(pl.n);
    if ((ldbt + 31) / 32 > 65535)
        return fail(NMFCU_ERR_UNSUPPORTED, "the split-bf16 form supports at most 2097120 rows");
    unsigned char *vh = c->Vs.as<unsigned char>();
    unsigned char *vl = vh + (size_t)pl.n * ldb * 2;
    unsigned char *vth = vl + (size_t)pl.n * ldb * 2;
    unsigned char *vtl = vth + (size_t)pl.p * ldbt * 2;
    {
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
        tc_split_v(V64, ldv, vh, vl, ldb, vth, vtl, ldbt, pl.n, pl.p, s);
    }
    CUDA_TRY(cudaGetLastError());
    NMF_TRY(encode_2d_bf16(&ps->tmVhH, vth, pl.p, pl.n, ldbt, kTcUnit, kTcTile));
    NMF_TRY(encode_2d_bf16(&ps->tmVlH, vtl, pl.p, pl.n, ldbt, kTcUnit, kTcTile));
    NMF_TRY(encode_2d_bf16(&ps->tmVhW, vh, pl.n, pl.p, ldb, kTcUnit, kTcTile));
    NMF_TRY(encode_2d_bf16(&ps->tmVlW, vl, pl.n, pl.p, ldb, kTcUnit, kTcTile));
    unsigned char *f = c->Fs.as<unsigned char>();
    for (int i = 0; i < 3; i++) {
        NMF_TRY(encode_2d_bf16(&ps->tmFw[i], f + (size_t)i * ps->rpn * ps->ldw * 2, ps->rpn, pl.n,
                               ps->ldw, kTcUnit, ps->rpn));
        NMF_TRY(encode_2d_bf16(&ps->tmFh[i], f + (size_t)i * ps->rpn * ps->ldh * 2, ps->rpn, pl.p,
                               ps->ldh, kTcUnit, ps->rpn));
    }
    return NMFCU_OK;
}

// The split factors of brunet's tensor-core passes in c->Xs: W's rows then
// H's, each in the tile layout then the unit layout (xpad rows of
// tcr_concat_rank(r) bf16).
struct TcrTerms {
    void *w_tile, *w_unit, *h_tile, *h_unit;
};
TcrTerms tcr_terms(nmfcu_context *c, const PassSet &ps, int r) {
    const size_t row = 2 * (size_t)tcr_concat_rank(r);
    unsigned char *base = c->Xs.as<unsigned char>();
    TcrTerms x;
    x.w_tile = base;
    x.w_unit = base + row * ps.xpadW;
    x.h_tile = base + 2 * row * ps.xpadW;
    x.h_unit = base + 2 * row * ps.xpadW + row * ps.xpadH;
    return x;
}

// brunet's split-bf16 passes (tensor cores) over the f32 V (leading
// dimension ld32): added to the f32 pass set `ps` made for that V.
nmfcu_status add_tcr_passes(nmfcu_context *c, const Plan &pl, const void *V32, int64_t ld32,
                            PassSet *ps) {
    ps->tcr = true;
    ps->Ht = nullptr;  // no H^T copy: the W pass streams the split terms of H
    ps->xpadW = round128(pl.n);
    ps->xpadH = round128(pl.p);
    ps->ldw = round8(pl.n);
    ps->ldh = round8(pl.p);
    if (pl.n <= 0 || pl.p <= 0) return NMFCU_OK;
    if (pl.r > kTcrRank) return fail(NMFCU_ERR_UNSUPPORTED, "rank above 32");
    NMF_TRY(encode_2d(&ps->tmVrH, V32, true, pl.n, pl.p, ld32, 128, 64));
    NMF_TRY(encode_2d(&ps->tmVrW, V32, true, pl.n, pl.p, ld32, 32, 128,
                      CU_TENSOR_MAP_SWIZZLE_128B));
    const int kc = tcr_concat_rank(pl.r);
    const TcrTerms x = tcr_terms(c, *ps, pl.r);
    NMF_TRY(encode_2d_bf16(&ps->tmXwU, x.w_unit, ps->xpadW, kc, kc, 64, 128));
    NMF_TRY(encode_2d_bf16(&ps->tmXhU, x.h_unit, ps->xpadH, kc, kc, 64, 128));
    return NMFCU_OK;
}

// ===========================================================================
// The iteration loop
// ===========================================================================
struct RunArgs {
    const nmfcu_options *opt;
    Plan pl;
    const Ops *ops;
    PassSet main;        // the contractions' element type (f32 in the FP32 form)
    PassSet p64;         // f64 passes (plain method, refinement iterations)
    const double *V64;   // f64 V for the objective
    int64_t ldv64;
    double *W, *H;       // padded device factors
    double *dev;         // device deviances (or nullptr)
    double *Wns = nullptr, *Hns = nullptr;  // nsNMF: W S, S H
    double *off = nullptr, *rsv = nullptr, *addon = nullptr;  // offset
    double *Wprev = nullptr, *Hprev = nullptr;                // ehals
    // lsNMF: V holds V o S; S the weights (same pitch); NH / NW the
    // numerator contractions; pden the weighted passes' maps over S.
    const double *S64 = nullptr;
    double *NH = nullptr, *NW = nullptr;
    PassSet pden;
    bool weighted = false;  // h_step / w_step run the weighted passes
    double *Wout = nullptr;  // w_step's epilogue target when not W (column shards)
};

// The objective's per-block partials over this V (c->obj, pl.obj_blocks).
nmfcu_status enqueue_objective_partials(nmfcu_context *c, const RunArgs &a, cudaStream_t s) {
    const Plan &pl = a.pl;
    RunState *st = c->state.as<RunState>();
    const bool kl = (a.opt->method == NMFCU_BRUNET || a.opt->method == NMFCU_NSNMF);
    const double *West = a.W;
    if (a.opt->method == NMFCU_NSNMF) {  // KL of V against (W S) H, lib.rs:1779-1783
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
        a.ops->ns_right(a.W, pl.n, pl.r, a.opt->theta, a.Wns, st, s);
        West = a.Wns;
    }
    if (a.opt->method == NMFCU_LSNMF) {  // 0.5 ||(V - W H) o S||^2, lib.rs:1024-1035
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OBJECTIVE);
        a.ops->ls_objective(a.V64, a.S64, a.ldv64, pl.n, pl.p, a.W, a.H,
                            pl.n > 0 ? pl.obj_blocks : 0, c->obj.as<double>(), st, s);
    } else {
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OBJECTIVE);
        a.ops->objective(a.V64, a.ldv64, pl.n, pl.p, West, a.H, kl ? 2 : 3, pl.S2,
                         pl.cols_per_split, c->obj.as<double>(), st, s,
                         a.opt->method == NMFCU_OFFSET ? a.off : nullptr);
    }
    return NMFCU_OK;
}

StopParams stop_params(const nmfcu_options *o, long long iter) {
    StopParams sp;
    sp.stationary = 1;
    sp.iter = iter;
    sp.check_interval = o->check_interval;
    sp.check_niter = o->check_niter;
    sp.threshold = o->stationary_th;
    sp.scale = (o->method == NMFCU_BRUNET || o->method == NMFCU_NSNMF) ? 1.0 : 0.5;
    return sp;
}

// Objective of iteration `iter` into the deviances and the stationary stop.
nmfcu_status enqueue_objective(nmfcu_context *c, const RunArgs &a, long long iter,
                               cudaStream_t s) {
    NMF_TRY(enqueue_objective_partials(c, a, s));
    nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
    objective_finalize<<<1, kThreads, 0, s>>>(c->obj.as<double>(),
                                              a.pl.n > 0 ? a.pl.obj_blocks : 0, a.dev,
                                              stop_params(a.opt, iter), c->state.as<RunState>());
    return NMFCU_OK;
}

// The Grams and sums in one launch each; the ticket lives in the run state,
// which every run zeroes before its first launch.
void gram_w_full(nmfcu_context *c, const RunArgs &a, double *G, double *sums, cudaStream_t s) {
    const Plan &pl = a.pl;
    RunState *st = c->state.as<RunState>();
    nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
    a.ops->gram_w_fin(a.W, pl.n, pl.Bw, pl.rows_per_gram, c->pg.as<double>(), c->ps.as<double>(),
                      G, sums, &st->gram_ticket, st, s);
}
void gram_h_full(nmfcu_context *c, const RunArgs &a, double *G, double *sums, cudaStream_t s) {
    const Plan &pl = a.pl;
    RunState *st = c->state.as<RunState>();
    nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
    a.ops->gram_h_fin(a.H, pl.p, pl.Bh, pl.cols_per_gram, c->pg.as<double>(), c->ps.as<double>(),
                      G, sums, &st->gram_ticket, st, s);
}

// H step: the streaming contraction over all rows, then the per-column update.
nmfcu_status h_step(nmfcu_context *c, const RunArgs &a, const PassSet &ps, const EpiParams &e,
                    bool ratio, cudaStream_t s) {
    const Plan &pl = a.pl;
    RunState *st = c->state.as<RunState>();
    if (ps.tcr) {
        // brunet, split-bf16 form: W's bf16 terms in the unit layout (the
        // streamed operand of both MMAs) and H's in the tile layout (the
        // tile operand of W H); tensor-core ratio pass; update.
        const StreamK sk = plan_tcr_h(pl.n, pl.p, c->sms);
        const TcrTerms x = tcr_terms(c, ps, pl.r);
        {
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
            tcr_split_factor(a.W, 1, pl.RP, pl.r, pl.n, ps.xpadW, nullptr, x.w_unit, st, c->sms,
                             s);
            tcr_split_factor(a.H, pl.p, 1, pl.r, pl.p, ps.xpadH, x.h_tile, nullptr, st, c->sms,
                             s);
        }
        if (sk.G > 0) {
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_HSTEP);
            CUDA_TRY(tcr_pass_launch(true, ps.tmVrH, x.h_tile, ps.tmXwU, pl.n, pl.r, pl.RP, sk,
                                     c->part.as<double>(), st, s));
        }
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
        ps.so->h_epi(a.H, nullptr, pl.p, c->part.as<double>(), sk, kTcTile, e, st, s);
        return NMFCU_OK;
    }
    if (ps.tc) {
        // W (n x RP f64) -> three bf16 terms of W^T; tensor-core pass; update.
        const StreamK sk = plan_tc_h(pl.n, pl.p, c->sms);
        if (pl.n > 0) {
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
            tc_split_factor(a.W, 1, pl.RP, pl.r, pl.n, c->Fs.ptr, ps.rpn, ps.ldw, st, c->sms, s);
        }
        if (sk.G > 0) {
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_HSTEP);
            CUDA_TRY(tc_pass_launch(true, ps.rpn, ps.tmVhH, ps.tmVlH, ps.tmFw, pl.n, pl.RP, sk,
                                    c->part.as<double>(), st, s));
        }
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
        ps.so->h_epi(a.H, ps.Ht, pl.p, c->part.as<double>(), sk, kTcTile, e, st, s);
        return NMFCU_OK;
    }
    const int tcols = ps.so->h_tcols(ratio);
    const StreamK sk = plan_h(ps.so, ratio, pl.n, pl.p, c->sms);
    // An f64 pass in a reduced-precision run is a refinement iteration.
    const int kclass = (!ps.f32 && a.opt->precision != NMFCU_PREC_FP64)
                           ? NMFCU_KCLASS_HSTEP_REFINE : NMFCU_KCLASS_HSTEP;
    if (ps.f32 && pl.n > 0) {
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
        ps.so->w_copy(a.W, ps.Wc, pl.n, st, s);
    }
    if (sk.G > 0) {
        nmfcu_context::Scope sc(c, s, kclass);
        if (a.weighted)
            CUDA_TRY(ps.so->hpass_weighted(ps.tmVh, ps.tmW, a.H, pl.n, pl.p, sk,
                                           c->part.as<double>(), st, sk.G, s));
        else
            CUDA_TRY(ps.so->hpass(ratio, ps.tmVh, ps.tmW, a.H, pl.n, pl.p, sk,
                                  c->part.as<double>(), st, sk.G, s));
    }
    nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
    ps.so->h_epi(a.H, ps.Ht, pl.p, c->part.as<double>(), sk, tcols, e, st, s);
    return NMFCU_OK;
}

// W step: the streaming contraction over all columns, then the per-row update.
nmfcu_status w_step(nmfcu_context *c, const RunArgs &a, const PassSet &ps, const EpiParams &e,
                    bool ratio, cudaStream_t s) {
    const Plan &pl = a.pl;
    RunState *st = c->state.as<RunState>();
    if (ps.tcr) {
        // brunet, split-bf16 form: H's bf16 terms in the unit layout (the
        // streamed operand) and W's in the tile layout; tensor-core ratio
        // pass; update.
        const StreamK sk = plan_tcr_w(pl.n, pl.p, c->sms);
        const TcrTerms x = tcr_terms(c, ps, pl.r);
        {
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
            tcr_split_factor(a.H, pl.p, 1, pl.r, pl.p, ps.xpadH, nullptr, x.h_unit, st, c->sms,
                             s);
            tcr_split_factor(a.W, 1, pl.RP, pl.r, pl.n, ps.xpadW, x.w_tile, nullptr, st, c->sms,
                             s);
        }
        if (sk.G > 0) {
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_WSTEP);
            CUDA_TRY(tcr_pass_launch(false, ps.tmVrW, x.w_tile, ps.tmXhU, pl.p, pl.r, pl.RP, sk,
                                     c->part.as<double>(), st, s));
        }
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
        ps.so->w_epi(a.Wout ? a.Wout : a.W, pl.n, c->part.as<double>(), sk, kTcTile, e, st, s);
        return NMFCU_OK;
    }
    if (ps.tc) {
        // H (RP x p f64) -> three bf16 terms; tensor-core pass; update.
        const StreamK sk = plan_tc_w(pl.n, pl.p, c->sms);
        if (pl.p > 0) {
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
            tc_split_factor(a.H, pl.p, 1, pl.r, pl.p, c->Fs.ptr, ps.rpn, ps.ldh, st, c->sms, s);
        }
        if (sk.G > 0) {
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_WSTEP);
            CUDA_TRY(tc_pass_launch(false, ps.rpn, ps.tmVhW, ps.tmVlW, ps.tmFh, pl.p, pl.RP, sk,
                                    c->part.as<double>(), st, s));
        }
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
        ps.so->w_epi(a.Wout ? a.Wout : a.W, pl.n, c->part.as<double>(), sk, kTcTile, e, st, s);
        return NMFCU_OK;
    }
    const int trows = ps.so->w_trows(ratio);
    const StreamK sk = plan_w(ps.so, ratio, pl.n, pl.p, c->sms);
    const int kclass = (!ps.f32 && a.opt->precision != NMFCU_PREC_FP64)
                           ? NMFCU_KCLASS_WSTEP_REFINE : NMFCU_KCLASS_WSTEP;
    if (sk.G > 0) {
        nmfcu_context::Scope sc(c, s, kclass);
        if (a.weighted)
            CUDA_TRY(ps.so->wpass_weighted(ps.tmVw, ps.tmHt, a.W, pl.n, pl.p, sk,
                                           c->part.as<double>(), st, sk.G, s));
        else
            CUDA_TRY(ps.so->wpass(ratio, ps.tmVw, ps.tmHt, a.W, pl.n, pl.p, sk,
                                  c->part.as<double>(), st, sk.G, s));
    }
    nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
    ps.so->w_epi(a.Wout ? a.Wout : a.W, pl.n, c->part.as<double>(), sk, trows, e, st, s);
    return NMFCU_OK;
}

// H^T copy of the current H (for a W step that is not preceded by an H step).
void transpose_h(nmfcu_context *c, const RunArgs &a, const PassSet &ps, cudaStream_t s) {
    const Plan &pl = a.pl;
    if (pl.p <= 0) return;
    const int rps = ps.so->rps();
    const unsigned blocks = std::max(1u, std::min<unsigned>(cdiv((int64_t)pl.p * rps, kThreads), 4096u));
    nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
    if (ps.f32)
        h_transpose<float><<<blocks, kThreads, 0, s>>>(a.H, static_cast<float *>(ps.Ht), pl.p, pl.r, rps);
    else
        h_transpose<double><<<blocks, kThreads, 0, s>>>(a.H, static_cast<double *>(ps.Ht), pl.p, pl.r, rps);
}

EpiParams epi(const nmfcu_options *o, int r, const double *G, const double *sums, bool hside) {
    EpiParams e;
    e.method = o->method;
    e.r = r;
    e.eps = o->eps;
    e.lambda = hside ? o->sparsity_h : o->sparsity_w;
    e.gamma = hside ? o->smoothness_h : o->smoothness_w;
    e.G = G;
    e.sums = sums;
    return e;
}

// Enqueue one full iteration `it` (1-based).
nmfcu_status enqueue_iteration(nmfcu_context *c, const RunArgs &a, long long it, bool fp64,
                               cudaStream_t s) {
    const Plan &pl = a.pl;
    const nmfcu_options *o = a.opt;
    RunState *st = c->state.as<RunState>();
    const PassSet &ps = fp64 ? a.p64 : a.main;
    double *Gw = c->Gw.as<double>(), *sw = c->sw.as<double>();
    double *Gh = c->Gh.as<double>(), *sh = c->sh.as<double>();

    switch (o->method) {
        case NMFCU_BRUNET: {
            // nmf_run_brunet lib.rs:1558-1575.
            gram_w_full(c, a, Gw, sw, s);  // sum_w (lib.rs:1563-1568)
            NMF_TRY(h_step(c, a, ps, epi(o, pl.r, Gw, sw, true), true, s));
            gram_h_full(c, a, Gh, sh, s);  // sum_h (lib.rs:161-169)
            NMF_TRY(w_step(c, a, ps, epi(o, pl.r, Gh, sh, false), true, s));
            if (it % 10 == 0) {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->clamp(a.W, a.H, pl.n, pl.p, pl.r, DBL_EPSILON, st, s);
            }
            break;
        }
        case NMFCU_LEE: {
            // nmf_run_lee lib.rs:1618-1636.
            gram_w_full(c, a, Gw, sw, s);  // W^T W (lib.rs:1622-1631)
            NMF_TRY(h_step(c, a, ps, epi(o, pl.r, Gw, sw, true), false, s));
            gram_h_full(c, a, Gh, sh, s);  // H H^T (lib.rs:293-302)
            NMF_TRY(w_step(c, a, ps, epi(o, pl.r, Gh, sh, false), false, s));
            if (o->rescale) {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER, 2);
                a.ops->gram_w(a.W, pl.n, pl.Bw, pl.rows_per_gram, c->pg.as<double>(),
                              c->ps.as<double>(), st, s);
                a.ops->rescale(a.W, pl.n, pl.r, c->ps.as<double>(), pl.Bw, st, s);
            }
            break;
        }
        case NMFCU_NSNMF: {
            // nmf_run_nsnmf lib.rs:1804-1821: H update with W S, W update with
            // S H, then col_rescale(W).
            RunArgs aw = a;
            aw.W = a.Wns;
            {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->ns_right(a.W, pl.n, pl.r, o->theta, a.Wns, st, s);
            }
            gram_w_full(c, aw, Gw, sw, s);  // colsum(W S)
            NMF_TRY(h_step(c, aw, ps, epi(o, pl.r, Gw, sw, true), true, s));
            RunArgs ah = a;
            ah.H = a.Hns;
            {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->ns_left(a.H, pl.p, pl.r, o->theta, a.Hns, st, s);
            }
            // The W pass streams (S H)^T (the tensor-core passes split S H
            // themselves).
            if (!ps.tcr) transpose_h(c, ah, ps, s);
            gram_h_full(c, ah, Gh, sh, s);  // rowsum(S H)
            NMF_TRY(w_step(c, ah, ps, epi(o, pl.r, Gh, sh, false), true, s));
            {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER, 2);
                a.ops->gram_w(a.W, pl.n, pl.Bw, pl.rows_per_gram, c->pg.as<double>(),
                              c->ps.as<double>(), st, s);
                a.ops->rescale(a.W, pl.n, pl.r, c->ps.as<double>(), pl.Bw, st, s);
            }
            break;
        }
        case NMFCU_OFFSET: {
            // nmf_run_offset lib.rs:1694-1742: lee updates with the offset
            // terms, then the offset update.
            gram_w_full(c, a, Gw, sw, s);  // W^T W
            {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->off_addon(a.W, pl.n, pl.r, a.off, a.addon, st, s);
            }
            EpiParams eh = epi(o, pl.r, Gw, sw, true);
            eh.addon = a.addon;
            NMF_TRY(h_step(c, a, ps, eh, false, s));
            gram_h_full(c, a, Gh, sh, s);  // H H^T, rowSums(H)
            EpiParams ew = epi(o, pl.r, Gh, sh, false);
            ew.roff = a.off;
            NMF_TRY(w_step(c, a, ps, ew, false, s));
            {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->off_update(a.W, pl.n, pl.r, sh, a.rsv, pl.p, o->eps, a.off, st, s);
            }
            break;
        }
        case NMFCU_LSNMF: {
            // nmf_run_lsnmf lib.rs:978-1019.  H: numerator W^T (V o S) by a
            // plain pass over V o S into NH, denominator W^T ((W H) o S) by
            // the weighted pass over S, whose epilogue applies the update.
            // W: the same with the new H (its H^T copy from the H epilogue).
            RunArgs an = a;
            an.H = a.NH;
            EpiParams ep = epi(o, pl.r, nullptr, nullptr, true);
            ep.method = nmfcu::M_PRODUCT;
            NMF_TRY(h_step(c, an, a.p64, ep, false, s));
            RunArgs ad = a;
            ad.weighted = true;
            EpiParams eh = epi(o, pl.r, nullptr, nullptr, true);
            eh.aux = a.NH;
            NMF_TRY(h_step(c, ad, a.pden, eh, true, s));
            an = a;
            an.W = a.NW;
            NMF_TRY(w_step(c, an, a.p64, ep, false, s));
            EpiParams ew = epi(o, pl.r, nullptr, nullptr, false);
            ew.aux = a.NW;
            NMF_TRY(w_step(c, ad, a.pden, ew, true, s));
            break;
        }
        case NMFCU_EHALS: {
            // nmf_run_ehals lib.rs:753-776: extrapolate W and H (beta 0.5),
            // then one HALS sweep from there.
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER, 2);
            ehals_extrapolate<<<grid_for((int64_t)pl.n * pl.r), kThreads, 0, s>>>(
                a.W, a.Wprev, pl.n, pl.RP, pl.r, 0.5, o->eps, st);
            ehals_extrapolate<<<grid_for((int64_t)pl.r * pl.p), kThreads, 0, s>>>(
                a.H, a.Hprev, pl.r, pl.p, pl.p, 0.5, o->eps, st);
        }
            [[fallthrough]];
        default: {
            // nmf_run_hals lib.rs:667-676; nmf_run_dnmf lib.rs:862-884.
            gram_w_full(c, a, Gw, sw, s);
            NMF_TRY(h_step(c, a, ps, epi(o, pl.r, Gw, sw, true), false, s));
            gram_h_full(c, a, Gh, sh, s);
            NMF_TRY(w_step(c, a, ps, epi(o, pl.r, Gh, sh, false), false, s));
            if (o->method == NMFCU_DNMF) {
                gram_w_full(c, a, c->Gw2.as<double>(), c->sw2.as<double>(), s);
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->dnmf_scale(a.W, a.H, pl.n, pl.p, pl.r, c->Gw2.as<double>(), Gh, st, s);
            }
            break;
        }
    }
    return NMFCU_OK;
}

// Every workspace buffer one run of this plan needs, with its size: the
// single list behind both the allocation (ensure_workspace) and the
// serving layer's memory accounting (nmfcu_internal::context_growth).
struct WsNeed {
    DevBuf *buf;
    size_t bytes;
};

std::vector<WsNeed> workspace_needs(nmfcu_context *c, const Plan &pl, bool need_f32,
                                    bool need_tc, int method, bool need_tcr = false) {
    std::vector<WsNeed> v;
    const size_t RP = pl.RP;
    v.push_back({&c->W, sizeof(double) * (size_t)pl.n * RP});
    v.push_back({&c->H, sizeof(double) * RP * (size_t)pl.p});
    const bool ratio = true;  // sized for the larger of the two tilings
    size_t part = 0;
    for (bool rt : {ratio, !ratio}) {
        part = std::max(part, pass_partial_bytes(stream_ops_f64(pl.RP), pl, rt, c->sms));
        if (need_f32) part = std::max(part, pass_partial_bytes(stream_ops_f32(pl.RP), pl, rt, c->sms));
    }
    if (need_tc || need_tcr) part = std::max(part, tc_partial_bytes(pl, c->sms));
    v.push_back({&c->part, part});
    if (need_tc)
        v.push_back({&c->Fs, 3 * 2 * (size_t)tc_rpn(pl.RP) *
                                 (size_t)std::max(round8(pl.n), round8(pl.p))});
    if (need_tc)
        v.push_back({&c->Vs, 2 * 2 * ((size_t)pl.n * (size_t)round8(pl.p) +
                                      (size_t)pl.p * (size_t)round8(pl.n))});
    if (need_tcr)
        v.push_back({&c->Xs, 4 * (size_t)tcr_concat_rank(std::min(pl.r, kTcrRank)) *
                                 (size_t)(round128(pl.n) + round128(pl.p))});
    v.push_back({&c->Ht64, sizeof(double) * (size_t)pl.p * stream_ops_f64(pl.RP)->rps()});
    if (need_f32) {
        const size_t rps = stream_ops_f32(pl.RP)->rps();
        v.push_back({&c->Ht32, sizeof(float) * (size_t)pl.p * rps});
        v.push_back({&c->Wf32, sizeof(float) * (size_t)pl.n * rps});
    }
    const size_t B = (size_t)std::max(pl.Bw, pl.Bh);
    v.push_back({&c->pg, sizeof(double) * B * RP * RP});
    v.push_back({&c->ps, sizeof(double) * B * RP});
    v.push_back({&c->Gw, sizeof(double) * RP * RP});
    v.push_back({&c->Gh, sizeof(double) * RP * RP});
    v.push_back({&c->Gw2, sizeof(double) * RP * RP});
    v.push_back({&c->sw, sizeof(double) * RP});
    v.push_back({&c->sh, sizeof(double) * RP});
    v.push_back({&c->sw2, sizeof(double) * RP});
    v.push_back({&c->obj, sizeof(double) * (size_t)std::max(pl.obj_blocks, 1)});
    v.push_back({&c->state, sizeof(RunState)});
    if (method == NMFCU_NSNMF) {
        v.push_back({&c->Wns, sizeof(double) * (size_t)pl.n * RP});
        v.push_back({&c->Hns, sizeof(double) * RP * (size_t)pl.p});
    }
    if (method == NMFCU_LSNMF || method == NMFCU_SNMF_R || method == NMFCU_SNMF_L) {
        v.push_back({&c->NW, sizeof(double) * (size_t)pl.n * RP});
        v.push_back({&c->NH, sizeof(double) * RP * (size_t)pl.p});
    }
    if (method == NMFCU_SNMF_R || method == NMFCU_SNMF_L) {
        const size_t P = (size_t)std::max(pl.n, pl.p);
        v.push_back({&c->fcK, sizeof(double) * P * pl.r});
        v.push_back({&c->fcD, sizeof(double) * P * pl.r});
        v.push_back({&c->fcP, sizeof(unsigned) * P});
        v.push_back({&c->fcF, 2 * P});
        v.push_back({&c->fcC, sizeof(double) * (nmfcu::kFcMax * nmfcu::kFcMax + 4)});
    }
    if (method == NMFCU_EHALS) {
        v.push_back({&c->Wprev, sizeof(double) * (size_t)pl.n * RP});
        v.push_back({&c->Hprev, sizeof(double) * RP * (size_t)pl.p});
    }
    if (method == NMFCU_OFFSET) {
        v.push_back({&c->off, sizeof(double) * (size_t)pl.n});
        v.push_back({&c->rsv, sizeof(double) * (size_t)pl.n});
        v.push_back({&c->addon, sizeof(double) * RP});
    }
    return v;
}

nmfcu_status ensure_workspace(nmfcu_context *c, const Plan &pl, bool need_f32,
                              bool need_tc = false, int method = -1, bool need_tcr = false) {
    for (const WsNeed &w : workspace_needs(c, pl, need_f32 || need_tc, need_tc, method, need_tcr))
        NMF_TRY(w.buf->ensure(w.bytes));
    if (!c->h_state) CUDA_TRY(cudaMallocHost((void **)&c->h_state, sizeof(RunState)));
    if (!c->h_count) CUDA_TRY(cudaMallocHost((void **)&c->h_count, sizeof(int)));
    return NMFCU_OK;
}

nmfcu_status validate_options_rank(const nmfcu_options *o, int64_t n, int64_t p, int64_t r,
                                   int64_t max_rank) {
    if (!o) return fail(NMFCU_ERR_INVALID_ARG, "options pointer is NULL");
    if (n < 0 || p < 0) return fail(NMFCU_ERR_INVALID_ARG, "negative matrix dimension");
    if (r < 1) return fail(NMFCU_ERR_INVALID_ARG, "rank must be >= 1");
    if (n > INT32_MAX || p > INT32_MAX)
        return fail(NMFCU_ERR_UNSUPPORTED, "n and p must each fit in 32 bits");
    if (r > max_rank)
        return fail(NMFCU_ERR_UNSUPPORTED,
                    "rank " + std::to_string(r) + " exceeds the largest built rank (" +
                        std::to_string(max_rank) + ")");
    switch (o->method) {
        case NMFCU_BRUNET:
        case NMFCU_LEE:
        case NMFCU_OFFSET:
        case NMFCU_NSNMF:
        case NMFCU_HALS:
        case NMFCU_EHALS:
        case NMFCU_LSNMF:
        case NMFCU_SNMF_R:
        case NMFCU_SNMF_L:
        case NMFCU_DNMF: break;
        default: return fail(NMFCU_ERR_INVALID_ARG, "unknown method id");
    }
    if (o->stop != NMFCU_STOP_MAX_ITER && o->stop != NMFCU_STOP_STATIONARY)
        return fail(NMFCU_ERR_INVALID_ARG, "unknown stop id");
    if (o->precision != NMFCU_PREC_FP64 && o->precision != NMFCU_PREC_FP32 &&
        o->precision != NMFCU_PREC_BF16X3)
        return fail(NMFCU_ERR_INVALID_ARG, "unknown precision id");
    if (o->max_iter < 0) return fail(NMFCU_ERR_INVALID_ARG, "max_iter must be >= 0");
    if (o->method == NMFCU_LSNMF && o->precision != NMFCU_PREC_FP64)
        return fail(NMFCU_ERR_UNSUPPORTED, "lsNMF runs in FP64 only");
    if ((o->method == NMFCU_SNMF_R || o->method == NMFCU_SNMF_L) &&
        o->precision != NMFCU_PREC_FP64)
        return fail(NMFCU_ERR_UNSUPPORTED, "snmf/r and snmf/l run in FP64 only");
    if (o->check_niter < 0 || o->check_interval < 0)
        return fail(NMFCU_ERR_INVALID_ARG, "check_interval / check_niter must be >= 0");
    if (o->refine_iters < 0) return fail(NMFCU_ERR_INVALID_ARG, "refine_iters must be >= 0");
    return NMFCU_OK;
}

nmfcu_status validate_options(const nmfcu_options *o, int64_t n, int64_t p, int64_t r) {
    return validate_options_rank(o, n, p, r, NMFCU_MAX_RANK);
}

// Runs the loop on prepared device buffers; fills n_iter / n_dev.
// Waits for the stream and reports a streaming kernel that gave up waiting
// for its copies (the device state's timeout flag).
nmfcu_status finish_checked(nmfcu_context *c, cudaStream_t s) {
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(c->h_state, c->state.ptr, sizeof(RunState), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (c->h_state->timeout != 0)
        return fail(NMFCU_ERR_TIMEOUT, "a streaming kernel gave up waiting for its copies (code " +
                                           std::to_string(c->h_state->timeout) + ")");
    return NMFCU_OK;
}

// FCNNLS over P columns (fcnnls.rs:297-470): the kernels of fcnnls.cuh in
// the reference's loop order, with its one iteration counter (cap 3 l) and
// its tests for empty sets read back after each set update.
nmfcu_status fcnnls_device(nmfcu_context *c, int l, int64_t P, const double *ctc,
                           const double *cta, int64_t cs, int64_t js, double eps,
                           cudaStream_t s) {
    if (P <= 0) return NMFCU_OK;
    nmfcu::FcState fs;
    fs.K = c->fcK.as<double>();
    fs.D = c->fcD.as<double>();
    fs.pset = c->fcP.as<unsigned>();
    fs.fflag = c->fcF.as<uint8_t>();
    fs.hflag = fs.fflag + P;
    fs.count = reinterpret_cast<int *>(c->fcC.as<double>() + nmfcu::kFcMax * nmfcu::kFcMax + 2);
    constexpr int kT = 128;
    const unsigned g = (unsigned)cdiv(P, kT);
    int launches = 0;
    auto counted = [&](auto &&launch) -> nmfcu_status {
        CUDA_TRY(cudaMemsetAsync(fs.count, 0, sizeof(int), s));
        launch();
        launches++;
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(c->h_count, fs.count, sizeof(int), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        return NMFCU_OK;
    };
    NMF_TRY(counted([&] { nmfcu::fc_start<<<g, kT, 0, s>>>(l, P, ctc, cta, cs, js, fs); }));
    int nf = *c->h_count;
    int iter = 0;
    const int max_iter = 3 * l;
    while (nf > 0) {
        nmfcu::fc_solve<<<g, kT, 0, s>>>(l, P, ctc, cta, cs, js, fs, fs.fflag);
        launches++;
        NMF_TRY(counted([&] { nmfcu::fc_hset<<<g, kT, 0, s>>>(l, P, eps, fs, 1); }));
        int nh = *c->h_count;
        while (nh > 0 && iter < max_iter) {
            iter++;
            NMF_TRY(counted([&] { nmfcu::fc_any_ij<<<g, kT, 0, s>>>(l, P, eps, fs); }));
            if (*c->h_count == 0) break;
            nmfcu::fc_step<<<g, kT, 0, s>>>(l, P, eps, fs);
            nmfcu::fc_solve<<<g, kT, 0, s>>>(l, P, ctc, cta, cs, js, fs, fs.hflag);
            launches += 2;
            NMF_TRY(counted([&] { nmfcu::fc_hset<<<g, kT, 0, s>>>(l, P, eps, fs, 0); }));
            nh = *c->h_count;
        }
        NMF_TRY(counted([&] { nmfcu::fc_tail<<<g, kT, 0, s>>>(l, P, ctc, cta, cs, js, eps, fs); }));
        nf = *c->h_count;
        if (iter >= max_iter) break;
    }
    c->launch_total += launches;
    return NMFCU_OK;
}

// Kim-Park sparse NMF (nmf_run_snmf_kim_park, lib.rs:1216-1320): ANLS with
// FCNNLS.  snmf/r solves H from [W; sqrt(beta) 1^T] against [V; 0], then W
// from [H^T; eta I] against [V^T; 0]; snmf/l works on V^T, so it solves W
// first (normal equations H H^T + beta, right-hand sides V H^T) and then H
// (W^T W + eta^2 I, W^T V).  The right-hand sides are the plain passes'
// products; the Grams are the iteration's own.  Every iteration records
// 0.5 ||V - W H||^2; there is no stop test (the reference runs max_iter).
nmfcu_status run_snmf(nmfcu_context *c, RunArgs &a, cudaStream_t s, double *dev) {
    const nmfcu_options *o = a.opt;
    const Plan &pl = a.pl;
    const bool left = (o->method == NMFCU_SNMF_L);
    RunState *st = c->state.as<RunState>();
    CUDA_TRY(cudaMemsetAsync(c->state.ptr, 0, sizeof(RunState), s));
    // snmf/r: eta = smoothness_w, beta = sparsity_h; snmf/l: the mirror
    // (lib.rs:2117-2148).
    const double eta = left ? o->smoothness_h : o->smoothness_w;
    const double beta = left ? o->sparsity_w : o->sparsity_h;
    double *ctc = c->fcC.as<double>();
    double *misc = ctc + nmfcu::kFcMax * nmfcu::kFcMax;  // [vmax, -, count]
    double eta_eff = eta;
    if (eta < 0.0) {  // max(V) (and 0), lib.rs:1252-1256
        nmfcu::fc_vmax<<<1, 256, 0, s>>>(a.V64, a.ldv64, pl.n, pl.p, misc);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(&eta_eff, misc, sizeof(double), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
    }
    const double beta_eff = beta > 1e-30 ? beta : 1e-30;
    const double sb = std::sqrt(beta_eff);
    const int r = pl.r, RP = pl.RP;
    double *Gw = c->Gw.as<double>(), *sw = c->sw.as<double>();
    double *Gh = c->Gh.as<double>(), *sh = c->sh.as<double>();
    double *NH = c->NH.as<double>(), *NW = c->NW.as<double>();
    EpiParams ep = epi(o, r, nullptr, nullptr, true);
    ep.method = nmfcu::M_PRODUCT;
    // The factor normalised first: W's columns (snmf/r) or H's rows (snmf/l).
    if (left)
        nmfcu::fc_normalize<<<r, 256, 0, s>>>(a.H, pl.p, r, RP, 1);
    else
        nmfcu::fc_normalize<<<r, 256, 0, s>>>(a.W, pl.n, r, RP, 0);
    CUDA_TRY(cudaGetLastError());
    auto solve_h = [&](double add_all, double add_diag) -> nmfcu_status {
        // ctc = W^T W + ..., right-hand sides W^T V (the H pass's product).
        gram_w_full(c, a, Gw, sw, s);
        nmfcu::fc_normal<<<1, r * r, 0, s>>>(Gw, RP, r, add_all, add_diag, ctc);
        RunArgs an = a;
        an.H = NH;
        NMF_TRY(h_step(c, an, a.p64, ep, false, s));
        NMF_TRY(fcnnls_device(c, r, pl.p, ctc, NH, pl.p, 1, o->eps, s));
        if (pl.p > 0)
            nmfcu::fc_scatter<<<grid_for((int64_t)pl.p * r), kThreads, 0, s>>>(
                c->fcK.as<double>(), r, pl.p, RP, 1, a.H);
        CUDA_TRY(cudaGetLastError());
        return NMFCU_OK;
    };
    auto solve_w = [&](double add_all, double add_diag) -> nmfcu_status {
        // ctc = H H^T + ..., right-hand sides V H^T (the W pass's product).
        gram_h_full(c, a, Gh, sh, s);
        nmfcu::fc_normal<<<1, r * r, 0, s>>>(Gh, RP, r, add_all, add_diag, ctc);
        transpose_h(c, a, a.p64, s);
        RunArgs aw = a;
        aw.Wout = NW;
        NMF_TRY(w_step(c, aw, a.p64, ep, false, s));
        NMF_TRY(fcnnls_device(c, r, pl.n, ctc, NW, 1, RP, o->eps, s));
        if (pl.n > 0)
            nmfcu::fc_scatter<<<grid_for((int64_t)pl.n * r), kThreads, 0, s>>>(
                c->fcK.as<double>(), r, pl.n, RP, 0, a.W);
        CUDA_TRY(cudaGetLastError());
        return NMFCU_OK;
    };
    StopParams sp{};
    sp.stationary = 0;
    sp.scale = 0.5;
    for (long long it = 0; it < o->max_iter; it++) {
        if (left) {
            NMF_TRY(solve_w(sb * sb, 0.0));        // user W from [H^T; sqrt(beta) 1^T]
            NMF_TRY(solve_h(0.0, eta_eff * eta_eff));  // user H from [W; eta I]
        } else {
            NMF_TRY(solve_h(sb * sb, 0.0));
            NMF_TRY(solve_w(0.0, eta_eff * eta_eff));
        }
        NMF_TRY(enqueue_objective_partials(c, a, s));
        sp.iter = it;
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
        objective_finalize<<<1, kThreads, 0, s>>>(c->obj.as<double>(),
                                                  pl.n > 0 ? pl.obj_blocks : 0, dev, sp, st);
    }
    return finish_checked(c, s);
}

// Iterations whose kernels repeat with this period: the only iteration-
// dependent work is brunet's clamp every 10 iterations.
constexpr long long kGraphPeriod = 10;

// The main-precision iterations of a fixed-length run as a CUDA graph: the
// first iteration is enqueued directly (its launches set the kernels'
// one-time attributes), the next kGraphPeriod are captured and the graph is
// launched while a whole period of main-precision iterations remains; *it
// is the next iteration still to enqueue.  Small problems are bound by
// launch overhead, which the graph's launches cut.  If capture or
// instantiation fails nothing of the captured work ran: *it stays at the
// first captured iteration and the caller enqueues the rest directly.
nmfcu_status run_graphed(nmfcu_context *c, RunArgs &a, long long refine_from, cudaStream_t s,
                         long long *it) {
    const nmfcu_options *o = a.opt;
    const long long main_end = std::min<long long>(o->max_iter, refine_from);
    if (main_end < 1 + 3 * kGraphPeriod) return NMFCU_OK;
    // Not on the legacy or per-thread default streams (they cannot be
    // captured), nor on a stream the caller is capturing already.
    if (s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread) return NMFCU_OK;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(s, &cap));
    if (cap != cudaStreamCaptureStatusNone) return NMFCU_OK;
    const bool fp64 = (o->precision == NMFCU_PREC_FP64);
    NMF_TRY(enqueue_iteration(c, a, 1, fp64, s));
    *it = 2;
    const int64_t launches0 = c->launch_total;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    nmfcu_status st = NMFCU_OK;
    for (long long k = 0; k < kGraphPeriod && st == NMFCU_OK; k++)
        st = enqueue_iteration(c, a, *it + k, fp64, s);
    const cudaError_t ec = cudaStreamEndCapture(s, &graph);
    if (st == NMFCU_OK && ec == cudaSuccess && graph &&
        cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        const int64_t per_graph = c->launch_total - launches0;
        c->launch_total = launches0;
        cudaError_t el = cudaSuccess;
        while (el == cudaSuccess && *it + kGraphPeriod - 1 <= main_end) {
            el = cudaGraphLaunch(exec, s);
            if (el == cudaSuccess) {
                c->launch_total += per_graph;
                *it += kGraphPeriod;
            }
        }
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        CUDA_TRY(el);
        return NMFCU_OK;
    }
    // Capture did not give a graph: nothing captured ran; enqueue directly.
    c->launch_total = launches0;
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return NMFCU_OK;
}

nmfcu_status run_loop(nmfcu_context *c, RunArgs &a, cudaStream_t s, int64_t *n_dev,
                      int64_t *n_iter) {
    const nmfcu_options *o = a.opt;
    const bool stat = (o->stop == NMFCU_STOP_STATIONARY);
    CUDA_TRY(cudaMemsetAsync(c->state.ptr, 0, sizeof(RunState), s));
    if (stat) NMF_TRY(enqueue_objective(c, a, 0, s));
    const long long refine_from =
        (o->precision != NMFCU_PREC_FP64) ? (long long)o->max_iter - o->refine_iters : LLONG_MAX;
    long long it = 1;
    if (!stat && !c->timing) NMF_TRY(run_graphed(c, a, refine_from, s, &it));
    for (; it <= o->max_iter; it++) {
        const bool fp64 = (o->precision == NMFCU_PREC_FP64) || (it > refine_from);
        NMF_TRY(enqueue_iteration(c, a, it, fp64, s));
        if (stat) NMF_TRY(enqueue_objective(c, a, it, s));
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(c->h_state, c->state.ptr, sizeof(RunState), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (c->timing) c->drain_timing();
    const RunState &hs = *c->h_state;
    if (hs.timeout != 0)
        return fail(NMFCU_ERR_TIMEOUT, "a streaming kernel gave up waiting for its copies (code " +
                                           std::to_string(hs.timeout) + ")");
    if (hs.error == 1)
        return fail(NMFCU_ERR_INVALID_ARG,
                    "check_interval must be > 0 (the stationary stop evaluates iter % check_interval)");
    int64_t iters = hs.stopped ? hs.n_iter : o->max_iter;
    *n_iter = iters;
    *n_dev = stat ? iters + 1 : 0;
    return NMFCU_OK;
}

// ===========================================================================
// Per-device default contexts for the host-pointer API
// ===========================================================================
std::mutex g_ctx_mu;
std::map<int, std::unique_ptr<nmfcu_context>> g_ctx;

nmfcu_status check_device(int device) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(NMFCU_ERR_NO_DEVICE,
                    std::string("no CUDA device available: ") +
                        (e != cudaSuccess ? cudaGetErrorString(e) : "0 devices"));
    }
    if (device < 0 || device >= count)
        return fail(NMFCU_ERR_INVALID_ARG, "device ordinal out of range");
    return NMFCU_OK;
}

nmfcu_status context_init(nmfcu_context *c, int device) {
    c->device = device;
    CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    c->sms = prop.multiProcessorCount;
    CUDA_TRY(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    return NMFCU_OK;
}

nmfcu_status default_context(int device, nmfcu_context **out) {
    NMF_TRY(check_device(device));
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = g_ctx.find(device);
    if (it == g_ctx.end()) {
        std::unique_ptr<nmfcu_context> c(new nmfcu_context());
        NMF_TRY(context_init(c.get(), device));
        it = g_ctx.emplace(device, std::move(c)).first;
    }
    *out = it->second.get();
    return NMFCU_OK;
}

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            prev = -1;
            cudaGetLastError();
        }
        cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Upload host V (n x p f64) into the context's pitched V64.
nmfcu_status upload_v(nmfcu_context *c, const double *V, int64_t n, int64_t p, int64_t *ldv,
                      cudaStream_t s) {
    const int64_t ld = std::max<int64_t>(16, round_up(p, 16));
    NMF_TRY(c->V64.ensure(sizeof(double) * (size_t)(n * ld)));
    if (n > 0 && p > 0)
        CUDA_TRY(cudaMemcpy2DAsync(c->V64.ptr, ld * sizeof(double), V, p * sizeof(double),
                                   p * sizeof(double), n, cudaMemcpyHostToDevice, s));
    *ldv = ld;
    return NMFCU_OK;
}

nmfcu_status make_f32(nmfcu_context *c, const double *V64, int64_t ldv64, int64_t n, int64_t p,
                      int64_t *ldv32, cudaStream_t s) {
    const int64_t ld = std::max<int64_t>(32, round_up(p, 32));
    NMF_TRY(c->V32.ensure(sizeof(float) * (size_t)(n * ld)));
    if (n > 0 && p > 0) {
        const unsigned blocks = std::min<unsigned>(cdiv(n * p, kThreads), (unsigned)c->sms * 16);
        convert_f64_f32<<<blocks, kThreads, 0, s>>>(V64, ldv64, c->V32.as<float>(), ld, (int)n, (int)p);
        CUDA_TRY(cudaGetLastError());
    }
    *ldv32 = ld;
    return NMFCU_OK;
}

// Padded factor copies.  W (n x r) <-> Wd (n x RP); H (r x p) <-> Hd (RP x p).
nmfcu_status put_factors(nmfcu_context *c, const Plan &pl, const double *W, const double *H,
                         cudaMemcpyKind kind, cudaStream_t s) {
    const size_t RP = pl.RP;
    CUDA_TRY(cudaMemsetAsync(c->W.ptr, 0, sizeof(double) * (size_t)pl.n * RP, s));
    CUDA_TRY(cudaMemsetAsync(c->H.ptr, 0, sizeof(double) * RP * (size_t)pl.p, s));
    if (pl.n > 0)
        CUDA_TRY(cudaMemcpy2DAsync(c->W.ptr, RP * sizeof(double), W, pl.r * sizeof(double),
                                   pl.r * sizeof(double), pl.n, kind, s));
    if (pl.p > 0)
        CUDA_TRY(cudaMemcpyAsync(c->H.ptr, H, sizeof(double) * (size_t)pl.r * pl.p, kind, s));
    return NMFCU_OK;
}

nmfcu_status get_factors(nmfcu_context *c, const Plan &pl, double *W, double *H,
                         cudaMemcpyKind kind, cudaStream_t s) {
    const size_t RP = pl.RP;
    if (W && pl.n > 0)
        CUDA_TRY(cudaMemcpy2DAsync(W, pl.r * sizeof(double), c->W.ptr, RP * sizeof(double),
                                   pl.r * sizeof(double), pl.n, kind, s));
    if (H && pl.p > 0)
        CUDA_TRY(cudaMemcpyAsync(H, c->H.ptr, sizeof(double) * (size_t)pl.r * pl.p, kind, s));
    return NMFCU_OK;
}

bool ieq(const char *a, const char *b) {
    for (; *a && *b; a++, b++)
        if (tolower((unsigned char)*a) != tolower((unsigned char)*b)) return false;
    return *a == 0 && *b == 0;
}

// Columns [c0, c0 + kc) of X (rows x ldx) into out (rows x ld, zero padded).
__global__ void pack_cols(const double *__restrict__ X, int64_t ldx, int rows, int c0, int kc,
                          double *__restrict__ out, int ld) {
    const int64_t total = (int64_t)rows * ld;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / ld;
        const int k = (int)(t - i * ld);
        out[t] = (k < kc) ? X[i * ldx + c0 + k] : 0.0;
    }
}
// Rows [0, kc) of H (RP x p) into columns [c0, c0 + kc) of out (p x ldo).
__global__ void unpack_rows_t(const double *__restrict__ H, int p, int kc, double *__restrict__ out,
                              int64_t ldo, int c0) {
    const int64_t total = (int64_t)p * kc;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / kc;
        const int k = (int)(t - j * kc);
        out[j * ldo + c0 + k] = H[(int64_t)k * p + j];
    }
}

// Single-step driver used by the four update entry points.
enum StepKind { STEP_H_KL, STEP_W_KL, STEP_H_EUC, STEP_W_EUC };

nmfcu_status single_step(StepKind kind, int64_t n, int64_t p, int64_t r, const double *V,
                         const double *W, const double *H, double eps, double *out) {
    if (!V || !W || !H || !out) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    nmfcu_options o;
    nmfcu_options_default(&o);
    o.method = (kind == STEP_H_KL || kind == STEP_W_KL) ? NMFCU_BRUNET : NMFCU_LEE;
    o.eps = eps;
    NMF_TRY(validate_options(&o, n, p, r));
    nmfcu_context *c = nullptr;
    NMF_TRY(default_context(0, &c));
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    cudaStream_t s = c->own_stream;
    const Plan pl = make_plan(n, p, r, c->sms);
    NMF_TRY(ensure_workspace(c, pl, false));
    int64_t ldv = 0;
    NMF_TRY(upload_v(c, V, n, p, &ldv, s));
    NMF_TRY(put_factors(c, pl, W, H, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemsetAsync(c->state.ptr, 0, sizeof(RunState), s));
    RunArgs a;
    a.opt = &o;
    a.pl = pl;
    a.ops = ops_for(pl.RP);
    NMF_TRY(make_passset(c, pl, false, o.method == NMFCU_BRUNET, c->V64.ptr, ldv, &a.p64));
    a.main = a.p64;
    a.V64 = c->V64.as<double>();
    a.ldv64 = ldv;
    a.W = c->W.as<double>();
    a.H = c->H.as<double>();
    a.dev = nullptr;
    double *Gw = c->Gw.as<double>(), *sw = c->sw.as<double>();
    double *Gh = c->Gh.as<double>(), *sh = c->sh.as<double>();
    switch (kind) {
        case STEP_H_KL:
            gram_w_full(c, a, Gw, sw, s);
            NMF_TRY(h_step(c, a, a.p64, epi(&o, pl.r, Gw, sw, true), true, s));
            NMF_TRY(get_factors(c, pl, nullptr, out, cudaMemcpyDeviceToHost, s));
            break;
        case STEP_W_KL:
            gram_h_full(c, a, Gh, sh, s);
            transpose_h(c, a, a.p64, s);
            NMF_TRY(w_step(c, a, a.p64, epi(&o, pl.r, Gh, sh, false), true, s));
            NMF_TRY(get_factors(c, pl, out, nullptr, cudaMemcpyDeviceToHost, s));
            break;
        case STEP_H_EUC:
            gram_w_full(c, a, Gw, sw, s);
            NMF_TRY(h_step(c, a, a.p64, epi(&o, pl.r, Gw, sw, true), false, s));
            NMF_TRY(get_factors(c, pl, nullptr, out, cudaMemcpyDeviceToHost, s));
            break;
        case STEP_W_EUC:
            gram_h_full(c, a, Gh, sh, s);
            transpose_h(c, a, a.p64, s);
            NMF_TRY(w_step(c, a, a.p64, epi(&o, pl.r, Gh, sh, false), false, s));
            NMF_TRY(get_factors(c, pl, out, nullptr, cudaMemcpyDeviceToHost, s));
            break;
    }
    return finish_checked(c, s);
}

nmfcu_status objective_host(bool kl, int64_t n, int64_t p, int64_t r, const double *V,
                            const double *W, const double *H, double *out) {
    if (!V || !W || !H || !out) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    nmfcu_options o;
    nmfcu_options_default(&o);
    o.method = kl ? NMFCU_BRUNET : NMFCU_LEE;
    NMF_TRY(validate_options(&o, n, p, r));
    nmfcu_context *c = nullptr;
    NMF_TRY(default_context(0, &c));
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    cudaStream_t s = c->own_stream;
    const Plan pl = make_plan(n, p, r, c->sms);
    NMF_TRY(ensure_workspace(c, pl, false));
    NMF_TRY(c->dev.ensure(sizeof(double)));
    int64_t ldv = 0;
    NMF_TRY(upload_v(c, V, n, p, &ldv, s));
    NMF_TRY(put_factors(c, pl, W, H, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemsetAsync(c->state.ptr, 0, sizeof(RunState), s));
    const Ops *ops = ops_for(pl.RP);
    RunState *st = c->state.as<RunState>();
    ops->objective(c->V64.as<double>(), ldv, pl.n, pl.p, c->W.as<double>(), c->H.as<double>(),
                   kl ? 2 : 3, pl.S2, pl.cols_per_split, c->obj.as<double>(), st, s);
    StopParams sp{};
    sp.stationary = 0;
    sp.iter = 0;
    sp.scale = kl ? 1.0 : 0.5;
    objective_finalize<<<1, kThreads, 0, s>>>(c->obj.as<double>(), pl.n > 0 ? pl.obj_blocks : 0,
                                              c->dev.as<double>(), sp, st);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, c->dev.ptr, sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return NMFCU_OK;
}

}  // namespace

// ===========================================================================
// Services for the other translation units (internal.h)
// ===========================================================================
namespace nmfcu_internal {

nmfcu_status default_context(int device, nmfcu_context **out) { return ::default_context(device, out); }

nmfcu_status validate_options(const nmfcu_options *o, int64_t n, int64_t p, int64_t r) {
    return ::validate_options(o, n, p, r);
}
nmfcu_status validate_options_rank(const nmfcu_options *o, int64_t n, int64_t p, int64_t r,
                                   int64_t max_rank) {
    return ::validate_options_rank(o, n, p, r, max_rank);
}
nmfcu_status context_prepare(nmfcu_context *c, int64_t n, int64_t p) {
    return ensure_workspace(c, make_plan(n, p, NMFCU_MAX_RANK, c->sms), false);
}

nmfcu_status context_buffer(nmfcu_context *c, int slot, size_t bytes, void **out) {
    if (slot < 0 || slot >= kContextSlots) return fail(NMFCU_ERR_INVALID_ARG, "bad scratch slot");
    NMF_TRY(c->extra[slot].ensure(bytes));
    *out = c->extra[slot].ptr;
    return NMFCU_OK;
}

cudaStream_t context_stream(nmfcu_context *c) { return c->own_stream; }
int context_sms(nmfcu_context *c) { return c->sms; }
int context_device(nmfcu_context *c) { return c->device; }
std::mutex &context_mutex(nmfcu_context *c) { return c->mu; }
void count_launches(nmfcu_context *c, int64_t launches) { c->launch_total += launches; }

TimedScope::TimedScope(nmfcu_context *c_, cudaStream_t s_, int k, int launches)
    : c(c_), s(s_), kclass(k), a(nullptr) {
    c->launch_total += launches;
    if (c->timing) {
        cudaEvent_t e = c->get_event();
        cudaEventRecord(e, s);
        a = e;
    }
}
TimedScope::~TimedScope() {
    if (c->timing && a) {
        cudaEvent_t b = c->get_event();
        cudaEventRecord(b, s);
        c->events.push_back({static_cast<cudaEvent_t>(a), b, kclass});
    }
}
void drain_timing(nmfcu_context *c) {
    if (c->timing) c->drain_timing();
}

size_t context_bytes(nmfcu_context *c) {
    size_t t = 0;
    for (const DevBuf *b : {&c->V64, &c->V32, &c->W, &c->H, &c->part, &c->pg, &c->ps, &c->Gw,
                            &c->sw, &c->Gh, &c->sh, &c->Gw2, &c->sw2, &c->obj, &c->dev, &c->state,
                            &c->Wf32, &c->Ht64, &c->Ht32, &c->Vs, &c->Fs, &c->Xs, &c->Wns, &c->Hns,
                            &c->off, &c->rsv, &c->addon, &c->Wprev, &c->Hprev,
                            &c->S64, &c->NH, &c->NW,
                            &c->fcK, &c->fcD, &c->fcP, &c->fcF, &c->fcC})
        t += b->bytes;
    for (const DevBuf &b : c->extra) t += b.bytes;
    return t;
}

// A DevBuf grows to max(want, 256) bytes (DevBuf::ensure).
static size_t grow_by(const DevBuf &b, size_t want) {
    want = std::max<size_t>(want, 256);
    return want > b.bytes ? want - b.bytes : 0;
}

size_t context_growth(nmfcu_context *c, int64_t n, int64_t p, int64_t r, bool f32, bool tc,
                      int method, bool tcr) {
    const Plan pl = make_plan(n, p, r, c->sms);
    size_t g = 0;
    for (const WsNeed &w : workspace_needs(c, pl, f32 || tc, tc, method, tcr))
        g += grow_by(*w.buf, w.bytes);
    if (f32 && !tc) g += grow_by(c->V32, sizeof(float) * (size_t)n * std::max<int64_t>(32, round_up(p, 32)));
    return g;
}

size_t slot_growth(nmfcu_context *c, int slot, size_t bytes) {
    if (slot < 0 || slot >= kContextSlots) return 0;
    return grow_by(c->extra[slot], bytes);
}

void context_release(nmfcu_context *c) {
    DeviceGuard dg(c->device);
    for (DevBuf *b : {&c->V64, &c->V32, &c->W, &c->H, &c->part, &c->pg, &c->ps, &c->Gw, &c->sw,
                      &c->Gh, &c->sh, &c->Gw2, &c->sw2, &c->obj, &c->dev, &c->state, &c->Wf32,
                      &c->Ht64, &c->Ht32, &c->Vs, &c->Fs, &c->Xs, &c->Wns, &c->Hns,
                            &c->off, &c->rsv, &c->addon, &c->Wprev, &c->Hprev,
                            &c->S64, &c->NH, &c->NW,
                            &c->fcK, &c->fcD, &c->fcP, &c->fcF, &c->fcC})
        b->release();
    for (DevBuf &b : c->extra) b.release();
}

}  // namespace nmfcu_internal

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

void nmfcu_options_default(nmfcu_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->method = NMFCU_BRUNET;
    o->stop = NMFCU_STOP_MAX_ITER;
    o->precision = NMFCU_PREC_FP64;
    o->rescale = 1;
    o->max_iter = 2000;
    o->eps = 1e-9;
    o->theta = 0.5;
    o->stationary_th = DBL_EPSILON;
    o->check_interval = 50;
    o->check_niter = 10;
    o->refine_iters = 2;
    o->device = 0;
}

nmfcu_status nmfcu_parse_method(const char *name, int32_t *method) {
    if (!name || !method) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    static const struct {
        const char *n;
        int32_t id;
    } table[] = {
        {"brunet", NMFCU_BRUNET}, {"kl", NMFCU_BRUNET},
        {"lee", NMFCU_LEE}, {"frobenius", NMFCU_LEE}, {"euclidean", NMFCU_LEE},
        {"offset", NMFCU_OFFSET},
        {"nsnmf", NMFCU_NSNMF}, {"ns", NMFCU_NSNMF}, {"ns_nmf", NMFCU_NSNMF},
        {"hals", NMFCU_HALS},
        {"ehals", NMFCU_EHALS}, {"e-hals", NMFCU_EHALS}, {"extrap_hals", NMFCU_EHALS},
        {"dnmf", NMFCU_DNMF}, {"diag_nmf", NMFCU_DNMF}, {"diagonalised_nmf", NMFCU_DNMF},
        {"rcppml", NMFCU_DNMF},
        {"ls-nmf", NMFCU_LSNMF}, {"lsnmf", NMFCU_LSNMF},
        {"snmf/r", NMFCU_SNMF_R}, {"snmf_r", NMFCU_SNMF_R}, {"snmfr", NMFCU_SNMF_R},
        {"snmf/l", NMFCU_SNMF_L}, {"snmf_l", NMFCU_SNMF_L}, {"snmfl", NMFCU_SNMF_L},
    };
    for (const auto &t : table)
        if (ieq(name, t.n)) {
            *method = t.id;
            return NMFCU_OK;
        }
    return fail(NMFCU_ERR_INVALID_ARG,
                std::string("unknown algorithm '") + name +
                    "': supported: brunet, lee, offset, nsNMF, hals, ehals, dnmf, lsNMF, snmf/r, snmf/l");
}

nmfcu_status nmfcu_parse_stop(const char *name, int32_t *stop) {
    if (!name || !stop) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    if (ieq(name, "max_iter") || ieq(name, "fixed") || ieq(name, "none")) {
        *stop = NMFCU_STOP_MAX_ITER;
        return NMFCU_OK;
    }
    if (ieq(name, "stationary")) {
        *stop = NMFCU_STOP_STATIONARY;
        return NMFCU_OK;
    }
    return fail(NMFCU_ERR_INVALID_ARG, std::string("unknown stopping criterion '") + name +
                                           "': supported: max_iter, stationary");
}

}  // extern "C"

// One rank's column shard of a solve (nmfcu_shard_*): its context (used by
// this shard alone while it lives), plan, passes and the caller's buffers.
struct nmfcu_shard {
    nmfcu_context *c = nullptr;
    nmfcu_options opt{};
    Plan pl{};
    RunArgs a{};
    double *R = nullptr;     // [W contraction n x RP | H H^T RP x RP | rowSums(H) RP]
    double *Robj = nullptr;  // this shard's objective term, then the sum over shards
    long long it = 0;        // iterations whose W update has been applied
    long long refine_from = LLONG_MAX;
};

namespace {

// Method state set up before the first iteration: nsNMF's W S / S H buffers;
// the offset method's row sums of V and its starting offsets (off0 when
// given, on the host or the device, else rowMeans(V) as in lib.rs:1667-1679).
nmfcu_status setup_method(nmfcu_context *c, const Plan &pl, const nmfcu_options *o, RunArgs &a,
                          const double *off0, bool off0_host, cudaStream_t s) {
    if (o->method == NMFCU_NSNMF) {
        a.Wns = c->Wns.as<double>();
        a.Hns = c->Hns.as<double>();
    }
    if (o->method == NMFCU_EHALS) {  // the previous iterate starts as the start
        a.Wprev = c->Wprev.as<double>();
        a.Hprev = c->Hprev.as<double>();
        CUDA_TRY(cudaMemcpyAsync(a.Wprev, a.W, sizeof(double) * (size_t)pl.n * pl.RP,
                                 cudaMemcpyDeviceToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(a.Hprev, a.H, sizeof(double) * (size_t)pl.RP * pl.p,
                                 cudaMemcpyDeviceToDevice, s));
    }
    if (o->method == NMFCU_OFFSET) {
        a.off = c->off.as<double>();
        a.rsv = c->rsv.as<double>();
        a.addon = c->addon.as<double>();
        if (pl.n > 0) {
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER, off0 ? 1 : 2);
            v_row_sums<<<(unsigned)cdiv((int64_t)pl.n * 32, kThreads), kThreads, 0, s>>>(
                a.V64, a.ldv64, pl.n, pl.p, a.rsv);
            if (off0)
                CUDA_TRY(cudaMemcpyAsync(a.off, off0, sizeof(double) * (size_t)pl.n,
                                         off0_host ? cudaMemcpyHostToDevice
                                                   : cudaMemcpyDeviceToDevice, s));
            else
                off_init<<<(unsigned)cdiv(pl.n, kThreads), kThreads, 0, s>>>(a.rsv, pl.n, pl.p,
                                                                            a.off);
        }
    }
    CUDA_TRY(cudaGetLastError());
    return NMFCU_OK;
}

// nmfcu_run for a rank above NMFCU_MAX_RANK (nmfcu_internal::wide_run).
nmfcu_status run_host_wide(const nmfcu_options *opt, int64_t n, int64_t p, int64_t r,
                           const double *V, const double *W0, const double *H0, double *W,
                           double *H, double *deviances, int64_t deviances_cap,
                           int64_t *n_deviances, int64_t *n_iter) {
    NMF_TRY(nmfcu_internal::wide_validate(opt, n, p, r));
    if (!V || !W0 || !H0 || !W || !H || !n_deviances || !n_iter)
        return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    const bool stat = opt->stop == NMFCU_STOP_STATIONARY;
    if (stat && (!deviances || deviances_cap < opt->max_iter + 1))
        return fail(NMFCU_ERR_INVALID_ARG, "deviances must hold max_iter + 1 values");
    nmfcu_context *c = nullptr;
    NMF_TRY(default_context(opt->device, &c));
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    cudaStream_t s = c->own_stream;
    if (stat) NMF_TRY(c->dev.ensure(sizeof(double) * (size_t)(opt->max_iter + 1)));
    int64_t ldv = 0;
    NMF_TRY(upload_v(c, V, n, p, &ldv, s));
    int64_t nd = 0, ni = 0;
    NMF_TRY(nmfcu_internal::wide_run(c, opt, n, p, r, c->V64.as<double>(), ldv, W0, H0, W, H,
                                     cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost,
                                     stat ? c->dev.as<double>() : nullptr, s, &nd, &ni));
    if (stat && nd > 0)
        CUDA_TRY(cudaMemcpyAsync(deviances, c->dev.ptr, sizeof(double) * (size_t)nd,
                                 cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    *n_deviances = nd;
    *n_iter = ni;
    return NMFCU_OK;
}

// The host-buffer run shared by nmfcu_run, nmfcu_run_offset and
// nmfcu_run_weighted.
nmfcu_status run_host(const nmfcu_options *opt, int64_t n, int64_t p, int64_t r,
                      const double *V, const double *weight, const double *W0,
                      const double *H0, const double *offset0, double *W, double *H,
                      double *offset, double *deviances, int64_t deviances_cap,
                      int64_t *n_deviances, int64_t *n_iter) {
    if (opt && r > NMFCU_MAX_RANK)
        return run_host_wide(opt, n, p, r, V, W0, H0, W, H, deviances, deviances_cap,
                             n_deviances, n_iter);
    NMF_TRY(validate_options(opt, n, p, r));
    if (!V || !W0 || !H0 || !W || !H || !n_deviances || !n_iter)
        return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    const bool snmf = opt->method == NMFCU_SNMF_R || opt->method == NMFCU_SNMF_L;
    if (snmf && (!deviances || deviances_cap < opt->max_iter))
        return fail(NMFCU_ERR_INVALID_ARG,
                    "snmf records a deviance every iteration: deviances must hold max_iter values");
    const bool ls = opt->method == NMFCU_LSNMF;
    if (ls && !weight)  // py_nmf_run, lib.rs:1967-1971
        return fail(NMFCU_ERR_INVALID_ARG,
                    "method='lsnmf' requires a `weight` matrix of the same shape as V "
                    "(nmfcu_run_weighted)");
    const bool stat = opt->stop == NMFCU_STOP_STATIONARY;
    if (stat && (!deviances || deviances_cap < opt->max_iter + 1))
        return fail(NMFCU_ERR_INVALID_ARG, "deviances must hold max_iter + 1 values");
    nmfcu_context *c = nullptr;
    NMF_TRY(default_context(opt->device, &c));
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    cudaStream_t s = c->own_stream;
    const Plan pl = make_plan(n, p, r, c->sms);
    const bool f32 = f32_form(opt), tc = tc_form(opt);
    NMF_TRY(ensure_workspace(c, pl, f32, tc, opt->method, tcr_form(opt)));
    if (stat) NMF_TRY(c->dev.ensure(sizeof(double) * (size_t)(opt->max_iter + 1)));
    int64_t ldv = 0, ld32 = 0;
    NMF_TRY(upload_v(c, V, n, p, &ldv, s));
    if (f32) NMF_TRY(make_f32(c, c->V64.as<double>(), ldv, n, p, &ld32, s));
    NMF_TRY(put_factors(c, pl, W0, H0, cudaMemcpyHostToDevice, s));
    RunArgs a;
    a.opt = opt;
    a.pl = pl;
    a.ops = ops_for(pl.RP);
    const bool ratio = (opt->method == NMFCU_BRUNET || opt->method == NMFCU_NSNMF);
    const double *wsrc = (opt->method == NMFCU_NSNMF) ? c->Wns.as<double>() : nullptr;
    NMF_TRY(make_passset(c, pl, false, ratio, c->V64.ptr, ldv, &a.p64, wsrc));
    if (tc)
        NMF_TRY(make_tc_passset(c, pl, c->V64.as<double>(), ldv, s, &a.main));
    else if (f32)
        NMF_TRY(make_passset(c, pl, true, ratio, c->V32.ptr, ld32, &a.main));
    else
        a.main = a.p64;
    if (tcr_form(opt)) NMF_TRY(add_tcr_passes(c, pl, c->V32.ptr, ld32, &a.main));
    a.V64 = c->V64.as<double>();
    a.ldv64 = ldv;
    a.W = c->W.as<double>();
    a.H = c->H.as<double>();
    a.dev = stat ? c->dev.as<double>() : nullptr;
    if (ls) {
        // S next to V with V's pitch, then V <- V o S (lib.rs:961).
        NMF_TRY(c->S64.ensure(sizeof(double) * (size_t)(n * ldv)));
        if (n > 0 && p > 0) {
            CUDA_TRY(cudaMemcpy2DAsync(c->S64.ptr, ldv * 8, weight, p * 8, p * 8, n,
                                       cudaMemcpyHostToDevice, s));
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
            mul_weight<<<grid_for(n * p), kThreads, 0, s>>>(c->V64.as<double>(),
                                                            c->S64.as<double>(), ldv, (int)n,
                                                            (int)p);
        }
        a.S64 = c->S64.as<double>();
        a.NH = c->NH.as<double>();
        a.NW = c->NW.as<double>();
        NMF_TRY(make_passset(c, pl, false, true, c->S64.ptr, ldv, &a.pden));
    }
    NMF_TRY(setup_method(c, pl, opt, a, offset0, true, s));
    int64_t nd = 0, ni = 0;
    if (snmf) {
        NMF_TRY(c->dev.ensure(sizeof(double) * (size_t)std::max<int64_t>(1, opt->max_iter)));
        NMF_TRY(run_snmf(c, a, s, c->dev.as<double>()));
        ni = nd = opt->max_iter;
        NMF_TRY(get_factors(c, pl, W, H, cudaMemcpyDeviceToHost, s));
        if (nd > 0)
            CUDA_TRY(cudaMemcpyAsync(deviances, c->dev.ptr, sizeof(double) * (size_t)nd,
                                     cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        *n_deviances = nd;
        *n_iter = ni;
        return NMFCU_OK;
    }
    NMF_TRY(run_loop(c, a, s, &nd, &ni));
    NMF_TRY(get_factors(c, pl, W, H, cudaMemcpyDeviceToHost, s));
    if (offset && opt->method == NMFCU_OFFSET && n > 0)
        CUDA_TRY(cudaMemcpyAsync(offset, a.off, sizeof(double) * (size_t)n,
                                 cudaMemcpyDeviceToHost, s));
    if (stat && nd > 0)
        CUDA_TRY(cudaMemcpyAsync(deviances, c->dev.ptr, sizeof(double) * (size_t)nd,
                                 cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    *n_deviances = nd;
    *n_iter = ni;
    return NMFCU_OK;
}

}  // namespace

extern "C" {

nmfcu_status nmfcu_run(const nmfcu_options *opt, int64_t n, int64_t p, int64_t r,
                       const double *V, const double *W0, const double *H0, double *W,
                       double *H, double *deviances, int64_t deviances_cap,
                       int64_t *n_deviances, int64_t *n_iter) {
    return run_host(opt, n, p, r, V, nullptr, W0, H0, nullptr, W, H, nullptr, deviances,
                    deviances_cap, n_deviances, n_iter);
}

nmfcu_status nmfcu_run_weighted(const nmfcu_options *opt, int64_t n, int64_t p, int64_t r,
                                const double *V, const double *weight, const double *W0,
                                const double *H0, double *W, double *H, double *deviances,
                                int64_t deviances_cap, int64_t *n_deviances, int64_t *n_iter) {
    if (!opt) return fail(NMFCU_ERR_INVALID_ARG, "NULL options");
    if (opt->method != NMFCU_LSNMF)
        return fail(NMFCU_ERR_INVALID_ARG, "nmfcu_run_weighted runs method NMFCU_LSNMF only");
    if (!weight && n > 0 && p > 0) return fail(NMFCU_ERR_INVALID_ARG, "NULL weight");
    static const double kNone = 0.0;
    return run_host(opt, n, p, r, V, weight ? weight : &kNone, W0, H0, nullptr, W, H, nullptr,
                    deviances, deviances_cap, n_deviances, n_iter);
}

nmfcu_status nmfcu_run_offset(const nmfcu_options *opt, int64_t n, int64_t p, int64_t r,
                              const double *V, const double *W0, const double *H0,
                              const double *offset0, double *W, double *H, double *offset,
                              double *deviances, int64_t deviances_cap, int64_t *n_deviances,
                              int64_t *n_iter) {
    if (!opt) return fail(NMFCU_ERR_INVALID_ARG, "NULL options");
    if (opt->method != NMFCU_OFFSET)
        return fail(NMFCU_ERR_INVALID_ARG, "nmfcu_run_offset runs method NMFCU_OFFSET only");
    if (!offset && n > 0) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    return run_host(opt, n, p, r, V, nullptr, W0, H0, offset0, W, H, offset, deviances,
                    deviances_cap, n_deviances, n_iter);
}

nmfcu_status nmfcu_update_h_divergence(int64_t n, int64_t p, int64_t r, const double *V,
                                       const double *W, const double *H, double *H_out) {
    return single_step(STEP_H_KL, n, p, r, V, W, H, 0.0, H_out);
}
nmfcu_status nmfcu_update_w_divergence(int64_t n, int64_t p, int64_t r, const double *V,
                                       const double *W, const double *H, double *W_out) {
    return single_step(STEP_W_KL, n, p, r, V, W, H, 0.0, W_out);
}
nmfcu_status nmfcu_update_h_euclidean(int64_t n, int64_t p, int64_t r, const double *V,
                                      const double *W, const double *H, double eps,
                                      double *H_out) {
    return single_step(STEP_H_EUC, n, p, r, V, W, H, eps, H_out);
}
nmfcu_status nmfcu_update_w_euclidean(int64_t n, int64_t p, int64_t r, const double *V,
                                      const double *W, const double *H, double eps,
                                      double *W_out) {
    return single_step(STEP_W_EUC, n, p, r, V, W, H, eps, W_out);
}

nmfcu_status nmfcu_divergence(int64_t n, int64_t p, int64_t r, const double *V, const double *W,
                              const double *H, double *out) {
    return objective_host(true, n, p, r, V, W, H, out);
}
nmfcu_status nmfcu_distance(int64_t n, int64_t p, int64_t r, const double *V, const double *W,
                            const double *H, double *out) {
    return objective_host(false, n, p, r, V, W, H, out);
}

nmfcu_status nmfcu_smoothing_matrix(int64_t r, double theta, double *S) {
    if (r < 0) return fail(NMFCU_ERR_INVALID_ARG, "rank must be >= 0");
    if (r > 0 && !S) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    // smoothing_matrix, lib.rs:458-466.
    const double off = theta / (double)r;
    const double diag = (1.0 - theta) + off;
    for (int64_t i = 0; i < r; i++)
        for (int64_t j = 0; j < r; j++) S[i * r + j] = (i == j) ? diag : off;
    return NMFCU_OK;
}

int32_t nmfcu_set_num_threads(int64_t n) {
    (void)n;
    return 0;
}

nmfcu_status nmfcu_context_create(int32_t device, nmfcu_context **ctx) {
    if (!ctx) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    *ctx = nullptr;
    NMF_TRY(check_device(device));
    std::unique_ptr<nmfcu_context> c(new nmfcu_context());
    DeviceGuard dg(device);
    NMF_TRY(context_init(c.get(), device));
    *ctx = c.release();
    return NMFCU_OK;
}

void nmfcu_context_destroy(nmfcu_context *ctx) { delete ctx; }

}  // extern "C"

namespace {
// nmfcu_run_device, and with `d_off` the offset method's run on device
// pointers (d_off0: the starting row offsets, or NULL for rowMeans(V);
// d_off receives the final ones).
nmfcu_status run_device_impl(nmfcu_context *c, const nmfcu_options *opt, int64_t n, int64_t p,
                             int64_t r, const void *dV, int32_t v_dtype, int64_t ldv,
                             const double *dV64, int64_t ldv64, double *dW, double *dH,
                             const double *d_off0, double *d_off, double *d_dev,
                             int64_t *n_deviances, int64_t *n_iter, void *stream) {
    if (!c) return fail(NMFCU_ERR_INVALID_ARG, "NULL context");
    if (opt && r > NMFCU_MAX_RANK) {
        // Ranks above the streaming passes' buckets: the FP64 wide loop.
        NMF_TRY(nmfcu_internal::wide_validate(opt, n, p, r));
        if (!dV || !dW || !dH || !n_deviances || !n_iter)
            return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
        if (v_dtype != NMFCU_F64)
            return fail(NMFCU_ERR_INVALID_ARG, "ranks above 32 run in FP64: pass an f64 V");
        if (ldv < p) return fail(NMFCU_ERR_INVALID_ARG, "ldv must be >= p");
        const bool stat = opt->stop == NMFCU_STOP_STATIONARY;
        if (stat && !d_dev) return fail(NMFCU_ERR_INVALID_ARG, "stationary stop needs d_dev");
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard dg(c->device);
        cudaStream_t s = (cudaStream_t)stream;
        const double *V64 = (const double *)dV;
        int64_t ld64 = ldv;
        if (!tma_layout_ok(V64, ld64, 8)) {
            const int64_t ld = std::max<int64_t>(16, round_up(p, 16));
            NMF_TRY(c->V64.ensure(sizeof(double) * (size_t)(n * ld)));
            if (n > 0 && p > 0)
                CUDA_TRY(cudaMemcpy2DAsync(c->V64.ptr, ld * 8, V64, ld64 * 8, p * 8, n,
                                           cudaMemcpyDeviceToDevice, s));
            V64 = c->V64.as<double>();
            ld64 = ld;
        }
        return nmfcu_internal::wide_run(c, opt, n, p, r, V64, ld64, dW, dH, dW, dH,
                                        cudaMemcpyDeviceToDevice, cudaMemcpyDeviceToDevice,
                                        stat ? d_dev : nullptr, s, n_deviances, n_iter);
    }
    NMF_TRY(validate_options(opt, n, p, r));
    if (opt->method == NMFCU_OFFSET && !d_off)
        return fail(NMFCU_ERR_UNSUPPORTED,
                    "the offset method returns its row offsets: run it through "
                    "nmfcu_run_offset or nmfcu_run_offset_device");
    if (opt->method == NMFCU_LSNMF)
        return fail(NMFCU_ERR_UNSUPPORTED,
                    "lsNMF takes a weight matrix: run it through nmfcu_run_weighted");
    if (opt->method == NMFCU_SNMF_R || opt->method == NMFCU_SNMF_L)
        return fail(NMFCU_ERR_UNSUPPORTED, "snmf/r and snmf/l run through nmfcu_run");
    if (!dV || !dW || !dH || !n_deviances || !n_iter)
        return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    if (v_dtype != NMFCU_F64 && v_dtype != NMFCU_F32)
        return fail(NMFCU_ERR_INVALID_ARG, "v_dtype must be NMFCU_F64 or NMFCU_F32");
    if (ldv < p) return fail(NMFCU_ERR_INVALID_ARG, "ldv must be >= p");
    const bool f32 = f32_form(opt), tc = tc_form(opt);
    const bool stat = opt->stop == NMFCU_STOP_STATIONARY;
    if (!f32 && v_dtype != NMFCU_F64 && !(tc && dV64))
        return fail(NMFCU_ERR_INVALID_ARG, "precision FP64 and the split-bf16 form need an f64 V");
    const double *V64 = (v_dtype == NMFCU_F64) ? (const double *)dV : dV64;
    int64_t ld64 = (v_dtype == NMFCU_F64) ? ldv : ldv64;
    if (V64 && dV64 && v_dtype == NMFCU_F32 && ldv64 < p)
        return fail(NMFCU_ERR_INVALID_ARG, "ldv64 must be >= p");
    if (f32 && (stat || opt->refine_iters > 0) && !V64)
        return fail(NMFCU_ERR_INVALID_ARG,
                    "precision FP32 with a stationary stop or refinement needs the f64 V (dV64)");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    cudaStream_t s = (cudaStream_t)stream;
    const Plan pl = make_plan(n, p, r, c->sms);
    NMF_TRY(ensure_workspace(c, pl, f32, tc, opt->method, tcr_form(opt)));
    // The streaming passes read V through TMA, which needs a 16-byte aligned
    // base and row pitch; a V that is not laid out so is copied into the
    // context's pitched buffer first.
    if (V64 && !tma_layout_ok(V64, ld64, 8)) {
        const int64_t ld = std::max<int64_t>(16, round_up(p, 16));
        NMF_TRY(c->V64.ensure(sizeof(double) * (size_t)(n * ld)));
        if (n > 0 && p > 0)
            CUDA_TRY(cudaMemcpy2DAsync(c->V64.ptr, ld * 8, V64, ld64 * 8, p * 8, n,
                                       cudaMemcpyDeviceToDevice, s));
        V64 = c->V64.as<double>();
        ld64 = ld;
    }
    const void *Vmain = (v_dtype == NMFCU_F64) ? (const void *)V64 : dV;
    int64_t ldmain = (v_dtype == NMFCU_F64) ? ld64 : ldv;
    if (f32 && v_dtype == NMFCU_F64) {
        int64_t ld32 = 0;
        NMF_TRY(make_f32(c, V64, ld64, n, p, &ld32, s));
        Vmain = c->V32.ptr;
        ldmain = ld32;
    } else if (f32 && !tma_layout_ok(dV, ldv, 4)) {
        const int64_t ld = std::max<int64_t>(32, round_up(p, 32));
        NMF_TRY(c->V32.ensure(sizeof(float) * (size_t)(n * ld)));
        if (n > 0 && p > 0)
            CUDA_TRY(cudaMemcpy2DAsync(c->V32.ptr, ld * 4, dV, ldv * 4, p * 4, n,
                                       cudaMemcpyDeviceToDevice, s));
        Vmain = c->V32.ptr;
        ldmain = ld;
    }
    NMF_TRY(put_factors(c, pl, dW, dH, cudaMemcpyDeviceToDevice, s));
    RunArgs a;
    a.opt = opt;
    a.pl = pl;
    a.ops = ops_for(pl.RP);
    const bool ratio = (opt->method == NMFCU_BRUNET || opt->method == NMFCU_NSNMF);
    const double *wsrc = (opt->method == NMFCU_NSNMF) ? c->Wns.as<double>() : nullptr;
    if (V64) NMF_TRY(make_passset(c, pl, false, ratio, V64, ld64, &a.p64, wsrc));
    if (tc)
        NMF_TRY(make_tc_passset(c, pl, V64, ld64, s, &a.main));
    else if (f32)
        NMF_TRY(make_passset(c, pl, true, ratio, Vmain, ldmain, &a.main));
    else
        a.main = a.p64;
    if (tcr_form(opt)) NMF_TRY(add_tcr_passes(c, pl, Vmain, ldmain, &a.main));
    if (f32 && !V64) {
        // No f64 V: no refinement iterations and no objective (checked above).
        a.p64 = a.main;
    }
    a.V64 = V64;
    a.ldv64 = ld64;
    a.W = c->W.as<double>();
    a.H = c->H.as<double>();
    a.dev = stat ? d_dev : nullptr;
    if (stat && !d_dev) return fail(NMFCU_ERR_INVALID_ARG, "stationary stop needs d_dev");
    if (opt->method == NMFCU_OFFSET && !V64)
        return fail(NMFCU_ERR_INVALID_ARG, "the offset method needs the f64 V (dV64)");
    NMF_TRY(setup_method(c, pl, opt, a, d_off0, false, s));
    int64_t nd = 0, ni = 0;
    NMF_TRY(run_loop(c, a, s, &nd, &ni));
    NMF_TRY(get_factors(c, pl, dW, dH, cudaMemcpyDeviceToDevice, s));
    if (opt->method == NMFCU_OFFSET && n > 0)
        CUDA_TRY(cudaMemcpyAsync(d_off, a.off, sizeof(double) * (size_t)n,
                                 cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    *n_deviances = nd;
    *n_iter = ni;
    return NMFCU_OK;
}
}  // namespace

extern "C" {

nmfcu_status nmfcu_run_device(nmfcu_context *c, const nmfcu_options *opt, int64_t n, int64_t p,
                              int64_t r, const void *dV, int32_t v_dtype, int64_t ldv,
                              const double *dV64, int64_t ldv64, double *dW, double *dH,
                              double *d_dev, int64_t *n_deviances, int64_t *n_iter,
                              void *stream) {
    return run_device_impl(c, opt, n, p, r, dV, v_dtype, ldv, dV64, ldv64, dW, dH, nullptr,
                           nullptr, d_dev, n_deviances, n_iter, stream);
}

nmfcu_status nmfcu_run_offset_device(nmfcu_context *c, const nmfcu_options *opt, int64_t n,
                                     int64_t p, int64_t r, const void *dV, int32_t v_dtype,
                                     int64_t ldv, const double *dV64, int64_t ldv64, double *dW,
                                     double *dH, const double *d_offset0, double *d_offset,
                                     double *d_dev, int64_t *n_deviances, int64_t *n_iter,
                                     void *stream) {
    if (!opt) return fail(NMFCU_ERR_INVALID_ARG, "NULL options");
    if (opt->method != NMFCU_OFFSET)
        return fail(NMFCU_ERR_INVALID_ARG, "nmfcu_run_offset_device runs method NMFCU_OFFSET only");
    if (!d_offset) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    return run_device_impl(c, opt, n, p, r, dV, v_dtype, ldv, dV64, ldv64, dW, dH, d_offset0,
                           d_offset, d_dev, n_deviances, n_iter, stream);
}

int64_t nmfcu_shard_reduce_len(int64_t n, int64_t r) {
    const int RP = (r >= 1 && r <= NMFCU_MAX_RANK) ? bucket_for(r) : 0;
    if (RP == 0 || n < 0) return 0;
    return n * RP + (int64_t)RP * RP + RP;
}

nmfcu_status nmfcu_shard_create(nmfcu_context *c, const nmfcu_options *opt, int64_t n,
                                int64_t p_local, int64_t r, const double *dV, int64_t ldv,
                                const double *dW0, const double *dH0, double *dReduce,
                                double *dObjective, nmfcu_shard **out, void *stream) {
    if (!c || !out) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    *out = nullptr;
    NMF_TRY(validate_options(opt, n, p_local, r));
    switch (opt->method) {
        case NMFCU_BRUNET: case NMFCU_LEE: case NMFCU_HALS: case NMFCU_DNMF: break;
        default:
            return fail(NMFCU_ERR_UNSUPPORTED,
                        "column shards run brunet, lee, hals and dnmf");
    }
    if (!dW0 || !dReduce || !dObjective || (p_local > 0 && (!dV || !dH0)))
        return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    if (ldv < p_local) return fail(NMFCU_ERR_INVALID_ARG, "ldv must be >= p_local");
    if (p_local > 0 && !tma_layout_ok(dV, ldv, 8))
        return fail(NMFCU_ERR_INVALID_ARG,
                    "the shard's V must be 16-byte aligned with a 16-byte row pitch");
    std::unique_ptr<nmfcu_shard> sh(new nmfcu_shard());
    sh->c = c;
    sh->opt = *opt;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    cudaStream_t s = (cudaStream_t)stream;
    const nmfcu_options *o = &sh->opt;
    const Plan pl = make_plan(n, p_local, r, c->sms);
    const bool f32 = f32_form(o), tc = tc_form(o);
    const bool stat = o->stop == NMFCU_STOP_STATIONARY;
    NMF_TRY(ensure_workspace(c, pl, f32, tc, o->method, tcr_form(o)));
    if (stat) NMF_TRY(c->dev.ensure(sizeof(double) * (size_t)(o->max_iter + 1)));
    NMF_TRY(put_factors(c, pl, dW0, dH0, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaMemsetAsync(c->state.ptr, 0, sizeof(RunState), s));
    CUDA_TRY(cudaMemsetAsync(dReduce, 0, sizeof(double) * (size_t)nmfcu_shard_reduce_len(n, r), s));
    RunArgs &a = sh->a;
    a.opt = o;
    a.pl = pl;
    a.ops = ops_for(pl.RP);
    const bool ratio = (o->method == NMFCU_BRUNET);
    NMF_TRY(make_passset(c, pl, false, ratio, dV, ldv, &a.p64));
    if (tc) {
        NMF_TRY(make_tc_passset(c, pl, dV, ldv, s, &a.main));
    } else if (f32) {
        int64_t ld32 = 0;
        NMF_TRY(make_f32(c, dV, ldv, n, p_local, &ld32, s));
        NMF_TRY(make_passset(c, pl, true, ratio, c->V32.ptr, ld32, &a.main));
        if (tcr_form(o)) NMF_TRY(add_tcr_passes(c, pl, c->V32.ptr, ld32, &a.main));
    } else {
        a.main = a.p64;
    }
    a.V64 = dV;
    a.ldv64 = ldv;
    a.W = c->W.as<double>();
    a.H = c->H.as<double>();
    a.dev = stat ? c->dev.as<double>() : nullptr;
    sh->pl = pl;
    sh->R = dReduce;
    sh->Robj = dObjective;
    sh->refine_from =
        (o->precision != NMFCU_PREC_FP64) ? (long long)o->max_iter - o->refine_iters : LLONG_MAX;
    CUDA_TRY(cudaGetLastError());
    *out = sh.release();
    return NMFCU_OK;
}

nmfcu_status nmfcu_shard_step(nmfcu_shard *sh, int32_t phase, void *stream) {
    if (!sh) return fail(NMFCU_ERR_INVALID_ARG, "NULL shard");
    nmfcu_context *c = sh->c;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    cudaStream_t s = (cudaStream_t)stream;
    const nmfcu_options *o = &sh->opt;
    const RunArgs &a = sh->a;
    const Plan &pl = sh->pl;
    RunState *st = c->state.as<RunState>();
    double *Rnum = sh->R;
    double *RG = Rnum + (size_t)pl.n * pl.RP;
    double *Rs = RG + (size_t)pl.RP * pl.RP;
    switch (phase) {
        case NMFCU_SHARD_HALF_STEP: {
            // The H update on this shard's columns (W replicated), then this
            // shard's terms of H H^T / rowSums(H) and of the W contraction.
            const long long itn = sh->it + 1;
            if (itn > o->max_iter) return fail(NMFCU_ERR_INVALID_ARG, "max_iter reached");
            const bool fp64 = (o->precision == NMFCU_PREC_FP64) || (itn > sh->refine_from);
            const PassSet &ps = fp64 ? a.p64 : a.main;
            const bool ratio = (o->method == NMFCU_BRUNET);
            double *Gw = c->Gw.as<double>(), *sw = c->sw.as<double>();
            gram_w_full(c, a, Gw, sw, s);
            NMF_TRY(h_step(c, a, ps, epi(o, pl.r, Gw, sw, true), ratio, s));
            gram_h_full(c, a, RG, Rs, s);
            RunArgs aw = a;
            aw.Wout = Rnum;
            EpiParams ep = epi(o, pl.r, nullptr, nullptr, false);
            ep.method = nmfcu::M_PRODUCT;
            NMF_TRY(w_step(c, aw, ps, ep, ratio, s));
            break;
        }
        case NMFCU_SHARD_W_UPDATE: {
            // The W update from the contraction and Grams summed over shards;
            // every shard applies it to its identical copy of W.
            const long long itn = sh->it + 1;
            {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->w_apply(a.W, pl.n, Rnum, epi(o, pl.r, RG, Rs, false), st, s);
            }
            if (o->method == NMFCU_BRUNET && itn % 10 == 0) {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->clamp(a.W, a.H, pl.n, pl.p, pl.r, DBL_EPSILON, st, s);
            } else if (o->method == NMFCU_LEE && o->rescale) {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER, 2);
                a.ops->gram_w(a.W, pl.n, pl.Bw, pl.rows_per_gram, c->pg.as<double>(),
                              c->ps.as<double>(), st, s);
                a.ops->rescale(a.W, pl.n, pl.r, c->ps.as<double>(), pl.Bw, st, s);
            } else if (o->method == NMFCU_DNMF) {
                gram_w_full(c, a, c->Gw2.as<double>(), c->sw2.as<double>(), s);
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->dnmf_scale(a.W, a.H, pl.n, pl.p, pl.r, c->Gw2.as<double>(), RG, st, s);
            }
            sh->it = itn;
            break;
        }
        case NMFCU_SHARD_OBJECTIVE: {
            if (o->stop != NMFCU_STOP_STATIONARY)
                return fail(NMFCU_ERR_INVALID_ARG, "the objective runs with stop stationary");
            NMF_TRY(enqueue_objective_partials(c, a, s));
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
            sum_partials<<<1, kThreads, 0, s>>>(c->obj.as<double>(),
                                                pl.n > 0 ? pl.obj_blocks : 0, sh->Robj);
            break;
        }
        case NMFCU_SHARD_STOP: {
            if (o->stop != NMFCU_STOP_STATIONARY)
                return fail(NMFCU_ERR_INVALID_ARG, "the stop test runs with stop stationary");
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
            objective_finalize<<<1, kThreads, 0, s>>>(sh->Robj, 1, a.dev,
                                                      stop_params(o, sh->it), st);
            break;
        }
        default: return fail(NMFCU_ERR_INVALID_ARG, "unknown shard phase");
    }
    CUDA_TRY(cudaGetLastError());
    return NMFCU_OK;
}

nmfcu_status nmfcu_shard_status(nmfcu_shard *sh, int64_t *n_iter, int32_t *stopped, void *stream) {
    if (!sh || !n_iter || !stopped) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    nmfcu_context *c = sh->c;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    NMF_TRY(finish_checked(c, (cudaStream_t)stream));
    const RunState &hs = *c->h_state;
    if (hs.error == 1)
        return fail(NMFCU_ERR_INVALID_ARG,
                    "check_interval must be > 0 (the stationary stop evaluates iter % check_interval)");
    *stopped = hs.stopped ? 1 : 0;
    *n_iter = hs.stopped ? hs.n_iter : sh->it;
    return NMFCU_OK;
}

nmfcu_status nmfcu_shard_result(nmfcu_shard *sh, double *dW, double *dH, double *d_dev,
                                int64_t *n_deviances, int64_t *n_iter, void *stream) {
    if (!sh || !dW || !n_deviances || !n_iter || (sh->pl.p > 0 && !dH))
        return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    int32_t stopped = 0;
    NMF_TRY(nmfcu_shard_status(sh, n_iter, &stopped, stream));
    nmfcu_context *c = sh->c;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    cudaStream_t s = (cudaStream_t)stream;
    NMF_TRY(get_factors(c, sh->pl, dW, dH, cudaMemcpyDeviceToDevice, s));
    const bool stat = sh->opt.stop == NMFCU_STOP_STATIONARY;
    *n_deviances = stat ? *n_iter + 1 : 0;
    if (stat && d_dev && *n_deviances > 0)
        CUDA_TRY(cudaMemcpyAsync(d_dev, c->dev.ptr, sizeof(double) * (size_t)*n_deviances,
                                 cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return NMFCU_OK;
}

void nmfcu_shard_destroy(nmfcu_shard *sh) { delete sh; }

extern "C++" {
namespace nmfcu_internal {
// out = V X (trans 0) or V^T X (trans 1) with the context locked and its
// device current; see nmfcu_v_product_device.  `reset_state` clears the
// context's run state first (a standalone product); a caller that keeps its
// own loop's stop state there passes false, and the passes then do no work
// once that loop has stopped.  `sync` waits for the stream and reports a
// streaming kernel that gave up waiting.
nmfcu_status v_product_locked(nmfcu_context *c, int32_t trans, int64_t n, int64_t p, int64_t l,
                              const double *dV, int64_t ldv, const double *dX, int64_t ldx,
                              double *dOut, int64_t ldo, cudaStream_t s, bool reset_state,
                              bool sync);
void *context_state(nmfcu_context *c) { return c->state.ptr; }
}  // namespace nmfcu_internal
}  // extern "C++"

nmfcu_status nmfcu_v_product_device(nmfcu_context *c, int32_t trans, int64_t n, int64_t p,
                                    int64_t l, const double *dV, int64_t ldv, const double *dX,
                                    int64_t ldx, double *dOut, int64_t ldo, void *stream) {
    if (!c) return fail(NMFCU_ERR_INVALID_ARG, "NULL context");
    if (trans != 0 && trans != 1) return fail(NMFCU_ERR_INVALID_ARG, "trans must be 0 or 1");
    if (n < 0 || p < 0 || l < 0) return fail(NMFCU_ERR_INVALID_ARG, "negative dimension");
    if (n > INT32_MAX || p > INT32_MAX)
        return fail(NMFCU_ERR_UNSUPPORTED, "n and p must each fit in 32 bits");
    if (ldv < p || ldx < l || ldo < l)
        return fail(NMFCU_ERR_INVALID_ARG, "leading dimensions must be >= the row lengths");
    const int64_t xrows = trans ? n : p, orows = trans ? p : n;
    if (l == 0 || orows == 0) return NMFCU_OK;
    if (!dOut || (xrows > 0 && (!dV || !dX))) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    return nmfcu_internal::v_product_locked(c, trans, n, p, l, dV, ldv, dX, ldx, dOut, ldo,
                                            (cudaStream_t)stream, true, true);
}

extern "C++" nmfcu_status nmfcu_internal::v_product_locked(nmfcu_context *c, int32_t trans, int64_t n,
                                              int64_t p, int64_t l, const double *dV, int64_t ldv,
                                              const double *dX, int64_t ldx, double *dOut,
                                              int64_t ldo, cudaStream_t s, bool reset_state,
                                              bool sync) {
    const int64_t xrows = trans ? n : p, orows = trans ? p : n;
    if (l == 0 || orows == 0) return NMFCU_OK;
    if (xrows == 0) {  // an empty sum: the product is zero
        CUDA_TRY(cudaMemset2DAsync(dOut, ldo * 8, 0, l * 8, orows, s));
        if (sync) CUDA_TRY(cudaStreamSynchronize(s));
        return NMFCU_OK;
    }
    // TMA needs a 16-byte aligned base and row pitch: otherwise V is copied
    // into the context's pitched buffer once for all column chunks.
    if (!tma_layout_ok(dV, ldv, 8)) {
        const int64_t ld = std::max<int64_t>(16, round_up(p, 16));
        NMF_TRY(c->V64.ensure(sizeof(double) * (size_t)(n * ld)));
        CUDA_TRY(cudaMemcpy2DAsync(c->V64.ptr, ld * 8, dV, ldv * 8, p * 8, n,
                                   cudaMemcpyDeviceToDevice, s));
        dV = c->V64.as<double>();
        ldv = ld;
    }
    nmfcu_options o;
    nmfcu_options_default(&o);
    o.method = NMFCU_LEE;
    // Column chunks of at most the largest built rank; each is one pass over V.
    for (int64_t c0 = 0; c0 < l; c0 += NMFCU_MAX_RANK) {
        const int kc = (int)std::min<int64_t>(NMFCU_MAX_RANK, l - c0);
        const Plan pl = make_plan(n, p, kc, c->sms);
        NMF_TRY(ensure_workspace(c, pl, false));  // allocates the device state too
        if (c0 == 0 && reset_state) CUDA_TRY(cudaMemsetAsync(c->state.ptr, 0, sizeof(RunState), s));
        RunArgs a;
        a.opt = &o;
        a.pl = pl;
        a.ops = ops_for(pl.RP);
        NMF_TRY(make_passset(c, pl, false, false, dV, ldv, &a.p64));
        a.main = a.p64;
        a.V64 = dV;
        a.ldv64 = ldv;
        a.W = c->W.as<double>();
        a.H = c->H.as<double>();
        a.dev = nullptr;
        EpiParams e = epi(&o, kc, nullptr, nullptr, trans != 0);
        e.method = nmfcu::M_PRODUCT;
        if (trans) {
            // V^T X: X's columns as the H pass's W (n x RP); the product lands
            // in H (RP x p) and is transposed out.
            {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                pack_cols<<<grid_for(n * pl.RP), kThreads, 0, s>>>(dX, ldx, (int)n, (int)c0, kc,
                                                                   a.W, pl.RP);
            }
            NMF_TRY(h_step(c, a, a.p64, e, false, s));
            nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
            unpack_rows_t<<<grid_for(p * kc), kThreads, 0, s>>>(a.H, (int)p, kc, dOut, ldo,
                                                                (int)c0);
        } else {
            // V X: X's columns as the W pass's H^T (p x rps); the product lands
            // in W (n x RP).
            const int rps = a.p64.so->rps();
            {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                pack_cols<<<grid_for(p * rps), kThreads, 0, s>>>(
                    dX, ldx, (int)p, (int)c0, kc, static_cast<double *>(a.p64.Ht), rps);
            }
            NMF_TRY(w_step(c, a, a.p64, e, false, s));
            CUDA_TRY(cudaMemcpy2DAsync(dOut + c0, ldo * 8, a.W, (size_t)pl.RP * 8, (size_t)kc * 8,
                                       n, cudaMemcpyDeviceToDevice, s));
        }
    }
    return sync ? finish_checked(c, s) : NMFCU_OK;
}

nmfcu_status nmfcu_context_set_timing(nmfcu_context *ctx, int32_t enabled) {
    if (!ctx) return fail(NMFCU_ERR_INVALID_ARG, "NULL context");
    ctx->timing = enabled != 0;
    return NMFCU_OK;
}

nmfcu_status nmfcu_context_kernel_time(nmfcu_context *ctx, int32_t kclass, int64_t *launches,
                                       double *total_ms) {
    if (!ctx || !launches || !total_ms) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    if (kclass < 0 || kclass >= NMFCU_KCLASS_COUNT)
        return fail(NMFCU_ERR_INVALID_ARG, "kernel class out of range");
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    ctx->drain_timing();
    *launches = ctx->count[kclass];
    *total_ms = ctx->total_ms[kclass];
    return NMFCU_OK;
}

nmfcu_status nmfcu_context_reset_timing(nmfcu_context *ctx) {
    if (!ctx) return fail(NMFCU_ERR_INVALID_ARG, "NULL context");
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    ctx->drain_timing();
    for (int k = 0; k < NMFCU_KCLASS_COUNT; k++) {
        ctx->total_ms[k] = 0;
        ctx->count[k] = 0;
    }
    ctx->launch_total = 0;
    return NMFCU_OK;
}

int64_t nmfcu_context_launch_count(nmfcu_context *ctx) { return ctx ? ctx->launch_total : 0; }

const char *nmfcu_last_error(void) { return g_last_error.c_str(); }

const char *nmfcu_status_string(nmfcu_status s) {
    switch (s) {
        case NMFCU_OK: return "ok";
        case NMFCU_ERR_INVALID_ARG: return "invalid argument";
        case NMFCU_ERR_UNSUPPORTED: return "unsupported";
        case NMFCU_ERR_OOM: return "out of device memory";
        case NMFCU_ERR_CUDA: return "CUDA error";
        case NMFCU_ERR_NUMERIC: return "numeric error";
        case NMFCU_ERR_TIMEOUT: return "device wait timed out";
        case NMFCU_ERR_NO_DEVICE: return "no CUDA device";
        case NMFCU_ERR_CANCELLED: return "request cancelled";
    }
    return "unknown status";
}

int32_t nmfcu_abi_version(void) { return NMFCU_ABI_VERSION; }

int32_t nmfcu_device_count(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return count;
}

}  // extern "C"

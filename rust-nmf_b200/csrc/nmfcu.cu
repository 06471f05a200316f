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

#include "../../include/nmfcu.h"
#include "kernels.cuh"

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
// Rank buckets and per-bucket kernel launchers
// ===========================================================================
constexpr int kBuckets[] = {2, 4, 6, 8, 10, 12, 14, 16, 20, 24, 28, 32};

int bucket_for(int64_t r) {
    for (int b : kBuckets)
        if (r <= b) return b;
    return 0;
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// V element type of a pass.
enum VType { VT_F64 = 0, VT_F32 = 1 };

struct Ops {
    virtual ~Ops() = default;
    virtual void hstep(VType vt, const void *V, int64_t ldv, int n, int p, const double *W,
                       const double *H, bool ratio, int S, int rows_per_split, double *part,
                       const RunState *st, cudaStream_t s) const = 0;
    // mode 0 plain, 1 ratio, 2 KL objective, 3 Frobenius objective
    virtual void rowpass(VType vt, const void *V, int64_t ldv, int n, int p, const double *W,
                         const double *H, int mode, int S2, int cols_per_split, double *part,
                         double *obj, const RunState *st, cudaStream_t s) const = 0;
    virtual void h_epi(double *H, int p, const double *part, int S, const EpiParams &e,
                       const RunState *st, cudaStream_t s) const = 0;
    virtual void w_epi(double *W, int n, const double *part, int S, const EpiParams &e,
                       const RunState *st, cudaStream_t s) const = 0;
    virtual void gram_w(const double *W, int n, int B, int rows_per_block, double *pg,
                        double *ps, const RunState *st, cudaStream_t s) const = 0;
    virtual void gram_h(const double *H, int p, int B, int cols_per_block, double *pg,
                        double *ps, const RunState *st, cudaStream_t s) const = 0;
    virtual void gram_fin(const double *pg, const double *ps, int B, double *G, double *sums,
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
    void hstep(VType vt, const void *V, int64_t ldv, int n, int p, const double *W,
               const double *H, bool ratio, int S, int rows_per_split, double *part,
               const RunState *st, cudaStream_t s) const override {
        if (p <= 0 || S <= 0) return;
        dim3 grid(cdiv(p, 32), S), block(32, kWarps);
        if (vt == VT_F64) {
            if (ratio)
                hstep_contract<double, double, RP, true><<<grid, block, 0, s>>>(
                    (const double *)V, ldv, n, p, W, H, rows_per_split, part, st);
            else
                hstep_contract<double, double, RP, false><<<grid, block, 0, s>>>(
                    (const double *)V, ldv, n, p, W, H, rows_per_split, part, st);
        } else {
            if (ratio)
                hstep_contract<float, float, RP, true><<<grid, block, 0, s>>>(
                    (const float *)V, ldv, n, p, W, H, rows_per_split, part, st);
            else
                hstep_contract<float, float, RP, false><<<grid, block, 0, s>>>(
                    (const float *)V, ldv, n, p, W, H, rows_per_split, part, st);
        }
    }
    void rowpass(VType vt, const void *V, int64_t ldv, int n, int p, const double *W,
                 const double *H, int mode, int S2, int cols_per_split, double *part,
                 double *obj, const RunState *st, cudaStream_t s) const override {
        if (n <= 0 || S2 <= 0) return;
        dim3 grid(cdiv(n, kThreads), S2), block(kThreads);
        if (vt == VT_F64) {
            const double *v = (const double *)V;
            switch (mode) {
                case 0: nmfcu::rowpass<double, double, RP, 0><<<grid, block, 0, s>>>(v, ldv, n, p, W, H, cols_per_split, part, obj, st); break;
                case 1: nmfcu::rowpass<double, double, RP, 1><<<grid, block, 0, s>>>(v, ldv, n, p, W, H, cols_per_split, part, obj, st); break;
                case 2: nmfcu::rowpass<double, double, RP, 2><<<grid, block, 0, s>>>(v, ldv, n, p, W, H, cols_per_split, part, obj, st); break;
                default: nmfcu::rowpass<double, double, RP, 3><<<grid, block, 0, s>>>(v, ldv, n, p, W, H, cols_per_split, part, obj, st); break;
            }
        } else {
            const float *v = (const float *)V;
            switch (mode) {
                case 0: nmfcu::rowpass<float, float, RP, 0><<<grid, block, 0, s>>>(v, ldv, n, p, W, H, cols_per_split, part, obj, st); break;
                case 1: nmfcu::rowpass<float, float, RP, 1><<<grid, block, 0, s>>>(v, ldv, n, p, W, H, cols_per_split, part, obj, st); break;
                default: break;  // objectives always run on the f64 V
            }
        }
    }
    void h_epi(double *H, int p, const double *part, int S, const EpiParams &e,
               const RunState *st, cudaStream_t s) const override {
        if (p <= 0) return;
        h_epilogue<RP><<<cdiv(p, kThreads), kThreads, 0, s>>>(H, p, part, S, e, st);
    }
    void w_epi(double *W, int n, const double *part, int S, const EpiParams &e,
               const RunState *st, cudaStream_t s) const override {
        if (n <= 0) return;
        w_epilogue<RP><<<cdiv(n, kThreads), kThreads, 0, s>>>(W, n, part, S, e, st);
    }
    void gram_w(const double *W, int n, int B, int rows_per_block, double *pg, double *ps,
                const RunState *st, cudaStream_t s) const override {
        gram_w_partial<RP><<<B, RP * RP, 0, s>>>(W, n, rows_per_block, pg, ps, st);
    }
    void gram_h(const double *H, int p, int B, int cols_per_block, double *pg, double *ps,
                const RunState *st, cudaStream_t s) const override {
        gram_h_partial<RP><<<B, RP * RP, 0, s>>>(H, p, cols_per_block, pg, ps, st);
    }
    void gram_fin(const double *pg, const double *ps, int B, double *G, double *sums,
                  const RunState *st, cudaStream_t s) const override {
        gram_finalize<RP><<<1, RP * RP, 0, s>>>(pg, ps, B, G, sums, st);
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
    template <typename T>
    T *as() const { return static_cast<T *>(ptr); }
};

// Launch geometry of one problem shape.
struct Plan {
    int n = 0, p = 0, r = 0, RP = 0;
    int S = 1, rows_per_split = 1;     // H-step row splits
    int S2 = 1, cols_per_split = 1;    // W-step / objective column splits
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
    // H step: 32-column tiles, split rows until there are ~8 CTAs per SM.
    const int64_t tiles = std::max<int64_t>(1, (p + 31) / 32);
    int64_t S = std::max<int64_t>(1, (target + tiles - 1) / tiles);
    S = std::min<int64_t>(S, std::max<int64_t>(1, n / 64));
    int64_t rps = std::max<int64_t>(1, (n + S - 1) / S);
    pl.rows_per_split = (int)rps;
    pl.S = (int)std::max<int64_t>(1, (n + rps - 1) / rps);
    // W step: 256-row blocks, split columns in multiples of 32.
    const int64_t rb = std::max<int64_t>(1, (n + kThreads - 1) / kThreads);
    int64_t S2 = std::max<int64_t>(1, (target + rb - 1) / rb);
    S2 = std::min<int64_t>(S2, std::max<int64_t>(1, p / 256));
    int64_t cps = std::max<int64_t>(32, ((p + S2 - 1) / S2 + 31) / 32 * 32);
    pl.cols_per_split = (int)cps;
    pl.S2 = (int)std::max<int64_t>(1, (p + cps - 1) / cps);
    pl.obj_blocks = (int)(((n + kThreads - 1) / kThreads) * pl.S2);
    // Grams.
    pl.Bw = (int)std::max<int64_t>(1, std::min<int64_t>((n + 63) / 64, sms));
    pl.rows_per_gram = (int)std::max<int64_t>(1, (n + pl.Bw - 1) / pl.Bw);
    pl.Bh = (int)std::max<int64_t>(1, std::min<int64_t>((p + 63) / 64, sms));
    pl.cols_per_gram = (int)std::max<int64_t>(1, (p + pl.Bh - 1) / pl.Bh);
    return pl;
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

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
    DevBuf V64, V32, W, H, part_h, part_w, pg, ps, Gw, sw, Gh, sh, Gw2, sw2, obj, dev, state;
    // Pinned staging for the small run state.
    RunState *h_state = nullptr;

    // Timing.
    bool timing = false;
    struct Ev {
        cudaEvent_t a, b;
        int kclass;
    };
    std::vector<Ev> events;
    std::vector<cudaEvent_t> pool;
    int64_t launches = 0;
    double total_ms[NMFCU_KCLASS_COUNT] = {0, 0, 0, 0};
    int64_t count[NMFCU_KCLASS_COUNT] = {0, 0, 0, 0};
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

    // Bracket one launch for the timing hooks.
    struct Scope {
        nmfcu_context *c;
        cudaStream_t s;
        int kclass;
        cudaEvent_t a = nullptr;
        Scope(nmfcu_context *c_, cudaStream_t s_, int k) : c(c_), s(s_), kclass(k) {
            c->launch_total++;
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
            if (cudaEventSynchronize(e.b) == cudaSuccess && cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
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
// The iteration loop
// ===========================================================================
struct RunArgs {
    const nmfcu_options *opt;
    Plan pl;
    const Ops *ops;
    VType vt_main;          // element type of Vmain
    const void *Vmain;      // V used by the contractions (f64 or f32)
    int64_t ldv_main;
    const double *V64;      // f64 V for objective and refinement iterations
    int64_t ldv64;
    double *W, *H;          // padded device factors
    double *dev;            // device deviances (or nullptr)
};

nmfcu_status enqueue_objective(nmfcu_context *c, const RunArgs &a, long long iter,
                               cudaStream_t s) {
    const Plan &pl = a.pl;
    RunState *st = c->state.as<RunState>();
    const bool kl = (a.opt->method == NMFCU_BRUNET);
    {
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OBJECTIVE);
        a.ops->rowpass(VT_F64, a.V64, a.ldv64, pl.n, pl.p, a.W, a.H, kl ? 2 : 3, pl.S2,
                       pl.cols_per_split, nullptr, c->obj.as<double>(), st, s);
    }
    StopParams sp;
    sp.stationary = 1;
    sp.iter = iter;
    sp.check_interval = a.opt->check_interval;
    sp.check_niter = a.opt->check_niter;
    sp.threshold = a.opt->stationary_th;
    sp.scale = kl ? 1.0 : 0.5;
    {
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
        objective_finalize<<<1, kThreads, 0, s>>>(c->obj.as<double>(), pl.n > 0 ? pl.obj_blocks : 0,
                                                  a.dev, sp, st);
    }
    return NMFCU_OK;
}

// Gram + sums of W (or H) into G / sums.
void gram_w_full(nmfcu_context *c, const RunArgs &a, double *G, double *sums, cudaStream_t s) {
    const Plan &pl = a.pl;
    RunState *st = c->state.as<RunState>();
    nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
    a.ops->gram_w(a.W, pl.n, pl.Bw, pl.rows_per_gram, c->pg.as<double>(), c->ps.as<double>(), st, s);
    a.ops->gram_fin(c->pg.as<double>(), c->ps.as<double>(), pl.Bw, G, sums, st, s);
}
void gram_h_full(nmfcu_context *c, const RunArgs &a, double *G, double *sums, cudaStream_t s) {
    const Plan &pl = a.pl;
    RunState *st = c->state.as<RunState>();
    nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
    a.ops->gram_h(a.H, pl.p, pl.Bh, pl.cols_per_gram, c->pg.as<double>(), c->ps.as<double>(), st, s);
    a.ops->gram_fin(c->pg.as<double>(), c->ps.as<double>(), pl.Bh, G, sums, st, s);
}

// H step: contraction + epilogue.
void h_step(nmfcu_context *c, const RunArgs &a, VType vt, const void *V, int64_t ldv,
            const EpiParams &e, bool ratio, cudaStream_t s) {
    const Plan &pl = a.pl;
    RunState *st = c->state.as<RunState>();
    {
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_HSTEP);
        a.ops->hstep(vt, V, ldv, pl.n, pl.p, a.W, a.H, ratio, pl.S, pl.rows_per_split,
                     c->part_h.as<double>(), st, s);
    }
    nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
    a.ops->h_epi(a.H, pl.p, c->part_h.as<double>(), pl.p > 0 ? pl.S : 0, e, st, s);
}

// W step: contraction + epilogue.
void w_step(nmfcu_context *c, const RunArgs &a, VType vt, const void *V, int64_t ldv,
            const EpiParams &e, bool ratio, cudaStream_t s) {
    const Plan &pl = a.pl;
    RunState *st = c->state.as<RunState>();
    {
        nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_WSTEP);
        a.ops->rowpass(vt, V, ldv, pl.n, pl.p, a.W, a.H, ratio ? 1 : 0, pl.S2,
                       pl.cols_per_split, c->part_w.as<double>(), nullptr, st, s);
    }
    nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
    a.ops->w_epi(a.W, pl.n, c->part_w.as<double>(), pl.S2, e, st, s);
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
void enqueue_iteration(nmfcu_context *c, const RunArgs &a, long long it, bool fp64,
                       cudaStream_t s) {
    const Plan &pl = a.pl;
    const nmfcu_options *o = a.opt;
    RunState *st = c->state.as<RunState>();
    const VType vt = fp64 ? VT_F64 : a.vt_main;
    const void *V = fp64 ? (const void *)a.V64 : a.Vmain;
    const int64_t ldv = fp64 ? a.ldv64 : a.ldv_main;
    double *Gw = c->Gw.as<double>(), *sw = c->sw.as<double>();
    double *Gh = c->Gh.as<double>(), *sh = c->sh.as<double>();

    switch (o->method) {
        case NMFCU_BRUNET: {
            // nmf_run_brunet lib.rs:1558-1575.
            gram_w_full(c, a, Gw, sw, s);  // sum_w (lib.rs:1563-1568)
            h_step(c, a, vt, V, ldv, epi(o, pl.r, Gw, sw, true), true, s);
            gram_h_full(c, a, Gh, sh, s);  // sum_h (lib.rs:161-169)
            w_step(c, a, vt, V, ldv, epi(o, pl.r, Gh, sh, false), true, s);
            if (it % 10 == 0) {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->clamp(a.W, a.H, pl.n, pl.p, pl.r, DBL_EPSILON, st, s);
            }
            break;
        }
        case NMFCU_LEE: {
            // nmf_run_lee lib.rs:1618-1636.
            gram_w_full(c, a, Gw, sw, s);  // W^T W (lib.rs:1622-1631)
            h_step(c, a, vt, V, ldv, epi(o, pl.r, Gw, sw, true), false, s);
            gram_h_full(c, a, Gh, sh, s);  // H H^T (lib.rs:293-302)
            w_step(c, a, vt, V, ldv, epi(o, pl.r, Gh, sh, false), false, s);
            if (o->rescale) {
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->gram_w(a.W, pl.n, pl.Bw, pl.rows_per_gram, c->pg.as<double>(),
                              c->ps.as<double>(), st, s);
                a.ops->rescale(a.W, pl.n, pl.r, c->ps.as<double>(), pl.Bw, st, s);
            }
            break;
        }
        default: {
            // nmf_run_hals lib.rs:667-676; nmf_run_dnmf lib.rs:862-884.
            gram_w_full(c, a, Gw, sw, s);
            h_step(c, a, vt, V, ldv, epi(o, pl.r, Gw, sw, true), false, s);
            gram_h_full(c, a, Gh, sh, s);
            w_step(c, a, vt, V, ldv, epi(o, pl.r, Gh, sh, false), false, s);
            if (o->method == NMFCU_DNMF) {
                gram_w_full(c, a, c->Gw2.as<double>(), c->sw2.as<double>(), s);
                nmfcu_context::Scope sc(c, s, NMFCU_KCLASS_OTHER);
                a.ops->dnmf_scale(a.W, a.H, pl.n, pl.p, pl.r, c->Gw2.as<double>(), Gh, st, s);
            }
            break;
        }
    }
}

nmfcu_status ensure_workspace(nmfcu_context *c, const Plan &pl) {
    const size_t RP = pl.RP;
    NMF_TRY(c->W.ensure(sizeof(double) * (size_t)pl.n * RP));
    NMF_TRY(c->H.ensure(sizeof(double) * RP * (size_t)pl.p));
    NMF_TRY(c->part_h.ensure(sizeof(double) * (size_t)pl.S * RP * (size_t)pl.p));
    NMF_TRY(c->part_w.ensure(sizeof(double) * (size_t)pl.S2 * (size_t)pl.n * RP));
    const size_t B = (size_t)std::max(pl.Bw, pl.Bh);
    NMF_TRY(c->pg.ensure(sizeof(double) * B * RP * RP));
    NMF_TRY(c->ps.ensure(sizeof(double) * B * RP));
    NMF_TRY(c->Gw.ensure(sizeof(double) * RP * RP));
    NMF_TRY(c->Gh.ensure(sizeof(double) * RP * RP));
    NMF_TRY(c->Gw2.ensure(sizeof(double) * RP * RP));
    NMF_TRY(c->sw.ensure(sizeof(double) * RP));
    NMF_TRY(c->sh.ensure(sizeof(double) * RP));
    NMF_TRY(c->sw2.ensure(sizeof(double) * RP));
    NMF_TRY(c->obj.ensure(sizeof(double) * (size_t)std::max(pl.obj_blocks, 1)));
    NMF_TRY(c->state.ensure(sizeof(RunState)));
    if (!c->h_state) CUDA_TRY(cudaMallocHost((void **)&c->h_state, sizeof(RunState)));
    return NMFCU_OK;
}

nmfcu_status validate_options(const nmfcu_options *o, int64_t n, int64_t p, int64_t r) {
    if (!o) return fail(NMFCU_ERR_INVALID_ARG, "options pointer is NULL");
    if (n < 0 || p < 0) return fail(NMFCU_ERR_INVALID_ARG, "negative matrix dimension");
    if (r < 1) return fail(NMFCU_ERR_INVALID_ARG, "rank must be >= 1");
    if (n > INT32_MAX || p > INT32_MAX)
        return fail(NMFCU_ERR_UNSUPPORTED, "n and p must each fit in 32 bits");
    if (r > NMFCU_MAX_RANK)
        return fail(NMFCU_ERR_UNSUPPORTED,
                    "rank " + std::to_string(r) + " exceeds the largest built rank (" +
                        std::to_string(NMFCU_MAX_RANK) + ")");
    switch (o->method) {
        case NMFCU_BRUNET:
        case NMFCU_LEE:
        case NMFCU_HALS:
        case NMFCU_DNMF: break;
        case NMFCU_OFFSET: case NMFCU_NSNMF: case NMFCU_EHALS: case NMFCU_LSNMF:
        case NMFCU_SNMF_R: case NMFCU_SNMF_L:
            return fail(NMFCU_ERR_UNSUPPORTED,
                        "method is not built in the GPU engine (built: brunet, lee, hals, dnmf)");
        default: return fail(NMFCU_ERR_INVALID_ARG, "unknown method id");
    }
    if (o->stop != NMFCU_STOP_MAX_ITER && o->stop != NMFCU_STOP_STATIONARY)
        return fail(NMFCU_ERR_INVALID_ARG, "unknown stop id");
    if (o->precision != NMFCU_PREC_FP64 && o->precision != NMFCU_PREC_FP32)
        return fail(NMFCU_ERR_INVALID_ARG, "unknown precision id");
    if (o->max_iter < 0) return fail(NMFCU_ERR_INVALID_ARG, "max_iter must be >= 0");
    if (o->check_niter < 0 || o->check_interval < 0)
        return fail(NMFCU_ERR_INVALID_ARG, "check_interval / check_niter must be >= 0");
    if (o->refine_iters < 0) return fail(NMFCU_ERR_INVALID_ARG, "refine_iters must be >= 0");
    return NMFCU_OK;
}

// Runs the loop on prepared device buffers; fills n_iter / n_dev.
nmfcu_status run_loop(nmfcu_context *c, RunArgs &a, cudaStream_t s, int64_t *n_dev,
                      int64_t *n_iter) {
    const nmfcu_options *o = a.opt;
    const bool stat = (o->stop == NMFCU_STOP_STATIONARY);
    CUDA_TRY(cudaMemsetAsync(c->state.ptr, 0, sizeof(RunState), s));
    if (stat) NMF_TRY(enqueue_objective(c, a, 0, s));
    const long long refine_from =
        (o->precision == NMFCU_PREC_FP32) ? (long long)o->max_iter - o->refine_iters : LLONG_MAX;
    for (long long it = 1; it <= o->max_iter; it++) {
        const bool fp64 = (o->precision == NMFCU_PREC_FP64) || (it > refine_from);
        enqueue_iteration(c, a, it, fp64, s);
        if (stat) NMF_TRY(enqueue_objective(c, a, it, s));
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(c->h_state, c->state.ptr, sizeof(RunState), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (c->timing) c->drain_timing();
    const RunState &hs = *c->h_state;
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
    NMF_TRY(ensure_workspace(c, pl));
    int64_t ldv = 0;
    NMF_TRY(upload_v(c, V, n, p, &ldv, s));
    NMF_TRY(put_factors(c, pl, W, H, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemsetAsync(c->state.ptr, 0, sizeof(RunState), s));
    RunArgs a;
    a.opt = &o;
    a.pl = pl;
    a.ops = ops_for(pl.RP);
    a.vt_main = VT_F64;
    a.Vmain = c->V64.ptr;
    a.ldv_main = ldv;
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
            h_step(c, a, VT_F64, a.V64, ldv, epi(&o, pl.r, Gw, sw, true), true, s);
            NMF_TRY(get_factors(c, pl, nullptr, out, cudaMemcpyDeviceToHost, s));
            break;
        case STEP_W_KL:
            gram_h_full(c, a, Gh, sh, s);
            w_step(c, a, VT_F64, a.V64, ldv, epi(&o, pl.r, Gh, sh, false), true, s);
            NMF_TRY(get_factors(c, pl, out, nullptr, cudaMemcpyDeviceToHost, s));
            break;
        case STEP_H_EUC:
            gram_w_full(c, a, Gw, sw, s);
            h_step(c, a, VT_F64, a.V64, ldv, epi(&o, pl.r, Gw, sw, true), false, s);
            NMF_TRY(get_factors(c, pl, nullptr, out, cudaMemcpyDeviceToHost, s));
            break;
        case STEP_W_EUC:
            gram_h_full(c, a, Gh, sh, s);
            w_step(c, a, VT_F64, a.V64, ldv, epi(&o, pl.r, Gh, sh, false), false, s);
            NMF_TRY(get_factors(c, pl, out, nullptr, cudaMemcpyDeviceToHost, s));
            break;
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s));
    return NMFCU_OK;
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
    NMF_TRY(ensure_workspace(c, pl));
    NMF_TRY(c->dev.ensure(sizeof(double)));
    int64_t ldv = 0;
    NMF_TRY(upload_v(c, V, n, p, &ldv, s));
    NMF_TRY(put_factors(c, pl, W, H, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemsetAsync(c->state.ptr, 0, sizeof(RunState), s));
    const Ops *ops = ops_for(pl.RP);
    RunState *st = c->state.as<RunState>();
    ops->rowpass(VT_F64, c->V64.ptr, ldv, pl.n, pl.p, c->W.as<double>(), c->H.as<double>(),
                 kl ? 2 : 3, pl.S2, pl.cols_per_split, nullptr, c->obj.as<double>(), st, s);
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

nmfcu_status nmfcu_run(const nmfcu_options *opt, int64_t n, int64_t p, int64_t r,
                       const double *V, const double *W0, const double *H0, double *W,
                       double *H, double *deviances, int64_t deviances_cap,
                       int64_t *n_deviances, int64_t *n_iter) {
    NMF_TRY(validate_options(opt, n, p, r));
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
    const Plan pl = make_plan(n, p, r, c->sms);
    NMF_TRY(ensure_workspace(c, pl));
    if (stat) NMF_TRY(c->dev.ensure(sizeof(double) * (size_t)(opt->max_iter + 1)));
    int64_t ldv = 0, ld32 = 0;
    NMF_TRY(upload_v(c, V, n, p, &ldv, s));
    if (opt->precision == NMFCU_PREC_FP32)
        NMF_TRY(make_f32(c, c->V64.as<double>(), ldv, n, p, &ld32, s));
    NMF_TRY(put_factors(c, pl, W0, H0, cudaMemcpyHostToDevice, s));
    RunArgs a;
    a.opt = opt;
    a.pl = pl;
    a.ops = ops_for(pl.RP);
    const bool f32 = opt->precision == NMFCU_PREC_FP32;
    a.vt_main = f32 ? VT_F32 : VT_F64;
    a.Vmain = f32 ? c->V32.ptr : c->V64.ptr;
    a.ldv_main = f32 ? ld32 : ldv;
    a.V64 = c->V64.as<double>();
    a.ldv64 = ldv;
    a.W = c->W.as<double>();
    a.H = c->H.as<double>();
    a.dev = stat ? c->dev.as<double>() : nullptr;
    int64_t nd = 0, ni = 0;
    NMF_TRY(run_loop(c, a, s, &nd, &ni));
    NMF_TRY(get_factors(c, pl, W, H, cudaMemcpyDeviceToHost, s));
    if (stat && nd > 0)
        CUDA_TRY(cudaMemcpyAsync(deviances, c->dev.ptr, sizeof(double) * (size_t)nd,
                                 cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    *n_deviances = nd;
    *n_iter = ni;
    return NMFCU_OK;
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

nmfcu_status nmfcu_run_device(nmfcu_context *c, const nmfcu_options *opt, int64_t n, int64_t p,
                              int64_t r, const void *dV, int32_t v_dtype, int64_t ldv,
                              const double *dV64, int64_t ldv64, double *dW, double *dH,
                              double *d_dev, int64_t *n_deviances, int64_t *n_iter,
                              void *stream) {
    if (!c) return fail(NMFCU_ERR_INVALID_ARG, "NULL context");
    NMF_TRY(validate_options(opt, n, p, r));
    if (!dV || !dW || !dH || !n_deviances || !n_iter)
        return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    if (v_dtype != NMFCU_F64 && v_dtype != NMFCU_F32)
        return fail(NMFCU_ERR_INVALID_ARG, "v_dtype must be NMFCU_F64 or NMFCU_F32");
    if (ldv < p) return fail(NMFCU_ERR_INVALID_ARG, "ldv must be >= p");
    const bool f32 = (opt->precision == NMFCU_PREC_FP32);
    const bool stat = opt->stop == NMFCU_STOP_STATIONARY;
    if (!f32 && v_dtype != NMFCU_F64)
        return fail(NMFCU_ERR_INVALID_ARG, "precision FP64 needs an f64 V");
    const double *V64 = (v_dtype == NMFCU_F64) ? (const double *)dV : dV64;
    int64_t ld64 = (v_dtype == NMFCU_F64) ? ldv : ldv64;
    if (f32 && (stat || opt->refine_iters > 0) && !V64)
        return fail(NMFCU_ERR_INVALID_ARG,
                    "precision FP32 with a stationary stop or refinement needs the f64 V (dV64)");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard dg(c->device);
    cudaStream_t s = (cudaStream_t)stream;
    const Plan pl = make_plan(n, p, r, c->sms);
    NMF_TRY(ensure_workspace(c, pl));
    const void *Vmain = dV;
    int64_t ldmain = ldv;
    if (f32 && v_dtype == NMFCU_F64) {
        int64_t ld32 = 0;
        NMF_TRY(make_f32(c, (const double *)dV, ldv, n, p, &ld32, s));
        Vmain = c->V32.ptr;
        ldmain = ld32;
    }
    NMF_TRY(put_factors(c, pl, dW, dH, cudaMemcpyDeviceToDevice, s));
    RunArgs a;
    a.opt = opt;
    a.pl = pl;
    a.ops = ops_for(pl.RP);
    a.vt_main = f32 ? VT_F32 : VT_F64;
    a.Vmain = Vmain;
    a.ldv_main = ldmain;
    a.V64 = V64;
    a.ldv64 = ld64;
    a.W = c->W.as<double>();
    a.H = c->H.as<double>();
    a.dev = stat ? d_dev : nullptr;
    if (stat && !d_dev) return fail(NMFCU_ERR_INVALID_ARG, "stationary stop needs d_dev");
    int64_t nd = 0, ni = 0;
    NMF_TRY(run_loop(c, a, s, &nd, &ni));
    NMF_TRY(get_factors(c, pl, dW, dH, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    *n_deviances = nd;
    *n_iter = ni;
    return NMFCU_OK;
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

// stream_inst.cuh -- StreamOps for one element type STREAM_T (included by
// stream_f32.cu / stream_f64.cu).
#include <algorithm>

#include "launch.h"
#include "stream.cuh"

namespace nmfcu {
namespace {

template <int RP>
struct StreamOpsT final : StreamOps {
    using T = STREAM_T;
    static constexpr int RPS = RankPad<T, RP>::RPS;
    // Every f64 pass runs on the FP64 tensor cores (hpass_dmma / wpass_dmma,
    // and the *_dmma_ratio kernels for the ratio and weighted forms); the f32
    // passes on the CUDA cores.
    static constexpr bool kDmma = sizeof(T) == 8;
    using HP = HCfg<T, RP, false>;
    using WP = WCfg<T, RP, false>;
    using HR = HCfg<T, RP, true>;
    using WR = WCfg<T, RP, true>;

    int elem_bytes() const override { return (int)sizeof(T); }
    int rps() const override { return RPS; }
    int h_tcols(bool ratio) const override {
        return ratio ? (kDmma ? DHRCfg<RP>::TCOLS : HR::TCOLS)
                     : (kDmma ? DHCfg<RP>::TCOLS : HP::TCOLS);
    }
    int h_brows(bool ratio) const override {
        return ratio ? (kDmma ? DHRCfg<RP>::BROWS : HR::BROWS)
                     : (kDmma ? DHCfg<RP>::BROWS : HP::BROWS);
    }
    int h_boxc(bool ratio) const override {
        return ratio ? (kDmma ? DHRCfg<RP>::BOXC : HR::BOXC)
                     : (kDmma ? DHCfg<RP>::BOXC : HP::BOXC);
    }
    int h_segu(bool ratio) const override {
        return ratio ? (kDmma ? DHRCfg<RP>::SEGU : HR::SEGU)
                     : (kDmma ? DHCfg<RP>::SEGU : HP::SEGU);
    }
    int w_trows(bool ratio) const override {
        return ratio ? (kDmma ? DWRCfg<RP>::TROWS : WR::TROWS)
                     : (kDmma ? DWCfg<RP>::TROWS : WP::TROWS);
    }
    int w_bcols(bool ratio) const override {
        return ratio ? (kDmma ? DWRCfg<RP>::BCOLS : WR::BCOLS)
                     : (kDmma ? DWCfg<RP>::BCOLS : WP::BCOLS);
    }
    int w_segu(bool ratio) const override {
        return ratio ? (kDmma ? DWRCfg<RP>::SEGU : WR::SEGU)
                     : (kDmma ? DWCfg<RP>::SEGU : WP::SEGU);
    }
    int w_rowb(bool ratio) const override {
        return ratio ? (kDmma ? DWRCfg<RP>::ROWB : WR::ROWB)
                     : (kDmma ? DWCfg<RP>::ROWB : WP::ROWB);
    }
    int w_boxr(bool ratio) const override {
        return ratio ? (kDmma ? DWRCfg<RP>::BOXR : WR::BOXR)
                     : (kDmma ? DWCfg<RP>::BOXR : WP::BOXR);
    }

    template <bool RATIO, bool WEIGHTED = false>
    static cudaError_t launch_h(const CUtensorMap &tmV, const CUtensorMap &tmW, const double *H,
                                int n, int p, const StreamK &sk, double *part, RunState *st,
                                int grid, cudaStream_t s) {
        using C = HCfg<T, RP, RATIO>;
        static_assert(C::BOXC * C::NBOX == C::TCOLS, "tile / box mismatch");
        static_assert(C::BROWS == HCfg<T, RP, !RATIO>::BROWS, "one W box");
        auto *kern = nmfcu::hpass<T, RP, RATIO, WEIGHTED>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             C::SMEM);
        if (e != cudaSuccess) return e;
        kern<<<grid, 32 * C::kWarps, C::SMEM, s>>>(tmV, tmW, H, n, p, sk, part, st);
        return cudaGetLastError();
    }
    template <bool RATIO, bool WEIGHTED = false>
    static cudaError_t launch_w(const CUtensorMap &tmV, const CUtensorMap &tmH, const double *W,
                                int n, int p, const StreamK &sk, double *part, RunState *st,
                                int grid, cudaStream_t s) {
        using C = WCfg<T, RP, RATIO>;
        auto *kern = nmfcu::wpass<T, RP, RATIO, WEIGHTED>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             C::SMEM);
        if (e != cudaSuccess) return e;
        kern<<<grid, 32 * C::kWarps, C::SMEM, s>>>(tmV, tmH, W, n, p, sk, part, st);
        return cudaGetLastError();
    }

    // f64 ratio / weighted passes on the FP64 tensor cores.
    template <bool WEIGHTED>
    static cudaError_t launch_hr(const CUtensorMap &tmV, const CUtensorMap &tmW, const double *H,
                                 int n, int p, const StreamK &sk, double *part, RunState *st,
                                 int grid, cudaStream_t s) {
        using C = DHRCfg<RP>;
        auto *kern = nmfcu::hpass_dmma_ratio<RP, WEIGHTED>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             C::SMEM);
        if (e != cudaSuccess) return e;
        kern<<<grid, 32 * C::kWarps, C::SMEM, s>>>(tmV, tmW, H, n, p, sk, part, st);
        return cudaGetLastError();
    }
    template <bool WEIGHTED>
    static cudaError_t launch_wr(const CUtensorMap &tmV, const CUtensorMap &tmH, const double *W,
                                 int n, int p, const StreamK &sk, double *part, RunState *st,
                                 int grid, cudaStream_t s) {
        using C = DWRCfg<RP>;
        auto *kern = nmfcu::wpass_dmma_ratio<RP, WEIGHTED>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             C::SMEM);
        if (e != cudaSuccess) return e;
        kern<<<grid, 32 * C::kWarps, C::SMEM, s>>>(tmV, tmH, W, n, p, sk, part, st);
        return cudaGetLastError();
    }

    cudaError_t hpass(bool ratio, const CUtensorMap &tmV, const CUtensorMap &tmW,
                      const double *H, int n, int p, const StreamK &sk, double *part,
                      RunState *st, int grid, cudaStream_t s) const override {
        if constexpr (kDmma) {
            if (ratio) return launch_hr<false>(tmV, tmW, H, n, p, sk, part, st, grid, s);
            using C = DHCfg<RP>;
            cudaError_t e = cudaFuncSetAttribute(nmfcu::hpass_dmma<RP>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 C::SMEM);
            if (e != cudaSuccess) return e;
            nmfcu::hpass_dmma<RP><<<grid, 32 * C::kWarps, C::SMEM, s>>>(tmV, tmW, n, p, sk, part,
                                                                        st);
            return cudaGetLastError();
        } else {
            if (ratio) return launch_h<true>(tmV, tmW, H, n, p, sk, part, st, grid, s);
            return launch_h<false>(tmV, tmW, H, n, p, sk, part, st, grid, s);
        }
    }
    cudaError_t wpass(bool ratio, const CUtensorMap &tmV, const CUtensorMap &tmH,
                      const double *W, int n, int p, const StreamK &sk, double *part,
                      RunState *st, int grid, cudaStream_t s) const override {
        if constexpr (kDmma) {
            if (ratio) return launch_wr<false>(tmV, tmH, W, n, p, sk, part, st, grid, s);
            using C = DWCfg<RP>;
            cudaError_t e = cudaFuncSetAttribute(nmfcu::wpass_dmma<RP>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 C::SMEM);
            if (e != cudaSuccess) return e;
            nmfcu::wpass_dmma<RP><<<grid, 32 * C::kWarps, C::SMEM, s>>>(tmV, tmH, n, p, sk, part,
                                                                        st);
            return cudaGetLastError();
        } else {
            if (ratio) return launch_w<true>(tmV, tmH, W, n, p, sk, part, st, grid, s);
            return launch_w<false>(tmV, tmH, W, n, p, sk, part, st, grid, s);
        }
    }
    cudaError_t hpass_weighted(const CUtensorMap &tmV, const CUtensorMap &tmW, const double *H,
                               int n, int p, const StreamK &sk, double *part, RunState *st,
                               int grid, cudaStream_t s) const override {
        if constexpr (kDmma)
            return launch_hr<true>(tmV, tmW, H, n, p, sk, part, st, grid, s);
        else
            return cudaErrorNotSupported;
    }
    cudaError_t wpass_weighted(const CUtensorMap &tmV, const CUtensorMap &tmH, const double *W,
                               int n, int p, const StreamK &sk, double *part, RunState *st,
                               int grid, cudaStream_t s) const override {
        if constexpr (kDmma)
            return launch_wr<true>(tmV, tmH, W, n, p, sk, part, st, grid, s);
        else
            return cudaErrorNotSupported;
    }
    void h_epi(double *H, void *Ht, int p, const double *part, const StreamK &sk, int tcols,
               const EpiParams &e, const RunState *st, cudaStream_t s) const override {
        if (p <= 0) return;
        h_epilogue_sk<RP, T, RPS><<<(p + kThreads - 1) / kThreads, kThreads, 0, s>>>(
            H, static_cast<T *>(Ht), p, part, sk, tcols, e, st);
    }
    void w_epi(double *W, int n, const double *part, const StreamK &sk, int trows,
               const EpiParams &e, const RunState *st, cudaStream_t s) const override {
        if (n <= 0) return;
        w_epilogue_sk<RP><<<(unsigned)(((size_t)n * 32 + kThreads - 1) / kThreads), kThreads, 0, s>>>(W, n, part, sk,
                                                                            trows, e, st);
    }
    void w_copy(const double *W, void *Wc, int n, const RunState *st,
                cudaStream_t s) const override {
        if (n <= 0) return;
        const long long total = (long long)n * RPS;
        const int blocks = (int)std::min<long long>((total + kThreads - 1) / kThreads, 4096);
        w_to_f32<RP, RPS><<<blocks, kThreads, 0, s>>>(W, static_cast<float *>(Wc), n, st);
    }
};

}  // namespace

const StreamOps *STREAM_FACTORY(int rp) {
    static const StreamOpsT<2> o2;
    static const StreamOpsT<4> o4;
    static const StreamOpsT<6> o6;
    static const StreamOpsT<8> o8;
    static const StreamOpsT<10> o10;
    static const StreamOpsT<12> o12;
    static const StreamOpsT<14> o14;
    static const StreamOpsT<16> o16;
    static const StreamOpsT<20> o20;
    static const StreamOpsT<24> o24;
    static const StreamOpsT<28> o28;
    static const StreamOpsT<32> o32;
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

}  // namespace nmfcu

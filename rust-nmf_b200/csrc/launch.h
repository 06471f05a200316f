// launch.h -- host-side interface to the TMA streaming passes (stream.cuh),
// instantiated once per V element type in stream_f32.cu / stream_f64.cu.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace nmfcu {

struct StreamK;

// Geometry and launchers of the two passes for one (element type, rank
// bucket).  All pointers are device pointers.
struct StreamOps {
    virtual ~StreamOps() = default;
    virtual int elem_bytes() const = 0;          // 4 or 8
    virtual int rps() const = 0;                 // padded rank of the W / H^T copies
    virtual int h_tcols(bool ratio) const = 0;   // H pass tile width (columns)
    virtual int h_brows(bool ratio) const = 0;   // H pass rows per unit
    virtual int h_boxc(bool ratio) const = 0;    // H pass V box width
    virtual int h_segu(bool ratio) const = 0;    // H pass max units per segment
    virtual int w_trows(bool ratio) const = 0;   // W pass tile height (rows)
    virtual int w_bcols(bool ratio) const = 0;   // W pass columns per unit
    virtual int w_segu(bool ratio) const = 0;    // W pass max units per segment
    virtual int w_rowb(bool ratio) const = 0;    // W pass row bytes per unit (= swizzle span)
    virtual int w_boxr(bool ratio) const = 0;    // W pass V box height (rows)
    virtual cudaError_t hpass(bool ratio, const CUtensorMap &tmV, const CUtensorMap &tmW,
                              const double *H, int n, int p, const StreamK &sk, double *part,
                              RunState *st, int grid, cudaStream_t s) const = 0;
    virtual cudaError_t wpass(bool ratio, const CUtensorMap &tmV, const CUtensorMap &tmH,
                              const double *W, int n, int p, const StreamK &sk, double *part,
                              RunState *st, int grid, cudaStream_t s) const = 0;
    // The ratio passes' tiling with each V element entering as v (W H)_ij
    // (lsNMF's denominators; V holds the weights).  f64 only.
    virtual cudaError_t hpass_weighted(const CUtensorMap &tmV, const CUtensorMap &tmW,
                                       const double *H, int n, int p, const StreamK &sk,
                                       double *part, RunState *st, int grid,
                                       cudaStream_t s) const = 0;
    virtual cudaError_t wpass_weighted(const CUtensorMap &tmV, const CUtensorMap &tmH,
                                       const double *W, int n, int p, const StreamK &sk,
                                       double *part, RunState *st, int grid,
                                       cudaStream_t s) const = 0;
    virtual void h_epi(double *H, void *Ht, int p, const double *part, const StreamK &sk,
                       int tcols, const EpiParams &e, const RunState *st,
                       cudaStream_t s) const = 0;
    virtual void w_epi(double *W, int n, const double *part, const StreamK &sk, int trows,
                       const EpiParams &e, const RunState *st, cudaStream_t s) const = 0;
    // f32 only: W (n x RP f64) -> the f32 copy (n x rps()) that the H pass streams.
    virtual void w_copy(const double *W, void *Wc, int n, const RunState *st,
                        cudaStream_t s) const = 0;
};

const StreamOps *stream_ops_f32(int rp);
const StreamOps *stream_ops_f64(int rp);

// Tensor-core passes of the split-bf16 form (stream_tc.cu).  Tiles are 128
// outputs wide, units 64 streamed elements, segments at most 32 units.
constexpr int kTcTile = 128, kTcUnit = 64, kTcSegUnits = 32;
// brunet's tensor-core passes (tcr.cuh) stream units of 128 elements,
// segments of 16 units (the same 2048 terms per f32 sum).
constexpr int kTcrUnit = 128, kTcrSegUnits = 16;
// hpass: D[j][k] = sum_i V[i][j] W[i][k] (ah/al: the split V^T, p x n);
// otherwise D[i][k] = sum_j V[i][j] H[k][j] (ah/al: the split V).  Maps of
// A have box {64, 128}; b3: the factor's three bf16 terms (box {64, RPN});
// RPN 16 or 32.
cudaError_t tc_pass_launch(bool hpass, int RPN, const CUtensorMap &ah, const CUtensorMap &al,
                           const CUtensorMap *b3, int kext, int RP, const StreamK &sk,
                           double *part, RunState *st, cudaStream_t s);
// V (f64) -> Vh, Vl (bf16, n x ldb) and Vth, Vtl (bf16 V^T, p x ldbt), one read of V.
void tc_split_v(const double *V, int64_t ldv, void *Vh, void *Vl, int64_t ldb, void *Vth,
                void *Vtl, int64_t ldbt, int n, int p, cudaStream_t s);
// F(k, x) = F[k * fk + x * fx] (R x K) -> three bf16 planes of RPN x ldk.
void tc_split_factor(const double *F, int64_t fk, int64_t fx, int R, int K, void *out, int RPN,
                     int64_t ldk, const RunState *st, int sms, cudaStream_t s);

// brunet's tensor-core passes (stream_tcr.cu), on their own stream-K split
// (units of kTcrUnit elements, kTcrSegUnits units a segment).  hpass:
// N[j][k] = sum_i W[i][k] V[i][j] / (W H)[i][j]; otherwise N[i][k] =
// sum_j H[k][j] V[i][j] / (W H)[i][j].  v: the f32 V (H pass box {128, 64};
// W pass box {32, 128}, 128-B swizzle); t: the tile factor's rows in the
// tile layout (device pointer, rows of tcr_concat_rank(rank) bf16, from
// tcr_split_factor); f1: the unit factor's rows in the unit layout (box
// {64, 128}, 128-B swizzle).
cudaError_t tcr_pass_launch(bool hpass, const CUtensorMap &v, const void *t,
                            const CUtensorMap &f1, int kext, int rank, int RP, const StreamK &sk,
                            double *part, RunState *st, cudaStream_t s);
// The padded concatenated rank (row length, bf16) of the two layouts:
// 128 for rank <= 21, 192 up to 32.
int tcr_concat_rank(int rank);
// F(k, x) = F[k * fk + x * fx] (R x K) -> xpad rows of tcr_concat_rank(R)
// bf16 in the tile layout ([Th Th Th Tm Tm Tl], blocks of R) and the unit
// layout ([Fh Fm Fl Fh Fm Fh]), zero-padded; either output may be null.
void tcr_split_factor(const double *F, int64_t fk, int64_t fx, int R, int K, int64_t xpad,
                      void *tile, void *unit, const RunState *st, int sms, cudaStream_t s);

}  // namespace nmfcu

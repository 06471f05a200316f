/*
 * nmfcu.h -- C ABI of the B200 NMF engine (libnmfcu.so).
 *
 * The reference, omicverse/rust-NMF, exposes its numerics only through the
 * PyO3 module `nmf_rs._rust` (rust/src/lib.rs:2177-2187).  Every entry point
 * below replaces one callable of that module, or one step of the loop behind
 * it, and is cited to it.  Plain pointers and sizes only: no allocation
 * crosses this boundary, the caller owns every buffer it passes.
 *
 * Conventions
 *   - Matrices are row-major (C-contiguous) f64: V is n x p, W is n x r,
 *     H is r x p -- the layout numpy hands the reference
 *     (python/nmf_rs/__init__.py:235-240).
 *   - Every call returns an nmfcu_status; on failure nmfcu_last_error()
 *     returns a message for the calling thread.  Nothing aborts the process.
 *   - All compute runs on the GPU.  There is no CPU fallback: without a
 *     usable CUDA device the compute entry points return
 *     NMFCU_ERR_NO_DEVICE.
 */
#ifndef NMFCU_H
#define NMFCU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NMFCU_ABI_VERSION 1
/* Largest factorisation rank the GPU kernels are built for. */
#define NMFCU_MAX_RANK 32
/* Ranks above NMFCU_MAX_RANK, up to NMFCU_MAX_WIDE_RANK, run lee, brunet, hals
 * and dnmf in FP64 through nmfcu_run / nmfcu_run_device: the V contractions
 * as streaming passes over 32-rank chunks (one pass over V each), the rest in
 * kernels with the rank as a run-time value. */
#define NMFCU_MAX_WIDE_RANK 256

typedef enum nmfcu_status {
    NMFCU_OK = 0,
    NMFCU_ERR_INVALID_ARG = 1, /* bad shape / value; Python maps to ValueError      */
    NMFCU_ERR_UNSUPPORTED = 2, /* method or rank not built; NotImplementedError      */
    NMFCU_ERR_OOM = 3,         /* device allocation failed; MemoryError              */
    NMFCU_ERR_CUDA = 4,        /* CUDA runtime error; RuntimeError                   */
    NMFCU_ERR_NUMERIC = 5,     /* non-finite value where the contract forbids one   */
    NMFCU_ERR_TIMEOUT = 6,     /* a bounded device wait gave up; RuntimeError        */
    NMFCU_ERR_NO_DEVICE = 7,   /* no CUDA device visible; RuntimeError               */
    NMFCU_ERR_CANCELLED = 8    /* a served request was cancelled before it started  */
} nmfcu_status;

/* Algorithm ids: the variants of `Algo` (lib.rs:1472-1484), same order. */
enum {
    NMFCU_BRUNET = 0,
    NMFCU_LEE = 1,
    NMFCU_OFFSET = 2, /* through nmfcu_run / nmfcu_run_offset (host buffers) */
    NMFCU_NSNMF = 3,
    NMFCU_HALS = 4,
    NMFCU_EHALS = 5,
    NMFCU_DNMF = 6,
    NMFCU_LSNMF = 7,  /* through nmfcu_run_weighted (FP64) */
    NMFCU_SNMF_R = 8, /* FP64 */
    NMFCU_SNMF_L = 9  /* FP64 */
};

/* Stop ids: the variants of `Stop` (lib.rs:1507-1513). */
enum { NMFCU_STOP_MAX_ITER = 0, NMFCU_STOP_STATIONARY = 1 };

/* Arithmetic of the V contractions.  The reference is f64 throughout.
 *   FP64   -- f64 V, f64 products and sums (the plain method).
 *   FP32   -- V stored f32, products and per-thread sums in f32; every
 *             reduction across threads, all update epilogues, Gram matrices,
 *             rescaling, objective and stop test stay f64, and the last
 *             `refine_iters` iterations run the FP64 path on the f64 V.
 *   BF16X3 -- lee / offset / hals / ehals / dnmf: V stored as two bf16 terms (hi + lo, 4 bytes
 *             an element), the factor of each contraction split into three
 *             bf16 terms, products on the tensor cores with f32 sums of at
 *             most 2048 terms; everything else as FP32.  brunet / nsNMF:
 *             W H and the contraction on the tensor cores (three bf16 terms
 *             per factor), the ratio V / (W H) in f32 over the f32 V, written
 *             as bf16 hi + lo.  Needs the f64 V. */
enum { NMFCU_PREC_FP64 = 0, NMFCU_PREC_FP32 = 1, NMFCU_PREC_BF16X3 = 2 };

/* Keyword arguments of py_nmf_run (lib.rs:1912-1933), plus engine knobs. */
typedef struct nmfcu_options {
    int32_t method;        /* NMFCU_BRUNET ...                                  */
    int32_t stop;          /* NMFCU_STOP_*                                      */
    int32_t precision;     /* NMFCU_PREC_*  (engine knob, default FP64)         */
    int32_t rescale;       /* lee: W columns to sum 1 each iteration (1)        */
    int64_t max_iter;      /* iterations (the reference has no default here)   */
    double eps;            /* 1e-9; brunet ignores it and uses DBL_EPSILON      */
    double theta;          /* nsNMF smoothing (0.5)                             */
    double sparsity_h;     /* dnmf L1 on H (0)                                  */
    double sparsity_w;     /* dnmf L1 on W (0)                                  */
    double smoothness_h;   /* dnmf L2 on H (0)                                  */
    double smoothness_w;   /* dnmf L2 on W (0)                                  */
    double stationary_th;  /* DBL_EPSILON                                       */
    int64_t check_interval; /* 50                                               */
    int64_t check_niter;    /* 10                                               */
    int32_t refine_iters;  /* FP32 precision: trailing FP64 iterations (2)      */
    int32_t device;        /* CUDA device ordinal (0)                           */
} nmfcu_options;

/* Fill `o` with the py_nmf_run defaults (lib.rs:1919-1932); method brunet,
 * max_iter 2000 (the Python default, python/nmf_rs/__init__.py:403). */
void nmfcu_options_default(nmfcu_options *o);

/* Algo::from_str (lib.rs:1486-1505): case-insensitive name or alias ->
 * method id.  NMFCU_ERR_INVALID_ARG for an unknown name. */
nmfcu_status nmfcu_parse_method(const char *name, int32_t *method);

/* Stop::from_str (lib.rs:1515-1526). */
nmfcu_status nmfcu_parse_stop(const char *name, int32_t *stop);

/*
 * nmfcu_run -- replaces py_nmf_run (lib.rs:1934-2169) for brunet, lee,
 * offset, nsNMF, hals, ehals and dnmf: the whole iteration loop
 * (nmf_run_brunet :1529-1586, nmf_run_lee :1589-1647, nmf_run_offset
 * :1650-1760, nmf_run_nsnmf :1762-1830, nmf_run_hals :638-688,
 * nmf_run_ehals :711-786, nmf_run_dnmf :827-906) and the Kim-Park snmf/r,
 * snmf/l (nmf_run_snmf_kim_park :1216-1320, FP64; deviances then hold one
 * value an iteration whatever the stop, as the reference returns).
 * For offset it starts from rowMeans(V) and drops the final offsets; use
 * nmfcu_run_offset to pass and receive them.
 *
 * Host pointers.  V (n x p), W0 (n x r), H0 (r x p) are read; W (n x r) and
 * H (r x p) receive the result (they may alias W0 / H0).  `deviances` must
 * hold `deviances_cap` >= max_iter + 1 doubles when stop is stationary (it
 * may be NULL otherwise); *n_deviances receives how many were written and
 * *n_iter the iteration count -- the `deviances` and `n_iter` of the
 * reference's result dict (lib.rs:2158-2168).
 */
nmfcu_status nmfcu_run(const nmfcu_options *opt, int64_t n, int64_t p, int64_t r,
                       const double *V, const double *W0, const double *H0, double *W,
                       double *H, double *deviances, int64_t deviances_cap,
                       int64_t *n_deviances, int64_t *n_iter);

/*
 * nmfcu_run_offset -- py_nmf_run with method "offset" (lib.rs:2023-2037, 2163-2165): as
 * nmfcu_run, plus the row offsets.  offset0 (n doubles) is the `offset`
 * keyword (NULL: rowMeans(V), lib.rs:1667-1679); `offset` (n doubles)
 * receives the final offsets, the result dict's "offset" entry.  opt->method
 * must be NMFCU_OFFSET.
 */
nmfcu_status nmfcu_run_offset(const nmfcu_options *opt, int64_t n, int64_t p, int64_t r,
                              const double *V, const double *W0, const double *H0,
                              const double *offset0, double *W, double *H, double *offset,
                              double *deviances, int64_t deviances_cap, int64_t *n_deviances,
                              int64_t *n_iter);

/*
 * nmfcu_run_weighted -- py_nmf_run with method "lsnmf" (lib.rs:2101-2115 ->
 * nmf_run_lsnmf :945-1043): as nmfcu_run, plus the per-entry weights
 * `weight` (n x p, the `weight` keyword), minimising 0.5 ||(V - W H) o
 * weight||^2.  opt->method must be NMFCU_LSNMF and opt->precision FP64.
 */
nmfcu_status nmfcu_run_weighted(const nmfcu_options *opt, int64_t n, int64_t p, int64_t r,
                                const double *V, const double *weight, const double *W0,
                                const double *H0, double *W, double *H, double *deviances,
                                int64_t deviances_cap, int64_t *n_deviances, int64_t *n_iter);

/* Single-step updates on host pointers; each writes a fresh factor.
 *   py_divergence_update_h (lib.rs:1851-1862 -> divergence_update_h_impl :120-144)
 *   py_divergence_update_w (lib.rs:1866-1877 -> divergence_update_w_impl :151-204)
 *   py_euclidean_update_h  (lib.rs:1880-1892 -> euclidean_update_h_impl  :249-276)
 *   py_euclidean_update_w  (lib.rs:1895-1907 -> euclidean_update_w_impl  :281-322) */
nmfcu_status nmfcu_update_h_divergence(int64_t n, int64_t p, int64_t r, const double *V,
                                       const double *W, const double *H, double *H_out);
nmfcu_status nmfcu_update_w_divergence(int64_t n, int64_t p, int64_t r, const double *V,
                                       const double *W, const double *H, double *W_out);
nmfcu_status nmfcu_update_h_euclidean(int64_t n, int64_t p, int64_t r, const double *V,
                                      const double *W, const double *H, double eps,
                                      double *H_out);
nmfcu_status nmfcu_update_w_euclidean(int64_t n, int64_t p, int64_t r, const double *V,
                                      const double *W, const double *H, double eps,
                                      double *W_out);

/* py_smoothing_matrix (lib.rs:2172-2175 -> smoothing_matrix :458-466):
 * S = (1 - theta) I + (theta / r) 1 1^T into S (r x r).  Host arithmetic. */
nmfcu_status nmfcu_smoothing_matrix(int64_t r, double theta, double *S);

/* set_num_threads (lib.rs:1841-1847).  The GPU engine has no CPU thread
 * pool; returns 0 (the reference's `false`, "pool not rebuilt"). */
int32_t nmfcu_set_num_threads(int64_t n);

/* Objectives on host pointers: kl_divergence (lib.rs:1410-1431) and
 * euclidean_distance (lib.rs:1434-1445) of V against W H, computed on the
 * GPU in f64 without materialising W H. */
nmfcu_status nmfcu_divergence(int64_t n, int64_t p, int64_t r, const double *V,
                              const double *W, const double *H, double *out);
nmfcu_status nmfcu_distance(int64_t n, int64_t p, int64_t r, const double *V, const double *W,
                            const double *H, double *out);

/* ---------------------------------------------------------------------- */
/* Device-resident API (inputs already in HBM).                            */
/* ---------------------------------------------------------------------- */

typedef struct nmfcu_context nmfcu_context;

/* A context owns the device scratch of one device and is reused across
 * calls; one context per host thread (calls on one context serialise). */
nmfcu_status nmfcu_context_create(int32_t device, nmfcu_context **ctx);
void nmfcu_context_destroy(nmfcu_context *ctx);

/* Element type of a device V. */
enum { NMFCU_F64 = 0, NMFCU_F32 = 1 };

/*
 * nmfcu_run_device -- nmfcu_run on device pointers, enqueued on `stream`
 * (a cudaStream_t, NULL for the legacy default stream).
 *   dV      n x p, leading dimension ldv (elements), type v_dtype.  For
 *           precision FP32 pass the f32 V here and the f64 V in dV64 (used by
 *           the FP64 refinement iterations and the objective); for FP64 pass
 *           the f64 V and dV64 = NULL.
 *   dW, dH  n x r and r x p f64, W0/H0 on entry, the result on exit.
 *   d_dev   device array of >= max_iter + 1 doubles (stationary stop) or NULL.
 * *n_iter / *n_deviances are written after the stream has been synchronised
 * (the call returns when the result is complete).
 */
nmfcu_status nmfcu_run_device(nmfcu_context *ctx, const nmfcu_options *opt, int64_t n,
                              int64_t p, int64_t r, const void *dV, int32_t v_dtype,
                              int64_t ldv, const double *dV64, int64_t ldv64, double *dW,
                              double *dH, double *d_dev, int64_t *n_deviances, int64_t *n_iter,
                              void *stream);

/*
 * nmfcu_run_csr -- nmfcu_run on a sparse V in compressed sparse row form.
 * No counterpart in the reference, whose nmf() densifies V first
 * (python/nmf_rs/__init__.py:495, `_f64_c(V)`), so it replaces that call
 * path for the sparse (AnnData CSR) inputs single-cell data arrives in: the
 * same loop (py_nmf_run, lib.rs:1934-2169) with V's zeros never stored or
 * read.  Methods lee, brunet, hals and dnmf (others: NMFCU_ERR_UNSUPPORTED),
 * FP64 only.
 *   indptr   n + 1 row offsets (indptr[0] = 0, non-decreasing, indptr[n] = nnz)
 *   indices  nnz column indices in [0, p), data nnz values (f64, >= 0): the
 *            canonical CSR of V -- each row's column indices strictly
 *            increasing (sorted, no duplicates); anything else is refused
 *            with NMFCU_ERR_INVALID_ARG.
 * W0, H0, W, H, deviances, n_deviances, n_iter as in nmfcu_run.  nnz is at
 * most 2^31 - 1.  The library keeps a column-sorted (CSC) copy of V for the
 * H step on the device for the run (12 bytes per stored entry).
 */
nmfcu_status nmfcu_run_csr(const nmfcu_options *opt, int64_t n, int64_t p, int64_t r,
                           int64_t nnz, const int64_t *indptr, const int32_t *indices,
                           const double *data, const double *W0, const double *H0, double *W,
                           double *H, double *deviances, int64_t deviances_cap,
                           int64_t *n_deviances, int64_t *n_iter);
/* nmfcu_run_csr on device pointers, enqueued on `stream`: the CSR arrays as
 * above, dW (n x r) and dH (r x p) f64 hold W0 / H0 on entry and the result
 * on exit, d_dev as in nmfcu_run_device.  The CSR's structure is checked on
 * the device before use (a bad indptr or index: NMFCU_ERR_INVALID_ARG). */
nmfcu_status nmfcu_run_csr_device(nmfcu_context *ctx, const nmfcu_options *opt, int64_t n,
                                  int64_t p, int64_t r, int64_t nnz, const int64_t *d_indptr,
                                  const int32_t *d_indices, const double *d_data, double *dW,
                                  double *dH, double *d_dev, int64_t *n_deviances,
                                  int64_t *n_iter, void *stream);

/*
 * nmfcu_run_offset_device -- nmfcu_run_offset on device pointers, enqueued on
 * `stream` (py_nmf_run with method "offset", lib.rs:2023-2037, 2163-2165):
 * the arguments of nmfcu_run_device plus d_offset0 (n doubles on the device,
 * the `offset` keyword; NULL: rowMeans(V), lib.rs:1667-1679) and d_offset (n
 * doubles on the device, receives the final offsets, the result dict's
 * "offset" entry).  opt->method must be NMFCU_OFFSET; the f64 V is needed
 * (dV, or dV64 beside an f32 dV) for the row sums the offset update uses.
 */
nmfcu_status nmfcu_run_offset_device(nmfcu_context *ctx, const nmfcu_options *opt, int64_t n,
                                     int64_t p, int64_t r, const void *dV, int32_t v_dtype,
                                     int64_t ldv, const double *dV64, int64_t ldv64, double *dW,
                                     double *dH, const double *d_offset0, double *d_offset,
                                     double *d_dev, int64_t *n_deviances, int64_t *n_iter,
                                     void *stream);

/*
 * nmfcu_v_product_device -- one V contraction of the randomized range finder
 * behind nndsvd_init (python/nmf_rs/__init__.py:129-219, which calls
 * scikit-learn's randomized_svd at :172-174; its products A @ Q, A.T @ Q and
 * Q.T @ A are these two with A = V or V^T):
 *   trans = 0:  out (n x l) = V X,    X (p x l)
 *   trans = 1:  out (p x l) = V^T X,  X (n x l)
 * All device pointers, f64, row-major, leading dimensions ldv / ldx / ldo,
 * enqueued on `stream`; returns once the product is complete.  One FP64
 * streaming pass over V per 32 columns of X.
 */
nmfcu_status nmfcu_v_product_device(nmfcu_context *ctx, int32_t trans, int64_t n, int64_t p,
                                    int64_t l, const double *dV, int64_t ldv, const double *dX,
                                    int64_t ldx, double *dOut, int64_t ldo, void *stream);

/*
 * Column shards -- one solve over several GPUs, one process a GPU.  The
 * reference has no multi-device path; this splits its loop (nmf_run_lee
 * lib.rs:1589-1647, nmf_run_brunet :1529-1586, nmf_run_hals :638-688,
 * nmf_run_dnmf :827-906) by columns of V.  Each rank holds V[:, c0:c1], its
 * H columns and a copy of W.  The H update is local; the W update needs
 * the W contraction (V H^T, or the ratio form for brunet), H H^T and
 * rowSums(H) summed over ranks: the caller all-reduces (sums) the reduce
 * buffer between the two halves of an iteration, and the objective scalar
 * between NMFCU_SHARD_OBJECTIVE and NMFCU_SHARD_STOP.  Every rank applies
 * the same W update to its copy, so the copies stay identical.
 *
 * One iteration:  HALF_STEP, all-reduce(reduce buffer), W_UPDATE
 *                 [stationary: OBJECTIVE, all-reduce(objective), STOP,
 *                  nmfcu_shard_status -> stop when `stopped`]
 * Before the first iteration with stop stationary: OBJECTIVE, all-reduce,
 * STOP.  Methods brunet, lee, hals, dnmf; all three precisions.
 *
 * nmfcu_shard_reduce_len(n, r): doubles in the reduce buffer.
 * nmfcu_shard_create: dV (n x p_local, pitch ldv, 16-byte aligned rows),
 *   dW0 (n x r) and dH0 (r x p_local) are device pointers; dReduce
 *   (reduce_len doubles) and dObjective (1 double) are the caller's device
 *   buffers that its collective sums.  The shard uses `ctx` until destroyed.
 * nmfcu_shard_status: synchronises `stream`; iterations done and the stop.
 * nmfcu_shard_result: W (n x r), this shard's H (r x p_local) and the
 *   deviances (n_iter + 1 with stop stationary) into device buffers.
 */
typedef struct nmfcu_shard nmfcu_shard;
enum {
    NMFCU_SHARD_HALF_STEP = 0,
    NMFCU_SHARD_W_UPDATE = 1,
    NMFCU_SHARD_OBJECTIVE = 2,
    NMFCU_SHARD_STOP = 3
};
int64_t nmfcu_shard_reduce_len(int64_t n, int64_t r);
nmfcu_status nmfcu_shard_create(nmfcu_context *ctx, const nmfcu_options *opt, int64_t n,
                                int64_t p_local, int64_t r, const double *dV, int64_t ldv,
                                const double *dW0, const double *dH0, double *dReduce,
                                double *dObjective, nmfcu_shard **shard, void *stream);
nmfcu_status nmfcu_shard_step(nmfcu_shard *shard, int32_t phase, void *stream);
nmfcu_status nmfcu_shard_status(nmfcu_shard *shard, int64_t *n_iter, int32_t *stopped,
                                void *stream);
nmfcu_status nmfcu_shard_result(nmfcu_shard *shard, double *dW, double *dH, double *d_dev,
                                int64_t *n_deviances, int64_t *n_iter, void *stream);
void nmfcu_shard_destroy(nmfcu_shard *shard);

/* Per-kernel CUDA-event timing inside nmfcu_run_device (off by default).
 * Kernel classes: 0 = H-step V contraction, 1 = W-step V contraction,
 * 2 = objective V pass, 3 = everything else (grams, epilogues, stop),
 * 4 / 5 = the H / W contractions of FP64 refinement iterations. */
enum { NMFCU_KCLASS_HSTEP = 0, NMFCU_KCLASS_WSTEP = 1, NMFCU_KCLASS_OBJECTIVE = 2,
       NMFCU_KCLASS_OTHER = 3,
       /* the FP64 refinement iterations of the FP32 / BF16X3 forms */
       NMFCU_KCLASS_HSTEP_REFINE = 4, NMFCU_KCLASS_WSTEP_REFINE = 5, NMFCU_KCLASS_COUNT = 6 };
nmfcu_status nmfcu_context_set_timing(nmfcu_context *ctx, int32_t enabled);
/* Launch count and summed event time (ms) of one kernel class since the
 * last reset; the call synchronises the context's events. */
nmfcu_status nmfcu_context_kernel_time(nmfcu_context *ctx, int32_t kclass, int64_t *launches,
                                       double *total_ms);
nmfcu_status nmfcu_context_reset_timing(nmfcu_context *ctx);
/* Kernels launched by this context since the last reset (all classes). */
int64_t nmfcu_context_launch_count(nmfcu_context *ctx);

/* ---------------------------------------------------------------------- */
/* Batched solves and consensus                                            */
/* ---------------------------------------------------------------------- */

/*
 * nmfcu_run_batch -- many brunet solves of one V at once: the restarts and
 * rank sweep of the reference's consensus workflow, which calls nmf() once
 * per (rank, run) in a Python loop (examples/build_scaling_notebook.py:
 * 157-208, each call nmf_run_brunet lib.rs:1529-1586 with stop="max_iter").
 * Solve s has rank ranks[s] (1..NMFCU_MAX_WIDE_RANK); ranks 1..16 run in the
 * batched kernels, higher ones one at a time through the single-solve
 * engine in FP64 within the same call.  The factors of all solves are stacked:
 *   W0, W  n x R f64, R = sum(ranks), solve s in columns [off_s, off_s + r_s)
 *   H0, H  R x p f64, solve s in rows [off_s, off_s + r_s)
 * with off_s = ranks[0] + ... + ranks[s-1].  Every solve runs exactly
 * max_iter iterations.  method must be NMFCU_BRUNET (others:
 * NMFCU_ERR_UNSUPPORTED).  precision FP64 gives each solve's single-solve
 * result to rounding; FP32 (and BF16X3, which runs brunet as FP32, as the
 * single solve does) computes in f32 from an f32 copy of V.
 */
nmfcu_status nmfcu_run_batch(int32_t method, int32_t precision, int64_t max_iter, int64_t n,
                             int64_t p, const double *V, int32_t nsolves, const int32_t *ranks,
                             const double *W0, const double *H0, double *W, double *H,
                             int32_t device);
/* The same on device pointers (V with leading dimension ldv), on `stream`;
 * dW/dH hold the stacked starts on entry and the results on exit. */
nmfcu_status nmfcu_run_batch_device(nmfcu_context *ctx, int32_t method, int32_t precision,
                                    int64_t max_iter, int64_t n, int64_t p, const double *dV,
                                    int64_t ldv, int32_t nsolves, const int32_t *ranks,
                                    double *dW, double *dH, void *stream);

/* Shape of the batched kernel: how many solves a CTA carries (and so how many
 * solves each V element it loads serves) and how many CTAs a multiprocessor
 * keeps resident.  With NMFCU_BATCH_SHAPE_AUTO (the default) the first
 * batched run of a problem -- device, precision, n, p and the multiset of
 * ranks -- with max_iter >= 20 times each candidate shape for a few
 * iterations on copies of its starting factors and keeps the fastest for
 * later runs of that problem; shorter runs take shape 0.  A shape changes
 * which solves share a CTA, not the arithmetic of a solve: every shape gives
 * the same results.  Process-wide. */
#define NMFCU_BATCH_SHAPE_AUTO (-1)
/* Selects NMFCU_BATCH_SHAPE_AUTO or forces shape 0 .. nmfcu_batch_shape_count() - 1. */
nmfcu_status nmfcu_batch_set_shape(int32_t shape);
int32_t nmfcu_batch_shape_count(void);
/* The shape the last batched run used (-1 before the first). */
int32_t nmfcu_batch_last_shape(void);

/* Consensus matrix of the selected solves `sel[0..nsel)` of a stacked H
 * (layout as above): C[j1][j2] = fraction of the selected solves that put
 * columns j1 and j2 in the same cluster, the cluster of column j being
 * argmax_k H_s[k][j] (first maximum) -- connectivity_matrix and the mean over
 * runs of examples/build_scaling_notebook.py:121-124, 179-186.  d_out is a
 * p x p f32 device array. */
nmfcu_status nmfcu_consensus_device(nmfcu_context *ctx, int64_t p, int32_t nsolves,
                                    const int32_t *ranks, const double *dH, int32_t nsel,
                                    const int32_t *sel, float *d_out, void *stream);

/*
 * nmfcu_consensus_stats_device -- the two summaries of a consensus matrix in
 * the reference's consensus workflow (examples/build_scaling_notebook.py
 * :126-141), computed on the device from C (p x p f32, pitch ldc, device):
 *   *cophenetic -- Brunet et al. (2004): the correlation over the pairs
 *     i < j between the distances 1 - C_ij and their cophenetic distances in
 *     the average-linkage tree of 1 - C (the tree scipy's linkage builds,
 *     ties included); 1 when either has no spread.
 *   *dispersion -- Kim & Park (2007): mean over all p^2 entries of
 *     4 (C_ij - 0.5)^2 (diagonal taken as 1).
 * Uses p^2 doubles of context scratch; returns once both are on the host.
 */
nmfcu_status nmfcu_consensus_stats_device(nmfcu_context *ctx, int64_t p, const float *dC,
                                          int64_t ldc, double *cophenetic, double *dispersion,
                                          void *stream);
/* The same for `count` consensus matrices at once (matrix m at dC + m *
 * stride elements, pitch ldc; the consensus matrices of a rank sweep, one per
 * rank): cophenetic[m], dispersion[m] (host arrays of `count`).  The
 * average-linkage trees of all matrices are built in one launch, one block
 * each, so they run concurrently.  Uses count * p^2 doubles of context
 * scratch. */
nmfcu_status nmfcu_consensus_stats_batch_device(nmfcu_context *ctx, int32_t count, int64_t p,
                                                const float *dC, int64_t ldc, int64_t stride,
                                                double *cophenetic, double *dispersion,
                                                void *stream);

/* ---------------------------------------------------------------------- */
/* Serving: continuous admission of independent factorisations            */
/* ---------------------------------------------------------------------- */

/*
 * No counterpart in the reference, whose nmf() runs each factorisation to
 * completion on the calling thread (python/nmf_rs/__init__.py:396-568).  A
 * server runs requests of any shape, rank and method concurrently on one
 * GPU: `slots` workers, each with its own engine context and stream, take
 * queued requests as slots and device memory free up; a request is admitted
 * when the device bytes its slot must add fit in `budget_bytes` (0: 90% of
 * the device's free memory at creation) next to what all slots hold.  Each
 * request computes exactly what nmfcu_run computes for the same arguments.
 */
typedef struct nmfcu_server nmfcu_server;

typedef struct nmfcu_server_stats {
    int64_t submitted, completed, failed, cancelled, queued, running;
    int64_t iterations;       /* iterations of the completed requests            */
    double wall_ms;           /* first submission to the last completion         */
    double p50_ms, p99_ms, max_ms; /* submit-to-complete latency, completed ones  */
    double mean_queue_ms;     /* submit-to-start, completed requests             */
    int64_t budget_bytes, in_use_bytes, peak_bytes; /* device memory of the slots */
    int64_t launches;         /* engine kernel launches of the completed requests */
    int32_t slots, peak_running;
} nmfcu_server_stats;

nmfcu_status nmfcu_server_create(int32_t device, int32_t slots, int64_t budget_bytes,
                                 nmfcu_server **out);
/* Cancels queued requests, waits for running ones, frees everything. */
void nmfcu_server_destroy(nmfcu_server *srv);
/* Queues one factorisation (arguments as nmfcu_run; V has leading dimension
 * ldv).  Every buffer stays owned by the caller and must stay valid until
 * nmfcu_server_wait has returned for the request.  A request that would not
 * fit in the budget even alone fails here with NMFCU_ERR_OOM. */
nmfcu_status nmfcu_server_submit(nmfcu_server *srv, const nmfcu_options *opt, int64_t n,
                                 int64_t p, int64_t r, const double *V, int64_t ldv,
                                 const double *W0, const double *H0, double *W, double *H,
                                 double *deviances, int64_t dev_cap, int64_t *request_id);
/* nmfcu_server_submit for the offset method (opt->method NMFCU_OFFSET): the
 * nmfcu_run_offset of a served request.  offset0 (n doubles, host; NULL:
 * rowMeans(V)) is read when the request starts, offset (n doubles, host)
 * receives the final row offsets; both stay owned by the caller until
 * nmfcu_server_wait has returned for the request. */
nmfcu_status nmfcu_server_submit_offset(nmfcu_server *srv, const nmfcu_options *opt, int64_t n,
                                        int64_t p, int64_t r, const double *V, int64_t ldv,
                                        const double *W0, const double *H0,
                                        const double *offset0, double *W, double *H,
                                        double *offset, double *deviances, int64_t dev_cap,
                                        int64_t *request_id);
/* state: 0 queued, 1 running, 2 done. */
nmfcu_status nmfcu_server_poll(nmfcu_server *srv, int64_t request_id, int32_t *state);
/* Waits up to timeout_ms (< 0: no limit) and returns the request's own
 * status (NMFCU_ERR_TIMEOUT if it has not finished; the request stays).
 * Once a final status is returned the id is released. */
nmfcu_status nmfcu_server_wait(nmfcu_server *srv, int64_t request_id, int64_t timeout_ms,
                               int64_t *n_iter, int64_t *n_deviances);
/* Cancels a request that has not started (its wait returns
 * NMFCU_ERR_CANCELLED); running requests finish. */
nmfcu_status nmfcu_server_cancel(nmfcu_server *srv, int64_t request_id);
nmfcu_status nmfcu_server_get_stats(nmfcu_server *srv, nmfcu_server_stats *out);
nmfcu_status nmfcu_server_reset_stats(nmfcu_server *srv);

/* ---------------------------------------------------------------------- */
/* Allocation-free objective                                               */
/* ---------------------------------------------------------------------- */

/* No counterpart in the reference.  For callers that may not allocate
 * device memory while they run (a server that reserves all device memory up
 * front, code under another framework's memory pool, a loop that cannot
 * take the synchronisation of cudaMalloc/cudaFree): the objective of V
 * against W H on device pointers, computed without any allocation.
 *
 *   kind   NMFCU_OBJECTIVE_KL (kl_divergence, lib.rs:1410-1431) or
 *          NMFCU_OBJECTIVE_FROBENIUS (0.5 ||V - WH||^2, lib.rs:1434-1445)
 *   dV     n x p f64, leading dimension ldv;  dW n x r;  dH r x p
 *   d_out  one f64 on the device, written when `stream` reaches the work
 *
 * Its scratch is a fixed 512 KB array compiled into the library (one f64 per
 * 8 rows), which every GPU that loads the library holds until the process
 * exits; n above NMFCU_NOALLOC_MAX_ROWS is rejected (NMFCU_ERR_INVALID_ARG).
 * It runs on the caller's current device.  The first call in a CUDA context
 * (the device's primary context, or one the caller created) looks up the
 * array's device address (cudaGetSymbolAddress) and caches it for that
 * context; make that first call before any stream capture.  The cache does
 * not survive cudaDeviceReset: a caller that resets the device must not call
 * this entry point again in the same process.  An empty V (n == 0 or
 * p == 0) writes 0 and reads none of dV, dW, dH (they may be NULL).  All
 * calls share the one array: calls whose work overlaps on the GPU
 * (different streams, or other host threads) race and may return wrong
 * values, so serialise them. */
#define NMFCU_NOALLOC_MAX_ROWS 524288
enum { NMFCU_OBJECTIVE_KL = 0, NMFCU_OBJECTIVE_FROBENIUS = 1 };
nmfcu_status nmfcu_objective_noalloc(int32_t kind, int64_t n, int64_t p, int64_t r,
                                     const double *dV, int64_t ldv, const double *dW,
                                     const double *dH, double *d_out, void *stream);

/* ---------------------------------------------------------------------- */
/* Misc                                                                    */
/* ---------------------------------------------------------------------- */

const char *nmfcu_last_error(void);
const char *nmfcu_status_string(nmfcu_status s);
int32_t nmfcu_abi_version(void);
/* Number of visible CUDA devices (0 without a GPU; never fails). */
int32_t nmfcu_device_count(void);

#ifdef __cplusplus
}
#endif

#endif /* NMFCU_H */

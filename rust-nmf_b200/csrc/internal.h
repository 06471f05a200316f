// internal.h -- services that nmfcu.cu offers the library's other
// translation units (C++ linkage: the nmfcu_* export list does not see them).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/nmfcu.h"

namespace nmfcu_internal {

// Records `msg` as the calling thread's nmfcu_last_error() and returns `s`.
nmfcu_status fail(nmfcu_status s, const std::string &msg);
// The same for a CUDA error (maps allocation failures to NMFCU_ERR_OOM).
nmfcu_status cuda_fail(cudaError_t e, const char *what);

// The option checks every run entry point applies (method, stop, sizes...).
nmfcu_status validate_options(const nmfcu_options *o, int64_t n, int64_t p, int64_t r);

// validate_options with another rank limit.
nmfcu_status validate_options_rank(const nmfcu_options *o, int64_t n, int64_t p, int64_t r,
                                   int64_t max_rank);
// Ranks above NMFCU_MAX_RANK (wide.cu): the option checks, and the FP64 loop
// on a device V (16-byte aligned base and pitch) with the factors copied in
// with `in_kind` and out with `out_kind`.  The caller holds the context's
// mutex with its device current.
nmfcu_status wide_validate(const nmfcu_options *o, int64_t n, int64_t p, int64_t r);
nmfcu_status wide_run(nmfcu_context *c, const nmfcu_options *o, int64_t n, int64_t p, int64_t r,
                      const double *V, int64_t ldv, const double *W0, const double *H0,
                      double *W, double *H, cudaMemcpyKind in_kind, cudaMemcpyKind out_kind,
                      double *d_dev, cudaStream_t s, int64_t *n_dev, int64_t *n_iter);
// Allocates the streaming passes' workspace (and the run state) of an
// n x p problem at the largest streaming rank.
nmfcu_status context_prepare(nmfcu_context *c, int64_t n, int64_t p);

// The per-device context behind the host-pointer API (created on first use).
nmfcu_status default_context(int device, nmfcu_context **out);

// A scratch buffer of the context that grows to at least `bytes` (slot
// 0..25, one owner per slot; the contents survive between calls).  Owners:
// 0..12, 16, 17 batch.cu; 13..15 linkage.cu; 18..23 sparse.cu (serve.cu
// uses the slots of its own contexts).
constexpr int kContextSlots = 26;
nmfcu_status context_buffer(nmfcu_context *c, int slot, size_t bytes, void **out);

cudaStream_t context_stream(nmfcu_context *c);
int context_sms(nmfcu_context *c);
int context_device(nmfcu_context *c);
std::mutex &context_mutex(nmfcu_context *c);
// Adds `launches` kernel launches to nmfcu_context_launch_count.
void count_launches(nmfcu_context *c, int64_t launches);

// Brackets the launches of one scope made by another translation unit for
// the context's timing hooks (the kernel classes of
// nmfcu_context_kernel_time) and its launch count.  The caller holds the
// context's mutex.
struct TimedScope {
    nmfcu_context *c;
    cudaStream_t s;
    int kclass;
    void *a;
    TimedScope(nmfcu_context *c, cudaStream_t s, int kclass, int launches = 1);
    ~TimedScope();
    TimedScope(const TimedScope &) = delete;
    TimedScope &operator=(const TimedScope &) = delete;
};
// Folds the recorded scopes into the per-class totals (waits for them).
void drain_timing(nmfcu_context *c);

// out = V X (trans 0) or V^T X (trans 1), V n x p f64 (pitch ldv), X with
// `l` columns, by the FP64 streaming passes in column chunks of at most
// NMFCU_MAX_RANK (one pass over V each).  The caller holds the context's
// mutex with its device current.  reset_state: clear the context's run state
// first; otherwise the passes do no work once the state says stopped.
// sync: wait for the stream and report a pass that gave up waiting.
nmfcu_status v_product_locked(nmfcu_context *c, int32_t trans, int64_t n, int64_t p, int64_t l,
                              const double *dV, int64_t ldv, const double *dX, int64_t ldx,
                              double *dOut, int64_t ldo, cudaStream_t s, bool reset_state,
                              bool sync);
// The context's device run state (an nmfcu::RunState).
void *context_state(nmfcu_context *c);

// Device bytes the context holds now.
size_t context_bytes(nmfcu_context *c);
// Bytes the context would add to run an n x p rank-r problem (f32: f32 main
// passes, including the f32 copy of an f64 V; tc: the split-bf16 tensor-core
// passes and their V / factor planes; method: the method's own buffers;
// tcr: brunet's split-bf16 tensor-core passes and their factor planes);
// 0 when its buffers suffice.
size_t context_growth(nmfcu_context *c, int64_t n, int64_t p, int64_t r, bool f32, bool tc,
                      int method, bool tcr = false);
// Bytes scratch slot `slot` would add to hold `bytes`.
size_t slot_growth(nmfcu_context *c, int slot, size_t bytes);
// Frees every device buffer of the context (it regrows on the next run).
void context_release(nmfcu_context *c);

// Makes `dev` current for the scope and restores the caller's device.
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            prev = -1;
            cudaGetLastError();
        }
        cudaSetDevice(dev);
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceScope(const DeviceScope &) = delete;
    DeviceScope &operator=(const DeviceScope &) = delete;
};

}  // namespace nmfcu_internal

#define NMFCU_CUDA_TRY(expr)                                                  \
    do {                                                                      \
        cudaError_t e_ = (expr);                                              \
        if (e_ != cudaSuccess) return nmfcu_internal::cuda_fail(e_, #expr);   \
    } while (0)

#define NMFCU_TRY(expr)                    \
    do {                                   \
        nmfcu_status s_ = (expr);          \
        if (s_ != NMFCU_OK) return s_;     \
    } while (0)

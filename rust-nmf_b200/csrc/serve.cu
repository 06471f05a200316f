// serve.cu -- request server for single factorisations, with continuous
// admission (each request still runs alone on its slot's stream; requests
// are not fused into shared launches).
//
// The reference has no server: every nmf() call runs to completion on the
// calling thread (python/nmf_rs/__init__.py:396-568, lib.rs:1934-2169).
// Here requests of any shape, rank and method are submitted from any host
// thread and run concurrently on one GPU:
//
//   * a fixed set of worker slots, each with its own engine context (device
//     workspace + CUDA stream) and host thread; the work of different slots
//     overlaps on the device;
//   * admission by device-memory footprint: a queued request starts on a free
//     slot when the bytes that slot would have to add (its V/W/H copies plus
//     the engine workspace of that shape, computed from the same list the
//     engine allocates from) fit in the server's budget next to what every
//     slot holds; requests that arrive while others run are admitted as
//     slots and memory free up, first come first served within two size
//     classes: large requests (V of at least 2^25 elements, whose passes
//     alone keep HBM busy) run on at most a quarter of the slots, so a
//     small request never queues behind a run of large ones and a large
//     one is never overtaken by later large ones;
//   * a slot keeps its buffers for the next request (no allocation on the
//     common path) and releases them when the request at the head of the
//     queue cannot fit otherwise;
//   * per-request results are those of the single-solve engine on the same
//     inputs: each request runs alone on its slot's stream with a plan that
//     depends only on its shape and the device, so a result does not depend
//     on what else is in flight.
//
// Latency is measured on the host from submission to completion.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/nmfcu.h"
#include "internal.h"

using nmfcu_internal::fail;

namespace {

using Clock = std::chrono::steady_clock;

// Scratch slots of a worker's context holding the request's device copies
// (offset method: the row offsets in and out).
constexpr int kSlotV = 12, kSlotW = 13, kSlotH = 14, kSlotDev = 15, kSlotOff = 16;
// A queued request that does not fit in device memory may be passed over
// this many times by later ones that do; after that nothing behind it is
// admitted before it.
constexpr int kMaxBypass = 8;
// Requests whose V has at least this many elements are "large".
constexpr int64_t kLargeElems = int64_t(1) << 25;

enum ReqState { kQueued = 0, kRunning = 1, kDone = 2 };

struct Request {
    int64_t id = 0;
    nmfcu_options opt{};
    int64_t n = 0, p = 0, r = 0, ldv = 0;
    const double *V = nullptr, *W0 = nullptr, *H0 = nullptr;
    double *W = nullptr, *H = nullptr, *dev = nullptr;
    const double *off0 = nullptr;  // offset method: starting offsets (NULL: rowMeans)
    double *off = nullptr;         // offset method: final offsets
    int64_t dev_cap = 0;
    int state = kQueued;
    int bypassed = 0;
    nmfcu_status status = NMFCU_OK;
    std::string error;
    int64_t n_iter = 0, n_dev = 0;
    Clock::time_point t_submit, t_start, t_done;
};

int64_t pitch_of(int64_t p) { return std::max<int64_t>(16, (p + 15) / 16 * 16); }

size_t v_bytes(const Request &q) { return sizeof(double) * (size_t)q.n * (size_t)pitch_of(q.p); }
size_t dev_slots(const Request &q) {
    return q.opt.stop == NMFCU_STOP_STATIONARY ? (size_t)q.opt.max_iter + 1 : 1;
}

// Bytes context `c` would add to run request q.
size_t growth_on(nmfcu_context *c, const Request &q) {
    const bool tc = q.opt.precision == NMFCU_PREC_BF16X3 && q.opt.method != NMFCU_BRUNET &&
                    q.opt.method != NMFCU_NSNMF;
    const bool f32 = q.opt.precision == NMFCU_PREC_FP32 || (q.opt.precision == NMFCU_PREC_BF16X3 && !tc);
    const bool tcr = q.opt.precision == NMFCU_PREC_BF16X3 &&
                     (q.opt.method == NMFCU_BRUNET || q.opt.method == NMFCU_NSNMF);
    return nmfcu_internal::context_growth(c, q.n, q.p, q.r, f32, tc, q.opt.method, tcr) +
           nmfcu_internal::slot_growth(c, kSlotV, v_bytes(q)) +
           nmfcu_internal::slot_growth(c, kSlotW, sizeof(double) * (size_t)(q.n * q.r)) +
           nmfcu_internal::slot_growth(c, kSlotH, sizeof(double) * (size_t)(q.r * q.p)) +
           nmfcu_internal::slot_growth(c, kSlotDev, sizeof(double) * dev_slots(q)) +
           (q.off ? nmfcu_internal::slot_growth(c, kSlotOff, 2 * sizeof(double) * (size_t)q.n)
                  : 0);
}

bool is_large(const Request &q) { return q.n * q.p >= kLargeElems; }

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct nmfcu_server {
    int device = 0;
    size_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work;  // queue, memory or shutdown changed
    std::condition_variable cv_done;  // a request finished
    bool stopping = false;
    int64_t next_id = 1;
    std::deque<Request *> queue;
    std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;

    struct Slot {
        nmfcu_context *ctx = nullptr;
        size_t held = 0;  // bytes the slot holds or has reserved
        bool busy = false;
        std::thread th;
    };
    std::vector<Slot> slots;
    nmfcu_context *probe = nullptr;  // never runs: sizes a request from nothing
    size_t in_use = 0, peak = 0;
    int running = 0, peak_running = 0, running_large = 0;

    // Statistics since creation or the last reset.
    int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, iterations = 0;
    int64_t launches = 0;
    std::vector<double> latency_ms, queue_ms;
    bool have_first = false;
    Clock::time_point first_submit, last_done;

    void worker(int k);
    Request *pick(int k, size_t *growth);
    void run(int k, Request *q);
};

// The oldest queued request that may start on slot k: a large one only
// while fewer than a quarter of the slots run large ones (later small ones
// go past it meanwhile), and only if what it adds fits in the budget next
// to what every slot holds.  A request passed over kMaxBypass times for
// memory blocks everything behind it until it fits, so no request waits
// for ever.
Request *nmfcu_server::pick(int k, size_t *growth) {
    Slot &sl = slots[k];
    const int max_large = std::max<int>(1, (int)slots.size() / 4);
    for (auto it = queue.begin(); it != queue.end(); ++it) {
        Request *q = *it;
        if (is_large(*q) && running_large >= max_large) continue;
        const size_t g = growth_on(sl.ctx, *q);
        if (in_use + g > budget) {
            if (q->bypassed >= kMaxBypass) return nullptr;
            continue;
        }
        // Requests ahead of it that did not fit were passed over once more.
        for (auto jt = queue.begin(); jt != it; ++jt)
            if (!(is_large(**jt) && running_large >= max_large)) (*jt)->bypassed++;
        queue.erase(it);
        *growth = g;
        return q;
    }
    return nullptr;
}

void nmfcu_server::worker(int k) {
    Slot &sl = slots[k];
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        if (stopping) return;
        size_t g = 0;
        Request *q = queue.empty() ? nullptr : pick(k, &g);
        if (!q) {
            if (!queue.empty() && sl.held > 0) {
                // The queue's head does not fit: give back this slot's cache.
                const size_t held = sl.held;
                lk.unlock();
                nmfcu_internal::context_release(sl.ctx);
                lk.lock();
                in_use -= held;
                sl.held = 0;
                cv_work.notify_all();
                continue;
            }
            cv_work.wait(lk);
            continue;
        }
        sl.held += g;
        in_use += g;
        peak = std::max(peak, in_use);
        sl.busy = true;
        running++;
        const bool large = is_large(*q);
        if (large) running_large++;
        peak_running = std::max(peak_running, running);
        q->state = kRunning;
        q->t_start = Clock::now();
        lk.unlock();
        const int64_t l0 = nmfcu_context_launch_count(sl.ctx);
        run(k, q);
        const int64_t dl = nmfcu_context_launch_count(sl.ctx) - l0;
        const size_t now_held = nmfcu_internal::context_bytes(sl.ctx);
        lk.lock();
        in_use = in_use - sl.held + now_held;
        sl.held = now_held;
        peak = std::max(peak, in_use);
        sl.busy = false;
        running--;
        if (large) running_large--;
        q->t_done = Clock::now();
        q->state = kDone;
        if (q->status == NMFCU_OK) {
            completed++;
            iterations += q->n_iter;
            launches += dl;
            latency_ms.push_back(ms_between(q->t_submit, q->t_done));
            queue_ms.push_back(ms_between(q->t_submit, q->t_start));
        } else {
            failed++;
        }
        last_done = q->t_done;
        cv_done.notify_all();
        cv_work.notify_all();
    }
}

// One request on slot k: copy in, the engine's device-pointer run on the
// slot's stream, copy out.  Errors are recorded on the request.
void nmfcu_server::run(int k, Request *q) {
    nmfcu_context *c = slots[k].ctx;
    auto record = [&](nmfcu_status s) {
        q->status = s;
        if (s != NMFCU_OK) q->error = nmfcu_last_error();
        return s;
    };
    nmfcu_internal::DeviceScope dg(device);
    cudaStream_t s = nmfcu_internal::context_stream(c);
    const int64_t ld = pitch_of(q->p);
    void *dV = nullptr, *dW = nullptr, *dH = nullptr, *dD = nullptr;
    if (record(nmfcu_internal::context_buffer(c, kSlotV, v_bytes(*q), &dV)) != NMFCU_OK) return;
    if (record(nmfcu_internal::context_buffer(c, kSlotW, sizeof(double) * (size_t)(q->n * q->r), &dW)) != NMFCU_OK) return;
    if (record(nmfcu_internal::context_buffer(c, kSlotH, sizeof(double) * (size_t)(q->r * q->p), &dH)) != NMFCU_OK) return;
    if (record(nmfcu_internal::context_buffer(c, kSlotDev, sizeof(double) * dev_slots(*q), &dD)) != NMFCU_OK) return;
    cudaError_t e = cudaSuccess;
    if (q->n > 0 && q->p > 0)
        e = cudaMemcpy2DAsync(dV, ld * 8, q->V, q->ldv * 8, q->p * 8, q->n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && q->n * q->r > 0)
        e = cudaMemcpyAsync(dW, q->W0, sizeof(double) * q->n * q->r, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && q->r * q->p > 0)
        e = cudaMemcpyAsync(dH, q->H0, sizeof(double) * q->r * q->p, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        record(nmfcu_internal::cuda_fail(e, "request upload"));
        return;
    }
    const bool stat = q->opt.stop == NMFCU_STOP_STATIONARY;
    int64_t nd = 0, ni = 0;
    if (q->off) {
        // The offset method: the starting offsets in, the final ones out.
        void *dO = nullptr;
        if (record(nmfcu_internal::context_buffer(c, kSlotOff, 2 * sizeof(double) * (size_t)q->n, &dO)) != NMFCU_OK)
            return;
        double *d_off0 = static_cast<double *>(dO), *d_off = d_off0 + q->n;
        if (q->off0 && q->n > 0)
            e = cudaMemcpyAsync(d_off0, q->off0, sizeof(double) * q->n, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
            record(nmfcu_internal::cuda_fail(e, "request upload"));
            return;
        }
        if (record(nmfcu_run_offset_device(c, &q->opt, q->n, q->p, q->r, dV, NMFCU_F64, ld,
                                           nullptr, 0, (double *)dW, (double *)dH,
                                           q->off0 ? d_off0 : nullptr, d_off,
                                           stat ? (double *)dD : nullptr, &nd, &ni, s)) != NMFCU_OK)
            return;
        if (q->n > 0)
            e = cudaMemcpyAsync(q->off, d_off, sizeof(double) * q->n, cudaMemcpyDeviceToHost, s);
    } else if (record(nmfcu_run_device(c, &q->opt, q->n, q->p, q->r, dV, NMFCU_F64, ld, nullptr,
                                       0, (double *)dW, (double *)dH,
                                       stat ? (double *)dD : nullptr, &nd, &ni, s)) != NMFCU_OK) {
        return;
    }
    if (e == cudaSuccess && q->n * q->r > 0)
        e = cudaMemcpyAsync(q->W, dW, sizeof(double) * q->n * q->r, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && q->r * q->p > 0)
        e = cudaMemcpyAsync(q->H, dH, sizeof(double) * q->r * q->p, cudaMemcpyDeviceToHost, s);
    const int64_t keep = std::min<int64_t>(nd, q->dev_cap);
    if (e == cudaSuccess && keep > 0 && q->dev)
        e = cudaMemcpyAsync(q->dev, dD, sizeof(double) * keep, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        record(nmfcu_internal::cuda_fail(e, "request download"));
        return;
    }
    q->n_iter = ni;
    q->n_dev = nd;
    record(NMFCU_OK);
}

namespace {

double percentile(std::vector<double> v, double pct) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    // nearest rank
    size_t idx = (size_t)std::ceil(pct / 100.0 * (double)v.size());
    idx = std::min(std::max<size_t>(idx, 1), v.size()) - 1;
    return v[idx];
}

}  // namespace

extern "C" {

nmfcu_status nmfcu_server_create(int32_t device, int32_t nslots, int64_t budget_bytes,
                                 nmfcu_server **out) {
    if (!out) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    *out = nullptr;
    if (nslots < 1 || nslots > 64) return fail(NMFCU_ERR_INVALID_ARG, "slots must be in [1, 64]");
    if (budget_bytes < 0) return fail(NMFCU_ERR_INVALID_ARG, "budget must be >= 0");
    std::unique_ptr<nmfcu_server> srv(new nmfcu_server());
    srv->device = device;
    NMFCU_TRY(nmfcu_context_create(device, &srv->probe));
    if (budget_bytes == 0) {
        nmfcu_internal::DeviceScope dg(device);
        size_t fr = 0, total = 0;
        NMFCU_CUDA_TRY(cudaMemGetInfo(&fr, &total));
        budget_bytes = (int64_t)(fr / 10 * 9);
    }
    srv->budget = (size_t)budget_bytes;
    srv->slots.resize(nslots);
    for (auto &sl : srv->slots) {
        nmfcu_status s = nmfcu_context_create(device, &sl.ctx);
        if (s != NMFCU_OK) {
            for (auto &t : srv->slots)
                if (t.ctx) nmfcu_context_destroy(t.ctx);
            nmfcu_context_destroy(srv->probe);
            return s;
        }
    }
    nmfcu_server *raw = srv.get();
    for (int k = 0; k < nslots; k++) raw->slots[k].th = std::thread([raw, k] { raw->worker(k); });
    *out = srv.release();
    return NMFCU_OK;
}

void nmfcu_server_destroy(nmfcu_server *srv) {
    if (!srv) return;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stopping = true;
        for (Request *q : srv->queue) {
            q->state = kDone;
            q->status = NMFCU_ERR_CANCELLED;
            q->error = "server destroyed before the request started";
        }
        srv->queue.clear();
        srv->cv_work.notify_all();
        srv->cv_done.notify_all();
    }
    for (auto &sl : srv->slots)
        if (sl.th.joinable()) sl.th.join();
    for (auto &sl : srv->slots) nmfcu_context_destroy(sl.ctx);
    nmfcu_context_destroy(srv->probe);
    delete srv;
}

namespace {
nmfcu_status submit(nmfcu_server *srv, const nmfcu_options *opt, int64_t n, int64_t p, int64_t r,
                    const double *V, int64_t ldv, const double *W0, const double *H0, double *W,
                    double *H, const double *off0, double *off, double *deviances,
                    int64_t dev_cap, int64_t *request_id) {
    if (!srv || !opt || !request_id) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    NMFCU_TRY(nmfcu_internal::validate_options(opt, n, p, r));
    if (opt->method == NMFCU_OFFSET && !off)
        return fail(NMFCU_ERR_UNSUPPORTED,
                    "the offset method returns its row offsets: submit it through "
                    "nmfcu_server_submit_offset");
    if (opt->method != NMFCU_OFFSET && off)
        return fail(NMFCU_ERR_INVALID_ARG, "nmfcu_server_submit_offset takes method offset only");
    if (opt->method == NMFCU_LSNMF)
        return fail(NMFCU_ERR_UNSUPPORTED,
                    "lsNMF takes a weight matrix: run it through nmfcu_run_weighted");
    if (opt->method == NMFCU_SNMF_R || opt->method == NMFCU_SNMF_L)
        return fail(NMFCU_ERR_UNSUPPORTED, "snmf/r and snmf/l run through nmfcu_run");
    if (!V || !W0 || !H0 || !W || !H) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    if (ldv < p) return fail(NMFCU_ERR_INVALID_ARG, "ldv must be >= p");
    if (dev_cap < 0 || (dev_cap > 0 && !deviances))
        return fail(NMFCU_ERR_INVALID_ARG, "deviances buffer missing");
    std::unique_ptr<Request> q(new Request());
    q->opt = *opt;
    q->opt.device = srv->device;
    q->n = n;
    q->p = p;
    q->r = r;
    q->ldv = ldv;
    q->V = V;
    q->W0 = W0;
    q->H0 = H0;
    q->W = W;
    q->H = H;
    q->dev = deviances;
    q->dev_cap = dev_cap;
    q->off0 = off0;
    q->off = off;
    // A request that cannot fit even on an empty server is refused now.
    const size_t need = growth_on(srv->probe, *q);
    if (need > srv->budget)
        return fail(NMFCU_ERR_OOM, "request needs " + std::to_string(need) +
                                       " device bytes; the server's budget is " +
                                       std::to_string(srv->budget));
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->stopping) return fail(NMFCU_ERR_INVALID_ARG, "server is shutting down");
    q->id = srv->next_id++;
    q->t_submit = Clock::now();
    if (!srv->have_first) {
        srv->have_first = true;
        srv->first_submit = q->t_submit;
    }
    srv->submitted++;
    *request_id = q->id;
    srv->queue.push_back(q.get());
    srv->reqs.emplace(q->id, std::move(q));
    srv->cv_work.notify_all();
    return NMFCU_OK;
}
}  // namespace

nmfcu_status nmfcu_server_submit(nmfcu_server *srv, const nmfcu_options *opt, int64_t n,
                                 int64_t p, int64_t r, const double *V, int64_t ldv,
                                 const double *W0, const double *H0, double *W, double *H,
                                 double *deviances, int64_t dev_cap, int64_t *request_id) {
    return submit(srv, opt, n, p, r, V, ldv, W0, H0, W, H, nullptr, nullptr, deviances, dev_cap,
                  request_id);
}

nmfcu_status nmfcu_server_submit_offset(nmfcu_server *srv, const nmfcu_options *opt, int64_t n,
                                        int64_t p, int64_t r, const double *V, int64_t ldv,
                                        const double *W0, const double *H0,
                                        const double *offset0, double *W, double *H,
                                        double *offset, double *deviances, int64_t dev_cap,
                                        int64_t *request_id) {
    if (!offset) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    if (opt && opt->method != NMFCU_OFFSET)
        return fail(NMFCU_ERR_INVALID_ARG, "nmfcu_server_submit_offset takes method offset only");
    return submit(srv, opt, n, p, r, V, ldv, W0, H0, W, H, offset0, offset, deviances, dev_cap,
                  request_id);
}

nmfcu_status nmfcu_server_poll(nmfcu_server *srv, int64_t request_id, int32_t *state) {
    if (!srv || !state) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(request_id);
    if (it == srv->reqs.end()) return fail(NMFCU_ERR_INVALID_ARG, "unknown request id");
    *state = it->second->state;
    return NMFCU_OK;
}

nmfcu_status nmfcu_server_wait(nmfcu_server *srv, int64_t request_id, int64_t timeout_ms,
                               int64_t *n_iter, int64_t *n_deviances) {
    if (!srv) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(request_id);
    if (it == srv->reqs.end()) return fail(NMFCU_ERR_INVALID_ARG, "unknown request id");
    Request *q = it->second.get();
    auto done = [&] { return q->state == kDone; };
    if (timeout_ms < 0) {
        srv->cv_done.wait(lk, done);
    } else if (!srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
        return fail(NMFCU_ERR_TIMEOUT, "request not finished within the wait's time limit");
    }
    if (n_iter) *n_iter = q->n_iter;
    if (n_deviances) *n_deviances = std::min(q->n_dev, q->dev_cap);
    const nmfcu_status s = q->status;
    const std::string msg = q->error;
    srv->reqs.erase(it);  // the id is released once its result is collected
    if (s != NMFCU_OK) return fail(s, msg);
    return NMFCU_OK;
}

nmfcu_status nmfcu_server_cancel(nmfcu_server *srv, int64_t request_id) {
    if (!srv) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(request_id);
    if (it == srv->reqs.end()) return fail(NMFCU_ERR_INVALID_ARG, "unknown request id");
    Request *q = it->second.get();
    if (q->state != kQueued)
        return fail(NMFCU_ERR_INVALID_ARG, "only a request that has not started can be cancelled");
    srv->queue.erase(std::find(srv->queue.begin(), srv->queue.end(), q));
    q->state = kDone;
    q->status = NMFCU_ERR_CANCELLED;
    q->error = "request cancelled before it started";
    srv->cancelled++;
    srv->cv_done.notify_all();
    srv->cv_work.notify_all();
    return NMFCU_OK;
}

nmfcu_status nmfcu_server_get_stats(nmfcu_server *srv, nmfcu_server_stats *out) {
    if (!srv || !out) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    std::lock_guard<std::mutex> lk(srv->mu);
    nmfcu_server_stats st{};
    st.submitted = srv->submitted;
    st.completed = srv->completed;
    st.failed = srv->failed;
    st.cancelled = srv->cancelled;
    st.queued = (int64_t)srv->queue.size();
    st.running = srv->running;
    st.iterations = srv->iterations;
    st.wall_ms = (srv->have_first && srv->completed + srv->failed > 0)
                     ? std::max(0.0, ms_between(srv->first_submit, srv->last_done))
                     : 0.0;
    st.p50_ms = percentile(srv->latency_ms, 50.0);
    st.p99_ms = percentile(srv->latency_ms, 99.0);
    st.max_ms = srv->latency_ms.empty()
                    ? 0.0
                    : *std::max_element(srv->latency_ms.begin(), srv->latency_ms.end());
    double qs = 0.0;
    for (double v : srv->queue_ms) qs += v;
    st.mean_queue_ms = srv->queue_ms.empty() ? 0.0 : qs / (double)srv->queue_ms.size();
    st.budget_bytes = (int64_t)srv->budget;
    st.in_use_bytes = (int64_t)srv->in_use;
    st.peak_bytes = (int64_t)srv->peak;
    st.launches = srv->launches;
    st.slots = (int32_t)srv->slots.size();
    st.peak_running = srv->peak_running;
    *out = st;
    return NMFCU_OK;
}

nmfcu_status nmfcu_server_reset_stats(nmfcu_server *srv) {
    if (!srv) return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->submitted = srv->completed = srv->failed = srv->cancelled = srv->iterations = 0;
    srv->launches = 0;
    srv->latency_ms.clear();
    srv->queue_ms.clear();
    srv->have_first = false;
    srv->peak = srv->in_use;
    srv->peak_running = srv->running;
    return NMFCU_OK;
}

}  // extern "C"

// linkage.cu -- consensus statistics on the device: Brunet's cophenetic
// correlation (average-linkage tree on the distances 1 - C) and Kim & Park's
// dispersion coefficient of a p x p consensus matrix C.
//
// The consensus workflow these summarise is examples/build_scaling_notebook.py
// :121-141 of the reference (connectivity -> consensus -> average linkage on
// 1 - C via scipy -> cophenetic correlation; dispersion = mean 4 (C - 0.5)^2).
//
// Average linkage (UPGMA) is built by the nearest-neighbour chain
// (Murtagh 1983; Muellner, "Modern hierarchical, agglomerative clustering
// algorithms", 2011): grow a chain of nearest neighbours from the first
// active cluster until its last two elements are reciprocal nearest
// neighbours, merge them (the merged cluster keeps the larger index), and
// update its distances with the Lance-Williams average rule
//   d(i, a u b) = (n_a d(i, a) + n_b d(i, b)) / (n_a + n_b).
// A nearest neighbour is the strictly smallest distance in index order,
// the chain's previous element winning ties -- the same choices (and the
// same f64 update, no FMA) as scipy.cluster.hierarchy.linkage's chain, so
// the tree is the same one even where consensus distances tie.
//
// The cophenetic distance of a pair is the height of the merge that joins
// it.  In an average-linkage tree a merge of clusters A and B happens at the
// mean original distance over A x B, so the sums the correlation needs come
// from the merges alone:  sum over A x B of d = |A||B| h, hence with
// N = p (p - 1) / 2 pairs, mean distance m_d and mean cophenetic distance
// m_c = sum_k n_k h_k / N (n_k = |A_k||B_k|),
//   cov = sum_k n_k (h_k - m_c)(h_k - m_d),  var_c = sum_k n_k (h_k - m_c)^2,
// and var_d from one pass over the pairs.  Nothing of size p^2 beyond D.
#include <cfloat>
#include <climits>
#include <cmath>
#include <vector>
#include <algorithm>

#include "internal.h"

namespace {

constexpr int kT = 1024;  // threads of the single-block kernels
constexpr int kR = 256;   // threads of the reduction kernels

// D = 1 - C in f64 (p x p, pitch p), zero diagonal (the reference fills the
// consensus diagonal with 1 before taking distances).
__global__ void distances_from_consensus(const float *__restrict__ C, int64_t ldc, int p,
                                         double *__restrict__ D) {
    const int64_t total = (int64_t)p * p;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / p, j = t - i * p;
        D[t] = (i == j) ? 0.0 : 1.0 - (double)C[i * ldc + j];
    }
}

__device__ double block_sum(double v, double *red) {
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    const double out = red[0];
    __syncthreads();
    return out;
}

// Per-block sums over the pairs i < j of d (mean == nullptr) or of
// (d - mean)^2; block b takes rows b, b + gridDim.x, ...
__global__ void __launch_bounds__(kR) pair_sums(const double *__restrict__ D, int p,
                                                const double *__restrict__ mean,
                                                double *__restrict__ part) {
    __shared__ double red[kR];
    const double m = mean ? *mean : 0.0;
    double acc = 0.0;
    for (int i = blockIdx.x; i < p; i += gridDim.x)
        for (int j = i + 1 + threadIdx.x; j < p; j += kR) {
            const double d = D[(size_t)i * p + j];
            acc += mean ? (d - m) * (d - m) : d;
        }
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Per-block sums of 4 (C - 0.5)^2 over all p x p entries (diagonal read as 1).
__global__ void __launch_bounds__(kR) dispersion_sums(const float *__restrict__ C, int64_t ldc,
                                                      int p, double *__restrict__ part) {
    __shared__ double red[kR];
    double acc = 0.0;
    for (int i = blockIdx.x; i < p; i += gridDim.x)
        for (int j = threadIdx.x; j < p; j += kR) {
            const double c = (i == j) ? 1.0 : (double)C[(size_t)i * ldc + j];
            acc += 4.0 * (c - 0.5) * (c - 0.5);
        }
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// out[0] = scale * (the B partials, summed in a fixed tree order).
__global__ void __launch_bounds__(kR) finish_sum(const double *__restrict__ part, int B,
                                                 double scale, double *__restrict__ out) {
    __shared__ double red[kR];
    double acc = 0.0;
    for (int b = threadIdx.x; b < B; b += kR) acc += part[b];
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) out[0] = s * scale;
}

struct VI {
    double v;
    int i;
};
__device__ __forceinline__ VI better(VI a, VI b) {
    return (b.v < a.v || (b.v == a.v && b.i < a.i)) ? b : a;
}
// The smallest (value, index) pair of the block, broadcast to every thread.
__device__ VI block_argmin(VI mine, VI *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        VI other;
        other.v = __shfl_down_sync(0xffffffffu, mine.v, o);
        other.i = __shfl_down_sync(0xffffffffu, mine.i, o);
        mine = better(mine, other);
    }
    if (lane == 0) red[warp] = mine;
    __syncthreads();
    if (warp == 0) {
        VI v = (lane < (int)(blockDim.x >> 5)) ? red[lane] : VI{INFINITY, INT_MAX};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            VI other;
            other.v = __shfl_down_sync(0xffffffffu, v.v, o);
            other.i = __shfl_down_sync(0xffffffffu, v.i, o);
            v = better(v, other);
        }
        if (lane == 0) red[32] = v;
    }
    __syncthreads();
    const VI out = red[32];
    __syncthreads();
    return out;
}

// Average-linkage tree of the p x p distances D (overwritten) by the
// nearest-neighbour chain, one block.  Writes each merge's height and pair
// count n_a n_b.  Every loop below ends: each merge takes at most p chain
// extensions (a chain holds distinct clusters), and there are p - 1 merges.
__device__ void nn_chain_tree(double *__restrict__ D, int p, int *__restrict__ size,
                              int *__restrict__ chain, double *__restrict__ height,
                              double *__restrict__ npair) {
    __shared__ VI red[33];
    __shared__ int s_len;
    const int tid = threadIdx.x;
    for (int i = tid; i < p; i += kT) size[i] = 1;
    if (tid == 0) s_len = 0;
    __syncthreads();
    for (int k = 0; k < p - 1; k++) {
        if (s_len == 0) {  // start a chain at the first active cluster
            VI mine{INFINITY, INT_MAX};
            for (int i = tid; i < p; i += kT)
                if (size[i] > 0) mine = better(mine, VI{0.0, i});
            const VI first = block_argmin(mine, red);
            if (tid == 0) {
                chain[0] = first.i;
                s_len = 1;
            }
            __syncthreads();
        }
        int x = -1, y = -1;
        double cur = 0.0;
        for (int guard = 0; guard <= p; guard++) {
            const int len = s_len;
            x = chain[len - 1];
            const int prev = (len > 1) ? chain[len - 2] : -1;
            const double *row = D + (size_t)x * p;
            VI mine{INFINITY, INT_MAX};
            for (int i = tid; i < p; i += kT)
                if (i != x && size[i] > 0) mine = better(mine, VI{row[i], i});
            const VI best = block_argmin(mine, red);
            if (prev >= 0 && !(best.v < row[prev])) {
                y = prev;  // reciprocal nearest neighbours: merge
                cur = row[prev];
                break;
            }
            y = best.i;
            cur = best.v;
            if (tid == 0) {
                chain[len] = y;
                s_len = len + 1;
            }
            __syncthreads();
        }
        const int a = x < y ? x : y, b = x < y ? y : x;  // b keeps the merged cluster
        const int na = size[a], nb = size[b];
        const double fa = (double)na, fb = (double)nb, fs = (double)(na + nb);
        const double *ra = D + (size_t)a * p;
        double *rb = D + (size_t)b * p;
        for (int i = tid; i < p; i += kT) {
            if (i == a || i == b || size[i] == 0) continue;
            const double d = __ddiv_rn(__dadd_rn(__dmul_rn(fa, ra[i]), __dmul_rn(fb, rb[i])), fs);
            rb[i] = d;
            D[(size_t)i * p + b] = d;
        }
        __syncthreads();
        if (tid == 0) {
            height[k] = cur;
            npair[k] = fa * fb;
            size[a] = 0;
            size[b] = na + nb;
            s_len -= 2;
        }
        __syncthreads();
    }
}

// One tree per block: block m builds the tree of matrix m (its distances,
// sizes and chain `dstride` / `istride` elements after matrix m - 1's, its
// merges `hstride` after).  The trees of a batch build concurrently on
// different multiprocessors.
__global__ void __launch_bounds__(kT) nn_chain_average(double *__restrict__ D, int p,
                                                       int64_t dstride, int *__restrict__ size,
                                                       int *__restrict__ chain, int64_t istride,
                                                       double *__restrict__ height,
                                                       double *__restrict__ npair,
                                                       int64_t hstride) {
    const int64_t m = blockIdx.x;
    nn_chain_tree(D + m * dstride, p, size + m * istride, chain + m * istride,
                  height + m * hstride, npair + m * hstride);
}

// out[0] = the cophenetic correlation from the merges (height, npair), the
// sum of the distances (dsum) and of their squared deviations (dvar); 1 when
// either side has no spread (the reference's convention).
__global__ void __launch_bounds__(kR) cophenetic_from_merges(
    const double *__restrict__ height, const double *__restrict__ npair, int m,
    const double *__restrict__ dsum, const double *__restrict__ dvar, double npairs,
    double *__restrict__ out) {
    __shared__ double red[kR];
    double a = 0.0;
    for (int k = threadIdx.x; k < m; k += kR) a += npair[k] * height[k];
    const double mc = block_sum(a, red) / npairs;
    const double md = dsum[0] / npairs;
    double cv = 0.0, vc = 0.0;
    for (int k = threadIdx.x; k < m; k += kR) {
        cv += npair[k] * (height[k] - mc) * (height[k] - md);
        vc += npair[k] * (height[k] - mc) * (height[k] - mc);
    }
    const double cov = block_sum(cv, red);
    const double var_c = block_sum(vc, red);
    if (threadIdx.x == 0) {
        const double var_d = dvar[0];
        out[0] = (var_d > 0.0 && var_c > 0.0) ? cov / sqrt(var_d * var_c) : 1.0;
    }
}

// The statistics of `count` consensus matrices (matrix m at dC + m * stride),
// the per-pair and dispersion sums one matrix at a time, the trees of all
// matrices in one launch (one block each).
nmfcu_status consensus_stats(nmfcu_context *ctx, int count, int64_t p, const float *dC,
                             int64_t ldc, int64_t stride, double *cophenetic, double *dispersion,
                             cudaStream_t s) {
    const int sms = nmfcu_internal::context_sms(ctx);
    const int B = sms * 8;
    const size_t pp = (size_t)p * (size_t)p;
    const size_t nd = 2 * (size_t)p + B + 8;  // doubles of one matrix: height, npair, part, stat
    void *pD = nullptr, *pi = nullptr, *pd = nullptr;
    NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 13, sizeof(double) * pp * count, &pD));
    NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 14, sizeof(int) * 2 * (size_t)p * count, &pi));
    NMFCU_TRY(nmfcu_internal::context_buffer(ctx, 15, sizeof(double) * nd * count, &pd));
    double *D0 = static_cast<double *>(pD);
    int *size0 = static_cast<int *>(pi);
    double *dbl0 = static_cast<double *>(pd);
    const double npairs = (double)p * (double)(p - 1) / 2.0;
    const unsigned g = (unsigned)std::min<int64_t>(((int64_t)p * p + kR - 1) / kR, 4096);
    int launches = 0;
    for (int m = 0; m < count; m++) {
        const float *C = dC + (size_t)m * stride;
        double *D = D0 + pp * m;
        double *part = dbl0 + nd * m + 2 * (size_t)p;
        double *stat = part + B;  // [sum d, mean d, sum (d - mean)^2, dispersion, cophenetic]
        distances_from_consensus<<<g, kR, 0, s>>>(C, ldc, (int)p, D);
        pair_sums<<<B, kR, 0, s>>>(D, (int)p, nullptr, part);
        finish_sum<<<1, kR, 0, s>>>(part, B, 1.0, stat);
        finish_sum<<<1, kR, 0, s>>>(part, B, npairs > 0 ? 1.0 / npairs : 0.0, stat + 1);
        pair_sums<<<B, kR, 0, s>>>(D, (int)p, stat + 1, part);
        finish_sum<<<1, kR, 0, s>>>(part, B, 1.0, stat + 2);
        dispersion_sums<<<B, kR, 0, s>>>(C, ldc, (int)p, part);
        finish_sum<<<1, kR, 0, s>>>(part, B, 1.0 / ((double)p * (double)p), stat + 3);
        launches += 8;
    }
    if (p >= 2) {
        nn_chain_average<<<count, kT, 0, s>>>(D0, (int)p, (int64_t)pp, size0, size0 + p,
                                              2 * p, dbl0, dbl0 + p, (int64_t)nd);
        launches += 1;
        for (int m = 0; m < count; m++) {
            double *h = dbl0 + nd * m;
            double *stat = h + 2 * (size_t)p + B;
            cophenetic_from_merges<<<1, kR, 0, s>>>(h, h + p, (int)p - 1, stat, stat + 2, npairs,
                                                    stat + 4);
        }
        launches += count;
    }
    NMFCU_CUDA_TRY(cudaGetLastError());
    nmfcu_internal::count_launches(ctx, launches);
    std::vector<double> host(5 * (size_t)count, 0.0);
    for (int m = 0; m < count; m++) {
        const double *stat = dbl0 + nd * m + 2 * (size_t)p + B;
        NMFCU_CUDA_TRY(cudaMemcpyAsync(host.data() + 5 * m, stat, sizeof(double) * (p >= 2 ? 5 : 4),
                                       cudaMemcpyDeviceToHost, s));
    }
    NMFCU_CUDA_TRY(cudaStreamSynchronize(s));
    for (int m = 0; m < count; m++) {
        dispersion[m] = host[5 * m + 3];
        cophenetic[m] = p >= 2 ? host[5 * m + 4] : 1.0;
    }
    return NMFCU_OK;
}

}  // namespace

extern "C" nmfcu_status nmfcu_consensus_stats_device(nmfcu_context *ctx, int64_t p,
                                                     const float *dC, int64_t ldc,
                                                     double *cophenetic, double *dispersion,
                                                     void *stream) {
    using nmfcu_internal::fail;
    if (!ctx || !dC || !cophenetic || !dispersion)
        return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    if (p < 1 || p > 200000) return fail(NMFCU_ERR_INVALID_ARG, "p must be in [1, 200000]");
    if (ldc < p) return fail(NMFCU_ERR_INVALID_ARG, "ldc must be >= p");
    std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(ctx));
    nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(ctx));
    return consensus_stats(ctx, 1, p, dC, ldc, 0, cophenetic, dispersion,
                           static_cast<cudaStream_t>(stream));
}

extern "C" nmfcu_status nmfcu_consensus_stats_batch_device(nmfcu_context *ctx, int32_t count,
                                                           int64_t p, const float *dC,
                                                           int64_t ldc, int64_t stride,
                                                           double *cophenetic,
                                                           double *dispersion, void *stream) {
    using nmfcu_internal::fail;
    if (!ctx || !dC || !cophenetic || !dispersion)
        return fail(NMFCU_ERR_INVALID_ARG, "NULL pointer");
    if (count < 1) return fail(NMFCU_ERR_INVALID_ARG, "count must be >= 1");
    if (p < 1 || p > 200000) return fail(NMFCU_ERR_INVALID_ARG, "p must be in [1, 200000]");
    if (ldc < p) return fail(NMFCU_ERR_INVALID_ARG, "ldc must be >= p");
    if (count > 1 && stride < ldc * p)
        return fail(NMFCU_ERR_INVALID_ARG, "stride must be >= ldc * p");
    std::lock_guard<std::mutex> lk(nmfcu_internal::context_mutex(ctx));
    nmfcu_internal::DeviceScope dg(nmfcu_internal::context_device(ctx));
    return consensus_stats(ctx, count, p, dC, ldc, stride, cophenetic, dispersion,
                           static_cast<cudaStream_t>(stream));
}

/*
 * device_common.cuh -- device helpers shared by the kernel translation units
 * (kernels_fast.cu for block size 9, kernels_nv.cu for the other sizes):
 * the fixed-order sums behind every residual norm.
 */
#ifndef TBS_DEVICE_COMMON_CUH
#define TBS_DEVICE_COMMON_CUH

#include "tbs_internal.hxx"

#include <cuda_runtime.h>

namespace tbs {

/* sum of p[t], p[t + stride], p[t + 2 stride], ... (t = threadIdx.x), added
 * in that order; eight loads are issued ahead of their adds so that their
 * latencies overlap without changing the sum */
static __device__ __forceinline__ double strided_sum(const double *p, int n, int stride) {
    double acc = 0.0;
    int t = threadIdx.x;
    for (; t + 7 * stride < n; t += 8 * stride) {
        double v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = __ldcg(p + t + k * stride);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc += v[k];
    }
    for (; t < n; t += stride) acc += __ldcg(p + t);
    return acc;
}

/* the device's global nanosecond clock */
static __device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

/* a launch's duration on the device clock, from its earliest CTA start to
 * the finish of its last CTA (called by that CTA's thread 0) */
static __device__ __forceinline__ void timer_launch_start(unsigned long long *timer) {
    if (timer && threadIdx.x == 0) atomicMin(timer, globaltimer_ns());
}
static __device__ __forceinline__ void timer_launch_end(unsigned long long *timer) {
    if (!timer || threadIdx.x != 0) return;
    const unsigned long long t1 = globaltimer_ns();
    const unsigned long long t0 = atomicExch(timer, ~0ull);
    if (t0 != ~0ull && t1 > t0) atomicAdd(timer + 1, t1 - t0);
    atomicAdd(timer + 2, 1ull);
}

/* Record the norm of a converged solve's true residual (NORM_CHECK): a
 * pass leaves the history alone and ends the solve; a failure counts a
 * restart, replaces the last history entry and the latest norm, and goes on
 * while sweeps are left.  Returns whether the solve goes on. */
static __device__ __forceinline__ bool record_check(SolveState *S, double *hist, double nrm) {
    const int sw = S->sweep;
    const bool pass = isfinite(nrm) && nrm <= S->tol * S->norm0;
    S->true_norm = nrm;
    S->checks += 1;
    if (!pass) {
        S->restarts += 1;
        if (sw < S->hist_cap) hist[sw] = nrm;
        S->last = nrm;
    }
    return !pass && isfinite(nrm) && sw < S->max_sweeps;
}

/* After a CTA's last tile: a ticket per CTA; the last CTA to finish adds
 * the n per-tile partials in a fixed order and, when asked, records the
 * norm like reduce_norm (history, sweep count, graph loop condition).
 * Called by every thread of the block. */
static __device__ bool finalize_total(const NormSink &ns, int n) {
    __shared__ unsigned ticket;
    __shared__ double red[32];
    if (!ns.partials || !ns.counter) return false;
    __syncthreads(); /* this CTA's partials are written */
    if (threadIdx.x == 0) {
        __threadfence();
        ticket = atomicAdd(ns.counter, 1u);
    }
    __syncthreads();
    if (ticket != gridDim.x - 1) return false;
    timer_launch_end(ns.timer); /* every other CTA has finished its tiles */
    if (!ns.state) {
        if (threadIdx.x == 0) *ns.counter = 0u;
        return true;
    }
    __threadfence();
    double acc = strided_sum(ns.partials, n, (int)blockDim.x);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) tot += red[w];
        const double nrm = sqrt(tot);
        SolveState *S = ns.state;
        if (ns.is_start == NORM_CHECK) {
            /* the true residual of a solve whose recursive residual passed */
            const bool go = record_check(S, ns.hist, nrm);
            if (ns.use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)ns.handle, go ? 1u : 0u);
            *ns.counter = 0u;
            return true;
        }
        if (ns.is_start) {
            S->sweep = 0;
            S->norm0 = nrm;
            S->true_norm = -1.0;
            S->checks = 0;
            S->restarts = 0;
        } else {
            S->sweep += 1;
        }
        const int sw = S->sweep;
        if (sw < S->hist_cap) ns.hist[sw] = nrm;
        S->last = nrm;
        const bool met = isfinite(nrm) && nrm <= S->tol * S->norm0;
        const bool go = isfinite(nrm) && !met && sw < S->max_sweeps;
        if (ns.use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)ns.handle, go ? 1u : 0u);
        if (ns.use_check)
            cudaGraphSetConditional((cudaGraphConditionalHandle)ns.check_handle,
                                    (!ns.is_start && met) ? 1u : 0u);
        *ns.counter = 0u;
    }
    return true;
}

}  // namespace tbs

#endif /* TBS_DEVICE_COMMON_CUH */

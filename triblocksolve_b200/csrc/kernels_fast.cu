/*
 * kernels_fast.cu -- TBS_ALGO_FP64 / TBS_ALGO_MIXED kernels for sm_100a,
 * plus the norm / permutation helpers every algorithm uses.
 *
 * The LIJ sweep of the reference (src/main.cxx:207-229) is
 *     dU = -M^-1 R ;  U += dU ;  R = rhs + J U
 * with M the block-tridiagonal part of J along each line.  Writing
 * J = M + O (O = couplings between different lines) and using M dU = -R,
 *     R_new = R + J dU = O dU,
 * so after the first sweep only the cross-line blocks are read to update
 * the residual.  The line solve is rewritten with explicit inverses:
 *     b_k  = -Dinv_k R_k                         (fast_resid, all cells)
 *     y_k  = b_k - G_k y_{k-1},   G_k = Dinv_k A_k (fast_thomas forward)
 *     dU_k = y_k - Gam_k dU_{k+1}, Gam_k = Dinv_k C_k (backward)
 * where Dinv_k = (D_k - A_k Gam_{k-1})^-1 is the inverse of the block-Thomas
 * pivot of src/okl/lineLU_v2.okl:58-182.  The recurrence on each line is
 * then one 9x9 matvec per cell; everything else is data parallel.
 *
 * Data are "position" ordered: cells in line order, each line starting at a
 * multiple of 4 positions, so that runs of cells are 16-byte aligned for
 * cp.async.bulk in FP64 and FP32 alike.
 */
#include "device_common.cuh"
#include "tbs_internal.hxx"
#include "tma.cuh"

#include <cuda_runtime.h>

#include <mutex>

namespace tbs {

constexpr int NV = 9;
constexpr int NB = 81;
constexpr unsigned FULL = 0xffffffffu;

/* ================================================================ helpers */

__global__ void zero_kernel(double *p, long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        p[t] = 0.0;
}

static int grid_for(long long n, int threads, int cap = 148 * 8) {
    long long b = (n + threads - 1) / threads;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

int launch_zero(cudaStream_t st, double *p, long long n) {
    zero_kernel<<<grid_for(n, 256), 256, 0, st>>>(p, n);
    return (int)cudaGetLastError();
}

/* block b sums v[b*chunk : (b+1)*chunk)^2 in a fixed order */
__global__ void norm_partials_kernel(const double *__restrict__ v, long long n, long long chunk,
                                     double *__restrict__ partials) {
    const long long lo = blockIdx.x * chunk;
    long long hi = lo + chunk;
    if (hi > n) hi = n;
    double s = 0.0;
    for (long long t = lo + threadIdx.x; t < hi; t += blockDim.x) s += v[t] * v[t];
    __shared__ double red[8];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(FULL, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        partials[blockIdx.x] = tot;
    }
}

int launch_norm_partials(cudaStream_t st, const double *v, long long n, double *partials,
                         int npart) {
    long long chunk = (n + npart - 1) / npart;
    if (chunk < 1) chunk = 1;
    norm_partials_kernel<<<npart, 256, 0, st>>>(v, n, chunk, partials);
    return (int)cudaGetLastError();
}

/* threads of the one-CTA norm sum (its order: thread t adds partials t,
 * t + REDUCE_THREADS, ..., then the warps' sums in order) */
constexpr int REDUCE_THREADS = 1024;

/* Sum the partials in a fixed order, record the norm and decide whether the
 * solve goes on.  The decision feeds the CUDA graph's while-node, so the
 * sweep loop never returns to the host.  n == 0 re-records the latest norm
 * (state->last) as the start of a new sweep sequence; is_start ==
 * NORM_CHECK records a converged solve's true residual. */
__global__ void reduce_norm_kernel(const double *__restrict__ partials, int n, SolveState *state,
                                   double *hist, int is_start,
                                   cudaGraphConditionalHandle handle, int use_cond,
                                   cudaGraphConditionalHandle handle2, int use2) {
    __shared__ double red[REDUCE_THREADS / 32];
    double acc = strided_sum(partials, n, REDUCE_THREADS);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(FULL, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < REDUCE_THREADS / 32; ++w) tot += red[w];
        const double nrm = n > 0 ? sqrt(tot) : state->last;
        if (is_start == NORM_CHECK) {
            /* the true residual of a solve whose recursive residual passed:
             * both conditions (the loop's, and the IF node that makes the
             * restart's input) say whether the solve goes on */
            const bool go = record_check(state, hist, nrm);
            if (use_cond) cudaGraphSetConditional(handle, go ? 1u : 0u);
            if (use2) cudaGraphSetConditional(handle2, go ? 1u : 0u);
            return;
        }
        if (is_start) {
            state->sweep = 0;
            state->norm0 = nrm;
            state->true_norm = -1.0;
            state->checks = 0;
            state->restarts = 0;
        } else {
            state->sweep += 1;
        }
        const int sw = state->sweep;
        if (sw < state->hist_cap) hist[sw] = nrm;
        state->last = nrm;
        const bool go = isfinite(nrm) && nrm > state->tol * state->norm0 && sw < state->max_sweeps;
        if (use_cond) cudaGraphSetConditional(handle, go ? 1u : 0u);
        if (use2) cudaGraphSetConditional(handle2, go ? 1u : 0u);
    }
}

int launch_reduce_norm(cudaStream_t st, const double *partials, int n, SolveState *state,
                       double *hist, int is_start, unsigned long long cond_handle, int use_cond,
                       unsigned long long cond_handle2, int use2) {
    reduce_norm_kernel<<<1, REDUCE_THREADS, 0, st>>>(partials, n, state, hist, is_start,
                                                     (cudaGraphConditionalHandle)cond_handle, use_cond,
                                                     (cudaGraphConditionalHandle)cond_handle2, use2);
    return (int)cudaGetLastError();
}

template <typename T>
__global__ void permute_to_pos_kernel(int nv, int nelem, const int *__restrict__ pos_of_elem,
                                      const double *__restrict__ src, T *__restrict__ dst) {
    long long n = (long long)nv * nelem;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int e = (int)(t / nv), i = (int)(t - (long long)e * nv);
        dst[(long long)pos_of_elem[e] * nv + i] = (T)src[t];
    }
}

__global__ void permute_to_elem_kernel(int nv, int nelem, const int *__restrict__ pos_of_elem,
                                       const double *__restrict__ src, double *__restrict__ dst) {
    long long n = (long long)nv * nelem;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int e = (int)(t / nv), i = (int)(t - (long long)e * nv);
        dst[t] = src[(long long)pos_of_elem[e] * nv + i];
    }
}

int launch_permute_to_pos(cudaStream_t st, int nv, int nelem, const int *pos_of_elem,
                          const double *src_elem, double *dst_pos) {
    permute_to_pos_kernel<double>
        <<<grid_for((long long)nv * nelem, 256), 256, 0, st>>>(nv, nelem, pos_of_elem, src_elem, dst_pos);
    return (int)cudaGetLastError();
}

int launch_permute_to_elem(cudaStream_t st, int nv, int nelem, const int *pos_of_elem,
                           const double *src_pos, double *dst_elem) {
    permute_to_elem_kernel<<<grid_for((long long)nv * nelem, 256), 256, 0, st>>>(
        nv, nelem, pos_of_elem, src_pos, dst_elem);
    return (int)cudaGetLastError();
}

__global__ void permute_f32_to_elem_kernel(int nv, int nelem, const int *__restrict__ pos_of_elem,
                                           const float *__restrict__ src,
                                           double *__restrict__ dst) {
    long long n = (long long)nv * nelem;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int e = (int)(t / nv), i = (int)(t - (long long)e * nv);
        dst[t] = (double)src[(long long)pos_of_elem[e] * nv + i];
    }
}

int launch_permute_f32_to_elem(cudaStream_t st, int nv, int nelem, const int *pos_of_elem,
                               const float *src_pos, double *dst_elem) {
    permute_f32_to_elem_kernel<<<grid_for((long long)nv * nelem, 256), 256, 0, st>>>(
        nv, nelem, pos_of_elem, src_pos, dst_elem);
    return (int)cudaGetLastError();
}

template <typename T>
__global__ void axpy_same_kernel(const T *__restrict__ d, T *__restrict__ U, long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        U[t] += d[t];
}

__global__ void cast_kernel(const double *__restrict__ s, float *__restrict__ d, long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        d[t] = (float)s[t];
}

int launch_cast_f64_f32(cudaStream_t st, const double *src, float *dst, long long n) {
    cast_kernel<<<grid_for(n, 256), 256, 0, st>>>(src, dst, n);
    return (int)cudaGetLastError();
}

__global__ void axpy_kernel(const float *__restrict__ d, double *__restrict__ U, long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        U[t] += (double)d[t];
}

int launch_axpy_f32_f64(cudaStream_t st, const float *d, double *U, long long n) {
    axpy_kernel<<<grid_for(n, 256), 256, 0, st>>>(d, U, n);
    return (int)cudaGetLastError();
}

__global__ void axpy2_kernel(const float *__restrict__ c, const float *__restrict__ d,
                             double *__restrict__ U, long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        U[t] += (double)c[t] + (double)d[t];
}

int launch_axpy_f64(cudaStream_t st, const double *d, double *U, long long n) {
    axpy_same_kernel<double><<<grid_for(n, 256), 256, 0, st>>>(d, U, n);
    return (int)cudaGetLastError();
}

int launch_axpy2_f32_f64(cudaStream_t st, const float *c, const float *d, double *U, long long n) {
    axpy2_kernel<<<grid_for(n, 256), 256, 0, st>>>(c, d, U, n);
    return (int)cudaGetLastError();
}

/* ====================================================== line factorization
 * Twisted block Thomas.  Each line is split into a top chain (cells
 * 0..m-1, eliminated downward as in src/okl/lineLU_v2.okl:58-182), a
 * bottom chain (cells n-1 down to m+1, the same elimination run upward) and
 * the twist cell m.  One warp per chain (grid = 2 x lines); lane j < 9 owns
 * column j of each 9x9 block.  For
 * chain step s >= 1 with A = block(row c_s, col c_{s-1}) and C =
 * block(row c_{s-1}, col c_s), both from the in-line face between them
 * (picked as in lineLU_v2.okl:116-117):
 *   Gam_{s-1} = Dinv_{s-1} C
 *   W         = D_s - A Gam_{s-1}          (block-Thomas pivot)
 *   Dinv_s    = W^-1   (in-place Gauss-Jordan, no pivoting, as the
 *                        reference's LU has none: lineLU_v2.okl:17-27)
 *   G_s       = Dinv_s A
 * and the chain's last Gam couples it to the twist cell.  The twist kernel
 * then forms Dinv_tw = (D_m - A_tw Gam_top - C_tw Gam_bot)^-1 and stores
 * Dinv_tw A_tw / Dinv_tw C_tw in the G / Gam slots of the twist position.
 * Dinv is stored column-major like the input blocks; G and Gam row-major
 * (entry (i,j) at 9i+j), the order the Thomas kernel reads them in.  The
 * FP32 arrays, when given, are the FP64 results rounded once. */
__device__ __forceinline__ void gj_invert(double *W, int t, unsigned *status) {
    const int i = t % NV, j = t / NV;
#pragma unroll 1
    for (int p = 0; p < NV; ++p) {
        double wpp = 0.0, wip = 0.0, wpj = 0.0, wij = 0.0;
        if (t < NB) {
            wpp = W[p * (NV + 1)];
            wip = W[i + NV * p];
            wpj = W[p + NV * j];
            wij = W[t];
        }
        __syncthreads();
        if (t < NB) {
            const double r = 1.0 / wpp;
            double v;
            if (i == p && j == p)
                v = r;
            else if (i == p)
                v = wpj * r;
            else if (j == p)
                v = -wip * r;
            else
                v = wij - wip * (wpj * r);
            W[t] = v;
        }
        if (t == 0 && !(fabs(wpp) > 0.0 && isfinite(wpp))) atomicOr(status, ST_PIVOT);
        __syncthreads();
    }
}

struct FactorOut {
    double *Dinv, *G, *Gam;
    float *Dinv32, *G32, *Gam32;
    __device__ void put_dinv(size_t p, int t, double w) const {
        if (Dinv) Dinv[p * NB + t] = w;
        if (Dinv32) Dinv32[p * NB + t] = (float)w;
    }
    /* row-major store of entry (i, j) */
    __device__ void put_g(size_t p, int i, int j, double v) const {
        if (G) G[p * NB + NV * i + j] = v;
        if (G32) G32[p * NB + NV * i + j] = (float)v;
    }
    __device__ void put_gam(size_t p, int i, int j, double v) const {
        if (Gam) Gam[p * NB + NV * i + j] = v;
        if (Gam32) Gam32[p * NB + NV * i + j] = (float)v;
    }
};

/* In-place Gauss-Jordan inverse of a 9x9 block distributed by columns:
 * lane j < 9 holds column j in w[0..8].  Pivot column p is broadcast with
 * shuffles; no pivoting, as the reference's LU has none. */
__device__ __forceinline__ void gj_invert_cols(double (&w)[NV], int j, unsigned *status) {
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        double colp[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) colp[i] = __shfl_sync(FULL, w[i], p);
        const double piv = colp[p];
        if (threadIdx.x == 0 && !(fabs(piv) > 0.0 && isfinite(piv))) atomicOr(status, ST_PIVOT);
        const double r = __drcp_rn(piv);
        const bool isp = (j == p);
        const double t = w[p] * r;
#pragma unroll
        for (int i = 0; i < NV; ++i)
            if (i != p) w[i] = isp ? -colp[i] * r : w[i] - colp[i] * t;
        w[p] = isp ? r : t;
    }
}

/* Gauss-Jordan inverse of a 9x9 block held by 27 lanes: lane j + 9g
 * (column j, row group g) holds rows 3g..3g+2 of column j in w[0..2].  For
 * pivot p, the pivot column's entries of this lane's rows come from lane
 * p + 9g, the pivot row's entry of this column and the pivot from the lanes
 * of row group p / 3 (their w[p % 3]).  Each entry is updated with the
 * operations of gj_invert_cols; no pivoting, as the reference's LU has none. */
__device__ __forceinline__ void gj_invert_27(double (&w)[3], int j, int g, unsigned *status) {
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        const int pg = p / 3, pr = p % 3;
        double colp[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) colp[k] = __shfl_sync(FULL, w[k], p + 9 * g);
        const double rowp = __shfl_sync(FULL, w[pr], j + 9 * pg);
        const double piv = __shfl_sync(FULL, w[pr], p + 9 * pg);
        if (threadIdx.x == 0 && !(fabs(piv) > 0.0 && isfinite(piv))) atomicOr(status, ST_PIVOT);
        const double r = __drcp_rn(piv);
        const bool isp = (j == p);
        const double t = rowp * r;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (3 * g + k != p)
                w[k] = isp ? -colp[k] * r : w[k] - colp[k] * t;
            else
                w[k] = isp ? r : t;
        }
    }
}

/* One warp per chain (grid = 2 x lines).  Lane j + 9g (27 lanes) owns rows
 * 3g..3g+2 of column j of every block, so 27 lanes share each product and
 * each pivot step; lanes 27..31 repeat lanes 18..22 and store nothing.  The
 * blocks every lane needs whole (Dinv_{s-1}, C, A, Gam_{s-1}, Dinv_s) are
 * published in shared memory.  Per entry the products add q = 0..8 in
 * order, as the column-per-lane form did. */
__global__ void __launch_bounds__(32) fast_factor_kernel(
    int nline, const int *__restrict__ line_start, const int *__restrict__ line_len,
    const int *__restrict__ line_twist, const int *__restrict__ fsrc,
    const double *__restrict__ jacD, const double *__restrict__ O1, const double *__restrict__ O2,
    FactorOut out, double *__restrict__ gamlast, unsigned *status) {
    const int l = blockIdx.x >> 1, chain = blockIdx.x & 1;
    if (l >= nline) return;
    const int lane = threadIdx.x;
    const bool act = lane < 27;
    const int jj = act ? lane % 9 : lane - 27; /* column */
    const int gg = act ? lane / 9 : 2;         /* row group: rows 3gg .. 3gg+2 */
    const int r0 = 3 * gg;
    __shared__ double sM[NB], sA[NB], sC[NB], sG[NB];
    const int ps = line_start[l], n = line_len[l], m = line_twist[l];
    const int len = chain ? n - 1 - m : m;
    const int cs = ps + (chain ? m : 0);
    const int ptw = ps + n - 1;
    if (len == 0) {
        for (int t = lane; t < NB; t += 32) gamlast[((size_t)l * 2 + chain) * NB + t] = 0.0;
        return;
    }
    double w[3], an[3], cn[3], dn[3];
    {
        const double *D0 = jacD + (size_t)fsrc[5 * cs] * NB + NV * jj + r0;
#pragma unroll
        for (int k = 0; k < 3; ++k) w[k] = D0[k];
    }
    auto fetch = [&](int p) {
        const int e = fsrc[5 * p], f = fsrc[5 * p + 1], side = fsrc[5 * p + 2];
        const double *Ap = (side ? O2 : O1) + (size_t)f * NB + NV * jj + r0;
        const double *Cp = (side ? O1 : O2) + (size_t)f * NB + NV * jj + r0;
        const double *Dp = jacD + (size_t)e * NB + NV * jj + r0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            an[k] = Ap[k];
            cn[k] = Cp[k];
            dn[k] = Dp[k];
        }
    };
    if (len > 1) fetch(cs + 1);
    gj_invert_27(w, jj, gg, status);
    if (act) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            out.put_dinv(cs, r0 + k + NV * jj, w[k]);
            out.put_g(cs, r0 + k, jj, 0.0);
            sM[r0 + k + NV * jj] = w[k];
        }
    }
    for (int s = 1; s < len; ++s) {
        const int p = cs + s;
        double a[3], c[3], d[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            a[k] = an[k];
            c[k] = cn[k];
            d[k] = dn[k];
        }
        if (s + 1 < len) fetch(p + 1);
        if (act) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                sC[r0 + k + NV * jj] = c[k];
                sA[r0 + k + NV * jj] = a[k];
            }
        }
        __syncwarp();
        /* Gam_{s-1}(:, j) = Dinv_{s-1} C(:, j) */
        double gm[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double acc = 0.0;
#pragma unroll
            for (int q = 0; q < NV; ++q) acc += sM[r0 + k + NV * q] * sC[q + NV * jj];
            gm[k] = acc;
        }
        if (act) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                out.put_gam(p - 1, r0 + k, jj, gm[k]);
                sG[r0 + k + NV * jj] = gm[k];
            }
        }
        __syncwarp();
        /* W(:, j) = D(:, j) - A Gam_{s-1}(:, j) */
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double acc = d[k];
#pragma unroll
            for (int q = 0; q < NV; ++q) acc -= sA[r0 + k + NV * q] * sG[q + NV * jj];
            w[k] = acc;
        }
        gj_invert_27(w, jj, gg, status);
        __syncwarp(); /* every lane has read Dinv_{s-1} */
        if (act) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                out.put_dinv(p, r0 + k + NV * jj, w[k]);
                sM[r0 + k + NV * jj] = w[k];
            }
        }
        __syncwarp();
        /* G_s(:, j) = Dinv_s A(:, j) */
        if (act) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double acc = 0.0;
#pragma unroll
                for (int q = 0; q < NV; ++q) acc += sM[r0 + k + NV * q] * sA[q + NV * jj];
                out.put_g(p, r0 + k, jj, acc);
            }
        }
        __syncwarp(); /* sA and sC are rewritten by the next cell */
    }
    /* coupling of the chain's last cell to the twist: Gam = Dinv_last block(row last, col m) */
    {
        const int f = fsrc[5 * ptw + (chain ? 3 : 1)], side = fsrc[5 * ptw + (chain ? 4 : 2)];
        const double *Cp = (side ? O1 : O2) + (size_t)f * NB + NV * jj + r0;
        if (act) {
#pragma unroll
            for (int k = 0; k < 3; ++k) sC[r0 + k + NV * jj] = Cp[k];
        }
        __syncwarp();
        if (act) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double acc = 0.0;
#pragma unroll
                for (int q = 0; q < NV; ++q) acc += sM[r0 + k + NV * q] * sC[q + NV * jj];
                out.put_gam(cs + len - 1, r0 + k, jj, acc);
                gamlast[((size_t)l * 2 + chain) * NB + r0 + k + NV * jj] = acc; /* column-major, FP64 */
            }
        }
    }
}

__global__ void __launch_bounds__(128) fast_twist_kernel(
    int nline, const int *__restrict__ line_start, const int *__restrict__ line_len,
    const int *__restrict__ line_twist, const int *__restrict__ fsrc,
    const double *__restrict__ jacD, const double *__restrict__ O1, const double *__restrict__ O2,
    FactorOut out, const double *__restrict__ gamlast, unsigned *status) {
    const int l = blockIdx.x;
    if (l >= nline) return;
    const int t = threadIdx.x;
    const bool act = t < NB;
    const int i = t % NV, j = t / NV;
    __shared__ double sW[NB], sA[NB], sC[NB], sGt[NB], sGb[NB];
    const int ps = line_start[l], n = line_len[l];
    const int ptw = ps + n - 1;
    if (act) {
        const int e = fsrc[5 * ptw];
        const int fa = fsrc[5 * ptw + 1], sa = fsrc[5 * ptw + 2];
        const int fb = fsrc[5 * ptw + 3], sb = fsrc[5 * ptw + 4];
        sW[t] = jacD[(size_t)e * NB + t];
        sA[t] = fa >= 0 ? (sa ? O2 : O1)[(size_t)fa * NB + t] : 0.0;
        sC[t] = fb >= 0 ? (sb ? O2 : O1)[(size_t)fb * NB + t] : 0.0;
        sGt[t] = gamlast[((size_t)l * 2 + 0) * NB + t];
        sGb[t] = gamlast[((size_t)l * 2 + 1) * NB + t];
    }
    __syncthreads();
    if (act) {
        double w = sW[t];
#pragma unroll
        for (int q = 0; q < NV; ++q) w -= sA[i + NV * q] * sGt[q + NV * j];
#pragma unroll
        for (int q = 0; q < NV; ++q) w -= sC[i + NV * q] * sGb[q + NV * j];
        sW[t] = w; /* only this thread reads or writes sW[t] in this phase */
    }
    __syncthreads();
    gj_invert(sW, t, status);
    if (act) {
        double ga = 0.0, gc = 0.0;
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            ga += sW[i + NV * q] * sA[q + NV * j];
            gc += sW[i + NV * q] * sC[q + NV * j];
        }
        out.put_dinv(ptw, t, sW[t]);
        out.put_g(ptw, i, j, ga);
        out.put_gam(ptw, i, j, gc);
    }
}

int launch_fast_factor(cudaStream_t st, const FastLayout &L, const double *jacD, const double *O1,
                       const double *O2, double *Dinv, double *G, double *Gam, float *Dinv32,
                       float *G32, float *Gam32, double *gamlast, unsigned *status) {
    if (L.nv != NV) return (int)cudaErrorInvalidValue;
    FactorOut out{Dinv, G, Gam, Dinv32, G32, Gam32};
    fast_factor_kernel<<<2 * L.nline, 32, 0, st>>>(L.nline, L.line_start, L.line_len, L.line_twist,
                                                   L.fsrc, jacD, O1, O2, out, gamlast, status);
    fast_twist_kernel<<<L.nline, 128, 0, st>>>(L.nline, L.line_start, L.line_len, L.line_twist,
                                               L.fsrc, jacD, O1, O2, out, gamlast, status);
    return (int)cudaGetLastError();
}

/* DX[q] = Dinv(p) X(q) for slot q = s*np16 + p, rounded once to FP32, from
 * the FP64 inverse and the original FP64 face block; one warp per slot */
__global__ void __launch_bounds__(256) fast_dx_kernel(long long nslots, int np16,
                                                      const int *__restrict__ xsrc,
                                                      const double *__restrict__ Dinv,
                                                      const double *__restrict__ O1,
                                                      const double *__restrict__ O2,
                                                      float *__restrict__ DX) {
    __shared__ double sm[8][2 * NB];
    const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    double *sD = sm[wb], *sX = sm[wb] + NB;
    for (long long q = w0; q < nslots; q += nw) {
        const int src = xsrc[q];
        const long long p = q % np16;
        __syncwarp();
        for (int t = lane; t < NB; t += 32) {
            sD[t] = Dinv[p * NB + t];
            sX[t] = src >= 0 ? ((src & 1) ? O2 : O1)[(size_t)(src >> 1) * NB + t] : 0.0;
        }
        __syncwarp();
        for (int t = lane; t < NB; t += 32) {
            const int i = t % NV, j = t / NV;
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < NV; ++k) acc += sD[i + NV * k] * sX[k + NV * j];
            DX[q * NB + t] = (float)acc;
        }
    }
}

int launch_fast_dx(cudaStream_t st, const FastLayout &L, const double *Dinv, const double *O1,
                   const double *O2, float *DX) {
    const long long nslots = (long long)L.np16 * L.nx;
    if (nslots == 0) return 0;
    fast_dx_kernel<<<grid_for(nslots * 32, 256), 256, 0, st>>>(nslots, L.np16, L.xsrc, Dinv, O1, O2, DX);
    return (int)cudaGetLastError();
}

/* X[q] = cross-line block of slot q = s*np16 + p (slot-major), or zeros;
 * one warp per slot */
__global__ void fast_xlayout_kernel(long long nslots, const int *__restrict__ xsrc,
                                    const double *__restrict__ O1, const double *__restrict__ O2,
                                    double *__restrict__ X, float *__restrict__ X32) {
    const int lane = threadIdx.x & 31;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long q = w0; q < nslots; q += nw) {
        const int src = xsrc[q];
        for (int tt = lane; tt < NB; tt += 32) {
            double v = 0.0;
            if (src >= 0) v = ((src & 1) ? O2 : O1)[(size_t)(src >> 1) * NB + tt];
            if (X) X[q * NB + tt] = v;
            if (X32) X32[q * NB + tt] = (float)v;
        }
    }
}

int launch_fast_xlayout(cudaStream_t st, const FastLayout &L, const double *O1, const double *O2,
                        double *X, float *X32) {
    const long long nslots = (long long)L.np16 * L.nx;
    if (nslots == 0) return 0;
    fast_xlayout_kernel<<<grid_for(nslots * 32, 256), 256, 0, st>>>(nslots, L.xsrc, O1, O2, X, X32);
    return (int)cudaGetLastError();
}

/* ================================================ residual -> Thomas RHS
 * Tiles of RES_TILE positions, each staged by one phase of the CTA's bulk
 * copy barrier; the single-system launches are persistent (as many CTAs
 * as fit, tiles round-robin per CTA).  Per tile:
 *   mode 0:  R = Rsrc (a residual already in position order)
 *   mode 1:  R = sum over slots X_slot dU[xnbr_slot]   (R_new = O dU)
 * then b = -Dinv R.  Thread t < 144 owns (cell c = t % 16, row i = t / 16):
 * with blocks 81 doubles apart, the 16 cells of a half-warp hit 16
 * distinct bank pairs, so the shared-memory reads are conflict-free.
 * X and xnbr are slot-major ([slot][position]) for the same reason.
 * Every tile writes its sum R^2; the last CTA to finish (atomic ticket)
 * adds the partials in tile order and, when asked, records the norm, the
 * sweep count and the graph's loop condition.
 */
constexpr int RES_THREADS_FAST = 160;

int fast_resid_grid(int np16) { return np16 / RES_TILE > 0 ? np16 / RES_TILE : 1; }

template <typename T>
__host__ __device__ inline size_t resid_smem_bytes(int nx) {
    const int nxa = nx > 0 ? nx : 1;
    return 128 + (size_t)RES_TILE * NB * sizeof(T) * (1 + nx) +
           (size_t)nxa * RES_TILE * NV * sizeof(T) + (size_t)RES_TILE * NV * sizeof(T) * 2;
}

/* The residual kernels' staging barrier sits at the start of the dynamic
 * shared memory; it is initialised once per CTA, and each tile the CTA
 * processes completes one phase of it. */
__device__ __forceinline__ uint64_t *resid_bar_init() {
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    return bar;
}

/* -(row of Dinv) . R for one (cell, row): dr points at entry (row, 0) of
 * the cell's column-major block, rv at the cell's R; three accumulators,
 * the order every b = -Dinv R of this file uses */
template <typename T>
__device__ __forceinline__ T neg_dinv_row(const T *dr, const T *rv) {
    T a0 = dr[0] * rv[0], a1 = dr[9] * rv[1], a2 = dr[18] * rv[2];
    a0 += dr[27] * rv[3];
    a1 += dr[36] * rv[4];
    a2 += dr[45] * rv[5];
    a0 += dr[54] * rv[6];
    a1 += dr[63] * rv[7];
    a2 += dr[72] * rv[8];
    return -(a0 + (a1 + a2));
}

/* One tile (positions blk*RES_TILE ..) with the staging barrier's phase of
 * the given parity.  Returns false (status set, copies landed) when the
 * wait for the tile's bulk copies ran out of time. */
template <typename T>
__device__ __forceinline__ bool fast_resid_body(
    int nx, int np16, int mode, const T *__restrict__ Dinv, const T *__restrict__ X,
    const int *__restrict__ xnbr, const T *__restrict__ dU, const T *__restrict__ Rsrc,
    T *__restrict__ b, T *__restrict__ Uacc, const NormSink &ns, unsigned *status, int blk,
    uint64_t *bar, uint32_t parity, const int *nbr_pre = nullptr, const T *__restrict__ Uin = nullptr) {
    extern __shared__ __align__(128) unsigned char smem[];
    T *sD = reinterpret_cast<T *>(smem + 128);
    T *sX = sD + RES_TILE * NB;
    const int nxa = nx > 0 ? nx : 1;
    T *sg = sX + nx * RES_TILE * NB;
    T *sr = sg + nxa * RES_TILE * NV;
    T *sb = sr + RES_TILE * NV;
    const int p0 = blk * RES_TILE;
    const int tid = threadIdx.x;
    const int c = tid % RES_TILE, i = tid / RES_TILE;
    const bool act = tid < RES_TILE * NV;
    const uint32_t szD = RES_TILE * NB * sizeof(T), szR = RES_TILE * NV * sizeof(T);

    if (tid == 0) {
        const uint64_t pol = policy_evict_first();
        const bool noD = mode == 3 || mode == 4;
        const uint32_t bytes = (noD ? 0u : szD) + (mode >= 1 ? nx * szD : szR);
        mbar_arrive_expect_tx(bar, bytes);
        if (!noD) bulk_g2s_hint(sD, Dinv + (size_t)p0 * NB, szD, bar, pol);
        if (mode >= 1) {
            for (int s = 0; s < nx; ++s)
                bulk_g2s_hint(sX + s * RES_TILE * NB, X + ((size_t)s * np16 + p0) * NB, szD, bar, pol);
        } else {
            bulk_g2s(sr, Rsrc + (size_t)p0 * NV, szR, bar);
        }
    }
    if (act && Uacc) {
        /* modes 1, 3: U += dU of this tile (the Thomas kernel leaves U to
         * this kernel), the previous U read from Uin when set; mode 0:
         * U = 0, the start of a sweep sequence */
        const size_t q = (size_t)p0 * NV + tid;
        Uacc[q] = (mode >= 1) ? (Uin ? Uin[q] : Uacc[q]) + dU[q] : T(0);
    }
    if (mode >= 1 && act) {
        /* neighbour dU gathers overlap the bulk copies (their indices
         * loaded during the previous tile when the caller prefetched them) */
        if (nbr_pre) {
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                if (s < nx) {
                    const int nb = nbr_pre[s];
                    sg[(s * RES_TILE + c) * NV + i] = (nb >= 0) ? dU[(size_t)nb * NV + i] : T(0);
                }
            }
        } else {
            for (int s = 0; s < nx; ++s) {
                const int nb = xnbr[(size_t)s * np16 + p0 + c];
                sg[(s * RES_TILE + c) * NV + i] = (nb >= 0) ? dU[(size_t)nb * NV + i] : T(0);
            }
        }
    }
    const bool ok = mbar_wait(bar, parity);
    if (__syncthreads_or(!ok)) {
        if (tid == 0) {
            atomicOr(status, ST_TIMEOUT);
            mbar_wait(bar, parity, 1LL << 28); /* let the copies land before the CTA retires */
        }
        return false;
    }
    T r = T(0);
    if (mode >= 1) {
        if (act) {
            T a0 = T(0), a1 = T(0), a2 = T(0);
            for (int s = 0; s < nx; ++s) {
                const T *xr = sX + (s * RES_TILE + c) * NB + i;
                const T *g = sg + (s * RES_TILE + c) * NV;
                a0 += xr[0] * g[0];
                a1 += xr[9] * g[1];
                a2 += xr[18] * g[2];
                a0 += xr[27] * g[3];
                a1 += xr[36] * g[4];
                a2 += xr[45] * g[5];
                a0 += xr[54] * g[6];
                a1 += xr[63] * g[7];
                a2 += xr[72] * g[8];
            }
            r = a0 + (a1 + a2);
            sr[c * NV + i] = r;
        }
        __syncthreads();
    } else if (act) {
        r = sr[c * NV + i];
    }
    double sq = act ? (double)r * (double)r : 0.0;
    if (mode == 3) {
        /* X held Dinv X: r is already Dinv R */
        if (act) sb[c * NV + i] = -r;
    } else if (mode == 4) {
        /* R = v + J z after the line solves, so J z = R - v */
        if (act) sb[c * NV + i] = r - Rsrc[(size_t)p0 * NV + c * NV + i];
    } else if (act) {
        sb[c * NV + i] = neg_dinv_row<T>(sD + c * NB + i, sr + c * NV);
    }
    __syncthreads();
    if (act) b[(size_t)p0 * NV + tid] = sb[tid]; /* contiguous tile store */
    if (ns.partials) {
        __shared__ double red[RES_THREADS_FAST / 32];
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(FULL, sq, o);
        if ((tid & 31) == 0) red[tid >> 5] = sq;
        __syncthreads();
        if (tid == 0) {
            double tot = 0.0;
            for (int w = 0; w < RES_THREADS_FAST / 32; ++w) tot += red[w];
            ns.partials[blk] = tot; /* the tile's sum R^2; totals by finalize_total */
        }
    }
    return true;
}

/* The single-system residual launches are persistent: CTA k takes tiles
 * k, k + grid, ...; each tile completes one phase of the CTA's barrier and
 * writes its partial; finalize_total then sums the tiles' partials in tile
 * order (the order of the batched norm kernel with 160 threads). */
template <typename T>
__device__ __forceinline__ bool resid_tiles(int nx, int np16, int mode, const T *Dinv, const T *X,
                                            const int *xnbr, const T *dU, const T *Rsrc, T *b,
                                            T *Uacc, const NormSink &ns, unsigned *status,
                                            int u_tile0 = 0, const T *Uin = nullptr) {
    timer_launch_start(ns.timer);
    uint64_t *bar = resid_bar_init();
    const int ntiles = np16 / RES_TILE;
    uint32_t parity = 0;
    /* the neighbour indices of a CTA's next tile are loaded while it works
     * on the current one, so that a tile's gathers wait for one memory
     * round trip, not two */
    constexpr int PRE = 4;
    const bool pre = mode >= 1 && nx <= PRE && threadIdx.x < RES_TILE * NV;
    const int c = threadIdx.x % RES_TILE;
    int nbr[PRE], nxt[PRE];
#pragma unroll
    for (int s = 0; s < PRE; ++s) nbr[s] = (pre && s < nx && blockIdx.x < ntiles)
                                               ? xnbr[(size_t)s * np16 + blockIdx.x * RES_TILE + c] : -1;
    for (int w = blockIdx.x; w < ntiles; w += gridDim.x) {
        const int wn = w + gridDim.x;
#pragma unroll
        for (int s = 0; s < PRE; ++s)
            nxt[s] = (pre && s < nx && wn < ntiles) ? xnbr[(size_t)s * np16 + wn * RES_TILE + c] : -1;
        const bool ok = fast_resid_body<T>(nx, np16, mode, Dinv, X, xnbr, dU, Rsrc, b,
                                           w >= u_tile0 ? Uacc : nullptr, ns, status, w, bar, parity,
                                           pre ? nbr : nullptr, Uin);
        parity ^= 1u;
        if (!ok) break;
#pragma unroll
        for (int s = 0; s < PRE; ++s) nbr[s] = nxt[s];
        __syncthreads(); /* the next tile's copies overwrite the stages */
    }
    /* a line partition's norm covers its owned lines, which come first */
    return finalize_total(ns, (ns.ntiles > 0 && ns.ntiles < ntiles) ? ns.ntiles : ntiles);
}

/* mode 1 (R = sum X dU over the cross-line slots); U += dU (Uacc = Uin +
 * dU when Uin is set) for the tiles from u_tile0 on: a line partition's
 * halo tiles, whose line solves leave U alone */
template <typename T>
__global__ void __launch_bounds__(RES_THREADS_FAST) fast_resid_kernel(
    int nx, int np16, const T *__restrict__ Dinv, const T *__restrict__ X,
    const int *__restrict__ xnbr, const T *__restrict__ dU, T *__restrict__ b,
    T *__restrict__ Uacc, NormSink ns, unsigned *status, int u_tile0, const T *__restrict__ Uin) {
    resid_tiles<T>(nx, np16, 1, Dinv, X, xnbr, dU, nullptr, b, Uacc, ns, status, u_tile0, Uin);
}

/* mode 3 (b = -sum (Dinv X) dU: premultiplied cross-line blocks, no norm) */
template <typename T>
__global__ void __launch_bounds__(RES_THREADS_FAST) fast_resid_dx_kernel(
    int nx, int np16, const T *__restrict__ DX, const int *__restrict__ xnbr,
    const T *__restrict__ dU, T *__restrict__ b, T *__restrict__ Uacc, unsigned *status) {
    resid_tiles<T>(nx, np16, 3, nullptr, DX, xnbr, dU, nullptr, b, Uacc, NormSink{}, status);
}

/* mode 4 (the product with J of a preconditioned direction: R = sum X dU
 * is the residual of v + J z after the line solves, so w = R - v; no
 * Dinv, no norm) */
template <typename T>
__global__ void __launch_bounds__(RES_THREADS_FAST) fast_resid_jv_kernel(
    int nx, int np16, const T *__restrict__ X, const int *__restrict__ xnbr,
    const T *__restrict__ dU, const T *__restrict__ v, T *__restrict__ w, T *__restrict__ Uacc,
    unsigned *status) {
    resid_tiles<T>(nx, np16, 4, nullptr, X, xnbr, dU, v, w, Uacc, NormSink{}, status);
}

/* mode 0 (R given in position order) */
template <typename T>
__global__ void __launch_bounds__(RES_THREADS_FAST) fast_resid_rhs_kernel(
    int np16, const T *__restrict__ Dinv, const T *__restrict__ Rsrc, T *__restrict__ b,
    T *__restrict__ Uzero, NormSink ns, unsigned *status) {
    resid_tiles<T>(0, np16, 0, Dinv, nullptr, nullptr, nullptr, Rsrc, b, Uzero, ns, status);
}

/* CTAs of a persistent single-system residual launch: as many as fit */
static int resid_grid_persistent(const void *fn, size_t smem, int ntiles) {
    int dev = 0, nsm = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, RES_THREADS_FAST, smem) != cudaSuccess ||
        per < 1)
        per = 1;
    const int g = per * nsm;
    return ntiles < g ? (ntiles > 0 ? ntiles : 1) : g;
}

template <typename T>
int launch_fast_resid(cudaStream_t st, const FastLayout &L, int mode, const T *Dinv, const T *X,
                      const T *dU, const T *Rsrc, T *b, const NormSink &ns, unsigned *status,
                      T *Uacc, int u_tile0, const T *Uin) {
    if (L.nv != NV) return (int)cudaErrorInvalidValue;
    const int grid = fast_resid_grid(L.np16);
    if (mode == 4) {
        /* nx == 0 runs the kernel too: no slot is read, w = -v */
        if (!Rsrc) return (int)cudaErrorInvalidValue;
        const size_t smem4 = resid_smem_bytes<T>(L.nx);
        fast_resid_jv_kernel<T><<<resid_grid_persistent((const void *)fast_resid_jv_kernel<T>, smem4, grid),
                                  RES_THREADS_FAST, smem4, st>>>(L.nx, L.np16, X, L.xnbr, dU, Rsrc, b,
                                                                 Uacc, status);
        return (int)cudaGetLastError();
    }
    if (mode >= 1 && L.nx == 0) {
        /* a mesh that is one line: the line solve is exact, R_new = 0 */
        if (Uacc) {
            const long long n = (long long)L.np16 * NV;
            axpy_same_kernel<T><<<grid_for(n, 256), 256, 0, st>>>(dU, Uacc, n);
        }
        cudaMemsetAsync(b, 0, (size_t)L.np16 * NV * sizeof(T), st);
        if (mode == 3) return (int)cudaGetLastError(); /* no norm wanted */
        /* run the kernel on a zero residual (read from b itself) so that the
         * norm bookkeeping happens */
        mode = 0;
        Rsrc = b;
        Uacc = nullptr;
    }
    if (mode == 0 && !Rsrc) return (int)cudaErrorInvalidValue;
    const size_t smem = resid_smem_bytes<T>(mode >= 1 ? L.nx : 0);
    if (mode == 3)
        fast_resid_dx_kernel<T><<<resid_grid_persistent((const void *)fast_resid_dx_kernel<T>, smem, grid),
                                  RES_THREADS_FAST, smem, st>>>(L.nx, L.np16, X, L.xnbr, dU, b, Uacc,
                                                                status);
    else if (mode == 1)
        fast_resid_kernel<T><<<resid_grid_persistent((const void *)fast_resid_kernel<T>, smem, grid),
                               RES_THREADS_FAST, smem, st>>>(L.nx, L.np16, Dinv, X, L.xnbr, dU, b, Uacc,
                                                             ns, status, u_tile0, Uin);
    else
        fast_resid_rhs_kernel<T><<<resid_grid_persistent((const void *)fast_resid_rhs_kernel<T>, smem, grid),
                                   RES_THREADS_FAST, smem, st>>>(L.np16, Dinv, Rsrc, b, Uacc, ns, status);
    return (int)cudaGetLastError();
}

template int launch_fast_resid<double>(cudaStream_t, const FastLayout &, int, const double *,
                                       const double *, const double *, const double *, double *,
                                       const NormSink &, unsigned *, double *, int, const double *);
template int launch_fast_resid<float>(cudaStream_t, const FastLayout &, int, const float *,
                                      const float *, const float *, const float *, float *,
                                      const NormSink &, unsigned *, float *, int, const float *);

/* =========================================================== line Thomas
 * One warp per line, twisted: lanes 0..8 run the top chain and lanes
 * 16..24 the bottom chain of the line with the same instruction stream, so
 * a line of n cells takes n+1 dependent steps instead of 2n.  Lane 0
 * streams "jobs" through an NS-stage bulk-copy ring, each stage holding one
 * chunk of P cells per chain: jobs 0..nf-1 forward chunks (G rows and b),
 * jobs nf..2nf-1 backward chunks in reverse (Gam rows).  G and Gam are
 * row-major; lane i owns row i and holds the row of the NEXT cell in
 * registers while the current cell's dot product runs.  The previous
 * cell's 9-vector is published through shared memory in two copies (at
 * offsets 0 and 11), so that every lane reads it with the 16-byte
 * alignment of its row.  Chain forward:  y_s = b_s - G_s y_{s-1};  twist:
 * x_m = b_m - G_tw y_top - Gam_tw y_bot;  chain backward:  x_s = y_s -
 * Gam_s x_{s+1} (s+1 toward the twist).
 * YS: the line's y and x live in shared memory, and dU / U are written with
 * coalesced 16-byte accesses after the line is solved; otherwise y goes to
 * global memory (read back one chunk ahead) and dU / U per step, U read
 * one chunk ahead with y (one-warp form) or staged behind the backward
 * chunk's Gam rows by the copy warp (warp-specialised form).
 *   accumulate = 0:  U = dU
 *   accumulate = 1:  U += dU (the FP64 sweeps of a context; U read from a
 *                    second buffer Uin when one is given: line partitions)
 *   accumulate = 2:  U untouched (the residual kernel that follows adds
 *                    dU to U for its tile, with coalesced tile accesses:
 *                    the batch engine)
 */
constexpr int THOMAS_P = 8;

template <typename T>
__host__ __device__ inline uint32_t thomas_half_bytes() {
    return (uint32_t)(THOMAS_P * (NB + NV) * sizeof(T));
}
template <typename T>
__host__ __device__ inline uint32_t thomas_stage_bytes() {
    return 2 * thomas_half_bytes<T>();
}

/* Lane constants for rows whose start parity is (q + i) & 1: pairs start at
 * row+par, the single element is row[8] (par 0) or row[0] (par 1); the
 * broadcast vector is read from copy A (offset 0) or copy B (offset 10,
 * holding y_j at 11+j) so that the pairs line up.  The same scheme serves
 * FP64 (16-byte pairs) and FP32 (8-byte pairs). */
struct LaneOff {
    int row;
    int rp[2], rs[2], vp[2], vs[2];
};

__device__ __forceinline__ LaneOff lane_offsets(int i) {
    LaneOff o;
    o.row = NV * i;
    for (int odd = 0; odd < 2; ++odd) {
        const int par = (i + odd) & 1;
        o.rp[odd] = NV * i + par;
        o.rs[odd] = NV * i + (par ? 0 : 8);
        o.vp[odd] = par ? 12 : 0;
        o.vs[odd] = par ? 0 : 8;
    }
    return o;
}

struct RowD {
    double2 r0, r1, r2, r3;
    double s;
};
struct RowF {
    float2 r0, r1, r2, r3;
    float s;
};
template <typename T> struct RowOf;
template <> struct RowOf<double> { using type = RowD; };
template <> struct RowOf<float> { using type = RowF; };

__device__ __forceinline__ void load_row(RowD &R, const double *rowbase, const LaneOff &o, int odd) {
    const double2 *r = reinterpret_cast<const double2 *>(rowbase + o.rp[odd]);
    R.r0 = r[0];
    R.r1 = r[1];
    R.r2 = r[2];
    R.r3 = r[3];
    R.s = rowbase[o.rs[odd]];
}

__device__ __forceinline__ void load_row(RowF &R, const float *rowbase, const LaneOff &o, int odd) {
    const float2 *r = reinterpret_cast<const float2 *>(rowbase + o.rp[odd]);
    R.r0 = r[0];
    R.r1 = r[1];
    R.r2 = r[2];
    R.r3 = r[3];
    R.s = rowbase[o.rs[odd]];
}

/* init - row . vec, vec from the broadcast buffer `cur` */
__device__ __forceinline__ double row_dot(const RowD &R, const double *cur, const LaneOff &o,
                                          int odd, double init) {
    const double2 *v = reinterpret_cast<const double2 *>(cur + o.vp[odd]);
    const double2 v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3];
    const double w = cur[o.vs[odd]];
    double a0 = init - R.s * w;
    double a1 = R.r0.x * v0.x;
    double a2 = R.r0.y * v0.y;
    a0 -= R.r1.x * v1.x;
    a1 += R.r1.y * v1.y;
    a2 += R.r2.x * v2.x;
    a0 -= R.r2.y * v2.y;
    a1 += R.r3.x * v3.x;
    a2 += R.r3.y * v3.y;
    return a0 - (a1 + a2);
}

__device__ __forceinline__ float row_dot(const RowF &R, const float *cur, const LaneOff &o,
                                         int odd, float init) {
    const float2 *v = reinterpret_cast<const float2 *>(cur + o.vp[odd]);
    const float2 v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3];
    const float w = cur[o.vs[odd]];
    float a0 = init - R.s * w;
    float a1 = R.r0.x * v0.x;
    float a2 = R.r0.y * v0.y;
    a0 -= R.r1.x * v1.x;
    a1 += R.r1.y * v1.y;
    a2 += R.r2.x * v2.x;
    a0 -= R.r2.y * v2.y;
    a1 += R.r3.x * v3.x;
    a2 += R.r3.y * v3.y;
    return a0 - (a1 + a2);
}

/* Forward steps kbase..kbase+P-1 of this half's chain (length len, first
 * position cpos relative to the line start).  CHECK: some steps of the
 * warp may lie beyond one chain's end; those compute but write nothing. */
template <typename T, int P, bool CHECK, bool YS>
__device__ __forceinline__ void fwd_chunk(const T *sG, const T *sB, T *bc, T *ys, T *yg, int kbase,
                                          int len, int cpos, int i, const LaneOff &o,
                                          uint64_t ypol) {
    typename RowOf<T>::type cur_row, next_row;
    load_row(cur_row, sG, o, 0);
    T cur_b = sB[i];
#pragma unroll
    for (int q = 0; q < P; ++q) {
        const int odd = q & 1;
        T next_b = T(0);
        if (q + 1 < P) {
            load_row(next_row, sG + (q + 1) * NB, o, odd ^ 1);
            next_b = sB[(q + 1) * NV + i];
        }
        const T *cur = bc + odd * 20;
        T *nxt = bc + (odd ^ 1) * 20;
        const T yi = row_dot(cur_row, cur, o, odd, cur_b);
        /* lanes 9..15 of a half compute row 8 from the same inputs as lane
         * 8 and store the same value to the same address: no divergence */
        if (!CHECK || kbase + q < len) {
            nxt[i] = yi;
            nxt[11 + i] = yi;
            const int pos = cpos + kbase + q;
            if (YS)
                ys[pos * NV + i] = yi;
            else /* kept in L2 for the backward chain (the blocks stream evict-first) */
                st_hint(yg + (size_t)pos * NV + i, yi, ypol);
        }
        __syncwarp();
        cur_row = next_row;
        cur_b = next_b;
    }
}

/* uv: U of the chunk's cells read ahead in registers, or sU (when set):
 * the chunk's U staged behind its Gam rows */
template <typename T, int P, bool CHECK, bool YS>
__device__ __forceinline__ void bwd_chunk(const T *sG, T *bc, T *ys, const T *yv, const T *uv,
                                          T *dUl, T *Ul, int kbase, int len, int cpos, int i,
                                          const LaneOff &o, const T *sU = nullptr) {
    typename RowOf<T>::type cur_row, next_row;
    load_row(cur_row, sG + (P - 1) * NB, o, (P - 1) & 1);
#pragma unroll
    for (int q = P - 1; q >= 0; --q) {
        const int odd = q & 1;
        if (q > 0) load_row(next_row, sG + (q - 1) * NB, o, odd ^ 1);
        const int f = (P - 1 - q) & 1; /* buffer alternates per step */
        const T *cur = bc + f * 20;
        T *nxt = bc + (f ^ 1) * 20;
        const bool valid = !CHECK || (kbase + q >= 0 && kbase + q < len);
        const int pos = cpos + kbase + q;
        T yk = T(0);
        if (valid) yk = YS ? ys[pos * NV + i] : yv[q];
        const T d = row_dot(cur_row, cur, o, odd, yk);
        if (valid) { /* lanes 9..15 repeat lane 8's row, value and address */
            nxt[i] = d;
            nxt[11 + i] = d;
            if (YS) {
                ys[pos * NV + i] = d;
            } else {
                dUl[(size_t)pos * NV + i] = d;
                if (Ul) Ul[(size_t)pos * NV + i] = (sU ? sU[q * NV + i] : uv[q]) + d;
            }
        }
        __syncwarp();
        cur_row = next_row;
    }
}

/* Solve one line (start ps, n cells, twist m) with the warp of the calling
 * CTA.  The staging barriers live at the start of `smem` and stay
 * initialised across the lines that a persistent CTA solves: bit s of
 * `pbase` is the parity with which barrier s completes its next phase.
 * Returns false when a staging wait ran out of time; the status bit is
 * then set and the copies in flight have landed. */
/* bytes before the first staging buffer: the barriers (and, in the
 * warp-specialised form, the producer's counters) */
template <bool WS>
__host__ __device__ constexpr int thomas_hdr() { return WS ? 256 : 128; }

/* accumulate = 1 reads U from Uin when it is set (a second buffer: the
 * previous U stays intact), else from U itself */
template <typename T, int P, bool YS, bool WS = false>
__device__ __forceinline__ bool thomas_line(
    int NS, int accumulate, int ps, int n, int m, const T *__restrict__ G,
    const T *__restrict__ Gam, const T *__restrict__ b, T *__restrict__ y, T *__restrict__ dU,
    T *__restrict__ U, unsigned *status, unsigned char *smem, uint32_t &pbase, uint64_t pol,
    const T *__restrict__ Uin = nullptr) {
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    /* WS (warp-specialised CTA of two warps): bars[0..NS) complete when a
     * stage's copies have landed, bars[8..8+NS) when warp 0 has consumed
     * it; warp 1 lane 0 issues the copies, warp 0 runs the chains */
    uint64_t *empty = bars + 8;
    volatile int *ws_issued = reinterpret_cast<volatile int *>(smem + 128);
    volatile int *ws_abort = ws_issued + 1;
    const uint32_t stage = 2 * P * (NB + NV) * sizeof(T);
    const uint32_t half = P * (NB + NV) * sizeof(T);
    unsigned char *st0 = smem + thomas_hdr<WS>();
    /* broadcast: 2 halves x 2 alternating buffers x [copy A: 10][copy B: 10] */
    T *bcall = reinterpret_cast<T *>(st0 + (size_t)NS * stage);
    T *ys = bcall + 80;
    const int lane = threadIdx.x & 31;
    const int h = lane >> 4, li = lane & 15;
    const int i = li < NV ? li : NV - 1;
    const LaneOff off = lane_offsets(i);
    const int nb = n - 1 - m;
    const int len = h ? nb : m;      /* this half's chain length */
    const int cpos = h ? m : 0;      /* its first position, relative to ps */
    const int nchT = (m + P - 1) / P, nchB = (nb + P - 1) / P;
    const int nch = h ? nchB : nchT;
    const int nf = nchT > nchB ? nchT : nchB;
    const int njobs = 2 * nf;
    T *bc = bcall + h * 40;
    T *yl = y + (size_t)ps * NV;
    T *dUl = dU + (size_t)ps * NV;
    T *Ul = U ? U + (size_t)ps * NV : nullptr;
    const T *Uil = Uin ? Uin + (size_t)ps * NV : Ul;
    auto parity = [&](int job) { return ((pbase >> (job % NS)) ^ (uint32_t)(job / NS)) & 1u; };

    const bool producer = WS && (threadIdx.x >> 5) == 1;
    /* warp-specialised form: the copy warp also stages U behind the
     * backward chunks' Gam rows (where the forward stages hold b), so the
     * chain warp reads it from shared memory */
    const bool stage_u = WS && !YS && accumulate == 1 && Ul != nullptr;
    __syncwarp(); /* the previous line's readers of the stages are done */
    if (!producer)
        for (int t = lane; t < 80; t += 32) bcall[t] = T(0);
    __syncwarp();

    /* copy size of chunk c of a chain of length ln, rounded up to 4 cells
     * (16-byte multiple); the extra cells stay inside the line's range */
    auto cells = [&](int ln, int c) { return ((min(P, ln - c * P) + 3) & ~3); };
    auto issue = [&](int job, int s) {
        unsigned char *base = st0 + (size_t)s * stage;
        uint32_t bytes = 0;
        if (job < nf) {
            const int c = job;
            if (c < nchT) bytes += cells(m, c) * (NB + NV) * sizeof(T);
            if (c < nchB) bytes += cells(nb, c) * (NB + NV) * sizeof(T);
        } else {
            const int jb = job - nf, bw = NB + (stage_u ? NV : 0);
            if (nchT - 1 - jb >= 0) bytes += cells(m, nchT - 1 - jb) * bw * sizeof(T);
            if (nchB - 1 - jb >= 0) bytes += cells(nb, nchB - 1 - jb) * bw * sizeof(T);
        }
        mbar_arrive_expect_tx(&bars[s], bytes);
        for (int hh = 0; hh < 2; ++hh) {
            const int ln = hh ? nb : m, nc = hh ? nchB : nchT, cp = hh ? m : 0;
            unsigned char *hb = base + hh * half;
            if (job < nf) {
                const int c = job;
                if (c >= nc) continue;
                const int cnt = cells(ln, c);
                bulk_g2s_hint(hb, G + (size_t)(ps + cp + c * P) * NB, cnt * NB * sizeof(T), &bars[s], pol);
                bulk_g2s(hb + P * NB * sizeof(T), b + (size_t)(ps + cp + c * P) * NV, cnt * NV * sizeof(T),
                         &bars[s]);
            } else {
                const int c = nc - 1 - (job - nf);
                if (c < 0) continue;
                const int cnt = cells(ln, c);
                bulk_g2s_hint(hb, Gam + (size_t)(ps + cp + c * P) * NB, cnt * NB * sizeof(T), &bars[s], pol);
                if (stage_u)
                    bulk_g2s(hb + P * NB * sizeof(T), Uil + (size_t)(cp + c * P) * NV, cnt * NV * sizeof(T),
                             &bars[s]);
            }
        }
    };
    if (producer) {
        /* every job as soon as the consumer has released its stage.  Each
         * empty barrier completes one phase per job consumed from its stage,
         * as each full barrier does per job landed, so the parity bits of
         * `pbase` serve both (a persistent CTA carries them across lines);
         * job j >= NS waits for the consumption of job j - NS */
        if (lane == 0) {
            for (int job = 0; job < njobs; ++job) {
                if (*ws_abort) break;
                const int s = job % NS;
                if (job >= NS && !mbar_wait(&empty[s], parity(job - NS))) {
                    atomicOr(status, ST_TIMEOUT);
                    break;
                }
                issue(job, s);
                *ws_issued = job + 1;
            }
        }
        __syncwarp();
        __syncthreads(); /* meets the consumer's */
        for (int s = 0; s < NS && s < njobs; ++s) {
            const int cnt = (njobs - 1 - s) / NS + 1;
            pbase ^= (uint32_t)(cnt & 1) << s;
        }
        return true;
    }
    int issued = 0;
    if (!WS && lane == 0) {
        for (; issued < NS && issued < njobs; ++issued) issue(issued, issued);
    }
    int consumed = 0;
    bool timed_out = false;
    const int both_full = (m < nb ? m : nb) / P; /* jobs where both chains run P steps */
    /* y, written by the forward chains and read once by the backward ones */
    const uint64_t ypol_last = YS ? 0ull : policy_evict_last();
    const uint64_t ypol_first = YS ? 0ull : policy_evict_first();

    /* ---------------- forward */
    for (int c = 0; c < nf; ++c) {
        const int s = c % NS;
        const bool ok = mbar_wait(&bars[s], parity(c));
        if (__any_sync(FULL, !ok)) {
            timed_out = true;
            break;
        }
        ++consumed;
        const T *sG = reinterpret_cast<const T *>(st0 + (size_t)s * stage + h * half);
        const T *sB = sG + P * NB;
        if (c < both_full)
            fwd_chunk<T, P, false, YS>(sG, sB, bc, ys, yl, c * P, len, cpos, i, off, ypol_last);
        else
            fwd_chunk<T, P, true, YS>(sG, sB, bc, ys, yl, c * P, len, cpos, i, off, ypol_last);
        __syncwarp();
        if (WS) {
            if (lane == 0) mbar_arrive(&empty[s]);
        } else if (lane == 0 && issued < njobs) {
            issue(issued, s);
            ++issued;
        }
    }

    if (!timed_out) {
        /* ---------------- twist: x_m = b_m - G_tw y_top - Gam_tw y_bot */
        const int ptw = n - 1; /* relative to ps */
        const T *ytop = bcall + 0 * 40 + (m & 1) * 20;
        const T *ybot = bcall + 1 * 40 + (nb & 1) * 20;
        T xm = T(0);
        if (lane < NV) {
            const T *gr = G + (size_t)(ps + ptw) * NB + NV * lane;
            const T *cr = Gam + (size_t)(ps + ptw) * NB + NV * lane;
            T acc = b[(size_t)(ps + ptw) * NV + lane];
#pragma unroll
            for (int j = 0; j < NV; ++j) acc -= gr[j] * ytop[j] + cr[j] * ybot[j];
            xm = acc;
        }
        __syncwarp();
        if (lane < NV) {
            for (int t = 0; t < 4; ++t) {
                bcall[t * 20 + lane] = xm;
                bcall[t * 20 + 11 + lane] = xm;
            }
            if (YS)
                ys[ptw * NV + lane] = xm;
            else {
                dUl[(size_t)ptw * NV + lane] = xm;
                if (accumulate < 2)
                    Ul[(size_t)ptw * NV + lane] = (accumulate ? Uil[(size_t)ptw * NV + lane] : T(0)) + xm;
            }
        }
        __syncwarp();

        /* ---------------- backward */
        T yv[P], uv[P], nyv[P], nuv[P];
        auto load_chunk = [&](int c, T *yy, T *uu) {
#pragma unroll
            for (int q = 0; q < P; ++q) {
                const int k = c * P + q;
                yy[q] = T(0);
                uu[q] = T(0);
                if (!YS && c >= 0 && k < len) { /* lanes 9..15: lane 8's values */
                    yy[q] = ld_hint(yl + (size_t)(cpos + k) * NV + i, ypol_first);
                    if (accumulate == 1 && !stage_u) uu[q] = Uil[(size_t)(cpos + k) * NV + i];
                }
            }
        };
        if (!YS) load_chunk(nch - 1, yv, uv);
        for (int jb = 0; jb < nf; ++jb) {
            const int job = nf + jb;
            const int c = nch - 1 - jb; /* this half's chunk (may be < 0) */
            if (!YS) load_chunk(c - 1, nyv, nuv);
            const int s = job % NS;
            const bool ok = mbar_wait(&bars[s], parity(job));
            if (__any_sync(FULL, !ok)) {
                timed_out = true;
                break;
            }
            ++consumed;
            const T *sG = reinterpret_cast<const T *>(st0 + (size_t)s * stage + h * half);
            const bool full = (nchT - 1 - jb) * P + P <= m && (nchB - 1 - jb) * P + P <= nb &&
                              nchT - 1 - jb >= 0 && nchB - 1 - jb >= 0;
            const T *sU = stage_u ? sG + P * NB : nullptr;
            if (full)
                bwd_chunk<T, P, false, YS>(sG, bc, ys, yv, uv, dUl, accumulate < 2 ? Ul : nullptr,
                                           c * P, len, cpos, i, off, sU);
            else
                bwd_chunk<T, P, true, YS>(sG, bc, ys, yv, uv, dUl, accumulate < 2 ? Ul : nullptr,
                                          c * P, len, cpos, i, off, sU);
            __syncwarp();
            if (WS) {
                if (lane == 0) mbar_arrive(&empty[s]);
            } else if (lane == 0 && issued < njobs) {
                issue(issued, s);
                ++issued;
            }
            if (!YS) {
#pragma unroll
                for (int q = 0; q < P; ++q) {
                    yv[q] = nyv[q];
                    uv[q] = nuv[q];
                }
            }
        }
        if (YS && !timed_out) {
            /* dU = x (and U = x or U += x) for the line's n cells; the U loads
             * of a batch are issued together so that their latencies overlap */
            const int nv = n * NV;
            constexpr int B = 8;
            for (int t0 = lane; t0 < nv; t0 += 32 * B) {
                T u[B];
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const int t = t0 + 32 * k;
                    u[k] = (accumulate == 1 && t < nv) ? Uil[t] : T(0);
                }
#pragma unroll
                for (int k = 0; k < B; ++k) {
                    const int t = t0 + 32 * k;
                    if (t < nv) {
                        const T x = ys[t];
                        dUl[t] = x;
                        if (accumulate < 2) Ul[t] = u[k] + x;
                    }
                }
            }
        }
    }
    if (timed_out) {
        if (WS) {
            /* stop the producer (its own waits are bounded), then wait for
             * the copies it issued */
            if (lane == 0) *ws_abort = 1;
            __syncwarp();
            __syncthreads();
            issued = *ws_issued;
        }
        if (lane == 0) {
            atomicOr(status, ST_TIMEOUT);
            for (int job = consumed; job < issued; ++job)
                mbar_wait(&bars[job % NS], parity(job), 1LL << 28);
        }
        __syncwarp();
        return false;
    }
    if (WS) __syncthreads(); /* meets the producer's */
    /* every job was waited for: barrier s completed one phase per job
     * j = s, s+NS, ... below njobs */
    for (int s = 0; s < NS && s < njobs; ++s) {
        const int cnt = (njobs - 1 - s) / NS + 1;
        pbase ^= (uint32_t)(cnt & 1) << s;
    }
    return true;
}

__device__ __forceinline__ void thomas_init_bars(unsigned char *smem, int NS) {
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    if ((threadIdx.x & 31) == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncwarp();
}

/* one CTA (one warp) per line */
/* lines from nacc on leave U alone (accumulate 2) */
template <typename T, int P, bool YS>
__global__ void __launch_bounds__(32) fast_thomas_kernel(
    int nline, int NS, int accumulate, int nacc, const int *__restrict__ line_start,
    const int *__restrict__ line_len, const int *__restrict__ line_twist, const T *__restrict__ G,
    const T *__restrict__ Gam, const T *__restrict__ b, T *__restrict__ y, T *__restrict__ dU,
    T *__restrict__ U, const T *__restrict__ Uin, unsigned *status) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int l = blockIdx.x;
    if (l >= nline) return;
    thomas_init_bars(smem, NS);
    const uint64_t pol = threadIdx.x == 0 ? policy_evict_first() : 0;
    uint32_t pbase = 0;
    thomas_line<T, P, YS>(NS, l < nacc ? accumulate : 2, line_start[l], line_len[l], line_twist[l], G,
                          Gam, b, y, dU, U, status, smem, pbase, pol, Uin);
}

/* Warp-specialised form, one CTA of two warps per line: warp 1 issues the
 * staging copies, warp 0 runs the chains with the same arithmetic as
 * fast_thomas_kernel, so its results are bit-identical; the chain warp no
 * longer stops every chunk to issue the next copies. */
template <typename T, int P, bool YS>
__global__ void __launch_bounds__(64) fast_thomas_ws_kernel(
    int nline, int NS, int accumulate, int nacc, const int *__restrict__ line_start,
    const int *__restrict__ line_len, const int *__restrict__ line_twist, const T *__restrict__ G,
    const T *__restrict__ Gam, const T *__restrict__ b, T *__restrict__ y, T *__restrict__ dU,
    T *__restrict__ U, const T *__restrict__ Uin, unsigned *status) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int l = blockIdx.x;
    if (l >= nline) return;
    if (threadIdx.x == 0) {
        uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
        for (int s = 0; s < NS; ++s) {
            mbar_init(&bars[s], 1);
            mbar_init(&bars[8 + s], 1);
        }
        int *cnt = reinterpret_cast<int *>(smem + 128);
        cnt[0] = 0;
        cnt[1] = 0;
        mbar_fence_init();
    }
    __syncthreads();
    const uint64_t pol = threadIdx.x == 32 ? policy_evict_first() : 0;
    uint32_t pbase = 0;
    thomas_line<T, P, YS, true>(NS, l < nacc ? accumulate : 2, line_start[l], line_len[l],
                                line_twist[l], G, Gam, b, y, dU, U, status, smem, pbase, pol, Uin);
}

/* Persistent form over many systems: each CTA (one warp) takes (system,
 * line) items from a device work queue, in the order of `work` (longest
 * lines first, so that the long lines do not start last), and skips the
 * lines of systems that have converged.  queue[0] is the next item,
 * queue[1] counts retired CTAs; the last CTA to retire resets both for the
 * next launch.  U is left to the residual kernel (accumulate = 2). */
template <typename T, int P>
__global__ void __launch_bounds__(32) fast_thomas_batch_kernel(
    const ThomasSys<T> *__restrict__ sys, const WorkItem *__restrict__ work,
    const int *__restrict__ nwork_p, const int *__restrict__ active, unsigned *queue, int NS,
    unsigned *status) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int nwork = *nwork_p;
    thomas_init_bars(smem, NS);
    const uint64_t pol = lane == 0 ? policy_evict_first() : 0;
    uint32_t pbase = 0;
    for (;;) {
        int w = 0;
        if (lane == 0) w = (int)atomicAdd(queue, 1u);
        w = __shfl_sync(FULL, w, 0);
        if (w >= nwork) break;
        const WorkItem it = work[w];
        if (active && !active[it.sys]) continue;
        const ThomasSys<T> S = sys[it.sys];
        const int l = it.unit;
        if (!thomas_line<T, P, false>(NS, 2, S.line_start[l], S.line_len[l], S.line_twist[l], S.G,
                                      S.Gam, S.b, S.y, S.dU, nullptr, status, smem, pbase, pol))
            break;
    }
    if (lane == 0) {
        __threadfence();
        if (atomicAdd(queue + 1, 1u) == gridDim.x - 1) {
            queue[0] = 0u;
            queue[1] = 0u;
            __threadfence();
        }
    }
}

/* The same persistent loop with two warps per CTA: warp 1 issues every
 * line's staging copies, warp 0 runs its chains (thomas_line's
 * warp-specialised form, bit-identical results).  Thread 0 takes the next
 * item for both warps; the staging barriers' parities carry across lines
 * in `pbase`, kept the same in both warps. */
template <typename T, int P>
__global__ void __launch_bounds__(64) fast_thomas_batch_ws_kernel(
    const ThomasSys<T> *__restrict__ sys, const WorkItem *__restrict__ work,
    const int *__restrict__ nwork_p, const int *__restrict__ active, unsigned *queue, int NS,
    unsigned *status) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_item, s_stop;
    const int nwork = *nwork_p;
    if (threadIdx.x == 0) {
        uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
        for (int s = 0; s < NS; ++s) {
            mbar_init(&bars[s], 1);
            mbar_init(&bars[8 + s], 1);
        }
        int *cnt = reinterpret_cast<int *>(smem + 128);
        cnt[0] = 0;
        cnt[1] = 0;
        s_stop = 0;
        mbar_fence_init();
    }
    __syncthreads();
    const uint64_t pol = threadIdx.x == 32 ? policy_evict_first() : 0;
    uint32_t pbase = 0;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int w = s_item;
        __syncthreads(); /* s_item is read before thread 0 takes the next item */
        if (w >= nwork) break;
        const WorkItem it = work[w];
        if (active && !active[it.sys]) continue;
        const ThomasSys<T> S = sys[it.sys];
        const int l = it.unit;
        const bool ok = thomas_line<T, P, false, true>(NS, 2, S.line_start[l], S.line_len[l],
                                                       S.line_twist[l], S.G, S.Gam, S.b, S.y, S.dU,
                                                       nullptr, status, smem, pbase, pol);
        if (!ok && (threadIdx.x & 31) == 0) s_stop = 1;
        __syncthreads();
        if (s_stop) break;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(queue + 1, 1u) == gridDim.x - 1) {
            queue[0] = 0u;
            queue[1] = 0u;
            __threadfence();
        }
    }
}

struct ThomasCfg {
    int NS;
    bool ys;
    size_t smem;
};

template <typename T, bool WS = false>
static ThomasCfg thomas_cfg(const FastLayout &L) {
    const size_t sb = thomas_stage_bytes<T>();
    /* lines resident per SM in one wave, and the shared memory each may use
     * so that they all are: the SM's capacity over them, less the per-CTA
     * reservation.  The deeper the copy ring, the more of the DRAM latency
     * the chain steps hide. */
    int dev = 0, nsm = 148, smem_sm = 228 * 1024, reserved = 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    if (nsm < 1) nsm = 148;
    const int per_sm = (L.nline + nsm - 1) / nsm;
    const long long budget = (long long)smem_sm / (per_sm > 0 ? per_sm : 1) - reserved;
    const size_t ys_bytes = (size_t)((L.max_len + 3) & ~3) * NV * sizeof(T);
    const size_t fixed = thomas_hdr<WS>() + 80 * sizeof(T);
    ThomasCfg c;
    c.ys = (long long)(fixed + ys_bytes + 3 * sb) <= budget;
    long long left = budget - (long long)fixed - (c.ys ? (long long)ys_bytes : 0);
    long long ns = left / (long long)sb;
    if (ns > 8) ns = 8;
    if (ns < 2) ns = 2;
    c.NS = (int)ns;
    c.smem = fixed + (size_t)c.NS * sb + (c.ys ? ys_bytes : 0);
    return c;
}

/* Which single-system line solve: the warp-specialised kernel (a copy
 * warp beside each chain warp) where few lines share an SM -- there the
 * launch is bound by the chain's step latency, and taking the copy issue
 * off the chain warp shortens every step (360 lines: 64 -> 51 us); the
 * one-warp kernel where many lines share an SM, whose warps hide each
 * other's latency and which holds more lines per SM in its registers
 * (1,200 lines: 409 us one-warp, 526 us warp-specialised).  At 600 lines
 * (5 per SM) the copy warp still pays: 117 -> 112 us (FP64), 87 -> 81 us
 * (FP32).  The
 * environment variable TBS_THOMAS_WS=0 / 1 forces one or the other. */
static bool thomas_ws(const FastLayout &L) {
    static const int forced = [] {
        const char *e = getenv("TBS_THOMAS_WS");
        return e && e[0] ? (e[0] == '0' ? 0 : 1) : -1;
    }();
    if (forced >= 0) return forced == 1;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm < 1) nsm = 148;
    return (L.nline + nsm - 1) / nsm <= 5;
}

template <typename T, bool WS, bool YS>
static const void *thomas_fn() {
    return WS ? (const void *)fast_thomas_ws_kernel<T, THOMAS_P, YS>
              : (const void *)fast_thomas_kernel<T, THOMAS_P, YS>;
}

template <typename T, bool WS>
static const void *thomas_fn(bool ys) {
    return ys ? thomas_fn<T, WS, true>() : thomas_fn<T, WS, false>();
}

template <typename T>
int launch_fast_thomas(cudaStream_t st, const FastLayout &L, const T *G, const T *Gam, const T *b,
                       T *y, T *dU, T *U, unsigned *status, int accumulate, int nacc, const T *Uin) {
    if (L.nv != NV) return (int)cudaErrorInvalidValue;
    const bool ws = thomas_ws(L);
    const ThomasCfg c = ws ? thomas_cfg<T, true>(L) : thomas_cfg<T>(L);
    const void *fn = ws ? thomas_fn<T, true>(c.ys) : thomas_fn<T, false>(c.ys);
    int ns = c.NS, nline = L.nline;
    if (nacc < 0 || nacc > nline) nacc = nline;
    const int *ls = L.line_start, *ll = L.line_len, *lt = L.line_twist;
    void *args[] = {&nline, &ns,  &accumulate, &nacc, &ls, &ll, &lt,
                    &G,     &Gam, &b,          &y,    &dU, &U,  &Uin, &status};
    return (int)cudaLaunchKernel(fn, dim3(L.nline), dim3(ws ? 64 : 32), args, c.smem, st);
}

template int launch_fast_thomas<double>(cudaStream_t, const FastLayout &, const double *,
                                        const double *, const double *, double *, double *,
                                        double *, unsigned *, int, int, const double *);
template int launch_fast_thomas<float>(cudaStream_t, const FastLayout &, const float *,
                                       const float *, const float *, float *, float *, float *,
                                       unsigned *, int, int, const float *);

static int smem_limit(const void *fn) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, fn);
    return optin - (int)fa.sharedSizeBytes;
}

int smem_raise(const void *fn, size_t need) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, fn) == cudaSuccess && (size_t)fa.maxDynamicSharedSizeBytes >= need)
        return 0;
    return (int)cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
}

static int set_smem(const void *fn, size_t need) {
    if ((long long)need > smem_limit(fn)) return (int)cudaErrorInvalidConfiguration;
    if (need <= 48 * 1024) return 0;
    return smem_raise(fn, need);
}

/* Called before any launch (and outside stream capture) once the layout is
 * known: opts the streaming kernels into the shared memory they need. */
int fast_prepare(const FastLayout &L) {
    int rc = set_smem((const void *)fast_resid_kernel<double>, resid_smem_bytes<double>(L.nx));
    if (!rc) rc = set_smem((const void *)fast_resid_jv_kernel<double>, resid_smem_bytes<double>(L.nx));
    if (!rc) rc = set_smem((const void *)fast_resid_kernel<float>, resid_smem_bytes<float>(L.nx));
    const ThomasCfg c64 = thomas_cfg<double>(L), c32 = thomas_cfg<float>(L);
    const ThomasCfg w64 = thomas_cfg<double, true>(L), w32 = thomas_cfg<float, true>(L);
    if (!rc) rc = set_smem(thomas_fn<double, false>(c64.ys), c64.smem);
    if (!rc) rc = set_smem(thomas_fn<float, false>(c32.ys), c32.smem);
    if (!rc) rc = set_smem(thomas_fn<double, true>(w64.ys), w64.smem);
    if (!rc) rc = set_smem(thomas_fn<float, true>(w32.ys), w32.smem);
    return rc;
}

int fast_kernels_init() { return 0; }

/* one CTA per line of the pack; the descriptor travels as a kernel parameter */
__global__ void __launch_bounds__(256) line_pack_kernel(LinePack lp, double *__restrict__ vec,
                                                        double *__restrict__ buf, int to_line) {
    const int k = blockIdx.x;
    if (k >= lp.n) return;
    const long long n = (long long)lp.len[k] * NV;
    double *v = vec + (long long)lp.start[k] * NV;
    double *b = buf + lp.off[k];
    for (long long t = threadIdx.x; t < n; t += blockDim.x) {
        if (to_line)
            v[t] = b[t];
        else
            b[t] = v[t];
    }
}

int launch_line_pack(cudaStream_t st, const LinePack &lp, double *vec, double *buf, int to_line) {
    if (lp.n <= 0) return 0;
    line_pack_kernel<<<lp.n, 256, 0, st>>>(lp, vec, buf, to_line);
    return (int)cudaGetLastError();
}

/* ============================================ true residual, any ordering
 * R(pos(e)) = rhs(e) + D_e U(pos(e)) + sum_{faces} offJ U(pos(nbr)) with the
 * original FP64 blocks (face rule of linesmoothLU_TriBlock_v3.okl:299-328),
 * output in position order as T, plus fixed-order per-block sum R^2.
 * Used for the FP64 outer residual of TBS_ALGO_MIXED, for a non-zero
 * starting solution, and for tbs_true_residual_norm / tbs_get_residual. */
constexpr int FULLRES_THREADS = 288;

template <typename T>
__device__ __forceinline__ void full_resid_body(
    int nelem, const int *__restrict__ epoint, const int *__restrict__ ef,
    const int *__restrict__ fc, const int *__restrict__ pos_of_elem,
    const double *__restrict__ D, const double *__restrict__ O1, const double *__restrict__ O2,
    const double *__restrict__ rhs, const double *__restrict__ Up, T *__restrict__ Rp,
    double *__restrict__ partials, int blk) {
    const int epb = FULLRES_THREADS / NV;
    const int le = threadIdx.x / NV;
    const int i = threadIdx.x - le * NV;
    const int e = blk * epb + le;
    double sq = 0.0;
    if (e < nelem) {
        const int pe = pos_of_elem[e];
        const double *u = Up + (size_t)pe * NV;
        const double *dr = D + (size_t)e * NB + i;
        double a0 = dr[0] * u[0], a1 = dr[9] * u[1], a2 = dr[18] * u[2];
        a0 += dr[27] * u[3];
        a1 += dr[36] * u[4];
        a2 += dr[45] * u[5];
        a0 += dr[54] * u[6];
        a1 += dr[63] * u[7];
        a2 += dr[72] * u[8];
        for (int k2 = epoint[e]; k2 < epoint[e + 1]; ++k2) {
            const int f = ef[k2];
            if (f >= 0) {
                const int e1 = fc[2 * f], e2 = fc[2 * f + 1];
                const double *o = ((e == e1) ? O2 : O1) + (size_t)f * NB + i;
                const double *un = Up + (size_t)pos_of_elem[(e == e1) ? e2 : e1] * NV;
                a0 += o[0] * un[0];
                a1 += o[9] * un[1];
                a2 += o[18] * un[2];
                a0 += o[27] * un[3];
                a1 += o[36] * un[4];
                a2 += o[45] * un[5];
                a0 += o[54] * un[6];
                a1 += o[63] * un[7];
                a2 += o[72] * un[8];
            }
        }
        const double r = (rhs ? rhs[(size_t)e * NV + i] : 0.0) + (a0 + (a1 + a2));
        Rp[(size_t)pe * NV + i] = (T)r;
        sq = r * r;
    }
    __shared__ double red[FULLRES_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(FULL, sq, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < FULLRES_THREADS / 32; ++w) tot += red[w];
        partials[blk] = tot;
    }
}

template <typename T>
__global__ void __launch_bounds__(FULLRES_THREADS) full_resid_kernel(
    int nelem, const int *__restrict__ epoint, const int *__restrict__ ef,
    const int *__restrict__ fc, const int *__restrict__ pos_of_elem,
    const double *__restrict__ D, const double *__restrict__ O1, const double *__restrict__ O2,
    const double *__restrict__ rhs, const double *__restrict__ Up, T *__restrict__ Rp,
    double *__restrict__ partials) {
    full_resid_body<T>(nelem, epoint, ef, fc, pos_of_elem, D, O1, O2, rhs, Up, Rp, partials,
                       blockIdx.x);
}

int full_resid_blocks(int nelem) { return (nelem + (FULLRES_THREADS / NV) - 1) / (FULLRES_THREADS / NV); }

template <typename T>
int launch_full_resid(cudaStream_t st, int nelem, const int *epoint, const int *ef, const int *fc,
                      const int *pos_of_elem, const double *D, const double *O1, const double *O2,
                      const double *rhs, const double *Up, T *Rp, double *partials) {
    full_resid_kernel<T><<<full_resid_blocks(nelem), FULLRES_THREADS, 0, st>>>(
        nelem, epoint, ef, fc, pos_of_elem, D, O1, O2, rhs, Up, Rp, partials);
    return (int)cudaGetLastError();
}

template int launch_full_resid<double>(cudaStream_t, int, const int *, const int *, const int *,
                                       const int *, const double *, const double *,
                                       const double *, const double *, const double *, double *,
                                       double *);
template int launch_full_resid<float>(cudaStream_t, int, const int *, const int *, const int *,
                                      const int *, const double *, const double *,
                                      const double *, const double *, const double *, float *,
                                      double *);


/* ============================================ full residual, position order
 * Dp = D blocks by position, XF[s][p] = the block of interior face s of the
 * cell (ef order) in the cell's row; both from the original FP64 arrays,
 * zero where absent.  One warp per block. */
__global__ void fullpos_layout_kernel(long long nblk, int np16, const int *__restrict__ elem_of_pos,
                                      const int *__restrict__ xsrcf, const double *__restrict__ D,
                                      const double *__restrict__ O1, const double *__restrict__ O2,
                                      double *__restrict__ Dp, double *__restrict__ XF) {
    const int lane = threadIdx.x & 31;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long q = w0; q < nblk; q += nw) {
        const double *src = nullptr;
        double *dst;
        if (q < np16) {
            const int e = elem_of_pos[q];
            if (e >= 0) src = D + (size_t)e * NB;
            dst = Dp + q * NB;
        } else {
            const long long k = q - np16; /* slot-major index s*np16 + p */
            const int f = xsrcf[k];
            if (f >= 0) src = ((f & 1) ? O2 : O1) + (size_t)(f >> 1) * NB;
            dst = XF + k * NB;
        }
        for (int tt = lane; tt < NB; tt += 32) dst[tt] = src ? src[tt] : 0.0;
    }
}

int launch_fullpos_layout(cudaStream_t st, const FastLayout &L, const double *jacD,
                          const double *O1, const double *O2, double *Dp, double *XF) {
    const long long nblk = (long long)L.np16 * (1 + L.nxf);
    fullpos_layout_kernel<<<grid_for(nblk * 32, 256), 256, 0, st>>>(nblk, L.np16, L.elem_of_pos,
                                                                    L.xsrcf, jacD, O1, O2, Dp, XF);
    return (int)cudaGetLastError();
}

__host__ __device__ inline size_t fullpos_smem_bytes(int nxf) {
    return 128 + (size_t)RES_TILE * NB * sizeof(double) * (1 + nxf) +
           (size_t)(nxf + 1) * RES_TILE * NV * sizeof(double) + (size_t)RES_TILE * NV * sizeof(double) +
           (size_t)RES_TILE * NB * sizeof(float) + 2 * (size_t)RES_TILE * NV * sizeof(float);
}

/* b = -Dinv R of one cell row in FP32, the operation order of the FP32
 * mode-0 residual (fast_resid_body): dr = column-major block row i, rv = R */

/* One tile of 16 positions (160 threads; thread t < 144 owns cell t % 16,
 * row t / 16).  R = rhs + D u + sum over faces (ef order) offJ u_nbr with
 * the accumulation pattern of full_resid_body; R32 out, partials[blk] =
 * the tile's sum R^2 (fixed order).  With Dinv32: also the next inner
 * solve's right-hand side b32 = -Dinv32 R32 and c32 = 0. */
__device__ __forceinline__ bool full_resid_pos_body(
    int nxf, int np16, const double *__restrict__ Dp, const double *__restrict__ XF,
    const int *__restrict__ xnbrf, const double *__restrict__ rhsp, const double *__restrict__ Up,
    float *__restrict__ R32, double *__restrict__ partials, const float *__restrict__ Dinv32,
    float *__restrict__ b32, float *__restrict__ c32, unsigned *status, int blk, uint64_t *bar,
    uint32_t parity, const int *nbr_pre = nullptr) {
    extern __shared__ __align__(128) unsigned char smem[];
    double *sD = reinterpret_cast<double *>(smem + 128);
    double *sX = sD + RES_TILE * NB;
    double *sg = sX + nxf * RES_TILE * NB;      /* [1 + nxf][16][9]: own u, then neighbours */
    double *sr = sg + (nxf + 1) * RES_TILE * NV; /* rhs tile */
    float *sDi = reinterpret_cast<float *>(sr + RES_TILE * NV); /* Dinv32 tile */
    float *so = sDi + RES_TILE * NB;
    float *sb = so + RES_TILE * NV;
    const int p0 = blk * RES_TILE;
    const int tid = threadIdx.x;
    const int c = tid % RES_TILE, i = tid / RES_TILE;
    const bool act = tid < RES_TILE * NV;
    const uint32_t szD = RES_TILE * NB * sizeof(double), szR = RES_TILE * NV * sizeof(double);
    const uint32_t szDi = RES_TILE * NB * sizeof(float);
    if (tid == 0) {
        const uint64_t pol = policy_evict_first();
        mbar_arrive_expect_tx(bar, szD * (1 + nxf) + szR + (Dinv32 ? szDi : 0u));
        bulk_g2s_hint(sD, Dp + (size_t)p0 * NB, szD, bar, pol);
        for (int s = 0; s < nxf; ++s)
            bulk_g2s_hint(sX + s * RES_TILE * NB, XF + ((size_t)s * np16 + p0) * NB, szD, bar, pol);
        bulk_g2s(sr, rhsp + (size_t)p0 * NV, szR, bar);
        if (Dinv32) bulk_g2s_hint(sDi, Dinv32 + (size_t)p0 * NB, szDi, bar, pol);
    }
    if (act && c32) c32[(size_t)p0 * NV + tid] = 0.0f;
    if (act) {
        sg[c * NV + i] = Up[(size_t)(p0 + c) * NV + i];
        if (nbr_pre) { /* indices loaded during the previous tile */
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                if (s < nxf) {
                    const int nb = nbr_pre[s];
                    sg[((s + 1) * RES_TILE + c) * NV + i] = (nb >= 0) ? Up[(size_t)nb * NV + i] : 0.0;
                }
            }
        } else {
            for (int s = 0; s < nxf; ++s) {
                const int nb = xnbrf[(size_t)s * np16 + p0 + c];
                sg[((s + 1) * RES_TILE + c) * NV + i] = (nb >= 0) ? Up[(size_t)nb * NV + i] : 0.0;
            }
        }
    }
    const bool ok = mbar_wait(bar, parity);
    if (__syncthreads_or(!ok)) {
        if (tid == 0) {
            atomicOr(status, ST_TIMEOUT);
            mbar_wait(bar, parity, 1LL << 28); /* let the copies land before the CTA retires */
        }
        return false;
    }
    double sq = 0.0;
    if (act) {
        const double *dr = sD + c * NB + i;
        const double *u = sg + c * NV;
        double a0 = dr[0] * u[0], a1 = dr[9] * u[1], a2 = dr[18] * u[2];
        a0 += dr[27] * u[3];
        a1 += dr[36] * u[4];
        a2 += dr[45] * u[5];
        a0 += dr[54] * u[6];
        a1 += dr[63] * u[7];
        a2 += dr[72] * u[8];
        for (int s = 0; s < nxf; ++s) {
            const double *o = sX + (s * RES_TILE + c) * NB + i;
            const double *un = sg + ((s + 1) * RES_TILE + c) * NV;
            a0 += o[0] * un[0];
            a1 += o[9] * un[1];
            a2 += o[18] * un[2];
            a0 += o[27] * un[3];
            a1 += o[36] * un[4];
            a2 += o[45] * un[5];
            a0 += o[54] * un[6];
            a1 += o[63] * un[7];
            a2 += o[72] * un[8];
        }
        const double r = sr[c * NV + i] + (a0 + (a1 + a2));
        so[c * NV + i] = (float)r;
        sq = r * r;
    }
    __syncthreads();
    if (act) R32[(size_t)p0 * NV + tid] = so[tid]; /* contiguous tile store */
    if (Dinv32) {
        if (act) sb[c * NV + i] = neg_dinv_row<float>(sDi + c * NB + i, so + c * NV);
        __syncthreads();
        if (act) b32[(size_t)p0 * NV + tid] = sb[tid];
    }
    __shared__ double red[RES_THREADS_FAST / 32];
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(FULL, sq, o);
    if ((tid & 31) == 0) red[tid >> 5] = sq;
    __syncthreads();
    if (tid == 0) {
        double tot = 0.0;
        for (int w = 0; w < RES_THREADS_FAST / 32; ++w) tot += red[w];
        partials[blk] = tot;
    }
    return true;
}

/* persistent: CTA k takes tiles k, k + grid, ... */
__global__ void __launch_bounds__(RES_THREADS_FAST) full_resid_pos_kernel(
    int nxf, int np16, const double *__restrict__ Dp, const double *__restrict__ XF,
    const int *__restrict__ xnbrf, const double *__restrict__ rhsp, const double *__restrict__ Up,
    float *__restrict__ R32, double *__restrict__ partials, const float *__restrict__ Dinv32,
    float *__restrict__ b32, float *__restrict__ c32, unsigned *status) {
    uint64_t *bar = resid_bar_init();
    const int ntiles = np16 / RES_TILE;
    uint32_t parity = 0;
    /* the next tile's neighbour indices load during the current one */
    const bool pre = nxf >= 1 && nxf <= 4 && threadIdx.x < RES_TILE * NV;
    const int c = threadIdx.x % RES_TILE;
    int nbr[4], nxt[4];
#pragma unroll
    for (int s = 0; s < 4; ++s)
        nbr[s] = (pre && s < nxf && (int)blockIdx.x < ntiles)
                     ? xnbrf[(size_t)s * np16 + blockIdx.x * RES_TILE + c] : -1;
    for (int w = blockIdx.x; w < ntiles; w += gridDim.x) {
        const int wn = w + gridDim.x;
#pragma unroll
        for (int s = 0; s < 4; ++s)
            nxt[s] = (pre && s < nxf && wn < ntiles) ? xnbrf[(size_t)s * np16 + wn * RES_TILE + c] : -1;
        const bool ok = full_resid_pos_body(nxf, np16, Dp, XF, xnbrf, rhsp, Up, R32, partials, Dinv32,
                                            b32, c32, status, w, bar, parity, pre ? nbr : nullptr);
        parity ^= 1u;
        if (!ok) break;
#pragma unroll
        for (int s = 0; s < 4; ++s) nbr[s] = nxt[s];
        __syncthreads(); /* the next tile's copies overwrite the stages */
    }
}

int launch_full_resid_pos(cudaStream_t st, const FastLayout &L, const double *Dp, const double *XF,
                          const double *rhsp, const double *Up, float *R32, double *partials,
                          const float *Dinv32, float *b32, float *c32, unsigned *status) {
    if (L.nxf < 0 || L.nxf > 4) return (int)cudaErrorInvalidValue;
    const size_t smem = fullpos_smem_bytes(L.nxf);
    const int grid = resid_grid_persistent((const void *)full_resid_pos_kernel, smem,
                                           fast_resid_grid(L.np16));
    full_resid_pos_kernel<<<grid, RES_THREADS_FAST, smem, st>>>(L.nxf, L.np16, Dp, XF, L.xnbrf, rhsp,
                                                                Up, R32, partials, Dinv32, b32, c32,
                                                                status);
    return (int)cudaGetLastError();
}

/* ================================================ mixed-precision prime
 * Per tile of RES_TILE positions (160 threads, 144 active): U = 0, the
 * FP32 copy of the residual R = rhs, and the tile's sum rhs^2 in a fixed
 * order (lane order within a warp, then warps in order). */
__device__ __forceinline__ void mixed_prime_body(const double *__restrict__ rhsp,
                                                 float *__restrict__ R32, double *__restrict__ Up,
                                                 double *__restrict__ partials,
                                                 const float *__restrict__ Dinv32,
                                                 float *__restrict__ b32, float *__restrict__ c32,
                                                 int blk) {
    const int tid = threadIdx.x;
    const bool act = tid < RES_TILE * NV;
    __shared__ float sR[RES_TILE * NV];
    double sq = 0.0;
    if (act) {
        const size_t q = (size_t)blk * RES_TILE * NV + tid;
        const double v = rhsp[q];
        R32[q] = (float)v;
        sR[tid] = (float)v;
        Up[q] = 0.0;
        if (c32) c32[q] = 0.0f;
        sq = v * v;
    }
    if (Dinv32) {
        /* the first inner solve's right-hand side b32 = -Dinv32 R32, from
         * the tile's Dinv32 blocks staged with coalesced loads */
        __shared__ float sDi[RES_TILE * NB];
        const float *src = Dinv32 + (size_t)blk * RES_TILE * NB;
        for (int t = tid; t < RES_TILE * NB; t += blockDim.x) sDi[t] = src[t];
        __syncthreads();
        if (act) {
            const int c = tid % RES_TILE, i = tid / RES_TILE;
            b32[((size_t)blk * RES_TILE + c) * NV + i] = neg_dinv_row<float>(sDi + c * NB + i, sR + c * NV);
        }
    }
    __shared__ double red[RES_THREADS_FAST / 32];
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(FULL, sq, o);
    if ((tid & 31) == 0) red[tid >> 5] = sq;
    __syncthreads();
    if (tid == 0) {
        double tot = 0.0;
        for (int w = 0; w < RES_THREADS_FAST / 32; ++w) tot += red[w];
        partials[blk] = tot;
    }
}

/* one CTA per tile (measured faster than a persistent loop here) */
__global__ void __launch_bounds__(RES_THREADS_FAST) mixed_prime_kernel(
    const double *__restrict__ rhsp, float *__restrict__ R32, double *__restrict__ Up,
    double *__restrict__ partials, const float *__restrict__ Dinv32, float *__restrict__ b32,
    float *__restrict__ c32) {
    mixed_prime_body(rhsp, R32, Up, partials, Dinv32, b32, c32, blockIdx.x);
}

int launch_mixed_prime(cudaStream_t st, const FastLayout &L, const double *rhsp, float *R32,
                       double *Up, double *partials, const float *Dinv32, float *b32, float *c32) {
    mixed_prime_kernel<<<fast_resid_grid(L.np16), RES_THREADS_FAST, 0, st>>>(rhsp, R32, Up, partials,
                                                                             Dinv32, b32, c32);
    return (int)cudaGetLastError();
}

/* ================================================================ batches
 * Every batched kernel reads its work count from device memory (a field of
 * the launch sequence's BatchCtl), so one instantiated graph serves any set
 * of members; all but the per-member norm kernel are persistent, with grids
 * sized to the SMs. */

/* Item w of a group index (layout in tbs_internal.hxx): the group by
 * binary search over the prefix sums, then unit-major within the group. */
__device__ __forceinline__ WorkItem group_item(const int *__restrict__ gi, int w) {
    const int ng = gi[0];
    const int *base = gi + 1;
    int lo = 0, hi = ng - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (base[mid] <= w) lo = mid;
        else hi = mid - 1;
    }
    const int *nmem = base + ng + 1, *moff = nmem + ng, *mlist = moff + ng;
    const int off = w - base[lo], r = nmem[lo];
    return WorkItem{mlist[moff[lo] + off % r], off / r};
}

__device__ __forceinline__ int group_items(const int *__restrict__ gi) { return gi[1 + gi[0]]; }

/* group_item for a CTA that visits items in increasing order: the group of
 * the last item (its range [lo, hi) and index g) is kept, so the binary
 * search runs only when the item leaves it */
struct GroupCursor {
    int lo = 0, hi = 0, g = -1;
    int r = 1, mo = 0, m0 = 0; /* the group's member count, list offset, first member */
};

__device__ __forceinline__ WorkItem group_item_next(const int *__restrict__ gi, int w, GroupCursor &c) {
    const int ng = gi[0];
    const int *base = gi + 1;
    const int *nmem = base + ng + 1, *moff = nmem + ng, *mlist = moff + ng;
    if (c.g < 0 || w < c.lo || w >= c.hi) {
        int lo = 0, hi = ng - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (base[mid] <= w) lo = mid;
            else hi = mid - 1;
        }
        c.g = lo;
        c.lo = base[lo];
        c.hi = base[lo + 1];
        c.r = nmem[lo];
        c.mo = moff[lo];
        c.m0 = mlist[c.mo];
    }
    const int off = w - c.lo;
    if (c.r == 1) return WorkItem{c.m0, off};
    return WorkItem{mlist[c.mo + off % c.r], off / c.r};
}

static int sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}

template <typename T>
size_t thomas_batch_smem(int stages, int warps) {
    return (warps == 2 ? thomas_hdr<true>() : thomas_hdr<false>()) +
           (size_t)stages * 2 * THOMAS_P * (NB + NV) * sizeof(T) + 80 * sizeof(T);
}

template <typename T>
int thomas_batch_fit(int stages, int warps) {
    int n = 0;
    const size_t smem = thomas_batch_smem<T>(stages, warps);
    const void *fn = warps == 2 ? (const void *)fast_thomas_batch_ws_kernel<T, THOMAS_P>
                                : (const void *)fast_thomas_batch_kernel<T, THOMAS_P>;
    if (smem_raise(fn, smem) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, 32 * warps, smem) != cudaSuccess)
        return 0;
    return n;
}

template <typename T>
int launch_thomas_batch(cudaStream_t st, const BatchSched &bs, const ThomasSys<T> *sys,
                        const WorkItem *work, const int *nwork, const int *active, unsigned *queue,
                        unsigned *status) {
    if (bs.stages < 2 || bs.stages > 8 || bs.ctas_per_sm < 1 || (bs.warps != 1 && bs.warps != 2))
        return (int)cudaErrorInvalidValue;
    const size_t smem = thomas_batch_smem<T>(bs.stages, bs.warps);
    const int grid = bs.ctas_per_sm * sm_count();
    if (bs.warps == 2)
        fast_thomas_batch_ws_kernel<T, THOMAS_P><<<grid, 64, smem, st>>>(sys, work, nwork, active,
                                                                          queue, bs.stages, status);
    else
        fast_thomas_batch_kernel<T, THOMAS_P><<<grid, 32, smem, st>>>(sys, work, nwork, active,
                                                                       queue, bs.stages, status);
    return (int)cudaGetLastError();
}

/* The tiles [unit * chunk, ...) of a member: the units of a group index
 * are single tiles (chunk 1) or chunks of BATCH_CHUNK tiles, which pay the
 * item's decode and descriptor load once for several tiles */
__device__ __forceinline__ int chunk_end(int unit, int chunk, int ntiles) {
    const int e = (unit + 1) * chunk;
    return e < ntiles ? e : ntiles;
}

/* persistent residual over (member, tile or chunk) items: CTA k takes
 * items k, k + grid, ...; each tile completes one phase of the CTA's
 * barrier and writes its own partial */
template <typename T, int CHUNK>
__global__ void __launch_bounds__(RES_THREADS_FAST, CHUNK == 1 ? 8 : 6) fast_resid_batch_kernel(
    const ResidSys<T> *__restrict__ sys, const int *__restrict__ groups, int mode,
    const int *__restrict__ active, unsigned *status) {
    constexpr int chunk = CHUNK;
    uint64_t *bar = resid_bar_init();
    const int nwork = group_items(groups);
    uint32_t parity = 0;
    GroupCursor gc;
    bool ok = true;
    for (int w = blockIdx.x; w < nwork && ok; w += gridDim.x) {
        const WorkItem it = group_item_next(groups, w, gc);
        if (active && !active[it.sys]) continue;
        const ResidSys<T> S = sys[it.sys];
        NormSink ns{};
        ns.partials = (mode == 3) ? nullptr : S.partials; /* no counter: partials only */
        const int t1 = chunk_end(it.unit, chunk, S.np16 / RES_TILE);
        /* the next tile's neighbour indices load during the current tile */
        const int nxm = mode == 0 ? 0 : S.nx;
        const bool pre = CHUNK > 1 && nxm >= 1 && nxm <= 4 && threadIdx.x < RES_TILE * NV;
        const int c = threadIdx.x % RES_TILE;
        int nbr[4], nxt[4];
        const int tb = it.unit * chunk;
#pragma unroll
        for (int s = 0; s < 4; ++s)
            nbr[s] = (pre && s < nxm && tb < t1) ? S.xnbr[(size_t)s * S.np16 + tb * RES_TILE + c] : -1;
        for (int t = tb; t < t1; ++t) {
#pragma unroll
            for (int s = 0; s < 4; ++s)
                nxt[s] = (pre && s < nxm && t + 1 < t1) ? S.xnbr[(size_t)s * S.np16 + (t + 1) * RES_TILE + c]
                                                        : -1;
            ok = fast_resid_body<T>(nxm, S.np16, mode, S.Dinv, S.X, S.xnbr, S.dU, S.Rsrc, S.b, S.Uacc, ns,
                                    status, t, bar, parity, pre ? nbr : nullptr);
            parity ^= 1u;
            if (!ok) break;
#pragma unroll
            for (int s = 0; s < 4; ++s) nbr[s] = nxt[s];
            __syncthreads(); /* the next tile's copies overwrite the stages */
        }
    }
}

/* Item w of a unit index (the group index layout with base[] the prefix
 * sums of each group's units, not units x members): (group, unit). */
__device__ __forceinline__ int2 group_unit(const int *__restrict__ gi, int w) {
    const int ng = gi[0];
    const int *base = gi + 1;
    int lo = 0, hi = ng - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (base[mid] <= w) lo = mid;
        else hi = mid - 1;
    }
    return make_int2(lo, w - base[lo]);
}

/* The sweep residual (mode 1) of the members of one system together: an
 * item is (system group, chunk of tiles); per tile the CTA stages the
 * system's Dinv and cross-line blocks once and then runs every active
 * member (one right-hand side each) over them, with fast_resid_body's
 * arithmetic, in its order, for each: U += dU, neighbour gathers, R, b,
 * the tile's partial.  The members' blocks are read from HBM once per tile
 * instead of once per member. */
template <typename T>
__global__ void __launch_bounds__(RES_THREADS_FAST) fast_resid_group_kernel(
    const ResidSys<T> *__restrict__ sys, const int *__restrict__ gunits, int chunk,
    const int *__restrict__ active, unsigned *status) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double red[RES_THREADS_FAST / 32];
    uint64_t *bar = resid_bar_init();
    const int ng = gunits[0];
    const int nwork = gunits[1 + ng];
    const int *nmem = gunits + 2 + ng, *moff = nmem + ng, *mlist = moff + ng;
    const int tid = threadIdx.x;
    const int c = tid % RES_TILE, i = tid / RES_TILE;
    const bool act = tid < RES_TILE * NV;
    uint32_t parity = 0;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 gu = group_unit(gunits, w);
        const int *ml = mlist + moff[gu.x];
        const int r = nmem[gu.x];
        const ResidSys<T> S0 = sys[ml[0]];
        const int nx = S0.nx, np16 = S0.np16;
        const int nxa = nx > 0 ? nx : 1;
        T *sD = reinterpret_cast<T *>(smem + 128);
        T *sX = sD + RES_TILE * NB;
        T *sg = sX + nx * RES_TILE * NB;
        T *sr = sg + nxa * RES_TILE * NV;
        T *sb = sr + RES_TILE * NV;
        const uint32_t szD = RES_TILE * NB * sizeof(T);
        const int t1 = chunk_end(gu.y, chunk, np16 / RES_TILE);
        const int tb = gu.y * chunk;
        /* a tile's neighbour indices serve every member; the next tile's
         * load while this one is worked on */
        int nb[4], nbn[4];
#pragma unroll
        for (int s = 0; s < 4; ++s)
            nb[s] = (act && s < nx && tb < t1) ? S0.xnbr[(size_t)s * np16 + tb * RES_TILE + c] : -1;
        for (int t = tb; t < t1; ++t) {
            const int p0 = t * RES_TILE;
            if (tid == 0) {
                const uint64_t pol = policy_evict_first();
                mbar_arrive_expect_tx(bar, (1 + nx) * szD);
                bulk_g2s_hint(sD, S0.Dinv + (size_t)p0 * NB, szD, bar, pol);
                for (int s = 0; s < nx; ++s)
                    bulk_g2s_hint(sX + s * RES_TILE * NB, S0.X + ((size_t)s * np16 + p0) * NB, szD, bar,
                                  pol);
            }
#pragma unroll
            for (int s = 0; s < 4; ++s)
                nbn[s] = (act && s < nx && t + 1 < t1) ? S0.xnbr[(size_t)s * np16 + (t + 1) * RES_TILE + c]
                                                       : -1;
            /* members in a software pipeline: the next active member's
             * loads (its U and dU, its neighbour gathers) are issued before
             * the current one's products, so they overlap them */
            const size_t q = (size_t)p0 * NV + tid;
            auto next_active = [&](int k) {
                while (k < r && active && !active[ml[k]]) ++k;
                return k;
            };
            auto load_member = [&](const ResidSys<T> &S, T &u, T &d, T (&g)[4]) {
                u = d = T(0);
#pragma unroll
                for (int s = 0; s < 4; ++s) g[s] = T(0);
                if (!act) return;
                d = S.dU[q];
                if (S.Uacc) u = S.Uacc[q];
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    if (s < nx && nb[s] >= 0) g[s] = S.dU[(size_t)nb[s] * NV + i];
            };
            bool staged = false;
            int k = next_active(0);
            ResidSys<T> Sc{};
            T cu, cd, cg[4];
            if (k < r) {
                Sc = sys[ml[k]];
                load_member(Sc, cu, cd, cg);
            }
            while (k < r) {
                if (act && Sc.Uacc) Sc.Uacc[q] = cu + cd;
                if (act) {
#pragma unroll
                    for (int s = 0; s < 4; ++s)
                        if (s < nx) sg[(s * RES_TILE + c) * NV + i] = cg[s];
                }
                const int kn = next_active(k + 1);
                ResidSys<T> Sn{};
                T nu = T(0), nd = T(0), ngv[4] = {T(0), T(0), T(0), T(0)};
                if (kn < r) {
                    Sn = sys[ml[kn]];
                    load_member(Sn, nu, nd, ngv);
                }
                if (!staged) {
                    const bool ok = mbar_wait(bar, parity);
                    parity ^= 1u;
                    staged = true;
                    if (__syncthreads_or(!ok)) {
                        if (tid == 0) {
                            atomicOr(status, ST_TIMEOUT);
                            mbar_wait(bar, parity ^ 1u, 1LL << 28);
                        }
                        return;
                    }
                } else {
                    __syncthreads();
                }
                T rr = T(0);
                if (act) {
                    T a0 = T(0), a1 = T(0), a2 = T(0);
                    for (int s = 0; s < nx; ++s) {
                        const T *xr = sX + (s * RES_TILE + c) * NB + i;
                        const T *g = sg + (s * RES_TILE + c) * NV;
                        a0 += xr[0] * g[0];
                        a1 += xr[9] * g[1];
                        a2 += xr[18] * g[2];
                        a0 += xr[27] * g[3];
                        a1 += xr[36] * g[4];
                        a2 += xr[45] * g[5];
                        a0 += xr[54] * g[6];
                        a1 += xr[63] * g[7];
                        a2 += xr[72] * g[8];
                    }
                    rr = a0 + (a1 + a2);
                    sr[c * NV + i] = rr;
                }
                __syncthreads();
                double sq = act ? (double)rr * (double)rr : 0.0;
                if (act) sb[c * NV + i] = neg_dinv_row<T>(sD + c * NB + i, sr + c * NV);
                __syncthreads();
                if (act) Sc.b[(size_t)p0 * NV + tid] = sb[tid];
                for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(FULL, sq, o);
                if ((tid & 31) == 0) red[tid >> 5] = sq;
                __syncthreads();
                if (tid == 0) {
                    double tot = 0.0;
                    for (int ww = 0; ww < RES_THREADS_FAST / 32; ++ww) tot += red[ww];
                    Sc.partials[t] = tot;
                }
                __syncthreads(); /* the next member overwrites sg, sr, sb and red */
                Sc = Sn;
                cu = nu;
                cd = nd;
#pragma unroll
                for (int s = 0; s < 4; ++s) cg[s] = ngv[s];
                k = kn;
            }
            if (!staged) { /* no member active: the tile's copies still land */
                const bool ok = mbar_wait(bar, parity);
                parity ^= 1u;
                if (__syncthreads_or(!ok)) {
                    if (tid == 0) {
                        atomicOr(status, ST_TIMEOUT);
                        mbar_wait(bar, parity ^ 1u, 1LL << 28);
                    }
                    return;
                }
            }
#pragma unroll
            for (int s = 0; s < 4; ++s) nb[s] = nbn[s];
            __syncthreads(); /* the next tile's copies overwrite the stages */
        }
    }
}

static int resid_batch_grid(size_t smem, const void *fn) {
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, RES_THREADS_FAST, smem) != cudaSuccess ||
        per < 1)
        per = 1;
    return per * sm_count();
}

template <typename T>
int launch_resid_batch(cudaStream_t st, int mode, int max_nx, const ResidSys<T> *sys,
                       const int *groups, int chunk, const int *active, unsigned *status) {
    if (mode != 0 && mode != 1 && mode != 3) return (int)cudaErrorInvalidValue;
    if (chunk != 1 && chunk != BATCH_CHUNK) return (int)cudaErrorInvalidValue;
    const size_t smem = resid_smem_bytes<T>(mode == 0 ? 0 : max_nx);
    if (chunk == 1) {
        const int grid = resid_batch_grid(smem, (const void *)fast_resid_batch_kernel<T, 1>);
        fast_resid_batch_kernel<T, 1><<<grid, RES_THREADS_FAST, smem, st>>>(sys, groups, mode, active,
                                                                            status);
    } else {
        const int grid = resid_batch_grid(smem, (const void *)fast_resid_batch_kernel<T, BATCH_CHUNK>);
        fast_resid_batch_kernel<T, BATCH_CHUNK><<<grid, RES_THREADS_FAST, smem, st>>>(sys, groups, mode,
                                                                                      active, status);
    }
    return (int)cudaGetLastError();
}

__global__ void __launch_bounds__(FULLRES_THREADS) full_resid_batch_kernel(
    const FullResSys *__restrict__ sys, const int *__restrict__ groups,
    const int *__restrict__ active) {
    const int nwork = group_items(groups);
    GroupCursor gc;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const WorkItem it = group_item_next(groups, w, gc);
        if (active && !active[it.sys]) continue;
        const FullResSys S = sys[it.sys];
        full_resid_body<float>(S.nelem, S.epoint, S.ef, S.fc, S.pos_of_elem, S.D, S.O1, S.O2,
                               S.rhs, S.Up, S.R32, S.partials, it.unit);
        __syncthreads(); /* the block sum's shared array is reused */
    }
}

static int plain_batch_grid(const void *fn, int threads) {
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, 0) != cudaSuccess || per < 1)
        per = 1;
    return per * sm_count();
}

int launch_full_resid_batch(cudaStream_t st, const FullResSys *sys, const int *groups,
                            const int *active) {
    const int grid = plain_batch_grid((const void *)full_resid_batch_kernel, FULLRES_THREADS);
    full_resid_batch_kernel<<<grid, FULLRES_THREADS, 0, st>>>(sys, groups, active);
    return (int)cudaGetLastError();
}

__global__ void __launch_bounds__(RES_THREADS_FAST) mixed_prime_batch_kernel(
    const VecSys *__restrict__ sys, const int *__restrict__ groups) {
    const int nwork = group_items(groups);
    GroupCursor gc;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const WorkItem it = group_item_next(groups, w, gc);
        const VecSys S = sys[it.sys];
        mixed_prime_body(S.rhsp, S.R32, S.Up, S.partials, S.Dinv32, S.b32, S.c32, it.unit);
        __syncthreads();
    }
}

int launch_mixed_prime_batch(cudaStream_t st, const VecSys *sys, const int *groups) {
    const int grid = plain_batch_grid((const void *)mixed_prime_batch_kernel, RES_THREADS_FAST);
    mixed_prime_batch_kernel<<<grid, RES_THREADS_FAST, 0, st>>>(sys, groups);
    return (int)cudaGetLastError();
}

/* U += c + d over one tile (elementwise: the same values as axpy2_kernel) */
__global__ void __launch_bounds__(RES_THREADS_FAST) axpy2_batch_kernel(
    const VecSys *__restrict__ sys, const int *__restrict__ groups,
    const int *__restrict__ active) {
    const int nwork = group_items(groups);
    GroupCursor gc;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const WorkItem it = group_item_next(groups, w, gc);
        if (active && !active[it.sys]) continue;
        if (threadIdx.x >= RES_TILE * NV) continue;
        const VecSys S = sys[it.sys];
        const size_t q = (size_t)it.unit * RES_TILE * NV + threadIdx.x;
        S.Up[q] += (double)S.c32[q] + (double)S.d32[q];
    }
}

int launch_axpy2_batch(cudaStream_t st, const VecSys *sys, const int *groups, const int *active) {
    const int grid = plain_batch_grid((const void *)axpy2_batch_kernel, RES_THREADS_FAST);
    axpy2_batch_kernel<<<grid, RES_THREADS_FAST, 0, st>>>(sys, groups, active);
    return (int)cudaGetLastError();
}

__global__ void __launch_bounds__(RES_THREADS_FAST) full_resid_pos_batch_kernel(
    const FullPosSys *__restrict__ sys, const int *__restrict__ groups, int chunk,
    const int *__restrict__ active, unsigned *status) {
    uint64_t *bar = resid_bar_init();
    const int nwork = group_items(groups);
    uint32_t parity = 0;
    GroupCursor gc;
    bool ok = true;
    for (int w = blockIdx.x; w < nwork && ok; w += gridDim.x) {
        const WorkItem it = group_item_next(groups, w, gc);
        if (active && !active[it.sys]) continue;
        const FullPosSys S = sys[it.sys];
        const int t1 = chunk_end(it.unit, chunk, S.np16 / RES_TILE);
        /* the next tile's neighbour indices load during the current one */
        const bool pre = chunk > 1 && S.nxf >= 1 && S.nxf <= 4 && threadIdx.x < RES_TILE * NV;
        const int c = threadIdx.x % RES_TILE;
        int nbr[4], nxt[4];
        const int tb = it.unit * chunk;
#pragma unroll
        for (int s = 0; s < 4; ++s)
            nbr[s] = (pre && s < S.nxf && tb < t1) ? S.xnbrf[(size_t)s * S.np16 + tb * RES_TILE + c] : -1;
        for (int t = tb; t < t1; ++t) {
#pragma unroll
            for (int s = 0; s < 4; ++s)
                nxt[s] = (pre && s < S.nxf && t + 1 < t1)
                             ? S.xnbrf[(size_t)s * S.np16 + (t + 1) * RES_TILE + c] : -1;
            ok = full_resid_pos_body(S.nxf, S.np16, S.Dp, S.XF, S.xnbrf, S.rhsp, S.Up, S.R32,
                                     S.partials, S.Dinv32, S.b32, S.c32, status, t, bar, parity,
                                     pre ? nbr : nullptr);
            parity ^= 1u;
            if (!ok) break;
#pragma unroll
            for (int s = 0; s < 4; ++s) nbr[s] = nxt[s];
            __syncthreads(); /* the next tile's copies overwrite the stages */
        }
    }
}

template <typename T>
int launch_resid_group(cudaStream_t st, int max_nx, const ResidSys<T> *sys, const int *gunits, int chunk,
                       const int *active, unsigned *status) {
    const size_t smem = resid_smem_bytes<T>(max_nx);
    const int grid = resid_batch_grid(smem, (const void *)fast_resid_group_kernel<T>);
    fast_resid_group_kernel<T><<<grid, RES_THREADS_FAST, smem, st>>>(sys, gunits, chunk, active, status);
    return (int)cudaGetLastError();
}
template int launch_resid_group<double>(cudaStream_t, int, const ResidSys<double> *, const int *, int,
                                        const int *, unsigned *);

int launch_full_resid_pos_batch(cudaStream_t st, int max_nxf, const FullPosSys *sys,
                                const int *groups, int chunk, const int *active, unsigned *status) {
    const size_t smem = fullpos_smem_bytes(max_nxf);
    const int grid = resid_batch_grid(smem, (const void *)full_resid_pos_batch_kernel);
    full_resid_pos_batch_kernel<<<grid, RES_THREADS_FAST, smem, st>>>(sys, groups, chunk, active,
                                                                      status);
    return (int)cudaGetLastError();
}

/* One CTA per descriptor (grid = capacity; CTAs beyond *nred only take
 * their ticket).  The last CTA to finish decides whether the graph's loop
 * goes on: some member is active, the sweep limit of the launch is not
 * reached and, when asked, no member stopped during the launch. */
__global__ void batch_reduce_kernel(const ReduceSys *__restrict__ sys, const int *__restrict__ nred_p,
                                    int is_start, int *active, BatchCtl *ctl, unsigned *counter,
                                    cudaGraphConditionalHandle handle, int use_cond,
                                    cudaGraphConditionalHandle handle2, int use2) {
    __shared__ double red[32];
    __shared__ unsigned ticket;
    const int s = blockIdx.x;
    if (s < *nred_p) {
        const ReduceSys R = sys[s];
        const int m = R.member;
        if (is_start || active[m]) {
            double acc = strided_sum(R.partials, R.n, (int)blockDim.x);
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(FULL, acc, o);
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
            __syncthreads();
            if (threadIdx.x == 0) {
                double tot = 0.0;
                for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) tot += red[w];
                const double nrm = sqrt(tot);
                SolveState *S = R.state;
                if (is_start) {
                    S->sweep = 0;
                    S->norm0 = nrm;
                } else {
                    S->sweep += 1;
                }
                const int sw = S->sweep;
                if (sw < S->hist_cap) R.hist[sw] = nrm;
                S->last = nrm;
                const bool go = isfinite(nrm) && nrm > S->tol * S->norm0 && sw < S->max_sweeps;
                active[m] = go ? 1 : 0;
                if (!go) ctl->finished = 1;
            }
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        ticket = atomicAdd(counter, 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0 && ticket == gridDim.x - 1) {
        __threadfence();
        int any = 0;
        const int n = ctl->nsys;
        for (int k = 0; k < n; ++k) any |= __ldcg(active + k);
        bool go = any != 0;
        if (!is_start && ctl->chunk_limit > 0) {
            ctl->chunk += 1;
            if (ctl->chunk >= ctl->chunk_limit) go = false;
        }
        if (ctl->stop_on_finish && __ldcg(&ctl->finished)) go = false;
        if (use_cond) cudaGraphSetConditional(handle, go ? 1u : 0u);
        if (use2) cudaGraphSetConditional(handle2, go ? 1u : 0u);
        *counter = 0u;
    }
}

int launch_reduce_batch(cudaStream_t st, int threads, const ReduceSys *sys, const int *nred,
                        int cap, int is_start, int *active, BatchCtl *ctl, unsigned *counter,
                        unsigned long long cond_handle, int use_cond,
                        unsigned long long cond_handle2, int use2) {
    if (cap <= 0) return 0;
    if (threads != RES_THREADS_FAST && threads != REDUCE_THREADS) return (int)cudaErrorInvalidValue;
    batch_reduce_kernel<<<cap, threads, 0, st>>>(sys, nred, is_start, active, ctl, counter,
                                                 (cudaGraphConditionalHandle)cond_handle, use_cond,
                                                 (cudaGraphConditionalHandle)cond_handle2, use2);
    return (int)cudaGetLastError();
}

/* opt the batched kernels into the shared memory of the widest member
 * (outside stream capture) */
int batch_prepare(int max_nx) {
    int rc = set_smem((const void *)fast_resid_batch_kernel<double, 1>, resid_smem_bytes<double>(max_nx));
    if (!rc)
        rc = set_smem((const void *)fast_resid_batch_kernel<double, BATCH_CHUNK>,
                      resid_smem_bytes<double>(max_nx));
    if (!rc)
        rc = set_smem((const void *)fast_resid_batch_kernel<float, 1>, resid_smem_bytes<float>(max_nx));
    if (!rc)
        rc = set_smem((const void *)fast_resid_batch_kernel<float, BATCH_CHUNK>,
                      resid_smem_bytes<float>(max_nx));
    if (!rc)
        rc = set_smem((const void *)fast_resid_group_kernel<double>, resid_smem_bytes<double>(max_nx));

    if (!rc) rc = set_smem((const void *)full_resid_pos_batch_kernel, fullpos_smem_bytes(4));
    return rc;
}

int fullpos_prepare(const FastLayout &L) {
    return set_smem((const void *)full_resid_pos_kernel, fullpos_smem_bytes(L.nxf));
}

template size_t thomas_batch_smem<double>(int, int);
template size_t thomas_batch_smem<float>(int, int);
template int thomas_batch_fit<double>(int, int);
template int thomas_batch_fit<float>(int, int);
template int launch_thomas_batch<double>(cudaStream_t, const BatchSched &, const ThomasSys<double> *,
                                         const WorkItem *, const int *, const int *, unsigned *,
                                         unsigned *);
template int launch_thomas_batch<float>(cudaStream_t, const BatchSched &, const ThomasSys<float> *,
                                        const WorkItem *, const int *, const int *, unsigned *,
                                        unsigned *);
template int launch_resid_batch<double>(cudaStream_t, int, int, const ResidSys<double> *,
                                        const int *, int, const int *, unsigned *);
template int launch_resid_batch<float>(cudaStream_t, int, int, const ResidSys<float> *,
                                       const int *, int, const int *, unsigned *);


/* ============================================== several right-hand sides
 * nr <= MULTI_MAX right-hand sides of one factored system swept together
 * (TBS_ALGO_FP64): the line blocks (G, Gam, Dinv, X) are read once per
 * sweep for all of them.  Vectors are RHS-major: right-hand side r of a
 * vector v starts at v + r * vs, vs = np16 * 9.  A right-hand side whose
 * solve has ended (active[r] == 0) is skipped by every kernel, so its
 * solution stays the one of its last sweep, and the per-element arithmetic
 * is the single-system kernels' own: every right-hand side's iterates,
 * norms and sweep count are bit-identical to a solve of it alone. */

/* Forward / backward chunk steps of thomas_line's chains for MULTI_RPW
 * right-hand sides at once: the row of G (Gam) is loaded once per step and
 * feeds one dot product per right-hand side, each with row_dot's own
 * expression, so every right-hand side's values are those of fwd_chunk /
 * bwd_chunk.  Right-hand side j reads its b chunk at sB[j], publishes its
 * vector through bc[j] and writes y (dU) through yg[j] (dUl[j]); only the
 * first `nown` of them write. */
constexpr int MULTI_RPW = 2;

template <int P, bool CHECK>
__device__ __forceinline__ void fwd_chunk_m(const double *sG, const double *const *sB,
                                            double *const *bc, double *const *yg, int nown,
                                            int kbase, int len, int cpos, int i,
                                            const LaneOff &o) {
    RowD cur_row, next_row;
    load_row(cur_row, sG, o, 0);
    double cur_b[MULTI_RPW], next_b[MULTI_RPW];
#pragma unroll
    for (int j = 0; j < MULTI_RPW; ++j) cur_b[j] = sB[j][i];
#pragma unroll
    for (int q = 0; q < P; ++q) {
        const int odd = q & 1;
#pragma unroll
        for (int j = 0; j < MULTI_RPW; ++j) next_b[j] = 0.0;
        if (q + 1 < P) {
            load_row(next_row, sG + (q + 1) * NB, o, odd ^ 1);
#pragma unroll
            for (int j = 0; j < MULTI_RPW; ++j) next_b[j] = sB[j][(q + 1) * NV + i];
        }
        double yi[MULTI_RPW];
#pragma unroll
        for (int j = 0; j < MULTI_RPW; ++j) yi[j] = row_dot(cur_row, bc[j] + odd * 20, o, odd, cur_b[j]);
        /* lanes 9..15 repeat lane 8's row, value and address: no divergence */
        if (!CHECK || kbase + q < len) {
            const int pos = cpos + kbase + q;
#pragma unroll
            for (int j = 0; j < MULTI_RPW; ++j) {
                if (j < nown) {
                    double *nxt = bc[j] + (odd ^ 1) * 20;
                    nxt[i] = yi[j];
                    nxt[11 + i] = yi[j];
                    yg[j][(size_t)pos * NV + i] = yi[j];
                }
            }
        }
        __syncwarp();
        cur_row = next_row;
#pragma unroll
        for (int j = 0; j < MULTI_RPW; ++j) cur_b[j] = next_b[j];
    }
}

template <int P, bool CHECK>
__device__ __forceinline__ void bwd_chunk_m(const double *sG, double *const *bc,
                                            const double (*yv)[P], double *const *dUl, int nown,
                                            int kbase, int len, int cpos, int i,
                                            const LaneOff &o) {
    RowD cur_row, next_row;
    load_row(cur_row, sG + (P - 1) * NB, o, (P - 1) & 1);
#pragma unroll
    for (int q = P - 1; q >= 0; --q) {
        const int odd = q & 1;
        if (q > 0) load_row(next_row, sG + (q - 1) * NB, o, odd ^ 1);
        const int f = (P - 1 - q) & 1;
        const bool valid = !CHECK || (kbase + q >= 0 && kbase + q < len);
        const int pos = cpos + kbase + q;
        double d[MULTI_RPW];
#pragma unroll
        for (int j = 0; j < MULTI_RPW; ++j)
            d[j] = row_dot(cur_row, bc[j] + f * 20, o, odd, valid ? yv[j][q] : 0.0);
        if (valid) { /* lanes 9..15 repeat lane 8's row, value and address */
#pragma unroll
            for (int j = 0; j < MULTI_RPW; ++j) {
                if (j < nown) {
                    double *nxt = bc[j] + (f ^ 1) * 20;
                    nxt[i] = d[j];
                    nxt[11 + i] = d[j];
                    dUl[j][(size_t)pos * NV + i] = d[j];
                }
            }
        }
        __syncwarp();
        cur_row = next_row;
    }
}

/* Thomas: one CTA per line; warp w solves the active right-hand sides
 * 2w and 2w+1 (in active order) with the chains of thomas_line (y in
 * global memory).  Thread 0 streams the jobs through an NS-stage ring; a
 * forward stage holds, for either chain, a chunk of G rows followed by the
 * chunks of b of the active right-hand sides, a backward stage a chunk of
 * Gam rows.  All warps have consumed a stage before it is refilled (one
 * CTA barrier per chunk). */
template <int P>
__device__ __forceinline__ void multi_thomas_line(const MultiLine &S, int l, int NS,
                                                  const int *__restrict__ active, unsigned *status) {
    using T = double;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned amask_s;
    __shared__ int rid[MULTI_MAX];
    /* the right-hand sides' vectors, indexed by slot */
    __shared__ const T *sbp[MULTI_MAX];
    __shared__ T *syp[MULTI_MAX], *sdp[MULTI_MAX];
    const int nr = S.nr;
    const int *__restrict__ line_start = S.line_start;
    const int *__restrict__ line_len = S.line_len;
    const int *__restrict__ line_twist = S.line_twist;
    const T *__restrict__ G = S.G;
    const T *__restrict__ Gam = S.Gam;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    if (tid == 0) {
        unsigned am = 0;
        int k = 0;
#pragma unroll
        for (int r = 0; r < MULTI_MAX; ++r) {
            sbp[r] = S.b[r];
            syp[r] = S.y[r];
            sdp[r] = S.dU[r];
            if (r < nr && active[S.aid[r]]) {
                am |= 1u << r;
                rid[k++] = r;
            }
        }
        amask_s = am;
        for (int s = 0; s < NS; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    const unsigned amask = amask_s;
    if (amask == 0u) return;
    const int nact = __popc(amask);
    const int k0 = w * MULTI_RPW;                  /* this warp's first active slot */
    const int nown = max(0, min(MULTI_RPW, nact - k0));
    const bool mine = nown > 0;
    const uint32_t halfb = P * (NB + nr * NV) * sizeof(T);
    const uint32_t stage = 2 * halfb;
    unsigned char *st0 = smem + 128;
    T *bcw = reinterpret_cast<T *>(st0 + (size_t)NS * stage) + w * MULTI_RPW * 80;
    const int ps = line_start[l], n = line_len[l], m = line_twist[l];
    const int h = lane >> 4, li = lane & 15;
    const int i = li < NV ? li : NV - 1;
    const LaneOff off = lane_offsets(i);
    const int nb = n - 1 - m;
    const int len = h ? nb : m;
    const int cpos = h ? m : 0;
    const int nchT = (m + P - 1) / P, nchB = (nb + P - 1) / P;
    const int nch = h ? nchB : nchT;
    const int nf = nchT > nchB ? nchT : nchB;
    const int njobs = 2 * nf;
    /* per owned right-hand side: its broadcast buffers (this half), y, dU
     * and b (slots beyond nown alias slot 0 and never write) */
    T *bc[MULTI_RPW], *yl[MULTI_RPW], *dUl[MULTI_RPW];
    const T *bg[MULTI_RPW];
    int slot[MULTI_RPW];
#pragma unroll
    for (int j = 0; j < MULTI_RPW; ++j) {
        const int jj = j < nown ? j : 0;
        slot[j] = mine ? k0 + jj : 0;
        const int rr = mine ? rid[k0 + jj] : 0;
        bc[j] = bcw + j * 80 + h * 40;
        yl[j] = syp[rr] + (size_t)ps * NV;
        dUl[j] = sdp[rr] + (size_t)ps * NV;
        bg[j] = sbp[rr] + (size_t)ps * NV;
    }
    const uint64_t pol = tid == 0 ? policy_evict_first() : 0;
    for (int t = lane; t < MULTI_RPW * 80; t += 32) bcw[t] = T(0);
    __syncwarp();

    auto cells = [&](int ln, int c) { return ((min(P, ln - c * P) + 3) & ~3); };
    auto issue = [&](int job, int s) {
        unsigned char *base = st0 + (size_t)s * stage;
        uint32_t bytes = 0;
        if (job < nf) {
            if (job < nchT) bytes += cells(m, job) * (NB + nact * NV) * sizeof(T);
            if (job < nchB) bytes += cells(nb, job) * (NB + nact * NV) * sizeof(T);
        } else {
            const int jb = job - nf;
            if (nchT - 1 - jb >= 0) bytes += cells(m, nchT - 1 - jb) * NB * sizeof(T);
            if (nchB - 1 - jb >= 0) bytes += cells(nb, nchB - 1 - jb) * NB * sizeof(T);
        }
        mbar_arrive_expect_tx(&bars[s], bytes);
        for (int hh = 0; hh < 2; ++hh) {
            const int ln = hh ? nb : m, nc = hh ? nchB : nchT, cp = hh ? m : 0;
            unsigned char *hb = base + hh * halfb;
            if (job < nf) {
                const int c = job;
                if (c >= nc) continue;
                const int cnt = cells(ln, c);
                const size_t p = (size_t)(ps + cp + c * P);
                bulk_g2s_hint(hb, G + p * NB, cnt * NB * sizeof(T), &bars[s], pol);
                for (int k = 0; k < nact; ++k)
                    bulk_g2s(hb + (size_t)(P * NB + k * P * NV) * sizeof(T), sbp[rid[k]] + p * NV,
                             cnt * NV * sizeof(T), &bars[s]);
            } else {
                const int c = nc - 1 - (job - nf);
                if (c < 0) continue;
                const int cnt = cells(ln, c);
                bulk_g2s_hint(hb, Gam + (size_t)(ps + cp + c * P) * NB, cnt * NB * sizeof(T),
                              &bars[s], pol);
            }
        }
    };
    int issued = 0;
    if (tid == 0) {
        for (; issued < NS && issued < njobs; ++issued) issue(issued, issued);
    }
    int consumed = 0;
    bool timed_out = false;
    const int both_full = (m < nb ? m : nb) / P;

    /* ---------------- forward */
    for (int c = 0; c < nf; ++c) {
        const int s = c % NS;
        const bool ok = __all_sync(FULL, mbar_wait(&bars[s], (uint32_t)(c / NS) & 1u));
        if (ok && mine) {
            const T *sG = reinterpret_cast<const T *>(st0 + (size_t)s * stage + h * halfb);
            const T *sB[MULTI_RPW];
#pragma unroll
            for (int j = 0; j < MULTI_RPW; ++j) sB[j] = sG + P * NB + slot[j] * P * NV;
            if (c < both_full)
                fwd_chunk_m<P, false>(sG, sB, bc, yl, nown, c * P, len, cpos, i, off);
            else
                fwd_chunk_m<P, true>(sG, sB, bc, yl, nown, c * P, len, cpos, i, off);
            __syncwarp();
        }
        if (__syncthreads_or(!ok)) {
            timed_out = true;
            break;
        }
        ++consumed;
        if (tid == 0 && issued < njobs) {
            issue(issued, s);
            ++issued;
        }
    }

    if (!timed_out) {
        /* ---------------- twist: x_m = b_m - G_tw y_top - Gam_tw y_bot */
        const int ptw = n - 1;
        T xm[MULTI_RPW];
#pragma unroll
        for (int j = 0; j < MULTI_RPW; ++j) xm[j] = T(0);
        if (mine && lane < NV) {
            const T *gr = G + (size_t)(ps + ptw) * NB + NV * lane;
            const T *cr = Gam + (size_t)(ps + ptw) * NB + NV * lane;
#pragma unroll
            for (int j = 0; j < MULTI_RPW; ++j) {
                const T *base = bcw + j * 80;
                const T *ytop = base + 0 * 40 + (m & 1) * 20;
                const T *ybot = base + 1 * 40 + (nb & 1) * 20;
                T acc = bg[j][(size_t)ptw * NV + lane];
#pragma unroll
                for (int jj = 0; jj < NV; ++jj) acc -= gr[jj] * ytop[jj] + cr[jj] * ybot[jj];
                xm[j] = acc;
            }
        }
        __syncwarp();
        if (mine && lane < NV) {
#pragma unroll
            for (int j = 0; j < MULTI_RPW; ++j) {
                if (j < nown) {
                    T *base = bcw + j * 80;
                    for (int t = 0; t < 4; ++t) {
                        base[t * 20 + lane] = xm[j];
                        base[t * 20 + 11 + lane] = xm[j];
                    }
                    dUl[j][(size_t)ptw * NV + lane] = xm[j];
                }
            }
        }
        __syncwarp();

        /* ---------------- backward */
        T yv[MULTI_RPW][P], nyv[MULTI_RPW][P];
        auto load_chunk = [&](int c, T (*yy)[P]) {
#pragma unroll
            for (int j = 0; j < MULTI_RPW; ++j)
#pragma unroll
                for (int q = 0; q < P; ++q) {
                    const int k = c * P + q;
                    yy[j][q] = T(0);
                    if (j < nown && c >= 0 && k < len) /* lanes 9..15: lane 8's values */
                        yy[j][q] = yl[j][(size_t)(cpos + k) * NV + i];
                }
        };
        load_chunk(nch - 1, yv);
        for (int jb = 0; jb < nf; ++jb) {
            const int job = nf + jb;
            const int c = nch - 1 - jb;
            load_chunk(c - 1, nyv);
            const int s = job % NS;
            const bool ok = __all_sync(FULL, mbar_wait(&bars[s], (uint32_t)(job / NS) & 1u));
            if (ok && mine) {
                const T *sG = reinterpret_cast<const T *>(st0 + (size_t)s * stage + h * halfb);
                const bool full = (nchT - 1 - jb) * P + P <= m && (nchB - 1 - jb) * P + P <= nb &&
                                  nchT - 1 - jb >= 0 && nchB - 1 - jb >= 0;
                if (full)
                    bwd_chunk_m<P, false>(sG, bc, yv, dUl, nown, c * P, len, cpos, i, off);
                else
                    bwd_chunk_m<P, true>(sG, bc, yv, dUl, nown, c * P, len, cpos, i, off);
                __syncwarp();
            }
            if (__syncthreads_or(!ok)) {
                timed_out = true;
                break;
            }
            ++consumed;
            if (tid == 0 && issued < njobs) {
                issue(issued, s);
                ++issued;
            }
#pragma unroll
            for (int j = 0; j < MULTI_RPW; ++j)
#pragma unroll
                for (int q = 0; q < P; ++q) yv[j][q] = nyv[j][q];
        }
    }
    if (timed_out && tid == 0) {
        atomicOr(status, ST_TIMEOUT);
        for (int job = consumed; job < issued; ++job)
            mbar_wait(&bars[job % NS], (uint32_t)(job / NS) & 1u, 1LL << 28);
    }
}

/* one line of one system per CTA: the context's solve (tbs_solve_multi) */
template <int P>
__global__ void __launch_bounds__(32 * MULTI_MAX / MULTI_RPW) multi_thomas_kernel(
    int nline, int NS, MultiLine S, const int *__restrict__ active, unsigned *status) {
    if ((int)blockIdx.x >= nline) return;
    multi_thomas_line<P>(S, blockIdx.x, NS, active, status);
}

/* the batch engine: item k = (group of one system's members, line) */
template <int P>
__global__ void __launch_bounds__(32 * MULTI_MAX / MULTI_RPW) multi_thomas_items_kernel(
    const MultiLine *__restrict__ sys, const WorkItem *__restrict__ items, const int *__restrict__ nitems,
    int NS, const int *__restrict__ active, unsigned *status) {
    if ((int)blockIdx.x >= *nitems) return;
    const WorkItem it = items[blockIdx.x];
    multi_thomas_line<P>(sys[it.sys], it.unit, NS, active, status);
}

static int multi_thomas_warps(int nr) { return (nr + MULTI_RPW - 1) / MULTI_RPW; }

static size_t multi_thomas_stage(int nr) {
    return 2 * (size_t)THOMAS_P * (NB + nr * NV) * sizeof(double);
}

static size_t multi_thomas_smem(int nr, int NS) {
    return 128 + (size_t)NS * multi_thomas_stage(nr) +
           (size_t)multi_thomas_warps(nr) * MULTI_RPW * 80 * sizeof(double);
}

/* ring depth: the shared memory each of the SM's resident lines may use,
 * at least 3 and at most 8 stages */
static int multi_thomas_ns(const FastLayout &L, int nr) {
    int dev = 0, nsm = 148, smem_sm = 228 * 1024, reserved = 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    if (nsm < 1) nsm = 148;
    int per_sm = (L.nline + nsm - 1) / nsm;
    const int by_threads = 2048 / (32 * multi_thomas_warps(nr));
    if (per_sm > by_threads) per_sm = by_threads;
    if (per_sm < 1) per_sm = 1;
    const long long budget = (long long)smem_sm / per_sm - reserved - (long long)multi_thomas_smem(nr, 0);
    long long ns = budget / (long long)multi_thomas_stage(nr);
    if (ns > 8) ns = 8;
    if (ns < 3) ns = 3;
    return (int)ns;
}

int launch_multi_thomas(cudaStream_t st, const FastLayout &L, int nr, const double *G,
                        const double *Gam, const double *b, double *y, double *dU,
                        const int *active, unsigned *status) {
    if (L.nv != NV || nr < 1 || nr > MULTI_MAX) return (int)cudaErrorInvalidValue;
    const int NS = multi_thomas_ns(L, nr);
    const long long vs = (long long)L.np16 * NV;
    MultiLine S{};
    S.line_start = L.line_start;
    S.line_len = L.line_len;
    S.line_twist = L.line_twist;
    S.G = G;
    S.Gam = Gam;
    S.nr = nr;
    for (int r = 0; r < MULTI_MAX; ++r) {
        const int rr = r < nr ? r : 0;
        S.aid[r] = rr;
        S.b[r] = b + (size_t)rr * vs;
        S.y[r] = y + (size_t)rr * vs;
        S.dU[r] = dU + (size_t)rr * vs;
    }
    multi_thomas_kernel<THOMAS_P><<<L.nline, 32 * multi_thomas_warps(nr), multi_thomas_smem(nr, NS), st>>>(
        L.nline, NS, S, active, status);
    return (int)cudaGetLastError();
}

/* ring depth of the engine's multi-RHS line solves (their shared memory
 * is sized for MULTI_MAX right-hand sides) */
constexpr int MULTI_ITEMS_NS = 3;

int multi_items_prepare() {
    return set_smem((const void *)multi_thomas_items_kernel<THOMAS_P>,
                    multi_thomas_smem(MULTI_MAX, MULTI_ITEMS_NS));
}

int launch_multi_thomas_items(cudaStream_t st, int grid, const MultiLine *sys, const WorkItem *items,
                              const int *nitems, const int *active, unsigned *status) {
    if (grid < 1) return 0;
    multi_thomas_items_kernel<THOMAS_P>
        <<<grid, 32 * multi_thomas_warps(MULTI_MAX), multi_thomas_smem(MULTI_MAX, MULTI_ITEMS_NS), st>>>(
            sys, items, nitems, MULTI_ITEMS_NS, active, status);
    return (int)cudaGetLastError();
}

/* Residual of several right-hand sides per tile: Dinv and the cross-line
 * blocks are staged once, then for every active right-hand side r
 *   mode 0 (the start):  R = Rsrc_r (staged), U_r = 0
 *   mode 1 (a sweep):    R = sum X dU_r (gathers of all r issued together),
 *                        U_r += dU_r
 * followed by b_r = -Dinv R and the tile's sum R^2 for r, each with the
 * expressions (and summation order) of fast_resid_body.  The last CTA to
 * finish adds every active r's partials in tile order (finalize_total's
 * order), records the norms, retires the right-hand sides whose solve has
 * ended and keeps the graph's loop running while any is active. */
static size_t multi_resid_smem(int nx, int nr) {
    const int nxa = nx > 0 ? nx : 1;
    return 128 + (size_t)RES_TILE * NB * sizeof(double) * (1 + nx) +
           (size_t)nr * nxa * RES_TILE * NV * sizeof(double) +
           (size_t)nr * RES_TILE * NV * sizeof(double);
}

template <int MODE>
__global__ void __launch_bounds__(RES_THREADS_FAST) multi_resid_kernel(
    MultiSys M, const double *__restrict__ Dinv, const double *__restrict__ X,
    const int *__restrict__ xnbr, const double *__restrict__ Rsrc, unsigned long long handle,
    int use_cond, unsigned *status) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned amask_s, ticket;
    __shared__ double red[MULTI_MAX][RES_THREADS_FAST / 32];
    const int tid = threadIdx.x;
    const int nx = MODE == 1 ? M.nx : 0;
    const int nxa = nx > 0 ? nx : 1;
    const int nr = M.nr;
    const long long vs = (long long)M.np16 * NV;
    const int ntiles = M.np16 / RES_TILE;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    double *sD = reinterpret_cast<double *>(smem + 128);
    double *sX = sD + RES_TILE * NB;
    double *sg = sX + nx * RES_TILE * NB; /* [k][s][c][i] gathers; mode 0: [k][c][i] R */
    double *sr = sg + (size_t)nr * nxa * RES_TILE * NV; /* [k][c][i] R, then b */
    __shared__ int rid[MULTI_MAX]; /* the k-th active right-hand side */
    if (tid == 0) {
        unsigned am = 0;
        int k = 0;
        for (int r = 0; r < nr; ++r)
            if (MODE == 0 || M.active[r]) {
                am |= 1u << r;
                rid[k++] = r;
            }
        amask_s = am;
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    const unsigned amask = amask_s;
    const int nact = __popc(amask);
    const int c = tid % RES_TILE, i = tid / RES_TILE;
    const bool act = tid < RES_TILE * NV;
    const uint32_t szD = RES_TILE * NB * sizeof(double), szR = RES_TILE * NV * sizeof(double);
    uint32_t parity = 0;
    bool failed = false;
    /* the neighbour indices of the CTA's next tile load during the current one */
    int pnbr[MULTI_NX];
#pragma unroll
    for (int s = 0; s < MULTI_NX; ++s)
        pnbr[s] = (MODE == 1 && act && s < nx && (int)blockIdx.x < ntiles)
                      ? __ldg(xnbr + (size_t)s * M.np16 + blockIdx.x * RES_TILE + c) : -1;
    for (int blk = blockIdx.x; blk < ntiles && nact > 0; blk += gridDim.x) {
        const int p0 = blk * RES_TILE;
        const int bn = blk + gridDim.x;
        int pnxt[MULTI_NX];
#pragma unroll
        for (int s = 0; s < MULTI_NX; ++s)
            pnxt[s] = (MODE == 1 && act && s < nx && bn < ntiles)
                          ? __ldg(xnbr + (size_t)s * M.np16 + bn * RES_TILE + c) : -1;
        if (tid == 0) {
            const uint64_t pol = policy_evict_first();
            mbar_arrive_expect_tx(bar, szD + (MODE == 1 ? nx * szD : nact * szR));
            bulk_g2s_hint(sD, Dinv + (size_t)p0 * NB, szD, bar, pol);
            if (MODE == 1) {
                for (int s = 0; s < nx; ++s)
                    bulk_g2s_hint(sX + s * RES_TILE * NB, X + ((size_t)s * M.np16 + p0) * NB, szD,
                                  bar, pol);
            } else {
                int k = 0;
                for (int r = 0; r < nr; ++r) {
                    if (!((amask >> r) & 1u)) continue;
                    bulk_g2s(sg + (size_t)k * RES_TILE * NV, Rsrc + (size_t)r * vs + (size_t)p0 * NV,
                             szR, bar);
                    ++k;
                }
            }
        }
        if (act) {
            const size_t q = (size_t)p0 * NV + tid;
            if (MODE == 1) {
                /* every load of the tile (the neighbour dU gathers, U and dU
                 * of each active r) is issued before the first store, so
                 * that their latencies overlap */
                int nbr[MULTI_NX];
#pragma unroll
                for (int s = 0; s < MULTI_NX; ++s) nbr[s] = pnbr[s];
                double gv[MULTI_MAX][MULTI_NX], uv[MULTI_MAX], dv[MULTI_MAX];
#pragma unroll
                for (int k = 0; k < MULTI_MAX; ++k) {
                    uv[k] = dv[k] = 0.0;
#pragma unroll
                    for (int s = 0; s < MULTI_NX; ++s) gv[k][s] = 0.0;
                    if (k < nact) {
                        const size_t ro = (size_t)rid[k] * vs;
#pragma unroll
                        for (int s = 0; s < MULTI_NX; ++s)
                            if (nbr[s] >= 0) gv[k][s] = __ldg(M.dU + ro + (size_t)nbr[s] * NV + i);
                        uv[k] = M.U[ro + q];
                        dv[k] = __ldg(M.dU + ro + q);
                    }
                }
#pragma unroll
                for (int k = 0; k < MULTI_MAX; ++k) {
                    if (k < nact) {
#pragma unroll
                        for (int s = 0; s < MULTI_NX; ++s)
                            if (s < nx) sg[((size_t)(k * nx + s) * RES_TILE + c) * NV + i] = gv[k][s];
                        M.U[(size_t)rid[k] * vs + q] = uv[k] + dv[k];
                    }
                }
            } else {
                for (int k = 0; k < nact; ++k) M.U[(size_t)rid[k] * vs + q] = 0.0;
            }
        }
        const bool ok = mbar_wait(bar, parity);
        parity ^= 1u;
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicOr(status, ST_TIMEOUT);
                mbar_wait(bar, parity ^ 1u, 1LL << 28);
            }
            failed = true;
            break;
        }
        /* R for every active r: the row of each slot's block is read once
         * and feeds every r; per r the products are added in
         * fast_resid_body's order (slots ascending, three accumulators) */
        double sq[MULTI_MAX];
#pragma unroll
        for (int k = 0; k < MULTI_MAX; ++k) sq[k] = 0.0;
        if (act) {
            if (MODE == 1) {
                double a0[MULTI_MAX], a1[MULTI_MAX], a2[MULTI_MAX];
#pragma unroll
                for (int k = 0; k < MULTI_MAX; ++k) a0[k] = a1[k] = a2[k] = 0.0;
                for (int s = 0; s < nx; ++s) {
                    const double *xr = sX + (s * RES_TILE + c) * NB + i;
                    double x[NV];
#pragma unroll
                    for (int j = 0; j < NV; ++j) x[j] = xr[9 * j];
#pragma unroll
                    for (int k = 0; k < MULTI_MAX; ++k) {
                        if (k < nact) {
                            const double *g = sg + ((size_t)(k * nx + s) * RES_TILE + c) * NV;
                            a0[k] += x[0] * g[0];
                            a1[k] += x[1] * g[1];
                            a2[k] += x[2] * g[2];
                            a0[k] += x[3] * g[3];
                            a1[k] += x[4] * g[4];
                            a2[k] += x[5] * g[5];
                            a0[k] += x[6] * g[6];
                            a1[k] += x[7] * g[7];
                            a2[k] += x[8] * g[8];
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < MULTI_MAX; ++k) {
                    if (k < nact) {
                        const double rr = a0[k] + (a1[k] + a2[k]);
                        sr[(size_t)k * RES_TILE * NV + c * NV + i] = rr;
                        sq[k] = rr * rr;
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < MULTI_MAX; ++k) {
                    if (k < nact) {
                        const double rr = sg[(size_t)k * RES_TILE * NV + c * NV + i];
                        sq[k] = rr * rr;
                    }
                }
            }
        }
        __syncthreads();
        /* b = -Dinv R for every active r (into sg, free now); the row of
         * Dinv is read once */
        const double *rsrc = MODE == 1 ? sr : sg;
        double *sb = MODE == 1 ? sg : sr;
        if (act) {
            const double *drow = sD + c * NB + i;
            double dr[NV];
#pragma unroll
            for (int j = 0; j < NV; ++j) dr[j] = drow[9 * j];
#pragma unroll
            for (int k = 0; k < MULTI_MAX; ++k) {
                if (k < nact) {
                    const double *rv = rsrc + (size_t)k * RES_TILE * NV + c * NV;
                    double a0 = dr[0] * rv[0], a1 = dr[1] * rv[1], a2 = dr[2] * rv[2];
                    a0 += dr[3] * rv[3];
                    a1 += dr[4] * rv[4];
                    a2 += dr[5] * rv[5];
                    a0 += dr[6] * rv[6];
                    a1 += dr[7] * rv[7];
                    a2 += dr[8] * rv[8];
                    sb[(size_t)k * RES_TILE * NV + c * NV + i] = -(a0 + (a1 + a2));
                }
            }
        }
        __syncthreads();
        if (act) {
            int k = 0;
            for (int r = 0; r < nr; ++r) {
                if (!((amask >> r) & 1u)) continue;
                M.b[(size_t)r * vs + (size_t)p0 * NV + tid] = sb[(size_t)k * RES_TILE * NV + tid];
                ++k;
            }
        }
        /* the tile's sum R^2 per r, in fast_resid_body's order */
#pragma unroll
        for (int k = 0; k < MULTI_MAX; ++k) {
            if (k < nact) {
                double v = sq[k];
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
                if ((tid & 31) == 0) red[k][tid >> 5] = v;
            }
        }
        __syncthreads();
        if (tid == 0) {
            int k = 0;
            for (int r = 0; r < nr; ++r) {
                if (!((amask >> r) & 1u)) continue;
                double tot = 0.0;
                for (int w = 0; w < RES_THREADS_FAST / 32; ++w) tot += red[k][w];
                M.partials[(size_t)r * ntiles + blk] = tot;
                ++k;
            }
        }
#pragma unroll
        for (int s = 0; s < MULTI_NX; ++s) pnbr[s] = pnxt[s];
        __syncthreads(); /* the next tile's copies overwrite the stages */
    }
    (void)failed;

    /* ---------------- the last CTA: norms of every active r */
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        ticket = atomicAdd(M.counter, 1u);
    }
    __syncthreads();
    if (ticket != gridDim.x - 1) return;
    __threadfence();
    __shared__ int any_go;
    if (tid == 0) any_go = 0;
    for (int r = 0; r < nr; ++r) {
        if (!((amask >> r) & 1u)) continue;
        double acc = strided_sum(M.partials + (size_t)r * ntiles, ntiles, (int)blockDim.x);
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(FULL, acc, o);
        __syncthreads(); /* red[0] of the previous r is read */
        if ((tid & 31) == 0) red[0][tid >> 5] = acc;
        __syncthreads();
        if (tid == 0) {
            double tot = 0.0;
            for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) tot += red[0][w];
            const double nrm = sqrt(tot);
            SolveState *S = M.state + r;
            if (MODE == 0) {
                S->sweep = 0;
                S->norm0 = nrm;
            } else {
                S->sweep += 1;
            }
            const int sw = S->sweep;
            if (sw < S->hist_cap) M.hist[(size_t)r * M.hist_stride + sw] = nrm;
            S->last = nrm;
            const bool go = isfinite(nrm) && nrm > S->tol * S->norm0 && sw < S->max_sweeps;
            M.active[r] = go ? 1 : 0;
            if (go) any_go = 1;
        }
    }
    __syncthreads();
    if (tid == 0) {
        if (use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)handle, any_go ? 1u : 0u);
        *M.counter = 0u;
    }
}

int launch_multi_resid(cudaStream_t st, const FastLayout &L, int mode, const MultiSys &M,
                       const double *Dinv, const double *X, const double *Rsrc,
                       unsigned long long cond_handle, int use_cond, unsigned *status) {
    if (L.nv != NV || M.nr < 1 || M.nr > MULTI_MAX || (mode != 0 && mode != 1))
        return (int)cudaErrorInvalidValue;
    const int ntiles = L.np16 / RES_TILE;
    if (mode == 1) {
        const size_t smem = multi_resid_smem(L.nx, M.nr);
        multi_resid_kernel<1><<<resid_grid_persistent((const void *)multi_resid_kernel<1>, smem, ntiles),
                                RES_THREADS_FAST, smem, st>>>(M, Dinv, X, L.xnbr, nullptr,
                                                              cond_handle, use_cond, status);
    } else {
        const size_t smem = multi_resid_smem(0, M.nr);
        multi_resid_kernel<0><<<resid_grid_persistent((const void *)multi_resid_kernel<0>, smem, ntiles),
                                RES_THREADS_FAST, smem, st>>>(M, Dinv, nullptr, nullptr, Rsrc,
                                                              cond_handle, use_cond, status);
    }
    return (int)cudaGetLastError();
}

/* opt the multi-RHS kernels into the shared memory of nr right-hand sides
 * (outside stream capture) */
int multi_prepare(const FastLayout &L, int nr) {
    if (nr < 1 || nr > MULTI_MAX) return (int)cudaErrorInvalidValue;
    int rc = set_smem((const void *)multi_thomas_kernel<THOMAS_P>,
                      multi_thomas_smem(nr, multi_thomas_ns(L, nr)));
    if (!rc) rc = set_smem((const void *)multi_resid_kernel<1>, multi_resid_smem(L.nx, nr));
    if (!rc) rc = set_smem((const void *)multi_resid_kernel<0>, multi_resid_smem(0, nr));
    return rc;
}


/* ================================================ point-implicit Jacobi
 * TBS_ALGO_PIJ: the sweep dU = -D^-1 R, U += dU, R = rhs + J U with the
 * diagonal block alone as the implicit operator (every cell its own
 * line).  As for the line form, D dU = -R makes the new residual
 * R + J dU = sum over the interior faces of offJ dU_nbr, so one sweep is
 * one streaming launch of the residual kernel over the position-ordered
 * face blocks (slot s = the s-th interior face of the cell in ef order):
 *     U += dU;  R = sum_s XF_s dU_nbr(s);  b = -Dinv R  (= the next dU)
 * with dU and b in two buffers that swap every sweep.  The buffer parity
 * lives in SolveState::pad, flipped by the launch's last CTA, so graph and
 * eager sweep sequences agree on where the latest update is. */

/* Dinv = D^-1 per position, in place (Gauss-Jordan without pivoting, as
 * the reference's LU has none); pads stay zero.  One warp per position. */
__global__ void __launch_bounds__(32) pij_invert_kernel(int np16, const int *__restrict__ elem_of_pos,
                                                        double *__restrict__ D, unsigned *status) {
    const int j = threadIdx.x;
    for (int p = blockIdx.x; p < np16; p += gridDim.x) {
        if (elem_of_pos[p] < 0) continue;
        double w[NV];
        double *blk = D + (size_t)p * NB;
#pragma unroll
        for (int i = 0; i < NV; ++i) w[i] = j < NV ? blk[NV * j + i] : (i == j ? 1.0 : 0.0);
        gj_invert_cols(w, j, status);
        if (j < NV) {
#pragma unroll
            for (int i = 0; i < NV; ++i) blk[NV * j + i] = w[i];
        }
        __syncwarp();
    }
}

int launch_pij_invert(cudaStream_t st, const FastLayout &L, double *D, unsigned *status) {
    const int grid = L.np16 < 148 * 32 ? (L.np16 > 0 ? L.np16 : 1) : 148 * 32;
    pij_invert_kernel<<<grid, 32, 0, st>>>(L.np16, L.elem_of_pos, D, status);
    return (int)cudaGetLastError();
}

__global__ void __launch_bounds__(RES_THREADS_FAST) pij_sweep_kernel(
    int nxf, int np16, const double *__restrict__ Dinv, const double *__restrict__ XF,
    const int *__restrict__ xnbrf, double *bufA, double *bufB, double *__restrict__ Up,
    NormSink ns, unsigned *status) {
    /* read before any CTA can finish: the last CTA flips it after every
     * CTA has taken its ticket */
    const int odd = ns.state->pad & 1;
    const double *dU = odd ? bufB : bufA;
    double *b = odd ? bufA : bufB;
    const bool last = resid_tiles<double>(nxf, np16, 1, Dinv, XF, xnbrf, dU, nullptr, b, Up, ns, status);
    if (last && threadIdx.x == 0) ns.state->pad = odd ^ 1;
}

int launch_pij_sweep(cudaStream_t st, const FastLayout &L, const double *Dinv, const double *XF,
                     double *bufA, double *bufB, double *Up, const NormSink &ns, unsigned *status) {
    /* nxf == 0 (no interior faces): no slot is read and R_new = 0 */
    if (L.nv != NV || L.nxf > 4 || !ns.state || !ns.partials) return (int)cudaErrorInvalidValue;
    const size_t smem = resid_smem_bytes<double>(L.nxf);
    pij_sweep_kernel<<<resid_grid_persistent((const void *)pij_sweep_kernel, smem, L.np16 / RES_TILE),
                       RES_THREADS_FAST, smem, st>>>(L.nxf, L.np16, Dinv, XF, L.xnbrf, bufA, bufB, Up,
                                                     ns, status);
    return (int)cudaGetLastError();
}

int pij_prepare(const FastLayout &L) {
    return set_smem((const void *)pij_sweep_kernel, resid_smem_bytes<double>(L.nxf));
}


/* =============================================== bounded-wait self-test
 * One thread arms an mbarrier for 16 bytes that no copy will deliver (no
 * copy is issued) and waits on it with the given clock budget, the wait
 * every staging pipeline uses: it must give up, and the status bit it then
 * records is the one the kernels record on a stalled copy. */
__global__ void selftest_timeout_kernel(long long budget, unsigned *status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    mbar_fence_init();
    mbar_arrive_expect_tx(&bar, 16);
    if (!mbar_wait(&bar, 0, budget)) atomicOr(status, ST_TIMEOUT);
}

int launch_selftest_timeout(cudaStream_t st, long long budget_cycles, unsigned *status) {
    if (budget_cycles < 0) return (int)cudaErrorInvalidValue;
    selftest_timeout_kernel<<<1, 32, 0, st>>>(budget_cycles, status);
    return (int)cudaGetLastError();
}

}  // namespace tbs

/*
 * kernels_ref.cu -- TBS_ALGO_REFERENCE: the reference's arithmetic, in its
 * operation order, on the GPU.  Built with -fmad=false so that every
 * multiply and add rounds separately, exactly like the CPU oracle built with
 * -ffp-contract=off; U, dU and R then agree bit for bit.
 *
 *   ref_line_lu      src/okl/lineLU_v2.okl:58-182 (LU 17-27, solveLU 30-52)
 *   ref_assemble_A   src/Jacobian.cxx:76-117 (done on the device here)
 *   ref_solve_du     src/okl/linesmoothLU_TriBlock_v3.okl:92-226
 *   ref_add_copy     src/okl/linesmoothLU_v5.okl:75-103 (addAtoB + copyAtoB)
 *   ref_line_res     src/okl/linesmoothLU_TriBlock_v3.okl:228-336
 *
 * Parallel decomposition differs from the reference (one warp per line,
 * rows spread over lanes; one thread per (element,row) for the residual)
 * but each scalar is produced by the same sequence of roundings: rows of
 * the Doolittle update are independent once the pivot row is final, the
 * nv columns of D'^-1 C are independent solves, and every dot product is
 * summed from 0.0 in ascending j as in the OKL loops.
 */
#include "tbs_internal.hxx"

#include <cuda_runtime.h>

namespace tbs {

constexpr int REF_MAXNV = 32;

#define MIDX(i, j, nv) ((i) + (nv) * (j))

/* x = (LU)^-1 b for one lane; A in shared memory, column-major.
 * lineLU_v2.okl:30-52 / linesmoothLU_TriBlock_v3.okl:23-45 */
template <int NV>
__device__ __forceinline__ void solve_lu_lane(const double *A, const double *b, double *x,
                                              int nv_rt) {
    const int nv = NV ? NV : nv_rt;
    double y[NV ? NV : REF_MAXNV];
#pragma unroll
    for (int i = 0; i < nv; ++i) {
        double tot = 0.0;
#pragma unroll
        for (int j = 0; j < i; ++j) tot += A[MIDX(i, j, nv)] * y[j];
        y[i] = b[i] - tot;
    }
#pragma unroll
    for (int i = nv - 1; i >= 0; --i) {
        double tot = 0.0;
#pragma unroll
        for (int j = i + 1; j < nv; ++j) tot += A[MIDX(i, j, nv)] * x[j];
        x[i] = (y[i] - tot) / A[MIDX(i, i, nv)];
    }
}

/* In-place no-pivot Doolittle on a shared-memory block, rows over lanes.
 * Row j is final when step j starts and only rows i > j change in it, so
 * lane i applying its own row's updates reproduces lineLU_v2.okl:17-27. */
template <int NV>
__device__ __forceinline__ void lu_rows(double *A, int lane, int nv_rt, unsigned *status) {
    const int nv = NV ? NV : nv_rt;
    for (int j = 0; j < nv; ++j) {
        __syncwarp();
        const double ajj = A[MIDX(j, j, nv)];
        if (lane == 0 && !(fabs(ajj) > 0.0 && isfinite(ajj))) atomicOr(status, ST_PIVOT);
        const double pivot = 1.0 / ajj;
        if (lane > j && lane < nv) {
            const double lij = A[MIDX(lane, j, nv)] * pivot;
            A[MIDX(lane, j, nv)] = lij;
            for (int k = j + 1; k < nv; ++k) A[MIDX(lane, k, nv)] -= lij * A[MIDX(j, k, nv)];
        }
    }
    __syncwarp();
}

template <int NV>
__global__ void __launch_bounds__(32) ref_line_lu_kernel(
    int nv_rt, int nline, const int *__restrict__ fc, const int *__restrict__ linesize,
    const int *__restrict__ linepoint, const int *__restrict__ lines,
    const int *__restrict__ lineface, double *__restrict__ Dia, const double *__restrict__ O1,
    const double *__restrict__ O2, double *__restrict__ DinvC, unsigned *status) {
    const int nv = NV ? NV : nv_rt;
    const int l = blockIdx.x;
    if (l >= nline) return;
    const int lane = threadIdx.x;
    const size_t bs = (size_t)nv * nv;
    extern __shared__ double sm[];
    double *sGamma = sm;
    double *sC = sGamma + bs;
    double *sAT = sC + bs;
    double *sDe = sAT + bs;
    double *sDl = sDe + bs;

    const int n = linesize[l];
    const int m0 = linepoint[l];
    int e = lines[m0];
    if (lane < nv)
        for (int j = 0; j < nv; ++j) sDe[MIDX(lane, j, nv)] = Dia[MIDX(lane, j, nv) + bs * e];
    lu_rows<NV>(sDe, lane, nv, status);
    if (lane < nv)
        for (int j = 0; j < nv; ++j) Dia[MIDX(lane, j, nv) + bs * e] = sDe[MIDX(lane, j, nv)];

    for (int k = 1; k < n; ++k) {
        const int m = m0 + k;
        const int elast = e;
        e = lines[m];
        const int f = lineface[m];
        const int e1 = fc[2 * f];
        const double *A = (e == e1) ? O2 : O1;
        const double *C = (e == e1) ? O1 : O2;
        __syncwarp();
        if (lane < nv) {
            for (int j = 0; j < nv; ++j) {
                /* D'_{k-1} is the block factored in the previous step; the
                 * reference re-reads it from global memory, same bits */
                sDl[MIDX(lane, j, nv)] = sDe[MIDX(lane, j, nv)];
            }
        }
        __syncwarp();
        if (lane < nv) {
            for (int j = 0; j < nv; ++j) {
                sC[MIDX(lane, j, nv)] = C[MIDX(lane, j, nv) + bs * f];
                sAT[MIDX(j, lane, nv)] = A[MIDX(lane, j, nv) + bs * f];
                sDe[MIDX(lane, j, nv)] = Dia[MIDX(lane, j, nv) + bs * e];
            }
        }
        __syncwarp();
        /* Gamma(:,i) = D'_{k-1}^-1 C(:,i)  (lineLU_v2.okl:142-144) */
        if (lane < nv) solve_lu_lane<NV>(sDl, &sC[MIDX(0, lane, nv)], &sGamma[MIDX(0, lane, nv)], nv);
        __syncwarp();
        /* D_k - A_k Gamma  (lineLU_v2.okl:147-161) */
        if (lane < nv) {
            for (int kk = 0; kk < nv; ++kk) {
                double tot = 0.0;
                for (int j = 0; j < nv; ++j) tot += sAT[MIDX(j, lane, nv)] * sGamma[MIDX(j, kk, nv)];
                sDe[MIDX(lane, kk, nv)] -= tot;
            }
        }
        lu_rows<NV>(sDe, lane, nv, status);
        if (lane < nv) {
            for (int j = 0; j < nv; ++j) {
                Dia[MIDX(lane, j, nv) + bs * e] = sDe[MIDX(lane, j, nv)];
                DinvC[MIDX(lane, j, nv) + bs * elast] = sGamma[MIDX(lane, j, nv)];
            }
        }
    }
}

int launch_ref_line_lu(cudaStream_t st, int nv, int nline, const int *fc, const int *linesize,
                       const int *linepoint, const int *lines, const int *lineface, double *DLU,
                       const double *O1, const double *O2, double *DinvC, unsigned *status) {
    if (nv < 1 || nv > REF_MAXNV) return (int)cudaErrorInvalidValue;
    const size_t smem = 5 * (size_t)nv * nv * sizeof(double);
    if (nv == 9) {
        ref_line_lu_kernel<9><<<nline, 32, smem, st>>>(nv, nline, fc, linesize, linepoint, lines,
                                                       lineface, DLU, O1, O2, DinvC, status);
    } else {
        if (smem > 48 * 1024) {
            const int e = smem_raise((const void *)ref_line_lu_kernel<0>, smem);
            if (e != 0) return e;
        }
        ref_line_lu_kernel<0><<<nline, 32, smem, st>>>(nv, nline, fc, linesize, linepoint, lines,
                                                       lineface, DLU, O1, O2, DinvC, status);
    }
    return (int)cudaGetLastError();
}

/* Jacobian.cxx:76-117: A[e] = (e == fc[2f]) ? O2[f] : O1[f], f = lineface[m],
 * for every line cell after the first.  One warp per line cell. */
__global__ void ref_assemble_A_kernel(int nv, int nline, const int *__restrict__ fc,
                                      const int *__restrict__ linesize,
                                      const int *__restrict__ linepoint,
                                      const int *__restrict__ lines,
                                      const int *__restrict__ lineface,
                                      const double *__restrict__ O1,
                                      const double *__restrict__ O2, double *__restrict__ A) {
    const int l = blockIdx.x;
    if (l >= nline) return;
    const size_t bs = (size_t)nv * nv;
    const int n = linesize[l];
    for (int k = 1 + threadIdx.y; k < n; k += blockDim.y) {
        const int m = linepoint[l] + k;
        const int f = lineface[m];
        const int e = lines[m];
        const double *src = (e == fc[2 * f]) ? &O2[bs * f] : &O1[bs * f];
        for (int t = threadIdx.x; t < (int)bs; t += 32) A[bs * e + t] = src[t];
    }
}

int launch_ref_assemble_A(cudaStream_t st, int nv, int nline, const int *fc, const int *linesize,
                          const int *linepoint, const int *lines, const int *lineface,
                          const double *O1, const double *O2, double *A) {
    ref_assemble_A_kernel<<<nline, dim3(32, 8), 0, st>>>(nv, nline, fc, linesize, linepoint, lines,
                                                         lineface, O1, O2, A);
    return (int)cudaGetLastError();
}

/* linesmoothLU_TriBlock_v3.okl:92-226.  Lane 0 runs solveLU as the
 * reference does (its `if(i==0)` guard, :154/:192); the other lanes do the
 * row-parallel matvecs and prefetch the next cell's blocks meanwhile. */
template <int NV>
__global__ void __launch_bounds__(32) ref_solve_du_kernel(
    int nv_rt, int nline, const int *__restrict__ linesize, const int *__restrict__ linepoint,
    const int *__restrict__ lines, const double *__restrict__ Dia,
    const double *__restrict__ DinvC, const double *__restrict__ A, double *__restrict__ dU,
    const double *__restrict__ R) {
    const int nv = NV ? NV : nv_rt;
    const int l = blockIdx.x;
    if (l >= nline) return;
    const int lane = threadIdx.x;
    const size_t bs = (size_t)nv * nv;
    extern __shared__ double sm[];
    double *sDia = sm;
    double *sAT = sDia + bs;
    double *sS = sAT + bs;
    double *sdU = sS + REF_MAXNV;

    const int n = linesize[l];
    const int m0 = linepoint[l];
    int e = lines[m0];
    if (lane < nv) {
        sS[lane] = -R[lane + (size_t)nv * e];
        for (int j = 0; j < nv; ++j) sDia[MIDX(lane, j, nv)] = Dia[MIDX(lane, j, nv) + bs * e];
    }
    __syncwarp();
    if (lane == 0) solve_lu_lane<NV>(sDia, sS, sdU, nv);
    __syncwarp();
    if (lane < nv) dU[lane + (size_t)nv * e] = sdU[lane];

    for (int k = 1; k < n; ++k) {
        e = lines[m0 + k];
        __syncwarp();
        if (lane < nv) {
            for (int j = 0; j < nv; ++j) {
                sAT[MIDX(j, lane, nv)] = A[MIDX(lane, j, nv) + bs * e];
                sDia[MIDX(lane, j, nv)] = Dia[MIDX(lane, j, nv) + bs * e];
            }
        }
        __syncwarp();
        if (lane < nv) {
            double tot = 0.0;
            for (int j = 0; j < nv; ++j) tot += sAT[MIDX(j, lane, nv)] * sdU[j];
            sS[lane] = -R[lane + (size_t)nv * e] - tot;
        }
        __syncwarp();
        if (lane == 0) solve_lu_lane<NV>(sDia, sS, sdU, nv);
        __syncwarp();
        if (lane < nv) dU[lane + (size_t)nv * e] = sdU[lane];
    }
    /* back substitution: dU_k -= DinvC_k dU_{k+1}; sdU holds dU of the
     * last cell, the value the reference reloads from global memory */
    for (int k = n - 2; k >= 0; --k) {
        e = lines[m0 + k];
        double mine = 0.0;
        if (lane < nv) {
            double tot = 0.0;
            for (int j = 0; j < nv; ++j) tot += DinvC[MIDX(lane, j, nv) + bs * e] * sdU[j];
            mine = dU[lane + (size_t)nv * e] - tot;
            dU[lane + (size_t)nv * e] = mine;
        }
        __syncwarp();
        if (lane < nv) sdU[lane] = mine;
        __syncwarp();
    }
}

int launch_ref_solve_du(cudaStream_t st, int nv, int nline, const int *linesize,
                        const int *linepoint, const int *lines, const double *DLU,
                        const double *DinvC, const double *A, double *dU, const double *R) {
    if (nv < 1 || nv > REF_MAXNV) return (int)cudaErrorInvalidValue;
    const size_t smem = (2 * (size_t)nv * nv + 2 * REF_MAXNV) * sizeof(double);
    if (nv == 9) {
        ref_solve_du_kernel<9><<<nline, 32, smem, st>>>(nv, nline, linesize, linepoint, lines, DLU,
                                                        DinvC, A, dU, R);
    } else {
        ref_solve_du_kernel<0><<<nline, 32, smem, st>>>(nv, nline, linesize, linepoint, lines, DLU,
                                                        DinvC, A, dU, R);
    }
    return (int)cudaGetLastError();
}

/* addAtoB (U += dU) and copyAtoB (R = rhs), linesmoothLU_v5.okl:75-103 */
__global__ void ref_add_copy_kernel(long long n, const double *__restrict__ dU,
                                    double *__restrict__ U, const double *__restrict__ rhs,
                                    double *__restrict__ R) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        U[t] += dU[t];
        R[t] = rhs[t];
    }
}

int launch_ref_add_copy(cudaStream_t st, long long n, const double *dU, double *U,
                        const double *rhs, double *R) {
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    ref_add_copy_kernel<<<(int)blocks, 256, 0, st>>>(n, dU, U, rhs, R);
    return (int)cudaGetLastError();
}

/* linesmoothLU_TriBlock_v3.okl:228-336, one thread per (element, row):
 * R(i,e) += [D U](i) + sum over faces in ef order of [offJ U_nbr](i).
 * Each block also writes the sum of R^2 over its entries (fixed-order tree)
 * for the residual norm the reference does not compute. */
constexpr int RES_THREADS = 288;

__global__ void __launch_bounds__(RES_THREADS) ref_line_res_kernel(
    int nv, int nelem, const int *__restrict__ epoint, const int *__restrict__ ef,
    const int *__restrict__ fc, const double *__restrict__ D, const double *__restrict__ O1,
    const double *__restrict__ O2, const double *__restrict__ U, double *__restrict__ R,
    double *__restrict__ partials) {
    const int epb = RES_THREADS / nv;
    const int le = threadIdx.x / nv;
    const int i = threadIdx.x - le * nv;
    const int e = blockIdx.x * epb + le;
    const size_t bs = (size_t)nv * nv;
    double sq = 0.0;
    if (le < epb && e < nelem) {
        double tot = 0.0;
        for (int j = 0; j < nv; ++j) tot += D[MIDX(i, j, nv) + bs * e] * U[j + (size_t)nv * e];
        double sR = tot;
        for (int k2 = epoint[e]; k2 < epoint[e + 1]; ++k2) {
            const int f = ef[k2];
            if (f >= 0) {
                const int e1 = fc[2 * f + 0];
                const int e2 = fc[2 * f + 1];
                const double *offJ = (e == e1) ? O2 : O1;
                const int nb = (e == e1) ? e2 : e1;
                double t2 = 0.0;
                for (int j = 0; j < nv; ++j) t2 += offJ[MIDX(i, j, nv) + bs * f] * U[j + (size_t)nv * nb];
                sR += t2;
            }
        }
        const double r = R[i + (size_t)nv * e] + sR;
        R[i + (size_t)nv * e] = r;
        sq = r * r;
    }
    /* deterministic block sum */
    __shared__ double red[RES_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < RES_THREADS / 32; ++w) s += red[w];
        partials[blockIdx.x] = s;
    }
}

int ref_line_res_partials(int nelem) { return (nelem + 31) / 32; }

int launch_ref_line_res(cudaStream_t st, int nv, int nline, int nelem, const int *epoint,
                        const int *ef, const int *fc, const int *linesize, const int *linepoint,
                        const int *lines, const double *D, const double *O1, const double *O2,
                        const double *U, double *R, double *partials, int *npartials_out) {
    (void)nline;
    (void)linesize;
    (void)linepoint;
    (void)lines;
    if (nv < 1 || nv > REF_MAXNV) return (int)cudaErrorInvalidValue;
    const int epb = RES_THREADS / nv;
    const int blocks = (nelem + epb - 1) / epb;
    if (npartials_out) *npartials_out = blocks;
    ref_line_res_kernel<<<blocks, RES_THREADS, 0, st>>>(nv, nelem, epoint, ef, fc, D, O1, O2, U, R,
                                                        partials);
    return (int)cudaGetLastError();
}

}  // namespace tbs

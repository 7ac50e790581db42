/*
 * lij_oracle.c -- CPU restatement of the reference's line-implicit Jacobi
 * (LIJ) path, run with "OCCA Serial" semantics (every @inner loop a plain
 * loop, @barrier a no-op).  TEST INFRASTRUCTURE: only the tests, the smoke
 * check and the CPU-baseline / reference arm of bench.py load this file's
 * library, and only as the results the GPU is compared against or as the
 * timed CPU baseline.  The product (libtriblock.so) never calls it.
 *
 * Parity status: the arithmetic is unpinned by reference outputs.  The
 * reference's kernels are OKL and need the OCCA translator (an empty,
 * unpinned submodule), MPI and gfortran to build, none of which exists
 * here, and the reference ships no golden vectors.  What is pinned: the
 * mesh format and numbering (the structured generator reproduces
 * data/ex05/gpuline.mesh.data.bin bit for bit) and the Jacobian layout
 * (size formula matches the data/ex06 LFS pointer).
 *
 * Operation order follows the reference exactly (no FMA contraction: build
 * with -ffp-contract=off), so that the GPU path compiled the same way
 * (TBS_ALGO_REFERENCE) can be compared bit for bit:
 *   lu_inplace            src/okl/lineLU_v2.okl:17-27
 *   solve_lu              src/okl/lineLU_v2.okl:30-52
 *                         (= src/okl/linesmoothLU_TriBlock_v3.okl:23-45)
 *   oracle_assemble_A     src/Jacobian.cxx:76-117
 *   oracle_line_lu        src/okl/lineLU_v2.okl:58-182 (after copyAtoBjac,
 *                         src/okl/linesmoothLU_v5.okl:85-93)
 *   oracle_solve_du       src/okl/linesmoothLU_TriBlock_v3.okl:92-226
 *   oracle_line_res       src/okl/linesmoothLU_TriBlock_v3.okl:228-336
 *   oracle_factor         src/main.cxx:90,180-190 (A packing, copy, lineLU)
 *   oracle_sweeps         src/main.cxx:207-229 (solveDU, U += dU, R = rhs,
 *                         R += J U), plus the per-sweep residual norm the
 *                         reference never prints
 *   oracle_lij            both, from U = 0 (src/main.cxx:180-229)
 *   oracle_resize_block_size  src/Jacobian.cxx:153-238
 * Block (i,j) of block b is at i + nv*j + nv*nv*b (OKL @dim, column-major).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXNV 64
#define M(A, i, j, nv) (A)[(size_t)(i) + (size_t)(nv) * (size_t)(j)]

static int g_threads = 1;

void oracle_set_threads(int n) { g_threads = n > 0 ? n : 1; }

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* lineLU_v2.okl:17-27: in-place Doolittle, unit L, multiply by 1/pivot */
static void lu_inplace(double *A, int nv) {
    for (int j = 0; j < nv; ++j) {
        double pivot = 1.0 / M(A, j, j, nv);
        for (int i = j + 1; i < nv; ++i) {
            M(A, i, j, nv) = M(A, i, j, nv) * pivot;
            for (int k = j + 1; k < nv; ++k) {
                M(A, i, k, nv) -= M(A, i, j, nv) * M(A, j, k, nv);
            }
        }
    }
}

/* lineLU_v2.okl:30-52: x = (LU)^-1 b */
static void solve_lu(const double *A, const double *b, double *x, int nv) {
    double y[MAXNV];
    for (int i = 0; i < nv; ++i) {
        double tot = 0.0;
        for (int j = 0; j < i; ++j) tot += M(A, i, j, nv) * y[j];
        y[i] = b[i] - tot;
    }
    for (int i = nv - 1; i >= 0; --i) {
        double tot = 0.0;
        for (int j = i + 1; j < nv; ++j) tot += M(A, i, j, nv) * x[j];
        x[i] = (y[i] - tot) / M(A, i, i, nv);
    }
}

/* Jacobian.cxx:76-117: A[e] = in-line lower block of row e (k >= 1) */
void oracle_assemble_A(int nv, int nline, const int *fc, const int *linesize,
                       const int *linepoint, const int *lines, const int *lineface,
                       const double *O1, const double *O2, double *A) {
    const size_t bs = (size_t)nv * nv;
    for (int l = 0; l < nline; ++l) {
        for (int k = 1; k < linesize[l]; ++k) {
            int m = linepoint[l] + k;
            int f = lineface[m];
            int e = lines[m];
            int e1 = fc[2 * f];
            const double *src = (e == e1) ? &O2[bs * f] : &O1[bs * f];
            memcpy(&A[bs * e], src, bs * sizeof(double));
        }
    }
}

/* lineLU_v2.okl:58-182 on one line.  Dia holds jacD on entry (copyAtoBjac)
 * and the packed L\U of D' on exit; DinvC[elast] = D'^-1 C. */
static void line_lu_one(int nv, int l, const int *fc, const int *linesize,
                        const int *linepoint, const int *lines, const int *lineface,
                        double *Dia, const double *O1, const double *O2, double *DinvC) {
    const size_t bs = (size_t)nv * nv;
    double Gamma[MAXNV * MAXNV], Alpha[MAXNV * MAXNV], sC[MAXNV * MAXNV];
    double sAT[MAXNV * MAXNV], sDe[MAXNV * MAXNV], sDl[MAXNV * MAXNV];
    const int n = linesize[l];
    const int m0 = linepoint[l];
    lu_inplace(&Dia[bs * lines[m0]], nv);
    for (int k = 1; k < n; ++k) {
        int m = m0 + k;
        int e = lines[m];
        const int f = lineface[m];
        int e1 = fc[2 * f];
        const int elast = lines[m0 + k - 1];
        const double *A = (e == e1) ? O2 : O1;
        const double *C = (e == e1) ? O1 : O2;
        for (int i = 0; i < nv; ++i) {
            for (int j = 0; j < nv; ++j) M(sC, i, j, nv) = C[i + nv * j + bs * f];
            for (int j = 0; j < nv; ++j) M(sAT, j, i, nv) = A[i + nv * j + bs * f];
            for (int j = 0; j < nv; ++j) M(sDl, i, j, nv) = Dia[i + nv * j + bs * elast];
            for (int j = 0; j < nv; ++j) M(sDe, i, j, nv) = Dia[i + nv * j + bs * e];
        }
        for (int i = 0; i < nv; ++i) solve_lu(sDl, &M(sC, 0, i, nv), &M(Gamma, 0, i, nv), nv);
        for (int i = 0; i < nv; ++i) {
            for (int kk = 0; kk < nv; ++kk) {
                double tot = 0.0;
                for (int j = 0; j < nv; ++j) tot += M(sAT, j, i, nv) * M(Gamma, j, kk, nv);
                M(Alpha, i, kk, nv) = tot;
            }
        }
        for (int i = 0; i < nv; ++i)
            for (int j = 0; j < nv; ++j) M(sDe, i, j, nv) -= M(Alpha, i, j, nv);
        lu_inplace(sDe, nv);
        for (int i = 0; i < nv; ++i) {
            for (int j = 0; j < nv; ++j) Dia[i + nv * j + bs * e] = M(sDe, i, j, nv);
            for (int j = 0; j < nv; ++j) DinvC[i + nv * j + bs * elast] = M(Gamma, i, j, nv);
        }
    }
}

void oracle_line_lu(int nv, int nline, const int *fc, const int *linesize,
                    const int *linepoint, const int *lines, const int *lineface, double *Dia,
                    const double *O1, const double *O2, double *DinvC) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads)
    for (int l = 0; l < nline; ++l)
        line_lu_one(nv, l, fc, linesize, linepoint, lines, lineface, Dia, O1, O2, DinvC);
}

/* linesmoothLU_TriBlock_v3.okl:92-226 on one line */
static void solve_du_one(int nv, int l, const int *linesize, const int *linepoint,
                         const int *lines, const double *Dia, const double *DinvC,
                         const double *A, double *dU, const double *R) {
    const size_t bs = (size_t)nv * nv;
    double S[MAXNV], x[MAXNV], dUe[MAXNV];
    double sAT[MAXNV * MAXNV], sDia[MAXNV * MAXNV], sDCT[MAXNV * MAXNV];
    const int n = linesize[l];
    const int m0 = linepoint[l];
    const int e0 = lines[m0];
    for (int i = 0; i < nv; ++i) {
        S[i] = -R[i + (size_t)nv * e0];
        for (int j = 0; j < nv; ++j) M(sDia, i, j, nv) = Dia[i + nv * j + bs * e0];
    }
    solve_lu(sDia, S, dUe, nv);
    for (int i = 0; i < nv; ++i) dU[i + (size_t)nv * e0] = dUe[i];
    for (int k = 1; k < n; ++k) {
        const int e = lines[m0 + k];
        for (int i = 0; i < nv; ++i) {
            for (int j = 0; j < nv; ++j) M(sAT, j, i, nv) = A[i + nv * j + bs * e];
            for (int j = 0; j < nv; ++j) M(sDia, i, j, nv) = Dia[i + nv * j + bs * e];
        }
        for (int i = 0; i < nv; ++i) {
            double tot = 0.0;
            for (int j = 0; j < nv; ++j) tot += M(sAT, j, i, nv) * dUe[j];
            x[i] = tot;
        }
        for (int i = 0; i < nv; ++i) S[i] = -R[i + (size_t)nv * e] - x[i];
        solve_lu(sDia, S, dUe, nv);
        for (int i = 0; i < nv; ++i) dU[i + (size_t)nv * e] = dUe[i];
    }
    for (int k = n - 2; k >= 0; --k) {
        const int e = lines[m0 + k];
        const int elast = lines[m0 + k + 1];
        for (int i = 0; i < nv; ++i) {
            for (int j = 0; j < nv; ++j) M(sDCT, j, i, nv) = DinvC[i + nv * j + bs * e];
            dUe[i] = dU[i + (size_t)nv * elast];
        }
        for (int i = 0; i < nv; ++i) {
            double tot = 0.0;
            for (int j = 0; j < nv; ++j) tot += M(sDCT, j, i, nv) * dUe[j];
            dU[i + (size_t)nv * e] -= tot;
        }
    }
}

void oracle_solve_du(int nv, int nline, const int *linesize, const int *linepoint,
                     const int *lines, const double *Dia, const double *DinvC, const double *A,
                     double *dU, const double *R) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads)
    for (int l = 0; l < nline; ++l)
        solve_du_one(nv, l, linesize, linepoint, lines, Dia, DinvC, A, dU, R);
}

/* linesmoothLU_TriBlock_v3.okl:228-336 for element e: R(e) += D U + sum O U */
static void line_res_elem(int nv, int e, const int *epoint, const int *ef, const int *fc,
                          const double *D, const double *O1, const double *O2, const double *U,
                          double *R) {
    const size_t bs = (size_t)nv * nv;
    double sR[MAXNV];
    for (int i = 0; i < nv; ++i) {
        double tot = 0.0;
        for (int j = 0; j < nv; ++j) tot += D[i + nv * j + bs * e] * U[j + (size_t)nv * e];
        sR[i] = tot;
    }
    for (int k2 = epoint[e]; k2 < epoint[e + 1]; ++k2) {
        const int f = ef[k2];
        if (f >= 0) {
            int e1 = fc[2 * f + 0];
            int e2 = fc[2 * f + 1];
            const double *offJ = (e == e1) ? O2 : O1;
            const int nb = (e == e1) ? e2 : e1;
            for (int i = 0; i < nv; ++i) {
                double tot = 0.0;
                for (int j = 0; j < nv; ++j) tot += offJ[i + nv * j + bs * f] * U[j + (size_t)nv * nb];
                sR[i] += tot;
            }
        }
    }
    for (int i = 0; i < nv; ++i) R[i + (size_t)nv * e] += sR[i];
}

void oracle_line_res(int nv, int nline, const int *epoint, const int *ef, const int *fc,
                     const int *linesize, const int *linepoint, const int *lines, const double *D,
                     const double *O1, const double *O2, const double *U, double *R) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads)
    for (int l = 0; l < nline; ++l)
        for (int k = 0; k < linesize[l]; ++k)
            line_res_elem(nv, lines[linepoint[l] + k], epoint, ef, fc, D, O1, O2, U, R);
}

double oracle_norm(const double *R, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += R[i] * R[i];
    return sqrt(s);
}

/* Setup phase of main.cxx:90 and :180-190: A packing, jacDLU = jacD,
 * lineLU.  DLU, DinvC, A are nv*nv*nelem each (zeroed here). */
int oracle_factor(int nv, int nelem, int nline, const int *fc, const int *linesize,
                  const int *linepoint, const int *lines, const int *lineface, const double *jacD,
                  const double *O1, const double *O2, double *DLU, double *DinvC, double *A) {
    if (nv < 1 || nv > MAXNV) return 1;
    const size_t bs = (size_t)nv * nv;
    memcpy(DLU, jacD, bs * nelem * sizeof(double));
    memset(DinvC, 0, bs * nelem * sizeof(double));
    memset(A, 0, bs * nelem * sizeof(double));
    oracle_assemble_A(nv, nline, fc, linesize, linepoint, lines, lineface, O1, O2, A);
    oracle_line_lu(nv, nline, fc, linesize, linepoint, lines, lineface, DLU, O1, O2, DinvC);
    return 0;
}

/* n sweeps of main.cxx:207-229 from the state (U, R); hist[p] (may be
 * NULL) receives ||R|| after sweep p. */
int oracle_sweeps(int nv, int nelem, int nline, const int *epoint, const int *ef, const int *fc,
                  const int *linesize, const int *linepoint, const int *lines, const double *jacD,
                  const double *O1, const double *O2, const double *rhs, const double *DLU,
                  const double *DinvC, const double *A, double *U, double *R, double *dU, int n,
                  double *hist) {
    const size_t nvec = (size_t)nv * nelem;
    for (int p = 0; p < n; ++p) {
        oracle_solve_du(nv, nline, linesize, linepoint, lines, DLU, DinvC, A, dU, R);
#pragma omp parallel for schedule(static) num_threads(g_threads)
        for (long long i = 0; i < (long long)nvec; ++i) {
            U[i] += dU[i];
            R[i] = rhs[i];
        }
        oracle_line_res(nv, nline, epoint, ef, fc, linesize, linepoint, lines, jacD, O1, O2, U, R);
        if (hist) hist[p] = oracle_norm(R, nvec);
    }
    return 0;
}

/* Whole reference flow (main.cxx:180-229) for `iters` sweeps from U = 0.
 * hist (iters+1 entries) gets ||R|| before the first sweep and after each.
 * Outputs U, R, dU (nv*nelem) and the factors (may be NULL). */
int oracle_lij(int nv, int nelem, int nintface, int nline, const int *epoint, const int *ef,
               const int *fc, const int *linesize, const int *linepoint, const int *lines,
               const int *lineface, const double *jacD, const double *O1, const double *O2,
               const double *rhs, int iters, double *U, double *R, double *dU, double *hist,
               double *jacDLU_out, double *DinvC_out) {
    if (nv < 1 || nv > MAXNV) return 1;
    const size_t bs = (size_t)nv * nv, nvec = (size_t)nv * nelem;
    (void)nintface;
    double *DLU = jacDLU_out ? jacDLU_out : (double *)malloc(bs * nelem * sizeof(double));
    double *DinvC = DinvC_out ? DinvC_out : (double *)malloc(bs * nelem * sizeof(double));
    double *A = (double *)malloc(bs * nelem * sizeof(double));
    if (!DLU || !DinvC || !A) return 2;
    oracle_factor(nv, nelem, nline, fc, linesize, linepoint, lines, lineface, jacD, O1, O2, DLU,
                  DinvC, A);
    memset(U, 0, nvec * sizeof(double));
    memset(dU, 0, nvec * sizeof(double));
    memcpy(R, rhs, nvec * sizeof(double));
    if (hist) hist[0] = oracle_norm(R, nvec);
    oracle_sweeps(nv, nelem, nline, epoint, ef, fc, linesize, linepoint, lines, jacD, O1, O2, rhs,
                  DLU, DinvC, A, U, R, dU, iters, hist ? hist + 1 : NULL);
    if (!jacDLU_out) free(DLU);
    if (!DinvC_out) free(DinvC);
    free(A);
    return 0;
}

/* Jacobian.cxx:153-238, including its quirks: the "clear" loops iterate
 * over copies (no effect), so std::vector::resize keeps the old flat
 * contents in the leading entries; diagonals of D, O1, O2 are then set to
 * 10.0 and the old min(nv)-square sub-blocks copied in; rhs and U0 copy
 * their first nelem*min_nv entries flat.  Arrays are sized by the caller
 * for nv_new; the *_old arrays hold the nv_old data. */
void oracle_resize_block_size(int nv_old, int nv_new, int nelem, int nintface,
                              const double *D_old, const double *O1_old, const double *O2_old,
                              const double *rhs_old, const double *U0_old, double *D,
                              double *O1, double *O2, double *rhs, double *U0) {
    const size_t bo = (size_t)nv_old * nv_old, bn = (size_t)nv_new * nv_new;
    const int mn = nv_new < nv_old ? nv_new : nv_old;
    const size_t nD_old = bo * nelem, nD_new = bn * nelem;
    const size_t nO_old = bo * nintface, nO_new = bn * nintface;
    const size_t nR_old = (size_t)nv_old * nelem, nR_new = (size_t)nv_new * nelem;
    for (size_t i = 0; i < nD_new; ++i) D[i] = i < nD_old ? D_old[i] : 0.0;
    for (size_t i = 0; i < nO_new; ++i) O1[i] = i < nO_old ? O1_old[i] : 0.0;
    for (size_t i = 0; i < nO_new; ++i) O2[i] = i < nO_old ? O2_old[i] : 0.0;
    for (size_t i = 0; i < nR_new; ++i) rhs[i] = i < nR_old ? rhs_old[i] : 0.0;
    for (size_t i = 0; i < nR_new; ++i) U0[i] = i < nR_old ? U0_old[i] : 0.0;
    for (int e = 0; e < nelem; ++e)
        for (int j = 0; j < nv_new; ++j) D[(size_t)e * bn + nv_new * j + j] = 10.0;
    for (int f = 0; f < nintface; ++f)
        for (int j = 0; j < nv_new; ++j) O1[(size_t)f * bn + nv_new * j + j] = 10.0;
    for (int f = 0; f < nintface; ++f)
        for (int j = 0; j < nv_new; ++j) O2[(size_t)f * bn + nv_new * j + j] = 10.0;
    for (int e = 0; e < nelem; ++e)
        for (int j = 0; j < mn; ++j)
            for (int i = 0; i < mn; ++i)
                D[(size_t)e * bn + nv_new * j + i] = D_old[(size_t)e * bo + nv_old * j + i];
    for (int e = 0; e < nintface; ++e)
        for (int j = 0; j < mn; ++j)
            for (int i = 0; i < mn; ++i) {
                O1[(size_t)e * bn + nv_new * j + i] = O1_old[(size_t)e * bo + nv_old * j + i];
                O2[(size_t)e * bn + nv_new * j + i] = O2_old[(size_t)e * bo + nv_old * j + i];
            }
    for (size_t eij = 0; eij < (size_t)nelem * mn; ++eij) rhs[eij] = rhs_old[eij];
    for (size_t eij = 0; eij < (size_t)nelem * mn; ++eij) U0[eij] = U0_old[eij];
}

/*
 * ref_driver.c -- drives the reference's own LIJ kernels, mechanically
 * translated from OKL to C by oracle/okl2c.py into oracle/_ref/ (generated,
 * git-ignored), in the order of the reference's driver (src/main.cxx:180-229).
 * TEST INFRASTRUCTURE: the tests use this library to pin oracle/lij_oracle.c
 * (the hand restatement) and the GPU's reference-order path to the
 * reference's own code; bench.py may time it as the CPU reference.  The
 * product (libtriblock.so) never calls it.
 *
 * Phases (all kernels are the translated reference kernels):
 *   A packing    Jacobian::assembleTriBlocks         src/Jacobian.cxx:76-117
 *   jacDLU = jacD copyAtoBjac                        src/okl/linesmoothLU_v5.okl:85-93
 *   factor       lineLU                              src/okl/lineLU_v2.okl:58-182
 *   R = rhs      copyAtoB                            src/okl/linesmoothLU_v5.okl:75-83
 *   per sweep    triblock_solveDU                    src/okl/linesmoothLU_TriBlock_v3.okl:92-226
 *                addAtoB (U += dU), copyAtoB (R = rhs)  linesmoothLU_v5.okl:95-103, :75-83
 *                triblock_lineRes (R += J U)         linesmoothLU_TriBlock_v3.okl:228-336
 * The per-sweep norm is not part of the reference (it prints none); it is
 * sqrt of the sum of squares in index order, as oracle_norm computes it.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "okl_kernels.h"

int okl_nvar = 9;
int okl_max_line_elem = 1;
int okl_threads = 1;

void okl_ref_assemble_tri_blocks(int nvar, int nelem, int nintface, int nline, int nlineelem,
                                 const int *fc, const int *linesize, const int *linepoint,
                                 const int *lines, const int *lineface, const double *jacO1,
                                 const double *jacO2, double *A);

void okl_ref_set_threads(int n) { okl_threads = n > 0 ? n : 1; }

static double norm2(const double *R, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += R[i] * R[i];
    return sqrt(s);
}

/* A reference run from U = 0: factor, then `iters` sweeps.
 *   hist       iters+1 norms of R (before the first sweep, after each), or NULL
 *   U, R, dU   final state (nv*nelem each)
 *   DLU, DinvC factors (nv*nv*nelem each) or NULL; A the packed lower blocks
 *              (nv*nv*nlineelem) or NULL
 *   U_all, R_all, dU_all  the state after every sweep (iters*nv*nelem each) or NULL
 * Returns 0, or 1 for sizes the reference cannot run, 2 on allocation failure. */
int okl_ref_lij(int nvar, int nelem, int nintface, int eftot, int nline, int nlineelem,
                int max_line_nelem, const int *epoint, const int *ef, const int *fc,
                const int *linesize, const int *linepoint, const int *lines, const int *lineface,
                const double *jacD, const double *jacO1, const double *jacO2, const double *rhs,
                int iters, double *U, double *R, double *dU, double *hist, double *DLU_out,
                double *DinvC_out, double *A_out, double *U_all, double *R_all, double *dU_all) {
    if (nvar < 1 || nelem < 0 || nline < 0 || nlineelem < nelem || max_line_nelem < 1 || iters < 0)
        return 1;
    okl_nvar = nvar;
    okl_max_line_elem = max_line_nelem;
    const size_t bs = (size_t)nvar * nvar, nvec = (size_t)nvar * nelem;
    /* the reference's host vectors are value-initialised by resize() (Jacobian.cxx:37-48) */
    double *DLU = (double *)calloc(bs * (size_t)nelem + 1, sizeof(double));
    double *DinvC = (double *)calloc(bs * (size_t)nelem + 1, sizeof(double));
    double *A = (double *)calloc(bs * (size_t)nlineelem + 1, sizeof(double));
    if (!DLU || !DinvC || !A) {
        free(DLU);
        free(DinvC);
        free(A);
        return 2;
    }
    okl_ref_assemble_tri_blocks(nvar, nelem, nintface, nline, nlineelem, fc, linesize, linepoint,
                                lines, lineface, jacO1, jacO2, A);
    memset(U, 0, nvec * sizeof(double));
    memset(dU, 0, nvec * sizeof(double));
    memset(R, 0, nvec * sizeof(double));

    v5__copyAtoBjac(nelem, jacD, DLU);
    lineLU_v2__lineLU(nelem, nintface, nline, fc, linesize, linepoint, lines, lineface, DLU, jacO1,
                      jacO2, DinvC);
    v5__copyAtoB(nelem, rhs, R);
    if (hist) hist[0] = norm2(R, nvec);
    for (int p = 0; p < iters; ++p) {
        TriBlock_v3__triblock_solveDU(nelem, nintface, eftot, nline, nlineelem, linesize,
                                      linepoint, lines, DLU, DinvC, A, dU, R);
        v5__addAtoB(nelem, dU, U);
        v5__copyAtoB(nelem, rhs, R);
        TriBlock_v3__triblock_lineRes(nelem, nintface, eftot, nline, nlineelem, epoint, ef, fc,
                                      linesize, linepoint, lines, jacD, jacO1, jacO2, U, R);
        if (hist) hist[p + 1] = norm2(R, nvec);
        if (U_all) memcpy(U_all + (size_t)p * nvec, U, nvec * sizeof(double));
        if (R_all) memcpy(R_all + (size_t)p * nvec, R, nvec * sizeof(double));
        if (dU_all) memcpy(dU_all + (size_t)p * nvec, dU, nvec * sizeof(double));
    }
    if (DLU_out) memcpy(DLU_out, DLU, bs * nelem * sizeof(double));
    if (DinvC_out) memcpy(DinvC_out, DinvC, bs * nelem * sizeof(double));
    if (A_out) memcpy(A_out, A, bs * nlineelem * sizeof(double));
    free(DLU);
    free(DinvC);
    free(A);
    return 0;
}

/* The reference's residual rule alone: R = rhs + J U (copyAtoB, then
 * triblock_lineRes). */
int okl_ref_true_residual(int nvar, int nelem, int nintface, int eftot, int nline, int nlineelem,
                          int max_line_nelem, const int *epoint, const int *ef, const int *fc,
                          const int *linesize, const int *linepoint, const int *lines,
                          const double *jacD, const double *jacO1, const double *jacO2,
                          const double *rhs, const double *U, double *R) {
    if (nvar < 1 || max_line_nelem < 1) return 1;
    okl_nvar = nvar;
    okl_max_line_elem = max_line_nelem;
    v5__copyAtoB(nelem, rhs, R);
    TriBlock_v3__triblock_lineRes(nelem, nintface, eftot, nline, nlineelem, epoint, ef, fc,
                                  linesize, linepoint, lines, jacD, jacO1, jacO2, U, R);
    return 0;
}

/* A reference factorization followed by `n` timed-style sweeps from the
 * state the caller holds (for the CPU baseline: factor once, sweep many). */
typedef struct {
    int nvar, nelem, nintface, eftot, nline, nlineelem, max_line_nelem;
    const int *epoint, *ef, *fc, *linesize, *linepoint, *lines;
    const double *jacD, *jacO1, *jacO2, *rhs;
    double *DLU, *DinvC, *A;
} okl_ref_state;

okl_ref_state *okl_ref_factor(int nvar, int nelem, int nintface, int eftot, int nline,
                              int nlineelem, int max_line_nelem, const int *epoint, const int *ef,
                              const int *fc, const int *linesize, const int *linepoint,
                              const int *lines, const int *lineface, const double *jacD,
                              const double *jacO1, const double *jacO2, const double *rhs) {
    if (nvar < 1 || nlineelem < nelem || max_line_nelem < 1) return NULL;
    okl_ref_state *s = (okl_ref_state *)calloc(1, sizeof(okl_ref_state));
    if (!s) return NULL;
    const size_t bs = (size_t)nvar * nvar;
    s->DLU = (double *)calloc(bs * (size_t)nelem + 1, sizeof(double));
    s->DinvC = (double *)calloc(bs * (size_t)nelem + 1, sizeof(double));
    s->A = (double *)calloc(bs * (size_t)nlineelem + 1, sizeof(double));
    if (!s->DLU || !s->DinvC || !s->A) {
        free(s->DLU);
        free(s->DinvC);
        free(s->A);
        free(s);
        return NULL;
    }
    s->nvar = nvar; s->nelem = nelem; s->nintface = nintface; s->eftot = eftot;
    s->nline = nline; s->nlineelem = nlineelem; s->max_line_nelem = max_line_nelem;
    s->epoint = epoint; s->ef = ef; s->fc = fc; s->linesize = linesize;
    s->linepoint = linepoint; s->lines = lines;
    s->jacD = jacD; s->jacO1 = jacO1; s->jacO2 = jacO2; s->rhs = rhs;
    okl_nvar = nvar;
    okl_max_line_elem = max_line_nelem;
    okl_ref_assemble_tri_blocks(nvar, nelem, nintface, nline, nlineelem, fc, linesize, linepoint,
                                lines, lineface, jacO1, jacO2, s->A);
    v5__copyAtoBjac(nelem, jacD, s->DLU);
    lineLU_v2__lineLU(nelem, nintface, nline, fc, linesize, linepoint, lines, lineface, s->DLU,
                      jacO1, jacO2, s->DinvC);
    return s;
}

/* n sweeps (src/main.cxx:207-229) on the caller's U, R, dU. */
void okl_ref_sweeps(okl_ref_state *s, double *U, double *R, double *dU, int n) {
    okl_nvar = s->nvar;
    okl_max_line_elem = s->max_line_nelem;
    for (int p = 0; p < n; ++p) {
        TriBlock_v3__triblock_solveDU(s->nelem, s->nintface, s->eftot, s->nline, s->nlineelem,
                                      s->linesize, s->linepoint, s->lines, s->DLU, s->DinvC, s->A,
                                      dU, R);
        v5__addAtoB(s->nelem, dU, U);
        v5__copyAtoB(s->nelem, s->rhs, R);
        TriBlock_v3__triblock_lineRes(s->nelem, s->nintface, s->eftot, s->nline, s->nlineelem,
                                      s->epoint, s->ef, s->fc, s->linesize, s->linepoint, s->lines,
                                      s->jacD, s->jacO1, s->jacO2, U, R);
    }
}

void okl_ref_free(okl_ref_state *s) {
    if (!s) return;
    free(s->DLU);
    free(s->DinvC);
    free(s->A);
    free(s);
}

/*
 * kernels_nv.cu -- TBS_ALGO_FP64 for block sizes other than 9 (nvar 2..16),
 * the block-size range of the reference's resizeBlockSize study
 * (src/Jacobian.cxx:153-238; the paper's Fig. 8).  Same algorithm, storage
 * and launch sequence as the size-9 kernels in kernels_fast.cu -- explicit
 * block inverses, twisted line elimination, the residual updated from the
 * cross-line couplings only, position order -- written once as templates
 * over the block size NV:
 *   nv_factor_kernel   one warp per chain, lane j < NV owns column j of
 *                      every block, Gauss-Jordan by columns with shuffles
 *   nv_twist_kernel    one CTA per line: the twist cell's pivot
 *   nv_thomas_kernel   one warp per line, the two half-warps on the two
 *                      chains, lane i < NV on row i; chunks of G (Gam)
 *                      and b stream through a ring of bulk copies in
 *                      shared memory and the previous vector arrives by
 *                      shuffles
 *   nv_resid_kernel    persistent over 16-position tiles, Dinv and the
 *                      cross-line blocks staged by bulk copies, thread
 *                      (cell, row) = (t / NV, t % NV)
 * All blocks are column-major (entry (i, j) at i + NV j), so that lane i
 * reading row i of a staged block hits consecutive shared-memory words.
 * The size-9 kernels stay the tuned path; these are their general form.
 */
#include "device_common.cuh"
#include "tbs_internal.hxx"
#include "tma.cuh"

#include <cuda_runtime.h>

namespace tbs {

namespace {

constexpr unsigned NFULL = 0xffffffffu;
constexpr int NV_MIN = 2, NV_MAX = 16;

template <int NV>
__device__ __forceinline__ void nv_gj_cols(double (&w)[NV], int j, unsigned *status) {
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        double colp[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) colp[i] = __shfl_sync(NFULL, w[i], p);
        const double piv = colp[p];
        if (threadIdx.x == 0 && !(fabs(piv) > 0.0 && isfinite(piv))) atomicOr(status, ST_PIVOT);
        const double r = 1.0 / piv;
        const bool isp = (j == p);
        const double t = w[p] * r;
#pragma unroll
        for (int i = 0; i < NV; ++i)
            if (i != p) w[i] = isp ? -colp[i] * r : w[i] - colp[i] * t;
        w[p] = isp ? r : t;
    }
}

/* in-place Gauss-Jordan of the NV x NV block W (column-major) in shared
 * memory, thread t < NV*NV on entry (t % NV, t / NV) */
template <int NV>
__device__ __forceinline__ void nv_gj_smem(double *W, int t, unsigned *status) {
    constexpr int NB = NV * NV;
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

/* one warp per chain (grid = 2 x lines); the layout's fsrc gives, per
 * position, the element, the face to the chain predecessor and its side */
template <int NV>
__global__ void __launch_bounds__(32) nv_factor_kernel(
    int nline, const int *__restrict__ line_start, const int *__restrict__ line_len,
    const int *__restrict__ line_twist, const int *__restrict__ fsrc,
    const double *__restrict__ jacD, const double *__restrict__ O1, const double *__restrict__ O2,
    double *__restrict__ Dinv, double *__restrict__ G, double *__restrict__ Gam,
    double *__restrict__ gamlast, unsigned *status) {
    constexpr int NB = NV * NV;
    const int l = blockIdx.x >> 1, g = blockIdx.x & 1;
    if (l >= nline) return;
    const int lane = threadIdx.x;
    const int j = lane < NV ? lane : NV - 1;
    const bool act = lane < NV;
    __shared__ double sM[NB], sA[NB];
    const int ps = line_start[l], n = line_len[l], m = line_twist[l];
    const int len = g ? n - 1 - m : m;
    const int cs = ps + (g ? m : 0);
    const int ptw = ps + n - 1;
    if (len == 0) {
        for (int t = lane; t < NB; t += 32) gamlast[((size_t)l * 2 + g) * NB + t] = 0.0;
        return;
    }
    double w[NV], an[NV], cn[NV], dn[NV];
    {
        const double *D0 = jacD + (size_t)fsrc[5 * cs] * NB + NV * j;
#pragma unroll
        for (int i = 0; i < NV; ++i) w[i] = D0[i];
    }
    auto fetch = [&](int p) {
        const int e = fsrc[5 * p], f = fsrc[5 * p + 1], side = fsrc[5 * p + 2];
        const double *Ap = (side ? O2 : O1) + (size_t)f * NB + NV * j;
        const double *Cp = (side ? O1 : O2) + (size_t)f * NB + NV * j;
        const double *Dp = jacD + (size_t)e * NB + NV * j;
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            an[i] = Ap[i];
            cn[i] = Cp[i];
            dn[i] = Dp[i];
        }
    };
    if (len > 1) fetch(cs + 1);
    nv_gj_cols<NV>(w, j, status);
    if (act) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            Dinv[(size_t)cs * NB + i + NV * j] = w[i];
            G[(size_t)cs * NB + i + NV * j] = 0.0;
            sM[i + NV * j] = w[i];
        }
    }
    for (int s = 1; s < len; ++s) {
        const int p = cs + s;
        double a[NV], c[NV], d[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            a[i] = an[i];
            c[i] = cn[i];
            d[i] = dn[i];
        }
        if (s + 1 < len) fetch(p + 1);
        __syncwarp();
        /* Gam_{s-1}(:, j) = Dinv_{s-1} C(:, j) */
        double gm[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double acc = 0.0;
#pragma unroll
            for (int q = 0; q < NV; ++q) acc += sM[i + NV * q] * c[q];
            gm[i] = acc;
        }
        if (act) {
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                Gam[(size_t)(p - 1) * NB + i + NV * j] = gm[i];
                sA[i + NV * j] = a[i];
            }
        }
        __syncwarp();
        /* W(:, j) = D(:, j) - A Gam_{s-1}(:, j) */
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double acc = d[i];
#pragma unroll
            for (int q = 0; q < NV; ++q) acc -= sA[i + NV * q] * gm[q];
            w[i] = acc;
        }
        nv_gj_cols<NV>(w, j, status);
        __syncwarp();
        if (act) {
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                Dinv[(size_t)p * NB + i + NV * j] = w[i];
                sM[i + NV * j] = w[i];
            }
        }
        __syncwarp();
        /* G_s(:, j) = Dinv_s A(:, j) */
        if (act) {
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                double acc = 0.0;
#pragma unroll
                for (int q = 0; q < NV; ++q) acc += sM[i + NV * q] * a[q];
                G[(size_t)p * NB + i + NV * j] = acc;
            }
        }
    }
    /* coupling of the chain's last cell to the twist */
    {
        const int f = fsrc[5 * ptw + (g ? 3 : 1)], side = fsrc[5 * ptw + (g ? 4 : 2)];
        const double *Cp = (side ? O1 : O2) + (size_t)f * NB + NV * j;
        double c[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) c[i] = Cp[i];
        __syncwarp();
        if (act) {
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                double acc = 0.0;
#pragma unroll
                for (int q = 0; q < NV; ++q) acc += sM[i + NV * q] * c[q];
                Gam[(size_t)(cs + len - 1) * NB + i + NV * j] = acc;
                gamlast[((size_t)l * 2 + g) * NB + i + NV * j] = acc;
            }
        }
    }
}

template <int NV>
constexpr int nv_block_threads() { return ((NV * NV + 31) / 32) * 32; }

template <int NV>
__global__ void __launch_bounds__(nv_block_threads<NV>()) nv_twist_kernel(
    int nline, const int *__restrict__ line_start, const int *__restrict__ line_len,
    const int *__restrict__ fsrc, const double *__restrict__ jacD, const double *__restrict__ O1,
    const double *__restrict__ O2, double *__restrict__ Dinv, double *__restrict__ G,
    double *__restrict__ Gam, const double *__restrict__ gamlast, unsigned *status) {
    constexpr int NB = NV * NV;
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
        sW[t] = w;
    }
    __syncthreads();
    nv_gj_smem<NV>(sW, t, status);
    if (act) {
        double ga = 0.0, gc = 0.0;
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            ga += sW[i + NV * q] * sA[q + NV * j];
            gc += sW[i + NV * q] * sC[q + NV * j];
        }
        Dinv[(size_t)ptw * NB + t] = sW[t];
        G[(size_t)ptw * NB + t] = ga;
        Gam[(size_t)ptw * NB + t] = gc;
    }
}

/* X[q] = cross-line block of slot q = s*np16 + p (slot-major), or zeros */
template <int NV>
__global__ void nv_xlayout_kernel(long long nslots, const int *__restrict__ xsrc,
                                  const double *__restrict__ O1, const double *__restrict__ O2,
                                  double *__restrict__ X) {
    constexpr int NB = NV * NV;
    const int lane = threadIdx.x & 31;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long q = w0; q < nslots; q += nw) {
        const int src = xsrc[q];
        for (int tt = lane; tt < NB; tt += 32)
            X[q * NB + tt] = src >= 0 ? ((src & 1) ? O2 : O1)[(size_t)(src >> 1) * NB + tt] : 0.0;
    }
}

/* init - row . v with the previous vector v held one component per lane of
 * this half-warp (lanes src0 .. src0+NV-1) */
/* init - row . v, row i of the column-major block at blk (entry (i, j)
 * at i + NV j), with the previous vector v held one component per lane
 * of this half-warp (lanes src0 .. src0+NV-1) */
template <int NV>
__device__ __forceinline__ double nv_row_step(const double *blk, int i, double init, double vmine,
                                              int src0) {
    double a0 = init, a1 = 0.0, a2 = 0.0;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const double vj = __shfl_sync(NFULL, vmine, src0 + j);
        const double g = blk[i + NV * j];
        if (j % 3 == 0)
            a0 -= g * vj;
        else if (j % 3 == 1)
            a1 += g * vj;
        else
            a2 += g * vj;
    }
    return a0 - (a1 + a2);
}

/* cells per chunk of a chain: 8, or 4 for blocks of 10..13 so that a
 * two-stage ring stays small enough for nine lines per SM (one wave at
 * 1,200 lines; measured: 10-25 % faster there, slower from 14 on, where
 * even 4-cell chunks do not reach one wave); a multiple of 4 keeps every
 * bulk copy 16-byte sized */
template <int NV>
constexpr int nv_chunk() { return (NV >= 10 && NV <= 13) ? 4 : 8; }

template <int NV>
__host__ __device__ inline size_t nv_thomas_stage() {
    return 2 * (size_t)nv_chunk<NV>() * (NV * NV + NV) * sizeof(double);
}

/* One warp per line: half-warp h runs chain h (top: positions 0..m-1 in
 * order, bottom: m..n-2 in elimination order), lane i < NV row i.  Lane 0
 * streams "jobs" through an NS-stage ring of bulk copies, each holding one
 * chunk of nv_chunk<NV>() cells of both chains: forward jobs the blocks of G and the
 * b vectors, backward jobs (in reverse) the blocks of Gam; y is read back
 * with plain loads one chunk ahead.  Forward y_s = b_s - G_s y_{s-1}, twist
 * x = b - G_tw y_top - Gam_tw y_bot, backward x_s = y_s - Gam_s x_{s+1};
 * accumulate 0: U = dU, 1: U += dU, 2: U untouched.  A staging wait that
 * runs out of time sets ST_TIMEOUT and the warp drains its copies. */
template <int NV>
__global__ void __launch_bounds__(32) nv_thomas_kernel(
    int nline, int NS, const int *__restrict__ line_start, const int *__restrict__ line_len,
    const int *__restrict__ line_twist, const double *__restrict__ G, const double *__restrict__ Gam,
    const double *__restrict__ b, double *__restrict__ y, double *__restrict__ dU,
    double *__restrict__ U, int accumulate, unsigned *status) {
    constexpr int NB = NV * NV, P = nv_chunk<NV>();
    extern __shared__ __align__(128) unsigned char smem[];
    const int l = blockIdx.x;
    if (l >= nline) return;
    const int lane = threadIdx.x, h = lane >> 4, i = lane & 15;
    const bool act = i < NV;
    const int ii = act ? i : 0;
    const int src0 = h << 4;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    const size_t half = (size_t)P * (NB + NV) * sizeof(double);
    const size_t stage = 2 * half;
    unsigned char *st0 = smem + 128;
    if (lane == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncwarp();
    const int ps = line_start[l], n = line_len[l], m = line_twist[l];
    const int nb = n - 1 - m;
    const int len = h ? nb : m;
    const size_t base = (size_t)ps + (h ? m : 0);
    const int nchT = (m + P - 1) / P, nchB = (nb + P - 1) / P;
    const int nch = h ? nchB : nchT;
    const int nf = nchT > nchB ? nchT : nchB;
    const int njobs = 2 * nf;
    const uint64_t pol = lane == 0 ? policy_evict_first() : 0;
    auto cells = [&](int ln, int c) { return ((min(P, ln - c * P) + 3) & ~3); };
    auto issue = [&](int job, int s) {
        unsigned char *st = st0 + (size_t)s * stage;
        uint32_t bytes = 0;
        if (job < nf) {
            if (job < nchT) bytes += cells(m, job) * (NB + NV) * sizeof(double);
            if (job < nchB) bytes += cells(nb, job) * (NB + NV) * sizeof(double);
        } else {
            const int jb = job - nf;
            if (nchT - 1 - jb >= 0) bytes += cells(m, nchT - 1 - jb) * NB * sizeof(double);
            if (nchB - 1 - jb >= 0) bytes += cells(nb, nchB - 1 - jb) * NB * sizeof(double);
        }
        mbar_arrive_expect_tx(&bars[s], bytes);
        for (int hh = 0; hh < 2; ++hh) {
            const int ln = hh ? nb : m, nc = hh ? nchB : nchT, cp = hh ? m : 0;
            unsigned char *hb = st + hh * half;
            if (job < nf) {
                const int c = job;
                if (c >= nc) continue;
                const int cnt = cells(ln, c);
                const size_t p = (size_t)(ps + cp + c * P);
                bulk_g2s_hint(hb, G + p * NB, cnt * NB * sizeof(double), &bars[s], pol);
                bulk_g2s(hb + (size_t)P * NB * sizeof(double), b + p * NV, cnt * NV * sizeof(double), &bars[s]);
            } else {
                const int c = nc - 1 - (job - nf);
                if (c < 0) continue;
                const int cnt = cells(ln, c);
                bulk_g2s_hint(hb, Gam + (size_t)(ps + cp + c * P) * NB, cnt * NB * sizeof(double),
                              &bars[s], pol);
            }
        }
    };
    /* u: U at p, read ahead when accumulate == 1 */
    auto put = [&](size_t p, double x, double u) {
        dU[p * NV + i] = x;
        if (accumulate == 0)
            U[p * NV + i] = x;
        else if (accumulate == 1)
            U[p * NV + i] = u + x;
    };
    int issued = 0;
    if (lane == 0)
        for (; issued < NS && issued < njobs; ++issued) issue(issued, issued);
    int consumed = 0;
    bool timed_out = false;

    /* ---------------- forward */
    double yp = 0.0;
    for (int c = 0; c < nf; ++c) {
        const int s = c % NS;
        if (!__all_sync(NFULL, mbar_wait(&bars[s], (uint32_t)(c / NS) & 1u))) {
            timed_out = true;
            break;
        }
        ++consumed;
        const double *sG = reinterpret_cast<const double *>(st0 + (size_t)s * stage + h * half);
        const double *sB = sG + P * NB;
#pragma unroll
        for (int q = 0; q < P; ++q) {
            const int k = c * P + q;
            const double yi = nv_row_step<NV>(sG + q * NB, ii, sB[q * NV + ii], yp, src0);
            if (k < len) {
                if (act) y[(base + k) * NV + i] = yi;
                yp = yi;
            }
        }
        __syncwarp();
        if (lane == 0 && issued < njobs) {
            issue(issued, s);
            ++issued;
        }
    }
    if (!timed_out) {
        /* ---------------- twist (both halves compute the same values) */
        const size_t ptw = (size_t)ps + n - 1;
        double xm = b[ptw * NV + ii];
        {
            const double *gr = G + ptw * NB + ii;
            const double *cr = Gam + ptw * NB + ii;
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                const double yt = __shfl_sync(NFULL, yp, j);
                const double yb = __shfl_sync(NFULL, yp, 16 + j);
                xm -= gr[NV * j] * yt + cr[NV * j] * yb;
            }
        }
        if (h == 0 && act) put(ptw, xm, accumulate == 1 ? U[ptw * NV + i] : 0.0);
        /* ---------------- backward */
        /* y, and U when the solve adds dU to it, read one chunk ahead */
        double yv[P], nyv[P], uv[P], nuv[P];
        auto load_y = [&](int c, double *yy, double *uu) {
#pragma unroll
            for (int q = 0; q < P; ++q) {
                const int k = c * P + q;
                const bool ok = c >= 0 && k < len;
                yy[q] = ok ? y[(base + k) * NV + ii] : 0.0;
                uu[q] = (ok && accumulate == 1) ? U[(base + k) * NV + ii] : 0.0;
            }
        };
        __syncwarp();
        load_y(nch - 1, yv, uv);
        double xp = xm;
        for (int jb = 0; jb < nf; ++jb) {
            const int job = nf + jb;
            const int c = nch - 1 - jb; /* this half's chunk (may be < 0) */
            load_y(c - 1, nyv, nuv);
            const int s = job % NS;
            if (!__all_sync(NFULL, mbar_wait(&bars[s], (uint32_t)(job / NS) & 1u))) {
                timed_out = true;
                break;
            }
            ++consumed;
            const double *sG = reinterpret_cast<const double *>(st0 + (size_t)s * stage + h * half);
#pragma unroll
            for (int q = P - 1; q >= 0; --q) {
                const int k = c * P + q;
                const bool valid = c >= 0 && k < len;
                const double xi = nv_row_step<NV>(sG + q * NB, ii, valid ? yv[q] : 0.0, xp, src0);
                if (valid) {
                    if (act) put(base + k, xi, uv[q]);
                    xp = xi;
                }
            }
            __syncwarp();
            if (lane == 0 && issued < njobs) {
                issue(issued, s);
                ++issued;
            }
#pragma unroll
            for (int q = 0; q < P; ++q) {
                yv[q] = nyv[q];
                uv[q] = nuv[q];
            }
        }
    }
    if (timed_out && lane == 0) {
        atomicOr(status, ST_TIMEOUT);
        for (int job = consumed; job < issued; ++job)
            mbar_wait(&bars[job % NS], (uint32_t)(job / NS) & 1u, 1LL << 28);
    }
}

/* positions per residual tile: 16 (the layout's granule), up to 64 for
 * small blocks so that a tile still moves several KB per barrier phase */
template <int NV>
constexpr int nv_tile() {
    return RES_TILE * (128 / (NV * NV) < 1 ? 1 : (128 / (NV * NV) > 4 ? 4 : 128 / (NV * NV)));
}

template <int NV>
constexpr int nv_resid_threads() { return ((nv_tile<NV>() * NV + 31) / 32) * 32; }

template <int NV>
__host__ __device__ inline size_t nv_resid_smem(int nx) {
    const int nxa = nx > 0 ? nx : 1;
    constexpr size_t T = nv_tile<NV>();
    return 128 + T * NV * NV * sizeof(double) * (1 + nx) + (size_t)nxa * T * NV * sizeof(double) +
           T * NV * sizeof(double) * 2;
}

template <int NV>
inline int nv_resid_tiles(int np16) { return (np16 + nv_tile<NV>() - 1) / nv_tile<NV>(); }

/* persistent over the tiles of nv_tile<NV>() positions (the last one may
 * be shorter, by whole 16-position granules); per tile
 *   MODE 0:  R = Rsrc, Uacc = 0 (the start of a sweep sequence)
 *   MODE 1:  R = sum over slots X dU[nbr], Uacc += dU
 * then b = -Dinv R and the tile's sum R^2; thread t < 16 NV owns cell
 * t / NV, row t % NV, so that the threads of a warp read consecutive rows
 * of a block in shared memory (no bank conflicts at any NV) and gather a
 * neighbour's vector with consecutive loads */
template <int NV, int MODE>
__global__ void __launch_bounds__(nv_resid_threads<NV>()) nv_resid_kernel(
    int nx, int np16, const double *__restrict__ Dinv, const double *__restrict__ X,
    const int *__restrict__ xnbr, const double *__restrict__ dU, const double *__restrict__ Rsrc,
    double *__restrict__ b, double *__restrict__ Uacc, NormSink ns, unsigned *status) {
    constexpr int NB = NV * NV, TH = nv_resid_threads<NV>(), TL = nv_tile<NV>();
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    double *sD = reinterpret_cast<double *>(smem + 128);
    double *sX = sD + TL * NB;
    const int nxa = nx > 0 ? nx : 1;
    double *sg = sX + (MODE == 1 ? nx : 0) * TL * NB;
    double *sr = sg + nxa * TL * NV;
    double *sb = sr + TL * NV;
    __shared__ double red[TH / 32];
    const int tid = threadIdx.x;
    const int c = tid / NV, i = tid % NV;
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    const int ntiles = (np16 + TL - 1) / TL;
    uint32_t parity = 0;
    for (int blk = blockIdx.x; blk < ntiles; blk += gridDim.x) {
        const int p0 = blk * TL;
        const int cnt = np16 - p0 < TL ? np16 - p0 : TL; /* a multiple of 16 */
        const bool act = tid < cnt * NV;
        const uint32_t szD = cnt * NB * sizeof(double), szR = cnt * NV * sizeof(double);
        if (tid == 0) {
            const uint64_t pol = policy_evict_first();
            mbar_arrive_expect_tx(bar, szD + (MODE == 1 ? nx * szD : szR));
            bulk_g2s_hint(sD, Dinv + (size_t)p0 * NB, szD, bar, pol);
            if (MODE == 1) {
                for (int s = 0; s < nx; ++s)
                    bulk_g2s_hint(sX + s * TL * NB, X + ((size_t)s * np16 + p0) * NB, szD, bar, pol);
            } else {
                bulk_g2s(sr, Rsrc + (size_t)p0 * NV, szR, bar);
            }
        }
        if (act && Uacc) {
            const size_t q = (size_t)p0 * NV + tid;
            Uacc[q] = MODE == 1 ? Uacc[q] + dU[q] : 0.0;
        }
        if (MODE == 1 && act) {
            for (int s = 0; s < nx; ++s) {
                const int nb = xnbr[(size_t)s * np16 + p0 + c];
                sg[(s * TL + c) * NV + i] = nb >= 0 ? dU[(size_t)nb * NV + i] : 0.0;
            }
        }
        const bool ok = mbar_wait(bar, parity);
        parity ^= 1u;
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicOr(status, ST_TIMEOUT);
                mbar_wait(bar, parity ^ 1u, 1LL << 28);
            }
            break;
        }
        double r = 0.0;
        if (MODE == 1) {
            if (act) {
                double a0 = 0.0, a1 = 0.0, a2 = 0.0;
                for (int s = 0; s < nx; ++s) {
                    const double *xr = sX + (s * TL + c) * NB + i;
                    const double *g = sg + (s * TL + c) * NV;
#pragma unroll
                    for (int j = 0; j < NV; ++j) {
                        if (j % 3 == 0)
                            a0 += xr[NV * j] * g[j];
                        else if (j % 3 == 1)
                            a1 += xr[NV * j] * g[j];
                        else
                            a2 += xr[NV * j] * g[j];
                    }
                }
                r = a0 + (a1 + a2);
                sr[c * NV + i] = r;
            }
            __syncthreads();
        } else if (act) {
            r = sr[c * NV + i];
        }
        double sq = act ? r * r : 0.0;
        if (act) {
            const double *dr = sD + c * NB + i;
            const double *rv = sr + c * NV;
            double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                if (j % 3 == 0)
                    a0 += dr[NV * j] * rv[j];
                else if (j % 3 == 1)
                    a1 += dr[NV * j] * rv[j];
                else
                    a2 += dr[NV * j] * rv[j];
            }
            sb[c * NV + i] = -(a0 + (a1 + a2));
        }
        __syncthreads();
        if (act) b[(size_t)p0 * NV + tid] = sb[tid];
        if (ns.partials) {
            for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(NFULL, sq, o);
            if ((tid & 31) == 0) red[tid >> 5] = sq;
            __syncthreads();
            if (tid == 0) {
                double tot = 0.0;
                for (int w = 0; w < TH / 32; ++w) tot += red[w];
                ns.partials[blk] = tot;
            }
        }
        __syncthreads(); /* the next tile's copies overwrite the stages */
    }
    finalize_total(ns, ntiles);
}


/* ---------------------------------------------------------------- host */

int nv_smem_limit(const void *fn) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, fn);
    return optin - (int)fa.sharedSizeBytes;
}

int nv_set_smem(const void *fn, size_t need) {
    if ((long long)need > nv_smem_limit(fn)) return (int)cudaErrorInvalidConfiguration;
    if (need <= 48 * 1024) return 0;
    return smem_raise(fn, need);
}

int nv_grid_persistent(const void *fn, int threads, size_t smem, int ntiles) {
    int dev = 0, nsm = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem) != cudaSuccess || per < 1)
        per = 1;
    const int g = per * nsm;
    return ntiles < g ? (ntiles > 0 ? ntiles : 1) : g;
}

int grid_cap(long long n, int threads) {
    long long g = (n + threads - 1) / threads;
    if (g > 148 * 8) g = 148 * 8;
    return g < 1 ? 1 : (int)g;
}

template <int NV>
struct NvOps {
    static int factor(cudaStream_t st, const FastLayout &L, const double *jacD, const double *O1,
                      const double *O2, double *Dinv, double *G, double *Gam, double *gamlast,
                      unsigned *status) {
        nv_factor_kernel<NV><<<2 * L.nline, 32, 0, st>>>(L.nline, L.line_start, L.line_len,
                                                         L.line_twist, L.fsrc, jacD, O1, O2, Dinv,
                                                         G, Gam, gamlast, status);
        nv_twist_kernel<NV><<<L.nline, nv_block_threads<NV>(), 0, st>>>(
            L.nline, L.line_start, L.line_len, L.fsrc, jacD, O1, O2, Dinv, G, Gam, gamlast, status);
        return (int)cudaGetLastError();
    }
    static int xlayout(cudaStream_t st, const FastLayout &L, const double *O1, const double *O2,
                       double *X) {
        const long long nslots = (long long)L.np16 * L.nx;
        if (nslots == 0) return 0;
        nv_xlayout_kernel<NV><<<grid_cap(nslots * 32, 256), 256, 0, st>>>(nslots, L.xsrc, O1, O2, X);
        return (int)cudaGetLastError();
    }
    /* ring depth: the SM's shared memory over its resident lines, 2..6 */
    static int thomas_ns(const FastLayout &L) {
        int dev = 0, nsm = 148, smem_sm = 228 * 1024, reserved = 1024;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
        int per_sm = (L.nline + (nsm > 0 ? nsm : 148) - 1) / (nsm > 0 ? nsm : 148);
        if (per_sm < 1) per_sm = 1;
        long long ns = ((long long)smem_sm / per_sm - reserved - 128) / (long long)nv_thomas_stage<NV>();
        if (ns > 6) ns = 6;
        if (ns < 2) ns = 2;
        return (int)ns;
    }
    static size_t thomas_smem(int ns) { return 128 + (size_t)ns * nv_thomas_stage<NV>(); }
    static int thomas(cudaStream_t st, const FastLayout &L, const double *G, const double *Gam,
                      const double *b, double *y, double *dU, double *U, int accumulate,
                      unsigned *status) {
        const int ns = thomas_ns(L);
        const size_t smem = thomas_smem(ns);
        int rc = nv_set_smem((const void *)nv_thomas_kernel<NV>, smem);
        if (rc) return rc;
        nv_thomas_kernel<NV><<<L.nline, 32, smem, st>>>(L.nline, ns, L.line_start, L.line_len,
                                                        L.line_twist, G, Gam, b, y, dU, U,
                                                        accumulate, status);
        return (int)cudaGetLastError();
    }
    static int resid(cudaStream_t st, const FastLayout &L, int mode, const double *Dinv,
                     const double *X, const double *dU, const double *Rsrc, double *b,
                     const NormSink &ns, unsigned *status, double *Uacc) {
        constexpr int TH = nv_resid_threads<NV>();
        const int ntiles = nv_resid_tiles<NV>(L.np16);
        if (mode == 1) {
            const size_t smem = nv_resid_smem<NV>(L.nx);
            nv_resid_kernel<NV, 1><<<nv_grid_persistent((const void *)nv_resid_kernel<NV, 1>, TH, smem, ntiles),
                                     TH, smem, st>>>(L.nx, L.np16, Dinv, X, L.xnbr, dU, nullptr, b,
                                                     Uacc, ns, status);
        } else {
            const size_t smem = nv_resid_smem<NV>(0);
            nv_resid_kernel<NV, 0><<<nv_grid_persistent((const void *)nv_resid_kernel<NV, 0>, TH, smem, ntiles),
                                     TH, smem, st>>>(0, L.np16, Dinv, nullptr, nullptr, nullptr, Rsrc,
                                                     b, Uacc, ns, status);
        }
        return (int)cudaGetLastError();
    }
    static int prepare(const FastLayout &L) {
        int rc = nv_set_smem((const void *)nv_thomas_kernel<NV>, thomas_smem(thomas_ns(L)));
        if (!rc) rc = nv_set_smem((const void *)nv_resid_kernel<NV, 1>, nv_resid_smem<NV>(L.nx));
        if (!rc) rc = nv_set_smem((const void *)nv_resid_kernel<NV, 0>, nv_resid_smem<NV>(0));
        return rc;
    }
};

/* a call on NvOps<nv> for nv in NV_MIN..NV_MAX */
template <typename F, int NV = NV_MIN>
int nv_dispatch(int nv, F &&f) {
    if constexpr (NV > NV_MAX) {
        return (int)cudaErrorInvalidValue;
    } else {
        if (nv == NV) return f(NvOps<NV>{});
        return nv_dispatch<F, NV + 1>(nv, static_cast<F &&>(f));
    }
}

}  // namespace

bool nv_supported(int nv) { return nv >= NV_MIN && nv <= NV_MAX; }

int nv_prepare(int nv, const FastLayout &L) {
    return nv_dispatch(nv, [&](auto ops) { return decltype(ops)::prepare(L); });
}

int launch_nv_factor(cudaStream_t st, int nv, const FastLayout &L, const double *jacD,
                     const double *O1, const double *O2, double *Dinv, double *G, double *Gam,
                     double *gamlast, unsigned *status) {
    return nv_dispatch(nv, [&](auto ops) {
        return decltype(ops)::factor(st, L, jacD, O1, O2, Dinv, G, Gam, gamlast, status);
    });
}

int launch_nv_xlayout(cudaStream_t st, int nv, const FastLayout &L, const double *O1,
                      const double *O2, double *X) {
    return nv_dispatch(nv, [&](auto ops) { return decltype(ops)::xlayout(st, L, O1, O2, X); });
}

int launch_nv_thomas(cudaStream_t st, int nv, const FastLayout &L, const double *G,
                     const double *Gam, const double *b, double *y, double *dU, double *U,
                     int accumulate, unsigned *status) {
    return nv_dispatch(nv, [&](auto ops) {
        return decltype(ops)::thomas(st, L, G, Gam, b, y, dU, U, accumulate, status);
    });
}

int launch_nv_resid(cudaStream_t st, int nv, const FastLayout &L, int mode, const double *Dinv,
                    const double *X, const double *dU, const double *Rsrc, double *b,
                    const NormSink &ns, unsigned *status, double *Uacc) {
    if (mode != 0 && mode != 1) return (int)cudaErrorInvalidValue;
    if (mode == 0 && !Rsrc) return (int)cudaErrorInvalidValue;
    return nv_dispatch(nv, [&](auto ops) {
        return decltype(ops)::resid(st, L, mode, Dinv, X, dU, Rsrc, b, ns, status, Uacc);
    });
}

}  // namespace tbs

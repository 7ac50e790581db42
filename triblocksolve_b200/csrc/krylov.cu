/*
 * krylov.cu -- tbs_gmres: restarted GMRES(m) on J U = -rhs, right
 * preconditioned by LIJ sweeps, the solver the paper pairs with the line
 * sweep (p.14, Table 6; the reference repository has no code for it).
 *
 * Preconditioner: P v = the iterate after k LIJ sweeps from zero on the
 * system v + J z = 0, i.e. z ~ -J^-1 v (k = 1: z = -M^-1 v, M the line
 * block-tridiagonal part), run with the TBS_ALGO_FP64 factors and kernels.
 * The product J z of each new direction comes out of the preconditioner's
 * last residual launch (J z = R - v, see precond_product).
 * Arnoldi on A = J P with classical Gram-Schmidt done twice; the basis of
 * preconditioned directions z_j is kept (flexible storage), so
 * U = sum_j y_j z_j.  The (m+1) x m Hessenberg least-squares problem is
 * solved on the host with Givens rotations after each Arnoldi step (one
 * small read-back per step); every restart recomputes the true residual.
 * Every reduction is a fixed-order sum, so runs are deterministic.
 *
 * Vectors are position ordered (np16 * 9 doubles, pads zero).
 */
#include "ctx.hxx"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using namespace tbs;

namespace {

constexpr int KR_THREADS = 256;
constexpr int KR_BLOCKS = 296;
constexpr int KR_CHUNK = 8;  /* vectors per pass of the dot kernel */
constexpr int KRYLOV_MAX = 64;
constexpr unsigned KFULL = 0xffffffffu;

/* partials[c * KR_BLOCKS + block] = this block's part of V_c . w for
 * c < count, and of w . w for c == count when self != 0.  Each thread
 * keeps KR_UNROLL grid-stride elements' loads in flight at once. */
constexpr int KR_UNROLL = 4;

__global__ void __launch_bounds__(KR_THREADS) kr_dots_kernel(long long n, const double *__restrict__ w,
                                                             const double *__restrict__ V, long long ldv,
                                                             int count, int self, double *partials) {
    __shared__ double red[KR_CHUNK][KR_THREADS / 32];
    const int total = count + (self ? 1 : 0);
    const long long t0 = blockIdx.x * (long long)KR_THREADS + threadIdx.x;
    const long long stride = (long long)gridDim.x * KR_THREADS;
    for (int c0 = 0; c0 < total; c0 += KR_CHUNK) {
        double acc[KR_CHUNK];
#pragma unroll
        for (int k = 0; k < KR_CHUNK; ++k) acc[k] = 0.0;
        long long t = t0;
        for (; t + (KR_UNROLL - 1) * stride < n; t += KR_UNROLL * stride) {
            double wt[KR_UNROLL];
#pragma unroll
            for (int u = 0; u < KR_UNROLL; ++u) wt[u] = w[t + u * stride];
#pragma unroll
            for (int k = 0; k < KR_CHUNK; ++k) {
                const int c = c0 + k;
                if (c < count) {
                    const double *vc = V + (size_t)c * ldv + t;
                    double x[KR_UNROLL];
#pragma unroll
                    for (int u = 0; u < KR_UNROLL; ++u) x[u] = vc[u * stride];
#pragma unroll
                    for (int u = 0; u < KR_UNROLL; ++u) acc[k] += x[u] * wt[u];
                } else if (c == count && self) {
#pragma unroll
                    for (int u = 0; u < KR_UNROLL; ++u) acc[k] += wt[u] * wt[u];
                }
            }
        }
        for (; t < n; t += stride) {
            const double wt = w[t];
#pragma unroll
            for (int k = 0; k < KR_CHUNK; ++k) {
                const int c = c0 + k;
                if (c < count)
                    acc[k] += V[(size_t)c * ldv + t] * wt;
                else if (c == count && self)
                    acc[k] += wt * wt;
            }
        }
#pragma unroll
        for (int k = 0; k < KR_CHUNK; ++k) {
            double v = acc[k];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(KFULL, v, o);
            if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
        }
        __syncthreads();
        if (threadIdx.x < KR_CHUNK && c0 + (int)threadIdx.x < total) {
            double tot = 0.0;
            for (int q = 0; q < KR_THREADS / 32; ++q) tot += red[threadIdx.x][q];
            partials[(size_t)(c0 + threadIdx.x) * KR_BLOCKS + blockIdx.x] = tot;
        }
        __syncthreads();
    }
}

/* out[c] = sum of the KR_BLOCKS partials of c, in a fixed order */
__global__ void __launch_bounds__(KR_THREADS) kr_reduce_kernel(const double *__restrict__ partials,
                                                               double *out) {
    __shared__ double red[KR_THREADS / 32];
    const double *p = partials + (size_t)blockIdx.x * KR_BLOCKS;
    double v = 0.0;
    for (int t = threadIdx.x; t < KR_BLOCKS; t += KR_THREADS) v += p[t];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(KFULL, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int q = 0; q < KR_THREADS / 32; ++q) tot += red[q];
        out[blockIdx.x] = tot;
    }
}

/* x += sign * sum_c coef[c] V_c (coef in device memory) */
__global__ void __launch_bounds__(KR_THREADS) kr_combine_kernel(long long n, double *__restrict__ x,
                                                                const double *__restrict__ V, long long ldv,
                                                                int count, const double *__restrict__ coef,
                                                                double sign) {
    __shared__ double cs[KRYLOV_MAX + 1];
    for (int c = threadIdx.x; c < count; c += KR_THREADS) cs[c] = sign * coef[c];
    __syncthreads();
    const long long stride = (long long)gridDim.x * KR_THREADS;
    long long t = blockIdx.x * (long long)KR_THREADS + threadIdx.x;
    for (; t + (KR_UNROLL - 1) * stride < n; t += KR_UNROLL * stride) {
        double acc[KR_UNROLL];
#pragma unroll
        for (int u = 0; u < KR_UNROLL; ++u) acc[u] = x[t + u * stride];
#pragma unroll 4
        for (int c = 0; c < count; ++c) {
            const double *vc = V + (size_t)c * ldv + t;
#pragma unroll
            for (int u = 0; u < KR_UNROLL; ++u) acc[u] += cs[c] * vc[u * stride];
        }
#pragma unroll
        for (int u = 0; u < KR_UNROLL; ++u) x[t + u * stride] = acc[u];
    }
    for (; t < n; t += stride) {
        double acc = x[t];
        for (int c = 0; c < count; ++c) acc += cs[c] * V[(size_t)c * ldv + t];
        x[t] = acc;
    }
}

__global__ void __launch_bounds__(KR_THREADS) kr_scale_kernel(long long n, double *__restrict__ dst,
                                                              const double *__restrict__ src, double a) {
    const long long stride = (long long)gridDim.x * KR_THREADS;
    long long t = blockIdx.x * (long long)KR_THREADS + threadIdx.x;
    for (; t + (KR_UNROLL - 1) * stride < n; t += KR_UNROLL * stride) {
        double v[KR_UNROLL];
#pragma unroll
        for (int u = 0; u < KR_UNROLL; ++u) v[u] = src[t + u * stride];
#pragma unroll
        for (int u = 0; u < KR_UNROLL; ++u) dst[t + u * stride] = a * v[u];
    }
    for (; t < n; t += stride) dst[t] = a * src[t];
}

}  // namespace

struct KrylovBufs {
    int m = 0;              /* restart length the basis holds */
    long long n = 0;        /* vector length */
    size_t bytes = 0;
    std::vector<void *> allocs;
    double *V = nullptr;    /* (m+1) x n */
    double *Z = nullptr;    /* m x n */
    double *w = nullptr;
    double *partials = nullptr;  /* (KRYLOV_MAX + 2) x KR_BLOCKS */
    double *h = nullptr, *h2 = nullptr, *y = nullptr;  /* KRYLOV_MAX + 2 each */
    double *h_host = nullptr;    /* pinned: h and h2 read-backs */
};

static int kfail(tbs_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    set_thread_error(msg);
    return code;
}

#define KCK(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return kfail(ctx, TBS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define KRUN(name, call)                                                                   \
    do {                                                                                   \
        const int h_ = ctx_prof_begin(ctx, name);                                          \
        const int rv_ = (int)(call);                                                       \
        ctx_prof_end(ctx, h_);                                                             \
        if (rv_ != 0)                                                                      \
            return kfail(ctx, TBS_ERR_CUDA,                                                \
                         std::string(name) + ": " + cudaGetErrorString((cudaError_t)rv_)); \
    } while (0)

static void krylov_free_vectors(KrylovBufs *k) {
    for (void *p : k->allocs) cudaFree(p);
    k->allocs.clear();
    k->bytes = 0;
    k->V = k->Z = k->w = k->partials = k->h = k->h2 = k->y = nullptr;
    k->m = 0;
    k->n = 0;
}

void krylov_free(tbs_ctx *ctx) {
    if (!ctx || !ctx->krylov) return;
    krylov_free_vectors(ctx->krylov);
    if (ctx->krylov->h_host) cudaFreeHost(ctx->krylov->h_host);
    delete ctx->krylov;
    ctx->krylov = nullptr;
}

size_t krylov_bytes(const tbs_ctx *ctx) { return ctx && ctx->krylov ? ctx->krylov->bytes : 0; }

template <typename T>
static int kalloc(tbs_ctx *ctx, KrylovBufs *k, T **p, size_t count) {
    const size_t nbytes = std::max<size_t>(count, 1) * sizeof(T);
    void *q = nullptr;
    if (cudaMalloc(&q, nbytes) != cudaSuccess) {
        cudaGetLastError();
        return kfail(ctx, TBS_ERR_NOMEM, "cudaMalloc of " + std::to_string(nbytes) + " bytes failed");
    }
    k->allocs.push_back(q);
    k->bytes += nbytes;
    *p = static_cast<T *>(q);
    KCK(cudaMemsetAsync(q, 0, nbytes, ctx->stream)); /* pads stay zero */
    return TBS_OK;
}

#define KA(ptr, cnt)                                 \
    do {                                             \
        int s_ = kalloc(ctx, k, &(ptr), (cnt));      \
        if (s_) return s_;                           \
    } while (0)

static int krylov_ensure(tbs_ctx *ctx, int m) {
    if (!ctx->krylov) {
        ctx->krylov = new KrylovBufs();
        if (cudaMallocHost((void **)&ctx->krylov->h_host, 2 * (KRYLOV_MAX + 2) * sizeof(double)) !=
            cudaSuccess) {
            cudaGetLastError();
            krylov_free(ctx);
            return kfail(ctx, TBS_ERR_NOMEM, "pinned host allocation failed");
        }
    }
    KrylovBufs *k = ctx->krylov;
    const long long n = (long long)ctx->L.np16 * 9;
    if (k->m >= m && k->n == n) return TBS_OK;
    KCK(cudaStreamSynchronize(ctx->stream));
    m = std::max(m, k->n == n ? k->m : 0);
    krylov_free_vectors(k);
    KA(k->V, (size_t)(m + 1) * n);
    KA(k->Z, (size_t)m * n);
    KA(k->w, (size_t)n);
    KA(k->partials, (size_t)(KRYLOV_MAX + 2) * KR_BLOCKS);
    KA(k->h, (size_t)KRYLOV_MAX + 2);
    KA(k->h2, (size_t)KRYLOV_MAX + 2);
    KA(k->y, (size_t)KRYLOV_MAX + 2);
    k->m = m;
    k->n = n;
    return TBS_OK;
}

/* out[0..count) (+ w.w at out[count] when self) on the device */
static int dots(tbs_ctx *ctx, const double *w, const double *V, int count, int self, double *out) {
    KrylovBufs *k = ctx->krylov;
    KRUN("kr_dots", (kr_dots_kernel<<<KR_BLOCKS, KR_THREADS, 0, ctx->stream>>>(
                         k->n, w, V, k->n, count, self, k->partials),
                     cudaGetLastError()));
    KRUN("kr_dots", (kr_reduce_kernel<<<count + (self ? 1 : 0), KR_THREADS, 0, ctx->stream>>>(
                         k->partials, out),
                     cudaGetLastError()));
    return TBS_OK;
}

static int combine(tbs_ctx *ctx, double *x, const double *V, int count, const double *coef,
                   double sign) {
    KrylovBufs *k = ctx->krylov;
    KRUN("kr_combine", (kr_combine_kernel<<<148 * 8, KR_THREADS, 0, ctx->stream>>>(
                            k->n, x, V, k->n, count, coef, sign),
                        cudaGetLastError()));
    return TBS_OK;
}

static int scale(tbs_ctx *ctx, double *dst, const double *src, double a) {
    KrylovBufs *k = ctx->krylov;
    KRUN("kr_scale", (kr_scale_kernel<<<148 * 8, KR_THREADS, 0, ctx->stream>>>(k->n, dst, src, a),
                      cudaGetLastError()));
    return TBS_OK;
}

/* z = P v: `sweeps` LIJ sweeps from zero on v + J z = 0 (TBS_ALGO_FP64),
 * and w = J z.  The sweeps track their residual R = v + J z recursively
 * (R = sum of the cross-line blocks times the last update, exact for exact
 * line solves), so the last sweep's residual launch gives J z = R - v
 * without a separate product with J. */
static int precond_product(tbs_ctx *ctx, const double *v, double *z, double *w, int sweeps) {
    cudaStream_t st = ctx->stream;
    const FastLayout &L = ctx->L;
    const NormSink none{};
    /* b = -Dinv v, z = 0 */
    KRUN("fast_resid_rhs", launch_fast_resid<double>(st, L, 0, ctx->d_Dinv, ctx->d_X, ctx->d_dUp, v,
                                                     ctx->d_b, none, ctx->d_status, z));
    /* each line solve adds its update to z as it writes it */
    for (int s = 0; s < sweeps; ++s) {
        KRUN("fast_thomas", launch_fast_thomas<double>(st, L, ctx->d_G, ctx->d_Gam, ctx->d_b, ctx->d_y,
                                                       ctx->d_dUp, z, ctx->d_status, 1));
        if (s + 1 < sweeps)
            KRUN("fast_resid", launch_fast_resid<double>(st, L, 1, ctx->d_Dinv, ctx->d_X, ctx->d_dUp,
                                                         nullptr, ctx->d_b, none, ctx->d_status,
                                                         nullptr));
        else
            KRUN("fast_resid_jv", launch_fast_resid<double>(st, L, 4, nullptr, ctx->d_X, ctx->d_dUp, v,
                                                            w, none, ctx->d_status, nullptr));
    }
    return TBS_OK;
}

/* w = rhs + J z from the original blocks (the true residual) */
static int matvec(tbs_ctx *ctx, const double *z, double *w, const double *rhs_elem) {
    KRUN("full_resid", launch_full_resid<double>(ctx->stream, ctx->nelem, ctx->d_epoint, ctx->d_ef,
                                                 ctx->d_fc, ctx->L.pos_of_elem, ctx->d_jacD, ctx->d_O1,
                                                 ctx->d_O2, rhs_elem, z, w, ctx->d_partials2));
    return TBS_OK;
}

static int read_back(tbs_ctx *ctx, const double *d, int count, double *host) {
    KCK(cudaMemcpyAsync(host, d, count * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    KCK(cudaStreamSynchronize(ctx->stream));
    return TBS_OK;
}

static int gmres(tbs_ctx *ctx, int m, int psweeps, double tol, int max_iters, int *iters_out,
                 double *hist) {
    int rc = krylov_ensure(ctx, m);
    if (rc) return rc;
    KrylovBufs *k = ctx->krylov;
    cudaStream_t st = ctx->stream;
    const long long n = k->n;
    double *hh = k->h_host;
    int iters = 0;
    /* U = 0; R = rhs (position order) */
    KCK(cudaMemsetAsync(ctx->d_Up, 0, (size_t)n * sizeof(double), st));
    KCK((cudaError_t)xfer_copy(st, ctx->d_rhsp, k->w, (size_t)n * sizeof(double), 0));
    rc = dots(ctx, k->w, nullptr, 0, 1, k->h);
    if (rc) return rc;
    rc = read_back(ctx, k->h, 1, hh);
    if (rc) return rc;
    const double beta0 = std::sqrt(hh[0]);
    if (hist) hist[0] = beta0;
    double beta = beta0;
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    while (beta > tol * beta0 && std::isfinite(beta) && iters < max_iters) {
        /* V_0 = -R / beta (A y = -rhs - J U = -R) */
        rc = scale(ctx, k->V, k->w, -1.0 / beta);
        if (rc) return rc;
        std::fill(H.begin(), H.end(), 0.0);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        bool stop = false;
        for (; j < m && !stop; ++j) {
            double *Vj = k->V + (size_t)j * n;
            double *Zj = k->Z + (size_t)j * n;
            rc = precond_product(ctx, Vj, Zj, k->w, psweeps);
            if (rc) return rc;
            /* classical Gram-Schmidt, twice; the second pass also gives w.w */
            rc = dots(ctx, k->w, k->V, j + 1, 0, k->h);
            if (rc) return rc;
            rc = combine(ctx, k->w, k->V, j + 1, k->h, -1.0);
            if (rc) return rc;
            rc = dots(ctx, k->w, k->V, j + 1, 1, k->h2);
            if (rc) return rc;
            rc = combine(ctx, k->w, k->V, j + 1, k->h2, -1.0);
            if (rc) return rc;
            KCK(cudaMemcpyAsync(hh, k->h, (j + 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
            rc = read_back(ctx, k->h2, j + 2, hh + KRYLOV_MAX + 2);
            if (rc) return rc;
            const double *h1 = hh, *h2 = hh + KRYLOV_MAX + 2;
            double ww = h2[j + 1], s2 = 0.0;
            for (int i = 0; i <= j; ++i) {
                H[(size_t)i * m + j] = h1[i] + h2[i];
                s2 += h2[i] * h2[i];
            }
            const double hn = std::sqrt(std::max(ww - s2, 0.0));
            H[(size_t)(j + 1) * m + j] = hn;
            /* previous rotations on column j, then a new one */
            for (int i = 0; i < j; ++i) {
                const double a = H[(size_t)i * m + j], b = H[(size_t)(i + 1) * m + j];
                H[(size_t)i * m + j] = cs[i] * a + sn[i] * b;
                H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * b;
            }
            const double a = H[(size_t)j * m + j], b = H[(size_t)(j + 1) * m + j];
            const double r = std::hypot(a, b);
            cs[j] = r > 0.0 ? a / r : 1.0;
            sn[j] = r > 0.0 ? b / r : 0.0;
            H[(size_t)j * m + j] = r;
            H[(size_t)(j + 1) * m + j] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            ++iters;
            const double res = std::fabs(g[j + 1]);
            if (hist) hist[iters] = res;
            if (res <= tol * beta0 || iters >= max_iters || !(hn > 0.0) || !std::isfinite(res))
                stop = true;
            else if (j + 1 < m) {
                rc = scale(ctx, k->V + (size_t)(j + 1) * n, k->w, 1.0 / hn);
                if (rc) return rc;
            }
        }
        /* y = R^-1 g (upper triangular, the rotated H), U += sum y_i z_i */
        for (int i = j - 1; i >= 0; --i) {
            double s = g[i];
            for (int c = i + 1; c < j; ++c) s -= H[(size_t)i * m + c] * y[c];
            const double d = H[(size_t)i * m + i];
            y[i] = d != 0.0 ? s / d : 0.0;
        }
        KCK(cudaMemcpyAsync(k->y, y.data(), j * sizeof(double), cudaMemcpyHostToDevice, st));
        rc = combine(ctx, ctx->d_Up, k->Z, j, k->y, 1.0);
        if (rc) return rc;
        /* the true residual R = rhs + J U opens the next cycle */
        rc = matvec(ctx, ctx->d_Up, k->w, ctx->d_rhs);
        if (rc) return rc;
        rc = dots(ctx, k->w, nullptr, 0, 1, k->h);
        if (rc) return rc;
        rc = read_back(ctx, k->h, 1, hh);
        if (rc) return rc;
        beta = std::sqrt(hh[0]);
        if (hist) hist[iters] = beta; /* the estimate replaced by the true norm */
    }
    if (iters_out) *iters_out = iters;
    /* the solve state: sweeps = Arnoldi steps, norms of the true residual */
    SolveState *S = ctx->h_state;
    std::memset(S, 0, sizeof(*S));
    S->norm0 = beta0;
    S->last = beta;
    S->sweep = iters;
    S->tol = tol;
    S->max_sweeps = max_iters;
    S->hist_cap = ctx->hist_cap;
    KCK(cudaMemcpyAsync(ctx->d_state, S, sizeof(SolveState), cudaMemcpyHostToDevice, st));
    KCK(cudaStreamSynchronize(st));
    if (ctx->prof) ctx_prof_resolve(ctx);
    return ctx_status(ctx);
}

extern "C" int tbs_gmres(tbs_ctx *ctx, int restart, int precond_sweeps, double rel_tol,
                         int max_iters, int *iters_out, double *hist_out) {
    if (!ctx) return kfail(nullptr, TBS_ERR_ARG, "null context");
    try {
        if (cudaSetDevice(ctx->device) != cudaSuccess)
            return kfail(ctx, TBS_ERR_CUDA, "cudaSetDevice failed");
        if (!ctx->factored) return kfail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
        if (ctx->algo != TBS_ALGO_FP64 || ctx->nvar != 9)
            return kfail(ctx, TBS_ERR_UNSUPPORTED,
                         "GMRES uses the TBS_ALGO_FP64 line factors of nvar == 9");
        if (ctx->lagged)
            return kfail(ctx, TBS_ERR_UNSUPPORTED,
                         "block values are newer than the factorization (tbs_update_values); GMRES "
                         "forms its products with J from the factorization's blocks: re-factor");
        if (ctx->nhalo > 0) return kfail(ctx, TBS_ERR_UNSUPPORTED, "a line partition sweeps with tbs_part_solve_du / tbs_part_line_res");
        if (restart < 1 || restart > KRYLOV_MAX || precond_sweeps < 1 || max_iters < 0 ||
            !(rel_tol >= 0.0))
            return kfail(ctx, TBS_ERR_ARG, "bad restart (1..64), preconditioner sweeps, "
                                           "iteration limit or tolerance");
        return gmres(ctx, restart, precond_sweeps, rel_tol, max_iters, iters_out, hist_out);
    } catch (const std::bad_alloc &) {
        return kfail(ctx, TBS_ERR_NOMEM, "host allocation failed");
    } catch (...) {
        return kfail(ctx, TBS_ERR_STATE, "internal error");
    }
}

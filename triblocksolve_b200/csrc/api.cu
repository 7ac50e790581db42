/*
 * api.cu -- the tbs_* solver entry points: device context, memory, the
 * line-ordered layout, and the launch sequences of the three algorithms.
 *
 * Reference flow replaced (src/main.cxx):
 *   Platform gpu(...)              :80    -> tbs_create
 *   mesh.setupDevice/toDevice      :84-85 -> tbs_set_mesh
 *   Jac.setupDevice/toDevice       :92-93 -> tbs_set_jacobian
 *   copyAtoBjac + lineLU_v2        :180-190 -> tbs_factor
 *   copyAtoB; loop{solveDU; addAtoB; copyAtoB; lineRes} :201-229
 *                                  -> tbs_sweep / tbs_solve
 * tbs_solve runs the sweep loop as one CUDA graph whose while-node is
 * driven by a device-side convergence test, so a solve costs one launch.
 */
#include "ctx.hxx"

#include <cuda_runtime.h>

#include <algorithm>
#include <utility>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <cstdlib>
#include <new>
#include <string>
#include <vector>

using namespace tbs;

/* ================================================================ errors */

static int ctx_fail(tbs_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    set_thread_error(msg);
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return ctx_fail(ctx, TBS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CKL(call)                                                                         \
    do {                                                                                  \
        int e_ = (call);                                                                  \
        if (e_ != 0)                                                                      \
            return ctx_fail(ctx, TBS_ERR_CUDA,                                            \
                            std::string(#call) + ": " + cudaGetErrorString((cudaError_t)e_)); \
    } while (0)

#define GUARD_BEGIN try {
#define GUARD_END                                                                        \
    }                                                                                     \
    catch (const std::bad_alloc &) {                                                      \
        return ctx_fail(ctx, TBS_ERR_NOMEM, "host allocation failed");                    \
    }                                                                                     \
    catch (const std::exception &ex) {                                                    \
        return ctx_fail(ctx, TBS_ERR_STATE, std::string("internal error: ") + ex.what()); \
    }                                                                                     \
    catch (...) {                                                                         \
        return ctx_fail(ctx, TBS_ERR_STATE, "internal error");                            \
    }

/* ================================================================ memory */

template <typename T>
static int dalloc(tbs_ctx *ctx, T **p, size_t count) {
    if (*p) return TBS_OK;
    size_t nbytes = std::max<size_t>(count, 1) * sizeof(T);
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, nbytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_fail(ctx, TBS_ERR_NOMEM,
                        "cudaMalloc of " + std::to_string(nbytes) + " bytes failed: " +
                            cudaGetErrorString(e));
    }
    e = cudaMemsetAsync(q, 0, nbytes, ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(q);
        return ctx_fail(ctx, TBS_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    }
    ctx->allocs.push_back({q, nbytes});
    ctx->bytes += nbytes;
    *p = static_cast<T *>(q);
    return TBS_OK;
}

template <typename T>
static void dfree(tbs_ctx *ctx, T **p) {
    if (!*p) return;
    for (size_t i = 0; i < ctx->allocs.size(); ++i) {
        if (ctx->allocs[i].first == (void *)*p) {
            ctx->bytes -= ctx->allocs[i].second;
            ctx->allocs.erase(ctx->allocs.begin() + i);
            break;
        }
    }
    cudaFree(*p);
    *p = nullptr;
}

#define DA(ptr, n)                          \
    do {                                    \
        int s_ = dalloc(ctx, &(ptr), (n));  \
        if (s_) return s_;                  \
    } while (0)

static void drop_graph(tbs_ctx *ctx) {
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    if (ctx->graph) cudaGraphDestroy(ctx->graph);
    ctx->gexec = nullptr;
    ctx->graph = nullptr;
    ctx->graph_algo = -1;
}

/* free everything that depends on the mesh */
static void drop_mesh(tbs_ctx *ctx) {
    if (ctx->copy) cudaStreamSynchronize(ctx->copy); /* a staged upload may be in flight */
    multi_free(ctx);
    krylov_free(ctx);
    drop_graph(ctx);
    for (auto &slot : ctx->d_land)
        for (auto &p : slot) p = nullptr; /* freed with the other allocations below */
    ctx->land_count = 0;
    ctx->land_head = 0;
    for (auto &a : ctx->allocs) cudaFree(a.first);
    ctx->allocs.clear();
    ctx->bytes = 0;
    double **dps[] = {&ctx->d_jacD, &ctx->d_O1, &ctx->d_O2, &ctx->d_rhs, &ctx->d_U, &ctx->d_dU,
                      &ctx->d_R, &ctx->d_Uinit, &ctx->d_scratch, &ctx->d_DLU, &ctx->d_DinvC,
                      &ctx->d_A, &ctx->d_Dinv, &ctx->d_G, &ctx->d_Gam, &ctx->d_X, &ctx->d_Up,
                      &ctx->d_Up_alt, &ctx->d_dUp, &ctx->d_b, &ctx->d_y, &ctx->d_rhsp, &ctx->d_Rp,
                      &ctx->d_partials, &ctx->d_partials2, &ctx->d_hist, &ctx->d_gamlast,
                      &ctx->d_Dp, &ctx->d_XF};
    for (auto p : dps) *p = nullptr;
    float **fps[] = {&ctx->d_Dinv32, &ctx->d_G32, &ctx->d_Gam32, &ctx->d_X32, &ctx->d_b32,
                     &ctx->d_y32, &ctx->d_d32, &ctx->d_c32, &ctx->d_R32};
    for (auto p : fps) *p = nullptr;
    int **ips[] = {&ctx->d_epoint, &ctx->d_ef, &ctx->d_fc, &ctx->d_linesize, &ctx->d_linepoint,
                   &ctx->d_lines, &ctx->d_lineface, &ctx->d_identity, &ctx->L.line_start,
                   &ctx->L.line_len, &ctx->L.line_twist, &ctx->L.pos_of_elem, &ctx->L.elem_of_pos, &ctx->L.xnbr,
                   &ctx->L.xsrc, &ctx->L.fsrc, &ctx->L.xsrcf, &ctx->L.xnbrf};
    for (auto p : ips) *p = nullptr;
    ctx->d_state = nullptr;
    ctx->d_status = nullptr;
    ctx->d_ktimer = nullptr;
    ctx->d_counter = nullptr;
    ctx->npart_cap = 0;
    ctx->hist_cap = 0;
    ctx->have_mesh = ctx->have_jac = ctx->factored = false;
    ctx->layout_ok = false;
    ctx->algo = -1;
}

/* ============================================================= profiling */

static int prof_slot(tbs_ctx *ctx, const char *name) {
    for (size_t i = 0; i < ctx->slots.size(); ++i)
        if (std::strcmp(ctx->slots[i].name, name) == 0) return (int)i;
    if (ctx->slots.size() >= TBS_PROFILE_MAX) return -1;
    ctx->slots.push_back({name, 0, 0.0});
    return (int)ctx->slots.size() - 1;
}

static cudaEvent_t prof_event(tbs_ctx *ctx) {
    if (!ctx->pool.empty()) {
        cudaEvent_t e = ctx->pool.back();
        ctx->pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

static void prof_resolve(tbs_ctx *ctx) {
    if (ctx->pending.empty()) return;
    cudaStreamSynchronize(ctx->stream);
    for (auto &p : ctx->pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess && p.slot >= 0) {
            ctx->slots[p.slot].ms += ms;
            ctx->slots[p.slot].launches += 1;
        }
        ctx->pool.push_back(p.a);
        ctx->pool.push_back(p.b);
    }
    ctx->pending.clear();
}

static bool capturing(tbs_ctx *ctx) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(ctx->stream, &cs);
    return cs != cudaStreamCaptureStatusNone;
}

/* run one launch, bracketed by events when profiling */
template <typename F>
static int timed(tbs_ctx *ctx, const char *name, F &&launch) {
    if (!ctx->prof || capturing(ctx)) return launch();
    if (ctx->pending.size() > 4000) prof_resolve(ctx);
    PendingEvent pe{prof_slot(ctx, name), prof_event(ctx), prof_event(ctx)};
    cudaEventRecord(pe.a, ctx->stream);
    int rc = launch();
    cudaEventRecord(pe.b, ctx->stream);
    ctx->pending.push_back(pe);
    return rc;
}

#define RUN(name, call) CKL(timed(ctx, name, [&]() { return (int)(call); }))

/* ======================================== host transfers off the copy engine
 * A cudaMemcpyAsync between host and device waits in the copy engine's
 * queue behind every copy issued before it: a 5 GB staged Jacobian
 * (tbs_stage_jacobian) would hold a solve's 32-byte control block for the
 * whole upload.  So the solve and factorization paths move their small
 * words with kernels (xfer.cu): the control block as kernel parameters,
 * the state, status and history into mapped pinned host memory, and a
 * result into the caller's buffer when that is pinned host memory the
 * device can address. */
__global__ void set_state_kernel(SolveState *s, double tol, int max_sweeps, int hist_cap) {
    s->tol = tol;
    s->max_sweeps = max_sweeps;
    s->hist_cap = hist_cap;
}

/* device -> device (or into mapped host memory) on the SMs */
static int copy_words(cudaStream_t st, const void *src, void *dst, size_t bytes) {
    return xfer_copy(st, src, dst, bytes, 0);
}

/* device -> host of `bytes`: a kernel when the destination is
 * device-addressable pinned memory, else a copy (which may queue behind a
 * staged upload) */
static int to_host(tbs_ctx *ctx, void *dst, const void *src, size_t bytes) {
    CKL(xfer_to_host(ctx->stream, dst, src, bytes, 0));
    return TBS_OK;
}

/* the mapped host copy of the history, at least n doubles */
static int ensure_h_hist(tbs_ctx *ctx, int n) {
    if (n <= ctx->h_hist_cap) return TBS_OK;
    if (ctx->h_hist) cudaFreeHost(ctx->h_hist);
    ctx->h_hist = nullptr;
    ctx->h_hist_dev = nullptr;
    ctx->h_hist_cap = 0;
    const int cap = std::max(n, 1024);
    CK(cudaHostAlloc((void **)&ctx->h_hist, (size_t)cap * sizeof(double), cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer((void **)&ctx->h_hist_dev, ctx->h_hist, 0));
    ctx->h_hist_cap = cap;
    return TBS_OK;
}

/* the first n norms of the device history into `out` (host) */
static int hist_to_host(tbs_ctx *ctx, double *out, int n) {
    int rc = ensure_h_hist(ctx, n);
    if (rc) return rc;
    CKL(copy_words(ctx->stream, ctx->d_hist, ctx->h_hist_dev, (size_t)n * sizeof(double)));
    CK(cudaStreamSynchronize(ctx->stream));
    std::memcpy(out, ctx->h_hist, (size_t)n * sizeof(double));
    return TBS_OK;
}

int ctx_prof_begin(tbs_ctx *ctx, const char *name) {
    if (!ctx->prof || capturing(ctx)) return -1;
    if (ctx->pending.size() > 4000) prof_resolve(ctx);
    PendingEvent pe{prof_slot(ctx, name), prof_event(ctx), prof_event(ctx)};
    cudaEventRecord(pe.a, ctx->stream);
    ctx->pending.push_back(pe);
    return (int)ctx->pending.size() - 1;
}

void ctx_prof_end(tbs_ctx *ctx, int h) {
    if (h >= 0 && h < (int)ctx->pending.size()) cudaEventRecord(ctx->pending[h].b, ctx->stream);
}

void ctx_prof_resolve(tbs_ctx *ctx) { prof_resolve(ctx); }

/* ============================================================ layout (host) */

static int build_layout(tbs_ctx *ctx) {
    const int nline = ctx->nline, nelem = ctx->nelem;
    const int *ls = ctx->h_linesize.data(), *lp = ctx->h_linepoint.data();
    const int *lines = ctx->h_lines.data(), *lf = ctx->h_lineface.data();
    const int *fc = ctx->h_fc.data(), *ep = ctx->h_epoint.data(), *ef = ctx->h_ef.data();
    std::vector<int> start(nline), len(nline), twist(nline);
    long long np = 0;
    const int nown = nline - ctx->nhalo;
    long long np_own = 0;
    for (int l = 0; l < nline; ++l) {
        if (l == nown) {
            /* halo lines start on a tile boundary: no residual tile mixes
             * owned and halo cells, so the norm can stop at the owned tiles */
            np = (np + RES_TILE - 1) / RES_TILE * RES_TILE;
            np_own = np;
        }
        start[l] = (int)np;
        len[l] = ls[l];
        twist[l] = line_twist_of(ls[l]);
        np += (ls[l] + 3) & ~3;
    }
    if (np > 0x7fffffffLL / ((long long)ctx->nvar * ctx->nvar))
        return ctx_fail(ctx, TBS_ERR_UNSUPPORTED, "mesh too large for int32 block offsets");
    const int np16 = (int)((np + RES_TILE - 1) / RES_TILE * RES_TILE);
    std::vector<int> pos_of_elem(nelem), elem_of_pos(np16, -1), fsrc((size_t)np16 * 5, -1);
    auto side_of = [&](int e, int f) { return (e == fc[2 * f]) ? 1 : 0; };
    for (int l = 0; l < nline; ++l) {
        const int n = ls[l], m = twist[l], ps = start[l];
        for (int k = 0; k < n; ++k) {
            const int e = lines[lp[l] + k];
            const int p = (k < m) ? ps + k : (k > m) ? ps + m + (n - 1 - k) : ps + n - 1;
            pos_of_elem[e] = p;
            elem_of_pos[p] = e;
            int *fs = &fsrc[5 * (size_t)p];
            fs[0] = e;
            if (k < m) { /* top chain: predecessor k-1 */
                if (k >= 1) {
                    fs[1] = lf[lp[l] + k];
                    fs[2] = side_of(e, fs[1]);
                }
            } else if (k > m) { /* bottom chain: predecessor k+1 */
                if (k + 1 < n) {
                    fs[1] = lf[lp[l] + k + 1];
                    fs[2] = side_of(e, fs[1]);
                }
            } else { /* twist: faces to m-1 and m+1 */
                if (m >= 1) {
                    fs[1] = lf[lp[l] + m];
                    fs[2] = side_of(e, fs[1]);
                }
                if (m + 1 < n) {
                    fs[3] = lf[lp[l] + m + 1];
                    fs[4] = side_of(e, fs[3]);
                }
            }
        }
    }
    /* cross-line slots: every interior face of the cell that is not one of
     * the (at most two) in-line faces used by the line factorization */
    std::vector<std::vector<std::pair<int, int>>> xs(np16);
    int nx = 0;
    long long nreal = 0;
    for (int l = 0; l < nline; ++l) {
        for (int k = 0; k < ls[l]; ++k) {
            const int m = lp[l] + k, e = lines[m], p = pos_of_elem[e];
            int fprev = (k >= 1) ? lf[m] : -1;
            int fnext = (k + 1 < ls[l]) ? lf[m + 1] : -1;
            auto &v = xs[p];
            for (int k2 = ep[e]; k2 < ep[e + 1]; ++k2) {
                const int f = ef[k2];
                if (f < 0) continue;
                if (f == fprev) {
                    fprev = -2;
                    continue;
                }
                if (f == fnext) {
                    fnext = -2;
                    continue;
                }
                const bool is1 = (e == fc[2 * f]);
                const int nb = is1 ? fc[2 * f + 1] : fc[2 * f];
                v.push_back({2 * f + (is1 ? 1 : 0), pos_of_elem[nb]});
            }
            nx = std::max<int>(nx, (int)v.size());
            nreal += (long long)v.size();
        }
    }
    std::vector<int> xsrc((size_t)np16 * std::max(nx, 1), -1), xnbr((size_t)np16 * std::max(nx, 1), -1);
    for (int p = 0; p < np16; ++p)
        for (size_t q = 0; q < xs[p].size(); ++q) {
            xsrc[q * (size_t)np16 + p] = xs[p][q].first;
            xnbr[q * (size_t)np16 + p] = xs[p][q].second;
        }
    /* all-face slots (in-line and cross-line, ef order): the full residual
     * in position order (TBS_ALGO_MIXED's outer residual) */
    int nxf = 0;
    long long nfreal = 0;
    for (int e = 0; e < nelem; ++e) {
        int cnt = 0;
        for (int k2 = ep[e]; k2 < ep[e + 1]; ++k2) cnt += ef[k2] >= 0;
        nxf = std::max(nxf, cnt);
        nfreal += cnt;
    }
    const int nxfa = std::max(nxf, 1);
    std::vector<int> xsrcf((size_t)np16 * nxfa, -1), xnbrf((size_t)np16 * nxfa, -1);
    for (int e = 0; e < nelem; ++e) {
        const int p = pos_of_elem[e];
        int q = 0;
        for (int k2 = ep[e]; k2 < ep[e + 1]; ++k2) {
            const int f = ef[k2];
            if (f < 0) continue;
            const bool is1 = (e == fc[2 * f]);
            xsrcf[q * (size_t)np16 + p] = 2 * f + (is1 ? 1 : 0);
            xnbrf[q * (size_t)np16 + p] = pos_of_elem[is1 ? fc[2 * f + 1] : fc[2 * f]];
            ++q;
        }
    }
    FastLayout &L = ctx->L;
    L.nv = ctx->nvar;
    L.np = (int)np;
    L.np16 = np16;
    L.ntile_own = (ctx->nhalo > 0 ? (int)np_own : np16) / RES_TILE;
    ctx->h_line_start = start;
    L.nx = nx;
    L.nxf = nxf;
    L.nline = nline;
    L.max_len = ctx->max_line;
    ctx->n_xslots_real = nreal;
    ctx->n_fslots_real = nfreal;
    DA(L.line_start, nline);
    DA(L.line_len, nline);
    DA(L.line_twist, nline);
    DA(L.pos_of_elem, nelem);
    DA(L.elem_of_pos, np16);
    DA(L.fsrc, (size_t)np16 * 5);
    DA(L.xsrc, (size_t)np16 * std::max(nx, 1));
    DA(L.xnbr, (size_t)np16 * std::max(nx, 1));
    DA(L.xsrcf, (size_t)np16 * nxfa);
    DA(L.xnbrf, (size_t)np16 * nxfa);
    DA(ctx->d_gamlast, (size_t)nline * 2 * ctx->nvar * ctx->nvar);
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(L.line_start, start.data(), nline * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.line_len, len.data(), nline * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.line_twist, twist.data(), nline * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.pos_of_elem, pos_of_elem.data(), nelem * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.elem_of_pos, elem_of_pos.data(), np16 * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.fsrc, fsrc.data(), fsrc.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.xsrc, xsrc.data(), xsrc.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.xnbr, xnbr.data(), xnbr.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.xsrcf, xsrcf.data(), xsrcf.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.xnbrf, xnbrf.data(), xnbrf.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    /* the residual kernel stages RES_TILE cells x nx blocks per tile; beyond
     * 4 cross-line couplings per cell it would not fit in shared memory,
     * and such meshes use TBS_ALGO_REFERENCE */
    ctx->layout_ok = (ctx->nvar == 9 || nv_supported(ctx->nvar)) && nx <= 4;
    return TBS_OK;
}

/* ============================================================ sequences */

/* the error of a status word read from the device (0: none); clears it */
static int status_error(tbs_ctx *ctx, unsigned s) {
    if (s) {
        CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned), ctx->stream));
        if (ctx->d_counter) CK(cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned), ctx->stream));
        if (s & ST_PIVOT)
            return ctx_fail(ctx, TBS_ERR_NUMERIC,
                            "zero or non-finite pivot in the no-pivot block factorization");
        if (s & ST_TIMEOUT)
            return ctx_fail(ctx, TBS_ERR_CUDA, "a device-side wait ran out of its time budget");
        return ctx_fail(ctx, TBS_ERR_CUDA, "device status " + std::to_string(s));
    }
    return TBS_OK;
}

static int status_check(tbs_ctx *ctx) {
    /* the status word (4 bytes) travels in an 8-byte copy: h_status and
     * d_status are 8-byte allocations */
    CKL(copy_words(ctx->stream, ctx->d_status, ctx->h_status_dev, 8));
    CK(cudaStreamSynchronize(ctx->stream));
    return status_error(ctx, *ctx->h_status);
}

int ctx_status(tbs_ctx *ctx) { return status_check(ctx); }

/* Everything a finished solve reports, in one launch and one
 * synchronisation: the state, the status word and the first nh norms of the
 * history, into the context's mapped host memory. */
__global__ void solve_readback_kernel(const SolveState *__restrict__ st,
                                      const unsigned long long *__restrict__ status,
                                      const double *__restrict__ hist, int nh, SolveState *o_state,
                                      unsigned long long *o_status, double *o_hist) {
    if (threadIdx.x == 0) {
        *o_state = *st;
        *o_status = *status;
    }
    for (int t = threadIdx.x; t < nh; t += blockDim.x) o_hist[t] = hist[t];
}

static long long nvec(tbs_ctx *ctx) { return (long long)ctx->nvar * ctx->nelem; }

/* TBS_ALGO_MIXED's outer residual streams position-ordered copies of the
 * blocks when a cell has at most 4 interior faces (one shared-memory tile) */
bool fullpos_ok(const tbs_ctx *ctx) { return ctx->L.nxf <= 4; }


/* The TBS_ALGO_FP64 sweep kernels for the context's block size: the tuned
 * size-9 kernels or their general form (kernels_nv.cu). */
static int thomas64(tbs_ctx *ctx, const double *b, double *dU, double *U, int accumulate) {
    if (ctx->nvar == 9)
        return launch_fast_thomas<double>(ctx->stream, ctx->L, ctx->d_G, ctx->d_Gam, b, ctx->d_y, dU, U,
                                          ctx->d_status, accumulate);
    return launch_nv_thomas(ctx->stream, ctx->nvar, ctx->L, ctx->d_G, ctx->d_Gam, b, ctx->d_y, dU, U,
                            accumulate, ctx->d_status);
}

static int resid64(tbs_ctx *ctx, int mode, const double *dU, const double *Rsrc, double *b,
                   const NormSink &ns, double *Uacc) {
    if (ctx->nvar == 9) {
        /* the sweeps' residual launches keep a device-clock record of their
         * durations (tbs_resid_timer), graph-launched ones included */
        NormSink nt = ns;
        if (mode == 1) nt.timer = ctx->d_ktimer;
        return launch_fast_resid<double>(ctx->stream, ctx->L, mode, ctx->d_Dinv, ctx->d_X, dU, Rsrc, b,
                                         nt, ctx->d_status, Uacc);
    }
    return launch_nv_resid(ctx->stream, ctx->nvar, ctx->L, mode, ctx->d_Dinv, ctx->d_X, dU, Rsrc, b, ns,
                           ctx->d_status, Uacc);
}

/* R = rhs + J U in element order by the reference-order residual kernel
 * (any block size); U in element order */
/* R = rhs + J U in element order, its norm partials in d_partials2 (*np_out
 * of them, may be null) */
static int ref_residual(tbs_ctx *ctx, const double *U, double *R, int *np_out = nullptr) {
    int np = 0;
    CKL(copy_words(ctx->stream, ctx->d_rhs, R, (size_t)ctx->nvar * ctx->nelem * sizeof(double)));
    CKL(launch_ref_line_res(ctx->stream, ctx->nvar, ctx->nline, ctx->nelem, ctx->d_epoint, ctx->d_ef,
                            ctx->d_fc, ctx->d_linesize, ctx->d_linepoint, ctx->d_lines, ctx->d_jacD,
                            ctx->d_O1, ctx->d_O2, U, R, ctx->d_partials2, &np));
    if (np_out) *np_out = np;
    return TBS_OK;
}

/* How a sequence ends: the norm of its residual is recorded as the start
 * of a solve (is_start) or as one more sweep, and, inside the solve graph,
 * sets the while-node's condition. */
struct CondCtl {
    unsigned long long handle;
    int use_cond;
    unsigned long long handle2; /* a second condition set to the same value (0: none) */
    int use2;
    unsigned long long check;   /* set to 1 when a sweep's recursive residual meets the
                                 * tolerance (the true-residual check's IF node) */
    int use_check;
};

static NormSink sink(tbs_ctx *ctx, int is_start, CondCtl cc) {
    NormSink ns{};
    ns.partials = ctx->d_partials;
    ns.counter = ctx->d_counter;
    ns.state = ctx->d_state;
    ns.hist = ctx->d_hist;
    ns.is_start = is_start;
    ns.use_cond = cc.use_cond;
    ns.handle = cc.handle;
    ns.ntiles = ctx->nhalo > 0 ? ctx->L.ntile_own : 0;
    ns.use_check = cc.use_check;
    ns.check_handle = cc.check;
    return ns;
}

static NormSink no_sink() { return NormSink{}; }

static int reduce(tbs_ctx *ctx, int npart, int is_start, CondCtl cc) {
    RUN("reduce_norm", launch_reduce_norm(ctx->stream, ctx->d_partials, npart, ctx->d_state,
                                          ctx->d_hist, is_start, cc.handle, cc.use_cond, cc.handle2,
                                          cc.use2));
    return TBS_OK;
}

/* Bring the state to "U = U_init, residual of U known and recorded as
 * ||R_0||", with the first sweep's inputs ready. */
static int prime(tbs_ctx *ctx, CondCtl cc) {
    cudaStream_t st = ctx->stream;
    ctx->outer_done = 0;
    const int nv = ctx->nvar, ne = ctx->nelem;
    const size_t vb = (size_t)nvec(ctx) * sizeof(double);
    if (ctx->algo == TBS_ALGO_REFERENCE) {
        int np = 0;
        CKL(copy_words(st, ctx->d_rhs, ctx->d_R, vb));
        if (ctx->d_Uinit) {
            CKL(copy_words(st, ctx->d_Uinit, ctx->d_U, vb));
            RUN("ref_line_res", launch_ref_line_res(st, nv, ctx->nline, ne, ctx->d_epoint, ctx->d_ef,
                                                    ctx->d_fc, ctx->d_linesize, ctx->d_linepoint,
                                                    ctx->d_lines, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                                    ctx->d_U, ctx->d_R, ctx->d_partials, &np));
        } else {
            CK(cudaMemsetAsync(ctx->d_U, 0, vb, st));
            np = ref_line_res_partials(ne);
            RUN("norm_partials", launch_norm_partials(st, ctx->d_R, nvec(ctx), ctx->d_partials, np));
        }
        CK(cudaMemsetAsync(ctx->d_dU, 0, vb, st));
        return reduce(ctx, np, 1, cc);
    }
    const FastLayout &L = ctx->L;
    if (ctx->algo == TBS_ALGO_FP64 || ctx->algo == TBS_ALGO_PIJ) {
        const bool pij = ctx->algo == TBS_ALGO_PIJ;
        const double *Rsrc = ctx->d_rhsp;
        /* TBS_ALGO_PIJ: the first update goes to buffer A (d_b), parity 0 */
        if (pij) CK(cudaMemsetAsync(&ctx->d_state->pad, 0, sizeof(int), st));
        if (ctx->d_Uinit) {
            RUN("permute", launch_permute_to_pos(st, nv, ne, L.pos_of_elem, ctx->d_Uinit, ctx->d_Up));
            if (nv == 9) {
                RUN("full_resid", launch_full_resid<double>(st, ne, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
                                                            L.pos_of_elem, ctx->d_jacD, ctx->d_O1,
                                                            ctx->d_O2, ctx->d_rhs, ctx->d_Up, ctx->d_Rp,
                                                            ctx->d_partials2));
            } else {
                int rc = ref_residual(ctx, ctx->d_Uinit, ctx->d_R);
                if (rc) return rc;
                RUN("permute", launch_permute_to_pos(st, nv, ne, L.pos_of_elem, ctx->d_R, ctx->d_Rp));
            }
            Rsrc = ctx->d_Rp;
        }
        /* from U = 0 the same launch clears U */
        RUN("fast_resid_rhs", resid64(ctx, 0, ctx->d_dUp, Rsrc, ctx->d_b, sink(ctx, 1, cc),
                                      ctx->d_Uinit ? nullptr : ctx->d_Up));
        return TBS_OK;
    }
    /* TBS_ALGO_MIXED: R32, its norm, and the first inner right-hand side
     * b32 = -Dinv32 R32 with c32 = 0 */
    if (ctx->d_Uinit) {
        RUN("permute", launch_permute_to_pos(st, 9, ne, L.pos_of_elem, ctx->d_Uinit, ctx->d_Up));
        RUN("full_resid", launch_full_resid<float>(st, ne, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
                                                   L.pos_of_elem, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                                   ctx->d_rhs, ctx->d_Up, ctx->d_R32,
                                                   ctx->d_partials));
        RUN("fast_resid32_rhs", launch_fast_resid<float>(st, L, 0, ctx->d_Dinv32, ctx->d_X32, ctx->d_d32,
                                                         ctx->d_R32, ctx->d_b32, no_sink(), ctx->d_status,
                                                         ctx->d_c32));
        return reduce(ctx, full_resid_blocks(ne), 1, cc);
    }
    RUN("mixed_prime", launch_mixed_prime(st, L, ctx->d_rhsp, ctx->d_R32, ctx->d_Up, ctx->d_partials,
                                          ctx->d_Dinv32, ctx->d_b32, ctx->d_c32));
    return reduce(ctx, fast_resid_grid(L.np16), 1, cc);
}

/* One sweep from the primed state, ending with the new residual's norm
 * recorded as one more sweep. */
/* the inner FP32 sweeps of the next TBS_ALGO_MIXED outer step */
static int inner_for_next(const tbs_ctx *ctx) {
    return (ctx->outer_done == 0 && ctx->inner_first > 0) ? ctx->inner_first : ctx->inner_sweeps;
}

static int body(tbs_ctx *ctx, CondCtl cc, int inner) {
    ctx->outer_done += 1;
    cudaStream_t st = ctx->stream;
    const int nv = ctx->nvar, ne = ctx->nelem;
    if (ctx->algo == TBS_ALGO_REFERENCE) {
        RUN("ref_solve_du", launch_ref_solve_du(st, nv, ctx->nline, ctx->d_linesize, ctx->d_linepoint,
                                                ctx->d_lines, ctx->d_DLU, ctx->d_DinvC, ctx->d_A,
                                                ctx->d_dU, ctx->d_R));
        RUN("ref_add_copy", launch_ref_add_copy(st, nvec(ctx), ctx->d_dU, ctx->d_U, ctx->d_rhs, ctx->d_R));
        int np = 0;
        RUN("ref_line_res", launch_ref_line_res(st, nv, ctx->nline, ne, ctx->d_epoint, ctx->d_ef,
                                                ctx->d_fc, ctx->d_linesize, ctx->d_linepoint,
                                                ctx->d_lines, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                                ctx->d_U, ctx->d_R, ctx->d_partials, &np));
        return reduce(ctx, np, 0, cc);
    }
    const FastLayout &L = ctx->L;
    if (ctx->algo == TBS_ALGO_PIJ) {
        RUN("pij_sweep", launch_pij_sweep(st, L, ctx->d_Dinv, ctx->d_XF, ctx->d_b, ctx->d_dUp, ctx->d_Up,
                                          sink(ctx, 0, cc), ctx->d_status));
        return TBS_OK;
    }
    if (ctx->algo == TBS_ALGO_FP64) {
        /* the Thomas kernel adds dU to U as it writes dU (U read one chunk
         * ahead of the backward chains), so the residual kernel reads
         * neither its own dU nor U (72 bytes a cell fewer per sweep at
         * size 9) */
        RUN("fast_thomas", thomas64(ctx, ctx->d_b, ctx->d_dUp, ctx->d_Up, 1));
        RUN("fast_resid", resid64(ctx, 1, ctx->d_dUp, nullptr, ctx->d_b, sink(ctx, 0, cc), nullptr));
        return TBS_OK;
    }
    /* TBS_ALGO_MIXED: inner FP32 LIJ sweeps on J d = -R, then U += d and the
     * FP64 residual R = rhs + J U from the original blocks */
    /* b32 = -Dinv32 R32 and c = 0 come from the previous step's residual
     * (or the prime) when the position-ordered residual runs; c = sum of
     * the inner updates but the last: each inner residual kernel adds its
     * sweep's d to c; the last d is added with c to U below */
    const bool pos = fullpos_ok(ctx);
    if (!pos)
        RUN("fast_resid32_rhs", launch_fast_resid<float>(st, L, 0, ctx->d_Dinv32, ctx->d_X32, ctx->d_d32,
                                                         ctx->d_R32, ctx->d_b32, no_sink(), ctx->d_status,
                                                         ctx->d_c32));
    /* every inner line solve but the last adds its d to c as it writes d
     * (the same FP32 sum c + d the residual kernel formed before; the line
     * solve is bound by its chain, the residual by HBM) */
    for (int m = 0; m < inner; ++m) {
        RUN("fast_thomas32", launch_fast_thomas<float>(st, L, ctx->d_G32, ctx->d_Gam32, ctx->d_b32,
                                                       ctx->d_y32, ctx->d_d32, ctx->d_c32,
                                                       ctx->d_status, m + 1 < inner ? 1 : 2));
        if (m + 1 < inner)
            RUN("fast_resid32", launch_fast_resid<float>(st, L, 3, nullptr, ctx->d_X32, ctx->d_d32,
                                                         nullptr, ctx->d_b32, no_sink(),
                                                         ctx->d_status, nullptr));
    }
    RUN("axpy", launch_axpy2_f32_f64(st, ctx->d_c32, ctx->d_d32, ctx->d_Up, (long long)L.np16 * 9));
    if (pos) {
        RUN("full_resid", launch_full_resid_pos(st, L, ctx->d_Dp, ctx->d_XF, ctx->d_rhsp, ctx->d_Up,
                                                ctx->d_R32, ctx->d_partials, ctx->d_Dinv32, ctx->d_b32,
                                                ctx->d_c32, ctx->d_status));
        return reduce(ctx, fast_resid_grid(L.np16), 0, cc);
    }
    RUN("full_resid", launch_full_resid<float>(st, ne, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
                                               L.pos_of_elem, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                               ctx->d_rhs, ctx->d_Up, ctx->d_R32, ctx->d_partials));
    return reduce(ctx, full_resid_blocks(ne), 0, cc);
}

/* Whether tbs_solve checks a converged solve against the true residual:
 * TBS_ALGO_FP64 tracks its residual recursively (R = X dU over the
 * cross-line blocks), so rounding, or Jacobian values changed after the
 * factorization (tbs_update_values), can make it differ from rhs + J U.
 * The other algorithms form the true residual every sweep (REFERENCE, the
 * MIXED outer step) or are point sweeps (PIJ). */
static bool checks_solve(const tbs_ctx *ctx) { return ctx->check && ctx->algo == TBS_ALGO_FP64; }

/* The check of a converged TBS_ALGO_FP64 solve: R = rhs + J U from the
 * original blocks (the rule of linesmoothLU_TriBlock_v3.okl:228-336) and
 * its norm, recorded as NORM_CHECK: a pass ends the solve; a failure
 * replaces the sweep's history entry, and the solve continues from the true
 * residual, for which the next sweep's input b = -Dinv R is made
 * (check_restart).  In the graph the restart is an IF node whose condition
 * the norm's reduction sets, so a passing check reads no factor block. */
static int check_residual(tbs_ctx *ctx, CondCtl cc) {
    cudaStream_t st = ctx->stream;
    const FastLayout &L = ctx->L;
    const int nv = ctx->nvar, ne = ctx->nelem;
    int np = 0;
    if (nv == 9) {
        RUN("full_resid", launch_full_resid<double>(st, ne, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
                                                    L.pos_of_elem, ctx->d_jacD, ctx->d_O1,
                                                    ctx->d_O2, ctx->d_rhs, ctx->d_Up, ctx->d_Rp,
                                                    ctx->d_partials2));
        np = full_resid_blocks(ne);
    } else {
        RUN("permute", launch_permute_to_elem(st, nv, ne, L.pos_of_elem, ctx->d_Up, ctx->d_U));
        int rc = ref_residual(ctx, ctx->d_U, ctx->d_R, &np);
        if (rc) return rc;
        RUN("permute", launch_permute_to_pos(st, nv, ne, L.pos_of_elem, ctx->d_R, ctx->d_Rp));
    }
    RUN("reduce_norm", launch_reduce_norm(st, ctx->d_partials2, np, ctx->d_state, ctx->d_hist,
                                          NORM_CHECK, cc.handle, cc.use_cond, cc.handle2, cc.use2));
    return TBS_OK;
}

/* b = -Dinv R of the true residual, for the sweeps after a failed check */
static int check_restart(tbs_ctx *ctx) {
    RUN("fast_resid_check", resid64(ctx, 0, ctx->d_dUp, ctx->d_Rp, ctx->d_b, no_sink(), nullptr));
    return TBS_OK;
}

/* eager form: the host reads the recorded check and makes b only after a
 * failure that leaves sweeps to do (the graph's IF node) */
static int read_state(tbs_ctx *ctx);
static int check_true_eager(tbs_ctx *ctx) {
    int rc = check_residual(ctx, CondCtl{});
    if (rc) return rc;
    rc = read_state(ctx);
    if (rc) return rc;
    const SolveState &S = *ctx->h_state;
    const bool pass = std::isfinite(S.true_norm) && S.true_norm <= S.tol * S.norm0;
    if (!pass && std::isfinite(S.true_norm) && S.sweep < S.max_sweeps) return check_restart(ctx);
    return TBS_OK;
}

int ctx_ensure_hist(tbs_ctx *ctx, int need) {
    if (need <= ctx->hist_cap) return TBS_OK;
    drop_graph(ctx);
    dfree(ctx, &ctx->d_hist);
    int cap = std::max(need, 1024);
    DA(ctx->d_hist, (size_t)cap);
    ctx->hist_cap = cap;
    return TBS_OK;
}

/* write the control block of the device SolveState (tol, max_sweeps,
 * hist_cap), leaving the recorded norms alone */
int ctx_set_state(tbs_ctx *ctx, double tol, int max_sweeps) {
    SolveState *h = ctx->h_state;
    h->tol = tol;
    h->max_sweeps = max_sweeps;
    h->hist_cap = ctx->hist_cap;
    set_state_kernel<<<1, 1, 0, ctx->stream>>>(ctx->d_state, tol, max_sweeps, ctx->hist_cap);
    CK(cudaGetLastError());
    return TBS_OK;
}

static_assert(sizeof(SolveState) % 8 == 0, "SolveState is copied in 8-byte words");

static int read_state(tbs_ctx *ctx) {
    CKL(copy_words(ctx->stream, ctx->d_state, ctx->h_state_dev, sizeof(SolveState)));
    CK(cudaStreamSynchronize(ctx->stream));
    return TBS_OK;
}

/* capture `fn` into the body graph of a conditional node */
template <typename F>
static int capture_into(tbs_ctx *ctx, cudaGraph_t g, F &&fn) {
    cudaStream_t st = ctx->stream;
    CK(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int rc = fn();
    cudaGraph_t outg = nullptr;
    cudaError_t ee = cudaStreamEndCapture(st, &outg);
    if (rc == TBS_OK && ee != cudaSuccess)
        rc = ctx_fail(ctx, TBS_ERR_CUDA, std::string("end body capture: ") + cudaGetErrorString(ee));
    return rc;
}

/* append a conditional node (type) after the capture's current nodes;
 * returns its body graph */
static int add_conditional(tbs_ctx *ctx, cudaGraph_t g, cudaGraphConditionalHandle h,
                           cudaGraphConditionalNodeType type, cudaGraph_t *body_out) {
    cudaStream_t st = ctx->stream;
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &ndeps);
    if (e != cudaSuccess) return ctx_fail(ctx, TBS_ERR_CUDA, std::string("capture info: ") + cudaGetErrorString(e));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    e = cudaGraphAddNode(&node, g, deps, ndeps, &cp);
    if (e != cudaSuccess) return ctx_fail(ctx, TBS_ERR_CUDA, std::string("conditional node: ") + cudaGetErrorString(e));
    *body_out = cp.conditional.phGraph_out[0];
    e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return ctx_fail(ctx, TBS_ERR_CUDA, std::string("capture deps: ") + cudaGetErrorString(e));
    return TBS_OK;
}

/* Graph: prime (records ||R_0||, sets the condition) -> while (cond) { sweep }.
 * TBS_ALGO_MIXED with its own inner sweep count for the first outer step:
 * prime -> if (cond) { first step } -> while (cond) { step }, the prime
 * setting both conditions and every step the loop's. */
static int build_graph(tbs_ctx *ctx) {
    drop_graph(ctx);
    cudaStream_t st = ctx->stream;
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    ctx->graph = g;
    const bool sched = ctx->algo == TBS_ALGO_MIXED && ctx->inner_first > 0 &&
                       ctx->inner_first != ctx->inner_sweeps;
    cudaGraphConditionalHandle hw, hf = 0;
    CK(cudaGraphConditionalHandleCreate(&hw, g, 0, cudaGraphCondAssignDefault));
    if (sched) CK(cudaGraphConditionalHandleCreate(&hf, g, 0, cudaGraphCondAssignDefault));
    const bool chk = checks_solve(ctx);
    cudaGraphConditionalHandle hc = 0, hr = 0;
    if (chk) {
        CK(cudaGraphConditionalHandleCreate(&hc, g, 0, cudaGraphCondAssignDefault));
        CK(cudaGraphConditionalHandleCreate(&hr, g, 0, cudaGraphCondAssignDefault));
    }
    const CondCtl loop{(unsigned long long)hw, 1, 0, 0, (unsigned long long)hc, chk ? 1 : 0};
    const CondCtl both{(unsigned long long)hw, 1, (unsigned long long)hf, sched ? 1 : 0, 0, 0};
    CK(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int rc = prime(ctx, both);
    cudaGraph_t firstg = nullptr, bodyg = nullptr;
    if (rc == TBS_OK && sched) rc = add_conditional(ctx, g, hf, cudaGraphCondTypeIf, &firstg);
    if (rc == TBS_OK) rc = add_conditional(ctx, g, hw, cudaGraphCondTypeWhile, &bodyg);
    cudaGraph_t outg = nullptr;
    cudaError_t ee = cudaStreamEndCapture(st, &outg);
    if (rc == TBS_OK && ee != cudaSuccess) rc = ctx_fail(ctx, TBS_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ee));
    if (rc == TBS_OK && sched)
        rc = capture_into(ctx, firstg, [&]() { return body(ctx, loop, ctx->inner_first); });
    /* the loop's body; with the check, an IF node after the sweep runs the
     * true residual when the sweep met the tolerance, and an IF node inside
     * it makes the next sweep's input when the check failed:
     * while (go) { sweep; if (met) { true residual; if (failed) { b } } } */
    cudaGraph_t checkg = nullptr;
    if (rc == TBS_OK)
        rc = capture_into(ctx, bodyg, [&]() {
            int r = body(ctx, loop, ctx->inner_sweeps);
            if (r == TBS_OK && chk) r = add_conditional(ctx, bodyg, hc, cudaGraphCondTypeIf, &checkg);
            return r;
        });
    if (rc == TBS_OK && chk) {
        /* the check's reduction sets the loop's condition and the restart's */
        const CondCtl ck{(unsigned long long)hw, 1, (unsigned long long)hr, 1, 0, 0};
        cudaGraph_t restartg = nullptr;
        rc = capture_into(ctx, checkg, [&]() {
            int r = check_residual(ctx, ck);
            if (r == TBS_OK) r = add_conditional(ctx, checkg, hr, cudaGraphCondTypeIf, &restartg);
            return r;
        });
        if (rc == TBS_OK) rc = capture_into(ctx, restartg, [&]() { return check_restart(ctx); });
    }
    if (rc != TBS_OK) {
        drop_graph(ctx);
        return rc;
    }
    cudaError_t ie = cudaGraphInstantiate(&ctx->gexec, g, 0);
    if (ie != cudaSuccess) {
        drop_graph(ctx);
        return ctx_fail(ctx, TBS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    }
    ctx->graph_algo = ctx->algo;
    return TBS_OK;
}

/* =========================================================== algorithms */

static int alloc_algo(tbs_ctx *ctx, int algo) {
    const size_t bs = (size_t)ctx->nvar * ctx->nvar, ne = ctx->nelem;
    DA(ctx->d_U, (size_t)nvec(ctx));
    DA(ctx->d_dU, (size_t)nvec(ctx));
    DA(ctx->d_R, (size_t)nvec(ctx));
    DA(ctx->d_scratch, (size_t)nvec(ctx));
    const int npmax = std::max({ref_line_res_partials(ctx->nelem) * 8, fast_resid_grid(ctx->L.np16),
                                full_resid_blocks(ctx->nelem), 1024});
    DA(ctx->d_counter, 1);
    if (ctx->npart_cap < npmax) {
        dfree(ctx, &ctx->d_partials);
        dfree(ctx, &ctx->d_partials2);
        DA(ctx->d_partials, (size_t)npmax);
        DA(ctx->d_partials2, (size_t)npmax);
        ctx->npart_cap = npmax;
    }
    if (algo == TBS_ALGO_REFERENCE) {
        const size_t nb = (size_t)ctx->nvar * ctx->nvar * ne;
        DA(ctx->d_DLU, nb);
        DA(ctx->d_DinvC, nb);
        DA(ctx->d_A, nb);
        return TBS_OK;
    }
    const FastLayout &L = ctx->L;
    const size_t npb = (size_t)L.np16 * bs, npv = (size_t)L.np16 * ctx->nvar;
    const size_t nxb = (size_t)L.np16 * std::max(L.nx, 1) * bs;
    DA(ctx->d_Up, npv);
    DA(ctx->d_rhsp, npv);
    DA(ctx->d_Rp, npv);
    if (algo == TBS_ALGO_PIJ) {
        DA(ctx->d_Dinv, npb); /* D^-1 per position, built in place */
        if (L.nxf > 0) DA(ctx->d_XF, (size_t)L.np16 * L.nxf * bs);
        DA(ctx->d_dUp, npv);  /* the two update buffers */
        DA(ctx->d_b, npv);
        return TBS_OK;
    }
    if (algo == TBS_ALGO_FP64) {
        DA(ctx->d_Dinv, npb);
        DA(ctx->d_G, npb);
        DA(ctx->d_Gam, npb);
        DA(ctx->d_X, nxb);
        DA(ctx->d_dUp, npv);
        DA(ctx->d_b, npv);
        DA(ctx->d_y, npv);
    } else {
        DA(ctx->d_Dinv, npb); /* FP64 inverse, input of the premultiplied DX blocks */
        DA(ctx->d_Dinv32, npb);
        DA(ctx->d_G32, npb);
        DA(ctx->d_Gam32, npb);
        DA(ctx->d_X32, nxb); /* holds DX = Dinv X in FP32 */
        if (fullpos_ok(ctx)) {
            DA(ctx->d_Dp, npb);
            DA(ctx->d_XF, (size_t)L.np16 * L.nxf * bs);
        }
        DA(ctx->d_b32, npv);
        DA(ctx->d_y32, npv);
        DA(ctx->d_d32, npv);
        DA(ctx->d_c32, npv);
        DA(ctx->d_R32, npv);
    }
    return TBS_OK;
}

static int run_factor(tbs_ctx *ctx, int algo) {
    cudaStream_t st = ctx->stream;
    const int nv = ctx->nvar;
    if (algo == TBS_ALGO_REFERENCE) {
        const size_t nb = (size_t)nv * nv * ctx->nelem;
        CKL(copy_words(st, ctx->d_jacD, ctx->d_DLU, nb * sizeof(double)));
        CK(cudaMemsetAsync(ctx->d_DinvC, 0, nb * sizeof(double), st));
        CK(cudaMemsetAsync(ctx->d_A, 0, nb * sizeof(double), st));
        RUN("ref_assemble_A", launch_ref_assemble_A(st, nv, ctx->nline, ctx->d_fc, ctx->d_linesize,
                                                    ctx->d_linepoint, ctx->d_lines, ctx->d_lineface,
                                                    ctx->d_O1, ctx->d_O2, ctx->d_A));
        RUN("ref_line_lu", launch_ref_line_lu(st, nv, ctx->nline, ctx->d_fc, ctx->d_linesize,
                                              ctx->d_linepoint, ctx->d_lines, ctx->d_lineface,
                                              ctx->d_DLU, ctx->d_O1, ctx->d_O2, ctx->d_DinvC,
                                              ctx->d_status));
        return TBS_OK;
    }
    const FastLayout &L = ctx->L;
    RUN("permute", launch_permute_to_pos(st, nv, ctx->nelem, L.pos_of_elem, ctx->d_rhs, ctx->d_rhsp));
    if (nv != 9) {
        /* TBS_ALGO_FP64, general block size */
        CKL(nv_prepare(nv, L));
        RUN("fast_factor", launch_nv_factor(st, nv, L, ctx->d_jacD, ctx->d_O1, ctx->d_O2, ctx->d_Dinv,
                                            ctx->d_G, ctx->d_Gam, ctx->d_gamlast, ctx->d_status));
        RUN("fast_xlayout", launch_nv_xlayout(st, nv, L, ctx->d_O1, ctx->d_O2, ctx->d_X));
        return TBS_OK;
    }
    CKL(fast_prepare(L));
    if (algo == TBS_ALGO_PIJ) {
        CKL(pij_prepare(L));
        RUN("fullpos_layout", launch_fullpos_layout(st, L, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                                    ctx->d_Dinv, ctx->d_XF));
        RUN("pij_invert", launch_pij_invert(st, L, ctx->d_Dinv, ctx->d_status));
        return TBS_OK;
    }
    if (algo == TBS_ALGO_FP64) {
        RUN("fast_factor", launch_fast_factor(st, L, ctx->d_jacD, ctx->d_O1, ctx->d_O2, ctx->d_Dinv,
                                              ctx->d_G, ctx->d_Gam, nullptr, nullptr, nullptr,
                                              ctx->d_gamlast, ctx->d_status));
        RUN("fast_xlayout", launch_fast_xlayout(st, L, ctx->d_O1, ctx->d_O2, ctx->d_X, nullptr));
    } else {
        RUN("fast_factor", launch_fast_factor(st, L, ctx->d_jacD, ctx->d_O1, ctx->d_O2, ctx->d_Dinv,
                                              nullptr, nullptr, ctx->d_Dinv32, ctx->d_G32,
                                              ctx->d_Gam32, ctx->d_gamlast, ctx->d_status));
        RUN("fast_dx", launch_fast_dx(st, L, ctx->d_Dinv, ctx->d_O1, ctx->d_O2, ctx->d_X32));
        if (fullpos_ok(ctx)) {
            CKL(fullpos_prepare(L));
            RUN("fullpos_layout", launch_fullpos_layout(st, L, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                                        ctx->d_Dp, ctx->d_XF));
        }
    }
    return TBS_OK;
}

/* ============================================================ C entry points */

extern "C" {

const char *tbs_last_error(const tbs_ctx *ctx) {
    if (ctx) return ctx->err.c_str();
    return thread_error();
}

int tbs_create(int device_id, tbs_ctx **out) {
    tbs_ctx *ctx = nullptr;
    if (!out) return ctx_fail(nullptr, TBS_ERR_ARG, "tbs_create: null output pointer");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return ctx_fail(nullptr, TBS_ERR_CUDA,
                        std::string("no CUDA device available (") + cudaGetErrorString(e) +
                            "); this library has no CPU path");
    }
    if (device_id < 0 || device_id >= ndev)
        return ctx_fail(nullptr, TBS_ERR_ARG, "device_id " + std::to_string(device_id) +
                                                  " out of range (" + std::to_string(ndev) + " devices)");
    ctx = new (std::nothrow) tbs_ctx();
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_NOMEM, "host allocation failed");
    ctx->device = device_id;
    e = cudaSetDevice(device_id);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&ctx->h_state, sizeof(SolveState), cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&ctx->h_state_dev, ctx->h_state, 0);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&ctx->h_status, 8, cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&ctx->h_status_dev, ctx->h_status, 0);
    if (e == cudaSuccess) e = (cudaError_t)fast_kernels_init();
    if (e != cudaSuccess) {
        std::string msg = std::string("device setup failed: ") + cudaGetErrorString(e);
        if (ctx->own) cudaStreamDestroy(ctx->own);
        delete ctx;
        return ctx_fail(nullptr, TBS_ERR_CUDA, msg);
    }
    ctx->stream = ctx->own;
    *out = ctx;
    return TBS_OK;
}

int tbs_destroy(tbs_ctx *ctx) {
    if (!ctx) return TBS_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    drop_mesh(ctx);
    for (auto &p : ctx->pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto ev : ctx->pool) cudaEventDestroy(ev);
    if (ctx->h_state) cudaFreeHost(ctx->h_state);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    if (ctx->h_hist) cudaFreeHost(ctx->h_hist);
    for (int k = 0; k < tbs_ctx::kLandSlots; ++k) {
        if (ctx->land_ready[k]) cudaEventDestroy(ctx->land_ready[k]);
        if (ctx->land_free[k]) cudaEventDestroy(ctx->land_free[k]);
    }
    if (ctx->copy) cudaStreamDestroy(ctx->copy);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
    return TBS_OK;
}

int tbs_set_stream(tbs_ctx *ctx, void *cuda_stream) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    cudaStream_t ns = cuda_stream ? (cudaStream_t)cuda_stream : ctx->own;
    if (ns != ctx->stream) {
        cudaStreamSynchronize(ctx->stream);
        drop_graph(ctx); /* graphs are launched on, and captured from, the stream */
        multi_drop_graph(ctx);
        ctx->stream = ns;
    }
    return TBS_OK;
}

/* tbs_set_mesh with the last nhalo lines marked as halo lines (0: none) */
static int set_mesh(tbs_ctx *ctx, int nhalo, int nvar, int nelem, int nintface, int eftot,
                    int nline, int nlineelem, const int *epoint, const int *ef, const int *fc,
                    const int *linesize, const int *linepoint, const int *lines,
                    const int *lineface) {
    CK(cudaSetDevice(ctx->device));
    int hdr[6] = {nvar, nelem, nintface, eftot, nline, nlineelem};
    int st = validate_mesh(hdr, epoint, ef, fc, linesize, linepoint, lines, lineface);
    if (st) return ctx_fail(ctx, st, thread_error());
    if (nvar > 32) return ctx_fail(ctx, TBS_ERR_UNSUPPORTED, "nvar > 32 is not supported");
    int nelem_own = nelem;
    if (nhalo > 0) {
        if (nhalo >= nline)
            return ctx_fail(ctx, TBS_ERR_ARG, "a line partition needs at least one owned line");
        /* the owned lines' cells must be exactly elements 0..nelem_own-1 */
        nelem_own = linepoint[nline - nhalo];
        for (int k = 0; k < nelem_own; ++k)
            if (lines[k] >= nelem_own)
                return ctx_fail(ctx, TBS_ERR_FORMAT,
                                "line partition: the owned lines' cells must be numbered before "
                                "the halo lines' cells");
    }
    CK(cudaStreamSynchronize(ctx->stream));
    drop_mesh(ctx);
    ctx->nhalo = nhalo;
    ctx->nelem_own = nelem_own;
    /* 8 bytes: the status word is read back in one 8-byte copy */
    CK(cudaMalloc((void **)&ctx->d_status, 8));
    ctx->allocs.push_back({ctx->d_status, 8});
    CK(cudaMemsetAsync(ctx->d_status, 0, 8, ctx->stream));
    DA(ctx->d_state, 1);
    DA(ctx->d_ktimer, 3);
    {
        const unsigned long long init[3] = {~0ull, 0ull, 0ull};
        CKL(xfer_put(ctx->stream, ctx->d_ktimer, init, sizeof(init)));
    }
    ctx->nvar = nvar;
    ctx->nelem = nelem;
    ctx->nintface = nintface;
    ctx->eftot = eftot;
    ctx->nline = nline;
    ctx->nlineelem = nlineelem;
    ctx->h_epoint.assign(epoint, epoint + nelem + 1);
    ctx->h_ef.assign(ef, ef + eftot);
    ctx->h_fc.assign(fc, fc + 2 * (size_t)nintface);
    ctx->h_linesize.assign(linesize, linesize + nline);
    ctx->h_linepoint.assign(linepoint, linepoint + nline + 1);
    ctx->h_lines.assign(lines, lines + nlineelem);
    ctx->h_lineface.assign(lineface, lineface + nlineelem);
    ctx->max_line = 0;
    for (int l = 0; l < nline; ++l) ctx->max_line = std::max(ctx->max_line, linesize[l]);
    DA(ctx->d_epoint, (size_t)nelem + 1);
    DA(ctx->d_ef, (size_t)eftot);
    DA(ctx->d_fc, 2 * (size_t)nintface);
    DA(ctx->d_linesize, (size_t)nline);
    DA(ctx->d_linepoint, (size_t)nline + 1);
    DA(ctx->d_lines, (size_t)nlineelem);
    DA(ctx->d_lineface, (size_t)nlineelem);
    DA(ctx->d_identity, (size_t)nelem);
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->d_epoint, epoint, (nelem + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    if (eftot) CK(cudaMemcpyAsync(ctx->d_ef, ef, eftot * sizeof(int), cudaMemcpyHostToDevice, s));
    if (nintface) CK(cudaMemcpyAsync(ctx->d_fc, fc, 2 * (size_t)nintface * sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->d_linesize, linesize, nline * sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->d_linepoint, linepoint, (nline + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->d_lines, lines, nlineelem * sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->d_lineface, lineface, nlineelem * sizeof(int), cudaMemcpyHostToDevice, s));
    {
        std::vector<int> id(nelem);
        for (int e = 0; e < nelem; ++e) id[e] = e;
        CK(cudaMemcpyAsync(ctx->d_identity, id.data(), nelem * sizeof(int), cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
    }
    int rc = build_layout(ctx);
    if (rc) return rc;
    ctx->have_mesh = true;
    return TBS_OK;
}

int tbs_set_mesh(tbs_ctx *ctx, int nvar, int nelem, int nintface, int eftot, int nline,
                 int nlineelem, const int *epoint, const int *ef, const int *fc,
                 const int *linesize, const int *linepoint, const int *lines,
                 const int *lineface) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    return set_mesh(ctx, 0, nvar, nelem, nintface, eftot, nline, nlineelem, epoint, ef, fc,
                    linesize, linepoint, lines, lineface);
    GUARD_END
}

int tbs_set_partition_mesh(tbs_ctx *ctx, int nhalo_lines, int nvar, int nelem, int nintface,
                           int eftot, int nline, int nlineelem, const int *epoint, const int *ef,
                           const int *fc, const int *linesize, const int *linepoint,
                           const int *lines, const int *lineface) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    if (nhalo_lines < 0) return ctx_fail(ctx, TBS_ERR_ARG, "negative halo line count");
    GUARD_BEGIN
    return set_mesh(ctx, nhalo_lines, nvar, nelem, nintface, eftot, nline, nlineelem, epoint, ef,
                    fc, linesize, linepoint, lines, lineface);
    GUARD_END
}

/* piece > 0: the copies go in pieces of at most `piece` bytes with at most
 * two in flight (the call returns when the last is issued), so that copies
 * from other threads wait behind two pieces, not the whole Jacobian */
static int upload_jacobian(tbs_ctx *ctx, const double *jacD, const double *O1, const double *O2,
                           const double *rhs, cudaMemcpyKind kind, size_t piece = 0) {
    if (!ctx->have_mesh) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_set_mesh must come first");
    if (!jacD || (ctx->nintface > 0 && (!O1 || !O2)) || !rhs)
        return ctx_fail(ctx, TBS_ERR_ARG, "null Jacobian array");
    const size_t nb = (size_t)ctx->nvar * ctx->nvar;
    DA(ctx->d_jacD, nb * ctx->nelem);
    DA(ctx->d_O1, nb * ctx->nintface);
    DA(ctx->d_O2, nb * ctx->nintface);
    DA(ctx->d_rhs, (size_t)nvec(ctx));
    cudaStream_t s = ctx->stream;
    struct Part {
        void *dst;
        const void *src;
        size_t bytes;
    };
    std::vector<Part> parts{{ctx->d_jacD, jacD, nb * ctx->nelem * sizeof(double)}};
    if (ctx->nintface) {
        parts.push_back({ctx->d_O1, O1, nb * ctx->nintface * sizeof(double)});
        parts.push_back({ctx->d_O2, O2, nb * ctx->nintface * sizeof(double)});
    }
    parts.push_back({ctx->d_rhs, rhs, (size_t)nvec(ctx) * sizeof(double)});
    if (piece == 0) {
        for (const Part &p : parts) CK(cudaMemcpyAsync(p.dst, p.src, p.bytes, kind, s));
    } else {
        cudaEvent_t ev[2] = {nullptr, nullptr};
        int rc = TBS_OK;
        long long n = 0;
        for (int k = 0; k < 2 && rc == TBS_OK; ++k)
            if (cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming) != cudaSuccess)
                rc = ctx_fail(ctx, TBS_ERR_CUDA, "cudaEventCreate failed");
        for (const Part &p : parts) {
            for (size_t off = 0; off < p.bytes && rc == TBS_OK; off += piece, ++n) {
                const size_t b = std::min(piece, p.bytes - off);
                cudaEvent_t e = ev[n & 1];
                if ((n >= 2 && cudaEventSynchronize(e) != cudaSuccess) ||
                    cudaMemcpyAsync(static_cast<char *>(p.dst) + off,
                                    static_cast<const char *>(p.src) + off, b, kind, s) != cudaSuccess ||
                    cudaEventRecord(e, s) != cudaSuccess)
                    rc = ctx_fail(ctx, TBS_ERR_CUDA, "paced Jacobian upload failed");
            }
        }
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        if (rc) return rc;
    }
    /* same mesh -> same allocations, so an instantiated solve graph stays valid */
    ctx->have_jac = true;
    ctx->factored = false;
    ctx->land_count = 0; /* these values, not a staged set, are the ones to factor */
    return TBS_OK;
}

int tbs_set_jacobian(tbs_ctx *ctx, const double *jacD, const double *jacO1, const double *jacO2,
                     const double *rhs, const double *U0) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    (void)U0; /* read but unused, as in the reference (U starts at zero) */
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    return upload_jacobian(ctx, jacD, jacO1, jacO2, rhs, cudaMemcpyHostToDevice);
    GUARD_END
}

int tbs_set_jacobian_device(tbs_ctx *ctx, const double *d_jacD, const double *d_jacO1,
                            const double *d_jacO2, const double *d_rhs) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    return upload_jacobian(ctx, d_jacD, d_jacO1, d_jacO2, d_rhs, cudaMemcpyDeviceToDevice);
    GUARD_END
}

int tbs_stage_jacobian(tbs_ctx *ctx, const double *jacD, const double *jacO1, const double *jacO2,
                       const double *rhs) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->have_mesh) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_set_mesh must come first");
    if (!jacD || (ctx->nintface > 0 && (!jacO1 || !jacO2)) || !rhs)
        return ctx_fail(ctx, TBS_ERR_ARG, "null Jacobian array");
    if (ctx->land_count == tbs_ctx::kLandSlots)
        return ctx_fail(ctx, TBS_ERR_STATE,
                        "two systems are already staged: tbs_factor takes the older one first");
    if (!ctx->copy) {
        CK(cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking));
        for (int k = 0; k < tbs_ctx::kLandSlots; ++k) {
            CK(cudaEventCreateWithFlags(&ctx->land_ready[k], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ctx->land_free[k], cudaEventDisableTiming));
        }
    }
    const int slot = (ctx->land_head + ctx->land_count) % tbs_ctx::kLandSlots;
    double **d = ctx->d_land[slot];
    const size_t nb = (size_t)ctx->nvar * ctx->nvar;
    const bool fresh = !d[0]; /* the four buffers are made and given up together */
    DA(d[0], nb * ctx->nelem);
    DA(d[1], nb * ctx->nintface);
    DA(d[2], nb * ctx->nintface);
    DA(d[3], (size_t)nvec(ctx));
    /* The copies wait for the slot's last reader, the copy that took its
     * previous system (tbs_factor), or, for new buffers, for their clearing
     * on the context's stream. */
    if (fresh) CK(cudaEventRecord(ctx->land_free[slot], ctx->stream));
    cudaStream_t c = ctx->copy;
    CK(cudaStreamWaitEvent(c, ctx->land_free[slot], 0));
    CK(cudaMemcpyAsync(d[0], jacD, nb * ctx->nelem * sizeof(double), cudaMemcpyDefault, c));
    if (ctx->nintface) {
        CK(cudaMemcpyAsync(d[1], jacO1, nb * ctx->nintface * sizeof(double), cudaMemcpyDefault, c));
        CK(cudaMemcpyAsync(d[2], jacO2, nb * ctx->nintface * sizeof(double), cudaMemcpyDefault, c));
    }
    CK(cudaMemcpyAsync(d[3], rhs, (size_t)nvec(ctx) * sizeof(double), cudaMemcpyDefault, c));
    CK(cudaEventRecord(ctx->land_ready[slot], c));
    ctx->land_count++;
    return TBS_OK;
    GUARD_END
}

/* make the oldest staged system the active one (tbs_factor): the context's
 * stream waits for its upload, then a kernel copies the slot over the
 * active buffers.  The active buffers keep their addresses, so the solve
 * graph captured on them stays the one launched: a graph launched for the
 * first time since another was launched on the stream re-uploads itself
 * through the copy engine, which would hold the solve behind the next
 * system's staged upload. */
static int take_staged(tbs_ctx *ctx) {
    const int slot = ctx->land_head;
    double **d = ctx->d_land[slot];
    CK(cudaStreamWaitEvent(ctx->stream, ctx->land_ready[slot], 0));
    if (!ctx->d_jacD) {
        /* no active set yet (nothing set before the first stage), so no
         * graph holds its addresses: the slot's buffers become the active
         * set and the slot allocates new ones when it is next staged */
        double **act[] = {&ctx->d_jacD, &ctx->d_O1, &ctx->d_O2, &ctx->d_rhs};
        for (int k = 0; k < 4; ++k) {
            *act[k] = d[k];
            d[k] = nullptr;
        }
    } else {
        const size_t nb = (size_t)ctx->nvar * ctx->nvar * sizeof(double);
        CKL(copy_words(ctx->stream, d[0], ctx->d_jacD, nb * ctx->nelem));
        if (ctx->nintface) {
            CKL(copy_words(ctx->stream, d[1], ctx->d_O1, nb * ctx->nintface));
            CKL(copy_words(ctx->stream, d[2], ctx->d_O2, nb * ctx->nintface));
        }
        CKL(copy_words(ctx->stream, d[3], ctx->d_rhs, (size_t)nvec(ctx) * sizeof(double)));
        CK(cudaEventRecord(ctx->land_free[slot], ctx->stream));
    }
    ctx->land_head = (slot + 1) % tbs_ctx::kLandSlots;
    ctx->land_count--;
    ctx->have_jac = true;
    ctx->factored = false;
    return TBS_OK;
}

int tbs_factor(tbs_ctx *ctx, int algo) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (ctx->land_count > 0) {
        int rs = take_staged(ctx);
        if (rs) return rs;
    }
    if (!ctx->have_jac) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_set_jacobian must come first");
    if (algo != TBS_ALGO_REFERENCE && algo != TBS_ALGO_FP64 && algo != TBS_ALGO_MIXED &&
        algo != TBS_ALGO_PIJ)
        return ctx_fail(ctx, TBS_ERR_ARG, "unknown algorithm " + std::to_string(algo));
    if (algo == TBS_ALGO_PIJ && (ctx->nvar != 9 || !fullpos_ok(ctx)))
        return ctx_fail(ctx, TBS_ERR_UNSUPPORTED,
                        "TBS_ALGO_PIJ needs nvar == 9 and at most 4 interior faces per cell");
    if (algo != TBS_ALGO_REFERENCE && algo != TBS_ALGO_PIJ && !ctx->layout_ok)
        return ctx_fail(ctx, TBS_ERR_UNSUPPORTED,
                        "TBS_ALGO_FP64 needs nvar 2..16 and at most 4 cross-line faces per cell; "
                        "use TBS_ALGO_REFERENCE");
    if (algo == TBS_ALGO_MIXED && ctx->nvar != 9)
        return ctx_fail(ctx, TBS_ERR_UNSUPPORTED, "TBS_ALGO_MIXED needs nvar == 9");
    int rc = alloc_algo(ctx, algo);
    if (rc) return rc;
    if (ctx->algo != algo) drop_graph(ctx);
    ctx->algo = algo;
    ctx->factored = false;
    rc = run_factor(ctx, algo);
    if (rc) return rc;
    rc = prime(ctx, CondCtl{});
    if (rc) return rc;
    rc = status_check(ctx);
    if (rc) return rc;
    ctx->factored = true;
    ctx->lagged = false;
    return TBS_OK;
    GUARD_END
}

int tbs_set_rhs(tbs_ctx *ctx, const double *rhs) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->factored) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
    if (!rhs) return ctx_fail(ctx, TBS_ERR_ARG, "null rhs");
    CK(cudaMemcpyAsync(ctx->d_rhs, rhs, (size_t)nvec(ctx) * sizeof(double), cudaMemcpyHostToDevice,
                       ctx->stream));
    if (ctx->algo != TBS_ALGO_REFERENCE) {
        RUN("permute", launch_permute_to_pos(ctx->stream, ctx->nvar, ctx->nelem, ctx->L.pos_of_elem, ctx->d_rhs,
                                             ctx->d_rhsp));
    }
    return prime(ctx, CondCtl{});
    GUARD_END
}

int tbs_set_initial(tbs_ctx *ctx, const double *U) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->factored) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
    if (U) {
        DA(ctx->d_Uinit, (size_t)nvec(ctx));
        CK(cudaMemcpyAsync(ctx->d_Uinit, U, (size_t)nvec(ctx) * sizeof(double),
                           cudaMemcpyHostToDevice, ctx->stream));
    } else {
        dfree(ctx, &ctx->d_Uinit);
    }
    drop_graph(ctx);
    return prime(ctx, CondCtl{});
    GUARD_END
}

int tbs_sweep(tbs_ctx *ctx, int n, double *rnorm_out) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->factored) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
    if (n < 0) return ctx_fail(ctx, TBS_ERR_ARG, "negative sweep count");
    if (ctx->nhalo > 0) return ctx_fail(ctx, TBS_ERR_UNSUPPORTED, "a line partition sweeps with tbs_part_solve_du / tbs_part_line_res");
    int rc = ctx_ensure_hist(ctx, n + 1);
    if (rc) return rc;
    rc = ctx_set_state(ctx, 0.0, n);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    /* the current residual norm (recorded by the last sequence) opens the history */
    rc = reduce(ctx, 0, 1, CondCtl{});
    if (rc) return rc;
    for (int s = 0; s < n; ++s) {
        rc = body(ctx, CondCtl{}, inner_for_next(ctx));
        if (rc) return rc;
    }
    if (rnorm_out) {
        rc = hist_to_host(ctx, rnorm_out, n + 1);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(st));
    if (ctx->prof) prof_resolve(ctx);
    return status_check(ctx);
    GUARD_END
}

int tbs_solve(tbs_ctx *ctx, double rel_tol, int max_sweeps, int *sweeps_out, double *hist_out) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->factored) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
    if (max_sweeps < 0 || !(rel_tol >= 0.0)) return ctx_fail(ctx, TBS_ERR_ARG, "bad tolerance or sweep limit");
    if (ctx->nhalo > 0) return ctx_fail(ctx, TBS_ERR_UNSUPPORTED, "a line partition sweeps with tbs_part_solve_du / tbs_part_line_res");
    int rc = ctx_ensure_hist(ctx, max_sweeps + 1);
    if (rc) return rc;
    rc = ctx_set_state(ctx, rel_tol, max_sweeps);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    if (ctx->prof) {
        /* eager form with a host-side test, so that every kernel is timed */
        rc = prime(ctx, CondCtl{});
        if (rc) return rc;
        bool checked = true; /* the primed residual is a true residual */
        for (;;) {
            rc = read_state(ctx);
            if (rc) return rc;
            const SolveState &S = *ctx->h_state;
            const bool met = std::isfinite(S.last) && S.last <= S.tol * S.norm0;
            const bool go = std::isfinite(S.last) && !met && S.sweep < S.max_sweeps;
            if (!go) {
                if (met && !checked && checks_solve(ctx)) {
                    /* as the graph's IF node: the true residual of the converged solve */
                    rc = check_true_eager(ctx);
                    if (rc) return rc;
                    checked = true;
                    continue;
                }
                break;
            }
            rc = body(ctx, CondCtl{}, inner_for_next(ctx));
            if (rc) return rc;
            checked = false;
        }
        prof_resolve(ctx);
    } else {
        if (!ctx->gexec || ctx->graph_algo != ctx->algo) {
            rc = build_graph(ctx);
            if (rc) return rc;
        }
        CK(cudaGraphLaunch(ctx->gexec, st));
        ctx->outer_done = 1; /* later tbs_sweep calls continue with the steady schedule */
        /* state, status and history in one read-back */
        const int nh = hist_out ? max_sweeps + 1 : 0;
        rc = ensure_h_hist(ctx, std::max(nh, 1));
        if (rc) return rc;
        solve_readback_kernel<<<1, 256, 0, st>>>(
            ctx->d_state, reinterpret_cast<const unsigned long long *>(ctx->d_status), ctx->d_hist,
            std::min(nh, ctx->hist_cap), ctx->h_state_dev,
            reinterpret_cast<unsigned long long *>(ctx->h_status_dev), ctx->h_hist_dev);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        const int sw = ctx->h_state->sweep;
        if (sweeps_out) *sweeps_out = sw;
        if (hist_out)
            std::memcpy(hist_out, ctx->h_hist, (size_t)(std::min(sw, max_sweeps) + 1) * sizeof(double));
        return status_error(ctx, *ctx->h_status);
    }
    const int sw = ctx->h_state->sweep;
    if (sweeps_out) *sweeps_out = sw;
    if (hist_out) {
        rc = hist_to_host(ctx, hist_out, std::min(sw, max_sweeps) + 1);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(st));
    return status_check(ctx);
    GUARD_END
}

static int get_vec(tbs_ctx *ctx, int which, double *out) {
    if (!ctx->factored) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
    if (!out) return ctx_fail(ctx, TBS_ERR_ARG, "null output");
    cudaStream_t st = ctx->stream;
    const size_t vb = (size_t)nvec(ctx) * sizeof(double);
    const double *src = nullptr;
    if (ctx->algo == TBS_ALGO_REFERENCE) {
        src = which == 0 ? ctx->d_U : which == 1 ? ctx->d_R : ctx->d_dU;
    } else {
        const FastLayout &L = ctx->L;
        const int nv = ctx->nvar;
        if (which == 0) {
            RUN("permute", launch_permute_to_elem(st, nv, ctx->nelem, L.pos_of_elem, ctx->d_Up, ctx->d_scratch));
        } else if (which == 1 && nv != 9) {
            /* general block size: the reference-order residual of U */
            RUN("permute", launch_permute_to_elem(st, nv, ctx->nelem, L.pos_of_elem, ctx->d_Up, ctx->d_U));
            int rc = ref_residual(ctx, ctx->d_U, ctx->d_scratch);
            if (rc) return rc;
        } else if (which == 1) {
            RUN("full_resid", launch_full_resid<double>(st, ctx->nelem, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
                                                        L.pos_of_elem, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                                        ctx->d_rhs, ctx->d_Up, ctx->d_Rp, ctx->d_partials2));
            RUN("permute", launch_permute_to_elem(st, 9, ctx->nelem, L.pos_of_elem, ctx->d_Rp, ctx->d_scratch));
        } else if (ctx->algo == TBS_ALGO_FP64) {
            RUN("permute", launch_permute_to_elem(st, nv, ctx->nelem, L.pos_of_elem, ctx->d_dUp, ctx->d_scratch));
        } else if (ctx->algo == TBS_ALGO_PIJ) {
            /* the last sweep added the buffer it read: A (d_b) when the
             * parity it flipped is now 1 */
            int rc = read_state(ctx);
            if (rc) return rc;
            const double *du = (ctx->h_state->pad & 1) ? ctx->d_b : ctx->d_dUp;
            RUN("permute", launch_permute_to_elem(st, 9, ctx->nelem, L.pos_of_elem, du, ctx->d_scratch));
        } else {
            RUN("permute", launch_permute_f32_to_elem(st, 9, ctx->nelem, L.pos_of_elem, ctx->d_c32, ctx->d_scratch));
            /* the outer correction is c + d (see body()); add d */
            RUN("permute", launch_permute_f32_to_elem(st, 9, ctx->nelem, L.pos_of_elem, ctx->d_d32, ctx->d_R));
            RUN("axpy", launch_axpy_f64(st, ctx->d_R, ctx->d_scratch, (long long)nvec(ctx)));
        }
        src = ctx->d_scratch;
    }
    int rc = to_host(ctx, out, src, vb);
    if (rc) return rc;
    CK(cudaStreamSynchronize(st));
    return TBS_OK;
}

int tbs_get_solution(tbs_ctx *ctx, double *U) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    return get_vec(ctx, 0, U);
    GUARD_END
}

int tbs_get_residual(tbs_ctx *ctx, double *R) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    return get_vec(ctx, 1, R);
    GUARD_END
}

int tbs_get_update(tbs_ctx *ctx, double *dU) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    return get_vec(ctx, 2, dU);
    GUARD_END
}

int tbs_true_residual_norm(tbs_ctx *ctx, double *out) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->factored) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
    if (!out) return ctx_fail(ctx, TBS_ERR_ARG, "null output");
    if (ctx->nvar != 9) {
        /* generic block size: the reference path's R is the true residual */
        std::vector<double> R((size_t)nvec(ctx));
        int rc = get_vec(ctx, 1, R.data());
        if (rc) return rc;
        double s = 0.0;
        for (size_t k = 0; k < (size_t)ctx->nelem_own * ctx->nvar; ++k) s += R[k] * R[k];
        *out = std::sqrt(s);
        return TBS_OK;
    }
    cudaStream_t st = ctx->stream;
    /* a line partition: the owned cells (elements 0..nelem_own-1); their
     * neighbours in halo lines are read from the halo copies of U */
    const int nb = full_resid_blocks(ctx->nelem_own);
    const bool ref = ctx->algo == TBS_ALGO_REFERENCE;
    RUN("full_resid", launch_full_resid<double>(st, ctx->nelem_own, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
                                                ref ? ctx->d_identity : ctx->L.pos_of_elem,
                                                ctx->d_jacD, ctx->d_O1, ctx->d_O2, ctx->d_rhs,
                                                ref ? ctx->d_U : ctx->d_Up,
                                                ref ? ctx->d_scratch : ctx->d_Rp, ctx->d_partials2));
    std::vector<double> part(nb);
    CK(cudaMemcpyAsync(part.data(), ctx->d_partials2, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double s = 0.0;
    for (double v : part) s += v;
    *out = std::sqrt(s);
    return TBS_OK;
    GUARD_END
}

int tbs_set_check(tbs_ctx *ctx, int on) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    if (on != 0 && on != 1) return ctx_fail(ctx, TBS_ERR_ARG, "tbs_set_check takes 0 or 1");
    if (ctx->check != on) {
        GUARD_BEGIN
        CK(cudaSetDevice(ctx->device));
        CK(cudaStreamSynchronize(ctx->stream));
        drop_graph(ctx);
        ctx->check = on;
        return TBS_OK;
        GUARD_END
    }
    return TBS_OK;
}

int tbs_solve_check(tbs_ctx *ctx, double *true_norm, int *checks, int *restarts) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->factored) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
    int rc = read_state(ctx);
    if (rc) return rc;
    if (true_norm) *true_norm = ctx->h_state->true_norm;
    if (checks) *checks = ctx->h_state->checks;
    if (restarts) *restarts = ctx->h_state->restarts;
    return TBS_OK;
    GUARD_END
}

int tbs_update_values(tbs_ctx *ctx, const double *jacD, const double *jacO1, const double *jacO2) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->factored) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
    if (!jacD || (ctx->nintface > 0 && (!jacO1 || !jacO2)))
        return ctx_fail(ctx, TBS_ERR_ARG, "null Jacobian array");
    if (ctx->algo == TBS_ALGO_PIJ)
        return ctx_fail(ctx, TBS_ERR_UNSUPPORTED,
                        "TBS_ALGO_PIJ tracks its residual with the factorization's face blocks; "
                        "re-factor instead (tbs_set_jacobian + tbs_factor)");
    if (ctx->nhalo > 0)
        return ctx_fail(ctx, TBS_ERR_UNSUPPORTED,
                        "a line partition tracks its residual with the factorization's blocks; "
                        "re-factor instead");
    if (ctx->algo == TBS_ALGO_FP64 && !ctx->check)
        return ctx_fail(ctx, TBS_ERR_STATE,
                        "TBS_ALGO_FP64 with the true-residual check off would converge to the "
                        "factored system; enable it (tbs_set_check) or re-factor");
    const size_t nb = (size_t)ctx->nvar * ctx->nvar;
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(ctx->d_jacD, jacD, nb * ctx->nelem * sizeof(double), cudaMemcpyHostToDevice, st));
    if (ctx->nintface) {
        CK(cudaMemcpyAsync(ctx->d_O1, jacO1, nb * ctx->nintface * sizeof(double), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->d_O2, jacO2, nb * ctx->nintface * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    if (ctx->algo == TBS_ALGO_MIXED && fullpos_ok(ctx))
        RUN("fullpos_layout", launch_fullpos_layout(st, ctx->L, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                                    ctx->d_Dp, ctx->d_XF));
    ctx->lagged = true;
    return prime(ctx, CondCtl{});
    GUARD_END
}

int tbs_selftest_timeout(tbs_ctx *ctx, long long budget_cycles) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->d_status) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_set_mesh must come first");
    if (budget_cycles < 0) return ctx_fail(ctx, TBS_ERR_ARG, "negative budget");
    CKL(launch_selftest_timeout(ctx->stream, budget_cycles, ctx->d_status));
    return status_check(ctx);
    GUARD_END
}

int tbs_memory_allocated(const tbs_ctx *ctx, size_t *bytes) {
    if (!ctx || !bytes) return ctx_fail(nullptr, TBS_ERR_ARG, "null argument");
    *bytes = ctx->bytes + multi_bytes(ctx) + krylov_bytes(ctx);
    return TBS_OK;
}

int tbs_set_inner_sweeps(tbs_ctx *ctx, int m) { return tbs_set_inner_schedule(ctx, m, m); }

int tbs_set_inner_schedule(tbs_ctx *ctx, int first, int rest) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    if (first < 1 || first > 64 || rest < 1 || rest > 64)
        return ctx_fail(ctx, TBS_ERR_ARG, "inner sweeps must be in 1..64");
    const int f = first == rest ? 0 : first;
    if (rest != ctx->inner_sweeps || f != ctx->inner_first) drop_graph(ctx);
    ctx->inner_sweeps = rest;
    ctx->inner_first = f;
    return TBS_OK;
}

int tbs_get_inner_schedule(const tbs_ctx *ctx, int *first, int *rest) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    if (first) *first = ctx->inner_first > 0 ? ctx->inner_first : ctx->inner_sweeps;
    if (rest) *rest = ctx->inner_sweeps;
    return TBS_OK;
}

/* device time of a solve to rel_tol with the schedule (first, rest): best
 * of two after a warm-up; +inf when it does not reach the tolerance */
static int time_schedule(tbs_ctx *ctx, int first, int rest, double rel_tol, int max_sweeps,
                         cudaEvent_t e0, cudaEvent_t e1, double *ms_out) {
    int rc = tbs_set_inner_schedule(ctx, first, rest);
    int sw = 0;
    if (!rc) rc = tbs_solve(ctx, rel_tol, max_sweeps, &sw, nullptr); /* builds the graph */
    double t = 1e300;
    for (int rep = 0; rep < 2 && !rc; ++rep) {
        cudaEventRecord(e0, ctx->stream);
        rc = tbs_solve(ctx, rel_tol, max_sweeps, &sw, nullptr);
        cudaEventRecord(e1, ctx->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        t = std::min(t, (double)ms);
    }
    if (rc) return rc;
    const SolveState &S = *ctx->h_state;
    const bool conv = std::isfinite(S.last) && S.last <= S.tol * S.norm0;
    *ms_out = conv ? t : 1e300;
    return TBS_OK;
}

int tbs_tune_inner(tbs_ctx *ctx, double rel_tol, int max_sweeps, int *best_m, double *best_ms) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->factored || ctx->algo != TBS_ALGO_MIXED)
        return ctx_fail(ctx, TBS_ERR_STATE, "tbs_tune_inner needs a TBS_ALGO_MIXED factorization");
    const bool prof = ctx->prof;
    ctx->prof = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int bf = -1, br = -1;
    double best_t = 1e300;
    int rc = TBS_OK;
    auto consider = [&](int f, int r) {
        if (rc || f < 1 || r < 1) return;
        double t = 1e300;
        rc = time_schedule(ctx, f, r, rel_tol, max_sweeps, e0, e1, &t);
        if (!rc && t < best_t) {
            best_t = t;
            bf = f;
            br = r;
        }
    };
    /* one count for every outer step, then the first step's own count
     * around the best one (the first step starts from the largest
     * residual, and one inner sweep fewer or more there can save an outer
     * step or an inner sweep overall) */
    for (int m : {2, 3, 4, 5, 6, 8, 10}) consider(m, m);
    if (!rc && br > 0) {
        const int m = br;
        for (int r : {m - 1, m, m + 1})
            for (int f : {m - 2, m - 1, m, m + 1, m + 2})
                if (!(f == r && (r == m - 1 || r == m || r == m + 1))) consider(f, r);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->prof = prof;
    if (rc) return rc;
    if (bf < 0) return ctx_fail(ctx, TBS_ERR_NUMERIC, "no inner sweep schedule reached the tolerance");
    rc = tbs_set_inner_schedule(ctx, bf, br);
    if (rc) return rc;
    if (best_m) *best_m = br;
    if (best_ms) *best_ms = best_t;
    return TBS_OK;
    GUARD_END
}

int tbs_profile_enable(tbs_ctx *ctx, int on) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    if (!on) prof_resolve(ctx);
    ctx->prof = on != 0;
    return TBS_OK;
}

int tbs_profile_reset(tbs_ctx *ctx) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    prof_resolve(ctx);
    ctx->slots.clear();
    return TBS_OK;
}

int tbs_profile_read(tbs_ctx *ctx, int *n, const char **names, long long *launches, double *ms) {
    if (!ctx || !n) return ctx_fail(ctx, TBS_ERR_ARG, "null argument");
    prof_resolve(ctx);
    const int cap = *n;
    const int cnt = (int)ctx->slots.size();
    for (int i = 0; i < cnt && i < cap; ++i) {
        if (names) names[i] = ctx->slots[i].name;
        if (launches) launches[i] = ctx->slots[i].launches;
        if (ms) ms[i] = ctx->slots[i].ms;
    }
    *n = cnt;
    return TBS_OK;
}

/* Algorithmic bytes of one launch: every array the kernel must read or
 * write, counted once per read and once per write (block = 648 B, vector
 * entry = 72 B per cell in FP64; halves in FP32). */
int tbs_kernel_bytes(tbs_ctx *ctx, const char *kernel, double *bytes) {
    if (!ctx || !kernel || !bytes) return ctx_fail(ctx, TBS_ERR_ARG, "null argument");
    if (!ctx->have_mesh) return ctx_fail(ctx, TBS_ERR_STATE, "no mesh");
    const double N = ctx->nelem, F = ctx->nintface, nv = ctx->nvar;
    const double blk = nv * nv * 8.0, vec = nv * 8.0;
    const double X = (double)ctx->n_xslots_real;
    const std::string k(kernel);
    double b = -1.0;
    if (k == "fast_resid") /* Dinv, X blocks, xnbr, neighbour dU, b out */
        b = N * (blk + vec) + X * (blk + 4.0 + vec);
    else if (k == "fast_resid_U")
        /* the form that adds dU to U (the batch engine): own dU and U in/out
         * on top */
        b = N * (blk + vec + 3 * vec) + X * (blk + 4.0 + vec);
    else if (k == "fast_resid_rhs" || k == "fast_resid_check") /* Dinv, R in, b out */
        b = N * (blk + 2 * vec);
    else if (k == "fast_resid32_rhs")
        b = N * (blk + 2 * vec) / 2;
    else if (k == "fast_resid32") /* DX blocks, xnbr, neighbour d, b out */
        b = N * vec / 2 + X * (blk / 2 + 4.0 + vec / 2);
    else if (k == "fast_resid32_U") /* the batch engine's: own d + c in/out on top */
        b = N * (4 * vec) / 2 + X * (blk / 2 + 4.0 + vec / 2);
    else if (k == "fast_thomas") /* G, b | Gam, dU out, U in/out (y stays on chip when the
                                  * line fits) */
        b = N * (2 * blk + 4 * vec);
    else if (k == "fast_thomas_dU") /* dU out only (the batch engine) */
        b = N * (2 * blk + 2 * vec);
    else if (k == "fast_thomas32") /* c in/out of all inner solves but the last not counted */
        b = N * (2 * blk + 2 * vec) / 2;
    else if (k == "full_resid" && ctx->algo == TBS_ALGO_MIXED && fullpos_ok(ctx))
        /* position order: D, one block + index + neighbour U per face slot, own U, rhs, R32
         * out, and the next inner right-hand side: Dinv32 in, b32 and c32 out */
        b = N * blk + (double)ctx->n_fslots_real * (blk + 4.0 + vec) + N * (2 * vec + vec / 2) +
            N * (blk / 2 + vec);
    else if (k == "full_resid") /* D, 2 blocks per face, U (own + nbrs), rhs, R out, ints */
        b = N * blk + 2 * F * blk + N * vec + 2 * F * vec + N * vec + N * vec / 2 +
            4.0 * (N + 1 + ctx->eftot + 2 * F + N);
    else if (k == "ref_solve_du") /* DLU, A, DinvC, R, dU out, dU in+out (back) */
        b = N * (3 * blk + 4 * vec) + 4.0 * N;
    else if (k == "ref_add_copy")
        b = N * 5 * vec;
    else if (k == "ref_line_res")
        b = N * blk + 2 * F * blk + N * vec + 2 * F * vec + 2 * N * vec +
            4.0 * (N + 1 + ctx->eftot + 2 * F);
    else if (k.rfind("multi_thomas/", 0) == 0 || k.rfind("multi_resid/", 0) == 0) {
        const int nr = std::atoi(k.c_str() + k.find('/') + 1);
        if (nr >= 1 && nr <= MULTI_MAX) {
            if (k[6] == 't') /* G, Gam once; per r: b in, y out and back in, dU out */
                b = N * 2 * blk + nr * N * 4 * vec;
            else /* Dinv, X blocks + xnbr once; per r: neighbour dU, b out, own dU + U in/out */
                b = N * blk + X * (blk + 4.0) + nr * (N * 4 * vec + X * vec);
        }
    }
    else if (k == "fast_resid_jv") /* X blocks, xnbr, neighbour dU, v in, w out */
        b = N * 2 * vec + X * (blk + 4.0 + vec);
    else if (k == "pij_sweep") /* Dinv, face blocks + index + neighbour dU, own dU, U in/out, b out */
        b = N * (blk + 4 * vec) + (double)ctx->n_fslots_real * (blk + 4.0 + vec);
    else if (k == "fast_factor") /* D, A, C in; Dinv, G, Gam out */
        b = N * blk + 2 * (N - ctx->nline) * blk + 3 * N * blk;
    if (b < 0) return ctx_fail(ctx, TBS_ERR_ARG, "unknown kernel name " + k);
    *bytes = b;
    return TBS_OK;
}

/* ======================================================= line partitions
 * One mesh split into contiguous line ranges, one context per range; each
 * context's mesh ends in halo lines (copies of the neighbouring partitions'
 * boundary lines).  A sweep is split where the halo update goes:
 *   tbs_part_solve_du   line solves of every line (halo lines included)
 *   -- the caller copies each halo line's dU from the line's owner --
 *   tbs_part_line_res   residual from dU, U += dU, norm over the owned lines
 * The per-position arithmetic is that of tbs_sweep on the whole mesh. */

static int part_check(tbs_ctx *ctx) {
    if (!ctx->factored) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
    if (ctx->algo != TBS_ALGO_FP64 || ctx->nvar != 9)
        return ctx_fail(ctx, TBS_ERR_UNSUPPORTED,
                        "line-partition sweeps need TBS_ALGO_FP64 with nvar == 9");
    return TBS_OK;
}

/* the norm that the last residual launch recorded (owned lines only) */
static int part_norm(tbs_ctx *ctx, double *out) {
    int rc = read_state(ctx);
    if (rc) return rc;
    rc = status_check(ctx);
    if (rc) return rc;
    if (out) *out = ctx->h_state->last;
    return TBS_OK;
}

int tbs_part_start(tbs_ctx *ctx, double *owned_norm) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    int rc = part_check(ctx);
    if (rc) return rc;
    rc = ctx_ensure_hist(ctx, 1);
    if (rc) return rc;
    rc = ctx_set_state(ctx, 0.0, 0x7fffffff);
    if (rc) return rc;
    ctx->part_restart = false;
    rc = prime(ctx, CondCtl{});
    if (rc) return rc;
    return part_norm(ctx, owned_norm);
    GUARD_END
}

int tbs_part_solve_du(tbs_ctx *ctx) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    int rc = part_check(ctx);
    if (rc) return rc;
    /* The owned lines' solves write U + dU into the second U buffer as they
     * write dU; tbs_part_line_res adds the halo lines' (copied) dU there and
     * makes it the current U.  Until then U stays the last counted sweep's,
     * so a line solve issued ahead of the convergence test changes nothing
     * that the solve reports. */
    DA(ctx->d_Up_alt, (size_t)ctx->L.np16 * ctx->nvar);
    if (ctx->part_restart) {
        /* the sweeps go on from the true residual of the last check */
        RUN("fast_resid_check", resid64(ctx, 0, ctx->d_dUp, ctx->d_Rp, ctx->d_b, no_sink(), nullptr));
        ctx->part_restart = false;
    }
    RUN("fast_thomas", launch_fast_thomas<double>(ctx->stream, ctx->L, ctx->d_G, ctx->d_Gam, ctx->d_b,
                                                  ctx->d_y, ctx->d_dUp, ctx->d_Up_alt, ctx->d_status, 1,
                                                  ctx->nline - ctx->nhalo, ctx->d_Up));
    return TBS_OK;
    GUARD_END
}

int tbs_part_line_res(tbs_ctx *ctx, double *owned_norm) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    int rc = part_check(ctx);
    if (rc) return rc;
    if (!ctx->d_Up_alt) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_part_solve_du must come first");
    {
        /* the halo tiles' U + dU into the second buffer (the owned lines'
         * were written by their line solves), which becomes the current U */
        NormSink ns = sink(ctx, 0, CondCtl{});
        ns.timer = ctx->d_ktimer;
        RUN("fast_resid", launch_fast_resid<double>(ctx->stream, ctx->L, 1, ctx->d_Dinv, ctx->d_X,
                                                    ctx->d_dUp, nullptr, ctx->d_b, ns, ctx->d_status,
                                                    ctx->d_Up_alt, ctx->L.ntile_own, ctx->d_Up));
        std::swap(ctx->d_Up, ctx->d_Up_alt);
        drop_graph(ctx); /* a captured solve holds the old address */
    }
    if (!owned_norm) return TBS_OK;
    rc = part_norm(ctx, owned_norm);
    if (ctx->prof) prof_resolve(ctx);
    return rc;
    GUARD_END
}

int tbs_part_line_vector(tbs_ctx *ctx, int which, int line, double *d_buf, int to_line) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    int rc = part_check(ctx);
    if (rc) return rc;
    if (which != TBS_VEC_SOLUTION && which != TBS_VEC_UPDATE)
        return ctx_fail(ctx, TBS_ERR_ARG, "which must be TBS_VEC_SOLUTION or TBS_VEC_UPDATE");
    if (line < 0 || line >= ctx->nline) return ctx_fail(ctx, TBS_ERR_ARG, "line out of range");
    if (!d_buf) return ctx_fail(ctx, TBS_ERR_ARG, "null buffer");
    double *v = (which == TBS_VEC_SOLUTION ? ctx->d_Up : ctx->d_dUp) +
                (size_t)ctx->h_line_start[line] * 9;
    const size_t bytes = (size_t)ctx->h_linesize[line] * 9 * sizeof(double);
    if (to_line)
        CK(cudaMemcpyAsync(v, d_buf, bytes, cudaMemcpyDefault, ctx->stream));
    else
        CK(cudaMemcpyAsync(d_buf, v, bytes, cudaMemcpyDefault, ctx->stream));
    return TBS_OK;
    GUARD_END
}

int tbs_part_check(tbs_ctx *ctx, double *owned_norm) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    int rc = part_check(ctx);
    if (rc) return rc;
    /* R = rhs + J U of the owned cells (their halo neighbours' U are the
     * owners' copies) and its owned norm; b = -Dinv R for the next line
     * solves only if sweeps follow (the next tbs_part_solve_du forms it, so
     * a passing check costs no factor read) */
    cudaStream_t st = ctx->stream;
    RUN("full_resid", launch_full_resid<double>(st, ctx->nelem_own, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
                                                ctx->L.pos_of_elem, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                                ctx->d_rhs, ctx->d_Up, ctx->d_Rp, ctx->d_partials2));
    RUN("reduce_norm", launch_reduce_norm(st, ctx->d_partials2, full_resid_blocks(ctx->nelem_own),
                                          ctx->d_state, ctx->d_hist, NORM_CHECK, 0, 0, 0, 0));
    ctx->part_restart = true;
    if (!owned_norm) return TBS_OK;
    return part_norm(ctx, owned_norm);
    GUARD_END
}

int tbs_resid_timer(tbs_ctx *ctx, double *total_us, long long *launches, int reset) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->d_ktimer) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_set_mesh must come first");
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned long long t[3] = {0, 0, 0};
    CK(cudaMemcpy(t, ctx->d_ktimer, sizeof(t), cudaMemcpyDeviceToHost));
    if (total_us) *total_us = 1e-3 * (double)t[1];
    if (launches) *launches = (long long)t[2];
    if (reset) {
        const unsigned long long init[3] = {~0ull, 0ull, 0ull};
        CKL(xfer_put(ctx->stream, ctx->d_ktimer, init, sizeof(init)));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return TBS_OK;
    GUARD_END
}

int tbs_sync(tbs_ctx *ctx) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->d_status) return TBS_OK;
    int rc = status_check(ctx);
    if (rc == TBS_OK && ctx->prof) prof_resolve(ctx);
    return rc;
    GUARD_END
}

int tbs_part_owned_norm(tbs_ctx *ctx, double *d_out) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    int rc = part_check(ctx);
    if (rc) return rc;
    if (!d_out) return ctx_fail(ctx, TBS_ERR_ARG, "null output");
    CK(cudaMemcpyAsync(d_out, &ctx->d_state->last, sizeof(double), cudaMemcpyDefault, ctx->stream));
    return TBS_OK;
    GUARD_END
}

int tbs_part_lines_vector(tbs_ctx *ctx, int which, int nlines, const int *lines, double *d_buf,
                          int to_line) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    int rc = part_check(ctx);
    if (rc) return rc;
    if (which != TBS_VEC_SOLUTION && which != TBS_VEC_UPDATE)
        return ctx_fail(ctx, TBS_ERR_ARG, "which must be TBS_VEC_SOLUTION or TBS_VEC_UPDATE");
    if (nlines < 0 || (nlines > 0 && (!lines || !d_buf)))
        return ctx_fail(ctx, TBS_ERR_ARG, "bad line list or null buffer");
    double *vec = which == TBS_VEC_SOLUTION ? ctx->d_Up : ctx->d_dUp;
    long long off = 0;
    for (int k0 = 0; k0 < nlines; k0 += PACK_MAX_LINES) {
        LinePack lp{};
        lp.n = std::min(PACK_MAX_LINES, nlines - k0);
        for (int j = 0; j < lp.n; ++j) {
            const int l = lines[k0 + j];
            if (l < 0 || l >= ctx->nline) return ctx_fail(ctx, TBS_ERR_ARG, "line out of range");
            lp.start[j] = ctx->h_line_start[l];
            lp.len[j] = ctx->h_linesize[l];
            lp.off[j] = off;
            off += (long long)ctx->h_linesize[l] * 9;
        }
        RUN("line_pack", launch_line_pack(ctx->stream, lp, vec, d_buf, to_line));
    }
    return TBS_OK;
    GUARD_END
}

}  // extern "C"

/* the server's re-factorizations (csrc/server.cu) */
int ctx_set_jacobian_paced(tbs_ctx *ctx, const double *jacD, const double *jacO1, const double *jacO2,
                           const double *rhs, size_t piece) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    return upload_jacobian(ctx, jacD, jacO1, jacO2, rhs, cudaMemcpyHostToDevice, piece);
    GUARD_END
}



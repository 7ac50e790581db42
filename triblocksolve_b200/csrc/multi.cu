/*
 * multi.cu -- tbs_solve_multi / tbs_solve_multi_device: several
 * right-hand sides of one factored system (TBS_ALGO_FP64) solved together.
 *
 * Groups of up to MULTI_MAX right-hand sides run as one CUDA graph
 *     prime (R = rhs_r, U_r = 0, b_r = -Dinv R, norms; all r active)
 *     -> while (any r active) { line solves of the active r;
 *                               residual, U_r += dU_r, norms }
 * so the line blocks (G, Gam, Dinv, X) cross HBM once per sweep for the
 * whole group instead of once per right-hand side.  A right-hand side
 * retires at the sweep where its own test ends a tbs_solve of it, and the
 * per-element arithmetic and norm sums are those of tbs_solve: each
 * right-hand side's solution, sweep count and norm history equal
 * tbs_set_rhs + tbs_solve of it alone, bit for bit.
 *
 * The reference's driver solves one right-hand side per run
 * (src/main.cxx:180-229); this is the multi-RHS form of that loop.
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

struct MultiBufs {
    int cap = 0;          /* right-hand sides the vectors hold */
    int hist_stride = 0;  /* device history entries per right-hand side */
    size_t bytes = 0;
    std::vector<void *> allocs;
    double *U = nullptr, *dU = nullptr, *b = nullptr, *y = nullptr, *rhsp = nullptr;
    double *partials = nullptr, *hist = nullptr, *elem = nullptr;
    SolveState *state = nullptr;
    SolveState *h_state = nullptr; /* pinned [MULTI_MAX] */
    int *active = nullptr;
    int *h_active = nullptr;       /* pinned [MULTI_MAX] */
    unsigned *counter = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int graph_nr = 0;
    const void *graph_key[5] = {};
};

static int mfail(tbs_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    set_thread_error(msg);
    return code;
}

#define MCK(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return mfail(ctx, TBS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define MCKL(call)                                                                         \
    do {                                                                                   \
        int e_ = (call);                                                                   \
        if (e_ != 0)                                                                       \
            return mfail(ctx, TBS_ERR_CUDA,                                                \
                         std::string(#call) + ": " + cudaGetErrorString((cudaError_t)e_)); \
    } while (0)

#define MRUN(name, call)                         \
    do {                                         \
        const int h_ = ctx_prof_begin(ctx, name); \
        const int rv_ = (int)(call);             \
        ctx_prof_end(ctx, h_);                   \
        MCKL(rv_);                               \
    } while (0)

static void multi_drop_graph_(MultiBufs *m) {
    if (m->gexec) cudaGraphExecDestroy(m->gexec);
    if (m->graph) cudaGraphDestroy(m->graph);
    m->gexec = nullptr;
    m->graph = nullptr;
    m->graph_nr = 0;
}

void multi_drop_graph(tbs_ctx *ctx) {
    if (ctx && ctx->multi) multi_drop_graph_(ctx->multi);
}

static void multi_free_vectors(MultiBufs *m) {
    multi_drop_graph_(m);
    for (void *p : m->allocs) cudaFree(p);
    m->allocs.clear();
    m->bytes = 0;
    m->U = m->dU = m->b = m->y = m->rhsp = m->partials = m->hist = m->elem = nullptr;
    m->state = nullptr;
    m->active = nullptr;
    m->counter = nullptr;
    m->cap = 0;
    m->hist_stride = 0;
}

void multi_free(tbs_ctx *ctx) {
    if (!ctx || !ctx->multi) return;
    MultiBufs *m = ctx->multi;
    multi_free_vectors(m);
    if (m->h_state) cudaFreeHost(m->h_state);
    if (m->h_active) cudaFreeHost(m->h_active);
    delete m;
    ctx->multi = nullptr;
}

size_t multi_bytes(const tbs_ctx *ctx) { return ctx && ctx->multi ? ctx->multi->bytes : 0; }

template <typename T>
static int malloc_zero(tbs_ctx *ctx, MultiBufs *m, T **p, size_t count) {
    const size_t nbytes = std::max<size_t>(count, 1) * sizeof(T);
    void *q = nullptr;
    if (cudaMalloc(&q, nbytes) != cudaSuccess) {
        cudaGetLastError();
        return mfail(ctx, TBS_ERR_NOMEM, "cudaMalloc of " + std::to_string(nbytes) + " bytes failed");
    }
    m->allocs.push_back(q);
    m->bytes += nbytes;
    *p = static_cast<T *>(q);
    MCK(cudaMemsetAsync(q, 0, nbytes, ctx->stream)); /* pads of every vector stay zero */
    return TBS_OK;
}

#define MA(ptr, n)                                  \
    do {                                            \
        int s_ = malloc_zero(ctx, m, &(ptr), (n));  \
        if (s_) return s_;                          \
    } while (0)

/* vectors for `cap` right-hand sides and `hist` norms each */
static int multi_ensure(tbs_ctx *ctx, int cap, int hist) {
    if (!ctx->multi) {
        ctx->multi = new MultiBufs();
        MultiBufs *m = ctx->multi;
        if (cudaMallocHost((void **)&m->h_state, MULTI_MAX * sizeof(SolveState)) != cudaSuccess ||
            cudaMallocHost((void **)&m->h_active, MULTI_MAX * sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            multi_free(ctx);
            return mfail(ctx, TBS_ERR_NOMEM, "pinned host allocation failed");
        }
    }
    MultiBufs *m = ctx->multi;
    if (m->cap >= cap && m->hist_stride >= hist) return TBS_OK;
    MCK(cudaStreamSynchronize(ctx->stream));
    cap = std::max(cap, m->cap);
    hist = std::max({hist, m->hist_stride, 1024});
    multi_free_vectors(m);
    const size_t vs = (size_t)ctx->L.np16 * 9;
    const size_t ne = (size_t)ctx->nelem * 9;
    const size_t ntiles = (size_t)ctx->L.np16 / RES_TILE;
    MA(m->U, cap * vs);
    MA(m->dU, cap * vs);
    MA(m->b, cap * vs);
    MA(m->y, cap * vs);
    MA(m->rhsp, cap * vs);
    MA(m->elem, cap * ne);
    MA(m->partials, cap * ntiles);
    MA(m->hist, (size_t)cap * hist);
    MA(m->state, (size_t)MULTI_MAX);
    MA(m->active, (size_t)MULTI_MAX);
    MA(m->counter, (size_t)1);
    m->cap = cap;
    m->hist_stride = hist;
    return TBS_OK;
}

static MultiSys multi_sys(tbs_ctx *ctx, int nr) {
    MultiBufs *m = ctx->multi;
    MultiSys M{};
    M.nr = nr;
    M.np16 = ctx->L.np16;
    M.nx = ctx->L.nx;
    M.hist_stride = m->hist_stride;
    M.U = m->U;
    M.b = m->b;
    M.partials = m->partials;
    M.hist = m->hist;
    M.dU = m->dU;
    M.state = m->state;
    M.active = m->active;
    M.counter = m->counter;
    return M;
}

static int multi_prime(tbs_ctx *ctx, int nr, unsigned long long h, int use_cond) {
    MultiBufs *m = ctx->multi;
    MRUN("multi_resid_rhs", launch_multi_resid(ctx->stream, ctx->L, 0, multi_sys(ctx, nr), ctx->d_Dinv,
                                               ctx->d_X, m->rhsp, h, use_cond, ctx->d_status));
    return TBS_OK;
}

static int multi_sweep(tbs_ctx *ctx, int nr, unsigned long long h, int use_cond) {
    MultiBufs *m = ctx->multi;
    MRUN("multi_thomas", launch_multi_thomas(ctx->stream, ctx->L, nr, ctx->d_G, ctx->d_Gam, m->b, m->y,
                                             m->dU, m->active, ctx->d_status));
    MRUN("multi_resid", launch_multi_resid(ctx->stream, ctx->L, 1, multi_sys(ctx, nr), ctx->d_Dinv,
                                           ctx->d_X, nullptr, h, use_cond, ctx->d_status));
    return TBS_OK;
}

/* prime -> while (any active) { sweep } for nr right-hand sides */
static int multi_build_graph(tbs_ctx *ctx, int nr) {
    MultiBufs *m = ctx->multi;
    multi_drop_graph_(m);
    cudaStream_t st = ctx->stream;
    MCK(cudaGraphCreate(&m->graph, 0));
    cudaGraphConditionalHandle hw;
    MCK(cudaGraphConditionalHandleCreate(&hw, m->graph, 0, cudaGraphCondAssignDefault));
    MCK(cudaStreamBeginCaptureToGraph(st, m->graph, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal));
    int rc = multi_prime(ctx, nr, (unsigned long long)hw, 1);
    cudaGraph_t bodyg = nullptr;
    if (rc == TBS_OK) {
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &ndeps);
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hw;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        if (e == cudaSuccess) e = cudaGraphAddNode(&node, m->graph, deps, ndeps, &cp);
        if (e == cudaSuccess) {
            bodyg = cp.conditional.phGraph_out[0];
            e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
        }
        if (e != cudaSuccess)
            rc = mfail(ctx, TBS_ERR_CUDA, std::string("while node: ") + cudaGetErrorString(e));
    }
    cudaGraph_t outg = nullptr;
    cudaError_t ee = cudaStreamEndCapture(st, &outg);
    if (rc == TBS_OK && ee != cudaSuccess)
        rc = mfail(ctx, TBS_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ee));
    if (rc == TBS_OK) {
        MCK(cudaStreamBeginCaptureToGraph(st, bodyg, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal));
        rc = multi_sweep(ctx, nr, (unsigned long long)hw, 1);
        ee = cudaStreamEndCapture(st, &outg);
        if (rc == TBS_OK && ee != cudaSuccess)
            rc = mfail(ctx, TBS_ERR_CUDA, std::string("end body capture: ") + cudaGetErrorString(ee));
    }
    if (rc == TBS_OK) {
        ee = cudaGraphInstantiate(&m->gexec, m->graph, 0);
        if (ee != cudaSuccess)
            rc = mfail(ctx, TBS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ee));
    }
    if (rc != TBS_OK) {
        multi_drop_graph_(m);
        return rc;
    }
    m->graph_nr = nr;
    m->graph_key[0] = ctx->d_G;
    m->graph_key[1] = ctx->d_Gam;
    m->graph_key[2] = ctx->d_Dinv;
    m->graph_key[3] = ctx->d_X;
    m->graph_key[4] = m->U;
    return TBS_OK;
}

static bool graph_valid(const tbs_ctx *ctx, int nr) {
    const MultiBufs *m = ctx->multi;
    return m->gexec && m->graph_nr == nr && m->graph_key[0] == ctx->d_G &&
           m->graph_key[1] == ctx->d_Gam && m->graph_key[2] == ctx->d_Dinv &&
           m->graph_key[3] == ctx->d_X && m->graph_key[4] == m->U;
}

/* one group: rhs (device, element order, nr vectors) -> U (device,
 * element order); sweeps / hist (host) per right-hand side */
static int multi_group(tbs_ctx *ctx, int nr, const double *d_rhs, double *d_U, double tol,
                       int max_sweeps, int *sweeps, double *hist, int hist_stride) {
    MultiBufs *m = ctx->multi;
    cudaStream_t st = ctx->stream;
    const int ne = ctx->nelem;
    const size_t nv = (size_t)ne * 9, vs = (size_t)ctx->L.np16 * 9;
    for (int r = 0; r < nr; ++r)
        MRUN("permute", launch_permute_to_pos(st, 9, ne, ctx->L.pos_of_elem, d_rhs + r * nv, m->rhsp + r * vs));
    for (int r = 0; r < nr; ++r) {
        SolveState &S = m->h_state[r];
        std::memset(&S, 0, sizeof(S));
        S.tol = tol;
        S.max_sweeps = max_sweeps;
        S.hist_cap = m->hist_stride;
    }
    MCK(cudaMemcpyAsync(m->state, m->h_state, nr * sizeof(SolveState), cudaMemcpyHostToDevice, st));
    MCKL(multi_prepare(ctx->L, nr));
    if (ctx->prof) {
        /* eager form with a host-side test */
        int rc = multi_prime(ctx, nr, 0, 0);
        if (rc) return rc;
        for (;;) {
            MCK(cudaMemcpyAsync(m->h_active, m->active, nr * sizeof(int), cudaMemcpyDeviceToHost, st));
            MCK(cudaStreamSynchronize(st));
            bool any = false;
            for (int r = 0; r < nr; ++r) any = any || m->h_active[r] != 0;
            if (!any) break;
            rc = multi_sweep(ctx, nr, 0, 0);
            if (rc) return rc;
        }
        ctx_prof_resolve(ctx);
    } else {
        if (!graph_valid(ctx, nr)) {
            int rc = multi_build_graph(ctx, nr);
            if (rc) return rc;
        }
        MCK(cudaGraphLaunch(m->gexec, st));
    }
    for (int r = 0; r < nr; ++r)
        MRUN("permute", launch_permute_to_elem(st, 9, ne, ctx->L.pos_of_elem, m->U + r * vs, d_U + r * nv));
    MCK(cudaMemcpyAsync(m->h_state, m->state, nr * sizeof(SolveState), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    int rc = ctx_status(ctx);
    if (rc) return rc;
    for (int r = 0; r < nr; ++r) {
        const int sw = m->h_state[r].sweep;
        if (sweeps) sweeps[r] = sw;
        if (hist && hist_stride > 0) {
            const int nh = std::min(std::min(sw, max_sweeps) + 1, hist_stride);
            MCK(cudaMemcpyAsync(hist + (size_t)r * hist_stride, m->hist + (size_t)r * m->hist_stride,
                                nh * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
    }
    MCK(cudaStreamSynchronize(st));
    return TBS_OK;
}

static int multi_check(tbs_ctx *ctx, int nrhs, const void *rhs, const void *U, double tol,
                       int max_sweeps, const double *hist, int hist_stride) {
    if (!ctx->factored) return mfail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
    if (ctx->algo != TBS_ALGO_FP64 || ctx->nvar != 9)
        return mfail(ctx, TBS_ERR_UNSUPPORTED, "several right-hand sides need TBS_ALGO_FP64 and nvar == 9");
    if (ctx->nhalo > 0) return mfail(ctx, TBS_ERR_UNSUPPORTED, "a line partition sweeps with tbs_part_solve_du / tbs_part_line_res");
    if (ctx->lagged)
        return mfail(ctx, TBS_ERR_UNSUPPORTED,
                     "block values are newer than the factorization (tbs_update_values); several "
                     "right-hand sides track the residual with the factorization's blocks: re-factor");
    if (nrhs < 0 || (nrhs > 0 && (!rhs || !U)))
        return mfail(ctx, TBS_ERR_ARG, "bad right-hand-side count or null arrays");
    if (max_sweeps < 0 || !(tol >= 0.0)) return mfail(ctx, TBS_ERR_ARG, "bad tolerance or sweep limit");
    if (hist && hist_stride < 1) return mfail(ctx, TBS_ERR_ARG, "hist_stride must be >= 1");
    return TBS_OK;
}

static int multi_run(tbs_ctx *ctx, int nrhs, const double *rhs, double *U, bool host, double tol,
                     int max_sweeps, int *sweeps, double *hist, int hist_stride) {
    cudaStream_t st = ctx->stream;
    const int g = std::min(nrhs, MULTI_MAX);
    int rc = multi_ensure(ctx, g, max_sweeps + 1);
    if (rc) return rc;
    MultiBufs *m = ctx->multi;
    const size_t nv = (size_t)ctx->nelem * 9;
    for (int r0 = 0; r0 < nrhs; r0 += MULTI_MAX) {
        const int nr = std::min(MULTI_MAX, nrhs - r0);
        const double *d_rhs = rhs + r0 * nv;
        double *d_U = U + r0 * nv;
        if (host) {
            MCK(cudaMemcpyAsync(m->elem, rhs + r0 * nv, nr * nv * sizeof(double),
                                cudaMemcpyHostToDevice, st));
            d_rhs = m->elem;
            d_U = m->elem; /* each r's rhs is permuted before any U lands here */
        }
        rc = multi_group(ctx, nr, d_rhs, d_U, tol, max_sweeps, sweeps ? sweeps + r0 : nullptr,
                         hist ? hist + (size_t)r0 * hist_stride : nullptr, hist_stride);
        if (rc) return rc;
        if (host) {
            MCK(cudaMemcpyAsync(U + r0 * nv, m->elem, nr * nv * sizeof(double),
                                cudaMemcpyDeviceToHost, st));
            MCK(cudaStreamSynchronize(st));
        }
    }
    return TBS_OK;
}

#define MGUARD_BEGIN try {
#define MGUARD_END                                                  \
    }                                                               \
    catch (const std::bad_alloc &) {                                \
        return mfail(ctx, TBS_ERR_NOMEM, "host allocation failed"); \
    }                                                               \
    catch (...) {                                                   \
        return mfail(ctx, TBS_ERR_STATE, "internal error");         \
    }

extern "C" {

int tbs_solve_multi(tbs_ctx *ctx, int nrhs, const double *rhs, double *U, double rel_tol,
                    int max_sweeps, int *sweeps, double *hist, int hist_stride) {
    if (!ctx) return mfail(nullptr, TBS_ERR_ARG, "null context");
    MGUARD_BEGIN
    MCK(cudaSetDevice(ctx->device));
    int rc = multi_check(ctx, nrhs, rhs, U, rel_tol, max_sweeps, hist, hist_stride);
    if (rc || nrhs == 0) return rc;
    return multi_run(ctx, nrhs, rhs, U, true, rel_tol, max_sweeps, sweeps, hist, hist_stride);
    MGUARD_END
}

int tbs_solve_multi_device(tbs_ctx *ctx, int nrhs, const double *d_rhs, double *d_U,
                           double rel_tol, int max_sweeps, int *sweeps, double *hist,
                           int hist_stride) {
    if (!ctx) return mfail(nullptr, TBS_ERR_ARG, "null context");
    MGUARD_BEGIN
    MCK(cudaSetDevice(ctx->device));
    int rc = multi_check(ctx, nrhs, d_rhs, d_U, rel_tol, max_sweeps, hist, hist_stride);
    if (rc || nrhs == 0) return rc;
    return multi_run(ctx, nrhs, d_rhs, d_U, false, rel_tol, max_sweeps, sweeps, hist, hist_stride);
    MGUARD_END
}

} /* extern "C" */

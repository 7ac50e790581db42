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
#include "tbs_internal.hxx"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using namespace tbs;

namespace {

struct ProfSlot {
    const char *name;
    long long launches;
    double ms;
};

struct PendingEvent {
    int slot;
    cudaEvent_t a, b;
};

}  // namespace

struct tbs_ctx {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;

    /* ---- mesh ---- */
    bool have_mesh = false, have_jac = false, factored = false;
    int nvar = 0, nelem = 0, nintface = 0, eftot = 0, nline = 0, nlineelem = 0, max_line = 0;
    std::vector<int> h_epoint, h_ef, h_fc, h_linesize, h_linepoint, h_lines, h_lineface;
    int *d_epoint = nullptr, *d_ef = nullptr, *d_fc = nullptr, *d_linesize = nullptr;
    int *d_linepoint = nullptr, *d_lines = nullptr, *d_lineface = nullptr, *d_identity = nullptr;

    /* ---- Jacobian (element / face order, as read) ---- */
    double *d_jacD = nullptr, *d_O1 = nullptr, *d_O2 = nullptr, *d_rhs = nullptr;
    double *d_U = nullptr, *d_dU = nullptr, *d_R = nullptr, *d_Uinit = nullptr;
    double *d_scratch = nullptr; /* 9*nelem element-order scratch */

    /* ---- TBS_ALGO_REFERENCE ---- */
    double *d_DLU = nullptr, *d_DinvC = nullptr, *d_A = nullptr;

    /* ---- line-ordered layout (FP64 / MIXED) ---- */
    FastLayout L{};
    bool layout_ok = false;
    double *d_gamlast = nullptr; /* per line and chain: last Gam toward the twist, FP64 */
    long long n_xslots_real = 0;
    double *d_Dinv = nullptr, *d_G = nullptr, *d_Gam = nullptr, *d_X = nullptr;
    double *d_Up = nullptr, *d_dUp = nullptr, *d_b = nullptr, *d_y = nullptr;
    double *d_rhsp = nullptr, *d_Rp = nullptr;
    float *d_Dinv32 = nullptr, *d_G32 = nullptr, *d_Gam32 = nullptr, *d_X32 = nullptr;
    float *d_b32 = nullptr, *d_y32 = nullptr, *d_d32 = nullptr, *d_c32 = nullptr,
          *d_R32 = nullptr;
    int inner_sweeps = 4;

    /* ---- norms / solve state ---- */
    double *d_partials = nullptr, *d_partials2 = nullptr;
    int npart_cap = 0;
    SolveState *d_state = nullptr;
    SolveState *h_state = nullptr; /* pinned */
    double *d_hist = nullptr;
    int hist_cap = 0;
    unsigned *d_status = nullptr;
    unsigned *h_status = nullptr; /* pinned */
    unsigned *d_counter = nullptr; /* last-CTA ticket of the fused norm */
    int algo = -1;

    /* ---- graph cache ---- */
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    int graph_algo = -1;

    /* ---- memory accounting ---- */
    std::vector<std::pair<void *, size_t>> allocs;
    size_t bytes = 0;

    /* ---- profiling ---- */
    bool prof = false;
    std::vector<ProfSlot> slots;
    std::vector<PendingEvent> pending;
    std::vector<cudaEvent_t> pool;
};

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
    drop_graph(ctx);
    for (auto &a : ctx->allocs) cudaFree(a.first);
    ctx->allocs.clear();
    ctx->bytes = 0;
    double **dps[] = {&ctx->d_jacD, &ctx->d_O1, &ctx->d_O2, &ctx->d_rhs, &ctx->d_U, &ctx->d_dU,
                      &ctx->d_R, &ctx->d_Uinit, &ctx->d_scratch, &ctx->d_DLU, &ctx->d_DinvC,
                      &ctx->d_A, &ctx->d_Dinv, &ctx->d_G, &ctx->d_Gam, &ctx->d_X, &ctx->d_Up,
                      &ctx->d_dUp, &ctx->d_b, &ctx->d_y, &ctx->d_rhsp, &ctx->d_Rp,
                      &ctx->d_partials, &ctx->d_partials2, &ctx->d_hist, &ctx->d_gamlast};
    for (auto p : dps) *p = nullptr;
    float **fps[] = {&ctx->d_Dinv32, &ctx->d_G32, &ctx->d_Gam32, &ctx->d_X32, &ctx->d_b32,
                     &ctx->d_y32, &ctx->d_d32, &ctx->d_c32, &ctx->d_R32};
    for (auto p : fps) *p = nullptr;
    int **ips[] = {&ctx->d_epoint, &ctx->d_ef, &ctx->d_fc, &ctx->d_linesize, &ctx->d_linepoint,
                   &ctx->d_lines, &ctx->d_lineface, &ctx->d_identity, &ctx->L.line_start,
                   &ctx->L.line_len, &ctx->L.line_twist, &ctx->L.pos_of_elem, &ctx->L.elem_of_pos, &ctx->L.xnbr,
                   &ctx->L.xsrc, &ctx->L.fsrc};
    for (auto p : ips) *p = nullptr;
    ctx->d_state = nullptr;
    ctx->d_status = nullptr;
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

/* ============================================================ layout (host) */

static int build_layout(tbs_ctx *ctx) {
    const int nline = ctx->nline, nelem = ctx->nelem;
    const int *ls = ctx->h_linesize.data(), *lp = ctx->h_linepoint.data();
    const int *lines = ctx->h_lines.data(), *lf = ctx->h_lineface.data();
    const int *fc = ctx->h_fc.data(), *ep = ctx->h_epoint.data(), *ef = ctx->h_ef.data();
    std::vector<int> start(nline), len(nline), twist(nline);
    long long np = 0;
    for (int l = 0; l < nline; ++l) {
        start[l] = (int)np;
        len[l] = ls[l];
        twist[l] = line_twist_of(ls[l]);
        np += (ls[l] + 3) & ~3;
    }
    if (np > 0x7fffffffLL / 81)
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
    FastLayout &L = ctx->L;
    L.nv = ctx->nvar;
    L.np = (int)np;
    L.np16 = np16;
    L.nx = nx;
    L.nline = nline;
    L.max_len = ctx->max_line;
    ctx->n_xslots_real = nreal;
    DA(L.line_start, nline);
    DA(L.line_len, nline);
    DA(L.line_twist, nline);
    DA(L.pos_of_elem, nelem);
    DA(L.elem_of_pos, np16);
    DA(L.fsrc, (size_t)np16 * 5);
    DA(L.xsrc, (size_t)np16 * std::max(nx, 1));
    DA(L.xnbr, (size_t)np16 * std::max(nx, 1));
    DA(ctx->d_gamlast, (size_t)nline * 2 * 81);
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(L.line_start, start.data(), nline * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.line_len, len.data(), nline * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.line_twist, twist.data(), nline * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.pos_of_elem, pos_of_elem.data(), nelem * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.elem_of_pos, elem_of_pos.data(), np16 * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.fsrc, fsrc.data(), fsrc.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.xsrc, xsrc.data(), xsrc.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(L.xnbr, xnbr.data(), xnbr.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    /* the residual kernel stages RES_TILE cells x nx blocks per tile; beyond
     * 4 cross-line couplings per cell it would not fit in shared memory,
     * and such meshes use TBS_ALGO_REFERENCE */
    ctx->layout_ok = (ctx->nvar == 9) && nx <= 4;
    return TBS_OK;
}

/* ============================================================ sequences */

static int status_check(tbs_ctx *ctx) {
    CK(cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const unsigned s = *ctx->h_status;
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

static long long nvec(tbs_ctx *ctx) { return (long long)ctx->nvar * ctx->nelem; }

/* How a sequence ends: the norm of its residual is recorded as the start
 * of a solve (is_start) or as one more sweep, and, inside the solve graph,
 * sets the while-node's condition. */
struct CondCtl {
    unsigned long long handle;
    int use_cond;
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
    return ns;
}

static NormSink no_sink() { return NormSink{}; }

static int reduce(tbs_ctx *ctx, int npart, int is_start, CondCtl cc) {
    RUN("reduce_norm", launch_reduce_norm(ctx->stream, ctx->d_partials, npart, ctx->d_state,
                                          ctx->d_hist, is_start, cc.handle, cc.use_cond));
    return TBS_OK;
}

/* Bring the state to "U = U_init, residual of U known and recorded as
 * ||R_0||", with the first sweep's inputs ready. */
static int prime(tbs_ctx *ctx, CondCtl cc) {
    cudaStream_t st = ctx->stream;
    const int nv = ctx->nvar, ne = ctx->nelem;
    const size_t vb = (size_t)nvec(ctx) * sizeof(double);
    if (ctx->algo == TBS_ALGO_REFERENCE) {
        int np = 0;
        CK(cudaMemcpyAsync(ctx->d_R, ctx->d_rhs, vb, cudaMemcpyDeviceToDevice, st));
        if (ctx->d_Uinit) {
            CK(cudaMemcpyAsync(ctx->d_U, ctx->d_Uinit, vb, cudaMemcpyDeviceToDevice, st));
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
    if (ctx->algo == TBS_ALGO_FP64) {
        const double *Rsrc = ctx->d_rhsp;
        if (ctx->d_Uinit) {
            RUN("permute", launch_permute_to_pos(st, 9, ne, L.pos_of_elem, ctx->d_Uinit, ctx->d_Up));
            RUN("full_resid", launch_full_resid<double>(st, ne, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
                                                        L.pos_of_elem, ctx->d_jacD, ctx->d_O1,
                                                        ctx->d_O2, ctx->d_rhs, ctx->d_Up, ctx->d_Rp,
                                                        ctx->d_partials2));
            Rsrc = ctx->d_Rp;
        }
        /* from U = 0 the same launch clears U */
        RUN("fast_resid_rhs", launch_fast_resid<double>(st, L, 0, ctx->d_Dinv, ctx->d_X, ctx->d_dUp,
                                                        Rsrc, ctx->d_b, sink(ctx, 1, cc),
                                                        ctx->d_status,
                                                        ctx->d_Uinit ? nullptr : ctx->d_Up));
        return TBS_OK;
    }
    /* TBS_ALGO_MIXED */
    if (ctx->d_Uinit) {
        RUN("permute", launch_permute_to_pos(st, 9, ne, L.pos_of_elem, ctx->d_Uinit, ctx->d_Up));
        RUN("full_resid", launch_full_resid<float>(st, ne, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
                                                   L.pos_of_elem, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                                   ctx->d_rhs, ctx->d_Up, ctx->d_R32,
                                                   ctx->d_partials));
        return reduce(ctx, full_resid_blocks(ne), 1, cc);
    }
    RUN("mixed_prime", launch_mixed_prime(st, L, ctx->d_rhsp, ctx->d_R32, ctx->d_Up, ctx->d_partials));
    return reduce(ctx, fast_resid_grid(L.np16), 1, cc);
}

/* One sweep from the primed state, ending with the new residual's norm
 * recorded as one more sweep. */
static int body(tbs_ctx *ctx, CondCtl cc) {
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
    if (ctx->algo == TBS_ALGO_FP64) {
        /* the Thomas kernel writes dU; the residual kernel adds it to U */
        RUN("fast_thomas", launch_fast_thomas<double>(st, L, ctx->d_G, ctx->d_Gam, ctx->d_b, ctx->d_y,
                                                      ctx->d_dUp, ctx->d_Up, ctx->d_status, 2));
        RUN("fast_resid", launch_fast_resid<double>(st, L, 1, ctx->d_Dinv, ctx->d_X, ctx->d_dUp,
                                                    nullptr, ctx->d_b, sink(ctx, 0, cc),
                                                    ctx->d_status, ctx->d_Up));
        return TBS_OK;
    }
    /* TBS_ALGO_MIXED: inner FP32 LIJ sweeps on J d = -R, then U += d and the
     * FP64 residual R = rhs + J U from the original blocks */
    /* c = sum of the inner updates but the last: this launch clears c, each
     * inner residual kernel adds its sweep's d to c; the last d is added
     * with c to U below */
    RUN("fast_resid32_rhs", launch_fast_resid<float>(st, L, 0, ctx->d_Dinv32, ctx->d_X32, ctx->d_d32,
                                                     ctx->d_R32, ctx->d_b32, no_sink(), ctx->d_status,
                                                     ctx->d_c32));
    for (int m = 0; m < ctx->inner_sweeps; ++m) {
        RUN("fast_thomas32", launch_fast_thomas<float>(st, L, ctx->d_G32, ctx->d_Gam32, ctx->d_b32,
                                                       ctx->d_y32, ctx->d_d32, ctx->d_c32,
                                                       ctx->d_status, 2));
        if (m + 1 < ctx->inner_sweeps)
            RUN("fast_resid32", launch_fast_resid<float>(st, L, 3, nullptr, ctx->d_X32, ctx->d_d32,
                                                         nullptr, ctx->d_b32, no_sink(),
                                                         ctx->d_status, ctx->d_c32));
    }
    RUN("axpy", launch_axpy2_f32_f64(st, ctx->d_c32, ctx->d_d32, ctx->d_Up, (long long)L.np16 * 9));
    RUN("full_resid", launch_full_resid<float>(st, ne, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
                                               L.pos_of_elem, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                               ctx->d_rhs, ctx->d_Up, ctx->d_R32, ctx->d_partials));
    return reduce(ctx, full_resid_blocks(ne), 0, cc);
}

static int ensure_hist(tbs_ctx *ctx, int need) {
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
static int set_state(tbs_ctx *ctx, double tol, int max_sweeps) {
    SolveState *h = ctx->h_state;
    h->tol = tol;
    h->max_sweeps = max_sweeps;
    h->hist_cap = ctx->hist_cap;
    const size_t off = offsetof(SolveState, tol);
    CK(cudaMemcpyAsync(reinterpret_cast<char *>(ctx->d_state) + off,
                       reinterpret_cast<char *>(h) + off, sizeof(SolveState) - off,
                       cudaMemcpyHostToDevice, ctx->stream));
    return TBS_OK;
}

static int read_state(tbs_ctx *ctx) {
    CK(cudaMemcpyAsync(ctx->h_state, ctx->d_state, sizeof(SolveState), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TBS_OK;
}

/* Graph: prime (records ||R_0||, sets the condition) -> while (cond) { sweep } */
static int build_graph(tbs_ctx *ctx) {
    drop_graph(ctx);
    cudaStream_t st = ctx->stream;
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    ctx->graph = g;
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    const CondCtl cc{(unsigned long long)h, 1};
    CK(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int rc = prime(ctx, cc);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    if (rc == TBS_OK) {
        cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &ndeps);
        if (e != cudaSuccess) rc = ctx_fail(ctx, TBS_ERR_CUDA, std::string("capture info: ") + cudaGetErrorString(e));
    }
    cudaGraphNode_t cnode = nullptr;
    cudaGraph_t bodyg = nullptr;
    if (rc == TBS_OK) {
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaError_t e = cudaGraphAddNode(&cnode, g, deps, ndeps, &cp);
        if (e != cudaSuccess) rc = ctx_fail(ctx, TBS_ERR_CUDA, std::string("conditional node: ") + cudaGetErrorString(e));
        else bodyg = cp.conditional.phGraph_out[0];
    }
    if (rc == TBS_OK) {
        cudaError_t e = cudaStreamUpdateCaptureDependencies(st, &cnode, 1, cudaStreamSetCaptureDependencies);
        if (e != cudaSuccess) rc = ctx_fail(ctx, TBS_ERR_CUDA, std::string("capture deps: ") + cudaGetErrorString(e));
    }
    cudaGraph_t outg = nullptr;
    cudaError_t ee = cudaStreamEndCapture(st, &outg);
    if (rc == TBS_OK && ee != cudaSuccess) rc = ctx_fail(ctx, TBS_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ee));
    if (rc != TBS_OK) {
        drop_graph(ctx);
        return rc;
    }
    CK(cudaStreamBeginCaptureToGraph(st, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    rc = body(ctx, cc);
    ee = cudaStreamEndCapture(st, &outg);
    if (rc == TBS_OK && ee != cudaSuccess) rc = ctx_fail(ctx, TBS_ERR_CUDA, std::string("end body capture: ") + cudaGetErrorString(ee));
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
    const size_t bs = 81, ne = ctx->nelem;
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
    const size_t npb = (size_t)L.np16 * bs, npv = (size_t)L.np16 * 9;
    const size_t nxb = (size_t)L.np16 * std::max(L.nx, 1) * bs;
    DA(ctx->d_Up, npv);
    DA(ctx->d_rhsp, npv);
    DA(ctx->d_Rp, npv);
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
        CK(cudaMemcpyAsync(ctx->d_DLU, ctx->d_jacD, nb * sizeof(double), cudaMemcpyDeviceToDevice, st));
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
    CKL(fast_prepare(L));
    RUN("permute", launch_permute_to_pos(st, 9, ctx->nelem, L.pos_of_elem, ctx->d_rhs, ctx->d_rhsp));
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
    if (e == cudaSuccess) e = cudaMallocHost((void **)&ctx->h_state, sizeof(SolveState));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&ctx->h_status, sizeof(unsigned));
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
        ctx->stream = ns;
    }
    return TBS_OK;
}

int tbs_set_mesh(tbs_ctx *ctx, int nvar, int nelem, int nintface, int eftot, int nline,
                 int nlineelem, const int *epoint, const int *ef, const int *fc,
                 const int *linesize, const int *linepoint, const int *lines,
                 const int *lineface) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    int hdr[6] = {nvar, nelem, nintface, eftot, nline, nlineelem};
    int st = validate_mesh(hdr, epoint, ef, fc, linesize, linepoint, lines, lineface);
    if (st) return ctx_fail(ctx, st, thread_error());
    if (nvar > 32) return ctx_fail(ctx, TBS_ERR_UNSUPPORTED, "nvar > 32 is not supported");
    CK(cudaStreamSynchronize(ctx->stream));
    drop_mesh(ctx);
    CK(cudaMalloc((void **)&ctx->d_status, sizeof(unsigned)));
    ctx->allocs.push_back({ctx->d_status, sizeof(unsigned)});
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned), ctx->stream));
    DA(ctx->d_state, 1);
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
    GUARD_END
}

static int upload_jacobian(tbs_ctx *ctx, const double *jacD, const double *O1, const double *O2,
                           const double *rhs, cudaMemcpyKind kind) {
    if (!ctx->have_mesh) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_set_mesh must come first");
    if (!jacD || (ctx->nintface > 0 && (!O1 || !O2)) || !rhs)
        return ctx_fail(ctx, TBS_ERR_ARG, "null Jacobian array");
    const size_t nb = (size_t)ctx->nvar * ctx->nvar;
    DA(ctx->d_jacD, nb * ctx->nelem);
    DA(ctx->d_O1, nb * ctx->nintface);
    DA(ctx->d_O2, nb * ctx->nintface);
    DA(ctx->d_rhs, (size_t)nvec(ctx));
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->d_jacD, jacD, nb * ctx->nelem * sizeof(double), kind, s));
    if (ctx->nintface) {
        CK(cudaMemcpyAsync(ctx->d_O1, O1, nb * ctx->nintface * sizeof(double), kind, s));
        CK(cudaMemcpyAsync(ctx->d_O2, O2, nb * ctx->nintface * sizeof(double), kind, s));
    }
    CK(cudaMemcpyAsync(ctx->d_rhs, rhs, (size_t)nvec(ctx) * sizeof(double), kind, s));
    /* same mesh -> same allocations, so an instantiated solve graph stays valid */
    ctx->have_jac = true;
    ctx->factored = false;
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

int tbs_factor(tbs_ctx *ctx, int algo) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->have_jac) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_set_jacobian must come first");
    if (algo != TBS_ALGO_REFERENCE && algo != TBS_ALGO_FP64 && algo != TBS_ALGO_MIXED)
        return ctx_fail(ctx, TBS_ERR_ARG, "unknown algorithm " + std::to_string(algo));
    if (algo != TBS_ALGO_REFERENCE && !ctx->layout_ok)
        return ctx_fail(ctx, TBS_ERR_UNSUPPORTED,
                        "TBS_ALGO_FP64 / TBS_ALGO_MIXED need nvar == 9 and at most 4 cross-line "
                        "faces per cell; use TBS_ALGO_REFERENCE");
    int rc = alloc_algo(ctx, algo);
    if (rc) return rc;
    if (ctx->algo != algo) drop_graph(ctx);
    ctx->algo = algo;
    ctx->factored = false;
    rc = run_factor(ctx, algo);
    if (rc) return rc;
    rc = prime(ctx, CondCtl{0, 0});
    if (rc) return rc;
    rc = status_check(ctx);
    if (rc) return rc;
    ctx->factored = true;
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
        RUN("permute", launch_permute_to_pos(ctx->stream, 9, ctx->nelem, ctx->L.pos_of_elem, ctx->d_rhs,
                                             ctx->d_rhsp));
    }
    return prime(ctx, CondCtl{0, 0});
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
    return prime(ctx, CondCtl{0, 0});
    GUARD_END
}

int tbs_sweep(tbs_ctx *ctx, int n, double *rnorm_out) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->factored) return ctx_fail(ctx, TBS_ERR_STATE, "tbs_factor must come first");
    if (n < 0) return ctx_fail(ctx, TBS_ERR_ARG, "negative sweep count");
    int rc = ensure_hist(ctx, n + 1);
    if (rc) return rc;
    rc = set_state(ctx, 0.0, n);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    /* the current residual norm (recorded by the last sequence) opens the history */
    rc = reduce(ctx, 0, 1, CondCtl{0, 0});
    if (rc) return rc;
    for (int s = 0; s < n; ++s) {
        rc = body(ctx, CondCtl{0, 0});
        if (rc) return rc;
    }
    if (rnorm_out)
        CK(cudaMemcpyAsync(rnorm_out, ctx->d_hist, (n + 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
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
    int rc = ensure_hist(ctx, max_sweeps + 1);
    if (rc) return rc;
    rc = set_state(ctx, rel_tol, max_sweeps);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    if (ctx->prof) {
        /* eager form with a host-side test, so that every kernel is timed */
        rc = prime(ctx, CondCtl{0, 0});
        if (rc) return rc;
        for (;;) {
            rc = read_state(ctx);
            if (rc) return rc;
            const SolveState &S = *ctx->h_state;
            const bool go = std::isfinite(S.last) && S.last > S.tol * S.norm0 && S.sweep < S.max_sweeps;
            if (!go) break;
            rc = body(ctx, CondCtl{0, 0});
            if (rc) return rc;
        }
        prof_resolve(ctx);
    } else {
        if (!ctx->gexec || ctx->graph_algo != ctx->algo) {
            rc = build_graph(ctx);
            if (rc) return rc;
        }
        CK(cudaGraphLaunch(ctx->gexec, st));
        rc = read_state(ctx);
        if (rc) return rc;
    }
    const int sw = ctx->h_state->sweep;
    if (sweeps_out) *sweeps_out = sw;
    if (hist_out)
        CK(cudaMemcpyAsync(hist_out, ctx->d_hist, (size_t)(std::min(sw, max_sweeps) + 1) * sizeof(double),
                           cudaMemcpyDeviceToHost, st));
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
        if (which == 0) {
            RUN("permute", launch_permute_to_elem(st, 9, ctx->nelem, L.pos_of_elem, ctx->d_Up, ctx->d_scratch));
        } else if (which == 1) {
            RUN("full_resid", launch_full_resid<double>(st, ctx->nelem, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
                                                        L.pos_of_elem, ctx->d_jacD, ctx->d_O1, ctx->d_O2,
                                                        ctx->d_rhs, ctx->d_Up, ctx->d_Rp, ctx->d_partials2));
            RUN("permute", launch_permute_to_elem(st, 9, ctx->nelem, L.pos_of_elem, ctx->d_Rp, ctx->d_scratch));
        } else if (ctx->algo == TBS_ALGO_FP64) {
            RUN("permute", launch_permute_to_elem(st, 9, ctx->nelem, L.pos_of_elem, ctx->d_dUp, ctx->d_scratch));
        } else {
            RUN("permute", launch_permute_f32_to_elem(st, 9, ctx->nelem, L.pos_of_elem, ctx->d_c32, ctx->d_scratch));
            /* the outer correction is c + d (see body()); add d */
            RUN("permute", launch_permute_f32_to_elem(st, 9, ctx->nelem, L.pos_of_elem, ctx->d_d32, ctx->d_R));
            RUN("axpy", launch_axpy_f64(st, ctx->d_R, ctx->d_scratch, (long long)nvec(ctx)));
        }
        src = ctx->d_scratch;
    }
    CK(cudaMemcpyAsync(out, src, vb, cudaMemcpyDeviceToHost, st));
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
        for (double v : R) s += v * v;
        *out = std::sqrt(s);
        return TBS_OK;
    }
    cudaStream_t st = ctx->stream;
    const int nb = full_resid_blocks(ctx->nelem);
    const bool ref = ctx->algo == TBS_ALGO_REFERENCE;
    RUN("full_resid", launch_full_resid<double>(st, ctx->nelem, ctx->d_epoint, ctx->d_ef, ctx->d_fc,
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

int tbs_memory_allocated(const tbs_ctx *ctx, size_t *bytes) {
    if (!ctx || !bytes) return ctx_fail(nullptr, TBS_ERR_ARG, "null argument");
    *bytes = ctx->bytes;
    return TBS_OK;
}

int tbs_set_inner_sweeps(tbs_ctx *ctx, int m) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    if (m < 1 || m > 64) return ctx_fail(ctx, TBS_ERR_ARG, "inner sweeps must be in 1..64");
    if (m != ctx->inner_sweeps) drop_graph(ctx);
    ctx->inner_sweeps = m;
    return TBS_OK;
}

int tbs_tune_inner(tbs_ctx *ctx, double rel_tol, int max_sweeps, int *best_m, double *best_ms) {
    if (!ctx) return ctx_fail(nullptr, TBS_ERR_ARG, "null context");
    GUARD_BEGIN
    CK(cudaSetDevice(ctx->device));
    if (!ctx->factored || ctx->algo != TBS_ALGO_MIXED)
        return ctx_fail(ctx, TBS_ERR_STATE, "tbs_tune_inner needs a TBS_ALGO_MIXED factorization");
    const int cand[] = {2, 3, 4, 5, 6, 8, 10};
    const bool prof = ctx->prof;
    ctx->prof = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int best = -1;
    double best_t = 0.0;
    int rc = TBS_OK;
    for (int m : cand) {
        if (rc) break;
        rc = tbs_set_inner_sweeps(ctx, m);
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
        if (rc) break;
        const SolveState &S = *ctx->h_state;
        const bool conv = std::isfinite(S.last) && S.last <= S.tol * S.norm0;
        if (conv && (best < 0 || t < best_t)) {
            best = m;
            best_t = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->prof = prof;
    if (rc) return rc;
    if (best < 0) return ctx_fail(ctx, TBS_ERR_NUMERIC, "no inner sweep count reached the tolerance");
    rc = tbs_set_inner_sweeps(ctx, best);
    if (rc) return rc;
    if (best_m) *best_m = best;
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
    if (k == "fast_resid") /* Dinv, X blocks, xnbr, neighbour dU, b out, own dU + U in/out */
        b = N * (blk + vec + 3 * vec) + X * (blk + 4.0 + vec);
    else if (k == "fast_resid_rhs") /* Dinv, R in, b out */
        b = N * (blk + 2 * vec);
    else if (k == "fast_resid32_rhs")
        b = N * (blk + 2 * vec) / 2;
    else if (k == "fast_resid32") /* DX blocks, xnbr, neighbour d, b out, own d + c in/out */
        b = N * (4 * vec) / 2 + X * (blk / 2 + 4.0 + vec / 2);
    else if (k == "fast_thomas") /* G, b | Gam, dU out (y stays on chip when the line fits) */
        b = N * (2 * blk + 2 * vec);
    else if (k == "fast_thomas32")
        b = N * (2 * blk + 2 * vec) / 2;
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
    else if (k == "fast_factor") /* D, A, C in; Dinv, G, Gam out */
        b = N * blk + 2 * (N - ctx->nline) * blk + 3 * N * blk;
    if (b < 0) return ctx_fail(ctx, TBS_ERR_ARG, "unknown kernel name " + k);
    *bytes = b;
    return TBS_OK;
}

}  // extern "C"

/* ================================================================ batches
 * Many independent systems (contexts factored with the same algorithm on
 * one GPU) solved together.  Every launch covers the work units of all
 * systems still above their tolerance: one persistent Thomas launch over
 * their lines from a device work queue, one residual launch over their
 * tiles, one launch for the per-system norms.  The per-unit arithmetic and
 * the order of every norm sum are those of the single-system sequences
 * (prime / body above), so each system's iterates are bit-identical to a
 * tbs_solve of its context alone. */

struct tbs_batch {
    int device = 0;
    cudaStream_t own = nullptr;    /* created with the batch */
    cudaStream_t stream = nullptr; /* where the launches go: own or the caller's */
    std::string err;
    std::vector<tbs_ctx *> sys;
    int algo = -1;
    int inner = 4;
    BatchSched sched{8, 2};
    int order = 0; /* 0: longest lines first, 1: mesh order */
    int max_nx = 0;
    /* device: descriptors and work lists (one allocation each) */
    std::vector<void *> allocs;
    ThomasSys<double> *d_th64 = nullptr;
    ThomasSys<float> *d_th32 = nullptr;
    ResidSys<double> *d_rs_prime = nullptr, *d_rs_body = nullptr;
    ResidSys<float> *d_rs32_rhs = nullptr, *d_rs32_dx = nullptr;
    FullResSys *d_fr = nullptr;
    VecSys *d_vec = nullptr;
    ReduceSys *d_red_prime = nullptr, *d_red_body = nullptr;
    WorkItem *d_lines_lpt = nullptr, *d_lines_mesh = nullptr, *d_tiles = nullptr,
             *d_prime_tiles = nullptr, *d_blocks = nullptr;
    int nlines = 0, ntiles = 0, nprime_tiles = 0, nblocks = 0;
    int *d_active = nullptr;
    unsigned *d_queue = nullptr, *d_counter = nullptr, *d_status = nullptr;
    unsigned *h_status = nullptr; /* pinned */
    /* what the descriptors and the graph were built from */
    std::vector<const void *> fingerprint;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool graph_ok = false;
    /* profiling (eager launches bracketed by events) */
    bool prof = false;
    std::vector<ProfSlot> slots;
    std::vector<PendingEvent> pending;
    std::vector<cudaEvent_t> pool;
};

static int bfail(tbs_batch *b, int code, const std::string &msg) {
    if (b) b->err = msg;
    set_thread_error(msg);
    return code;
}

#define BCK(call)                                                                         \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return bfail(b, TBS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define BCKL(call)                                                                        \
    do {                                                                                  \
        int e_ = (call);                                                                  \
        if (e_ != 0)                                                                      \
            return bfail(b, TBS_ERR_CUDA,                                                 \
                         std::string(#call) + ": " + cudaGetErrorString((cudaError_t)e_)); \
    } while (0)

template <typename T>
static int balloc(tbs_batch *b, T **p, size_t count) {
    void *q = nullptr;
    const size_t nbytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&q, nbytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, TBS_ERR_NOMEM, "cudaMalloc of " + std::to_string(nbytes) + " bytes failed");
    }
    b->allocs.push_back(q);
    *p = static_cast<T *>(q);
    return TBS_OK;
}

template <typename T>
static int bupload(tbs_batch *b, T **p, const std::vector<T> &h) {
    if (!*p) {
        int rc = balloc(b, p, h.size());
        if (rc) return rc;
    }
    if (!h.empty())
        BCK(cudaMemcpyAsync(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, b->stream));
    return TBS_OK;
}

static void bdrop_graph(tbs_batch *b) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
    b->graph_ok = false;
}

/* every device pointer and setting the descriptors and graph depend on */
static std::vector<const void *> batch_fingerprint(tbs_batch *b) {
    std::vector<const void *> f;
    for (tbs_ctx *c : b->sys) {
        const void *p[] = {c->d_G, c->d_Gam, c->d_Dinv, c->d_X, c->d_b, c->d_y, c->d_dUp, c->d_Up,
                           c->d_rhsp, c->d_Rp, c->d_partials, c->d_state, c->d_hist, c->d_Uinit,
                           c->d_G32, c->d_Gam32, c->d_Dinv32, c->d_X32, c->d_b32, c->d_y32,
                           c->d_d32, c->d_c32, c->d_R32, c->L.line_start, c->L.xnbr, c->d_jacD,
                           c->d_O1, c->d_O2, c->d_rhs, c->d_epoint};
        f.insert(f.end(), std::begin(p), std::end(p));
        f.push_back(reinterpret_cast<const void *>((uintptr_t)c->algo));
    }
    f.push_back(reinterpret_cast<const void *>((uintptr_t)b->inner));
    return f;
}

static int batch_check_members(tbs_batch *b) {
    for (size_t s = 0; s < b->sys.size(); ++s) {
        tbs_ctx *c = b->sys[s];
        if (!c->factored || !c->layout_ok)
            return bfail(b, TBS_ERR_STATE, "batch member " + std::to_string(s) + " is not factored");
        if (c->algo != b->algo)
            return bfail(b, TBS_ERR_STATE,
                         "batch member " + std::to_string(s) + " was re-factored with another algorithm");
    }
    return TBS_OK;
}

/* descriptors of every launch, from the members' current arrays */
static int batch_descriptors(tbs_batch *b) {
    const int n = (int)b->sys.size();
    std::vector<ThomasSys<double>> th64;
    std::vector<ThomasSys<float>> th32;
    std::vector<ResidSys<double>> rsp, rsb;
    std::vector<ResidSys<float>> rs32r, rs32d;
    std::vector<FullResSys> fr;
    std::vector<VecSys> vec;
    std::vector<ReduceSys> redp, redb;
    std::vector<WorkItem> prime_tiles;
    const bool mixed = b->algo == TBS_ALGO_MIXED;
    for (int s = 0; s < n; ++s) {
        tbs_ctx *c = b->sys[s];
        const FastLayout &L = c->L;
        const int nt = fast_resid_grid(L.np16);
        if (!mixed) {
            th64.push_back({L.line_start, L.line_len, L.line_twist, c->d_G, c->d_Gam, c->d_b, c->d_y,
                            c->d_dUp});
            /* prime: R = rhs (U = 0, cleared here) or the residual of U_init */
            rsp.push_back({L.np16, L.nx, L.xnbr, c->d_Dinv, c->d_X, c->d_dUp,
                           c->d_Uinit ? c->d_Rp : c->d_rhsp, c->d_b, c->d_Uinit ? nullptr : c->d_Up,
                           c->d_partials});
            rsb.push_back({L.np16, L.nx, L.xnbr, c->d_Dinv, c->d_X, c->d_dUp, nullptr, c->d_b,
                           c->d_Up, c->d_partials});
            redp.push_back({c->d_partials, nt, 0, c->d_state, c->d_hist});
            redb.push_back({c->d_partials, nt, 0, c->d_state, c->d_hist});
        } else {
            th32.push_back({L.line_start, L.line_len, L.line_twist, c->d_G32, c->d_Gam32, c->d_b32,
                            c->d_y32, c->d_d32});
            rs32r.push_back({L.np16, L.nx, L.xnbr, c->d_Dinv32, c->d_X32, c->d_d32, c->d_R32,
                             c->d_b32, c->d_c32, nullptr});
            rs32d.push_back({L.np16, L.nx, L.xnbr, nullptr, c->d_X32, c->d_d32, nullptr, c->d_b32,
                             c->d_c32, nullptr});
            fr.push_back({c->nelem, 0, c->d_epoint, c->d_ef, c->d_fc, L.pos_of_elem, c->d_jacD,
                          c->d_O1, c->d_O2, c->d_rhs, c->d_Up, c->d_R32, c->d_partials});
            vec.push_back({c->d_rhsp, c->d_R32, c->d_c32, c->d_d32, c->d_Up, c->d_partials});
            redp.push_back({c->d_partials, c->d_Uinit ? full_resid_blocks(c->nelem) : nt, 0,
                            c->d_state, c->d_hist});
            redb.push_back({c->d_partials, full_resid_blocks(c->nelem), 0, c->d_state, c->d_hist});
            if (!c->d_Uinit)
                for (int t = 0; t < nt; ++t) prime_tiles.push_back({s, t});
        }
    }
    int rc = TBS_OK;
    if (!mixed) {
        if (!rc) rc = bupload(b, &b->d_th64, th64);
        if (!rc) rc = bupload(b, &b->d_rs_prime, rsp);
        if (!rc) rc = bupload(b, &b->d_rs_body, rsb);
    } else {
        if (!rc) rc = bupload(b, &b->d_th32, th32);
        if (!rc) rc = bupload(b, &b->d_rs32_rhs, rs32r);
        if (!rc) rc = bupload(b, &b->d_rs32_dx, rs32d);
        if (!rc) rc = bupload(b, &b->d_fr, fr);
        if (!rc) rc = bupload(b, &b->d_vec, vec);
        /* the prime tile list depends on which members start from U_init */
        if (!rc && b->d_prime_tiles && (int)prime_tiles.size() > b->nprime_tiles) {
            cudaFree(b->d_prime_tiles);
            b->allocs.erase(std::find(b->allocs.begin(), b->allocs.end(), (void *)b->d_prime_tiles));
            b->d_prime_tiles = nullptr;
        }
        if (!rc) rc = bupload(b, &b->d_prime_tiles, prime_tiles);
        b->nprime_tiles = (int)prime_tiles.size();
    }
    if (!rc) rc = bupload(b, &b->d_red_prime, redp);
    if (!rc) rc = bupload(b, &b->d_red_body, redb);
    if (!rc) BCK(cudaStreamSynchronize(b->stream));
    return rc;
}

static cudaEvent_t bprof_event(tbs_batch *b) {
    if (!b->pool.empty()) {
        cudaEvent_t e = b->pool.back();
        b->pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

static void bprof_resolve(tbs_batch *b) {
    if (b->pending.empty()) return;
    cudaStreamSynchronize(b->stream);
    for (auto &p : b->pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess && p.slot >= 0) {
            b->slots[p.slot].ms += ms;
            b->slots[p.slot].launches += 1;
        }
        b->pool.push_back(p.a);
        b->pool.push_back(p.b);
    }
    b->pending.clear();
}

template <typename F>
static int btimed(tbs_batch *b, const char *name, F &&launch) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(b->stream, &cs);
    if (!b->prof || cs != cudaStreamCaptureStatusNone) return launch();
    int slot = -1;
    for (size_t i = 0; i < b->slots.size(); ++i)
        if (std::strcmp(b->slots[i].name, name) == 0) slot = (int)i;
    if (slot < 0 && b->slots.size() < TBS_PROFILE_MAX) {
        b->slots.push_back({name, 0, 0.0});
        slot = (int)b->slots.size() - 1;
    }
    if (b->pending.size() > 4000) bprof_resolve(b);
    PendingEvent pe{slot, bprof_event(b), bprof_event(b)};
    cudaEventRecord(pe.a, b->stream);
    int rc = launch();
    cudaEventRecord(pe.b, b->stream);
    b->pending.push_back(pe);
    return rc;
}

#define BRUN(name, call) BCKL(btimed(b, name, [&]() { return (int)(call); }))

static const WorkItem *batch_lines(tbs_batch *b) {
    return b->order == 0 ? b->d_lines_lpt : b->d_lines_mesh;
}

/* start of a batched solve: every member's residual of U_init (or rhs),
 * its norm recorded as ||R_0|| and its active flag */
static int batch_prime(tbs_batch *b, CondCtl cc) {
    cudaStream_t st = b->stream;
    const int n = (int)b->sys.size();
    for (tbs_ctx *c : b->sys) {
        if (!c->d_Uinit) continue;
        const FastLayout &L = c->L;
        BRUN("permute", launch_permute_to_pos(st, 9, c->nelem, L.pos_of_elem, c->d_Uinit, c->d_Up));
        if (b->algo == TBS_ALGO_FP64)
            BRUN("full_resid", launch_full_resid<double>(st, c->nelem, c->d_epoint, c->d_ef, c->d_fc,
                                                         L.pos_of_elem, c->d_jacD, c->d_O1, c->d_O2,
                                                         c->d_rhs, c->d_Up, c->d_Rp, c->d_partials2));
        else
            BRUN("full_resid", launch_full_resid<float>(st, c->nelem, c->d_epoint, c->d_ef, c->d_fc,
                                                        L.pos_of_elem, c->d_jacD, c->d_O1, c->d_O2,
                                                        c->d_rhs, c->d_Up, c->d_R32, c->d_partials));
    }
    if (b->algo == TBS_ALGO_FP64) {
        BRUN("fast_resid_rhs", launch_resid_batch<double>(st, 0, b->max_nx, b->d_rs_prime, b->d_tiles,
                                                          b->ntiles, nullptr, b->d_status));
        BRUN("reduce_norm", launch_reduce_batch(st, 160, b->d_red_prime, n, 1, b->d_active,
                                                b->d_counter, cc.handle, cc.use_cond));
    } else {
        BRUN("mixed_prime", launch_mixed_prime_batch(st, b->d_vec, b->d_prime_tiles, b->nprime_tiles));
        BRUN("reduce_norm", launch_reduce_batch(st, 256, b->d_red_prime, n, 1, b->d_active,
                                                b->d_counter, cc.handle, cc.use_cond));
    }
    return TBS_OK;
}

/* one sweep of every active member */
static int batch_body(tbs_batch *b, CondCtl cc) {
    cudaStream_t st = b->stream;
    const int n = (int)b->sys.size();
    if (b->algo == TBS_ALGO_FP64) {
        BRUN("fast_thomas", launch_thomas_batch<double>(st, b->sched, b->d_th64, batch_lines(b),
                                                        b->nlines, b->d_active, b->d_queue,
                                                        b->d_status));
        BRUN("fast_resid", launch_resid_batch<double>(st, 1, b->max_nx, b->d_rs_body, b->d_tiles,
                                                      b->ntiles, b->d_active, b->d_status));
        BRUN("reduce_norm", launch_reduce_batch(st, 160, b->d_red_body, n, 0, b->d_active,
                                                b->d_counter, cc.handle, cc.use_cond));
        return TBS_OK;
    }
    BRUN("fast_resid32_rhs", launch_resid_batch<float>(st, 0, b->max_nx, b->d_rs32_rhs, b->d_tiles,
                                                       b->ntiles, b->d_active, b->d_status));
    for (int m = 0; m < b->inner; ++m) {
        BRUN("fast_thomas32", launch_thomas_batch<float>(st, b->sched, b->d_th32, batch_lines(b),
                                                         b->nlines, b->d_active, b->d_queue,
                                                         b->d_status));
        if (m + 1 < b->inner)
            BRUN("fast_resid32", launch_resid_batch<float>(st, 3, b->max_nx, b->d_rs32_dx, b->d_tiles,
                                                           b->ntiles, b->d_active, b->d_status));
    }
    BRUN("axpy", launch_axpy2_batch(st, b->d_vec, b->d_tiles, b->ntiles, b->d_active));
    BRUN("full_resid", launch_full_resid_batch(st, b->d_fr, b->d_blocks, b->nblocks, b->d_active));
    BRUN("reduce_norm", launch_reduce_batch(st, 256, b->d_red_body, n, 0, b->d_active, b->d_counter,
                                            cc.handle, cc.use_cond));
    return TBS_OK;
}

static int batch_build_graph(tbs_batch *b) {
    bdrop_graph(b);
    cudaStream_t st = b->stream;
    cudaGraph_t g = nullptr;
    BCK(cudaGraphCreate(&g, 0));
    b->graph = g;
    cudaGraphConditionalHandle h;
    BCK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    const CondCtl cc{(unsigned long long)h, 1};
    BCK(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int rc = batch_prime(b, cc);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    if (rc == TBS_OK) {
        cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &ndeps);
        if (e != cudaSuccess) rc = bfail(b, TBS_ERR_CUDA, std::string("capture info: ") + cudaGetErrorString(e));
    }
    cudaGraphNode_t cnode = nullptr;
    cudaGraph_t bodyg = nullptr;
    if (rc == TBS_OK) {
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaError_t e = cudaGraphAddNode(&cnode, g, deps, ndeps, &cp);
        if (e != cudaSuccess) rc = bfail(b, TBS_ERR_CUDA, std::string("conditional node: ") + cudaGetErrorString(e));
        else bodyg = cp.conditional.phGraph_out[0];
    }
    if (rc == TBS_OK) {
        cudaError_t e = cudaStreamUpdateCaptureDependencies(st, &cnode, 1, cudaStreamSetCaptureDependencies);
        if (e != cudaSuccess) rc = bfail(b, TBS_ERR_CUDA, std::string("capture deps: ") + cudaGetErrorString(e));
    }
    cudaGraph_t outg = nullptr;
    cudaError_t ee = cudaStreamEndCapture(st, &outg);
    if (rc == TBS_OK && ee != cudaSuccess) rc = bfail(b, TBS_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ee));
    if (rc != TBS_OK) {
        bdrop_graph(b);
        return rc;
    }
    BCK(cudaStreamBeginCaptureToGraph(st, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    rc = batch_body(b, cc);
    ee = cudaStreamEndCapture(st, &outg);
    if (rc == TBS_OK && ee != cudaSuccess) rc = bfail(b, TBS_ERR_CUDA, std::string("end body capture: ") + cudaGetErrorString(ee));
    if (rc != TBS_OK) {
        bdrop_graph(b);
        return rc;
    }
    cudaError_t ie = cudaGraphInstantiate(&b->gexec, g, 0);
    if (ie != cudaSuccess) {
        bdrop_graph(b);
        return bfail(b, TBS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    }
    b->graph_ok = true;
    return TBS_OK;
}

static int batch_status(tbs_batch *b) {
    BCK(cudaMemcpyAsync(b->h_status, b->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    const unsigned s = *b->h_status;
    if (s) {
        BCK(cudaMemsetAsync(b->d_status, 0, sizeof(unsigned), b->stream));
        BCK(cudaMemsetAsync(b->d_queue, 0, 2 * sizeof(unsigned), b->stream));
        BCK(cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned), b->stream));
        BCK(cudaStreamSynchronize(b->stream));
        if (s & ST_TIMEOUT) return bfail(b, TBS_ERR_CUDA, "a device-side wait ran out of its time budget");
        return bfail(b, TBS_ERR_CUDA, "device status " + std::to_string(s));
    }
    return TBS_OK;
}

/* members' device state (tolerance, sweep limit, history capacity) and
 * the descriptors / graph, refreshed when a member's arrays changed */
static int batch_ready(tbs_batch *b, double tol, int max_sweeps) {
    int rc = batch_check_members(b);
    if (rc) return rc;
    for (tbs_ctx *c : b->sys) {
        BCK(cudaStreamSynchronize(c->stream));
        rc = ensure_hist(c, max_sweeps + 1);
        if (!rc) rc = set_state(c, tol, max_sweeps);
        if (rc) return bfail(b, rc, "batch member: " + c->err);
        BCK(cudaStreamSynchronize(c->stream));
    }
    std::vector<const void *> fp = batch_fingerprint(b);
    if (fp != b->fingerprint) {
        bdrop_graph(b);
        rc = batch_descriptors(b);
        if (rc) return rc;
        b->fingerprint = fp;
    }
    return TBS_OK;
}

static int batch_destroy_all(tbs_batch *b) {
    if (!b) return TBS_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    bprof_resolve(b);
    bdrop_graph(b);
    for (void *p : b->allocs) cudaFree(p);
    for (cudaEvent_t e : b->pool) cudaEventDestroy(e);
    if (b->h_status) cudaFreeHost(b->h_status);
    if (b->own) cudaStreamDestroy(b->own);
    delete b;
    return TBS_OK;
}

extern "C" {

const char *tbs_batch_last_error(const tbs_batch *b) {
    if (!b) return thread_error();
    return b->err.c_str();
}

int tbs_batch_create(tbs_ctx *const *systems, int nsys, tbs_batch **out) {
    tbs_batch *b = nullptr;
    if (!out || !systems || nsys < 1) return bfail(nullptr, TBS_ERR_ARG, "tbs_batch_create: bad arguments");
    *out = nullptr;
    try {
        b = new tbs_batch();
    } catch (...) {
        return bfail(nullptr, TBS_ERR_NOMEM, "host allocation failed");
    }
    auto fail = [&](int rc) {
        std::string msg = b->err;
        batch_destroy_all(b);
        set_thread_error(msg);
        return rc;
    };
    try {
        for (int s = 0; s < nsys; ++s) {
            tbs_ctx *c = systems[s];
            if (!c) return fail(bfail(b, TBS_ERR_ARG, "null system " + std::to_string(s)));
            for (int t = 0; t < s; ++t)
                if (systems[t] == c)
                    return fail(bfail(b, TBS_ERR_ARG, "system " + std::to_string(s) + " appears twice"));
            if (!c->factored)
                return fail(bfail(b, TBS_ERR_STATE, "system " + std::to_string(s) + " is not factored"));
            if (c->algo != TBS_ALGO_FP64 && c->algo != TBS_ALGO_MIXED)
                return fail(bfail(b, TBS_ERR_UNSUPPORTED,
                                  "batches take TBS_ALGO_FP64 or TBS_ALGO_MIXED systems"));
            if (s > 0 && (c->algo != systems[0]->algo || c->device != systems[0]->device))
                return fail(bfail(b, TBS_ERR_ARG,
                                  "all systems of a batch need the same algorithm and GPU"));
            b->sys.push_back(c);
        }
        b->algo = systems[0]->algo;
        b->device = systems[0]->device;
        b->inner = systems[0]->inner_sweeps;
        if (cudaSetDevice(b->device) != cudaSuccess)
            return fail(bfail(b, TBS_ERR_CUDA, "cudaSetDevice failed"));
        if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess)
            return fail(bfail(b, TBS_ERR_CUDA, "cudaStreamCreate failed"));
        b->stream = b->own;
        if (cudaMallocHost(&b->h_status, sizeof(unsigned)) != cudaSuccess)
            return fail(bfail(b, TBS_ERR_NOMEM, "pinned allocation failed"));
        /* work lists */
        std::vector<WorkItem> lines, tiles, blocks;
        std::vector<int> len;
        for (int s = 0; s < nsys; ++s) {
            tbs_ctx *c = b->sys[s];
            b->max_nx = std::max(b->max_nx, c->L.nx);
            for (int l = 0; l < c->nline; ++l) {
                lines.push_back({s, l});
                len.push_back(c->h_linesize[l]);
            }
            for (int t = 0; t < fast_resid_grid(c->L.np16); ++t) tiles.push_back({s, t});
            for (int k = 0; k < full_resid_blocks(c->nelem); ++k) blocks.push_back({s, k});
        }
        std::vector<int> idx(lines.size());
        for (size_t k = 0; k < idx.size(); ++k) idx[k] = (int)k;
        std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return len[x] > len[y]; });
        std::vector<WorkItem> lpt(lines.size());
        for (size_t k = 0; k < idx.size(); ++k) lpt[k] = lines[idx[k]];
        b->nlines = (int)lines.size();
        b->ntiles = (int)tiles.size();
        b->nblocks = (int)blocks.size();
        int rc = bupload(b, &b->d_lines_lpt, lpt);
        if (!rc) rc = bupload(b, &b->d_lines_mesh, lines);
        if (!rc) rc = bupload(b, &b->d_tiles, tiles);
        if (!rc && b->algo == TBS_ALGO_MIXED) rc = bupload(b, &b->d_blocks, blocks);
        if (!rc) rc = balloc(b, &b->d_active, (size_t)nsys);
        if (!rc) rc = balloc(b, &b->d_queue, 2);
        if (!rc) rc = balloc(b, &b->d_counter, 1);
        if (!rc) rc = balloc(b, &b->d_status, 1);
        if (rc) return fail(rc);
        if (cudaMemsetAsync(b->d_active, 0, nsys * sizeof(int), b->stream) != cudaSuccess ||
            cudaMemsetAsync(b->d_queue, 0, 2 * sizeof(unsigned), b->stream) != cudaSuccess ||
            cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned), b->stream) != cudaSuccess ||
            cudaMemsetAsync(b->d_status, 0, sizeof(unsigned), b->stream) != cudaSuccess)
            return fail(bfail(b, TBS_ERR_CUDA, "cudaMemsetAsync failed"));
        if (batch_prepare(b->max_nx)) return fail(bfail(b, TBS_ERR_CUDA, "shared-memory opt-in failed"));
        /* default schedule: 2 stages, as many CTAs per SM as fit, at most 8 */
        const int fit = b->algo == TBS_ALGO_FP64 ? thomas_batch_fit<double>(2) : thomas_batch_fit<float>(2);
        if (fit < 1) return fail(bfail(b, TBS_ERR_CUDA, "the batched Thomas kernel does not fit on an SM"));
        b->sched = BatchSched{std::min(fit, 8), 2};
        if (cudaStreamSynchronize(b->stream) != cudaSuccess)
            return fail(bfail(b, TBS_ERR_CUDA, "cudaStreamSynchronize failed"));
    } catch (...) {
        return fail(bfail(b, TBS_ERR_NOMEM, "host allocation failed"));
    }
    *out = b;
    return TBS_OK;
}

int tbs_batch_destroy(tbs_batch *b) { return batch_destroy_all(b); }

int tbs_batch_set_stream(tbs_batch *b, void *cuda_stream) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    cudaStream_t ns = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : b->own;
    if (ns != b->stream) {
        cudaStreamSynchronize(b->stream);
        bdrop_graph(b);
        b->stream = ns;
    }
    return TBS_OK;
}

int tbs_batch_size(const tbs_batch *b, int *nsys) {
    if (!b || !nsys) return bfail(nullptr, TBS_ERR_ARG, "null argument");
    *nsys = (int)b->sys.size();
    return TBS_OK;
}

int tbs_batch_set_inner_sweeps(tbs_batch *b, int m) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (m < 1 || m > 64) return bfail(b, TBS_ERR_ARG, "inner sweeps must be in 1..64");
    if (m != b->inner) bdrop_graph(b);
    b->inner = m;
    b->fingerprint.clear();
    return TBS_OK;
}

int tbs_batch_set_schedule(tbs_batch *b, int ctas_per_sm, int stages, int order) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (stages < 2 || stages > 8 || ctas_per_sm < 1 || (order != 0 && order != 1))
        return bfail(b, TBS_ERR_ARG, "bad schedule");
    try {
        BCK(cudaSetDevice(b->device));
        const int fit = b->algo == TBS_ALGO_FP64 ? thomas_batch_fit<double>(stages)
                                                 : thomas_batch_fit<float>(stages);
        if (ctas_per_sm > fit)
            return bfail(b, TBS_ERR_ARG, "schedule does not fit: at most " + std::to_string(fit) +
                                             " CTAs per SM with " + std::to_string(stages) + " stages");
        b->sched = BatchSched{ctas_per_sm, stages};
        b->order = order;
        bdrop_graph(b);
    } catch (...) {
        return bfail(b, TBS_ERR_STATE, "internal error");
    }
    return TBS_OK;
}

int tbs_batch_get_schedule(const tbs_batch *b, int *ctas_per_sm, int *stages, int *order) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (ctas_per_sm) *ctas_per_sm = b->sched.ctas_per_sm;
    if (stages) *stages = b->sched.stages;
    if (order) *order = b->order;
    return TBS_OK;
}

int tbs_batch_solve(tbs_batch *b, double rel_tol, int max_sweeps, int *sweeps_out,
                    double *hist_out) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (max_sweeps < 0 || !(rel_tol >= 0.0)) return bfail(b, TBS_ERR_ARG, "bad tolerance or sweep limit");
    try {
        BCK(cudaSetDevice(b->device));
        int rc = batch_ready(b, rel_tol, max_sweeps);
        if (rc) return rc;
        cudaStream_t st = b->stream;
        const int n = (int)b->sys.size();
        if (b->prof) {
            /* eager form with a host-side test, so that every kernel is timed */
            rc = batch_prime(b, CondCtl{0, 0});
            if (rc) return rc;
            std::vector<int> act(n);
            for (;;) {
                BCK(cudaMemcpyAsync(act.data(), b->d_active, n * sizeof(int), cudaMemcpyDeviceToHost, st));
                BCK(cudaStreamSynchronize(st));
                bool any = false;
                for (int v : act) any = any || v;
                if (!any) break;
                rc = batch_body(b, CondCtl{0, 0});
                if (rc) return rc;
            }
            bprof_resolve(b);
        } else {
            if (!b->graph_ok) {
                rc = batch_build_graph(b);
                if (rc) return rc;
            }
            BCK(cudaGraphLaunch(b->gexec, st));
        }
        rc = batch_status(b);
        if (rc) return rc;
        for (int s = 0; s < n; ++s) {
            tbs_ctx *c = b->sys[s];
            BCK(cudaMemcpyAsync(c->h_state, c->d_state, sizeof(SolveState), cudaMemcpyDeviceToHost, st));
        }
        BCK(cudaStreamSynchronize(st));
        for (int s = 0; s < n; ++s) {
            tbs_ctx *c = b->sys[s];
            const int sw = c->h_state->sweep;
            if (sweeps_out) sweeps_out[s] = sw;
            if (hist_out)
                BCK(cudaMemcpyAsync(hist_out + (size_t)s * (max_sweeps + 1), c->d_hist,
                                    (size_t)(std::min(sw, max_sweeps) + 1) * sizeof(double),
                                    cudaMemcpyDeviceToHost, st));
        }
        BCK(cudaStreamSynchronize(st));
    } catch (...) {
        return bfail(b, TBS_ERR_STATE, "internal error");
    }
    return TBS_OK;
}

int tbs_batch_tune(tbs_batch *b, int *ctas_per_sm, int *stages, int *order, double *best_ms) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    try {
        BCK(cudaSetDevice(b->device));
        int rc = batch_ready(b, 0.0, 1);
        if (rc) return rc;
        cudaStream_t st = b->stream;
        const int n = (int)b->sys.size();
        std::vector<int> ones(n, 1);
        BCK(cudaMemcpyAsync(b->d_active, ones.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
        cudaEvent_t e0, e1;
        BCK(cudaEventCreate(&e0));
        BCK(cudaEventCreate(&e1));
        const BatchSched keep = b->sched;
        const int keep_order = b->order;
        double best = 1e30;
        BatchSched best_s = keep;
        int best_o = keep_order;
        const int cand_ctas[] = {2, 3, 4, 6, 8, 12, 16};
        for (int ns = 2; ns <= 4 && !rc; ++ns) {
            const int fit = b->algo == TBS_ALGO_FP64 ? thomas_batch_fit<double>(ns)
                                                     : thomas_batch_fit<float>(ns);
            for (int cps : cand_ctas) {
                if (cps > fit || rc) continue;
                for (int o = 0; o < 2 && !rc; ++o) {
                    b->sched = BatchSched{cps, ns};
                    b->order = o;
                    auto launch = [&]() {
                        return b->algo == TBS_ALGO_FP64
                                   ? launch_thomas_batch<double>(st, b->sched, b->d_th64, batch_lines(b),
                                                                 b->nlines, b->d_active, b->d_queue,
                                                                 b->d_status)
                                   : launch_thomas_batch<float>(st, b->sched, b->d_th32, batch_lines(b),
                                                                b->nlines, b->d_active, b->d_queue,
                                                                b->d_status);
                    };
                    int e = launch();
                    const int reps = 3;
                    if (!e) cudaEventRecord(e0, st);
                    for (int r = 0; r < reps && !e; ++r) e = launch();
                    if (!e) cudaEventRecord(e1, st);
                    if (e) {
                        rc = bfail(b, TBS_ERR_CUDA, std::string("tuning launch: ") +
                                                        cudaGetErrorString((cudaError_t)e));
                        break;
                    }
                    cudaEventSynchronize(e1);
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    rc = batch_status(b);
                    if (rc) break;
                    if (ms / reps < best) {
                        best = ms / reps;
                        best_s = b->sched;
                        best_o = o;
                    }
                }
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        b->sched = rc ? keep : best_s;
        b->order = rc ? keep_order : best_o;
        bdrop_graph(b);
        if (rc) return rc;
        if (ctas_per_sm) *ctas_per_sm = best_s.ctas_per_sm;
        if (stages) *stages = best_s.stages;
        if (order) *order = best_o;
        if (best_ms) *best_ms = best;
    } catch (...) {
        return bfail(b, TBS_ERR_STATE, "internal error");
    }
    return TBS_OK;
}

int tbs_batch_profile_enable(tbs_batch *b, int on) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (!on) bprof_resolve(b);
    b->prof = on != 0;
    return TBS_OK;
}

int tbs_batch_profile_reset(tbs_batch *b) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    bprof_resolve(b);
    b->slots.clear();
    return TBS_OK;
}

int tbs_batch_profile_read(tbs_batch *b, int *n, const char **names, long long *launches,
                           double *ms) {
    if (!b || !n) return bfail(b, TBS_ERR_ARG, "null argument");
    bprof_resolve(b);
    const int cap = *n, cnt = (int)b->slots.size();
    for (int i = 0; i < cnt && i < cap; ++i) {
        if (names) names[i] = b->slots[i].name;
        if (launches) launches[i] = b->slots[i].launches;
        if (ms) ms[i] = b->slots[i].ms;
    }
    *n = cnt;
    return TBS_OK;
}

}  // extern "C"

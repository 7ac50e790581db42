/*
 * ctx.hxx -- the solver context (struct tbs_ctx) shared by the host
 * translation units: api.cu (single systems), batch.cu (batched launch
 * sequences over many systems) and server.cu (the request loop).
 * Not installed; the public surface is include/triblock.h.
 */
#ifndef TBS_CTX_HXX
#define TBS_CTX_HXX

#include "tbs_internal.hxx"

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

struct ProfSlot {
    const char *name;
    long long launches;
    double ms;
};

struct PendingEvent {
    int slot;
    cudaEvent_t a, b;
};

struct MultiBufs;  /* several right-hand sides (multi.cu) */
struct KrylovBufs; /* line-preconditioned GMRES (krylov.cu) */

struct tbs_ctx {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;

    /* ---- mesh ---- */
    bool have_mesh = false, have_jac = false, factored = false;
    int nvar = 0, nelem = 0, nintface = 0, eftot = 0, nline = 0, nlineelem = 0, max_line = 0;
    std::vector<int> h_epoint, h_ef, h_fc, h_linesize, h_linepoint, h_lines, h_lineface;
    /* line partition of a larger mesh: the last nhalo lines are copies of
     * lines another partition owns (swept, never counted in a norm); the
     * owned lines' cells are elements 0..nelem_own-1 */
    int nhalo = 0, nelem_own = 0;
    /* tbs_part_check left a true residual that the next tbs_part_solve_du
     * turns into its line solves' input (b = -Dinv R) */
    bool part_restart = false;
    std::vector<int> h_line_start; /* first position of every line */
    int *d_epoint = nullptr, *d_ef = nullptr, *d_fc = nullptr, *d_linesize = nullptr;
    int *d_linepoint = nullptr, *d_lines = nullptr, *d_lineface = nullptr, *d_identity = nullptr;

    /* ---- Jacobian (element / face order, as read) ---- */
    double *d_jacD = nullptr, *d_O1 = nullptr, *d_O2 = nullptr, *d_rhs = nullptr;
    double *d_U = nullptr, *d_dU = nullptr, *d_R = nullptr, *d_Uinit = nullptr;
    double *d_scratch = nullptr; /* 9*nelem element-order scratch */

    /* ---- TBS_ALGO_REFERENCE ---- */
    double *d_DLU = nullptr, *d_DinvC = nullptr, *d_A = nullptr;

    /* ---- line-ordered layout (FP64 / MIXED) ---- */
    tbs::FastLayout L{};
    bool layout_ok = false;
    double *d_gamlast = nullptr; /* per line and chain: last Gam toward the twist, FP64 */
    long long n_xslots_real = 0;
    long long n_fslots_real = 0; /* interior face slots of all cells */
    double *d_Dinv = nullptr, *d_G = nullptr, *d_Gam = nullptr, *d_X = nullptr;
    double *d_Dp = nullptr, *d_XF = nullptr; /* MIXED: position-ordered original blocks */
    double *d_Up = nullptr, *d_dUp = nullptr, *d_b = nullptr, *d_y = nullptr;
    /* a line partition's second U: its line solves write U + dU there and
     * its residual launch makes it the current U (swapped with d_Up) */
    double *d_Up_alt = nullptr;
    double *d_rhsp = nullptr, *d_Rp = nullptr;
    float *d_Dinv32 = nullptr, *d_G32 = nullptr, *d_Gam32 = nullptr, *d_X32 = nullptr;
    float *d_b32 = nullptr, *d_y32 = nullptr, *d_d32 = nullptr, *d_c32 = nullptr,
          *d_R32 = nullptr;
    int inner_sweeps = 4;  /* TBS_ALGO_MIXED inner sweeps per outer step */
    int inner_first = 0;   /* > 0: the first outer step's inner sweeps */
    int outer_done = 0;    /* outer steps since the last prime (eager sequences) */
    bool lagged = false;   /* block values replaced since the factorization (tbs_update_values) */
    int check = 1;         /* tbs_solve checks a converged TBS_ALGO_FP64 solve against
                            * the true residual (tbs_set_check) */

    /* ---- norms / solve state ---- */
    double *d_partials = nullptr, *d_partials2 = nullptr;
    int npart_cap = 0;
    tbs::SolveState *d_state = nullptr;
    tbs::SolveState *h_state = nullptr; /* pinned, mapped: written by a kernel */
    tbs::SolveState *h_state_dev = nullptr; /* its device address */
    double *d_hist = nullptr;
    int hist_cap = 0;
    double *h_hist = nullptr;     /* pinned, mapped copy of the history for the host */
    double *h_hist_dev = nullptr;
    int h_hist_cap = 0;
    unsigned *d_status = nullptr;
    unsigned long long *d_ktimer = nullptr; /* device-clock record of the sweeps' residual launches */
    unsigned *h_status = nullptr; /* pinned, mapped */
    unsigned *h_status_dev = nullptr;
    unsigned *d_counter = nullptr; /* last-CTA ticket of the fused norm */
    int algo = -1;

    /* ---- graph cache ---- */
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    int graph_algo = -1;

    /* ---- staged Jacobians (tbs_stage_jacobian): up to two next systems'
     * jacD, O1, O2 and rhs, uploaded on the copy stream into landing slots
     * while the current system is solved; tbs_factor copies the oldest over
     * the active set on the device ---- */
    static constexpr int kLandSlots = 2;
    double *d_land[kLandSlots][4] = {};
    cudaStream_t copy = nullptr;
    cudaEvent_t land_ready[kLandSlots] = {}; /* the slot's upload has landed */
    cudaEvent_t land_free[kLandSlots] = {};  /* the copy out of the slot is done */
    int land_head = 0;                       /* oldest staged slot */
    int land_count = 0;                      /* staged systems waiting for tbs_factor */

    /* ---- several right-hand sides: vectors and graph, made on first use ---- */
    MultiBufs *multi = nullptr;
    /* ---- GMRES: Krylov basis and work vectors, made on first use ---- */
    KrylovBufs *krylov = nullptr;

    /* ---- memory accounting ---- */
    std::vector<std::pair<void *, size_t>> allocs;
    size_t bytes = 0;

    /* ---- profiling ---- */
    bool prof = false;
    std::vector<ProfSlot> slots;
    std::vector<PendingEvent> pending;
    std::vector<cudaEvent_t> pool;
};

/* whether TBS_ALGO_MIXED's outer residual uses the position-ordered blocks */
bool fullpos_ok(const tbs_ctx *ctx);
/* device history of at least `need` norms (drops the cached graph when it grows) */
int ctx_ensure_hist(tbs_ctx *ctx, int need);
/* tolerance, sweep limit and history capacity of the device SolveState */
int ctx_set_state(tbs_ctx *ctx, double tol, int max_sweeps);
/* reads and clears the device status word; a set bit becomes the error */
int ctx_status(tbs_ctx *ctx);
/* tbs_set_jacobian from host memory in pieces of at most `piece` bytes, at
 * most two in flight (returns when the last piece is issued) */
int ctx_set_jacobian_paced(tbs_ctx *ctx, const double *jacD, const double *jacO1, const double *jacO2,
                           const double *rhs, size_t piece);
/* profiling brackets (a no-op unless profiling, outside stream capture):
 * begin records the start event of a launch named `name` and returns its
 * handle, end records its end event; resolve adds the finished pairs up */
int ctx_prof_begin(tbs_ctx *ctx, const char *name);
void ctx_prof_end(tbs_ctx *ctx, int h);
void ctx_prof_resolve(tbs_ctx *ctx);
/* multi.cu: free the multi-RHS vectors and graph / drop only the graph /
 * their device bytes */
void multi_free(tbs_ctx *ctx);
void multi_drop_graph(tbs_ctx *ctx);
size_t multi_bytes(const tbs_ctx *ctx);
/* krylov.cu: free the GMRES vectors / their device bytes */
void krylov_free(tbs_ctx *ctx);
size_t krylov_bytes(const tbs_ctx *ctx);

#endif /* TBS_CTX_HXX */

/*
 * engine.hxx -- batched launch sequences over many factored systems, shared
 * by tbs_batch (a fixed set of systems, batch.cu) and tbs_server (a request
 * loop whose in-flight set changes between graph launches, server.cu).
 *
 * A member is one right-hand side in flight: the factors and layout of a
 * system (a tbs_ctx) plus its own vectors.  Members of the same system
 * share the factors.  One instantiated CUDA graph runs
 *     prime(members marked fresh) -> while (rule) { one sweep of every
 *     active member }
 * where every kernel reads its work count from the device BatchCtl, so
 * the graph is rebuilt only when the capacity, the algorithm or the
 * schedule changes, not when members come and go.
 */
#ifndef TBS_ENGINE_HXX
#define TBS_ENGINE_HXX

#include "ctx.hxx"

#include <string>
#include <vector>

namespace tbs {

/* the vectors of one right-hand side in flight, position order unless
 * noted; the TBS_ALGO_FP64 or the TBS_ALGO_MIXED set is used */
struct VecSet {
    double *Up = nullptr, *dUp = nullptr, *b = nullptr, *y = nullptr, *rhsp = nullptr;
    const double *rhs = nullptr;   /* element order: the full residual's rhs */
    double *Rp = nullptr;          /* FP64 residual of U_init */
    double *partials = nullptr;
    double *partials2 = nullptr;   /* scratch partials of the U_init residual */
    const double *Uinit = nullptr; /* element order, or null: start from U = 0 */
    SolveState *state = nullptr;
    double *hist = nullptr;
    float *b32 = nullptr, *y32 = nullptr, *d32 = nullptr, *c32 = nullptr, *R32 = nullptr;
};

/* a context's own vectors */
VecSet ctx_vectors(tbs_ctx *c);

struct Member {
    tbs_ctx *sys;  /* factors, layout, mesh */
    VecSet v;
    bool fresh;    /* started (primed) by the next run */
};

struct Engine {
    int device = 0;
    int algo = -1;
    int inner = 4;            /* TBS_ALGO_MIXED inner sweeps per outer step */
    int inner_first = 0;      /* > 0: the first outer step's (all members fresh together) */
    cudaStream_t stream = nullptr;
    BatchSched sched{8, 2, 1};
    int order = 0;            /* Thomas items: 0 longest lines first, 1 mesh order */
    int max_nx = 0;           /* widest member (shared-memory size of the residual) */
    std::string err;

    /* capacity-sized device arrays (reallocated, and the graph rebuilt, on growth) */
    int cap_mem = 0, cap_lines = 0;
    std::vector<void *> allocs;
    ThomasSys<double> *d_th64 = nullptr;
    ThomasSys<float> *d_th32 = nullptr;
    ResidSys<double> *d_rs_prime = nullptr, *d_rs_body = nullptr;
    ResidSys<float> *d_rs32_rhs = nullptr, *d_rs32_dx = nullptr;
    FullResSys *d_fr = nullptr;
    FullPosSys *d_fp = nullptr;
    bool fullpos = false;     /* MIXED outer residual from position-ordered blocks */
    int max_nxf = 0;
    VecSys *d_vec = nullptr;
    ReduceSys *d_red_prime = nullptr, *d_red_body = nullptr;
    WorkItem *d_lines = nullptr;                       /* Thomas items, explicit */
    /* FP64: line solves of groups of one system's members (multi-RHS) */
    MultiLine *d_ml = nullptr;
    WorkItem *d_mitems = nullptr;
    int cap_mitems = 0;
    int *d_g_tiles = nullptr, *d_g_prime = nullptr, *d_g_blocks = nullptr; /* group indices */
    int *d_g_chunks = nullptr; /* every member, units of BATCH_CHUNK tiles */
    int *d_g_solo = nullptr;   /* members alone in their system, units of BATCH_CHUNK tiles */
    int *d_g_units = nullptr;  /* systems with several members, units of BATCH_CHUNK tiles */
    int *d_active = nullptr;
    unsigned *d_queue = nullptr, *d_counter = nullptr, *d_status = nullptr;
    BatchCtl *d_ctl = nullptr;
    BatchCtl *h_ctl = nullptr;     /* pinned */
    unsigned *h_status = nullptr;  /* pinned, written by the device */
    std::vector<int> h_active;
    int *h_active_pin = nullptr;   /* pinned, written by the device */
    int h_active_cap = 0;
    /* pinned staging of the descriptor and work-list uploads, read by one
     * copy launch (never by the copy engine, never a synchronisation with
     * the stream); reused once stage_ev has passed */
    char *h_stage = nullptr;
    size_t stage_cap = 0;
    cudaEvent_t stage_ev = nullptr;

    /* the members of the last engine_set_members */
    std::vector<Member> members;
    /* members with a starting solution: their U_init residual is one
     * launch each inside the graph, so the graph depends on this list */
    std::vector<int> uinit;

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool graph_ok = false;

    bool prof = false;
    std::vector<ProfSlot> slots;
    std::vector<PendingEvent> pending;
    std::vector<cudaEvent_t> pool;
};

int engine_init(Engine &e, int device, cudaStream_t stream, int algo);
void engine_free(Engine &e);
void engine_drop_graph(Engine &e);
/* descriptors, work lists and counts for `members`; active flags: fresh
 * members 0 (their prime sets them), the others 1 */
int engine_set_members(Engine &e, const std::vector<Member> &members);
/* same members, all fresh again (a new solve of a fixed set) */
int engine_restart(Engine &e);
/* after a run: the members primed by it are no longer fresh (no upload of
 * descriptors or work lists, only the prime counts change) */
void engine_mark_started(Engine &e);
/* one graph launch (eager launches while profiling) and the device status;
 * chunk_limit > 0 ends the sweep loop after that many sweeps, and
 * stop_on_finish ends it as soon as a member stops */
int engine_run(Engine &e, int chunk_limit, int stop_on_finish);
/* the same as an asynchronous graph launch (engine_finish waits for it and
 * checks the device status); while profiling it runs engine_run */
int engine_launch(Engine &e, int chunk_limit, int stop_on_finish);
int engine_finish(Engine &e);
/* times the persistent Thomas launch for each schedule that fits */
int engine_tune(Engine &e, BatchSched *best, int *best_order, double *best_ms);
int engine_set_schedule(Engine &e, BatchSched s, int order);
/* the active flags after the last run */
int engine_read_active(Engine &e);

}  // namespace tbs

#endif /* TBS_ENGINE_HXX */

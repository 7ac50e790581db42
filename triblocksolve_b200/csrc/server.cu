/*
 * server.cu -- tbs_server_*: a request loop over systems whose factors stay
 * resident in HBM (continuous batching).  No counterpart in the reference,
 * whose driver (src/main.cxx) factors and sweeps one system per run.
 *
 * Requests carry right-hand sides for a registered system and, optionally,
 * new Jacobian values that re-factor the system first.  A loop thread
 *   - admits queued requests in arrival order while their right-hand sides
 *     fit the device budget and the slot limit (admission by footprint;
 *     a request that does not fit holds back the ones behind it, so that
 *     large requests are not starved),
 *   - runs every admitted right-hand side together through the batched
 *     engine (engine.hxx): one graph launch primes the newly admitted ones
 *     and sweeps all of them until one reaches its tolerance or a chunk of
 *     sweeps is done, so new arrivals join at the next sweep boundary,
 *   - retires each right-hand side as soon as it stops and completes a
 *     request when all of its right-hand sides have.
 * A factor thread per lane re-factors systems (upload of the new values
 * and the factorization on the system's own stream) into a spare copy of the
 * system's factors, so that the right-hand sides already admitted keep
 * sweeping on the current copy; the system's later requests wait for the
 * new factors.  When the spare copy does not fit the budget, the system is
 * re-factored in place once none of its right-hand sides is in flight.
 *
 * The per-right-hand-side arithmetic is that of tbs_solve: a result does
 * not depend on what else was in flight.
 */
#include "engine.hxx"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

using namespace tbs;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct SrvSystem {
    /* two versions of the system's factors: new Jacobian values are
     * uploaded and factored into the spare while the right-hand sides
     * already admitted keep sweeping on the current one */
    tbs_ctx *ctx[2] = {nullptr, nullptr};
    int cur = 0;
    int inflight[2] = {0, 0}; /* right-hand sides in flight per version */
    bool refactoring = false;
    bool broken = false;      /* an in-place re-factorization failed */
    size_t bytes = 0;         /* device bytes of one version */
    int lane = 0;
};

struct SrvRequest {
    long long id = 0;
    int sys = 0;
    int ver = 0;                 /* the system version it runs on (set at admission) */
    int target = 0;              /* the version a re-factorization writes */
    bool new_version = false;    /* that version's context is created by the factor thread */
    tbs_ctx *ctx = nullptr;      /* the version's context (stable while the server lives) */
    int nrhs = 0;
    const double *rhs = nullptr; /* caller's: nrhs x 9 nelem, valid until completion */
    double *U = nullptr;         /* caller's output */
    double tol = 0.0;
    int max_sweeps = 0;
    const double *jacD = nullptr, *jacO1 = nullptr, *jacO2 = nullptr; /* re-factor first */
    bool refactored = false;
    std::vector<int> sweeps;
    std::vector<double> rel;
    int remaining = 0;
    enum { QUEUED, FACTORING, RUNNING, DONE, FAILED } state = QUEUED;
    int err = 0;
    std::string msg;
    size_t bytes = 0;            /* device bytes of its right-hand sides */
    Clock::time_point t_submit, t_admit, t_done;
};

struct SrvSlot {               /* one right-hand side in flight (an engine member) */
    SrvRequest *req = nullptr;
    int k = 0;                 /* which right-hand side of the request */
    void *mem = nullptr;       /* one stream-ordered allocation for all its vectors */
    size_t bytes = 0;
    VecSet v;
    double *rhs_elem = nullptr; /* element-order rhs, reused for the solution read-back */
    bool fresh = true;
};

}  // namespace

struct SrvIncoming {               /* uploads issued, not yet members */
    std::vector<SrvSlot> slots;
    cudaEvent_t ev;                /* their uploads are done */
};

struct SrvPending {                /* read-backs in flight */
    std::vector<SrvSlot> slots;
    std::vector<SolveState> st;
    cudaEvent_t ev;
};

struct SrvLane {
    int id = 0;
    Engine eng;
    cudaStream_t stream = nullptr;     /* graph launches */
    cudaStream_t up = nullptr;         /* uploads of admitted right-hand sides */
    cudaStream_t down = nullptr;       /* read-back of finished solutions */
    std::vector<SrvSlot> slots;        /* members of the engine */
    std::deque<SrvIncoming> incoming;
    cudaEvent_t ev_up = nullptr;       /* the last batch of uploads is done */
    std::deque<SrvPending> pending;
    std::vector<cudaEvent_t> ev_pool;
    SolveState *h_states = nullptr;    /* pinned, max_slots: read-back of states */
    std::string err;
    std::thread th;
    /* re-factorizations of this lane's systems, by the lane's own factor
     * thread: a small system's new Jacobian never waits behind a large one */
    std::deque<SrvRequest *> factor_jobs;
    std::thread factor;
};

struct tbs_server {
    int device = 0;
    int algo = TBS_ALGO_FP64;
    size_t budget = 0;         /* device bytes for systems + right-hand sides in flight */
    int max_slots = 64;
    int chunk = 4;             /* sweeps per graph launch at most */
    std::string err;

    std::mutex mu;
    std::condition_variable cv_loop, cv_done, cv_factor;
    bool stopping = false;
    std::vector<SrvSystem> systems;
    size_t sys_bytes = 0;
    size_t slot_bytes_in_flight = 0;
    std::deque<SrvRequest *> queue;
    std::map<long long, std::unique_ptr<SrvRequest>> requests;
    long long next_id = 1;

    /* one loop thread per lane: a system sweeps in the lane given by how
     * many of the ascending lane_splits its cell count reaches, so that
     * small systems are not held to the pace of large ones (by default
     * three lanes: below 262,144 cells, below 1,048,576, and larger) */
    std::vector<long long> lane_splits{262144, 1048576};
    std::vector<std::unique_ptr<struct SrvLane>> lanes;
    cudaMemPool_t pool = nullptr;
    bool pool_reserved = false;
    int rhs_in_flight = 0;             /* admitted, not yet read back (all lanes) */

    /* statistics */
    long long n_done = 0, n_rhs_done = 0, n_launches = 0, n_refactor = 0;
    long long peak_rhs = 0, peak_bytes = 0;
    /* loop-thread time (microseconds): starting admitted right-hand sides
     * (clear, upload, permute), rebuilding the member set, graph launches
     * until they return, retiring (read-back) */
    double us_start = 0, us_members = 0, us_run = 0, us_retire = 0;
};

static int sfail(tbs_server *s, int code, const std::string &msg) {
    if (s) s->err = msg;
    set_thread_error(msg);
    return code;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

/* CTAs of a right-hand side's or solution's copy through pinned host
 * memory: enough 16-byte accesses in flight for the host link, while the
 * sweeps keep the rest of the SMs */
constexpr int kSysmemCtas = 32;

/* lanes (loop and factor threads, engines) a server runs; the lane splits
 * decide how many of them receive systems */
constexpr int kMaxLanes = 4;

/* a re-factorization's Jacobian goes up in pieces of this size, at most two
 * in flight, so that the loop threads' copies never wait behind more than
 * two pieces (about 2.4 ms of the host link) */
constexpr size_t kRefactorPiece = 64ull << 20;

/* device bytes of one right-hand side of system c with a history of hist_n */
static size_t slot_bytes(const tbs_ctx *c, int algo, int hist_n) {
    const size_t npv = (size_t)c->L.np16 * 9, ne = (size_t)c->nelem * 9;
    const size_t nt = (size_t)fast_resid_grid(c->L.np16);
    size_t b = 0;
    if (algo == TBS_ALGO_FP64) {
        b += 5 * align256(npv * sizeof(double)); /* Up, dUp, b, y, rhsp */
        b += align256(nt * sizeof(double));
    } else {
        b += 2 * align256(npv * sizeof(double)); /* Up, rhsp */
        b += 5 * align256(npv * sizeof(float));  /* b32, y32, d32, c32, R32 */
        b += align256(std::max(nt, (size_t)full_resid_blocks(c->nelem)) * sizeof(double));
    }
    b += align256(ne * sizeof(double));          /* rhs, element order */
    b += align256(sizeof(SolveState));
    b += align256((size_t)hist_n * sizeof(double));
    return b;
}

/* carve a slot's vectors out of its allocation */
static void slot_layout(SrvSlot &sl, const tbs_ctx *c, int algo, int hist_n) {
    const size_t npv = (size_t)c->L.np16 * 9, ne = (size_t)c->nelem * 9;
    const size_t nt = (size_t)fast_resid_grid(c->L.np16);
    char *p = static_cast<char *>(sl.mem);
    auto take = [&](size_t n) {
        char *q = p;
        p += align256(n);
        return q;
    };
    VecSet v;
    if (algo == TBS_ALGO_FP64) {
        v.Up = (double *)take(npv * sizeof(double));
        v.dUp = (double *)take(npv * sizeof(double));
        v.b = (double *)take(npv * sizeof(double));
        v.y = (double *)take(npv * sizeof(double));
        v.rhsp = (double *)take(npv * sizeof(double));
        v.partials = (double *)take(nt * sizeof(double));
    } else {
        v.Up = (double *)take(npv * sizeof(double));
        v.rhsp = (double *)take(npv * sizeof(double));
        v.b32 = (float *)take(npv * sizeof(float));
        v.y32 = (float *)take(npv * sizeof(float));
        v.d32 = (float *)take(npv * sizeof(float));
        v.c32 = (float *)take(npv * sizeof(float));
        v.R32 = (float *)take(npv * sizeof(float));
        v.partials = (double *)take(std::max(nt, (size_t)full_resid_blocks(c->nelem)) * sizeof(double));
    }
    sl.rhs_elem = (double *)take(ne * sizeof(double));
    v.rhs = sl.rhs_elem;
    v.state = (SolveState *)take(sizeof(SolveState));
    v.hist = (double *)take((size_t)hist_n * sizeof(double));
    sl.v = v;
}

static void complete(tbs_server *s, SrvRequest *r, int err, const std::string &msg) {
    r->t_done = Clock::now();
    r->state = err ? SrvRequest::FAILED : SrvRequest::DONE;
    r->err = err;
    r->msg = msg;
    if (!err) {
        s->n_done += 1;
        s->n_rhs_done += r->nrhs;
    }
}

/* ---------------------------------------------------------------- factor thread */

static void factor_main(tbs_server *s, SrvLane *L) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_factor.wait(lk, [&] { return s->stopping || !L->factor_jobs.empty(); });
        if (L->factor_jobs.empty()) {
            if (s->stopping) break;
            continue;
        }
        SrvRequest *r = L->factor_jobs.front();
        L->factor_jobs.pop_front();
        tbs_ctx *c = s->systems[r->sys].ctx[r->target];
        const tbs_ctx *model = s->systems[r->sys].ctx[s->systems[r->sys].cur];
        const bool fresh = r->new_version;
        lk.unlock();
        int rc = TBS_OK;
        if (fresh) {
            /* the spare version: same mesh as the current one */
            rc = tbs_create(s->device, &c);
            if (!rc)
                rc = tbs_set_mesh(c, model->nvar, model->nelem, model->nintface, model->eftot,
                                  model->nline, model->nlineelem, model->h_epoint.data(),
                                  model->h_ef.data(), model->h_fc.data(), model->h_linesize.data(),
                                  model->h_linepoint.data(), model->h_lines.data(),
                                  model->h_lineface.data());
        }
        if (!rc) rc = ctx_set_jacobian_paced(c, r->jacD, r->jacO1, r->jacO2, r->rhs, kRefactorPiece);
        if (!rc) rc = tbs_factor(c, s->algo);
        std::string msg = rc ? std::string(c ? tbs_last_error(c) : thread_error()) : std::string();
        lk.lock();
        SrvSystem &sys = s->systems[r->sys]; /* re-read: systems may have been added */
        sys.refactoring = false;
        s->n_refactor += 1;
        if (rc) {
            if (fresh) {
                /* the current version is untouched: only this request fails */
                if (c) tbs_destroy(c);
                s->sys_bytes -= sys.bytes;
            } else if (r->target == sys.cur) {
                /* in place: the factors may be half replaced */
                sys.broken = true;
            }
            complete(s, r, rc, "re-factorization failed: " + msg);
            s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
            s->cv_done.notify_all();
        } else {
            if (fresh) sys.ctx[r->target] = c;
            sys.cur = r->target;
            r->refactored = true;
            r->state = SrvRequest::QUEUED;
        }
        s->cv_loop.notify_all();
    }
}

/* ---------------------------------------------------------------- loop threads */

/* Admission scan of one lane under the lock: the lane's requests in
 * arrival order; a request that needs a re-factorization goes to the
 * factor thread once its target copy is idle; later requests of a system
 * that is being re-factored wait; the first request whose right-hand sides
 * do not fit (budget, or right-hand sides in flight) ends the scan. */
static void admit_scan(tbs_server *s, SrvLane *L, std::vector<SrvRequest *> &admitted) {
    std::vector<char> blocked(s->systems.size(), 0);
    const size_t avail = s->budget > s->sys_bytes ? s->budget - s->sys_bytes : 0;
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        SrvRequest *r = *it;
        SrvSystem &sys = s->systems[r->sys];
        if (sys.lane != L->id) {
            ++it;
            continue;
        }
        if (sys.broken && r->state == SrvRequest::QUEUED) {
            complete(s, r, TBS_ERR_STATE, "the system's re-factorization failed");
            s->cv_done.notify_all();
            it = s->queue.erase(it);
            continue;
        }
        if (r->state == SrvRequest::FACTORING || blocked[r->sys] || sys.refactoring) {
            blocked[r->sys] = 1;
            ++it;
            continue;
        }
        if (r->jacD && !r->refactored) {
            /* into the spare copy while the current one keeps sweeping;
             * in place (after the system drains) when a spare does not fit */
            const int spare = 1 - sys.cur;
            const bool have = sys.ctx[spare] != nullptr;
            const bool fits = have || s->sys_bytes + sys.bytes + s->slot_bytes_in_flight <= s->budget;
            const int target = fits ? spare : sys.cur;
            if (sys.inflight[target] == 0) {
                sys.refactoring = true;
                r->target = target;
                r->new_version = fits && !have;
                if (r->new_version) s->sys_bytes += sys.bytes;
                r->state = SrvRequest::FACTORING;
                L->factor_jobs.push_back(r);
                s->cv_factor.notify_all();
            }
            blocked[r->sys] = 1;
            ++it;
            continue;
        }
        if (s->rhs_in_flight + r->nrhs > s->max_slots || s->slot_bytes_in_flight + r->bytes > avail) break;
        s->slot_bytes_in_flight += r->bytes;
        s->rhs_in_flight += r->nrhs;
        r->ver = sys.cur;
        r->ctx = sys.ctx[sys.cur];
        sys.inflight[r->ver] += r->nrhs;
        r->state = SrvRequest::RUNNING;
        r->t_admit = Clock::now();
        admitted.push_back(r);
        it = s->queue.erase(it);
    }
}

/* Keep freed right-hand-side memory in the pool and grow it once to the
 * room the budget leaves after the resident systems, so that admissions do
 * not pay for mapping new device memory. */
static void reserve_pool(tbs_server *s, SrvLane *L, size_t avail) {
    if (avail == 0) return;
    void *p = nullptr;
    if (cudaMallocFromPoolAsync(&p, avail, s->pool, L->up) == cudaSuccess) {
        cudaFreeAsync(p, L->up);
        cudaStreamSynchronize(L->up);
    } else {
        cudaGetLastError(); /* not fatal: the pool then grows on demand */
    }
}

static cudaEvent_t take_event(SrvLane *L) {
    if (!L->ev_pool.empty()) {
        cudaEvent_t e = L->ev_pool.back();
        L->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return e;
}

static int lfail(SrvLane *L, int code, const std::string &msg) {
    L->err = msg;
    set_thread_error(msg);
    return code;
}

/* allocate, clear and fill the right-hand sides of newly admitted requests
 * on the upload stream (overlapping the running graph); they become engine
 * members once their uploads are done */
static int start_requests(tbs_server *s, SrvLane *L, const std::vector<SrvRequest *> &admitted,
                          std::vector<SrvRequest *> &failed) {
    if (admitted.empty()) return TBS_OK;
    /* the staging of the previous uploads is free once they have run */
    if (cudaEventSynchronize(L->ev_up) != cudaSuccess) return lfail(L, TBS_ERR_CUDA, "event failed");
    SrvIncoming batch;
    for (SrvRequest *r : admitted) {
        tbs_ctx *c = r->ctx;
        const size_t nv = (size_t)c->nelem * 9;
        const size_t per = r->bytes / r->nrhs;
        bool ok = true;
        std::vector<SrvSlot> mine;
        for (int k = 0; k < r->nrhs && ok; ++k) {
            SrvSlot sl;
            sl.req = r;
            sl.k = k;
            sl.bytes = per;
            if (cudaMallocFromPoolAsync(&sl.mem, per, s->pool, L->up) != cudaSuccess) {
                cudaGetLastError();
                ok = false;
                break;
            }
            mine.push_back(sl);
            SrvSlot &m = mine.back();
            slot_layout(m, c, s->algo, r->max_sweeps + 1);
            /* pad positions of the layout are never written by the kernels
             * but enter the first norm (rhs) and the U accumulation: start
             * from zeros, as a context's arrays do */
            /* the state by kernel parameter and the right-hand side by the
             * SMs when the caller's memory is pinned: neither waits in the
             * copy engine behind a re-factorization's Jacobian upload */
            SolveState st{};
            st.tol = r->tol;
            st.max_sweeps = r->max_sweeps;
            st.hist_cap = r->max_sweeps + 1;
            ok = launch_zero(L->up, static_cast<double *>(m.mem), (long long)(per / sizeof(double))) == 0 &&
                 xfer_put(L->up, m.v.state, &st, sizeof(st)) == 0 &&
                 xfer_to_device(L->up, m.rhs_elem, r->rhs + k * nv, nv * sizeof(double), kSysmemCtas) == 0 &&
                 launch_permute_to_pos(L->up, 9, c->nelem, c->L.pos_of_elem, m.rhs_elem, m.v.rhsp) == 0;
        }
        if (!ok) {
            for (SrvSlot &sl : mine)
                if (sl.mem) cudaFreeAsync(sl.mem, L->up);
            failed.push_back(r);
            continue;
        }
        for (SrvSlot &sl : mine) batch.slots.push_back(sl);
    }
    if (cudaEventRecord(L->ev_up, L->up) != cudaSuccess) return lfail(L, TBS_ERR_CUDA, "event record failed");
    if (!batch.slots.empty()) {
        batch.ev = take_event(L);
        if (cudaEventRecord(batch.ev, L->up) != cudaSuccess) return lfail(L, TBS_ERR_CUDA, "event record failed");
        L->incoming.push_back(std::move(batch));
    }
    return TBS_OK;
}

static int engine_members(SrvLane *L) {
    std::vector<Member> m;
    m.reserve(L->slots.size());
    for (SrvSlot &sl : L->slots) m.push_back({sl.req->ctx, sl.v, sl.fresh});
    return engine_set_members(L->eng, m);
}

/* the members that stopped: their states now (pinned, main stream), their
 * solutions permuted to element order on the main stream and copied to the
 * caller on the read-back stream (overlapping the next graph) */
static int retire(SrvLane *L) {
    std::vector<SrvSlot> keep, out;
    for (size_t k = 0; k < L->slots.size(); ++k)
        (L->eng.h_active[k] ? keep : out).push_back(L->slots[k]);
    if (out.empty()) return TBS_OK;
    for (size_t k = 0; k < out.size(); ++k) {
        SrvSlot &sl = out[k];
        tbs_ctx *c = sl.req->ctx;
        if (xfer_to_host(L->stream, &L->h_states[k], sl.v.state, sizeof(SolveState), 1) != 0 ||
            launch_permute_to_elem(L->stream, 9, c->nelem, c->L.pos_of_elem, sl.v.Up, sl.rhs_elem) != 0)
            return lfail(L, TBS_ERR_CUDA, "solution read-back failed");
    }
    cudaEvent_t ready = take_event(L);
    if (cudaEventRecord(ready, L->stream) != cudaSuccess ||
        cudaStreamWaitEvent(L->down, ready, 0) != cudaSuccess)
        return lfail(L, TBS_ERR_CUDA, "event failed");
    L->ev_pool.push_back(ready); /* reusable: the wait is already enqueued */
    SrvPending p;
    for (SrvSlot &sl : out) {
        tbs_ctx *c = sl.req->ctx;
        const size_t nv = (size_t)c->nelem * 9;
        if (xfer_to_host(L->down, sl.req->U + sl.k * nv, sl.rhs_elem, nv * sizeof(double), kSysmemCtas) != 0)
            return lfail(L, TBS_ERR_CUDA, "solution read-back failed");
        cudaFreeAsync(sl.mem, L->down);
    }
    if (cudaStreamSynchronize(L->stream) != cudaSuccess) return lfail(L, TBS_ERR_CUDA, "state read-back failed");
    p.st.assign(L->h_states, L->h_states + out.size());
    p.slots.swap(out);
    p.ev = take_event(L);
    if (cudaEventRecord(p.ev, L->down) != cudaSuccess) return lfail(L, TBS_ERR_CUDA, "event failed");
    L->pending.push_back(std::move(p));
    L->slots.swap(keep);
    return TBS_OK;
}

/* read-backs that finished; called without the lock */
static int collect(SrvLane *L, std::vector<SrvPending> &done) {
    while (!L->pending.empty()) {
        SrvPending &p = L->pending.front();
        if (cudaEventSynchronize(p.ev) != cudaSuccess) return lfail(L, TBS_ERR_CUDA, "read-back failed");
        L->ev_pool.push_back(p.ev);
        done.push_back(std::move(p));
        L->pending.pop_front();
    }
    return TBS_OK;
}

static void loop_main(tbs_server *s, SrvLane *L) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        const int chunk = s->chunk;
        lk.unlock();
        auto t0 = Clock::now();
        /* 1. sweep the members while the host admits and copies */
        int rc = TBS_OK;
        const bool running = !L->slots.empty();
        if (running) rc = engine_launch(L->eng, chunk, 1);
        /* 2. admission and uploads */
        std::vector<SrvRequest *> admitted, failed;
        lk.lock();
        admit_scan(s, L, admitted);
        size_t reserve = 0;
        if (!admitted.empty() && !s->pool_reserved) {
            s->pool_reserved = true;
            reserve = s->budget > s->sys_bytes ? s->budget - s->sys_bytes : 0;
        }
        lk.unlock();
        if (reserve) reserve_pool(s, L, reserve);
        auto t1 = Clock::now();
        if (!rc) rc = start_requests(s, L, admitted, failed);
        /* 3. solutions that reached the caller */
        std::vector<SrvPending> copied;
        if (!rc) rc = collect(L, copied);
        auto t2 = Clock::now();
        /* 4. the sweeps' end: retire the members that stopped */
        if (running && !rc) rc = engine_finish(L->eng);
        if (running && !rc) rc = engine_read_active(L->eng);
        auto t3 = Clock::now();
        if (running && !rc) {
            for (SrvSlot &sl : L->slots) sl.fresh = false;
            engine_mark_started(L->eng);
            rc = retire(L);
        }
        auto t4 = Clock::now();
        /* 5. the next member set: the remaining ones and the arrivals whose
         * uploads are done (the sweeps never wait for a copy; with nothing
         * to sweep the loop waits for the oldest upload) */
        bool changed = running && L->eng.h_ctl->nsys != (int)L->slots.size();
        while (!rc && !L->incoming.empty()) {
            SrvIncoming &in = L->incoming.front();
            const cudaError_t q = L->slots.empty() ? cudaEventSynchronize(in.ev) : cudaEventQuery(in.ev);
            if (q == cudaErrorNotReady) break;
            if (q != cudaSuccess) {
                rc = lfail(L, TBS_ERR_CUDA, "upload failed");
                break;
            }
            for (SrvSlot &sl : in.slots) L->slots.push_back(sl);
            L->ev_pool.push_back(in.ev);
            L->incoming.pop_front();
            changed = true;
        }
        if (!rc && changed && !L->slots.empty()) rc = engine_members(L);
        auto t5 = Clock::now();
        std::string msg = rc ? L->eng.err + L->err : std::string();
        lk.lock();
        s->us_start += 1e3 * ms_between(t1, t2);
        s->us_members += 1e3 * ms_between(t4, t5);
        s->us_run += 1e3 * (ms_between(t0, t1) + ms_between(t2, t3));
        s->us_retire += 1e3 * ms_between(t3, t4);
        if (running) s->n_launches += 1;
        s->peak_rhs = std::max<long long>(s->peak_rhs, (long long)s->rhs_in_flight);
        s->peak_bytes = std::max<long long>(s->peak_bytes, (long long)s->slot_bytes_in_flight);
        for (SrvRequest *r : failed) {
            s->systems[r->sys].inflight[r->ver] -= r->nrhs;
            s->slot_bytes_in_flight -= r->bytes;
            s->rhs_in_flight -= r->nrhs;
            complete(s, r, TBS_ERR_NOMEM, "device allocation for the right-hand sides failed");
        }
        for (SrvPending &p : copied) {
            for (size_t k = 0; k < p.slots.size(); ++k) {
                SrvSlot &sl = p.slots[k];
                SrvRequest *r = sl.req;
                const SolveState &st = p.st[k];
                r->sweeps[sl.k] = st.sweep;
                r->rel[sl.k] = st.norm0 > 0.0 ? st.last / st.norm0 : 0.0;
                s->systems[r->sys].inflight[r->ver] -= 1;
                s->slot_bytes_in_flight -= sl.bytes;
                s->rhs_in_flight -= 1;
                if (--r->remaining == 0) complete(s, r, 0, "");
            }
        }
        if (rc) {
            /* a device error ends every request in flight in this lane */
            std::vector<SrvSlot> all = L->slots;
            for (SrvIncoming &in : L->incoming) all.insert(all.end(), in.slots.begin(), in.slots.end());
            for (SrvPending &p : L->pending) all.insert(all.end(), p.slots.begin(), p.slots.end());
            for (SrvSlot &sl : all) {
                SrvRequest *r = sl.req;
                s->systems[r->sys].inflight[r->ver] -= 1;
                s->slot_bytes_in_flight -= sl.bytes;
                s->rhs_in_flight -= 1;
                if (r->state == SrvRequest::RUNNING) complete(s, r, rc, msg);
            }
            L->slots.clear();
            L->incoming.clear();
            L->pending.clear();
            s->err = msg;
        }
        if (!failed.empty() || !copied.empty() || rc) {
            s->cv_done.notify_all();
            s->cv_loop.notify_all(); /* room freed: the other lane may admit */
        }
        /* 6. idle: nothing to sweep or copy; new requests, freed room or
         * the end of a re-factorization wake the loop */
        if (L->slots.empty() && L->incoming.empty() && L->pending.empty() && admitted.empty()) {
            bool mine = false, ready = false;
            for (SrvRequest *r : s->queue) {
                if (s->systems[r->sys].lane != L->id) continue;
                mine = true;
                if (r->state == SrvRequest::QUEUED && !s->systems[r->sys].refactoring) ready = true;
            }
            if (s->stopping && !mine && L->factor_jobs.empty()) break;
            if (!mine)
                s->cv_loop.wait(lk);
            else if (!ready) /* queued behind a re-factorization */
                s->cv_loop.wait_for(lk, std::chrono::milliseconds(1));
            else /* queued but did not fit: wait for room */
                s->cv_loop.wait_for(lk, std::chrono::milliseconds(1));
        }
    }
}

/* ---------------------------------------------------------------- entry points */

static void lane_free(SrvLane *L) {
    for (cudaStream_t x : {L->stream, L->up, L->down})
        if (x) cudaStreamSynchronize(x);
    if (L->eng.h_ctl) engine_free(L->eng);
    for (cudaEvent_t e : L->ev_pool) cudaEventDestroy(e);
    L->ev_pool.clear();
    if (L->ev_up) cudaEventDestroy(L->ev_up);
    if (L->h_states) cudaFreeHost(L->h_states);
    for (cudaStream_t x : {L->stream, L->up, L->down})
        if (x) cudaStreamDestroy(x);
    L->ev_up = nullptr;
    L->h_states = nullptr;
    L->stream = L->up = L->down = nullptr;
}

static int lane_init(tbs_server *s, SrvLane *L, int id) {
    L->id = id;
    if (cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&L->up, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&L->down, cudaStreamNonBlocking) != cudaSuccess)
        return lfail(L, TBS_ERR_CUDA, "cudaStreamCreate failed");
    if (cudaEventCreateWithFlags(&L->ev_up, cudaEventDisableTiming) != cudaSuccess)
        return lfail(L, TBS_ERR_CUDA, "cudaEventCreate failed");
    if (cudaMallocHost(&L->h_states, sizeof(SolveState) * (size_t)s->max_slots) != cudaSuccess)
        return lfail(L, TBS_ERR_NOMEM, "pinned allocation failed");
    int rc = engine_init(L->eng, s->device, L->stream, s->algo);
    if (rc) return lfail(L, rc, L->eng.err);
    return TBS_OK;
}

static void server_stop(tbs_server *s) {
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        /* queued requests that never started fail */
        for (SrvRequest *r : s->queue)
            if (r->state == SrvRequest::QUEUED) complete(s, r, TBS_ERR_STATE, "server stopped");
        std::deque<SrvRequest *> keep;
        for (SrvRequest *r : s->queue)
            if (r->state == SrvRequest::FACTORING) keep.push_back(r);
        s->queue.swap(keep);
        s->cv_loop.notify_all();
        s->cv_factor.notify_all();
        s->cv_done.notify_all();
    }
    for (auto &L : s->lanes)
        if (L->factor.joinable()) L->factor.join();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (SrvRequest *r : s->queue) complete(s, r, TBS_ERR_STATE, "server stopped");
        s->queue.clear();
        s->cv_loop.notify_all();
    }
    for (auto &L : s->lanes)
        if (L->th.joinable()) L->th.join();
}

extern "C" {

const char *tbs_server_last_error(const tbs_server *s) {
    if (!s) return thread_error();
    return s->err.c_str();
}

int tbs_server_create(int device_id, int algo, size_t device_budget_bytes, int max_rhs_in_flight,
                      tbs_server **out) {
    if (!out) return sfail(nullptr, TBS_ERR_ARG, "null output");
    *out = nullptr;
    if (algo != TBS_ALGO_FP64 && algo != TBS_ALGO_MIXED)
        return sfail(nullptr, TBS_ERR_UNSUPPORTED, "the server runs TBS_ALGO_FP64 or TBS_ALGO_MIXED");
    if (max_rhs_in_flight < 1 || device_budget_bytes == 0)
        return sfail(nullptr, TBS_ERR_ARG, "bad budget or slot limit");
    tbs_server *s = nullptr;
    try {
        s = new tbs_server();
        for (int k = 0; k < kMaxLanes; ++k) s->lanes.emplace_back(new SrvLane());
    } catch (...) {
        delete s;
        return sfail(nullptr, TBS_ERR_NOMEM, "host allocation failed");
    }
    s->device = device_id;
    s->algo = algo;
    s->budget = device_budget_bytes;
    s->max_slots = max_rhs_in_flight;
    auto fail = [&](int code, const std::string &msg) {
        for (auto &L : s->lanes) lane_free(L.get());
        if (s->pool) cudaMemPoolDestroy(s->pool);
        delete s;
        return sfail(nullptr, code, msg);
    };
    if (cudaSetDevice(device_id) != cudaSuccess) return fail(TBS_ERR_CUDA, "cudaSetDevice failed");
    for (size_t k = 0; k < s->lanes.size(); ++k) {
        int rc = lane_init(s, s->lanes[k].get(), (int)k);
        if (rc) return fail(rc, s->lanes[k]->err);
    }
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device_id;
    if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess)
        return fail(TBS_ERR_CUDA, "cudaMemPoolCreate failed");
    uint64_t keep = ~0ull; /* freed right-hand-side memory stays in the pool */
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    try {
        for (auto &L : s->lanes) {
            L->th = std::thread(loop_main, s, L.get());
            L->factor = std::thread(factor_main, s, L.get());
        }
    } catch (...) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stopping = true;
            s->cv_loop.notify_all();
            s->cv_factor.notify_all();
        }
        for (auto &L : s->lanes) {
            if (L->th.joinable()) L->th.join();
            if (L->factor.joinable()) L->factor.join();
        }
        return fail(TBS_ERR_STATE, "thread start failed");
    }
    *out = s;
    return TBS_OK;
}

int tbs_server_destroy(tbs_server *s) {
    if (!s) return TBS_OK;
    server_stop(s);
    cudaSetDevice(s->device);
    for (auto &L : s->lanes) lane_free(L.get());
    for (SrvSystem &sys : s->systems)
        for (tbs_ctx *c : sys.ctx)
            if (c) tbs_destroy(c);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return TBS_OK;
}

int tbs_server_set_lanes(tbs_server *s, long long split_cells) {
    if (!s) return sfail(nullptr, TBS_ERR_ARG, "null server");
    if (split_cells < 0) return sfail(s, TBS_ERR_ARG, "negative split");
    return tbs_server_set_lane_splits(s, &split_cells, split_cells > 0 ? 1 : 0);
}

int tbs_server_set_lane_splits(tbs_server *s, const long long *splits, int n) {
    if (!s) return sfail(nullptr, TBS_ERR_ARG, "null server");
    if (n < 0 || n > kMaxLanes - 1 || (n > 0 && !splits))
        return sfail(s, TBS_ERR_ARG, "at most " + std::to_string(kMaxLanes - 1) + " lane splits");
    for (int k = 0; k < n; ++k)
        if (splits[k] <= 0 || (k > 0 && splits[k] <= splits[k - 1]))
            return sfail(s, TBS_ERR_ARG, "lane splits must be positive and ascending");
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->systems.empty()) return sfail(s, TBS_ERR_STATE, "lanes are set before systems are added");
    s->lane_splits.assign(splits, splits + n);
    return TBS_OK;
}

int tbs_server_set_chunk(tbs_server *s, int sweeps) {
    if (!s) return sfail(nullptr, TBS_ERR_ARG, "null server");
    if (sweeps < 1) return sfail(s, TBS_ERR_ARG, "chunk must be at least one sweep");
    std::lock_guard<std::mutex> lk(s->mu);
    s->chunk = sweeps;
    return TBS_OK;
}

int tbs_server_add_system(tbs_server *s, int nvar, int nelem, int nintface, int eftot, int nline,
                          int nlineelem, const int *epoint, const int *ef, const int *fc,
                          const int *linesize, const int *linepoint, const int *lines,
                          const int *lineface, const double *jacD, const double *jacO1,
                          const double *jacO2, int *system_id) {
    if (!s || !system_id) return sfail(s, TBS_ERR_ARG, "null argument");
    if (nvar != 9) return sfail(s, TBS_ERR_UNSUPPORTED, "the server takes systems of nvar 9");
    tbs_ctx *c = nullptr;
    int rc = tbs_create(s->device, &c);
    if (rc) return sfail(s, rc, thread_error());
    auto fail = [&](int code) {
        std::string msg = tbs_last_error(c);
        tbs_destroy(c);
        return sfail(s, code, msg);
    };
    rc = tbs_set_mesh(c, nvar, nelem, nintface, eftot, nline, nlineelem, epoint, ef, fc, linesize,
                      linepoint, lines, lineface);
    if (rc) return fail(rc);
    try {
        std::vector<double> zero((size_t)nvar * nelem, 0.0);
        rc = tbs_set_jacobian(c, jacD, jacO1, jacO2, zero.data(), nullptr);
    } catch (...) {
        rc = TBS_ERR_NOMEM;
    }
    if (rc) return fail(rc);
    rc = tbs_factor(c, s->algo);
    if (rc) return fail(rc);
    size_t bytes = 0;
    tbs_memory_allocated(c, &bytes);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->sys_bytes + bytes > s->budget) {
        tbs_destroy(c);
        return sfail(s, TBS_ERR_NOMEM, "the system does not fit the server's device budget");
    }
    s->sys_bytes += bytes;
    SrvSystem sys;
    sys.ctx[0] = c;
    sys.bytes = bytes;
    sys.lane = 0;
    for (long long split : s->lane_splits)
        if (nelem >= split) sys.lane += 1;
    s->systems.push_back(sys);
    *system_id = (int)s->systems.size() - 1;
    return TBS_OK;
}

int tbs_server_system_bytes(tbs_server *s, int system_id, int max_sweeps, size_t *resident,
                            size_t *per_rhs) {
    if (!s) return sfail(nullptr, TBS_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (system_id < 0 || system_id >= (int)s->systems.size())
        return sfail(s, TBS_ERR_ARG, "unknown system");
    const SrvSystem &sys = s->systems[system_id];
    tbs_ctx *c = sys.ctx[sys.cur];
    if (resident) tbs_memory_allocated(c, resident);
    if (per_rhs) *per_rhs = slot_bytes(c, s->algo, std::max(max_sweeps, 0) + 1);
    return TBS_OK;
}

int tbs_server_submit(tbs_server *s, int system_id, int nrhs, const double *rhs, double *U_out,
                      double rel_tol, int max_sweeps, const double *jacD, const double *jacO1,
                      const double *jacO2, long long *request_id) {
    if (!s || !request_id) return sfail(s, TBS_ERR_ARG, "null argument");
    if (nrhs < 1 || !rhs || !U_out || max_sweeps < 0 || !(rel_tol >= 0.0))
        return sfail(s, TBS_ERR_ARG, "bad request");
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->stopping) return sfail(s, TBS_ERR_STATE, "server stopping");
    if (system_id < 0 || system_id >= (int)s->systems.size())
        return sfail(s, TBS_ERR_ARG, "unknown system");
    const SrvSystem &sys = s->systems[system_id];
    tbs_ctx *c = sys.ctx[sys.cur];
    if (jacD && (!jacO1 || !jacO2) && c->nintface > 0)
        return sfail(s, TBS_ERR_ARG, "new Jacobian values need jacD, jacO1 and jacO2");
    const size_t per = slot_bytes(c, s->algo, max_sweeps + 1);
    const size_t avail = s->budget > s->sys_bytes ? s->budget - s->sys_bytes : 0;
    if (nrhs > s->max_slots || per * nrhs > avail)
        return sfail(s, TBS_ERR_NOMEM, "the request can never fit the server's budget or slot limit");
    std::unique_ptr<SrvRequest> r;
    try {
        r.reset(new SrvRequest());
        r->sweeps.assign(nrhs, 0);
        r->rel.assign(nrhs, 0.0);
    } catch (...) {
        return sfail(s, TBS_ERR_NOMEM, "host allocation failed");
    }
    r->id = s->next_id++;
    r->sys = system_id;
    r->ctx = c;
    r->nrhs = nrhs;
    r->rhs = rhs;
    r->U = U_out;
    r->tol = rel_tol;
    r->max_sweeps = max_sweeps;
    r->jacD = jacD;
    r->jacO1 = jacO1;
    r->jacO2 = jacO2;
    r->remaining = nrhs;
    r->bytes = per * nrhs;
    r->t_submit = Clock::now();
    SrvRequest *raw = r.get();
    s->requests[raw->id] = std::move(r);
    s->queue.push_back(raw);
    *request_id = raw->id;
    s->cv_loop.notify_all();
    return TBS_OK;
}

int tbs_server_poll(tbs_server *s, long long request_id, int *done) {
    if (!s || !done) return sfail(s, TBS_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) return sfail(s, TBS_ERR_ARG, "unknown request");
    const auto st = it->second->state;
    *done = (st == SrvRequest::DONE || st == SrvRequest::FAILED) ? 1 : 0;
    return TBS_OK;
}

int tbs_server_wait(tbs_server *s, long long request_id, int *sweeps, double *rel_residual,
                    double *latency_ms, double *queue_ms) {
    if (!s) return sfail(nullptr, TBS_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) return sfail(s, TBS_ERR_ARG, "unknown request");
    SrvRequest *r = it->second.get();
    s->cv_done.wait(lk, [&] { return r->state == SrvRequest::DONE || r->state == SrvRequest::FAILED; });
    const int err = r->err;
    const std::string msg = r->msg;
    if (!err) {
        for (int k = 0; k < r->nrhs; ++k) {
            if (sweeps) sweeps[k] = r->sweeps[k];
            if (rel_residual) rel_residual[k] = r->rel[k];
        }
        if (latency_ms) *latency_ms = ms_between(r->t_submit, r->t_done);
        if (queue_ms) *queue_ms = ms_between(r->t_submit, r->t_admit);
    }
    s->requests.erase(it);
    if (err) return sfail(s, err, msg);
    return TBS_OK;
}

int tbs_server_stats(tbs_server *s, long long *stats, int n) {
    if (!s || !stats) return sfail(s, TBS_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    const long long v[] = {s->n_done, s->n_rhs_done, s->n_launches, s->n_refactor, s->peak_rhs,
                           s->peak_bytes, (long long)s->sys_bytes, (long long)s->queue.size(),
                           (long long)s->us_start, (long long)s->us_members, (long long)s->us_run,
                           (long long)s->us_retire};
    for (int k = 0; k < n && k < (int)(sizeof(v) / sizeof(v[0])); ++k) stats[k] = v[k];
    return TBS_OK;
}

}  // extern "C"

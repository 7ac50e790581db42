/*
 * batch.cu -- the batched launch engine (engine.hxx) and the tbs_batch_*
 * entry points: many independent factored systems solved together.
 *
 * Every launch covers the work units of all members still above their
 * tolerance: one persistent Thomas launch over their lines from a device
 * work queue, one persistent residual launch over their tiles and one
 * launch for the per-member norms.  The per-unit arithmetic and the order
 * of every norm sum are those of the single-system sequences in api.cu, so
 * each member's iterates are bit-identical to a tbs_solve of it alone.
 * No counterpart in the reference, whose driver (src/main.cxx) solves one
 * system per process.
 */
#include "engine.hxx"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using namespace tbs;

namespace tbs {

/* ================================================================ helpers */

static int efail(Engine &e, int code, const std::string &msg) {
    e.err = msg;
    set_thread_error(msg);
    return code;
}

#define ECK(call)                                                                         \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return efail(e, TBS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define ECKL(call)                                                                        \
    do {                                                                                  \
        int e_ = (call);                                                                  \
        if (e_ != 0)                                                                      \
            return efail(e, TBS_ERR_CUDA,                                                 \
                         std::string(#call) + ": " + cudaGetErrorString((cudaError_t)e_)); \
    } while (0)

template <typename T>
static int ealloc(Engine &e, T **p, size_t count) {
    void *q = nullptr;
    const size_t nbytes = std::max<size_t>(count, 1) * sizeof(T);
    if (cudaMalloc(&q, nbytes) != cudaSuccess) {
        cudaGetLastError();
        return efail(e, TBS_ERR_NOMEM, "cudaMalloc of " + std::to_string(nbytes) + " bytes failed");
    }
    e.allocs.push_back(q);
    *p = static_cast<T *>(q);
    return TBS_OK;
}

template <typename T>
static void efree(Engine &e, T **p) {
    if (!*p) return;
    auto it = std::find(e.allocs.begin(), e.allocs.end(), (void *)*p);
    if (it != e.allocs.end()) e.allocs.erase(it);
    cudaFree(*p);
    *p = nullptr;
}

/* the capacity-sized arrays are stream-ordered: growing them does not
 * synchronise the device (other engines' graphs keep running) */
template <typename T>
static int ealloc_async(Engine &e, T **p, size_t count) {
    void *q = nullptr;
    const size_t nbytes = std::max<size_t>(count, 1) * sizeof(T);
    if (cudaMallocAsync(&q, nbytes, e.stream) != cudaSuccess) {
        cudaGetLastError();
        return efail(e, TBS_ERR_NOMEM, "cudaMallocAsync of " + std::to_string(nbytes) + " bytes failed");
    }
    e.allocs.push_back(q);
    *p = static_cast<T *>(q);
    return TBS_OK;
}

template <typename T>
static void efree_async(Engine &e, T **p) {
    if (!*p) return;
    auto it = std::find(e.allocs.begin(), e.allocs.end(), (void *)*p);
    if (it != e.allocs.end()) e.allocs.erase(it);
    cudaFreeAsync(*p, e.stream);
    *p = nullptr;
}

template <typename T>
static int eupload(Engine &e, T *dst, const std::vector<T> &h) {
    if (!h.empty())
        ECK(cudaMemcpyAsync(dst, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, e.stream));
    return TBS_OK;
}

/* Uploads through the engine's pinned staging buffer: asynchronous on the
 * engine's stream without a synchronisation; the buffer is reused after
 * the previous batch of uploads has been consumed (stage_ev). */
struct Stager {
    Engine &e;
    size_t used = 0;
    std::vector<std::pair<void *, std::pair<size_t, size_t>>> jobs; /* dst, (offset, bytes) */
    std::vector<char> host;
    explicit Stager(Engine &en) : e(en) {}
    template <typename T>
    void put(T *dst, const std::vector<T> &v) {
        static_assert(sizeof(T) % 4 == 0 && alignof(T) >= 4,
                      "xfer_jobs copies whole, aligned 4-byte words");
        if (v.empty()) return;
        const size_t b = v.size() * sizeof(T);
        const size_t off = host.size();
        const char *src = reinterpret_cast<const char *>(v.data());
        host.insert(host.end(), src, src + b);
        host.resize(off + ((b + 255) & ~(size_t)255));
        jobs.push_back({(void *)dst, {off, b}});
    }
    /* the staged bytes, then the job table, into the pinned buffer; one
     * launch copies every job from it (the SMs read the host memory) */
    int flush() {
        if (jobs.empty()) return TBS_OK;
        if (e.stage_ev) ECK(cudaEventSynchronize(e.stage_ev));
        const size_t table = host.size();
        const size_t need = table + jobs.size() * sizeof(XferJob);
        if (need > e.stage_cap) {
            if (e.h_stage) cudaFreeHost(e.h_stage);
            e.h_stage = nullptr;
            e.stage_cap = 0;
            const size_t cap = need + need / 2;
            if (cudaMallocHost(&e.h_stage, cap) != cudaSuccess)
                return efail(e, TBS_ERR_NOMEM, "pinned staging allocation failed");
            e.stage_cap = cap;
        }
        char *dev = static_cast<char *>(xfer_device_view(e.h_stage));
        if (!dev) return efail(e, TBS_ERR_CUDA, "the staging buffer is not device-addressable");
        std::memcpy(e.h_stage, host.data(), table);
        XferJob *tab = reinterpret_cast<XferJob *>(e.h_stage + table);
        size_t most = 0;
        for (size_t k = 0; k < jobs.size(); ++k) {
            tab[k].dst = (unsigned long long)(uintptr_t)jobs[k].first;
            tab[k].src = (unsigned long long)(uintptr_t)(dev + jobs[k].second.first);
            tab[k].bytes = jobs[k].second.second;
            most = std::max(most, jobs[k].second.second);
        }
        ECKL(xfer_jobs(e.stream, reinterpret_cast<const XferJob *>(dev + table), (int)jobs.size(), most));
        if (!e.stage_ev) ECK(cudaEventCreateWithFlags(&e.stage_ev, cudaEventDisableTiming));
        ECK(cudaEventRecord(e.stage_ev, e.stream));
        return TBS_OK;
    }
};

static cudaEvent_t eprof_event(Engine &e) {
    if (!e.pool.empty()) {
        cudaEvent_t ev = e.pool.back();
        e.pool.pop_back();
        return ev;
    }
    cudaEvent_t ev = nullptr;
    cudaEventCreate(&ev);
    return ev;
}

static void eprof_resolve(Engine &e) {
    if (e.pending.empty()) return;
    cudaStreamSynchronize(e.stream);
    for (auto &p : e.pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess && p.slot >= 0) {
            e.slots[p.slot].ms += ms;
            e.slots[p.slot].launches += 1;
        }
        e.pool.push_back(p.a);
        e.pool.push_back(p.b);
    }
    e.pending.clear();
}

template <typename F>
static int etimed(Engine &e, const char *name, F &&launch) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(e.stream, &cs);
    if (!e.prof || cs != cudaStreamCaptureStatusNone) return launch();
    int slot = -1;
    for (size_t i = 0; i < e.slots.size(); ++i)
        if (std::strcmp(e.slots[i].name, name) == 0) slot = (int)i;
    if (slot < 0 && e.slots.size() < TBS_PROFILE_MAX) {
        e.slots.push_back({name, 0, 0.0});
        slot = (int)e.slots.size() - 1;
    }
    if (e.pending.size() > 4000) eprof_resolve(e);
    PendingEvent pe{slot, eprof_event(e), eprof_event(e)};
    cudaEventRecord(pe.a, e.stream);
    int rc = launch();
    cudaEventRecord(pe.b, e.stream);
    e.pending.push_back(pe);
    return rc;
}

#define ERUN(name, call) ECKL(etimed(e, name, [&]() { return (int)(call); }))

VecSet ctx_vectors(tbs_ctx *c) {
    VecSet v;
    v.Up = c->d_Up;
    v.dUp = c->d_dUp;
    v.b = c->d_b;
    v.y = c->d_y;
    v.rhsp = c->d_rhsp;
    v.rhs = c->d_rhs;
    v.Rp = c->d_Rp;
    v.partials = c->d_partials;
    v.partials2 = c->d_partials2;
    v.Uinit = c->d_Uinit;
    v.state = c->d_state;
    v.hist = c->d_hist;
    v.b32 = c->d_b32;
    v.y32 = c->d_y32;
    v.d32 = c->d_d32;
    v.c32 = c->d_c32;
    v.R32 = c->d_R32;
    return v;
}

/* ================================================================ engine */

int engine_init(Engine &e, int device, cudaStream_t stream, int algo) {
    e.device = device;
    e.stream = stream;
    e.algo = algo;
    int rc = ealloc(e, &e.d_queue, 2);
    if (!rc) rc = ealloc(e, &e.d_counter, 1);
    if (!rc) rc = ealloc(e, &e.d_status, 1);
    if (!rc) rc = ealloc(e, &e.d_ctl, 1);
    if (rc) return rc;
    if (cudaMallocHost(&e.h_ctl, sizeof(BatchCtl)) != cudaSuccess ||
        cudaMallocHost(&e.h_status, sizeof(unsigned)) != cudaSuccess)
        return efail(e, TBS_ERR_NOMEM, "pinned allocation failed");
    std::memset(e.h_ctl, 0, sizeof(BatchCtl));
    if (algo == TBS_ALGO_FP64 && multi_items_prepare() != 0)
        return efail(e, TBS_ERR_CUDA, "shared-memory opt-in failed");
    ECK(cudaMemsetAsync(e.d_queue, 0, 2 * sizeof(unsigned), e.stream));
    ECK(cudaMemsetAsync(e.d_counter, 0, sizeof(unsigned), e.stream));
    ECK(cudaMemsetAsync(e.d_status, 0, sizeof(unsigned), e.stream));
    ECK(cudaMemsetAsync(e.d_ctl, 0, sizeof(BatchCtl), e.stream));
    /* default schedule: 2 stages, as many CTAs per SM as fit, at most 8 */
    const int fit = algo == TBS_ALGO_FP64 ? thomas_batch_fit<double>(2, 1) : thomas_batch_fit<float>(2, 1);
    if (fit < 1) return efail(e, TBS_ERR_CUDA, "the batched Thomas kernel does not fit on an SM");
    e.sched = BatchSched{std::min(fit, 8), 2, 1};
    ECK(cudaStreamSynchronize(e.stream));
    return TBS_OK;
}

void engine_drop_graph(Engine &e) {
    if (e.gexec) cudaGraphExecDestroy(e.gexec);
    if (e.graph) cudaGraphDestroy(e.graph);
    e.gexec = nullptr;
    e.graph = nullptr;
    e.graph_ok = false;
}

void engine_free(Engine &e) {
    if (e.stream) cudaStreamSynchronize(e.stream);
    eprof_resolve(e);
    engine_drop_graph(e);
    for (void *p : e.allocs) cudaFree(p);
    e.allocs.clear();
    for (cudaEvent_t ev : e.pool) cudaEventDestroy(ev);
    e.pool.clear();
    if (e.h_ctl) cudaFreeHost(e.h_ctl);
    if (e.h_status) cudaFreeHost(e.h_status);
    if (e.h_active_pin) cudaFreeHost(e.h_active_pin);
    if (e.h_stage) cudaFreeHost(e.h_stage);
    if (e.stage_ev) cudaEventDestroy(e.stage_ev);
    e.h_ctl = nullptr;
    e.h_status = nullptr;
    e.h_active_pin = nullptr;
    e.h_active_cap = 0;
    e.h_stage = nullptr;
    e.stage_cap = 0;
    e.stage_ev = nullptr;
}

/* grow the capacity-sized arrays (never shrinks); growth invalidates the graph */
static int ensure_capacity(Engine &e, int nmem, int nlines, int nmitems = 0) {
    auto grow = [](int need, int have, int least) {
        return need <= have ? have : std::max({need, 2 * have, least});
    };
    int rc = TBS_OK;
    if (nmem > e.cap_mem) {
        const int c = grow(nmem, e.cap_mem, 64);
        efree_async(e, &e.d_th64);
        efree_async(e, &e.d_th32);
        efree_async(e, &e.d_rs_prime);
        efree_async(e, &e.d_rs_body);
        efree_async(e, &e.d_rs32_rhs);
        efree_async(e, &e.d_rs32_dx);
        efree_async(e, &e.d_fr);
        efree_async(e, &e.d_fp);
        efree_async(e, &e.d_vec);
        efree_async(e, &e.d_red_prime);
        efree_async(e, &e.d_red_body);
        efree_async(e, &e.d_active);
        efree_async(e, &e.d_g_tiles);
        efree_async(e, &e.d_g_prime);
        efree_async(e, &e.d_g_blocks);
        efree_async(e, &e.d_g_chunks);
        efree_async(e, &e.d_g_units);
        efree_async(e, &e.d_g_solo);
        efree_async(e, &e.d_ml);
        if (e.algo == TBS_ALGO_FP64) {
            if (!rc) rc = ealloc_async(e, &e.d_ml, c);
            if (!rc) rc = ealloc_async(e, &e.d_th64, c);
            if (!rc) rc = ealloc_async(e, &e.d_rs_prime, c);
            if (!rc) rc = ealloc_async(e, &e.d_rs_body, c);
        } else {
            if (!rc) rc = ealloc_async(e, &e.d_th32, c);
            if (!rc) rc = ealloc_async(e, &e.d_rs32_rhs, c);
            if (!rc) rc = ealloc_async(e, &e.d_rs32_dx, c);
            if (!rc) rc = ealloc_async(e, &e.d_fr, c);
            if (!rc) rc = ealloc_async(e, &e.d_fp, c);
            if (!rc) rc = ealloc_async(e, &e.d_vec, c);
        }
        if (!rc) rc = ealloc_async(e, &e.d_red_prime, c);
        if (!rc) rc = ealloc_async(e, &e.d_red_body, c);
        if (!rc) rc = ealloc_async(e, &e.d_active, c);
        const size_t gi = group_index_ints(c, c);
        if (!rc) rc = ealloc_async(e, &e.d_g_tiles, gi);
        if (!rc) rc = ealloc_async(e, &e.d_g_prime, gi);
        if (!rc) rc = ealloc_async(e, &e.d_g_blocks, gi);
        if (!rc) rc = ealloc_async(e, &e.d_g_chunks, gi);
        if (!rc) rc = ealloc_async(e, &e.d_g_units, gi);
        if (!rc) rc = ealloc_async(e, &e.d_g_solo, gi);
        e.cap_mem = rc ? 0 : c;
        engine_drop_graph(e);
    }
    if (!rc && nlines > e.cap_lines) {
        const int c = grow(nlines, e.cap_lines, 1 << 16);
        efree_async(e, &e.d_lines);
        rc = ealloc_async(e, &e.d_lines, c);
        e.cap_lines = rc ? 0 : c;
        engine_drop_graph(e);
    }
    /* the multi-RHS line solves launch one CTA per item up to capacity (the
     * graph holds the grid), so the capacity starts small */
    if (!rc && e.algo == TBS_ALGO_FP64 && (nmitems > e.cap_mitems || !e.d_mitems)) {
        const int c = grow(std::max(nmitems, 1), e.cap_mitems, 1024);
        efree_async(e, &e.d_mitems);
        rc = ealloc_async(e, &e.d_mitems, c);
        e.cap_mitems = rc ? 0 : c;
        engine_drop_graph(e);
    }
    return rc;
}

/* members grouped by system, in order of first appearance */
static std::vector<std::vector<int>> group_members(const std::vector<Member> &m,
                                                   const std::vector<char> &take) {
    std::vector<std::vector<int>> g;
    std::vector<const tbs_ctx *> key;
    for (size_t k = 0; k < m.size(); ++k) {
        if (!take[k]) continue;
        size_t j = 0;
        while (j < key.size() && key[j] != m[k].sys) ++j;
        if (j == key.size()) {
            key.push_back(m[k].sys);
            g.emplace_back();
        }
        g[j].push_back((int)k);
    }
    return g;
}

/* host image of a group index (layout in tbs_internal.hxx); per_member:
 * a group's items are its units times its members (an item is one member's
 * unit), else its units (an item is a unit of every member) */
static std::vector<int> group_index(const std::vector<std::vector<int>> &g,
                                    const std::vector<int> &units_per_group, bool per_member = true) {
    const int ng = (int)g.size();
    std::vector<int> v;
    v.push_back(ng);
    long long base = 0;
    for (int j = 0; j < ng; ++j) {
        v.push_back((int)base);
        base += (long long)units_per_group[j] * (per_member ? (long long)g[j].size() : 1LL);
    }
    v.push_back((int)base);
    for (int j = 0; j < ng; ++j) v.push_back((int)g[j].size());
    int off = 0;
    for (int j = 0; j < ng; ++j) {
        v.push_back(off);
        off += (int)g[j].size();
    }
    for (int j = 0; j < ng; ++j)
        for (int k : g[j]) v.push_back(k);
    return v;
}

/* Thomas items in the engine's order.  Longest lines first; the items of
 * one line of one system (several right-hand sides) are adjacent, so that
 * the warps running them together share the line's blocks in L2. */
/* the members whose lines the batched line solve runs: all of them, but
 * for FP64 the members of a system with several members, whose line
 * solves run together (multi_items) */
static std::vector<char> thomas_take(const Engine &e, const std::vector<Member> &m) {
    std::vector<char> take(m.size(), 1);
    if (e.algo != TBS_ALGO_FP64) return take;
    std::vector<char> all(m.size(), 1);
    for (const auto &grp : group_members(m, all))
        if (grp.size() > 1)
            for (int k : grp) take[k] = 0;
    return take;
}

static std::vector<WorkItem> line_items(const Engine &e, const std::vector<Member> &m) {
    const std::vector<char> all = thomas_take(e, m);
    const std::vector<std::vector<int>> g = group_members(m, all);
    struct GL {
        int len, group, line;
    };
    std::vector<GL> gl;
    for (size_t j = 0; j < g.size(); ++j) {
        const tbs_ctx *c = m[g[j][0]].sys;
        for (int l = 0; l < c->nline; ++l) gl.push_back({c->h_linesize[l], (int)j, l});
    }
    if (e.order == 0)
        std::stable_sort(gl.begin(), gl.end(), [](const GL &a, const GL &b) { return a.len > b.len; });
    std::vector<WorkItem> items;
    if (e.order == 0) {
        for (const GL &x : gl)
            for (int k : g[x.group]) items.push_back({k, x.line});
    } else {
        for (size_t k = 0; k < m.size(); ++k)
            if (all[k])
                for (int l = 0; l < m[k].sys->nline; ++l) items.push_back({(int)k, l});
    }
    return items;
}

/* FP64: the line solves of the members of a system with several members,
 * up to MULTI_MAX of them per CTA (their lines' blocks read once): one
 * MultiLine per such group of members, and its (group, line) items,
 * longest lines first */
static void multi_items(const std::vector<Member> &m, std::vector<MultiLine> &sys,
                        std::vector<WorkItem> &items) {
    sys.clear();
    items.clear();
    std::vector<char> all(m.size(), 1);
    struct GL {
        int len, grp, line;
    };
    std::vector<GL> gl;
    for (const auto &grp : group_members(m, all)) {
        if (grp.size() < 2) continue;
        for (size_t k0 = 0; k0 < grp.size(); k0 += MULTI_MAX) {
            const tbs_ctx *c = m[grp[k0]].sys;
            MultiLine L{};
            L.line_start = c->L.line_start;
            L.line_len = c->L.line_len;
            L.line_twist = c->L.line_twist;
            L.G = c->d_G;
            L.Gam = c->d_Gam;
            L.nr = (int)std::min<size_t>(MULTI_MAX, grp.size() - k0);
            for (int r = 0; r < MULTI_MAX; ++r) {
                const int k = grp[k0 + (r < L.nr ? r : 0)];
                L.aid[r] = k;
                L.b[r] = m[k].v.b;
                L.y[r] = m[k].v.y;
                L.dU[r] = m[k].v.dUp;
            }
            const int gi = (int)sys.size();
            sys.push_back(L);
            for (int l = 0; l < c->nline; ++l) gl.push_back({c->h_linesize[l], gi, l});
        }
    }
    std::stable_sort(gl.begin(), gl.end(), [](const GL &a, const GL &b) { return a.len > b.len; });
    for (const GL &x : gl) items.push_back({x.grp, x.line});
}

int engine_set_members(Engine &e, const std::vector<Member> &members) {
    const int n = (int)members.size();
    const bool mixed = e.algo == TBS_ALGO_MIXED;
    int nx = e.max_nx;
    long long nlines = 0, ntiles = 0, nblocks = 0;
    for (const Member &m : members) {
        nx = std::max(nx, m.sys->L.nx);
        nlines += m.sys->nline;
        ntiles += fast_resid_grid(m.sys->L.np16);
        if (mixed) nblocks += full_resid_blocks(m.sys->nelem);
    }
    if (nlines > 0x7fffffff || ntiles > 0x7fffffff || nblocks > 0x7fffffff)
        return efail(e, TBS_ERR_UNSUPPORTED, "batch too large for int32 work indices");
    if (nx > e.max_nx) {
        if (batch_prepare(nx)) return efail(e, TBS_ERR_CUDA, "shared-memory opt-in failed");
        e.max_nx = nx;
        engine_drop_graph(e);
    }
    std::vector<MultiLine> mls;
    std::vector<WorkItem> mitems;
    if (!mixed) multi_items(members, mls, mitems);
    int rc = ensure_capacity(e, std::max(n, 1), (int)std::max(nlines, 1LL), (int)mitems.size());
    if (rc) return rc;

    std::vector<ThomasSys<double>> th64;
    std::vector<ThomasSys<float>> th32;
    std::vector<ResidSys<double>> rsp, rsb;
    std::vector<ResidSys<float>> rs32r, rs32d;
    std::vector<FullResSys> fr;
    std::vector<FullPosSys> fp;
    std::vector<VecSys> vec;
    bool fullpos = mixed;
    int max_nxf = 0;
    for (const Member &m : members) {
        fullpos = fullpos && fullpos_ok(m.sys) && m.sys->d_Dp;
        max_nxf = std::max(max_nxf, m.sys->L.nxf);
    }
    std::vector<ReduceSys> redp, redb;
    std::vector<int> uinit;
    std::vector<char> all(n, 1), prime(n, 0);
    e.h_active.assign(n, 0);
    for (int k = 0; k < n; ++k) {
        const Member &m = members[k];
        tbs_ctx *c = m.sys;
        const VecSet &v = m.v;
        const FastLayout &L = c->L;
        const int nt = fast_resid_grid(L.np16);
        const bool ui = m.fresh && v.Uinit;
        if (!mixed) {
            th64.push_back({L.line_start, L.line_len, L.line_twist, c->d_G, c->d_Gam, v.b, v.y, v.dUp});
            /* prime: R = rhs (U = 0, cleared by the same launch) or the residual of U_init */
            rsp.push_back({L.np16, L.nx, L.xnbr, c->d_Dinv, c->d_X, v.dUp, ui ? v.Rp : v.rhsp, v.b,
                           ui ? nullptr : v.Up, v.partials});
            rsb.push_back({L.np16, L.nx, L.xnbr, c->d_Dinv, c->d_X, v.dUp, nullptr, v.b, v.Up,
                           v.partials});
            if (m.fresh) redp.push_back({v.partials, nt, k, v.state, v.hist});
            redb.push_back({v.partials, nt, k, v.state, v.hist});
        } else {
            th32.push_back({L.line_start, L.line_len, L.line_twist, c->d_G32, c->d_Gam32, v.b32, v.y32,
                            v.d32});
            rs32r.push_back({L.np16, L.nx, L.xnbr, c->d_Dinv32, c->d_X32, v.d32, v.R32, v.b32, v.c32,
                             nullptr});
            rs32d.push_back({L.np16, L.nx, L.xnbr, nullptr, c->d_X32, v.d32, nullptr, v.b32, v.c32,
                             nullptr});
            fr.push_back({c->nelem, 0, c->d_epoint, c->d_ef, c->d_fc, L.pos_of_elem, c->d_jacD, c->d_O1,
                          c->d_O2, v.rhs, v.Up, v.R32, v.partials});
            fp.push_back({L.np16, L.nxf, L.xnbrf, c->d_Dp, c->d_XF, v.rhsp, v.Up, v.R32, v.partials,
                          c->d_Dinv32, v.b32, v.c32});
            vec.push_back({v.rhsp, v.R32, v.c32, v.d32, v.Up, v.partials, c->d_Dinv32, v.b32});
            if (m.fresh) redp.push_back({v.partials, ui ? full_resid_blocks(c->nelem) : nt, k, v.state, v.hist});
            redb.push_back({v.partials, fullpos ? nt : full_resid_blocks(c->nelem), k, v.state, v.hist});
        }
        prime[k] = m.fresh && !(mixed && ui);
        if (ui) uinit.push_back(k);
        e.h_active[k] = m.fresh ? 0 : 1;
    }
    if (uinit != e.uinit || fullpos != e.fullpos || max_nxf > e.max_nxf) {
        e.uinit = uinit;
        e.fullpos = fullpos;
        e.max_nxf = std::max(e.max_nxf, max_nxf);
        engine_drop_graph(e);
    }
    /* group indices of the residual-type launches */
    /* units: 0 residual tiles, 1 element blocks, 2 chunks of BATCH_CHUNK tiles */
    auto units = [&](const std::vector<std::vector<int>> &g, int kind) {
        std::vector<int> u;
        for (const auto &grp : g) {
            const tbs_ctx *c = members[grp[0]].sys;
            const int nt = fast_resid_grid(c->L.np16);
            u.push_back(kind == 1 ? full_resid_blocks(c->nelem) : kind == 2 ? batch_chunks(nt) : nt);
        }
        return u;
    };
    const auto g_all = group_members(members, all);
    const auto g_prime = group_members(members, prime);
    const std::vector<int> gi_tiles = group_index(g_all, units(g_all, 0));
    const std::vector<int> gi_prime = group_index(g_prime, units(g_prime, 0));
    e.members = members;
    std::vector<WorkItem> lines = line_items(e, members);
    Stager up(e);
    if (!mixed) {
        up.put(e.d_th64, th64);
        up.put(e.d_ml, mls);
        up.put(e.d_mitems, mitems);
        up.put(e.d_rs_prime, rsp);
        up.put(e.d_rs_body, rsb);
    } else {
        up.put(e.d_th32, th32);
        up.put(e.d_rs32_rhs, rs32r);
        up.put(e.d_rs32_dx, rs32d);
        up.put(e.d_fr, fr);
        up.put(e.d_fp, fp);
        up.put(e.d_vec, vec);
        up.put(e.d_g_blocks, group_index(g_all, units(g_all, 1)));
    }
    up.put(e.d_red_prime, redp);
    up.put(e.d_red_body, redb);
    up.put(e.d_lines, lines);
    up.put(e.d_g_tiles, gi_tiles);
    up.put(e.d_g_chunks, group_index(g_all, units(g_all, 2)));
    {
        /* the sweep residual: members alone in their system run per member,
         * several members of one system together over one staging of its
         * blocks per tile */
        std::vector<std::vector<int>> g_solo, g_multi;
        for (const auto &grp : g_all) (grp.size() > 1 ? g_multi : g_solo).push_back(grp);
        up.put(e.d_g_solo, group_index(g_solo, units(g_solo, 2)));
        up.put(e.d_g_units, group_index(g_multi, units(g_multi, 2), false));
    }
    up.put(e.d_g_prime, gi_prime);
    up.put(e.d_active, e.h_active);
    rc = up.flush();
    if (rc) return rc;
    BatchCtl &C = *e.h_ctl;
    C.nsys = n;
    C.nlines = (int)lines.size();
    C.nmitems = (int)mitems.size();
    C.ntiles = gi_tiles[1 + gi_tiles[0]];
    C.nblocks = (int)nblocks;
    C.nprime_sys = (int)redp.size();
    C.nprime_tiles = gi_prime[1 + gi_prime[0]];
    return TBS_OK;
}

int engine_restart(Engine &e) {
    bool all_fresh = true;
    for (const Member &m : e.members) all_fresh = all_fresh && m.fresh;
    if (!all_fresh) {
        std::vector<Member> m = e.members;
        for (Member &x : m) x.fresh = true;
        return engine_set_members(e, m);
    }
    std::fill(e.h_active.begin(), e.h_active.end(), 0);
    Stager up(e);
    up.put(e.d_active, e.h_active);
    return up.flush();
}

void engine_mark_started(Engine &e) {
    for (Member &m : e.members) m.fresh = false;
    e.h_ctl->nprime_sys = 0;
    e.h_ctl->nprime_tiles = 0;
    /* an empty prime group index (the count is read from it on the device) */
    Stager up(e);
    up.put(e.d_g_prime, std::vector<int>{0, 0});
    up.flush();
}

struct Cond {
    unsigned long long handle;
    int use;
    unsigned long long handle2; /* a second condition set to the same value (0: none) */
    int use2;
};

static int engine_prime(Engine &e, Cond cc) {
    cudaStream_t st = e.stream;
    for (int k : e.uinit) {
        const Member &m = e.members[k];
        tbs_ctx *c = m.sys;
        const VecSet &v = m.v;
        const FastLayout &L = c->L;
        ERUN("permute", launch_permute_to_pos(st, 9, c->nelem, L.pos_of_elem, v.Uinit, v.Up));
        if (e.algo == TBS_ALGO_FP64)
            ERUN("full_resid", launch_full_resid<double>(st, c->nelem, c->d_epoint, c->d_ef, c->d_fc,
                                                         L.pos_of_elem, c->d_jacD, c->d_O1, c->d_O2,
                                                         v.rhs, v.Up, v.Rp, v.partials2));
        else {
            ERUN("full_resid", launch_full_resid<float>(st, c->nelem, c->d_epoint, c->d_ef, c->d_fc,
                                                        L.pos_of_elem, c->d_jacD, c->d_O1, c->d_O2,
                                                        v.rhs, v.Up, v.R32, v.partials));
            /* the first inner right-hand side, as the single-system prime */
            ERUN("fast_resid32_rhs", launch_fast_resid<float>(st, L, 0, c->d_Dinv32, c->d_X32, v.d32,
                                                              v.R32, v.b32, NormSink{}, e.d_status, v.c32));
        }
    }
    BatchCtl *C = e.d_ctl;
    if (e.algo == TBS_ALGO_FP64) {
        ERUN("fast_resid_rhs", launch_resid_batch<double>(st, 0, e.max_nx, e.d_rs_prime, e.d_g_prime, 1,
                                                          nullptr, e.d_status));
        ERUN("reduce_norm", launch_reduce_batch(st, 160, e.d_red_prime, &C->nprime_sys, e.cap_mem, 1,
                                                e.d_active, C, e.d_counter, cc.handle, cc.use,
                                                cc.handle2, cc.use2));
    } else {
        ERUN("mixed_prime", launch_mixed_prime_batch(st, e.d_vec, e.d_g_prime));
        ERUN("reduce_norm", launch_reduce_batch(st, 1024, e.d_red_prime, &C->nprime_sys, e.cap_mem, 1,
                                                e.d_active, C, e.d_counter, cc.handle, cc.use,
                                                cc.handle2, cc.use2));
    }
    return TBS_OK;
}

static int engine_body(Engine &e, Cond cc, int inner) {
    cudaStream_t st = e.stream;
    BatchCtl *C = e.d_ctl;
    if (e.algo == TBS_ALGO_FP64) {
        ERUN("fast_thomas", launch_thomas_batch<double>(st, e.sched, e.d_th64, e.d_lines, &C->nlines,
                                                        e.d_active, e.d_queue, e.d_status));
        /* the line solves of several members of one system: their blocks
         * read once per line for up to MULTI_MAX of them */
        ERUN("multi_thomas", launch_multi_thomas_items(st, e.cap_mitems, e.d_ml, e.d_mitems, &C->nmitems,
                                                       e.d_active, e.d_status));
        ERUN("fast_resid", launch_resid_batch<double>(st, 1, e.max_nx, e.d_rs_body, e.d_g_solo,
                                                      BATCH_CHUNK, e.d_active, e.d_status));
        ERUN("fast_resid_group", launch_resid_group<double>(st, e.max_nx, e.d_rs_body, e.d_g_units,
                                                            BATCH_CHUNK, e.d_active, e.d_status));
        ERUN("reduce_norm", launch_reduce_batch(st, 160, e.d_red_body, &C->nsys, e.cap_mem, 0,
                                                e.d_active, C, e.d_counter, cc.handle, cc.use));
        return TBS_OK;
    }
    /* c (the sum of the inner updates but the last) is cleared by the first
     * launch, each inner residual adds its sweep's d to it, and the last d
     * goes to U with c (the order of the single-system sequence) */
    if (!e.fullpos)
        ERUN("fast_resid32_rhs", launch_resid_batch<float>(st, 0, e.max_nx, e.d_rs32_rhs, e.d_g_tiles, 1,
                                                           e.d_active, e.d_status));
    for (int m = 0; m < inner; ++m) {
        ERUN("fast_thomas32", launch_thomas_batch<float>(st, e.sched, e.d_th32, e.d_lines, &C->nlines,
                                                         e.d_active, e.d_queue, e.d_status));
        if (m + 1 < inner)
            ERUN("fast_resid32", launch_resid_batch<float>(st, 3, e.max_nx, e.d_rs32_dx, e.d_g_tiles, 1,
                                                           e.d_active, e.d_status));
    }
    ERUN("axpy", launch_axpy2_batch(st, e.d_vec, e.d_g_tiles, e.d_active));
    if (e.fullpos)
        ERUN("full_resid", launch_full_resid_pos_batch(st, e.max_nxf, e.d_fp, e.d_g_chunks, BATCH_CHUNK,
                                                       e.d_active, e.d_status));
    else
        ERUN("full_resid", launch_full_resid_batch(st, e.d_fr, e.d_g_blocks, e.d_active));
    ERUN("reduce_norm", launch_reduce_batch(st, 1024, e.d_red_body, &C->nsys, e.cap_mem, 0, e.d_active,
                                            C, e.d_counter, cc.handle, cc.use));
    return TBS_OK;
}

/* capture `fn` into a conditional node's body graph */
template <typename F>
static int engine_capture_into(Engine &e, cudaGraph_t g, F &&fn) {
    ECK(cudaStreamBeginCaptureToGraph(e.stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int rc = fn();
    cudaGraph_t outg = nullptr;
    cudaError_t ee = cudaStreamEndCapture(e.stream, &outg);
    if (rc == TBS_OK && ee != cudaSuccess)
        rc = efail(e, TBS_ERR_CUDA, std::string("end body capture: ") + cudaGetErrorString(ee));
    return rc;
}

static int engine_add_conditional(Engine &e, cudaGraph_t g, cudaGraphConditionalHandle h,
                                  cudaGraphConditionalNodeType type, cudaGraph_t *body_out) {
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaError_t x = cudaStreamGetCaptureInfo(e.stream, &cs, nullptr, nullptr, &deps, &ndeps);
    if (x != cudaSuccess) return efail(e, TBS_ERR_CUDA, std::string("capture info: ") + cudaGetErrorString(x));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    x = cudaGraphAddNode(&node, g, deps, ndeps, &cp);
    if (x != cudaSuccess) return efail(e, TBS_ERR_CUDA, std::string("conditional node: ") + cudaGetErrorString(x));
    *body_out = cp.conditional.phGraph_out[0];
    x = cudaStreamUpdateCaptureDependencies(e.stream, &node, 1, cudaStreamSetCaptureDependencies);
    if (x != cudaSuccess) return efail(e, TBS_ERR_CUDA, std::string("capture deps: ") + cudaGetErrorString(x));
    return TBS_OK;
}

/* prime -> while (rule) { sweep }; MIXED with its own inner count for the
 * first outer step (all members start together, as in tbs_batch):
 * prime -> if (rule) { first step } -> while (rule) { step } */
static bool engine_sched(const Engine &e) {
    return e.algo == TBS_ALGO_MIXED && e.inner_first > 0 && e.inner_first != e.inner;
}

static int engine_build_graph(Engine &e) {
    engine_drop_graph(e);
    cudaGraph_t g = nullptr;
    ECK(cudaGraphCreate(&g, 0));
    e.graph = g;
    const bool sched = engine_sched(e);
    cudaGraphConditionalHandle hw, hf = 0;
    ECK(cudaGraphConditionalHandleCreate(&hw, g, 0, cudaGraphCondAssignDefault));
    if (sched) ECK(cudaGraphConditionalHandleCreate(&hf, g, 0, cudaGraphCondAssignDefault));
    const Cond loop{(unsigned long long)hw, 1, 0, 0};
    const Cond both{(unsigned long long)hw, 1, (unsigned long long)hf, sched ? 1 : 0};
    ECK(cudaStreamBeginCaptureToGraph(e.stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int rc = engine_prime(e, both);
    cudaGraph_t firstg = nullptr, bodyg = nullptr;
    if (rc == TBS_OK && sched) rc = engine_add_conditional(e, g, hf, cudaGraphCondTypeIf, &firstg);
    if (rc == TBS_OK) rc = engine_add_conditional(e, g, hw, cudaGraphCondTypeWhile, &bodyg);
    cudaGraph_t outg = nullptr;
    cudaError_t ee = cudaStreamEndCapture(e.stream, &outg);
    if (rc == TBS_OK && ee != cudaSuccess) rc = efail(e, TBS_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ee));
    if (rc == TBS_OK && sched)
        rc = engine_capture_into(e, firstg, [&]() { return engine_body(e, loop, e.inner_first); });
    if (rc == TBS_OK) rc = engine_capture_into(e, bodyg, [&]() { return engine_body(e, loop, e.inner); });
    if (rc != TBS_OK) {
        engine_drop_graph(e);
        return rc;
    }
    cudaError_t ie = cudaGraphInstantiate(&e.gexec, g, 0);
    if (ie != cudaSuccess) {
        engine_drop_graph(e);
        return efail(e, TBS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    }
    e.graph_ok = true;
    return TBS_OK;
}

static int engine_status(Engine &e) {
    ECKL(xfer_to_host(e.stream, e.h_status, e.d_status, sizeof(unsigned), 1));
    ECK(cudaStreamSynchronize(e.stream));
    const unsigned s = *e.h_status;
    if (s) {
        ECK(cudaMemsetAsync(e.d_status, 0, sizeof(unsigned), e.stream));
        ECK(cudaMemsetAsync(e.d_queue, 0, 2 * sizeof(unsigned), e.stream));
        ECK(cudaMemsetAsync(e.d_counter, 0, sizeof(unsigned), e.stream));
        ECK(cudaStreamSynchronize(e.stream));
        if (s & ST_TIMEOUT) return efail(e, TBS_ERR_CUDA, "a device-side wait ran out of its time budget");
        return efail(e, TBS_ERR_CUDA, "device status " + std::to_string(s));
    }
    return TBS_OK;
}

int engine_read_active(Engine &e) {
    const int n = e.h_ctl->nsys;
    e.h_active.resize(n);
    if (n > e.h_active_cap) {
        if (e.h_active_pin) cudaFreeHost(e.h_active_pin);
        e.h_active_pin = nullptr;
        e.h_active_cap = 0;
        const int cap = std::max(n, 256);
        if (cudaMallocHost(&e.h_active_pin, cap * sizeof(int)) != cudaSuccess)
            return efail(e, TBS_ERR_NOMEM, "pinned allocation failed");
        e.h_active_cap = cap;
    }
    if (n > 0) ECKL(xfer_to_host(e.stream, e.h_active_pin, e.d_active, n * sizeof(int), 1));
    ECK(cudaStreamSynchronize(e.stream));
    if (n > 0) std::memcpy(e.h_active.data(), e.h_active_pin, n * sizeof(int));
    return TBS_OK;
}

int engine_run(Engine &e, int chunk_limit, int stop_on_finish) {
    BatchCtl &C = *e.h_ctl;
    C.chunk = 0;
    C.finished = 0;
    C.chunk_limit = chunk_limit;
    C.stop_on_finish = stop_on_finish;
    ECKL(xfer_put(e.stream, e.d_ctl, e.h_ctl, sizeof(BatchCtl)));
    if (e.prof) {
        /* eager form with the graph's loop rule tested on the host, so
         * that every kernel is timed */
        int rc = engine_prime(e, Cond{});
        if (rc) return rc;
        BatchCtl now{};
        for (int step = 0;; ++step) {
            ECK(cudaMemcpyAsync(&now, e.d_ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, e.stream));
            rc = engine_read_active(e);
            if (rc) return rc;
            bool any = false;
            for (int v : e.h_active) any = any || v;
            bool go = any;
            if (chunk_limit > 0 && now.chunk >= chunk_limit) go = false;
            if (stop_on_finish && now.finished) go = false;
            if (!go) break;
            rc = engine_body(e, Cond{}, (step == 0 && engine_sched(e)) ? e.inner_first : e.inner);
            if (rc) return rc;
        }
        eprof_resolve(e);
    } else {
        if (!e.graph_ok) {
            int rc = engine_build_graph(e);
            if (rc) return rc;
        }
        ECK(cudaGraphLaunch(e.gexec, e.stream));
    }
    return engine_status(e);
}

int engine_launch(Engine &e, int chunk_limit, int stop_on_finish) {
    if (e.prof) return engine_run(e, chunk_limit, stop_on_finish);
    BatchCtl &C = *e.h_ctl;
    C.chunk = 0;
    C.finished = 0;
    C.chunk_limit = chunk_limit;
    C.stop_on_finish = stop_on_finish;
    ECKL(xfer_put(e.stream, e.d_ctl, e.h_ctl, sizeof(BatchCtl)));
    if (!e.graph_ok) {
        int rc = engine_build_graph(e);
        if (rc) return rc;
    }
    ECK(cudaGraphLaunch(e.gexec, e.stream));
    return TBS_OK;
}

int engine_finish(Engine &e) { return engine_status(e); }

static int engine_upload_lines(Engine &e) {
    std::vector<WorkItem> lines = line_items(e, e.members);
    int rc = eupload(e, e.d_lines, lines);
    if (rc) return rc;
    ECK(cudaStreamSynchronize(e.stream));
    return TBS_OK;
}

int engine_set_schedule(Engine &e, BatchSched s, int order) {
    if (s.warps != 1 && s.warps != 2) return efail(e, TBS_ERR_ARG, "warps per line must be 1 or 2");
    if (s.stages < 2 || s.stages > 8) return efail(e, TBS_ERR_ARG, "stages must be in 2..8");
    const int fit = e.algo == TBS_ALGO_FP64 ? thomas_batch_fit<double>(s.stages, s.warps)
                                            : thomas_batch_fit<float>(s.stages, s.warps);
    if (s.ctas_per_sm < 1 || s.ctas_per_sm > fit)
        return efail(e, TBS_ERR_ARG, "schedule does not fit: at most " + std::to_string(fit) +
                                         " CTAs per SM with " + std::to_string(s.stages) +
                                         " stages and " + std::to_string(s.warps) + " warp(s) per line");
    const bool new_order = order != e.order;
    e.sched = s;
    e.order = order;
    engine_drop_graph(e);
    if (new_order && !e.members.empty()) return engine_upload_lines(e);
    return TBS_OK;
}

int engine_tune(Engine &e, BatchSched *best_s, int *best_o, double *best_ms) {
    cudaStream_t st = e.stream;
    const int n = e.h_ctl->nsys;
    if (n < 1) return efail(e, TBS_ERR_STATE, "no members to tune on");
    std::vector<int> ones(n, 1);
    int rc = eupload(e, e.d_active, ones);
    if (rc) return rc;
    ECK(cudaMemcpyAsync(e.d_ctl, e.h_ctl, sizeof(BatchCtl), cudaMemcpyHostToDevice, st));
    cudaEvent_t e0, e1;
    ECK(cudaEventCreate(&e0));
    ECK(cudaEventCreate(&e1));
    const BatchSched keep = e.sched;
    const int keep_order = e.order;
    double best = 1e30;
    BatchSched bs = keep;
    int bo = keep_order;
    const int cand_ctas[] = {2, 3, 4, 6, 8, 12, 16};
    for (int o = 0; o < 2 && !rc; ++o) {
        e.order = o;
        rc = engine_upload_lines(e);
        for (int wpl = 1; wpl <= 2 && !rc; ++wpl)
        for (int ns = 2; ns <= 4 && !rc; ++ns) {
            const int fit = e.algo == TBS_ALGO_FP64 ? thomas_batch_fit<double>(ns, wpl)
                                                    : thomas_batch_fit<float>(ns, wpl);
            for (int cps : cand_ctas) {
                if (cps > fit || rc) continue;
                e.sched = BatchSched{cps, ns, wpl};
                auto launch = [&]() {
                    return e.algo == TBS_ALGO_FP64
                               ? launch_thomas_batch<double>(st, e.sched, e.d_th64, e.d_lines,
                                                             &e.d_ctl->nlines, e.d_active, e.d_queue,
                                                             e.d_status)
                               : launch_thomas_batch<float>(st, e.sched, e.d_th32, e.d_lines,
                                                            &e.d_ctl->nlines, e.d_active, e.d_queue,
                                                            e.d_status);
                };
                int x = launch();
                const int reps = 3;
                if (!x) cudaEventRecord(e0, st);
                for (int r = 0; r < reps && !x; ++r) x = launch();
                if (!x) cudaEventRecord(e1, st);
                if (x) {
                    rc = efail(e, TBS_ERR_CUDA,
                               std::string("tuning launch: ") + cudaGetErrorString((cudaError_t)x));
                    break;
                }
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                rc = engine_status(e);
                if (rc) break;
                if (ms / reps < best) {
                    best = ms / reps;
                    bs = e.sched;
                    bo = o;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    e.sched = rc ? keep : bs;
    e.order = rc ? keep_order : bo;
    engine_drop_graph(e);
    int rc2 = engine_upload_lines(e);
    if (rc) return rc;
    if (rc2) return rc2;
    if (best_s) *best_s = bs;
    if (best_o) *best_o = bo;
    if (best_ms) *best_ms = best;
    return TBS_OK;
}

}  // namespace tbs

/* ============================================================= tbs_batch */

struct tbs_batch {
    Engine eng;
    cudaStream_t own = nullptr;
    std::vector<tbs_ctx *> sys;
    std::vector<const void *> fingerprint;
};

static int bfail(tbs_batch *b, int code, const std::string &msg) {
    if (b) b->eng.err = msg;
    set_thread_error(msg);
    return code;
}

/* every device pointer and setting the members' descriptors depend on */
static std::vector<const void *> batch_fingerprint(tbs_batch *b) {
    std::vector<const void *> f;
    for (tbs_ctx *c : b->sys) {
        const void *p[] = {c->d_G, c->d_Gam, c->d_Dinv, c->d_X, c->d_b, c->d_y, c->d_dUp, c->d_Up,
                           c->d_rhsp, c->d_Rp, c->d_partials, c->d_partials2, c->d_state, c->d_hist,
                           c->d_Uinit, c->d_G32, c->d_Gam32, c->d_Dinv32, c->d_X32, c->d_b32,
                           c->d_y32, c->d_d32, c->d_c32, c->d_R32, c->L.line_start, c->L.xnbr,
                           c->d_jacD, c->d_O1, c->d_O2, c->d_rhs, c->d_epoint};
        f.insert(f.end(), std::begin(p), std::end(p));
        f.push_back(reinterpret_cast<const void *>((uintptr_t)c->algo));
    }
    return f;
}

static int batch_check_members(tbs_batch *b) {
    for (size_t s = 0; s < b->sys.size(); ++s) {
        tbs_ctx *c = b->sys[s];
        if (!c->factored || !c->layout_ok)
            return bfail(b, TBS_ERR_STATE, "batch member " + std::to_string(s) + " is not factored");
        if (c->nhalo > 0)
            return bfail(b, TBS_ERR_UNSUPPORTED,
                         "batch member " + std::to_string(s) + " is a line partition of a larger mesh");
        if (c->algo != b->eng.algo)
            return bfail(b, TBS_ERR_STATE,
                         "batch member " + std::to_string(s) + " was re-factored with another algorithm");
        if (c->lagged && c->algo == TBS_ALGO_FP64)
            return bfail(b, TBS_ERR_UNSUPPORTED,
                         "batch member " + std::to_string(s) +
                             " has block values newer than its FP64 factorization (tbs_update_values); "
                             "the batch tracks the residual with the factorization's blocks: re-factor "
                             "it or solve it with tbs_solve");
    }
    return TBS_OK;
}

/* members' device state (tolerance, sweep limit, history capacity) and the
 * engine's descriptors, rebuilt when a member's arrays changed */
static int batch_ready(tbs_batch *b, double tol, int max_sweeps) {
    int rc = batch_check_members(b);
    if (rc) return rc;
    for (tbs_ctx *c : b->sys) {
        if (cudaStreamSynchronize(c->stream) != cudaSuccess)
            return bfail(b, TBS_ERR_CUDA, "member stream synchronisation failed");
        rc = ctx_ensure_hist(c, max_sweeps + 1);
        if (!rc) rc = ctx_set_state(c, tol, max_sweeps);
        if (rc) return bfail(b, rc, "batch member: " + c->err);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess)
            return bfail(b, TBS_ERR_CUDA, "member stream synchronisation failed");
    }
    std::vector<const void *> fp = batch_fingerprint(b);
    if (fp != b->fingerprint) {
        std::vector<Member> m;
        for (tbs_ctx *c : b->sys) m.push_back({c, ctx_vectors(c), true});
        rc = engine_set_members(b->eng, m);
        if (rc) return rc;
        b->fingerprint = fp;
        return TBS_OK;
    }
    return engine_restart(b->eng);
}

static int batch_destroy_all(tbs_batch *b) {
    if (!b) return TBS_OK;
    cudaSetDevice(b->eng.device);
    engine_free(b->eng);
    if (b->own) cudaStreamDestroy(b->own);
    delete b;
    return TBS_OK;
}

#define BGUARD_BEGIN try {
#define BGUARD_END                                                                        \
    }                                                                                     \
    catch (const std::bad_alloc &) {                                                      \
        return bfail(b, TBS_ERR_NOMEM, "host allocation failed");                         \
    }                                                                                     \
    catch (...) {                                                                         \
        return bfail(b, TBS_ERR_STATE, "internal error");                                 \
    }

extern "C" {

const char *tbs_batch_last_error(const tbs_batch *b) {
    if (!b) return thread_error();
    return b->eng.err.c_str();
}

int tbs_batch_create(tbs_ctx *const *systems, int nsys, tbs_batch **out) {
    if (!out || !systems || nsys < 1) return bfail(nullptr, TBS_ERR_ARG, "tbs_batch_create: bad arguments");
    *out = nullptr;
    tbs_batch *b = nullptr;
    try {
        b = new tbs_batch();
    } catch (...) {
        return bfail(nullptr, TBS_ERR_NOMEM, "host allocation failed");
    }
    auto fail = [&](int rc) {
        std::string msg = b->eng.err;
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
            if ((c->algo != TBS_ALGO_FP64 && c->algo != TBS_ALGO_MIXED) || c->nvar != 9)
                return fail(bfail(b, TBS_ERR_UNSUPPORTED,
                                  "batches take TBS_ALGO_FP64 or TBS_ALGO_MIXED systems of nvar 9"));
            if (s > 0 && (c->algo != systems[0]->algo || c->device != systems[0]->device))
                return fail(bfail(b, TBS_ERR_ARG,
                                  "all systems of a batch need the same algorithm and GPU"));
            b->sys.push_back(c);
        }
        const int dev = systems[0]->device;
        if (cudaSetDevice(dev) != cudaSuccess) return fail(bfail(b, TBS_ERR_CUDA, "cudaSetDevice failed"));
        if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess)
            return fail(bfail(b, TBS_ERR_CUDA, "cudaStreamCreate failed"));
        int rc = engine_init(b->eng, dev, b->own, systems[0]->algo);
        if (rc) return fail(rc);
        b->eng.inner = systems[0]->inner_sweeps;
        b->eng.inner_first = systems[0]->inner_first;
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
    if (ns != b->eng.stream) {
        cudaStreamSynchronize(b->eng.stream);
        engine_drop_graph(b->eng);
        b->eng.stream = ns;
    }
    return TBS_OK;
}

int tbs_batch_size(const tbs_batch *b, int *nsys) {
    if (!b || !nsys) return bfail(nullptr, TBS_ERR_ARG, "null argument");
    *nsys = (int)b->sys.size();
    return TBS_OK;
}

int tbs_batch_set_inner_sweeps(tbs_batch *b, int m) { return tbs_batch_set_inner_schedule(b, m, m); }

int tbs_batch_set_inner_schedule(tbs_batch *b, int first, int rest) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (first < 1 || first > 64 || rest < 1 || rest > 64)
        return bfail(b, TBS_ERR_ARG, "inner sweeps must be in 1..64");
    const int f = first == rest ? 0 : first;
    if (rest != b->eng.inner || f != b->eng.inner_first) engine_drop_graph(b->eng);
    b->eng.inner = rest;
    b->eng.inner_first = f;
    return TBS_OK;
}

int tbs_batch_set_schedule(tbs_batch *b, int ctas_per_sm, int stages, int order) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (order != 0 && order != 1) return bfail(b, TBS_ERR_ARG, "bad line order");
    BGUARD_BEGIN
    if (cudaSetDevice(b->eng.device) != cudaSuccess) return bfail(b, TBS_ERR_CUDA, "cudaSetDevice failed");
    return engine_set_schedule(b->eng, BatchSched{ctas_per_sm, stages, b->eng.sched.warps}, order);
    BGUARD_END
}

int tbs_batch_set_warps_per_line(tbs_batch *b, int warps) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (warps != 1 && warps != 2) return bfail(b, TBS_ERR_ARG, "warps per line must be 1 or 2");
    BGUARD_BEGIN
    if (cudaSetDevice(b->eng.device) != cudaSuccess) return bfail(b, TBS_ERR_CUDA, "cudaSetDevice failed");
    BatchSched s = b->eng.sched;
    const int fit = b->eng.algo == TBS_ALGO_FP64 ? thomas_batch_fit<double>(s.stages, warps)
                                                 : thomas_batch_fit<float>(s.stages, warps);
    s.warps = warps;
    s.ctas_per_sm = std::max(1, std::min(s.ctas_per_sm, fit));
    return engine_set_schedule(b->eng, s, b->eng.order);
    BGUARD_END
}

int tbs_batch_get_warps_per_line(const tbs_batch *b, int *warps) {
    if (!b || !warps) return bfail(const_cast<tbs_batch *>(b), TBS_ERR_ARG, "null argument");
    *warps = b->eng.sched.warps;
    return TBS_OK;
}

int tbs_batch_get_schedule(const tbs_batch *b, int *ctas_per_sm, int *stages, int *order) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (ctas_per_sm) *ctas_per_sm = b->eng.sched.ctas_per_sm;
    if (stages) *stages = b->eng.sched.stages;
    if (order) *order = b->eng.order;
    return TBS_OK;
}

int tbs_batch_solve(tbs_batch *b, double rel_tol, int max_sweeps, int *sweeps_out,
                    double *hist_out) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (max_sweeps < 0 || !(rel_tol >= 0.0)) return bfail(b, TBS_ERR_ARG, "bad tolerance or sweep limit");
    BGUARD_BEGIN
    if (cudaSetDevice(b->eng.device) != cudaSuccess) return bfail(b, TBS_ERR_CUDA, "cudaSetDevice failed");
    int rc = batch_ready(b, rel_tol, max_sweeps);
    if (rc) return rc;
    rc = engine_run(b->eng, 0, 0);
    if (rc) return rc;
    cudaStream_t st = b->eng.stream;
    const int n = (int)b->sys.size();
    for (int s = 0; s < n; ++s) {
        tbs_ctx *c = b->sys[s];
        if (xfer_to_host(st, c->h_state, c->d_state, sizeof(SolveState), 1) != 0)
            return bfail(b, TBS_ERR_CUDA, "state read-back failed");
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return bfail(b, TBS_ERR_CUDA, "synchronisation failed");
    for (int s = 0; s < n; ++s) {
        tbs_ctx *c = b->sys[s];
        const int sw = c->h_state->sweep;
        if (sweeps_out) sweeps_out[s] = sw;
        if (hist_out &&
            xfer_to_host(st, hist_out + (size_t)s * (max_sweeps + 1), c->d_hist,
                         (size_t)(std::min(sw, max_sweeps) + 1) * sizeof(double), 1) != 0)
            return bfail(b, TBS_ERR_CUDA, "history read-back failed");
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return bfail(b, TBS_ERR_CUDA, "synchronisation failed");
    return TBS_OK;
    BGUARD_END
}

int tbs_batch_tune(tbs_batch *b, int *ctas_per_sm, int *stages, int *order, double *best_ms) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    BGUARD_BEGIN
    if (cudaSetDevice(b->eng.device) != cudaSuccess) return bfail(b, TBS_ERR_CUDA, "cudaSetDevice failed");
    int rc = batch_ready(b, 0.0, 1);
    if (rc) return rc;
    BatchSched s{};
    int o = 0;
    double ms = 0.0;
    rc = engine_tune(b->eng, &s, &o, &ms);
    if (rc) return rc;
    if (ctas_per_sm) *ctas_per_sm = s.ctas_per_sm;
    if (stages) *stages = s.stages;
    if (order) *order = o;
    if (best_ms) *best_ms = ms;
    return TBS_OK;
    BGUARD_END
}

/* one timed batch solve (best of two after a first one that builds the
 * graph); +inf unless every member reached the tolerance */
static int batch_time_schedule(tbs_batch *b, int first, int rest, double rel_tol, int max_sweeps,
                               cudaEvent_t e0, cudaEvent_t e1, double *ms_out) {
    int rc = tbs_batch_set_inner_schedule(b, first, rest);
    if (!rc) rc = tbs_batch_solve(b, rel_tol, max_sweeps, nullptr, nullptr);
    double t = 1e300;
    for (int rep = 0; rep < 2 && !rc; ++rep) {
        cudaEventRecord(e0, b->eng.stream);
        rc = tbs_batch_solve(b, rel_tol, max_sweeps, nullptr, nullptr);
        cudaEventRecord(e1, b->eng.stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        t = std::min(t, (double)ms);
    }
    if (rc) return rc;
    bool conv = true;
    for (tbs_ctx *c : b->sys) {
        const SolveState &S = *c->h_state;
        conv = conv && std::isfinite(S.last) && S.last <= S.tol * S.norm0;
    }
    *ms_out = conv ? t : 1e300;
    return TBS_OK;
}

int tbs_batch_tune_inner(tbs_batch *b, double rel_tol, int max_sweeps, int *first_out,
                         int *rest_out, double *best_ms) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (b->eng.algo != TBS_ALGO_MIXED)
        return bfail(b, TBS_ERR_STATE, "tbs_batch_tune_inner needs TBS_ALGO_MIXED systems");
    if (max_sweeps < 1 || !(rel_tol >= 0.0)) return bfail(b, TBS_ERR_ARG, "bad tolerance or sweep limit");
    BGUARD_BEGIN
    if (cudaSetDevice(b->eng.device) != cudaSuccess) return bfail(b, TBS_ERR_CUDA, "cudaSetDevice failed");
    const bool prof = b->eng.prof;
    b->eng.prof = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return bfail(b, TBS_ERR_CUDA, "cudaEventCreate failed");
    int bf = -1, br = -1, rc = TBS_OK;
    double best_t = 1e300;
    auto consider = [&](int f, int r) {
        if (rc || f < 1 || r < 1) return;
        double t = 1e300;
        rc = batch_time_schedule(b, f, r, rel_tol, max_sweeps, e0, e1, &t);
        if (!rc && t < best_t) {
            best_t = t;
            bf = f;
            br = r;
        }
    };
    /* the search of tbs_tune_inner: one count for every outer step, then
     * the first step's own count around the best */
    for (int m : {2, 3, 4, 5, 6, 8}) consider(m, m);
    if (!rc && br > 0) {
        const int m = br;
        for (int r : {m - 1, m, m + 1})
            for (int f : {m - 2, m - 1, m, m + 1, m + 2})
                if (!(f == r && (r == m - 1 || r == m || r == m + 1))) consider(f, r);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->eng.prof = prof;
    if (rc) return rc;
    if (bf < 0) return bfail(b, TBS_ERR_NUMERIC, "no inner sweep schedule reached the tolerance");
    rc = tbs_batch_set_inner_schedule(b, bf, br);
    if (rc) return rc;
    if (first_out) *first_out = bf;
    if (rest_out) *rest_out = br;
    if (best_ms) *best_ms = best_t;
    return TBS_OK;
    BGUARD_END
}

int tbs_batch_profile_enable(tbs_batch *b, int on) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    if (!on) eprof_resolve(b->eng);
    b->eng.prof = on != 0;
    return TBS_OK;
}

int tbs_batch_profile_reset(tbs_batch *b) {
    if (!b) return bfail(nullptr, TBS_ERR_ARG, "null batch");
    eprof_resolve(b->eng);
    b->eng.slots.clear();
    return TBS_OK;
}

int tbs_batch_profile_read(tbs_batch *b, int *n, const char **names, long long *launches,
                           double *ms) {
    if (!b || !n) return bfail(b, TBS_ERR_ARG, "null argument");
    eprof_resolve(b->eng);
    const int cap = *n, cnt = (int)b->eng.slots.size();
    for (int i = 0; i < cnt && i < cap; ++i) {
        if (names) names[i] = b->eng.slots[i].name;
        if (launches) launches[i] = b->eng.slots[i].launches;
        if (ms) ms[i] = b->eng.slots[i].ms;
    }
    *n = cnt;
    return TBS_OK;
}

}  // extern "C"

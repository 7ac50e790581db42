/*
 * tbs_internal.hxx -- declarations shared by the host code (formats.cpp,
 * api.cu) and the kernel translation units (kernels_ref.cu,
 * kernels_fast.cu).  Not installed; the public surface is include/triblock.h.
 */
#ifndef TBS_INTERNAL_HXX
#define TBS_INTERNAL_HXX

#include "../../include/triblock.h"

#include <cstddef>
#include <cstdint>
#include <string>

#ifdef __CUDACC__
#include <cuda_runtime.h>
#else
typedef struct CUstream_st *cudaStream_t;
#endif

namespace tbs {

/* -------------------------------------------------------------- formats */
void set_thread_error(const std::string &msg);
const char *thread_error();
long long mesh_file_bytes(const int hdr[6]);
long long jacobian_file_bytes(const int hdr[3]);
int read_mesh_header(const char *path, int hdr[6]);
int read_mesh(const char *path, const int hdr[6], int *epoint, int *ef, int *fc, int *linesize,
              int *linepoint, int *lines, int *lineface);
int write_mesh(const char *path, const int hdr[6], const int *epoint, const int *ef, const int *fc,
               const int *linesize, const int *linepoint, const int *lines, const int *lineface);
int read_jacobian_header(const char *path, int hdr[3]);
int read_jacobian(const char *path, const int hdr[3], double *jacD, double *jacO1, double *jacO2,
                  double *rhs, double *U0);
int write_jacobian(const char *path, const int hdr[3], const double *jacD, const double *jacO1,
                   const double *jacO2, const double *rhs, const double *U0);
int validate_mesh(const int hdr[6], const int *epoint, const int *ef, const int *fc,
                  const int *linesize, const int *linepoint, const int *lines,
                  const int *lineface);
int gen_structured_header(int L, int K, int nvar, int hdr[6]);
int gen_structured_mesh(int L, int K, int *epoint, int *ef, int *fc, int *linesize,
                        int *linepoint, int *lines, int *lineface);
int gen_jacobian(int nvar, int nelem, int nintface, double shift, uint64_t seed, double *jacD,
                 double *jacO1, double *jacO2, double *rhs, double *U0);

/* ------------------------------------------------------ device status bits
 * Kernels never trap: they OR one of these into a device status word that
 * the host reads after the launch sequence. */
enum : unsigned {
    ST_PIVOT = 1u,       /* zero or non-finite pivot in a block factorization */
    ST_TIMEOUT = 2u,     /* an mbarrier wait ran out of its clock budget */
    ST_BOUNDS = 4u,      /* an index failed a device-side range check */
};

/* Per-solve state that lives in device memory so that one instantiated
 * CUDA graph serves every tolerance and sweep limit. */
struct SolveState {
    double norm0;      /* ||R_0|| of the current solve */
    double last;       /* latest ||R|| */
    int sweep;         /* sweeps done in the current solve */
    int pad;
    /* control block, written by the host before a solve (offset 24) */
    double tol;        /* relative tolerance */
    int max_sweeps;
    int hist_cap;      /* entries available in hist */
    /* checks of a converged solve against the true residual (device-written;
     * reset by the solve's start) */
    double true_norm;  /* ||rhs + J U|| at the last check, -1 when none ran */
    int checks;        /* checks run in the current solve */
    int restarts;      /* checks that failed: the solve went on from the true residual */
};

/* ------------------------------------------------- fast (line-ordered) layout
 * Each line of n cells is solved as a twisted block-Thomas system: a top
 * chain (cells 0..m-1, eliminated downward), a bottom chain (cells n-1
 * down to m+1, eliminated upward) and the twist cell m where they meet.
 * Positions p give every line a contiguous range starting at a multiple of
 * 4: [top chain in order][bottom chain in elimination order][twist], then
 * zero pad cells up to the next multiple of 4.  m is a multiple of 4, so
 * both chains start 16-byte aligned for cp.async.bulk in FP64 and FP32
 * (4 cells of 9x9 blocks = 2592 / 1296 B).  np16 = positions rounded up to
 * a multiple of RES_TILE, the residual kernel's tile. */
constexpr int RES_TILE = 16;

/* twist cell of a line of n cells: the top chain gets m = 4*round((n-1)/8)
 * cells, the bottom chain n-1-m */
inline int line_twist_of(int n) {
    if (n < 2) return 0;
    int m = 4 * (int)((n - 1 + 4) / 8);
    if (m > n - 1) m = n - 1 - ((n - 1) % 4);
    return m;
}

struct FastLayout {
    int nv;        /* block size (9) */
    int np;        /* positions incl. line pads */
    int np16;      /* np rounded up to RES_TILE */
    int ntile_own; /* tiles of the owned lines (all tiles unless the mesh ends in halo lines) */
    int nx;        /* cross-line coupling slots per position */
    int nline;
    int max_len;   /* longest line */
    /* device arrays */
    int *line_start;   /* [nline] multiple of 4 */
    int *line_len;     /* [nline] */
    int *line_twist;   /* [nline] m: top chain length (multiple of 4) */
    int *pos_of_elem;  /* [nelem] */
    int *elem_of_pos;  /* [np16], -1 for pads */
    int *xnbr;         /* [nx*np16] slot-major: neighbour position or -1 */
    int *xsrc;         /* [nx*np16] 2*face + (1 if the block is O2), or -1 */
    int nxf;           /* all-face slots per position (the full residual) */
    int *xnbrf;        /* [nxf*np16] slot-major: neighbour position over every interior
                        * face of the cell in ef order, or -1 */
    int *xsrcf;        /* [nxf*np16] 2*face + (1 if the block is O2), or -1 */
    int *fsrc;         /* [np16*5] factor sources: elem, face to the chain
                        * predecessor (-1 at a chain start), side (1 if elem is
                        * fc[2f]); the twist position adds the face to its
                        * bottom neighbour and its side (its top face in 1-2) */
};

/* Raise kernel fn's dynamic shared-memory limit to at least `need` bytes.
 * The limit is one value per kernel for the whole process, shared by every
 * context (and thread) that launches the kernel, so it is only ever raised:
 * a context with a smaller mesh must not lower it under a larger one.
 * Returns a cudaError_t as an int. */
int smem_raise(const void *fn, size_t need);

/* ------------------------------------------------------ kernel launchers
 * All launches go on `st`; they return cudaGetLastError() as an int. */

/* reference-order kernels (kernels_ref.cu, built with -fmad=false) */
int launch_ref_line_lu(cudaStream_t st, int nv, int nline, const int *fc, const int *linesize,
                       const int *linepoint, const int *lines, const int *lineface, double *DLU,
                       const double *O1, const double *O2, double *DinvC, unsigned *status);
int launch_ref_assemble_A(cudaStream_t st, int nv, int nline, const int *fc, const int *linesize,
                          const int *linepoint, const int *lines, const int *lineface,
                          const double *O1, const double *O2, double *A);
int launch_ref_solve_du(cudaStream_t st, int nv, int nline, const int *linesize,
                        const int *linepoint, const int *lines, const double *DLU,
                        const double *DinvC, const double *A, double *dU, const double *R);
int launch_ref_add_copy(cudaStream_t st, long long n, const double *dU, double *U,
                        const double *rhs, double *R);
int launch_ref_line_res(cudaStream_t st, int nv, int nline, int nelem, const int *epoint,
                        const int *ef, const int *fc, const int *linesize, const int *linepoint,
                        const int *lines, const double *D, const double *O1, const double *O2,
                        const double *U, double *R, double *partials, int *npartials_out);
int ref_line_res_partials(int nelem);

/* generic helpers (kernels_fast.cu) */
int launch_norm_partials(cudaStream_t st, const double *v, long long n, double *partials,
                         int npart);
int launch_reduce_norm(cudaStream_t st, const double *partials, int n, SolveState *state,
                       double *hist, int is_start, unsigned long long cond_handle, int use_cond,
                       unsigned long long cond_handle2 = 0, int use2 = 0);
int launch_zero(cudaStream_t st, double *p, long long n);
int launch_permute_to_pos(cudaStream_t st, int nv, int nelem, const int *pos_of_elem,
                          const double *src_elem, double *dst_pos);
int launch_permute_to_elem(cudaStream_t st, int nv, int nelem, const int *pos_of_elem,
                           const double *src_pos, double *dst_elem);
int launch_permute_f32_to_elem(cudaStream_t st, int nv, int nelem, const int *pos_of_elem,
                               const float *src_pos, double *dst_elem);

/* fast FP64 / FP32 kernels (kernels_fast.cu) */
int launch_fast_factor(cudaStream_t st, const FastLayout &L, const double *jacD,
                       const double *O1, const double *O2, double *Dinv, double *G, double *Gam,
                       float *Dinv32, float *G32, float *Gam32, double *gamlast,
                       unsigned *status);
int launch_fast_xlayout(cudaStream_t st, const FastLayout &L, const double *O1, const double *O2,
                        double *X, float *X32);
/* DX = Dinv X per cross-line slot, FP32 (TBS_ALGO_MIXED inner sweeps) */
int launch_fast_dx(cudaStream_t st, const FastLayout &L, const double *Dinv, const double *O1,
                   const double *O2, float *DX);
int fast_resid_grid(int np16);
/* Where a streaming kernel's sum of R^2 goes: per-CTA partials, and, when
 * `state` is set, the last CTA's fixed-order total recorded like
 * reduce_norm (norm history, sweep count, graph loop condition). */
struct NormSink {
    double *partials;            /* [grid] or null: no norm */
    unsigned *counter;           /* zero between launches */
    SolveState *state;           /* null: partials only */
    double *hist;
    int is_start;                /* 1: the norm opens a solve; 0: one more sweep;
                                  * NORM_CHECK: the true residual of a converged solve */
    int use_cond;
    unsigned long long handle;   /* cudaGraphConditionalHandle */
    int ntiles;                  /* > 0: the norm sums the first ntiles tiles only (the
                                  * owned lines of a line partition); 0: every tile */
    int use_check;               /* a sweep's norm also sets check_handle: 1 when the
                                  * recursive residual has met the tolerance */
    unsigned long long check_handle;
    unsigned long long *timer;   /* null, or the launch's device-clock record: [0] the
                                  * earliest CTA start (all ones between launches),
                                  * [1] += last finish - [0] in ns, [2] += 1 launch */
};
/* NormSink::is_start of the check of a converged solve: a norm at or below
 * the tolerance ends the solve with the history unchanged; a larger one
 * replaces the sweep's entry and the solve goes on from it */
constexpr int NORM_CHECK = 2;

/* mode 0: R given (Rsrc); 1: R = sum X dU (with norm); 3: X holds Dinv X,
 * b = -sum X dU, no norm; 4: b = sum X dU - Rsrc (the product with J of
 * the iterate of line sweeps on Rsrc + J z = 0), no Dinv, no norm.  Uacc
 * (may be null): modes 1, 3 add dU to it for the tile's positions, mode 0
 * sets it to zero there; mode 1 only from tile u_tile0 on, and with Uin
 * set as Uacc = Uin + dU */
template <typename T>
int launch_fast_resid(cudaStream_t st, const FastLayout &L, int mode, const T *Dinv,
                      const T *X, const T *dU, const T *Rsrc, T *b, const NormSink &ns,
                      unsigned *status, T *Uacc = nullptr, int u_tile0 = 0,
                      const T *Uin = nullptr);
/* accumulate 0: U = dU, 1: U += dU (U = Uin + dU when Uin is set), 2: U
 * left alone; lines from nacc on (nacc >= 0) leave U alone */
template <typename T>
int launch_fast_thomas(cudaStream_t st, const FastLayout &L, const T *G, const T *Gam,
                       const T *b, T *y, T *dU, T *U, unsigned *status, int accumulate,
                       int nacc = -1, const T *Uin = nullptr);
int fast_kernels_init();
/* Several lines' vectors packed into (or unpacked from) one contiguous
 * buffer by one launch: line k's span is [start[k]*9, start[k]*9 + len[k]*9)
 * of `vec` and [off[k], off[k] + len[k]*9) of `buf`. */
constexpr int PACK_MAX_LINES = 64;
struct LinePack {
    int n;
    int start[PACK_MAX_LINES];
    int len[PACK_MAX_LINES];
    long long off[PACK_MAX_LINES];
};
int launch_line_pack(cudaStream_t st, const LinePack &lp, double *vec, double *buf, int to_line);
int fast_prepare(const FastLayout &L);
int full_resid_blocks(int nelem);
/* rhs may be null (zero): Rp = J U, the matrix-vector product */
template <typename T>
int launch_full_resid(cudaStream_t st, int nelem, const int *epoint, const int *ef, const int *fc,
                      const int *pos_of_elem, const double *D, const double *O1, const double *O2,
                      const double *rhs, const double *Up, T *Rp, double *partials);

/* The FP64 residual R = rhs + J U in position order from position-ordered
 * copies of the original blocks (Dp: diagonal, XF: one slot per interior
 * face in ef order), streamed per tile with bulk copies like the sweep
 * residual; R goes out in FP32 (the inner solve's right-hand side) with
 * per-tile partials of R^2; with Dinv32 also b32 = -Dinv32 R32 and
 * c32 = 0 for the next inner solve.  Needs L.nxf <= 4. */
int launch_fullpos_layout(cudaStream_t st, const FastLayout &L, const double *jacD,
                          const double *O1, const double *O2, double *Dp, double *XF);
int launch_full_resid_pos(cudaStream_t st, const FastLayout &L, const double *Dp,
                          const double *XF, const double *rhsp, const double *Up, float *R32,
                          double *partials, const float *Dinv32, float *b32, float *c32,
                          unsigned *status);
int fullpos_prepare(const FastLayout &L);

/* mixed-precision glue (kernels_fast.cu) */
int launch_cast_f64_f32(cudaStream_t st, const double *src, float *dst, long long n);
int launch_axpy_f32_f64(cudaStream_t st, const float *d, double *U, long long n);
int launch_axpy2_f32_f64(cudaStream_t st, const float *c, const float *d, double *U, long long n);
int launch_axpy_f64(cudaStream_t st, const double *d, double *U, long long n);
/* per tile of RES_TILE positions: Up = 0, R32 = (float)rhsp, partials[tile]
 * = sum rhsp^2 in a fixed order (the start of a TBS_ALGO_MIXED solve); with
 * Dinv32 also the first inner right-hand side b32 = -Dinv32 R32, c32 = 0 */
int launch_mixed_prime(cudaStream_t st, const FastLayout &L, const double *rhsp, float *R32,
                       double *Up, double *partials, const float *Dinv32, float *b32, float *c32);

/* TBS_ALGO_FP64 for the block sizes other than 9 (kernels_nv.cu): the
 * same launch sequence with kernels templated on nv (2..16); G and Gam are
 * column-major here (the size-9 kernels keep them row-major). */
bool nv_supported(int nv);
int nv_prepare(int nv, const FastLayout &L);
int launch_nv_factor(cudaStream_t st, int nv, const FastLayout &L, const double *jacD,
                     const double *O1, const double *O2, double *Dinv, double *G, double *Gam,
                     double *gamlast, unsigned *status);
int launch_nv_xlayout(cudaStream_t st, int nv, const FastLayout &L, const double *O1,
                      const double *O2, double *X);
int launch_nv_thomas(cudaStream_t st, int nv, const FastLayout &L, const double *G,
                     const double *Gam, const double *b, double *y, double *dU, double *U,
                     int accumulate, unsigned *status);
/* modes 0 and 1 of launch_fast_resid */
int launch_nv_resid(cudaStream_t st, int nv, const FastLayout &L, int mode, const double *Dinv,
                    const double *X, const double *dU, const double *Rsrc, double *b,
                    const NormSink &ns, unsigned *status, double *Uacc);

/* a staging wait that is made to run out: ST_TIMEOUT into *status */
int launch_selftest_timeout(cudaStream_t st, long long budget_cycles, unsigned *status);

/* point-implicit Jacobi (TBS_ALGO_PIJ): D^-1 in place of the
 * position-ordered diagonal blocks; one sweep = U += dU, R = sum over the
 * interior faces of XF dU_nbr, b = -Dinv R, with dU / b alternating between
 * bufA and bufB by SolveState::pad (flipped by each sweep) */
int launch_pij_invert(cudaStream_t st, const FastLayout &L, double *D, unsigned *status);
int launch_pij_sweep(cudaStream_t st, const FastLayout &L, const double *Dinv, const double *XF,
                     double *bufA, double *bufB, double *Up, const NormSink &ns, unsigned *status);
int pij_prepare(const FastLayout &L);

/* ------------------------------------- several right-hand sides (FP64)
 * Up to MULTI_MAX right-hand sides of one system swept together, the line
 * blocks read once per sweep for all of them.  Vectors are RHS-major with
 * stride np16 * 9; state, active and the history rows are per right-hand
 * side, partials [nr][np16 / RES_TILE]. */
constexpr int MULTI_MAX = 8;
constexpr int MULTI_NX = 4;     /* cross-line slots per position of the fast layout */
struct MultiSys {
    int nr, np16, nx, hist_stride;
    double *U, *b, *partials, *hist;
    const double *dU;
    SolveState *state;
    int *active;
    unsigned *counter;
};
/* The line solves of up to MULTI_MAX right-hand sides of one system: its
 * line layout and factors, and per slot r < nr its vectors and the index
 * of its flag in the active array. */
struct MultiLine {
    const int *line_start, *line_len, *line_twist;
    const double *G, *Gam;
    int nr;
    int aid[MULTI_MAX];
    const double *b[MULTI_MAX];
    double *y[MULTI_MAX], *dU[MULTI_MAX];
};
/* dU of every active right-hand side from its b (the line solves) */
int launch_multi_thomas(cudaStream_t st, const FastLayout &L, int nr, const double *G,
                        const double *Gam, const double *b, double *y, double *dU,
                        const int *active, unsigned *status);
/* mode 0: R = Rsrc (position order, RHS-major), U = 0, the solve's start
 * (every r becomes active); mode 1: R = sum X dU, U += dU.  Then b = -Dinv R,
 * the norms, and the graph condition (any right-hand side still active). */
int launch_multi_resid(cudaStream_t st, const FastLayout &L, int mode, const MultiSys &M,
                       const double *Dinv, const double *X, const double *Rsrc,
                       unsigned long long cond_handle, int use_cond, unsigned *status);
int multi_prepare(const FastLayout &L, int nr);


/* ------------------------------------------------------------ batches
 * Many independent systems swept together.  Each kernel takes one
 * descriptor per system and a list of work items (system, unit), so that
 * a launch covers the units of every system that has not converged
 * (active[system] != 0).  The per-unit arithmetic is the one of the
 * single-system kernels, unit for unit, so a system's iterates do not
 * depend on the batch it is solved in. */
struct alignas(8) WorkItem {
    int sys;                    /* index into the launch's descriptors */
    int unit;                   /* line, residual tile or element block */
};
/* the batch engine's line solves of groups of one system's members: item k
 * (k < *nitems, grid = capacity) = (index into sys, line) */
int launch_multi_thomas_items(cudaStream_t st, int grid, const MultiLine *sys, const WorkItem *items,
                              const int *nitems, const int *active, unsigned *status);
int multi_items_prepare(); /* shared-memory opt-in of that launch (outside stream capture) */
template <typename T>
struct ThomasSys {
    const int *line_start, *line_len, *line_twist;
    const T *G, *Gam, *b;
    T *y, *dU;
};
template <typename T>
struct ResidSys {
    int np16, nx;
    const int *xnbr;
    const T *Dinv, *X, *dU, *Rsrc;
    T *b, *Uacc;
    double *partials;
};
struct FullResSys {
    int nelem, pad;
    const int *epoint, *ef, *fc, *pos_of_elem;
    const double *D, *O1, *O2, *rhs, *Up;
    float *R32;
    double *partials;
};
struct FullPosSys {
    int np16, nxf;
    const int *xnbrf;
    const double *Dp, *XF, *rhsp, *Up;
    float *R32;
    double *partials;
    const float *Dinv32;        /* non-null: also b32 = -Dinv32 R32, c32 = 0 */
    float *b32, *c32;
};
struct VecSys {                 /* mixed-precision glue of one system */
    const double *rhsp;
    float *R32, *c32, *d32;
    double *Up;
    double *partials;
    const float *Dinv32;        /* non-null: the prime also sets b32 (and c32 = 0) */
    float *b32;
};
struct ReduceSys {
    const double *partials;
    int n;                      /* partials to sum */
    int member;                 /* index into active[] */
    SolveState *state;
    double *hist;
};
/* Device-side control of a batched launch sequence: the work counts the
 * kernels read (so that one graph serves any set of members) and the rule
 * by which the per-member norm launch ends the graph's sweep loop. */
struct BatchCtl {
    int nsys;                   /* members: active[0..nsys) */
    int nlines;                 /* Thomas work items */
    int ntiles;                 /* residual tiles */
    int nblocks;                /* full-residual element blocks */
    int nprime_sys;             /* norm descriptors of the members started now */
    int nprime_tiles;           /* their tiles */
    int chunk;                  /* sweeps done by the current graph launch */
    int chunk_limit;            /* > 0: the loop ends after this many sweeps */
    int stop_on_finish;         /* 1: the loop ends when a member stops */
    int finished;               /* set by the norm launch when a member stops */
    int nmitems;                /* FP64: (group of one system's members, line) items */
};
struct BatchSched {             /* persistent Thomas launch shape */
    int ctas_per_sm;            /* CTAs per SM, each solving one line at a time */
    int stages;                 /* bulk-copy ring depth */
    int warps;                  /* warps per line: 1 (the chain warp issues its own copies)
                                 * or 2 (a second warp issues them) */
};

template <typename T>
size_t thomas_batch_smem(int stages, int warps);
/* CTAs of the persistent Thomas kernel that fit on one SM with `stages` */
template <typename T>
int thomas_batch_fit(int stages, int warps);
template <typename T>
int launch_thomas_batch(cudaStream_t st, const BatchSched &bs, const ThomasSys<T> *sys,
                        const WorkItem *work, const int *nwork, const int *active, unsigned *queue,
                        unsigned *status);
/* Group index: the work items of the residual-type launches without a
 * list of them.  Members that share a system form a group; group g covers
 * items [base[g], base[g+1]) = (its units) x (its members), unit-major, so
 * that the right-hand sides of one system run each unit side by side and
 * share its blocks in L2.  Device layout (ints):
 *   [ng][base[0..ng]][nmem[0..ng)][moff[0..ng)][mlist[...]]
 * item w -> member mlist[moff[g] + (w - base[g]) % nmem[g]],
 *           unit (w - base[g]) / nmem[g]. */
/* units of the chunked group index: up to BATCH_CHUNK residual tiles */
constexpr int BATCH_CHUNK = 8;
inline int batch_chunks(int ntiles) { return (ntiles + BATCH_CHUNK - 1) / BATCH_CHUNK; }
inline size_t group_index_ints(int max_groups, int max_members) {
    return 1 + (size_t)(max_groups + 1) + 2 * (size_t)max_groups + (size_t)max_members;
}
template <typename T>
/* units of `groups`: single tiles (chunk 1) or chunks of BATCH_CHUNK tiles */
int launch_resid_batch(cudaStream_t st, int mode, int max_nx, const ResidSys<T> *sys,
                       const int *groups, int chunk, const int *active, unsigned *status);
/* the sweep residual (mode 1) of every member, the members of one system
 * together over one staging of its blocks per tile; gunits: the group
 * index of the members with base[] the prefix sums of units (chunks of
 * `chunk` tiles) per group */
template <typename T>
int launch_resid_group(cudaStream_t st, int max_nx, const ResidSys<T> *sys, const int *gunits, int chunk,
                       const int *active, unsigned *status);
int launch_full_resid_batch(cudaStream_t st, const FullResSys *sys, const int *groups,
                            const int *active);
int launch_full_resid_pos_batch(cudaStream_t st, int max_nxf, const FullPosSys *sys,
                                const int *groups, int chunk, const int *active, unsigned *status);
int launch_mixed_prime_batch(cudaStream_t st, const VecSys *sys, const int *groups);
int launch_axpy2_batch(cudaStream_t st, const VecSys *sys, const int *groups, const int *active);
/* one CTA of `threads` threads per norm descriptor (grid = cap, *nred in
 * use): the fixed-order sum of the member's partials (the order of
 * finalize_total for threads = 160 and of reduce_norm for threads = 1024),
 * its norm history and active flag; the last CTA sets the graph condition
 * by the rule in `ctl` */
int launch_reduce_batch(cudaStream_t st, int threads, const ReduceSys *sys, const int *nred,
                        int cap, int is_start, int *active, BatchCtl *ctl, unsigned *counter,
                        unsigned long long cond_handle, int use_cond,
                        unsigned long long cond_handle2 = 0, int use2 = 0);
int batch_prepare(int max_nx);

}  // namespace tbs

/* ------------------------------------------ transfers off the copy engine
 * (xfer.cu).  Host memory below is pinned memory the device can address;
 * the functions return a cudaError_t value (0 = success). */
struct XferJob {               /* one copy of a batched job list */
    unsigned long long dst, src, bytes; /* device addresses; bytes % 4 == 0 */
};
constexpr int kXferPutMax = 256;
/* bytes (a multiple of 4, both addresses 4-aligned) on the SMs, at most
 * max_blocks CTAs of 256 threads (< 1: 4 per SM) */
int xfer_copy(cudaStream_t st, const void *src, void *dst, size_t bytes, int max_blocks);
/* a small value (at most kXferPutMax bytes) written by a kernel that takes
 * it as a parameter */
int xfer_put(cudaStream_t st, void *dst, const void *value, size_t bytes);
/* njobs copies in one launch; jobs_dev is readable by the device (e.g. the
 * device view of a pinned staging buffer); max_bytes bounds the largest */
int xfer_jobs(cudaStream_t st, const XferJob *jobs_dev, int njobs, size_t max_bytes);
/* the device address of pinned host memory, or null */
void *xfer_device_view(const void *host);
/* device -> host / host -> device: by the SMs when the host side is
 * device-addressable pinned memory, else cudaMemcpyAsync */
int xfer_to_host(cudaStream_t st, void *dst, const void *src, size_t bytes, int max_blocks);
int xfer_to_device(cudaStream_t st, void *dst, const void *src, size_t bytes, int max_blocks);

#endif /* TBS_INTERNAL_HXX */

/*
 * triblock.h -- C ABI of libtriblock.so, the B200 line-implicit Jacobi (LIJ) solver.
 *
 * The reference (ackirby88/triblocksolve) exposes no plugin API.  Its de-facto
 * boundary is (1) the two Fortran bind(C) readers, (2) the Mesh/Jacobian
 * classes, (3) the OKL kernel argument lists launched from src/main.cxx and
 * (4) the CLI `triblock.exe <compute_mode> <device_id> <block_size>`.  Every
 * entry point below names the reference interface it replaces.
 *
 * Conventions
 *   - Every tbs_* function returns an int status (TBS_OK == 0).  Nothing
 *     exits the process and no C++ exception crosses this boundary.
 *   - Index arrays passed to tbs_* are 0-based, i.e. exactly what the
 *     reference holds in memory after read_mesh_data_ shifted them
 *     (src/F90/read_mesh_data.F90:41-64).
 *   - Block storage is column-major FP64: entry (row i, col j) of block b is
 *     at i + nvar*j + nvar*nvar*b, the OKL @dim(NVAR,NVAR,n) convention
 *     (src/okl/linesmoothLU_TriBlock_v3.okl:7).
 *   - A context owns one CUDA stream and all of its device memory; one
 *     context must be used from one host thread at a time.
 *   - There is no CPU fallback: a context can only be created on a CUDA
 *     device, and compute_mode values other than 2 (CUDA) are rejected.
 */
#ifndef TRIBLOCK_H
#define TRIBLOCK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define TBS_OK               0
#define TBS_ERR_ARG          1  /* bad argument (null pointer, negative size, ...) */
#define TBS_ERR_IO           2  /* file missing, short read, write failure */
#define TBS_ERR_FORMAT       3  /* header/array inconsistency in mesh or Jacobian */
#define TBS_ERR_CUDA         4  /* CUDA runtime error or no device */
#define TBS_ERR_STATE        5  /* call out of order (e.g. sweep before factor) */
#define TBS_ERR_NUMERIC      6  /* zero / non-finite pivot in the no-pivot block LU */
#define TBS_ERR_UNSUPPORTED  7  /* nvar or mode this build does not support */
#define TBS_ERR_NOMEM        8  /* device or host allocation refused */

/* ---------------------------------------------------- algorithm / precision
 * TBS_ALGO_REFERENCE  reference operation order (LU-form blocks, solveLU,
 *                     full residual R = rhs + J U each sweep).  Compiled
 *                     without FMA contraction so that U, dU and R are
 *                     bit-identical to the CPU oracle.
 * TBS_ALGO_FP64       FP64, line-ordered storage, explicit block inverses,
 *                     residual updated from the cross-line couplings only
 *                     (R_{s+1} = O dU_{s+1}, exact for an exact line solve).
 * TBS_ALGO_MIXED      FP32 line factors and FP32 inner sweeps on the
 *                     correction equation; residual, solution accumulation
 *                     and convergence test in FP64 (outer refinement).
 * TBS_ALGO_PIJ        point-implicit Jacobi, the line sweep's sibling with
 *                     the diagonal block alone as the implicit operator
 *                     (dU = -D^-1 R, U += dU, R = rhs + J U; every cell its
 *                     own line), FP64, residual updated from the face
 *                     couplings like TBS_ALGO_FP64.
 */
#define TBS_ALGO_REFERENCE 0
#define TBS_ALGO_FP64      1
#define TBS_ALGO_MIXED     2
#define TBS_ALGO_PIJ       3

/* compute modes of the reference CLI (include/Platform.hxx:17-23) */
#define TBS_SERIAL_MODE 0
#define TBS_HIP_MODE    1
#define TBS_CUDA_MODE   2
#define TBS_OPENCL_MODE 3
#define TBS_OPENMP_MODE 4
#define TBS_DPCPP_MODE  5
#define TBS_METAL_MODE  6

typedef struct tbs_ctx tbs_ctx;

/* ============================================================ file formats */

/* Replaces the Fortran reader src/F90/read_mesh_data.F90:8-65 (declared at
 * include/Mesh.hxx:22-25).  Same signature and semantics: reads
 * ./gpuline.mesh.data.bin (stream binary, little-endian int32), fills the
 * caller-sized arrays and converts 1-based indices to 0-based.  The Fortran
 * routine reports nothing; failures here leave the arrays untouched and are
 * reported by tbs_last_error(NULL). */
void read_mesh_data_(int *nvar, int *nelem, int *nintface,
                     int *eftot, int *nline, int *nlineelem,
                     int *epoint, int *ef, int *fc, int *lines,
                     int *linesize, int *linepoint, int *lineface);

/* Replaces src/F90/read_jacobian_data.F90:8-33 (declared at
 * include/Jacobian.hxx:23-25): reads ./gpuline.jacobian.data.bin. */
void read_jacobian_data_(int *nvar, int *nelem, int *nintface,
                         double *jacD, double *jacO1, double *jacO2,
                         double *rhs, double *U0);

/* Header of a mesh file: hdr = {nvar, nelem, nintface, eftot, nline, nlineelem}
 * (src/Mesh.cxx:21-32).  Also checks that the file size matches the header. */
int tbs_read_mesh_header(const char *path, int hdr[6]);

/* Path form of read_mesh_data_ with a status; outputs are 0-based. */
int tbs_read_mesh(const char *path, const int hdr[6],
                  int *epoint, int *ef, int *fc, int *linesize,
                  int *linepoint, int *lines, int *lineface);

/* Writes a mesh file in the reference layout (inputs 0-based, written 1-based). */
int tbs_write_mesh(const char *path, const int hdr[6],
                   const int *epoint, const int *ef, const int *fc,
                   const int *linesize, const int *linepoint,
                   const int *lines, const int *lineface);

/* Header of a Jacobian file: hdr = {nvar, nelem, nintface}
 * (src/Jacobian.cxx:22-27); checks the file size. */
int tbs_read_jacobian_header(const char *path, int hdr[3]);

int tbs_read_jacobian(const char *path, const int hdr[3],
                      double *jacD, double *jacO1, double *jacO2,
                      double *rhs, double *U0);

int tbs_write_jacobian(const char *path, const int hdr[3],
                       const double *jacD, const double *jacO1,
                       const double *jacO2, const double *rhs,
                       const double *U0);

/* Checks the index invariants every solver path relies on: index ranges,
 * linepoint prefix sums, lines a permutation of the elements, lineface[m]
 * (k >= 1) joining lines[m-1] and lines[m].  The reference checks nothing. */
int tbs_validate_mesh(const int hdr[6],
                      const int *epoint, const int *ef, const int *fc,
                      const int *linesize, const int *linepoint,
                      const int *lines, const int *lineface);

/* ======================================================= synthetic inputs
 * Structured L x K quad mesh in the reference's numbering; it reproduces
 * data/ex05/gpuline.mesh.data.bin (L=60, K=64) bit for bit. */
int tbs_gen_structured_header(int L, int K, int nvar, int hdr[6]);
int tbs_gen_structured_mesh(int L, int K,
                            int *epoint, int *ef, int *fc, int *linesize,
                            int *linepoint, int *lines, int *lineface);

/* Seeded values in file order: jacD = U(-1,1) + shift*I, jacO1/jacO2 =
 * 0.1*U(-1,1), rhs = U(-1,1), U0 = 0.  U(-1,1) of stream position n is
 * splitmix64(seed + (n+1)*0x9E3779B97F4A7C15) mapped to [-1,1) with 53
 * bits, so host and device generation agree bit for bit.  Runs on all host
 * threads. */
int tbs_gen_jacobian(int nvar, int nelem, int nintface, double shift,
                     uint64_t seed, double *jacD, double *jacO1,
                     double *jacO2, double *rhs, double *U0);

/* Block-size change of src/Jacobian.cxx:153-238 with the same resulting
 * arrays: new diagonals of D, O1, O2 set to 10.0, the old min(nv)-square
 * sub-blocks copied in, and -- as the reference's vector::resize leaves
 * them -- the leading entries of every array keeping the old flat data
 * wherever neither rule writes.  rhs and U0 copy their first
 * nelem*min(nv) entries flat.  Output arrays are sized for nv_new. */
int tbs_resize_block_size(int nv_old, int nv_new, int nelem, int nintface,
                          const double *D_old, const double *O1_old,
                          const double *O2_old, const double *rhs_old,
                          const double *U0_old, double *D, double *O1,
                          double *O2, double *rhs, double *U0);

/* ================================================================ solver */

/* Device selection, replacing Platform(comm, mode, device_id)
 * (src/Platform.cxx:11-78).  Fails with TBS_ERR_CUDA when no device exists. */
int tbs_create(int device_id, tbs_ctx **out);
int tbs_destroy(tbs_ctx *ctx);

/* Last error text of ctx, or of the calling thread when ctx is NULL. */
const char *tbs_last_error(const tbs_ctx *ctx);

/* Launch on a caller-owned cudaStream_t instead of the context's own
 * stream (pass NULL to return to the context's stream). */
int tbs_set_stream(tbs_ctx *ctx, void *cuda_stream);

/* Replaces Mesh::setupDevice/toDevice (src/Mesh.cxx:75-94).  Copies the
 * 0-based mesh in; the caller keeps ownership of its arrays. */
int tbs_set_mesh(tbs_ctx *ctx, int nvar, int nelem, int nintface, int eftot,
                 int nline, int nlineelem,
                 const int *epoint, const int *ef, const int *fc,
                 const int *linesize, const int *linepoint,
                 const int *lines, const int *lineface);

/* Replaces Jacobian::setupDevice/toDevice (src/Jacobian.cxx:240-277).
 * Host pointers; U0 may be NULL.  As in the reference, the solution
 * starts at zero (U0 is kept only for tbs_set_initial). */
int tbs_set_jacobian(tbs_ctx *ctx, const double *jacD, const double *jacO1,
                     const double *jacO2, const double *rhs, const double *U0);

/* Same, from device pointers already resident on the context's device
 * (copied device-to-device on the context's stream). */
int tbs_set_jacobian_device(tbs_ctx *ctx, const double *d_jacD,
                            const double *d_jacO1, const double *d_jacO2,
                            const double *d_rhs);

/* New right-hand side for the already factored Jacobian (host pointer);
 * resets U to zero and R to rhs. */
int tbs_set_rhs(tbs_ctx *ctx, const double *rhs);

/* Starting solution (host pointer, 9*nelem): R becomes rhs + J U.
 * Checkpoint/resume of a solve; the reference always starts from 0. */
int tbs_set_initial(tbs_ctx *ctx, const double *U);

/* The next system's Jacobian (host or device pointers, the layout of
 * tbs_set_jacobian) uploaded into a landing set of device buffers on the
 * context's own copy stream, while the current system is still being
 * solved: the call returns at once, and a later tbs_factor waits for the
 * upload and switches to the staged values (its rhs included).  Up to two
 * systems may be staged; each tbs_factor takes the older one.  A stream of
 * systems then keeps the host-to-device link busy, the factorizations
 * included:
 *   tbs_stage_jacobian(ctx, J0...);  tbs_stage_jacobian(ctx, J1...);
 *   tbs_factor(ctx, algo);                  -- system 0
 *   for each system k:
 *     tbs_solve(ctx, ...);  tbs_get_solution(ctx, U_k);
 *     tbs_stage_jacobian(ctx, J[k+2]...);   -- queued behind J[k+1]
 *     tbs_factor(ctx, algo);                -- now the system k+1
 * The copies overlap the solve only from pinned (page-locked) host memory;
 * the host arrays must stay unchanged until the tbs_factor that takes them
 * returns.  A third stage before a tbs_factor is refused (TBS_ERR_STATE);
 * tbs_set_jacobian discards the staged systems.  Each landing set costs
 * the device memory of one more Jacobian; tbs_factor copies the set it
 * takes over the active one on the device (about 1.6 ms for 5 GB), so the
 * solve graph keeps its addresses and no host copy of the solve waits
 * behind an upload.  No counterpart in the reference,
 * which reads one Jacobian per run (src/main.cxx:86-93). */
int tbs_stage_jacobian(tbs_ctx *ctx, const double *jacD, const double *jacO1,
                       const double *jacO2, const double *rhs);

/* Replaces copyAtoBjac + lineLU (src/main.cxx:180-190,
 * src/okl/lineLU_v2.okl:58-182, src/okl/linesmoothLU_v5.okl:85-93) and the
 * host packing Jacobian::assembleTriBlocks (src/Jacobian.cxx:76-117).
 * algo is one of TBS_ALGO_*.  Resets U to zero and R to rhs. */
int tbs_factor(tbs_ctx *ctx, int algo);

/* n LIJ sweeps (src/main.cxx:207-229: solveDU -> U += dU -> R = rhs ->
 * R += J U).  rnorm_out (may be NULL) receives n+1 values: ||R|| before
 * the first sweep and after each sweep (2-norm over all 9*nelem entries).
 * TBS_ALGO_MIXED counts one outer refinement step as one sweep. */
int tbs_sweep(tbs_ctx *ctx, int n, double *rnorm_out);

/* Sweeps until ||R|| <= rel_tol * ||R_0|| or max_sweeps, with the
 * convergence test on the device (one CUDA graph launch, no host round
 * trip per sweep).  *sweeps_out = sweeps done; hist_out (may be NULL)
 * receives sweeps+1 norms, hist[0] = ||R_0||.
 * TBS_ALGO_FP64 tracks R recursively; when that R meets the tolerance the
 * solve recomputes the true residual rhs + J U from the original blocks
 * (the rule of src/okl/linesmoothLU_TriBlock_v3.okl:228-336).  If it also
 * meets the tolerance the solve ends (history unchanged); if not, its norm
 * replaces the sweep's history entry and the sweeps go on from it.  So a
 * reported convergence is never one that tbs_true_residual_norm
 * contradicts.  tbs_set_check(ctx, 0) turns the check off. */
int tbs_solve(tbs_ctx *ctx, double rel_tol, int max_sweeps,
              int *sweeps_out, double *hist_out);

/* nrhs right-hand sides with the factors of the last
 * tbs_factor(TBS_ALGO_FP64), each from U = 0: the multi-RHS form of the
 * sweep loop of src/main.cxx:180-229 (the reference solves one per run).
 * rhs and U hold nrhs vectors of 9*nelem doubles, element order, one after
 * the other.  Groups of up to 8 sweep together in one CUDA graph launch,
 * the line blocks read once per sweep for the group; each right-hand side
 * stops at its own tolerance or max_sweeps.  sweeps (may be NULL) gets
 * nrhs counts; hist (may be NULL) row r, at hist + r * hist_stride, gets
 * min(sweeps[r] + 1, hist_stride) norms as tbs_solve's hist_out.  Every
 * right-hand side's U, sweep count and norms are bit-identical to
 * tbs_set_rhs + tbs_solve of it alone.  The context's own rhs and solution
 * are left alone.  TBS_ERR_UNSUPPORTED for the other algorithms.
 * tbs_solve_multi takes host arrays; tbs_solve_multi_device device arrays
 * (work on the context's stream; returns after it is done). */
int tbs_solve_multi(tbs_ctx *ctx, int nrhs, const double *rhs, double *U,
                    double rel_tol, int max_sweeps, int *sweeps, double *hist,
                    int hist_stride);
int tbs_solve_multi_device(tbs_ctx *ctx, int nrhs, const double *d_rhs,
                           double *d_U, double rel_tol, int max_sweeps,
                           int *sweeps, double *hist, int hist_stride);

/* Restarted GMRES(restart) on J U = -rhs from U = 0, right preconditioned
 * by precond_sweeps LIJ sweeps from zero with the TBS_ALGO_FP64 factors
 * (one sweep: the line block-tridiagonal solve) -- the Krylov caller of the
 * line sweep in the paper (p.14, Table 6), which the reference repository
 * does not contain.  Stops when the residual norm reaches rel_tol * ||rhs||
 * or after max_iters Arnoldi steps (each one preconditioner application
 * and one product with J).  *iters_out = Arnoldi steps; hist_out (may be
 * NULL, max_iters + 1 entries) gets ||rhs|| and then the GMRES residual
 * estimate after each step, replaced by the true ||rhs + J U|| at the end
 * of every restart cycle.  The solution is read with tbs_get_solution;
 * tbs_solve / tbs_set_rhs start over from U = 0.  restart <= 64. */
int tbs_gmres(tbs_ctx *ctx, int restart, int precond_sweeps, double rel_tol,
              int max_iters, int *iters_out, double *hist_out);

/* ======================================================= line partitions
 * One mesh split over several contexts (one per GPU, or several on one
 * GPU), each owning a contiguous range of lines.  The reference solves a
 * mesh on one device; this splits its sweep loop (src/main.cxx:207-229) at
 * the one place where partitions need each other's data: the residual
 * (triblock_lineRes, src/okl/linesmoothLU_TriBlock_v3.okl:228-336) reads
 * the update of the neighbouring lines.
 *
 * tbs_set_partition_mesh: tbs_set_mesh for one partition.  The mesh holds
 * the owned lines followed by nhalo_lines halo lines: whole copies of the
 * lines of other partitions that hold a neighbour of an owned cell (their
 * faces to cells outside this mesh dropped).  The owned lines' cells must
 * be elements 0..nelem_own-1.  Halo lines are swept like the others, but
 * no norm counts them; tbs_solve / tbs_sweep / multi-RHS / GMRES / batches
 * refuse such a context (TBS_ERR_UNSUPPORTED): it sweeps as below.  Needs
 * tbs_factor(TBS_ALGO_FP64), nvar 9.
 *
 * A solve from U = 0:
 *   tbs_part_start(ctx, &n0)          ||R_0|| over the owned cells
 *   repeat:
 *     tbs_part_solve_du(ctx)          line solves, dU of every line (the
 *                                     owned lines' U + dU into a second U
 *                                     buffer; the current U is untouched)
 *     for each halo line h: copy dU of h from its owner into this context
 *       (tbs_part_line_vector: owner to_line=0 into a device buffer, the
 *        buffer to another GPU by NCCL or a peer copy, then to_line=1 here)
 *     tbs_part_line_res(ctx, &n)      R from dU, the halo lines' U + dU,
 *                                     the second buffer becomes the
 *                                     current U, ||R|| over owned
 *   the global norm is sqrt(sum over partitions of n^2).  A
 *   tbs_part_solve_du issued before the norm is read (and dropped when the
 *   solve ends there) leaves the solution unchanged.
 * Owned cells' U and dU are bit-identical to a tbs_sweep of the whole mesh;
 * a halo line's U is its owner's (it accumulates the copied dU).
 * tbs_true_residual_norm, on such a context, covers the owned cells.
 * owned_norm may be NULL in tbs_part_line_res: no host synchronisation,
 * the norm stays in the context (read by the next call that returns one). */
int tbs_set_partition_mesh(tbs_ctx *ctx, int nhalo_lines, int nvar, int nelem,
                           int nintface, int eftot, int nline, int nlineelem,
                           const int *epoint, const int *ef, const int *fc,
                           const int *linesize, const int *linepoint,
                           const int *lines, const int *lineface);
int tbs_part_start(tbs_ctx *ctx, double *owned_norm);
int tbs_part_solve_du(tbs_ctx *ctx);
int tbs_part_line_res(tbs_ctx *ctx, double *owned_norm);

/* Copies line `line`'s part of the solution (TBS_VEC_SOLUTION) or of the
 * last update (TBS_VEC_UPDATE) to (to_line = 0) or from (to_line = 1) the
 * device buffer d_buf: linesize[line] * 9 doubles, in the line's internal
 * cell order, which depends only on the line's length, so a buffer taken
 * from a line's owner fits the same line's halo copy.  Asynchronous on the
 * context's stream; d_buf may be any address the device can reach. */
#define TBS_VEC_SOLUTION 0
#define TBS_VEC_UPDATE   2
int tbs_part_line_vector(tbs_ctx *ctx, int which, int line, double *d_buf,
                         int to_line);

/* The true-residual check of a partitioned solve: R = rhs + J U of the
 * owned cells from the original blocks and its owned norm in *owned_norm
 * (or, with NULL, kept for tbs_part_owned_norm).  The next
 * tbs_part_solve_du forms its line solves' input from that R (so the
 * sweeps go on from the true residual); a check that ends the solve forms
 * nothing more.  The loop runs it when the global recursive norm meets the
 * tolerance, as tbs_solve does. */
int tbs_part_check(tbs_ctx *ctx, double *owned_norm);

/* The device-clock record of the sweeps' cross-line residual launches
 * (block size 9; every launch, graph-launched ones included): the sum of
 * their durations in microseconds, each from its earliest CTA start to the
 * finish of its last CTA on the GPU's global nanosecond clock, and their
 * number.  reset != 0 starts a new record.  Waits for the context's
 * stream.  No counterpart in the reference (its timing is host-side,
 * src/main.cxx:233-252). */
int tbs_resid_timer(tbs_ctx *ctx, double *total_us, long long *launches, int reset);

/* Waits for the context's stream and reports a device-side failure (a
 * zero pivot, a staging wait that ran out of time) of the launches since
 * the last call that returned a status: the end of a sequence of calls
 * that do not synchronise (tbs_part_line_res with a NULL norm). */
int tbs_sync(tbs_ctx *ctx);

/* The owned norm of the last tbs_part_start / tbs_part_line_res copied to
 * d_out (one double, any address the device can reach), in stream order,
 * without a host synchronisation: the input of a device-side all-reduce.
 * tbs_part_line_res(ctx, NULL) followed by this keeps the sweep loop free
 * of host round trips until the global norm is read. */
int tbs_part_owned_norm(tbs_ctx *ctx, double *d_out);

/* The same for several lines in one launch: lines[0..nlines) (host array
 * of local line indices) packed back to back into d_buf (to_line = 0) or
 * unpacked from it (to_line = 1), each line's span as tbs_part_line_vector
 * gives it.  A halo exchange with one neighbour is one call per side. */
int tbs_part_lines_vector(tbs_ctx *ctx, int which, int nlines, const int *lines,
                          double *d_buf, int to_line);

/* Jacobian::fromDevice (src/Jacobian.cxx:279-290) for the vectors, in the
 * element order of the input (9*nelem doubles each). */
int tbs_get_solution(tbs_ctx *ctx, double *U);
int tbs_get_residual(tbs_ctx *ctx, double *R);
int tbs_get_update(tbs_ctx *ctx, double *dU);

/* ||rhs + J U|| recomputed from the original FP64 blocks, whatever the
 * algorithm (the check behind every reported convergence). */
int tbs_true_residual_norm(tbs_ctx *ctx, double *out);

/* The true-residual check of TBS_ALGO_FP64 solves (on by default, no
 * counterpart in the reference, which prints no residual): 1 on, 0 off. */
int tbs_set_check(tbs_ctx *ctx, int on);

/* The checks of the last solve: *true_norm = ||rhs + J U|| at the last
 * check (-1 when none ran), *checks = checks run, *restarts = checks whose
 * true residual missed the tolerance (the solve went on).  Any output may
 * be NULL. */
int tbs_solve_check(tbs_ctx *ctx, double *true_norm, int *checks, int *restarts);

/* New values of the factored Jacobian's blocks (host pointers, the layout
 * of tbs_set_jacobian) for the residual, keeping the line factorization:
 * the factors of the old values become the preconditioner of the new
 * system (a lagged factorization, as between the time steps of the flow
 * solver the reference serves).  TBS_ALGO_REFERENCE and TBS_ALGO_FP64 (with
 * the true-residual check on) then converge to the new system's solution,
 * TBS_ALGO_MIXED's FP64 outer residual uses the new values.  Resets U to
 * zero (or the starting solution) and R to its residual.  TBS_ALGO_PIJ
 * and line partitions refuse (re-factor); so do, until the next
 * tbs_factor, the TBS_ALGO_FP64 paths that track the residual with the
 * factorization's blocks alone: batches, several right-hand sides, GMRES.
 * No counterpart in the reference, which re-reads and re-factors
 * (src/main.cxx:86-93,180-190). */
int tbs_update_values(tbs_ctx *ctx, const double *jacD, const double *jacO1,
                      const double *jacO2);

/* Device bytes held by the context (replaces
 * gpu.device.memoryAllocated(), src/main.cxx:97-99). */
int tbs_memory_allocated(const tbs_ctx *ctx, size_t *bytes);

/* TBS_ALGO_MIXED: FP32 inner sweeps per FP64 outer refinement step
 * (default 4, range 1..64), the same for every outer step. */
int tbs_set_inner_sweeps(tbs_ctx *ctx, int m);

/* TBS_ALGO_MIXED: `first` inner sweeps in the first outer step of a solve
 * (or of a tbs_sweep sequence after a new rhs, initial solution or
 * factorization), `rest` in the others. */
int tbs_set_inner_schedule(tbs_ctx *ctx, int first, int rest);
int tbs_get_inner_schedule(const tbs_ctx *ctx, int *first, int *rest);

/* Autotuner for TBS_ALGO_MIXED: times a solve to rel_tol on the device for
 * each uniform inner sweep count in {2,3,4,5,6,8,10}, then for first-step
 * counts within 2 of the best and steady counts within 1 of it; keeps the
 * fastest schedule that converges (set in the context) and reports its
 * steady count and its time in ms (tbs_get_inner_schedule gives both). */
int tbs_tune_inner(tbs_ctx *ctx, double rel_tol, int max_sweeps, int *best_m,
                   double *best_ms);

/* Per-kernel CUDA-event timing.  While enabled, every launch is bracketed
 * by events on the launching stream; tbs_profile_read returns, for kernel
 * slot k < *n, its name, launch count and total milliseconds. */
#define TBS_PROFILE_MAX 16
int tbs_profile_enable(tbs_ctx *ctx, int on);
int tbs_profile_reset(tbs_ctx *ctx);
int tbs_profile_read(tbs_ctx *ctx, int *n, const char **names,
                     long long *launches, double *ms);

/* Self-test of the failure path of every staging wait: a kernel waits
 * budget_cycles (clock64) on a copy barrier that nothing completes, gives
 * up and records the timeout in the context's device status, which this
 * call reads like any launch sequence: it returns TBS_ERR_CUDA ("a
 * device-side wait ran out of its time budget") and leaves the context
 * usable.  The kernels' own waits use a budget of 2^31 cycles (about one
 * second).  No copy is issued, so nothing is left in flight. */
int tbs_selftest_timeout(tbs_ctx *ctx, long long budget_cycles);

/* Algorithmic bytes one launch of each kernel moves (reads + writes of
 * every array it must touch once), for the roofline numerator.  The
 * multi-RHS kernels take the group size as a suffix: "multi_thomas/8",
 * "multi_resid/8" (every right-hand side active).  "fast_thomas" and
 * "fast_resid" are the forms the FP64 sweeps of a context run (the line
 * solve adds dU to U); "fast_thomas_dU", "fast_resid_U" and
 * "fast_resid32_U" are the batch engine's forms, whose residual kernels add
 * the update instead. */
int tbs_kernel_bytes(tbs_ctx *ctx, const char *kernel, double *bytes);

/* Linear residual R = rhs + D U + (sum over each cell's interior faces of
 * offJ U_nbr) and its 2-norm for nvar = 9, on device buffers owned by the
 * caller, without
 * allocating device memory -- for callers that cannot call cudaMalloc
 * (a solver whose memory pool owns the GPU, a time loop that must not
 * allocate).  No counterpart in the reference.  Arrays are device pointers
 * in element order (epoint, ef, fc 0-based; jacD, jacO1, jacO2, rhs, U as
 * in the Jacobian file); d_R may be NULL; *norm_out is written on the host
 * (the call synchronises `cuda_stream`, NULL = legacy default stream).
 * Its only work array is a fixed file-scope device array: at most 2,097,152
 * cells (TBS_ERR_ARG beyond), kept by every GPU that loads the library
 * until exit, shared by all calls (calls that overlap on the GPU race).
 * The first call on a device looks up that array's address and should come
 * before any stream capture; the address is kept for the life of the
 * process, so a device or primary-context reset (cudaDeviceReset) after
 * that first call is not supported. */
int tbs_residual_noalloc(int device_id, void *cuda_stream, int nelem,
                         const int *d_epoint, const int *d_ef, const int *d_fc,
                         const double *d_jacD, const double *d_jacO1,
                         const double *d_jacO2, const double *d_rhs,
                         const double *d_U, double *d_R, double *norm_out);

/* ======================================================== batched solves
 * Many independent systems solved together on one GPU (no counterpart in
 * the reference, whose driver solves one system per process).  A batch is
 * built over contexts factored with the same algorithm (TBS_ALGO_FP64 or
 * TBS_ALGO_MIXED) on the same device; each keeps its own blocks, rhs,
 * starting solution (tbs_set_initial) and result, read with
 * tbs_get_solution as after tbs_solve.  tbs_batch_solve runs one CUDA
 * graph launch: every sweep is one persistent Thomas launch over the lines
 * of all systems still above their tolerance, taken from a device work
 * queue (longest lines first by default), one residual launch over their
 * tiles and one launch for the per-system norms; each system stops at its
 * own tolerance or sweep limit.  Each system's iterates, norm history and
 * sweep count are bit-identical to tbs_solve on that context alone.
 * The batch reads the members' device arrays at each solve; re-factoring
 * a member with the same algorithm or giving it a new rhs is allowed,
 * tbs_set_mesh or tbs_destroy on a member is not while the batch lives.
 * Calls on one batch and on its members must not overlap. */
typedef struct tbs_batch tbs_batch;
int tbs_batch_create(tbs_ctx *const *systems, int nsys, tbs_batch **out);
int tbs_batch_destroy(tbs_batch *batch);
const char *tbs_batch_last_error(const tbs_batch *batch);
int tbs_batch_size(const tbs_batch *batch, int *nsys);
/* Launch on `cuda_stream` (not the legacy default stream; NULL: the
 * batch's own stream). */
int tbs_batch_set_stream(tbs_batch *batch, void *cuda_stream);

/* sweeps_out[nsys]; hist_out: nsys rows of (max_sweeps + 1) norms, row s
 * valid up to entry sweeps_out[s]; either may be NULL */
int tbs_batch_solve(tbs_batch *batch, double rel_tol, int max_sweeps,
                    int *sweeps_out, double *hist_out);

/* Shape of the persistent Thomas launch: CTAs (each one line at a time)
 * per SM, bulk-copy ring stages (2..8), line order (0: longest first,
 * 1: mesh order).  TBS_ERR_ARG when the shape does not fit. */
int tbs_batch_set_schedule(tbs_batch *batch, int ctas_per_sm, int stages, int order);
int tbs_batch_get_schedule(const tbs_batch *batch, int *ctas_per_sm, int *stages,
                           int *order);

/* Warps per line of the persistent Thomas launch: 1 (the warp running the
 * line's two chains also issues its staging copies) or 2 (a second warp
 * issues them, so that the chains never stop for it).  Results are
 * bit-identical either way; CTAs per SM are lowered to what fits. */
int tbs_batch_set_warps_per_line(tbs_batch *batch, int warps);
int tbs_batch_get_warps_per_line(const tbs_batch *batch, int *warps);

/* Autotuner: times the persistent Thomas launch over every warps-per-line
 * / CTAs-per-SM / stage count / line order that fits, keeps the fastest
 * and reports it and its time per launch in ms (any output may be NULL;
 * tbs_batch_get_warps_per_line gives the warps). */
int tbs_batch_tune(tbs_batch *batch, int *ctas_per_sm, int *stages, int *order,
                   double *best_ms);

/* TBS_ALGO_MIXED: FP32 inner sweeps per outer step for every member, or
 * a first-step / steady schedule as tbs_set_inner_schedule (default: the
 * first member's setting). */
int tbs_batch_set_inner_sweeps(tbs_batch *batch, int m);
int tbs_batch_set_inner_schedule(tbs_batch *batch, int first, int rest);

/* TBS_ALGO_MIXED: times batched solves to rel_tol under the inner sweep
 * schedules tbs_tune_inner tries, keeps the fastest one with which every
 * member reaches the tolerance, and reports it (outputs may be NULL). */
int tbs_batch_tune_inner(tbs_batch *batch, double rel_tol, int max_sweeps,
                         int *first, int *rest, double *best_ms);

/* Per-kernel CUDA-event timing of batched solves (eager launches while
 * enabled), as tbs_profile_*. */
int tbs_batch_profile_enable(tbs_batch *batch, int on);
int tbs_batch_profile_reset(tbs_batch *batch);
int tbs_batch_profile_read(tbs_batch *batch, int *n, const char **names,
                           long long *launches, double *ms);

/* ================================================================= serving
 * A request loop on one GPU (no counterpart in the reference).  Systems are
 * registered once and stay factored in HBM.  Requests bring 1.. right-hand
 * sides for a system and, optionally, new Jacobian values (same mesh) that
 * re-factor it before the request's solves; the loop runs on a thread of
 * the server.  It admits queued requests in arrival order while their
 * right-hand sides fit the device budget (resident systems plus the
 * vectors of every right-hand side in flight) and the limit on right-hand
 * sides in flight; a request that does not fit holds back the later ones.
 * All admitted right-hand sides are swept together (continuous batching):
 * a request that arrives while others are on the GPU joins them at the
 * next sweep boundary, and each right-hand side leaves when it reaches its
 * tolerance or sweep limit.  Re-factorizations run on a second thread into
 * a spare copy of the system's factors (counted against the budget; when
 * it does not fit, in place once the system's right-hand sides are done),
 * so the right-hand sides already admitted keep sweeping on the current
 * factors; the system's later requests use the new ones.  Every solution
 * is bit-identical to tbs_solve of the same system and right-hand side on
 * its own.
 * The rhs, U_out and new Jacobian arrays stay owned by the caller and must
 * stay valid until tbs_server_wait returns for the request. */
typedef struct tbs_server tbs_server;
/* algo: TBS_ALGO_FP64 or TBS_ALGO_MIXED; device_budget_bytes: systems plus
 * right-hand sides in flight; max_rhs_in_flight >= 1 */
int tbs_server_create(int device_id, int algo, size_t device_budget_bytes,
                      int max_rhs_in_flight, tbs_server **out);
/* finishes the right-hand sides in flight; queued requests fail */
int tbs_server_destroy(tbs_server *srv);
const char *tbs_server_last_error(const tbs_server *srv);
/* sweeps per graph launch at most (default 4): how long a new arrival can
 * wait for the next sweep boundary */
int tbs_server_set_chunk(tbs_server *srv, int sweeps);
/* Lanes, each its own loop thread, factor thread, engine and streams,
 * sharing the budget and the limit on right-hand sides in flight, so that
 * small systems are not held to the pace of large ones.  A system sweeps in
 * lane k = how many of the ascending splits its cell count reaches.
 * Default: three lanes, splits 262,144 and 1,048,576 cells.
 * tbs_server_set_lanes: two lanes split at split_cells (0: one lane).
 * tbs_server_set_lane_splits: up to three splits (four lanes).  Set before
 * any system is added. */
int tbs_server_set_lanes(tbs_server *srv, long long split_cells);
int tbs_server_set_lane_splits(tbs_server *srv, const long long *splits, int n);
/* uploads and factors a system (blocking); arrays as tbs_set_mesh and
 * tbs_set_jacobian */
int tbs_server_add_system(tbs_server *srv, int nvar, int nelem, int nintface, int eftot,
                          int nline, int nlineelem, const int *epoint, const int *ef,
                          const int *fc, const int *linesize, const int *linepoint,
                          const int *lines, const int *lineface, const double *jacD,
                          const double *jacO1, const double *jacO2, int *system_id);
/* device bytes the system holds and one right-hand side of it needs in
 * flight with a sweep limit of max_sweeps (the admission footprint) */
int tbs_server_system_bytes(tbs_server *srv, int system_id, int max_sweeps,
                            size_t *resident, size_t *per_rhs);
/* rhs and U_out: nrhs x 9*nelem doubles, element order; jacD/jacO1/jacO2
 * NULL keeps the factors.  Returns at once with the request's id. */
int tbs_server_submit(tbs_server *srv, int system_id, int nrhs, const double *rhs,
                      double *U_out, double rel_tol, int max_sweeps, const double *jacD,
                      const double *jacO1, const double *jacO2, long long *request_id);
int tbs_server_poll(tbs_server *srv, long long request_id, int *done);
/* blocks until the request is done, then forgets it: sweeps[nrhs],
 * rel_residual[nrhs] (final / initial norm), latency (submit to done) and
 * queueing time (submit to admission) in ms; any output may be NULL */
int tbs_server_wait(tbs_server *srv, long long request_id, int *sweeps,
                    double *rel_residual, double *latency_ms, double *queue_ms);
/* stats[0..n): requests done, right-hand sides done, graph launches,
 * re-factorizations, peak right-hand sides in flight, peak bytes of
 * right-hand sides in flight, bytes of resident systems, requests queued,
 * then the loop thread's microseconds spent starting right-hand sides,
 * rebuilding the member set, in graph launches, and reading results back */
int tbs_server_stats(tbs_server *srv, long long *stats, int n);

/* Library version string. */
const char *tbs_version(void);

#ifdef __cplusplus
}
#endif
#endif /* TRIBLOCK_H */

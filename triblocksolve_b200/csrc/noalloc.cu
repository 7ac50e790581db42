/*
 * noalloc.cu -- tbs_residual_noalloc: the linear residual R = rhs + J U of
 * a 9x9-block line Jacobian and its 2-norm, computed on device buffers the
 * caller owns, without allocating any device memory.
 *
 * Some callers cannot allocate: a flow solver that hands the whole GPU to
 * its own memory pool (and forbids cudaMalloc behind its back), or a time
 * loop that must not allocate between steps.  They still need the residual
 * norm of the current iterate to steer their nonlinear iteration.  The
 * context API (tbs_create ... tbs_true_residual_norm) allocates its work
 * arrays with cudaMalloc; this entry point keeps its only work array -- one
 * partial sum per CTA, the final norm and the last-CTA ticket -- in a
 * file-scope __device__ array of fixed size instead.
 *
 * Limits and sharing:
 *   - at most NOALLOC_MAX_CELLS cells (NOALLOC_MAX_BLOCKS CTAs of 32 cells);
 *     larger meshes are rejected with TBS_ERR_ARG before any launch;
 *   - every GPU that loads the library holds the array (~512 KiB) until the
 *     process exits;
 *   - every call shares the array, which keeps the last call's contents:
 *     the ticket is cleared at the start of each call, and calls whose work
 *     overlaps on the GPU (different streams, or different host threads)
 *     race on it, so callers must serialise them;
 *   - the first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress with that device current); that first call
 *     should come before any stream capture.  The address is kept for the
 *     life of the process: resetting the device or its primary context
 *     (cudaDeviceReset) after the first call is not supported.
 */
#include "tbs_internal.hxx"

#include <cuda_runtime.h>

#include <mutex>
#include <string>

namespace tbs {

constexpr int NOALLOC_THREADS = 288;            /* 9 threads per cell */
constexpr int NOALLOC_CELLS_PER_BLOCK = NOALLOC_THREADS / 9;
constexpr int NOALLOC_MAX_BLOCKS = 65536;
constexpr long long NOALLOC_MAX_CELLS = (long long)NOALLOC_MAX_BLOCKS * NOALLOC_CELLS_PER_BLOCK;
constexpr int NOALLOC_NORM = NOALLOC_MAX_BLOCKS;       /* slot of the final norm */
constexpr int NOALLOC_TICKET = NOALLOC_MAX_BLOCKS + 1; /* slot of the CTA ticket */

/* partial sums [0, MAX_BLOCKS), norm, ticket (an unsigned in a double slot) */
static __device__ __align__(256) double tbs_noalloc_scratch[NOALLOC_MAX_BLOCKS + 2];

/* R(e) = rhs(e) + D_e U_e + sum over the faces of e of offJ U_nbr, with the
 * face rule of src/okl/linesmoothLU_TriBlock_v3.okl:299-328, one thread per
 * (cell, row); the same arithmetic as the context path's residual kernel. */
__global__ void __launch_bounds__(NOALLOC_THREADS) noalloc_resid_kernel(
    int nelem, const int *__restrict__ epoint, const int *__restrict__ ef,
    const int *__restrict__ fc, const double *__restrict__ D, const double *__restrict__ O1,
    const double *__restrict__ O2, const double *__restrict__ rhs, const double *__restrict__ U,
    double *__restrict__ R, double *scratch) {
    const int le = threadIdx.x / 9;
    const int i = threadIdx.x - le * 9;
    const int e = blockIdx.x * NOALLOC_CELLS_PER_BLOCK + le;
    double sq = 0.0;
    if (e < nelem) {
        const double *u = U + (size_t)e * 9;
        const double *dr = D + (size_t)e * 81 + i;
        double a0 = dr[0] * u[0], a1 = dr[9] * u[1], a2 = dr[18] * u[2];
        a0 += dr[27] * u[3];
        a1 += dr[36] * u[4];
        a2 += dr[45] * u[5];
        a0 += dr[54] * u[6];
        a1 += dr[63] * u[7];
        a2 += dr[72] * u[8];
        for (int k2 = epoint[e]; k2 < epoint[e + 1]; ++k2) {
            const int f = ef[k2];
            if (f >= 0) {
                const int e1 = fc[2 * f], e2 = fc[2 * f + 1];
                const double *o = ((e == e1) ? O2 : O1) + (size_t)f * 81 + i;
                const double *un = U + (size_t)((e == e1) ? e2 : e1) * 9;
                a0 += o[0] * un[0];
                a1 += o[9] * un[1];
                a2 += o[18] * un[2];
                a0 += o[27] * un[3];
                a1 += o[36] * un[4];
                a2 += o[45] * un[5];
                a0 += o[54] * un[6];
                a1 += o[63] * un[7];
                a2 += o[72] * un[8];
            }
        }
        const double r = rhs[(size_t)e * 9 + i] + (a0 + (a1 + a2));
        if (R) R[(size_t)e * 9 + i] = r;
        sq = r * r;
    }
    __shared__ double red[NOALLOC_THREADS / 32];
    __shared__ unsigned ticket;
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
    __syncthreads();
    unsigned *tk = reinterpret_cast<unsigned *>(scratch + NOALLOC_TICKET);
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < NOALLOC_THREADS / 32; ++w) tot += red[w];
        scratch[blockIdx.x] = tot;
        __threadfence();
        ticket = atomicAdd(tk, 1u);
    }
    __syncthreads();
    if (ticket != gridDim.x - 1) return;
    /* last CTA: fixed-order sum of all partials */
    __threadfence();
    double acc = 0.0;
    for (unsigned t = threadIdx.x; t < gridDim.x; t += blockDim.x) acc += __ldcg(scratch + t);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < NOALLOC_THREADS / 32; ++w) tot += red[w];
        scratch[NOALLOC_NORM] = sqrt(tot);
        *tk = 0u;
    }
}

/* device address of the scratch array, looked up once per device */
static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[64];

static int noalloc_scratch(int device, double **out) {
    if (device < 0 || device >= 64) {
        set_thread_error("tbs_residual_noalloc: device id out of range");
        return TBS_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        double *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, tbs_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_thread_error(std::string("tbs_residual_noalloc: cudaGetSymbolAddress failed: ") +
                             cudaGetErrorString(e));
            return TBS_ERR_CUDA;
        }
        g_noalloc_ptr[device] = p;
    }
    *out = g_noalloc_ptr[device];
    return TBS_OK;
}

}  // namespace tbs

using namespace tbs;

extern "C" int tbs_residual_noalloc(int device_id, void *cuda_stream, int nelem,
                                    const int *d_epoint, const int *d_ef, const int *d_fc,
                                    const double *d_jacD, const double *d_jacO1,
                                    const double *d_jacO2, const double *d_rhs,
                                    const double *d_U, double *d_R, double *norm_out) {
    if (nelem < 1) {
        set_thread_error("tbs_residual_noalloc: nelem must be >= 1");
        return TBS_ERR_ARG;
    }
    if ((long long)nelem > NOALLOC_MAX_CELLS) {
        set_thread_error("tbs_residual_noalloc: " + std::to_string(nelem) +
                         " cells exceed the fixed scratch limit of " +
                         std::to_string(NOALLOC_MAX_CELLS) + " cells");
        return TBS_ERR_ARG;
    }
    if (!d_epoint || !d_ef || !d_fc || !d_jacD || !d_jacO1 || !d_jacO2 || !d_rhs || !d_U ||
        !norm_out) {
        set_thread_error("tbs_residual_noalloc: null argument");
        return TBS_ERR_ARG;
    }
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) {
        cudaGetLastError();
        set_thread_error("tbs_residual_noalloc: no CUDA device");
        return TBS_ERR_CUDA;
    }
    int rc = TBS_OK;
    cudaError_t e = cudaSetDevice(device_id);
    double *scratch = nullptr;
    if (e == cudaSuccess) rc = noalloc_scratch(device_id, &scratch);
    if (e == cudaSuccess && rc == TBS_OK) {
        cudaStream_t st = (cudaStream_t)cuda_stream;
        const int blocks = (nelem + NOALLOC_CELLS_PER_BLOCK - 1) / NOALLOC_CELLS_PER_BLOCK;
        /* the ticket must start at zero; the partials are overwritten */
        e = cudaMemsetAsync(scratch + NOALLOC_TICKET, 0, sizeof(double), st);
        if (e == cudaSuccess) {
            noalloc_resid_kernel<<<blocks, NOALLOC_THREADS, 0, st>>>(
                nelem, d_epoint, d_ef, d_fc, d_jacD, d_jacO1, d_jacO2, d_rhs, d_U, d_R, scratch);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(norm_out, scratch + NOALLOC_NORM, sizeof(double),
                                cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) {
        set_thread_error(std::string("tbs_residual_noalloc: ") + cudaGetErrorString(e));
        rc = TBS_ERR_CUDA;
    }
    cudaSetDevice(prev);
    return rc;
}

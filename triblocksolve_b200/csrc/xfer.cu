/* Host <-> device transfers that stay off the copy engine.
 *
 * Every cudaMemcpyAsync between host and device, whatever its stream, waits
 * in the copy engine's queue behind the copies issued before it (measured
 * on B200: a 32-byte state read-back issued during a 5 GB Jacobian upload
 * returned after the whole upload, 91 ms later).  Paths whose latency
 * matters -- a solve's control words, the batch engine's control block and
 * member tables, a served request's right-hand side and solution -- move
 * their bytes with the kernels below instead: the SMs read or write pinned
 * host memory through its device address, or take a small value as a
 * kernel parameter.  Bulk uploads (Jacobians) keep the copy engine. */
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "tbs_internal.hxx"

namespace {

template <typename W>
__global__ void xfer_copy_kernel(const W *__restrict__ src, W *__restrict__ dst, long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        dst[t] = src[t];
}

/* one job per grid row: 16-byte words where both addresses allow, 4-byte
 * words for the rest */
__global__ void xfer_jobs_kernel(const XferJob *__restrict__ jobs) {
    __shared__ XferJob sj; /* the job table may be host memory: read it once per CTA */
    if (threadIdx.x == 0) sj = jobs[blockIdx.y];
    __syncthreads();
    const XferJob j = sj;
    const char *src = reinterpret_cast<const char *>(j.src);
    char *dst = reinterpret_cast<char *>(j.dst);
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long head = 0;
    if (((j.src | j.dst) & 15) == 0) {
        const long long n16 = (long long)(j.bytes / 16);
        const uint4 *s = reinterpret_cast<const uint4 *>(src);
        uint4 *d = reinterpret_cast<uint4 *>(dst);
        for (long long t = t0; t < n16; t += stride) d[t] = s[t];
        head = n16 * 16;
    }
    const long long n4 = (long long)((j.bytes - head) / 4);
    const unsigned *s4 = reinterpret_cast<const unsigned *>(src + head);
    unsigned *d4 = reinterpret_cast<unsigned *>(dst + head);
    for (long long t = t0; t < n4; t += stride) d4[t] = s4[t];
}

struct Blob {
    unsigned char b[kXferPutMax];
};

__global__ void xfer_put_kernel(unsigned char *dst, Blob v, int bytes) {
    for (int t = threadIdx.x; t < bytes; t += blockDim.x) dst[t] = v.b[t];
}

int blocks_for(long long words, int max_blocks) {
    return (int)std::min<long long>(std::max<long long>((words + 255) / 256, 1), max_blocks);
}

}  // namespace

int xfer_copy(cudaStream_t st, const void *src, void *dst, size_t bytes, int max_blocks) {
    if (bytes == 0) return 0;
    const uintptr_t a = (uintptr_t)src | (uintptr_t)dst;
    if (bytes % 4 != 0 || a % 4 != 0) return (int)cudaErrorMisalignedAddress;
    if (max_blocks < 1) max_blocks = 4 * 148;
    const size_t w = (a % 16 == 0 && bytes % 16 == 0) ? 16 : (a % 8 == 0 && bytes % 8 == 0) ? 8 : 4;
    const long long n = (long long)(bytes / w);
    const int blocks = blocks_for(n, max_blocks);
    if (w == 16)
        xfer_copy_kernel<uint4><<<blocks, 256, 0, st>>>(static_cast<const uint4 *>(src),
                                                        static_cast<uint4 *>(dst), n);
    else if (w == 8)
        xfer_copy_kernel<unsigned long long><<<blocks, 256, 0, st>>>(
            static_cast<const unsigned long long *>(src), static_cast<unsigned long long *>(dst), n);
    else
        xfer_copy_kernel<unsigned><<<blocks, 256, 0, st>>>(static_cast<const unsigned *>(src),
                                                           static_cast<unsigned *>(dst), n);
    return (int)cudaGetLastError();
}

int xfer_put(cudaStream_t st, void *dst, const void *value, size_t bytes) {
    if (bytes == 0) return 0;
    if (bytes > (size_t)kXferPutMax) return (int)cudaErrorInvalidValue;
    Blob v;
    std::memset(&v, 0, sizeof(v));
    std::memcpy(v.b, value, bytes);
    xfer_put_kernel<<<1, 128, 0, st>>>(static_cast<unsigned char *>(dst), v, (int)bytes);
    return (int)cudaGetLastError();
}

int xfer_jobs(cudaStream_t st, const XferJob *jobs_dev, int njobs, size_t max_bytes) {
    if (njobs <= 0) return 0;
    if (njobs > 65535) return (int)cudaErrorInvalidValue;
    const int bx = blocks_for((long long)(max_bytes / 16), 32);
    xfer_jobs_kernel<<<dim3(bx, njobs), 256, 0, st>>>(jobs_dev);
    return (int)cudaGetLastError();
}

void *xfer_device_view(const void *host) {
    if (!host) return nullptr;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, host) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return (a.type == cudaMemoryTypeHost && a.devicePointer) ? a.devicePointer : nullptr;
}

int xfer_to_host(cudaStream_t st, void *dst, const void *src, size_t bytes, int max_blocks) {
    void *dv = xfer_device_view(dst);
    if (dv && bytes % 4 == 0 && ((uintptr_t)dv | (uintptr_t)src) % 4 == 0)
        return xfer_copy(st, src, dv, bytes, max_blocks);
    return (int)cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
}

int xfer_to_device(cudaStream_t st, void *dst, const void *src, size_t bytes, int max_blocks) {
    const void *sv = xfer_device_view(src);
    if (sv && bytes % 4 == 0 && ((uintptr_t)sv | (uintptr_t)dst) % 4 == 0)
        return xfer_copy(st, sv, dst, bytes, max_blocks);
    return (int)cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
}

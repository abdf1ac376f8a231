/*
 * dsh_noalloc.cu — residual and L2 misfit without any device allocation.
 *
 * Same arithmetic and reduction order as the residual step of dsh_gradient
 * (residual time-reversed as the adjoint source, first observed sample
 * replaced by the synthetic one, per-block double partial sums reduced in a
 * fixed order), but the partial sums live in a file-scope __device__ array
 * instead of context memory, so a call allocates nothing.
 *
 * The array is a single fixed buffer per GPU that loads this library: every
 * call on a device reuses it and it keeps the previous call's contents (each
 * call overwrites every partial it later reads, so nothing needs clearing).
 * Calls that overlap on the GPU (concurrent streams, or threads sharing a
 * device) race on it and must be serialised by the caller.
 */
#include "dsh.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

namespace {

constexpr int NA_BLOCKS = 296;            /* blocks per shot (same partition as dsh_gradient) */
constexpr int NA_THREADS = 256;
constexpr int NA_MAX_DEVICES = 64;

/* static scratch: NA_BLOCKS double partial sums per shot, for up to
 * DSH_NOALLOC_MAX_SHOTS shots (296 * 64 * 8 B = 151,552 B per device) */
static __device__ __align__(256) double g_partials[DSH_NOALLOC_MAX_SHOTS * NA_BLOCKS];

/* host-side device addresses of g_partials per device.  The address is
 * looked up again on every call whose stream is not capturing (cheap once
 * the module is loaded), so a device reset between calls, which unloads the
 * module, cannot leave a stale address behind; a capturing call uses the
 * address an earlier call on that device found. */
std::mutex g_mu;
double *g_partials_dev[NA_MAX_DEVICES] = {};

int partials_address(cudaStream_t st, double **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) return DSH_ERR_CUDA;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return DSH_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if (cs != cudaStreamCaptureStatusNone && !g_partials_dev[dev]) {
        fprintf(stderr, "dsh_residual_noalloc: the first call on device %d must come before any stream capture\n", dev);
        return DSH_ERR_STATE;
    }
    if (cs == cudaStreamCaptureStatusNone) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_partials);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "dsh_residual_noalloc: cudaGetSymbolAddress failed on device %d (%s)\n", dev,
                    cudaGetErrorString(e));
            return DSH_ERR_CUDA;
        }
        g_partials_dev[dev] = static_cast<double *>(p);
    }
    *out = g_partials_dev[dev];
    return DSH_OK;
}

/* residual of shot s (blockIdx.y): syn, obs, res are [ntr][nt];
 * res[r][t-1] = syn[r][nt-t] - obs[r][nt-t], the first observed sample being
 * replaced by the synthetic one (src/calc_res.c:115,172-177) */
__global__ void residual_static_kernel(int nt, int ntr, const float *syn, const float *obs, float *res, double *part)
{
    const int s = blockIdx.y;
    const long long n = (long long)ntr * nt;
    const float *sy = syn + (long long)s * n;
    const float *ob = obs + (long long)s * n;
    float *rs = res + (long long)s * n;
    double acc = 0.0;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx / nt);
        const int t = (int)(idx % nt) + 1;
        const int tf = nt - t + 1;
        const float a = sy[(long long)r * nt + (tf - 1)];
        const float b = (tf == 1) ? a : ob[(long long)r * nt + (tf - 1)];
        const float v = a - b;
        rs[(long long)r * nt + (t - 1)] = v;
        acc += (double)v * (double)v;
    }
    __shared__ double sh[NA_THREADS];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(long long)s * gridDim.x + blockIdx.x] = sh[0];
}

__global__ void reduce_static_kernel(const double *part, int nparts, double *l2)
{
    const int s = blockIdx.x;
    __shared__ double sh[NA_THREADS];
    double acc = 0.0;
    for (int k = threadIdx.x; k < nparts; k += blockDim.x) acc += part[(long long)s * nparts + k];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) l2[s] = sh[0];
}

/* whether the float ranges [a, a+n) and [b, b+n) share any element */
bool overlap(const float *a, const float *b, long long n)
{
    const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b, len = (uintptr_t)n * sizeof(float);
    return x < y + len && y < x + len;
}

}  // namespace

extern "C" int dsh_residual_noalloc(int nshots, int ntr, int nt, const float *syn, const float *obs, float *res,
                                    double *l2, void *stream)
{
    if (nshots < 1 || ntr < 1 || nt < 1 || !syn || !obs || !res || !l2) return DSH_ERR_PARAM;
    if (nshots > DSH_NOALLOC_MAX_SHOTS) {
        fprintf(stderr, "dsh_residual_noalloc: %d shots exceed the static scratch capacity of %d shots per call\n",
                nshots, DSH_NOALLOC_MAX_SHOTS);
        return DSH_ERR_PARAM;
    }
    /* each thread writes res[r][t-1] from syn/obs sample nt-t, which another
       thread may be writing: the residual cannot be formed in place */
    const long long total = (long long)nshots * ntr * nt;
    if (overlap(res, syn, total) || overlap(res, obs, total)) {
        fprintf(stderr, "dsh_residual_noalloc: res must not overlap syn or obs\n");
        return DSH_ERR_PARAM;
    }
    /* an error left by earlier, unrelated work on this device is reported as
       such, not as a failure of these launches */
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "dsh_residual_noalloc: a CUDA error from earlier work was pending (%s); nothing launched\n",
                cudaGetErrorString(e));
        return DSH_ERR_CUDA;
    }
    cudaStream_t st = (cudaStream_t)stream;
    double *part = nullptr;
    int rc = partials_address(st, &part);
    if (rc != DSH_OK) return rc;
    residual_static_kernel<<<dim3(NA_BLOCKS, nshots), NA_THREADS, 0, st>>>(nt, ntr, syn, obs, res, part);
    if ((e = cudaGetLastError()) != cudaSuccess) {
        fprintf(stderr, "dsh_residual_noalloc: residual launch failed (%s)\n", cudaGetErrorString(e));
        return DSH_ERR_CUDA;
    }
    reduce_static_kernel<<<nshots, NA_THREADS, 0, st>>>(part, NA_BLOCKS, l2);
    if ((e = cudaGetLastError()) != cudaSuccess) {
        fprintf(stderr, "dsh_residual_noalloc: reduction launch failed (%s)\n", cudaGetErrorString(e));
        return DSH_ERR_CUDA;
    }
    return DSH_OK;
}

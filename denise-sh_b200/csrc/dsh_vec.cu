/*
 * dsh_vec.cu — the FWI loop's vector steps on the device, so that a gradient
 * the engine left in HBM (dsh_gradient_device) can become a search direction
 * without a round trip through host memory:
 *   dsh_lbfgs_direction_device  two-loop recursion (src/LBFGS.c:12-95)
 *   dsh_pcg_direction_device    conjugate-gradient direction per parameter
 *                               class (src/PCG.c:10-107)
 * The arithmetic is that of the host versions in dsh_fwi.c (dsh_lbfgs_direction,
 * dsh_pcg_direction) except the order of the dot-product sums: every dot
 * product is a double sum over a fixed partition (VB blocks of VT threads,
 * grid-stride slices, then a fixed tree), so a result does not depend on the
 * launch or the device, and it agrees with the host's to float rounding.
 * Scalars (rho, alpha, gamma, beta) stay in the caller's workspace on the
 * device; nothing is allocated and nothing is copied to the host.
 */
#include "dsh.h"
#include "dsh_fwi.h"

#include <cuda_runtime.h>

#include <cstdio>

namespace {

constexpr int VB = 296;        /* blocks of every partial reduction (2 x 148 SMs) */
constexpr int VT = 256;

/* workspace layout (doubles) */
constexpr int W_PART = 0;                  /* VB partials */
constexpr int W_PART2 = VB;                /* VB partials of a second sum */
constexpr int W_SCAL = 2 * VB;             /* scalars: gamma, beta, spare */
constexpr int W_ARR = 2 * VB + 8;          /* rho[count], alpha[count] | beta[nclass] */

__device__ double block_sum(double v)
{
    __shared__ double sh[VT];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = VT / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();                      /* every thread has read sh[0] before a next call writes it */
    return r;
}

/* part[b] = sum of a[i] * b[i] over block b's grid-stride slice */
__global__ void __launch_bounds__(VT) dot_part(long long n, const float *a, const float *b, double *part)
{
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * VT + threadIdx.x; i < n; i += (long long)VB * VT)
        acc += (double)a[i] * (double)b[i];
    const double s = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__device__ double sum_parts(const double *part)
{
    double acc = 0.0;
    for (int k = threadIdx.x; k < VB; k += VT) acc += part[k];
    return block_sum(acc);
}

/* rho[k] = 1 / (y_k . s_k), or 0 when that product is 0 */
__global__ void __launch_bounds__(VT) set_rho(const double *part, double *rho)
{
    const double ys = sum_parts(part);
    if (threadIdx.x == 0) *rho = fabs(ys) > 0.0 ? 1.0 / ys : 0.0;
}

/* alpha = rho * (s . r) */
__global__ void __launch_bounds__(VT) set_alpha(const double *part, const double *rho, double *alpha)
{
    const double sr = sum_parts(part);
    if (threadIdx.x == 0) *alpha = *rho * sr;
}

/* gamma = (y.s) / (y.y) of the newest pair, 1 when y.y is 0 */
__global__ void __launch_bounds__(VT) set_gamma(const double *part_yy, const double *part_ys, double *gamma)
{
    const double yy = sum_parts(part_yy);
    const double ys = sum_parts(part_ys);
    if (threadIdx.x == 0) *gamma = yy > 0.0 ? ys / yy : 1.0;
}

/* coef = alpha[k] - rho[k] * (y . r) */
__global__ void __launch_bounds__(VT) set_coef2(const double *part, const double *rho, const double *alpha, double *coef)
{
    const double yr = sum_parts(part);
    if (threadIdx.x == 0) *coef = *alpha - *rho * yr;
}

/* r = (float)(r - alpha * y) */
__global__ void __launch_bounds__(VT) sub_scaled(long long n, const double *alpha, const float *y, float *r)
{
    const double a = *alpha;
    for (long long i = (long long)blockIdx.x * VT + threadIdx.x; i < n; i += (long long)gridDim.x * VT)
        r[i] = (float)((double)r[i] - a * (double)y[i]);
}

/* r = (float)(gamma * r) */
__global__ void __launch_bounds__(VT) scale(long long n, const double *gamma, float *r)
{
    const double g = *gamma;
    for (long long i = (long long)blockIdx.x * VT + threadIdx.x; i < n; i += (long long)gridDim.x * VT)
        r[i] = (float)(g * (double)r[i]);
}

/* r = (float)(r + s * coef) */
__global__ void __launch_bounds__(VT) add_scaled(long long n, const double *coef, const float *s, float *r)
{
    const double c = *coef;
    for (long long i = (long long)blockIdx.x * VT + threadIdx.x; i < n; i += (long long)gridDim.x * VT)
        r[i] = (float)((double)r[i] + (double)s[i] * c);
}

/* partial numerator and denominator of the PCG beta (src/PCG.c:25-83) */
__global__ void __launch_bounds__(VT) pcg_part(int kind, long long n, const float *a, const float *b, const float *d,
                                               double *part_num, double *part_den)
{
    double num = 0.0, den = 0.0;
    for (long long i = (long long)blockIdx.x * VT + threadIdx.x; i < n; i += (long long)VB * VT) {
        const double x = a[i], y = b[i], z = d[i];
        switch (kind) {
        case 1: num += x * x; den += y * y; break;                 /* Fletcher-Reeves */
        case 2: num += x * (x - y); den += y * y; break;           /* Polak-Ribiere */
        case 3: num += -x * (x - y); den += z * (x - y); break;    /* Hestenes-Stiefel */
        default: num += -x * x; den += z * (x - y); break;         /* Dai-Yuan */
        }
    }
    const double sn = block_sum(num);
    const double sd = block_sum(den);
    if (threadIdx.x == 0) {
        part_num[blockIdx.x] = sn;
        part_den[blockIdx.x] = sd;
    }
}

/* beta = num / den as a float (0 when den is 0; Polak-Ribiere resets a negative beta) */
__global__ void __launch_bounds__(VT) set_beta(int kind, const double *part_num, const double *part_den, float *beta)
{
    const double num = sum_parts(part_num);
    const double den = sum_parts(part_den);
    if (threadIdx.x == 0) {
        float b = 0.0f;
        if ((float)den != 0.0f) b = (float)(num / den);
        if (kind == 2 && b < 0.0f) b = 0.0f;
        *beta = b;
    }
}

/* dir = g_new + beta * dir (float, src/PCG.c:88-102) */
__global__ void __launch_bounds__(VT) pcg_update(long long n, const float *beta, const float *a, float *d)
{
    const float b = *beta;
    for (long long i = (long long)blockIdx.x * VT + threadIdx.x; i < n; i += (long long)gridDim.x * VT)
        d[i] = a[i] + b * d[i];
}

int launch_ok(const char *what)
{
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return DSH_OK;
    fprintf(stderr, "%s: launch failed (%s)\n", what, cudaGetErrorString(e));
    return DSH_ERR_CUDA;
}

}  // namespace

extern "C" long long dsh_vec_work_doubles(int count)
{
    if (count < 0 || count > 64) return -1;
    return (long long)W_ARR + 2LL * (count > DSH_PCG_MAX_CLASSES ? count : DSH_PCG_MAX_CLASSES);
}

extern "C" int dsh_lbfgs_direction_device(long long n, int count, const float *S, const float *Y, const float *q,
                                          float *r, double *work, void *stream)
{
    if (n <= 0 || count < 0 || count > 64 || !q || !r || !work || (count > 0 && (!S || !Y))) return DSH_ERR_PARAM;
    cudaStream_t st = (cudaStream_t)stream;
    if (r != q && cudaMemcpyAsync(r, q, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return DSH_ERR_CUDA;
    if (count == 0) return launch_ok("dsh_lbfgs_direction_device");
    double *part = work + W_PART, *part2 = work + W_PART2, *gamma = work + W_SCAL, *coef = work + W_SCAL + 1;
    double *rho = work + W_ARR, *alpha = work + W_ARR + count;
    const int gb = VB;
    for (int k = 0; k < count; k++) {
        dot_part<<<VB, VT, 0, st>>>(n, Y + (long long)k * n, S + (long long)k * n, part);
        set_rho<<<1, VT, 0, st>>>(part, rho + k);
    }
    for (int k = count - 1; k >= 0; k--) {            /* newest to oldest (src/LBFGS.c:56-70) */
        const float *s = S + (long long)k * n, *y = Y + (long long)k * n;
        dot_part<<<VB, VT, 0, st>>>(n, s, r, part);
        set_alpha<<<1, VT, 0, st>>>(part, rho + k, alpha + k);
        sub_scaled<<<gb, VT, 0, st>>>(n, alpha + k, y, r);
    }
    const float *sn = S + (long long)(count - 1) * n, *yn = Y + (long long)(count - 1) * n;
    dot_part<<<VB, VT, 0, st>>>(n, yn, yn, part);
    dot_part<<<VB, VT, 0, st>>>(n, yn, sn, part2);
    set_gamma<<<1, VT, 0, st>>>(part, part2, gamma);   /* initial inverse Hessian (src/LBFGS.c:30-38) */
    scale<<<gb, VT, 0, st>>>(n, gamma, r);
    for (int k = 0; k < count; k++) {                 /* oldest to newest (src/LBFGS.c:78-92) */
        const float *s = S + (long long)k * n, *y = Y + (long long)k * n;
        dot_part<<<VB, VT, 0, st>>>(n, y, r, part);
        set_coef2<<<1, VT, 0, st>>>(part, rho + k, alpha + k, coef);
        add_scaled<<<gb, VT, 0, st>>>(n, coef, s, r);
    }
    return launch_ok("dsh_lbfgs_direction_device");
}

extern "C" int dsh_pcg_direction_device(long long n, int nclass, const float *g_new, const float *g_old, float *dir,
                                        int beta_kind, float *beta_dev, double *work, void *stream)
{
    if (n <= 0 || nclass < 1 || nclass > DSH_PCG_MAX_CLASSES || !g_new || !g_old || !dir || !work || beta_kind < 1 ||
        beta_kind > 4)
        return DSH_ERR_PARAM;
    cudaStream_t st = (cudaStream_t)stream;
    float *beta = beta_dev ? beta_dev : reinterpret_cast<float *>(work + W_ARR);
    for (int k = 0; k < nclass; k++) {                /* every beta from the old direction first */
        pcg_part<<<VB, VT, 0, st>>>(beta_kind, n, g_new + (long long)k * n, g_old + (long long)k * n,
                                    dir + (long long)k * n, work + W_PART, work + W_PART2);
        set_beta<<<1, VT, 0, st>>>(beta_kind, work + W_PART, work + W_PART2, beta + k);
    }
    for (int k = 0; k < nclass; k++)
        pcg_update<<<VB, VT, 0, st>>>(n, beta + k, g_new + (long long)k * n, dir + (long long)k * n);
    return launch_ok("dsh_pcg_direction_device");
}

/*
 * dsh_post.cu — processing around the gradient on the device: the
 * SPATFILTER=3 Gaussian smoothing of src/gauss_filt.c (src/smooth_grad.c:27-29),
 * the application of the gradient tapers (src/taper_grad.c; coefficients from
 * dsh_taper.c) and the Butterworth filtering of source signals and traces of the
 * multi-scale workflow stages (src/timedomain_filt.c, libcseife).
 * Each output point sums the (2h+1)^2 taps of the edge-replicated gradient
 * in the reference's order (ii outer, jj inner) in FP32 without contraction,
 * so it is bit-identical to the reference's loop (with its normalising sum
 * started at 0).
 */
#include "dsh.h"
#include "dsh_setup.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

namespace {

constexpr int GAUSS_MAX = 45;                 /* largest filter length (odd) */

struct GaussW {
    float w[GAUSS_MAX * GAUSS_MAX];
};

__global__ void gauss_filt_kernel(int nx, int ny, int hfs, const __grid_constant__ GaussW k, const float *in,
                                  float *out)
{
    const int n = 2 * hfs + 1;
    const long long total = (long long)nx * ny;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nx) + 1, j = (int)(idx / nx) + 1;
        float conv = 0.0f;
        for (int ii = -hfs; ii <= hfs; ii++) {
            int ix = i + ii;
            ix = ix < 1 ? 1 : ix > nx ? nx : ix;
            for (int jj = -hfs; jj <= hfs; jj++) {
                int jy = j + jj;
                jy = jy < 1 ? 1 : jy > ny ? ny : jy;
                conv += __ldg(in + (long long)(jy - 1) * nx + (ix - 1)) * k.w[(jj + hfs) * n + (ii + hfs)];
            }
        }
        out[idx] = conv;
    }
}

struct IIRChain {
    int n;
    double c[9][5];                  /* f0, f1, f2, g1, g2 per section */
};

/* [ntr][ns] float -> [ns][ntr] double; the highpass first subtracts each
 * trace's first sample (cseife.c:139-144) */
__global__ void iir_load(const float *d, int ntr, int ns, int highpass, double *x)
{
    const long long total = (long long)ntr * ns;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(idx / ntr), t = (int)(idx % ntr);
        double v = (double)d[(long long)t * ns + j];
        if (highpass) v -= (double)d[(long long)t * ns];
        x[idx] = v;
    }
}

/* the recursive sections of one trace per thread (cseife_rekfl.c:62-73),
 * in place, samples [ns][ntr] so neighbouring threads touch neighbouring words */
__global__ void iir_run(double *x, int ntr, int ns, const __grid_constant__ IIRChain ch)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntr) return;
    for (int s = 0; s < ch.n; s++) {
        const double f0 = ch.c[s][0], f1 = ch.c[s][1], f2 = ch.c[s][2], g1 = ch.c[s][3], g2 = ch.c[s][4];
        double xa = 0., xaa = 0., ya = 0., yaa = 0.;
        for (int j = 0; j < ns; j++) {
            double *p = x + (long long)j * ntr + t;
            const double xn = *p;
            const double y = f0 * xn + f1 * xa + f2 * xaa + g1 * ya + g2 * yaa;
            *p = y;
            xaa = xa;
            xa = xn;
            yaa = ya;
            ya = y;
        }
    }
}

__global__ void iir_store(const double *x, int ntr, int ns, float *d)
{
    const long long total = (long long)ntr * ns;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(idx / ntr), t = (int)(idx % ntr);
        d[(long long)t * ns + j] = (float)x[idx];
    }
}

/* SPATFILTER=4: out = sum_k w_k in(edge-replicated tap k) / sum_k w_k with the
 * point's own kernel (ii outer, jj inner, float, no contraction), or the
 * input where the point has none (src/gauss_filt_var.c:150-205) */
__global__ void gauss_var_kernel(int nx, int ny, const int *map, const int *pairs, const float *w, const float *in,
                                 float *out)
{
    const long long total = (long long)nx * ny;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int k = map[idx];
        if (k < 0) { out[idx] = in[idx]; continue; }
        const int i = (int)(idx % nx), j = (int)(idx / nx);
        const int hx = pairs[4 * k], hz = pairs[4 * k + 1];
        const float *wk = w + pairs[4 * k + 2];
        const float sum = __int_as_float(pairs[4 * k + 3]);
        float conv = 0.0f;
        int q = 0;
        for (int ii = -hx; ii <= hx; ii++) {
            const int ic = min(max(i + ii, 0), nx - 1);
            for (int jj = -hz; jj <= hz; jj++) {
                const int jc = min(max(j + jj, 0), ny - 1);
                conv = conv + in[(long long)jc * nx + ic] * wk[q++];
            }
        }
        out[idx] = conv / sum;
    }
}

/* g = zero ? 0 : g*coeff (src/taper_grad.c: waveconv *= taper_coeff, then
 * the zeroed points are set to 0.0) */
__global__ void taper_kernel(long long n, float *g, const float *c, const unsigned char *z)
{
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        g[k] = z[k] ? 0.0f : g[k] * c[k];
}

}  // namespace

extern "C" int dsh_taper_apply(float *g_dev, int nx, int ny, const float *coeff_dev, const unsigned char *zero_dev,
                               void *stream)
{
    if (nx < 1 || ny < 1 || !g_dev || !coeff_dev || !zero_dev) return DSH_ERR_PARAM;
    const long long total = (long long)nx * ny;
    const int blocks = (int)((total + 255) / 256 < 148 * 8 ? (total + 255) / 256 : 148 * 8);
    taper_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(total, g_dev, coeff_dev, zero_dev);
    return cudaGetLastError() == cudaSuccess ? DSH_OK : DSH_ERR_CUDA;
}

/* Butterworth filtering of traces (src/timedomain_filt.c with libcseife's
 * seife_lpb / seife_hpb): data_dev [ntr][ns] float on the device, filtered in
 * double like the reference and rounded back; method 1 lowpass, 2 highpass.
 * compat = 1 reproduces the reference's indexing (it passes its 1-based
 * vector as 0-based: a zero lead-in sample is filtered instead of the last
 * one, which is returned unfiltered, and the highpass removes that zero
 * instead of the first sample). */
extern "C" int dsh_timedomain_filt(float *data_dev, int ntr, int ns, float dt, float fc, int order, int method,
                                   int compat, void *stream)
{
    if (!data_dev || ntr < 1 || ns < 1 || (method != 1 && method != 2)) return DSH_ERR_PARAM;
    IIRChain ch;
    ch.n = dsh_setup_butterworth((double)dt, fc, order, method == 2, &ch.c[0][0]);
    if (ch.n < 0) return DSH_ERR_PARAM;
    const cudaStream_t st = (cudaStream_t)stream;
    double *x = nullptr;
    if (cudaMallocAsync(&x, (size_t)ntr * ns * sizeof(double), st) != cudaSuccess) return DSH_ERR_OOM;
    const long long total = (long long)ntr * ns;
    const int blocks = (int)((total + 255) / 256 < 148 * 16 ? (total + 255) / 256 : 148 * 16);
    /* compat: samples 0 .. ns-2 are filtered (a zero lead-in with zero
       filter state changes nothing), sample ns-1 stays, no offset removal */
    const int nf = compat ? ns - 1 : ns;
    iir_load<<<blocks, 256, 0, st>>>(data_dev, ntr, ns, method == 2 && !compat, x);
    if (nf > 0) iir_run<<<(ntr + 127) / 128, 128, 0, st>>>(x, ntr, nf, ch);
    iir_store<<<blocks, 256, 0, st>>>(x, ntr, ns, data_dev);
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(x, st);
    return e == cudaSuccess ? DSH_OK : DSH_ERR_CUDA;
}

extern "C" int dsh_smooth_gauss(int nx, int ny, int filt, const float *in_dev, float *out_dev, void *stream)
{
    if (nx < 1 || ny < 1 || !in_dev || !out_dev || in_dev == out_dev) return DSH_ERR_PARAM;
    const cudaStream_t st = (cudaStream_t)stream;
    if (filt == 0)
        return cudaMemcpyAsync(out_dev, in_dev, (size_t)nx * ny * sizeof(float), cudaMemcpyDeviceToDevice, st) ==
                       cudaSuccess ? DSH_OK : DSH_ERR_CUDA;
    const int hfs = (filt < 0 ? -filt : filt) / 2;
    if (2 * hfs + 1 > GAUSS_MAX) return DSH_ERR_PARAM;
    GaussW k;
    if (dsh_setup_gauss_kernel(filt, k.w) != 0) return DSH_ERR_PARAM;
    const long long total = (long long)nx * ny;
    const int blocks = (int)((total + 255) / 256 < 148 * 16 ? (total + 255) / 256 : 148 * 16);
    gauss_filt_kernel<<<blocks, 256, 0, st>>>(nx, ny, hfs, k, in_dev, out_dev);
    return cudaGetLastError() == cudaSuccess ? DSH_OK : DSH_ERR_CUDA;
}

extern "C" int dsh_smooth_gauss_var(int nx, int ny, float dh, float wd_damp, float wd_damp1, float fc_end,
                                    const float *vel_host, const float *in_dev, float *out_dev, void *stream)
{
    if (nx < 1 || ny < 1 || !vel_host || !in_dev || !out_dev || in_dev == out_dev || !(dh > 0) || !(fc_end > 0))
        return DSH_ERR_PARAM;
    const long long n = (long long)nx * ny;
    const int max_pairs = 4096, max_weights = 1 << 22;
    std::vector<int> map((size_t)n), pairs(4 * (size_t)max_pairs);
    std::vector<float> w((size_t)max_weights);
    const int np = dsh_setup_gauss_var(nx, ny, dh, wd_damp, wd_damp1, fc_end, vel_host, map.data(), max_pairs,
                                       pairs.data(), max_weights, w.data());
    if (np < 0) return DSH_ERR_PARAM;
    int nw = 0;
    for (int k = 0; k < np; k++) nw = std::max(nw, pairs[4 * k + 2] + (2 * pairs[4 * k] + 1) * (2 * pairs[4 * k + 1] + 1));
    const cudaStream_t st = (cudaStream_t)stream;
    int *d_map = nullptr, *d_pairs = nullptr;
    float *d_w = nullptr;
    if (cudaMallocAsync(&d_map, (size_t)n * sizeof(int), st) != cudaSuccess ||
        cudaMallocAsync(&d_pairs, (size_t)std::max(np, 1) * 4 * sizeof(int), st) != cudaSuccess ||
        cudaMallocAsync(&d_w, (size_t)std::max(nw, 1) * sizeof(float), st) != cudaSuccess) {
        cudaFreeAsync(d_map, st); cudaFreeAsync(d_pairs, st); cudaFreeAsync(d_w, st);
        cudaGetLastError();
        return DSH_ERR_OOM;
    }
    cudaMemcpyAsync(d_map, map.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st);
    if (np > 0) {
        cudaMemcpyAsync(d_pairs, pairs.data(), (size_t)np * 4 * sizeof(int), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_w, w.data(), (size_t)nw * sizeof(float), cudaMemcpyHostToDevice, st);
    }
    const int blocks = (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
    gauss_var_kernel<<<blocks, 256, 0, st>>>(nx, ny, d_map, d_pairs, d_w, in_dev, out_dev);
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(d_map, st); cudaFreeAsync(d_pairs, st); cudaFreeAsync(d_w, st);
    /* the host tables must outlive the asynchronous copies */
    if (cudaStreamSynchronize(st) != cudaSuccess || e != cudaSuccess) return DSH_ERR_CUDA;
    return DSH_OK;
}

extern "C" int dsh_gauss_filter_size(float wd_damp, float c_vs, float fc_end, float dh)
{
    return dsh_setup_gauss_size(wd_damp, c_vs, fc_end, dh);
}

/*
 * dsh_post.cu — gradient post-processing on the device: the SPATFILTER=3
 * Gaussian smoothing of src/gauss_filt.c (src/smooth_grad.c:27-29).
 * Each output point sums the (2h+1)^2 taps of the edge-replicated gradient
 * in the reference's order (ii outer, jj inner) in FP32 without contraction,
 * so it is bit-identical to the reference's loop (with its normalising sum
 * started at 0).
 */
#include "dsh.h"
#include "dsh_setup.h"

#include <cuda_runtime.h>

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

}  // namespace

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

extern "C" int dsh_gauss_filter_size(float wd_damp, float c_vs, float fc_end, float dh)
{
    return dsh_setup_gauss_size(wd_damp, c_vs, fc_end, dh);
}

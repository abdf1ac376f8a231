/*
 * dsh_nn_ops.cu — layout, activation, pooling, loss and optimiser kernels of
 * the pseudo-Hessian U-Net (everything except the tensor-core GEMM).  All
 * are bandwidth-bound grid-stride loops over NHWC tensors.
 */
#include "dsh_nn.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

namespace {

typedef __nv_bfloat16 bf16;

inline int grid_for(long long n, int threads = 256)
{
    return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 16));
}

inline int status() { return cudaGetLastError() == cudaSuccess ? DSH_NN_OK : DSH_NN_ERR_CUDA; }

#define GRID_LOOP(i, n) \
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

/* one thread per (pixel, tap, channel) column entry */
__global__ void im2col_k(const bf16 *x, int B, int H, int W, int C, bf16 *col, long long ldk)
{
    const long long P = (long long)B * H * W, K = 9LL * C;
    GRID_LOOP(idx, P * K)
    {
        const long long p = idx / K;
        const int k = (int)(idx % K), tap = k / C, c = k % C;
        const int xw = (int)(p % W), yh = (int)((p / W) % H);
        const long long b = p / ((long long)W * H);
        const int yy = yh + tap / 3 - 1, xx = xw + tap % 3 - 1;
        bf16 v = __float2bfloat16_rn(0.0f);
        if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = x[((b * H + yy) * W + xx) * C + c];
        col[p * ldk + k] = v;
    }
}

/* transposed: colT[k][p], consecutive threads along p */
__global__ void im2col_t_k(const bf16 *x, int B, int H, int W, int C, bf16 *colT, long long ldp)
{
    const long long P = (long long)B * H * W, K = 9LL * C;
    GRID_LOOP(idx, P * K)
    {
        const long long k = idx / P, p = idx % P;
        const int tap = (int)(k / C), c = (int)(k % C);
        const int xw = (int)(p % W), yh = (int)((p / W) % H);
        const long long b = p / ((long long)W * H);
        const int yy = yh + tap / 3 - 1, xx = xw + tap % 3 - 1;
        bf16 v = __float2bfloat16_rn(0.0f);
        if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = x[((b * H + yy) * W + xx) * C + c];
        colT[k * ldp + p] = v;
    }
}

/* 32 x 32 tile transpose through shared memory */
__global__ void transpose_k(const bf16 *y, long long P, int C, bf16 *yT, long long ldp)
{
    __shared__ bf16 t[32][33];
    const long long p0 = (long long)blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const long long p = p0 + r;
        const int c = c0 + threadIdx.x;
        t[r][threadIdx.x] = (p < P && c < C) ? y[p * C + c] : __float2bfloat16_rn(0.0f);
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int c = c0 + r;
        const long long p = p0 + threadIdx.x;
        if (c < C && p < P) yT[(long long)c * ldp + p] = t[threadIdx.x][r];
    }
}

__global__ void prep_weights_k(const float *w, int Cout, int Cin, bf16 *wb, long long ldk, bf16 *wf, long long ldf)
{
    const long long K = 9LL * Cin;
    GRID_LOOP(idx, (long long)Cout * K)
    {
        const int co = (int)(idx / K), k = (int)(idx % K);
        const bf16 v = __float2bfloat16_rn(w[idx]);
        wb[(long long)co * ldk + k] = v;
        const int tap = k / Cin, ci = k % Cin;
        wf[(long long)ci * ldf + (long long)(8 - tap) * Cout + co] = v;
    }
}

__global__ void to_bf16_k(const float *x, bf16 *y, long long n)
{
    GRID_LOOP(i, n) y[i] = __float2bfloat16_rn(x[i]);
}

__global__ void relu_bwd_k(const float *dy, const bf16 *y, bf16 *dx, float *dx32, long long n)
{
    GRID_LOOP(i, n)
    {
        const float d = __bfloat162float(y[i]) > 0.0f ? dy[i] : 0.0f;
        dx[i] = __float2bfloat16_rn(d);
        if (dx32) dx32[i] = d;
    }
}

__global__ void add_k(float *y, const float *x, long long n)
{
    GRID_LOOP(i, n) y[i] += x[i];
}

__global__ void maxpool_fwd_k(const bf16 *x, int B, int H, int W, int C, bf16 *y, unsigned char *arg)
{
    const int h = H / 2, w = W / 2;
    GRID_LOOP(idx, (long long)B * h * w * C)
    {
        const int c = (int)(idx % C);
        const long long q = idx / C;
        const int xo = (int)(q % w), yo = (int)((q / w) % h);
        const long long b = q / ((long long)w * h);
        float best = -3.0e38f;
        int a = 0;
        for (int k = 0; k < 4; k++) {
            const float v = __bfloat162float(x[((b * H + 2 * yo + k / 2) * W + 2 * xo + k % 2) * C + c]);
            if (v > best) { best = v; a = k; }
        }
        y[idx] = __float2bfloat16_rn(best);
        arg[idx] = (unsigned char)a;
    }
}

__global__ void maxpool_bwd_k(const float *dy, const unsigned char *arg, int B, int H, int W, int C, float *dx)
{
    GRID_LOOP(idx, (long long)B * H * W * C)
    {
        const int c = (int)(idx % C);
        const long long q = idx / C;
        const int xx = (int)(q % W), yy = (int)((q / W) % H);
        const long long b = q / ((long long)W * H);
        const long long o = ((b * (H / 2) + yy / 2) * (W / 2) + xx / 2) * C + c;
        dx[idx] = (arg[o] == (yy % 2) * 2 + (xx % 2)) ? dy[o] : 0.0f;
    }
}

__global__ void upsample_fwd_k(const bf16 *x, int B, int h, int w, int C, bf16 *y)
{
    const int H = 2 * h, W = 2 * w;
    GRID_LOOP(idx, (long long)B * H * W * C)
    {
        const int c = (int)(idx % C);
        const long long q = idx / C;
        const int xx = (int)(q % W), yy = (int)((q / W) % H);
        const long long b = q / ((long long)W * H);
        y[idx] = x[((b * h + yy / 2) * w + xx / 2) * C + c];
    }
}

__global__ void upsample_bwd_k(const float *dy, int B, int h, int w, int C, float *dx)
{
    const int W = 2 * w;
    GRID_LOOP(idx, (long long)B * h * w * C)
    {
        const int c = (int)(idx % C);
        const long long q = idx / C;
        const int xs = (int)(q % w), ys = (int)((q / w) % h);
        const long long b = q / ((long long)w * h);
        const long long r0 = ((b * 2 * h + 2 * ys) * W + 2 * xs) * C + c;
        dx[idx] = dy[r0] + dy[r0 + C] + dy[r0 + (long long)W * C] + dy[r0 + (long long)W * C + C];
    }
}

__global__ void concat_k(const bf16 *a, int C1, const bf16 *b, int C2, long long P, bf16 *y)
{
    const int C = C1 + C2;
    GRID_LOOP(idx, P * C)
    {
        const long long p = idx / C;
        const int c = (int)(idx % C);
        y[idx] = c < C1 ? a[p * C1 + c] : b[p * C2 + (c - C1)];
    }
}

__global__ void split_k(const float *dy, int C1, int C2, long long P, float *da, float *db)
{
    const int C = C1 + C2;
    GRID_LOOP(idx, P * C)
    {
        const long long p = idx / C;
        const int c = (int)(idx % C);
        if (c < C1) da[p * C1 + c] = dy[idx];
        else db[p * C2 + (c - C1)] = dy[idx];
    }
}

__global__ void head_fwd_k(const bf16 *x, long long P, int C, const float *w, const float *b, float *out)
{
    GRID_LOOP(p, P)
    {
        float s = 0.0f;
        for (int c = 0; c < C; c++) s += __bfloat162float(x[p * C + c]) * w[c];
        out[p] = s + b[0];
    }
}

/* dx[p][c] = dout[p] w[c], and per block b the partial sums
 * part[b][c] = sum over its rows of dout[p] x[p][c] (c < C) and
 * part[b][C] = sum of dout[p]: thread t of a block owns column t % (C+1) and
 * the rows r = t / (C+1) + k * (256 / (C+1)) of the block's chunk, partials
 * are combined in a fixed order, so the result does not depend on timing. */
__global__ void head_bwd_k(const float *dout, const bf16 *x, long long P, int C, const float *w, float *dx, float *part)
{
    const long long rows = (P + gridDim.x - 1) / gridDim.x;
    const long long r0 = (long long)blockIdx.x * rows, r1 = min(P, r0 + rows);
    for (long long idx = r0 * C + threadIdx.x; idx < r1 * C; idx += blockDim.x) {
        const long long p = idx / C;
        dx[idx] = dout[p] * w[idx % C];
    }
    extern __shared__ float acc[];                 /* blockDim.x */
    const int W = C + 1, lanes = blockDim.x / W;
    float s = 0.0f;
    if ((int)threadIdx.x < lanes * W) {
        const int c = threadIdx.x % W, lane = threadIdx.x / W;
        for (long long p = r0 + lane; p < r1; p += lanes)
            s += c < C ? dout[p] * __bfloat162float(x[p * C + c]) : dout[p];
    }
    acc[threadIdx.x] = s;
    __syncthreads();
    if ((int)threadIdx.x < W) {
        float t = 0.0f;
        for (int lane = 0; lane < lanes; lane++) t += acc[lane * W + threadIdx.x];
        part[(long long)blockIdx.x * W + threadIdx.x] = t;
    }
}

/* per-block partial column sums of dy [P][N] (fixed order, as head_bwd_k) */
__global__ void colsum_k(const float *dy, long long P, int N, float *part)
{
    const long long rows = (P + gridDim.x - 1) / gridDim.x;
    const long long r0 = (long long)blockIdx.x * rows, r1 = min(P, r0 + rows);
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        float s = 0.0f;
        for (long long p = r0; p < r1; p++) s += dy[p * N + n];
        part[(long long)blockIdx.x * N + n] = s;
    }
}

/* g[n] += sum over blocks of part[b*stride + n], blocks in order */
__global__ void sum_parts_k(const float *part, int nblocks, int N, int stride, float *g)
{
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int b = 0; b < nblocks; b++) s += part[(long long)b * stride + n];
        g[n] += s;
    }
}

__global__ void mse_k(const float *pred, const float *target, const unsigned char *mask, long long n, float count,
                      float *grad, float *loss)
{
    __shared__ float red[256];
    float s = 0.0f;
    GRID_LOOP(i, n)
    {
        const bool on = !mask || mask[i];
        const float d = on ? pred[i] - target[i] : 0.0f;
        grad[i] = 2.0f * d / count;
        s += d * d;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0] / count);
}

__global__ void adam_k(float *w, float *m, float *v, const float *g, int rows, int cols, int transposed, float lr,
                       float b1, float b2, float eps, float c1, float c2)
{
    GRID_LOOP(i, (long long)rows * cols)
    {
        const long long r = i / cols, c = i % cols;
        const float gr = transposed ? g[c * rows + r] : g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gr;
        const float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

}  // namespace

#define ST ((cudaStream_t)stream)

extern "C" int dsh_nn_im2col(const void *x, int B, int H, int W, int C, void *col, long long ldk, void *stream)
{
    if (!x || !col || B <= 0 || H <= 0 || W <= 0 || C <= 0 || ldk < 9LL * C) return DSH_NN_ERR_PARAM;
    const long long n = (long long)B * H * W * 9 * C;
    im2col_k<<<grid_for(n), 256, 0, ST>>>((const bf16 *)x, B, H, W, C, (bf16 *)col, ldk);
    return status();
}

extern "C" int dsh_nn_im2col_t(const void *x, int B, int H, int W, int C, void *colT, long long ldp, void *stream)
{
    if (!x || !colT || B <= 0 || H <= 0 || W <= 0 || C <= 0 || ldp < (long long)B * H * W) return DSH_NN_ERR_PARAM;
    const long long n = (long long)B * H * W * 9 * C;
    im2col_t_k<<<grid_for(n), 256, 0, ST>>>((const bf16 *)x, B, H, W, C, (bf16 *)colT, ldp);
    return status();
}

extern "C" int dsh_nn_transpose(const void *y, long long P, int C, void *yT, long long ldp, void *stream)
{
    if (!y || !yT || P <= 0 || C <= 0 || ldp < P) return DSH_NN_ERR_PARAM;
    dim3 grid((unsigned)((P + 31) / 32), (unsigned)((C + 31) / 32));
    transpose_k<<<grid, dim3(32, 8), 0, ST>>>((const bf16 *)y, P, C, (bf16 *)yT, ldp);
    return status();
}

extern "C" int dsh_nn_prep_weights(const float *w, int Cout, int Cin, void *wb, long long ldk, void *wf, long long ldf,
                                   void *stream)
{
    if (!w || !wb || !wf || Cout <= 0 || Cin <= 0 || ldk < 9LL * Cin || ldf < 9LL * Cout) return DSH_NN_ERR_PARAM;
    prep_weights_k<<<grid_for(9LL * Cin * Cout), 256, 0, ST>>>(w, Cout, Cin, (bf16 *)wb, ldk, (bf16 *)wf, ldf);
    return status();
}

extern "C" int dsh_nn_to_bf16(const float *x, void *y, long long n, void *stream)
{
    if (!x || !y || n < 0) return DSH_NN_ERR_PARAM;
    if (n) to_bf16_k<<<grid_for(n), 256, 0, ST>>>(x, (bf16 *)y, n);
    return status();
}

extern "C" int dsh_nn_relu_bwd(const float *dy, const void *y, void *dx, float *dx32, long long n, void *stream)
{
    if (!dy || !y || !dx || n < 0) return DSH_NN_ERR_PARAM;
    if (n) relu_bwd_k<<<grid_for(n), 256, 0, ST>>>(dy, (const bf16 *)y, (bf16 *)dx, dx32, n);
    return status();
}

extern "C" int dsh_nn_add(float *y, const float *x, long long n, void *stream)
{
    if (!y || !x || n < 0) return DSH_NN_ERR_PARAM;
    if (n) add_k<<<grid_for(n), 256, 0, ST>>>(y, x, n);
    return status();
}

extern "C" int dsh_nn_maxpool_fwd(const void *x, int B, int H, int W, int C, void *y, unsigned char *arg, void *stream)
{
    if (!x || !y || !arg || H % 2 || W % 2 || B <= 0 || C <= 0) return DSH_NN_ERR_PARAM;
    maxpool_fwd_k<<<grid_for((long long)B * H * W * C / 4), 256, 0, ST>>>((const bf16 *)x, B, H, W, C, (bf16 *)y, arg);
    return status();
}

extern "C" int dsh_nn_maxpool_bwd(const float *dy, const unsigned char *arg, int B, int H, int W, int C, float *dx,
                                  void *stream)
{
    if (!dy || !arg || !dx || H % 2 || W % 2 || B <= 0 || C <= 0) return DSH_NN_ERR_PARAM;
    maxpool_bwd_k<<<grid_for((long long)B * H * W * C), 256, 0, ST>>>(dy, arg, B, H, W, C, dx);
    return status();
}

extern "C" int dsh_nn_upsample_fwd(const void *x, int B, int h, int w, int C, void *y, void *stream)
{
    if (!x || !y || B <= 0 || h <= 0 || w <= 0 || C <= 0) return DSH_NN_ERR_PARAM;
    upsample_fwd_k<<<grid_for(4LL * B * h * w * C), 256, 0, ST>>>((const bf16 *)x, B, h, w, C, (bf16 *)y);
    return status();
}

extern "C" int dsh_nn_upsample_bwd(const float *dy, int B, int h, int w, int C, float *dx, void *stream)
{
    if (!dy || !dx || B <= 0 || h <= 0 || w <= 0 || C <= 0) return DSH_NN_ERR_PARAM;
    upsample_bwd_k<<<grid_for((long long)B * h * w * C), 256, 0, ST>>>(dy, B, h, w, C, dx);
    return status();
}

extern "C" int dsh_nn_concat(const void *a, int C1, const void *b, int C2, long long P, void *y, void *stream)
{
    if (!a || !b || !y || C1 <= 0 || C2 <= 0 || P <= 0) return DSH_NN_ERR_PARAM;
    concat_k<<<grid_for(P * (C1 + C2)), 256, 0, ST>>>((const bf16 *)a, C1, (const bf16 *)b, C2, P, (bf16 *)y);
    return status();
}

extern "C" int dsh_nn_split(const float *dy, int C1, int C2, long long P, float *da, float *db, void *stream)
{
    if (!dy || !da || !db || C1 <= 0 || C2 <= 0 || P <= 0) return DSH_NN_ERR_PARAM;
    split_k<<<grid_for(P * (C1 + C2)), 256, 0, ST>>>(dy, C1, C2, P, da, db);
    return status();
}

extern "C" int dsh_nn_head_fwd(const void *x, long long P, int C, const float *w, const float *b, float *out,
                               void *stream)
{
    if (!x || !w || !b || !out || P <= 0 || C <= 0) return DSH_NN_ERR_PARAM;
    head_fwd_k<<<grid_for(P), 256, 0, ST>>>((const bf16 *)x, P, C, w, b, out);
    return status();
}

constexpr int RED_BLOCKS = DSH_NN_RED_BLOCKS;

extern "C" int dsh_nn_head_bwd(const float *dout, const void *x, long long P, int C, const float *w, float *dx,
                               float *gw, float *gb, float *part, void *stream)
{
    if (!dout || !x || !w || !dx || !gw || !gb || !part || P <= 0 || C <= 0 || C + 1 > 256) return DSH_NN_ERR_PARAM;
    head_bwd_k<<<RED_BLOCKS, 256, 256 * sizeof(float), ST>>>(dout, (const bf16 *)x, P, C, w, dx, part);
    sum_parts_k<<<1, 256, 0, ST>>>(part, RED_BLOCKS, C, C + 1, gw);
    sum_parts_k<<<1, 32, 0, ST>>>(part + C, RED_BLOCKS, 1, C + 1, gb);   /* column C of the (C+1)-wide table */
    return status();
}

extern "C" int dsh_nn_colsum(const float *dy, long long P, int N, float *g, float *part, void *stream)
{
    if (!dy || !g || !part || P <= 0 || N <= 0) return DSH_NN_ERR_PARAM;
    colsum_k<<<RED_BLOCKS, 256, 0, ST>>>(dy, P, N, part);
    sum_parts_k<<<(N + 255) / 256, 256, 0, ST>>>(part, RED_BLOCKS, N, N, g);
    return status();
}

extern "C" int dsh_nn_mse(const float *pred, const float *target, const unsigned char *mask, long long n, float count,
                          float *grad, float *loss, void *stream)
{
    if (!pred || !target || !grad || !loss || n <= 0 || !(count > 0)) return DSH_NN_ERR_PARAM;
    mse_k<<<grid_for(n), 256, 0, ST>>>(pred, target, mask, n, count, grad, loss);
    return status();
}

extern "C" int dsh_nn_adam(float *w, float *m, float *v, const float *g, int rows, int cols, int transposed, float lr,
                           float beta1, float beta2, float eps, int step, void *stream)
{
    if (!w || !m || !v || !g || rows <= 0 || cols <= 0 || step < 1) return DSH_NN_ERR_PARAM;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    adam_k<<<grid_for((long long)rows * cols), 256, 0, ST>>>(w, m, v, g, rows, cols, transposed, lr, beta1, beta2, eps,
                                                             c1, c2);
    return status();
}

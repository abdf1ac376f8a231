/*
 * dsh_nn.h — C ABI of the kernels behind the learned pseudo-Hessian
 * preconditioner: a 4-level U-Net (BF16 weights and activations, FP32
 * accumulation) that predicts the pseudo-Hessian diagonal of the SH FWI
 * gradient (src/hessian.c, src/hessian_out.c) from the raw gradient, the
 * eprecond energies Ws, Wr (src/eprecond.c) and the current vs model.  The
 * reference has no learned component; these entry points have no
 * counterpart there.
 *
 * Layouts: activations NHWC ([batch][ny][nx][channels], channels fastest),
 * "pixels" P = batch*ny*nx; bf16 buffers are uint16 bit patterns of
 * __nv_bfloat16.  3x3 convolutions use zero ("same") padding and
 * tap-major columns: k = tap*C + c with tap = (dy+1)*3 + (dx+1).
 * All pointers are device pointers; every call is asynchronous on `stream`
 * (a cudaStream_t as void*, NULL = default stream) and returns DSH_NN_OK or a
 * negative code.  Kernels that wait on a barrier record DSH_NN_ERR_TIMEOUT in
 * the caller's device int *err instead of hanging.
 */
#ifndef DSH_NN_H
#define DSH_NN_H

#ifdef __cplusplus
extern "C" {
#endif

#define DSH_NN_OK 0
#define DSH_NN_ERR_PARAM (-1)
#define DSH_NN_ERR_CUDA (-2)
#define DSH_NN_ERR_TIMEOUT (-6)

/* C[M][N] = A[M][K] . B[N][K]^T (+ bias[N]) (ReLU) on the tensor cores.
 * A, B: bf16, row strides lda, ldb elements (multiples of 8, >= K; 16-byte
 * aligned bases).  Outputs: C32 (float) and/or C16 (bf16), row stride ldc.
 * splits > 1 divides K over CTAs (FP32 partials in `partial`, splits*M*ldc
 * floats, then summed into C32; no bias/ReLU/C16 then); accumulate = 1 adds
 * the product to C32 (uses `partial` for M*ldc floats). */
/* Poll limit of the GEMM pipeline's mbarrier waits for the following
 * launches (process-wide; default 2^22, <= 0 restores it).  On expiry a CTA
 * records DSH_NN_ERR_TIMEOUT in the caller's err word, stops issuing, waits
 * for the copies and multiply operations it already issued, frees its tensor
 * memory and exits; a small limit exercises that path on a healthy run.  No
 * counterpart in the reference. */
int dsh_nn_set_wait_limit(long long polls);

int dsh_nn_gemm(int M, int N, int K, const void *A, long long lda, const void *B, long long ldb, float *C32, void *C16,
                long long ldc, const float *bias, int relu, int splits, float *partial, int accumulate, int *err,
                void *stream);

/* im2col of a 3x3 same-padded convolution: x bf16 [B][H][W][C] ->
 * col bf16 [P][ldk] (columns 9C..ldk-1 are left untouched) */
int dsh_nn_im2col(const void *x, int B, int H, int W, int C, void *col, long long ldk, void *stream);
/* the transposed columns colT bf16 [9C][ldp] (ldp >= P, multiple of 8) */
int dsh_nn_im2col_t(const void *x, int B, int H, int W, int C, void *colT, long long ldp, void *stream);
/* y bf16 [P][C] -> yT bf16 [C][ldp] */
int dsh_nn_transpose(const void *y, long long P, int C, void *yT, long long ldp, void *stream);
/* FP32 master weights w [Cout][9*Cin] -> bf16 forward operand wb [Cout][ldk]
 * and the flipped, transposed operand of the input gradient
 * wf [Cin][ldf]: wf[ci][tap*Cout + co] = w[co][(8-tap)*Cin + ci] */
int dsh_nn_prep_weights(const float *w, int Cout, int Cin, void *wb, long long ldk, void *wf, long long ldf,
                        void *stream);
/* float -> bf16 (n elements) */
int dsh_nn_to_bf16(const float *x, void *y, long long n, void *stream);
/* dx = dy * (y > 0) (ReLU backward through the stored activation): bf16 dx,
 * and the same values as float in dx32 when it is not NULL (may alias dy) */
int dsh_nn_relu_bwd(const float *dy, const void *y, void *dx, float *dx32, long long n, void *stream);
/* y += x (n floats) */
int dsh_nn_add(float *y, const float *x, long long n, void *stream);
/* 2x2 max pooling: x bf16 [B][H][W][C] -> y bf16 [B][H/2][W/2][C], arg uint8 (0..3) */
int dsh_nn_maxpool_fwd(const void *x, int B, int H, int W, int C, void *y, unsigned char *arg, void *stream);
/* dx float [B][H][W][C] = dy routed to the argmax (others 0) */
int dsh_nn_maxpool_bwd(const float *dy, const unsigned char *arg, int B, int H, int W, int C, float *dx, void *stream);
/* nearest 2x upsampling: x bf16 [B][h][w][C] -> y bf16 [B][2h][2w][C] */
int dsh_nn_upsample_fwd(const void *x, int B, int h, int w, int C, void *y, void *stream);
/* dx float [B][h][w][C] = sum of dy over each 2x2 block */
int dsh_nn_upsample_bwd(const float *dy, int B, int h, int w, int C, float *dx, void *stream);
/* channel concatenation y [P][C1+C2] = (a [P][C1], b [P][C2]) (bf16) */
int dsh_nn_concat(const void *a, int C1, const void *b, int C2, long long P, void *y, void *stream);
/* split of the concatenation's gradient: dy float [P][C1+C2] -> da [P][C1], db [P][C2] (float) */
int dsh_nn_split(const float *dy, int C1, int C2, long long P, float *da, float *db, void *stream);
/* out[p] = sum_c x[p][c] w[c] + b (1x1 convolution to one channel, x bf16, out float) */
int dsh_nn_head_fwd(const void *x, long long P, int C, const float *w, const float *b, float *out, void *stream);
/* dx[p][c] = dout[p] w[c] (float); gw[c] += sum_p dout[p] x[p][c]; gb += sum_p dout[p].
 * part: scratch of DSH_NN_RED_BLOCKS*(C+1) floats; the sums are formed in a
 * fixed order (no atomics), so training is reproducible run to run. */
#define DSH_NN_RED_BLOCKS 296
int dsh_nn_head_bwd(const float *dout, const void *x, long long P, int C, const float *w, float *dx, float *gw,
                    float *gb, float *part, void *stream);
/* column sums: g[n] += sum_p dy[p][n] (bias gradient), dy float [P][N];
 * part: scratch of DSH_NN_RED_BLOCKS*N floats, fixed summation order */
int dsh_nn_colsum(const float *dy, long long P, int N, float *g, float *part, void *stream);
/* masked mean-square loss: d = pred - target on mask != 0; loss[0] += sum d^2 / count,
 * grad = 2 d / count (0 outside the mask) */
int dsh_nn_mse(const float *pred, const float *target, const unsigned char *mask, long long n, float count,
               float *grad, float *loss, void *stream);
/* Adam (FP32 master weights): w -= lr * mhat / (sqrt(vhat) + eps); with
 * transposed = 1 the gradient is stored [K][N] for weights [N][K] */
int dsh_nn_adam(float *w, float *m, float *v, const float *g, int rows, int cols, int transposed, float lr,
                float beta1, float beta2, float eps, int step, void *stream);

#ifdef __cplusplus
}
#endif
#endif

/*
 * dsh_engine.cu — device-resident engine behind include/dsh.h.
 *
 * One context = one model on one GPU with `max_shots` shot slots advanced
 * together (grid z = slot).  A pass (forward, forward with storage, forward
 * with Hessian accumulation, adjoint) is a loop over NT steps of
 *     v_step -> inject_sample -> s_step
 * replayed from a CUDA graph that holds `chunk` steps; the kernels read the
 * step number from a device counter that the graph's last node advances, so
 * one small graph serves every step of every pass.
 *
 * Reference correspondence (src/...): forward loop denise.c:1179-1346,
 * residual calc_res.c:94-232, adjoint loop denise.c:1452-1654, energy
 * preconditioning eprecond1.c + denise.c:1665-1678, shot sum :1689-1694,
 * conversion :1743-1813, Hessian hessian.c:91-94 + hessian_out.c:20-31.
 */
#include "dsh.h"
#include "dsh_engine_int.h"
#include "dsh_fs.h"
#include "dsh_pf.h"
#include "dsh_cl.h"
#include "dsh_tb.h"
#include "dsh_fused.cuh"
#include "dsh_setup.h"

#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

using namespace dsh;
using namespace dsh::eng;

static void build_tmaps(dsh_ctx *ctx);

namespace {


constexpr int RED_BLOCKS = 296;        /* 2 x 148 SMs for reductions */
constexpr int RED_THREADS = 256;

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

/* ---------------- epilogue kernels ---------------- */

/* Residual of one slot, stored as the adjoint source of step t (1-based):
 * res[r][t-1] = syn(NT-t+1) - obs(NT-t+1), with the first observed sample
 * replaced by the synthetic one (calc_res.c:115,172-177).  Also the per-block
 * partial sums of res^2 (double) for a deterministic L2. */
__global__ void residual_kernel(int nt_total, const int *rec_off, const float *seis, const long long *seis_off,
                                const float *obs, const long long *obs_off, float *res, double *part)
{
    const int s = blockIdx.y;
    const int ntr = rec_off[s + 1] - rec_off[s];
    const long long n = (long long)ntr * nt_total;
    const float *syn = seis + seis_off[s];
    const float *ob = obs + obs_off[s];
    float *rs = res + seis_off[s];
    double acc = 0.0;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx / nt_total);
        const int t = (int)(idx % nt_total) + 1;       /* adjoint step */
        const int tf = nt_total - t + 1;                /* forward sample */
        const float sy = syn[(long long)(tf - 1) * ntr + r];
        const float od = (tf == 1) ? sy : ob[(long long)r * nt_total + (tf - 1)];
        const float v = sy - od;
        rs[(long long)r * nt_total + (t - 1)] = v;
        acc += (double)v * (double)v;
    }
    __shared__ double sh[RED_THREADS];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(long long)s * gridDim.x + blockIdx.x] = sh[0];
}

/* Residual of LNORM 1, 3, 4 (calc_res.c:156-189) with the same layout and
 * first-sample replacement: sign(obs - syn), (obs - syn)/(1 + (obs - syn)^2),
 * tanh(obs - syn) (double tanh rounded to float, as the reference's C call).
 * The reference adds nothing to the misfit for these norms (:250-260). */
__global__ void residual_elem_kernel(int lnorm, int nt_total, const int *rec_off, const float *seis,
                                     const long long *seis_off, const float *obs, const long long *obs_off, float *res,
                                     double *part)
{
    const int s = blockIdx.y;
    const int ntr = rec_off[s + 1] - rec_off[s];
    const long long n = (long long)ntr * nt_total;
    const float *syn = seis + seis_off[s];
    const float *ob = obs + obs_off[s];
    float *rs = res + seis_off[s];
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx / nt_total);
        const int t = (int)(idx % nt_total) + 1;
        const int tf = nt_total - t + 1;
        const float sy = syn[(long long)(tf - 1) * ntr + r];
        const float od = (tf == 1) ? sy : ob[(long long)r * nt_total + (tf - 1)];
        float v;
        if (lnorm == 1) v = (od - sy) > 0.0f ? 1.0f : ((od - sy) < 0.0f ? -1.0f : 0.0f);
        else if (lnorm == 3) v = (od - sy) / (1.0f + ((od - sy) * (od - sy)));
        else v = (float)tanh((double)(od - sy));
        rs[(long long)r * nt_total + (t - 1)] = v;
    }
    if (threadIdx.x == 0) part[(long long)s * gridDim.x + blockIdx.x] = 0.0;
}

/* Global-correlation residual, LNORM=5 (calc_res.c:119-147,192-217): per
 * trace the float norms |obs|, |syn| and syn.obs in sample order (before the
 * first observed sample is replaced), then
 *   res = syn (syn.obs) / (|syn|^3 |obs|) - obs / (|syn| |obs|)
 * time-reversed, and the misfit term -obs syn / (|obs| |syn|) per sample
 * (summed in double; the reference subtracts it from its float L2).  One
 * thread per trace. */
__global__ void residual_gc_kernel(int nt_total, const int *rec_off, const float *seis, const long long *seis_off,
                                   const float *obs, const long long *obs_off, float *res, double *part)
{
    const int s = blockIdx.y;
    const int ntr = rec_off[s + 1] - rec_off[s];
    const float *syn = seis + seis_off[s];
    float *rs = res + seis_off[s];
    double acc = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < ntr; r += gridDim.x * blockDim.x) {
        const float *ob = obs + obs_off[s] + (long long)r * nt_total;
        float ad = 0.0f, as = 0.0f, dms = 0.0f;
#pragma unroll 8
        for (int t = 0; t < nt_total; t++) {
            const float d = ob[t], y = syn[(long long)t * ntr + r];
            ad = ad + d * d;
            as = as + y * y;
            dms = dms + y * d;
        }
        ad = (float)sqrt((double)ad);
        as = (float)sqrt((double)as);
        const float tmp = as * as * as * ad, tmp1 = as * ad, tmp2 = ad * as;
#pragma unroll 4
        for (int tf = 1; tf <= nt_total; tf++) {
            const float y = syn[(long long)(tf - 1) * ntr + r];
            const float d = (tf == 1) ? y : ob[tf - 1];
            rs[(long long)r * nt_total + (nt_total - tf)] = ((y * dms) / (tmp + 0.0f)) - (d / (tmp1 + 0.0f));
            acc -= (double)((d * y) / (tmp2 + 0.0f));
        }
    }
    __shared__ double sh[RED_THREADS];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(long long)s * gridDim.x + blockIdx.x] = sh[0];
}

__global__ void reduce_parts(const double *part, int nparts, int nslots, double *out)
{
    const int s = blockIdx.x;
    __shared__ double sh[RED_THREADS];
    double acc = 0.0;
    for (int k = threadIdx.x; k < nparts; k += blockDim.x) acc += part[(long long)s * nparts + k];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0 && s < nslots) out[s] = sh[0];
}

struct EpiArgs {
    int nx, ny, pitch;
    long long slot_stride;
    float *ws, *wr, *we, *gu, *grho;
    unsigned *wemax;
    float cvs, crho, dh;
    int eprecond;
};

/* We = sqrt(Ws*Wr) (EPRECOND=1) or sqrt(Ws)*(asinh((xmax-x)/y)-asinh((xmin-x)/y))
 * (EPRECOND=3, Plessix & Mulder), and its maximum (eprecond1.c:17-57). */
__global__ void eprecond_we_kernel(EpiArgs a)
{
    const int s = blockIdx.y;
    const long long so = (long long)s * a.slot_stride;
    const long long n = (long long)a.nx * a.ny;
    float mx = 0.0f;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % a.nx) + 1, j = (int)(idx / a.nx) + 1;
        const long long o = so + (long long)(j - 1) * a.pitch + (i - 1 + HX);
        float we;
        if (a.eprecond == 1) {
            we = sqrtf(a.ws[o] * a.wr[o]);
        } else {
            const float x = i * a.dh, y = j * a.dh, xmin = a.dh, xmax = a.nx * a.dh;
            we = (float)(sqrt((double)a.ws[o]) * (asinh((double)((xmax - x) / y)) - asinh((double)((xmin - x) / y))));
        }
        a.we[o] = we;
        if (we > mx) mx = we;
    }
    /* float max of non-negative values == unsigned max of their bits */
    for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_down_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0 && mx > 0.0f) atomicMax(a.wemax + s, __float_as_uint(mx));
}

/* We += 0.005*max(We); per-shot gradients /= We*C^2 (eprecond1.c:59-73, denise.c:1670-1675) */
__global__ void eprecond_scale_kernel(EpiArgs a)
{
    const int s = blockIdx.y;
    const long long so = (long long)s * a.slot_stride;
    const long long n = (long long)a.nx * a.ny;
    const float eps = 0.005f;
    const float mx = __uint_as_float(a.wemax[s]);
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % a.nx) + 1, j = (int)(idx / a.nx) + 1;
        const long long o = so + (long long)(j - 1) * a.pitch + (i - 1 + HX);
        const float we = a.we[o] + (eps * mx);
        a.we[o] = we;
        a.gu[o] = a.gu[o] / (we * a.cvs * a.cvs);
        a.grho[o] = a.grho[o] / (we * a.crho * a.crho);
    }
}

/* sum += per-shot field, slots in shot order (denise.c:1689-1694) */
__global__ void shot_sum_kernel(int nx, int ny, int pitch, long long slot_stride, int nslots, const float *a_u,
                                const float *a_r, float *sum_u, float *sum_r)
{
    const long long n = (long long)nx * ny;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nx) + 1, j = (int)(idx / nx) + 1;
        const long long o = (long long)(j - 1) * pitch + (i - 1 + HX);
        float su = sum_u[o], sr = sum_r[o];
        for (int s = 0; s < nslots; s++) {
            su = su + a_u[(long long)s * slot_stride + o];
            sr = sr + a_r[(long long)s * slot_stride + o];
        }
        sum_u[o] = su;
        sum_r[o] = sr;
    }
}

/* per-shot circular taper of one slot (src/taper_grad_shot.c) */
struct TaperShot {
    int i1, j1;
    float minm, maxm;
};

/* sum += tapered per-shot field: the shot's coefficient (min(1, box value)
 * - minm) / maxm, 0 within filt points of its source
 * (src/taper_grad_shot.c:126-190, then denise.c:1689-1694) */
__global__ void shot_sum_taper_kernel(int nx, int ny, int pitch, long long slot_stride, int nslots, const float *a_u,
                                      const float *a_r, float *sum_u, float *sum_r, const float *box, int g, int ijc,
                                      int filt, const TaperShot *ts)
{
    const long long n = (long long)nx * ny;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nx) + 1, j = (int)(idx / nx) + 1;
        const long long o = (long long)(j - 1) * pitch + (i - 1 + HX);
        float su = sum_u[o], sr = sum_r[o];
        for (int s = 0; s < nslots; s++) {
            const TaperShot t = ts[s];
            const int ix = i - t.i1 + ijc, iy = j - t.j1 + ijc;
            float mm = 1.0f;
            if (ix >= 1 && ix <= g && iy >= 1 && iy <= g) mm = box[(iy - 1) * g + (ix - 1)];
            float ms = 1.0f;
            if (ms > mm) ms = mm;
            const float c = (ms - t.minm) / t.maxm;
            const bool z = abs(i - t.i1) <= filt && abs(j - t.j1) <= filt;
            su = su + (z ? 0.0f : a_u[(long long)s * slot_stride + o] * c);
            sr = sr + (z ? 0.0f : a_r[(long long)s * slot_stride + o] * c);
        }
        sum_u[o] = su;
        sum_r[o] = sr;
    }
}

/* waveconv_mu = -DT*sum_u; g_vs = 2 rho vs mu (double, as the reference's
 * double literal promotes it); g_rho = vs^2 mu - DT*sum_rho (denise.c:1752-1800) */
__global__ void convert_kernel(int nx, int ny, int pitch, float dt, const float *vs, const float *rho,
                               const float *sum_u, const float *sum_r, float *g_vs, float *g_rho)
{
    const long long n = (long long)nx * ny;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nx) + 1, j = (int)(idx / nx) + 1;
        const long long o = (long long)(j - 1) * pitch + (i - 1 + HX);
        const float u = vs[o], r = rho[o];
        const float mu = -dt * sum_u[o];
        const float gv = (float)(2.0 * (double)r * (double)u * (double)mu);
        const float rho_s = -dt * sum_r[o];
        const float gr = (u * u * mu) + rho_s;
        g_vs[idx] = gv;
        g_rho[idx] = gr;
    }
}

/* Qs gradient from the shot sums of the two correlations (no counterpart in
 * the reference, which has no Q gradient): the stress multiplier of forward
 * update k is (2/rho) times the back-propagated adjoint strain, so
 * dJ/dtau_ipjp = -(2/rho) sum_x and dJ/dtau = -(2/rho) sum_y; tau_ipjp is the
 * four-point average of tau (av_tau.c:12, one-rank periodic wrap) and
 * tau = 2/Qs (readmod.c:99).  Double arithmetic in the oracle's order. */
__global__ void q_convert_kernel(int nx, int ny, int pitch, const float *rho, const float *qs, const float *sum_x,
                                 const float *sum_y, float *g_qs)
{
    const long long n = (long long)nx * ny;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nx) + 1, j = (int)(idx / nx) + 1;
        const int im = i > 1 ? i - 1 : nx, jm = j > 1 ? j - 1 : ny;
        const long long nb[4] = {(long long)(j - 1) * pitch + (i - 1 + HX), (long long)(j - 1) * pitch + (im - 1 + HX),
                                 (long long)(jm - 1) * pitch + (i - 1 + HX), (long long)(jm - 1) * pitch + (im - 1 + HX)};
        double gx = 0.0;
        for (int k = 0; k < 4; k++) gx += -2.0 / (double)rho[nb[k]] * (double)sum_x[nb[k]];
        const double gy = -2.0 / (double)rho[nb[0]] * (double)sum_y[nb[0]];
        const double q = (double)qs[nb[0]];
        g_qs[idx] = (float)((gy + 0.25 * gx) * (-2.0 / (q * q)));
    }
}

/* hessian_out.c:20-31: H_rho += vs^4 H_mu; H_vs = 4 rho^2 vs^2 H_mu (double) */
__global__ void hessian_convert_kernel(int nx, int ny, int pitch, const float *vs, const float *rho, const float *hu,
                                       const float *hr, float *h_vs, float *h_rho)
{
    const long long n = (long long)nx * ny;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nx) + 1, j = (int)(idx / nx) + 1;
        const long long o = (long long)(j - 1) * pitch + (i - 1 + HX);
        const float u = vs[o], r = rho[o];
        float a = hu[o], b = hr[o];
        b += u * u * u * u * a;
        a = (float)(4.0 * (double)r * (double)r * (double)u * (double)u * (double)a);
        h_vs[idx] = a;
        h_rho[idx] = b;
    }
}

/* [NT][ntr] (device seismogram layout) -> [ntr][NT] */
__global__ void seis_transpose_kernel(int nt_total, const int *rec_off, const float *in, const long long *in_off,
                                      float *out, const long long *out_off)
{
    const int s = blockIdx.y;
    const int ntr = rec_off[s + 1] - rec_off[s];
    const long long n = (long long)ntr * nt_total;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx / nt_total), t = (int)(idx % nt_total);
        out[out_off[s] + idx] = in[in_off[s] + (long long)t * ntr + r];
    }
}

/* dense pitched interior field of slot s -> [ny][nx] */
__global__ void gather_dense_kernel(int nx, int ny, int pitch, const float *src, float *dst)
{
    const long long n = (long long)nx * ny;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nx), j = (int)(idx / nx);
        dst[idx] = src[(long long)j * pitch + i + HX];
    }
}

__global__ void set_int_kernel(int *p, int v) { *p = v; }

}  // namespace

/* ======================= context (struct dsh_ctx: dsh_engine_int.h) ======================= */

static int fail_cuda(dsh_ctx *c, cudaError_t e)
{
    if (c) c->last_cuda = (int)e;
    fprintf(stderr, "dsh: CUDA error %d (%s)\n", (int)e, cudaGetErrorString(e));
    return DSH_ERR_CUDA;
}
#define CK(x)                                              \
    do {                                                   \
        cudaError_t e_ = (x);                              \
        if (e_ != cudaSuccess) return fail_cuda(ctx, e_);  \
    } while (0)

namespace dsh::eng {
int wait_stream(dsh_ctx *ctx)
{
    CK(cudaEventRecord(ctx->ev_wait, ctx->st));
    const int rc = wait_event(ctx->ev_wait, ctx->host_timeout_s);
    if (rc == DSH_ERR_TIMEOUT)
        fprintf(stderr, "dsh: the device did not finish within %.3g s; the call returns DSH_ERR_TIMEOUT\n",
                ctx->host_timeout_s);
    if (rc == DSH_ERR_CUDA) return fail_cuda(ctx, cudaGetLastError());
    return rc;
}
}  // namespace dsh::eng

/* bounded host waits (no cudaStreamSynchronize / cudaEventSynchronize): for
 * the context's stream, and for an event already recorded on it */
#define WAIT(c)                                            \
    do {                                                   \
        const int w_ = wait_stream(c);                     \
        if (w_ != DSH_OK) return w_;                       \
    } while (0)
#define WAIT_EV(c, ev)                                     \
    do {                                                   \
        const int w_ = wait_event((ev), (c)->host_timeout_s); \
        if (w_ == DSH_ERR_CUDA) return fail_cuda((c), cudaGetLastError()); \
        if (w_ != DSH_OK) return w_;                       \
    } while (0)

extern "C" void dsh_params_default(dsh_params *p)
{
    memset(p, 0, sizeof(*p));
    p->fdorder = 4;
    p->maxrelerror = 1;
    p->fw = 20;
    p->free_surf = 1;
    p->npower = 4.0f;
    p->k_max_pml = 1.0f;
    p->fpml = 30.0f;
    p->quellart = 1;
    p->eprecond = 1;
    p->max_shots = 1;
    p->compat_fd12 = 1;
}

extern "C" const char *dsh_error_string(int s)
{
    switch (s) {
    case DSH_OK: return "ok";
    case DSH_ERR_PARAM: return "invalid parameter";
    case DSH_ERR_CUDA: return "CUDA error";
    case DSH_ERR_OOM: return "out of device memory or budget";
    case DSH_ERR_UNSTABLE: return "simulation is unstable (non-finite wavefield)";
    case DSH_ERR_STATE: return "call out of order";
    case DSH_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
    }
}

static int check_params(const dsh_params *p)
{
    if (p->nx < 1 || p->ny < 1 || p->nt < 1) return DSH_ERR_PARAM;
    if (p->fdorder < 2 || p->fdorder > 12 || (p->fdorder & 1)) return DSH_ERR_PARAM;
    if (p->maxrelerror < 0 || p->maxrelerror > 4) return DSH_ERR_PARAM;
    if (p->fw < 0 || p->fw > DSH_MAX_FW || p->fw > p->nx || p->fw > p->ny) return DSH_ERR_PARAM;
    if (p->l < 0 || p->l > DSH_MAX_L) return DSH_ERR_PARAM;
    if (!(p->dh > 0) || !(p->dt > 0)) return DSH_ERR_PARAM;
    for (int l = 0; l < p->l; l++)
        if (!(p->fl[l] > 0)) return DSH_ERR_PARAM;
    if (p->eprecond != 0 && p->eprecond != 1 && p->eprecond != 3 && p->eprecond != DSH_EPRECOND_ENERGY_ONLY)
        return DSH_ERR_PARAM;
    if (p->max_shots < 1 || p->max_shots > 65535) return DSH_ERR_PARAM;
    if (p->ckpt_every < 0) return DSH_ERR_PARAM;
    if (p->grad_q != 0 && (p->grad_q != 1 || p->l < 1)) return DSH_ERR_PARAM;   /* Qs gradient: viscoelastic only */
    if (p->nx > 65000 || p->ny > 65000) return DSH_ERR_PARAM;
    if (p->quellart != 1 && p->quellart != 2 && p->quellart != 3 && p->quellart != 4 && p->quellart != 5 &&
        p->quellart != 6)
        return DSH_ERR_PARAM;
    return DSH_OK;
}

extern "C" dsh_ctx *dsh_create(const dsh_params *p, int device, int *status)
{
    int rc = check_params(p);
    if (rc != DSH_OK) { if (status) *status = rc; return nullptr; }
    dsh_ctx *ctx = new dsh_ctx();
    ctx->p = *p;
    ctx->dev = device;
    auto bail = [&](int code) { if (status) *status = code; dsh_destroy(ctx); return (dsh_ctx *)nullptr; };
    if (cudaSetDevice(device) != cudaSuccess) return bail(DSH_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&ctx->own_st, cudaStreamNonBlocking) != cudaSuccess) return bail(DSH_ERR_CUDA);
    ctx->st = ctx->own_st;
    for (int k = 0; k < 4; k++) cudaEventCreate(&ctx->ev[k]);
    if (cudaEventCreateWithFlags(&ctx->ev_wait, cudaEventDisableTiming) != cudaSuccess) return bail(DSH_ERR_CUDA);
    const int nx = p->nx, ny = p->ny, L = p->l, fw = p->fw;
    ctx->H = p->fdorder / 2;
    ctx->hy = ctx->H;
    ctx->pitch = (int)round_up(nx + 32, 32);
    ctx->S = p->max_shots;
    ctx->fstride = round_up((long long)(ny + 2 * ctx->hy) * ctx->pitch, 32);
    ctx->dstride = round_up((long long)ny * ctx->pitch, 32);
    long long o = 0;
    ctx->o_vy = o; o += ctx->fstride;
    ctx->o_sxy = o; o += ctx->fstride;
    ctx->o_syz = o; o += ctx->fstride;
    ctx->o_r = o; o += (long long)L * ctx->dstride;
    ctx->o_q = o; o += (long long)L * ctx->dstride;
    ctx->o_pvxx = o; o += round_up((long long)ny * 2 * fw + 4, 32);
    ctx->o_psxx = o; o += round_up((long long)ny * 2 * fw + 4, 32);
    ctx->o_pvyy = o; o += round_up((long long)2 * fw * ctx->pitch + 4, 32);
    ctx->o_psyy = o; o += round_up((long long)2 * fw * ctx->pitch + 4, 32);
    /* second buffers of the fused step (vy, sxy, syz, velocity CPML memory);
       inside the state region so checkpoints hold both */
    ctx->fused_ok = p->fdorder <= 8;
    if (ctx->fused_ok) {
        ctx->o_vy_b = o; o += ctx->fstride;
        ctx->o_sxy_b = o; o += ctx->fstride;
        ctx->o_syz_b = o; o += ctx->fstride;
        ctx->o_pvxx_b = o; o += round_up((long long)ny * 2 * fw + 4, 32);
        ctx->o_pvyy_b = o; o += round_up((long long)2 * fw * ctx->pitch + 4, 32);
    }
    ctx->o_state_end = o;
    ctx->o_ws = o; o += ctx->dstride;
    ctx->o_wr = o; o += ctx->dstride;
    ctx->o_we = o; o += ctx->dstride;
    ctx->o_gu = o; o += ctx->dstride;
    ctx->o_grho = o; o += ctx->dstride;
    ctx->o_hu = o; o += ctx->dstride;
    ctx->o_hrho = o; o += ctx->dstride;
    if (p->grad_q) {                      /* Qs gradient: adjoint strains and correlation sums */
        ctx->o_exy = o; o += ctx->dstride;
        ctx->o_eyz = o; o += ctx->dstride;
        ctx->o_gqx = o; o += ctx->dstride;
        ctx->o_gqy = o; o += ctx->dstride;
    }
    ctx->slot_stride = o;
    if (cudaMalloc(&ctx->slab, (size_t)ctx->S * ctx->slot_stride * sizeof(float)) != cudaSuccess) return bail(DSH_ERR_OOM);
    build_tmaps(ctx);
    const long long nmodel = 10LL * ctx->dstride;
    if (cudaMalloc(&ctx->model, (size_t)nmodel * sizeof(float)) != cudaSuccess) return bail(DSH_ERR_OOM);
    cudaMemset(ctx->model, 0, (size_t)nmodel * sizeof(float));
    float *m = ctx->model;
    ctx->m_brho = m; m += ctx->dstride;
    ctx->m_uip = m; m += ctx->dstride;
    ctx->m_ujp = m; m += ctx->dstride;
    ctx->m_muip = m; m += ctx->dstride;
    ctx->m_mujp = m; m += ctx->dstride;
    ctx->m_tip = m; m += ctx->dstride;
    ctx->m_taus = m; m += ctx->dstride;
    ctx->m_vs = m; m += ctx->dstride;
    ctx->m_rho = m; m += ctx->dstride;
    ctx->m_qs = m;
    if (cudaMalloc(&ctx->pml, 12 * (size_t)(2 * DSH_MAX_FW + 1) * sizeof(float)) != cudaSuccess) return bail(DSH_ERR_OOM);
    if (cudaMalloc(&ctx->sums, (p->grad_q ? 8 : 6) * (size_t)ctx->dstride * sizeof(float)) != cudaSuccess)
        return bail(DSH_ERR_OOM);
    if (p->grad_q && cudaMalloc(&ctx->d_gq, (size_t)nx * ny * sizeof(float)) != cudaSuccess) return bail(DSH_ERR_OOM);
    if (cudaMalloc(&ctx->d_out, 2 * (size_t)nx * ny * sizeof(float)) != cudaSuccess) return bail(DSH_ERR_OOM);
    if (cudaMalloc(&ctx->d_nt, 4 * sizeof(int)) != cudaSuccess) return bail(DSH_ERR_OOM);
    ctx->d_status = ctx->d_nt + 1;
    ctx->d_bar = reinterpret_cast<unsigned *>(ctx->d_nt + 2);
    cudaMemset(ctx->d_nt, 0, 4 * sizeof(int));
    if (cudaMalloc(&ctx->d_part, (size_t)ctx->S * RED_BLOCKS * sizeof(double)) != cudaSuccess) return bail(DSH_ERR_OOM);
    if (cudaMalloc(&ctx->d_l2, (size_t)ctx->S * sizeof(double)) != cudaSuccess) return bail(DSH_ERR_OOM);
    if (cudaMalloc(&ctx->d_wemax, (size_t)ctx->S * sizeof(unsigned)) != cudaSuccess) return bail(DSH_ERR_OOM);
    if (cudaMalloc(&ctx->d_offs, 4 * (size_t)ctx->S * sizeof(long long)) != cudaSuccess) return bail(DSH_ERR_OOM);
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(DSH_ERR_CUDA);
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    if (status) *status = DSH_OK;
    return ctx;
}

namespace dsh::eng {
void drop_graphs(dsh_ctx *ctx)
{
    for (auto &kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
    ctx->graphs.clear();
}
}  // namespace dsh::eng

extern "C" int dsh_destroy(dsh_ctx *ctx)
{
    if (!ctx) return DSH_OK;
    cudaSetDevice(ctx->dev);
    if (ctx->st && ctx->ev_wait) wait_stream(ctx);     /* bounded: the device waits are bounded too */
    drop_graphs(ctx);
    cudaFree(ctx->slab); cudaFree(ctx->model); cudaFree(ctx->pml); cudaFree(ctx->sums); cudaFree(ctx->fwd);
    cudaFree(ctx->ckpt); cudaFree(ctx->shadow);
    cudaFree(ctx->d_geo); cudaFree(ctx->d_offs); cudaFree(ctx->d_sig); cudaFree(ctx->d_seis); cudaFree(ctx->d_res);
    cudaFree(ctx->d_obs); cudaFree(ctx->d_tmp); cudaFree(ctx->d_out); cudaFree(ctx->d_nt); cudaFree(ctx->d_part); cudaFree(ctx->d_l2);
    cudaFree(ctx->d_wemax); cudaFree(ctx->d_gq); cudaFree(ctx->d_flags);
    cudaFree(ctx->d_taper_box); cudaFree(ctx->d_taper_shot); cudaFree(ctx->d_tmap);
    for (int k = 0; k < 4; k++) if (ctx->ev[k]) cudaEventDestroy(ctx->ev[k]);
    if (ctx->ev_wait) cudaEventDestroy(ctx->ev_wait);
    if (ctx->own_st) cudaStreamDestroy(ctx->own_st);
    delete ctx;
    return DSH_OK;
}

/* ---------------- tensor maps of the TMA-staged velocity kernel ---------------- */

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn tmap_encoder()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

/* one haloed field of every shot slot: dims (pitch, ny + 2hy, S) floats,
 * row and slot strides in bytes (multiples of 16), box (bx floats, by rows,
 * 1 slot), zero fill outside */
static bool field_map(CUtensorMap *m, const dsh_ctx *ctx, const float *field, int bx, int by)
{
    EncodeTiledFn enc = tmap_encoder();
    if (!enc || !field) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)ctx->pitch, (cuuint64_t)(ctx->p.ny + 2 * ctx->hy), (cuuint64_t)ctx->S};
    const cuuint64_t strides[2] = {(cuuint64_t)ctx->pitch * 4, (cuuint64_t)ctx->slot_stride * 4};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(field), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

/* maps of sxy and syz for the slab and the shadow state (the slab's again
 * while no shadow exists); on any failure the TMA variant stays off */
static void build_tmaps(dsh_ctx *ctx)
{
    ctx->tma_ok = 0;
    const int H = ctx->p.fdorder / 2, NL = (H + 3) / 4, NR = (H - 1 + 3) / 4;
    const int bxs = 4 * (BX + NL + NR), bys = BY, bxy = 4 * BX, byy = BY + 2 * H - 1;
    alignas(64) CUtensorMap maps[4];
    const float *sh = ctx->shadow ? ctx->shadow : ctx->slab;
    if (!field_map(&maps[0], ctx, ctx->slab + ctx->o_sxy, bxs, bys) ||
        !field_map(&maps[1], ctx, ctx->slab + ctx->o_syz, bxy, byy) ||
        !field_map(&maps[2], ctx, sh + ctx->o_sxy, bxs, bys) || !field_map(&maps[3], ctx, sh + ctx->o_syz, bxy, byy))
        return;
    if (!ctx->d_tmap && cudaMalloc(&ctx->d_tmap, sizeof(maps)) != cudaSuccess) {
        cudaGetLastError();
        ctx->d_tmap = nullptr;
        return;
    }
    if (cudaMemcpy(ctx->d_tmap, maps, sizeof(maps), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    ctx->tma_ok = 1;
}

/* The per-point model coefficients on the device: the loops of
 * dsh_setup_model (brho, the harmonic averages uip/ujp with the periodic
 * one-rank neighbour) and dsh_setup_visc_base (taus = 2/Qs, its four-point
 * average tausipjp, the relaxed moduli muip/mujp) in csrc/dsh_setup.c, with
 * the same float/double expressions in the same order and no multiply-add
 * contraction, so every field is identical to the host's.  Inputs and
 * outputs are [ny][pitch] fields, point (i, j) at (j-1)*pitch + i-1+HX. */
struct ModelArgs {
    int nx, ny, pitch, l;
    float sumu;
    const float *vs, *rho, *qs;
    float *brho, *uip, *ujp, *muip, *mujp, *tip, *taus;
};

static __global__ void model_coef_kernel(ModelArgs m)
{
    const long long n = (long long)m.nx * m.ny;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(q / m.nx) + 1, i = (int)(q % m.nx) + 1;
        const int ie = i < m.nx ? i + 1 : 1, je = j < m.ny ? j + 1 : 1;   /* periodic neighbour (one rank) */
        const long long c = (long long)(j - 1) * m.pitch + (i - 1 + HX), e = (long long)(j - 1) * m.pitch + (ie - 1 + HX);
        const long long sx = (long long)(je - 1) * m.pitch + (i - 1 + HX);
        const float rho_c = m.rho[c], vs_c = m.vs[c];
        float b = 1.0 / rho_c;
        if (rho_c < 1e-20) b = 0.0;
        m.brho[c] = b;
        const float mu_c = rho_c * vs_c * vs_c;
        const float mu_e = m.rho[e] * m.vs[e] * m.vs[e];
        const float mu_s = m.rho[sx] * m.vs[sx] * m.vs[sx];
        float ui = 2.0 / ((1.0 / mu_c) + (1.0 / mu_e));
        float uj = 2.0 / ((1.0 / mu_c) + (1.0 / mu_s));
        if ((mu_c == 0.0) || (mu_e == 0.0)) ui = 0.0;
        if ((mu_c == 0.0) || (mu_s == 0.0)) uj = 0.0;
        m.uip[c] = ui;
        m.ujp[c] = uj;
        if (m.l > 0) {
            const long long se = (long long)(je - 1) * m.pitch + (ie - 1 + HX);
            const float t_c = 2.0 / m.qs[c], t_e = 2.0 / m.qs[e], t_s = 2.0 / m.qs[sx], t_se = 2.0 / m.qs[se];
            const float t_ip = 0.25 * (t_c + t_e + t_s + t_se);
            const float u_jp = uj / (1.0 + m.sumu * t_c);
            const float u_ip = ui / (1.0 + m.sumu * t_ip);
            m.taus[c] = t_c;
            m.tip[c] = t_ip;
            m.mujp[c] = u_jp;
            m.muip[c] = u_ip;
        }
    }
}

static int upload_field(dsh_ctx *ctx, float *dst, const float *src)
{
    CK(cudaMemcpy2DAsync(dst + HX, (size_t)ctx->pitch * sizeof(float), src, (size_t)ctx->p.nx * sizeof(float),
                         (size_t)ctx->p.nx * sizeof(float), ctx->p.ny, cudaMemcpyHostToDevice, ctx->st));
    return DSH_OK;
}

extern "C" int dsh_set_model(dsh_ctx *ctx, const float *vs, const float *rho, const float *qs)
{
    if (!ctx || !vs || !rho || (ctx->p.l > 0 && !qs)) return DSH_ERR_PARAM;
    CK(cudaSetDevice(ctx->dev));
    const dsh_params &p = ctx->p;
    const int L = p.l;
    const size_t n = (size_t)p.nx * p.ny;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (long long k = 0; k < (long long)n; k++) {
        if (!std::isfinite(vs[k]) || !std::isfinite(rho[k]) || vs[k] < 0 || rho[k] < 0) bad |= 1;
        if (L > 0 && !(qs[k] > 0)) bad |= 1;
    }
    if (bad) return DSH_ERR_PARAM;
    if (dsh_setup_holberg(p.fdorder, p.maxrelerror, ctx->hc) != 0) return DSH_ERR_PARAM;
    if (L > 0) {
        if (dsh_setup_sls(L, p.fl, p.dt, ctx->eta, ctx->bip, ctx->bjm, ctx->cip, ctx->cjm) != 0) return DSH_ERR_PARAM;
        ctx->sumu = dsh_setup_sumu(L, p.fl);
    }
    dsh_pml pml;
    float damping = p.damping;
    if (!(damping > 0)) damping = *std::max_element(vs, vs + n);
    dsh_setup_pml(p.nx, p.ny, p.fw, p.dh, p.dt, damping, p.fpml, p.npower, p.k_max_pml, &pml);
    const float *vecs[12] = {pml.K_x, pml.a_x, pml.b_x, pml.K_x_half, pml.a_x_half, pml.b_x_half,
                             pml.K_y, pml.a_y, pml.b_y, pml.K_y_half, pml.a_y_half, pml.b_y_half};
    const size_t vlen = 2 * DSH_MAX_FW + 1;
    std::vector<float> pmlh(12 * vlen);
    for (int k = 0; k < 12; k++) memcpy(&pmlh[k * vlen], vecs[k], vlen * sizeof(float));
    CK(cudaMemcpyAsync(ctx->pml, pmlh.data(), pmlh.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->st));
    /* the model in, the coefficient fields formed on the device */
    int rc;
    if ((rc = upload_field(ctx, ctx->m_vs, vs)) != DSH_OK) return rc;
    if ((rc = upload_field(ctx, ctx->m_rho, rho)) != DSH_OK) return rc;
    if (L > 0 && (rc = upload_field(ctx, ctx->m_qs, qs)) != DSH_OK) return rc;
    ModelArgs ma;
    ma.nx = p.nx; ma.ny = p.ny; ma.pitch = ctx->pitch; ma.l = L; ma.sumu = ctx->sumu;
    ma.vs = ctx->m_vs; ma.rho = ctx->m_rho; ma.qs = ctx->m_qs;
    ma.brho = ctx->m_brho; ma.uip = ctx->m_uip; ma.ujp = ctx->m_ujp;
    ma.muip = ctx->m_muip; ma.mujp = ctx->m_mujp; ma.tip = ctx->m_tip; ma.taus = ctx->m_taus;
    model_coef_kernel<<<(unsigned)std::min<long long>(((long long)n + 255) / 256, 148LL * 8), 256, 0, ctx->st>>>(ma);
    CK(cudaGetLastError());
    /* meanwhile on the host: the vs/rho means (a sequential float sum in the reference's order) */
    dsh_setup_cnorm(p.nx, p.ny, vs, rho, ctx->cnorm);
    ctx->gq_valid = 0;
    WAIT(ctx);   /* the caller's arrays and the staging vector are free again once this returns */
    ctx->model_set = 1;
    return DSH_OK;
}

/* ---------------- geometry of one batch ---------------- */

static bool in_grid(const dsh_params &p, int i, int j) { return i >= 0 && i <= p.nx + 1 && j >= 0 && j <= p.ny + 1; }

/* Uploads sources, receivers, forward signals and (optionally) observed data
 * of shots[0..nb) into slots 0..nb).  Sources at one grid point form a group
 * (members in source order); groups and receivers are also listed per thread
 * block tile for the fused injection/sampling of the velocity kernel. */
namespace dsh::eng {
int upload_batch(dsh_ctx *ctx, const dsh_shot *shots, int nb, const float *obs_host, const float *obs_dev,
                 long long obs_dev_off)
{
    const dsh_params &p = ctx->p;
    const int NT = p.nt, S = ctx->S;
    const int gx = (p.nx + 4 * BX - 1) / (4 * BX), gy = (p.ny + BY - 1) / BY, T = gx * gy;
    std::vector<int> fgrp_off(S + 1), agrp_off(S + 1), rec_off(S + 1);
    std::vector<int> ftile(S * (T + 1)), atile(S * (T + 1)), rtile(S * (T + 1));
    std::vector<int> grp_pt, grp_beg, src_id, rec_pt, gpk, rpk, rid;
    std::vector<long long> sig_off(S, 0), seis_off(S, 0), obs_off(S, 0), out_off(S, 0);
    long long nsig = 0, nseis = 0;
    bool fused = true;
    ctx->ntr_b.assign(nb, 0);
    auto pt_of = [&](int i, int j) { return (int)((long long)(j - 1 + ctx->hy) * ctx->pitch + (i - 1 + HX)); };
    auto tile_of = [&](int i, int j) {
        if (i < 1 || i > p.nx || j < 1 || j > p.ny) return -1;
        return ((j - 1) / BY) * gx + (i - 1) / (4 * BX);
    };
    struct Grp { int i, j, tile; std::vector<int> members; };
    /* appends groups (sorted by tile, stable) and fills the tile table of slot s */
    auto emit = [&](std::vector<Grp> &gs, int *tab) {
        std::stable_sort(gs.begin(), gs.end(), [](const Grp &x, const Grp &y) { return x.tile < y.tile; });
        size_t k = 0;
        for (int t = 0; t <= T; t++) {
            while (k < gs.size() && gs[k].tile < t) k++;
            tab[t] = (int)grp_pt.size() + (int)k;
        }
        for (auto &g : gs) {
            grp_pt.push_back(pt_of(g.i, g.j));
            gpk.push_back((g.j << 16) | (g.i & 0xffff));
            grp_beg.push_back((int)src_id.size());
            for (int m : g.members) src_id.push_back(m);
        }
    };
    auto group = [&](int n, auto pos_i, auto pos_j, auto use) {
        std::map<int, int> idx;
        std::vector<Grp> gs;
        for (int k = 0; k < n; k++) {
            if (!use(k)) continue;
            const int i = pos_i(k), j = pos_j(k);
            const int key = pt_of(i, j);
            auto it = idx.find(key);
            if (it == idx.end()) { idx[key] = (int)gs.size(); gs.push_back({i, j, tile_of(i, j), {k}}); }
            else gs[it->second].members.push_back(k);
            if (tile_of(i, j) < 0) fused = false;
        }
        return gs;
    };
    for (int s = 0; s < nb; s++) {
        const dsh_shot &sh = shots[s];
        if (sh.nsrc < 0 || sh.ntr < 0 || (sh.nsrc > 0 && !sh.srcpos) || (sh.ntr > 0 && !sh.recpos)) return DSH_ERR_PARAM;
        for (int k = 0; k < sh.nsrc; k++)
            if (!in_grid(p, (int)sh.srcpos[k], (int)sh.srcpos[sh.nsrc + k])) return DSH_ERR_PARAM;
        for (int r = 0; r < sh.ntr; r++)
            if (!in_grid(p, sh.recpos[r], sh.recpos[sh.ntr + r])) return DSH_ERR_PARAM;
    }
    /* forward groups: type-3 sources (update_v_PML.c:569) */
    for (int s = 0; s < S; s++) {
        fgrp_off[s] = (int)grp_pt.size();
        std::vector<Grp> gs;
        if (s < nb) {
            const dsh_shot &sh = shots[s];
            gs = group(sh.nsrc, [&](int k) { return (int)sh.srcpos[k]; },
                       [&](int k) { return (int)sh.srcpos[sh.nsrc + k]; },
                       [&](int k) { return (int)sh.srcpos[7 * sh.nsrc + k] == 3; });
            sig_off[s] = nsig;
            nsig += (long long)sh.nsrc * NT;
        }
        emit(gs, &ftile[s * (T + 1)]);
    }
    fgrp_off[S] = (int)grp_pt.size();
    /* adjoint groups: receivers inject the residual (update_v_PML.c:576-583) */
    for (int s = 0; s < S; s++) {
        agrp_off[s] = (int)grp_pt.size();
        std::vector<Grp> gs;
        if (s < nb) {
            const dsh_shot &sh = shots[s];
            gs = group(sh.ntr, [&](int r) { return sh.recpos[r]; }, [&](int r) { return sh.recpos[sh.ntr + r]; },
                       [](int) { return true; });
        }
        emit(gs, &atile[s * (T + 1)]);
    }
    agrp_off[S] = (int)grp_pt.size();
    grp_beg.push_back((int)src_id.size());
    /* receivers: original order (fallback kernel) and per tile (fused sampling) */
    for (int s = 0; s < S; s++) {
        rec_off[s] = (int)rec_pt.size();
        std::vector<std::pair<int, int>> ent;       /* (tile, r) */
        if (s < nb) {
            const dsh_shot &sh = shots[s];
            for (int r = 0; r < sh.ntr; r++) {
                const int i = sh.recpos[r], j = sh.recpos[sh.ntr + r];
                rec_pt.push_back(pt_of(i, j));
                ent.push_back({tile_of(i, j), r});
            }
            std::stable_sort(ent.begin(), ent.end(), [](auto &x, auto &y) { return x.first < y.first; });
            ctx->ntr_b[s] = sh.ntr;
            seis_off[s] = nseis;
            out_off[s] = nseis;
            obs_off[s] = obs_dev ? obs_dev_off + nseis : nseis;
            nseis += (long long)sh.ntr * NT;
        }
        size_t k = 0;
        for (int t = 0; t <= T; t++) {
            while (k < ent.size() && ent[k].first < t) k++;
            rtile[s * (T + 1) + t] = (int)rpk.size() + (int)k;
        }
        for (auto &e : ent) {
            const int r = e.second;
            rpk.push_back((shots[s].recpos[shots[s].ntr + r] << 16) | (shots[s].recpos[r] & 0xffff));
            rid.push_back(r);
        }
    }
    rec_off[S] = (int)rec_pt.size();
    ctx->geo_max_groups = ctx->geo_max_members = ctx->geo_max_ntr = 0;
    for (int s = 0; s < nb; s++) {
        ctx->geo_max_groups = std::max(ctx->geo_max_groups, fgrp_off[s + 1] - fgrp_off[s]);
        for (int g = fgrp_off[s]; g < fgrp_off[s + 1]; g++)
            ctx->geo_max_members = std::max(ctx->geo_max_members, grp_beg[g + 1] - grp_beg[g]);
        ctx->geo_max_ntr = std::max(ctx->geo_max_ntr, ctx->ntr_b[s]);
    }

    /* fused step: per slot and 128 x 16 tile, the groups whose point lies in
     * the tile's velocity region (the tile grown by H-1 points left / above
     * and H right / below) */
    const int H = p.fdorder / 2;
    const int fgx = (p.nx + FTX - 1) / FTX, fgy = (p.ny + FTY - 1) / FTY, FT = fgx * fgy;
    std::vector<int> fvoff(2 * S * (FT + 1)), fvids;
    for (int pass = 0; pass < 2; pass++) {
        const std::vector<int> &goff_s = pass ? agrp_off : fgrp_off;
        for (int s = 0; s < S; s++) {
            std::vector<std::pair<int, int>> ent;     /* (tile, group) */
            for (int g = goff_s[s]; g < goff_s[s + 1]; g++) {
                const int i = gpk[g] & 0xffff, j = gpk[g] >> 16;
                for (int ty = std::max(0, (j - 1) / FTY - 1); ty <= std::min(fgy - 1, (j - 1) / FTY + 1); ty++)
                    for (int tx = std::max(0, (i - 1) / FTX - 1); tx <= std::min(fgx - 1, (i - 1) / FTX + 1); tx++)
                        if (i >= tx * FTX + 2 - H && i <= tx * FTX + FTX + H && j >= ty * FTY + 2 - H &&
                            j <= ty * FTY + FTY + H)
                            ent.push_back({ty * fgx + tx, g});
            }
            std::stable_sort(ent.begin(), ent.end(), [](auto &x, auto &y) { return x.first < y.first; });
            int *tab = &fvoff[(size_t)(pass * S + s) * (FT + 1)];
            size_t k = 0;
            for (int t = 0; t <= FT; t++) {
                while (k < ent.size() && ent[k].first < t) k++;
                tab[t] = (int)fvids.size() + (int)k;
            }
            for (auto &e : ent) fvids.push_back(e.second);
        }
    }

    /* one int buffer: fixed tables, then 8 variable sections of capacity cp */
    const long long F = 3LL * (S + 1) + 3LL * S * (T + 1) + 2LL * S * (FT + 1);
    const long long maxlen = (long long)std::max({grp_pt.size(), grp_beg.size(), src_id.size(), rec_pt.size(),
                                                  gpk.size(), rpk.size(), rid.size(), fvids.size()}) + 1;
    bool realloc = false;
    if (F + 8 * maxlen > ctx->geo_cap) {
        cudaFree(ctx->d_geo);
        ctx->d_geo = nullptr;
        const long long cp_old = ctx->geo_cap > F ? (ctx->geo_cap - F) / 8 : 0;
        ctx->geo_cap = F + 8 * std::max(maxlen, 2 * cp_old);
        CK(cudaMalloc(&ctx->d_geo, (size_t)ctx->geo_cap * sizeof(int)));
        realloc = true;
    }
    const long long cp = (ctx->geo_cap - F) / 8;
    int *G = ctx->d_geo;
    ctx->d_fgrp_off = G; ctx->d_agrp_off = G + (S + 1); ctx->d_rec_off = G + 2 * (S + 1);
    ctx->d_ftile = G + 3 * (S + 1); ctx->d_atile = ctx->d_ftile + S * (T + 1); ctx->d_rtile = ctx->d_atile + S * (T + 1);
    ctx->d_grp_pt = G + F; ctx->d_grp_beg = ctx->d_grp_pt + cp; ctx->d_src_id = ctx->d_grp_beg + cp;
    ctx->d_rec_pt = ctx->d_src_id + cp; ctx->d_gpk = ctx->d_rec_pt + cp; ctx->d_rpk = ctx->d_gpk + cp;
    ctx->d_rid = ctx->d_rpk + cp;
    ctx->d_fvoff = ctx->d_rtile + S * (T + 1); ctx->d_avoff = ctx->d_fvoff + S * (FT + 1);
    ctx->d_fvids = ctx->d_rid + cp;
    ctx->fvg_ntiles = FT;
    ctx->ntiles = T;
    ctx->fused_inject = fused && getenv("DSH_NO_FUSED_INJECT") == nullptr;
    std::vector<int> host((size_t)ctx->geo_cap, 0);
    auto put = [&](long long off, const std::vector<int> &v) { if (!v.empty()) memcpy(&host[off], v.data(), v.size() * sizeof(int)); };
    put(0, fgrp_off); put(S + 1, agrp_off); put(2 * (S + 1), rec_off);
    put(3 * (S + 1), ftile); put(3 * (S + 1) + S * (T + 1), atile); put(3 * (S + 1) + 2 * S * (T + 1), rtile);
    put(F, grp_pt); put(F + cp, grp_beg); put(F + 2 * cp, src_id); put(F + 3 * cp, rec_pt);
    put(F + 4 * cp, gpk); put(F + 5 * cp, rpk); put(F + 6 * cp, rid);
    put(3 * (S + 1) + 3 * S * (T + 1), fvoff); put(F + 7 * cp, fvids);
    CK(cudaMemcpyAsync(ctx->d_geo, host.data(), (size_t)ctx->geo_cap * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    WAIT(ctx);

    /* signals */
    if (nsig > ctx->cap_sig) {
        cudaFree(ctx->d_sig);
        ctx->cap_sig = std::max(nsig, 2 * ctx->cap_sig);
        CK(cudaMalloc(&ctx->d_sig, (size_t)ctx->cap_sig * sizeof(float)));
        realloc = true;
    }
    if (nsig > 0) {
        std::vector<float> sig((size_t)nsig);
        for (int s = 0; s < nb; s++) {
            const dsh_shot &sh = shots[s];
            if (sh.nsrc == 0) continue;
            float *dst = &sig[(size_t)sig_off[s]];
            if (sh.signals) memcpy(dst, sh.signals, (size_t)sh.nsrc * NT * sizeof(float));
            else if (p.quellart == 3 || dsh_setup_wavelet(p.quellart, NT, p.dt, sh.nsrc, sh.srcpos, dst) != 0)
                return DSH_ERR_PARAM;
        }
        CK(cudaMemcpyAsync(ctx->d_sig, sig.data(), (size_t)nsig * sizeof(float), cudaMemcpyHostToDevice, ctx->st));
        WAIT(ctx);
    }
    /* seismograms, residuals, observed data, transposed output */
    const long long nseis_cap = std::max(nseis, 1LL);
    if (nseis_cap > ctx->cap_seis) {
        cudaFree(ctx->d_seis); cudaFree(ctx->d_res); cudaFree(ctx->d_tmp);
        ctx->cap_seis = std::max(nseis_cap, 2 * ctx->cap_seis);
        CK(cudaMalloc(&ctx->d_seis, (size_t)ctx->cap_seis * sizeof(float)));
        CK(cudaMalloc(&ctx->d_res, (size_t)ctx->cap_seis * sizeof(float)));
        CK(cudaMalloc(&ctx->d_tmp, (size_t)ctx->cap_seis * sizeof(float)));
        realloc = true;
    }
    if (obs_host) {
        if (nseis_cap > ctx->cap_obs) {
            cudaFree(ctx->d_obs);
            ctx->cap_obs = std::max(nseis_cap, 2 * ctx->cap_obs);
            CK(cudaMalloc(&ctx->d_obs, (size_t)ctx->cap_obs * sizeof(float)));
        }
        if (nseis > 0)
            CK(cudaMemcpyAsync(ctx->d_obs, obs_host, (size_t)nseis * sizeof(float), cudaMemcpyHostToDevice, ctx->st));
    }
    std::vector<long long> offs(4 * (size_t)ctx->S);
    memcpy(&offs[0], sig_off.data(), ctx->S * sizeof(long long));
    memcpy(&offs[ctx->S], seis_off.data(), ctx->S * sizeof(long long));
    memcpy(&offs[2 * ctx->S], obs_off.data(), ctx->S * sizeof(long long));
    memcpy(&offs[3 * ctx->S], out_off.data(), ctx->S * sizeof(long long));
    CK(cudaMemcpyAsync(ctx->d_offs, offs.data(), offs.size() * sizeof(long long), cudaMemcpyHostToDevice, ctx->st));
    WAIT(ctx);
    if (realloc) { drop_graphs(ctx); ctx->geo_version++; }
    return DSH_OK;
}
}  // namespace dsh::eng

/* ---------------- passes ---------------- */

/* DH = 2^k: x/DH and x*(1/DH) are the same correctly rounded number */
namespace dsh::eng {
bool dh_pow2(float dh)
{
    int e;
    return dh > 0 && std::frexp(dh, &e) == 0.5f;
}
}  // namespace dsh::eng

namespace dsh::eng {
/* L2 policy of a pass (StepArgs::l2_stream): the fields the velocity kernel
 * reads every half-step (vy, sxy, syz of every slot, 1/rho, and in the
 * adjoint the g_rho, g_u and Wr sums) stay evict-last.  If they fit half the
 * L2, the memory variables (read and written once per step, bit 0) are
 * streamed evict-first so that they do not displace those fields, and with a
 * single shot slot the stress model factors too (bit 1; with several slots
 * every slot of the launch re-reads them).  A single-shot 2000 x 800
 * viscoelastic gradient: 38.0 -> 42.0 Gpt/s.  With more (64 slots of
 * 1000 x 300: 230 MB) everything keeps the evict-last policy, which measured
 * faster there.  DSH_L2_STREAM=<mask> fixes the choice. */
int l2_stream(const dsh_ctx *ctx, Pass pass)
{
    static const char *env = getenv("DSH_L2_STREAM");
    if (env) return atoi(env) & 3;
    int l2 = 0;
    if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, ctx->dev) != cudaSuccess || l2 <= 0) return 0;
    const long long per_slot = 3 * ctx->fstride + (pass == P_ADJ ? 3 * ctx->dstride : 0);
    const long long bytes = 4 * ((long long)ctx->S * per_slot + ctx->dstride);
    if (bytes > (long long)l2 / 2) return 0;
    return ctx->S == 1 ? 3 : 1;
}

StepArgs step_args(dsh_ctx *ctx, Pass pass)
{
    const dsh_params &p = ctx->p;
    StepArgs a;
    memset(&a, 0, sizeof(a));
    a.nx = p.nx; a.ny = p.ny; a.pitch = ctx->pitch; a.hy = ctx->hy; a.fw = p.fw; a.free_surf = p.free_surf;
    a.l = p.l; a.fd12_compat = p.compat_fd12;
    a.fdo = p.fdorder; a.p2 = dh_pow2(p.dh) ? 1 : 0; a.nslots = ctx->S;
    a.l2_stream = l2_stream(ctx, pass);
    a.nt_last = p.nt; a.nt_total = p.nt; a.nt_base = ctx->d_nt;
    a.chk_mask = 15;
    a.fstride = ctx->fstride; a.dstride = ctx->dstride; a.slot_stride = ctx->slot_stride;
    for (int k = 0; k < 7; k++) a.hc[k] = ctx->hc[k];
    a.dt = p.dt; a.dh = p.dh;
    a.inv_dh = (float)(1.0 / (double)p.dh);
    a.dhi_el = p.dt / p.dh;
    a.dhi_visc = (float)(1.0 / (double)p.dh);
    a.dthalbe = (float)((double)p.dt / 2.0);
    const size_t vlen = 2 * DSH_MAX_FW + 1;
    const float *pm = ctx->pml;
    a.pml.K_x = pm; a.pml.a_x = pm + vlen; a.pml.b_x = pm + 2 * vlen;
    a.pml.K_x_half = pm + 3 * vlen; a.pml.a_x_half = pm + 4 * vlen; a.pml.b_x_half = pm + 5 * vlen;
    a.pml.K_y = pm + 6 * vlen; a.pml.a_y = pm + 7 * vlen; a.pml.b_y = pm + 8 * vlen;
    a.pml.K_y_half = pm + 9 * vlen; a.pml.a_y_half = pm + 10 * vlen; a.pml.b_y_half = pm + 11 * vlen;
    float *sl = (pass == P_RECOMP) ? ctx->shadow : ctx->slab;
    a.vy = sl + ctx->o_vy; a.sxy = sl + ctx->o_sxy; a.syz = sl + ctx->o_syz;
    a.r = sl + ctx->o_r; a.q = sl + ctx->o_q;
    a.psi_vxx = sl + ctx->o_pvxx; a.psi_sxx = sl + ctx->o_psxx;
    a.psi_vyy_v = sl + ctx->o_pvyy; a.psi_syy = sl + ctx->o_psyy;
    a.gu = sl + ctx->o_gu; a.grho = sl + ctx->o_grho; a.hu = sl + ctx->o_hu; a.hrho = sl + ctx->o_hrho;
    if (ctx->fused_ok) {
        a.vy_b = sl + ctx->o_vy_b; a.sxy_b = sl + ctx->o_sxy_b; a.syz_b = sl + ctx->o_syz_b;
        a.psi_vxx_b = sl + ctx->o_pvxx_b; a.psi_vyy_v_b = sl + ctx->o_pvyy_b;
        a.fvg_off = pass == P_ADJ ? ctx->d_avoff : ctx->d_fvoff;
        a.fvg_ids = ctx->d_fvids;
        a.fvg_ntiles = ctx->fvg_ntiles;
    }
    a.brho = ctx->m_brho; a.uip = ctx->m_uip; a.ujp = ctx->m_ujp;
    a.muip = ctx->m_muip; a.mujp = ctx->m_mujp; a.tausipjp = ctx->m_tip; a.taus = ctx->m_taus;
    for (int l = 0; l < 4; l++) a.eta[l] = ctx->eta[l];
    a.lf = (float)p.l;
    a.sumu = ctx->sumu;
    if (p.grad_q) {
        a.exy = sl + ctx->o_exy; a.eyz = sl + ctx->o_eyz; a.gqx = sl + ctx->o_gqx; a.gqy = sl + ctx->o_gqy;
    }
    for (int l = 0; l < 4; l++) { a.bip[l] = ctx->bip[l]; a.bjm[l] = ctx->bjm[l]; a.cip[l] = ctx->cip[l]; a.cjm[l] = ctx->cjm[l]; }
    a.fwd_slot_stride = ctx->fwd_slot_stride;
    a.fwd_mod = ctx->fwd_mod > 0 ? ctx->fwd_mod : p.nt;
    a.fwd_step_stride = ctx->fwd_step_stride;
    a.status = ctx->d_status;
    a.wait_polls = ctx->device_polls;
    if (ctx->tma_ok) {
        const CUtensorMap *tm = (const CUtensorMap *)ctx->d_tmap + (pass == P_RECOMP ? 2 : 0);
        a.tm_sxy = tm;
        a.tm_syz = tm + 1;
    }
    /* fused injection / sampling lists */
    a.tl.on = ctx->fused_inject;
    a.tl.ntiles = ctx->ntiles;
    a.tl.ntx = (p.nx + 4 * BX - 1) / (4 * BX);
    a.tl.gpt = ctx->d_gpk; a.tl.gbeg = ctx->d_grp_beg; a.tl.src_id = ctx->d_src_id;
    a.tl.roff = ctx->d_rtile; a.tl.rpt = ctx->d_rpk; a.tl.rid = ctx->d_rid; a.tl.rec_off = ctx->d_rec_off;
    a.tl.seis = ctx->d_seis; a.tl.seis_off = ctx->d_offs + ctx->S;
    if (pass == P_ADJ) {
        a.tl.goff = ctx->d_atile;
        a.tl.sig = ctx->d_res; a.tl.sig_off = ctx->d_offs + ctx->S;
        a.tl.sig_ss = p.nt; a.tl.sig_ts = 1;
        a.tl.sample = 0;
    } else {
        a.tl.goff = ctx->d_ftile;
        a.tl.sig = ctx->d_sig; a.tl.sig_off = ctx->d_offs;
        a.tl.sig_ss = p.nt; a.tl.sig_ts = 1;
        a.tl.sample = (pass == P_FWD_HESS || pass == P_RECOMP) ? 0 : 1;
    }
    switch (pass) {
    case P_FWD_PLAIN:
        break;
    case P_FWD_STORE:
        a.fwd = ctx->fwd;
        if (p.eprecond == 1 || p.eprecond == 3 || p.eprecond == DSH_EPRECOND_ENERGY_ONLY) a.ws = sl + ctx->o_ws;
        break;
    case P_FWD_CKPT:
        if (p.eprecond == 1 || p.eprecond == 3 || p.eprecond == DSH_EPRECOND_ENERGY_ONLY) a.ws = sl + ctx->o_ws;
        break;
    case P_RECOMP:
        a.fwd = ctx->fwd;
        break;
    case P_FWD_HESS:
        break;
    case P_ADJ:
        a.fwd = ctx->fwd;
        if (p.eprecond == 1 || p.eprecond == DSH_EPRECOND_ENERGY_ONLY) a.ws = sl + ctx->o_wr;
        break;
    }
    return a;
}
}  // namespace dsh::eng

namespace dsh::eng {
InjectArgs inject_args(dsh_ctx *ctx, Pass pass)
{
    InjectArgs a;
    memset(&a, 0, sizeof(a));
    a.nt_base = ctx->d_nt;
    a.nt_last = ctx->p.nt;
    a.nt_total = ctx->p.nt;
    a.slot_stride = ctx->slot_stride;
    a.vy = (pass == P_RECOMP ? ctx->shadow : ctx->slab) + ctx->o_vy;
    a.grp_pt = ctx->d_grp_pt; a.grp_beg = ctx->d_grp_beg; a.src_id = ctx->d_src_id;
    a.rec_off = ctx->d_rec_off; a.rec_pt = ctx->d_rec_pt;
    a.seis = ctx->d_seis; a.seis_off = ctx->d_offs + ctx->S;
    if (pass == P_ADJ) {
        a.grp_off = ctx->d_agrp_off;
        a.sig = ctx->d_res; a.sig_off = ctx->d_offs + ctx->S;   /* residual [ntr][NT] at the seismogram offsets */
        a.sig_ss = ctx->p.nt; a.sig_ts = 1;
        a.sample = 0;
    } else {
        a.grp_off = ctx->d_fgrp_off;
        a.sig = ctx->d_sig; a.sig_off = ctx->d_offs;
        a.sig_ss = ctx->p.nt; a.sig_ts = 1;
        a.sample = (pass == P_FWD_HESS || pass == P_RECOMP) ? 0 : 1;
    }
    return a;
}
}  // namespace dsh::eng

/* Velocity kernel of the kernel pair: v_step (stress taps from global
 * memory through L1); DSH_VSTAGE=1 selects the shared-memory staged
 * v_step_st, which measured slower on B200 (19.2 vs 14.7 us per launch at
 * 2000 x 800, FDORDER 8: the block-wide staging and barrier cost more than the
 * L1 hits they replace). */
static int env_flag(const char *name)
{
    const char *e = getenv(name);
    return e && atoi(e) != 0;
}

/* rows per block of the stress kernel and of the velocity kernel v_step
 * (128 x rows points): 4 by default, 8 or 2 through DSH_SROWS / DSH_VBROWS.
 * On the 2000 x 800 FDORDER 8 gradient 4-row blocks measured 2 % faster
 * than 8-row ones (the stress launches 6 % faster: a shorter block lifetime
 * shortens the last, partly idle wave of each launch); 2 rows gained
 * nothing more. */
static int env_rows(const char *name)
{
    const char *e = getenv(name);
    const int r = e ? atoi(e) : 4;
    return (r == 2 || r == 4 || r == 8) ? r : 4;
}
static int s_rows()
{
    static const int r = env_rows("DSH_SROWS");
    return r;
}
static int v_rows()
{
    static const int r = env_rows("DSH_VBROWS");
    return r;
}

/* the velocity kernel of the pair: code 0 v_step, 1 v_step_st (DSH_VSTAGE=1
 * or the autotuner), 2 the persistent TMA-staged v_step_tp (DSH_VTMA=1; it
 * needs the context's tensor maps) */
struct VPick {
    KFn k;
    int code;
};

static VPick pick_v(const dsh_ctx *ctx, int fdo, int vflags, bool p2)
{
    static const int env = env_flag("DSH_VSTAGE");
    static const int env_tma = env_flag("DSH_VTMA");
    static const int env_rows = getenv("DSH_VROWS") ? atoi(getenv("DSH_VROWS")) : 1;
    const bool staged = ctx->sel_staged >= 0 ? ctx->sel_staged != 0 : env != 0;
    KFn k = staged ? v_kernel_st(fdo, vflags, p2) : nullptr;
    if (k) return {k, 1};
    if (env_tma && ctx->tma_ok && (k = v_kernel_tp(fdo, vflags, p2))) return {k, 2};
    const bool rows2 = ctx->sel_rows >= 0 ? ctx->sel_rows != 0 : env_rows == 2;
    if (rows2 && (k = v_kernel_r2(fdo, vflags, p2))) return {k, 3};
    return {v_kernel(fdo, vflags, p2), 0};
}

/* launch shape of the picked velocity kernel for nb slots: the tile grid, or
 * for the persistent one about two blocks per SM shared among the slots */
static void v_shape(const dsh_ctx *ctx, const VPick &v, int nb, dim3 *grid, dim3 *block)
{
    const dsh_params &p = ctx->p;
    const unsigned gx = (unsigned)((p.nx + 4 * BX - 1) / (4 * BX)), gy = (unsigned)((p.ny + BY - 1) / BY);
    if (v.code == 2) {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->dev);
        const unsigned per = (unsigned)std::max(1, 2 * nsm / std::max(1, nb));
        *grid = dim3(std::min(per, gx * gy), (unsigned)nb, 1);
        *block = dim3(BX, BY + 1, 1);           /* 8 computing warps + 1 producer warp */
    } else if (v.code == 0) {
        const int vr = v_rows();
        *grid = dim3(gx, (unsigned)((p.ny + vr - 1) / vr), (unsigned)nb);
        *block = dim3(BX, vr, 1);
    } else {
        *grid = dim3(gx, gy, (unsigned)nb);
        *block = dim3(BX, v.code == 3 ? BY / 2 : BY, 1);
    }
}

/* graph key code of the velocity kernel in use */
static long long v_code(const dsh_ctx *ctx) { return pick_v(ctx, ctx->p.fdorder, 0, dh_pow2(ctx->p.dh)).code; }

/* The fused step (one kernel per time step, dsh_fused.cuh) serves every pass
 * but the Hessian one when FDORDER <= 8 and injection/sampling are fused;
 * DSH_FUSED=0 selects the velocity + stress kernel pair instead. */
static bool use_fused(dsh_ctx *ctx, Pass pass)
{
    static const int env = env_flag("DSH_FUSED");
    const bool on = ctx->sel_fused >= 0 ? ctx->sel_fused != 0 : env != 0;
    return on && ctx->fused_ok && ctx->fused_inject && pass != P_FWD_HESS && !ctx->p.grad_q;
}

static int fused_mode(Pass pass)
{
    return pass == P_ADJ ? FM_ADJ : (pass == P_FWD_STORE || pass == P_RECOMP) ? FM_STORE : FM_FWD;
}

static int launch_fused_chunk(dsh_ctx *ctx, Pass pass, int nb, int nsteps_in_chunk, long long *nlaunch)
{
    const dsh_params &p = ctx->p;
    KFn fk = fs_kernel(p.fdorder, p.l, fused_mode(pass), dh_pow2(p.dh));
    if (!fk) return DSH_ERR_PARAM;
    StepArgs sa = step_args(ctx, pass);
    dim3 grid((unsigned)((p.nx + FTX - 1) / FTX), (unsigned)((p.ny + FTY - 1) / FTY), (unsigned)nb);
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(256, 1, 1);
    cfg.stream = ctx->st;
    static const bool use_pdl = getenv("DSH_NO_PDL") == nullptr;
    for (int k = 0; k < nsteps_in_chunk; k++) {
        int off = k;
        void *args[2] = {&sa, &off};
        cfg.attrs = (use_pdl && k > 0) ? &attr : nullptr;
        cfg.numAttrs = (use_pdl && k > 0) ? 1 : 0;
        CK(cudaLaunchKernelExC(&cfg, (const void *)fk, args));
        *nlaunch += 1;
    }
    advance_step<<<1, 1, 0, ctx->st>>>(ctx->d_nt, nsteps_in_chunk);
    *nlaunch += 1;
    CK(cudaGetLastError());
    return DSH_OK;
}

static int launch_step_chunk(dsh_ctx *ctx, Pass pass, int nb, int nsteps_in_chunk, long long *nlaunch)
{
    if (use_fused(ctx, pass)) return launch_fused_chunk(ctx, pass, nb, nsteps_in_chunk, nlaunch);
    const dsh_params &p = ctx->p;
    int vflags = 0, sflags = 0;
    switch (pass) {
    case P_FWD_PLAIN: break;
    case P_FWD_STORE: sflags = SF_STRAIN_OUT; break;
    case P_FWD_HESS: vflags = VF_HESS; sflags = SF_HESS; break;
    case P_ADJ: vflags = VF_ADJOINT | VF_CORR; sflags = SF_CORR; break;
    case P_FWD_CKPT: break;
    case P_RECOMP: sflags = SF_STRAIN_OUT; break;
    }
    if (p.grad_q && (sflags == SF_STRAIN_OUT || sflags == SF_CORR))   /* the Qs gradient's two halves */
        sflags |= sflags == SF_CORR ? SF_CORRQ : SF_QSENS;
    const VPick vp = pick_v(ctx, p.fdorder, vflags, dh_pow2(p.dh));
    KFn vk = vp.k, sk = s_kernel(p.fdorder, p.l, sflags);
    if (!vk || !sk) return DSH_ERR_PARAM;
    StepArgs sa = step_args(ctx, pass);
    InjectArgs ia = inject_args(ctx, pass);
    const int sr = s_rows();
    dim3 block(BX, sr, 1);
    dim3 grid((unsigned)((p.nx + 4 * BX - 1) / (4 * BX)), (unsigned)((p.ny + sr - 1) / sr), (unsigned)nb);
    dim3 vgrid, vblock;
    v_shape(ctx, vp, nb, &vgrid, &vblock);
    /* velocity and stress kernels overlap their prologues with the
     * predecessor through programmatic dependent launch; the first velocity
     * kernel of a chunk follows the step-counter update and is launched plainly */
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ctx->st;
    static const bool use_pdl = getenv("DSH_NO_PDL") == nullptr;
    for (int k = 0; k < nsteps_in_chunk; k++) {
        int off = k;
        void *args[2] = {&sa, &off};
        cfg.attrs = (use_pdl && k > 0) ? &attr : nullptr;
        cfg.numAttrs = (use_pdl && k > 0) ? 1 : 0;
        cfg.gridDim = vgrid;
        cfg.blockDim = vblock;
        CK(cudaLaunchKernelExC(&cfg, (const void *)vk, args));
        cfg.gridDim = grid;
        cfg.blockDim = block;
        if (!sa.tl.on) {
            void *iargs[2] = {&ia, &off};
            CK(cudaLaunchKernel((const void *)inject_sample, dim3(nb), dim3(128), iargs, 0, ctx->st));
            *nlaunch += 1;
        }
        cfg.attrs = use_pdl ? &attr : nullptr;
        cfg.numAttrs = use_pdl ? 1 : 0;
        CK(cudaLaunchKernelExC(&cfg, (const void *)sk, args));
        *nlaunch += 2;
    }
    advance_step<<<1, 1, 0, ctx->st>>>(ctx->d_nt, nsteps_in_chunk);
    *nlaunch += 1;
    CK(cudaGetLastError());
    return DSH_OK;
}

static int get_graph(dsh_ctx *ctx, Pass pass, int nb, int K, cudaGraphExec_t *out)
{
    const long long vcode = v_code(ctx);
    const long long key = ((long long)pass << 52) | ((long long)ctx->fused_inject << 51) |
                          ((long long)use_fused(ctx, pass) << 50) | (vcode << 45) | ((long long)K << 32) |
                          ((long long)nb << 16) | (long long)(ctx->geo_version & 0xffff);
    auto it = ctx->graphs.find(key);
    if (it != ctx->graphs.end()) { *out = it->second; return DSH_OK; }
    cudaGraph_t g;
    long long nl = 0;
    CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal));
    int rc = launch_step_chunk(ctx, pass, nb, K, &nl);
    cudaError_t e = cudaStreamEndCapture(ctx->st, &g);
    if (rc != DSH_OK) return rc;
    CK(e);
    cudaGraphExec_t exec;
    CK(cudaGraphInstantiate(&exec, g, 0));
    cudaGraphDestroy(g);
    ctx->graphs[key] = exec;
    *out = exec;
    return DSH_OK;
}

/* Small grids, plain forward modelling: the whole pass in one cooperative
 * launch of persist_fwd when all tiles of all slots fit in one wave.  Opt-in
 * (DSH_PERSIST=1): on the 500 x 200 FDORDER 4 case it measured 16.8 us per
 * step against 12.5 us for the graph-replayed kernel pair — two bounded grid
 * barriers per step cost more than the two launches they replace.  Returns
 * the grid size, 0 when not used. */
static int persistent_grid(dsh_ctx *ctx, Pass pass, int nb)
{
    static const int env = env_flag("DSH_PERSIST");
    const bool on = ctx->sel_persist >= 0 ? ctx->sel_persist != 0 : env != 0;
    const dsh_params &p = ctx->p;
    if (!on || pass != P_FWD_PLAIN || !ctx->fused_inject || p.fdorder > 8) return 0;
    PFn fk = pf_kernel(p.fdorder, p.l, dh_pow2(p.dh));
    if (!fk) return 0;
    int per_sm = 0, nsm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fk, BX * BY, 0) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->dev) != cudaSuccess) return 0;
    const long long tiles = (long long)((p.nx + 4 * BX - 1) / (4 * BX)) * ((p.ny + BY - 1) / BY) * nb;
    return tiles <= (long long)per_sm * nsm ? (int)tiles : 0;
}

static int run_persistent(dsh_ctx *ctx, Pass pass, int nb, int n0, int count, int grid)
{
    const dsh_params &p = ctx->p;
    PFn fk = pf_kernel(p.fdorder, p.l, dh_pow2(p.dh));
    StepArgs sa = step_args(ctx, pass);
    sa.nslots = nb;
    set_int_kernel<<<1, 1, 0, ctx->st>>>(ctx->d_nt, n0);
    /* completion flags of the tiles (velocity and stress step per tile and slot) */
    const long long nflags = 2LL * grid;
    if (nflags > ctx->flags_cap) {
        cudaFree(ctx->d_flags);
        ctx->d_flags = nullptr;
        ctx->flags_cap = 0;
        if (cudaMalloc(&ctx->d_flags, (size_t)nflags * sizeof(unsigned)) != cudaSuccess) {
            cudaGetLastError();
            return DSH_ERR_OOM;
        }
        ctx->flags_cap = nflags;
    }
    CK(cudaMemsetAsync(ctx->d_flags, 0, (size_t)nflags * sizeof(unsigned), ctx->st));
    unsigned *bar = ctx->d_flags;
    void *args[3] = {&sa, &count, &bar};
    CK(cudaLaunchCooperativeKernel((const void *)fk, dim3(grid), dim3(BX, BY), args, 0, ctx->st));
    ctx->launches += 2;
    ctx->state_b = 0;
    return DSH_OK;
}

/* Small elastic grids, plain forward modelling: the whole pass in one launch
 * of cl_fwd (dsh_cluster.cuh), one thread-block cluster per shot slot that
 * holds the slot's wavefield and the model in its CTAs' shared memory.  On
 * by DSH_CLUSTER=1 or the autotuner's choice; false when it does not apply
 * (viscoelastic, FDORDER > 8, positions outside the grid, strips too large
 * for one CTA's shared memory). */
static bool cluster_cfg(dsh_ctx *ctx, Pass pass, int nb, ClCfg *cfg)
{
    static const int env = env_flag("DSH_CLUSTER");
    const bool on = ctx->sel_cluster >= 0 ? ctx->sel_cluster != 0 : env != 0;
    const dsh_params &p = ctx->p;
    if (!on || pass != P_FWD_PLAIN || !ctx->fused_inject || p.l != 0 || p.fdorder > 8) return false;
    ClProblem pb;
    pb.fdorder = p.fdorder; pb.p2 = dh_pow2(p.dh) ? 1 : 0; pb.nx = p.nx; pb.ny = p.ny; pb.pitch = ctx->pitch;
    pb.fw = p.fw; pb.free_surf = p.free_surf; pb.nb = nb;
    pb.max_groups = ctx->geo_max_groups; pb.max_members = ctx->geo_max_members;
    pb.max_receivers = ctx->geo_max_ntr;
    return cl_config(pb, cfg);
}

static int run_cluster(dsh_ctx *ctx, Pass pass, int nb, int n0, int count, const ClCfg &cfg)
{
    const dsh_params &p = ctx->p;
    StepArgs sa = step_args(ctx, pass);
    sa.nslots = nb;
    set_int_kernel<<<1, 1, 0, ctx->st>>>(ctx->d_nt, n0);
    CK(cl_launch(cfg, p.fdorder, dh_pow2(p.dh), sa, count, nb, ctx->st));
    ctx->launches += 2;
    ctx->state_b = 0;
    return DSH_OK;
}

/* Small elastic grids, plain forward modelling: k time steps per launch of
 * tb_fwd (dsh_tblock.cuh), each CTA advancing its tile and a recomputed halo
 * in shared memory.  On by DSH_TBLOCK=1 or the autotuner's choice; false
 * when it does not apply (viscoelastic, FDORDER > 8, positions outside the
 * grid, more sources or receivers per shot than its lists hold). */
static bool tblock_cfg(dsh_ctx *ctx, Pass pass, int nb, TbCfg *cfg)
{
    static const int env = env_flag("DSH_TBLOCK");
    const bool on = ctx->sel_tblock >= 0 ? ctx->sel_tblock != 0 : env != 0;
    const dsh_params &p = ctx->p;
    if (!on || pass != P_FWD_PLAIN || !ctx->fused_inject || p.l != 0 || p.fdorder > 8) return false;
    TbProblem pb;
    pb.fdorder = p.fdorder; pb.p2 = dh_pow2(p.dh) ? 1 : 0; pb.nx = p.nx; pb.ny = p.ny; pb.fw = p.fw; pb.nb = nb;
    pb.max_groups = ctx->geo_max_groups; pb.max_members = ctx->geo_max_members;
    pb.max_receivers = ctx->geo_max_ntr;
    return tb_config(pb, cfg);
}

static int run_tblock(dsh_ctx *ctx, Pass pass, int nb, int n0, int count, const TbCfg &cfg)
{
    const dsh_params &p = ctx->p;
    StepArgs sa = step_args(ctx, pass);
    sa.nslots = nb;
    long long nl = 0;
    const cudaError_t e = tb_launch(cfg, p.fdorder, dh_pow2(p.dh), sa, n0, count, nb, ctx->st, &nl);
    ctx->launches += nl;
    CK(e);
    ctx->state_b = 0;
    return DSH_OK;
}

/* Steps n0 .. n0+count-1 of a pass: graphs of `chunk` steps replayed
 * count/chunk times, then one graph for the remaining steps. */
static int run_steps(dsh_ctx *ctx, Pass pass, int nb, int n0, int count)
{
    if (count <= 0) return DSH_OK;
    ClCfg ccfg;
    if (cluster_cfg(ctx, pass, nb, &ccfg)) return run_cluster(ctx, pass, nb, n0, count, ccfg);
    TbCfg tcfg;
    if (tblock_cfg(ctx, pass, nb, &tcfg)) return run_tblock(ctx, pass, nb, n0, count, tcfg);
    if (const int grid = persistent_grid(ctx, pass, nb)) return run_persistent(ctx, pass, nb, n0, count, grid);
    const int K = std::min(ctx->chunk, count);
    const int nfull = count / K, rem = count % K;
    const bool fused = use_fused(ctx, pass);
    const long long per_step = fused ? 1 : ctx->fused_inject ? 2 : 3;
    /* the fused step leaves the state of step n in buffer n & 1 */
    if (pass != P_RECOMP) ctx->state_b = fused ? ((n0 + count - 1) & 1) : 0;
    set_int_kernel<<<1, 1, 0, ctx->st>>>(ctx->d_nt, n0);
    ctx->launches += 1;
    static const bool use_graphs = getenv("DSH_NO_GRAPHS") == nullptr;
    if (!use_graphs) {
        for (int c = 0; c < nfull + (rem ? 1 : 0); c++) {
            long long nl = 0;
            int rc = launch_step_chunk(ctx, pass, nb, c < nfull ? K : rem, &nl);
            if (rc != DSH_OK) return rc;
            ctx->launches += nl;
        }
        return DSH_OK;
    }
    cudaGraphExec_t full, tail = nullptr;
    int rc = get_graph(ctx, pass, nb, K, &full);
    if (rc != DSH_OK) return rc;
    if (rem && (rc = get_graph(ctx, pass, nb, rem, &tail)) != DSH_OK) return rc;
    for (int c = 0; c < nfull; c++) CK(cudaGraphLaunch(full, ctx->st));
    if (rem) CK(cudaGraphLaunch(tail, ctx->st));
    ctx->launches += (per_step * K + 1) * nfull + (rem ? per_step * rem + 1 : 0);
    return DSH_OK;
}

static int run_pass(dsh_ctx *ctx, Pass pass, int nb) { return run_steps(ctx, pass, nb, 1, ctx->p.nt); }

/* state (wavefields, memory variables, CPML memory) of slots [0, nb):
 * copy between a slab and checkpoint k */
static int copy_state(dsh_ctx *ctx, int nb, float *dst, size_t dpitch, const float *src, size_t spitch)
{
    CK(cudaMemcpy2DAsync(dst, dpitch * sizeof(float), src, spitch * sizeof(float),
                         (size_t)ctx->o_state_end * sizeof(float), nb, cudaMemcpyDeviceToDevice, ctx->st));
    return DSH_OK;
}

/* Forward pass of a gradient: every step stored (full storage), or the state
 * saved after every C steps (checkpoint k = state after step (k+1)*C). */
static int forward_for_gradient(dsh_ctx *ctx, int nb)
{
    const int NT = ctx->p.nt;
    if (!ctx->ckpt_c) return run_pass(ctx, P_FWD_STORE, nb);
    const int C = ctx->ckpt_c, nseg = (NT + C - 1) / C;
    for (int k = 0; k < nseg; k++) {
        const int a = k * C, len = std::min(C, NT - a);
        int rc = run_steps(ctx, P_FWD_CKPT, nb, a + 1, len);
        if (rc != DSH_OK) return rc;
        if (k < nseg - 1) {
            float *dst = ctx->ckpt + (size_t)k * ctx->S * ctx->o_state_end;
            if ((rc = copy_state(ctx, nb, dst, ctx->o_state_end, ctx->slab, ctx->slot_stride)) != DSH_OK) return rc;
        }
    }
    return DSH_OK;
}

/* Adjoint pass: with checkpoints, segments are processed last to first:
 * restore the checkpoint into the shadow state, recompute the segment's
 * forward steps into the C-step buffer, then run the adjoint steps that
 * correlate with them (adjoint step nt uses forward step NT-nt+1). */
static int adjoint_for_gradient(dsh_ctx *ctx, int nb)
{
    const int NT = ctx->p.nt;
    if (!ctx->ckpt_c) return run_pass(ctx, P_ADJ, nb);
    const int C = ctx->ckpt_c, nseg = (NT + C - 1) / C;
    for (int k = nseg - 1; k >= 0; k--) {
        const int a = k * C, b = std::min(a + C, NT);
        int rc;
        if (k == 0) {
            CK(cudaMemset2DAsync(ctx->shadow, (size_t)ctx->slot_stride * sizeof(float), 0,
                                 (size_t)ctx->o_state_end * sizeof(float), nb, ctx->st));
        } else {
            const float *src = ctx->ckpt + (size_t)(k - 1) * ctx->S * ctx->o_state_end;
            if ((rc = copy_state(ctx, nb, ctx->shadow, ctx->slot_stride, src, ctx->o_state_end)) != DSH_OK) return rc;
        }
        if ((rc = run_steps(ctx, P_RECOMP, nb, a + 1, b - a)) != DSH_OK) return rc;
        if ((rc = run_steps(ctx, P_ADJ, nb, NT - b + 1, b - a)) != DSH_OK) return rc;
    }
    return DSH_OK;
}

/* zero the wavefield state of slots [0, nb) (zero_fdveps(_visc)); with
 * accumulators also the per-shot energies, gradients and Hessian sums */
namespace dsh::eng {
int zero_slots(dsh_ctx *ctx, int nb, bool accumulators)
{
    const size_t w = (size_t)(accumulators ? ctx->slot_stride : ctx->o_state_end) * sizeof(float);
    CK(cudaMemset2DAsync(ctx->slab, (size_t)ctx->slot_stride * sizeof(float), 0, w, nb, ctx->st));
    return DSH_OK;
}
}  // namespace dsh::eng

namespace dsh::eng {
int check_status(dsh_ctx *ctx)
{
    int h = 0;
    WAIT(ctx);
    CK(cudaMemcpyAsync(&h, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    WAIT(ctx);
    if (h) {
        cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->st);
        WAIT(ctx);
        return (h & 2) ? DSH_ERR_TIMEOUT : DSH_ERR_UNSTABLE;   /* bit 2: a bounded grid barrier expired */
    }
    return DSH_OK;
}
}  // namespace dsh::eng

/* Storage for the adjoint's forward wavefields.  Full storage (3 fields per
 * step and shot) when it fits the budget (mem_budget, or the free device
 * memory less a 2 GiB reserve when mem_budget is 0); otherwise checkpoints
 * every C steps, C = sqrt(NT*(3+2L)/3) (minimises checkpoints + C-step buffer),
 * with one recomputed forward pass.  ckpt_every > 0 asks for checkpoints every
 * ckpt_every steps whatever the budget. */
static int ensure_storage(dsh_ctx *ctx)
{
    const dsh_params &p = ctx->p;
    const size_t S = ctx->S, D = ctx->dstride, st = ctx->o_state_end;
    const size_t NS = p.grad_q ? 5 : 3;   /* stored fields per step: acc, uy, uyx (+ the two tau sensitivities) */
    const size_t full = S * (size_t)p.nt * NS * D * sizeof(float);
    int C = p.ckpt_every > 0 ? p.ckpt_every
                             : (int)std::lround(std::sqrt((double)p.nt * (3.0 + 2.0 * p.l) / 3.0));
    C = std::max(1, std::min(C, p.nt));
    const int nck = (p.nt + C - 1) / C - 1;
    const size_t ckpt_need = S * (size_t)C * NS * D * sizeof(float) + (size_t)nck * S * st * sizeof(float) +
                             S * (size_t)ctx->slot_stride * sizeof(float);
    if (ctx->fwd && ((ctx->ckpt_c == 0 && ctx->fwd_bytes >= full) || (ctx->ckpt_c == C && ctx->ckpt))) return DSH_OK;
    cudaFree(ctx->fwd); cudaFree(ctx->ckpt); cudaFree(ctx->shadow);
    ctx->fwd = ctx->ckpt = ctx->shadow = nullptr;
    ctx->fwd_bytes = ctx->ckpt_bytes = 0;
    drop_graphs(ctx);
    ctx->geo_version++;
    long long budget = p.mem_budget;
    if (budget <= 0) {
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        budget = (long long)fr - (2LL << 30);
    }
    ctx->fwd_step_stride = NS * D;
    if (p.ckpt_every <= 0 && (long long)full <= budget) {
        if (cudaMalloc(&ctx->fwd, full) != cudaSuccess) { cudaGetLastError(); return DSH_ERR_OOM; }
        ctx->fwd_bytes = full;
        ctx->fwd_mod = p.nt;
        ctx->ckpt_c = 0;
    } else {
        if ((long long)ckpt_need > budget) return DSH_ERR_OOM;
        const size_t seg = S * (size_t)C * NS * D * sizeof(float);
        if (cudaMalloc(&ctx->fwd, seg) != cudaSuccess) { cudaGetLastError(); return DSH_ERR_OOM; }
        if (nck > 0 && cudaMalloc(&ctx->ckpt, (size_t)nck * S * st * sizeof(float)) != cudaSuccess) {
            cudaGetLastError(); return DSH_ERR_OOM;
        }
        if (cudaMalloc(&ctx->shadow, S * (size_t)ctx->slot_stride * sizeof(float)) != cudaSuccess) {
            cudaGetLastError(); return DSH_ERR_OOM;
        }
        ctx->fwd_bytes = seg;
        ctx->ckpt_bytes = (size_t)nck * S * st * sizeof(float) + S * (size_t)ctx->slot_stride * sizeof(float);
        ctx->fwd_mod = C;
        ctx->ckpt_c = C;
    }
    ctx->fwd_slot_stride = (long long)ctx->fwd_mod * ctx->fwd_step_stride;
    build_tmaps(ctx);                     /* the shadow state may have changed */
    return DSH_OK;
}

static dim3 epi_grid(dsh_ctx *ctx, int nb)
{
    const long long n = (long long)ctx->p.nx * ctx->p.ny;
    return dim3((unsigned)std::min<long long>((n + 255) / 256, 4 * 148), (unsigned)nb, 1);
}

namespace dsh::eng {
int copy_seis_out(dsh_ctx *ctx, int nb, float *host_out, float *dev_out)
{
    long long tot = 0;
    for (int s = 0; s < nb; s++) tot += (long long)ctx->ntr_b[s] * ctx->p.nt;
    if (tot == 0) return DSH_OK;
    float *dst = dev_out ? dev_out : ctx->d_tmp;
    seis_transpose_kernel<<<dim3(256, nb), 256, 0, ctx->st>>>(ctx->p.nt, ctx->d_rec_off, ctx->d_seis, ctx->d_offs + ctx->S,
                                                             dst, ctx->d_offs + 3 * ctx->S);
    ctx->launches++;
    CK(cudaGetLastError());
    if (host_out) {
        WAIT(ctx);     /* a copy to pageable host memory would wait for the stream without a limit */
        CK(cudaMemcpyAsync(host_out, ctx->d_tmp, (size_t)tot * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    }
    return DSH_OK;
}
}  // namespace dsh::eng

namespace dsh::eng {
long long batch_seis_len(dsh_ctx *ctx, const dsh_shot *shots, int nb)
{
    long long t = 0;
    for (int s = 0; s < nb; s++) t += (long long)shots[s].ntr * ctx->p.nt;
    return t;
}
}  // namespace dsh::eng

static int forward_impl(dsh_ctx *ctx, const dsh_shot *shots, int nshots, float *seis_host, float *seis_dev)
{
    if (!ctx || !shots || nshots < 0) return DSH_ERR_PARAM;
    if (!ctx->model_set) return DSH_ERR_STATE;
    CK(cudaSetDevice(ctx->dev));
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    ctx->launches = 0;
    long long out = 0;
    for (int b0 = 0; b0 < nshots; b0 += ctx->S) {
        const int nb = std::min(ctx->S, nshots - b0);
        int rc = upload_batch(ctx, shots + b0, nb, nullptr, nullptr, 0);
        if (rc != DSH_OK) return rc;
        if ((rc = zero_slots(ctx, nb, false)) != DSH_OK) return rc;
        if ((rc = run_pass(ctx, P_FWD_PLAIN, nb)) != DSH_OK) return rc;
        if ((rc = copy_seis_out(ctx, nb, seis_host ? seis_host + out : nullptr, seis_dev ? seis_dev + out : nullptr)) != DSH_OK)
            return rc;
        out += batch_seis_len(ctx, shots + b0, nb);
        WAIT(ctx);
    }
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    WAIT_EV(ctx, ctx->ev[1]);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    ctx->stats.ms_forward = ms; ctx->stats.ms_adjoint = 0; ctx->stats.ms_total = ms;
    ctx->stats.kernel_launches = ctx->launches;
    ctx->stats.point_updates = (long long)ctx->p.nx * ctx->p.ny * ctx->p.nt * nshots;
    ctx->stats.storage_bytes = 0;
    ctx->stats.checkpoint_interval = 0;
    return check_status(ctx);
}

extern "C" int dsh_forward(dsh_ctx *ctx, const dsh_shot *shots, int nshots, float *seis_out)
{
    return forward_impl(ctx, shots, nshots, seis_out, nullptr);
}

extern "C" int dsh_forward_device(dsh_ctx *ctx, const dsh_shot *shots, int nshots, float *seis_dev)
{
    return forward_impl(ctx, shots, nshots, nullptr, seis_dev);
}

static int gradient_impl(dsh_ctx *ctx, const dsh_shot *shots, int nshots, const float *obs_host, const float *obs_dev,
                         float *g_vs_host, float *g_rho_host, float *g_vs_dev, float *g_rho_dev, double *l2,
                         float *seis_host, float *ws_host, float *wr_host)
{
    if (!ctx || !shots || nshots < 1 || (!obs_host && !obs_dev)) return DSH_ERR_PARAM;
    if (!ctx->model_set) return DSH_ERR_STATE;
    CK(cudaSetDevice(ctx->dev));
    int rc = ensure_storage(ctx);
    if (rc != DSH_OK) return rc;
    const dsh_params &p = ctx->p;
    const long long n = (long long)p.nx * p.ny;
    float *sum_u = ctx->sums, *sum_r = ctx->sums + ctx->dstride;
    float *esum_s = ctx->sums + 4 * ctx->dstride, *esum_r = ctx->sums + 5 * ctx->dstride;
    const bool energies = p.eprecond == 1 || p.eprecond == 3 || p.eprecond == DSH_EPRECOND_ENERGY_ONLY;
    CK(cudaMemsetAsync(ctx->sums, 0, 2 * (size_t)ctx->dstride * sizeof(float), ctx->st));
    CK(cudaMemsetAsync(esum_s, 0, 2 * (size_t)ctx->dstride * sizeof(float), ctx->st));
    if (p.grad_q) CK(cudaMemsetAsync(ctx->sums + 6 * ctx->dstride, 0, 2 * (size_t)ctx->dstride * sizeof(float), ctx->st));
    ctx->gq_valid = 0;
    ctx->launches = 0;
    ctx->shot_l2.clear();
    double l2_total = 0.0;
    float ms_f = 0, ms_a = 0;
    long long out = 0;
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    for (int b0 = 0; b0 < nshots; b0 += ctx->S) {
        const int nb = std::min(ctx->S, nshots - b0);
        const float *obs_h = obs_host ? obs_host + out : nullptr;
        if ((rc = upload_batch(ctx, shots + b0, nb, obs_h, obs_dev, out)) != DSH_OK) return rc;
        const float *obs_base = obs_dev ? obs_dev : ctx->d_obs;
        if ((rc = zero_slots(ctx, nb, true)) != DSH_OK) return rc;
        cudaEvent_t e0, e1, e2;
        cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2);
        cudaEventRecord(e0, ctx->st);
        if ((rc = forward_for_gradient(ctx, nb)) != DSH_OK) return rc;
        cudaEventRecord(e1, ctx->st);
        /* residual + misfit (LNORM of dsh_set_misfit) */
        if (ctx->lnorm == 2)
            residual_kernel<<<dim3(RED_BLOCKS, nb), RED_THREADS, 0, ctx->st>>>(p.nt, ctx->d_rec_off, ctx->d_seis,
                                                                              ctx->d_offs + ctx->S, obs_base,
                                                                              ctx->d_offs + 2 * ctx->S, ctx->d_res,
                                                                              ctx->d_part);
        else if (ctx->lnorm == 5)
            residual_gc_kernel<<<dim3(RED_BLOCKS, nb), RED_THREADS, 0, ctx->st>>>(
                p.nt, ctx->d_rec_off, ctx->d_seis, ctx->d_offs + ctx->S, obs_base, ctx->d_offs + 2 * ctx->S,
                ctx->d_res, ctx->d_part);
        else
            residual_elem_kernel<<<dim3(RED_BLOCKS, nb), RED_THREADS, 0, ctx->st>>>(
                ctx->lnorm, p.nt, ctx->d_rec_off, ctx->d_seis, ctx->d_offs + ctx->S, obs_base,
                ctx->d_offs + 2 * ctx->S, ctx->d_res, ctx->d_part);
        reduce_parts<<<nb, RED_THREADS, 0, ctx->st>>>(ctx->d_part, RED_BLOCKS, nb, ctx->d_l2);
        ctx->launches += 2;
        CK(cudaGetLastError());
        if (seis_host) {
            if ((rc = copy_seis_out(ctx, nb, seis_host + out, nullptr)) != DSH_OK) return rc;
        }
        if ((rc = zero_slots(ctx, nb, false)) != DSH_OK) return rc;
        if ((rc = adjoint_for_gradient(ctx, nb)) != DSH_OK) return rc;
        cudaEventRecord(e2, ctx->st);
        if (ws_host || wr_host) {
            WAIT(ctx);
            for (int s = 0; s < nb; s++) {
                if (ws_host) {
                    gather_dense_kernel<<<256, 256, 0, ctx->st>>>(p.nx, p.ny, ctx->pitch,
                                                                  ctx->slab + s * ctx->slot_stride + ctx->o_ws, ctx->d_out);
                    CK(cudaMemcpyAsync(ws_host + (size_t)(b0 + s) * n, ctx->d_out, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
                }
                if (wr_host) {
                    gather_dense_kernel<<<256, 256, 0, ctx->st>>>(p.nx, p.ny, ctx->pitch,
                                                                  ctx->slab + s * ctx->slot_stride + ctx->o_wr, ctx->d_out + n);
                    CK(cudaMemcpyAsync(wr_host + (size_t)(b0 + s) * n, ctx->d_out + n, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
                }
                WAIT(ctx);
            }
        }
        if (p.eprecond == 1 || p.eprecond == 3) {
            EpiArgs ea;
            ea.nx = p.nx; ea.ny = p.ny; ea.pitch = ctx->pitch; ea.slot_stride = ctx->slot_stride;
            ea.ws = ctx->slab + ctx->o_ws; ea.wr = ctx->slab + ctx->o_wr; ea.we = ctx->slab + ctx->o_we;
            ea.gu = ctx->slab + ctx->o_gu; ea.grho = ctx->slab + ctx->o_grho;
            ea.wemax = ctx->d_wemax; ea.cvs = ctx->cnorm[0]; ea.crho = ctx->cnorm[1]; ea.dh = p.dh;
            ea.eprecond = p.eprecond;
            CK(cudaMemsetAsync(ctx->d_wemax, 0, (size_t)nb * sizeof(unsigned), ctx->st));
            eprecond_we_kernel<<<epi_grid(ctx, nb), 256, 0, ctx->st>>>(ea);
            eprecond_scale_kernel<<<epi_grid(ctx, nb), 256, 0, ctx->st>>>(ea);
            ctx->launches += 2;
        }
        if (ctx->taper_on) {
            std::vector<TaperShot> ts(nb);
            for (int s = 0; s < nb; s++) {
                const dsh_shot &sh = shots[b0 + s];
                ts[s].i1 = (int)sh.srcpos[0];
                ts[s].j1 = (int)sh.srcpos[sh.nsrc];
                dsh_setup_taper_norm(p.nx, p.ny, ctx->taper_g, ctx->taper_ijc, ctx->taper_box.data(), ts[s].i1,
                                     ts[s].j1, &ts[s].minm, &ts[s].maxm);
            }
            CK(cudaMemcpyAsync(ctx->d_taper_shot, ts.data(), nb * sizeof(TaperShot), cudaMemcpyHostToDevice, ctx->st));
            shot_sum_taper_kernel<<<epi_grid(ctx, 1), 256, 0, ctx->st>>>(
                p.nx, p.ny, ctx->pitch, ctx->slot_stride, nb, ctx->slab + ctx->o_gu, ctx->slab + ctx->o_grho, sum_u,
                sum_r, ctx->d_taper_box, ctx->taper_g, ctx->taper_ijc, ctx->taper_filt,
                (const TaperShot *)ctx->d_taper_shot);
        } else {
            shot_sum_kernel<<<epi_grid(ctx, 1), 256, 0, ctx->st>>>(p.nx, p.ny, ctx->pitch, ctx->slot_stride, nb,
                                                                   ctx->slab + ctx->o_gu, ctx->slab + ctx->o_grho,
                                                                   sum_u, sum_r);
        }
        ctx->launches++;
        if (p.grad_q) {            /* shot sums of the Qs-gradient correlations */
            shot_sum_kernel<<<epi_grid(ctx, 1), 256, 0, ctx->st>>>(p.nx, p.ny, ctx->pitch, ctx->slot_stride, nb,
                                                                   ctx->slab + ctx->o_gqx, ctx->slab + ctx->o_gqy,
                                                                   ctx->sums + 6 * ctx->dstride,
                                                                   ctx->sums + 7 * ctx->dstride);
            ctx->launches++;
        }
        if (energies) {            /* shot sums of Ws and Wr (dsh_get_energy_sums) */
            shot_sum_kernel<<<epi_grid(ctx, 1), 256, 0, ctx->st>>>(p.nx, p.ny, ctx->pitch, ctx->slot_stride, nb,
                                                                   ctx->slab + ctx->o_ws, ctx->slab + ctx->o_wr,
                                                                   esum_s, esum_r);
            ctx->launches++;
        }
        CK(cudaGetLastError());
        std::vector<double> l2b(nb);
        WAIT(ctx);
        CK(cudaMemcpyAsync(l2b.data(), ctx->d_l2, nb * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
        WAIT(ctx);
        for (int s = 0; s < nb; s++) { l2_total += l2b[s]; ctx->shot_l2.push_back(l2b[s]); }
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, e0, e1);
        cudaEventElapsedTime(&b, e1, e2);
        ms_f += a; ms_a += b;
        cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
        out += batch_seis_len(ctx, shots + b0, nb);
    }
    float *gv = g_vs_dev ? g_vs_dev : ctx->d_out;
    float *gr = g_rho_dev ? g_rho_dev : ctx->d_out + n;
    convert_kernel<<<epi_grid(ctx, 1), 256, 0, ctx->st>>>(p.nx, p.ny, ctx->pitch, p.dt, ctx->m_vs, ctx->m_rho, sum_u,
                                                          sum_r, gv, gr);
    ctx->launches++;
    if (p.grad_q) {
        q_convert_kernel<<<epi_grid(ctx, 1), 256, 0, ctx->st>>>(p.nx, p.ny, ctx->pitch, ctx->m_rho, ctx->m_qs,
                                                                ctx->sums + 6 * ctx->dstride,
                                                                ctx->sums + 7 * ctx->dstride, ctx->d_gq);
        ctx->launches++;
    }
    CK(cudaGetLastError());
    if (g_vs_host || g_rho_host) WAIT(ctx);
    if (g_vs_host) CK(cudaMemcpyAsync(g_vs_host, gv, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    if (g_rho_host) CK(cudaMemcpyAsync(g_rho_host, gr, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    WAIT_EV(ctx, ctx->ev[1]);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    ctx->stats.ms_forward = ms_f; ctx->stats.ms_adjoint = ms_a; ctx->stats.ms_total = ms;
    ctx->stats.kernel_launches = ctx->launches;
    ctx->stats.point_updates = 2LL * p.nx * p.ny * p.nt * nshots;
    ctx->stats.storage_bytes = (long long)(ctx->fwd_bytes + ctx->ckpt_bytes);
    ctx->stats.checkpoint_interval = ctx->ckpt_c;
    if (l2) *l2 = l2_total;
    const int st = check_status(ctx);
    ctx->gq_valid = p.grad_q && st == DSH_OK;
    return st;
}

extern "C" int dsh_get_gradient_q(dsh_ctx *ctx, float *g_qs_host, float *g_qs_dev)
{
    if (!ctx || (!g_qs_host && !g_qs_dev)) return DSH_ERR_PARAM;
    if (!ctx->p.grad_q || !ctx->gq_valid) return DSH_ERR_STATE;
    CK(cudaSetDevice(ctx->dev));
    const size_t bytes = (size_t)ctx->p.nx * ctx->p.ny * sizeof(float);
    if (g_qs_dev) CK(cudaMemcpyAsync(g_qs_dev, ctx->d_gq, bytes, cudaMemcpyDeviceToDevice, ctx->st));
    if (g_qs_host) {
        WAIT(ctx);
        CK(cudaMemcpyAsync(g_qs_host, ctx->d_gq, bytes, cudaMemcpyDeviceToHost, ctx->st));
    }
    WAIT(ctx);
    return DSH_OK;
}

extern "C" int dsh_gradient(dsh_ctx *ctx, const dsh_shot *shots, int nshots, const float *obs, float *g_vs,
                            float *g_rho, double *l2, float *seis_out, float *ws, float *wr)
{
    if (!obs) return DSH_ERR_PARAM;
    return gradient_impl(ctx, shots, nshots, obs, nullptr, g_vs, g_rho, nullptr, nullptr, l2, seis_out, ws, wr);
}

extern "C" int dsh_gradient_device(dsh_ctx *ctx, const dsh_shot *shots, int nshots, const float *obs_dev,
                                   float *g_vs_dev, float *g_rho_dev, double *l2)
{
    if (!obs_dev) return DSH_ERR_PARAM;
    return gradient_impl(ctx, shots, nshots, nullptr, obs_dev, nullptr, nullptr, g_vs_dev, g_rho_dev, l2, nullptr,
                         nullptr, nullptr);
}

extern "C" int dsh_set_wait_limits(dsh_ctx *ctx, long long device_polls, double host_seconds)
{
    if (!ctx) return DSH_ERR_PARAM;
    const long long polls = device_polls > 0 ? device_polls : DEVICE_POLLS_DEFAULT;
    if (polls != ctx->device_polls) drop_graphs(ctx);      /* the limit is baked into captured launches */
    ctx->device_polls = polls;
    ctx->host_timeout_s = host_seconds > 0 ? host_seconds : HOST_TIMEOUT_DEFAULT_S;
    return DSH_OK;
}

/* step-kernel variants: staged velocity taps, fused step, persistent launch, cluster-resident launch,
 * temporally blocked launches */
static const int VARIANT_SEL[DSH_STEP_VARIANTS][5] = {
    {0, 0, 0, 0, 0}, {1, 0, 0, 0, 0}, {0, 1, 0, 0, 0}, {0, 0, 1, 0, 0}, {0, 0, 0, 1, 0}, {0, 0, 0, 0, 1}};

static void select_variant(dsh_ctx *ctx, int v)
{
    ctx->sel_staged = v < 0 ? -1 : VARIANT_SEL[v][0];
    ctx->sel_fused = v < 0 ? -1 : VARIANT_SEL[v][1];
    ctx->sel_persist = v < 0 ? -1 : VARIANT_SEL[v][2];
    ctx->sel_cluster = v < 0 ? -1 : VARIANT_SEL[v][3];
    ctx->sel_tblock = v < 0 ? -1 : VARIANT_SEL[v][4];
}

extern "C" int dsh_set_step_variant(dsh_ctx *ctx, int variant)
{
    if (!ctx || variant < -1 || variant >= DSH_STEP_VARIANTS) return DSH_ERR_PARAM;
    if (variant == 2 && !ctx->fused_ok) return DSH_ERR_PARAM;
    select_variant(ctx, variant);
    drop_graphs(ctx);
    return DSH_OK;
}

extern "C" int dsh_set_misfit(dsh_ctx *ctx, int lnorm)
{
    if (!ctx || lnorm < 1 || lnorm > 5) return DSH_ERR_PARAM;
    ctx->lnorm = lnorm;
    return DSH_OK;
}

extern "C" int dsh_set_shot_taper(dsh_ctx *ctx, int enable, int srtshape, float srtradius, int filtsize)
{
    if (!ctx) return DSH_ERR_PARAM;
    if (!enable) {
        ctx->taper_on = 0;
        return DSH_OK;
    }
    int g = 0, ijc = 0;
    if (filtsize < 0 || dsh_setup_taper_box(srtshape, srtradius, ctx->p.dh, &g, &ijc, nullptr) != 0)
        return DSH_ERR_PARAM;
    if (g > 4096) return DSH_ERR_PARAM;
    std::vector<float> box((size_t)g * g);
    dsh_setup_taper_box(srtshape, srtradius, ctx->p.dh, &g, &ijc, box.data());
    CK(cudaSetDevice(ctx->dev));
    WAIT(ctx);
    ctx->taper_on = 0;
    cudaFree(ctx->d_taper_box);
    ctx->d_taper_box = nullptr;
    if (cudaMalloc(&ctx->d_taper_box, box.size() * sizeof(float)) != cudaSuccess) return DSH_ERR_OOM;
    if (!ctx->d_taper_shot && cudaMalloc(&ctx->d_taper_shot, (size_t)ctx->S * sizeof(TaperShot)) != cudaSuccess)
        return DSH_ERR_OOM;
    CK(cudaMemcpy(ctx->d_taper_box, box.data(), box.size() * sizeof(float), cudaMemcpyHostToDevice));
    ctx->taper_box.swap(box);
    ctx->taper_g = g;
    ctx->taper_ijc = ijc;
    ctx->taper_filt = filtsize;
    ctx->taper_on = 1;
    return DSH_OK;
}

extern "C" int dsh_hessian_diag(dsh_ctx *ctx, const dsh_shot *shots, int nshots, float *h_vs, float *h_rho)
{
    if (!ctx || !shots || nshots < 1) return DSH_ERR_PARAM;
    if (!ctx->model_set) return DSH_ERR_STATE;
    CK(cudaSetDevice(ctx->dev));
    const dsh_params &p = ctx->p;
    const long long n = (long long)p.nx * p.ny;
    float *sum_u = ctx->sums, *sum_r = ctx->sums + ctx->dstride;
    CK(cudaMemsetAsync(ctx->sums, 0, 2 * (size_t)ctx->dstride * sizeof(float), ctx->st));
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    ctx->launches = 0;
    int rc;
    for (int b0 = 0; b0 < nshots; b0 += ctx->S) {
        const int nb = std::min(ctx->S, nshots - b0);
        if ((rc = upload_batch(ctx, shots + b0, nb, nullptr, nullptr, 0)) != DSH_OK) return rc;
        if ((rc = zero_slots(ctx, nb, true)) != DSH_OK) return rc;
        if ((rc = run_pass(ctx, P_FWD_HESS, nb)) != DSH_OK) return rc;
        shot_sum_kernel<<<epi_grid(ctx, 1), 256, 0, ctx->st>>>(p.nx, p.ny, ctx->pitch, ctx->slot_stride, nb,
                                                               ctx->slab + ctx->o_hu, ctx->slab + ctx->o_hrho, sum_u, sum_r);
        ctx->launches++;
        WAIT(ctx);
    }
    hessian_convert_kernel<<<epi_grid(ctx, 1), 256, 0, ctx->st>>>(p.nx, p.ny, ctx->pitch, ctx->m_vs, ctx->m_rho, sum_u,
                                                                  sum_r, ctx->d_out, ctx->d_out + n);
    ctx->launches++;
    CK(cudaGetLastError());
    if (h_vs || h_rho) WAIT(ctx);
    if (h_vs) CK(cudaMemcpyAsync(h_vs, ctx->d_out, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    if (h_rho) CK(cudaMemcpyAsync(h_rho, ctx->d_out + n, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    WAIT_EV(ctx, ctx->ev[1]);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    ctx->stats.ms_forward = ms; ctx->stats.ms_adjoint = 0; ctx->stats.ms_total = ms;
    ctx->stats.kernel_launches = ctx->launches;
    ctx->stats.point_updates = (long long)p.nx * p.ny * p.nt * nshots;
    return check_status(ctx);
}

extern "C" int dsh_get_field(dsh_ctx *ctx, int shot, int which, float *out)
{
    if (!ctx || !out || shot < 0 || shot >= ctx->S) return DSH_ERR_PARAM;
    CK(cudaSetDevice(ctx->dev));
    const dsh_params &p = ctx->p;
    const long long n = (long long)p.nx * p.ny;
    const float *base = ctx->slab + (long long)shot * ctx->slot_stride;
    const float *src;
    int pitch = ctx->pitch;
    switch (which) {
    case 0: src = base + (ctx->state_b ? ctx->o_vy_b : ctx->o_vy) + (long long)ctx->hy * pitch; break;
    case 1: src = base + (ctx->state_b ? ctx->o_sxy_b : ctx->o_sxy) + (long long)ctx->hy * pitch; break;
    case 2: src = base + (ctx->state_b ? ctx->o_syz_b : ctx->o_syz) + (long long)ctx->hy * pitch; break;
    case 12: src = base + ctx->o_ws; break;
    case 13: src = base + ctx->o_wr; break;
    case 14: src = base + ctx->o_we; break;
    case 15: src = base + ctx->o_gu; break;
    case 16: src = base + ctx->o_grho; break;
    case 17: src = base + ctx->o_hu; break;
    case 18: src = base + ctx->o_hrho; break;
    case 300: src = ctx->m_brho; break;
    case 301: src = ctx->m_uip; break;
    case 302: src = ctx->m_ujp; break;
    case 303: case 304: case 305: case 306:
        if (p.l < 1) return DSH_ERR_PARAM;
        src = which == 303 ? ctx->m_muip : which == 304 ? ctx->m_mujp : which == 305 ? ctx->m_tip : ctx->m_taus;
        break;
    default: {
        const int l = which % 100;
        if (l >= p.l) return DSH_ERR_PARAM;
        if (which >= 100 && which < 200) src = base + ctx->o_r + (long long)l * ctx->dstride;
        else if (which >= 200 && which < 300) src = base + ctx->o_q + (long long)l * ctx->dstride;
        else return DSH_ERR_PARAM;
    }
    }
    WAIT(ctx);
    CK(cudaMemcpy2DAsync(out, (size_t)p.nx * sizeof(float), src + HX, (size_t)pitch * sizeof(float),
                         (size_t)p.nx * sizeof(float), p.ny, cudaMemcpyDeviceToHost, ctx->st));
    WAIT(ctx);
    (void)n;
    return DSH_OK;
}

/* Times plain forward steps of each step-kernel variant the context can run
 * on these shots — kernel pair (v_step), pair with v_step_st, fused step,
 * persistent launch, cluster-resident launch, temporally blocked launches —
 * and keeps the fastest for the context's later calls (the fused choice also
 * serves the gradient passes, the last three only plain forward modelling).
 * ms_per_step[DSH_STEP_VARIANTS] (optional): mean device ms per step of each
 * variant, 0 where it does not apply. */
extern "C" int dsh_autotune(dsh_ctx *ctx, const dsh_shot *shots, int nshots, int nsteps, float *ms_per_step,
                            int *choice)
{
    if (!ctx || !shots || nshots < 1 || nsteps < 1) return DSH_ERR_PARAM;
    if (!ctx->model_set) return DSH_ERR_STATE;
    CK(cudaSetDevice(ctx->dev));
    const int nb = std::min(ctx->S, nshots);
    int rc = upload_batch(ctx, shots, nb, nullptr, nullptr, 0);
    if (rc != DSH_OK) return rc;
    nsteps = std::min(nsteps, ctx->p.nt);
    float ms[DSH_STEP_VARIANTS] = {0};
    int best = 0;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (int v = 0; v < DSH_STEP_VARIANTS; v++) {
        select_variant(ctx, v);
        drop_graphs(ctx);                              /* graphs hold the previous variant's kernels */
        ClCfg ccfg;
        if (v == 2 && !use_fused(ctx, P_FWD_PLAIN)) continue;
        if (v == 3 && !persistent_grid(ctx, P_FWD_PLAIN, nb)) continue;
        if (v == 4 && !cluster_cfg(ctx, P_FWD_PLAIN, nb, &ccfg)) continue;
        TbCfg tcfg;
        if (v == 5 && !tblock_cfg(ctx, P_FWD_PLAIN, nb, &tcfg)) continue;
        for (int rep = 0; rep < 2; rep++) {            /* first round warms up (graphs, lazy loading) */
            if ((rc = zero_slots(ctx, nb, false)) != DSH_OK) break;
            CK(cudaEventRecord(e0, ctx->st));
            if ((rc = run_steps(ctx, P_FWD_PLAIN, nb, 1, nsteps)) != DSH_OK) break;
            CK(cudaEventRecord(e1, ctx->st));
        }
        if (rc != DSH_OK) break;
        WAIT_EV(ctx, e1);
        cudaEventElapsedTime(&ms[v], e0, e1);
        ms[v] /= nsteps;
        if (ms[v] < ms[best]) best = v;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    select_variant(ctx, best);
    drop_graphs(ctx);
    if (ms_per_step) for (int v = 0; v < DSH_STEP_VARIANTS; v++) ms_per_step[v] = ms[v];
    if (choice) *choice = best;
    if (rc != DSH_OK) return rc;
    return check_status(ctx);
}

extern "C" int dsh_profile_fused(dsh_ctx *ctx, int pass, int nsteps, float *out_ms)
{
    if (!ctx || !out_ms || pass < 0 || pass > 3 || pass == P_FWD_HESS || nsteps < 1 || nsteps > ctx->p.nt)
        return DSH_ERR_PARAM;
    if (ctx->ckpt_c && (pass == P_FWD_STORE || pass == P_ADJ) && nsteps > ctx->ckpt_c) nsteps = ctx->ckpt_c;
    if (!ctx->model_set || ctx->ntr_b.empty() || ((pass == P_FWD_STORE || pass == P_ADJ) && !ctx->fwd)) return DSH_ERR_STATE;
    if (!use_fused(ctx, (Pass)pass)) return DSH_ERR_STATE;
    CK(cudaSetDevice(ctx->dev));
    const dsh_params &p = ctx->p;
    const int nb = (int)ctx->ntr_b.size();
    KFn fk = fs_kernel(p.fdorder, p.l, fused_mode((Pass)pass), dh_pow2(p.dh));
    if (!fk) return DSH_ERR_PARAM;
    StepArgs sa = step_args(ctx, (Pass)pass);
    dim3 grid((unsigned)((p.nx + FTX - 1) / FTX), (unsigned)((p.ny + FTY - 1) / FTY), (unsigned)nb);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    set_int_kernel<<<1, 1, 0, ctx->st>>>(ctx->d_nt, 1);
    {   /* one untimed launch first (lazy module loading) */
        int off = 0;
        void *args[2] = {&sa, &off};
        CK(cudaLaunchKernel((const void *)fk, grid, dim3(256), args, 0, ctx->st));
    }
    CK(cudaEventRecord(e0, ctx->st));
    for (int k = 0; k < nsteps; k++) {
        int off = k;
        void *args[2] = {&sa, &off};
        CK(cudaLaunchKernel((const void *)fk, grid, dim3(256), args, 0, ctx->st));
    }
    CK(cudaEventRecord(e1, ctx->st));
    WAIT(ctx);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *out_ms = ms / nsteps;
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->st);
    return check_status(ctx);
}

extern "C" int dsh_get_shot_misfits(dsh_ctx *ctx, int nshots, double *out)
{
    if (!ctx || !out || nshots < 0) return DSH_ERR_PARAM;
    if (nshots > (int)ctx->shot_l2.size()) return DSH_ERR_STATE;
    for (int s = 0; s < nshots; s++) out[s] = ctx->shot_l2[s];
    return DSH_OK;
}

extern "C" int dsh_get_energy_sums(dsh_ctx *ctx, float *ws_sum, float *wr_sum)
{
    if (!ctx || (!ws_sum && !wr_sum)) return DSH_ERR_PARAM;
    const dsh_params &p = ctx->p;
    if (p.eprecond != 1 && p.eprecond != 3 && p.eprecond != DSH_EPRECOND_ENERGY_ONLY) return DSH_ERR_STATE;
    CK(cudaSetDevice(ctx->dev));
    const long long n = (long long)p.nx * p.ny;
    float *src[2] = {ctx->sums + 4 * ctx->dstride, ctx->sums + 5 * ctx->dstride};
    float *dst[2] = {ws_sum, wr_sum};
    for (int k = 0; k < 2; k++) {
        if (!dst[k]) continue;
        gather_dense_kernel<<<256, 256, 0, ctx->st>>>(p.nx, p.ny, ctx->pitch, src[k], ctx->d_out);
        CK(cudaGetLastError());
        WAIT(ctx);
        CK(cudaMemcpyAsync(dst[k], ctx->d_out, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
        WAIT(ctx);
    }
    return DSH_OK;
}

extern "C" int dsh_get_stats(dsh_ctx *ctx, dsh_stats *out)
{
    if (!ctx || !out) return DSH_ERR_PARAM;
    *out = ctx->stats;
    return DSH_OK;
}

extern "C" int dsh_set_stream(dsh_ctx *ctx, void *stream)
{
    if (!ctx) return DSH_ERR_PARAM;
    CK(cudaSetDevice(ctx->dev));
    WAIT(ctx);
    ctx->st = stream ? (cudaStream_t)stream : ctx->own_st;
    return DSH_OK;
}

extern "C" int dsh_profile_step(dsh_ctx *ctx, int pass, int nsteps, float *out_ms3)
{
    if (!ctx || !out_ms3 || pass < 0 || pass > 3 || nsteps < 1 || nsteps > ctx->p.nt) return DSH_ERR_PARAM;
    if (ctx->ckpt_c && (pass == P_FWD_STORE || pass == P_ADJ) && nsteps > ctx->ckpt_c) nsteps = ctx->ckpt_c;
    if (!ctx->model_set || ctx->ntr_b.empty() || ((pass == P_FWD_STORE || pass == P_ADJ) && !ctx->fwd)) return DSH_ERR_STATE;
    CK(cudaSetDevice(ctx->dev));
    const dsh_params &p = ctx->p;
    const int nb = (int)ctx->ntr_b.size();
    int vflags = 0, sflags = 0;
    if (pass == P_FWD_STORE) sflags = SF_STRAIN_OUT;
    if (pass == P_FWD_HESS) { vflags = VF_HESS; sflags = SF_HESS; }
    if (pass == P_ADJ) { vflags = VF_ADJOINT | VF_CORR; sflags = SF_CORR; }
    const VPick vp = pick_v(ctx, p.fdorder, vflags, dh_pow2(p.dh));
    KFn vk = vp.k, sk = s_kernel(p.fdorder, p.l, sflags);
    if (!vk || !sk) return DSH_ERR_PARAM;
    StepArgs sa = step_args(ctx, (Pass)pass);
    InjectArgs ia = inject_args(ctx, (Pass)pass);
    const int sr = s_rows();
    dim3 block(BX, sr, 1);
    dim3 grid((unsigned)((p.nx + 4 * BX - 1) / (4 * BX)), (unsigned)((p.ny + sr - 1) / sr), (unsigned)nb);
    dim3 vgrid, vblock;
    v_shape(ctx, vp, nb, &vgrid, &vblock);
    /* each kernel launched nsteps times back to back between one event pair */
    cudaEvent_t ev[6];
    for (auto &e : ev) CK(cudaEventCreate(&e));
    set_int_kernel<<<1, 1, 0, ctx->st>>>(ctx->d_nt, 1);
    {   /* one untimed launch of each kernel first (lazy module loading) */
        int off = 0;
        void *args[2] = {&sa, &off};
        void *iargs[2] = {&ia, &off};
        CK(cudaLaunchKernel((const void *)vk, vgrid, vblock, args, 0, ctx->st));
        if (!sa.tl.on) CK(cudaLaunchKernel((const void *)inject_sample, dim3(nb), dim3(128), iargs, 0, ctx->st));
        CK(cudaLaunchKernel((const void *)sk, grid, block, args, 0, ctx->st));
    }
    for (int q = 0; q < 3; q++) {
        CK(cudaEventRecord(ev[2 * q], ctx->st));
        for (int k = 0; k < nsteps; k++) {
            int off = k;
            void *args[2] = {&sa, &off};
            void *iargs[2] = {&ia, &off};
            if (q == 0) CK(cudaLaunchKernel((const void *)vk, vgrid, vblock, args, 0, ctx->st));
            if (q == 1 && !sa.tl.on) CK(cudaLaunchKernel((const void *)inject_sample, dim3(nb), dim3(128), iargs, 0, ctx->st));
            if (q == 2) CK(cudaLaunchKernel((const void *)sk, grid, block, args, 0, ctx->st));
        }
        CK(cudaEventRecord(ev[2 * q + 1], ctx->st));
    }
    WAIT(ctx);
    double acc[3] = {0, 0, 0};
    for (int q = 0; q < 3; q++) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev[2 * q], ev[2 * q + 1]);
        acc[q] = ms;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    for (int q = 0; q < 3; q++) out_ms3[q] = (float)(acc[q] / nsteps);
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->st);   /* repeated steps of one kernel may overflow */
    return check_status(ctx);
}

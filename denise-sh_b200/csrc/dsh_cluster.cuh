/*
 * dsh_cluster.cuh — small elastic grids: a whole forward-modelling pass in one
 * launch, with the wavefield, the model and the CPML memory held in the
 * shared memory of one thread-block cluster per shot.
 *
 * The kernel pair pays two launches per time step (~12 us per step on the
 * 500 x 200 elastic case, whose state is 1.2 MB), and a grid-wide persistent
 * kernel pays for global-memory flags, fences and L2 round trips between its
 * blocks.  Here the C CTAs of a cluster (C = 16 where the device allows it,
 * one CTA per SM) split the grid into row strips; CTA k keeps its rows
 * j0[k] .. j0[k+1]-1 of vy, sxy, syz, of the model factors 1/rho, uip, ujp
 * and of the CPML memory in its shared memory for the whole pass, plus
 * H = FDORDER/2 halo rows of vy and syz above and below.  One time step is
 *     velocity update of the own rows -> injection (one warp) -> cluster
 *     barrier -> sampling; copy the neighbours' H boundary rows of vy into
 *     the halo (distributed shared memory) -> stress update of the own rows ->
 *     cluster barrier -> copy the neighbours' boundary rows of syz
 * (sxy is only differentiated along x, inside a row, so it needs no halo).
 * The barriers are the hardware cluster barrier (arrive with release, wait
 * with acquire semantics), not polls on memory: every CTA of a cluster is
 * resident by construction and every thread of every CTA takes the same
 * barriers in the same order.  A CTA copies its neighbour's rows after the
 * barrier that ends the phase writing them and before it arrives at the next
 * one, and the neighbour overwrites those rows only after that next barrier,
 * so no copy races with an update.
 *
 * Inside the time loop a CTA touches global memory only to write receiver
 * samples and to prefetch the next step's source signals: the CPML
 * coefficient vectors, the CTA's source groups and receivers are copied into
 * shared memory before the loop.  (A barrier with acquire semantics at
 * cluster scope leaves nothing in L1 that another SM may have written, so
 * every global read after it would pay an L2 round trip on the step's
 * critical path.)  CTAs whose rows lie in a CPML depth strip also hold that
 * strip's memory rows and therefore take fewer rows (cl_partition).
 *
 * Per point the arithmetic is that of v_body / s_body (dsh_kernels.cuh) for
 * plain elastic forward modelling — the same expressions in the same order,
 * compiled with -fmad=false — so results are bit-identical to the kernel
 * pair.  At the end of the pass the own rows of vy, sxy, syz and the CPML
 * memory go back to the slot's global state.
 */
#pragma once
#include <cooperative_groups.h>

#include "dsh_kernels.cuh"

namespace dsh {

/* threads per CTA at most (80 registers each: at 1024 threads the 64-register
 * limit spills the stencil taps) */
__host__ __device__ constexpr int cl_max_threads(int) { return 768; }
constexpr int CL_MAX_ITEMS = 4;   /* 4-point items per thread and phase */
constexpr int CL_MAX_C = 16;      /* CTAs per cluster at most */
constexpr int CL_MAX_GRP = 32;    /* source points (groups) of a slot */
constexpr int CL_MAX_MEM = 4;     /* sources at one point */
constexpr int CL_MAX_REC = 512;   /* receivers of a slot */

/* row strips of the CTAs: CTA k owns grid rows j0[k] .. j0[k+1]-1 (none when
 * equal); j0[0] = 1, j0[C] = ny + 1; every CTA but the last one with rows
 * owns at least H rows */
struct ClGeom {
    int C;
    int j0[CL_MAX_C + 1];
};

/* rows of the CPML depth strips among rows [ja, jb): top strip (j <= fw,
 * only without a free surface) and bottom strip (j >= ny - fw + 1) */
__host__ __device__ inline int cl_top_rows(int ja, int jb, int fw, int free_surf)
{
    if (free_surf || fw <= 0) return 0;
    const int e = jb < fw + 1 ? jb : fw + 1;
    return e > ja ? e - ja : 0;
}
__host__ __device__ inline int cl_bot_rows(int ja, int jb, int ny, int fw)
{
    if (fw <= 0) return 0;
    const int b = ja > ny - fw + 1 ? ja : ny - fw + 1;
    return jb > b ? jb - b : 0;
}

/* Shared-memory layout of one CTA with r own rows and y CPML depth-strip
 * rows: float4 fields (p4 float4s per row), then float arrays, then int
 * lists.  Offsets in units of the element type, all from the same base. */
struct ClLayout {
    long long vy, syz, sxy, br, ui, uj, pyv, pys;   /* float4 index */
    long long pxv, pxs, coef;                         /* float index */
    long long grp, rec, cnt;                          /* int index */
    long long bytes;
};
__host__ __device__ inline ClLayout cl_layout(int r, int y, int H, int p4, int fw)
{
    ClLayout L;
    long long o = 0;
    L.vy = o; o += (long long)(r + 2 * H) * p4;
    L.syz = o; o += (long long)(r + 2 * H) * p4;
    L.sxy = o; o += (long long)r * p4;
    L.br = o; o += (long long)r * p4;
    L.ui = o; o += (long long)r * p4;
    L.uj = o; o += (long long)r * p4;
    L.pyv = o; o += (long long)y * p4;
    L.pys = o; o += (long long)y * p4;
    long long f = 4 * o;
    L.pxv = f; f += (long long)r * 2 * fw;
    L.pxs = f; f += (long long)r * 2 * fw;
    L.coef = f; f += 12LL * (2 * fw + 1);
    long long n = f;               /* ints share the 4-byte index */
    L.grp = n; n += (long long)CL_MAX_GRP * (2 + CL_MAX_MEM);
    L.rec = n; n += 2LL * CL_MAX_REC;
    L.cnt = n; n += 4;
    L.bytes = 4 * n;
    return L;
}

/* store the lanes of v inside the grid (the others stay 0) */
__device__ __forceinline__ void sts4m(float4 *p, float4 v, int nvalid)
{
    if (nvalid >= 4) { *p = v; return; }
    float *q = reinterpret_cast<float *>(p);
    if (nvalid > 0) q[0] = v.x;
    if (nvalid > 1) q[1] = v.y;
    if (nvalid > 2) q[2] = v.z;
}

extern __shared__ float4 cl_smem[];

/* The CTA's view of its shared memory (32-bit offsets from cl_smem, so the
 * addresses stay shared-window offsets in registers) and the CPML geometry. */
struct ClView {
    int vy, syz, sxy, br, ui, uj;  /* float4 index */
    int pyv, pys, pxv, pxs, coef;  /* float index; coef: 12 vectors of 2fw+1: K_x a_x b_x K_x_half a_x_half
                                      b_x_half, then the same six for y */
    int p4, pitch, fw2;            /* fw2 = 2fw + 1 */
    int j0, yt, ybeg;              /* first own row; top-strip rows; first bottom-strip row */
};
__device__ __forceinline__ float4 *cl_f4(int off) { return cl_smem + off; }
__device__ __forceinline__ float *cl_f(int off) { return reinterpret_cast<float *>(cl_smem) + off; }

/* psi row of own grid row j in the depth strips (top rows first, then bottom) */
__device__ __forceinline__ int cl_top_idx(const ClView &v, int j) { return j - v.j0; }
__device__ __forceinline__ int cl_bot_idx(const ClView &v, int j) { return v.yt + (j - v.ybeg); }

/* Velocity update of the four points i0..i0+3 of own local row lr (v_body,
 * FLAGS = 0, no injection or sampling: those follow for the whole CTA). */
template <int FDO, bool P2>
__device__ __forceinline__ void cl_v_points(const StepArgs &a, const ClView &v, int lr, int g)
{
    constexpr int H = FDO / 2;
    constexpr int NL = (H + 3) / 4;
    constexpr int NR = (H - 1 + 3) / 4;
    constexpr int NXS = 4 * (NL + 1 + NR);
    const int i0 = 1 + 4 * g, j = v.j0 + lr;
    const int c4 = g + HX / 4;
    const int p4 = v.p4;
    const float4 *sxr = cl_f4(v.sxy + lr * p4 + c4);
    const float4 *syc = cl_f4(v.syz + lr * p4 + c4);              /* syz row j-H */
    float4 *vyp = cl_f4(v.vy + (lr + H) * p4 + c4);
    float xs[NXS];
#pragma unroll
    for (int q = 0; q < NL + 1 + NR; q++) {
        const float4 t = sxr[q - NL];
        xs[4 * q] = t.x; xs[4 * q + 1] = t.y; xs[4 * q + 2] = t.z; xs[4 * q + 3] = t.w;
    }
    float4 ys[2 * H];
#pragma unroll
    for (int r = 0; r < 2 * H; r++) ys[r] = syc[r * p4];
    float4 vy4 = *vyp;
    const float4 b4 = *cl_f4(v.br + lr * p4 + c4);

    const int col0 = i0 - 1 + HX;
    const int nvalid = min(4, a.nx - i0 + 1);
    const bool in_pml = a.fw > 0 && (i0 <= a.fw || i0 + 3 >= a.nx - a.fw + 1 || (!a.free_surf && j <= a.fw) ||
                                     j >= a.ny - a.fw + 1);
    const float *K_x = cl_f(v.coef), *a_x = cl_f(v.coef + v.fw2), *b_x = cl_f(v.coef + 2 * v.fw2);
    const float *K_y = cl_f(v.coef + 6 * v.fw2), *a_y = cl_f(v.coef + 7 * v.fw2), *b_y = cl_f(v.coef + 8 * v.fw2);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int i = i0 + k;
        float sxy_x, syy_y;
#pragma unroll
        for (int m = 1; m <= H; m++) {
            float tx = a.hc[m] * (xs[4 * NL + k + m - 1] - xs[4 * NL + k - m]);
            float ty = a.hc[m] * (get(ys[H + m - 1], k) - get(ys[H - m], k));
            if (m == 1) { sxy_x = tx; syy_y = ty; }
            else { sxy_x = sxy_x + tx; syy_y = syy_y + ty; }
        }
        const int fw = a.fw;
        if (in_pml && i <= a.nx) {
            if (i <= fw) {
                float *p = cl_f(v.pxv + lr * 2 * fw + (i - 1));
                float ps = b_x[i] * *p + a_x[i] * sxy_x;
                *p = ps;
                sxy_x = sxy_x / K_x[i] + ps;
            }
            if (i >= a.nx - fw + 1) {
                const int h1 = i - a.nx + 2 * fw;
                float *p = cl_f(v.pxv + lr * 2 * fw + (h1 - 1));
                float ps = b_x[h1] * *p + a_x[h1] * sxy_x;
                *p = ps;
                sxy_x = sxy_x / K_x[h1] + ps;
            }
            if (!a.free_surf && j <= fw) {
                float *p = cl_f(v.pyv + cl_top_idx(v, j) * v.pitch + (col0 + k));
                float ps = b_y[j] * *p + a_y[j] * syy_y;
                *p = ps;
                syy_y = syy_y / K_y[j] + ps;
            }
            if (j >= a.ny - fw + 1) {
                const int h1 = j - a.ny + 2 * fw;
                float *p = cl_f(v.pyv + cl_bot_idx(v, j) * v.pitch + (col0 + k));
                float ps = b_y[h1] * *p + a_y[h1] * syy_y;
                *p = ps;
                syy_y = syy_y / K_y[h1] + ps;
            }
        }
        const float b = get(b4, k);
        const float s = sxy_x + syy_y;
        set(vy4, k, get(vy4, k) + div_dh<P2>(b * a.dt * s, a));
    }
    sts4m(vyp, vy4, nvalid);
}

/* Elastic stress update of the four points i0..i0+3 of own local row lr
 * (s_body, L = 0, FLAGS = 0). */
template <int FDO>
__device__ __forceinline__ void cl_s_points(const StepArgs &a, const ClView &v, int lr, int g, int nt)
{
    constexpr int H = FDO / 2;
    constexpr int NL = (H - 1 + 3) / 4;
    constexpr int NR = (H + 3) / 4;
    constexpr int NXS = 4 * (NL + 1 + NR);
    const int i0 = 1 + 4 * g, j = v.j0 + lr;
    const int c4 = g + HX / 4;
    const int p4 = v.p4;
    const float4 *vyr = cl_f4(v.vy + (lr + H) * p4 + c4);
    const float4 *vyc = cl_f4(v.vy + (lr + 1) * p4 + c4);           /* vy row j-H+1 */
    float4 *sxyp = cl_f4(v.sxy + lr * p4 + c4);
    float4 *syzp = cl_f4(v.syz + (lr + H) * p4 + c4);
    float xs[NXS];
#pragma unroll
    for (int q = 0; q < NL + 1 + NR; q++) {
        const float4 t = vyr[q - NL];
        xs[4 * q] = t.x; xs[4 * q + 1] = t.y; xs[4 * q + 2] = t.z; xs[4 * q + 3] = t.w;
    }
    float4 ys[2 * H];
#pragma unroll
    for (int r = 0; r < 2 * H; r++) ys[r] = vyc[r * p4];
    float4 sxy4 = *sxyp, syz4 = *syzp;
    const float4 c1 = *cl_f4(v.ui + lr * p4 + c4), c2 = *cl_f4(v.uj + lr * p4 + c4);

    const int col0 = i0 - 1 + HX;
    const int nvalid = min(4, a.nx - i0 + 1);
    const float dhi = a.dhi_el;
    const bool in_pml = a.fw > 0 && (i0 <= a.fw || i0 + 3 >= a.nx - a.fw + 1 || (!a.free_surf && j <= a.fw) ||
                                     j >= a.ny - a.fw + 1);
    const float *K_xh = cl_f(v.coef + 3 * v.fw2), *a_xh = cl_f(v.coef + 4 * v.fw2), *b_xh = cl_f(v.coef + 5 * v.fw2);
    const float *K_yh = cl_f(v.coef + 9 * v.fw2), *a_yh = cl_f(v.coef + 10 * v.fw2), *b_yh = cl_f(v.coef + 11 * v.fw2);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int i = i0 + k;
        float vyx, vyy;
#pragma unroll
        for (int m = 1; m <= H; m++) {
            float tx = a.hc[m] * (xs[4 * NL + k + m] - xs[4 * NL + k - m + 1]);
            float ty = a.hc[m] * (get(ys[H - 1 + m], k) - get(ys[H - m], k));
            if (m == 1) { vyx = tx; vyy = ty; }
            else { vyx = vyx + tx; vyy = vyy + ty; }
        }
        vyx = vyx * dhi;
        vyy = vyy * dhi;
        const int fw = a.fw;
        if (in_pml && i <= a.nx) {
            if (i <= fw) {
                float *p = cl_f(v.pxs + lr * 2 * fw + (i - 1));
                float ps = b_xh[i] * *p + a_xh[i] * vyx;
                *p = ps;
                vyx = vyx / K_xh[i] + ps;
            }
            if (i >= a.nx - fw + 1) {
                const int h1 = i - a.nx + 2 * fw;
                float *p = cl_f(v.pxs + lr * 2 * fw + (h1 - 1));
                float ps = b_xh[h1] * *p + a_xh[h1] * vyx;
                *p = ps;
                vyx = vyx / K_xh[h1] + ps;
            }
            if (!a.free_surf && j <= fw) {
                float *p = cl_f(v.pys + cl_top_idx(v, j) * v.pitch + (col0 + k));
                float ps = b_yh[j] * *p + a_yh[j] * vyy;
                *p = ps;
                vyy = vyy / K_yh[j] + ps;
            }
            if (j >= a.ny - fw + 1) {
                const int h1 = j - a.ny + 2 * fw;
                float *p = cl_f(v.pys + cl_bot_idx(v, j) * v.pitch + (col0 + k));
                float ps = b_yh[h1] * *p + a_yh[h1] * vyy;
                *p = ps;
                vyy = vyy / K_yh[h1] + ps;
            }
        }
        set(sxy4, k, get(sxy4, k) + get(c1, k) * vyx);
        set(syz4, k, get(syz4, k) + get(c2, k) * vyy);
    }
    if (((nt & a.chk_mask) == 0 || nt >= a.nt_last) &&
        !(isfinite(sxy4.x) && isfinite(sxy4.y) && isfinite(sxy4.z) && isfinite(sxy4.w) && isfinite(syz4.x) &&
          isfinite(syz4.y) && isfinite(syz4.z) && isfinite(syz4.w) && isfinite(xs[4 * NL])))
        atomicOr(a.status, 1);
    sts4m(sxyp, sxy4, nvalid);
    sts4m(syzp, syz4, nvalid);
}

/* The H halo rows of a haloed shared field (float4 offset `off` of the field
 * in every CTA; own rows at H .. r+H-1) from the neighbouring CTAs' boundary
 * rows: rows 0..H-1 from the last H own rows of rank-1 (which owns ru rows),
 * rows r+H .. r+2H-1 from the first H own rows of rank+1 when it owns rows;
 * otherwise the halo keeps the zeros of the grid's padding. */
__device__ __forceinline__ void cl_halo(cooperative_groups::cluster_group &cl, float4 *base, long long off_me,
                                        long long off_up, long long off_dn, int rank, bool has_up, bool has_dn,
                                        int r, int ru, int H, int p4)
{
    const int n = H * p4;
    float4 *f = base + off_me;
    const float4 *up = has_up ? cl.map_shared_rank(base, rank - 1) + off_up + (long long)ru * p4 : nullptr;
    const float4 *dn = has_dn ? cl.map_shared_rank(base, rank + 1) + off_dn + (long long)H * p4 : nullptr;
    for (int k = threadIdx.x; k < 2 * n; k += blockDim.x) {
        if (k < n) {
            if (up) f[k] = up[k];
        } else if (dn) {
            f[(long long)(r + H) * p4 + (k - n)] = dn[k - n];
        }
    }
}

/* Grid: C CTAs per shot slot (cluster dims (C,1,1), slot = blockIdx.x / C),
 * rows per CTA from g, dynamic shared memory the largest cl_layout(...).bytes
 * of the CTAs; steps *nt_base .. *nt_base + nsteps - 1. */
/* Items of a CTA (a 4-point group g of own row lr): first the groups of
 * every row that no CPML x strip touches, row by row, then the x-strip groups
 * (left, then right), so that the strip work, which costs about twice as
 * much, fills warps of its own.  gl = left-strip groups, gr0 = first
 * right-strip group. */
__device__ __forceinline__ int cl_item(int it, int r, int ng, int gl, int gr0)
{
    const int nint = gr0 - gl, nstr = ng - nint;
    int lr, g;
    if (it < r * nint) {
        lr = it / nint;
        g = gl + (it - lr * nint);
    } else {
        const int q = it - r * nint;
        lr = q / nstr;
        const int e = q - lr * nstr;
        g = e < gl ? e : gr0 + (e - gl);
    }
    return (lr << 16) | g;
}

template <int FDO, bool P2>
__global__ void __launch_bounds__(cl_max_threads(FDO), 1) cl_fwd(StepArgs a, int nsteps, ClGeom geo)
{
    namespace cg = cooperative_groups;
    constexpr int H = FDO / 2;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int C = geo.C;
    const int slot = blockIdx.x / C;
    const long long so = (long long)slot * a.slot_stride;
    const int pitch = a.pitch, p4 = pitch / 4, fw = a.fw;
    const int ng = (a.nx + 3) / 4;
    const int j0 = geo.j0[rank], j1 = geo.j0[rank + 1];
    const int r = j1 - j0;
    const int yt = cl_top_rows(j0, j1, fw, a.free_surf), yb = cl_bot_rows(j0, j1, a.ny, fw);
    const ClLayout L = cl_layout(r, yt + yb, H, p4, fw);
    float *fs = reinterpret_cast<float *>(cl_smem);
    int *is = reinterpret_cast<int *>(cl_smem);
    ClView v;
    v.vy = (int)L.vy; v.syz = (int)L.syz; v.sxy = (int)L.sxy;
    v.br = (int)L.br; v.ui = (int)L.ui; v.uj = (int)L.uj;
    v.pyv = (int)(4 * L.pyv); v.pys = (int)(4 * L.pys);
    v.pxv = (int)L.pxv; v.pxs = (int)L.pxs; v.coef = (int)L.coef;
    v.p4 = p4; v.pitch = pitch; v.fw2 = 2 * fw + 1;
    v.j0 = j0; v.yt = yt;
    v.ybeg = max(j0, a.ny - fw + 1);
    int *grp = is + L.grp, *rec = is + L.rec, *cnt = is + L.cnt;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    const int tid = threadIdx.x, nthr = blockDim.x;

    /* ---- the pass's starting state, the model, the CPML memory and coefficients ---- */
    const int grows = a.ny + 2 * a.hy;
    for (long long k = tid; k < (long long)(r + 2 * H) * p4; k += nthr) {
        const int lr = (int)(k / p4), c = (int)(k - (long long)lr * p4);
        const int row = j0 - 1 + lr;                  /* haloed global row of grid row j0 - H + lr */
        float4 vv = zero, s = zero;
        if (row < grows) {
            const long long off = so + (long long)row * pitch + 4 * c;
            vv = *reinterpret_cast<const float4 *>(a.vy + off);
            s = *reinterpret_cast<const float4 *>(a.syz + off);
        }
        cl_smem[L.vy + k] = vv;
        cl_smem[L.syz + k] = s;
    }
    for (long long k = tid; k < (long long)r * p4; k += nthr) {
        const int lr = (int)(k / p4), c = (int)(k - (long long)lr * p4);
        const int j = j0 + lr;
        const long long d = (long long)(j - 1) * pitch + 4 * c;
        cl_smem[L.sxy + k] = *reinterpret_cast<const float4 *>(a.sxy + so + (long long)(j - 1 + a.hy) * pitch + 4 * c);
        cl_smem[L.br + k] = __ldg(reinterpret_cast<const float4 *>(a.brho + d));
        cl_smem[L.ui + k] = __ldg(reinterpret_cast<const float4 *>(a.uip + d));
        cl_smem[L.uj + k] = __ldg(reinterpret_cast<const float4 *>(a.ujp + d));
    }
    for (long long k = tid; k < (long long)(yt + yb) * p4; k += nthr) {
        const int q = (int)(k / p4), c = (int)(k - (long long)q * p4);
        const int prow = q < yt ? (j0 + q - 1) : (v.ybeg + (q - yt) - a.ny + 2 * fw - 1);   /* psi strip row */
        const long long off = so + (long long)prow * pitch + 4 * c;
        cl_smem[L.pyv + k] = *reinterpret_cast<const float4 *>(a.psi_vyy_v + off);
        cl_smem[L.pys + k] = *reinterpret_cast<const float4 *>(a.psi_syy + off);
    }
    for (int k = tid; k < r * 2 * fw; k += nthr) {
        const long long off = so + (long long)(j0 - 1) * 2 * fw + k;
        fs[L.pxv + k] = a.psi_vxx[off];
        fs[L.pxs + k] = a.psi_sxx[off];
    }
    {
        const float *src[12] = {a.pml.K_x, a.pml.a_x, a.pml.b_x, a.pml.K_x_half, a.pml.a_x_half, a.pml.b_x_half,
                                a.pml.K_y, a.pml.a_y, a.pml.b_y, a.pml.K_y_half, a.pml.a_y_half, a.pml.b_y_half};
        for (int k = tid; k < 12 * v.fw2; k += nthr) fs[L.coef + k] = __ldg(src[k / v.fw2] + k % v.fw2);
    }
    /* the slot's source groups and receivers that lie in the own rows
       (all of the slot's tiles: the per-tile tables are cumulative) */
    if (tid == 0) { cnt[0] = 0; cnt[1] = 0; }
    __syncthreads();
    const int T = a.tl.ntiles;
    const int g_beg = a.tl.goff[(long long)slot * (T + 1)], g_end = a.tl.goff[(long long)slot * (T + 1) + T];
    for (int gi = g_beg + tid; gi < g_end; gi += nthr) {
        const int pk = __ldg(a.tl.gpt + gi);
        const int i = pk & 0xffff, j = pk >> 16;
        if (j < j0 || j >= j1) continue;
        const int e = atomicAdd(&cnt[0], 1);
        int *gr = grp + e * (2 + CL_MAX_MEM);
        gr[0] = (j - j0 + H) * pitch + (i - 1 + HX);  /* float index in the CTA's vy rows */
        const int m0 = __ldg(a.tl.gbeg + gi), m1 = __ldg(a.tl.gbeg + gi + 1);
        gr[1] = m1 - m0;
        for (int m = m0; m < m1; m++) gr[2 + (m - m0)] = __ldg(a.tl.src_id + m);
    }
    const int r_beg = a.tl.roff[(long long)slot * (T + 1)], r_end = a.tl.roff[(long long)slot * (T + 1) + T];
    for (int e = r_beg + tid; e < r_end; e += nthr) {
        const int pk = __ldg(a.tl.rpt + e);
        const int i = pk & 0xffff, j = pk >> 16;
        if (j < j0 || j >= j1) continue;
        const int q = atomicAdd(&cnt[1], 1);
        rec[2 * q] = (j - j0 + H) * pitch + (i - 1 + HX);
        rec[2 * q + 1] = __ldg(a.tl.rid + e);
    }
    const int nt0 = *a.nt_base;
    __syncthreads();
    const int ngrp = cnt[0], nrec = cnt[1];
    const int rec0 = a.tl.rec_off[slot], ntr = a.tl.rec_off[slot + 1] - rec0;
    float *seis = a.tl.seis + a.tl.seis_off[slot];
    const float *sig = a.tl.sig + a.tl.sig_off[slot];
    /* injection warp: lane q < ngrp adds the signals of group q; the signals of
       the coming step are loaded one step ahead */
    int gpt = 0, gn = 0, gsid[CL_MAX_MEM];
    float gnext[CL_MAX_MEM];
    if (tid < 32 && tid < ngrp) {
        const int *gr = grp + tid * (2 + CL_MAX_MEM);
        gpt = gr[0];
        gn = gr[1];
#pragma unroll
        for (int m = 0; m < CL_MAX_MEM; m++) {
            gsid[m] = m < gn ? gr[2 + m] : 0;
            gnext[m] = m < gn ? sig[(long long)gsid[m] * a.tl.sig_ss + (long long)(nt0 - 1) * a.tl.sig_ts] : 0.f;
        }
    }
    float *vyf = cl_f(4 * v.vy);

    const bool has_up = rank > 0 && r > 0;
    const bool has_dn = rank + 1 < C && geo.j0[rank + 2] > j1 && r > 0;
    const int ru = rank > 0 ? j0 - geo.j0[rank - 1] : 0;
    const int rd = rank + 1 < C ? geo.j0[rank + 2] - j1 : 0;
    /* the neighbours' field offsets (their layouts differ by their row counts) */
    const int yu = rank > 0 ? cl_top_rows(geo.j0[rank - 1], j0, fw, a.free_surf) + cl_bot_rows(geo.j0[rank - 1], j0, a.ny, fw) : 0;
    const int yd = rank + 1 < C ? cl_top_rows(j1, geo.j0[rank + 2], fw, a.free_surf) + cl_bot_rows(j1, geo.j0[rank + 2], a.ny, fw) : 0;
    const ClLayout Lu = cl_layout(ru, yu, H, p4, fw), Ld = cl_layout(rd, yd, H, p4, fw);
    /* this thread's items: tid, tid + nthr, ... (the host sizes the CTA so
       that no thread has more than CL_MAX_ITEMS) */
    const int gl = fw > 0 ? min(ng, (fw + 3) / 4) : 0;
    const int gr0 = fw > 0 ? max(gl, min(ng, (a.nx - fw - 3 + 3) / 4)) : ng;
    const int nmy = tid < r * ng ? (r * ng - tid + nthr - 1) / nthr : 0;

    for (int step = 0; step < nsteps; step++) {
        const int nt = nt0 + step;
        const bool run = nt <= a.nt_last;
        if (run) {
#pragma unroll 1
            for (int q = 0; q < nmy; q++) {
                const int m = cl_item(tid + q * nthr, r, ng, gl, gr0);
                cl_v_points<FDO, P2>(a, v, m >> 16, m & 0xffff);
            }
        }
        __syncthreads();
        if (run && tid < ngrp) {                      /* injection: sources of a point in the reference's order */
            float x = vyf[gpt];
            for (int m = 0; m < gn; m++) x = x + gnext[m];
            vyf[gpt] = x;
        }
        cl.sync();                                    /* every velocity of the step is in place */
        if (tid < 32) {
            /* sampling and the next step's signals after the barrier, so that
               these global accesses complete during the stress phase instead of
               holding the barrier's release (own rows of vy stay unchanged
               until the next velocity phase) */
            if (run && a.tl.sample)
                for (int e = tid; e < nrec; e += 32) seis[(long long)(nt - 1) * ntr + rec[2 * e + 1]] = vyf[rec[2 * e]];
            if (tid < ngrp && nt + 1 <= a.nt_last)
                for (int m = 0; m < gn; m++)
                    gnext[m] = sig[(long long)gsid[m] * a.tl.sig_ss + (long long)nt * a.tl.sig_ts];
        }
        cl_halo(cl, cl_smem, L.vy, Lu.vy, Ld.vy, rank, has_up, has_dn, r, ru, H, p4);
        __syncthreads();
        if (run) {
#pragma unroll 1
            for (int q = 0; q < nmy; q++) {
                const int m = cl_item(tid + q * nthr, r, ng, gl, gr0);
                cl_s_points<FDO>(a, v, m >> 16, m & 0xffff, nt);
            }
        }
        cl.sync();                                    /* every stress of the step is in place */
        cl_halo(cl, cl_smem, L.syz, Lu.syz, Ld.syz, rank, has_up, has_dn, r, ru, H, p4);
        __syncthreads();
    }
    cl.sync();                                        /* no CTA reads another's rows after this */

    /* ---- own rows and CPML memory back to the slot's global state ---- */
    for (long long k = tid; k < (long long)r * p4; k += nthr) {
        const int lr = (int)(k / p4), c = (int)(k - (long long)lr * p4);
        const long long off = so + (long long)(j0 - 1 + lr + a.hy) * pitch + 4 * c;
        *reinterpret_cast<float4 *>(a.vy + off) = cl_smem[L.vy + (long long)(lr + H) * p4 + c];
        *reinterpret_cast<float4 *>(a.syz + off) = cl_smem[L.syz + (long long)(lr + H) * p4 + c];
        *reinterpret_cast<float4 *>(a.sxy + off) = cl_smem[L.sxy + k];
    }
    for (long long k = tid; k < (long long)(yt + yb) * p4; k += nthr) {
        const int q = (int)(k / p4), c = (int)(k - (long long)q * p4);
        const int prow = q < yt ? (j0 + q - 1) : (v.ybeg + (q - yt) - a.ny + 2 * fw - 1);
        const long long off = so + (long long)prow * pitch + 4 * c;
        *reinterpret_cast<float4 *>(a.psi_vyy_v + off) = cl_smem[L.pyv + k];
        *reinterpret_cast<float4 *>(a.psi_syy + off) = cl_smem[L.pys + k];
    }
    for (int k = tid; k < r * 2 * fw; k += nthr) {
        const long long off = so + (long long)(j0 - 1) * 2 * fw + k;
        a.psi_vxx[off] = fs[L.pxv + k];
        a.psi_sxx[off] = fs[L.pxs + k];
    }
}

}  // namespace dsh

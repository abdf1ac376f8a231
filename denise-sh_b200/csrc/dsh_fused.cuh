/*
 * dsh_fused.cuh — one kernel per time step: velocity and stress half-steps
 * fused through shared memory.
 *
 * A thread block owns a 128 x 16-point tile of one shot slot.  It
 *   1. stages sxy and syz of the previous step (with the halo its velocity
 *      region needs) in shared memory,
 *   2. computes the new velocity on the tile plus a halo of H-1 points left /
 *      above and H right / below (the points the stress stencil of the tile
 *      reads) into shared memory — halo points are recomputed, not read from
 *      the neighbouring tiles, so no grid-wide synchronisation is needed;
 *      injection is applied to every point of that region, and only owned
 *      points are stored (vy, forward storage, correlation, CPML memory,
 *      receiver samples),
 *   3. computes the stress / memory-variable update of the owned points from
 *      the shared velocities.
 * The stress and velocity fields and the velocity CPML memory are read by
 * neighbouring tiles during the step, so they are double-buffered: step n
 * reads buffer (n-1)&1 and writes buffer n&1 (buffer 0 = vy/sxy/syz/psi_v,
 * buffer 1 = the *_b fields).  Per-point arithmetic is the reference's
 * expression order exactly as in v_body / s_body (the file is compiled with
 * -fmad=false), so results are bit-identical to the two-kernel path.
 *
 * Saves, per grid point and step, the second pass over sxy and syz (8 B),
 * the re-read of vy (4 B) and one launch.  FDORDER <= 8 (the 8 halo columns
 * of the layout cover the staged region); fused injection lists required.
 */
#pragma once
#include "dsh_kernels.cuh"

namespace dsh {

constexpr int FTX = 128, FTY = 16;       /* owned tile */
constexpr int FSW = FTX + 16;            /* staged row: global columns x0 .. x0+143 = points x0-7 .. x0+136 */

/* passes of the fused kernel */
constexpr int FM_FWD = 0;      /* forward, no storage (plain modelling, checkpointed forward) */
constexpr int FM_STORE = 1;    /* forward storing acceleration and strains (full storage, recompute) */
constexpr int FM_ADJ = 2;      /* adjoint with g_rho / g_u correlation */

__device__ __forceinline__ float4 ld4z(const float *p, bool ok)
{
    return ok ? *reinterpret_cast<const float4 *>(p) : make_float4(0.f, 0.f, 0.f, 0.f);
}

template <int FDO, int L, int MODE, bool P2>
__global__ void __launch_bounds__(256, 2) fs_step(StepArgs a, int nt_off)
{
    constexpr int H = FDO / 2;
    constexpr int VH = FTY + 2 * H - 1;      /* velocity rows: j = y0+2-H .. y0+FTY+H */
    constexpr int ZH = FTY + 4 * H - 2;      /* staged syz rows: j = y0+2-2H .. y0+FTY+2H-1 */
    constexpr int NG = FSW / 4;              /* float4 groups per staged row */
    constexpr int G0 = (9 - H) / 4;          /* first group holding velocity-region points */
    constexpr int G1 = (FTX + H + 7) / 4;    /* last one */
    constexpr int LL = L > 0 ? L : 1;
    static_assert(H <= 4, "staged halo covers FDORDER <= 8");
    __shared__ __align__(16) float s_sxy[VH][FSW];
    __shared__ __align__(16) float s_syz[ZH][FSW];
    __shared__ __align__(16) float s_v[VH][FSW];

    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * FTX, y0 = blockIdx.y * FTY;
    const int slot = blockIdx.z;
    const long long so = (long long)slot * a.slot_stride;
    const int pitch = a.pitch;
    const int nt = *a.nt_base + nt_off;
    if (nt > a.nt_last) return;
    const bool odd = ((nt - 1) & 1) != 0;   /* previous step's state in buffer 1 */
    const float *vy_r = (odd ? a.vy_b : a.vy) + so;
    const float *sxy_r = (odd ? a.sxy_b : a.sxy) + so;
    const float *syz_r = (odd ? a.syz_b : a.syz) + so;
    float *vy_w = (odd ? a.vy : a.vy_b) + so;
    float *sxy_w = (odd ? a.sxy : a.sxy_b) + so;
    float *syz_w = (odd ? a.syz : a.syz_b) + so;
    const float *pvx_r = (odd ? a.psi_vxx_b : a.psi_vxx) + so;
    const float *pvy_r = (odd ? a.psi_vyy_v_b : a.psi_vyy_v) + so;
    float *pvx_w = (odd ? a.psi_vxx : a.psi_vxx_b) + so;
    float *pvy_w = (odd ? a.psi_vyy_v : a.psi_vyy_v_b) + so;
    const int rows_total = a.ny + 2 * a.hy;

    pdl_wait();                              /* the previous step is complete */
    pdl_trigger();

    /* ---- 1. stage sxy (velocity rows) and syz (velocity rows +- H) ---- */
    for (int idx = tid; idx < VH * NG; idx += 256) {
        const int r = idx / NG, g = idx % NG;
        const int row = (y0 + 2 - H + r) - 1 + a.hy;
        const int col = x0 + 4 * g;
        const bool ok = row >= 0 && row < rows_total && col + 3 < pitch;
        *reinterpret_cast<float4 *>(&s_sxy[r][4 * g]) = ld4z(sxy_r + (long long)row * pitch + col, ok);
    }
    for (int idx = tid; idx < ZH * NG; idx += 256) {
        const int r = idx / NG, g = idx % NG;
        const int row = (y0 + 2 - 2 * H + r) - 1 + a.hy;
        const int col = x0 + 4 * g;
        const bool ok = row >= 0 && row < rows_total && col + 3 < pitch;
        *reinterpret_cast<float4 *>(&s_syz[r][4 * g]) = ld4z(syz_r + (long long)row * pitch + col, ok);
    }
    /* injection groups whose point lies in this tile's velocity region */
    const int ftile = blockIdx.y * gridDim.x + blockIdx.x;
    int fg0 = 0, fg1 = 0;
    if (a.tl.on) {
        const int *fo = a.fvg_off + (long long)slot * (a.fvg_ntiles + 1) + ftile;
        fg0 = __ldg(fo);
        fg1 = __ldg(fo + 1);
    }
    __syncthreads();

    /* ---- 2. velocities of the region (update_v_PML.c:51-198, 564-583) ---- */
    for (int idx = tid; idx < VH * (G1 - G0 + 1); idx += 256) {
        const int r = idx / (G1 - G0 + 1), g = G0 + idx % (G1 - G0 + 1);
        const int j = y0 + 2 - H + r;
        const int i0 = x0 - 7 + 4 * g;
        const bool rowin = j >= 1 && j <= a.ny;
        const bool owned = rowin && j > y0 && j <= y0 + FTY && g >= 2 && g <= FTX / 4 + 1 && i0 <= a.nx;
        float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
        if (rowin && i0 + 3 >= 1 && i0 <= a.nx) {
            const long long hrow = (long long)(j - 1 + a.hy) * pitch;
            const long long drow = (long long)(j - 1) * pitch;
            const int col0 = i0 - 1 + HX;
            const float4 b4 = ldg4(a.brho + drow + col0);
            float4 vy4 = ld4(vy_r + hrow + col0);
            const float4 old4 = vy4;
            float4 acc4 = make_float4(0.f, 0.f, 0.f, 0.f);
            /* taps as float4 rows of shared memory (conflict-free): xs[p] =
               sxy[i0 - 4*NLV + p] of row j, ys[q] = syz rows j-H .. j+H-1 */
            constexpr int NLV = (H + 3) / 4, NRV = (H - 1 + 3) / 4;
            float xs[4 * (NLV + 1 + NRV)];
#pragma unroll
            for (int v = 0; v < NLV + 1 + NRV; v++) {
                const float4 t = *reinterpret_cast<const float4 *>(&s_sxy[r][4 * (g - NLV + v)]);
                xs[4 * v] = t.x; xs[4 * v + 1] = t.y; xs[4 * v + 2] = t.z; xs[4 * v + 3] = t.w;
            }
            float4 ys[2 * H];
#pragma unroll
            for (int q = 0; q < 2 * H; q++) ys[q] = *reinterpret_cast<const float4 *>(&s_syz[r + q][4 * g]);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int i = i0 + k;
                if (i < 1 || i > a.nx) continue;
                float sxy_x, syy_y;
#pragma unroll
                for (int m = 1; m <= H; m++) {
                    float tx = a.hc[m] * (xs[4 * NLV + k + m - 1] - xs[4 * NLV + k - m]);
                    float ty = a.hc[m] * (get(ys[H + m - 1], k) - get(ys[H - m], k));
                    if (m == 1) { sxy_x = tx; syy_y = ty; }
                    else { sxy_x = sxy_x + tx; syy_y = syy_y + ty; }
                }
                const int fw = a.fw;
                if (fw > 0) {
                    if (i <= fw) {
                        const long long o = (long long)(j - 1) * 2 * fw + (i - 1);
                        float ps = __ldg(a.pml.b_x + i) * pvx_r[o] + __ldg(a.pml.a_x + i) * sxy_x;
                        if (owned) pvx_w[o] = ps;
                        sxy_x = sxy_x / __ldg(a.pml.K_x + i) + ps;
                    }
                    if (i >= a.nx - fw + 1) {
                        const int h1 = i - a.nx + 2 * fw;
                        const long long o = (long long)(j - 1) * 2 * fw + (h1 - 1);
                        float ps = __ldg(a.pml.b_x + h1) * pvx_r[o] + __ldg(a.pml.a_x + h1) * sxy_x;
                        if (owned) pvx_w[o] = ps;
                        sxy_x = sxy_x / __ldg(a.pml.K_x + h1) + ps;
                    }
                    if (!a.free_surf && j <= fw) {
                        const long long o = (long long)(j - 1) * pitch + (col0 + k);
                        float ps = __ldg(a.pml.b_y + j) * pvy_r[o] + __ldg(a.pml.a_y + j) * syy_y;
                        if (owned) pvy_w[o] = ps;
                        syy_y = syy_y / __ldg(a.pml.K_y + j) + ps;
                    }
                    if (j >= a.ny - fw + 1) {
                        const int h1 = j - a.ny + 2 * fw;
                        const long long o = (long long)(h1 - 1) * pitch + (col0 + k);
                        float ps = __ldg(a.pml.b_y + h1) * pvy_r[o] + __ldg(a.pml.a_y + h1) * syy_y;
                        if (owned) pvy_w[o] = ps;
                        syy_y = syy_y / __ldg(a.pml.K_y + h1) + ps;
                    }
                }
                const float b = get(b4, k);
                const float s = sxy_x + syy_y;
                if (MODE != FM_ADJ) set(acc4, k, div_dh<P2>(b * s, a));
                set(vy4, k, get(vy4, k) + div_dh<P2>(b * a.dt * s, a));
            }
            /* injection, sources of one point in the reference's order */
            for (int e = fg0; e < fg1; e++) {
                const int gi_ = __ldg(a.fvg_ids + e);
                const int pk = __ldg(a.tl.gpt + gi_);
                const int gi = pk & 0xffff, gj = pk >> 16;
                if (gj == j && gi >= i0 && gi < i0 + 4) {
                    float v = lane(vy4, gi - i0);
                    const float *sg = a.tl.sig + a.tl.sig_off[slot] + (long long)(nt - 1) * a.tl.sig_ts;
                    for (int m = __ldg(a.tl.gbeg + gi_); m < __ldg(a.tl.gbeg + gi_ + 1); m++)
                        v = v + sg[(long long)__ldg(a.tl.src_id + m) * a.tl.sig_ss];
                    set_lane(vy4, gi - i0, v);
                }
            }
            /* points outside the grid stay zero (the reference's padding) */
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (i0 + k >= 1 && i0 + k <= a.nx) set(out, k, get(vy4, k));
            if (owned) {
                const int nvalid = min(4, a.nx - i0 + 1);
                st4m(vy_w + hrow + col0, vy4, nvalid);
                if (a.tl.sample) {          /* receivers of the two 128 x 8 list tiles of this row */
                    const int ltile = ((j - 1) / BY) * a.tl.ntx + (i0 - 1) / (4 * BX);
                    const int *ro = a.tl.roff + (long long)slot * (a.tl.ntiles + 1) + ltile;
                    const int tr0 = __ldg(ro), tr1 = __ldg(ro + 1);
                    if (tr1 > tr0) {
                        const int r0 = a.tl.rec_off[slot], ntr = a.tl.rec_off[slot + 1] - r0;
                        float *sm = a.tl.seis + a.tl.seis_off[slot] + (long long)(nt - 1) * ntr;
                        for (int e = tr0; e < tr1; e++) {
                            const int pk = __ldg(a.tl.rpt + e);
                            const int ri = pk & 0xffff, rj = pk >> 16;
                            if (rj == j && ri >= i0 && ri < i0 + 4) sm[__ldg(a.tl.rid + e)] = lane(vy4, ri - i0);
                        }
                    }
                }
                if (MODE == FM_STORE) {      /* forward storage of vyp1 */
                    const long long k = store_idx(nt - 1, a.fwd_mod);
                    st4ms(a.fwd + (long long)slot * a.fwd_slot_stride + k * a.fwd_step_stride + drow + col0, acc4,
                          nvalid);
                }
                if (MODE == FM_ADJ) {        /* g_rho += vyp1 * forward acceleration (denise.c:1589) */
                    const long long k = store_idx(a.nt_total - nt, a.fwd_mod);
                    const float4 f4 =
                        ldcs4(a.fwd + (long long)slot * a.fwd_slot_stride + k * a.fwd_step_stride + drow + col0);
                    float4 g4 = ld4(a.grho + so + drow + col0);
                    g4.x = g4.x + (old4.x * f4.x); g4.y = g4.y + (old4.y * f4.y);
                    g4.z = g4.z + (old4.z * f4.z); g4.w = g4.w + (old4.w * f4.w);
                    st4m(a.grho + so + drow + col0, g4, nvalid);
                }
            }
        }
        *reinterpret_cast<float4 *>(&s_v[r][4 * g]) = out;
    }
    /* the staged groups left of G0 / right of G1 are read by no stencil */
    __syncthreads();

    /* ---- 3. stresses and memory variables of the owned tile ---- */
    const float dhi = (L > 0) ? a.dhi_visc : a.dhi_el;
#pragma unroll 1
    for (int half = 0; half < 2; half++) {
        const int g = 2 + (tid & 31);
        const int ro = (tid >> 5) + 8 * half;        /* owned row 0..15 */
        const int j = y0 + 1 + ro;
        const int i0 = x0 + 1 + 4 * (tid & 31);
        if (j > a.ny || i0 > a.nx) continue;
        const int rv = ro + H - 1, rz = ro + 2 * H - 1;
        const int c = 4 * g;
        (void)c;
        const long long drow = (long long)(j - 1) * pitch;
        const long long hrow = (long long)(j - 1 + a.hy) * pitch;
        const int col0 = i0 - 1 + HX;
        const int nvalid = min(4, a.nx - i0 + 1);
        float4 sxy4 = *reinterpret_cast<const float4 *>(&s_sxy[rv][c]);
        float4 syz4 = *reinterpret_cast<const float4 *>(&s_syz[rz][c]);
        float4 c1, c2;
        float4 rr[LL], qq[LL];
        float4 mi4, mj4, ti4, tj4;
        if (L == 0) {
            c1 = ldg4(a.uip + drow + col0);
            c2 = ldg4(a.ujp + drow + col0);
        } else {
#pragma unroll
            for (int l = 0; l < L; l++) {
                rr[l] = ld4(a.r + so + l * a.dstride + drow + col0);
                qq[l] = ld4(a.q + so + l * a.dstride + drow + col0);
            }
            mi4 = ldg4(a.muip + drow + col0);
            mj4 = ldg4(a.mujp + drow + col0);
            ti4 = ldg4(a.tausipjp + drow + col0);
            tj4 = ldg4(a.taus + drow + col0);
        }
        float4 w4, g4, fy, fu;
        if (a.ws) w4 = ld4(a.ws + so + drow + col0);
        if (MODE == FM_ADJ) {
            g4 = ld4(a.gu + so + drow + col0);
            const long long k = store_idx(a.nt_total - nt, a.fwd_mod);
            const float *base = a.fwd + (long long)slot * a.fwd_slot_stride + k * a.fwd_step_stride + drow + col0;
            fy = ldcs4(base + a.dstride);
            fu = ldcs4(base + 2 * a.dstride);
        }
        /* velocity taps: xs[p] = vy[i0 - 4*NLS + p] of row j, ys[q] = vy rows j-H+1 .. j+H */
        constexpr int NLS = (H - 1 + 3) / 4, NRS = (H + 3) / 4;
        float xs[4 * (NLS + 1 + NRS)];
#pragma unroll
        for (int v = 0; v < NLS + 1 + NRS; v++) {
            const float4 t = *reinterpret_cast<const float4 *>(&s_v[rv][4 * (g - NLS + v)]);
            xs[4 * v] = t.x; xs[4 * v + 1] = t.y; xs[4 * v + 2] = t.z; xs[4 * v + 3] = t.w;
        }
        float4 ys[2 * H];
#pragma unroll
        for (int q = 0; q < 2 * H; q++) ys[q] = *reinterpret_cast<const float4 *>(&s_v[rv - H + 1 + q][4 * g]);
        float4 vyx4 = make_float4(0.f, 0.f, 0.f, 0.f), vyy4 = vyx4;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int i = i0 + k;
            float vyx, vyy;
#pragma unroll
            for (int m = 1; m <= H; m++) {
                float tx = a.hc[m] * (xs[4 * NLS + k + m] - xs[4 * NLS + k - m + 1]);
                float ty = a.hc[m] * (get(ys[H - 1 + m], k) - get(ys[H - m], k));
                if (m == 1) { vyx = tx; vyy = ty; }
                else { vyx = vyx + tx; vyy = vyy + ty; }
            }
            vyx = vyx * dhi;
            vyy = vyy * dhi;
            const int fw = a.fw;
            if (fw > 0 && i <= a.nx) {
                if (i <= fw) {
                    float *p = a.psi_sxx + so + (long long)(j - 1) * 2 * fw + (i - 1);
                    float ps = __ldg(a.pml.b_x_half + i) * *p + __ldg(a.pml.a_x_half + i) * vyx;
                    *p = ps;
                    vyx = vyx / __ldg(a.pml.K_x_half + i) + ps;
                }
                if (i >= a.nx - fw + 1) {
                    const int h1 = i - a.nx + 2 * fw;
                    float *p = a.psi_sxx + so + (long long)(j - 1) * 2 * fw + (h1 - 1);
                    float ps = __ldg(a.pml.b_x_half + h1) * *p + __ldg(a.pml.a_x_half + h1) * vyx;
                    *p = ps;
                    vyx = vyx / __ldg(a.pml.K_x_half + h1) + ps;
                }
                if (!a.free_surf && j <= fw) {
                    float *p = a.psi_syy + so + (long long)(j - 1) * pitch + (col0 + k);
                    if (L > 0) {
                        float ps = __ldg(a.pml.b_y + j) * *p + __ldg(a.pml.a_y + j) * vyy;
                        *p = ps;
                        vyy = vyy / __ldg(a.pml.K_y + j) + ps;
                    } else {
                        float ps = __ldg(a.pml.b_y_half + j) * *p + __ldg(a.pml.a_y_half + j) * vyy;
                        *p = ps;
                        vyy = vyy / __ldg(a.pml.K_y_half + j) + ps;
                    }
                }
                if (j >= a.ny - fw + 1) {
                    const int h1 = j - a.ny + 2 * fw;
                    float *p = a.psi_syy + so + (long long)(h1 - 1) * pitch + (col0 + k);
                    float ps = __ldg(a.pml.b_y_half + h1) * *p + __ldg(a.pml.a_y_half + h1) * vyy;
                    *p = ps;
                    vyy = vyy / __ldg(a.pml.K_y_half + h1) + ps;
                }
            }
            set(vyx4, k, vyx);
            set(vyy4, k, vyy);
        }
        if (L == 0) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                set(sxy4, k, get(sxy4, k) + get(c1, k) * get(vyx4, k));
                set(syz4, k, get(syz4, k) + get(c2, k) * get(vyy4, k));
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                set(c1, k, (float)((double)(get(mi4, k) * a.dt) * (1.0 + (double)(a.lf * get(ti4, k)))));
                set(c2, k, (float)((double)(get(mj4, k) * a.dt) * (1.0 + (double)(a.lf * get(tj4, k)))));
            }
            float4 sumr4 = make_float4(0.f, 0.f, 0.f, 0.f), sumq4 = sumr4;
#pragma unroll
            for (int l = 0; l < L; l++) {
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    set(sumr4, k, get(sumr4, k) + get(rr[l], k));
                    set(sumq4, k, get(sumq4, k) + get(qq[l], k));
                }
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                set(sxy4, k, get(sxy4, k) + ((get(c1, k) * get(vyx4, k)) + (a.dthalbe * get(sumr4, k))));
                set(syz4, k, get(syz4, k) + ((get(c2, k) * get(vyy4, k)) + (a.dthalbe * get(sumq4, k))));
            }
            sumr4 = make_float4(0.f, 0.f, 0.f, 0.f);
            sumq4 = sumr4;
#pragma unroll
            for (int l = 0; l < L; l++) {
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const float dipv = (get(mi4, k) * a.eta[l]) * get(ti4, k);
                    const float dv = (get(mj4, k) * a.eta[l]) * get(tj4, k);
                    float rn = a.bip[l] * (get(rr[l], k) * a.cip[l] - (dipv * get(vyx4, k)));
                    float qn = a.bjm[l] * (get(qq[l], k) * a.cjm[l] - (dv * get(vyy4, k)));
                    set(rr[l], k, rn);
                    set(qq[l], k, qn);
                    set(sumr4, k, get(sumr4, k) + rn);
                    set(sumq4, k, get(sumq4, k) + qn);
                }
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                set(sxy4, k, get(sxy4, k) + (a.dthalbe * get(sumr4, k)));
                set(syz4, k, get(syz4, k) + (a.dthalbe * get(sumq4, k)));
            }
        }
        st4m(sxy_w + hrow + col0, sxy4, nvalid);
        st4m(syz_w + hrow + col0, syz4, nvalid);
#pragma unroll
        for (int l = 0; l < L; l++) {
            st4m(a.r + so + l * a.dstride + drow + col0, rr[l], nvalid);
            st4m(a.q + so + l * a.dstride + drow + col0, qq[l], nvalid);
        }
        const float4 vnow = *reinterpret_cast<const float4 *>(&s_v[rv][c]);
        if (!(isfinite(sxy4.x) && isfinite(sxy4.y) && isfinite(sxy4.z) && isfinite(sxy4.w) && isfinite(syz4.x) &&
              isfinite(syz4.y) && isfinite(syz4.z) && isfinite(syz4.w) && isfinite(vnow.x)))
            atomicOr(a.status, 1);
        if (MODE == FM_STORE) {
            const long long k = store_idx(nt - 1, a.fwd_mod);
            float *base = a.fwd + (long long)slot * a.fwd_slot_stride + k * a.fwd_step_stride + drow + col0;
            st4ms(base + a.dstride, vyy4, nvalid);
            st4ms(base + 2 * a.dstride, vyx4, nvalid);
        }
        if (a.ws) {                       /* energy W += vy^2 (eprecond.c:11) */
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float v = get(vnow, k);
                set(w4, k, get(w4, k) + v * v);
            }
            st4m(a.ws + so + drow + col0, w4, nvalid);
        }
        if (MODE == FM_ADJ) {             /* g_u += uyx_fwd*sxy + uy_fwd*syz (denise.c:1609) */
#pragma unroll
            for (int kk = 0; kk < 4; kk++)
                set(g4, kk, get(g4, kk) + ((get(fu, kk) * get(sxy4, kk)) + (get(fy, kk) * get(syz4, kk))));
            st4m(a.gu + so + drow + col0, g4, nvalid);
        }
    }
}

}  // namespace dsh

/*
 * dsh_tblock.cuh — small elastic grids: several time steps of plain forward
 * modelling per launch (temporal blocking with overlapped tiles).
 *
 * The kernel pair pays two launches per time step, and on a 500 x 200 grid
 * (1e5 points, less than one wave of blocks) each launch is mostly latency:
 * ~12 us per step for 1.2 MB of state.  Here one launch advances k steps.
 * Thread block (CTA) b owns a tw x th tile of grid points and holds, in its
 * shared memory, that tile grown by g = kmax * (FDORDER - 1) points on every
 * side: vy, sxy, syz, the model factors 1/rho, uip, ujp and the four CPML
 * memory fields.  One step of the velocity update at a point reads sxy and
 * syz up to H = FDORDER/2 points away (H left, H-1 right), one step of the
 * stress update reads vy up to H points away (H-1 left, H right), so a full
 * step shrinks the region of valid values by 2H - 1 = FDORDER - 1 points per
 * side.  Step s (0-based) of a k-step launch therefore updates
 *     velocity on the own tile grown by (k-1-s)(2H-1) + H-1 (left/top) and
 *              (k-1-s)(2H-1) + H (right/bottom) points,
 *     stress   on the own tile grown by (k-1-s)(2H-1) points,
 * both clipped to the grid; after step k-1 the own tile is exact and goes
 * back to global memory (the halo was recomputed redundantly by this CTA
 * and, exactly, by its neighbours).  Points outside the grid stay 0, as the
 * global arrays' padding does.  Between the phases of a step the CTA
 * synchronises with __syncthreads only: no CTA waits for another, so
 * neighbouring tiles never depend on each other inside a launch.
 *
 * Source groups whose point lies in the shared-memory tile and receivers in
 * the own tile are listed in shared memory at the start of the launch.  The
 * injection of step nt is applied to every group point inside the step's
 * velocity region (every CTA that recomputes the point adds the same
 * signal), the samples are written by the owner only, after the injection,
 * as in v_body.
 *
 * Per point the arithmetic is that of v_body / s_body (dsh_kernels.cuh) for
 * plain elastic forward modelling — the same expressions in the same order,
 * compiled with -fmad=false — so results are bit-identical to the kernel
 * pair (update_v_PML.c:51-198, update_s_elastic_PML.c:51-455,
 * seismo_ssg.c:17-27).  A point lies in at most one CPML strip per axis
 * (the host requires NX, NY >= 2 FW), so one memory value per field and
 * point suffices.
 */
#pragma once

#include "dsh_kernels.cuh"

namespace dsh {

constexpr int TB_THREADS = 512;  /* threads per CTA */
constexpr int TB_MAX_GRP = 32;   /* source points (groups) of a slot */
constexpr int TB_MAX_MEM = 4;    /* sources at one point */
constexpr int TB_MAX_REC = 512;  /* receivers of a slot */
constexpr int TB_FIELDS = 10;    /* vy sxy syz 1/rho uip ujp psi_vxx psi_vyy psi_sxx psi_syy */

struct TbGeom {
    int tw, th;                  /* own tile: tw x th grid points */
    int g;                       /* shared-memory halo per side: kmax * (FDORDER - 1) */
    int ew, eh;                  /* shared-memory tile: (tw + 2g) x (th + 2g) */
};

/* dynamic shared memory of one CTA in bytes: the fields, then the lists
 * (groups: local index, member count, packed point, member ids; receivers:
 * local index, receiver id; two counters) */
__host__ __device__ inline long long tb_smem_bytes(const TbGeom &g)
{
    return 4LL * (TB_FIELDS * (long long)g.ew * g.eh + TB_MAX_GRP * (3 + TB_MAX_MEM) + 2LL * TB_MAX_REC + 2);
}

template <int FDO, bool P2>
__global__ void __launch_bounds__(TB_THREADS) tb_fwd(StepArgs a, TbGeom geo, int n_first, int ksteps)
{
    constexpr int H = FDO / 2, R = FDO - 1;
    extern __shared__ float tb_smem[];
    const int slot = blockIdx.z;
    const long long so = (long long)slot * a.slot_stride;
    const int nx = a.nx, ny = a.ny, fw = a.fw, pitch = a.pitch;
    const bool top = !a.free_surf;
    const int ox = 1 + blockIdx.x * geo.tw, oy = 1 + blockIdx.y * geo.th;      /* first own point */
    const int ox1 = min(ox + geo.tw - 1, nx), oy1 = min(oy + geo.th - 1, ny);  /* last own point */
    const int gx0 = ox - geo.g, gy0 = oy - geo.g, ew = geo.ew, eh = geo.eh;
    const int np = ew * eh;
    float *vy = tb_smem, *sxy = vy + np, *syz = sxy + np, *br = syz + np, *ui = br + np, *uj = ui + np;
    float *pvx = uj + np, *pvy = pvx + np, *psx = pvy + np, *psy = psx + np;
    int *gl = reinterpret_cast<int *>(psy + np);   /* group k: local index gl[k], members gl[MAX+k], point gl[2MAX+k] */
    int *gs = gl + 3 * TB_MAX_GRP;                  /* member ids of group k: gs[k*TB_MAX_MEM + m] */
    int *rl = gs + TB_MAX_GRP * TB_MAX_MEM;         /* own receiver e: local index rl[e], id rl[TB_MAX_REC + e] */
    int *cnt = rl + 2 * TB_MAX_REC;                 /* groups, receivers */
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = TB_THREADS / 32;

    if (tid == 0) { cnt[0] = 0; cnt[1] = 0; }
    pdl_wait();                                     /* the previous launch's steps are complete */
    pdl_trigger();

    /* ---- the shared-memory tile from the slot's state and the model ---- */
    for (int y = warp; y < eh; y += NW) {
        const int j = gy0 + y;
        const bool jin = j >= 1 && j <= ny;
        for (int x = lane; x < ew; x += 32) {
            const int i = gx0 + x, p = y * ew + x;
            float v = 0.f, sx = 0.f, sz = 0.f, b = 0.f, u1 = 0.f, u2 = 0.f, q0 = 0.f, q1 = 0.f, q2 = 0.f, q3 = 0.f;
            if (jin && i >= 1 && i <= nx) {
                const long long h = so + (long long)(j - 1 + a.hy) * pitch + (i - 1 + HX);
                const long long d = (long long)(j - 1) * pitch + (i - 1 + HX);
                v = a.vy[h]; sx = a.sxy[h]; sz = a.syz[h];
                b = __ldg(a.brho + d); u1 = __ldg(a.uip + d); u2 = __ldg(a.ujp + d);
                if (fw > 0) {
                    const int xi = i <= fw ? i - 1 : (i >= nx - fw + 1 ? i - nx + 2 * fw - 1 : -1);
                    const int yr = (top && j <= fw) ? j - 1 : (j >= ny - fw + 1 ? j - ny + 2 * fw - 1 : -1);
                    if (xi >= 0) {
                        const long long o = so + (long long)(j - 1) * 2 * fw + xi;
                        q0 = a.psi_vxx[o]; q2 = a.psi_sxx[o];
                    }
                    if (yr >= 0) {
                        const long long o = so + (long long)yr * pitch + (i - 1 + HX);
                        q1 = a.psi_vyy_v[o]; q3 = a.psi_syy[o];
                    }
                }
            }
            vy[p] = v; sxy[p] = sx; syz[p] = sz; br[p] = b; ui[p] = u1; uj[p] = u2;
            pvx[p] = q0; pvy[p] = q1; psx[p] = q2; psy[p] = q3;
        }
    }
    __syncthreads();                                /* counters zeroed */

    /* ---- source groups in the tile, receivers in the own tile ---- */
    if (a.tl.on) {
        const int T = a.tl.ntiles;
        const int *go = a.tl.goff + (long long)slot * (T + 1);
        const int g0 = __ldg(go), g1 = __ldg(go + T);
        for (int g = g0 + tid; g < g1; g += TB_THREADS) {
            const int pk = __ldg(a.tl.gpt + g), gi = pk & 0xffff, gj = pk >> 16;
            if (gi >= gx0 && gi < gx0 + ew && gj >= gy0 && gj < gy0 + eh) {
                const int k = atomicAdd(&cnt[0], 1);
                if (k < TB_MAX_GRP) {                /* the host admits at most TB_MAX_GRP groups per slot */
                    const int b0 = __ldg(a.tl.gbeg + g), nm = min(__ldg(a.tl.gbeg + g + 1) - b0, TB_MAX_MEM);
                    gl[k] = (gj - gy0) * ew + (gi - gx0);
                    gl[TB_MAX_GRP + k] = nm;
                    gl[2 * TB_MAX_GRP + k] = pk;
                    for (int m = 0; m < nm; m++) gs[k * TB_MAX_MEM + m] = __ldg(a.tl.src_id + b0 + m);
                }
            }
        }
        if (a.tl.sample) {
            const int *ro = a.tl.roff + (long long)slot * (T + 1);
            const int e0 = __ldg(ro), e1 = __ldg(ro + T);
            for (int e = e0 + tid; e < e1; e += TB_THREADS) {
                const int pk = __ldg(a.tl.rpt + e), ri = pk & 0xffff, rj = pk >> 16;
                if (ri >= ox && ri <= ox1 && rj >= oy && rj <= oy1) {
                    const int k = atomicAdd(&cnt[1], 1);
                    if (k < TB_MAX_REC) {
                        rl[k] = (rj - gy0) * ew + (ri - gx0);
                        rl[TB_MAX_REC + k] = __ldg(a.tl.rid + e);
                    }
                }
            }
        }
    }
    __syncthreads();
    const int ngrp = min(cnt[0], TB_MAX_GRP), nrec = min(cnt[1], TB_MAX_REC);
    const int ntr = nrec > 0 ? a.tl.rec_off[slot + 1] - a.tl.rec_off[slot] : 0;
    float *seis = nrec > 0 ? a.tl.seis + a.tl.seis_off[slot] : nullptr;
    const float *sig = ngrp > 0 ? a.tl.sig + a.tl.sig_off[slot] : nullptr;

    int bad = 0;
    for (int s = 0; s < ksteps; s++) {
        const int nt = n_first + s;
        const int e = (ksteps - 1 - s) * R;
        /* this step's signals of the CTA's groups, fetched before the velocity
           update so that their latency overlaps it */
        float sv[TB_MAX_MEM];
        if (tid < ngrp) {
            const float *sg = sig + (long long)(nt - 1) * a.tl.sig_ts;
#pragma unroll
            for (int m = 0; m < TB_MAX_MEM; m++)
                if (m < gl[TB_MAX_GRP + tid]) sv[m] = sg[(long long)gs[tid * TB_MAX_MEM + m] * a.tl.sig_ss];
        }

        /* ---- velocity half-step (v_body) ---- */
        const int vx0 = max(1, ox - e - (H - 1)), vx1 = min(nx, ox1 + e + H);
        const int vy0 = max(1, oy - e - (H - 1)), vy1 = min(ny, oy1 + e + H);
        for (int j = vy0 + warp; j <= vy1; j += NW) {
            const int row = (j - gy0) * ew - gx0;
            for (int i = vx0 + lane; i <= vx1; i += 32) {
                const int p = row + i;
                float sxy_x, syy_y;
#pragma unroll
                for (int m = 1; m <= H; m++) {
                    const float tx = a.hc[m] * (sxy[p + m - 1] - sxy[p - m]);
                    const float ty = a.hc[m] * (syz[p + (m - 1) * ew] - syz[p - m * ew]);
                    if (m == 1) { sxy_x = tx; syy_y = ty; }
                    else { sxy_x = sxy_x + tx; syy_y = syy_y + ty; }
                }
                if (fw > 0) {
                    if (i <= fw) {
                        const float ps = __ldg(a.pml.b_x + i) * pvx[p] + __ldg(a.pml.a_x + i) * sxy_x;
                        pvx[p] = ps;
                        sxy_x = sxy_x / __ldg(a.pml.K_x + i) + ps;
                    } else if (i >= nx - fw + 1) {
                        const int h1 = i - nx + 2 * fw;
                        const float ps = __ldg(a.pml.b_x + h1) * pvx[p] + __ldg(a.pml.a_x + h1) * sxy_x;
                        pvx[p] = ps;
                        sxy_x = sxy_x / __ldg(a.pml.K_x + h1) + ps;
                    }
                    if (top && j <= fw) {
                        const float ps = __ldg(a.pml.b_y + j) * pvy[p] + __ldg(a.pml.a_y + j) * syy_y;
                        pvy[p] = ps;
                        syy_y = syy_y / __ldg(a.pml.K_y + j) + ps;
                    } else if (j >= ny - fw + 1) {
                        const int h1 = j - ny + 2 * fw;
                        const float ps = __ldg(a.pml.b_y + h1) * pvy[p] + __ldg(a.pml.a_y + h1) * syy_y;
                        pvy[p] = ps;
                        syy_y = syy_y / __ldg(a.pml.K_y + h1) + ps;
                    }
                }
                const float b = br[p];
                const float sum = sxy_x + syy_y;
                vy[p] = vy[p] + div_dh<P2>(b * a.dt * sum, a);
            }
        }
        __syncthreads();

        /* ---- injection of step nt (sources of a point in the reference's order) ---- */
        if (tid < ngrp) {
            const int pk = gl[2 * TB_MAX_GRP + tid], gi = pk & 0xffff, gj = pk >> 16;
            if (gi >= vx0 && gi <= vx1 && gj >= vy0 && gj <= vy1) {
                const int p = gl[tid], nm = gl[TB_MAX_GRP + tid];
                float v = vy[p];
#pragma unroll
                for (int m = 0; m < TB_MAX_MEM; m++)
                    if (m < nm) v = v + sv[m];
                vy[p] = v;
            }
        }
        __syncthreads();

        /* ---- receiver samples (own points; vy after the injection) ---- */
        if (nrec > 0) {
            float *sm = seis + (long long)(nt - 1) * ntr;
            for (int r = tid; r < nrec; r += TB_THREADS) sm[rl[TB_MAX_REC + r]] = vy[rl[r]];
        }

        /* ---- stress half-step (s_body, L = 0) ---- */
        const bool chk = (nt & a.chk_mask) == 0 || nt >= a.nt_last;
        const int sx0 = max(1, ox - e), sx1 = min(nx, ox1 + e);
        const int sy0 = max(1, oy - e), sy1 = min(ny, oy1 + e);
        for (int j = sy0 + warp; j <= sy1; j += NW) {
            const int row = (j - gy0) * ew - gx0;
            for (int i = sx0 + lane; i <= sx1; i += 32) {
                const int p = row + i;
                float vyx, vyy;
#pragma unroll
                for (int m = 1; m <= H; m++) {
                    const float tx = a.hc[m] * (vy[p + m] - vy[p - m + 1]);
                    const float ty = a.hc[m] * (vy[p + m * ew] - vy[p - (m - 1) * ew]);
                    if (m == 1) { vyx = tx; vyy = ty; }
                    else { vyx = vyx + tx; vyy = vyy + ty; }
                }
                vyx = vyx * a.dhi_el;
                vyy = vyy * a.dhi_el;
                if (fw > 0) {
                    if (i <= fw) {
                        const float ps = __ldg(a.pml.b_x_half + i) * psx[p] + __ldg(a.pml.a_x_half + i) * vyx;
                        psx[p] = ps;
                        vyx = vyx / __ldg(a.pml.K_x_half + i) + ps;
                    } else if (i >= nx - fw + 1) {
                        const int h1 = i - nx + 2 * fw;
                        const float ps = __ldg(a.pml.b_x_half + h1) * psx[p] + __ldg(a.pml.a_x_half + h1) * vyx;
                        psx[p] = ps;
                        vyx = vyx / __ldg(a.pml.K_x_half + h1) + ps;
                    }
                    if (top && j <= fw) {
                        const float ps = __ldg(a.pml.b_y_half + j) * psy[p] + __ldg(a.pml.a_y_half + j) * vyy;
                        psy[p] = ps;
                        vyy = vyy / __ldg(a.pml.K_y_half + j) + ps;
                    } else if (j >= ny - fw + 1) {
                        const int h1 = j - ny + 2 * fw;
                        const float ps = __ldg(a.pml.b_y_half + h1) * psy[p] + __ldg(a.pml.a_y_half + h1) * vyy;
                        psy[p] = ps;
                        vyy = vyy / __ldg(a.pml.K_y_half + h1) + ps;
                    }
                }
                const float nsx = sxy[p] + ui[p] * vyx, nsz = syz[p] + uj[p] * vyy;
                sxy[p] = nsx;
                syz[p] = nsz;
                /* finite check of the own points (a non-finite value never turns finite again) */
                if (chk && i >= ox && i <= ox1 && j >= oy && j <= oy1 &&
                    !(isfinite(nsx) && isfinite(nsz) && isfinite(vy[p])))
                    bad = 1;
            }
        }
        __syncthreads();
    }

    /* ---- the own tile back to the slot's state ---- */
    for (int j = oy + warp; j <= oy1; j += NW) {
        const int row = (j - gy0) * ew - gx0;
        for (int i = ox + lane; i <= ox1; i += 32) {
            const int p = row + i;
            const long long h = so + (long long)(j - 1 + a.hy) * pitch + (i - 1 + HX);
            a.vy[h] = vy[p]; a.sxy[h] = sxy[p]; a.syz[h] = syz[p];
            if (fw > 0) {
                const int xi = i <= fw ? i - 1 : (i >= nx - fw + 1 ? i - nx + 2 * fw - 1 : -1);
                const int yr = (top && j <= fw) ? j - 1 : (j >= ny - fw + 1 ? j - ny + 2 * fw - 1 : -1);
                if (xi >= 0) {
                    const long long o = so + (long long)(j - 1) * 2 * fw + xi;
                    a.psi_vxx[o] = pvx[p]; a.psi_sxx[o] = psx[p];
                }
                if (yr >= 0) {
                    const long long o = so + (long long)yr * pitch + (i - 1 + HX);
                    a.psi_vyy_v[o] = pvy[p]; a.psi_syy[o] = psy[p];
                }
            }
        }
    }
    if (__syncthreads_or(bad) && tid == 0) atomicOr(a.status, 1);
}

}  // namespace dsh

/*
 * dsh_kernels.cuh — sm_100a kernels of the SH time step.
 *
 * Layout in HBM (one "slot" per concurrently advanced shot):
 *   haloed fields vy, sxy, syz   [ny + 2*hy][pitch], element (i,j) at
 *                                 (j-1+hy)*pitch + (i-1+hx); the halo stays 0
 *   interior fields (model coefficients, memory variables, energies,
 *   gradients, stored forward wavefields)   [ny][pitch], element at
 *                                 (j-1)*pitch + (i-1+hx)
 *   CPML memory psi: x strips [ny][2fw], y strips [2fw][pitch]
 * hx = 8 and pitch % 32 == 0, so the four x-consecutive points a thread owns
 * start on a 16-byte boundary and every row access is a float4.
 *
 * Arithmetic: every point is computed with the reference's expression order
 * (src/update_v_PML.c, src/update_s_elastic_PML.c, src/update_s_visc_PML.c)
 * and the file is compiled with -fmad=false, so no multiply-add is fused:
 * results are bit-identical to the reference's FP32 CPU code.
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dsh {

constexpr int HX = 8;            /* left halo / alignment columns */
constexpr int BX = 32;           /* threads per block along x (4 points each) */
constexpr int BY = 8;            /* threads per block along depth */
#ifndef SSTEP_MIN_BLOCKS
#define SSTEP_MIN_BLOCKS 2       /* resident stress-kernel blocks per SM the register budget targets */
#endif
#ifndef VSTEP_MIN_BLOCKS
#define VSTEP_MIN_BLOCKS 3       /* resident velocity-kernel blocks per SM the register budget targets */
#endif
#ifndef VSTEP_MIN_BLOCKS_FWD
#define VSTEP_MIN_BLOCKS_FWD 4   /* the same for the forward velocity kernel (no correlation), which fits
                                    64 registers */
#endif

/* flags of the velocity kernel */
constexpr int VF_ADJOINT = 1;    /* sw=1: vyp1 = old vy (update_v_PML.c:189-192) */
constexpr int VF_ACC_OUT = 2;    /* write vyp1 (acceleration or old vy) to acc_out */
constexpr int VF_CORR = 4;       /* g_rho += vyp1 * stored forward acceleration (denise.c:1589) */
constexpr int VF_HESS = 8;       /* H_rho += acc^2 (hessian.c:93) */
/* flags of the stress kernel */
constexpr int SF_STRAIN_OUT = 1; /* write uy = vyy, uyx = vyx (GRAD_FORM=2) */
constexpr int SF_ENERGY = 2;     /* unused: the energy W += vy^2 (eprecond.c:11) runs when ws != nullptr */
constexpr int SF_CORR = 4;       /* g_u += uyx_fwd*sxy + uy_fwd*syz (denise.c:1609) */
constexpr int SF_HESS = 8;       /* H_u += uy^2 + (0.5 uyx)^2 (hessian.c:92) */
constexpr int SF_PARAMS = 16;    /* viscoelastic: read precomputed fipjp, f, dip_l, d_l (the compat layer)
                                    instead of forming them from muip, mujp, tausipjp, taus */
constexpr int SF_QSENS = 32;     /* with SF_STRAIN_OUT: also store the step's stress-increment
                                    sensitivities to tau (the Qs gradient's forward part) */
constexpr int SF_CORRQ = 64;     /* with SF_CORR: accumulate the Qs-gradient correlation */

struct PmlCoef {                 /* device copies, index 1..2fw */
    const float *K_x, *a_x, *b_x, *K_x_half, *a_x_half, *b_x_half;
    const float *K_y, *a_y, *b_y, *K_y_half, *a_y_half, *b_y_half;
};

/* Source injection and receiver sampling fused into the velocity kernel:
 * per slot, the groups of sources (one group per grid point, members in the
 * reference's order) and the receivers are listed per thread block tile. */
struct TileLists {
    const int *goff;             /* [slot][ntiles+1] -> group index range of a tile */
    const int *gpt;              /* packed point (j << 16 | i) of group g */
    const int *gbeg;             /* members of group g: src_id[gbeg[g] .. gbeg[g+1]) */
    const int *src_id;
    const float *sig;            /* signal of source sid at step nt: sig[sig_off[s] + sid*sig_ss + (nt-1)*sig_ts] */
    const long long *sig_off;
    long long sig_ss, sig_ts;
    const int *roff;             /* [slot][ntiles+1] -> receiver entries of a tile */
    const int *rpt;              /* packed point of receiver entry e */
    const int *rid;              /* receiver index (within its slot) of entry e */
    const int *rec_off;          /* [slot+1]: receivers of slot s are rec_off[s] .. rec_off[s+1] */
    float *seis;                 /* slot s: seis[seis_off[s] + (nt-1)*ntr_s + r] */
    const long long *seis_off;
    int ntiles;
    int ntx;                     /* list tiles along x: ceil(nx / 128); tile of (i, j) = ((j-1)/8)*ntx + (i-1)/128 */
    int on;                      /* fused path active (all positions inside the grid) */
    int sample;
};

struct StepArgs {
    int nx, ny, pitch, hy, fw, free_surf, l;
    int fd12_compat;
    int fdo, p2;                 /* FDORDER; DH a power of two (multi-model launches pick the body from these) */
    int nslots;                  /* shot slots allocated (multi-model launches skip slots >= nslots) */
    int l2_stream;               /* evict-first in L2: bit 0 memory variables, bit 1 stress model factors */
    int nt_last;                 /* last valid step of this pass (1-based) */
    int nt_total;                /* NT of the pass (for the Hessian's nt < NTDTINV) */
    int chk_mask;                /* finite check of the updated fields on steps with (nt & chk_mask) == 0
                                    and on the pass's last step (0: every step) */
    const int *nt_base;          /* device step counter; step = *nt_base + nt_off */
    long long fstride;           /* floats per haloed field */
    long long dstride;           /* floats per interior field */
    long long slot_stride;       /* floats between consecutive shot slots */
    float hc[7];
    float dt, dh, inv_dh, dhi_el, dhi_visc, dthalbe;
    PmlCoef pml;
    /* per-slot state (slot 0 base; slot s at + s*slot_stride) */
    float *vy, *sxy, *syz, *r, *q, *psi_vxx, *psi_vyy_v, *psi_sxx, *psi_syy;
    float *ws, *gu, *grho, *hu, *hrho;
    /* model (shared by all slots) */
    const float *brho, *uip, *ujp, *fipjp, *f, *dip, *d;
    const float *muip, *mujp, *tausipjp, *taus;   /* viscoelastic base factors */
    float eta[4];                /* DT / tau_l */
    float lf;                    /* L as a float */
    float sumu;                  /* sum_l w^2 tau_l^2 / (1 + w^2 tau_l^2) (prepare_update_s.c:29-32) */
    float *exy, *eyz, *gqx, *gqy;   /* Qs gradient (per slot): adjoint strains, correlation sums */
    float bip[4], bjm[4], cip[4], cjm[4];
    /* stored forward wavefields: slot s, stored step k (0-based) at
       fwd + s*fwd_slot_stride + k*fwd_step_stride (+ 0/1/2 * dstride for acc/uy/uyx) */
    float *fwd;
    long long fwd_slot_stride, fwd_step_stride;
    int fwd_mod;                 /* stored-step index: forward (nt-1) % fwd_mod, adjoint (NT-nt) % fwd_mod
                                    (fwd_mod = NT: full storage; = C: a C-step segment buffer) */
    /* compat outputs (Layer-1): explicit vyp1/uy/uyx haloed fields */
    float *out_acc, *out_uy, *out_uyx;
    int *status;                 /* device error word (non-finite detection) */
    long long wait_polls;        /* poll limit of bounded device waits (the persistent launch's grid barrier) */
    const void *tm_sxy, *tm_syz;   /* tensor maps (CUtensorMap, device memory) of sxy / syz over all slots,
                                      for the TMA-staged velocity kernel; NULL when not built */
    TileLists tl;
    /* fused step (dsh_fused.cuh): second buffers of the fields neighbouring
       tiles read during a step, and the injection groups of each 128 x 16
       tile's velocity region: fvg_ids[fvg_off[slot*(fvg_ntiles+1) + tile] ..] */
    float *vy_b, *sxy_b, *syz_b, *psi_vxx_b, *psi_vyy_v_b;
    const int *fvg_off, *fvg_ids;
    int fvg_ntiles;
};

#ifndef DSH_L2_KEEP
#define DSH_L2_KEEP 1
#endif
#if DSH_L2_KEEP
/* The fields that every time step reads again (wavefield state, memory
 * variables, model factors, energies, gradient sums) are loaded and stored
 * with an L2 evict-last policy, so that a working set smaller than the L2
 * stays there from one step to the next; the stored forward wavefield is
 * streamed (st4ms / ldcs4 below). */
__device__ __forceinline__ uint64_t l2_keep()
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ float4 ld4(const float *p)
{
    float4 v;
    asm volatile("ld.global.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(l2_keep()));
    return v;
}
__device__ __forceinline__ float4 ldg4(const float *p)
{
    float4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(l2_keep()));
    return v;
}
__device__ __forceinline__ void st4(float *p, float4 v)
{
    asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(v.x), "f"(v.y),
                 "f"(v.z), "f"(v.w), "l"(l2_keep())
                 : "memory");
}
__device__ __forceinline__ void st1(float *p, float v)
{
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(l2_keep()) : "memory");
}
#else
__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float4 ldg4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ void st1(float *p, float v) { *p = v; }
#endif
#if DSH_L2_KEEP
/* The memory variables (StepArgs::l2_stream bit 0) and the stress kernel's
 * model factors (bit 1) are loaded and stored evict-first when the host finds
 * that the velocity kernel's read set then stays in L2 from one half-step to
 * the next; otherwise they keep the evict-last policy. */
__device__ __forceinline__ uint64_t l2_drop()
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ float4 ld4p(const float *p, uint64_t pol)
{
    float4 v;
    asm volatile("ld.global.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float4 ldg4p(const float *p, uint64_t pol)
{
    float4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ void st4p(float *p, float4 v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(v.x), "f"(v.y),
                 "f"(v.z), "f"(v.w), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void st1p(float *p, float v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol) : "memory");
}
#define DSH_L2_POL(a, bit) (((a).l2_stream & (bit)) ? l2_drop() : l2_keep())
#else
__device__ __forceinline__ float4 ld4p(const float *p, uint64_t) { return ld4(p); }
__device__ __forceinline__ float4 ldg4p(const float *p, uint64_t) { return ldg4(p); }
__device__ __forceinline__ void st4p(float *p, float4 v, uint64_t) { st4(p, v); }
__device__ __forceinline__ void st1p(float *p, float v, uint64_t) { st1(p, v); }
#define DSH_L2_POL(a, bit) 0ull
#endif
/* state loads of the persistent kernel: other blocks wrote them earlier in the
 * same launch, so they bypass L1 (ld.global.cg) */
template <bool CG>
__device__ __forceinline__ float4 lds4(const float *p)
{
    if (CG) return __ldcg(reinterpret_cast<const float4 *>(p));
    return ld4(p);
}
__device__ __forceinline__ float get(const float4 &v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }
__device__ __forceinline__ void set(float4 &v, int k, float x)
{
    if (k == 0) v.x = x; else if (k == 1) v.y = x; else if (k == 2) v.z = x; else v.w = x;
}

/* store the lanes of v that lie inside the grid (i0+k <= nx) */
__device__ __forceinline__ void st4m(float *p, float4 v, int nvalid)
{
    if (nvalid >= 4) { st4(p, v); return; }
    if (nvalid > 0) st1(p, v.x);
    if (nvalid > 1) st1(p + 1, v.y);
    if (nvalid > 2) st1(p + 2, v.z);
}
__device__ __forceinline__ void st4mp(float *p, float4 v, int nvalid, uint64_t pol)
{
    if (nvalid >= 4) { st4p(p, v, pol); return; }
    if (nvalid > 0) st1p(p, v.x, pol);
    if (nvalid > 1) st1p(p + 1, v.y, pol);
    if (nvalid > 2) st1p(p + 2, v.z, pol);
}

/* forward-storage traffic is written once per pass and read once by the
 * adjoint, so it is streamed (st.global.cs / ld.global.cs: evict-first in L2)
 * and leaves the L2 to the fields that every time step reads again */
__device__ __forceinline__ void st4ms(float *p, float4 v, int nvalid)
{
    if (nvalid >= 4) { __stcs(reinterpret_cast<float4 *>(p), v); return; }
    if (nvalid > 0) __stcs(p, v.x);
    if (nvalid > 1) __stcs(p + 1, v.y);
    if (nvalid > 2) __stcs(p + 2, v.z);
}
__device__ __forceinline__ float4 ldcs4(const float *p) { return __ldcs(reinterpret_cast<const float4 *>(p)); }

/* Programmatic dependent launch (PTX griddepcontrol): a kernel launched with
 * programmatic stream serialization may start while its predecessor drains.
 * It reads only data its predecessor does not write until pdl_wait() returns
 * (the predecessor grid has completed and its writes are visible), and calls
 * pdl_trigger() after its own wait so the next kernel can start prefetching.
 * Without the launch attribute both are no-ops. */
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" :::); }

/* lane k of a float4 with a runtime k (rare paths only) */
__device__ __forceinline__ float lane(const float4 &v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }
__device__ __forceinline__ void set_lane(float4 &v, int k, float x)
{
    if (k == 0) v.x = x; else if (k == 1) v.y = x; else if (k == 2) v.z = x; else v.w = x;
}

/* stored-step index s % mod (s >= 0); no division when the pass stores
 * every step (mod = NT > s), the case of full storage */
__device__ __forceinline__ long long store_idx(int s, int mod) { return s < mod ? s : s % mod; }

/* x / DH: when DH is a power of two the product with the exact reciprocal is
 * the same correctly rounded value, so P2 kernels multiply. */
template <bool P2>
__device__ __forceinline__ float div_dh(float x, const StepArgs &a) { return P2 ? x * a.inv_dh : x / a.dh; }

/*
 * Velocity half-step (update_v_PML.c:51-198 for FDORDER = FDO): per point
 *   sxy_x = sum_m hc[m] (sxy[i+m-1] - sxy[i-m]),  syy_y = sum_m hc[m] (syz[j+m-1] - syz[j-m])
 *   CPML strips: psi = b*psi + a*d;  d = d/K + psi   (full-grid profiles)
 *   vy += b*DT*(sxy_x+syy_y)/DH with b = 1/rho
 * followed, when the tile holds any, by the source injection of this step
 * (update_v_PML.c:564-583) and the receiver samples (seismo_ssg.c:17-27).
 * Thread = 4 x-consecutive points (i0 .. i0+3) of row j of shot slot `slot`;
 * `tile` = the 128 x 8-point tile of the injection / sampling lists holding
 * them, ((j-1)/8) * ceil(nx/128) + (i0-1)/128.
 * All global loads are issued before any store so their latencies overlap.
 */
/* Stress taps of the velocity update straight from global memory:
 * xs[p] = sxy[i0 - 4*NL + p] of row j, ys[r] = syz rows j-H .. j+H-1. */
template <bool CG = false>
struct GlobalTaps {
    template <int H, int NL, int NR>
    __device__ __forceinline__ void load(const StepArgs &a, long long so, long long hrow, int col0, int j, float *xs,
                                         float4 *ys) const
    {
        const float *row = a.sxy + so + hrow + col0 - 4 * NL;
#pragma unroll
        for (int v = 0; v < NL + 1 + NR; v++) {
            float4 t = lds4<CG>(row + 4 * v);
            xs[4 * v] = t.x; xs[4 * v + 1] = t.y; xs[4 * v + 2] = t.z; xs[4 * v + 3] = t.w;
        }
        const float *col = a.syz + so + (long long)(j - 1 + a.hy - H) * a.pitch + col0;
#pragma unroll
        for (int r = 0; r < 2 * H; r++) ys[r] = lds4<CG>(col + (long long)r * a.pitch);
    }
};

/* The same taps from a block's shared-memory staging (v_step_st): sx[ty][v]
 * = sxy row of thread row ty, float4 group v counted from the block's first
 * point minus 4*NL; sy[r][tx] = syz row j0-H+r at the thread's four points. */
struct SharedTaps {
    const float4 *sx, *sy;
    int sx_pitch, tx, ty;
    template <int H, int NL, int NR>
    __device__ __forceinline__ void load(const StepArgs &, long long, long long, int, int, float *xs,
                                         float4 *ys) const
    {
#pragma unroll
        for (int v = 0; v < NL + 1 + NR; v++) {
            const float4 t = sx[ty * sx_pitch + tx + v];
            xs[4 * v] = t.x; xs[4 * v + 1] = t.y; xs[4 * v + 2] = t.z; xs[4 * v + 3] = t.w;
        }
#pragma unroll
        for (int r = 0; r < 2 * H; r++) ys[r] = sy[(ty + r) * BX + tx];
    }
};

template <int FDO, int FLAGS, bool P2, class Taps = GlobalTaps<>, bool CG = false>
__device__ __forceinline__ void v_body(const StepArgs &a, int nt_off, int i0, int j, int slot, int tile,
                                       const Taps &taps = Taps())
{
    constexpr int H = FDO / 2;
    constexpr int NL = (H + 3) / 4;          /* float4s left of the own vector (needs H)   */
    constexpr int NR = (H - 1 + 3) / 4;      /* float4s right of the own vector (needs H-1) */
    constexpr int NXS = 4 * (NL + 1 + NR);
    if (i0 > a.nx || j > a.ny) return;
    const int nt = *a.nt_base + nt_off;
    const long long so = (long long)slot * a.slot_stride;
    const int pitch = a.pitch;
    const int col0 = i0 - 1 + HX;
    const long long hrow = (long long)(j - 1 + a.hy) * pitch;
    const long long drow = (long long)(j - 1) * pitch;

    /* ---- loads of data the preceding stress kernel does not write ---- */
    const float4 b4 = ldg4(a.brho + drow + col0);
    float4 vy4 = lds4<CG>(a.vy + so + hrow + col0);
    float4 g4, h4, f4;
    if (FLAGS & VF_CORR) g4 = ld4(a.grho + so + drow + col0);
    if (FLAGS & VF_HESS) h4 = ld4(a.hrho + so + drow + col0);
    int tg0 = 0, tg1 = 0, tr0 = 0, tr1 = 0;
    if (a.tl.on) {
        const int *go = a.tl.goff + (long long)slot * (a.tl.ntiles + 1) + tile;
        tg0 = __ldg(go); tg1 = __ldg(go + 1);
        if (a.tl.sample) {
            const int *ro = a.tl.roff + (long long)slot * (a.tl.ntiles + 1) + tile;
            tr0 = __ldg(ro); tr1 = __ldg(ro + 1);
        }
    }
    if (FLAGS & VF_CORR) {                   /* stored forward acceleration of step NT-nt+1 (the address
                                                clamped so that a step beyond the pass stays in range) */
        const long long k = store_idx(max(a.nt_total - nt, 0), a.fwd_mod);
        f4 = ldcs4(a.fwd + (long long)slot * a.fwd_slot_stride + k * a.fwd_step_stride + drow + col0);
    }
    pdl_wait();                              /* stresses of the previous step are complete */
    pdl_trigger();

    /* ---- stress taps (issued before the step test below: their addresses do not
       depend on the step, so they need not wait for the step counter) ---- */
    float xs[NXS];                           /* xs[p] = sxy[i0 - 4*NL + p] */
    float4 ys[2 * H];                        /* syz rows j-H .. j+H-1 */
    taps.template load<H, NL, NR>(a, so, hrow, col0, j, xs, ys);
    if (nt > a.nt_last) return;

    /* ---- compute ---- */
    float4 acc4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 old4 = vy4;
    const int nvalid = min(4, a.nx - i0 + 1);
    /* whether a CPML strip holds any of the four points (false for the whole
       warp almost everywhere: one branch instead of four tests per point) */
    const bool in_pml = a.fw > 0 && (i0 <= a.fw || i0 + 3 >= a.nx - a.fw + 1 || (!a.free_surf && j <= a.fw) ||
                                     j >= a.ny - a.fw + 1);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int i = i0 + k;
        float sxy_x, syy_y;
#pragma unroll
        for (int m = 1; m <= H; m++) {
            const int my = (FDO == 12 && m == 6 && a.fd12_compat) ? 5 : m;
            float tx = a.hc[m] * (xs[4 * NL + k + m - 1] - xs[4 * NL + k - m]);
            float ty = a.hc[my] * (get(ys[H + m - 1], k) - get(ys[H - m], k));
            if (m == 1) { sxy_x = tx; syy_y = ty; }
            else { sxy_x = sxy_x + tx; syy_y = syy_y + ty; }
        }
        const int fw = a.fw;
        if (in_pml && i <= a.nx) {
            if (i <= fw) {
                float *p = a.psi_vxx + so + (long long)(j - 1) * 2 * fw + (i - 1);
                float ps = __ldg(a.pml.b_x + i) * *p + __ldg(a.pml.a_x + i) * sxy_x;
                *p = ps;
                sxy_x = sxy_x / __ldg(a.pml.K_x + i) + ps;
            }
            if (i >= a.nx - fw + 1) {
                const int h1 = i - a.nx + 2 * fw;
                float *p = a.psi_vxx + so + (long long)(j - 1) * 2 * fw + (h1 - 1);
                float ps = __ldg(a.pml.b_x + h1) * *p + __ldg(a.pml.a_x + h1) * sxy_x;
                *p = ps;
                sxy_x = sxy_x / __ldg(a.pml.K_x + h1) + ps;
            }
            if (!a.free_surf && j <= fw) {
                float *p = a.psi_vyy_v + so + (long long)(j - 1) * pitch + (col0 + k);
                float ps = __ldg(a.pml.b_y + j) * *p + __ldg(a.pml.a_y + j) * syy_y;
                *p = ps;
                syy_y = syy_y / __ldg(a.pml.K_y + j) + ps;
            }
            if (j >= a.ny - fw + 1) {
                const int h1 = j - a.ny + 2 * fw;
                float *p = a.psi_vyy_v + so + (long long)(h1 - 1) * pitch + (col0 + k);
                float ps = __ldg(a.pml.b_y + h1) * *p + __ldg(a.pml.a_y + h1) * syy_y;
                *p = ps;
                syy_y = syy_y / __ldg(a.pml.K_y + h1) + ps;
            }
        }
        const float b = get(b4, k);
        const float s = sxy_x + syy_y;
        if (!(FLAGS & VF_ADJOINT)) set(acc4, k, div_dh<P2>(b * s, a));
        set(vy4, k, get(vy4, k) + div_dh<P2>(b * a.dt * s, a));
    }

    /* ---- fused injection (sources in order per point) and sampling ---- */
    for (int g = tg0; g < tg1; g++) {
        const int pk = __ldg(a.tl.gpt + g);
        const int gi = pk & 0xffff, gj = pk >> 16;
        if (gj == j && gi >= i0 && gi < i0 + 4) {
            float v = lane(vy4, gi - i0);
            const float *sg = a.tl.sig + a.tl.sig_off[slot] + (long long)(nt - 1) * a.tl.sig_ts;
            for (int e = __ldg(a.tl.gbeg + g); e < __ldg(a.tl.gbeg + g + 1); e++)
                v = v + sg[(long long)__ldg(a.tl.src_id + e) * a.tl.sig_ss];
            set_lane(vy4, gi - i0, v);
        }
    }
    if (tr1 > tr0) {
        const int r0 = a.tl.rec_off[slot], ntr = a.tl.rec_off[slot + 1] - r0;
        float *sm = a.tl.seis + a.tl.seis_off[slot] + (long long)(nt - 1) * ntr;
        for (int e = tr0; e < tr1; e++) {
            const int pk = __ldg(a.tl.rpt + e);
            const int ri = pk & 0xffff, rj = pk >> 16;
            if (rj == j && ri >= i0 && ri < i0 + 4) sm[__ldg(a.tl.rid + e)] = lane(vy4, ri - i0);
        }
    }

    /* ---- stores ---- */
    st4m(a.vy + so + hrow + col0, vy4, nvalid);
    if (FLAGS & VF_ACC_OUT) st4m(a.out_acc + so + hrow + col0, (FLAGS & VF_ADJOINT) ? old4 : acc4, nvalid);
    if (FLAGS & VF_CORR) {          /* adjoint: g_rho += vyp1 * forward acceleration (denise.c:1589) */
        g4.x = g4.x + (old4.x * f4.x); g4.y = g4.y + (old4.y * f4.y);
        g4.z = g4.z + (old4.z * f4.z); g4.w = g4.w + (old4.w * f4.w);
        st4m(a.grho + so + drow + col0, g4, nvalid);
    }
    if (!(FLAGS & VF_ADJOINT) && a.fwd && !(FLAGS & VF_CORR)) {   /* forward storage of vyp1 */
        const long long k = store_idx(nt - 1, a.fwd_mod);
        st4ms(a.fwd + (long long)slot * a.fwd_slot_stride + k * a.fwd_step_stride + drow + col0, acc4, nvalid);
    }
    if ((FLAGS & VF_HESS) && nt < a.nt_total) {
        h4.x = h4.x + (acc4.x * acc4.x); h4.y = h4.y + (acc4.y * acc4.y);
        h4.z = h4.z + (acc4.z * acc4.z); h4.w = h4.w + (acc4.w * acc4.w);
        st4m(a.hrho + so + drow + col0, h4, nvalid);
    }
}

/* one thread block = 128 x blockDim.y points of one shot slot (grid z),
 * blockDim.y dividing the 8 rows of an injection / sampling list tile */
template <int FDO, int FLAGS, bool P2>
__global__ void __launch_bounds__(BX *BY, (FLAGS & (VF_CORR | VF_HESS)) ? VSTEP_MIN_BLOCKS : VSTEP_MIN_BLOCKS_FWD)
    v_step(StepArgs a, int nt_off)
{
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    v_body<FDO, FLAGS, P2>(a, nt_off, 1 + 4 * (blockIdx.x * BX + threadIdx.x), j, blockIdx.z,
                           ((j - 1) / BY) * gridDim.x + blockIdx.x);
}

/*
 * The velocity step for R vertically adjacent rows per thread (j0 .. j0+R-1,
 * the same 4 points in x): the syz column window of the rows overlaps, so R
 * rows need 2H+R-1 syz rows instead of 2H*R, and every load of all R rows is
 * issued before the first computation.  Per point the arithmetic, CPML,
 * injection, sampling and stores are those of v_body (bit-identical).  The
 * rows lie in one 128 x 8 tile of the injection / sampling lists.
 */
template <int FDO, int FLAGS, bool P2, int R>
__device__ __forceinline__ void v_body_rows(const StepArgs &a, int nt_off, int i0, int j0, int slot)
{
    constexpr int H = FDO / 2;
    constexpr int NL = (H + 3) / 4;
    constexpr int NR = (H - 1 + 3) / 4;
    constexpr int NXS = 4 * (NL + 1 + NR);
    if (i0 > a.nx || j0 > a.ny) return;
    const int nt = *a.nt_base + nt_off;
    const long long so = (long long)slot * a.slot_stride;
    const int pitch = a.pitch;
    const int col0 = i0 - 1 + HX;
    const int tile = ((j0 - 1) / BY) * a.tl.ntx + (i0 - 1) / (4 * BX);
    const int nrows = min(R, a.ny - j0 + 1);

    /* ---- loads of data the preceding stress kernel does not write ---- */
    float4 b4[R], vy4[R], g4[R], h4[R], f4[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        if (r < nrows) {
            const long long drow = (long long)(j0 + r - 1) * pitch;
            b4[r] = ldg4(a.brho + drow + col0);
            vy4[r] = ld4(a.vy + so + (long long)(j0 + r - 1 + a.hy) * pitch + col0);
            if (FLAGS & VF_CORR) g4[r] = ld4(a.grho + so + drow + col0);
            if (FLAGS & VF_HESS) h4[r] = ld4(a.hrho + so + drow + col0);
        }
    }
    int tg0 = 0, tg1 = 0, tr0 = 0, tr1 = 0;
    if (a.tl.on) {
        const int *go = a.tl.goff + (long long)slot * (a.tl.ntiles + 1) + tile;
        tg0 = __ldg(go); tg1 = __ldg(go + 1);
        if (a.tl.sample) {
            const int *ro = a.tl.roff + (long long)slot * (a.tl.ntiles + 1) + tile;
            tr0 = __ldg(ro); tr1 = __ldg(ro + 1);
        }
    }
    if (nt > a.nt_last) return;
    if (FLAGS & VF_CORR) {
        const long long k = store_idx(a.nt_total - nt, a.fwd_mod);
        const float *fb = a.fwd + (long long)slot * a.fwd_slot_stride + k * a.fwd_step_stride + col0;
#pragma unroll
        for (int r = 0; r < R; r++)
            if (r < nrows) f4[r] = ldcs4(fb + (long long)(j0 + r - 1) * pitch);
    }
    pdl_wait();
    pdl_trigger();

    /* ---- stress taps: sxy of each row, the shared syz column window ---- */
    float xs[R][NXS];
    float4 ys[2 * H + R - 1];                /* syz rows j0-H .. j0+H+R-2 */
#pragma unroll
    for (int r = 0; r < R; r++) {
        if (r < nrows) {
            const float *row = a.sxy + so + (long long)(j0 + r - 1 + a.hy) * pitch + col0 - 4 * NL;
#pragma unroll
            for (int v = 0; v < NL + 1 + NR; v++) {
                const float4 t = ld4(row + 4 * v);
                xs[r][4 * v] = t.x; xs[r][4 * v + 1] = t.y; xs[r][4 * v + 2] = t.z; xs[r][4 * v + 3] = t.w;
            }
        }
    }
    {
        const float *col = a.syz + so + (long long)(j0 - 1 + a.hy - H) * pitch + col0;
#pragma unroll
        for (int q = 0; q < 2 * H + R - 1; q++)
            if (q < 2 * H + nrows - 1) ys[q] = ld4(col + (long long)q * pitch);
    }

    const int nvalid = min(4, a.nx - i0 + 1);
#pragma unroll
    for (int r = 0; r < R; r++) {
        if (r >= nrows) break;
        const int j = j0 + r;
        const long long hrow = (long long)(j - 1 + a.hy) * pitch;
        const long long drow = (long long)(j - 1) * pitch;
        float4 acc4 = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 old4 = vy4[r];
        const bool in_pml = a.fw > 0 && (i0 <= a.fw || i0 + 3 >= a.nx - a.fw + 1 || (!a.free_surf && j <= a.fw) ||
                                         j >= a.ny - a.fw + 1);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int i = i0 + k;
            float sxy_x, syy_y;
#pragma unroll
            for (int m = 1; m <= H; m++) {
                const int my = (FDO == 12 && m == 6 && a.fd12_compat) ? 5 : m;
                float tx = a.hc[m] * (xs[r][4 * NL + k + m - 1] - xs[r][4 * NL + k - m]);
                float ty = a.hc[my] * (get(ys[r + H + m - 1], k) - get(ys[r + H - m], k));
                if (m == 1) { sxy_x = tx; syy_y = ty; }
                else { sxy_x = sxy_x + tx; syy_y = syy_y + ty; }
            }
            const int fw = a.fw;
            if (in_pml && i <= a.nx) {
                if (i <= fw) {
                    float *p = a.psi_vxx + so + (long long)(j - 1) * 2 * fw + (i - 1);
                    float ps = __ldg(a.pml.b_x + i) * *p + __ldg(a.pml.a_x + i) * sxy_x;
                    *p = ps;
                    sxy_x = sxy_x / __ldg(a.pml.K_x + i) + ps;
                }
                if (i >= a.nx - fw + 1) {
                    const int h1 = i - a.nx + 2 * fw;
                    float *p = a.psi_vxx + so + (long long)(j - 1) * 2 * fw + (h1 - 1);
                    float ps = __ldg(a.pml.b_x + h1) * *p + __ldg(a.pml.a_x + h1) * sxy_x;
                    *p = ps;
                    sxy_x = sxy_x / __ldg(a.pml.K_x + h1) + ps;
                }
                if (!a.free_surf && j <= fw) {
                    float *p = a.psi_vyy_v + so + (long long)(j - 1) * pitch + (col0 + k);
                    float ps = __ldg(a.pml.b_y + j) * *p + __ldg(a.pml.a_y + j) * syy_y;
                    *p = ps;
                    syy_y = syy_y / __ldg(a.pml.K_y + j) + ps;
                }
                if (j >= a.ny - fw + 1) {
                    const int h1 = j - a.ny + 2 * fw;
                    float *p = a.psi_vyy_v + so + (long long)(h1 - 1) * pitch + (col0 + k);
                    float ps = __ldg(a.pml.b_y + h1) * *p + __ldg(a.pml.a_y + h1) * syy_y;
                    *p = ps;
                    syy_y = syy_y / __ldg(a.pml.K_y + h1) + ps;
                }
            }
            const float b = get(b4[r], k);
            const float s = sxy_x + syy_y;
            if (!(FLAGS & VF_ADJOINT)) set(acc4, k, div_dh<P2>(b * s, a));
            set(vy4[r], k, get(vy4[r], k) + div_dh<P2>(b * a.dt * s, a));
        }

        for (int g = tg0; g < tg1; g++) {
            const int pk = __ldg(a.tl.gpt + g);
            const int gi = pk & 0xffff, gj = pk >> 16;
            if (gj == j && gi >= i0 && gi < i0 + 4) {
                float v = lane(vy4[r], gi - i0);
                const float *sg = a.tl.sig + a.tl.sig_off[slot] + (long long)(nt - 1) * a.tl.sig_ts;
                for (int e = __ldg(a.tl.gbeg + g); e < __ldg(a.tl.gbeg + g + 1); e++)
                    v = v + sg[(long long)__ldg(a.tl.src_id + e) * a.tl.sig_ss];
                set_lane(vy4[r], gi - i0, v);
            }
        }
        if (tr1 > tr0) {
            const int r0 = a.tl.rec_off[slot], ntr = a.tl.rec_off[slot + 1] - r0;
            float *sm = a.tl.seis + a.tl.seis_off[slot] + (long long)(nt - 1) * ntr;
            for (int e = tr0; e < tr1; e++) {
                const int pk = __ldg(a.tl.rpt + e);
                const int ri = pk & 0xffff, rj = pk >> 16;
                if (rj == j && ri >= i0 && ri < i0 + 4) sm[__ldg(a.tl.rid + e)] = lane(vy4[r], ri - i0);
            }
        }

        st4m(a.vy + so + hrow + col0, vy4[r], nvalid);
        if (FLAGS & VF_ACC_OUT) st4m(a.out_acc + so + hrow + col0, (FLAGS & VF_ADJOINT) ? old4 : acc4, nvalid);
        if (FLAGS & VF_CORR) {
            float4 g = g4[r];
            const float4 f = f4[r];
            g.x = g.x + (old4.x * f.x); g.y = g.y + (old4.y * f.y);
            g.z = g.z + (old4.z * f.z); g.w = g.w + (old4.w * f.w);
            st4m(a.grho + so + drow + col0, g, nvalid);
        }
        if (!(FLAGS & VF_ADJOINT) && a.fwd && !(FLAGS & VF_CORR)) {
            const long long k = store_idx(nt - 1, a.fwd_mod);
            st4ms(a.fwd + (long long)slot * a.fwd_slot_stride + k * a.fwd_step_stride + drow + col0, acc4, nvalid);
        }
        if ((FLAGS & VF_HESS) && nt < a.nt_total) {
            float4 h = h4[r];
            h.x = h.x + (acc4.x * acc4.x); h.y = h.y + (acc4.y * acc4.y);
            h.z = h.z + (acc4.z * acc4.z); h.w = h.w + (acc4.w * acc4.w);
            st4m(a.hrho + so + drow + col0, h, nvalid);
        }
    }
}

/* R rows per thread: a block of 32 x (8/R) threads covers a 128 x 8 tile */
#ifndef VSTEP_R2_MIN_BLOCKS
#define VSTEP_R2_MIN_BLOCKS 5
#endif
template <int FDO, int FLAGS, bool P2>
__global__ void __launch_bounds__(BX *BY / 2, VSTEP_R2_MIN_BLOCKS) v_step_r2(StepArgs a, int nt_off)
{
    v_body_rows<FDO, FLAGS, P2, 2>(a, nt_off, 1 + 4 * (blockIdx.x * BX + threadIdx.x),
                                   1 + blockIdx.y * BY + 2 * threadIdx.y, blockIdx.z);
}

/* The velocity step with the block's stress taps staged in shared memory
 * first: 8 sxy rows of 128 + 4*(NL+NR) points and 8+2H-1 syz rows of 128
 * points, loaded once per block (about 3 float4 loads per thread instead of
 * NL+1+NR+2H), then read by every thread of the block. */
template <int FDO, int FLAGS, bool P2>
__global__ void __launch_bounds__(BX *BY, 3) v_step_st(StepArgs a, int nt_off)
{
    constexpr int H = FDO / 2;
    constexpr int NL = (H + 3) / 4, NR = (H - 1 + 3) / 4;
    constexpr int SXP = BX + NL + NR;                 /* float4 groups per staged sxy row */
    constexpr int SYR = BY + 2 * H - 1;               /* staged syz rows */
    __shared__ float4 sx[BY * SXP];
    __shared__ float4 sy[SYR * BX];
    const int nt = *a.nt_base + nt_off;
    if (nt > a.nt_last) return;
    const int tid = threadIdx.y * BX + threadIdx.x;
    const int slot = blockIdx.z;
    const long long so = (long long)slot * a.slot_stride;
    const int j0 = 1 + blockIdx.y * BY;
    const int cb = 4 * blockIdx.x * BX + HX;          /* column of the block's first point */
    const int rows_total = a.ny + 2 * a.hy;
    pdl_wait();                                       /* stresses of the previous step are complete */
    for (int idx = tid; idx < BY * SXP; idx += BX * BY) {
        const int r = idx / SXP, v = idx % SXP;
        const int row = j0 + r - 1 + a.hy, col = cb - 4 * NL + 4 * v;
        sx[idx] = (row < rows_total && col + 3 < a.pitch) ? ld4(a.sxy + so + (long long)row * a.pitch + col)
                                                         : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    for (int idx = tid; idx < SYR * BX; idx += BX * BY) {
        const int r = idx / BX, v = idx % BX;
        const int row = j0 - H + r - 1 + a.hy, col = cb + 4 * v;
        sy[idx] = (row < rows_total && col + 3 < a.pitch) ? ld4(a.syz + so + (long long)row * a.pitch + col)
                                                         : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    SharedTaps taps{sx, sy, SXP, (int)threadIdx.x, (int)threadIdx.y};
    v_body<FDO, FLAGS, P2>(a, nt_off, 1 + 4 * (blockIdx.x * BX + threadIdx.x), 1 + blockIdx.y * BY + threadIdx.y,
                           slot, blockIdx.y * gridDim.x + blockIdx.x, taps);
}

/*
 * Stress half-step with CPML and, for L > 0, L standard-linear-solid memory
 * variables (update_s_elastic_PML.c:104-158, update_s_visc_PML.c:131-209):
 *   vyx = (sum_m hc[m] (vy[i+m]-vy[i-m+1])) * dhi,   vyy likewise in depth
 *   CPML on the half grid (the viscoelastic top strip uses full-grid profiles)
 *   elastic: sxy += uip*vyx, syz += ujp*vyy  (dhi = DT/DH)
 *   visc:    sxy += fipjp*vyx + DT/2*sum r;  r_l = bip_l (r_l cip_l - dip_l vyx);
 *            sxy += DT/2*sum r_new (same for syz / q)   (dhi = 1/DH)
 * All loads (taps, stresses, memory variables, coefficients, accumulators)
 * are issued before the first store.
 */
template <int FDO, int L, int FLAGS, bool CG = false>
__device__ __forceinline__ void s_body(const StepArgs &a, int nt_off, int i0, int j, int slot)
{
    constexpr int H = FDO / 2;
    constexpr int NL = (H - 1 + 3) / 4;      /* needs vy[i0-(H-1)] */
    constexpr int NR = (H + 3) / 4;          /* needs vy[i0+3+H]   */
    constexpr int NXS = 4 * (NL + 1 + NR);
    constexpr int LL = L > 0 ? L : 1;
    if (i0 > a.nx || j > a.ny) return;
    const int nt = *a.nt_base + nt_off;
    const long long so = (long long)slot * a.slot_stride;
    const int pitch = a.pitch;
    const int col0 = i0 - 1 + HX;
    const long long hrow = (long long)(j - 1 + a.hy) * pitch;
    const long long drow = (long long)(j - 1) * pitch;
    const int nvalid = min(4, a.nx - i0 + 1);

    /* ---- loads of data the preceding velocity kernel does not write ---- */
    float *sxy_p = a.sxy + so + hrow + col0;
    float *syz_p = a.syz + so + hrow + col0;
    float4 sxy4 = lds4<CG>(sxy_p), syz4 = lds4<CG>(syz_p);
    float4 c1, c2;                           /* uip/ujp (elastic) or fipjp/f (visc) */
    float4 rr[LL], qq[LL], dip4[LL], d4[LL];
    float4 mi4, mj4, ti4, tj4;               /* muip, mujp, tausipjp, taus */
    float4 sold_r, sold_q, qsx, qsy;         /* Qs gradient: memory sums before the update, sensitivities */
    float4 ex4, ey4, gx4, gy4, dsx4, dsy4;   /* Qs gradient, adjoint: strains, sums, stored sensitivities */
    const uint64_t pol_rq = DSH_L2_POL(a, 1), pol_f = DSH_L2_POL(a, 2);   /* memory variables, model factors */
    if (L == 0) {
        c1 = ldg4p(a.uip + drow + col0, pol_f);
        c2 = ldg4p(a.ujp + drow + col0, pol_f);
    } else {
#pragma unroll
        for (int l = 0; l < L; l++) {
            rr[l] = ld4p(a.r + so + l * a.dstride + drow + col0, pol_rq);
            qq[l] = ld4p(a.q + so + l * a.dstride + drow + col0, pol_rq);
        }
        if (FLAGS & SF_PARAMS) {
            c1 = ldg4p(a.fipjp + drow + col0, pol_f);
            c2 = ldg4p(a.f + drow + col0, pol_f);
#pragma unroll
            for (int l = 0; l < L; l++) {
                dip4[l] = ldg4p(a.dip + l * a.dstride + drow + col0, pol_f);
                d4[l] = ldg4p(a.d + l * a.dstride + drow + col0, pol_f);
            }
        } else {
            mi4 = ldg4p(a.muip + drow + col0, pol_f);
            mj4 = ldg4p(a.mujp + drow + col0, pol_f);
            ti4 = ldg4p(a.tausipjp + drow + col0, pol_f);
            tj4 = ldg4p(a.taus + drow + col0, pol_f);
        }
    }
    float4 w4, g4, h4, fy, fu;
    if (a.ws) w4 = ld4(a.ws + so + drow + col0);
    if (FLAGS & SF_CORR) g4 = ld4(a.gu + so + drow + col0);
    if (FLAGS & SF_HESS) h4 = ld4(a.hu + so + drow + col0);
    if (FLAGS & SF_CORR) {                   /* (address clamped as in v_body) */
        const long long k = store_idx(max(a.nt_total - nt, 0), a.fwd_mod);
        const float *base = a.fwd + (long long)slot * a.fwd_slot_stride + k * a.fwd_step_stride + drow + col0;
        fy = ldcs4(base + a.dstride);
        fu = ldcs4(base + 2 * a.dstride);
        if (FLAGS & SF_CORRQ) {
            dsx4 = ldcs4(base + 3 * a.dstride);
            dsy4 = ldcs4(base + 4 * a.dstride);
        }
    }
    if (FLAGS & SF_CORRQ) {
        ex4 = ld4(a.exy + so + drow + col0);
        ey4 = ld4(a.eyz + so + drow + col0);
        gx4 = ld4(a.gqx + so + drow + col0);
        gy4 = ld4(a.gqy + so + drow + col0);
    }
    pdl_wait();                              /* velocities of this step are complete */
    pdl_trigger();

    /* ---- velocity taps ---- */
    float xs[NXS];
    {
        const float *row = a.vy + so + hrow + col0 - 4 * NL;
#pragma unroll
        for (int v = 0; v < NL + 1 + NR; v++) {
            float4 t = lds4<CG>(row + 4 * v);
            xs[4 * v] = t.x; xs[4 * v + 1] = t.y; xs[4 * v + 2] = t.z; xs[4 * v + 3] = t.w;
        }
    }
    float4 ys[2 * H];                        /* vy rows j-H+1 .. j+H */
    {
        const float *col = a.vy + so + (long long)(j - 1 + a.hy - H + 1) * pitch + col0;
#pragma unroll
        for (int r = 0; r < 2 * H; r++) ys[r] = lds4<CG>(col + (long long)r * pitch);
    }
    if (nt > a.nt_last) return;              /* after every load: none depends on the step test */

    /* ---- derivatives and CPML ---- */
    const float dhi = (L > 0) ? a.dhi_visc : a.dhi_el;
    const bool in_pml = a.fw > 0 && (i0 <= a.fw || i0 + 3 >= a.nx - a.fw + 1 || (!a.free_surf && j <= a.fw) ||
                                     j >= a.ny - a.fw + 1);
    float4 vyx4 = make_float4(0.f, 0.f, 0.f, 0.f), vyy4 = vyx4;
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

    /* ---- stress and memory-variable update ---- */
    if (L == 0) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            set(sxy4, k, get(sxy4, k) + get(c1, k) * get(vyx4, k));
            set(syz4, k, get(syz4, k) + get(c2, k) * get(vyy4, k));
        }
    } else {
        if (!(FLAGS & SF_PARAMS)) {
            /* fipjp = muip*DT*(1+L*tausipjp), f = mujp*DT*(1+L*taus) with the
               reference's float/double mix (prepare_update_s.c:46-47) */
#pragma unroll
            for (int k = 0; k < 4; k++) {
                set(c1, k, (float)((double)(get(mi4, k) * a.dt) * (1.0 + (double)(a.lf * get(ti4, k)))));
                set(c2, k, (float)((double)(get(mj4, k) * a.dt) * (1.0 + (double)(a.lf * get(tj4, k)))));
            }
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
        if (FLAGS & SF_QSENS) { sold_r = sumr4; sold_q = sumq4; }
        sumr4 = make_float4(0.f, 0.f, 0.f, 0.f);
        sumq4 = sumr4;
#pragma unroll
        for (int l = 0; l < L; l++) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                /* dip_l = muip*eta_l*tausipjp, d_l = mujp*eta_l*taus (prepare_update_s.c:54-55) */
                const float dipv = (FLAGS & SF_PARAMS) ? get(dip4[l], k) : (get(mi4, k) * a.eta[l]) * get(ti4, k);
                const float dv = (FLAGS & SF_PARAMS) ? get(d4[l], k) : (get(mj4, k) * a.eta[l]) * get(tj4, k);
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
        if (FLAGS & SF_QSENS) {
            /* d(stress increment)/d(tau) with the strain history held fixed:
               dfipjp/dtau = muip DT (L - sumu) / (1 + sumu tau), and every memory
               variable scales with its dip_l, whose log-derivative is
               1 / (tau (1 + sumu tau)) (prepare_update_s.c:40-55) */
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float tx = get(ti4, k), ty = get(tj4, k);
                const float denx = 1.0f + a.sumu * tx, deny = 1.0f + a.sumu * ty;
                const float ax = ((get(mi4, k) * a.dt) * (a.lf - a.sumu)) / denx;
                const float ay = ((get(mj4, k) * a.dt) * (a.lf - a.sumu)) / deny;
                const float kx = a.dthalbe / (tx * denx), ky = a.dthalbe / (ty * deny);
                set(qsx, k, (ax * get(vyx4, k)) + (kx * (get(sold_r, k) + get(sumr4, k))));
                set(qsy, k, (ay * get(vyy4, k)) + (ky * (get(sold_q, k) + get(sumq4, k))));
            }
        }
    }

    /* ---- stores ---- */
    st4m(sxy_p, sxy4, nvalid);
    st4m(syz_p, syz4, nvalid);
#pragma unroll
    for (int l = 0; l < L; l++) {
        st4mp(a.r + so + l * a.dstride + drow + col0, rr[l], nvalid, pol_rq);
        st4mp(a.q + so + l * a.dstride + drow + col0, qq[l], nvalid, pol_rq);
    }
    /* a non-finite value never turns finite again in these updates, so a
       check every few steps and on the last one finds every instability */
    if (((nt & a.chk_mask) == 0 || nt >= a.nt_last) &&
        !(isfinite(sxy4.x) && isfinite(sxy4.y) && isfinite(sxy4.z) && isfinite(sxy4.w) && isfinite(syz4.x) &&
          isfinite(syz4.y) && isfinite(syz4.z) && isfinite(syz4.w) && isfinite(xs[4 * NL])))
        atomicOr(a.status, 1);
    if (FLAGS & SF_STRAIN_OUT) {
        if (a.out_uy) {               /* compat fields */
            st4m(a.out_uy + so + hrow + col0, vyy4, nvalid);
            st4m(a.out_uyx + so + hrow + col0, vyx4, nvalid);
        } else {                      /* forward storage: uy at +dstride, uyx at +2*dstride */
            const long long k = store_idx(nt - 1, a.fwd_mod);
            float *base = a.fwd + (long long)slot * a.fwd_slot_stride + k * a.fwd_step_stride + drow + col0;
            st4ms(base + a.dstride, vyy4, nvalid);
            st4ms(base + 2 * a.dstride, vyx4, nvalid);
            if ((FLAGS & SF_QSENS) && L > 0) {
                st4ms(base + 3 * a.dstride, qsx, nvalid);
                st4ms(base + 4 * a.dstride, qsy, nvalid);
            }
        }
    }
    if (a.ws) {                       /* energy W += vy^2 (eprecond.c:11); vy at the point is xs[4NL+k] */
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float v = xs[4 * NL + k];
            set(w4, k, get(w4, k) + v * v);
        }
        st4m(a.ws + so + drow + col0, w4, nvalid);
    }
    if (FLAGS & SF_CORR) {            /* g_u += uyx_fwd*sxy + uy_fwd*syz (denise.c:1609) */
#pragma unroll
        for (int kk = 0; kk < 4; kk++)
            set(g4, kk, get(g4, kk) + ((get(fu, kk) * get(sxy4, kk)) + (get(fy, kk) * get(syz4, kk))));
        st4m(a.gu + so + drow + col0, g4, nvalid);
    }
    if (FLAGS & SF_CORRQ) {           /* Qs gradient: adjoint strain of the earlier adjoint steps times the
                                         stored sensitivity of forward step NT-nt+1, then this step's strain */
#pragma unroll
        for (int k = 0; k < 4; k++) {
            set(gx4, k, get(gx4, k) + (get(ex4, k) * get(dsx4, k)));
            set(gy4, k, get(gy4, k) + (get(ey4, k) * get(dsy4, k)));
            set(ex4, k, get(ex4, k) + (get(vyx4, k) * a.dt));
            set(ey4, k, get(ey4, k) + (get(vyy4, k) * a.dt));
        }
        st4m(a.gqx + so + drow + col0, gx4, nvalid);
        st4m(a.gqy + so + drow + col0, gy4, nvalid);
        st4m(a.exy + so + drow + col0, ex4, nvalid);
        st4m(a.eyz + so + drow + col0, ey4, nvalid);
    }
    if ((FLAGS & SF_HESS) && nt < a.nt_total) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float eyy = get(vyy4, k), eyx = 0.5f * get(vyx4, k);
            set(h4, k, get(h4, k) + ((eyy * eyy) + (eyx * eyx)));
        }
        st4m(a.hu + so + drow + col0, h4, nvalid);
    }
}

/* one thread block = 128 x blockDim.y points of one shot slot (grid z);
 * blockDim.y = 8, 4 or 2 (a shorter block lifetime shortens the last,
 * partly idle wave of a launch) */
template <int FDO, int L, int FLAGS>
__global__ void __launch_bounds__(BX *BY, SSTEP_MIN_BLOCKS) s_step(StepArgs a, int nt_off)
{
    s_body<FDO, L, FLAGS>(a, nt_off, 1 + 4 * (blockIdx.x * BX + threadIdx.x), 1 + blockIdx.y * blockDim.y + threadIdx.y,
                          blockIdx.z);
}

/* Source injection then receiver sampling for one step, one block per slot
 * (update_v_PML.c:564-583, seismo_ssg.c:17-27).  Sources at the same grid
 * point are grouped so their additions keep the reference's order. */
struct InjectArgs {
    const int *nt_base;
    int nt_last;
    int nt_total;
    long long slot_stride;
    float *vy;
    /* per slot s: groups [grp_off[s], grp_off[s+1]) with point offset grp_pt[g]
       and source ids src_id[grp_beg[g] .. grp_beg[g+1]) */
    const int *grp_off, *grp_pt, *grp_beg, *src_id;
    const float *sig;             /* signal of source id sid at step nt: sig[sig_off[s] + sid*sig_ss + (nt-1)*sig_ts] */
    const long long *sig_off;
    long long sig_ss, sig_ts;
    int reverse_time;             /* unused (the adjoint signal is stored time-reversed) */
    /* receivers: slot s has rec_n[s] receivers at rec_pt[rec_off[s] + r] */
    const int *rec_off, *rec_pt;
    float *seis;                  /* slot s: seis[seis_off[s] + (nt-1)*ntr_s + r] */
    const long long *seis_off;
    int sample;
};

static __global__ void inject_sample(InjectArgs a, int nt_off)
{
    const int nt = *a.nt_base + nt_off;
    if (nt > a.nt_last) return;
    const int s = blockIdx.x;
    float *vy = a.vy + (long long)s * a.slot_stride;
    const int g0 = a.grp_off[s], g1 = a.grp_off[s + 1];
    for (int g = g0 + threadIdx.x; g < g1; g += blockDim.x) {
        const int pt = a.grp_pt[g];
        float v = vy[pt];
        for (int e = a.grp_beg[g]; e < a.grp_beg[g + 1]; e++)
            v = v + a.sig[a.sig_off[s] + (long long)a.src_id[e] * a.sig_ss + (long long)(nt - 1) * a.sig_ts];
        vy[pt] = v;
    }
    if (!a.sample) return;
    __syncthreads();
    const int r0 = a.rec_off[s], r1 = a.rec_off[s + 1], ntr = r1 - r0;
    float *seis = a.seis + a.seis_off[s] + (long long)(nt - 1) * ntr;
    for (int r = threadIdx.x; r < ntr; r += blockDim.x) seis[r] = vy[a.rec_pt[r0 + r]];
}

/* advance the device step counter of a captured chunk */
static __global__ void advance_step(int *nt_base, int by) { *nt_base += by; }

}  // namespace dsh

/*
 * dsh_setup.h — host-side coefficient generation (plain C, FP32 with the
 * reference's float/double mixture so every coefficient is bit-identical to
 * the one the reference's CPU code computes).
 */
#ifndef DSH_SETUP_H
#define DSH_SETUP_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DSH_MAX_FW 256
#define DSH_MAX_L 4

/* CPML profile vectors, index 1..2*fw (entry 0 unused). */
typedef struct dsh_pml {
    float K_x[2 * DSH_MAX_FW + 1], a_x[2 * DSH_MAX_FW + 1], b_x[2 * DSH_MAX_FW + 1];
    float K_x_half[2 * DSH_MAX_FW + 1], a_x_half[2 * DSH_MAX_FW + 1], b_x_half[2 * DSH_MAX_FW + 1];
    float K_y[2 * DSH_MAX_FW + 1], a_y[2 * DSH_MAX_FW + 1], b_y[2 * DSH_MAX_FW + 1];
    float K_y_half[2 * DSH_MAX_FW + 1], a_y_half[2 * DSH_MAX_FW + 1], b_y_half[2 * DSH_MAX_FW + 1];
    float d_x[2 * DSH_MAX_FW + 1], d_x_half[2 * DSH_MAX_FW + 1], d_y[2 * DSH_MAX_FW + 1], d_y_half[2 * DSH_MAX_FW + 1];
} dsh_pml;

/* Staggered-grid operator hc[1..6] (hc[0] = minimum points per wavelength). */
int dsh_setup_holberg(int fdorder, int maxrelerror, float hc[7]);

/* C-PML profiles for an nx x ny grid (src/PML_pro.c:65-295). */
void dsh_setup_pml(int nx, int ny, int fw, float dh, float dt, float damping, float fpml, float npower,
                   float k_max_pml, dsh_pml *out);

/* Model-dependent coefficients for dense [ny][nx] inputs.  Outputs (dense
 * [ny][nx] unless noted; pass NULL for what is not needed):
 *   brho  1/rho as the velocity update forms it (0 where rho < 1e-20)
 *   uip, ujp  harmonic shear-modulus averages with the periodic one-rank halo
 *   for l > 0: fipjp, f, dip [l][ny][nx], d [l][ny][nx], bip/bjm/cip/cjm [l]
 *   cnorm[2]  C_vs, C_rho */
int dsh_setup_model(int nx, int ny, int l, const float *fl, float dt, const float *vs, const float *rho,
                    const float *qs, float *brho, float *uip, float *ujp, float *fipjp, float *f, float *dip,
                    float *d, float *bip, float *bjm, float *cip, float *cjm, float *cnorm);

/* C_vs, C_rho: the means of vs and rho as float sums in the reference's loop
 * order (x outer, depth inner), as dsh_setup_model forms cnorm */
void dsh_setup_cnorm(int nx, int ny, const float *vs, const float *rho, float *cnorm);

/* The per-mechanism scalars of dsh_setup_model / dsh_setup_visc_base for
 * l >= 1 relaxation mechanisms: eta_l = DT/tau_l (readmod.c:30-33) and the
 * memory-variable factors bip, bjm, cip, cjm (prepare_update_s.c:52-55);
 * NULL outputs are skipped. */
int dsh_setup_sls(int l, const float *fl, float dt, float *eta, float *bip, float *bjm, float *cip, float *cjm);

/* sum_l w^2 tau_l^2 / (1 + w^2 tau_l^2), w = 2 pi FL[1] (prepare_update_s.c:24-32), as
 * dsh_setup_visc_base forms it */
float dsh_setup_sumu(int l, const float *fl);
/* The per-point factors from which every viscoelastic coefficient is a
 * product (src/prepare_update_s.c:43-57): relaxed moduli muip/mujp at the
 * two stress positions, tau at (i+1/2, j+1/2) and (i, j+1/2) (av_tau), and
 * eta_l = DT/tau_l.  fipjp = muip*DT*(1+L*tausipjp), f = mujp*DT*(1+L*taus),
 * dip_l = muip*eta_l*tausipjp, d_l = mujp*eta_l*taus are formed from them. */
int dsh_setup_visc_base(int nx, int ny, int l, const float *fl, float dt, const float *vs, const float *rho,
                        const float *qs, float *muip, float *mujp, float *tausipjp, float *taus, float *eta);

/* Source time functions (src/wavelet.c:26-84): out [nsrc][nt]. */
int dsh_setup_wavelet(int quellart, int nt, float dt, int nsrc, const float *srcpos8, float *out);

/* SPATFILTER=3 Gaussian gradient smoothing (src/gauss_filt.c): odd filter
 * length round(WD_DAMP*(C_vs/FC_END)/DH), and its normalised kernel [n][n],
 * n = 2*(|filt|/2)+1 (row jj, column ii). */
int dsh_setup_gauss_size(float wd_damp, float c_vs, float fc_end, float dh);
int dsh_setup_gauss_kernel(int filt, float *kernel);

/* SPATFILTER=4 spatially variable Gaussian smoothing (src/gauss_filt_var.c):
 * per-point kernel index and the distinct kernels' weights and sums. */
int dsh_setup_gauss_var(int nx, int ny, float dh, float wd_damp, float wd_damp1, float fc_end, const float *vel,
                        int *map, int max_pairs, int *pairs, int max_weights, float *weights);

/* Butterworth low-/highpass sections of timedomain_filt.c (libcseife):
 * returns the number of sections written to coef [n][5] = f0 f1 f2 g1 g2. */
int dsh_setup_butterworth(double dt, float fc, int order, int highpass, double *coef);

/* Circular source taper box of src/taper_grad.c:298-351 and
 * src/taper_grad_shot.c:47-96: size g (>= 5) and centre ijc in grid points,
 * and, when m is not NULL, the normalised box values m [g][g] (row iy-1,
 * column ix-1). */
int dsh_setup_taper_box(int srtshape, float srtradius, float dh, int *g, int *ijc, float *m);
/* For one source at grid point (i1, j1): the minimum of the source's
 * min-combined mask over the grid and the maximum after subtracting it
 * (src/taper_grad_shot.c:126-140); the coefficient at a point is then
 * (min(1, box value or 1) - minm) / maxm. */
void dsh_setup_taper_norm(int nx, int ny, int g, int ijc, const float *m, int i1, int j1, float *minm, float *maxm);

/* Largest stable DT of the staggered scheme (src/checkfd_ssg_elastic.c):
 * DH / (sqrt(2) * sum|hc| * vmax). */
double dsh_setup_dt_limit(int fdorder, int maxrelerror, float dh, float vmax);

#ifdef __cplusplus
}
#endif
#endif

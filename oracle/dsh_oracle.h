/*
 * dsh_oracle.h — TEST ORACLE ONLY (CPU restatement of the DENISE-SH hot path).
 *
 * A plain-C restatement, written for this repository, of the reference's SH
 * time-stepping path for one MPI rank: coefficients (holbergcoeff, PML_pro,
 * av_mue with the one-rank periodic model wrap of matcopy, av_tau,
 * prepare_update_s, wavelet), the velocity/stress updates with CPML and SLS
 * memory variables, source injection, receiver sampling, forward storage,
 * residual, adjoint back-propagation with gradient correlation, energy
 * preconditioning, gradient conversion and the pseudo-Hessian diagonal.
 *
 * The time stepping is compiled twice: in FP32 (bit-identical to the reference
 * built with -ffp-contract=off, checked by the test suite) and in FP64 (used to
 * state FP32 errors against a double-precision run with the same coefficients).
 * Only tests/, the smoke check and the CPU-baseline leg of bench.py use this.
 *
 * Array conventions match oracle/ref_harness.c: dense row-major [NY][NX] for
 * grid fields, [ntr][NT] for traces, [8][nsrc] for source tables (rows: grid x,
 * grid y, 0, tshift, fc, amp, angle, type), [2][ntr] for receiver grid indices.
 */
#ifndef DSH_ORACLE_H
#define DSH_ORACLE_H

typedef struct {
    int nx, ny, nt, fdorder, maxrelerror, fw, free_surf, l, quellart, eprecond;
    float dh, dt, damping, fpml, npower, k_max_pml;
    float fl[8];
} dsho_params;

int dsho_init(const dsho_params *p, const float *vs, const float *rho, const float *qs, int fp64);
void dsho_free(void);
void dsho_set_fd12_compat(int on);
/* misfit norm of dsho_residual (calc_res.c LNORM 1..5, GRAD_FORM=2); dsho_init resets it to 2 */
int dsho_set_lnorm(int lnorm);
void dsho_get_hc(float *out7);
void dsho_get_cnorm(float *out2);
int dsho_get_pml(int which, float *out);
void dsho_get_sls(float *bip, float *bjm, float *cip, float *cjm);
int dsho_get_field(int which, float *out);
int dsho_get_field_f64(int which, double *out);
int dsho_get_psi(int which, float *out);
int dsho_wavelet(int nsrc, const float *srcpos8, float *out);
int dsho_forward(int nsrc, const float *srcpos8, const float *signals, int ntr, const int *recpos,
                 int nsteps, int store, int hessian, float *seis);
int dsho_forward_f64(int nsrc, const float *srcpos8, const float *signals, int ntr, const int *recpos,
                     int nsteps, int store, int hessian, double *seis);
int dsho_residual(const float *obs, float *res, double *l2);
int dsho_adjoint(const float *adj, int nsteps);
int dsho_eprecond_scale(void);
int dsho_convert(const float *wu, const float *wrho, float *g_vs, float *g_rho);
int dsho_hessian_out(float *h_vs, float *h_rho);
/* Qs gradient (no counterpart in the reference): set before dsho_init, read
 * after the adjoint of one shot (dJ/dQs, J = sum res^2, double [NY][NX]) */
void dsho_set_grad_q(int on);
int dsho_get_grad_q(double *g_qs);
int dsho_psource(int nt, float *sxx, float *syy, int nsrc, const float *srcpos8, const float *signals);

/* SPATFILTER=3 gradient smoothing (src/gauss_filt.c) */
int dsho_gauss_filter_size(float wd_damp, float c_vs, float fc_end, float dh);
int dsho_gauss_kernel(int filt, float *kernel);
int dsho_gauss_filt(int nx, int ny, int filt, const float *in, float *out);
#endif

/*
 * dsh_compat.h — the reference's hot-path functions with their own names and
 * signatures, implemented by libdsh_compat.so on the GPU (velocity/stress
 * updates, energy accumulation) or with the reference's arithmetic on the
 * host (bookkeeping).  A program that defines the reference's global
 * parameters (src/globvar.h: DT, DH, NX, NY, FDORDER, FW, FREE_SURF, L, ...)
 * links this library in place of the corresponding reference objects.
 * Supported: NPROCX = NPROCY = 1, BOUNDARY = 0, GRAD_FORM = 2, full-grid
 * ranges (1..NX, 1..NY), L <= 4.  Arrays are the reference's Numerical-Recipes
 * row-pointer arrays (float **m, m[j][i]; float ***t, t[j][i][l]).
 */
#ifndef DSH_COMPAT_H
#define DSH_COMPAT_H

#ifdef __cplusplus
extern "C" {
#endif

/* replaces src/update_v_PML.c:12-16 (velocity half-step, CPML, injection; writes QUELLTYP) */
void update_v_PML(int nx1, int nx2, int ny1, int ny2, int nt, float **vy, float **vyp1, float **vym1, float **utty,
                  float **syz, float **sxy, float **rho, float **srcpos_loc, float **signals1, int nsrc,
                  float **absorb_coeff, float *hc, int infoout, int sw, float *K_x, float *a_x, float *b_x,
                  float *K_x_half, float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                  float *K_y_half, float *a_y_half, float *b_y_half, float **psi_syy_y, float **psi_sxy_x);

/* replaces src/update_s_elastic_PML.c:12-16 */
void update_s_elastic_PML(int nx1, int nx2, int ny1, int ny2, float **vy, float **uy, float **uyx, float **syz,
                          float **sxy, float **u, float **uip, float **ujp, float **absorb_coeff, float **rho,
                          float *hc, int infoout, float *K_x, float *a_x, float *b_x, float *K_x_half,
                          float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y, float *K_y_half,
                          float *a_y_half, float *b_y_half, float **psi_vyy, float **psi_vyx);

/* replaces src/update_s_visc_PML.c:12-17 */
void update_s_visc_PML(int nx1, int nx2, int ny1, int ny2, float **vy, float **uy, float **uyx, float **syz,
                       float **sxy, float **ujp, float **uip, float **rho, float *hc, int infoout, float ***r,
                       float ***p, float ***q, float **fipjp, float **f, float **g, float *bip, float *bjm,
                       float *cip, float *cjm, float ***d, float ***e, float ***dip, float *K_x, float *a_x,
                       float *b_x, float *K_x_half, float *a_x_half, float *b_x_half, float *K_y, float *a_y,
                       float *b_y, float *K_y_half, float *a_y_half, float *b_y_half, float **psi_vyy,
                       float **psi_vyx);

/* replaces src/seismo_ssg.c:9 */
void seismo_ssg(int lsamp, int ntr, int **recpos, float **sectionvy, float **vy, float **syy, float **u, float *hc);

/* replaces src/eprecond.c:2 */
void eprecond(float **W, float **vy);

/* replaces src/eprecond1.c:2 (the one-rank maximum; the reference's MPI_Allreduce of it is the identity) */
void eprecond1(float **We, float **Ws, float **Wr);

/* replaces src/hess_save.c:2 */
void hess_save(int nt, float **uy, float **uyx, float **vyp1, float ***hess_eyy, float ***hess_eyx,
               float ***hess_utty);

/* replaces src/hessian.c:9 */
void hessian(int NTDTINV, float ***hess_eyy, float ***hess_eyx, float ***hess_utty, float **hessian_u,
             float **hessian_rho);

/* replace src/zero_fdveps.c:11 and src/zero_fdveps_visc.c:11 */
void zero_fdveps(int ny1, int ny2, int nx1, int nx2, float **vy, float **syy, float **sxy, float **vym1,
                 float **vyp1, float **psi_sxy_x, float **psi_vyx, float **psi_syy_y, float **psi_vyy);
void zero_fdveps_visc(int ny1, int ny2, int nx1, int nx2, float **vy, float **syy, float **sxy, float **vym1,
                      float **vyp1, float **psi_sxy_x, float **psi_vyx, float **psi_syy_y, float **psi_vyy,
                      float ***pr, float ***pp, float ***pq);

/* replaces src/psource.c:9 (P-SV explosive source; not used by the SH program) */
void psource(int nt, float **sxx, float **syy, float **srcpos_loc, float **signals, int nsrc);

/* Errors of the functions above, which keep the reference's void
 * signatures: the first error code (dsh.h's DSH_ERR_*) since the previous
 * call, then cleared — DSH_ERR_UNSTABLE when a stress or velocity update left
 * a non-finite value, DSH_ERR_PARAM for an unsupported configuration,
 * DSH_ERR_CUDA / DSH_ERR_OOM for device failures.  Each error is also
 * printed.  With DSH_COMPAT_ABORT=1 in the environment an error ends the
 * run the way the reference's err() does (src/util.c:7-15: the rank and the
 * message on stdout, then a non-zero exit), as the reference does for its
 * own fatal errors (src/denise.c:1183-1185 for an unstable simulation).
 * No counterpart in the reference. */
int dsh_compat_status(void);

#ifdef __cplusplus
}
#endif
#endif

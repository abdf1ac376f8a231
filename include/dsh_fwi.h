/*
 * dsh_fwi.h — host-side optimisation steps of the FWI loop, in plain C as in
 * the reference (which keeps L-BFGS and the line search on the host):
 *   dsh_lbfgs_direction   two-loop recursion (src/LBFGS.c:12-95), with the
 *                         pairs of model and gradient differences stored as
 *                         src/store_LBFGS_SH.c does (gradient x C_vs,
 *                         model / C_vs)
 *   dsh_pcg_direction     conjugate-gradient direction update per
 *                         parameter class (src/PCG.c:10-107)
 *   dsh_opt_step          step length from three test misfits: the extremum
 *                         of the parabola through them with the reference's
 *                         guards (src/calc_opt_step.c:20-111)
 *   dsh_line_search_next  one decision of the reference's bracketing loop
 *                         (src/line_search.c:316-360)
 */
#ifndef DSH_FWI_H
#define DSH_FWI_H

#ifdef __cplusplus
extern "C" {
#endif

/* r = H q for the stored pairs: S, Y hold `count` pairs [count][n], oldest
 * first; gamma = (y.s)/(y.y) of the newest pair scales the initial inverse
 * Hessian; rho_k = 1/(y_k.s_k), or 0 when y_k.s_k = 0.  count = 0 gives r = q.
 * Dot products in double. */
int dsh_lbfgs_direction(long long n, int count, const float *S, const float *Y, const float *q, float *r);

/* The reference's own L-BFGS step (src/LBFGS.c:12-107) on its ring buffers:
 * y and s hold nlbfgs slots of nvec values (slot k, 1-based, at
 * (k-1)*nvec), the newest pair in slot `pointer`; q is the preconditioned
 * gradient vector (overwritten, as the reference overwrites q_LBFGS) and r
 * receives H q.  As the reference: nothing is done for iter <= 1; gamma from
 * slot `pointer`; the two loops run over the slots in slot order (k = nlbfgs
 * .. 1, then 1 .. nlbfgs) whatever their age, empty slots included (their
 * rho is 0); every dot product is a float sum in index order (src/dotp.c). */
int dsh_lbfgs_ring(int iter, const float *y, const float *s, float *q, float *r, int pointer, int nlbfgs,
                   long long nvec);

/* Median smoothing of the updated model (MODEL_FILTER=1, src/smooth_model.c,
 * called at src/denise.c:1948, with the median of src/median.c): each point
 * of vs and rho [ny][nx] becomes the median of its window of side |FILT_SIZE|
 * (an even FILT_SIZE grows by one away from 0, as the reference does),
 * edges replicated; the window values are taken depth offset outer, x offset
 * inner, and the median is element (k+1)/2 of their ascending order, ties in
 * that order.  filt_size = 0 copies the fields.  Writes *filt_size_used
 * (optional): the reference keeps the grown size in FILT_SIZE. */
int dsh_smooth_model_median(int nx, int ny, int filt_size, const float *vs, const float *rho, float *vs_out,
                            float *rho_out, int *filt_size_used);

/* Conjugate-gradient direction (src/PCG.c:10-107, called at
 * src/denise.c:1850-1871 on the steepest-descent directions of vs and rho):
 * the vectors hold nclass parameter classes of n values each, class after
 * class, in the caller's point order (the reference stores each class x-major,
 * src/store_PCG_SH.c).  Per class, beta = num/den from float sums taken in
 * vector order, 0 when den = 0:
 *   beta_kind 1 Fletcher-Reeves   num = g_new.g_new          den = g_old.g_old
 *             2 Polak-Ribiere     num = g_new.(g_new-g_old)  den = g_old.g_old,
 *                                 beta < 0 reset to 0 (the reference's setting,
 *                                 PCG_BETA = 2 at src/PCG.c:17)
 *             3 Hestenes-Stiefel  num = -g_new.(g_new-g_old) den = dir.(g_new-g_old)
 *             4 Dai-Yuan          num = -g_new.g_new         den = dir.(g_new-g_old)
 * then dir = g_new + beta*dir in place.  beta_out (nclass floats) may be NULL.
 * Returns 0, or -1 for invalid arguments (nclass outside 1..DSH_PCG_MAX_CLASSES). */
#define DSH_PCG_MAX_CLASSES 8
int dsh_pcg_direction(long long n, int nclass, const float *g_new, const float *g_old, float *dir, int beta_kind,
                      float *beta_out);

/* Device versions of dsh_lbfgs_direction and dsh_pcg_direction (no
 * counterpart in the reference, whose optimiser runs on the host): every
 * vector is a device array, the work runs on `stream` (a cudaStream_t as
 * void*, NULL = the default stream) and nothing is allocated or copied to the
 * host.  Same steps as the host functions; each dot product is a double sum
 * over a fixed partition of the vector (296 blocks, then a fixed tree), so
 * results are reproducible and agree with the host versions to float
 * rounding.  work: dsh_vec_work_doubles(count) doubles of device memory that
 * the call owns until its stream reaches the end of it (count = the L-BFGS
 * pairs; also enough for any nclass of the PCG step).  The PCG betas go to
 * beta_dev (nclass floats on the device) or, when NULL, stay in work.
 * Returns DSH_ERR_PARAM for invalid arguments, DSH_ERR_CUDA when a launch fails. */
long long dsh_vec_work_doubles(int count);
int dsh_lbfgs_direction_device(long long n, int count, const float *S, const float *Y, const float *q, float *r,
                               double *work, void *stream);
int dsh_pcg_direction_device(long long n, int nclass, const float *g_new, const float *g_old, float *dir,
                             int beta_kind, float *beta_dev, double *work, void *stream);

/* epst[0..2], L2t[0..2]: test step lengths (epst[0] = 0) and their misfits */
float dsh_opt_step(const float L2t[3], const float epst[3]);
/* The same step as src/calc_opt_step.c:20-111 computes it, bit for bit: the
 * 3 x 3 system [1, eps, eps^2] x = L2 solved by the reference's float Gauss
 * elimination without pivoting (src/solvelin.c:9-60); a singular system gives
 * what the reference gives (a non-finite step).  dsh_opt_step (used by
 * dsh_line_search_next) solves in double and guards the singular case. */
float dsh_opt_step_ref(const float L2t[3], const float epst[3]);

/* Line-search state of src/line_search.c: feed the misfits of the steps the
 * previous call asked for; returns 1 while another test forward is needed
 * (its relative step length in *eps_scale and its slot, 1 or 2, in *slot),
 * 0 when done (*eps_scale = the chosen step) and -1 when no step reduced the
 * misfit within stepmax tries (*eps_scale = 0). */
typedef struct dsh_line_search {
    float epst[3], L2t[3];
    float eps_scale, scalefac;
    int step1, step2, countstep, stepmax, slot;
} dsh_line_search;
void dsh_line_search_init(dsh_line_search *ls, float L2_now, float eps_scale, float scalefac, int stepmax);
int dsh_line_search_next(dsh_line_search *ls, float L2_test, float *eps_scale, int *slot);

/* Misfit and data energy of the FWI loop's reported objective and of the
 * line search's test shots (called at src/denise.c:1423-1425 and in
 * src/line_search.c), over traces [ntr][ns] (row-major, sample 1 first), with
 * the reference's float accumulation; trace killing (TRKILL) is not built.
 *   dsh_calc_misfit (src/calc_misfit.c:7-100, itest = 0, sws = 1,
 *   swstestshot = 1): LNORM 2 and 6 add, per trace, the squared running
 *   integral of syn - obs times DT^2; LNORM 5 subtracts, per trace, the
 *   normalised correlation of the running integrals of obs and syn; other
 *   LNORMs add nothing.  The sum starts from l2_in (the running total the
 *   reference passes in).
 *   dsh_calc_energy (src/calc_energy.c:7-65): adds the squared running
 *   integral of obs times DT^2 to energy_in.
 * The L2 misfit the reference reports is L2 / energy for LNORM=2
 * (src/denise.c:1719-1723). */
double dsh_calc_misfit(const float *obs, const float *syn, int ntr, int ns, int lnorm, float dt, float l2_in);

/* Model update along the search direction (src/calc_mat_change_test.c:9-170,
 * INVMAT1=1), on dense [ny][nx] fields: eps_u = eps_scale * max(vs)/max|d_vs|
 * and eps_rho = eps_scale * max(rho)/max|d_rho| * SCALERHO (0 before
 * INV_VS_ITER / INV_RHO_ITER), vs_new = vs - eps_u d_vs, rho_new = rho -
 * eps_rho d_rho, then the reference's bounds in its order: a new vs below
 * VSLOWERLIM (but above 1e-6) or above VSUPPERLIM keeps the old value, a new
 * rho outside [RHOLOWERLIM, RHOUPPERLIM] keeps the old value, before the
 * INV_*_ITER iterations the old values are kept, negative values keep the old
 * ones.  Returns eps_u (the reference's eps_true); *eps_rho (optional) gets
 * eps_rho.  limits = {VSLOWERLIM, VSUPPERLIM, RHOLOWERLIM, RHOUPPERLIM}. */
float dsh_model_update(int nx, int ny, const float *vs, const float *rho, const float *d_vs, const float *d_rho,
                       float eps_scale, float scalerho, int iter, int inv_vs_iter, int inv_rho_iter,
                       const float limits[4], float *vs_new, float *rho_new, float *eps_rho);
double dsh_calc_energy(const float *obs, int ntr, int ns, float dt, float energy_in);
/* Relative model change sum (u - u0)^2 / sum u0^2 over dense [ny][nx]
 * fields, float sums in the reference's order (src/calc_mres.c:7-25; the FWI
 * loop reports it for vs and rho against the starting model,
 * src/denise.c:1733-1738). */
float dsh_calc_mres(int nx, int ny, const float *u, const float *u0);

#ifdef __cplusplus
}
#endif
#endif

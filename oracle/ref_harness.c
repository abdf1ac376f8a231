/*
 * ref_harness.c — TEST ORACLE ONLY.
 *
 * Drives the reference's own compiled CPU functions (update_v_PML,
 * update_s_elastic_PML, update_s_visc_PML, seismo_ssg, eprecond, eprecond1,
 * hess_save, hessian, matcopy, av_mue, av_tau, prepare_update_s, PML_pro,
 * holbergcoeff, wavelet, calc_res, zero_fdveps*) through the same per-shot
 * time loops that the reference's main program runs for one MPI rank
 * (NPROCX=NPROCY=1).  The reference sources are compiled in place by
 * oracle/Makefile into oracle/_ref/; nothing here is linked into the product.
 *
 * The loop bodies restated here follow:
 *   forward loop         src/denise.c:1179-1346
 *   residual             src/denise.c:1364-1428 (calc_res with LNORM=2)
 *   adjoint loop         src/denise.c:1452-1654 (correlation :1580-1625)
 *   eprecond scaling     src/denise.c:1665-1678
 *   shot summation       src/denise.c:1689-1694
 *   gradient conversion  src/denise.c:1743-1813 (INVMAT=0, INVMAT1=1)
 *   normalisers C_vs/C_rho  src/denise.c:778-816
 *   Hessian output conversion src/hessian_out.c:20-31 (file output omitted)
 * All arrays crossing this API are dense row-major [NY][NX] (index j*NX+i for
 * grid point (i+1, j+1)); seismograms are [ntr][NT].
 */
#include "fd.h"

/* reference globals referenced here (defined by the reference's globvar.h) */
extern float DT, DH, DAMPING, FPML, *FL, TIME;
extern int NX, NY, NXG, NYG, NT, FDORDER, MAXRELERROR, FW, FREE_SURF, BOUNDARY, L;
extern int IDX, IDY, NPROCX, NPROCY, MYID, POS[3], INDEX[5], INVMAT1, INVMAT, GRAD_FORM;
extern int QUELLART, QUELLTYP, QUELLTYPB, EPRECOND, DTINV, SEISMO, NDT, HESSIAN;
extern int IENDX, IENDY, NP, NPROC;
extern int TRKILL, TIMEWIN, RTM, OFFSET_MUTE, NORMALIZE;
extern float npower, k_max_PML, C_vs, C_rho;
extern FILE *FP;

typedef struct {
    int nx, ny, nt, fdorder, maxrelerror, fw, free_surf, l, quellart, eprecond;
    float dh, dt, damping, fpml, npower, k_max_pml;
    float fl[8];
} refh_params;

/* Implementation switch (tests of a reference-signature replacement):
 * the loops below call these pointers; NULL restores the reference's own. */
typedef void (*fn_v_t)(int, int, int, int, int, float **, float **, float **, float **, float **, float **, float **,
                       float **, float **, int, float **, float *, int, int, float *, float *, float *, float *,
                       float *, float *, float *, float *, float *, float *, float *, float *, float **, float **);
typedef void (*fn_se_t)(int, int, int, int, float **, float **, float **, float **, float **, float **, float **,
                        float **, float **, float **, float *, int, float *, float *, float *, float *, float *,
                        float *, float *, float *, float *, float *, float *, float *, float **, float **);
typedef void (*fn_sv_t)(int, int, int, int, float **, float **, float **, float **, float **, float **, float **,
                        float **, float *, int, float ***, float ***, float ***, float **, float **, float **,
                        float *, float *, float *, float *, float ***, float ***, float ***, float *, float *,
                        float *, float *, float *, float *, float *, float *, float *, float *, float *, float *,
                        float **, float **);
typedef void (*fn_ep_t)(float **, float **);
typedef void (*fn_ep1_t)(float **, float **, float **);
static fn_v_t impl_v = NULL;
static fn_se_t impl_se = NULL;
static fn_sv_t impl_sv = NULL;
static fn_ep_t impl_ep = NULL;
static fn_ep1_t impl_ep1 = NULL;
static int cur_lnorm = 2;         /* LNORM of refh_residual (refh_set_lnorm; reset by refh_init) */

void refh_set_impl(void *v, void *s_el, void *s_visc, void *ep, void *ep1)
{
    impl_v = (fn_v_t)v;
    impl_se = (fn_se_t)s_el;
    impl_sv = (fn_sv_t)s_visc;
    impl_ep = (fn_ep_t)ep;
    impl_ep1 = (fn_ep1_t)ep1;
}
/* The same for the bookkeeping functions of the loops (seismo_ssg,
 * hess_save, hessian, zero_fdveps, zero_fdveps_visc) and psource. */
typedef void (*fn_seis_t)(int, int, int **, float **, float **, float **, float **, float *);
typedef void (*fn_hsave_t)(int, float **, float **, float **, float ***, float ***, float ***);
typedef void (*fn_hess_t)(int, float ***, float ***, float ***, float **, float **);
typedef void (*fn_zero_t)(int, int, int, int, float **, float **, float **, float **, float **, float **, float **,
                          float **, float **);
typedef void (*fn_zerov_t)(int, int, int, int, float **, float **, float **, float **, float **, float **, float **,
                           float **, float **, float ***, float ***, float ***);
typedef void (*fn_psrc_t)(int, float **, float **, float **, float **, int);
void psource(int nt, float **sxx, float **syy, float **srcpos_loc, float **signals, int nsrc);   /* src/psource.c:9; fd.h has no prototype */
static fn_seis_t impl_seis = NULL;
static fn_hsave_t impl_hsave = NULL;
static fn_hess_t impl_hess = NULL;
static fn_zero_t impl_zero = NULL;
static fn_zerov_t impl_zerov = NULL;
static fn_psrc_t impl_psrc = NULL;

void refh_set_impl_aux(void *seis, void *hsave, void *hess, void *zero, void *zerov, void *psrc)
{
    impl_seis = (fn_seis_t)seis;
    impl_hsave = (fn_hsave_t)hsave;
    impl_hess = (fn_hess_t)hess;
    impl_zero = (fn_zero_t)zero;
    impl_zerov = (fn_zerov_t)zerov;
    impl_psrc = (fn_psrc_t)psrc;
}
#define CALL_SEIS (impl_seis ? impl_seis : seismo_ssg)
#define CALL_HSAVE (impl_hsave ? impl_hsave : hess_save)
#define CALL_HESS (impl_hess ? impl_hess : hessian)
#define CALL_ZERO (impl_zero ? impl_zero : zero_fdveps)
#define CALL_ZEROV (impl_zerov ? impl_zerov : zero_fdveps_visc)
#define CALL_PSRC (impl_psrc ? impl_psrc : psource)

#define CALL_V (impl_v ? impl_v : update_v_PML)
#define CALL_SE (impl_se ? impl_se : update_s_elastic_PML)
#define CALL_SV (impl_sv ? impl_sv : update_s_visc_PML)
#define CALL_EP (impl_ep ? impl_ep : eprecond)
#define CALL_EP1 (impl_ep1 ? impl_ep1 : eprecond1)

static int nd;
static float **pvy, **psxy, **psyz, **pvyp1, **pvym1, **uy, **uyx, **utty;
static float **prho, **pu, **puip, **pujp, **absorb_coeff;
static float ***pr, ***pp, ***pq, ***dip, ***d, ***e;
static float **ptaus, **ptausipjp, **fipjp, **f, **g;
static float *peta, *etaip, *etajm, *bip, *bjm, *cip, *cjm;
static float *hc;
static float *d_x, *K_x, *alpha_prime_x, *a_x, *b_x, *d_x_half, *K_x_half, *alpha_prime_x_half, *a_x_half, *b_x_half;
static float *d_y, *K_y, *alpha_prime_y, *a_y, *b_y, *d_y_half, *K_y_half, *alpha_prime_y_half, *a_y_half, *b_y_half;
static float **psi_syz_y, **psi_sxy_x, **psi_vyy, **psi_vyx;
static float **Ws, **Wr, **We, **g_u_shot, **g_rho_shot, **hessian_u, **hessian_rho;
static float *fwd_rho_y, *fwd_y, *fwd_u;         /* forward_prop_* of denise.c:467-478 */
static float ***hess_eyy, ***hess_eyx, ***hess_utty;
static int fwd_stored = 0, hess_alloc = 0, alive = 0;
static int cur_ntr = 0;
static int **recpos_loc = NULL;
static float **sectionvy = NULL, **sectionvydiff = NULL, **sectionvydata = NULL, **sectionvydiffold = NULL;

static void harness_free_shot(void)
{
    if (recpos_loc) { free_imatrix(recpos_loc, 1, 3, 1, cur_ntr); recpos_loc = NULL; }
    if (sectionvy) { free_matrix(sectionvy, 1, cur_ntr, 1, NT); sectionvy = NULL; }
    if (sectionvydiff) { free_matrix(sectionvydiff, 1, cur_ntr, 1, NT); sectionvydiff = NULL; }
    if (sectionvydata) { free_matrix(sectionvydata, 1, cur_ntr, 1, NT); sectionvydata = NULL; }
    if (sectionvydiffold) { free_matrix(sectionvydiffold, 1, cur_ntr, 1, NT); sectionvydiffold = NULL; }
    cur_ntr = 0;
}

void refh_free(void)
{
    if (!alive) return;
    harness_free_shot();
    free_matrix(pvy, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(psxy, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(psyz, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(pvyp1, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(pvym1, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(uy, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(uyx, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(utty, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(prho, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(pu, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(puip, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(pujp, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(absorb_coeff, 1, NY, 1, NX);
    free_matrix(Ws, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(Wr, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(We, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(g_u_shot, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(g_rho_shot, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(hessian_u, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(hessian_rho, -nd + 1, NY + nd, -nd + 1, NX + nd);
    if (L) {
        free_f3tensor(pr, -nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        free_f3tensor(pp, -nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        free_f3tensor(pq, -nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        free_f3tensor(dip, -nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        free_f3tensor(d, -nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        free_f3tensor(e, -nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        free_matrix(ptaus, -nd + 1, NY + nd, -nd + 1, NX + nd);
        free_matrix(ptausipjp, -nd + 1, NY + nd, -nd + 1, NX + nd);
        free_matrix(fipjp, -nd + 1, NY + nd, -nd + 1, NX + nd);
        free_matrix(f, -nd + 1, NY + nd, -nd + 1, NX + nd);
        free_matrix(g, -nd + 1, NY + nd, -nd + 1, NX + nd);
        free_vector(peta, 1, L); free_vector(etaip, 1, L); free_vector(etajm, 1, L);
        free_vector(bip, 1, L); free_vector(bjm, 1, L); free_vector(cip, 1, L); free_vector(cjm, 1, L);
        free_vector(FL, 1, L);
    }
    free_vector(hc, 0, 6);
    if (FW > 0) {
        free_vector(d_x, 1, 2 * FW); free_vector(K_x, 1, 2 * FW); free_vector(alpha_prime_x, 1, 2 * FW);
        free_vector(a_x, 1, 2 * FW); free_vector(b_x, 1, 2 * FW);
        free_vector(d_x_half, 1, 2 * FW); free_vector(K_x_half, 1, 2 * FW); free_vector(alpha_prime_x_half, 1, 2 * FW);
        free_vector(a_x_half, 1, 2 * FW); free_vector(b_x_half, 1, 2 * FW);
        free_vector(d_y, 1, 2 * FW); free_vector(K_y, 1, 2 * FW); free_vector(alpha_prime_y, 1, 2 * FW);
        free_vector(a_y, 1, 2 * FW); free_vector(b_y, 1, 2 * FW);
        free_vector(d_y_half, 1, 2 * FW); free_vector(K_y_half, 1, 2 * FW); free_vector(alpha_prime_y_half, 1, 2 * FW);
        free_vector(a_y_half, 1, 2 * FW); free_vector(b_y_half, 1, 2 * FW);
        free_matrix(psi_syz_y, 1, 2 * FW, 1, NX);
        free_matrix(psi_sxy_x, 1, NY, 1, 2 * FW);
        free_matrix(psi_vyy, 1, 2 * FW, 1, NX);
        free_matrix(psi_vyx, 1, NY, 1, 2 * FW);
    }
    if (fwd_stored) {
        free_vector(fwd_rho_y, 1, NX * NY * NT);
        free_vector(fwd_y, 1, NX * NY * NT);
        free_vector(fwd_u, 1, NX * NY * NT);
        fwd_stored = 0;
    }
    if (hess_alloc) {
        free_f3tensor(hess_eyy, 1, NY, 1, NX, 1, NT);
        free_f3tensor(hess_eyx, 1, NY, 1, NX, 1, NT);
        free_f3tensor(hess_utty, 1, NY, 1, NX, 1, NT);
        hess_alloc = 0;
    }
    alive = 0;
}

/* Sets the reference globals for one rank and builds every coefficient the
 * time loop consumes, in the order of denise.c:598-627 and :726-743. */
int refh_init(const refh_params *p, const float *vs, const float *rho, const float *qs)
{
    int i, j, l;
    refh_free();
    cur_lnorm = 2;
    FP = stderr;
    NX = NXG = p->nx; NY = NYG = p->ny; NT = p->nt;
    FDORDER = p->fdorder; MAXRELERROR = p->maxrelerror; FW = p->fw; FREE_SURF = p->free_surf;
    L = p->l; QUELLART = p->quellart; EPRECOND = p->eprecond;
    DH = p->dh; DT = p->dt; DAMPING = p->damping; FPML = p->fpml; npower = p->npower; k_max_PML = p->k_max_pml;
    TIME = NT * DT;
    BOUNDARY = 0; IDX = IDY = 1; NPROCX = NPROCY = 1; NP = NPROC = 1; MYID = 0;
    POS[1] = POS[2] = 0; INDEX[1] = INDEX[2] = INDEX[3] = INDEX[4] = 0;
    IENDX = NX; IENDY = NY;
    INVMAT1 = 1; INVMAT = 0; GRAD_FORM = 2; QUELLTYPB = 2; DTINV = 1; SEISMO = 1; NDT = 1; HESSIAN = 0;
    TRKILL = 0; TIMEWIN = 0; RTM = 0; OFFSET_MUTE = 0; NORMALIZE = 0;
    if (L > 0) {
        FL = vector(1, L);
        for (l = 1; l <= L; l++) FL[l] = p->fl[l - 1];
    }
    nd = FDORDER / 2 + 1;

    pvy = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    psxy = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    psyz = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    pvyp1 = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    pvym1 = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    uy = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    uyx = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    utty = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    prho = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    pu = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    puip = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    pujp = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    absorb_coeff = matrix(1, NY, 1, NX);
    Ws = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    Wr = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    We = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    g_u_shot = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    g_rho_shot = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    hessian_u = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    hessian_rho = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    if (L) {
        pr = f3tensor(-nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        pp = f3tensor(-nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        pq = f3tensor(-nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        dip = f3tensor(-nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        d = f3tensor(-nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        e = f3tensor(-nd + 1, NY + nd, -nd + 1, NX + nd, 1, L);
        ptaus = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
        ptausipjp = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
        fipjp = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
        f = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
        g = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
        peta = vector(1, L); etaip = vector(1, L); etajm = vector(1, L);
        bip = vector(1, L); bjm = vector(1, L); cip = vector(1, L); cjm = vector(1, L);
    }
    /* CPML arrays: denise.c:528-555 */
    if (FW > 0) {
        d_x = vector(1, 2 * FW); K_x = vector(1, 2 * FW); alpha_prime_x = vector(1, 2 * FW);
        a_x = vector(1, 2 * FW); b_x = vector(1, 2 * FW);
        d_x_half = vector(1, 2 * FW); K_x_half = vector(1, 2 * FW); alpha_prime_x_half = vector(1, 2 * FW);
        a_x_half = vector(1, 2 * FW); b_x_half = vector(1, 2 * FW);
        d_y = vector(1, 2 * FW); K_y = vector(1, 2 * FW); alpha_prime_y = vector(1, 2 * FW);
        a_y = vector(1, 2 * FW); b_y = vector(1, 2 * FW);
        d_y_half = vector(1, 2 * FW); K_y_half = vector(1, 2 * FW); alpha_prime_y_half = vector(1, 2 * FW);
        a_y_half = vector(1, 2 * FW); b_y_half = vector(1, 2 * FW);
        psi_syz_y = matrix(1, 2 * FW, 1, NX);
        psi_sxy_x = matrix(1, NY, 1, 2 * FW);
        psi_vyy = matrix(1, 2 * FW, 1, NX);
        psi_vyx = matrix(1, NY, 1, 2 * FW);
    }
    alive = 1;

    hc = holbergcoeff();                                  /* denise.c:598 */

    /* model: readmod.c:82-99 (u=vs, rho, taus=2/qs; eta=DT/pts) */
    for (j = 1; j <= NY; j++)
        for (i = 1; i <= NX; i++) {
            pu[j][i] = vs[(j - 1) * NX + (i - 1)];
            prho[j][i] = rho[(j - 1) * NX + (i - 1)];
            if (L) ptaus[j][i] = 2.0 / qs[(j - 1) * NX + (i - 1)];
        }
    if (L) {
        for (l = 1; l <= L; l++) {
            float pts = 1.0 / (2.0 * PI * FL[l]);
            peta[l] = DT / pts;
        }
    }

    if (FW > 0)                                           /* denise.c:626-627 */
        PML_pro(d_x, K_x, alpha_prime_x, a_x, b_x, d_x_half, K_x_half, alpha_prime_x_half, a_x_half, b_x_half,
                d_y, K_y, alpha_prime_y, a_y, b_y, d_y_half, K_y_half, alpha_prime_y_half, a_y_half, b_y_half);

    /* per-iteration preparation: denise.c:726-743 */
    if (L) matcopy(prho, pu, ptaus);
    else matcopy_elastic(prho, pu);
    av_mue(pu, puip, pujp, prho);
    if (L) av_tau(ptaus, ptausipjp);
    if (L) prepare_update_s(etajm, etaip, peta, fipjp, pujp, puip, prho, ptaus, ptausipjp, f, g, bip, bjm, cip, cjm, dip, d, e);

    /* normalisers: denise.c:778-816 (first iteration) */
    {
        float Vs_avg = 0.0, rho_avg = 0.0;
        int Lcount = 1;
        for (i = 1; i <= NX; i = i + IDX)
            for (j = 1; j <= NY; j = j + IDY) {
                Vs_avg += pu[j][i];
                rho_avg += prho[j][i];
                Lcount++;
            }
        Lcount--;
        Vs_avg /= Lcount;
        rho_avg /= Lcount;
        C_vs = Vs_avg;
        C_rho = rho_avg;
    }
    /* Hessian accumulators start at zero (matrix() zero-fills; denise.c:673-674) */
    return 0;
}

/* Coefficient export (for parity of the product's own host-side setup). */
void refh_get_hc(float *out7) { int i; for (i = 0; i <= 6; i++) out7[i] = hc[i]; }
void refh_get_cnorm(float *out2) { out2[0] = C_vs; out2[1] = C_rho; }

/* which: 0..9 = K_x a_x b_x K_x_half a_x_half b_x_half K_y a_y b_y K_y_half;
 * 10 a_y_half 11 b_y_half 12 d_x 13 d_x_half 14 d_y 15 d_y_half */
int refh_get_pml(int which, float *out)
{
    float *v[] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half,
                  d_x, d_x_half, d_y, d_y_half};
    int i;
    if (FW <= 0 || which < 0 || which > 15) return -1;
    for (i = 1; i <= 2 * FW; i++) out[i - 1] = v[which][i];
    return 0;
}

/* Dense [NY][NX] export of a grid field.
 * 0 vy 1 sxy 2 syz 3 vyp1 4 uy 5 uyx 6 uip 7 ujp 8 rho 9 u(vs) 10 fipjp 11 f
 * 12 Ws 13 Wr 14 We 15 g_u_shot 16 g_rho_shot 17 hessian_u 18 hessian_rho 19 taus 20 tausipjp
 * 100+l: r[.][.][l+1]; 200+l: q[.][.][l+1]; 300+l: dip[l+1]; 400+l: d[l+1] */
int refh_get_field(int which, float *out)
{
    float **m = NULL;
    float ***t = NULL;
    int i, j, l = 0;
    switch (which) {
    case 0: m = pvy; break;  case 1: m = psxy; break; case 2: m = psyz; break;
    case 3: m = pvyp1; break; case 4: m = uy; break; case 5: m = uyx; break;
    case 6: m = puip; break; case 7: m = pujp; break; case 8: m = prho; break;
    case 9: m = pu; break;
    case 10: m = L ? fipjp : NULL; break; case 11: m = L ? f : NULL; break;
    case 12: m = Ws; break; case 13: m = Wr; break; case 14: m = We; break;
    case 15: m = g_u_shot; break; case 16: m = g_rho_shot; break;
    case 17: m = hessian_u; break; case 18: m = hessian_rho; break;
    case 19: m = L ? ptaus : NULL; break; case 20: m = L ? ptausipjp : NULL; break;
    default:
        if (!L) return -1;
        l = which % 100 + 1;
        if (l > L) return -1;
        if (which >= 100 && which < 200) t = pr;
        else if (which >= 200 && which < 300) t = pq;
        else if (which >= 300 && which < 400) t = dip;
        else if (which >= 400 && which < 500) t = d;
        else return -1;
    }
    if (!m && !t) return -1;
    for (j = 1; j <= NY; j++)
        for (i = 1; i <= NX; i++)
            out[(j - 1) * NX + (i - 1)] = m ? m[j][i] : t[j][i][l];
    return 0;
}

void refh_get_sls(float *bip_o, float *bjm_o, float *cip_o, float *cjm_o)
{
    int l;
    for (l = 1; l <= L; l++) { bip_o[l - 1] = bip[l]; bjm_o[l - 1] = bjm[l]; cip_o[l - 1] = cip[l]; cjm_o[l - 1] = cjm[l]; }
}

/* psi export: 0 psi_sxy_x [NY][2FW], 1 psi_vyx [NY][2FW], 2 psi_syz_y [2FW][NX], 3 psi_vyy [2FW][NX] */
int refh_get_psi(int which, float *out)
{
    int i, j;
    if (FW <= 0) return -1;
    if (which == 0 || which == 1) {
        float **m = which == 0 ? psi_sxy_x : psi_vyx;
        for (j = 1; j <= NY; j++) for (i = 1; i <= 2 * FW; i++) out[(j - 1) * 2 * FW + i - 1] = m[j][i];
    } else if (which == 2 || which == 3) {
        float **m = which == 2 ? psi_syz_y : psi_vyy;
        for (j = 1; j <= 2 * FW; j++) for (i = 1; i <= NX; i++) out[(j - 1) * NX + i - 1] = m[j][i];
    } else return -1;
    return 0;
}

/* Ricker (or other QUELLART) wavelets through the reference's wavelet():
 * srcpos rows 4..6 = tshift, fc, amp (wavelet.c:33-45). out: [nsrc][NT] */
int refh_wavelet(int nsrc, const float *srcpos8, float *out)
{
    float **sp = matrix(1, 8, 1, nsrc);
    float **sig;
    int k, r, n;
    for (r = 1; r <= 8; r++) for (k = 1; k <= nsrc; k++) sp[r][k] = srcpos8[(r - 1) * nsrc + (k - 1)];
    sig = wavelet(sp, nsrc, 1);
    for (k = 1; k <= nsrc; k++) for (n = 1; n <= NT; n++) out[(k - 1) * NT + (n - 1)] = sig[k][n];
    free_matrix(sig, 1, nsrc, 1, NT);
    free_matrix(sp, 1, 8, 1, nsrc);
    return 0;
}

static void zero_state(void)
{
    if (L) CALL_ZEROV(-nd + 1, NY + nd, -nd + 1, NX + nd, pvy, psyz, psxy, uy, pvyp1,
                            psi_sxy_x, psi_vyx, psi_syz_y, psi_vyy, pr, pp, pq);
    else CALL_ZERO(-nd + 1, NY + nd, -nd + 1, NX + nd, pvy, psyz, psxy, uy, pvyp1,
                     psi_sxy_x, psi_vyx, psi_syz_y, psi_vyy);
}

static void step_stress(void)
{
    if (L)
        CALL_SV(1, NX, 1, NY, pvy, uy, uyx, psyz, psxy, pujp, puip, prho, hc, 0,
                          pr, pp, pq, fipjp, f, g, bip, bjm, cip, cjm, d, e, dip,
                          K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half,
                          psi_vyy, psi_vyx);
    else
        CALL_SE(1, NX, 1, NY, pvy, uy, uyx, psyz, psxy, pu, puip, pujp, absorb_coeff, prho, hc, 0,
                             K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half,
                             psi_vyy, psi_vyx);
}

/*
 * One shot forward: denise.c:1126-1346.
 *   srcpos8: [8][nsrc] rows as srcpos_loc (grid x, grid y, 0, tshift, fc, amp, angle, type)
 *   signals: [nsrc][NT] source time functions (or NULL -> reference wavelet())
 *   recpos:  [2][ntr] grid x, grid y
 *   nsteps:  number of steps to run (<= NT); store: keep forward_prop_* for the adjoint
 *   hessian: run hess_save each step and hessian() at the end (denise.c:1312-1315, :1350-1352)
 *   seis:    [ntr][NT] output (columns beyond nsteps stay 0)
 */
int refh_forward(int nsrc, const float *srcpos8, const float *signals_in, int ntr, const int *recpos,
                 int nsteps, int store, int hessian_on, float *seis)
{
    float **sp, **signals;
    int i, j, k, r, nt, hin, hin1, imat, imat1, imat2;
    if (!alive) return -1;
    if (nsteps > NT) nsteps = NT;
    harness_free_shot();
    cur_ntr = ntr;
    recpos_loc = imatrix(1, 3, 1, ntr > 0 ? ntr : 1);
    for (k = 1; k <= ntr; k++) {
        recpos_loc[1][k] = recpos[k - 1];
        recpos_loc[2][k] = recpos[ntr + k - 1];
        recpos_loc[3][k] = k;
    }
    sectionvy = matrix(1, ntr > 0 ? ntr : 1, 1, NT);
    cur_ntr = ntr > 0 ? ntr : 1;
    sp = matrix(1, 8, 1, nsrc);
    for (r = 1; r <= 8; r++) for (k = 1; k <= nsrc; k++) sp[r][k] = srcpos8[(r - 1) * nsrc + (k - 1)];
    if (signals_in) {
        signals = matrix(1, nsrc, 1, NT);
        for (k = 1; k <= nsrc; k++) for (nt = 1; nt <= NT; nt++) signals[k][nt] = signals_in[(k - 1) * NT + nt - 1];
    } else {
        signals = wavelet(sp, nsrc, 1);
    }

    zero_state();
    /* per-shot gradient / energy accumulators: denise.c:1138-1161 */
    for (i = 1; i <= NX; i++)
        for (j = 1; j <= NY; j++) {
            g_rho_shot[j][i] = 0.0; g_u_shot[j][i] = 0.0;
            Ws[j][i] = 0.0; Wr[j][i] = 0.0; We[j][i] = 0.0;
        }
    if (store && !fwd_stored) {
        fwd_rho_y = vector(1, NX * NY * NT);
        fwd_y = vector(1, NX * NY * NT);
        fwd_u = vector(1, NX * NY * NT);
        fwd_stored = 1;
    }
    if (hessian_on && !hess_alloc) {
        hess_eyy = f3tensor(1, NY, 1, NX, 1, NT);
        hess_eyx = f3tensor(1, NY, 1, NX, 1, NT);
        hess_utty = f3tensor(1, NY, 1, NX, 1, NT);
        hess_alloc = 1;
    }
    hin = 1; hin1 = 1; imat = 1; imat1 = 1; imat2 = 1;
    for (nt = 1; nt <= nsteps; nt++) {
        CALL_V(1, NX, 1, NY, nt, pvy, pvyp1, pvym1, utty, psyz, psxy, prho, sp, signals, nsrc, absorb_coeff,
                     hc, 0, 0, K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half,
                     b_y_half, psi_syz_y, psi_sxy_x);
        step_stress();
        if (ntr > 0) CALL_SEIS(nt, ntr, recpos_loc, sectionvy, pvy, psyz, pu, hc);
        if (nt == hin1) {
            if (store) {                                  /* denise.c:1261-1301 */
                for (i = 1; i <= NX; i++) for (j = 1; j <= NY; j++) fwd_rho_y[imat1++] = pvyp1[j][i];
                for (i = 1; i <= NX; i++) for (j = 1; j <= NY; j++) fwd_y[imat++] = uy[j][i];
                for (i = 1; i <= NX; i++) for (j = 1; j <= NY; j++) fwd_u[imat2++] = uyx[j][i];
            }
            if (hessian_on) CALL_HSAVE(hin, uy, uyx, pvyp1, hess_eyy, hess_eyx, hess_utty);
            if ((EPRECOND == 1) || (EPRECOND == 3)) CALL_EP(Ws, pvy);
            hin++;
            hin1 = hin1 + DTINV;
        }
    }
    if (hessian_on) CALL_HESS(nsteps, hess_eyy, hess_eyx, hess_utty, hessian_u, hessian_rho);
    for (k = 1; k <= ntr; k++) for (nt = 1; nt <= NT; nt++) seis[(k - 1) * NT + nt - 1] = sectionvy[k][nt];
    free_matrix(signals, 1, nsrc, 1, NT);
    free_matrix(sp, 1, 8, 1, nsrc);
    return 0;
}

/* Residual and misfit (calc_res.c, GRAD_FORM=2, LNORM from refh_set_lnorm,
 * default 2): obs [ntr][NT]; res out [ntr][NT] (time-reversed); the reference
 * also overwrites obs sample 1 with the synthetic one. */
int refh_set_lnorm(int lnorm)
{
    if (lnorm < 1 || lnorm > 5) return -1;
    cur_lnorm = lnorm;
    return 0;
}
int refh_residual(const float *obs, float *res, double *l2)
{
    int k, nt, ntr = cur_ntr;
    if (!sectionvy) return -1;
    sectionvydata = matrix(1, ntr, 1, NT);
    sectionvydiff = matrix(1, ntr, 1, NT);
    sectionvydiffold = matrix(1, ntr, 1, NT);
    for (k = 1; k <= ntr; k++) for (nt = 1; nt <= NT; nt++) sectionvydata[k][nt] = obs[(k - 1) * NT + nt - 1];
    {
        int **recpos_glob = recpos_loc;
        float **srcdummy = matrix(1, 8, 1, 1);
        *l2 = calc_res(sectionvydata, sectionvy, sectionvydiff, sectionvydiffold, ntr, NT, cur_lnorm, 0.0, 0, 1, 1, ntr,
                       recpos_glob, recpos_loc, srcdummy, 1, 1, 1);
        free_matrix(srcdummy, 1, 8, 1, 1);
    }
    for (k = 1; k <= ntr; k++) for (nt = 1; nt <= NT; nt++) res[(k - 1) * NT + nt - 1] = sectionvydiff[k][nt];
    return 0;
}

/*
 * Adjoint loop with correlation: denise.c:1452-1654, nsteps <= NT
 * (for a full run nsteps = NT; the snapshot index follows :1582 with NTDTINV = nsteps).
 * adj: [ntr][NT] adjoint source (time-reversed residual) or NULL -> last refh_residual output.
 */
int refh_adjoint(const float *adj, int nsteps)
{
    int i, j, k, nt, hin, imat, ntr = cur_ntr, NTD;
    float **srcpos_loc_back, **sig;
    if (!fwd_stored) return -1;
    if (nsteps > NT) nsteps = NT;
    NTD = nsteps;
    srcpos_loc_back = matrix(1, 6, 1, ntr);
    for (i = 1; i <= ntr; i++) {
        srcpos_loc_back[1][i] = recpos_loc[1][i];
        srcpos_loc_back[2][i] = recpos_loc[2][i];
    }
    sig = matrix(1, ntr, 1, NT);
    for (k = 1; k <= ntr; k++) for (nt = 1; nt <= NT; nt++)
        sig[k][nt] = adj ? adj[(k - 1) * NT + nt - 1] : sectionvydiff[k][nt];
    zero_state();
    hin = 1;
    for (nt = 1; nt <= nsteps; nt++) {
        CALL_V(1, NX, 1, NY, nt, pvy, pvyp1, pvym1, utty, psyz, psxy, prho, srcpos_loc_back, sig, ntr,
                     absorb_coeff, hc, 0, 1, K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half,
                     a_y_half, b_y_half, psi_syz_y, psi_sxy_x);
        step_stress();
        /* DTINV=1: every step is a stored step (DTINV_help[NT-nt+1]==1) */
        imat = ((NX * NY * NTD) - hin * NX * NY) + 1;
        for (i = 1; i <= NX; i++)
            for (j = 1; j <= NY; j++) {
                g_rho_shot[j][i] += (pvyp1[j][i] * fwd_rho_y[imat]);
                g_u_shot[j][i] += (fwd_u[imat] * psxy[j][i]) + (fwd_y[imat] * psyz[j][i]);
                imat++;
            }
        if (EPRECOND == 1) CALL_EP(Wr, pvy);
        hin++;
    }
    free_matrix(sig, 1, ntr, 1, NT);
    free_matrix(srcpos_loc_back, 1, 6, 1, ntr);
    return 0;
}

/* eprecond1 + per-shot scaling: denise.c:1665-1678 */
int refh_eprecond_scale(void)
{
    int i, j;
    if ((EPRECOND == 1) || (EPRECOND == 3)) {
        CALL_EP1(We, Ws, Wr);
        for (i = 1; i <= NX; i = i + IDX)
            for (j = 1; j <= NY; j = j + IDY) {
                g_u_shot[j][i] = g_u_shot[j][i] / (We[j][i] * C_vs * C_vs);
                g_rho_shot[j][i] = g_rho_shot[j][i] / (We[j][i] * C_rho * C_rho);
            }
    }
    return 0;
}

/* Gradient conversion, denise.c:1743-1813 (INVMAT=0, INVMAT1=1):
 * waveconv_u / waveconv_rho are the shot sums [NY][NX]; outputs g_vs, g_rho. */
int refh_convert(const float *wu, const float *wrho, float *g_vs, float *g_rho)
{
    int i, j;
    for (i = 1; i <= NX; i++)
        for (j = 1; j <= NY; j++) {
            int o = (j - 1) * NX + (i - 1);
            float waveconv_u = wu[o], waveconv_rho = wrho[o];
            float waveconv_mu, waveconv_rho_s;
            waveconv_mu = -DT * waveconv_u;
            waveconv_u = 2.0 * prho[j][i] * pu[j][i] * waveconv_mu;
            waveconv_rho_s = -DT * waveconv_rho;
            waveconv_rho = (pu[j][i] * pu[j][i] * waveconv_mu) + waveconv_rho_s;
            g_vs[o] = waveconv_u;
            g_rho[o] = waveconv_rho;
        }
    return 0;
}

/* Hessian output conversion, hessian_out.c:20-31 (INVMAT1=1), applied to the
 * accumulated hessian_u / hessian_rho; outputs H_vs, H_rho. */
int refh_hessian_out(float *h_vs, float *h_rho)
{
    int i, j;
    for (i = 1; i <= NX; i++)
        for (j = 1; j <= NY; j++) {
            float hu = hessian_u[j][i], hr = hessian_rho[j][i];
            hr += pu[j][i] * pu[j][i] * pu[j][i] * pu[j][i] * hu;
            hu = 4.0 * prho[j][i] * prho[j][i] * pu[j][i] * pu[j][i] * hu;
            h_vs[(j - 1) * NX + i - 1] = hu;
            h_rho[(j - 1) * NX + i - 1] = hr;
        }
    return 0;
}

/* P-SV explosive source of the reference (psource.c), run in isolation on
 * dense [NY][NX] sxx/syy fields. srcpos8 [8][nsrc], signals [nsrc][NT]. */
int refh_psource(int nt, float *sxx, float *syy, int nsrc, const float *srcpos8, const float *signals_in)
{
    float **a = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd), **b = matrix(-nd + 1, NY + nd, -nd + 1, NX + nd);
    float **sp = matrix(1, 8, 1, nsrc), **sig = matrix(1, nsrc, 1, NT);
    int i, j, k, r, n;
    for (j = 1; j <= NY; j++) for (i = 1; i <= NX; i++) { a[j][i] = sxx[(j - 1) * NX + i - 1]; b[j][i] = syy[(j - 1) * NX + i - 1]; }
    for (r = 1; r <= 8; r++) for (k = 1; k <= nsrc; k++) sp[r][k] = srcpos8[(r - 1) * nsrc + (k - 1)];
    for (k = 1; k <= nsrc; k++) for (n = 1; n <= NT; n++) sig[k][n] = signals_in[(k - 1) * NT + n - 1];
    CALL_PSRC(nt, a, b, sp, sig, nsrc);
    for (j = 1; j <= NY; j++) for (i = 1; i <= NX; i++) { sxx[(j - 1) * NX + i - 1] = a[j][i]; syy[(j - 1) * NX + i - 1] = b[j][i]; }
    free_matrix(a, -nd + 1, NY + nd, -nd + 1, NX + nd); free_matrix(b, -nd + 1, NY + nd, -nd + 1, NX + nd);
    free_matrix(sp, 1, 8, 1, nsrc); free_matrix(sig, 1, nsrc, 1, NT);
    return 0;
}

/* ---------------- the reference's file readers / writers ---------------- */
extern char SOURCE_FILE[], REC_FILE[], MFILE[], SEIS_FILE_VY[], DATA_DIR[], SIGNAL_FILE[];
extern int NPROCX, NPROCY, MAXRELERROR, QUELLTYP, SRCREC, RUN_MULTIPLE_SHOTS, READMOD, READREC, SEIS_FORMAT;
extern int HESSIAN, GRAD_METHOD, LNORM, DTINV, INVMAT1, INVMAT;
extern float TAU, FC_HESSIAN, REFREC[4];
extern int IENDX, IENDY;

/* read_par() on a .inp file; numeric results in a fixed order, strings
 * concatenated with '\n' separators into strs (6 names). */
int refh_read_par(const char *path, double *v, char *strs, int nstr)
{
    FILE *fp = fopen(path, "r");
    int k = 0, l;
    if (!fp) return -1;
    FP = stderr;
    MYID = 0;
    read_par(fp);   /* closes fp */
    v[k++] = NPROCX; v[k++] = NPROCY; v[k++] = FDORDER; v[k++] = MAXRELERROR; v[k++] = NX; v[k++] = NY;
    v[k++] = DH; v[k++] = TIME; v[k++] = DT; v[k++] = QUELLART; v[k++] = QUELLTYP; v[k++] = SRCREC;
    v[k++] = RUN_MULTIPLE_SHOTS; v[k++] = READMOD; v[k++] = L;
    for (l = 1; l <= 8; l++) v[k++] = (l <= L) ? FL[l] : 0.0;
    v[k++] = TAU; v[k++] = FREE_SURF; v[k++] = FW; v[k++] = DAMPING; v[k++] = FPML; v[k++] = BOUNDARY;
    v[k++] = SEISMO; v[k++] = READREC; v[k++] = REFREC[1]; v[k++] = REFREC[2]; v[k++] = NDT; v[k++] = SEIS_FORMAT;
    v[k++] = INVMAT1; v[k++] = INVMAT; v[k++] = QUELLTYPB; v[k++] = npower; v[k++] = k_max_PML; v[k++] = HESSIAN;
    v[k++] = FC_HESSIAN; v[k++] = GRAD_METHOD; v[k++] = LNORM; v[k++] = DTINV;
    snprintf(strs, nstr, "%s\n%s\n%s\n%s\n%s\n%s", SIGNAL_FILE, SOURCE_FILE, MFILE, REC_FILE, SEIS_FILE_VY, DATA_DIR);
    return k;
}

/* sources() + splitsrc() for one rank: srcpos_m [8][max] (metres), srcpos_loc [8][max] (grid) */
int refh_sources(const char *path, float dh, int nx, int ny, int max, float *srcpos_m, float *srcpos_loc, int *nloc)
{
    float **sp, **spl;
    int nsrc = 0, n, r, k;
    FP = stderr; MYID = 0; SRCREC = 1; DH = dh; NX = NXG = nx; NY = NYG = ny; IENDX = nx; IENDY = ny;
    POS[1] = POS[2] = 0;
    strncpy(SOURCE_FILE, path, 73); SOURCE_FILE[73] = 0;
    sp = sources(&nsrc);
    if (nsrc > max) return -1;
    for (r = 1; r <= 8; r++) for (k = 1; k <= nsrc; k++) srcpos_m[(r - 1) * max + k - 1] = sp[r][k];
    spl = splitsrc(sp, &n, nsrc);
    for (r = 1; r <= 8; r++) for (k = 1; k <= n; k++) srcpos_loc[(r - 1) * max + k - 1] = spl[r][k];
    *nloc = n;
    return nsrc;
}

/* receiver() with READREC=1: recpos [3][max] */
int refh_receivers(const char *path, float dh, float refx, float refy, int max, int *recpos)
{
    int ntr = 0, r, k;
    int **rp;
    FP = stderr; MYID = 0; READREC = 1; DH = dh; REFREC[1] = refx; REFREC[2] = refy; REFREC[3] = 0.0;
    strncpy(REC_FILE, path, 73); REC_FILE[73] = 0;
    rp = receiver(stderr, &ntr);
    if (ntr > max) return -1;
    for (r = 1; r <= 3; r++) for (k = 1; k <= ntr; k++) recpos[(r - 1) * max + k - 1] = rp[r][k];
    return ntr;
}

/* outseis_glob() in SU format for one shot: section [ntr][ns], recpos [3][ntr],
 * source (xs, ys) in metres */
int refh_write_su(const char *path, int ntr, int ns, const float *section, const int *recpos, float xs, float ys,
                  float dh, float dt, float refx, float refy)
{
    float **sec = matrix(1, ntr, 1, ns), **sp = matrix(1, 8, 1, 1);
    int **rp = imatrix(1, 3, 1, ntr);
    int k, s;
    FILE *fp = fopen(path, "wb");
    if (!fp) return -1;
    FP = stderr; DH = dh; DT = dt; NDT = 1; TIME = ns * dt; REFREC[1] = refx; REFREC[2] = refy;
    for (k = 1; k <= ntr; k++) {
        for (s = 1; s <= ns; s++) sec[k][s] = section[(k - 1) * ns + s - 1];
        rp[1][k] = recpos[k - 1]; rp[2][k] = recpos[ntr + k - 1]; rp[3][k] = recpos[2 * ntr + k - 1];
    }
    sp[1][1] = xs; sp[2][1] = ys;
    outseis_glob(stderr, fp, 0, sec, rp, rp, ntr, sp, 1, ns, 1, 1, 0);   /* closes fp */
    free_matrix(sec, 1, ntr, 1, ns);
    free_matrix(sp, 1, 8, 1, 1);
    free_imatrix(rp, 1, 3, 1, ntr);
    return 0;
}

/* The reference's Butterworth filtering of traces (timedomain_filt.c with
 * libcseife's seife_lpb / seife_hpb), on dense data [ntr][ns]. */
void timedomain_filt(float **data, float fc, int order, int ntr, int ns, int method);
int refh_timedomain_filt(float *data, int ntr, int ns, float dt, float fc, int order, int method)
{
    float **d = matrix(1, ntr, 1, ns);
    int t, j;
    for (t = 1; t <= ntr; t++) for (j = 1; j <= ns; j++) d[t][j] = data[(t - 1) * ns + j - 1];
    DT = dt;
    /* timedomain_filt hands libcseife its 1-based dvector as a 0-based array,
     * so element 0 of that allocation (never initialised) is filtered as the
     * first sample; releasing a zeroed block of the same size first makes the
     * allocator hand that block back, so the element is 0 as in a fresh process */
    free(calloc((size_t)ns + 1, sizeof(double)));
    timedomain_filt(d, fc, order, ntr, ns, method);
    for (t = 1; t <= ntr; t++) for (j = 1; j <= ns; j++) data[(t - 1) * ns + j - 1] = d[t][j];
    free_matrix(d, 1, ntr, 1, ns);
    return 0;
}

/* The reference's conjugate-gradient direction update (src/PCG.c, which fixes
 * PCG_BETA = 2, Polak-Ribiere with reset) on nclass classes of nx*ny values,
 * in the order src/store_PCG_SH.c stores them; dir is updated in place and
 * the reference's 1-based vectors are filled from and copied back to it. */
void PCG(float *PCG_new, float *PCG_old, float *PCG_dir, int PCG_class);
int refh_pcg(int nx, int ny, int nclass, const float *g_new, const float *g_old, float *dir)
{
    const int n = nclass * nx * ny, nx0 = NX, ny0 = NY, idx0 = IDX, idy0 = IDY, myid0 = MYID;
    float *a = vector(1, n), *b = vector(1, n), *d = vector(1, n);
    int h;
    for (h = 1; h <= n; h++) { a[h] = g_new[h - 1]; b[h] = g_old[h - 1]; d[h] = dir[h - 1]; }
    NX = nx; NY = ny; IDX = IDY = 1; MYID = 1;   /* MYID != 0: no progress printout */
    PCG(a, b, d, nclass);
    NX = nx0; NY = ny0; IDX = idx0; IDY = idy0; MYID = myid0;
    for (h = 1; h <= n; h++) dir[h - 1] = d[h];
    free_vector(a, 1, n); free_vector(b, 1, n); free_vector(d, 1, n);
    return 0;
}

/* The reference's gradient tapers on a dense gradient g [ny][nx] (in place):
 * shot = 0 runs src/taper_grad.c with the given sws, shot = k >= 1 runs
 * src/taper_grad_shot.c for source k.  src_xy [2][nsrc] in metres, recpos
 * [2][ntr]; the coefficient field comes back in taper [ny][nx].  The
 * coefficient files taper_grad writes (and taper.bin it reads for sws 5/6)
 * live in the directory dir. */
void taper_grad(float **waveconv, float **taper_coeff, float **srcpos, int nshots, int **recpos, int ntr, int iter,
                int sws);
void taper_grad_shot(float **waveconv, float **taper_coeff, float **srcpos, int nshots, int **recpos, int ntr,
                     int ishot);
extern int GRADT1, GRADT2, GRADT3, GRADT4, SRTSHAPE, FILTSIZE;
extern float SRTRADIUS;
#include <unistd.h>
int refh_taper(const char *dir, int sws, int shot, int nx, int ny, float dh, const int *gradt, int srtshape,
               float srtradius, int filtsize, int nsrc, const float *src_xy, int ntr, const int *recpos, float *g,
               float *taper)
{
    char cwd[4096];
    int i, j, k;
    const int nx0 = NX, ny0 = NY, nxg0 = NXG, nyg0 = NYG, myid0 = MYID;
    const float dh0 = DH;
    FILE *fp0 = FP, *quiet;
    float **w, **tc, **sp;
    int **rp;
    if (!getcwd(cwd, sizeof cwd) || chdir(dir) != 0) return -1;
    quiet = fopen("/dev/null", "w");
    NX = NXG = nx; NY = NYG = ny; DH = dh; POS[1] = POS[2] = 0; IDX = IDY = 1;
    NPROCX = NPROCY = 1; MYID = 1;   /* MYID != 0: no merge of the per-rank coefficient files */
    FP = quiet ? quiet : stderr;
    GRADT1 = gradt[0]; GRADT2 = gradt[1]; GRADT3 = gradt[2]; GRADT4 = gradt[3];
    SRTSHAPE = srtshape; SRTRADIUS = srtradius; FILTSIZE = filtsize;
    w = matrix(1, ny, 1, nx); tc = matrix(1, ny, 1, nx);
    sp = matrix(1, 8, 1, nsrc > 0 ? nsrc : 1); rp = imatrix(1, 3, 1, ntr > 0 ? ntr : 1);
    for (j = 1; j <= ny; j++) for (i = 1; i <= nx; i++) { w[j][i] = g[(j - 1) * nx + i - 1]; tc[j][i] = 0.0f; }
    for (k = 1; k <= nsrc; k++) { sp[1][k] = src_xy[k - 1]; sp[2][k] = src_xy[nsrc + k - 1]; }
    for (k = 1; k <= ntr; k++) { rp[1][k] = recpos[k - 1]; rp[2][k] = recpos[ntr + k - 1]; rp[3][k] = 0; }
    if (shot == 0) taper_grad(w, tc, sp, nsrc, rp, ntr, 1, sws);
    else taper_grad_shot(w, tc, sp, nsrc, rp, ntr, shot);
    for (j = 1; j <= ny; j++) for (i = 1; i <= nx; i++) { g[(j - 1) * nx + i - 1] = w[j][i]; taper[(j - 1) * nx + i - 1] = tc[j][i]; }
    free_matrix(w, 1, ny, 1, nx); free_matrix(tc, 1, ny, 1, nx);
    free_matrix(sp, 1, 8, 1, nsrc > 0 ? nsrc : 1); free_imatrix(rp, 1, 3, 1, ntr > 0 ? ntr : 1);
    FP = fp0;
    NX = nx0; NY = ny0; NXG = nxg0; NYG = nyg0; MYID = myid0; DH = dh0;
    if (quiet) fclose(quiet);
    return chdir(cwd) == 0 ? 0 : -1;
}

/* The reference's spatially variable Gaussian smoothing (src/gauss_filt_var.c,
 * SPATFILTER=4) of a dense gradient g [ny][nx] (in place) for the velocity
 * model vel [ny][nx]; the files it writes and reads back go to the directory
 * dir (JACOBIAN = dir/jac). */
void gauss_filt_var(float **waveconv, float **vel_mod);
extern float WD_DAMP, WD_DAMP1, FC_END;
extern char JACOBIAN[];
int refh_gauss_filt_var(const char *dir, int nx, int ny, float dh, float wd_damp, float wd_damp1, float fc_end,
                        const float *vel, float *g)
{
    int i, j;
    if (strlen(dir) + 4 + 18 >= STRING_SIZE) return -1;   /* its file names live in char[STRING_SIZE] */
    const int nx0 = NX, ny0 = NY, nxg0 = NXG, nyg0 = NYG, myid0 = MYID;
    const float dh0 = DH;
    FILE *fp0 = FP, *quiet = fopen("/dev/null", "w");
    float **w = matrix(1, ny, 1, nx), **v = matrix(1, ny, 1, nx);
    NX = NXG = nx; NY = NYG = ny; DH = dh; POS[1] = POS[2] = 0; IDX = IDY = 1;
    NPROCX = NPROCY = 1; MYID = 0;
    FP = quiet ? quiet : stderr;
    WD_DAMP = wd_damp; WD_DAMP1 = wd_damp1; FC_END = fc_end;
    snprintf(JACOBIAN, STRING_SIZE, "%s/jac", dir);   /* the reference appends up to 18 characters */
    for (j = 1; j <= ny; j++) for (i = 1; i <= nx; i++) { w[j][i] = g[(j - 1) * nx + i - 1]; v[j][i] = vel[(j - 1) * nx + i - 1]; }
    gauss_filt_var(w, v);
    for (j = 1; j <= ny; j++) for (i = 1; i <= nx; i++) g[(j - 1) * nx + i - 1] = w[j][i];
    free_matrix(w, 1, ny, 1, nx); free_matrix(v, 1, ny, 1, nx);
    NX = nx0; NY = ny0; NXG = nxg0; NYG = nyg0; MYID = myid0; DH = dh0; FP = fp0;
    if (quiet) fclose(quiet);
    return 0;
}

/* The reference's built-in start models (READMOD=0, src/denise.c:609-615):
 * model() of src/model_grad_visc.c when l > 0 (vs, rho, taus, eta) and
 * model_elastic() of src/check_start.c when l == 0 (vs, rho), as dense
 * [ny][nx] arrays; the model files they write go to dir (INV_MODELFILE =
 * dir/inv, MFILE = dir/mod). */
void model(float **rho, float **u, float **taus, float *eta);
void model_elastic(float **rho, float **u);
extern char MFILE[], INV_MODELFILE[];
int refh_builtin_model(const char *dir, int l, int nx, int ny, float dh, float dt, const float *fl, float *vs,
                       float *rho, float *taus, float *eta)
{
    int i, j, k;
    if (strlen(dir) + 4 + 17 >= STRING_SIZE) return -1;   /* dir/inv_rho_it_0.bin.0.0 in char[STRING_SIZE] */
    const int nx0 = NX, ny0 = NY, nxg0 = NXG, nyg0 = NYG, myid0 = MYID, l0 = L;
    const float dh0 = DH, dt0 = DT;
    float *fl0 = FL;
    FILE *fp0 = FP, *quiet = fopen("/dev/null", "w");
    NX = NXG = nx; NY = NYG = ny; DH = dh; DT = dt; L = l; POS[1] = POS[2] = 0; IDX = IDY = 1;
    NPROCX = NPROCY = 1; NPROC = 1; MYID = 0;
    FP = quiet ? quiet : stderr;
    snprintf(INV_MODELFILE, STRING_SIZE, "%s/inv", dir);
    snprintf(MFILE, STRING_SIZE, "%s/mod", dir);
    float **r = matrix(1, ny, 1, nx), **u = matrix(1, ny, 1, nx), **t = NULL, *e = NULL;
    if (l > 0) {
        FL = vector(1, l);
        for (k = 1; k <= l; k++) FL[k] = fl[k - 1];
        t = matrix(1, ny, 1, nx);
        e = vector(1, l);
        model(r, u, t, e);
    } else {
        model_elastic(r, u);
    }
    for (j = 1; j <= ny; j++)
        for (i = 1; i <= nx; i++) {
            vs[(j - 1) * nx + i - 1] = u[j][i];
            rho[(j - 1) * nx + i - 1] = r[j][i];
            if (l > 0) taus[(j - 1) * nx + i - 1] = t[j][i];
        }
    if (l > 0) {
        for (k = 1; k <= l; k++) eta[k - 1] = e[k];
        free_matrix(t, 1, ny, 1, nx);
        free_vector(e, 1, l);
        free_vector(FL, 1, l);
    }
    free_matrix(r, 1, ny, 1, nx); free_matrix(u, 1, ny, 1, nx);
    FL = fl0;
    NX = nx0; NY = ny0; NXG = nxg0; NYG = nyg0; MYID = myid0; L = l0; DH = dh0; DT = dt0; FP = fp0;
    if (quiet) fclose(quiet);
    return 0;
}

/* The reference's FD grid check (src/checkfd_ssg_visc.c for l > 0,
 * src/checkfd_ssg_elastic.c for l == 0) on dense [ny][nx] vs, rho, qs; its
 * report goes to the file log.  Only for arguments that pass the check: where
 * it fails the reference ends the process (err). */
void checkfd_ssg_visc(FILE *fp, float **prho, float **pu, float **ptaus, float *peta, float *hc);
void checkfd_ssg_elastic(FILE *fp, float **prho, float **pu, float *hc);
extern float TS;
int refh_checkfd(const char *log, int l, int nx, int ny, const float *fl, float dh, float dt, float ts, int fdorder,
                 int maxrelerror, int fw, const float *vs, const float *rho, const float *qs)
{
    int i, j, k;
    FILE *fp = fopen(log, "w");
    if (!fp) return -1;
    const int nx0 = NX, ny0 = NY, myid0 = MYID, l0 = L, fdo0 = FDORDER, mre0 = MAXRELERROR, fw0 = FW, inv0 = INVMAT1;
    const float dh0 = DH, dt0 = DT, ts0 = TS;
    NX = nx; NY = ny; DH = dh; DT = dt; TS = ts; L = l; MYID = 0; FDORDER = fdorder; MAXRELERROR = maxrelerror;
    FW = fw; INVMAT1 = 1;
    float *h = holbergcoeff();
    float **r = matrix(1, ny, 1, nx), **u = matrix(1, ny, 1, nx);
    for (j = 1; j <= ny; j++)
        for (i = 1; i <= nx; i++) {
            u[j][i] = vs[(j - 1) * nx + i - 1];
            r[j][i] = rho[(j - 1) * nx + i - 1];
        }
    if (l > 0) {
        float **t = matrix(1, ny, 1, nx), *e = vector(1, l);
        for (j = 1; j <= ny; j++)
            for (i = 1; i <= nx; i++) t[j][i] = 2.0 / qs[(j - 1) * nx + i - 1];   /* readmod.c:99 */
        for (k = 1; k <= l; k++) {                                                 /* readmod.c:32-33 */
            float pts = 1.0 / (2.0 * PI * fl[k - 1]);
            e[k] = DT / pts;
        }
        checkfd_ssg_visc(fp, r, u, t, e, h);
        free_matrix(t, 1, ny, 1, nx);
        free_vector(e, 1, l);
    } else {
        checkfd_ssg_elastic(fp, r, u, h);
    }
    fclose(fp);
    free_matrix(r, 1, ny, 1, nx); free_matrix(u, 1, ny, 1, nx); free_vector(h, 0, 6);
    NX = nx0; NY = ny0; MYID = myid0; L = l0; FDORDER = fdo0; MAXRELERROR = mre0; FW = fw0; INVMAT1 = inv0;
    DH = dh0; DT = dt0; TS = ts0;
    return 0;
}

/* The reference's misfit and data energy of traces [ntr][ns]
 * (src/calc_misfit.c, src/calc_energy.c; TRKILL off), called as
 * src/denise.c:1423-1425 calls them. */
double calc_misfit(float **sectiondata, float **section, int ntr, int ns, int LNORM, float L2, int itest, int sws,
                   int swstestshot, int ntr_glob, int **recpos_loc, int nsrc_glob, int ishot);
double calc_energy(float **sectiondata, int ntr, int ns, float energy, int ntr_glob, int **recpos_loc, int nsrc_glob,
                   int ishot);
static float **traces_in(const float *a, int ntr, int ns)
{
    int i, j;
    float **m = matrix(1, ntr, 1, ns);
    for (i = 1; i <= ntr; i++) for (j = 1; j <= ns; j++) m[i][j] = a[(i - 1) * ns + j - 1];
    return m;
}
double refh_calc_misfit(const float *obs, const float *syn, int ntr, int ns, int lnorm, float dt, float l2_in)
{
    const float dt0 = DT;
    const int trk0 = TRKILL;
    float **d = traces_in(obs, ntr, ns), **s = traces_in(syn, ntr, ns);
    DT = dt; TRKILL = 0;
    const double r = calc_misfit(d, s, ntr, ns, lnorm, l2_in, 0, 1, 1, ntr, NULL, 1, 1);
    DT = dt0; TRKILL = trk0;
    free_matrix(d, 1, ntr, 1, ns); free_matrix(s, 1, ntr, 1, ns);
    return r;
}
double refh_calc_energy(const float *obs, int ntr, int ns, float dt, float energy_in)
{
    const float dt0 = DT;
    const int trk0 = TRKILL;
    float **d = traces_in(obs, ntr, ns);
    DT = dt; TRKILL = 0;
    const double r = calc_energy(d, ntr, ns, energy_in, ntr, NULL, 1, 1);
    DT = dt0; TRKILL = trk0;
    free_matrix(d, 1, ntr, 1, ns);
    return r;
}

/* The reference's model update (src/calc_mat_change_test.c, itest = 1) on
 * dense [ny][nx] fields; returns eps_true, *eps_rho = EPSILON_rho. */
float calc_mat_change_test(float **waveconv_rho, float **waveconv_u, float **rho, float **rhonp1, float **u,
                           float **unp1, int iter, int epstest, int INVMAT, float eps_scale, int itest, int nfstart);
extern float SCALERHO, EPSILON_u, EPSILON_rho, VSUPPERLIM, VSLOWERLIM, RHOUPPERLIM, RHOLOWERLIM;
extern int INV_RHO_ITER, INV_VS_ITER;
static float **field_in(const float *a, int nx, int ny)
{
    int i, j;
    float **m = matrix(1, ny, 1, nx);
    for (j = 1; j <= ny; j++) for (i = 1; i <= nx; i++) m[j][i] = a[(j - 1) * nx + i - 1];
    return m;
}
float refh_model_update(int nx, int ny, const float *vs, const float *rho, const float *d_vs, const float *d_rho,
                        float eps_scale, float scalerho, int iter, int inv_vs_iter, int inv_rho_iter,
                        const float *limits, float *vs_new, float *rho_new, float *eps_rho)
{
    int i, j;
    const int nx0 = NX, ny0 = NY, myid0 = MYID, inv0 = INVMAT1;
    NX = nx; NY = ny; MYID = 0; INVMAT1 = 1;
    SCALERHO = scalerho; INV_VS_ITER = inv_vs_iter; INV_RHO_ITER = inv_rho_iter;
    VSLOWERLIM = limits[0]; VSUPPERLIM = limits[1]; RHOLOWERLIM = limits[2]; RHOUPPERLIM = limits[3];
    float **u = field_in(vs, nx, ny), **r = field_in(rho, nx, ny), **gu = field_in(d_vs, nx, ny),
          **gr = field_in(d_rho, nx, ny), **un = matrix(1, ny, 1, nx), **rn = matrix(1, ny, 1, nx);
    const float eps = calc_mat_change_test(gr, gu, r, rn, u, un, iter, 1, 0, eps_scale, 1, 0);
    for (j = 1; j <= ny; j++)
        for (i = 1; i <= nx; i++) {
            vs_new[(j - 1) * nx + i - 1] = un[j][i];
            rho_new[(j - 1) * nx + i - 1] = rn[j][i];
        }
    *eps_rho = EPSILON_rho;
    free_matrix(u, 1, ny, 1, nx); free_matrix(r, 1, ny, 1, nx); free_matrix(gu, 1, ny, 1, nx);
    free_matrix(gr, 1, ny, 1, nx); free_matrix(un, 1, ny, 1, nx); free_matrix(rn, 1, ny, 1, nx);
    NX = nx0; NY = ny0; MYID = myid0; INVMAT1 = inv0;
    return eps;
}

/* The reference's L-BFGS step (src/LBFGS.c) on its ring buffers y, s
 * [nlbfgs*nvec] and the vector q [nvec] (overwritten); r [nvec] out. */
void LBFGS(int iter, float *y_LBFGS, float *s_LBFGS, float *rho_LBFGS, float *alpha_LBFGS, float *q_LBFGS,
           float *r_LBFGS, float *beta_LBFGS, int LBFGS_pointer, int NLBFGS, int NLBFGS_vec);
int refh_lbfgs(int iter, const float *y, const float *s, float *q, float *r, int pointer, int nlbfgs, int nvec)
{
    int i;
    const int n = nlbfgs * nvec, myid0 = MYID;
    float *yv = vector(1, n), *sv = vector(1, n), *qv = vector(1, nvec), *rv = vector(1, nvec);
    float *rho = vector(1, nlbfgs), *alpha = vector(1, nlbfgs), *beta = vector(1, nlbfgs);
    for (i = 1; i <= n; i++) { yv[i] = y[i - 1]; sv[i] = s[i - 1]; }
    for (i = 1; i <= nvec; i++) { qv[i] = q[i - 1]; rv[i] = r[i - 1]; }
    MYID = 1;                                    /* no per-slot printout */
    LBFGS(iter, yv, sv, rho, alpha, qv, rv, beta, pointer, nlbfgs, nvec);
    MYID = myid0;
    for (i = 1; i <= nvec; i++) { q[i - 1] = qv[i]; r[i - 1] = rv[i]; }
    free_vector(yv, 1, n); free_vector(sv, 1, n); free_vector(qv, 1, nvec); free_vector(rv, 1, nvec);
    free_vector(rho, 1, nlbfgs); free_vector(alpha, 1, nlbfgs); free_vector(beta, 1, nlbfgs);
    return 0;
}

/* The reference's parabolic step (src/calc_opt_step.c with src/solvelin.c)
 * for test misfits L2t[3] at steps epst[3]. */
float calc_opt_step(float *L2t, float **waveconv, float **gradg, float *epst, int sws, float C_vp);
float refh_opt_step(const float *l2t, const float *epst)
{
    float L[5] = {0}, E[5] = {0};
    int i;
    for (i = 0; i < 3; i++) { L[i + 1] = l2t[i]; E[i + 1] = epst[i]; }
    return calc_opt_step(L, NULL, NULL, E, 1, 0.0f);
}

/* The reference's model smoothing (src/smooth_model.c, MODEL_FILTER=1, with
 * src/median.c) of dense [ny][nx] vs, rho in place; its model files go to
 * dir (INV_MODELFILE = dir/inv).  Returns FILT_SIZE after the call. */
void smooth_model(float **pu, float **prho, int iter);
extern int MODEL_FILTER, FILT_SIZE;
int refh_smooth_model(const char *dir, int nx, int ny, int filt_size, float *vs, float *rho)
{
    if (strlen(dir) + 4 + 12 >= STRING_SIZE) return -999;
    const int nx0 = NX, ny0 = NY, nxg0 = NXG, nyg0 = NYG, myid0 = MYID;
    FILE *fp0 = FP, *quiet = fopen("/dev/null", "w");
    char path[STRING_SIZE + 16];
    int i, j, rc;
    NX = NXG = nx; NY = NYG = ny; POS[1] = POS[2] = 0; NPROCX = NPROCY = 1; MYID = 0;
    FP = quiet ? quiet : stderr;
    MODEL_FILTER = 1; FILT_SIZE = filt_size;
    snprintf(INV_MODELFILE, STRING_SIZE, "%s/inv", dir);
    float **u = matrix(1, ny, 1, nx), **r = matrix(1, ny, 1, nx);
    for (j = 1; j <= ny; j++) for (i = 1; i <= nx; i++) { u[j][i] = vs[(j - 1) * nx + i - 1]; r[j][i] = rho[(j - 1) * nx + i - 1]; }
    /* the model files it reads: x outer, depth inner */
    snprintf(path, sizeof path, "%s_vs.bin", INV_MODELFILE);
    FILE *f = fopen(path, "wb");
    for (i = 1; i <= nx; i++) for (j = 1; j <= ny; j++) fwrite(&u[j][i], sizeof(float), 1, f);
    fclose(f);
    snprintf(path, sizeof path, "%s_rho.bin", INV_MODELFILE);
    f = fopen(path, "wb");
    for (i = 1; i <= nx; i++) for (j = 1; j <= ny; j++) fwrite(&r[j][i], sizeof(float), 1, f);
    fclose(f);
    smooth_model(u, r, 1);
    for (j = 1; j <= ny; j++) for (i = 1; i <= nx; i++) { vs[(j - 1) * nx + i - 1] = u[j][i]; rho[(j - 1) * nx + i - 1] = r[j][i]; }
    free_matrix(u, 1, ny, 1, nx); free_matrix(r, 1, ny, 1, nx);
    rc = FILT_SIZE;
    MODEL_FILTER = 0;
    NX = nx0; NY = ny0; NXG = nxg0; NYG = nyg0; MYID = myid0; FP = fp0;
    if (quiet) fclose(quiet);
    return rc;
}

/* The reference's relative model change (src/calc_mres.c) of dense fields. */
float calc_mres(int nx1, int nx2, int ny1, int ny2, float **u, float **u0);
float refh_calc_mres(int nx, int ny, const float *u, const float *u0)
{
    float **a = field_in(u, nx, ny), **b = field_in(u0, nx, ny);
    const float m = calc_mres(1, nx, 1, ny, a, b);
    free_matrix(a, 1, ny, 1, nx); free_matrix(b, 1, ny, 1, nx);
    return m;
}

/*
 * dsh_oracle.c — TEST ORACLE ONLY.  CPU restatement of the DENISE-SH hot path
 * (see dsh_oracle.h).  Coefficients are built once in FP32 with the same C
 * types and expression order as the reference; the time stepping is compiled
 * for FP32 and FP64 from dsh_oracle_step.inc.
 */
#include "dsh_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define HX 7                                    /* uniform halo, > FDORDER/2 for every order */
#define ORACLE_PI (3.141592653589793)
#define IX(i, j) ((size_t)((j) - 1 + HX) * (size_t)G.pitch + (size_t)((i) - 1 + HX))

/* Holberg (1987) staggered-grid operator coefficients hc[1..6] per FD order
 * and maximum relative group-velocity error, as tabulated by the reference in
 * holbergcoeff.c:25-66; level 0 holds the Taylor coefficients.  Only the
 * operator coefficients are kept (the reference's column 0, the minimum
 * points per wavelength, is not used by the time stepping). */
static const double HOLBERG[5][6][6] = {
    {{1.0, 0, 0, 0, 0, 0},
     {9.0 / 8.0, -1.0 / 24.0, 0, 0, 0, 0},
     {75.0 / 64.0, -25.0 / 384.0, 3.0 / 640.0, 0, 0, 0},
     {1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0, 0, 0},
     {19845.0 / 16384.0, -735.0 / 8192.0, 567.0 / 40960.0, -405.0 / 229376.0, 35.0 / 294912.0, 0},
     {160083.0 / 131072.0, -12705.0 / 131072.0, 22869.0 / 1310720.0, -5445.0 / 1835008.0, 847.0 / 2359296.0,
      -63.0 / 2883584.0}},
    {{1.0010, 0, 0, 0, 0, 0},
     {1.1382, -0.046414, 0, 0, 0, 0},
     {1.1965, -0.078804, 0.0081781, 0, 0, 0},
     {1.2257, -0.099537, 0.018063, -0.0026274, 0, 0},
     {1.2415, -0.11231, 0.026191, -0.0064682, 0.001191, 0},
     {1.2508, -0.12034, 0.032131, -0.010142, 0.0029857, -0.00066667}},
    {{1.0050, 0, 0, 0, 0, 0},
     {1.1534, -0.052806, 0, 0, 0, 0},
     {1.2111, -0.088313, 0.011768, 0, 0, 0},
     {1.2367, -0.10815, 0.023113, -0.0046905, 0, 0},
     {1.2496, -0.11921, 0.031130, -0.0093272, 0.0025161, 0},
     {1.2568, -0.12573, 0.036423, -0.013132, 0.0047484, -0.0015979}},
    {{1.0100, 0, 0, 0, 0, 0},
     {1.1640, -0.057991, 0, 0, 0, 0},
     {1.2192, -0.094070, 0.014608, 0, 0, 0},
     {1.2422, -0.11269, 0.026140, -0.0064054, 0, 0},
     {1.2534, -0.12257, 0.033755, -0.011081, 0.0036784, 0},
     {1.2596, -0.12825, 0.038550, -0.014763, 0.0058619, -0.0024538}},
    {{1.0300, 0, 0, 0, 0, 0},
     {1.1876, -0.072518, 0, 0, 0, 0},
     {1.2341, -0.10569, 0.022589, 0, 0, 0},
     {1.2516, -0.12085, 0.032236, -0.011459, 0, 0},
     {1.2596, -0.12829, 0.038533, -0.014681, 0.0072580, 0},
     {1.2640, -0.13239, 0.042217, -0.017803, 0.0081959, -0.0051848}},
};

/* Global oracle session (one model at a time; test infrastructure). */
static struct {
    int alive, fp64, fd12_compat, lnorm;
    int nx, ny, nt, fdorder, maxrelerror, fw, free_surf, l, quellart, eprecond;
    float dh, dt, damping, fpml, npower, k_max_pml, fl[8];
    int pitch, rows;
    float hc[7];
    float K_x[64 + 1], a_x[64 + 1], b_x[64 + 1], K_x_half[64 + 1], a_x_half[64 + 1], b_x_half[64 + 1];
    float K_y[64 + 1], a_y[64 + 1], b_y[64 + 1], K_y_half[64 + 1], a_y_half[64 + 1], b_y_half[64 + 1];
    float d_x[64 + 1], d_x_half[64 + 1], d_y[64 + 1], d_y_half[64 + 1];
    float *vs, *rho, *uip, *ujp, *taus, *tausipjp, *fipjp, *f, *dip, *d; /* dense [NY][NX] ([L][NY][NX]) */
    float *muip, *mujp, *qs;                    /* relaxed-modulus factors and Qs (Q gradient) */
    float bip[8], bjm[8], cip[8], cjm[8], eta[8];
    float sumu;                                 /* prepare_update_s.c:29-32 */
    int grad_q;                                 /* accumulate the Qs gradient (dsho_set_grad_q) */
    float c_vs, c_rho;
    int ntr, *recpos;
} G = {.fd12_compat = 1, .lnorm = 2};

#define REAL float
#define SFX f32
#include "dsh_oracle_step.inc"
#undef REAL
#undef SFX
#define REAL double
#define SFX f64
#include "dsh_oracle_step.inc"
#undef REAL
#undef SFX

void dsho_set_fd12_compat(int on) { G.fd12_compat = on; }
void dsho_set_grad_q(int on) { G.grad_q = on; }
int dsho_set_lnorm(int lnorm)
{
    if (lnorm < 1 || lnorm > 5) return -1;
    G.lnorm = lnorm;
    return 0;
}

void dsho_free(void)
{
    state_free_f32();
    state_free_f64();
    free(G.vs); free(G.rho); free(G.uip); free(G.ujp); free(G.taus); free(G.tausipjp);
    free(G.fipjp); free(G.f); free(G.dip); free(G.d); free(G.recpos);
    free(G.muip); free(G.mujp); free(G.qs);
    G.vs = G.rho = G.uip = G.ujp = G.taus = G.tausipjp = G.fipjp = G.f = G.dip = G.d = NULL;
    G.muip = G.mujp = G.qs = NULL;
    G.recpos = NULL;
    G.alive = 0;
}

/* CPML profiles, PML_pro.c:65-295 (Komatitsch & Martin 2007 C-PML).  Kept
 * with the reference's float/double mix, including that a and the "a" guard
 * use the integer abs() of a float (so a stays 0 where |d| < 1). */
static void pml_profiles(void)
{
    const int FW = G.fw, NXG = G.nx, NYG = G.ny;
    const float DH = G.dh, DT = G.dt, npower = G.npower, k_max_PML = G.k_max_pml;
    const float alpha_max_PML = 2.0 * ORACLE_PI * (G.fpml / 2.0);
    float thickness_PML_x, thickness_PML_y, xoriginleft, xoriginright, yoriginbottom, yorigintop;
    float Rcoef, d0_x, d0_y, xval, yval, abscissa_in_PML, abscissa_normalized;
    float alpha_x[65] = {0}, alpha_x_half[65] = {0}, alpha_y[65] = {0}, alpha_y_half[65] = {0};
    int i, h;

    thickness_PML_x = FW * DH;
    thickness_PML_y = FW * DH;
    Rcoef = 0.001;
    d0_x = -(npower + 1) * G.damping * log(Rcoef) / (2.0 * thickness_PML_x);
    d0_y = -(npower + 1) * G.damping * log(Rcoef) / (2.0 * thickness_PML_y);
    xoriginleft = thickness_PML_x;
    xoriginright = (NXG - 1) * DH - thickness_PML_x;

    for (i = 1; i <= FW; i++) {
        G.K_x[i] = 1.0;
        G.K_x_half[i] = 1.0;
        xval = DH * (i - 1);
        abscissa_in_PML = xoriginleft - xval;
        if (abscissa_in_PML >= 0.0) {
            abscissa_normalized = abscissa_in_PML / thickness_PML_x;
            G.d_x[i] = d0_x * pow(abscissa_normalized, npower);
            G.K_x[i] = 1.0 + (k_max_PML - 1.0) * pow(abscissa_normalized, npower);
            alpha_x[i] = alpha_max_PML * (1.0 - abscissa_normalized) + 0.1 * alpha_max_PML;
        }
        abscissa_in_PML = xoriginleft - (xval + DH / 2.0);
        if (abscissa_in_PML >= 0.0) {
            abscissa_normalized = abscissa_in_PML / thickness_PML_x;
            G.d_x_half[i] = d0_x * pow(abscissa_normalized, npower);
            G.K_x_half[i] = 1.0 + (k_max_PML - 1.0) * pow(abscissa_normalized, npower);
            alpha_x_half[i] = alpha_max_PML * (1.0 - abscissa_normalized) + 0.1 * alpha_max_PML;
        }
        if (alpha_x[i] < 0.0) alpha_x[i] = 0.0;
        if (alpha_x_half[i] < 0.0) alpha_x_half[i] = 0.0;
        G.b_x[i] = exp(-(G.d_x[i] / G.K_x[i] + alpha_x[i]) * DT);
        G.b_x_half[i] = exp(-(G.d_x_half[i] / G.K_x_half[i] + alpha_x_half[i]) * DT);
        if (abs((int)G.d_x[i]) > 1.0e-6)
            G.a_x[i] = G.d_x[i] * (G.b_x[i] - 1.0) / (G.K_x[i] * (G.d_x[i] + G.K_x[i] * alpha_x[i]));
        if (abs((int)G.d_x_half[i]) > 1.0e-6)
            G.a_x_half[i] = G.d_x_half[i] * (G.b_x_half[i] - 1.0) /
                            (G.K_x_half[i] * (G.d_x_half[i] + G.K_x_half[i] * alpha_x_half[i]));
    }
    for (i = NXG - FW + 1; i <= NXG; i++) {
        h = i - NXG + 2 * FW;
        G.K_x[h] = 1.0;
        G.K_x_half[h] = 1.0;
        xval = DH * (i - 1);
        abscissa_in_PML = xval - xoriginright;
        if (abscissa_in_PML >= 0.0) {
            abscissa_normalized = abscissa_in_PML / thickness_PML_x;
            G.d_x[h] = d0_x * pow(abscissa_normalized, npower);
            G.K_x[h] = 1.0 + (k_max_PML - 1.0) * pow(abscissa_normalized, npower);
            alpha_x[h] = alpha_max_PML * (1.0 - abscissa_normalized) + 0.1 * alpha_max_PML;
        }
        abscissa_in_PML = xval + DH / 2.0 - xoriginright;
        if (abscissa_in_PML >= 0.0) {
            abscissa_normalized = abscissa_in_PML / thickness_PML_x;
            G.d_x_half[h] = d0_x * pow(abscissa_normalized, npower);
            G.K_x_half[h] = 1.0 + (k_max_PML - 1.0) * pow(abscissa_normalized, npower);
            alpha_x_half[h] = alpha_max_PML * (1.0 - abscissa_normalized) + 0.1 * alpha_max_PML;
        }
        if (alpha_x[h] < 0.0) alpha_x[h] = 0.0;
        if (alpha_x_half[h] < 0.0) alpha_x_half[h] = 0.0;
        G.b_x[h] = exp(-(G.d_x[h] / G.K_x[h] + alpha_x[h]) * DT);
        G.b_x_half[h] = exp(-(G.d_x_half[h] / G.K_x_half[h] + alpha_x_half[h]) * DT);
        if (abs((int)G.d_x[h]) > 1.0e-6)
            G.a_x[h] = G.d_x[h] * (G.b_x[h] - 1.0) / (G.K_x[h] * (G.d_x[h] + G.K_x[h] * alpha_x[h]));
        if (abs((int)G.d_x_half[h]) > 1.0e-6)
            G.a_x_half[h] = G.d_x_half[h] * (G.b_x_half[h] - 1.0) /
                            (G.K_x_half[h] * (G.d_x_half[h] + G.K_x_half[h] * alpha_x_half[h]));
    }

    yoriginbottom = thickness_PML_y;
    yorigintop = (NYG - 1) * DH - thickness_PML_y;
    for (i = 1; i <= FW; i++) {
        G.K_y[i] = 1.0;
        G.K_y_half[i] = 1.0;
        yval = DH * (i - 1);
        abscissa_in_PML = yoriginbottom - yval;
        if (abscissa_in_PML >= 0.0) {
            abscissa_normalized = abscissa_in_PML / thickness_PML_y;
            G.d_y[i] = d0_y * pow(abscissa_normalized, npower);
            G.K_y[i] = 1.0 + (k_max_PML - 1.0) * pow(abscissa_normalized, npower);
            alpha_y[i] = alpha_max_PML * (1.0 - abscissa_normalized) + 0.1 * alpha_max_PML;
        }
        abscissa_in_PML = yoriginbottom - (yval + DH / 2.0);
        if (abscissa_in_PML >= 0.0) {
            abscissa_normalized = abscissa_in_PML / thickness_PML_y;
            G.d_y_half[i] = d0_y * pow(abscissa_normalized, npower);
            G.K_y_half[i] = 1.0 + (k_max_PML - 1.0) * pow(abscissa_normalized, npower);
            alpha_y_half[i] = alpha_max_PML * (1.0 - abscissa_normalized) + 0.1 * alpha_max_PML;
        }
        G.b_y[i] = exp(-(G.d_y[i] / G.K_y[i] + alpha_y[i]) * DT);
        G.b_y_half[i] = exp(-(G.d_y_half[i] / G.K_y_half[i] + alpha_y_half[i]) * DT);
        if (abs((int)G.d_y[i]) > 1.0e-6)
            G.a_y[i] = G.d_y[i] * (G.b_y[i] - 1.0) / (G.K_y[i] * (G.d_y[i] + G.K_y[i] * alpha_y[i]));
        if (abs((int)G.d_y_half[i]) > 1.0e-6)
            G.a_y_half[i] = G.d_y_half[i] * (G.b_y_half[i] - 1.0) /
                            (G.K_y_half[i] * (G.d_y_half[i] + G.K_y_half[i] * alpha_y_half[i]));
    }
    for (i = NYG - FW + 1; i <= NYG; i++) {
        h = i - NYG + 2 * FW;
        G.K_y[h] = 1.0;
        G.K_y_half[h] = 1.0;
        yval = DH * (i - 1);
        abscissa_in_PML = yval - yorigintop;
        if (abscissa_in_PML >= 0.0) {
            abscissa_normalized = abscissa_in_PML / thickness_PML_y;
            G.d_y[h] = d0_y * pow(abscissa_normalized, npower);
            G.K_y[h] = 1.0 + (k_max_PML - 1.0) * pow(abscissa_normalized, npower);
            alpha_y[h] = alpha_max_PML * (1.0 - abscissa_normalized) + 0.1 * alpha_max_PML;
        }
        abscissa_in_PML = yval + DH / 2.0 - yorigintop;
        if (abscissa_in_PML >= 0.0) {
            abscissa_normalized = abscissa_in_PML / thickness_PML_y;
            G.d_y_half[h] = d0_x * pow(abscissa_normalized, npower);
            G.K_y_half[h] = 1.0 + (k_max_PML - 1.0) * pow(abscissa_normalized, npower);
            alpha_y_half[h] = alpha_max_PML * (1.0 - abscissa_normalized) + 0.1 * alpha_max_PML;
        }
        G.b_y[h] = exp(-(G.d_y[h] / G.K_y[h] + alpha_y[h]) * DT);
        G.b_y_half[h] = exp(-(G.d_y_half[h] / G.K_y_half[h] + alpha_y_half[h]) * DT);
        if (abs((int)G.d_y[h]) > 1.0e-6)
            G.a_y[h] = G.d_y[h] * (G.b_y[h] - 1.0) / (G.K_y[h] * (G.d_y[h] + G.K_y[h] * alpha_y[h]));
        if (abs((int)G.d_y_half[h]) > 1.0e-6)
            G.a_y_half[h] = G.d_y_half[h] * (G.b_y_half[h] - 1.0) /
                            (G.K_y_half[h] * (G.d_y_half[h] + G.K_y_half[h] * alpha_y_half[h]));
    }
}

/* One-rank periodic neighbour (matcopy.c / matcopy_elastic.c self-messages
 * wrap the model: index NX+1 reads column 1, NY+1 reads row 1). */
static inline size_t wrapo(int i, int j)
{
    if (i > G.nx) i -= G.nx;
    if (j > G.ny) j -= G.ny;
    return (size_t)(j - 1) * G.nx + (i - 1);
}

int dsho_init(const dsho_params *p, const float *vs, const float *rho, const float *qs, int fp64)
{
    int i, j, l, k;
    const size_t n = (size_t)p->nx * p->ny;
    dsho_free();
    G.lnorm = 2;
    if (p->fdorder < 2 || p->fdorder > 12 || (p->fdorder & 1) || p->maxrelerror < 0 || p->maxrelerror > 4 ||
        p->fw < 0 || p->fw > 64 || p->l < 0 || p->l > 8 || p->nx < 1 || p->ny < 1 || p->nt < 1)
        return -1;
    G.fp64 = fp64;
    G.nx = p->nx; G.ny = p->ny; G.nt = p->nt; G.fdorder = p->fdorder; G.maxrelerror = p->maxrelerror;
    G.fw = p->fw; G.free_surf = p->free_surf; G.l = p->l; G.quellart = p->quellart; G.eprecond = p->eprecond;
    G.dh = p->dh; G.dt = p->dt; G.damping = p->damping; G.fpml = p->fpml; G.npower = p->npower;
    G.k_max_pml = p->k_max_pml;
    for (l = 0; l < 8; l++) G.fl[l] = p->fl[l];
    G.pitch = G.nx + 2 * HX;
    G.rows = G.ny + 2 * HX;

    /* holbergcoeff.c:80-87 */
    G.hc[0] = 0;
    for (k = 1; k <= 6; k++) G.hc[k] = (float)HOLBERG[G.maxrelerror][G.fdorder / 2 - 1][k - 1];

    memset(G.K_x, 0, sizeof(G.K_x)); memset(G.a_x, 0, sizeof(G.a_x)); memset(G.b_x, 0, sizeof(G.b_x));
    memset(G.K_x_half, 0, sizeof(G.K_x_half)); memset(G.a_x_half, 0, sizeof(G.a_x_half));
    memset(G.b_x_half, 0, sizeof(G.b_x_half)); memset(G.K_y, 0, sizeof(G.K_y)); memset(G.a_y, 0, sizeof(G.a_y));
    memset(G.b_y, 0, sizeof(G.b_y)); memset(G.K_y_half, 0, sizeof(G.K_y_half));
    memset(G.a_y_half, 0, sizeof(G.a_y_half)); memset(G.b_y_half, 0, sizeof(G.b_y_half));
    memset(G.d_x, 0, sizeof(G.d_x)); memset(G.d_x_half, 0, sizeof(G.d_x_half));
    memset(G.d_y, 0, sizeof(G.d_y)); memset(G.d_y_half, 0, sizeof(G.d_y_half));
    if (G.fw > 0) pml_profiles();

    G.vs = malloc(n * sizeof(float)); G.rho = malloc(n * sizeof(float));
    G.uip = malloc(n * sizeof(float)); G.ujp = malloc(n * sizeof(float));
    memcpy(G.vs, vs, n * sizeof(float));
    memcpy(G.rho, rho, n * sizeof(float));

    /* av_mue.c:28-52 (INVMAT1=1) with the periodic wrap */
    for (j = 1; j <= G.ny; j++)
        for (i = 1; i <= G.nx; i++) {
            size_t o = wrapo(i, j), ox = wrapo(i + 1, j), oy = wrapo(i, j + 1);
            float u1 = G.rho[o] * G.vs[o] * G.vs[o];
            float u2 = G.rho[ox] * G.vs[ox] * G.vs[ox];
            float u3 = G.rho[oy] * G.vs[oy] * G.vs[oy];
            G.uip[o] = 2.0 / ((1.0 / u1) + (1.0 / u2));
            G.ujp[o] = 2.0 / ((1.0 / u1) + (1.0 / u3));
            if ((u1 == 0.0) || (u2 == 0.0)) G.uip[o] = 0.0;
            if ((u1 == 0.0) || (u3 == 0.0)) G.ujp[o] = 0.0;
        }

    if (G.l > 0) {
        float sumu = 0.0, ws, pts[8];
        G.taus = malloc(n * sizeof(float)); G.tausipjp = malloc(n * sizeof(float));
        G.fipjp = malloc(n * sizeof(float)); G.f = malloc(n * sizeof(float));
        G.dip = malloc(n * G.l * sizeof(float)); G.d = malloc(n * G.l * sizeof(float));
        G.muip = malloc(n * sizeof(float)); G.mujp = malloc(n * sizeof(float)); G.qs = malloc(n * sizeof(float));
        memcpy(G.qs, qs, n * sizeof(float));
        for (k = 0; k < (int)n; k++) G.taus[k] = 2.0 / qs[k];                 /* readmod.c:99 */
        for (l = 0; l < G.l; l++) {                                            /* readmod.c:30-33 */
            float p_ = 1.0 / (2.0 * ORACLE_PI * G.fl[l]);
            G.eta[l] = G.dt / p_;
        }
        for (j = 1; j <= G.ny; j++)                                            /* av_tau.c:12 */
            for (i = 1; i <= G.nx; i++)
                G.tausipjp[wrapo(i, j)] = 0.25 * (G.taus[wrapo(i, j)] + G.taus[wrapo(i + 1, j)] +
                                                  G.taus[wrapo(i, j + 1)] + G.taus[wrapo(i + 1, j + 1)]);
        /* prepare_update_s.c:24-62 */
        for (l = 0; l < G.l; l++) pts[l] = 1.0 / (2.0 * ORACLE_PI * G.fl[l]);
        ws = 2.0 * ORACLE_PI * G.fl[0];
        for (l = 0; l < G.l; l++) sumu = sumu + ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
        for (l = 0; l < G.l; l++) {
            G.bip[l] = 1.0 / (1.0 + (G.eta[l] * 0.5));
            G.bjm[l] = 1.0 / (1.0 + (G.eta[l] * 0.5));
            G.cip[l] = 1.0 - (G.eta[l] * 0.5);
            G.cjm[l] = 1.0 - (G.eta[l] * 0.5);
        }
        G.sumu = sumu;
        for (k = 0; k < (int)n; k++) {
            float mujp = G.ujp[k] / (1.0 + sumu * G.taus[k]);
            float muip = G.uip[k] / (1.0 + sumu * G.tausipjp[k]);
            G.muip[k] = muip;
            G.mujp[k] = mujp;
            G.fipjp[k] = muip * G.dt * (1.0 + G.l * G.tausipjp[k]);
            G.f[k] = mujp * G.dt * (1.0 + G.l * G.taus[k]);
            for (l = 0; l < G.l; l++) {
                G.dip[(size_t)l * n + k] = muip * G.eta[l] * G.tausipjp[k];
                G.d[(size_t)l * n + k] = mujp * G.eta[l] * G.taus[k];
            }
        }
    }

    /* C_vs, C_rho: denise.c:778-816 (float sums, x outer, y inner) */
    {
        float Vs_avg = 0.0, rho_avg = 0.0;
        int Lcount = 0;
        for (i = 1; i <= G.nx; i++)
            for (j = 1; j <= G.ny; j++) {
                Vs_avg += G.vs[(size_t)(j - 1) * G.nx + i - 1];
                rho_avg += G.rho[(size_t)(j - 1) * G.nx + i - 1];
                Lcount++;
            }
        Vs_avg /= Lcount;
        rho_avg /= Lcount;
        G.c_vs = Vs_avg;
        G.c_rho = rho_avg;
    }
    if (fp64) state_alloc_f64(); else state_alloc_f32();
    G.alive = 1;
    return 0;
}

void dsho_get_hc(float *out7) { int k; for (k = 0; k <= 6; k++) out7[k] = G.hc[k]; }
void dsho_get_cnorm(float *out2) { out2[0] = G.c_vs; out2[1] = G.c_rho; }
void dsho_get_sls(float *bip, float *bjm, float *cip, float *cjm)
{
    int l;
    for (l = 0; l < G.l; l++) { bip[l] = G.bip[l]; bjm[l] = G.bjm[l]; cip[l] = G.cip[l]; cjm[l] = G.cjm[l]; }
}

int dsho_get_pml(int which, float *out)
{
    const float *v[] = {G.K_x, G.a_x, G.b_x, G.K_x_half, G.a_x_half, G.b_x_half, G.K_y, G.a_y, G.b_y,
                        G.K_y_half, G.a_y_half, G.b_y_half, G.d_x, G.d_x_half, G.d_y, G.d_y_half};
    int i;
    if (G.fw <= 0 || which < 0 || which > 15) return -1;
    for (i = 1; i <= 2 * G.fw; i++) out[i - 1] = v[which][i];
    return 0;
}

/* Field codes as oracle/ref_harness.c refh_get_field. */
#define GET_FIELD_BODY(S, OUTT)                                                                     \
    const int NX = G.nx, NY = G.ny;                                                                 \
    const size_t n = (size_t)NX * NY;                                                               \
    int i, j;                                                                                       \
    const void *halo = NULL;                                                                        \
    const void *dense = NULL;                                                                       \
    int isfloat = 0;                                                                                \
    switch (which) {                                                                                \
    case 0: halo = S.vy; break; case 1: halo = S.sxy; break; case 2: halo = S.syz; break;           \
    case 3: halo = S.vyp1; break; case 4: halo = S.uy; break; case 5: halo = S.uyx; break;          \
    case 6: dense = G.uip; isfloat = 1; break; case 7: dense = G.ujp; isfloat = 1; break;           \
    case 8: dense = G.rho; isfloat = 1; break; case 9: dense = G.vs; isfloat = 1; break;            \
    case 10: dense = G.fipjp; isfloat = 1; break; case 11: dense = G.f; isfloat = 1; break;         \
    case 12: dense = S.Ws; break; case 13: dense = S.Wr; break; case 14: dense = S.We; break;       \
    case 15: dense = S.gu; break; case 16: dense = S.grho; break;                                   \
    case 17: dense = S.hu; break; case 18: dense = S.hrho; break;                                   \
    case 19: dense = G.taus; isfloat = 1; break; case 20: dense = G.tausipjp; isfloat = 1; break;   \
    default: {                                                                                      \
        int l = which % 100;                                                                        \
        if (l >= G.l) return -1;                                                                    \
        if (which >= 100 && which < 200) dense = S.r + (size_t)l * n;                               \
        else if (which >= 200 && which < 300) dense = S.q + (size_t)l * n;                          \
        else if (which >= 300 && which < 400) { dense = G.dip + (size_t)l * n; isfloat = 1; }       \
        else if (which >= 400 && which < 500) { dense = G.d + (size_t)l * n; isfloat = 1; }         \
        else return -1;                                                                             \
    }                                                                                               \
    }                                                                                               \
    if (!halo && !dense) return -1;                                                                 \
    for (j = 1; j <= NY; j++)                                                                       \
        for (i = 1; i <= NX; i++) {                                                                 \
            size_t o = (size_t)(j - 1) * NX + (i - 1);                                              \
            if (halo) out[o] = (OUTT)((const REALT *)halo)[IX(i, j)];                               \
            else if (isfloat) out[o] = (OUTT)((const float *)dense)[o];                             \
            else out[o] = (OUTT)((const REALT *)dense)[o];                                          \
        }                                                                                           \
    return 0;

int dsho_get_field(int which, float *out)
{
    if (!G.alive) return -1;
    if (G.fp64) {
#define REALT double
        GET_FIELD_BODY(st_f64, float)
#undef REALT
    } else {
#define REALT float
        GET_FIELD_BODY(st_f32, float)
#undef REALT
    }
}

int dsho_get_field_f64(int which, double *out)
{
    if (!G.alive) return -1;
    if (G.fp64) {
#define REALT double
        GET_FIELD_BODY(st_f64, double)
#undef REALT
    } else {
#define REALT float
        GET_FIELD_BODY(st_f32, double)
#undef REALT
    }
}

int dsho_get_psi(int which, float *out)
{
    int k, cnt;
    if (!G.alive || G.fw <= 0 || which < 0 || which > 3) return -1;
    cnt = (which < 2) ? G.ny * 2 * G.fw : 2 * G.fw * G.nx;
    for (k = 0; k < cnt; k++) {
        if (G.fp64) {
            const double *a[] = {st_f64.psi_sxy_x, st_f64.psi_vyx, st_f64.psi_syz_y, st_f64.psi_vyy};
            out[k] = (float)a[which][k];
        } else {
            const float *a[] = {st_f32.psi_sxy_x, st_f32.psi_vyx, st_f32.psi_syz_y, st_f32.psi_vyy};
            out[k] = a[which][k];
        }
    }
    return 0;
}

/* Source time functions, wavelet.c:26-84 (QUELLART 1, 2, 4, 5, 6; type 3
 * reads a file in the reference and is supplied by the caller here). */
int dsho_wavelet(int nsrc, const float *srcpos8, float *out)
{
    int nt, k;
    const float DT = G.dt;
    for (nt = 1; nt <= G.nt; nt++) {
        float t = (float)nt * DT;
        for (k = 1; k <= nsrc; k++) {
            float tshift = srcpos8[3 * nsrc + k - 1], fc = srcpos8[4 * nsrc + k - 1], a = srcpos8[5 * nsrc + k - 1];
            float ts = 1.0 / fc, ag = ORACLE_PI * ORACLE_PI * fc * fc, tau, amp = 0.0;
            switch (G.quellart) {
            case 1:
                tau = ORACLE_PI * (t - 1.5 * ts - tshift) / (1.5 * ts);
                amp = (((1.0 - 4.0 * tau * tau) * exp(-2.0 * tau * tau)));
                break;
            case 2:
                if ((t < tshift) || (t > (tshift + ts))) amp = 0.0;
                else amp = ((sin(2.0 * ORACLE_PI * (t - tshift) * fc) - 0.5 * sin(4.0 * ORACLE_PI * (t - tshift) * fc)));
                break;
            case 4:
                if ((t < tshift) || (t > (tshift + ts))) amp = 0.0;
                else amp = pow(sin(ORACLE_PI * (t + tshift) / ts), 3.0);
                break;
            case 5:
                ts = 1.2 / fc;
                ag = ORACLE_PI * ORACLE_PI * fc * fc;
                amp = -2.0 * ag * (t - ts) * exp(-ag * (t - ts) * (t - ts));
                break;
            case 6:
                amp = 0.0;
                if (nt == 1 + (int)floor(tshift / DT + 0.5)) amp = 1.0;
                break;
            default:
                return -1;
            }
            out[(size_t)(k - 1) * G.nt + nt - 1] = amp * a;
        }
    }
    return 0;
}

int dsho_forward(int nsrc, const float *srcpos8, const float *signals, int ntr, const int *recpos, int nsteps,
                 int store, int hessian, float *seis)
{
    int k;
    if (!G.alive) return -1;
    if (G.fp64) {
        forward_f64(nsrc, srcpos8, signals, ntr, recpos, nsteps, store, hessian);
        for (k = 0; k < ntr * G.nt; k++) seis[k] = (float)st_f64.seis[k];
    } else {
        forward_f32(nsrc, srcpos8, signals, ntr, recpos, nsteps, store, hessian);
        memcpy(seis, st_f32.seis, sizeof(float) * (size_t)ntr * G.nt);
    }
    return 0;
}

int dsho_forward_f64(int nsrc, const float *srcpos8, const float *signals, int ntr, const int *recpos, int nsteps,
                     int store, int hessian, double *seis)
{
    int k;
    if (!G.alive || !G.fp64) return -1;
    forward_f64(nsrc, srcpos8, signals, ntr, recpos, nsteps, store, hessian);
    for (k = 0; k < ntr * G.nt; k++) seis[k] = st_f64.seis[k];
    return 0;
}

int dsho_residual(const float *obs, float *res, double *l2)
{
    int k;
    if (!G.alive) return -1;
    if (G.fp64) {
        residual_f64(obs, l2);
        if (res) for (k = 0; k < G.ntr * G.nt; k++) res[k] = (float)st_f64.res[k];
    } else {
        residual_f32(obs, l2);
        if (res) memcpy(res, st_f32.res, sizeof(float) * (size_t)G.ntr * G.nt);
    }
    return 0;
}

int dsho_adjoint(const float *adj, int nsteps)
{
    if (!G.alive) return -1;
    return G.fp64 ? adjoint_f64(adj, nsteps) : adjoint_f32(adj, nsteps);
}

int dsho_eprecond_scale(void)
{
    if (!G.alive) return -1;
    return G.fp64 ? eprecond_scale_f64() : eprecond_scale_f32();
}

/* Gradient conversion, denise.c:1743-1813 (INVMAT=0, INVMAT1=1). */
int dsho_convert(const float *wu, const float *wrho, float *g_vs, float *g_rho)
{
    int i, j;
    const float DT = G.dt;
    if (!G.alive) return -1;
    for (i = 1; i <= G.nx; i++)
        for (j = 1; j <= G.ny; j++) {
            size_t o = (size_t)(j - 1) * G.nx + (i - 1);
            float waveconv_u = wu[o], waveconv_rho = wrho[o], waveconv_mu, waveconv_rho_s;
            waveconv_mu = -DT * waveconv_u;
            waveconv_u = 2.0 * G.rho[o] * G.vs[o] * waveconv_mu;
            waveconv_rho_s = -DT * waveconv_rho;
            waveconv_rho = (G.vs[o] * G.vs[o] * waveconv_mu) + waveconv_rho_s;
            g_vs[o] = waveconv_u;
            g_rho[o] = waveconv_rho;
        }
    return 0;
}

/* Gradient of the misfit J = sum res^2 with respect to Qs after one shot's
 * forward (stored) + residual + adjoint with dsho_set_grad_q(1) (no
 * counterpart in the reference, which has no Q gradient).  The velocity-stress
 * Lagrangian gives the stress multiplier of forward update k as (2/rho) times
 * the back-propagated adjoint strain e, so dJ/dtau_ipjp = -(2/rho) sum e dsx
 * and dJ/dtau = -(2/rho) sum e dsy; tau_ipjp is the four-point average of tau
 * (av_tau.c:12, one-rank periodic wrap), and tau = 2/Qs (readmod.c:99). */
int dsho_get_grad_q(double *g_qs)
{
    const int NX = G.nx, NY = G.ny;
    int i, j;
    if (!G.alive || G.l < 1 || !G.grad_q) return -1;
    for (j = 1; j <= NY; j++)
        for (i = 1; i <= NX; i++) {
            const int im = i > 1 ? i - 1 : NX, jm = j > 1 ? j - 1 : NY;
            const size_t o = (size_t)(j - 1) * NX + (i - 1);
            const size_t nb[4] = {o, (size_t)(j - 1) * NX + (im - 1), (size_t)(jm - 1) * NX + (i - 1),
                                  (size_t)(jm - 1) * NX + (im - 1)};
            double gx = 0.0, gy;
            int k;
            for (k = 0; k < 4; k++) {
                const double q = G.fp64 ? st_f64.gqx[nb[k]] : (double)st_f32.gqx[nb[k]];
                gx += -2.0 / (double)G.rho[nb[k]] * q;
            }
            gy = -2.0 / (double)G.rho[o] * (G.fp64 ? st_f64.gqy[o] : (double)st_f32.gqy[o]);
            g_qs[o] = (gy + 0.25 * gx) * (-2.0 / ((double)G.qs[o] * (double)G.qs[o]));
        }
    return 0;
}

/* hessian_out.c:20-31 (INVMAT1=1) on the accumulated diagonal. */
int dsho_hessian_out(float *h_vs, float *h_rho)
{
    int k;
    const int n = G.nx * G.ny;
    if (!G.alive) return -1;
    for (k = 0; k < n; k++) {
        float hu = G.fp64 ? (float)st_f64.hu[k] : st_f32.hu[k];
        float hr = G.fp64 ? (float)st_f64.hrho[k] : st_f32.hrho[k];
        float u = G.vs[k], r = G.rho[k];
        hr += u * u * u * u * hu;
        hu = 4.0 * r * r * u * u * hu;
        h_vs[k] = hu;
        h_rho[k] = hr;
    }
    return 0;
}

/* P-SV explosive source, psource.c:17-27 (not linked into the SH program). */
int dsho_psource(int nt, float *sxx, float *syy, int nsrc, const float *srcpos8, const float *signals)
{
    int l;
    const int NT = G.nt;
    const float DT = G.dt;
    for (l = 1; l <= nsrc; l++) {
        int i = (int)srcpos8[0 * nsrc + l - 1], j = (int)srcpos8[1 * nsrc + l - 1];
        const float *s = signals + (size_t)(l - 1) * NT;
        float amp = 0.0f;
        if (nt == 1) amp = s[nt + 1 - 1] / DT;
        if ((nt > 1) && (nt < NT)) amp = (s[nt + 1 - 1] - s[nt - 1 - 1]) / DT;
        if (nt == NT) amp = -s[nt - 1 - 1] / DT;
        sxx[(size_t)(j - 1) * G.nx + i - 1] += amp;
        syy[(size_t)(j - 1) * G.nx + i - 1] += amp;
    }
    return 0;
}

/* ---- SPATFILTER=3 Gaussian smoothing of a gradient (src/gauss_filt.c:58-160) ----
 * Filter length FILT_SIZE_GRAD = round(WD_DAMP*lam/DH) with lam = C_vs/FC_END,
 * made odd (:61-69); hfs = |filt|/2, sigma = hfs/2 in integer arithmetic, s =
 * 2 sigma^2 (:71-73); the model is extended by replicating its edge rows and
 * columns (:98-123); kernel exp(-(ii^2)/s - (jj^2)/s) normalised by its sum
 * (:126-141; the reference never initialises that sum, here it starts at 0);
 * conv summed in float with ii outer and jj inner (:144-157). */
int dsho_gauss_filter_size(float wd_damp, float c_vs, float fc_end, float dh)
{
    const float lam = c_vs / fc_end;
    int f = (int)round((wd_damp * lam) / dh);
    if (f == 0) return 0;
    if (!(f % 2)) f += f > 0 ? 1 : -1;
    return f;
}

int dsho_gauss_kernel(int filt, float *kernel /* [filt][filt], row jj, column ii */)
{
    if (filt == 0) return -1;
    const int hfs = abs(filt) / 2;
    const float sigma = hfs / 2;
    const float s = 2.0f * sigma * sigma;
    const int n = 2 * hfs + 1;
    float sum = 0.0f;
    for (int ii = -hfs; ii <= hfs; ii++)
        for (int jj = -hfs; jj <= hfs; jj++) {
            kernel[(jj + hfs) * n + (ii + hfs)] = exp(-((ii * ii) / s) - ((jj * jj) / s));
            sum += kernel[(jj + hfs) * n + (ii + hfs)];
        }
    for (int k = 0; k < n * n; k++) kernel[k] /= sum;
    return 0;
}

int dsho_gauss_filt(int nx, int ny, int filt, const float *in /* [ny][nx] */, float *out)
{
    if (filt == 0) { memcpy(out, in, (size_t)nx * ny * sizeof(float)); return 0; }
    const int hfs = abs(filt) / 2, n = 2 * hfs + 1;
    float *k = (float *)malloc((size_t)n * n * sizeof(float));
    if (!k) return -1;
    dsho_gauss_kernel(filt, k);
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
            float conv = 0.0f;
            for (int ii = -hfs; ii <= hfs; ii++)
                for (int jj = -hfs; jj <= hfs; jj++) {
                    int jy = j + jj, ix = i + ii;
                    jy = jy < 1 ? 1 : jy > ny ? ny : jy;
                    ix = ix < 1 ? 1 : ix > nx ? nx : ix;
                    conv += in[(size_t)(jy - 1) * nx + (ix - 1)] * k[(jj + hfs) * n + (ii + hfs)];
                }
            out[(size_t)(j - 1) * nx + (i - 1)] = conv;
        }
    free(k);
    return 0;
}

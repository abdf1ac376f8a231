/*
 * dsh_setup.c — host-side coefficient generation for the SH engine.
 *
 * Every coefficient is computed with the same C types (float storage, double
 * libm calls and double literals) and the same operation order as the
 * reference, so the device kernels see bit-identical inputs.  Compiled as C
 * (C++ would pick float overloads of pow/exp/log) with -ffp-contract=off.
 * The per-point loops run on the host's cores (OpenMP); every point is
 * computed by the same expression either way, and the reductions (the mean
 * model of the gradient normalisation) stay sequential in the reference's
 * order.
 */
#include "dsh_setup.h"
#include "dsh.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define DSH_PI (3.141592653589793)

/* Operator coefficients of the staggered first derivative, per half-order
 * (FDORDER/2 = 1..6) and error level.  Level 0 is the Taylor operator (exact
 * fractions); levels 1..4 are Holberg's (1987) optimised operators for a
 * maximum group-velocity error of 0.1, 0.5, 1 and 3 %.  Column 0 is the
 * minimum number of grid points per shortest wavelength of that operator.
 * The reference tabulates the same published numbers in holbergcoeff.c:25-66. */
static const double OPERATORS[5][6][7] = {
    {{23.0, 1.0, 0, 0, 0, 0, 0},
     {8.0, 9.0 / 8.0, -1.0 / 24.0, 0, 0, 0, 0},
     {6.0, 75.0 / 64.0, -25.0 / 384.0, 3.0 / 640.0, 0, 0, 0},
     {5.0, 1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0, 0, 0},
     {5.0, 19845.0 / 16384.0, -735.0 / 8192.0, 567.0 / 40960.0, -405.0 / 229376.0, 35.0 / 294912.0, 0},
     {4.0, 160083.0 / 131072.0, -12705.0 / 131072.0, 22869.0 / 1310720.0, -5445.0 / 1835008.0,
      847.0 / 2359296.0, -63.0 / 2883584.0}},
    {{49.7, 1.0010, 0, 0, 0, 0, 0},
     {8.32, 1.1382, -0.046414, 0, 0, 0, 0},
     {4.77, 1.1965, -0.078804, 0.0081781, 0, 0, 0},
     {3.69, 1.2257, -0.099537, 0.018063, -0.0026274, 0, 0},
     {3.19, 1.2415, -0.11231, 0.026191, -0.0064682, 0.001191, 0},
     {2.91, 1.2508, -0.12034, 0.032131, -0.010142, 0.0029857, -0.00066667}},
    {{22.2, 1.0050, 0, 0, 0, 0, 0},
     {5.65, 1.1534, -0.052806, 0, 0, 0, 0},
     {3.74, 1.2111, -0.088313, 0.011768, 0, 0, 0},
     {3.11, 1.2367, -0.10815, 0.023113, -0.0046905, 0, 0},
     {2.80, 1.2496, -0.11921, 0.031130, -0.0093272, 0.0025161, 0},
     {2.62, 1.2568, -0.12573, 0.036423, -0.013132, 0.0047484, -0.0015979}},
    {{15.8, 1.0100, 0, 0, 0, 0, 0},
     {4.80, 1.1640, -0.057991, 0, 0, 0, 0},
     {3.39, 1.2192, -0.094070, 0.014608, 0, 0, 0},
     {2.90, 1.2422, -0.11269, 0.026140, -0.0064054, 0, 0},
     {2.65, 1.2534, -0.12257, 0.033755, -0.011081, 0.0036784, 0},
     {2.51, 1.2596, -0.12825, 0.038550, -0.014763, 0.0058619, -0.0024538}},
    {{9.16, 1.0300, 0, 0, 0, 0, 0},
     {3.47, 1.1876, -0.072518, 0, 0, 0, 0},
     {2.91, 1.2341, -0.10569, 0.022589, 0, 0, 0},
     {2.61, 1.2516, -0.12085, 0.032236, -0.011459, 0, 0},
     {2.45, 1.2596, -0.12829, 0.038533, -0.014681, 0.0072580, 0},
     {2.36, 1.2640, -0.13239, 0.042217, -0.017803, 0.0081959, -0.0051848}},
};

int dsh_setup_holberg(int fdorder, int maxrelerror, float hc[7])
{
    int k;
    if (fdorder < 2 || fdorder > 12 || (fdorder & 1) || maxrelerror < 0 || maxrelerror > 4) return -1;
    for (k = 0; k < 7; k++) hc[k] = (float)OPERATORS[maxrelerror][fdorder / 2 - 1][k];
    return 0;
}

double dsh_setup_dt_limit(int fdorder, int maxrelerror, float dh, float vmax)
{
    float hc[7];
    double gamma = 0.0;
    int k;
    if (dsh_setup_holberg(fdorder, maxrelerror, hc) != 0 || vmax <= 0) return 0.0;
    for (k = 1; k <= 6; k++) gamma += fabs(hc[k]);
    return dh / (sqrt(2.0) * gamma * vmax);
}

/* FD grid check of the starting model (checkfd_ssg_visc.c:14-140,
 * checkfd_ssg_elastic.c), the reference's float/double mix kept: sumu, c,
 * gamma, dtstab and dhstab are floats formed from double expressions. */
int dsh_check_fd(int nx, int ny, int l, const float *fl, float dh, float dt, float ts, int fdorder, int maxrelerror,
                 int fw, const float *vs, const float *rho, const float *qs, float out[4], int *warn)
{
    float hc[7], peta[DSH_MAX_L];
    float cmax = 0.0f, cmin = 1e9f, c, ws, fmax, gamma, dtstab, dhstab;
    size_t k, n;
    int m;
    if (nx < 1 || ny < 1 || l < 0 || l > DSH_MAX_L || !vs || !rho || !out || !(ts > 0.0f) || !(dh > 0.0f) ||
        (l > 0 && (!fl || !qs)) || dsh_setup_holberg(fdorder, maxrelerror, hc) != 0)
        return DSH_ERR_PARAM;
    for (m = 0; m < l; m++) {                       /* readmod.c:32-33 */
        const float pts = 1.0 / (2.0 * DSH_PI * fl[m]);
        peta[m] = dt / pts;
    }
    ws = 2.0 * DSH_PI / ts;                         /* checkfd_ssg_visc.c:27 */
    n = (size_t)nx * ny;
    for (k = 0; k < n; k++) {
        const float u = vs[k], r = rho[k];
        if (l > 0) {
            const float taus = 2.0 / qs[k];         /* readmod.c:99 */
            const float pu_ref = r * u * u;
            float sumu = 0.0f;
            for (m = 0; m < l; m++) {
                const float tsl = dt / peta[m];
                sumu = sumu + ((ws * ws * tsl * tsl * taus) / (1.0 + ws * ws * tsl * tsl));
            }
            c = sqrt(pu_ref / (r * (1.0 + sumu)));
            if (cmin > c) cmin = c;
            c = sqrt(pu_ref * (1.0 + l * taus) / (r * (1.0 + sumu)));
            if (cmax < c) cmax = c;
        } else {
            c = u;
            if (cmax < c) cmax = c;
            if (cmin > c) cmin = c;
        }
    }
    fmax = 2.0 / ts;
    dhstab = (cmin / (hc[0] * fmax));
    gamma = fabs(hc[1]) + fabs(hc[2]) + fabs(hc[3]) + fabs(hc[4]) + fabs(hc[5]) + fabs(hc[6]);
    dtstab = dh / (sqrt(2) * gamma * cmax);
    out[0] = cmin; out[1] = cmax; out[2] = dtstab; out[3] = dhstab;
    if (warn) *warn = (dh > dhstab ? 1 : 0) | (fw < 10 ? 2 : 0);
    if (dt > dtstab) return DSH_ERR_UNSTABLE;
    if (fw > nx || fw > ny) return DSH_ERR_PARAM;
    return DSH_OK;
}

/* One C-PML node: damping d = d0 * x^npower, stretching K, frequency shift
 * alpha = alpha_max*(1-x) + 0.1*alpha_max (x = normalised depth into the
 * layer), recursion coefficients b = exp(-(d/K + alpha)*dt) and
 * a = d*(b-1)/(K*(d + K*alpha)).  The reference guards a with the integer
 * abs() of d, so a stays 0 where |d| < 1 (PML_pro.c:151-152); kept as is. */
static void pml_node(float abscissa, float thickness, float d0, float npower, float k_max, float alpha_max,
                     float dt, int clamp_alpha, float *d, float *K, float *a, float *b)
{
    float alpha = 0.0f, xn;
    *K = 1.0;
    if (abscissa >= 0.0) {
        xn = abscissa / thickness;
        *d = d0 * pow(xn, npower);
        *K = 1.0 + (k_max - 1.0) * pow(xn, npower);
        alpha = alpha_max * (1.0 - xn) + 0.1 * alpha_max;
    }
    if (clamp_alpha && alpha < 0.0) alpha = 0.0;
    *b = exp(-(*d / *K + alpha) * dt);
    if (abs((int)*d) > 1.0e-6) *a = *d * (*b - 1.0) / (*K * (*d + *K * alpha));
}

void dsh_setup_pml(int nx, int ny, int fw, float dh, float dt, float damping, float fpml, float npower,
                   float k_max_pml, dsh_pml *o)
{
    const float alpha_max = 2.0 * DSH_PI * (fpml / 2.0);
    float thickness, d0, origin_lo, origin_hi_x, origin_hi_y, pos, abscissa;
    int i, h;
    memset(o, 0, sizeof(*o));
    if (fw <= 0) return;
    thickness = fw * dh;
    d0 = -(npower + 1) * damping * log((float)0.001) / (2.0 * thickness);
    origin_lo = thickness;
    origin_hi_x = (nx - 1) * dh - thickness;
    origin_hi_y = (ny - 1) * dh - thickness;

    for (i = 1; i <= fw; i++) {                 /* left / top strip, index i */
        pos = dh * (i - 1);
        abscissa = origin_lo - pos;
        pml_node(abscissa, thickness, d0, npower, k_max_pml, alpha_max, dt, 1, &o->d_x[i], &o->K_x[i], &o->a_x[i],
                 &o->b_x[i]);
        abscissa = origin_lo - (pos + dh / 2.0);
        pml_node(abscissa, thickness, d0, npower, k_max_pml, alpha_max, dt, 1, &o->d_x_half[i], &o->K_x_half[i],
                 &o->a_x_half[i], &o->b_x_half[i]);
        abscissa = origin_lo - pos;
        pml_node(abscissa, thickness, d0, npower, k_max_pml, alpha_max, dt, 0, &o->d_y[i], &o->K_y[i], &o->a_y[i],
                 &o->b_y[i]);
        abscissa = origin_lo - (pos + dh / 2.0);
        pml_node(abscissa, thickness, d0, npower, k_max_pml, alpha_max, dt, 0, &o->d_y_half[i], &o->K_y_half[i],
                 &o->a_y_half[i], &o->b_y_half[i]);
    }
    for (i = nx - fw + 1; i <= nx; i++) {       /* right strip, index h = fw+1..2fw */
        h = i - nx + 2 * fw;
        pos = dh * (i - 1);
        abscissa = pos - origin_hi_x;
        pml_node(abscissa, thickness, d0, npower, k_max_pml, alpha_max, dt, 1, &o->d_x[h], &o->K_x[h], &o->a_x[h],
                 &o->b_x[h]);
        abscissa = pos + dh / 2.0 - origin_hi_x;
        pml_node(abscissa, thickness, d0, npower, k_max_pml, alpha_max, dt, 1, &o->d_x_half[h], &o->K_x_half[h],
                 &o->a_x_half[h], &o->b_x_half[h]);
    }
    for (i = ny - fw + 1; i <= ny; i++) {       /* bottom strip */
        h = i - ny + 2 * fw;
        pos = dh * (i - 1);
        abscissa = pos - origin_hi_y;
        pml_node(abscissa, thickness, d0, npower, k_max_pml, alpha_max, dt, 0, &o->d_y[h], &o->K_y[h], &o->a_y[h],
                 &o->b_y[h]);
        abscissa = pos + dh / 2.0 - origin_hi_y;
        pml_node(abscissa, thickness, d0, npower, k_max_pml, alpha_max, dt, 0, &o->d_y_half[h], &o->K_y_half[h],
                 &o->a_y_half[h], &o->b_y_half[h]);
    }
}

/* periodic neighbour of the one-rank model halo */
static size_t nb(int nx, int ny, int i, int j)
{
    if (i > nx) i -= nx;
    if (j > ny) j -= ny;
    return (size_t)(j - 1) * nx + (i - 1);
}

int dsh_setup_model(int nx, int ny, int l, const float *fl, float dt, const float *vs, const float *rho,
                    const float *qs, float *brho, float *uip, float *ujp, float *fipjp, float *f, float *dip,
                    float *d, float *bip, float *bjm, float *cip, float *cjm, float *cnorm)
{
    const size_t n = (size_t)nx * ny;
    float *mu_ip = NULL, *mu_jp = NULL, *taus = NULL, *tausipjp = NULL;
    int i, j, m;
    if (nx < 1 || ny < 1 || l < 0 || l > DSH_MAX_L) return -1;

    if (brho) {
#pragma omp parallel for schedule(static)
        for (long long kk = 0; kk < (long long)n; kk++) {
            float b = 1.0 / rho[kk];
            if (rho[kk] < 1e-20) b = 0.0;
            brho[kk] = b;
        }
    }

    /* shear modulus mu = rho*vs^2 and its harmonic means at (i+1/2, j) and
     * (i, j+1/2); zero if either side is zero */
    mu_ip = uip ? uip : (float *)malloc(n * sizeof(float));
    mu_jp = ujp ? ujp : (float *)malloc(n * sizeof(float));
    if (!mu_ip || !mu_jp) return -1;
#pragma omp parallel for schedule(static)
    for (int jj = 1; jj <= ny; jj++)
        for (int ii = 1; ii <= nx; ii++) {
            const int i = ii, j = jj;
            size_t c = nb(nx, ny, i, j), e = nb(nx, ny, i + 1, j), s = nb(nx, ny, i, j + 1);
            float mu_c = rho[c] * vs[c] * vs[c];
            float mu_e = rho[e] * vs[e] * vs[e];
            float mu_s = rho[s] * vs[s] * vs[s];
            mu_ip[c] = 2.0 / ((1.0 / mu_c) + (1.0 / mu_e));
            mu_jp[c] = 2.0 / ((1.0 / mu_c) + (1.0 / mu_s));
            if ((mu_c == 0.0) || (mu_e == 0.0)) mu_ip[c] = 0.0;
            if ((mu_c == 0.0) || (mu_s == 0.0)) mu_jp[c] = 0.0;
        }

    if (l > 0) {
        float eta[DSH_MAX_L], tau_sls[DSH_MAX_L], omega, sumu = 0.0;
        taus = (float *)malloc(n * sizeof(float));
        tausipjp = (float *)malloc(n * sizeof(float));
        if (!taus || !tausipjp) { free(taus); free(tausipjp); return -1; }
        /* relaxation times and eta = DT/tau_l (readmod.c:30-33) */
        for (m = 0; m < l; m++) {
            tau_sls[m] = 1.0 / (2.0 * DSH_PI * fl[m]);
            eta[m] = dt / tau_sls[m];
        }
#pragma omp parallel for schedule(static)
        for (long long kk = 0; kk < (long long)n; kk++) taus[kk] = 2.0 / qs[kk];
#pragma omp parallel for schedule(static)
        for (int jj = 1; jj <= ny; jj++)
            for (int ii = 1; ii <= nx; ii++)
                tausipjp[nb(nx, ny, ii, jj)] = 0.25 * (taus[nb(nx, ny, ii, jj)] + taus[nb(nx, ny, ii + 1, jj)] +
                                                       taus[nb(nx, ny, ii, jj + 1)] + taus[nb(nx, ny, ii + 1, jj + 1)]);
        /* relaxed-modulus correction at the reference frequency FL[1] */
        omega = 2.0 * DSH_PI * fl[0];
        for (m = 0; m < l; m++)
            sumu = sumu + ((omega * omega * tau_sls[m] * tau_sls[m]) /
                           (1.0 + omega * omega * tau_sls[m] * tau_sls[m]));
        for (m = 0; m < l; m++) {
            if (bip) bip[m] = 1.0 / (1.0 + (eta[m] * 0.5));
            if (bjm) bjm[m] = 1.0 / (1.0 + (eta[m] * 0.5));
            if (cip) cip[m] = 1.0 - (eta[m] * 0.5);
            if (cjm) cjm[m] = 1.0 - (eta[m] * 0.5);
        }
#pragma omp parallel for schedule(static)
        for (long long kk = 0; kk < (long long)n; kk++) {
            const size_t q = (size_t)kk;
            float mujp = mu_jp[q] / (1.0 + sumu * taus[q]);
            float muip = mu_ip[q] / (1.0 + sumu * tausipjp[q]);
            if (fipjp) fipjp[q] = muip * dt * (1.0 + l * tausipjp[q]);
            if (f) f[q] = mujp * dt * (1.0 + l * taus[q]);
            for (int mm = 0; mm < l; mm++) {
                if (dip) dip[(size_t)mm * n + q] = muip * eta[mm] * tausipjp[q];
                if (d) d[(size_t)mm * n + q] = mujp * eta[mm] * taus[q];
            }
        }
        free(taus);
        free(tausipjp);
    }
    if (!uip) free(mu_ip);
    if (!ujp) free(mu_jp);

    if (cnorm) dsh_setup_cnorm(nx, ny, vs, rho, cnorm);
    (void)i;
    (void)j;
    return 0;
}

void dsh_setup_cnorm(int nx, int ny, const float *vs, const float *rho, float *cnorm)
{
    /* means in the reference's loop order (x outer, depth inner) */
    float vs_sum = 0.0, rho_sum = 0.0;
    int cnt = 0;
    int i, j;
    for (i = 1; i <= nx; i++)
        for (j = 1; j <= ny; j++) {
            vs_sum += vs[(size_t)(j - 1) * nx + i - 1];
            rho_sum += rho[(size_t)(j - 1) * nx + i - 1];
            cnt++;
        }
    vs_sum /= cnt;
    rho_sum /= cnt;
    cnorm[0] = vs_sum;
    cnorm[1] = rho_sum;
}

int dsh_setup_sls(int l, const float *fl, float dt, float *eta, float *bip, float *bjm, float *cip, float *cjm)
{
    float tau_sls[DSH_MAX_L], e[DSH_MAX_L];
    int m;
    if (l < 1 || l > DSH_MAX_L) return -1;
    for (m = 0; m < l; m++) {
        tau_sls[m] = 1.0 / (2.0 * DSH_PI * fl[m]);
        e[m] = dt / tau_sls[m];
    }
    for (m = 0; m < l; m++) {
        if (eta) eta[m] = e[m];
        if (bip) bip[m] = 1.0 / (1.0 + (e[m] * 0.5));
        if (bjm) bjm[m] = 1.0 / (1.0 + (e[m] * 0.5));
        if (cip) cip[m] = 1.0 - (e[m] * 0.5);
        if (cjm) cjm[m] = 1.0 - (e[m] * 0.5);
    }
    return 0;
}

int dsh_setup_visc_base(int nx, int ny, int l, const float *fl, float dt, const float *vs, const float *rho,
                        const float *qs, float *muip, float *mujp, float *tausipjp, float *taus, float *eta)
{
    const size_t n = (size_t)nx * ny;
    float tau_sls[DSH_MAX_L], omega, sumu = 0.0;
    int m;
    if (nx < 1 || ny < 1 || l < 1 || l > DSH_MAX_L) return -1;
    if (dsh_setup_model(nx, ny, 0, fl, dt, vs, rho, qs, NULL, muip, mujp, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                        NULL, NULL) != 0)
        return -1;                          /* harmonic means uip, ujp into muip, mujp */
    for (m = 0; m < l; m++) {
        tau_sls[m] = 1.0 / (2.0 * DSH_PI * fl[m]);
        eta[m] = dt / tau_sls[m];
    }
#pragma omp parallel for schedule(static)
    for (long long kk = 0; kk < (long long)n; kk++) taus[kk] = 2.0 / qs[kk];
#pragma omp parallel for schedule(static)
    for (int jj = 1; jj <= ny; jj++)
        for (int ii = 1; ii <= nx; ii++)
            tausipjp[nb(nx, ny, ii, jj)] = 0.25 * (taus[nb(nx, ny, ii, jj)] + taus[nb(nx, ny, ii + 1, jj)] +
                                                   taus[nb(nx, ny, ii, jj + 1)] + taus[nb(nx, ny, ii + 1, jj + 1)]);
    omega = 2.0 * DSH_PI * fl[0];
    for (m = 0; m < l; m++)
        sumu = sumu + ((omega * omega * tau_sls[m] * tau_sls[m]) / (1.0 + omega * omega * tau_sls[m] * tau_sls[m]));
#pragma omp parallel for schedule(static)
    for (long long kk = 0; kk < (long long)n; kk++) {
        float u_jp = mujp[kk] / (1.0 + sumu * taus[kk]);
        float u_ip = muip[kk] / (1.0 + sumu * tausipjp[kk]);
        mujp[kk] = u_jp;
        muip[kk] = u_ip;
    }
    return 0;
}

float dsh_setup_sumu(int l, const float *fl)
{
    float tau_sls[DSH_MAX_L], omega, sumu = 0.0;
    int m;
    if (l < 1 || l > DSH_MAX_L) return 0.0f;
    for (m = 0; m < l; m++) tau_sls[m] = 1.0 / (2.0 * DSH_PI * fl[m]);
    omega = 2.0 * DSH_PI * fl[0];
    for (m = 0; m < l; m++)
        sumu = sumu + ((omega * omega * tau_sls[m] * tau_sls[m]) / (1.0 + omega * omega * tau_sls[m] * tau_sls[m]));
    return sumu;
}

int dsh_setup_wavelet(int quellart, int nt, float dt, int nsrc, const float *srcpos8, float *out)
{
    int it, s;
    for (it = 1; it <= nt; it++) {
        float t = (float)it * dt;
        for (s = 0; s < nsrc; s++) {
            float tshift = srcpos8[3 * nsrc + s], fc = srcpos8[4 * nsrc + s], amp_scale = srcpos8[5 * nsrc + s];
            float ts = 1.0 / fc, tau, ag, amp;
            switch (quellart) {
            case 1:   /* Ricker, centred at 1.5/fc after tshift */
                tau = DSH_PI * (t - 1.5 * ts - tshift) / (1.5 * ts);
                amp = (((1.0 - 4.0 * tau * tau) * exp(-2.0 * tau * tau)));
                break;
            case 2:   /* one-period two-sine pulse */
                if ((t < tshift) || (t > (tshift + ts))) amp = 0.0;
                else amp = ((sin(2.0 * DSH_PI * (t - tshift) * fc) - 0.5 * sin(4.0 * DSH_PI * (t - tshift) * fc)));
                break;
            case 4:   /* sine cubed */
                if ((t < tshift) || (t > (tshift + ts))) amp = 0.0;
                else amp = pow(sin(DSH_PI * (t + tshift) / ts), 3.0);
                break;
            case 5:   /* first derivative of a Gaussian */
                ts = 1.2 / fc;
                ag = DSH_PI * DSH_PI * fc * fc;
                amp = -2.0 * ag * (t - ts) * exp(-ag * (t - ts) * (t - ts));
                break;
            case 6:   /* spike at sample 1 + round(tshift/dt) */
                amp = 0.0;
                if (it == 1 + (int)floor(tshift / dt + 0.5)) amp = 1.0;
                break;
            default:
                return -1;
            }
            out[(size_t)s * nt + it - 1] = amp * amp_scale;
        }
    }
    return 0;
}

/* SPATFILTER=3 (src/gauss_filt.c:58-141): filter length and normalised
 * kernel [n][n] (row jj, column ii), in the reference's float/double mix;
 * the normalising sum starts at 0 (the reference leaves it uninitialised). */
int dsh_setup_gauss_size(float wd_damp, float c_vs, float fc_end, float dh)
{
    const float lam = c_vs / fc_end;
    int f = (int)round((wd_damp * lam) / dh);
    if (f == 0) return 0;
    if (!(f % 2)) f += f > 0 ? 1 : -1;
    return f;
}

int dsh_setup_gauss_kernel(int filt, float *kernel)
{
    if (filt == 0 || !kernel) return -1;
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

/* Spatially variable Gaussian smoothing, SPATFILTER=4 (src/gauss_filt_var.c:
 * 150-205).  Per point: lam = vel/FC_END, filter sizes round(WD_DAMP1 lam/DH)
 * along x and round(WD_DAMP lam/DH) in depth (odd, at least 6); no filtering
 * where the depth size is <= 0.  The kernels depend only on the half sizes
 * (hx, hz); each distinct pair gets one entry: weights exp(-(ii^2)/sx -
 * (jj^2)/sz) for ii = -hx..hx (outer), jj = -hz..hz (inner) and their float
 * sum in that order, as the reference forms them at every point.
 * map[p] = pair index or -1; pairs[4k..4k+3] = hx, hz, offset of the
 * weights in `weights`, and the sum's bits.  Returns the number of pairs, or
 * -1 when more than max_pairs pairs or max_weights weights are needed. */
int dsh_setup_gauss_var(int nx, int ny, float dh, float wd_damp, float wd_damp1, float fc_end, const float *vel,
                        int *map, int max_pairs, int *pairs, int max_weights, float *weights)
{
    int npairs = 0, nw = 0;
    if (nx < 1 || ny < 1 || !vel || !map || !pairs || !weights) return -1;
    int (*slot)[256] = (int (*)[256])malloc(sizeof(int) * 256 * 256);   /* pair index by (hx, hz), -1 = none */
    if (!slot) return -1;
    for (int a = 0; a < 256; a++)
        for (int b = 0; b < 256; b++) slot[a][b] = -1;
    for (long long p = 0; p < (long long)nx * ny; p++) {
        const float lam = vel[p] / fc_end;
        int fx = (int)round((wd_damp1 * lam) / dh);
        int fz = (int)round((wd_damp * lam) / dh);
        if (!(fz > 0)) { map[p] = -1; continue; }
        if (!(fx % 2)) fx += 1;
        if (!(fz % 2)) fz += 1;
        if (fx < 6) fx = 6;
        if (fz < 6) fz = 6;
        const int hx = abs(fx) / 2, hz = abs(fz) / 2;
        if (hx > 255 || hz > 255) { free(slot); return -1; }
        if (slot[hx][hz] < 0) {
            const int need = (2 * hx + 1) * (2 * hz + 1);
            if (npairs >= max_pairs || nw + need > max_weights) { free(slot); return -1; }
            const float sigmax = hx / 2, sigmaz = hz / 2;
            const float sx = 2.0 * sigmax * sigmax, sz = 2.0 * sigmaz * sigmaz;
            float sum = 0.0;
            int k = nw;
            for (int ii = -hx; ii <= hx; ii++)
                for (int jj = -hz; jj <= hz; jj++) {
                    const float kernel = exp(-((ii * ii) / sx) - ((jj * jj) / sz));
                    weights[k++] = kernel;
                    sum += kernel;
                }
            pairs[4 * npairs] = hx;
            pairs[4 * npairs + 1] = hz;
            pairs[4 * npairs + 2] = nw;
            memcpy(&pairs[4 * npairs + 3], &sum, sizeof(float));
            slot[hx][hz] = npairs++;
            nw += need;
        }
        map[p] = slot[hx][hz];
    }
    free(slot);
    return npairs;
}

/* Butterworth sections of libcseife (cseife.c:147-177, cseife_rfk.c) for
 * timedomain_filt.c: period t0 = 1/fc, order m; an odd order adds a first
 * order section first, then m/2 second-order sections with damping
 * h_j = sin(pi/2 (2j-1)/m).  Each section: f0, f1, f2, g1, g2 (double). */
int dsh_setup_butterworth(double dt, float fc, int order, int highpass, double *coef /* [max 9][5] */)
{
    if (order < 1 || order > 16 || !(fc > 0) || !(dt > 0)) return -1;
    const double one = 1., two = 2., four = 4., eight = 8.;
    const double T0 = 1.0 / fc;
    const double t0 = T0 / dt;
    const double zpi = eight * atan(one), eps = zpi / t0;
    int n = 0;
    const int mm = order / 2;
    if (order > 2 * mm) {
        double *c = coef + 5 * n++;
        c[2] = 0.; c[4] = 0.;
        c[3] = (two - eps) / (two + eps);
        if (!highpass) { c[0] = eps / (two + eps); c[1] = c[0]; }
        else { c[0] = two / (two + eps); c[1] = -(c[0]); }
    }
    const double pih = 2. * atan(1.);
    for (int j = 1; j <= mm; ++j) {
        const double h = sin(pih * (2 * j - 1) / order);
        const double epsq = eps * eps;
        const double a = one - eps * h + epsq / four;
        const double b = -two + epsq / two;
        const double c0 = one + eps * h + epsq / four;
        double *c = coef + 5 * n++;
        c[3] = -b / c0;
        c[4] = -a / c0;
        if (!highpass) { c[0] = epsq / four / c0; c[1] = c[0] + c[0]; c[2] = c[0]; }
        else { c[0] = one / c0; c[1] = -(c[0]) - c[0]; c[2] = c[0]; }
    }
    return n;
}

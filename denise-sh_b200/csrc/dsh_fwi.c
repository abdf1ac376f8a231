/*
 * dsh_fwi.c — L-BFGS direction, parabolic step length and the bracketing
 * line search of the FWI loop (host C; see include/dsh_fwi.h).
 */
#include "dsh_fwi.h"

#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

static double dot(long long n, const float *a, const float *b)
{
    double s = 0.0;
    for (long long i = 0; i < n; i++) s += (double)a[i] * (double)b[i];
    return s;
}

int dsh_lbfgs_direction(long long n, int count, const float *S, const float *Y, const float *q, float *r)
{
    if (n <= 0 || count < 0 || !q || !r || (count > 0 && (!S || !Y)) || count > 64) return -1;
    double alpha[64], rho[64];
    for (long long i = 0; i < n; i++) r[i] = q[i];
    if (count == 0) return 0;
    for (int k = 0; k < count; k++) {
        const double ys = dot(n, Y + (long long)k * n, S + (long long)k * n);
        rho[k] = fabs(ys) > 0.0 ? 1.0 / ys : 0.0;
    }
    /* first loop: newest to oldest (src/LBFGS.c:56-70) */
    for (int k = count - 1; k >= 0; k--) {
        const float *s = S + (long long)k * n, *y = Y + (long long)k * n;
        alpha[k] = rho[k] * dot(n, s, r);
        for (long long i = 0; i < n; i++) r[i] = (float)((double)r[i] - alpha[k] * (double)y[i]);
    }
    /* initial inverse Hessian gamma I from the newest pair (src/LBFGS.c:30-38) */
    const float *sn = S + (long long)(count - 1) * n, *yn = Y + (long long)(count - 1) * n;
    const double yy = dot(n, yn, yn);
    const double gamma = yy > 0.0 ? dot(n, yn, sn) / yy : 1.0;
    for (long long i = 0; i < n; i++) r[i] = (float)(gamma * (double)r[i]);
    /* second loop: oldest to newest (src/LBFGS.c:78-92) */
    for (int k = 0; k < count; k++) {
        const float *s = S + (long long)k * n, *y = Y + (long long)k * n;
        const double beta = rho[k] * dot(n, y, r);
        for (long long i = 0; i < n; i++) r[i] = (float)((double)r[i] + (double)s[i] * (alpha[k] - beta));
    }
    return 0;
}

int dsh_pcg_direction(long long n, int nclass, const float *g_new, const float *g_old, float *dir, int beta_kind,
                      float *beta_out)
{
    if (n <= 0 || nclass < 1 || nclass > DSH_PCG_MAX_CLASSES || !g_new || !g_old || !dir || beta_kind < 1 ||
        beta_kind > 4)
        return -1;
    float beta[DSH_PCG_MAX_CLASSES];
    /* beta per class from float sums in vector order (src/PCG.c:25-83) */
    for (int k = 0; k < nclass; k++) {
        const float *a = g_new + (long long)k * n, *b = g_old + (long long)k * n, *d = dir + (long long)k * n;
        float num = 0.0f, den = 0.0f;
        for (long long i = 0; i < n; i++) {
            switch (beta_kind) {
            case 1: num += a[i] * a[i]; den += b[i] * b[i]; break;                    /* Fletcher-Reeves */
            case 2: num += a[i] * (a[i] - b[i]); den += b[i] * b[i]; break;           /* Polak-Ribiere */
            case 3: num += -a[i] * (a[i] - b[i]); den += d[i] * (a[i] - b[i]); break; /* Hestenes-Stiefel */
            default: num += -a[i] * a[i]; den += d[i] * (a[i] - b[i]); break;         /* Dai-Yuan */
            }
        }
        beta[k] = 0.0f;
        if (den != 0.0f) beta[k] = num / den;
        if (beta_kind == 2 && beta[k] < 0.0f) beta[k] = 0.0f;                     /* direction reset */
        if (beta_out) beta_out[k] = beta[k];
    }
    /* new conjugate direction (src/PCG.c:88-102) */
    for (int k = 0; k < nclass; k++) {
        const float *a = g_new + (long long)k * n;
        float *d = dir + (long long)k * n;
        for (long long i = 0; i < n; i++) d[i] = a[i] + beta[k] * d[i];
    }
    return 0;
}

/* 3x3 solve by Gaussian elimination with partial pivoting (double) */
static int solve3(double A[3][3], double b[3], double x[3])
{
    for (int c = 0; c < 3; c++) {
        int p = c;
        for (int r = c + 1; r < 3; r++)
            if (fabs(A[r][c]) > fabs(A[p][c])) p = r;
        if (A[p][c] == 0.0) return -1;
        for (int k = 0; k < 3; k++) { double t = A[c][k]; A[c][k] = A[p][k]; A[p][k] = t; }
        { double t = b[c]; b[c] = b[p]; b[p] = t; }
        for (int r = c + 1; r < 3; r++) {
            const double f = A[r][c] / A[c][c];
            for (int k = c; k < 3; k++) A[r][k] -= f * A[c][k];
            b[r] -= f * b[c];
        }
    }
    for (int r = 2; r >= 0; r--) {
        double s = b[r];
        for (int k = r + 1; k < 3; k++) s -= A[r][k] * x[k];
        x[r] = s / A[r][r];
    }
    return 0;
}

float dsh_opt_step(const float L2t[3], const float epst[3])
{
    double A[3][3], b[3], x[3];
    for (int i = 0; i < 3; i++) {
        A[i][0] = 1.0;
        A[i][1] = epst[i];
        A[i][2] = (double)epst[i] * epst[i];
        b[i] = L2t[i];
    }
    if (solve3(A, b, x) != 0) return epst[0] > 0 ? epst[0] : epst[1];
    float opteps = (float)(-x[1] / (2.0 * x[2]));
    if (2.0 * x[2] < 0.0 && L2t[1] > L2t[2]) opteps = epst[2];   /* misfit still falling at the 3rd step */
    if (opteps > epst[2]) opteps = epst[2];
    if (opteps < 0.0f) opteps = epst[0];
    return opteps;
}

void dsh_line_search_init(dsh_line_search *ls, float L2_now, float eps_scale, float scalefac, int stepmax)
{
    ls->epst[0] = 0.0f; ls->epst[1] = ls->epst[2] = 0.0f;
    ls->L2t[0] = L2_now; ls->L2t[1] = ls->L2t[2] = 0.0f;
    ls->eps_scale = eps_scale;
    ls->scalefac = scalefac;
    ls->step1 = ls->step2 = ls->countstep = 0;
    ls->stepmax = stepmax;
    ls->slot = 1;
}

int dsh_line_search_next(dsh_line_search *ls, float L2_test, float *eps_scale, int *slot)
{
    /* the misfit of the step just tested goes into its slot (epst1/L2t[itest]);
     * a non-finite misfit counts as no reduction */
    if (!isfinite(L2_test)) L2_test = INFINITY;
    ls->L2t[ls->slot] = L2_test;
    ls->epst[ls->slot] = ls->eps_scale;
    if (ls->step1 == 0 && ls->L2t[0] <= ls->L2t[1]) {          /* no reduction yet: shorter step */
        ls->eps_scale = ls->eps_scale / ls->scalefac;
        ls->countstep++;
    }
    if (ls->step1 == 1 && ls->L2t[1] < ls->L2t[2]) {           /* bracketed */
        ls->epst[2] = ls->eps_scale;
        ls->step2 = 1;
    }
    if (ls->step1 == 1 && ls->L2t[1] >= ls->L2t[2]) {          /* still falling: longer third step */
        ls->epst[2] = ls->eps_scale;
        ls->eps_scale = ls->eps_scale + ls->eps_scale / ls->scalefac;
        ls->countstep++;
    }
    if (ls->step1 == 0 && ls->L2t[0] > ls->L2t[1]) {           /* first reducing step found */
        ls->epst[1] = ls->eps_scale;
        ls->step1 = 1;
        ls->slot = 2;
        ls->countstep = 0;
        ls->eps_scale = ls->eps_scale + ls->eps_scale / ls->scalefac;
    }
    if (ls->step1 == 0 && ls->countstep > ls->stepmax) {
        *eps_scale = 0.0f;
        return -1;
    }
    if (ls->step1 == 1 && ls->countstep > ls->stepmax) ls->step2 = 1;
    if (ls->step1 == 1 && ls->step2 == 1) {
        *eps_scale = dsh_opt_step(ls->L2t, ls->epst);
        return 0;
    }
    *eps_scale = ls->eps_scale;
    *slot = ls->slot;
    return 1;
}

/* calc_misfit.c:51-86 for itest = 0, sws = 1, swstestshot = 1: float
 * running integrals and sums; the LNORM=5 correction is formed in double and
 * stored back to the float sum. */
double dsh_calc_misfit(const float *obs, const float *syn, int ntr, int ns, int lnorm, float dt, float l2_in)
{
    float L2 = l2_in;
    int i, j;
    if (!obs || !syn || ntr < 0 || ns < 0) return NAN;
    for (i = 0; i < ntr; i++) {
        const float *d = obs + (size_t)i * ns, *s = syn + (size_t)i * ns;
        float intseis = 0.0f, intseis_data = 0.0f, intseis_synthetics = 0.0f, abs_data = 0.0f, abs_synthetics = 0.0f;
        float L2_dummy = 0.0f;
        for (j = 0; j < ns; j++) {
            if (lnorm == 2 || lnorm == 6) intseis += s[j] - d[j];
            if (lnorm == 5) {
                intseis_data += d[j] * dt;
                intseis_synthetics += s[j] * dt;
                abs_data += intseis_data * intseis_data;
                abs_synthetics += intseis_synthetics * intseis_synthetics;
                L2_dummy += (intseis_data * intseis_synthetics);
            }
            if (lnorm == 2 || lnorm == 6) L2 += intseis * intseis * dt * dt;
        }
        if (lnorm == 5) L2 -= L2_dummy / (sqrt(abs_data) * sqrt(abs_synthetics));
    }
    return L2;
}

/* calc_energy.c:51-59 */
double dsh_calc_energy(const float *obs, int ntr, int ns, float dt, float energy_in)
{
    float energy = energy_in;
    int i, j;
    if (!obs || ntr < 0 || ns < 0) return NAN;
    for (i = 0; i < ntr; i++) {
        const float *d = obs + (size_t)i * ns;
        float intseis = 0.0f;
        for (j = 0; j < ns; j++) {
            intseis += d[j];
            energy += intseis * intseis * dt * dt;
        }
    }
    return energy;
}

/* calc_mat_change_test.c:31-170 (itest = 1: the caller keeps or adopts the
 * new fields); maxima over the grid in the reference's order, float steps */
float dsh_model_update(int nx, int ny, const float *vs, const float *rho, const float *d_vs, const float *d_rho,
                       float eps_scale, float scalerho, int iter, int inv_vs_iter, int inv_rho_iter,
                       const float limits[4], float *vs_new, float *rho_new, float *eps_rho)
{
    float umax = 0.0f, rhomax = 0.0f, gradmax_u = 0.0f, gradmax_rho = 0.0f, eps_u, eps_r;
    int i, j;
    if (nx < 1 || ny < 1 || !vs || !rho || !d_vs || !d_rho || !limits || !vs_new || !rho_new) return NAN;
    for (i = 0; i < nx; i++)
        for (j = 0; j < ny; j++) {
            const size_t k = (size_t)j * nx + i;
            const float gu = fabs(d_vs[k]), gr = fabs(d_rho[k]);
            if (vs[k] > umax) umax = vs[k];
            if ((i == 0 && j == 0) || gradmax_u == 0.0f) gradmax_u = gu;
            else if (gu > gradmax_u) gradmax_u = gu;
            if (rho[k] > rhomax) rhomax = rho[k];
            if ((i == 0 && j == 0) || gradmax_rho == 0.0f) gradmax_rho = gr;
            else if (gr > gradmax_rho) gradmax_rho = gr;
        }
    eps_u = eps_scale * (umax / gradmax_u);
    if (iter < inv_vs_iter) eps_u = 0.0f;
    eps_r = eps_scale * (rhomax / gradmax_rho) * scalerho;
    if (iter < inv_rho_iter) eps_r = 0.0f;
    for (i = 0; i < nx; i++)
        for (j = 0; j < ny; j++) {
            const size_t k = (size_t)j * nx + i;
            float un = vs[k] - eps_u * d_vs[k];
            float rn = rho[k] - eps_r * d_rho[k];
            if (un < limits[0] && un > 1e-6) un = vs[k];
            if (un > limits[1]) un = vs[k];
            if (rn < limits[2]) rn = rho[k];
            if (rn > limits[3]) rn = rho[k];
            if (inv_vs_iter > iter) un = vs[k];
            if (inv_rho_iter > iter) rn = rho[k];
            if (un < 0.0f) un = vs[k];
            if (rn < 0.0f) rn = rho[k];
            vs_new[k] = un;
            rho_new[k] = rn;
        }
    if (eps_rho) *eps_rho = eps_r;
    return eps_u;
}

/* dotp.c:12-40: float sum in index order */
static float dotp_f(const float *a, const float *b, long long n)
{
    float tmp = 0.0f;
    long long i;
    for (i = 0; i < n; i++) tmp += a[i] * b[i];
    return tmp;
}

/* LBFGS.c:25-104 */
int dsh_lbfgs_ring(int iter, const float *y, const float *s, float *q, float *r, int pointer, int nlbfgs,
                   long long nvec)
{
    float *rho, *alpha, gamma;
    long long i;
    int k;
    if (!y || !s || !q || !r || nlbfgs < 1 || nvec < 1 || pointer < 1 || pointer > nlbfgs) return -1;
    if (iter <= 1) return 0;
    rho = (float *)malloc(2 * (size_t)nlbfgs * sizeof(float));
    if (!rho) return -3;
    alpha = rho + nlbfgs;
    {
        const float *yp = y + (size_t)(pointer - 1) * nvec, *sp = s + (size_t)(pointer - 1) * nvec;
        const float sum_nom = dotp_f(yp, sp, nvec), sum_denom = dotp_f(yp, yp, nvec);
        gamma = sum_nom / sum_denom;
    }
    for (k = 1; k <= nlbfgs; k++) {
        const float sum_nom = dotp_f(y + (size_t)(k - 1) * nvec, s + (size_t)(k - 1) * nvec, nvec);
        rho[k - 1] = fabs(sum_nom) > 0.0 ? 1.0 / sum_nom : 0.0;
    }
    for (k = nlbfgs; k >= 1; k--) {
        const float *yk = y + (size_t)(k - 1) * nvec, *sk = s + (size_t)(k - 1) * nvec;
        alpha[k - 1] = rho[k - 1] * dotp_f(sk, q, nvec);
        for (i = 0; i < nvec; i++) q[i] = q[i] - alpha[k - 1] * yk[i];
    }
    for (i = 0; i < nvec; i++) r[i] = gamma * q[i];
    for (k = 1; k <= nlbfgs; k++) {
        const float *yk = y + (size_t)(k - 1) * nvec, *sk = s + (size_t)(k - 1) * nvec;
        const float beta = rho[k - 1] * dotp_f(yk, r, nvec);
        for (i = 0; i < nvec; i++) r[i] = r[i] + sk[i] * (alpha[k - 1] - beta);
    }
    free(rho);
    return 0;
}

/* calc_opt_step.c:61-103 with solvelin.c:29-52 (method 1) in float */
float dsh_opt_step_ref(const float L2t[3], const float epst[3])
{
    float A[3][3], b[3], x[3], a, c, opteps;
    int k, m, n;
    for (k = 0; k < 3; k++) {
        A[k][2] = (epst[k] * epst[k]);
        A[k][1] = (epst[k]);
        A[k][0] = (1.0);
        b[k] = L2t[k];
    }
    for (k = 0; k < 2; k++)
        for (n = k; n < 2; n++) {
            a = A[n + 1][k] / A[k][k];
            for (m = 0; m < 3; m++) A[n + 1][m] = A[n + 1][m] - a * A[k][m];
            b[n + 1] = b[n + 1] - a * b[k];
        }
    for (k = 2; k >= 0; k--) {
        c = b[k];
        for (m = 2; m >= k + 1; m--) c = c - A[k][m] * x[m];
        x[k] = c / A[k][k];
    }
    opteps = -x[1] / (2.0 * x[2]);
    if (((2.0 * x[2]) < 0.0) && (L2t[1] > L2t[2])) opteps = epst[2];
    if (opteps > epst[2]) opteps = epst[2];
    if (opteps < 0.0) opteps = epst[0];
    return opteps;
}

/* smooth_model.c:25-121 with median.c:12-38 (k successive first minima) */
static void median_field(int nx, int ny, int hfs, const float *in, float *out, float *win)
{
    const int side = 2 * hfs + 1, k = side * side;
    int i, j, ii, jj, a;
    for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++) {
            int n = 0;
            for (jj = -hfs; jj <= hfs; jj++)
                for (ii = -hfs; ii <= hfs; ii++) {
                    int y = j + jj, x = i + ii;
                    y = y < 0 ? 0 : (y >= ny ? ny - 1 : y);
                    x = x < 0 ? 0 : (x >= nx ? nx - 1 : x);
                    const float v = in[(size_t)y * nx + x];
                    /* stable insertion: equal values keep their window order, as
                       repeated first-minimum selection orders them */
                    for (a = n; a > 0 && v < win[a - 1]; a--) win[a] = win[a - 1];
                    win[a] = v;
                    n++;
                }
            out[(size_t)j * nx + i] = win[(k + 1) / 2 - 1];
        }
}

int dsh_smooth_model_median(int nx, int ny, int filt_size, const float *vs, const float *rho, float *vs_out,
                            float *rho_out, int *filt_size_used)
{
    int fs = filt_size, hfs;
    float *win;
    if (nx < 1 || ny < 1 || !vs || !rho || !vs_out || !rho_out) return -1;
    if (fs == 0) {
        memcpy(vs_out, vs, (size_t)nx * ny * sizeof(float));
        memcpy(rho_out, rho, (size_t)nx * ny * sizeof(float));
        if (filt_size_used) *filt_size_used = 0;
        return 0;
    }
    if (!(fs % 2)) fs = fs > 0 ? fs + 1 : fs - 1;
    hfs = abs(fs) / 2;
    if (hfs > 64) return -1;
    win = (float *)malloc((size_t)(2 * hfs + 1) * (2 * hfs + 1) * sizeof(float));
    if (!win) return -3;
    median_field(nx, ny, hfs, vs, vs_out, win);
    median_field(nx, ny, hfs, rho, rho_out, win);
    free(win);
    if (filt_size_used) *filt_size_used = fs;
    return 0;
}

/* calc_mres.c:12-24 */
float dsh_calc_mres(int nx, int ny, const float *u, const float *u0)
{
    float M2tmp = 0.0f, m20 = 0.0f;
    int i, j;
    if (nx < 1 || ny < 1 || !u || !u0) return NAN;
    for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++) {
            const size_t k = (size_t)j * nx + i;
            M2tmp += (u[k] - u0[k]) * (u[k] - u0[k]);
            m20 += u0[k] * u0[k];
        }
    return M2tmp / m20;
}

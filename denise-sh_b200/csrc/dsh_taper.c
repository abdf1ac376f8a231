/*
 * dsh_taper.c — coefficients of the gradient tapers (host C).
 *
 * src/taper_grad.c builds a coefficient field on the host, multiplies the
 * summed gradient by it and sets a few points to zero; src/taper_grad_shot.c
 * does the same with one shot's circular taper before the shot sum.  The
 * coefficients here follow the reference's C types and operation order
 * (float storage, double libm calls and literals), so they are bit-identical;
 * the multiplication runs on the device (dsh_taper_apply, and the engine's
 * shot sum for the per-shot taper).
 */
#include "dsh.h"
#include "dsh_setup.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* iround of src/fd.h:18 */
static int iround_f(float x) { return (int)floor(x + 0.5); }

int dsh_setup_taper_box(int srtshape, float srtradius, float dh, int *g_out, int *ijc_out, float *m)
{
    if (!(dh > 0) || !(srtradius >= 0) || (srtshape != 1 && srtshape != 2)) return -1;
    /* box size in grid points, at least 5 (src/taper_grad.c:303-305) */
    int g = (int)(ceil(2.0 * srtradius / dh));
    if (g < 5) g = 5;
    if (g_out) *g_out = g;
    if (ijc_out) *ijc_out = (int)(ceil((float)g / 2));          /* centre (src/taper_grad.c:351) */
    if (!m) return 0;
    const float a = 1.0f;
    const float maxrad = sqrt(2.0 * srtradius * srtradius);
    /* m[j][i] = erf(a rad/maxrad) or log(rad) of the distance to the centre (:318-335) */
    for (int j = 1; j <= g; j++)
        for (int i = 1; i <= g; i++) {
            const float x = ((float)i - ((float)g) / 2.0 - 0.5) * dh;
            const float y = ((float)j - ((float)g) / 2.0 - 0.5) * dh;
            const float rad = sqrt(x * x + y * y);
            float v;
            if (srtshape == 1) v = erf(a * rad / maxrad);
            else v = rad > 0 ? log(rad) : 0.0;
            m[(j - 1) * g + (i - 1)] = v;
        }
    /* minus the minimum (minimum_m, src/util.c:38-54: first element, then i outer, j inner) */
    float minm = m[0];
    for (int i = 1; i <= g; i++)
        for (int j = 1; j <= g; j++) {
            if (i * j == 1) continue;
            if (m[(j - 1) * g + (i - 1)] < minm) minm = m[(j - 1) * g + (i - 1)];
        }
    for (int k = 0; k < g * g; k++) m[k] -= minm;
    /* normalised to the largest of the four edge centres, capped at 1 (:340-349) */
    const float e[4] = {m[0 * g + (g / 2 - 1)], m[(g / 2 - 1) * g + 0], m[(g / 2 - 1) * g + (g - 1)],
                        m[(g - 1) * g + (g / 2 - 1)]};
    float maxm = e[0];
    for (int k = 1; k < 4; k++)
        if (e[k] > maxm) maxm = e[k];
    for (int k = 0; k < g * g; k++) {
        m[k] /= maxm;
        if (m[k] > 1.0) m[k] = 1.0;
    }
    return 0;
}

/* the min-combined source masks and their normalisation (src/taper_grad.c:353-393):
 * msum = 1, lowered to the box values of every source; then (msum - min) / max */
static void taper_sources(int nx, int ny, int g, int ijc, const float *m, int nsrc, const int *si, const int *sj,
                          float *msum)
{
    for (long long k = 0; k < (long long)nx * ny; k++) msum[k] = 1.0f;
    for (int n = 0; n < nsrc; n++)
        for (int iy = 1; iy <= g; iy++)
            for (int ix = 1; ix <= g; ix++) {
                const int xx = si[n] + ix - ijc, yy = sj[n] + iy - ijc;
                if ((xx < 1) || (xx > nx) || (yy < 1) || (yy > ny)) continue;
                float *p = msum + (long long)(yy - 1) * nx + (xx - 1);
                const float v = m[(iy - 1) * g + (ix - 1)];
                if (*p > v) *p = v;
            }
}

void dsh_setup_taper_norm(int nx, int ny, int g, int ijc, const float *m, int i1, int j1, float *minm_out,
                          float *maxm_out)
{
    /* One source: msum is 1 outside the box and min(1, m) inside it.  min
     * and max of non-NaN values do not depend on the visiting order, and
     * float subtraction is monotonic, so max(msum - minm) = max(msum) - minm. */
    long long covered = 0;
    float mn = INFINITY, mx = -INFINITY;
    for (int iy = 1; iy <= g; iy++)
        for (int ix = 1; ix <= g; ix++) {
            const int xx = i1 + ix - ijc, yy = j1 + iy - ijc;
            if ((xx < 1) || (xx > nx) || (yy < 1) || (yy > ny)) continue;
            covered++;
            float v = 1.0f;
            if (v > m[(iy - 1) * g + (ix - 1)]) v = m[(iy - 1) * g + (ix - 1)];
            if (v < mn) mn = v;
            if (v > mx) mx = v;
        }
    if (covered < (long long)nx * ny) {      /* some points keep msum = 1 */
        if (1.0f < mn) mn = 1.0f;
        if (1.0f > mx) mx = 1.0f;
    }
    *minm_out = mn;
    *maxm_out = mx - mn;
}

int dsh_taper_coeff(int sws, int nx, int ny, float dh, const int gradt[4], int srtshape, float srtradius,
                    int filtsize, int nsrc, const float *src_xy, int ntr, const int *recpos, const float *file_vals,
                    float *coeff, unsigned char *zero)
{
    if (nx < 1 || ny < 1 || !(dh > 0) || !coeff || !zero) return DSH_ERR_PARAM;
    if ((sws == 1 || sws == 2) && !gradt) return DSH_ERR_PARAM;
    if ((sws == 1 || sws == 3) && nsrc > 0 && !src_xy) return DSH_ERR_PARAM;
    if (sws == 1 && ntr > 0 && !recpos) return DSH_ERR_PARAM;
    if ((sws == 5 || sws == 6) && !file_vals) return DSH_ERR_PARAM;
    if (sws == 3 && filtsize < 0) return DSH_ERR_PARAM;
    const long long n = (long long)nx * ny;
    memset(zero, 0, (size_t)n);
#define C_(j, i) coeff[(long long)((j) - 1) * nx + ((i) - 1)]
#define Z_(j, i) zero[(long long)((j) - 1) * nx + ((i) - 1)]
#define IN_(j, i) ((i) >= 1 && (i) <= nx && (j) >= 1 && (j) <= ny)
    if (sws == 1) {
        /* vertical frame: Gaussian ramps over GRADT1..GRADT2 and GRADT3..GRADT4 (src/taper_grad.c:47-100) */
        const int taperlength = gradt[1] - gradt[0], taperlength2 = gradt[3] - gradt[2];
        const int ifw = gradt[3] - gradt[0];
        float *window = (float *)malloc(sizeof(float) * (size_t)(ifw > 0 ? ifw : 1));
        if (!window) return DSH_ERR_OOM;
        const float a = 3;
        for (int i = 1; i <= ifw; i++) {
            window[i - 1] = 1.0;
            if (i <= taperlength)
                window[i - 1] = exp(-(1.0 / 2.0) * (a * (i - taperlength) / (taperlength / 2.0)) *
                                    (a * (i - taperlength) / (taperlength / 2.0)));
            if (i >= (ifw - taperlength2))
                window[i - 1] = exp(-(1.0 / 2.0) * (a * (i - (ifw - taperlength2)) / (taperlength2 / 2.0)) *
                                    (a * (i - (ifw - taperlength2)) / (taperlength2 / 2.0)));
        }
        for (int j = 1; j <= ny; j++) {
            int h = 1;
            for (int i = 1; i <= nx; i++) {
                float t = 0.0;
                if ((i > gradt[0]) && (i < gradt[3])) t = window[(h++) - 1];
                C_(j, i) = t;
            }
        }
        free(window);
        /* zero at the source and receiver points (:118-160) */
        for (int k = 0; k < nsrc; k++) {
            const int i = iround_f(src_xy[k] / dh), j = iround_f(src_xy[nsrc + k] / dh);
            if (IN_(j, i)) Z_(j, i) = 1;
        }
        for (int k = 0; k < ntr; k++) {
            const int i = recpos[k], j = recpos[ntr + k];
            if (IN_(j, i)) Z_(j, i) = 1;
        }
    } else if (sws == 2) {
        /* horizontal: Gaussian ramp over rows GRADT1..GRADT2, depth j*DH below (src/taper_grad.c:177-241) */
        const int taperlength = gradt[1] - gradt[0];
        const int ifw = gradt[1] - gradt[0] + 1;
        float *window = (float *)malloc(sizeof(float) * (size_t)(ifw > 0 ? ifw : 1));
        if (!window) return DSH_ERR_OOM;
        const float a = 3;
        const float exp_hor = 1.0;
        for (int i = 1; i <= ifw; i++) {
            window[i - 1] = 1.0;
            if (i <= taperlength)
                window[i - 1] = exp(-(1.0 / 2.0) * (a * (i - taperlength) / (taperlength / 2.0)) *
                                    (a * (i - taperlength) / (taperlength / 2.0)));
        }
        int h = 1;
        for (int j = 1; j <= ny; j++) {
            for (int i = 1; i <= nx; i++) {
                float t = 0.0;
                if ((j >= gradt[0]) && (j <= gradt[1])) t = window[h - 1];
                if (j > gradt[1]) t = pow((float)(j * dh), exp_hor);
                C_(j, i) = t;
            }
            if (j >= gradt[0]) h++;
        }
        free(window);
    } else if (sws == 3) {
        /* circular tapers at the sources (src/taper_grad.c:298-436) */
        int g, ijc;
        if (dsh_setup_taper_box(srtshape, srtradius, dh, &g, &ijc, NULL) != 0) return DSH_ERR_PARAM;
        float *m = (float *)malloc(sizeof(float) * (size_t)g * g);
        int *si = (int *)malloc(sizeof(int) * (size_t)(nsrc > 0 ? nsrc : 1));
        int *sj = (int *)malloc(sizeof(int) * (size_t)(nsrc > 0 ? nsrc : 1));
        if (!m || !si || !sj) { free(m); free(si); free(sj); return DSH_ERR_OOM; }
        dsh_setup_taper_box(srtshape, srtradius, dh, &g, &ijc, m);
        for (int k = 0; k < nsrc; k++) {
            si[k] = iround_f(src_xy[k] / dh);
            sj[k] = iround_f(src_xy[nsrc + k] / dh);
        }
        taper_sources(nx, ny, g, ijc, m, nsrc, si, sj, coeff);
        /* minimum_m / maximum_m over the grid (src/util.c:38-72), then (msum - min)/max */
        float minm = coeff[0];
        for (int i = 1; i <= nx; i++)
            for (int j = 1; j <= ny; j++)
                if (i * j != 1 && C_(j, i) < minm) minm = C_(j, i);
        for (long long k = 0; k < n; k++) coeff[k] -= minm;
        float maxm = coeff[0];
        for (int i = 1; i <= nx; i++)
            for (int j = 1; j <= ny; j++)
                if (i * j != 1 && C_(j, i) > maxm) maxm = C_(j, i);
        for (long long k = 0; k < n; k++) coeff[k] = coeff[k] / maxm;
        /* zero within FILTSIZE points of each source (:400-428); box points
         * outside the grid are skipped */
        for (int k = 0; k < nsrc; k++)
            for (int i = si[k] - filtsize; i <= si[k] + filtsize; i++)
                for (int j = sj[k] - filtsize; j <= sj[k] + filtsize; j++)
                    if (IN_(j, i)) { Z_(j, i) = 1; C_(j, i) = 0.0; }
        free(m); free(si); free(sj);
    } else if (sws == 5 || sws == 6) {
        /* coefficients from a file of nx*ny floats, x outer (src/taper_grad.c:540-560) */
        for (int i = 1; i <= nx; i++)
            for (int j = 1; j <= ny; j++) C_(j, i) = file_vals[(long long)(i - 1) * ny + (j - 1)];
    } else {
        return DSH_ERR_PARAM;
    }
#undef C_
#undef Z_
#undef IN_
    return DSH_OK;
}

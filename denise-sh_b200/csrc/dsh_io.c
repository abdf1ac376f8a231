/*
 * dsh_io.c — the reference's file formats (see include/dsh_io.h).
 */
#include "dsh_io.h"

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int iround_f(float x) { return (int)floor(x + 0.5); }

/* Types of the parameter lines of a .inp file in the reference's order
 * (src/read_par.c): i int, f float, s string, L the FL list (L floats),
 * F two floats "a , b", A four ints "a, b, c, d", B three ints. */
static const char INP_SCHEMA[] =
    "iiiiii" "fff" "ii" "fff" "s" "f" "i" "s" "ii" "s" "i" "L" "f" "ii" "ff" "ii" "fff" "iii" "s" "ii" "s"
    "FFF" "ii" "ff" "iii" "ssssss" "iii" "s" "i" "ss" "iii" "A" "iii" "B" "iiiii" "f" "iii" "f" "iiii" "s"
    "iiii" "ffffffff" "i" "ff" "i" "f" "iiiii" "s" "iii" "fff" "iii" "f" "i" "ff" "i" "s" "i" "s" "fff"
    "i" "s" "iiiiii" "s";

/* 1-based parameter line of each field used here */
enum {
    LN_NPROCX = 1, LN_NPROCY = 2, LN_FDORDER = 3, LN_MAXRELERROR = 4, LN_NX = 5, LN_NY = 6, LN_DH = 7, LN_TIME = 8,
    LN_DT = 9, LN_QUELLART = 10, LN_QUELLTYP = 11, LN_ANGLE = 12, LN_PWD = 13, LN_PHI = 14, LN_SIGNAL_FILE = 15,
    LN_TS = 16, LN_SRCREC = 17, LN_SOURCE_FILE = 18, LN_RMS = 19, LN_READMOD = 20, LN_MFILE = 21, LN_L = 22,
    LN_FL = 23, LN_TAU = 24, LN_FREE_SURF = 25, LN_FW = 26, LN_DAMPING = 27, LN_FPML = 28, LN_BOUNDARY = 29,
    LN_SEISMO = 38, LN_READREC = 39, LN_REC_FILE = 40, LN_REFREC = 41, LN_NDT = 49, LN_SEIS_FORMAT = 50,
    LN_SEIS_FILE_VY = 52, LN_DATA_DIR = 63, LN_INVMAT1 = 68, LN_INVMAT = 69, LN_QUELLTYPB = 70, LN_NPOWER = 97,
    LN_KMAX = 98, LN_HESSIAN = 99, LN_FC_HESSIAN = 103, LN_GRAD_METHOD = 105, LN_LNORM = 117, LN_DTINV = 118
};

static void inp_defaults(dsh_inp *in)
{
    memset(in, 0, sizeof(*in));
    in->fdorder = 4; in->maxrelerror = 1; in->quellart = 1; in->quelltyp = 3; in->npower = 4.0f;
    in->k_max_pml = 1.0f; in->seismo = 1; in->ndt = 1; in->seis_format = 1; in->invmat1 = 1; in->quelltypb = 2;
    in->lnorm = 2; in->dtinv = 1; in->nprocx = in->nprocy = 1;
}

static void set_int(dsh_inp *in, int line, int v)
{
    switch (line) {
    case LN_NPROCX: in->nprocx = v; break;       case LN_NPROCY: in->nprocy = v; break;
    case LN_FDORDER: in->fdorder = v; break;     case LN_MAXRELERROR: in->maxrelerror = v; break;
    case LN_NX: in->nx = v; break;               case LN_NY: in->ny = v; break;
    case LN_QUELLART: in->quellart = v; break;   case LN_QUELLTYP: in->quelltyp = v; break;
    case LN_SRCREC: in->srcrec = v; break;       case LN_RMS: in->run_multiple_shots = v; break;
    case LN_READMOD: in->readmod = v; break;     case LN_L: in->l = v; break;
    case LN_FREE_SURF: in->free_surf = v; break; case LN_FW: in->fw = v; break;
    case LN_BOUNDARY: in->boundary = v; break;   case LN_SEISMO: in->seismo = v; break;
    case LN_READREC: in->readrec = v; break;     case LN_NDT: in->ndt = v; break;
    case LN_SEIS_FORMAT: in->seis_format = v; break; case LN_INVMAT1: in->invmat1 = v; break;
    case LN_INVMAT: in->invmat = v; break;       case LN_QUELLTYPB: in->quelltypb = v; break;
    case LN_HESSIAN: in->hessian = v; break;     case LN_GRAD_METHOD: in->grad_method = v; break;
    case LN_LNORM: in->lnorm = v; break;         case LN_DTINV: in->dtinv = v; break;
    default: break;
    }
}

static void set_float(dsh_inp *in, int line, float v)
{
    switch (line) {
    case LN_DH: in->dh = v; break;           case LN_TIME: in->time = v; break;
    case LN_DT: in->dt = v; break;           case LN_ANGLE: in->angle = v; break;
    case LN_PWD: in->plane_wave_depth = v; break; case LN_PHI: in->phi = v; break;
    case LN_TS: in->ts = v; break;           case LN_TAU: in->tau = v; break;
    case LN_DAMPING: in->damping = v; break; case LN_FPML: in->fpml = v; break;
    case LN_NPOWER: in->npower = v; break;   case LN_KMAX: in->k_max_pml = v; break;
    case LN_FC_HESSIAN: in->fc_hessian = v; break;
    default: break;
    }
}

static void set_string(dsh_inp *in, int line, const char *v)
{
    char *dst = NULL;
    switch (line) {
    case LN_SIGNAL_FILE: dst = in->signal_file; break; case LN_SOURCE_FILE: dst = in->source_file; break;
    case LN_MFILE: dst = in->mfile; break;             case LN_REC_FILE: dst = in->rec_file; break;
    case LN_SEIS_FILE_VY: dst = in->seis_file_vy; break; case LN_DATA_DIR: dst = in->data_dir; break;
    default: return;
    }
    strncpy(dst, v, DSH_PATH - 1);
    dst[DSH_PATH - 1] = 0;
}

int dsh_read_inp(const char *path, dsh_inp *out)
{
    FILE *fp;
    int c, line = 0, k;
    const int nlines = (int)strlen(INP_SCHEMA);
    char key[1024], sval[1024];
    if (!path || !out) return DSH_ERR_PARAM;
    fp = fopen(path, "r");
    if (!fp) return DSH_ERR_PARAM;
    inp_defaults(out);
    /* a parameter follows every newline whose next character is not '#';
     * that character is consumed and the key text is not interpreted */
    while ((c = getc(fp)) != EOF) {
        if (c != '\n' || getc(fp) == '#') continue;
        line++;
        if (line > nlines) continue;
        switch (INP_SCHEMA[line - 1]) {
        case 'i': {
            int v;
            if (fscanf(fp, "%1023s =%i", key, &v) == 2) set_int(out, line, v);
            break;
        }
        case 'f': {
            float v;
            if (fscanf(fp, "%1023s =%f", key, &v) == 2) set_float(out, line, v);
            break;
        }
        case 's':
            if (fscanf(fp, "%1023s =%1023s", key, sval) == 2) set_string(out, line, sval);
            break;
        case 'L': {
            float v;
            if (fscanf(fp, "%1023s =%f", key, &v) == 2) out->fl[0] = v;
            for (k = 2; k <= out->l && k <= 8; k++)
                if (fscanf(fp, "%f", &v) == 1) out->fl[k - 1] = v;
            break;
        }
        case 'F': {
            float a, b;
            if (fscanf(fp, "%1023s =%f ,%f", key, &a, &b) == 3 && line == LN_REFREC) {
                out->refrec[0] = a;
                out->refrec[1] = b;
            }
            break;
        }
        case 'A': {
            int a, b, cc, d;
            (void)!fscanf(fp, "%1023s =%i, %i, %i, %i", key, &a, &b, &cc, &d);
            break;
        }
        case 'B': {
            int a, b, cc;
            (void)!fscanf(fp, "%1023s =%i, %i, %i", key, &a, &b, &cc);
            break;
        }
        default: break;
        }
    }
    fclose(fp);
    out->lines = line;
    return (out->nx > 0 && out->ny > 0) ? DSH_OK : DSH_ERR_PARAM;
}

/* ---------------- JSON ---------------- */

/* Next "key" : value pair of a flat JSON object; value copied as text. */
static const char *json_pair(const char *p, char *key, size_t nk, char *val, size_t nv)
{
    size_t n;
    while (*p && *p != '"') p++;
    if (!*p) return NULL;
    p++;
    for (n = 0; *p && *p != '"'; p++)
        if (n + 1 < nk) key[n++] = *p;
    key[n] = 0;
    if (!*p) return NULL;
    p++;
    while (*p && isspace((unsigned char)*p)) p++;
    if (*p != ':') return p;
    p++;
    while (*p && isspace((unsigned char)*p)) p++;
    n = 0;
    if (*p == '"') {
        for (p++; *p && *p != '"'; p++)
            if (n + 1 < nv) val[n++] = *p;
        if (*p) p++;
    } else {
        for (; *p && *p != ',' && *p != '}' && *p != '\n'; p++)
            if (n + 1 < nv) val[n++] = *p;
        while (n > 0 && isspace((unsigned char)val[n - 1])) n--;
    }
    val[n] = 0;
    return p;
}

int dsh_read_json(const char *path, dsh_inp *out)
{
    FILE *fp;
    long len;
    char *buf, key[256], val[DSH_PATH];
    const char *p;
    static const struct { const char *k; char t; int line; } map[] = {
        {"NPROCX", 'i', LN_NPROCX}, {"NPROCY", 'i', LN_NPROCY}, {"FDORDER", 'i', LN_FDORDER},
        {"MAXRELERROR", 'i', LN_MAXRELERROR}, {"NX", 'i', LN_NX}, {"NY", 'i', LN_NY}, {"DH", 'f', LN_DH},
        {"TIME", 'f', LN_TIME}, {"DT", 'f', LN_DT}, {"QUELLART", 'i', LN_QUELLART}, {"QUELLTYP", 'i', LN_QUELLTYP},
        {"ANGLE", 'f', LN_ANGLE}, {"PLANE_WAVE_DEPTH", 'f', LN_PWD}, {"PHI", 'f', LN_PHI},
        {"SIGNAL_FILE", 's', LN_SIGNAL_FILE}, {"TS", 'f', LN_TS}, {"SRCREC", 'i', LN_SRCREC},
        {"SOURCE_FILE", 's', LN_SOURCE_FILE}, {"RUN_MULTIPLE_SHOTS", 'i', LN_RMS}, {"READMOD", 'i', LN_READMOD},
        {"MFILE", 's', LN_MFILE}, {"L", 'i', LN_L}, {"TAU", 'f', LN_TAU}, {"FREE_SURF", 'i', LN_FREE_SURF},
        {"FW", 'i', LN_FW}, {"DAMPING", 'f', LN_DAMPING}, {"FPML", 'f', LN_FPML}, {"BOUNDARY", 'i', LN_BOUNDARY},
        {"SEISMO", 'i', LN_SEISMO}, {"READREC", 'i', LN_READREC}, {"REC_FILE", 's', LN_REC_FILE},
        {"NDT", 'i', LN_NDT}, {"SEIS_FORMAT", 'i', LN_SEIS_FORMAT}, {"SEIS_FILE_VY", 's', LN_SEIS_FILE_VY},
        {"DATA_DIR", 's', LN_DATA_DIR}, {"INVMAT1", 'i', LN_INVMAT1}, {"INVMAT", 'i', LN_INVMAT},
        {"QUELLTYPB", 'i', LN_QUELLTYPB}, {"npower", 'f', LN_NPOWER}, {"k_max_PML", 'f', LN_KMAX},
        {"HESSIAN", 'i', LN_HESSIAN}, {"FC_HESSIAN", 'f', LN_FC_HESSIAN}, {"GRAD_METHOD", 'i', LN_GRAD_METHOD},
        {"LNORM", 'i', LN_LNORM}, {"DTINV", 'i', LN_DTINV},
    };
    if (!path || !out) return DSH_ERR_PARAM;
    fp = fopen(path, "rb");
    if (!fp) return DSH_ERR_PARAM;
    fseek(fp, 0, SEEK_END);
    len = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    buf = (char *)malloc((size_t)len + 1);
    if (!buf) { fclose(fp); return DSH_ERR_PARAM; }
    if (fread(buf, 1, (size_t)len, fp) != (size_t)len) { free(buf); fclose(fp); return DSH_ERR_PARAM; }
    buf[len] = 0;
    fclose(fp);
    inp_defaults(out);
    for (p = buf; (p = json_pair(p, key, sizeof key, val, sizeof val)) != NULL;) {
        size_t m;
        int handled = 0;
        for (m = 0; m < sizeof map / sizeof map[0]; m++) {
            if (strcmp(key, map[m].k) != 0) continue;
            if (map[m].t == 'i') set_int(out, map[m].line, atoi(val));
            else if (map[m].t == 'f') set_float(out, map[m].line, (float)atof(val));
            else set_string(out, map[m].line, val);
            handled = 1;
        }
        if (!handled) {
            if (strncmp(key, "FL", 2) == 0 && isdigit((unsigned char)key[2])) {
                int idx = atoi(key + 2);
                if (idx >= 1 && idx <= 8) out->fl[idx - 1] = (float)atof(val);
            } else if (strcmp(key, "REFRECX") == 0) {
                out->refrec[0] = (float)atof(val);
            } else if (strcmp(key, "REFRECY") == 0) {
                out->refrec[1] = (float)atof(val);
            }
        }
    }
    free(buf);
    return (out->nx > 0 && out->ny > 0) ? DSH_OK : DSH_ERR_PARAM;
}

int dsh_inp_params(const dsh_inp *in, dsh_params *p)
{
    int l;
    if (!in || !p) return DSH_ERR_PARAM;
    dsh_params_default(p);
    p->nx = in->nx; p->ny = in->ny; p->dh = in->dh; p->dt = in->dt;
    p->nt = (in->dt > 0) ? iround_f(in->time / in->dt) : 0;
    p->fdorder = in->fdorder; p->maxrelerror = in->maxrelerror; p->fw = in->fw; p->free_surf = in->free_surf;
    p->damping = in->damping; p->fpml = in->fpml; p->npower = in->npower; p->k_max_pml = in->k_max_pml;
    p->l = in->l;
    for (l = 0; l < 8; l++) p->fl[l] = in->fl[l];
    p->quellart = in->quellart;
    if (in->nprocx != 1 || in->nprocy != 1 || in->boundary != 0) return DSH_ERR_PARAM;
    return DSH_OK;
}

int dsh_read_workflow(const char *path, int stage, dsh_stage *out)
{
    FILE *fp;
    char str[256];
    int k;
    dsh_stage s;
    if (!path || !out || stage < 1) return DSH_ERR_PARAM;
    fp = fopen(path, "r");
    if (!fp) return DSH_ERR_PARAM;
    for (k = 0; k < 24; k++)
        if (fscanf(fp, "%255s", str) != 1) { fclose(fp); return DSH_ERR_PARAM; }
    for (k = 1; k <= stage; k++) {
        if (fscanf(fp, "%f%i%f%f%i%i%f%f%f%i%i%i%i%f%f%i%i%i%f%f%i%i%f%f", &s.pro, &s.time_filt, &s.fc_start,
                   &s.fc_end, &s.order, &s.timewin, &s.gamma, &s.twlength_minus, &s.twlength_plus, &s.inv_vp_iter,
                   &s.inv_vs_iter, &s.inv_rho_iter, &s.spatfilter, &s.wd_damp1, &s.wd_damp, &s.eprecond, &s.lnorm,
                   &s.inv_stf, &s.offsetc_stf, &s.eps_stf, &s.normalize, &s.offset_mute, &s.offsetc,
                   &s.scalerho) != 24) {
            fclose(fp);
            return DSH_ERR_PARAM;
        }
    }
    fclose(fp);
    *out = s;
    return DSH_OK;
}

/* ---------------- sources and receivers ---------------- */

int dsh_read_sources(const char *path, float dh, int nx, int ny, int max, int *nsrc, float *srcpos8, float *srcpos_m)
{
    FILE *fp;
    char line[256];
    int n = 0, l, kept = 0;
    if (!path || !nsrc || !srcpos8 || max < 1 || !(dh > 0)) return DSH_ERR_PARAM;
    fp = fopen(path, "r");
    if (!fp) return DSH_ERR_PARAM;
    if (fscanf(fp, "%d", &n) != 1 || n < 0) { fclose(fp); return DSH_ERR_PARAM; }
    rewind(fp);
    if (!fgets(line, sizeof line, fp)) { fclose(fp); return DSH_ERR_PARAM; }
    for (l = 0; l < n; l++) {
        float x, z, y, tshift, fc, amp, angle = 0.0f, type = 0.0f;   /* missing columns stay 0 (src/sources.c:49-62) */
        int nv, i, j;
        if (!fgets(line, sizeof line, fp)) { fclose(fp); return DSH_ERR_PARAM; }
        nv = sscanf(line, "%f%f%f%f%f%f%f%f", &x, &z, &y, &tshift, &fc, &amp, &angle, &type);
        if (nv < 6) { fclose(fp); return DSH_ERR_PARAM; }        /* sources.c:49-62: tshift, fc, amp required */
        if (nv == 6) angle = 0.0f;
        (void)z;
        i = iround_f(x / dh);
        j = iround_f(y / dh);
        /* one-rank splitsrc: keep a source when its rank coordinate is 0 */
        if ((i - 1) / nx != 0 || (j - 1) / ny != 0) continue;
        if (kept >= max) { fclose(fp); return DSH_ERR_PARAM; }
        srcpos8[0 * max + kept] = (float)(((i - 1) % nx) + 1);
        srcpos8[1 * max + kept] = (float)(((j - 1) % ny) + 1);
        srcpos8[2 * max + kept] = 0.0f;
        srcpos8[3 * max + kept] = tshift;
        srcpos8[4 * max + kept] = fc;
        srcpos8[5 * max + kept] = amp;
        srcpos8[6 * max + kept] = angle;
        srcpos8[7 * max + kept] = type;
        if (srcpos_m) { srcpos_m[kept] = x; srcpos_m[max + kept] = y; }
        kept++;
    }
    fclose(fp);
    *nsrc = kept;
    return DSH_OK;
}

int dsh_read_receivers(const char *path, float dh, const float refrec[2], int max, int *ntr, int *recpos)
{
    FILE *fp;
    int c, lines = 0, k, m, kept = 0;
    int *ii, *jj;
    float rx = refrec ? refrec[0] : 0.0f, ry = refrec ? refrec[1] : 0.0f;
    if (!path || !ntr || !recpos || max < 1 || !(dh > 0)) return DSH_ERR_PARAM;
    fp = fopen(path, "r");
    if (!fp) return DSH_ERR_PARAM;
    while ((c = fgetc(fp)) != EOF)
        if (c == '\n') ++lines;
    rewind(fp);
    ii = (int *)malloc(sizeof(int) * (size_t)(lines + 1));
    jj = (int *)malloc(sizeof(int) * (size_t)(lines + 1));
    if (!ii || !jj) { free(ii); free(jj); fclose(fp); return DSH_ERR_PARAM; }
    for (k = 0; k < lines; k++) {
        float x, y;
        if (fscanf(fp, "%f%f\n", &x, &y) != 2) { free(ii); free(jj); fclose(fp); return DSH_ERR_PARAM; }
        ii[k] = iround_f((x + rx) / dh);
        jj[k] = iround_f((y + ry) / dh);
    }
    fclose(fp);
    for (k = 0; k < lines; k++) {            /* later duplicates of a grid point are dropped */
        int dup = 0;
        for (m = 0; m < k && !dup; m++) dup = (ii[m] == ii[k] && jj[m] == jj[k]);
        if (dup) continue;
        if (kept >= max) { free(ii); free(jj); return DSH_ERR_PARAM; }
        recpos[kept] = ii[k];
        recpos[max + kept] = jj[k];
        kept++;
    }
    free(ii);
    free(jj);
    *ntr = kept;
    return DSH_OK;
}

/* ---------------- model files ---------------- */

static int read_xmajor(const char *path, int nx, int ny, float *dst, int transform_qs)
{
    FILE *fp = fopen(path, "rb");
    int i, j;
    if (!fp) return DSH_ERR_PARAM;
    for (i = 0; i < nx; i++)
        for (j = 0; j < ny; j++) {
            float v;
            if (fread(&v, sizeof(float), 1, fp) != 1) { fclose(fp); return DSH_ERR_PARAM; }
            dst[(size_t)j * nx + i] = v;
        }
    (void)transform_qs;
    fclose(fp);
    return DSH_OK;
}

int dsh_read_model(const char *mfile, int nx, int ny, int l, float *vs, float *rho, float *qs)
{
    char path[DSH_PATH + 16];
    int rc;
    if (!mfile || nx < 1 || ny < 1 || !vs || !rho || (l > 0 && !qs)) return DSH_ERR_PARAM;
    snprintf(path, sizeof path, "%s.vs", mfile);
    if ((rc = read_xmajor(path, nx, ny, vs, 0)) != DSH_OK) return rc;
    snprintf(path, sizeof path, "%s.rho", mfile);
    if ((rc = read_xmajor(path, nx, ny, rho, 0)) != DSH_OK) return rc;
    if (l > 0) {
        snprintf(path, sizeof path, "%s.qs", mfile);
        if ((rc = read_xmajor(path, nx, ny, qs, 1)) != DSH_OK) return rc;
    }
    return DSH_OK;
}

int dsh_write_model(const char *path, int nx, int ny, const float *field)
{
    FILE *fp;
    int i, j;
    if (!path || !field || nx < 1 || ny < 1) return DSH_ERR_PARAM;
    fp = fopen(path, "wb");
    if (!fp) return DSH_ERR_PARAM;
    for (i = 0; i < nx; i++)
        for (j = 0; j < ny; j++)
            if (fwrite(&field[(size_t)j * nx + i], sizeof(float), 1, fp) != 1) { fclose(fp); return DSH_ERR_PARAM; }
    fclose(fp);
    return DSH_OK;
}

int dsh_builtin_model(int l, int nx, int ny, float dh, float *vs, float *rho, float *qs)
{
    int i, j;
    if (l < 0 || nx < 1 || ny < 1 || !vs || !rho || (l > 0 && !qs)) return DSH_ERR_PARAM;
    for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++) {
            const size_t k = (size_t)j * nx + i;
            if (l > 0) {
                /* model_grad_visc.c:21,46: float constants, float arithmetic */
                const float grad0 = 2.80f, vs0 = 170.0f;
                vs[k] = grad0 * ((float)j * dh) + vs0;
                rho[k] = 1900.0f;
                qs[k] = 10.0f;
            } else {
                vs[k] = 164.0f;
                rho[k] = 1900.0f;
                if (qs) qs[k] = 0.0f;
            }
        }
    return DSH_OK;
}

/* ---------------- SU ---------------- */

static void put_i32(unsigned char *h, int off, int v) { memcpy(h + off, &v, 4); }
static void put_i16(unsigned char *h, int off, short v) { memcpy(h + off, &v, 2); }
static void put_u16(unsigned char *h, int off, unsigned short v) { memcpy(h + off, &v, 2); }
static void put_f32(unsigned char *h, int off, float v) { memcpy(h + off, &v, 4); }

int dsh_write_su(const char *path, int ntr, int ns, const float *section, const int *recpos, const int *tracl,
                 float xs, float ys, float dh, float dt, int ndt, const float refrec[2])
{
    /* 240-byte SU trace header, standard field offsets */
    enum { TRACL = 0, EP = 16, CDP = 20, TRID = 28, OFFSET = 36, GELEV = 40, SDEPTH = 48, SWDEP = 60,
           SCALEL = 68, SCALCO = 70, SX = 72, SY = 76, GX = 80, GY = 84, NS = 114, DT = 116, D1 = 180 };
    const float xshift = 800.0f, yshift = 800.0f;
    const double pi = 3.141592653589793;
    FILE *fp;
    int k;
    float rx = refrec ? refrec[0] : 0.0f, ry = refrec ? refrec[1] : 0.0f;
    if (!path || !section || !recpos || ntr < 0 || ns < 1 || ndt < 1) return DSH_ERR_PARAM;
    fp = fopen(path, "wb");
    if (!fp) return DSH_ERR_PARAM;
    for (k = 0; k < ntr; k++) {
        unsigned char h[240];
        const float *tr = section + (size_t)k * ns;
        const float xr = recpos[k] * dh, yr = recpos[ntr + k] * dh;
        const float x = xr - rx, y = yr - ry;
        const int num = tracl ? tracl[k] : k + 1;
        unsigned short dtus;
        memset(h, 0, sizeof h);
        put_i32(h, TRACL, num);
        put_i32(h, CDP, num);
        put_i32(h, EP, 0);
        put_i16(h, TRID, 1);
        put_i32(h, OFFSET, (int)floor(sqrt((xs - xr) * (xs - xr) + (ys - yr) * (ys - yr)) * 1000.0 + 0.5));
        put_i32(h, GELEV, (int)floor(yr * 1000.0 + 0.5));
        put_i32(h, SDEPTH, (int)floor(ys * 1000.0 + 0.5));
        put_i32(h, SWDEP, (int)floor(((360.0 / (2.0 * pi)) * atan2(x - xshift, y - yshift)) * 1000.0 + 0.5));
        put_i16(h, SCALEL, (short)-1000);
        put_i16(h, SCALCO, (short)-1000);
        put_i32(h, SX, (int)floor(xs * 1000.0 + 0.5));
        put_i32(h, SY, (int)floor(ys * 1000.0 + 0.5));
        put_i32(h, GX, (int)floor(xr * 1000.0 + 0.5));
        put_i32(h, GY, (int)floor(yr * 1000.0 + 0.5));
        put_u16(h, NS, (unsigned short)ns);
        dtus = (unsigned short)floor(((float)ndt * dt) * 1.0e6 + 0.5);
        put_u16(h, DT, dtus);
        put_f32(h, D1, (float)dtus * 1.0e-6);
        if (fwrite(h, 240, 1, fp) != 1 || fwrite(tr, sizeof(float), (size_t)ns, fp) != (size_t)ns) {
            fclose(fp);
            return DSH_ERR_PARAM;
        }
    }
    fclose(fp);
    return DSH_OK;
}

int dsh_read_su(const char *path, int ntr, int ns, float *section)
{
    FILE *fp;
    int k;
    if (!path || !section || ntr < 0 || ns < 1) return DSH_ERR_PARAM;
    fp = fopen(path, "rb");
    if (!fp) return DSH_ERR_PARAM;
    for (k = 0; k < ntr; k++) {
        unsigned char h[240];
        float *tr = section + (size_t)k * ns;
        if (fread(h, 240, 1, fp) != 1 || fread(tr, sizeof(float), (size_t)ns, fp) != (size_t)ns) {
            fclose(fp);
            return DSH_ERR_PARAM;
        }
        tr[0] = 0.0f;
    }
    fclose(fp);
    return DSH_OK;
}

/*
 * dsh_compat.cu — reference-signature layer (libdsh_compat.so).
 *
 * Exports the reference's own hot-path functions with their exact names and
 * signatures (src/fd.h), reading the same global parameters the reference's
 * globvar.h defines, so the reference program can be relinked against this
 * library instead of its CPU loops: update_v_PML, update_s_elastic_PML,
 * update_s_visc_PML, seismo_ssg, eprecond, eprecond1, hess_save, hessian,
 * zero_fdveps, zero_fdveps_visc, psource.
 *
 * The velocity and stress updates and eprecond copy the Numerical-Recipes
 * arrays they touch to the device, run the same sm_100a kernels as the
 * resident engine for one step (with the reference's side outputs vyp1 / uy /
 * uyx), and copy the results back; the bookkeeping functions (seismo_ssg,
 * hess_save, hessian, eprecond1, zero_fdveps*, psource) are host loops with
 * the reference's arithmetic.
 * That round trip makes it a parity and migration layer, not the fast path
 * (include/dsh.h keeps the wavefields resident).  Supported like the
 * one-rank program: NPROCX = NPROCY = 1, BOUNDARY = 0, GRAD_FORM = 2, the full
 * grid range (nx1..nx2 = 1..NX, ny1..ny2 = 1..NY), L <= 4.  Unsupported
 * settings print a message on stderr and leave the arrays unchanged.
 */
#include "dsh.h"
#include "dsh_compat.h"
#include "dsh_dispatch.h"
#include "dsh_setup.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

using namespace dsh;

/* the reference's globals (defined by the program that links this library) */
extern "C" {
extern float DT, DH;
extern int NX, NY, NXG, FDORDER, FW, FREE_SURF, BOUNDARY, NPROCX, NPROCY, POS[3], GRAD_FORM, L, IDX, IDY;
extern int EPRECOND, QUELLTYP, QUELLTYPB, NT, MYID;
}

namespace {

struct Compat {
    int nx = 0, ny = 0, fdo = 0, fw = 0, l = 0, hy = 0, pitch = 0;
    long long fstride = 0, dstride = 0;
    float *buf = nullptr;                 /* all device arrays */
    float *vy, *sxy, *syz, *acc, *uy, *uyx, *brho, *c1, *c2, *dip, *d, *r, *q;
    float *pvx, *pvy, *psx, *psy, *pml;
    float *w1, *w2;
    int *ints = nullptr;                  /* [0] step counter, [1] status */
    std::vector<float> host;
};
Compat G;

int last_status = DSH_OK;                 /* first error since the last dsh_compat_status() */

/* Records an error for dsh_compat_status() and prints it.  With
 * DSH_COMPAT_ABORT=1 in the environment the run ends as the reference ends
 * it on a fatal error (src/util.c:7-15: the rank, a run-time error banner
 * and the message on stdout, then a non-zero exit, which an MPI launcher
 * turns into the abort of the whole job). */
void fail(int code, const char *msg)
{
    if (last_status == DSH_OK) last_status = code;
    fprintf(stderr, "dsh compat: %s\n", msg);
    static const bool abort_mode = getenv("DSH_COMPAT_ABORT") && atoi(getenv("DSH_COMPAT_ABORT")) != 0;
    if (abort_mode) {
        fprintf(stdout, "Message from PE %d\n", MYID);
        fprintf(stdout, "R U N - T I M E  E R R O R: \n");
        fprintf(stdout, "%s\n", msg);
        fprintf(stdout, "...now exiting to system.\n");
        fflush(stdout);
        exit(1);
    }
}

void release()
{
    cudaFree(G.buf);
    cudaFree(G.ints);
    G.buf = nullptr;
    G.ints = nullptr;
    G.nx = 0;
}

bool supported(const char *fn, int nx1, int nx2, int ny1, int ny2)
{
    if (NPROCX != 1 || NPROCY != 1 || BOUNDARY != 0 || nx1 != 1 || ny1 != 1 || nx2 != NX || ny2 != NY ||
        FDORDER < 2 || FDORDER > 12 || (FDORDER & 1) || L < 0 || L > DSH_MAX_L || FW < 0 || FW > DSH_MAX_FW) {
        char msg[256];
        snprintf(msg, sizeof msg, "%s: only the one-rank full-grid configuration is supported "
                                  "(NPROCX=NPROCY=1, BOUNDARY=0, ranges 1..NX/1..NY, L<=4)", fn);
        fail(DSH_ERR_PARAM, msg);
        return false;
    }
    return true;
}

/* device arrays for the current NX, NY, FDORDER, FW, L */
bool ensure()
{
    if (G.buf && G.nx == NX && G.ny == NY && G.fdo == FDORDER && G.fw == FW && G.l == L) return true;
    release();
    G.nx = NX; G.ny = NY; G.fdo = FDORDER; G.fw = FW; G.l = L;
    G.hy = FDORDER / 2;
    G.pitch = (int)((NX + 32 + 31) / 32 * 32);
    G.fstride = ((long long)(NY + 2 * G.hy) * G.pitch + 31) / 32 * 32;
    G.dstride = ((long long)NY * G.pitch + 31) / 32 * 32;
    const long long psix = ((long long)NY * 2 * FW + 4 + 31) / 32 * 32, psiy = ((long long)2 * FW * G.pitch + 4 + 31) / 32 * 32;
    const long long vlen = 2 * DSH_MAX_FW + 1;
    const long long total = 6 * G.fstride + (5 + 4 * (long long)L + 2) * G.dstride + 2 * psix + 2 * psiy + 12 * vlen;
    if (cudaMalloc(&G.buf, total * sizeof(float)) != cudaSuccess || cudaMalloc(&G.ints, 2 * sizeof(int)) != cudaSuccess) {
        release();
        fail(DSH_ERR_OOM, "device allocation failed");
        return false;
    }
    cudaMemset(G.buf, 0, total * sizeof(float));
    cudaMemset(G.ints, 0, 2 * sizeof(int));
    float *p = G.buf;
    G.vy = p; p += G.fstride; G.sxy = p; p += G.fstride; G.syz = p; p += G.fstride;
    G.acc = p; p += G.fstride; G.uy = p; p += G.fstride; G.uyx = p; p += G.fstride;
    G.brho = p; p += G.dstride; G.c1 = p; p += G.dstride; G.c2 = p; p += G.dstride;
    G.w1 = p; p += G.dstride; G.w2 = p; p += G.dstride;
    G.dip = p; p += (long long)L * G.dstride; G.d = p; p += (long long)L * G.dstride;
    G.r = p; p += (long long)L * G.dstride; G.q = p; p += (long long)L * G.dstride;
    G.pvx = p; p += psix; G.psx = p; p += psix; G.pvy = p; p += psiy; G.psy = p; p += psiy;
    G.pml = p;
    return true;
}

/* ---- host <-> device transfers of NR arrays ---- */

/* haloed field: rows 1-h .. NY+h, columns 1-8 .. NX+8 of m (the caller's
 * arrays carry a halo of FDORDER/2+1 >= h rows/columns; columns beyond it stay 0) */
void put_haloed(float *dev, float **m, int halo_cols)
{
    const int h = G.hy;
    G.host.assign((size_t)G.fstride, 0.0f);
    for (int j = 1 - h; j <= NY + h; j++)
        for (int i = 1 - halo_cols; i <= NX + halo_cols; i++)
            G.host[(size_t)(j - 1 + h) * G.pitch + (i - 1 + HX)] = m[j][i];
    cudaMemcpy(dev, G.host.data(), (size_t)G.fstride * sizeof(float), cudaMemcpyHostToDevice);
}

void get_haloed(float **m, const float *dev, int halo_rows, int halo_cols)
{
    const int h = G.hy;
    G.host.resize((size_t)G.fstride);
    cudaMemcpy(G.host.data(), dev, (size_t)G.fstride * sizeof(float), cudaMemcpyDeviceToHost);
    for (int j = 1 - halo_rows; j <= NY + halo_rows; j++)
        for (int i = 1 - halo_cols; i <= NX + halo_cols; i++)
            m[j][i] = G.host[(size_t)(j - 1 + h) * G.pitch + (i - 1 + HX)];
}

void put_dense(float *dev, float **m)
{
    G.host.assign((size_t)G.dstride, 0.0f);
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) G.host[(size_t)(j - 1) * G.pitch + (i - 1 + HX)] = m[j][i];
    cudaMemcpy(dev, G.host.data(), (size_t)G.dstride * sizeof(float), cudaMemcpyHostToDevice);
}

void get_dense(float **m, const float *dev)
{
    G.host.resize((size_t)G.dstride);
    cudaMemcpy(G.host.data(), dev, (size_t)G.dstride * sizeof(float), cudaMemcpyDeviceToHost);
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) m[j][i] = G.host[(size_t)(j - 1) * G.pitch + (i - 1 + HX)];
}

/* f3tensor [j][i][l] (l = 1..L) <-> SoA [l][j][i] */
void put_tensor(float *dev, float ***t)
{
    G.host.assign((size_t)L * G.dstride, 0.0f);
    for (int l = 1; l <= L; l++)
        for (int j = 1; j <= NY; j++)
            for (int i = 1; i <= NX; i++)
                G.host[(size_t)(l - 1) * G.dstride + (size_t)(j - 1) * G.pitch + (i - 1 + HX)] = t[j][i][l];
    cudaMemcpy(dev, G.host.data(), (size_t)L * G.dstride * sizeof(float), cudaMemcpyHostToDevice);
}

void get_tensor(float ***t, const float *dev)
{
    G.host.resize((size_t)L * G.dstride);
    cudaMemcpy(G.host.data(), dev, (size_t)L * G.dstride * sizeof(float), cudaMemcpyDeviceToHost);
    for (int l = 1; l <= L; l++)
        for (int j = 1; j <= NY; j++)
            for (int i = 1; i <= NX; i++)
                t[j][i][l] = G.host[(size_t)(l - 1) * G.dstride + (size_t)(j - 1) * G.pitch + (i - 1 + HX)];
}

/* CPML memory: x strips m[1..NY][1..2FW], y strips m[1..2FW][1..NX] */
void put_psi_x(float *dev, float **m)
{
    if (FW <= 0) return;
    G.host.assign((size_t)NY * 2 * FW, 0.0f);
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= 2 * FW; i++) G.host[(size_t)(j - 1) * 2 * FW + (i - 1)] = m[j][i];
    cudaMemcpy(dev, G.host.data(), G.host.size() * sizeof(float), cudaMemcpyHostToDevice);
}
void get_psi_x(float **m, const float *dev)
{
    if (FW <= 0) return;
    G.host.resize((size_t)NY * 2 * FW);
    cudaMemcpy(G.host.data(), dev, G.host.size() * sizeof(float), cudaMemcpyDeviceToHost);
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= 2 * FW; i++) m[j][i] = G.host[(size_t)(j - 1) * 2 * FW + (i - 1)];
}
void put_psi_y(float *dev, float **m)
{
    if (FW <= 0) return;
    G.host.assign((size_t)2 * FW * G.pitch, 0.0f);
    for (int j = 1; j <= 2 * FW; j++)
        for (int i = 1; i <= NX; i++) G.host[(size_t)(j - 1) * G.pitch + (i - 1 + HX)] = m[j][i];
    cudaMemcpy(dev, G.host.data(), G.host.size() * sizeof(float), cudaMemcpyHostToDevice);
}
void get_psi_y(float **m, const float *dev)
{
    if (FW <= 0) return;
    G.host.resize((size_t)2 * FW * G.pitch);
    cudaMemcpy(G.host.data(), dev, G.host.size() * sizeof(float), cudaMemcpyDeviceToHost);
    for (int j = 1; j <= 2 * FW; j++)
        for (int i = 1; i <= NX; i++) m[j][i] = G.host[(size_t)(j - 1) * G.pitch + (i - 1 + HX)];
}

void put_pml(float *const v[12])
{
    const size_t vlen = 2 * DSH_MAX_FW + 1;
    G.host.assign(12 * vlen, 0.0f);
    for (int k = 0; k < 12; k++)
        if (v[k]) for (int i = 1; i <= 2 * FW; i++) G.host[k * vlen + i] = v[k][i];
    cudaMemcpy(G.pml, G.host.data(), G.host.size() * sizeof(float), cudaMemcpyHostToDevice);
}

StepArgs base_args(const float *hc)
{
    StepArgs a;
    memset(&a, 0, sizeof(a));
    a.nx = NX; a.ny = NY; a.pitch = G.pitch; a.hy = G.hy; a.fw = FW; a.free_surf = FREE_SURF; a.l = L;
    a.fd12_compat = 1;
    a.nt_last = 1 << 30; a.nt_total = 1 << 30; a.nt_base = G.ints;
    a.fstride = G.fstride; a.dstride = G.dstride; a.slot_stride = 0;
    for (int k = 0; k <= 6; k++) a.hc[k] = hc[k];
    a.dt = DT; a.dh = DH;
    a.inv_dh = (float)(1.0 / (double)DH);
    a.dhi_el = DT / DH;
    a.dhi_visc = (float)(1.0 / (double)DH);
    a.dthalbe = (float)((double)DT / 2.0);
    const size_t vlen = 2 * DSH_MAX_FW + 1;
    a.pml.K_x = G.pml; a.pml.a_x = G.pml + vlen; a.pml.b_x = G.pml + 2 * vlen;
    a.pml.K_x_half = G.pml + 3 * vlen; a.pml.a_x_half = G.pml + 4 * vlen; a.pml.b_x_half = G.pml + 5 * vlen;
    a.pml.K_y = G.pml + 6 * vlen; a.pml.a_y = G.pml + 7 * vlen; a.pml.b_y = G.pml + 8 * vlen;
    a.pml.K_y_half = G.pml + 9 * vlen; a.pml.a_y_half = G.pml + 10 * vlen; a.pml.b_y_half = G.pml + 11 * vlen;
    a.vy = G.vy; a.sxy = G.sxy; a.syz = G.syz; a.r = G.r; a.q = G.q;
    a.psi_vxx = G.pvx; a.psi_vyy_v = G.pvy; a.psi_sxx = G.psx; a.psi_syy = G.psy;
    a.brho = G.brho; a.uip = G.c1; a.ujp = G.c2; a.fipjp = G.c1; a.f = G.c2; a.dip = G.dip; a.d = G.d;
    a.fwd_mod = 1;
    a.status = G.ints + 1;
    return a;
}

bool launch(KFn fn, StepArgs &a)
{
    const int zero[2] = {0, 0};           /* step counter, status word */
    cudaMemcpy(G.ints, zero, sizeof(zero), cudaMemcpyHostToDevice);
    dim3 block(BX, BY, 1);
    dim3 grid((unsigned)((NX + 4 * BX - 1) / (4 * BX)), (unsigned)((NY + BY - 1) / BY), 1);
    int off = 1;                           /* the kernels read step = *nt_base + off */
    void *args[2] = {&a, &off};
    cudaError_t e = cudaLaunchKernel((const void *)fn, grid, block, args, 0, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof msg, "kernel failed (%s)", cudaGetErrorString(e));
        fail(DSH_ERR_CUDA, msg);
        return false;
    }
    int st = 0;
    cudaMemcpy(&st, G.ints + 1, sizeof(int), cudaMemcpyDeviceToHost);
    if (st) {   /* a non-finite stress or velocity (the reference's check at src/denise.c:1183-1185) */
        fail(DSH_ERR_UNSTABLE, " Simulation is unstable !");
        return false;
    }
    return true;
}

/* ordered point-source additions of one step (update_v_PML.c:564-583) */
__global__ void add_sources(float *vy, int pitch, int hy, int n, const int *ij, const float *val)
{
    for (int k = 0; k < n; k++) vy[(long long)(ij[2 * k + 1] - 1 + hy) * pitch + (ij[2 * k] - 1 + HX)] += val[k];
}

__global__ void energy_kernel(float *w, const float *vy, int nx, int ny, int pitch, int hy)
{
    const long long n = (long long)nx * ny;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nx), j = (int)(idx / nx);
        const float v = vy[(long long)(j + hy) * pitch + i + HX];
        float *p = w + (long long)j * pitch + i + HX;
        *p = *p + v * v;
    }
}

bool device_ok()
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
        fail(DSH_ERR_CUDA, "no CUDA device");
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

/* src/update_v_PML.c:12-16 */
void update_v_PML(int nx1, int nx2, int ny1, int ny2, int nt, float **vy, float **vyp1, float **vym1, float **utty,
                  float **syz, float **sxy, float **rho, float **srcpos_loc, float **signals1, int nsrc,
                  float **absorb_coeff, float *hc, int infoout, int sw, float *K_x, float *a_x, float *b_x,
                  float *K_x_half, float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                  float *K_y_half, float *a_y_half, float *b_y_half, float **psi_syy_y, float **psi_sxy_x)
{
    (void)vym1; (void)utty; (void)absorb_coeff; (void)infoout;
    if (!device_ok() || !supported("update_v_PML", nx1, nx2, ny1, ny2) || !ensure()) return;
    if (GRAD_FORM != 2 && sw == 1) {
        fail(DSH_ERR_PARAM, "update_v_PML: only GRAD_FORM=2 is supported");
        return;
    }
    const int H = G.hy;
    put_haloed(G.sxy, sxy, H);
    put_haloed(G.syz, syz, H);
    put_haloed(G.vy, vy, H);
    std::vector<float> b((size_t)NX * NY);
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) {
            float bb = 1.0 / rho[j][i];
            if (rho[j][i] < 1e-20) bb = 0.0;
            b[(size_t)(j - 1) * NX + (i - 1)] = bb;
        }
    cudaMemcpy2D(G.brho + HX, G.pitch * sizeof(float), b.data(), NX * sizeof(float), NX * sizeof(float), NY,
                 cudaMemcpyHostToDevice);
    put_psi_x(G.pvx, psi_sxy_x);
    put_psi_y(G.pvy, psi_syy_y);
    float *const v[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
    put_pml(v);
    int e;
    const bool p2 = DH > 0 && std::frexp(DH, &e) == 0.5f;
    KFn fn = v_kernel(FDORDER, VF_ACC_OUT | (sw == 1 ? VF_ADJOINT : 0), p2);
    StepArgs a = base_args(hc);
    a.out_acc = G.acc;
    if (!fn || !launch(fn, a)) return;
    /* injection after the update, in source order */
    std::vector<int> ij;
    std::vector<float> val;
    for (int l = 1; l <= nsrc; l++) {
        const int i = (int)srcpos_loc[1][l], j = (int)srcpos_loc[2][l];
        if (sw == 0) {
            QUELLTYP = (int)srcpos_loc[8][l];
            if (QUELLTYP != 3) continue;
        } else if (QUELLTYPB != 2) {
            continue;
        }
        ij.push_back(i); ij.push_back(j);
        val.push_back(signals1[l][nt]);
    }
    if (!val.empty()) {
        int *dij = nullptr;
        float *dval = nullptr;
        cudaMalloc(&dij, ij.size() * sizeof(int));
        cudaMalloc(&dval, val.size() * sizeof(float));
        cudaMemcpy(dij, ij.data(), ij.size() * sizeof(int), cudaMemcpyHostToDevice);
        cudaMemcpy(dval, val.data(), val.size() * sizeof(float), cudaMemcpyHostToDevice);
        add_sources<<<1, 1>>>(G.vy, G.pitch, G.hy, (int)val.size(), dij, dval);
        cudaDeviceSynchronize();
        cudaFree(dij);
        cudaFree(dval);
    }
    get_haloed(vy, G.vy, 1, 1);
    get_dense(vyp1, G.acc + (long long)G.hy * G.pitch);
    get_psi_x(psi_sxy_x, G.pvx);
    get_psi_y(psi_syy_y, G.pvy);
}

static void stress_common(const char *name, int nx1, int nx2, int ny1, int ny2, float **vy, float **uy, float **uyx,
                          float **syz, float **sxy, float *hc, float *const pml[12], float **psi_vyy, float **psi_vyx,
                          int l, float **c1, float **c2, float ***r, float ***q, float ***dip, float ***d,
                          const float *bip, const float *bjm, const float *cip, const float *cjm)
{
    if (!device_ok() || !supported(name, nx1, nx2, ny1, ny2) || !ensure()) return;
    put_haloed(G.vy, vy, G.hy);
    put_haloed(G.sxy, sxy, 0);
    put_haloed(G.syz, syz, 0);
    put_dense(G.c1, c1);
    put_dense(G.c2, c2);
    if (l > 0) {
        put_tensor(G.r, r);
        put_tensor(G.q, q);
        put_tensor(G.dip, dip);
        put_tensor(G.d, d);
    }
    put_psi_x(G.psx, psi_vyx);
    put_psi_y(G.psy, psi_vyy);
    put_pml(pml);
    KFn fn = s_kernel(FDORDER, l, SF_STRAIN_OUT | SF_PARAMS);
    StepArgs a = base_args(hc);
    for (int k = 0; k < l; k++) { a.bip[k] = bip[k + 1]; a.bjm[k] = bjm[k + 1]; a.cip[k] = cip[k + 1]; a.cjm[k] = cjm[k + 1]; }
    a.out_uy = G.uy;
    a.out_uyx = G.uyx;
    if (!fn || !launch(fn, a)) return;
    get_haloed(sxy, G.sxy, 0, 0);
    get_haloed(syz, G.syz, 0, 0);
    if (GRAD_FORM == 2) {
        get_haloed(uy, G.uy, 0, 0);
        get_haloed(uyx, G.uyx, 0, 0);
    }
    if (l > 0) {
        get_tensor(r, G.r);
        get_tensor(q, G.q);
    }
    get_psi_x(psi_vyx, G.psx);
    get_psi_y(psi_vyy, G.psy);
}

/* src/update_s_elastic_PML.c:12-16 (the program passes (pu, puip, pujp) as (u, uip, ujp)) */
void update_s_elastic_PML(int nx1, int nx2, int ny1, int ny2, float **vy, float **uy, float **uyx, float **syz,
                          float **sxy, float **u, float **uip, float **ujp, float **absorb_coeff, float **rho,
                          float *hc, int infoout, float *K_x, float *a_x, float *b_x, float *K_x_half,
                          float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y, float *K_y_half,
                          float *a_y_half, float *b_y_half, float **psi_vyy, float **psi_vyx)
{
    (void)u; (void)absorb_coeff; (void)rho; (void)infoout;
    float *const v[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
    stress_common("update_s_elastic_PML", nx1, nx2, ny1, ny2, vy, uy, uyx, syz, sxy, hc, v, psi_vyy, psi_vyx, 0, uip,
                  ujp, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
}

/* src/update_s_visc_PML.c:12-17 */
void update_s_visc_PML(int nx1, int nx2, int ny1, int ny2, float **vy, float **uy, float **uyx, float **syz,
                       float **sxy, float **ujp, float **uip, float **rho, float *hc, int infoout, float ***r,
                       float ***p, float ***q, float **fipjp, float **f, float **g, float *bip, float *bjm,
                       float *cip, float *cjm, float ***d, float ***e, float ***dip, float *K_x, float *a_x,
                       float *b_x, float *K_x_half, float *a_x_half, float *b_x_half, float *K_y, float *a_y,
                       float *b_y, float *K_y_half, float *a_y_half, float *b_y_half, float **psi_vyy,
                       float **psi_vyx)
{
    (void)ujp; (void)uip; (void)rho; (void)infoout; (void)p; (void)g; (void)e;
    float *const v[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
    stress_common("update_s_visc_PML", nx1, nx2, ny1, ny2, vy, uy, uyx, syz, sxy, hc, v, psi_vyy, psi_vyx, L, fipjp, f,
                  r, q, dip, d, bip, bjm, cip, cjm);
}

/* src/seismo_ssg.c:9 (SEISMO=1: vertical velocity) */
void seismo_ssg(int lsamp, int ntr, int **recpos, float **sectionvy, float **vy, float **syy, float **u, float *hc)
{
    (void)syy; (void)u; (void)hc;
    for (int itr = 1; itr <= ntr; itr++) sectionvy[itr][lsamp] = vy[recpos[2][itr]][recpos[1][itr]];
}

/* src/eprecond.c:2-15: W += vy^2 over the grid */
void eprecond(float **W, float **vy)
{
    if (!device_ok() || !ensure()) return;
    if (IDX != 1 || IDY != 1) {
        for (int i = 1; i <= NX; i += IDX)
            for (int j = 1; j <= NY; j += IDY) W[j][i] += vy[j][i] * vy[j][i];
        return;
    }
    put_dense(G.w1, W);
    put_haloed(G.vy, vy, 0);
    energy_kernel<<<296, 256>>>(G.w1, G.vy, NX, NY, G.pitch, G.hy);
    cudaDeviceSynchronize();
    get_dense(W, G.w1);
}

/* src/eprecond1.c:2-73 */
void eprecond1(float **We, float **Ws, float **Wr)
{
    float maxWe = 0.0f;
    const float eps = 0.005f, xmin = DH, xmax = NXG * DH;
    for (int i = 1; i <= NX; i += IDX)
        for (int j = 1; j <= NY; j += IDY) {
            if (EPRECOND == 1) We[j][i] = std::sqrt((double)(Ws[j][i] * Wr[j][i]));
            if (EPRECOND == 3) {
                const int ii = i + POS[1] * NX, jj = j + POS[2] * NY;
                const float x = ii * DH, y = jj * DH;
                We[j][i] = std::sqrt((double)Ws[j][i]) *
                           (std::asinh((double)((xmax - x) / y)) - std::asinh((double)((xmin - x) / y)));
            }
            if (We[j][i] > maxWe) maxWe = We[j][i];
        }
    for (int i = 1; i <= NX; i += IDX)
        for (int j = 1; j <= NY; j += IDY) We[j][i] = We[j][i] + (eps * maxWe);
}

/* src/hess_save.c:2-17 */
void hess_save(int nt, float **uy, float **uyx, float **vyp1, float ***hess_eyy, float ***hess_eyx,
               float ***hess_utty)
{
    for (int i = 1; i <= NX; i += IDX)
        for (int j = 1; j <= NY; j += IDY) {
            hess_eyy[j][i][nt] = uy[j][i];
            hess_eyx[j][i][nt] = 0.5 * uyx[j][i];
            hess_utty[j][i][nt] = vyp1[j][i];
        }
}

/* src/hessian.c:91-94 */
void hessian(int NTDTINV, float ***hess_eyy, float ***hess_eyx, float ***hess_utty, float **hessian_u,
             float **hessian_rho)
{
    for (int i = 1; i <= NX; i += IDX)
        for (int j = 1; j <= NY; j += IDY)
            for (int nt = 1; nt < NTDTINV; nt++) {
                hessian_u[j][i] += (hess_eyy[j][i][nt] * hess_eyy[j][i][nt]) + (hess_eyx[j][i][nt] * hess_eyx[j][i][nt]);
                hessian_rho[j][i] += (hess_utty[j][i][nt] * hess_utty[j][i][nt]);
            }
}

/* src/zero_fdveps.c:11-52 */
void zero_fdveps(int ny1, int ny2, int nx1, int nx2, float **vy, float **syy, float **sxy, float **vym1,
                 float **vyp1, float **psi_sxy_x, float **psi_vyx, float **psi_syy_y, float **psi_vyy)
{
    for (int j = ny1; j <= ny2; j++)
        for (int i = nx1; i <= nx2; i++) vy[j][i] = syy[j][i] = sxy[j][i] = vym1[j][i] = vyp1[j][i] = 0.0f;
    for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= 2 * FW; i++) psi_sxy_x[j][i] = psi_vyx[j][i] = 0.0f;
    for (int j = 1; j <= 2 * FW; j++)
        for (int i = 1; i <= NX; i++) psi_syy_y[j][i] = psi_vyy[j][i] = 0.0f;
}

/* src/zero_fdveps_visc.c:11-64 */
void zero_fdveps_visc(int ny1, int ny2, int nx1, int nx2, float **vy, float **syy, float **sxy, float **vym1,
                      float **vyp1, float **psi_sxy_x, float **psi_vyx, float **psi_syy_y, float **psi_vyy,
                      float ***pr, float ***pp, float ***pq)
{
    zero_fdveps(ny1, ny2, nx1, nx2, vy, syy, sxy, vym1, vyp1, psi_sxy_x, psi_vyx, psi_syy_y, psi_vyy);
    for (int j = ny1; j <= ny2; j++)
        for (int i = nx1; i <= nx2; i++)
            for (int l = 1; l <= L; l++) pr[j][i][l] = pp[j][i][l] = pq[j][i][l] = 0.0f;
}

/* src/psource.c:9-38: P-SV explosive source (not used by the SH program) */
void psource(int nt, float **sxx, float **syy, float **srcpos_loc, float **signals, int nsrc)
{
    for (int l = 1; l <= nsrc; l++) {
        const int i = (int)srcpos_loc[1][l], j = (int)srcpos_loc[2][l];
        float amp = 0.0f;
        if (nt == 1) amp = signals[l][nt + 1] / DT;
        if ((nt > 1) && (nt < NT)) amp = (signals[l][nt + 1] - signals[l][nt - 1]) / DT;
        if (nt == NT) amp = -signals[l][nt - 1] / DT;
        sxx[j][i] += amp;
        syy[j][i] += amp;
    }
}

}  /* extern "C" */

extern "C" int dsh_compat_status(void)
{
    const int st = last_status;
    last_status = DSH_OK;
    return st;
}

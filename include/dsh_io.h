/*
 * dsh_io.h — the reference's file formats, read and written by this
 * library's own code (host C), so existing DENISE-SH inputs drive the engine
 * and its outputs feed the reference's tools:
 *   .inp parameter file   positional "key = value" lines (src/read_par.c:80-470)
 *   .json parameter file  flat "KEY" : "value" pairs (src/read_par_json.c)
 *   workflow table        24 columns per FWI stage (src/read_par_inv.c:31-34)
 *   source file           nsrc, then x z y tshift fc amp angle type (src/sources.c:37-62)
 *   receiver file         x y per line, duplicates removed (src/receiver.c:25-72)
 *   model files           float32, x outer / depth inner (src/readmod.c:82-99)
 *   SU seismograms        240-byte trace header + samples (src/outseis_glob.c:45-265,
 *                         src/inseis.c:73-82)
 */
#ifndef DSH_IO_H
#define DSH_IO_H

#include "dsh.h"

#ifdef __cplusplus
extern "C" {
#endif

#define DSH_PATH 256

/* the parameters of a .inp / .json file that the hot path and its driver use */
typedef struct dsh_inp {
    int nprocx, nprocy, fdorder, maxrelerror, nx, ny;
    float dh, time, dt;
    int quellart, quelltyp;
    float angle, plane_wave_depth, phi;
    char signal_file[DSH_PATH];
    float ts;
    int srcrec;
    char source_file[DSH_PATH];
    int run_multiple_shots, readmod;
    char mfile[DSH_PATH];
    int l;
    float fl[8], tau;
    int free_surf, fw;
    float damping, fpml;
    int boundary, seismo, readrec;
    char rec_file[DSH_PATH];
    float refrec[2];
    int ndt, seis_format;
    char seis_file_vy[DSH_PATH], data_dir[DSH_PATH];
    int invmat1, invmat, quelltypb;
    float npower, k_max_pml;
    int hessian;
    float fc_hessian;
    int grad_method, lnorm, dtinv;
    int lines;                 /* parameter lines read */
} dsh_inp;

/* Positional .inp reader: every line after a newline that does not start
 * with '#' is the next parameter in the reference's fixed order; the key
 * text is ignored (src/read_par.c:80-470).  Returns DSH_OK or DSH_ERR_PARAM. */
int dsh_read_inp(const char *path, dsh_inp *out);

/* JSON reader: keys as in the reference's .json files ("NX", "FDORDER", ...). */
int dsh_read_json(const char *path, dsh_inp *out);

/* dsh_params from a parameter file: NT = iround(TIME/DT) (src/denise.c:231). */
int dsh_inp_params(const dsh_inp *in, dsh_params *p);

/* one stage of the FWI workflow table (src/read_par_inv.c:31-34) */
typedef struct dsh_stage {
    float pro;
    int time_filt;
    float fc_start, fc_end;
    int order, timewin;
    float gamma, twlength_minus, twlength_plus;
    int inv_vp_iter, inv_vs_iter, inv_rho_iter, spatfilter;
    float wd_damp1, wd_damp;
    int eprecond, lnorm, inv_stf;
    float offsetc_stf, eps_stf;
    int normalize, offset_mute;
    float offsetc, scalerho;
} dsh_stage;
int dsh_read_workflow(const char *path, int stage, dsh_stage *out);

/* Source file -> source table [8][max] in grid units as the one-rank program
 * holds it after src/splitsrc.c (grid x, grid y, 0, tshift, fc, amp, angle,
 * type); sources outside the grid's rank are dropped like splitsrc does. */
int dsh_read_sources(const char *path, float dh, int nx, int ny, int max, int *nsrc, float *srcpos8,
                     float *srcpos_m /* optional [2][max]: x, y in metres */);

/* Receiver file -> [2][max] grid indices (iround((x+REFREC)/DH)), later
 * duplicates of a grid point removed as src/receiver.c:50-72 does. */
int dsh_read_receivers(const char *path, float dh, const float refrec[2], int max, int *ntr, int *recpos);

/* MFILE.vs / .rho / .qs (qs only when l > 0) -> dense [ny][nx] arrays. */
int dsh_read_model(const char *mfile, int nx, int ny, int l, float *vs, float *rho, float *qs);
/* dense [ny][nx] -> float32 file, x outer / depth inner (src/writemod.c) */
int dsh_write_model(const char *path, int nx, int ny, const float *field);

/* The reference's built-in start models, used when READMOD=0
 * (src/denise.c:609-615), as dense [ny][nx] arrays: l > 0 the 1-D gradient
 * model of src/model_grad_visc.c:26-55 (vs = 2.8 (j-1) DH + 170 m/s,
 * rho = 1900 kg/m^3, Qs = 10, i.e. taus = 2/Qs), l == 0 the homogeneous
 * model of src/check_start.c:68-92 (vs = 164 m/s, rho = 1900); qs may be
 * NULL when l == 0.  The reference also writes these models to files
 * (writemod/mergemod); dsh_write_model does that here when wanted. */
int dsh_builtin_model(int l, int nx, int ny, float dh, float *vs, float *rho, float *qs);

/* SU output of one shot (SEIS_FORMAT=1): section [ntr][ns] (ns samples, every
 * ndt-th step), recpos [2][ntr] grid indices, tracl[k] trace numbers (NULL:
 * 1..ntr), source position (xs, ys) in metres; header values as
 * src/outseis_glob.c:45-265 writes them (header bytes 210-239 are not
 * assigned by the reference; they are 0 here). */
int dsh_write_su(const char *path, int ntr, int ns, const float *section, const int *recpos, const int *tracl,
                 float xs, float ys, float dh, float dt, int ndt, const float refrec[2]);

/* SU input as src/inseis.c:73-82 fills it: section [ntr][ns], sample 1 set to 0. */
int dsh_read_su(const char *path, int ntr, int ns, float *section);

/* Asynchronous staging of observed data for the shot loop, in place of the
 * synchronous inseis reads before each residual (src/denise.c:1364-1420).
 * A host thread reads the SU files of submitted batches (dsh_read_su, the
 * same values) into nbuf buffers of max_floats floats; with use_device = 1
 * the buffers are page-locked and dsh_stager_acquire copies the oldest batch
 * to device memory on the stager's own stream and makes `stream` (a
 * cudaStream_t as void*) wait for that copy, so reading and uploading overlap
 * the computation on the previous batch.  A batch is the files' sections
 * concatenated ([ntr[0]][ns], [ntr[1]][ns], ...), the layout dsh_gradient
 * takes as observed data.  Acquire and release alternate; the buffer returns
 * to the reader once `stream` has passed dsh_stager_release, and batch i is
 * read once batch i - nbuf is released.  acquire returns the batch's read
 * status (DSH_ERR_PARAM when a file could not be read; release it all the
 * same); with use_device = 0, dsh_stager_acquire_host returns the host
 * buffer instead (release with stream NULL).  Submitting needs no GPU. */
typedef struct dsh_stager dsh_stager;
dsh_stager *dsh_stager_create(int nbuf, long long max_floats, int use_device, int *status);
int dsh_stager_submit(dsh_stager *s, int nfiles, const char *const *paths, const int *ntr, int ns);
int dsh_stager_acquire(dsh_stager *s, void *stream, const float **dev, long long *nfloats);
int dsh_stager_acquire_host(dsh_stager *s, const float **host, long long *nfloats);
int dsh_stager_release(dsh_stager *s, void *stream);
int dsh_stager_destroy(dsh_stager *s);

#ifdef __cplusplus
}
#endif
#endif

/*
 * dsh.h — C ABI of the B200 SH time-stepping / FWI-gradient engine.
 *
 * Drop-in for the hot path of DENISE-SH's single-rank (NPROCX=NPROCY=1)
 * program: the per-shot forward loop (src/denise.c:1179-1346), the residual
 * (src/calc_res.c, LNORM=2), the adjoint back-propagation with vs/rho
 * correlation (src/denise.c:1452-1654), energy preconditioning
 * (src/eprecond.c, src/eprecond1.c, src/denise.c:1665-1678), the shot sum and
 * gradient conversion (src/denise.c:1689-1694, :1743-1813) and the
 * pseudo-Hessian diagonal (src/hess_save.c, src/hessian.c, src/hessian_out.c).
 * Each of these runs as sm_100a CUDA kernels on device-resident wavefields;
 * results are bit-identical to the reference's FP32 CPU code built without
 * fused multiply-add (see the parity tests), except the float-accumulated L2
 * misfit, which is summed in double here.
 *
 * Conventions
 *   grid fields        dense row-major [ny][nx]; element (i,j) of the reference
 *                      (1-based, i along x, j along depth) is at (j-1)*nx+(i-1)
 *   source table       [8][nsrc] floats, the rows of the reference's srcpos_loc
 *                      (src/splitsrc.c:20-29): grid x, grid y, 0, tshift, fc,
 *                      amplitude, angle, source type (3 = vertical force; only
 *                      type 3 injects in the forward pass, src/update_v_PML.c:569)
 *   receiver table     [2][ntr] ints: grid x, grid y (src/receiver.c:40-41)
 *   traces             per shot [ntr][nt], concatenated shot after shot
 * Every entry point returns DSH_OK (0) or a negative DSH_ERR_* code and never
 * aborts the process.  A context is not thread-safe; use one per host thread.
 */
#ifndef DSH_H
#define DSH_H

#ifdef __cplusplus
extern "C" {
#endif

#define DSH_OK 0
#define DSH_ERR_PARAM (-1)     /* invalid parameter or size */
#define DSH_ERR_CUDA (-2)      /* a CUDA call failed */
#define DSH_ERR_OOM (-3)       /* device allocation failed or budget too small */
#define DSH_ERR_UNSTABLE (-4)  /* non-finite wavefield detected (src/denise.c:1183-1185) */
#define DSH_ERR_STATE (-5)     /* call out of order (e.g. no model set) */
#define DSH_ERR_TIMEOUT (-6)   /* a bounded device wait expired */

#define DSH_EPRECOND_ENERGY_ONLY 10   /* dsh_params.eprecond: raw gradient plus energy maps */

/* Time-stepping parameters: the keys of the reference's .inp/.json files
 * that the hot path reads (src/read_par.c, src/globvar.h). */
typedef struct dsh_params {
    int nx, ny;               /* NX, NY: interior grid points */
    int nt;                   /* NT = iround(TIME/DT) (src/denise.c:231) */
    float dh, dt;             /* DH, DT */
    int fdorder;              /* FDORDER: 2, 4, 6, 8, 10, 12 */
    int maxrelerror;          /* MAXRELERROR 0..4 (0 = Taylor, 1..4 = Holberg) */
    int fw;                   /* FW: CPML width in grid points (0 = none) */
    int free_surf;            /* FREE_SURF: 1 disables the top CPML strip */
    float damping;            /* DAMPING: CPML reference velocity (m/s) */
    float fpml;               /* FPML: CPML frequency (Hz) */
    float npower, k_max_pml;  /* npower, k_max_PML */
    int l;                    /* L: relaxation mechanisms (0 = elastic, <= 4) */
    float fl[8];              /* FL[1..L]: relaxation frequencies (Hz) */
    int quellart;             /* QUELLART: source wavelet (1 Ricker, 2, 4, 5, 6); 3 = caller supplies signals */
    int eprecond;             /* EPRECOND: 0, 1 or 3 (energy preconditioning, src/eprecond1.c);
                                 DSH_EPRECOND_ENERGY_ONLY: accumulate the energies Ws, Wr as
                                 EPRECOND=1 does but leave the gradient unscaled */
    int max_shots;            /* shots advanced together in one launch (>= 1) */
    int compat_fd12;          /* 1: reuse hc[5] in the 6th y term of the FDORDER=12 velocity
                                 operator, as src/update_v_PML.c:469 does */
    long long mem_budget;     /* device bytes for the adjoint's stored forward wavefields;
                                 0 = the free device memory less 2 GiB.  Full storage
                                 when it fits, else checkpoints every
                                 C = sqrt(NT*(3+2L)/3) steps and one recomputed
                                 forward pass (DSH_ERR_OOM if even that does not fit) */
    int ckpt_every;           /* > 0: always checkpoint-and-recompute, one checkpoint every
                                 ckpt_every steps (e.g. ceil(sqrt(NT))), whatever the budget;
                                 0 = the automatic choice above */
    int grad_q;               /* 1: dsh_gradient also forms the gradient with respect to Qs
                                 (L > 0 only; read it with dsh_get_gradient_q).  The forward
                                 pass then stores 5 fields per step instead of 3 */
} dsh_params;

/* One shot (one source gather). */
typedef struct dsh_shot {
    int nsrc;
    const float *srcpos;      /* [8][nsrc] host */
    const float *signals;     /* [nsrc][nt] host, or NULL: computed from srcpos + quellart
                                 (src/wavelet.c:26-84) */
    int ntr;
    const int *recpos;        /* [2][ntr] host */
} dsh_shot;

typedef struct dsh_ctx dsh_ctx;

/* Fills a dsh_params with the values the reference's example parameter
 * file uses for keys the caller does not set (FDORDER 4, MAXRELERROR 1,
 * FW 20, FREE_SURF 1, npower 4, k_max_PML 1, EPRECOND 1, QUELLART 1). */
void dsh_params_default(dsh_params *p);

/* Creates a context on CUDA device `device`. */
dsh_ctx *dsh_create(const dsh_params *p, int device, int *status);
int dsh_destroy(dsh_ctx *ctx);
const char *dsh_error_string(int status);

/* Sets the model (host arrays [ny][nx]: vs in m/s, rho in kg/m^3, qs quality
 * factor, ignored when L=0) and builds every coefficient the kernels read:
 * Holberg operator (src/holbergcoeff.c), CPML profiles (src/PML_pro.c),
 * harmonic shear-modulus averages with the one-rank periodic model halo
 * (src/matcopy_elastic.c, src/av_mue.c), tau averages (src/av_tau.c),
 * SLS coefficients (src/prepare_update_s.c) and the C_vs / C_rho means
 * (src/denise.c:778-816).  Only vs, rho and qs are copied to the device;
 * the per-point coefficients are formed there, identical to the host
 * restatement.  The host arrays may be reused once the call returns. */
int dsh_set_model(dsh_ctx *ctx, const float *vs, const float *rho, const float *qs);

/* Forward modelling of nshots shots; seis_out receives the vertical-velocity
 * seismograms (src/seismo_ssg.c), per shot [ntr][nt]. */
int dsh_forward(dsh_ctx *ctx, const dsh_shot *shots, int nshots, float *seis_out);

/* FWI gradient over nshots shots: forward + residual against obs (per shot
 * [ntr][nt]) + adjoint with correlation + per-shot energy preconditioning +
 * shot sum + conversion to (vs, rho).  Outputs (any may be NULL):
 *   g_vs, g_rho [ny][nx]   gradients (waveconv_u, waveconv_rho after :1813)
 *   l2                     sum over shots of the residual L2 (double accumulation)
 *   seis_out               synthetic seismograms, per shot [ntr][nt]
 *   ws, wr                 [nshots][ny][nx] forward / adjoint energies */
int dsh_gradient(dsh_ctx *ctx, const dsh_shot *shots, int nshots, const float *obs, float *g_vs, float *g_rho,
                 double *l2, float *seis_out, float *ws, float *wr);

/* Pseudo-Hessian diagonal (src/hessian.c:91-94 summed over shots, then the
 * (vs, rho) conversion of src/hessian_out.c:20-31). */
int dsh_hessian_diag(dsh_ctx *ctx, const dsh_shot *shots, int nshots, float *h_vs, float *h_rho);

/* Device-resident variant of dsh_gradient for callers that keep data in HBM:
 * obs_dev is a device array [nshots][ntr][nt]; outputs are device arrays
 * (g_vs_dev, g_rho_dev [ny][nx]); l2 is a host double.  Shots' geometry is
 * host data as above (uploaded once per distinct geometry). */
int dsh_gradient_device(dsh_ctx *ctx, const dsh_shot *shots, int nshots, const float *obs_dev, float *g_vs_dev,
                        float *g_rho_dev, double *l2);

/* Gradient of the misfit J = sum over shots, traces and samples of res^2 (the
 * L2 value dsh_gradient returns, LNORM=2) with respect to the quality factor
 * Qs at every grid point, from the last dsh_gradient / dsh_gradient_device
 * call of a context created with grad_q = 1.  No counterpart in the
 * reference, which inverts vs and rho only.  It is the exact sensitivity of
 * the discrete viscoelastic update (prepare_update_s.c:40-55 through
 * tau = 2/Qs, readmod.c:99, and the four-point tau average, av_tau.c:12) to
 * the back-propagated wavefield: per forward step the stress increment's
 * derivative with respect to tau, with the strain history held fixed, is
 * stored next to the strains, and the adjoint pass correlates it with the
 * adjoint strain; it is neither energy-preconditioned nor scaled.  g_qs_host
 * and/or g_qs_dev receive [ny][nx] floats.  DSH_ERR_STATE when there is no
 * such gradient yet. */
int dsh_get_gradient_q(dsh_ctx *ctx, float *g_qs_host, float *g_qs_dev);

/* Device-resident forward: seis_dev receives [nshots][ntr][nt]. */
int dsh_forward_device(dsh_ctx *ctx, const dsh_shot *shots, int nshots, float *seis_dev);

/* Inspection of the last run (tests and tools): copies a wavefield of shot
 * slot `shot` to host [ny][nx].  which: 0 vy, 1 sxy, 2 syz, 100+l r_l, 200+l q_l,
 * 12 Ws, 13 Wr, 14 We, 15 per-shot g_u (scaled), 16 per-shot g_rho (scaled),
 * 17 / 18 Hessian sums; the model coefficients that dsh_set_model forms on
 * the device (any slot): 300 1/rho, 301 uip, 302 ujp, and for L > 0 the
 * relaxed moduli 303 muip, 304 mujp and 305 tausipjp, 306 taus. */
int dsh_get_field(dsh_ctx *ctx, int shot, int which, float *out);

/* Runs the context's work on the caller's CUDA stream (a cudaStream_t passed
 * as void*; NULL restores the context's own stream), so callers can order it
 * with their own work and time it with events on that stream. */
int dsh_set_stream(dsh_ctx *ctx, void *stream);

/* Per-kernel timing: launches each kernel of pass `pass` (0 forward,
 * 1 forward with storage, 2 forward with Hessian sums, 3 adjoint) `nsteps`
 * times back to back on the last batch between one CUDA event pair and
 * returns the mean device time per launch in ms: out[0] velocity step,
 * out[1] separate injection/sampling (0 when fused), out[2] stress step.
 * Call it after a dsh_gradient on the same shots; it overwrites the
 * wavefield state, which is rebuilt by the next call. */
int dsh_profile_step(dsh_ctx *ctx, int pass, int nsteps, float *out_ms3);

/* Step-kernel variants (dsh_autotune, dsh_set_step_variant): 0 kernel pair,
 * 1 pair with the shared-memory staged velocity kernel, 2 fused
 * velocity+stress step (FDORDER <= 8), 3 one persistent launch per pass of
 * plain forward modelling for grids whose tiles fit one wave, 4 one launch
 * per pass of plain elastic forward modelling with the wavefield and model
 * held in the shared memory of one 16-CTA (or 8-CTA) thread-block cluster
 * per shot (FDORDER <= 8, grids whose ceil(NY/16)-row strips fit one CTA's
 * shared memory, e.g. 500 x 200), 5 plain elastic forward modelling with k
 * time steps per launch (FDORDER 2/4/6/8: k = 8/4/3/2), each thread block
 * advancing a tile 32 points wide (and 8-64 rows high, so that all tiles run
 * in one wave where they can) and a recomputed halo of k*(FDORDER-1) points
 * in its shared memory (FDORDER <= 8, NX and NY >= 2 FW, at most 32 source
 * points, 4 sources per point and 512 receivers per shot). */
#define DSH_STEP_VARIANTS 6

/* Step-kernel autotuner: times nsteps plain forward steps of every variant
 * this context can run on these shots, keeps the fastest for the context's
 * later calls and reports ms_per_step[DSH_STEP_VARIANTS] (0 where a variant
 * does not apply) and *choice.  Results do not depend on the choice (all
 * variants are bit-identical). */
int dsh_autotune(dsh_ctx *ctx, const dsh_shot *shots, int nshots, int nsteps, float *ms_per_step, int *choice);

/* The same for the fused step kernel (one launch per time step; used when
 * FDORDER <= 8, injection/sampling positions lie inside the grid and
 * DSH_FUSED is set): mean ms per launch in *out_ms; DSH_ERR_STATE when the
 * fused kernel does not serve this context and pass. */
int dsh_profile_fused(dsh_ctx *ctx, int pass, int nsteps, float *out_ms);

/* Residual and L2 misfit with no device allocation at all.  This entry point
 * has no counterpart in the reference; it exists for callers that cannot
 * allocate device memory themselves or let a library do it — for instance an
 * application whose device memory is entirely owned by its own pool or arena,
 * or a misfit evaluation inside a loop that must not touch the allocator.
 * It computes, for nshots gathers of ntr traces x nt samples (device arrays
 * [nshots][ntr][nt]), the time-reversed residual res (the adjoint source, as
 * dsh_gradient forms it) and per-shot L2 = sum res^2 (device doubles [nshots]),
 * on the caller's stream (a cudaStream_t as void*, NULL = default stream) and
 * the caller's current device.  Its reduction scratch is a fixed array inside
 * the library (DSH_NOALLOC_MAX_SHOTS shots, 151,552 bytes held by every GPU
 * that loads the library until the process exits); larger nshots is rejected
 * with DSH_ERR_PARAM.  The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress), so make the first call on each device before
 * any stream capture.  All calls on a device share the array and it keeps the
 * last call's contents; calls that overlap on the GPU race on it and must be
 * serialised by the caller.  res must not overlap syn or obs (an in-place
 * residual is rejected with DSH_ERR_PARAM); a CUDA error left pending by
 * earlier work on the device is returned as DSH_ERR_CUDA before any launch. */
#define DSH_NOALLOC_MAX_SHOTS 64
int dsh_residual_noalloc(int nshots, int ntr, int nt, const float *syn, const float *obs, float *res, double *l2,
                         void *stream);

/* ---- Uneven batches: many models in few launches per half-step ----
 * A batch holds nmodels independent models, each with its own dsh_params
 * (grid, FDORDER, L, DT, NT, max_shots, ...).  dsh_batch_forward advances all
 * their shots together: per time step one velocity and one stress kernel
 * launch for all models of a register class (the same FDORDER and L; one
 * launch holding every body for batches of more than 36 models), each thread
 * block working on one 128-point tile of one model; models leave the
 * launches once their NT is reached.  Results are bit-identical to running
 * each model through its own context (and so to the reference's forward
 * loop, src/denise.c:1179-1346); the reference runs one model per program.
 * Supported per model: FDORDER 4, 6, 8 and L 0 or 2 (other combinations:
 * DSH_ERR_PARAM at creation).
 * Tile shape: each launch uses one of four block shapes (128 x 8 points x 1
 * shot, 128 x 4 x 2 shots, 128 x 2 x 4 shots, 128 x 4 x 1 shot); the first
 * run of a batch times them on the batch itself and keeps the fastest
 * (dsh_batch_set_variant fixes them instead). */
typedef struct dsh_batch dsh_batch;
dsh_batch *dsh_batch_create(const dsh_params *p, int nmodels, int device, int *status);
int dsh_batch_destroy(dsh_batch *b);
/* model k's vs, rho, qs as dsh_set_model takes them */
int dsh_batch_set_model(dsh_batch *b, int model, const float *vs, const float *rho, const float *qs);
/* Forward modelling of every model: shots holds nshots[0] shots of model 0,
 * then nshots[1] of model 1, ... (nshots[k] <= max_shots of model k, 0 skips
 * a model); seis_out receives, in the same order, per shot [ntr][nt_k]. */
int dsh_batch_forward(dsh_batch *b, const dsh_shot *shots, const int *nshots, float *seis_out);
int dsh_batch_forward_device(dsh_batch *b, const dsh_shot *shots, const int *nshots, float *seis_dev);
int dsh_batch_set_stream(dsh_batch *b, void *stream);
/* tile-shape variants for the velocity and stress launches: 0 128x8 points
 * x 1 shot, 1 128x4 x 2 shots, 2 128x2 x 4 shots (256-thread blocks), 3 128x4
 * x 1 shot (128 threads); -1 = autotune */
int dsh_batch_set_variant(dsh_batch *b, int v_variant, int s_variant);
/* Wall-clock limit of the batch's host waits (as dsh_set_wait_limits; <= 0 restores 1800 s). */
int dsh_batch_set_host_timeout(dsh_batch *b, double host_seconds);
typedef struct dsh_batch_stats {
    double ms_total;                 /* device time of the last run (CUDA events) */
    long long kernel_launches;
    long long point_updates;         /* sum over models of nx*ny*nt*shots */
    int v_variant, s_variant;        /* tile shapes in use */
    int phases;                      /* distinct NT values (launch grids shrink at each) */
    float v_ms[4], s_ms[4];          /* autotuner: mean ms per launch of each variant (0 = not timed) */
} dsh_batch_stats;
/* model_ms[k] (optional, nmodels doubles): device time from the start of
 * the last run until model k's last step completed */
int dsh_batch_get_stats(dsh_batch *b, double *model_ms, dsh_batch_stats *out);

/* Per-shot L2 misfits of the last dsh_gradient / dsh_gradient_device call
 * (the terms of its l2 total, in shot order; double accumulation). */
int dsh_get_shot_misfits(dsh_ctx *ctx, int nshots, double *out);

/* Shot sums of the energies Ws and Wr of the last gradient call (host dense
 * [ny][nx]; either pointer may be NULL).  Needs EPRECOND 1, 3 or
 * DSH_EPRECOND_ENERGY_ONLY; summed on the device, so no per-shot copies. */
int dsh_get_energy_sums(dsh_ctx *ctx, float *ws_sum, float *wr_sum);

/* Gradient smoothing SPATFILTER=3 (src/smooth_grad.c:27-29, src/gauss_filt.c):
 * out = in convolved with the normalised Gaussian of the given odd filter
 * length (dsh_gauss_filter_size: round(WD_DAMP*(C_vs/FC_END)/DH) made odd),
 * edges replicated; device arrays [ny][nx], in != out, |filt| <= 45
 * (0 copies).  The reference never initialises the kernel's normalising sum
 * (src/gauss_filt.c:26,130); here it starts at 0. */
int dsh_smooth_gauss(int nx, int ny, int filt, const float *in_dev, float *out_dev, void *stream);
int dsh_gauss_filter_size(float wd_damp, float c_vs, float fc_end, float dh);

/* Gradient smoothing SPATFILTER=4 (src/smooth_grad.c:31-33,
 * src/gauss_filt_var.c): a Gaussian whose size follows the local velocity
 * vel_host [ny][nx] (host): lam = vel/FC_END, kernel lengths
 * round(WD_DAMP1 lam/DH) along x and round(WD_DAMP lam/DH) in depth (odd, at
 * least 6; no smoothing where the depth length is <= 0), weights
 * exp(-ii^2/sx - jj^2/sz) normalised by their sum, edges replicated; device
 * arrays [ny][nx], in != out.  The kernels are tabulated on the host (glibc
 * exp, the reference's float/double mix); at most 4096 distinct kernel
 * sizes and 4 M weights (DSH_ERR_PARAM beyond).  Synchronises `stream`. */
int dsh_smooth_gauss_var(int nx, int ny, float dh, float wd_damp, float wd_damp1, float fc_end, const float *vel_host,
                         const float *in_dev, float *out_dev, void *stream);

/* Butterworth filtering of traces or source signals (TIME_FILT stages;
 * src/timedomain_filt.c with libcseife's seife_lpb/seife_hpb,
 * src/denise.c:908-918,1056-1059): data_dev [ntr][ns] device floats,
 * filtered in double by the reference's recursive sections (corner fc Hz,
 * order 1..16; method 1 lowpass, 2 highpass) and rounded back to float.
 * compat = 1 reproduces the reference's off-by-one (src/timedomain_filt.c:31,
 * :42-45 pass its 1-based vector to 0-based libcseife: the last sample is
 * returned unfiltered and the highpass removes a zero, not the first sample);
 * compat = 0 filters all ns samples as libcseife intends. */
int dsh_timedomain_filt(float *data_dev, int ntr, int ns, float dt, float fc, int order, int method, int compat,
                        void *stream);

/* Gradient tapers applied after the shot sum and the smoothing
 * (src/taper_grad.c, called at src/denise.c:1822-1846).  dsh_taper_coeff
 * computes on the host the coefficients coeff [ny][nx] and the mask
 * zero [ny][nx] (1 = the taper sets the point to 0) of
 *   sws 1     the vertical frame: Gaussian ramps over columns GRADT1..GRADT2
 *             and GRADT3..GRADT4, 0 outside, zero at every source and receiver
 *   sws 2     the horizontal taper: 0 above row GRADT1, a Gaussian ramp over
 *             rows GRADT1..GRADT2, the depth j*DH below
 *   sws 3     circular tapers around the sources (srtshape 1 erf, 2 log,
 *             radius srtradius m), zero within filtsize points of a source
 *   sws 5, 6  the values of a taper file (file_vals: nx*ny floats, x outer,
 *             as the reference reads taper.bin)
 * gradt = GRADT1..GRADT4; src_xy [2][nsrc] source x and y in metres (the
 * reference's srcpos rows 1-2, rounded to grid points as it does); recpos
 * [2][ntr] 1-based receiver grid points.  Points outside the grid are
 * ignored: the reference's zeroing writes for box points left of column 1
 * land in the halo or in the previous row's last columns, which is not
 * reproduced.  dsh_taper_apply then sets g = zero ? 0 : g*coeff on device
 * arrays [ny][nx] (coeff_dev, zero_dev: copies of the host arrays). */
int dsh_taper_coeff(int sws, int nx, int ny, float dh, const int gradt[4], int srtshape, float srtradius,
                    int filtsize, int nsrc, const float *src_xy, int ntr, const int *recpos, const float *file_vals,
                    float *coeff, unsigned char *zero);
int dsh_taper_apply(float *g_dev, int nx, int ny, const float *coeff_dev, const unsigned char *zero_dev,
                    void *stream);

/* Misfit norm of dsh_gradient / dsh_gradient_device (LNORM of calc_res.c,
 * GRAD_FORM=2; default 2): 1 L1 (residual sign(obs - syn)), 2 L2 (syn - obs),
 * 3 Cauchy, 4 sech (tanh residual), 5 global correlation
 * (syn (syn.obs)/(|syn|^3 |obs|) - obs/(|syn| |obs|) per trace).  The
 * misfit reported is the reference's: sum res^2 for 2, -sum obs syn/(|obs|
 * |syn|) for 5, and 0 for 1, 3 and 4 (src/calc_res.c:213-257 adds nothing
 * for them).  A trace with |syn| or |obs| = 0 (or whose norms underflow in
 * float) gives NaN residuals under LNORM=5, as in the reference, which carries
 * them into its gradient; here the adjoint pass then returns DSH_ERR_UNSTABLE.
 * LNORM=6 is
 * rejected: the reference reads integrated traces there that it allocates
 * only for LNORM=5 with GRAD_FORM=1 (src/calc_res.c:69-72,221). */
int dsh_set_misfit(dsh_ctx *ctx, int lnorm);

/* Limits of the context's waits (no counterpart in the reference, which
 * blocks in MPI and has no device).  host_seconds: wall-clock limit of every
 * host wait for the context's stream (default 1800 s; <= 0 restores it); when
 * it passes the call returns DSH_ERR_TIMEOUT while the device work goes on, a
 * later call on the stream waits behind that work, and outputs of the
 * timed-out call are undefined.  device_polls: poll limit of the bounded
 * device waits (the grid barrier of the persistent launch; default 2^24,
 * <= 0 restores it); on expiry the kernel sets an error bit, leaves its time
 * loop and the call returns DSH_ERR_TIMEOUT with the context still usable.
 * Small limits exist to exercise those paths. */
int dsh_set_wait_limits(dsh_ctx *ctx, long long device_polls, double host_seconds);

/* Pins the step-kernel variant (0 .. DSH_STEP_VARIANTS-1 as listed at
 * DSH_STEP_VARIANTS; 3, 4 and 5 fall back to the pair where they do not apply;
 * -1 the defaults) — what dsh_autotune picks by timing. */
int dsh_set_step_variant(dsh_ctx *ctx, int variant);

/* Per-shot circular taper (SWS_TAPER_CIRCULAR_PER_SHOT, src/taper_grad_shot.c,
 * applied at src/denise.c:1681-1687): in dsh_gradient / dsh_gradient_device
 * every shot's gradients, after the eprecond scaling and before the shot sum,
 * are multiplied by the circular taper (srtshape 1 erf, 2 log, radius
 * srtradius m) around the shot's first source and set to 0 within filtsize
 * points of it.  enable = 0 switches it off (the default). */
int dsh_set_shot_taper(dsh_ctx *ctx, int enable, int srtshape, float srtradius, int filtsize);

/* The FD grid check the reference runs once on the starting model
 * (src/denise.c:617-622: checkfd_ssg_visc, src/checkfd_ssg_visc.c:14-140,
 * for l > 0; checkfd_ssg_elastic, src/checkfd_ssg_elastic.c, for l == 0;
 * INVMAT1=1), on dense [ny][nx] vs, rho, qs with the reference's float /
 * double mix: out[0] = cmin, the smallest S velocity at zero frequency;
 * out[1] = cmax, the largest at infinite frequency; out[2] = dtstab =
 * DH / (sqrt(2) gamma cmax), gamma = sum |hc[1..6]|; out[3] = dhstab =
 * cmin / (hc[0] * 2/TS), the grid spacing for hc[0] points per minimum
 * wavelength.  Returns DSH_ERR_UNSTABLE where the reference stops with "The
 * simulation will get unstable" (DT > dtstab), DSH_ERR_PARAM where it stops
 * because FW exceeds NX or NY (and for invalid arguments); *warn (optional)
 * gets bit 0 for its grid-dispersion warning (DH > dhstab) and bit 1 for
 * FW < 10.  ts = the source duration TS of the parameter file. */
int dsh_check_fd(int nx, int ny, int l, const float *fl, float dh, float dt, float ts, int fdorder, int maxrelerror,
                 int fw, const float *vs, const float *rho, const float *qs, float out[4], int *warn);

/* Statistics of the last dsh_forward / dsh_gradient call. */
typedef struct dsh_stats {
    double ms_forward, ms_adjoint, ms_total;   /* device time (CUDA events) */
    long long kernel_launches;                  /* kernels of this library launched */
    long long point_updates;                    /* grid-point time steps advanced (all passes) */
    long long storage_bytes;                    /* device bytes used for forward storage */
    int checkpoint_interval;                    /* 0 = full storage */
} dsh_stats;
int dsh_get_stats(dsh_ctx *ctx, dsh_stats *out);

#ifdef __cplusplus
}
#endif
#endif

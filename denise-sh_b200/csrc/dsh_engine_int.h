/* dsh_engine_int.h — engine internals shared by the single-model engine
 * (dsh_engine.cu) and the multi-model batch (dsh_batch.cu). */
#pragma once
#include "dsh.h"
#include "dsh_dispatch.h"
#include "dsh_setup.h"

#include <chrono>
#include <map>
#include <thread>
#include <vector>

namespace dsh {
/* passes: plain forward (modelling), forward storing every step, forward
 * with Hessian sums, adjoint, forward saving only checkpoints, and the
 * recomputation of one segment from a checkpoint on the shadow state */
enum Pass { P_FWD_PLAIN = 0, P_FWD_STORE = 1, P_FWD_HESS = 2, P_ADJ = 3, P_FWD_CKPT = 4, P_RECOMP = 5 };
}  // namespace dsh

struct dsh_ctx {
    dsh_params p;
    int dev = 0;
    cudaStream_t st = nullptr;
    cudaStream_t own_st = nullptr;
    int H = 0, hy = 0, pitch = 0, S = 1, chunk = 32;
    long long fstride = 0, dstride = 0, slot_stride = 0;
    long long o_vy, o_sxy, o_syz, o_r, o_q, o_pvxx, o_psxx, o_pvyy, o_psyy, o_state_end;
    long long o_ws, o_wr, o_we, o_gu, o_grho, o_hu, o_hrho;
    long long o_exy = 0, o_eyz = 0, o_gqx = 0, o_gqy = 0;   /* Qs gradient (params.grad_q) */
    long long o_vy_b = 0, o_sxy_b = 0, o_syz_b = 0, o_pvxx_b = 0, o_pvyy_b = 0;   /* fused step's second buffers */
    int fused_ok = 0;                     /* FDORDER <= 8: the fused step kernel can run this context */
    int state_b = 0;                      /* the slab's current state is in the second buffers */
    int sel_staged = -1, sel_fused = -1, sel_persist = -1;   /* step-kernel variants chosen by dsh_autotune
                                                               (-1: the DSH_VSTAGE / DSH_FUSED / DSH_PERSIST defaults) */
    int sel_cluster = -1;                 /* cluster-resident forward modelling (-1: the DSH_CLUSTER default) */
    int sel_tblock = -1;                  /* temporally blocked forward modelling (-1: the DSH_TBLOCK default) */
    int sel_rows = -1;                    /* 1: the velocity kernel with two rows per thread (-1: DSH_VROWS=2) */
    float *slab = nullptr;
    float *model = nullptr;               /* brho uip ujp muip mujp tausipjp taus vs rho qs */
    float *m_brho, *m_uip, *m_ujp, *m_muip, *m_mujp, *m_tip, *m_taus, *m_vs, *m_rho, *m_qs;
    float sumu = 0.0f;                    /* SLS sum of prepare_update_s (Qs gradient) */
    float *d_gq = nullptr;                /* dJ/dQs of the last gradient (dense [ny][nx]) */
    int gq_valid = 0;
    float eta[4] = {0};
    float *pml = nullptr;
    float *sums = nullptr;                /* sum_u, sum_rho, out_a, out_b (dense pitched) */
    float hc[7] = {0}, bip[4] = {0}, bjm[4] = {0}, cip[4] = {0}, cjm[4] = {0}, cnorm[2] = {0};
    int model_set = 0;
    float *fwd = nullptr;
    long long fwd_slot_stride = 0, fwd_step_stride = 0;
    size_t fwd_bytes = 0;
    int fwd_mod = 0;                      /* stored steps per slot: NT (full storage) or C (checkpointing) */
    int ckpt_c = 0;                       /* checkpoint interval C; 0 = full storage */
    float *ckpt = nullptr;                /* checkpoints: [k][slot][state] */
    size_t ckpt_bytes = 0;
    float *shadow = nullptr;              /* recomputation state, same slot layout as slab */
    /* geometry */
    int *d_geo = nullptr;
    long long geo_cap = 0;
    int *d_fgrp_off, *d_agrp_off, *d_grp_pt, *d_grp_beg, *d_src_id, *d_rec_off, *d_rec_pt;
    int *d_ftile, *d_atile, *d_rtile, *d_gpk, *d_rpk, *d_rid;
    int ntiles = 0, fused_inject = 0;
    int *d_fvoff = nullptr, *d_avoff = nullptr, *d_fvids = nullptr;   /* fused-tile injection lists */
    int fvg_ntiles = 0;
    long long *d_offs = nullptr;          /* sig_off[S], seis_off[S], obs_off[S], out_off[S] */
    float *d_sig = nullptr, *d_seis = nullptr, *d_res = nullptr, *d_obs = nullptr, *d_tmp = nullptr;
    float *d_out = nullptr;               /* 2 x [ny][nx] dense outputs */
    long long cap_sig = 0, cap_seis = 0, cap_obs = 0;
    int geo_version = 0;
    int *d_nt = nullptr, *d_status = nullptr;
    unsigned *d_bar = nullptr;            /* (unused spare words after the status word) */
    unsigned *d_flags = nullptr;          /* tile completion flags of the persistent launch */
    long long flags_cap = 0;
    double *d_part = nullptr, *d_l2 = nullptr;
    unsigned *d_wemax = nullptr;
    std::vector<int> ntr_b;
    int geo_max_groups = 0, geo_max_members = 0, geo_max_ntr = 0;   /* last batch, per slot: forward source
                                                                       points, sources at one point, receivers */
    int lnorm = 2;                        /* misfit norm of the residual (dsh_set_misfit) */
    void *d_tmap = nullptr;               /* 4 CUtensorMap: sxy, syz of the slab, then of the shadow state */
    int tma_ok = 0;                       /* the maps are built (the TMA-staged velocity kernel can run) */
    /* per-shot circular gradient taper (dsh_set_shot_taper): box [g][g] and,
       per slot, the first source's grid point and the normalisation */
    int taper_on = 0, taper_g = 0, taper_ijc = 0, taper_filt = 0;
    std::vector<float> taper_box;
    float *d_taper_box = nullptr;
    void *d_taper_shot = nullptr;         /* S x TaperShot */
    std::vector<double> shot_l2;          /* per-shot L2 misfits of the last gradient */
    std::map<long long, cudaGraphExec_t> graphs;
    cudaEvent_t ev[4];
    cudaEvent_t ev_wait = nullptr;        /* recorded by the bounded host waits (timing disabled) */
    double host_timeout_s = 1800.0;       /* wall-clock limit of every host wait (dsh_set_wait_limits) */
    long long device_polls = 1LL << 24;   /* poll limit of the device's bounded waits (dsh_set_wait_limits) */
    dsh_stats stats;
    long long launches = 0;
    int last_cuda = 0;
};

namespace dsh::eng {
constexpr double HOST_TIMEOUT_DEFAULT_S = 1800.0;
constexpr long long DEVICE_POLLS_DEFAULT = 1LL << 24;

/* Bounded host wait on a recorded event: polls it (yielding, then sleeping
 * 20 us between polls) until it completes (DSH_OK), reports a device error
 * (DSH_ERR_CUDA) or timeout_s seconds of wall-clock time pass
 * (DSH_ERR_TIMEOUT; the device work goes on and a later call on the same
 * stream waits behind it). */
inline int wait_event(cudaEvent_t ev, double timeout_s)
{
    const auto t0 = std::chrono::steady_clock::now();
    for (int polls = 0;; polls++) {
        const cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return DSH_OK;
        if (e != cudaErrorNotReady) return DSH_ERR_CUDA;
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_s)
            return DSH_ERR_TIMEOUT;
        if (polls < 512) std::this_thread::yield();
        else std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

/* bounded wait for everything enqueued on the context's stream so far */
int wait_stream(dsh_ctx *ctx);

/* shots[0..nb) -> slots: sources, receivers, signals, optional observed data */
int upload_batch(dsh_ctx *ctx, const dsh_shot *shots, int nb, const float *obs_host, const float *obs_dev,
                 long long obs_dev_off);
StepArgs step_args(dsh_ctx *ctx, Pass pass);
InjectArgs inject_args(dsh_ctx *ctx, Pass pass);
int zero_slots(dsh_ctx *ctx, int nb, bool accumulators);
int copy_seis_out(dsh_ctx *ctx, int nb, float *host_out, float *dev_out);
int check_status(dsh_ctx *ctx);
bool dh_pow2(float dh);
int l2_stream(const dsh_ctx *ctx, Pass pass);
long long batch_seis_len(dsh_ctx *ctx, const dsh_shot *shots, int nb);
void drop_graphs(dsh_ctx *ctx);
}  // namespace dsh::eng

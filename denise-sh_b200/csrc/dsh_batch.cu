/*
 * dsh_batch.cu — uneven batches: many independent models (each with its own
 * grid, FDORDER, L, DT, NT and shots) advanced together, one velocity and one
 * stress launch per time step for the whole batch.
 *
 * Every model keeps a single-model context (its own slab, coefficients,
 * source/receiver lists); the batch owns one step counter, the models'
 * StepArgs in device memory and block maps listing (model, x tile, y tile,
 * slot group) for each tile-shape variant.  Models are ordered by NT,
 * longest first, so the models still running at step n are a prefix of the
 * map: phase p (steps T_{p-1}+1 .. T_p of the sorted distinct NTs) launches
 * that prefix.  With the StepArgs in the kernels' parameter space the map of
 * each half-step is further grouped by register class (the model's body key,
 * dsh_multi.cuh): one class kernel per key present, each over the NT-ordered
 * prefix of its own group.  Steps are replayed from CUDA graphs of up to 32
 * steps per phase; an event after each phase gives each model's completion
 * time.
 *
 * Reference correspondence: every model runs the forward loop of
 * src/denise.c:1179-1346 (update_v_PML, source injection, update_s_*_PML,
 * seismo_ssg) exactly as a single-model context does; the reference itself
 * runs one model per program invocation.
 */
#include "dsh.h"
#include "dsh_engine_int.h"
#include "dsh_multi.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <vector>

using namespace dsh;
using namespace dsh::eng;

namespace {
__global__ void batch_set_counter(int *p, int v) { *p = v; }
constexpr int CHUNK = 32;
}  // namespace

struct dsh_batch {
    int dev = 0;
    int n = 0;
    std::vector<dsh_ctx *> ctx;
    std::vector<dsh_params> p;
    cudaStream_t st = nullptr, own_st = nullptr;
    int *d_nt = nullptr;
    StepArgs *d_args = nullptr;
    std::unique_ptr<MultiParams> hp;       /* the same in the kernels' parameter space (batches of up to
                                              MULTI_PARAM_MODELS models; DSH_MULTI_ARGS_DEVICE=1: never) */
    int4 *d_map = nullptr;                 /* 2 x MULTI_NVAR maps (velocity, stress x tile-shape variant),
                                              each of map_cap entries */
    long long map_cap = 0;
    bool classed = false;                  /* class kernels, or the kernel with every body (key 0) */
    std::vector<int> order;                /* models by NT, longest first */
    std::vector<int> phase_nt;             /* distinct NTs ascending */
    struct MapClass {
        int key;                           /* body key; 0: every body */
        long long start;                   /* first entry in the map */
        std::vector<long long> count;      /* per phase: entries of the group's running models */
    };
    std::vector<MapClass> cls[2][MULTI_NVAR];
    std::vector<int> nb;                   /* shots per model of the current run */
    long long sig = -1;                    /* signature of the uploaded maps */
    long long geo = -1;                    /* sum of the models' geometry versions the graphs were made for */
    int var_v = -1, var_s = -1;            /* chosen tile-shape variants (-1: tune on next run) */
    int forced_v = -1, forced_s = -1;
    float tune_ms[2][MULTI_NVAR] = {{0}};
    std::map<long long, cudaGraphExec_t> graphs;
    std::vector<cudaEvent_t> ev;           /* start, then one per phase */
    std::vector<double> done_ms;           /* per model: completion time of the last run */
    double total_ms = 0;
    long long launches = 0, points = 0;
    int last_cuda = 0;
    cudaEvent_t ev_wait = nullptr;         /* recorded by the bounded host waits */
    double host_timeout_s = dsh::eng::HOST_TIMEOUT_DEFAULT_S;
};

static int bfail(dsh_batch *b, cudaError_t e)
{
    if (b) b->last_cuda = (int)e;
    fprintf(stderr, "dsh batch: CUDA error %d (%s)\n", (int)e, cudaGetErrorString(e));
    return DSH_ERR_CUDA;
}
#define BK(x)                                          \
    do {                                               \
        cudaError_t e_ = (x);                          \
        if (e_ != cudaSuccess) return bfail(b, e_);    \
    } while (0)

/* bounded host wait for the batch's stream (DSH_ERR_TIMEOUT after host_timeout_s) */
static int bwait(dsh_batch *b)
{
    BK(cudaEventRecord(b->ev_wait, b->st));
    const int rc = dsh::eng::wait_event(b->ev_wait, b->host_timeout_s);
    if (rc == DSH_ERR_CUDA) return bfail(b, cudaGetLastError());
    if (rc == DSH_ERR_TIMEOUT)
        fprintf(stderr, "dsh batch: the device did not finish within %.3g s; the call returns DSH_ERR_TIMEOUT\n",
                b->host_timeout_s);
    return rc;
}
#define BWAIT(b)                                       \
    do {                                               \
        const int w_ = bwait(b);                       \
        if (w_ != DSH_OK) return w_;                   \
    } while (0)

static void drop_batch_graphs(dsh_batch *b)
{
    for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
}

extern "C" dsh_batch *dsh_batch_create(const dsh_params *p, int nmodels, int device, int *status)
{
    auto fail = [&](int code, dsh_batch *b) {
        if (status) *status = code;
        dsh_batch_destroy(b);
        return (dsh_batch *)nullptr;
    };
    if (!p || nmodels <= 0) return fail(DSH_ERR_PARAM, nullptr);
    for (int k = 0; k < nmodels; k++)
        if (!multi_supported(p[k].fdorder, p[k].l)) return fail(DSH_ERR_PARAM, nullptr);
    dsh_batch *b = new dsh_batch();
    b->dev = device;
    b->n = nmodels;
    b->p.assign(p, p + nmodels);
    if (cudaSetDevice(device) != cudaSuccess) return fail(DSH_ERR_CUDA, b);
    if (cudaStreamCreateWithFlags(&b->own_st, cudaStreamNonBlocking) != cudaSuccess) return fail(DSH_ERR_CUDA, b);
    if (cudaEventCreateWithFlags(&b->ev_wait, cudaEventDisableTiming) != cudaSuccess) return fail(DSH_ERR_CUDA, b);
    b->st = b->own_st;
    for (int k = 0; k < nmodels; k++) {
        int rc = DSH_OK;
        dsh_ctx *c = dsh_create(&p[k], device, &rc);
        if (!c) return fail(rc, b);
        b->ctx.push_back(c);
        dsh_set_stream(c, b->st);
    }
    if (cudaMalloc(&b->d_nt, sizeof(int)) != cudaSuccess) return fail(DSH_ERR_OOM, b);
    if (cudaMalloc(&b->d_args, (size_t)nmodels * sizeof(StepArgs)) != cudaSuccess) return fail(DSH_ERR_OOM, b);
    b->order.resize(nmodels);
    std::iota(b->order.begin(), b->order.end(), 0);
    std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) { return p[x].nt > p[y].nt; });
    for (int k = 0; k < nmodels; k++) b->phase_nt.push_back(p[k].nt);
    std::sort(b->phase_nt.begin(), b->phase_nt.end());
    b->phase_nt.erase(std::unique(b->phase_nt.begin(), b->phase_nt.end()), b->phase_nt.end());
    b->ev.resize(b->phase_nt.size() + 1);
    for (auto &e : b->ev) cudaEventCreate(&e);
    b->done_ms.assign(nmodels, 0.0);
    const char *fv = getenv("DSH_BATCH_VARIANT");     /* "v,s": fixed variants, no tuning */
    if (fv && sscanf(fv, "%d,%d", &b->forced_v, &b->forced_s) != 2) b->forced_v = b->forced_s = -1;
    if (status) *status = DSH_OK;
    return b;
}

extern "C" int dsh_batch_destroy(dsh_batch *b)
{
    if (!b) return DSH_OK;
    cudaSetDevice(b->dev);
    if (b->st && b->ev_wait) bwait(b);
    drop_batch_graphs(b);
    for (dsh_ctx *c : b->ctx) dsh_destroy(c);
    cudaFree(b->d_nt); cudaFree(b->d_args); cudaFree(b->d_map);
    for (auto &e : b->ev) if (e) cudaEventDestroy(e);
    if (b->ev_wait) cudaEventDestroy(b->ev_wait);
    if (b->own_st) cudaStreamDestroy(b->own_st);
    delete b;
    return DSH_OK;
}

extern "C" int dsh_batch_set_model(dsh_batch *b, int model, const float *vs, const float *rho, const float *qs)
{
    if (!b || model < 0 || model >= b->n) return DSH_ERR_PARAM;
    return dsh_set_model(b->ctx[model], vs, rho, qs);
}

extern "C" int dsh_batch_set_stream(dsh_batch *b, void *stream)
{
    if (!b) return DSH_ERR_PARAM;
    if (b->st) BWAIT(b);
    b->st = stream ? (cudaStream_t)stream : b->own_st;
    for (dsh_ctx *c : b->ctx) dsh_set_stream(c, b->st);
    drop_batch_graphs(b);
    return DSH_OK;
}

extern "C" int dsh_batch_set_host_timeout(dsh_batch *b, double host_seconds)
{
    if (!b) return DSH_ERR_PARAM;
    b->host_timeout_s = host_seconds > 0 ? host_seconds : dsh::eng::HOST_TIMEOUT_DEFAULT_S;
    for (dsh_ctx *c : b->ctx) dsh_set_wait_limits(c, c->device_polls, b->host_timeout_s);
    return DSH_OK;
}

extern "C" int dsh_batch_set_variant(dsh_batch *b, int v_variant, int s_variant)
{
    if (!b || v_variant < -1 || v_variant >= MULTI_NVAR || s_variant < -1 || s_variant >= MULTI_NVAR)
        return DSH_ERR_PARAM;
    b->forced_v = v_variant;
    b->forced_s = s_variant;
    b->var_v = b->var_s = -1;
    return DSH_OK;
}

/* block maps of both half-steps and every variant for the current shot
 * counts, grouped by register class; per phase the number of entries of the
 * models still running in each group */
static int body_key(const dsh_batch *b, int kind, int k)
{
    if (!b->classed) return 0;
    const dsh_params &q = b->p[k];
    return kind ? multi_skey(q.fdorder, q.l) : multi_vkey(q.fdorder, dh_pow2(q.dh) ? 1 : 0);
}

static const int4 *map_of(const dsh_batch *b, int kind, int v)
{
    return b->d_map + ((size_t)kind * MULTI_NVAR + v) * b->map_cap;
}

static int build_maps(dsh_batch *b)
{
    unsigned long long h = 1469598103934665603ULL;     /* FNV-1a over the shot counts */
    for (int k = 0; k < b->n; k++) h = (h ^ (unsigned)b->nb[k]) * 1099511628211ULL;
    const long long sig = (long long)(h >> 1);
    if (sig == b->sig) return DSH_OK;
    static const bool mixed = getenv("DSH_MULTI_MIXED") != nullptr || getenv("DSH_MULTI_ARGS_DEVICE") != nullptr;
    b->classed = !mixed && b->n <= MULTI_PARAM_MODELS;
    std::vector<int4> maps[2][MULTI_NVAR];
    long long cap = 1;
    for (int kind = 0; kind < 2; kind++) {
        std::vector<int> keys;             /* keys present, in the order of the models' first appearance */
        for (int k : b->order) {
            const int key = body_key(b, kind, k);
            if (std::find(keys.begin(), keys.end(), key) == keys.end()) keys.push_back(key);
        }
        for (int v = 0; v < MULTI_NVAR; v++) {
            const int rows = MULTI_ROWS[v], spb = MULTI_SPB[v];
            std::vector<int4> &m = maps[kind][v];
            b->cls[kind][v].clear();
            for (int key : keys) {
                dsh_batch::MapClass c{key, (long long)m.size(), std::vector<long long>(b->phase_nt.size(), 0)};
                for (int k : b->order) {
                    if (body_key(b, kind, k) != key) continue;
                    const dsh_params &q = b->p[k];
                    const int gx = (q.nx + 4 * BX - 1) / (4 * BX), gy = (q.ny + rows - 1) / rows;
                    const int gz = (b->nb[k] + spb - 1) / spb;
                    for (int z = 0; z < gz; z++)
                        for (int y = 0; y < gy; y++)
                            for (int x = 0; x < gx; x++) m.push_back(make_int4(k, x, y, z));
                    const long long end = (long long)m.size() - c.start;
                    for (size_t ph = 0; ph < b->phase_nt.size(); ph++)
                        if (q.nt >= b->phase_nt[ph]) c.count[ph] = std::max(c.count[ph], end);
                }
                if ((long long)m.size() > c.start) b->cls[kind][v].push_back(c);
            }
            cap = std::max(cap, (long long)m.size());
        }
    }
    if (cap > b->map_cap) {
        cudaFree(b->d_map);
        b->d_map = nullptr;
        BK(cudaMalloc(&b->d_map, (size_t)2 * MULTI_NVAR * cap * sizeof(int4)));
        b->map_cap = cap;
    }
    for (int kind = 0; kind < 2; kind++)
        for (int v = 0; v < MULTI_NVAR; v++)
            if (!maps[kind][v].empty())
                BK(cudaMemcpyAsync((int4 *)map_of(b, kind, v), maps[kind][v].data(),
                                   maps[kind][v].size() * sizeof(int4), cudaMemcpyHostToDevice, b->st));
    BWAIT(b);
    drop_batch_graphs(b);
    b->sig = sig;
    b->var_v = b->var_s = -1;
    return DSH_OK;
}

/* StepArgs of every model for plain forward modelling on the batch counter */
static int upload_args(dsh_batch *b)
{
    std::vector<StepArgs> a(b->n);
    for (int k = 0; k < b->n; k++) {
        a[k] = step_args(b->ctx[k], P_FWD_PLAIN);
        a[k].nt_base = b->d_nt;
        a[k].nslots = b->nb[k];
        a[k].l2_stream = 0;            /* the batch's working set is every model's */
    }
    BK(cudaMemcpyAsync(b->d_args, a.data(), a.size() * sizeof(StepArgs), cudaMemcpyHostToDevice, b->st));
    static const bool device_only = getenv("DSH_MULTI_ARGS_DEVICE") != nullptr;
    if (b->n <= MULTI_PARAM_MODELS && !device_only) {
        if (!b->hp) b->hp.reset(new MultiParams());
        memset(b->hp.get(), 0, sizeof(MultiParams));
        for (int k = 0; k < b->n; k++) b->hp->m[k] = a[k];
    } else {
        b->hp.reset();
    }
    BWAIT(b);
    return DSH_OK;
}

/* the launches of one half-step (kind 0 velocity, 1 stress) over the
 * running models of phase ph: one per register class, or one mixed launch;
 * the first with programmatic serialization only if pdl_first */
static int launch_half(dsh_batch *b, int kind, int var, int ph, int off, bool pdl_first, long long *nl)
{
    static const bool use_pdl = getenv("DSH_NO_PDL") == nullptr;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    const int4 *map = map_of(b, kind, var);
    bool first = true;
    for (const auto &c : b->cls[kind][var]) {
        const long long nblk = c.count[ph];
        if (nblk == 0) continue;
        const bool pdl = use_pdl && (pdl_first || !first);
        first = false;
        cudaLaunchConfig_t cfg = {};
        cfg.blockDim = dim3(BX, MULTI_ROWS[var], MULTI_SPB[var]);
        cfg.gridDim = dim3((unsigned)nblk);
        cfg.stream = b->st;
        cfg.attrs = pdl ? &attr : nullptr;
        cfg.numAttrs = pdl ? 1 : 0;
        const int4 *m = map + c.start;
        if (b->classed) {
            MultiPFn f = kind ? s_multi_k_kernel(var, c.key) : v_multi_k_kernel(var, c.key);
            if (!f) return DSH_ERR_PARAM;
            BK(cudaLaunchKernelEx(&cfg, f, *b->hp, m, off));
        } else if (b->hp) {
            BK(cudaLaunchKernelEx(&cfg, kind ? s_multi_p_kernel(var) : v_multi_p_kernel(var), *b->hp, m, off));
        } else {
            const StepArgs *args = b->d_args;
            BK(cudaLaunchKernelEx(&cfg, kind ? s_multi_kernel(var) : v_multi_kernel(var), args, m, off));
        }
        *nl += 1;
    }
    return DSH_OK;
}

/* number of launches of one half-step in phase ph */
static int half_launches(const dsh_batch *b, int kind, int var, int ph)
{
    int n = 0;
    for (const auto &c : b->cls[kind][var]) n += c.count[ph] > 0;
    return n;
}

/* K steps of phase ph: velocity launches -> (separate injection for models
 * whose sources or receivers lie on the padding) -> stress launches, then
 * the counter */
static int launch_chunk(dsh_batch *b, int ph, int K, long long *nl)
{
    std::vector<std::pair<int, InjectArgs>> sep;
    for (int k = 0; k < b->n; k++) {
        dsh_ctx *c = b->ctx[k];
        if (b->p[k].nt < b->phase_nt[ph] || c->fused_inject || b->nb[k] == 0) continue;
        InjectArgs ia = inject_args(c, P_FWD_PLAIN);
        ia.nt_base = b->d_nt;
        sep.push_back({b->nb[k], ia});
    }
    if (half_launches(b, 0, b->var_v, ph) == 0 || half_launches(b, 1, b->var_s, ph) == 0)
        return DSH_OK;                                 /* no shots in this phase */
    int rc;
    for (int k = 0; k < K; k++) {
        int off = k;
        if ((rc = launch_half(b, 0, b->var_v, ph, off, k > 0, nl)) != DSH_OK) return rc;
        for (auto &s : sep) {
            void *iargs[2] = {&s.second, &off};
            BK(cudaLaunchKernel((const void *)inject_sample, dim3(s.first), dim3(128), iargs, 0, b->st));
            *nl += 1;
        }
        if ((rc = launch_half(b, 1, b->var_s, ph, off, true, nl)) != DSH_OK) return rc;
    }
    advance_step<<<1, 1, 0, b->st>>>(b->d_nt, K);
    *nl += 1;
    BK(cudaGetLastError());
    return DSH_OK;
}

static int run_phase(dsh_batch *b, int ph)
{
    const int n0 = ph ? b->phase_nt[ph - 1] + 1 : 1;
    const int count = b->phase_nt[ph] - n0 + 1;
    if (count <= 0) return DSH_OK;
    batch_set_counter<<<1, 1, 0, b->st>>>(b->d_nt, n0);
    b->launches += 1;
    const int K = std::min(CHUNK, count);
    const int nfull = count / K, rem = count % K;
    static const bool use_graphs = getenv("DSH_NO_GRAPHS") == nullptr;
    for (int c = 0; c < nfull + (rem ? 1 : 0); c++) {
        const int len = c < nfull ? K : rem;
        long long nl = 0;
        if (!use_graphs) {
            int rc = launch_chunk(b, ph, len, &nl);
            if (rc != DSH_OK) return rc;
            b->launches += nl;
            continue;
        }
        const long long key = ((long long)ph << 32) | ((long long)len << 16) | (b->var_v << 8) | b->var_s;
        auto it = b->graphs.find(key);
        if (it == b->graphs.end()) {
            cudaGraph_t g;
            BK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
            int rc = launch_chunk(b, ph, len, &nl);
            cudaError_t e = cudaStreamEndCapture(b->st, &g);
            if (rc != DSH_OK) return rc;
            BK(e);
            cudaGraphExec_t ex;
            BK(cudaGraphInstantiate(&ex, g, 0));
            cudaGraphDestroy(g);
            it = b->graphs.emplace(key, ex).first;
        }
        /* launches per chunk: the class launches of both half-steps per step
           (+ separate injections) + the counter */
        const int nv = half_launches(b, 0, b->var_v, ph), ns = half_launches(b, 1, b->var_s, ph);
        long long per = 0;
        for (int k = 0; k < b->n; k++)
            if (b->p[k].nt >= b->phase_nt[ph] && !b->ctx[k]->fused_inject && b->nb[k] > 0) per++;
        b->launches += nv && ns ? (nv + ns + per) * len + 1 : 0;
        BK(cudaGraphLaunch(it->second, b->st));
    }
    return DSH_OK;
}

/* Autotuner: the launches of each velocity and stress variant (one per
 * register class) repeated back to back over every model (phase 0), mean
 * device time per half-step; the fastest of each kind is kept for this
 * batch signature.  The wavefields it disturbs are zeroed again before the
 * run. */
static int tune(dsh_batch *b)
{
    const int reps = 8;
    cudaEvent_t e0 = b->ev[0], e1 = b->ev[1];
    for (int kind = 0; kind < 2; kind++) {
        const int forced = kind ? b->forced_s : b->forced_v;
        float best = 1e30f;
        int arg = forced >= 0 ? forced : 0;
        for (int v = 0; v < MULTI_NVAR; v++) {
            b->tune_ms[kind][v] = 0;
            if (forced >= 0 && v != forced) continue;
            if (half_launches(b, kind, v, 0) == 0) continue;
            batch_set_counter<<<1, 1, 0, b->st>>>(b->d_nt, 1);
            long long nl = 0;
            for (int r = 0; r < reps + 2; r++) {
                if (r == 2) BK(cudaEventRecord(e0, b->st));
                int rc = launch_half(b, kind, v, 0, 0, false, &nl);
                if (rc != DSH_OK) return rc;
            }
            BK(cudaEventRecord(e1, b->st));
            BWAIT(b);
            BK(cudaGetLastError());
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= reps;
            b->tune_ms[kind][v] = ms;
            if (forced < 0 && ms < best) { best = ms; arg = v; }
        }
        if (kind) b->var_s = arg; else b->var_v = arg;
    }
    return DSH_OK;
}

static int batch_forward(dsh_batch *b, const dsh_shot *shots, const int *nshots, float *seis_host, float *seis_dev)
{
    if (!b || !shots || !nshots) return DSH_ERR_PARAM;
    BK(cudaSetDevice(b->dev));
    b->nb.assign(nshots, nshots + b->n);
    std::vector<long long> first(b->n + 1, 0), out_off(b->n + 1, 0);
    for (int k = 0; k < b->n; k++) {
        if (nshots[k] < 0 || nshots[k] > b->ctx[k]->S) return DSH_ERR_PARAM;
        if (!b->ctx[k]->model_set) return DSH_ERR_STATE;
        first[k + 1] = first[k] + nshots[k];
        out_off[k + 1] = out_off[k] + batch_seis_len(b->ctx[k], shots + first[k], nshots[k]);
    }
    int rc;
    for (int k = 0; k < b->n; k++) {
        dsh_ctx *c = b->ctx[k];
        if (nshots[k] == 0) continue;
        if ((rc = upload_batch(c, shots + first[k], nshots[k], nullptr, nullptr, 0)) != DSH_OK) return rc;
    }
    if ((rc = build_maps(b)) != DSH_OK) return rc;
    if ((rc = upload_args(b)) != DSH_OK) return rc;
    long long geo = 0;                     /* separate-injection arguments are baked into the graphs */
    for (dsh_ctx *c : b->ctx) geo += c->geo_version;
    if (geo != b->geo) { drop_batch_graphs(b); b->geo = geo; }
    if (b->var_v < 0 || b->var_s < 0) {
        if ((rc = tune(b)) != DSH_OK) return rc;
    }
    for (int k = 0; k < b->n; k++)
        if (nshots[k] > 0 && (rc = zero_slots(b->ctx[k], nshots[k], false)) != DSH_OK) return rc;
    b->launches = 0;
    b->points = 0;
    BK(cudaEventRecord(b->ev[0], b->st));
    for (size_t ph = 0; ph < b->phase_nt.size(); ph++) {
        if ((rc = run_phase(b, (int)ph)) != DSH_OK) return rc;
        BK(cudaEventRecord(b->ev[ph + 1], b->st));
    }
    for (int k = 0; k < b->n; k++) {
        if (nshots[k] == 0) continue;
        dsh_ctx *c = b->ctx[k];
        if ((rc = copy_seis_out(c, nshots[k], seis_host ? seis_host + out_off[k] : nullptr,
                                seis_dev ? seis_dev + out_off[k] : nullptr)) != DSH_OK)
            return rc;
        b->launches += 1;
        b->points += (long long)b->p[k].nx * b->p[k].ny * b->p[k].nt * nshots[k];
    }
    BWAIT(b);
    for (int k = 0; k < b->n; k++) {
        const size_t ph = std::lower_bound(b->phase_nt.begin(), b->phase_nt.end(), b->p[k].nt) - b->phase_nt.begin();
        float ms = 0;
        cudaEventElapsedTime(&ms, b->ev[0], b->ev[ph + 1]);
        b->done_ms[k] = ms;
    }
    float tot = 0;
    cudaEventElapsedTime(&tot, b->ev[0], b->ev[b->phase_nt.size()]);
    b->total_ms = tot;
    int worst = DSH_OK;
    for (int k = 0; k < b->n; k++)
        if ((rc = check_status(b->ctx[k])) != DSH_OK) worst = rc;
    return worst;
}

extern "C" int dsh_batch_forward(dsh_batch *b, const dsh_shot *shots, const int *nshots, float *seis_out)
{
    return batch_forward(b, shots, nshots, seis_out, nullptr);
}

extern "C" int dsh_batch_forward_device(dsh_batch *b, const dsh_shot *shots, const int *nshots, float *seis_dev)
{
    return batch_forward(b, shots, nshots, nullptr, seis_dev);
}

extern "C" int dsh_batch_get_stats(dsh_batch *b, double *model_ms, dsh_batch_stats *out)
{
    if (!b) return DSH_ERR_PARAM;
    if (model_ms)
        for (int k = 0; k < b->n; k++) model_ms[k] = b->done_ms[k];
    if (out) {
        memset(out, 0, sizeof(*out));
        out->ms_total = b->total_ms;
        out->kernel_launches = b->launches;
        out->point_updates = b->points;
        out->v_variant = b->var_v;
        out->s_variant = b->var_s;
        for (int v = 0; v < MULTI_NVAR && v < 4; v++) {
            out->v_ms[v] = b->tune_ms[0][v];
            out->s_ms[v] = b->tune_ms[1][v];
        }
        out->phases = (int)b->phase_nt.size();
    }
    return DSH_OK;
}

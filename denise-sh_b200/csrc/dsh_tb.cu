/* Instantiations, launch shape and launches of the temporally blocked
 * forward-modelling kernel (dsh_tblock.cuh), FDORDER 2..8. */
#include <algorithm>
#include <cstdlib>

#include "dsh_tb.h"

namespace dsh {
using TbFn = void (*)(StepArgs, TbGeom, int, int);

template <bool P2>
static TbFn tb_pick(int fdo)
{
    switch (fdo) {
    case 2: return tb_fwd<2, P2>;
    case 4: return tb_fwd<4, P2>;
    case 6: return tb_fwd<6, P2>;
    case 8: return tb_fwd<8, P2>;
    default: return nullptr;
    }
}

static TbFn tb_fn(int fdo, bool p2) { return p2 ? tb_pick<true>(fdo) : tb_pick<false>(fdo); }

bool tb_config(const TbProblem &pb, TbCfg *cfg)
{
    const TbFn fk = tb_fn(pb.fdorder, pb.p2 != 0);
    if (!fk || pb.nb < 1 || pb.nx < 1 || pb.ny < 1 || pb.nx > 0xffff || pb.ny > 0x7fff) return false;
    if (pb.max_groups > TB_MAX_GRP || pb.max_members > TB_MAX_MEM || pb.max_receivers > TB_MAX_REC) return false;
    if (pb.fw > 0 && (pb.nx < 2 * pb.fw || pb.ny < 2 * pb.fw)) return false;
    int dev = 0, maxsm = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const int R = pb.fdorder - 1;
    int k = pb.fdorder == 2 ? 8 : pb.fdorder == 4 ? 4 : pb.fdorder == 6 ? 3 : 2;
    if (const char *e = getenv("DSH_TB_STEPS")) {
        const int v = atoi(e);
        if (v >= 1 && v <= 64) k = v;
    }
    int rows = 0;                                    /* tile height pinned by DSH_TB_ROWS */
    if (const char *e = getenv("DSH_TB_ROWS")) {
        const int v = atoi(e);
        if (v >= 1 && v <= 256) rows = v;
    }
    TbCfg c;
    c.geo.tw = 32;
    auto shape = [&](int th, int kk) {
        c.geo.th = th;
        c.geo.g = kk * R;
        c.geo.ew = c.geo.tw + 2 * c.geo.g;
        c.geo.eh = c.geo.th + 2 * c.geo.g;
        return tb_smem_bytes(c.geo) <= maxsm;
    };
    /* tile height: the smallest multiple of 8 rows (up to 64) for which every
       tile of every slot runs at once, one CTA per SM (a second wave, or SMs
       holding two tiles beside SMs holding one, would double the time of the
       slowest SM); 16 rows where no height does */
    int th = 16;
    if (rows) {
        th = rows;
    } else {
        const int ntx = (pb.nx + c.geo.tw - 1) / c.geo.tw;
        for (int t = 8; t <= 64; t += 8)
            if ((long long)ntx * ((pb.ny + t - 1) / t) * pb.nb <= nsm && shape(t, k)) {
                th = t;
                break;
            }
    }
    for (; k >= 1; k--)
        if (shape(th, k)) break;
    if (k < 1) return false;
    c.k = k;
    c.ntx = (pb.nx + c.geo.tw - 1) / c.geo.tw;
    c.nty = (pb.ny + c.geo.th - 1) / c.geo.th;
    c.smem = (size_t)tb_smem_bytes(c.geo);
    /* the opt-in maximum, not this problem's size: contexts of other sizes
       may launch the same kernel concurrently */
    if (cudaFuncSetAttribute((const void *)fk, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    *cfg = c;
    return true;
}

cudaError_t tb_launch(const TbCfg &cfg, int fdorder, bool p2, const StepArgs &a, int n0, int count, int nb,
                      cudaStream_t st, long long *nlaunch)
{
    const TbFn fk = tb_fn(fdorder, p2);
    if (!fk || cfg.k < 1) return cudaErrorInvalidValue;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)cfg.ntx, (unsigned)cfg.nty, (unsigned)nb);
    lc.blockDim = dim3(TB_THREADS);
    lc.dynamicSmemBytes = cfg.smem;
    lc.stream = st;
    static const bool use_pdl = getenv("DSH_NO_PDL") == nullptr;
    for (int c = 0; c < count; c += cfg.k) {
        const int ks = std::min(cfg.k, count - c);
        lc.attrs = (use_pdl && c > 0) ? &attr : nullptr;   /* the first one follows the pass's set-up plainly */
        lc.numAttrs = (use_pdl && c > 0) ? 1 : 0;
        const cudaError_t e = cudaLaunchKernelEx(&lc, fk, a, cfg.geo, n0 + c, ks);
        if (e != cudaSuccess) return e;
        *nlaunch += 1;
    }
    return cudaSuccess;
}
}  // namespace dsh

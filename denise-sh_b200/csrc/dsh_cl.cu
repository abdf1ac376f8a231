/* Instantiations, launch shape and launch of the cluster-resident
 * forward-modelling kernel (dsh_cluster.cuh), FDORDER 2..8. */
#include <algorithm>

#include "dsh_cl.h"

namespace dsh {
using ClFn = void (*)(StepArgs, int, ClGeom);

template <bool P2>
static ClFn cl_pick(int fdo)
{
    switch (fdo) {
    case 2: return cl_fwd<2, P2>;
    case 4: return cl_fwd<4, P2>;
    case 6: return cl_fwd<6, P2>;
    case 8: return cl_fwd<8, P2>;
    default: return nullptr;
    }
}

static cudaLaunchConfig_t launch_cfg(const ClCfg &c, int nb, cudaStream_t st, cudaLaunchAttribute *at)
{
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)(c.geo.C * nb));
    lc.blockDim = dim3((unsigned)c.nthr);
    lc.dynamicSmemBytes = c.smem;
    lc.stream = st;
    at->id = cudaLaunchAttributeClusterDimension;
    at->val.clusterDim.x = (unsigned)c.geo.C;
    at->val.clusterDim.y = 1;
    at->val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    return lc;
}

/* Row strips for C CTAs.  A row costs its 4-point groups, the groups a CPML
 * x strip touches once more and, in a CPML depth strip, all of them once
 * more (the CPML update about doubles a point's work); rows go to the CTAs
 * in order, each CTA taking rows while its cost stays within `cap`, its
 * shared-memory layout within `budget` and its items within what its threads
 * can hold; the smallest cap (from the mean cost per CTA) that places every
 * row wins.  A CTA followed by rows must own at least H rows (its last H rows
 * are the next CTA's upper halo). */
static bool cl_partition(const ClProblem &pb, int C, size_t budget, int max_items, ClGeom *g, size_t *smem,
                         int *max_rows)
{
    const int H = pb.fdorder / 2, p4 = pb.pitch / 4, ny = pb.ny, fw = pb.fw;
    const int ng = (pb.nx + 3) / 4;
    const int gl = fw > 0 ? std::min(ng, (fw + 3) / 4) : 0;
    const int gr0 = fw > 0 ? std::max(gl, std::min(ng, (pb.nx - fw) / 4)) : ng;
    const int nstr = ng - (gr0 - gl);
    auto bytes = [&](int ja, int jb) {
        const int y = cl_top_rows(ja, jb, fw, pb.free_surf) + cl_bot_rows(ja, jb, ny, fw);
        return (size_t)cl_layout(jb - ja, y, H, p4, fw).bytes;
    };
    auto row_cost = [&](int j) {
        const bool ystrip = fw > 0 && ((!pb.free_surf && j <= fw) || j >= ny - fw + 1);
        return (long long)ng + nstr + (ystrip ? ng : 0);
    };
    long long total = 0;
    for (int j = 1; j <= ny; j++) total += row_cost(j);
    for (long long cap = (total + C - 1) / C;; cap += std::max(1LL, cap / 64)) {
        int j = 1;
        bool ok = true;
        for (int k = 0; k < C; k++) {
            g->j0[k] = j;
            int r = 0;
            long long c = 0;
            while (j + r <= ny && c + row_cost(j + r) <= cap && bytes(j, j + r + 1) <= budget &&
                   (long long)(r + 1) * ng <= max_items) {
                c += row_cost(j + r);
                r++;
            }
            if (r < H && j + r <= ny) {
                ok = false;
                break;
            }
            j += r;
        }
        if (j > ny && ok) break;
        /* rows left over: a larger cap, unless no CTA could take one more row */
        if (cap > total) return false;
    }
    g->C = C;
    g->j0[C] = ny + 1;
    size_t mb = 0;
    int mr = 0;
    for (int k = 0; k < C; k++) {
        mb = std::max(mb, bytes(g->j0[k], g->j0[k + 1]));
        mr = std::max(mr, g->j0[k + 1] - g->j0[k]);
    }
    *smem = mb;
    *max_rows = mr;
    return true;
}

bool cl_config(const ClProblem &pb, ClCfg *cfg)
{
    const ClFn fk = pb.p2 ? cl_pick<true>(pb.fdorder) : cl_pick<false>(pb.fdorder);
    if (!fk || pb.nb < 1 || pb.pitch % 4 || pb.ny < 1 || pb.nx < 1) return false;
    if (pb.max_groups > CL_MAX_GRP || pb.max_members > CL_MAX_MEM || pb.max_receivers > CL_MAX_REC) return false;
    int dev = 0, maxsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const int ng = (pb.nx + 3) / 4, maxthr = cl_max_threads(pb.fdorder);
    for (int C : {16, 8}) {
        ClCfg c;
        size_t smem = 0;
        int max_rows = 0;
        if (!cl_partition(pb, C, (size_t)maxsm, maxthr * CL_MAX_ITEMS, &c.geo, &smem, &max_rows)) continue;
        const int items = max_rows * ng;
        const int per = (items + maxthr - 1) / maxthr;
        c.nthr = std::max(32, ((items + per - 1) / per + 31) / 32 * 32);
        c.smem = smem;
        /* the opt-in maximum, not this problem's size: contexts of other sizes
           may launch the same kernel concurrently */
        if (cudaFuncSetAttribute((const void *)fk, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm) !=
                cudaSuccess ||
            (C > 8 && cudaFuncSetAttribute((const void *)fk, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                          cudaSuccess)) {
            cudaGetLastError();
            continue;
        }
        cudaLaunchAttribute at;
        cudaLaunchConfig_t lc = launch_cfg(c, pb.nb, nullptr, &at);
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, (const void *)fk, &lc) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        if (ncl < 1) continue;
        *cfg = c;
        return true;
    }
    return false;
}

cudaError_t cl_launch(const ClCfg &cfg, int fdorder, bool p2, const StepArgs &a, int nsteps, int nb,
                      cudaStream_t st)
{
    const ClFn fk = p2 ? cl_pick<true>(fdorder) : cl_pick<false>(fdorder);
    if (!fk) return cudaErrorInvalidValue;
    cudaLaunchAttribute at;
    cudaLaunchConfig_t lc = launch_cfg(cfg, nb, st, &at);
    return cudaLaunchKernelEx(&lc, fk, a, nsteps, cfg.geo);
}
}  // namespace dsh

/* dsh_tb.h — the temporally blocked forward-modelling kernel (dsh_tblock.cuh):
 * its launch shape for a context and its launches. */
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include "dsh_tblock.cuh"

namespace dsh {
/* what decides whether and how the kernel serves a plain elastic forward pass */
struct TbProblem {
    int fdorder, p2, nx, ny, fw;
    int nb;                      /* shot slots (grid z) */
    int max_groups, max_members, max_receivers;   /* per slot: source points, sources at one point, receivers */
};

struct TbCfg {
    TbGeom geo;
    int k = 0;                   /* time steps per launch at most */
    int ntx = 0, nty = 0;        /* own tiles along x and depth */
    size_t smem = 0;             /* dynamic shared memory per CTA in bytes */
};

/* The launch shape on the current device: own tiles 32 points wide and as
 * few rows high (a multiple of 8, up to 64) as lets every tile of every slot
 * run at once with one CTA per SM, else 16 rows (DSH_TB_ROWS pins the
 * height); k steps per launch (FDORDER 2: 8, 4: 4, 6: 3, 8: 2; DSH_TB_STEPS
 * overrides it), k lowered until the tile fits the opt-in shared memory of
 * one CTA.  false
 * when the kernel cannot serve the problem (FDORDER > 8, more sources or
 * receivers per slot than its lists hold, NX or NY below 2 FW). */
bool tb_config(const TbProblem &pb, TbCfg *cfg);

/* Launches steps n0 .. n0 + count - 1 for nb slots: ceil(count / k)
 * launches of k steps (the last one the rest), each after the previous one
 * through programmatic dependent launch.  *nlaunch += the launches made. */
cudaError_t tb_launch(const TbCfg &cfg, int fdorder, bool p2, const StepArgs &a, int n0, int count, int nb,
                      cudaStream_t st, long long *nlaunch);
}  // namespace dsh

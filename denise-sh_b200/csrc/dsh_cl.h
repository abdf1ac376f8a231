/* dsh_cl.h — the cluster-resident forward-modelling kernel (dsh_cluster.cuh):
 * its launch shape for a context and its launch. */
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include "dsh_cluster.cuh"

namespace dsh {
/* what decides whether and how the kernel serves a plain elastic forward pass */
struct ClProblem {
    int fdorder, p2, nx, ny, pitch, fw, free_surf;
    int nb;                      /* shot slots (one cluster each) */
    int max_groups, max_members, max_receivers;   /* per slot: source points, sources at one point, receivers */
};

struct ClCfg {
    ClGeom geo;                  /* CTAs per cluster and their row strips */
    int nthr = 0;                /* threads per CTA */
    size_t smem = 0;             /* dynamic shared memory per CTA in bytes */
};

/* The cluster shape on the current device: 16 CTAs per cluster where the
 * device allows it, else 8; rows split so that every CTA's strip (its
 * fields, halo rows, CPML memory, lists) fits the opt-in shared memory of one
 * CTA, CTAs in a CPML depth strip taking fewer rows.  false when the kernel
 * cannot serve the problem (FDORDER > 8, too many sources or receivers, a
 * strip too large, no cluster fits). */
bool cl_config(const ClProblem &pb, ClCfg *cfg);

/* Launches the pass's steps *a.nt_base .. *a.nt_base + nsteps - 1 for nb slots. */
cudaError_t cl_launch(const ClCfg &cfg, int fdorder, bool p2, const StepArgs &a, int nsteps, int nb,
                      cudaStream_t st);
}  // namespace dsh

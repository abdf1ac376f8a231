/*
 * dsh_persist.cuh — small grids: a whole forward-modelling pass in one
 * cooperative launch.
 *
 * For a grid whose 128 x 8-point tiles (times shot slots) fit in one wave,
 * the per-step launch latency of the kernel pair dominates (the 500 x 200
 * elastic case is 100 tiles: ~13 us per step for ~3 us of work).  Here every
 * block owns tiles for the whole pass and loops over the time steps:
 *     velocity of its tiles -> grid barrier -> stress of its tiles -> grid barrier
 * with the same per-point bodies (v_body, s_body) as the kernel pair, so the
 * results are bit-identical.  Loads of fields other blocks wrote earlier in
 * the launch bypass L1 (ld.global.cg).  The barrier is a counter and a
 * generation word in device memory; its wait is bounded: on expiry the block
 * sets bit 2 of the status word and leaves the time loop, and the host
 * reports DSH_ERR_TIMEOUT.  The launch is cooperative, so all blocks are
 * resident and the barrier cannot wait on an unscheduled block.
 */
#pragma once
#include "dsh_kernels.cuh"

namespace dsh {

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

/* count[0]: arrivals of the current barrier, count[1]: generation.  The
 * block barrier before thread 0's fence makes the block's stores part of its
 * release (fences are cumulative); waiting threads poll the generation with
 * acquire loads, at most `limit` times (StepArgs::wait_polls). */
__device__ __forceinline__ bool grid_barrier(unsigned *count, int *status, long long limit)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const unsigned g = ld_acquire(count + 1);
        ok = 1;
        __threadfence();
        if (atomicAdd(count, 1u) == gridDim.x - 1) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(count + 1, 1u);
        } else {
            long long it = 0;
            while (ld_acquire(count + 1) == g) {
                if (++it >= limit) { atomicOr(status, 2); ok = 0; break; }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

template <int FDO, int L, bool P2>
__global__ void __launch_bounds__(BX *BY, 2) persist_fwd(StepArgs a, int nsteps, unsigned *bar)
{
    const int gx = (a.nx + 4 * BX - 1) / (4 * BX), gy = (a.ny + BY - 1) / BY;
    const int per_slot = gx * gy, ntiles = per_slot * a.nslots;
    for (int step = 0; step < nsteps; step++) {
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const int slot = t / per_slot, tile = t % per_slot;
            const int bx = tile % gx, by = tile / gx;
            v_body<FDO, 0, P2, GlobalTaps<true>, true>(a, step, 1 + 4 * (bx * BX + threadIdx.x),
                                                       1 + by * BY + threadIdx.y, slot, tile);
        }
        if (!grid_barrier(bar, a.status, a.wait_polls)) return;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const int slot = t / per_slot, tile = t % per_slot;
            const int bx = tile % gx, by = tile / gx;
            s_body<FDO, L, 0, true>(a, step, 1 + 4 * (bx * BX + threadIdx.x), 1 + by * BY + threadIdx.y, slot);
        }
        if (!grid_barrier(bar, a.status, a.wait_polls)) return;
    }
}

}  // namespace dsh

/*
 * dsh_persist.cuh — small grids: a whole forward-modelling pass in one
 * cooperative launch.
 *
 * For a grid whose 128 x 8-point tiles (times shot slots) fit in one wave,
 * the per-step launch latency of the kernel pair dominates (the 500 x 200
 * elastic case is 100 tiles: ~12 us per step for ~3 us of work).  Here every
 * block owns one tile for the whole pass and loops over the time steps:
 *     wait for the neighbouring tiles -> velocity -> publish ->
 *     wait for the neighbouring tiles -> stress -> publish
 * with the same per-point bodies (v_body, s_body) as the kernel pair, so the
 * results are bit-identical.  Loads of fields other blocks wrote earlier in
 * the launch bypass L1 (ld.global.cg).  A block waits only for its 8
 * neighbours' completion flags, not for the whole grid; every wait is
 * bounded.  The launch is cooperative, so all blocks are resident and no
 * wait depends on an unscheduled block.
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

/* Completion flags of the tiles: flags[0 .. nslots*ntiles) hold the last
 * step whose velocity a tile has finished, flags[nslots*ntiles ..) the last
 * step whose stresses it has finished.  A tile's velocity update of step k
 * reads the stresses of step k-1 of its own and the 8 neighbouring tiles
 * (H <= 6 points, less than a tile in either direction) and overwrites the
 * velocities they read in their stress update of step k-1, so it waits until
 * those tiles' stress flags reach k-1; the stress update of step k waits for
 * their velocity flags to reach k in the same way.  Eight threads poll the
 * eight flags with acquire loads, at most `limit` polls each
 * (StepArgs::wait_polls); on expiry the block sets bit 2 of the status word
 * and leaves its time loop,
 * and the host reports DSH_ERR_TIMEOUT.  A tile publishes a flag after a
 * block barrier and a fence (cumulative: the block's stores are ordered
 * before the flag). */
__device__ __forceinline__ void st_release(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ bool wait_tiles(const unsigned *flags, int bx, int by, int gx, int gy, unsigned need,
                                           long long limit, int *status)
{
    /* the 8 neighbours' flags are polled at once, one thread each (each
       acquire load is an L2 round trip; one thread polling them in turn paid
       eight per phase); the block barrier then orders every thread's loads
       after the acquiring loads */
    __shared__ int ok;
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    if (t == 0) ok = 1;
    __syncthreads();
    if (t < 9 && t != 4) {
        const int x = bx + t % 3 - 1, y = by + t / 3 - 1;
        if (x >= 0 && x < gx && y >= 0 && y < gy) {
            const unsigned *f = flags + y * gx + x;
            long long it = 0;
            while (ld_acquire(f) < need)
                if (++it >= limit) { atomicOr(status, 2); ok = 0; break; }
        }
    }
    __syncthreads();
    return ok != 0;
}

__device__ __forceinline__ void publish_tile(unsigned *flag, unsigned step)
{
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        __threadfence();
        st_release(flag, step);
    }
}

/* one block per 128 x 8 tile of one slot (grid = slots x tiles, all resident) */
template <int FDO, int L, bool P2>
__global__ void __launch_bounds__(BX *BY, 2) persist_fwd(StepArgs a, int nsteps, unsigned *flags)
{
    const int gx = (a.nx + 4 * BX - 1) / (4 * BX), gy = (a.ny + BY - 1) / BY;
    const int per_slot = gx * gy;
    const int t = blockIdx.x;
    if (t >= per_slot * a.nslots) return;
    const int slot = t / per_slot, tile = t % per_slot;
    const int bx = tile % gx, by = tile / gx;
    unsigned *vdone = flags + (long long)slot * per_slot;
    unsigned *sdone = flags + (long long)(a.nslots + slot) * per_slot;
    const int i0 = 1 + 4 * (bx * BX + threadIdx.x), j = 1 + by * BY + threadIdx.y;
    for (int step = 0; step < nsteps; step++) {
        if (!wait_tiles(sdone, bx, by, gx, gy, (unsigned)step, a.wait_polls, a.status)) return;
        v_body<FDO, 0, P2, GlobalTaps<true>, true>(a, step, i0, j, slot, tile);
        publish_tile(vdone + tile, (unsigned)(step + 1));
        if (!wait_tiles(vdone, bx, by, gx, gy, (unsigned)(step + 1), a.wait_polls, a.status)) return;
        s_body<FDO, L, 0, true>(a, step, i0, j, slot);
        publish_tile(sdone + tile, (unsigned)(step + 1));
    }
}

}  // namespace dsh

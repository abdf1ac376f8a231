/*
 * dsh_multi.cuh — step kernels for uneven batches of models.
 *
 * One launch advances every shot of every model of a batch by one half-step.
 * Each thread block reads one entry of a block map — (model, x tile, y tile,
 * slot group) — copies that model's StepArgs into shared memory and runs the
 * same per-point body as the single-model kernels, picked at run time from
 * the model's FDORDER and L (uniform across the block, so no divergence).
 * Results are therefore bit-identical to the single-model kernels.
 *
 * Tile-shape variants: a block is 32 threads along x (4 points each, 128
 * points), ROWS rows and SPB shot slots of the same model: 256 threads
 * (ROWS * SPB = 8) or, for 128 x 4 points of one shot, 128 threads (a
 * shorter block lifetime, a shorter partly idle last wave).  Blocks that
 * share a model's coefficients across SPB shots read them once from L2 per
 * block instead of once per shot; the batch autotuner times the variants on
 * the actual batch and keeps the fastest.
 *
 * Bodies compiled in: FDORDER 4, 6, 8 and L 0 (elastic), 2 (viscoelastic),
 * the operator and relaxation counts of uneven survey batches; the batch
 * rejects other combinations (they run through single-model contexts).
 */
#pragma once
#include "dsh_kernels.cuh"

namespace dsh {

constexpr int MULTI_NVAR = 4;
constexpr int MULTI_ROWS[MULTI_NVAR] = {8, 4, 2, 4};
constexpr int MULTI_SPB[MULTI_NVAR] = {1, 2, 4, 1};

__host__ __device__ constexpr bool multi_supported(int fdo, int l)
{
    return (fdo == 4 || fdo == 6 || fdo == 8) && (l == 0 || l == 2);
}

/* Batches of up to MULTI_PARAM_MODELS models pass every model's StepArgs in
 * the kernel's parameter space (840 B each, within the 32 KB parameter
 * limit): a block reads its model's fields there (constant cache) and starts
 * its loads at once, instead of first copying the 840 B into shared memory
 * behind a block barrier. */
constexpr int MULTI_PARAM_MODELS = 36;
struct MultiParams {
    StepArgs m[MULTI_PARAM_MODELS];
};
static_assert(sizeof(MultiParams) + 16 <= 32764, "kernel parameter space");

/* this thread's point vector, row, slot and injection/sampling list tile
 * for map entry m; false for threads on slots the model does not use */
template <int ROWS, int SPB>
__device__ __forceinline__ bool multi_point(const StepArgs &sa, const int4 &m, int &i0, int &j, int &slot, int &tile)
{
    static_assert(ROWS * SPB == BY || (ROWS == 4 && SPB == 1), "256-thread blocks or 128 x 4 points");
    i0 = 1 + 4 * (m.y * BX + threadIdx.x);
    j = 1 + m.z * ROWS + threadIdx.y;
    slot = m.w * SPB + threadIdx.z;
    tile = ((j - 1) / BY) * sa.tl.ntx + (i0 - 1) / (4 * BX);
    return slot < sa.nslots;
}

/* Block prologue of the device-array form: the model's StepArgs into shared
 * memory, then multi_point. */
template <int ROWS, int SPB>
__device__ __forceinline__ bool multi_setup(StepArgs &sa, const StepArgs *__restrict__ args,
                                            const int4 *__restrict__ map, int &i0, int &j, int &slot, int &tile)
{
    static_assert(sizeof(StepArgs) % 4 == 0, "word copy");
    const int4 m = map[blockIdx.x];
    const int tid = threadIdx.x + BX * (threadIdx.y + ROWS * threadIdx.z);
    const int *src = reinterpret_cast<const int *>(args + m.x);
    int *dst = reinterpret_cast<int *>(&sa);
    for (int k = tid; k < (int)(sizeof(StepArgs) / 4); k += BX * ROWS * SPB) dst[k] = __ldg(src + k);
    __syncthreads();
    return multi_point<ROWS, SPB>(sa, m, i0, j, slot, tile);
}

/* the per-point bodies, picked from the model's FDORDER, L and DH */
__device__ __forceinline__ void v_multi_body(const StepArgs &sa, int nt_off, int i0, int j, int slot, int tile)
{
    switch (sa.fdo * 2 + sa.p2) {
    case 8: v_body<4, 0, false>(sa, nt_off, i0, j, slot, tile); break;
    case 9: v_body<4, 0, true>(sa, nt_off, i0, j, slot, tile); break;
    case 12: v_body<6, 0, false>(sa, nt_off, i0, j, slot, tile); break;
    case 13: v_body<6, 0, true>(sa, nt_off, i0, j, slot, tile); break;
    case 16: v_body<8, 0, false>(sa, nt_off, i0, j, slot, tile); break;
    case 17: v_body<8, 0, true>(sa, nt_off, i0, j, slot, tile); break;
    default: break;
    }
}
__device__ __forceinline__ void s_multi_body(const StepArgs &sa, int nt_off, int i0, int j, int slot)
{
    switch (sa.fdo * 8 + sa.l) {
    case 32: s_body<4, 0, 0>(sa, nt_off, i0, j, slot); break;
    case 34: s_body<4, 2, 0>(sa, nt_off, i0, j, slot); break;
    case 48: s_body<6, 0, 0>(sa, nt_off, i0, j, slot); break;
    case 50: s_body<6, 2, 0>(sa, nt_off, i0, j, slot); break;
    case 64: s_body<8, 0, 0>(sa, nt_off, i0, j, slot); break;
    case 66: s_body<8, 2, 0>(sa, nt_off, i0, j, slot); break;
    default: break;
    }
}

/* velocity / stress half-step of plain forward modelling (flags 0) for all
 * models: StepArgs from a device array ... */
template <int ROWS, int SPB>
__global__ void __launch_bounds__(BX *BY, 3) v_multi(const StepArgs *__restrict__ args, const int4 *__restrict__ map,
                                                     int nt_off)
{
    __shared__ StepArgs sa;
    int i0, j, slot, tile;
    if (!multi_setup<ROWS, SPB>(sa, args, map, i0, j, slot, tile)) return;
    v_multi_body(sa, nt_off, i0, j, slot, tile);
}
template <int ROWS, int SPB>
__global__ void __launch_bounds__(BX *BY, 2) s_multi(const StepArgs *__restrict__ args, const int4 *__restrict__ map,
                                                     int nt_off)
{
    __shared__ StepArgs sa;
    int i0, j, slot, tile;
    if (!multi_setup<ROWS, SPB>(sa, args, map, i0, j, slot, tile)) return;
    s_multi_body(sa, nt_off, i0, j, slot);
}

/* ... or from the parameter space */
template <int ROWS, int SPB>
__global__ void __launch_bounds__(BX *BY, 3) v_multi_p(const __grid_constant__ MultiParams P,
                                                       const int4 *__restrict__ map, int nt_off)
{
    const int4 m = map[blockIdx.x];
    const StepArgs &sa = P.m[m.x];
    int i0, j, slot, tile;
    if (!multi_point<ROWS, SPB>(sa, m, i0, j, slot, tile)) return;
    v_multi_body(sa, nt_off, i0, j, slot, tile);
}
template <int ROWS, int SPB>
__global__ void __launch_bounds__(BX *BY, 2) s_multi_p(const __grid_constant__ MultiParams P,
                                                       const int4 *__restrict__ map, int nt_off)
{
    const int4 m = map[blockIdx.x];
    const StepArgs &sa = P.m[m.x];
    int i0, j, slot, tile;
    if (!multi_point<ROWS, SPB>(sa, m, i0, j, slot, tile)) return;
    s_multi_body(sa, nt_off, i0, j, slot);
}

using MultiFn = void (*)(const StepArgs *, const int4 *, int);
using MultiPFn = void (*)(const MultiParams, const int4 *, int);
MultiFn v_multi_kernel(int variant);
MultiFn s_multi_kernel(int variant);
MultiPFn v_multi_p_kernel(int variant);
MultiPFn s_multi_p_kernel(int variant);

}  // namespace dsh

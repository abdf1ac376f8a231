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

/* Register classes.  A kernel that holds every body needs the registers of
 * the largest one (FDORDER 8, L 2: 128 per thread, 16 warps per SM) for all
 * its blocks, elastic FDORDER-4 tiles included.  A class kernel holds the
 * body of one key alone and a register budget of its own (velocity: that of
 * the single-model kernel, 64 registers, 32 warps per SM; stress: below),
 * and the batch launches one per key present, back to back: every grid waits
 * for its predecessor (pdl_wait) before it reads stresses or velocities, so
 * the launches of one half-step run in order and the next one may begin its
 * prologue during the previous one's tail.  Keys: velocity FDORDER x 2 + (DH
 * a power of two), stress FDORDER x 8 + L. */
__host__ __device__ constexpr int multi_vkey(int fdo, int p2) { return fdo * 2 + (p2 ? 1 : 0); }
__host__ __device__ constexpr int multi_skey(int fdo, int l) { return fdo * 8 + l; }

template <int ROWS, int SPB, int KEY>
__global__ void __launch_bounds__(BX *BY, VSTEP_MIN_BLOCKS_FWD) v_multi_k(const __grid_constant__ MultiParams P,
                                                                          const int4 *__restrict__ map, int nt_off)
{
    const int4 m = map[blockIdx.x];
    const StepArgs &sa = P.m[m.x];
    int i0, j, slot, tile;
    if (!multi_point<ROWS, SPB>(sa, m, i0, j, slot, tile)) return;
    v_body<KEY / 2, 0, (KEY & 1) != 0>(sa, nt_off, i0, j, slot, tile);
}
/* stress: a register cap per key rather than the single-model kernel's
 * budget (a block of 128 threads resides 6 times per SM at <= 80 registers,
 * 5 times at <= 96, 4 times at 128): elastic bodies 80 registers (FDORDER 4
 * without spills, 6 and 8 a few words), viscoelastic 96 (a few words more);
 * measured 6.8 % faster per stress half-step of the 32-model survey batch
 * than the single-model budget, and the cap of 80 for the viscoelastic
 * bodies too 1.5 % slower than 96 */
__host__ __device__ constexpr int multi_sreg(int key) { return key % 8 ? 96 : 80; }
template <int ROWS, int SPB, int KEY>
__global__ void __maxnreg__(multi_sreg(KEY)) s_multi_k(const __grid_constant__ MultiParams P,
                                                        const int4 *__restrict__ map, int nt_off)
{
    const int4 m = map[blockIdx.x];
    const StepArgs &sa = P.m[m.x];
    int i0, j, slot, tile;
    if (!multi_point<ROWS, SPB>(sa, m, i0, j, slot, tile)) return;
    s_body<KEY / 8, KEY % 8, 0>(sa, nt_off, i0, j, slot);
}

using MultiFn = void (*)(const StepArgs *, const int4 *, int);
using MultiPFn = void (*)(const MultiParams, const int4 *, int);
MultiFn v_multi_kernel(int variant);
MultiFn s_multi_kernel(int variant);
MultiPFn v_multi_p_kernel(int variant);
MultiPFn s_multi_p_kernel(int variant);
/* class kernels: nullptr for a key of a body that is not compiled in */
MultiPFn v_multi_k_kernel(int variant, int key);
MultiPFn s_multi_k_kernel(int variant, int key);

}  // namespace dsh

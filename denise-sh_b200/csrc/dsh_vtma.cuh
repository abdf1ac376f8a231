/* dsh_vtma.cuh — the velocity half-step with its stress taps staged in
 * shared memory by the tensor-memory accelerator (opt-in, DSH_VTMA=1).
 *
 * Persistent and pipelined: blockIdx.y = shot slot; the x blocks of a slot
 * take its 128 x 8-point tiles in turn, t = blockIdx.x + k*gridDim.x.  For a
 * tile the block needs its sxy rows with the x halo of the x-derivative
 * (BY rows x 4*(32+NL+NR) floats) and its syz rows with the depth halo
 * (BY+2H-1 rows x 128 floats); a ninth warp produces them: its lane 0
 * issues two 3-D tiled bulk tensor loads per tile (no multicast) into one of
 * vtp_stages(FDO) shared-memory stages and keeps up to that many tiles in flight
 * (full barrier: the stage's bytes have landed; empty barrier: the 256
 * computing threads are done with it, after which the producer refills it),
 * while warps 0-7 run v_body on the staged taps (SharedTaps) — so the results
 * are bit-identical to v_step.  The tensor maps (built on the host, kept in
 * device memory) cover each slot's haloed field; positions outside it read
 * as zeros; the x coordinate of every box is a multiple of 4 floats (16
 * bytes).  Every wait is bounded: on expiry the block sets bit 2 of the
 * status word (DSH_ERR_TIMEOUT) and stops, and the producer waits (bounded)
 * for the loads it issued before the block exits.
 */
#pragma once
#include "dsh_kernels.cuh"

namespace dsh {

constexpr long long VTMA_WAIT_LIMIT = 1LL << 22;   /* mbarrier.try_wait polls before giving up */
/* shared-memory stages: 4 up to FDORDER 8, 3 above (static shared memory <= 48 KB) */
__host__ __device__ constexpr int vtp_stages(int fdo) { return fdo <= 8 ? 4 : 3; }

__device__ __forceinline__ uint32_t vt_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool vt_try_wait(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(vt_smem(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

/* bounded wait for the phase of the given parity; false on expiry or abort */
__device__ __forceinline__ bool vt_wait_flag(uint64_t *b, uint32_t parity, volatile int *abort)
{
    for (long long it = 0; it < VTMA_WAIT_LIMIT; it++) {
        if (vt_try_wait(b, parity)) return true;
        if (*abort) return false;
    }
    return false;
}

__device__ __forceinline__ void vt_load_3d(void *dst, const void *map, uint64_t *bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(vt_smem(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(vt_smem(bar))
        : "memory");
}

template <int FDO, int FLAGS, bool P2>
__global__ void __launch_bounds__(BX *(BY + 1), 2) v_step_tp(StepArgs a, int nt_off)
{
    constexpr int H = FDO / 2;
    constexpr int NL = (H + 3) / 4, NR = (H - 1 + 3) / 4;
    constexpr int SXP = BX + NL + NR;                 /* float4 groups per staged sxy row */
    constexpr int SYR = BY + 2 * H - 1;               /* staged syz rows */
    constexpr int NS = vtp_stages(FDO);
    constexpr uint32_t BYTES = (uint32_t)(BY * SXP + SYR * BX) * 16u;
    __shared__ __align__(128) float4 sx[NS][BY * SXP];
    __shared__ __align__(128) float4 sy[NS][SYR * BX];
    __shared__ __align__(8) uint64_t full[NS], empty[NS];
    __shared__ int abort_flag;
    const int nt = *a.nt_base + nt_off;
    if (nt > a.nt_last) return;
    const int slot = blockIdx.y;
    const int gx = (a.nx + 4 * BX - 1) / (4 * BX), gy = (a.ny + BY - 1) / BY, per_slot = gx * gy;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        for (int s = 0; s < NS; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(vt_smem(&full[s])), "r"(1) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(vt_smem(&empty[s])), "r"(BX * BY) : "memory");
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    pdl_wait();                                       /* stresses of the previous step are complete */
    if (threadIdx.y == BY) {                          /* producer warp */
        if (threadIdx.x != 0) return;
        /* the maps were written by the host before the launch */
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(a.tm_sxy) : "memory");
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(a.tm_syz) : "memory");
        int k = 0;
        for (int t = blockIdx.x; t < per_slot; t += gridDim.x, k++) {
            const int s = k % NS;
            if (k >= NS && !vt_wait_flag(&empty[s], (uint32_t)(k / NS - 1) & 1u, &abort_flag)) {
                abort_flag = 1;
                break;
            }
            const int bx = t % gx, by = t / gx;
            const int cb = 4 * bx * BX + HX, j0 = 1 + by * BY;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(vt_smem(&full[s])),
                         "r"(BYTES)
                         : "memory");
            vt_load_3d(sx[s], a.tm_sxy, &full[s], cb - 4 * NL, j0 - 1 + a.hy, slot);
            vt_load_3d(sy[s], a.tm_syz, &full[s], cb, j0 - H - 1 + a.hy, slot);
        }
        if (abort_flag) {
            atomicOr(a.status, 2);
            /* at most NS issued loads can be outstanding: the last ones */
            for (int q = k > NS ? k - NS : 0; q < k; q++)
                for (long long w = 0; w < VTMA_WAIT_LIMIT; w++)
                    if (vt_try_wait(&full[q % NS], (uint32_t)(q / NS) & 1u)) break;
        }
        return;
    }
    int it = 0;
    for (int t = blockIdx.x; t < per_slot; t += gridDim.x, it++) {
        const int s = it % NS;
        if (!vt_wait_flag(&full[s], (uint32_t)(it / NS) & 1u, &abort_flag)) {
            abort_flag = 1;
            break;
        }
        const int bx = t % gx, by = t / gx;
        SharedTaps taps{sx[s], sy[s], SXP, (int)threadIdx.x, (int)threadIdx.y};
        v_body<FDO, FLAGS, P2>(a, nt_off, 1 + 4 * (bx * BX + threadIdx.x), 1 + by * BY + threadIdx.y, slot,
                               by * gx + bx, taps);
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(vt_smem(&empty[s])) : "memory");
    }
}

}  // namespace dsh

/*
 * dsh_nn_gemm.cu — BF16 GEMM on the sm_100a tensor cores (tcgen05 + TMA),
 * FP32 accumulation in tensor memory, for the pseudo-Hessian U-Net.
 *
 *   C[M][N] = A[M][K] . B[N][K]^T  (+ bias[N]) (ReLU)    A, B bf16, K-major
 *
 * One CTA computes a 128 x BN tile of C (BN = 32, 64, 128 or 256) over a
 * range of K (split-K along grid z writes FP32 partials that a reduction
 * kernel sums).  128 threads:
 *   warp 0, one thread   TMA producer: 128 x 64 A and BN x 64 B tiles into a
 *                        4-stage ring of 128-byte-swizzled shared memory,
 *                        completion counted on the stage's "full" mbarrier
 *   warp 1, one thread   MMA issuer: per stage 4 x tcgen05.mma (M=128, N=BN,
 *                        K=16, kind::f16 with BF16 inputs, F32 accumulator in
 *                        TMEM), then tcgen05.commit to the stage's "empty"
 *                        mbarrier so the producer may refill it
 *   all 4 warps          epilogue: tcgen05.ld of the accumulator (warp w owns
 *                        TMEM lanes 32w..32w+31 = tile rows), bias, ReLU,
 *                        FP32 or BF16 stores
 * Every mbarrier wait is bounded; on expiry the CTA records an error code,
 * stops issuing work, waits (with a separate bound) for the copies and
 * matrix-multiply operations it already issued, and frees its tensor memory.
 */
#include "dsh_nn.h"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>

namespace {

constexpr int BM = 128, BK = 64, STAGES = 4, THREADS = 128;
constexpr long long WAIT_LIMIT = 1LL << 22;       /* mbarrier.try_wait polls before giving up (default) */
constexpr long long DRAIN_LIMIT = 1LL << 24;      /* polls while draining work in flight after an expiry */
long long g_wait_polls = WAIT_LIMIT;              /* dsh_nn_set_wait_limit */

struct GemmArgs {
    int M, N, K;
    int ktiles, kt_per_split;
    float *c32;
    __nv_bfloat16 *c16;
    long long ldc;
    long long split_stride;                      /* floats between split-K partial outputs */
    const float *bias;
    int relu;
    int *err;                                    /* set to DSH_NN_ERR_TIMEOUT by a CTA whose wait expired */
    long long wait_polls;                        /* poll limit of the pipeline's mbarrier waits */
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

/* bounded wait for the phase of the given parity; false on expiry or abort */
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, volatile int *abort, long long limit)
{
    for (long long it = 0; it < limit; it++) {
        if (mbar_try_wait(b, parity)) return true;
        if (*abort) return false;
    }
    return false;
}

/* bounded wait that ignores the abort flag: after an expiry, for the copies
   and multiply operations the CTA already issued to finish before it frees
   its tensor memory and exits */
__device__ __forceinline__ bool mbar_drain(uint64_t *b, uint32_t parity)
{
    for (long long it = 0; it < DRAIN_LIMIT; it++)
        if (mbar_try_wait(b, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

/* shared-memory matrix descriptor of a K-major tile with 128-byte rows in the
 * 128-byte swizzle (8-row, 1024-byte atoms): start >> 4 in bits 0-13,
 * leading offset 16 B (unused for this layout), stride offset 1024 B between
 * 8-row groups in bits 32-45, descriptor version 1 (bits 46-47), swizzle
 * mode 2 = 128 B (bits 61-63) */
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

/* instruction descriptor: F32 accumulator (bits 4-5 = 1), A and B BF16
 * (bits 7-9, 10-12 = 1), both K-major, N >> 3 in bits 17-22, M >> 4 in 24-28 */
template <int BN>
__device__ __forceinline__ uint32_t idesc_bf16()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

/* 16 consecutive FP32 accumulator columns of this thread's TMEM lane */
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

template <int BN>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_bf16_tc(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmArgs g)
{
    constexpr uint32_t A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE = A_BYTES + B_BYTES;
    constexpr uint32_t TCOLS = BN < 32 ? 32 : BN;                /* power of two >= 32 */
    extern __shared__ uint8_t dyn[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~(uintptr_t)1023);
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int kt0 = blockIdx.z * g.kt_per_split;
    const int kt1 = min(g.ktiles, kt0 + g.kt_per_split);
    const int nk = kt1 - kt0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(&done, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (nk > 0) {
        if (warp == 0 && lane == 0) {                 /* TMA producer */
            int issued = 0;
            for (int i = 0; i < nk; i++) {
                const int s = i % STAGES;
                const uint32_t ph = (uint32_t)(i / STAGES) & 1u;
                if (!mbar_wait(&empty[s], ph ^ 1u, &abort_flag, g.wait_polls)) { abort_flag = 1; break; }
                uint8_t *sa = smem + s * STAGE;
                mbar_expect_tx(&full[s], STAGE);
                tma_load_2d(sa, &ta, &full[s], (kt0 + i) * BK, m0);
                tma_load_2d(sa + A_BYTES, &tb, &full[s], (kt0 + i) * BK, n0);
                issued = i + 1;
            }
            if (abort_flag) {                         /* the last load of each stage lands before the CTA exits */
                for (int i = issued > STAGES ? issued - STAGES : 0; i < issued; i++)
                    mbar_drain(&full[i % STAGES], (uint32_t)(i / STAGES) & 1u);
            }
        } else if (warp == 1 && lane == 0) {          /* MMA issuer */
            const uint32_t idesc = idesc_bf16<BN>();
            for (int i = 0; i < nk; i++) {
                const int s = i % STAGES;
                const uint32_t ph = (uint32_t)(i / STAGES) & 1u;
                if (!mbar_wait(&full[s], ph, &abort_flag, g.wait_polls)) { abort_flag = 1; break; }
                tc_fence_after();
                const uint32_t sa = smem_u32(smem + s * STAGE), sb = sa + A_BYTES;
                const uint64_t da = sw128_desc(sa), db = sw128_desc(sb);
#pragma unroll
                for (int kk = 0; kk < BK / 16; kk++)  /* K step of 16 bf16 = 32 bytes = 2 descriptor units */
                    umma_bf16(tmem, da + 2 * kk, db + 2 * kk, idesc, (i > 0 || kk > 0) ? 1u : 0u);
                umma_commit(&empty[s]);
            }
            umma_commit(&done);                       /* also after an expiry: tracks every issued MMA */
        }
        __syncwarp();
        /* epilogue: every thread one row of the tile */
        bool ok = mbar_wait(&done, 0, &abort_flag, g.wait_polls) && !abort_flag;
        ok = __all_sync(0xffffffffu, ok);             /* tcgen05.ld below is warp-collective */
        if (!ok) mbar_drain(&done, 0);                /* the issued MMAs finish before TMEM is freed */
        tc_fence_after();
        const int row = m0 + warp * 32 + lane;
        if (ok) {
            float *c32 = g.c32 ? g.c32 + (long long)blockIdx.z * g.split_stride : nullptr;
#pragma unroll 1
            for (int c = 0; c < BN; c += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
                if (row >= g.M) continue;
                const int nb = n0 + c;
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    const int n = nb + k;
                    if (n >= g.N) break;
                    float x = v[k];
                    if (g.bias) x += g.bias[n];
                    if (g.relu) x = fmaxf(x, 0.0f);
                    if (c32) c32[(long long)row * g.ldc + n] = x;
                    if (g.c16) g.c16[(long long)row * g.ldc + n] = __float2bfloat16_rn(x);
                }
            }
        } else if (lane == 0) {                      /* any warp whose wait expired reports it */
            atomicExch(g.err, DSH_NN_ERR_TIMEOUT);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
}

/* sum of split-K partials: c[m][n] = sum_z part[z][m][n] (+ c if accumulate) */
__global__ void splitk_reduce(const float *part, int splits, long long stride, int M, int N, long long ldc, float *c,
                              int accumulate)
{
    const long long total = (long long)M * N;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long m = idx / N, n = idx % N;
        float s = accumulate ? c[m * ldc + n] : 0.0f;
        for (int z = 0; z < splits; z++) s += part[z * stride + m * ldc + n];
        c[m * ldc + n] = s;
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encoder()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

/* 2-D bf16 tensor map: rows x k (k contiguous, row stride ld elements),
 * box 64 (k) x box_rows, 128-byte swizzle, zero fill outside */
bool make_map(CUtensorMap *m, const void *ptr, long long rows, long long k, long long ld, int box_rows)
{
    EncodeTiledFn enc = encoder();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN>
int launch(const CUtensorMap &ta, const CUtensorMap &tb, const GemmArgs &g, int splits, cudaStream_t st)
{
    const size_t smem = (size_t)STAGES * (BM * BK * 2 + BN * BK * 2) + 1024;
    static bool attr_set = false;
    if (!attr_set) {
        if (cudaFuncSetAttribute(gemm_bf16_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return DSH_NN_ERR_CUDA;
        attr_set = true;
    }
    dim3 grid((unsigned)((g.M + BM - 1) / BM), (unsigned)((g.N + BN - 1) / BN), (unsigned)splits);
    gemm_bf16_tc<BN><<<grid, THREADS, smem, st>>>(ta, tb, g);
    return cudaGetLastError() == cudaSuccess ? DSH_NN_OK : DSH_NN_ERR_CUDA;
}

}  // namespace

extern "C" int dsh_nn_set_wait_limit(long long polls)
{
    g_wait_polls = polls > 0 ? polls : WAIT_LIMIT;
    return DSH_NN_OK;
}

extern "C" int dsh_nn_gemm(int M, int N, int K, const void *A, long long lda, const void *B, long long ldb, float *C32,
                           void *C16, long long ldc, const float *bias, int relu, int splits, float *partial,
                           int accumulate, int *err, void *stream)
{
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || (!C32 && !C16) || !err) return DSH_NN_ERR_PARAM;
    if (lda % 8 || ldb % 8 || lda < K || ldb < K || ((uintptr_t)A & 15) || ((uintptr_t)B & 15)) return DSH_NN_ERR_PARAM;
    if (splits < 1) splits = 1;
    if (splits > 1 && (!C32 || !partial || C16 || bias || relu)) return DSH_NN_ERR_PARAM;
    if (accumulate && (!C32 || C16)) return DSH_NN_ERR_PARAM;
    const int BN = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
    CUtensorMap ta, tb;
    if (!make_map(&ta, A, M, K, lda, BM) || !make_map(&tb, B, N, K, ldb, BN)) return DSH_NN_ERR_PARAM;
    GemmArgs g;
    g.M = M; g.N = N; g.K = K;
    g.ktiles = (K + BK - 1) / BK;
    splits = std::min(splits, g.ktiles);
    g.kt_per_split = (g.ktiles + splits - 1) / splits;
    splits = (g.ktiles + g.kt_per_split - 1) / g.kt_per_split;
    const bool direct = splits == 1 && !accumulate;
    g.c32 = direct ? C32 : partial;
    g.c16 = (__nv_bfloat16 *)C16;
    g.ldc = ldc;
    g.split_stride = (long long)M * ldc;
    g.bias = bias;
    g.relu = relu;
    g.err = err;
    g.wait_polls = g_wait_polls;
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    switch (BN) {
    case 32: rc = launch<32>(ta, tb, g, splits, st); break;
    case 64: rc = launch<64>(ta, tb, g, splits, st); break;
    case 128: rc = launch<128>(ta, tb, g, splits, st); break;
    default: rc = launch<256>(ta, tb, g, splits, st); break;
    }
    if (rc != DSH_NN_OK || direct) return rc;
    const long long total = (long long)M * N;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 8);
    splitk_reduce<<<blocks, 256, 0, st>>>(partial, splits, g.split_stride, M, N, ldc, C32, accumulate);
    return cudaGetLastError() == cudaSuccess ? DSH_NN_OK : DSH_NN_ERR_CUDA;
}

/* dsh_dispatch.h — kernel selection by FD order, relaxation count and mode. */
#pragma once
#include "dsh_kernels.cuh"

namespace dsh {
using KFn = void (*)(StepArgs, int);

#define DSH_DECLARE_FD(N)                     \
    KFn v_kernel_fd##N(int flags, bool p2);    \
    KFn v_kernel_st_fd##N(int flags, bool p2); \
    KFn v_kernel_tp_fd##N(int flags, bool p2); \
    KFn v_kernel_r2_fd##N(int flags, bool p2); \
    KFn s_kernel_fd##N(int l, int flags);
DSH_DECLARE_FD(2)
DSH_DECLARE_FD(4)
DSH_DECLARE_FD(6)
DSH_DECLARE_FD(8)
DSH_DECLARE_FD(10)
DSH_DECLARE_FD(12)
#undef DSH_DECLARE_FD

inline KFn v_kernel(int fdo, int flags, bool p2)
{
    switch (fdo) {
    case 2: return v_kernel_fd2(flags, p2);
    case 4: return v_kernel_fd4(flags, p2);
    case 6: return v_kernel_fd6(flags, p2);
    case 8: return v_kernel_fd8(flags, p2);
    case 10: return v_kernel_fd10(flags, p2);
    case 12: return v_kernel_fd12(flags, p2);
    default: return nullptr;
    }
}

/* velocity step with shared-memory staged stress taps */
inline KFn v_kernel_st(int fdo, int flags, bool p2)
{
    switch (fdo) {
    case 2: return v_kernel_st_fd2(flags, p2);
    case 4: return v_kernel_st_fd4(flags, p2);
    case 6: return v_kernel_st_fd6(flags, p2);
    case 8: return v_kernel_st_fd8(flags, p2);
    case 10: return v_kernel_st_fd10(flags, p2);
    case 12: return v_kernel_st_fd12(flags, p2);
    default: return nullptr;
    }
}

/* persistent velocity step with TMA-staged taps (dsh_vtma.cuh); grid (blocks per slot, slots),
 * block (32, 9) */
inline KFn v_kernel_tp(int fdo, int flags, bool p2)
{
    switch (fdo) {
    case 2: return v_kernel_tp_fd2(flags, p2);
    case 4: return v_kernel_tp_fd4(flags, p2);
    case 6: return v_kernel_tp_fd6(flags, p2);
    case 8: return v_kernel_tp_fd8(flags, p2);
    case 10: return v_kernel_tp_fd10(flags, p2);
    case 12: return v_kernel_tp_fd12(flags, p2);
    default: return nullptr;
    }
}

/* velocity step with two rows per thread (v_step_r2), block (32, 4) */
inline KFn v_kernel_r2(int fdo, int flags, bool p2)
{
    switch (fdo) {
    case 2: return v_kernel_r2_fd2(flags, p2);
    case 4: return v_kernel_r2_fd4(flags, p2);
    case 6: return v_kernel_r2_fd6(flags, p2);
    case 8: return v_kernel_r2_fd8(flags, p2);
    case 10: return v_kernel_r2_fd10(flags, p2);
    case 12: return v_kernel_r2_fd12(flags, p2);
    default: return nullptr;
    }
}

inline KFn s_kernel(int fdo, int l, int flags)
{
    switch (fdo) {
    case 2: return s_kernel_fd2(l, flags);
    case 4: return s_kernel_fd4(l, flags);
    case 6: return s_kernel_fd6(l, flags);
    case 8: return s_kernel_fd8(l, flags);
    case 10: return s_kernel_fd10(l, flags);
    case 12: return s_kernel_fd12(l, flags);
    default: return nullptr;
    }
}
}  // namespace dsh

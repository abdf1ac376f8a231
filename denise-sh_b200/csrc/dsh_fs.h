/* dsh_fs.h — selection of the fused step kernel (dsh_fused.cuh). */
#pragma once
#include "dsh_dispatch.h"

namespace dsh {
#define DSH_DECLARE_FS(N) KFn fs_kernel_fd##N(int l, int mode, bool p2);
DSH_DECLARE_FS(2)
DSH_DECLARE_FS(4)
DSH_DECLARE_FS(6)
DSH_DECLARE_FS(8)
#undef DSH_DECLARE_FS

inline KFn fs_kernel(int fdo, int l, int mode, bool p2)
{
    switch (fdo) {
    case 2: return fs_kernel_fd2(l, mode, p2);
    case 4: return fs_kernel_fd4(l, mode, p2);
    case 6: return fs_kernel_fd6(l, mode, p2);
    case 8: return fs_kernel_fd8(l, mode, p2);
    default: return nullptr;
    }
}
}  // namespace dsh

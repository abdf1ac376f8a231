/* dsh_pf.h — selection of the persistent forward-modelling kernel (dsh_persist.cuh). */
#pragma once
#include "dsh_kernels.cuh"

namespace dsh {
using PFn = void (*)(StepArgs, int, unsigned *);
PFn pf_kernel_fd2(int l, bool p2);
PFn pf_kernel_fd4(int l, bool p2);
PFn pf_kernel_fd6(int l, bool p2);
PFn pf_kernel_fd8(int l, bool p2);

inline PFn pf_kernel(int fdo, int l, bool p2)
{
    switch (fdo) {
    case 2: return pf_kernel_fd2(l, p2);
    case 4: return pf_kernel_fd4(l, p2);
    case 6: return pf_kernel_fd6(l, p2);
    case 8: return pf_kernel_fd8(l, p2);
    default: return nullptr;
    }
}
}  // namespace dsh

/* dsh_inst.cuh — instantiates the step kernels of one FD order (included by
 * dsh_fd<N>.cu so the orders compile in parallel). */
#pragma once
#include "dsh_dispatch.h"
#include "dsh_vtma.cuh"

#define DSH_INSTANTIATE_FD(N)                                                                 \
    namespace dsh {                                                                           \
    template <bool P2>                                                                        \
    static KFn v_pick_##N(int flags)                                                          \
    {                                                                                         \
        switch (flags) {                                                                      \
        case 0: return v_step<N, 0, P2>;                                                      \
        case VF_HESS: return v_step<N, VF_HESS, P2>;                                          \
        case VF_ADJOINT | VF_CORR: return v_step<N, VF_ADJOINT | VF_CORR, P2>;                \
        case VF_ACC_OUT: return v_step<N, VF_ACC_OUT, P2>;                                    \
        case VF_ADJOINT | VF_ACC_OUT: return v_step<N, VF_ADJOINT | VF_ACC_OUT, P2>;          \
        default: return nullptr;                                                              \
        }                                                                                     \
    }                                                                                         \
    KFn v_kernel_fd##N(int flags, bool p2) { return p2 ? v_pick_##N<true>(flags) : v_pick_##N<false>(flags); } \
    template <bool P2>                                                                        \
    static KFn v_pick_st_##N(int flags)                                                       \
    {                                                                                         \
        switch (flags) {                                                                      \
        case 0: return v_step_st<N, 0, P2>;                                                   \
        case VF_HESS: return v_step_st<N, VF_HESS, P2>;                                       \
        case VF_ADJOINT | VF_CORR: return v_step_st<N, VF_ADJOINT | VF_CORR, P2>;             \
        default: return nullptr;                                                              \
        }                                                                                     \
    }                                                                                         \
    KFn v_kernel_st_fd##N(int flags, bool p2) { return p2 ? v_pick_st_##N<true>(flags) : v_pick_st_##N<false>(flags); } \
    template <bool P2>                                                                        \
    static KFn v_pick_tp_##N(int flags)                                                       \
    {                                                                                         \
        switch (flags) {                                                                      \
        case 0: return v_step_tp<N, 0, P2>;                                                   \
        case VF_HESS: return v_step_tp<N, VF_HESS, P2>;                                       \
        case VF_ADJOINT | VF_CORR: return v_step_tp<N, VF_ADJOINT | VF_CORR, P2>;             \
        default: return nullptr;                                                              \
        }                                                                                     \
    }                                                                                         \
    KFn v_kernel_tp_fd##N(int flags, bool p2) { return p2 ? v_pick_tp_##N<true>(flags) : v_pick_tp_##N<false>(flags); } \
    template <bool P2>                                                                        \
    static KFn v_pick_r2_##N(int flags)                                                       \
    {                                                                                         \
        switch (flags) {                                                                      \
        case 0: return v_step_r2<N, 0, P2>;                                                   \
        case VF_HESS: return v_step_r2<N, VF_HESS, P2>;                                       \
        case VF_ADJOINT | VF_CORR: return v_step_r2<N, VF_ADJOINT | VF_CORR, P2>;             \
        default: return nullptr;                                                              \
        }                                                                                     \
    }                                                                                         \
    KFn v_kernel_r2_fd##N(int flags, bool p2) { return p2 ? v_pick_r2_##N<true>(flags) : v_pick_r2_##N<false>(flags); } \
    template <int L>                                                                          \
    static KFn s_pick_##N(int flags)                                                          \
    {                                                                                         \
        switch (flags) {                                                                      \
        case 0: return s_step<N, L, 0>;                                                       \
        case SF_STRAIN_OUT: return s_step<N, L, SF_STRAIN_OUT>;                               \
        case SF_HESS: return s_step<N, L, SF_HESS>;                                           \
        case SF_CORR: return s_step<N, L, SF_CORR>;                                           \
        case SF_STRAIN_OUT | SF_PARAMS: return s_step<N, L, SF_STRAIN_OUT | SF_PARAMS>;       \
        case SF_STRAIN_OUT | SF_QSENS:                                                        \
            if constexpr (L > 0) return s_step<N, L, SF_STRAIN_OUT | SF_QSENS>;               \
            else return nullptr;                                                              \
        case SF_CORR | SF_CORRQ:                                                              \
            if constexpr (L > 0) return s_step<N, L, SF_CORR | SF_CORRQ>;                     \
            else return nullptr;                                                              \
        default: return nullptr;                                                              \
        }                                                                                     \
    }                                                                                         \
    KFn s_kernel_fd##N(int l, int flags)                                                      \
    {                                                                                         \
        switch (l) {                                                                          \
        case 0: return s_pick_##N<0>(flags);                                                  \
        case 1: return s_pick_##N<1>(flags);                                                  \
        case 2: return s_pick_##N<2>(flags);                                                  \
        case 3: return s_pick_##N<3>(flags);                                                  \
        case 4: return s_pick_##N<4>(flags);                                                  \
        default: return nullptr;                                                              \
        }                                                                                     \
    }                                                                                         \
    }

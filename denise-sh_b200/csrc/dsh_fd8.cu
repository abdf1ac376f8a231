/* step kernels for FDORDER=8 */
#include "dsh_inst.cuh"
DSH_INSTANTIATE_FD(8)

/* experimental velocity-kernel variants (DSH_VVAR, FDORDER 8 only) */
namespace dsh {
template <int VAR, bool P2>
static KFn v_exp_pick(int flags)
{
    switch (flags) {
    case 0: return v_step_x<8, 0, P2, VAR>;
    case VF_ADJOINT | VF_CORR: return v_step_x<8, VF_ADJOINT | VF_CORR, P2, VAR>;
    default: return nullptr;
    }
}
KFn v_kernel_exp_fd8(int var, int flags, bool p2)
{
    switch (var) {
    case 1: return p2 ? v_exp_pick<1, true>(flags) : v_exp_pick<1, false>(flags);
    case 2: return p2 ? v_exp_pick<2, true>(flags) : v_exp_pick<2, false>(flags);
    case 3: return p2 ? v_exp_pick<3, true>(flags) : v_exp_pick<3, false>(flags);
    case 4:
        if (flags == 0) return p2 ? v_step_col<8, 0, true> : v_step_col<8, 0, false>;
        if (flags == (VF_ADJOINT | VF_CORR))
            return p2 ? v_step_col<8, VF_ADJOINT | VF_CORR, true> : v_step_col<8, VF_ADJOINT | VF_CORR, false>;
        return nullptr;
    default: return nullptr;
    }
}
}  // namespace dsh

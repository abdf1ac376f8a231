/* fused step kernels for FDORDER=2 */
#include "dsh_fs.h"
#include "dsh_fused.cuh"

namespace dsh {
template <int L, bool P2>
static KFn fs_pick(int mode)
{
    switch (mode) {
    case FM_FWD: return fs_step<2, L, FM_FWD, P2>;
    case FM_STORE: return fs_step<2, L, FM_STORE, P2>;
    case FM_ADJ: return fs_step<2, L, FM_ADJ, P2>;
    default: return nullptr;
    }
}
template <bool P2>
static KFn fs_pick_l(int l, int mode)
{
    switch (l) {
    case 0: return fs_pick<0, P2>(mode);
    case 1: return fs_pick<1, P2>(mode);
    case 2: return fs_pick<2, P2>(mode);
    case 3: return fs_pick<3, P2>(mode);
    case 4: return fs_pick<4, P2>(mode);
    default: return nullptr;
    }
}
KFn fs_kernel_fd2(int l, int mode, bool p2) { return p2 ? fs_pick_l<true>(l, mode) : fs_pick_l<false>(l, mode); }
}  // namespace dsh

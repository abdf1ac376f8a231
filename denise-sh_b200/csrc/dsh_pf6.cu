/* persistent forward-modelling kernels for FDORDER=6 */
#include "dsh_persist.cuh"
#include "dsh_pf.h"

namespace dsh {
template <bool P2>
static PFn pf_pick(int l)
{
    switch (l) {
    case 0: return persist_fwd<6, 0, P2>;
    case 1: return persist_fwd<6, 1, P2>;
    case 2: return persist_fwd<6, 2, P2>;
    case 3: return persist_fwd<6, 3, P2>;
    case 4: return persist_fwd<6, 4, P2>;
    default: return nullptr;
    }
}
PFn pf_kernel_fd6(int l, bool p2) { return p2 ? pf_pick<true>(l) : pf_pick<false>(l); }
}  // namespace dsh

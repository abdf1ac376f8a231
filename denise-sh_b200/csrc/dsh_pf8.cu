/* persistent forward-modelling kernels for FDORDER=8 */
#include "dsh_persist.cuh"
#include "dsh_pf.h"

namespace dsh {
template <bool P2>
static PFn pf_pick(int l)
{
    switch (l) {
    case 0: return persist_fwd<8, 0, P2>;
    case 1: return persist_fwd<8, 1, P2>;
    case 2: return persist_fwd<8, 2, P2>;
    case 3: return persist_fwd<8, 3, P2>;
    case 4: return persist_fwd<8, 4, P2>;
    default: return nullptr;
    }
}
PFn pf_kernel_fd8(int l, bool p2) { return p2 ? pf_pick<true>(l) : pf_pick<false>(l); }
}  // namespace dsh

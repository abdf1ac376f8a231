/* stress kernels of uneven multi-model batches, one per tile-shape variant */
#include "dsh_multi.cuh"

namespace dsh {
MultiFn s_multi_kernel(int variant)
{
    switch (variant) {
    case 0: return s_multi<8, 1>;
    case 1: return s_multi<4, 2>;
    case 2: return s_multi<2, 4>;
    case 3: return s_multi<4, 1>;
    default: return nullptr;
    }
}
MultiPFn s_multi_p_kernel(int variant)
{
    switch (variant) {
    case 0: return s_multi_p<8, 1>;
    case 1: return s_multi_p<4, 2>;
    case 2: return s_multi_p<2, 4>;
    case 3: return s_multi_p<4, 1>;
    default: return nullptr;
    }
}
}  // namespace dsh

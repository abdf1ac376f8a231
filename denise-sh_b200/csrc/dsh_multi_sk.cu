/* stress class kernels of uneven multi-model batches: tile-shape variant x body key */
#include "dsh_multi.cuh"

namespace dsh {
template <int ROWS, int SPB>
static MultiPFn s_key(int key)
{
    switch (key) {
    case 32: return s_multi_k<ROWS, SPB, 32>;
    case 34: return s_multi_k<ROWS, SPB, 34>;
    case 48: return s_multi_k<ROWS, SPB, 48>;
    case 50: return s_multi_k<ROWS, SPB, 50>;
    case 64: return s_multi_k<ROWS, SPB, 64>;
    case 66: return s_multi_k<ROWS, SPB, 66>;
    default: return nullptr;
    }
}
MultiPFn s_multi_k_kernel(int variant, int key)
{
    switch (variant) {
    case 0: return s_key<8, 1>(key);
    case 1: return s_key<4, 2>(key);
    case 2: return s_key<2, 4>(key);
    case 3: return s_key<4, 1>(key);
    default: return nullptr;
    }
}
}  // namespace dsh

/* velocity class kernels of uneven multi-model batches: tile-shape variant x body key */
#include "dsh_multi.cuh"

namespace dsh {
template <int ROWS, int SPB>
static MultiPFn v_key(int key)
{
    switch (key) {
    case 8: return v_multi_k<ROWS, SPB, 8>;
    case 9: return v_multi_k<ROWS, SPB, 9>;
    case 12: return v_multi_k<ROWS, SPB, 12>;
    case 13: return v_multi_k<ROWS, SPB, 13>;
    case 16: return v_multi_k<ROWS, SPB, 16>;
    case 17: return v_multi_k<ROWS, SPB, 17>;
    default: return nullptr;
    }
}
MultiPFn v_multi_k_kernel(int variant, int key)
{
    switch (variant) {
    case 0: return v_key<8, 1>(key);
    case 1: return v_key<4, 2>(key);
    case 2: return v_key<2, 4>(key);
    case 3: return v_key<4, 1>(key);
    default: return nullptr;
    }
}
}  // namespace dsh

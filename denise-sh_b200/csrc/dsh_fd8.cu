/* step kernels for FDORDER=8 */
#include "dsh_inst.cuh"
DSH_INSTANTIATE_FD(8)

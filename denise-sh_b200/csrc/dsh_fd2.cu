/* step kernels for FDORDER=2 */
#include "dsh_inst.cuh"
DSH_INSTANTIATE_FD(2)

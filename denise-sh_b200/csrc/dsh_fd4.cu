/* step kernels for FDORDER=4 */
#include "dsh_inst.cuh"
DSH_INSTANTIATE_FD(4)

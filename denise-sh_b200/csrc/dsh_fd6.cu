/* step kernels for FDORDER=6 */
#include "dsh_inst.cuh"
DSH_INSTANTIATE_FD(6)

/* step kernels for FDORDER=10 */
#include "dsh_inst.cuh"
DSH_INSTANTIATE_FD(10)

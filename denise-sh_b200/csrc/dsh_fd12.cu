/* step kernels for FDORDER=12 */
#include "dsh_inst.cuh"
DSH_INSTANTIATE_FD(12)

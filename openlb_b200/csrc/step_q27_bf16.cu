// D3Q27, bfloat16 storage of scaled shifted populations, float arithmetic
#include "launch_impl.cuh"
OLB_B200_INSTANTIATE(27, __nv_bfloat16, float)

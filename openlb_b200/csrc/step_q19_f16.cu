// D3Q19, IEEE half storage of scaled shifted populations, float arithmetic
#include "launch_impl.cuh"
OLB_B200_INSTANTIATE(19, __half, float)

// D3Q27, IEEE half storage of scaled shifted populations, float arithmetic
#include "launch_impl.cuh"
OLB_B200_INSTANTIATE(27, __half, float)

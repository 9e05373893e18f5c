// D3Q27, float storage, float arithmetic
#include "launch_impl.cuh"
OLB_B200_INSTANTIATE(27, float, float)

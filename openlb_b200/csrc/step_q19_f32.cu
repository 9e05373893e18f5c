// D3Q19, float storage, float arithmetic
#include "launch_impl.cuh"
OLB_B200_INSTANTIATE(19, float, float)

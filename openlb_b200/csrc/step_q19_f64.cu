// D3Q19, double storage, double arithmetic
#include "launch_impl.cuh"
OLB_B200_INSTANTIATE(19, double, double)

// D3Q27, double storage, double arithmetic
#include "launch_impl.cuh"
OLB_B200_INSTANTIATE(27, double, double)

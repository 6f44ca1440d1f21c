// FP64 instantiation of the GJK kernels (compiled with -fmad=false).
#include "gjk_kernels.cuh"

RBPS_INSTANTIATE_GJK(double, double)

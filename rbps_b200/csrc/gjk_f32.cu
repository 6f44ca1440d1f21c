// FP32 instantiation of the GJK kernels (compiled with
// -fmad=false: their GJK / EPA arithmetic is double).
#include "gjk_kernels.cuh"

RBPS_INSTANTIATE_GJK(float, float)

// FP32 instantiations of the step kernels: all-float, and float solver with
// double body positions (far-from-origin scenes).
#include "engine_impl.cuh"
RBPS_INSTANTIATE_ENGINE(float, float)
RBPS_INSTANTIATE_ENGINE(float, double)

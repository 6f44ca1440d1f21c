// FP32 instantiation of the step kernels (RBPS_PRECISION_FP32, and
// RBPS_PRECISION_FP32_POS64, whose positions are float relative to a
// per-world double origin).
#include "engine_impl.cuh"
RBPS_INSTANTIATE_ENGINE(float, float)

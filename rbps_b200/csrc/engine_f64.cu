// FP64 instantiation of the step kernels.  Compiled with -fmad=false so every
// double operation rounds exactly as the reference's x86-64 build (which has
// no FMA contraction).
#include "engine_impl.cuh"
RBPS_INSTANTIATE_ENGINE(double, double)

// FP32 instantiation of the loop kernels: the production path (FP32 state and
// fluxes; FP64 geometry, RK state w and residual norms). FMA contraction on.
#include "ops_impl.cuh"

template struct psst::Ops<float>;

// FP64 instantiation of the loop kernels: the parity path. Compiled with
// -fmad=false so that every multiply and add rounds separately, as in the
// reference built for x86-64 (no FMA contraction).
#include "ops_impl.cuh"

template struct psst::Ops<double>;

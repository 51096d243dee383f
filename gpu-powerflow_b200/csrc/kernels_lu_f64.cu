// kernels_lu_f64.cu -- FP64 instantiations of the front kernels (kernels_lu.cuh);
// split by precision so the two halves compile in parallel.
#include "kernels_lu.cuh"

namespace cupf_b200 {
template void configure_front_kernels<double, double>();
template void launch_factor_single_tree<double, double>(const FactorArgs<double, double>&,
                                                       const SingleTree&, cudaStream_t);
template void launch_factor_level<double, double>(const LevelLaunch&, const FactorArgs<double, double>&,
                                                  cudaStream_t);
template void launch_backward_top<double>(const LevelLaunch&, const int*, int, const SweepArgs<double>&, cudaStream_t);
template void launch_backward_level<double>(const LevelLaunch&, const SweepArgs<double>&, cudaStream_t);
template void launch_ut_forward_level<double>(const LevelLaunch&, const AdjointSweepArgs<double>&, cudaStream_t);
template void launch_l_forward_level<double>(const LevelLaunch&, const AdjointSweepArgs<double>&, cudaStream_t);
template void launch_lt_backward_level<double>(const LevelLaunch&, const AdjointSweepArgs<double>&, cudaStream_t);
}  // namespace cupf_b200

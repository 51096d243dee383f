// kernels_lu_f32.cu -- FP32 instantiations of the front kernels (kernels_lu.cuh);
// split by precision so the two halves compile in parallel.
#include "kernels_lu.cuh"

namespace cupf_b200 {
template void configure_front_kernels<float, float>();
template void launch_factor_single_tree<float, float>(const FactorArgs<float, float>&, const SingleTree&,
                                                cudaStream_t);
template void launch_factor_level<float, float>(const LevelLaunch&, const FactorArgs<float, float>&, cudaStream_t);
template void launch_backward_top<float>(const LevelLaunch&, const int*, int, const SweepArgs<float>&, cudaStream_t);
template void launch_backward_level<float>(const LevelLaunch&, const SweepArgs<float>&, cudaStream_t);
template void launch_ut_forward_level<float>(const LevelLaunch&, const AdjointSweepArgs<float>&, cudaStream_t);
template void launch_l_forward_level<float>(const LevelLaunch&, const AdjointSweepArgs<float>&, cudaStream_t);
template void launch_lt_backward_level<float>(const LevelLaunch&, const AdjointSweepArgs<float>&, cudaStream_t);
}  // namespace cupf_b200

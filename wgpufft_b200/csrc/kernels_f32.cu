// f32 instantiation of the transform kernels (kernels_impl.cuh).
#include "kernels_impl.cuh"
#include "regfft.cuh"

namespace b2f {
template cudaError_t launch_lines_t<float>(const LinesParams&, unsigned, unsigned, size_t,
                                              cudaStream_t);
template cudaError_t launch_rader_t<float>(const RaderParams&, unsigned, unsigned, size_t,
                                              cudaStream_t);
template cudaError_t launch_bluestein_t<float>(const BluesteinParams&, unsigned, unsigned,
                                                  size_t, cudaStream_t);
template cudaError_t launch_scale_copy_t<float>(const void*, void*, uint64_t, double, bool,
                                             cudaStream_t);
template cudaError_t launch_r2c_t<float>(const RealParams&, unsigned, unsigned, size_t,
                                            cudaStream_t);
template cudaError_t launch_c2r_t<float>(const RealParams&, unsigned, unsigned, size_t,
                                            cudaStream_t);
template cudaError_t launch_blue_elem_t<float>(const BlueElemParams&, cudaStream_t);
template cudaError_t launch_pow2_t<float, 16, false>(const LinesParams&, unsigned, unsigned, size_t, cudaStream_t);
template cudaError_t launch_pow2_t<float, 16, true>(const LinesParams&, unsigned, unsigned, size_t, cudaStream_t);
template cudaError_t launch_pow2_t<float, 32, true>(const LinesParams&, unsigned, unsigned, size_t, cudaStream_t);
template cudaError_t launch_real_elem_t<float>(const RealElemParams&, cudaStream_t);
template cudaError_t launch_small_volume_t<float>(const SmallVolumeParams&, unsigned, size_t,
                                                  cudaStream_t);
}  // namespace b2f

// f64 instantiation of the transform kernels (kernels_impl.cuh).
#include "kernels_impl.cuh"
#include "regfft.cuh"

namespace b2f {
template cudaError_t launch_lines_t<double>(const LinesParams&, unsigned, unsigned, size_t,
                                              cudaStream_t);
template cudaError_t launch_rader_t<double>(const RaderParams&, unsigned, unsigned, size_t,
                                              cudaStream_t);
template cudaError_t launch_bluestein_t<double>(const BluesteinParams&, unsigned, unsigned,
                                                  size_t, cudaStream_t);
template cudaError_t launch_scale_copy_t<double>(const void*, void*, uint64_t, double, bool,
                                             cudaStream_t);
template cudaError_t launch_r2c_t<double>(const RealParams&, unsigned, unsigned, size_t,
                                            cudaStream_t);
template cudaError_t launch_c2r_t<double>(const RealParams&, unsigned, unsigned, size_t,
                                            cudaStream_t);
template cudaError_t launch_blue_elem_t<double>(const BlueElemParams&, cudaStream_t);
template cudaError_t launch_pow2_t<double, 16, false>(const LinesParams&, unsigned, unsigned, size_t, cudaStream_t);
template cudaError_t launch_pow2_t<double, 16, true>(const LinesParams&, unsigned, unsigned, size_t, cudaStream_t);
template cudaError_t launch_real_elem_t<double>(const RealElemParams&, cudaStream_t);
}  // namespace b2f

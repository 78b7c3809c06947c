// df64 instantiation of the transform kernels (kernels_impl.cuh).
#include "kernels_impl.cuh"
#include "regfft.cuh"

namespace b2f {
template cudaError_t launch_lines_t<df>(const LinesParams&, unsigned, unsigned, size_t,
                                              cudaStream_t);
template cudaError_t launch_rader_t<df>(const RaderParams&, unsigned, unsigned, size_t,
                                              cudaStream_t);
template cudaError_t launch_bluestein_t<df>(const BluesteinParams&, unsigned, unsigned,
                                                  size_t, cudaStream_t);
template cudaError_t launch_scale_copy_t<df>(const void*, void*, uint64_t, double, bool,
                                             cudaStream_t);
template cudaError_t launch_blue_elem_t<df>(const BlueElemParams&, cudaStream_t);
template cudaError_t launch_pow2_t<df, 16, false>(const LinesParams&, unsigned, unsigned, size_t, cudaStream_t);
template cudaError_t launch_pow2_t<df, 16, true>(const LinesParams&, unsigned, unsigned, size_t, cudaStream_t);
}  // namespace b2f

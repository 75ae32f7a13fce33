// FFT pass launches of the FP32 transform precision (see fft_passes.cuh).
#include "fft_pass_launch.cuh"
#include "fft_plane.cuh"

namespace n2c {
template int fft_launch_pass<float2>(int, int, int, const PassArgs<float2> &, size_t, long long);
template int fft_zline_occupancy<float2>(int, int, int, size_t);
template int fft_plane_launch<float2>(bool, int, const PlaneArgs<float2> &, cudaStream_t);
}  // namespace n2c

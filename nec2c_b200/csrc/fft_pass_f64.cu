// FFT pass launches of the FP64 transform precision (see fft_passes.cuh).
#include "fft_pass_launch.cuh"
#include "fft_plane.cuh"

namespace n2c {
template int fft_launch_pass<double2>(int, int, int, const PassArgs<double2> &, size_t, long long);
template int fft_zline_occupancy<double2>(int, int, int, size_t);
template int fft_plane_launch<double2>(bool, int, const PlaneArgs<double2> &, cudaStream_t);
}  // namespace n2c

// Shared device helpers for the nec2c B200 backend (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

namespace n2c {

// Complex arithmetic on the native vector types: double2 / float2 hold (re, im).
template <typename R> struct cplx_of;
template <> struct cplx_of<double> { using type = double2; };
template <> struct cplx_of<float> { using type = float2; };

__host__ __device__ __forceinline__ double2 mk(double re, double im) { return make_double2(re, im); }
__host__ __device__ __forceinline__ float2 mk(float re, float im) { return make_float2(re, im); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
// conj(a) * b
template <typename C> __device__ __forceinline__ C cconjmul(C a, C b) {
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.x * b.y - a.y * b.x; return r;
}
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(a.x) s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }
template <typename C> __device__ __forceinline__ C czero() { C r; r.x = 0; r.y = 0; return r; }
// a / b with the textbook formula (the reference's complex division is C99's).
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
template <typename C> __device__ __forceinline__ C from_d(double2 a);
template <> __device__ __forceinline__ double2 from_d<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 from_d<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }

__device__ __forceinline__ bool finite2(double2 a) { return isfinite(a.x) && isfinite(a.y); }

// Block-wide sum of a double2 (all threads return the total).  blockDim.x must
// be a multiple of 32 and at most 1024.
__device__ __forceinline__ double2 block_sum(double2 v) {
  __shared__ double2 red[32];
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double2 t = make_double2(0, 0);
  if (lane < nw) t = red[lane];
  for (int o = 16; o > 0; o >>= 1) {
    t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
    t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
  }
  return t;
}

// Programmatic dependent launch.  A kernel launched with programmatic stream
// serialisation may be scheduled while its predecessor in the stream is still
// finishing: it first waits here for that grid to complete and its writes to
// be visible, then lets its own successor begin launching (whose CTAs take the
// SMs this grid's last wave leaves idle, and wait in turn).  Both are no-ops
// for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace n2c

#define N2C_CHECK(call)                                                        \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      n2c_set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
      return 0;                                                                \
    }                                                                          \
  } while (0)

extern "C" void n2c_set_error(const char *fmt, ...);

// Kernels around the split-precision dense LU: FP64 <-> FP32 block copies,
// the infinity norm of A, and the FP64 refinement residual r = b - A x with
// its norms.  The refinement itself (when to stop, when to fall back to the
// FP64 factorisation) is host logic in dense_cuda.c.
#include <float.h>
#include <math.h>
#include <string.h>
#include "common.cuh"
#include "device_api.h"
#include "runtime.cuh"

using namespace n2c;

namespace {

// |Re| + |Im|, the norm LAPACK's complex refinement uses.
__device__ __forceinline__ double cabs1(double2 z) { return fabs(z.x) + fabs(z.y); }

// Non-negative doubles order like their bit patterns: a max-reduction can use
// 64-bit integer atomics.
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *slot, double v) {
  atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

__global__ void narrow_kernel(const double2 *src, long long lds, float2 *dst, long long ldd, long long rows,
                              long long cols) {
  const long long total = rows * cols;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / cols, c = t - r * cols;
    const double2 v = src[r * lds + c];
    dst[r * ldd + c] = make_float2((float)v.x, (float)v.y);
  }
}

__global__ void widen_kernel(const float2 *src, long long lds, double2 *dst, long long ldd, long long rows,
                             long long cols) {
  const long long total = rows * cols;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / cols, c = t - r * cols;
    const float2 v = src[r * lds + c];
    dst[r * ldd + c] = make_double2(v.x, v.y);
  }
}

// Warp per row.
__global__ void norm_inf_kernel(const double2 *a, long long n, long long ld, unsigned long long *out) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long r = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
    double s = 0;
    for (long long c = lane; c < n; c += 32) s += cabs1(a[r * ld + c]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) atomic_max_nonneg(out, s);
  }
}

// r_j = b_j - A x_j, warp per row, all right-hand sides; rnorm[j] = max |r_j|.
__global__ void residual_kernel(const double2 *a, long long n, long long ld, const double2 *x, const double2 *b,
                                double2 *r, long long nrhs, long long ldb, unsigned long long *rnorm) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long row = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); row < n; row += warps) {
    for (long long j = 0; j < nrhs; ++j) {
      const double2 *xj = x + j * ldb;
      double2 s = make_double2(0, 0);
      for (long long c = lane; c < n; c += 32) s = cadd(s, cmul(a[row * ld + c], xj[c]));
      for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      }
      if (lane == 0) {
        const double2 v = csub(b[j * ldb + row], s);
        r[j * ldb + row] = v;
        atomic_max_nonneg(rnorm + j, cabs1(v));
      }
    }
  }
}

__global__ void add_kernel(double2 *x, const double2 *d, long long n, long long nrhs, long long ldb,
                           unsigned long long *xnorm) {
  const long long total = n * nrhs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long j = t / n, i = t - j * n;
    const double2 v = cadd(x[j * ldb + i], d[j * ldb + i]);
    x[j * ldb + i] = v;
    atomic_max_nonneg(xnorm + j, cabs1(v));
  }
}

unsigned grid_for(long long work, int threads) {
  long long b = (work + threads - 1) / threads;
  const long long cap = (long long)n2c_sm_count() * 16;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

// Per-column maxima: cleared, filled by a kernel, read back (synchronises).
int read_maxima(const unsigned long long *dev, long long count, double *host) {
  unsigned long long tmp[64];
  for (long long j0 = 0; j0 < count; j0 += 64) {
    const long long m = count - j0 < 64 ? count - j0 : 64;
    if (!n2d_download(tmp, dev + j0, (size_t)m * sizeof(unsigned long long))) return 0;
    for (long long j = 0; j < m; ++j) {
      double v;
      memcpy(&v, &tmp[j], sizeof(v));
      host[j0 + j] = v;
    }
  }
  return 1;
}

}  // namespace

extern "C" int n2d_narrow(const double *src, long long lds, float *dst, long long ldd, long long rows, long long cols) {
  if (rows <= 0 || cols <= 0) return 1;
  narrow_kernel<<<grid_for(rows * cols, 256), 256, 0, n2c_stream()>>>((const double2 *)src, lds, (float2 *)dst, ldd,
                                                                       rows, cols);
  return n2c_check_launch("narrow");
}

extern "C" int n2d_widen(const float *src, long long lds, double *dst, long long ldd, long long rows, long long cols) {
  if (rows <= 0 || cols <= 0) return 1;
  widen_kernel<<<grid_for(rows * cols, 256), 256, 0, n2c_stream()>>>((const float2 *)src, lds, (double2 *)dst, ldd,
                                                                      rows, cols);
  return n2c_check_launch("widen");
}

extern "C" int n2d_norm_inf(const double *a, long long n, long long ld, void *norm_dev, double *norm_host) {
  unsigned long long *m = (unsigned long long *)norm_dev;
  if (!n2d_memset(m, 0, sizeof(unsigned long long))) return 0;
  norm_inf_kernel<<<grid_for(n * 32, 256), 256, 0, n2c_stream()>>>((const double2 *)a, n, ld, m);
  return n2c_check_launch("norm") && (!norm_host || read_maxima(m, 1, norm_host));
}

extern "C" int n2d_residual(const double *a, long long n, long long ld, const double *x, const double *b, double *r,
                            long long nrhs, long long ldb, void *norm_dev, double *rnorm_host) {
  unsigned long long *m = (unsigned long long *)norm_dev;
  if (!n2d_memset(m, 0, (size_t)nrhs * sizeof(unsigned long long))) return 0;
  residual_kernel<<<grid_for(n * 32, 256), 256, 0, n2c_stream()>>>((const double2 *)a, n, ld, (const double2 *)x,
                                                                    (const double2 *)b, (double2 *)r, nrhs, ldb, m);
  return n2c_check_launch("residual") && (!rnorm_host || read_maxima(m, nrhs, rnorm_host));
}

extern "C" int n2d_add_correction(double *x, const double *d, long long n, long long nrhs, long long ldb,
                                  void *norm_dev, double *xnorm_host) {
  unsigned long long *m = (unsigned long long *)norm_dev;
  if (!n2d_memset(m, 0, (size_t)nrhs * sizeof(unsigned long long))) return 0;
  add_kernel<<<grid_for(n * nrhs, 256), 256, 0, n2c_stream()>>>((double2 *)x, (const double2 *)d, n, nrhs, ldb, m);
  return n2c_check_launch("correction") && (!xnorm_host || read_maxima(m, nrhs, xnorm_host));
}

extern "C" int n2d_read_norms(const void *norm_dev, long long count, double *host) {
  return read_maxima((unsigned long long *)norm_dev, count, host);
}

// Definitions behind fft_passes.cuh, included by the two per-precision
// translation units only.
#pragma once
#include <stdlib.h>

#include <atomic>

#include "fft_passes.cuh"
#include "runtime.cuh"

namespace n2c {

template <typename C, int R1, int R2>
static void (*pass_kernel(int mode))(PassArgs<C>) {
  return mode == 0 ? fft_forward_pass<C, R1, R2>
       : mode == 1 ? fft_inverse_pass<C, R1, R2>
       : mode == 2 ? fft_product_pass<C, R1, R2>
       : mode == 5 ? fft_zline_pass<C, R1, R2, false, false>
       : mode == 6 ? fft_zline_pass<C, R1, R2, true, false>
       : mode == 7 ? fft_zline_pass<C, R1, R2, false, true>
                   : fft_zline_pass<C, R1, R2, true, true>;
}

template <typename C, int R1, int R2>
static int launch_rr(int mode, const PassArgs<C> &a, size_t smem, long long tiles) {
  // Set by whichever worker thread launches a mode first (the attribute
  // calls are idempotent).
  static std::atomic<bool> configured[9];
  void (*k)(PassArgs<C>) = pass_kernel<C, R1, R2>(mode);
  if (!configured[mode].load(std::memory_order_acquire)) {
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess ||
        cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess) {
      n2c_set_error("cannot raise shared memory for FFT pass");
      return 0;
    }
    configured[mode].store(true, std::memory_order_release);
  }
  if (tiles > 0x7fffffffLL) { n2c_set_error("FFT pass grid too large"); return 0; }
  // Programmatic dependent launch (the kernels wait for their predecessor
  // first thing, pdl_begin), so a pass's launch and first CTAs overlap the
  // previous pass's last wave.  NEC2C_CUDA_PDL=0 (read once) turns it off.
  static const bool pdl = [] {
    const char *v = getenv("NEC2C_CUDA_PDL");
    return !(v && v[0] == '0');
  }();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)tiles);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = n2c_stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k, a);
  if (e != cudaSuccess) {
    n2c_set_error("fft pass launch: %s", cudaGetErrorString(e));
    return 0;
  }
  return n2c_check_launch("fft pass");
}

template <typename C, int R1, int R2>
static int occupancy_rr(int mode, size_t smem) {
  void (*k)(PassArgs<C>) = pass_kernel<C, R1, R2>(mode);
  int blocks = 0;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess ||
      cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, 256, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return blocks;
}

// Calls F::template run<R1, R2>() for the split of (L, variant); 0 with the
// error set when the pair is not instantiated.
template <typename F>
static int with_split(int L, int variant, F &&f) {
  if (variant == 1) {
    switch (L) {
      case 16: return f.template run<4, 4>();
      case 32: return f.template run<4, 8>();
      case 64: return f.template run<16, 4>();
      case 128: return f.template run<8, 16>();
    }
  } else if (variant == 0) {
    switch (L) {
      case 1: return f.template run<1, 1>();
      case 2: return f.template run<2, 1>();
      case 4: return f.template run<4, 1>();
      case 8: return f.template run<8, 1>();
      case 16: return f.template run<16, 1>();
      case 32: return f.template run<8, 4>();
      case 64: return f.template run<8, 8>();
      case 128: return f.template run<16, 8>();
      case 256: return f.template run<16, 16>();
      case 512: return f.template run<32, 16>();
      case 1024: return f.template run<32, 32>();
    }
  }
  n2c_set_error("unsupported FFT length %d (radix variant %d)", L, variant);
  return 0;
}

template <typename C>
struct LaunchF {
  int mode;
  const PassArgs<C> &a;
  size_t smem;
  long long tiles;
  template <int R1, int R2> int run() const { return launch_rr<C, R1, R2>(mode, a, smem, tiles); }
};

template <typename C>
struct OccupancyF {
  int mode;
  size_t smem;
  template <int R1, int R2> int run() const { return occupancy_rr<C, R1, R2>(mode, smem); }
};

template <typename C>
int fft_launch_pass(int mode, int L, int variant, const PassArgs<C> &a, size_t smem, long long tiles) {
  return with_split(L, variant, LaunchF<C>{mode, a, smem, tiles});
}

template <typename C>
int fft_zline_occupancy(int mode, int L, int variant, size_t smem) {
  if (mode < 5) return 0;
  const int r = with_split(L, variant, OccupancyF<C>{mode, smem});
  if (!r) cudaGetLastError();
  return r;
}

}  // namespace n2c

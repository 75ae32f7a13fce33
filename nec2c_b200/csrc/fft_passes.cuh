// Launch interface of the line-FFT passes (fft_engine.cuh).
//
// A pass is chosen by its mode, its line length L, the radix split L = R1*R2
// (a "variant" of L) and its tile height NL (PassArgs::NL).  The launches are
// instantiated once per transform precision, in fft_pass_f32.cu and
// fft_pass_f64.cu, so the two compile in parallel and the plan code in vie.cu
// does not carry the kernels.
//
// Modes: strided axes (y, x): 0 forward, 1 inverse, 2 forward x + spectrum
// product + inverse x.  Contiguous axis (z), staged through shared memory:
// 5 forward, 6 inverse, 7 forward with the cell scatter, 8 inverse with the
// permittivity epilogue.
#pragma once
#include <stddef.h>
#include "fft_engine.cuh"

namespace n2c {

// Radix splits on offer for a line of length L (a power of two <= 1024):
// variant 0 is the default split, variant 1 (where it exists) the transposed
// one, which moves work between the two register DFTs and changes how many
// work items each of the two steps has per tile.
inline int fft_radix_variants(int L) { return (L == 16 || L == 32 || L == 64 || L == 128) ? 2 : 1; }

// R1 of variant v of L (R2 = L / R1); 0 for an unsupported pair.
inline int fft_radix_r1(int L, int v) {
  if (v == 1) {
    switch (L) {
      case 16: return 4;
      case 32: return 4;
      case 64: return 16;
      case 128: return 8;
    }
    return 0;
  }
  switch (L) {
    case 1: return 1;
    case 2: return 2;
    case 4: return 4;
    case 8: return 8;
    case 16: return 16;
    case 32: return 8;
    case 64: return 8;
    case 128: return 16;
    case 256: return 16;
    case 512: return 32;
    case 1024: return 32;
  }
  return 0;
}

// One launch of `tiles` CTAs of 256 threads with `smem` bytes of dynamic
// shared memory on the current stream.  Returns 0 (error set) on failure.
template <typename C>
int fft_launch_pass(int mode, int L, int variant, const PassArgs<C> &a, size_t smem, long long tiles);

// Resident CTAs per SM of a staged z pass (modes 5-8) with smem bytes (0 on
// error).
template <typename C>
int fft_zline_occupancy(int mode, int L, int variant, size_t smem);

}  // namespace n2c

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

// ------------------------------------------------- fused yz-plane passes
// (fft_plane.cuh): the y and z transforms of a lattice plane in one kernel,
// for padded y and z axes of the same length P = 2Q.
template <typename C> struct PlaneArgs {
  C *grid;                       // [3][nx][P][P] (y, z padded to P)
  const C *twy, *twz;            // exp(-2 pi i m / P), m < P, of the y and z axes
  int nx, ny, nz;                // lattice
  const int *gate;               // skip all work when *gate == 0 (NULL: always run)
  const double2 *cx;             // cell vector x (3 per cell)
  double2 *cy;                   // cell vector y (inverse pass)
  const double2 *eps;            // per-cell permittivity
  const int *box_cell;           // box index -> cell (-1: empty)
  double2 self0, self1, self2;   // self terms of the Jacobi divisor
  long long mirror;              // PEC physical cells (0: none)
  int precondition;              // the operator acts on x ./ diag
  int *flag;                     // non-finite input / output
  double *partials, *norm;       // |y|^2 reduction (norm NULL: none)
  unsigned int *ticket;
};

// Shared memory of one plane CTA: a Q x (Q+1) tile.
template <typename C> constexpr size_t plane_smem(int Q) { return (size_t)Q * (Q + 1) * sizeof(C); }

// Q (= P/2 of the y and z axes) values the plane kernels are built for.
inline bool plane_supported(int Q) { return Q == 16 || Q == 32 || Q == 64; }

// One plane pass (forward with the cell scatter, or inverse with the
// epilogue) of 12 nx CTAs on stream.  Q as plane_supported; 0 with the error
// set otherwise.
template <typename C>
int fft_plane_launch(bool inverse, int Q, const PlaneArgs<C> &a, cudaStream_t stream);

}  // namespace n2c

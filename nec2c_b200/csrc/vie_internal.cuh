// Device-side state of one volume FFT plan (shared by vie.cu, hybrid.cu, gmres.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

// Tile height (lines per CTA) and radix variant (fft_passes.cuh) of one FFT
// pass; nl == 0 means the heuristic choice.
struct n2d_pass_choice {
  int nl, radix;
};

// The five passes of one matvec: 0 z forward with the cell scatter, 1 y
// forward, 2 x forward + spectrum product + x inverse, 3 y inverse, 4 z
// inverse with the permittivity epilogue.
enum { N2D_VIE_PASSES = 5 };

struct n2d_vie {
  int fp32;                 // 1: FP32 grids/spectrum (FP64 vectors and epilogue)
  long long S[3], P[3];     // lattice shape, padded FFT grid
  long long Ss[3];          // shape sorted descending (spectrum build)
  long long G, nbox, cells, count;
  long long mirror;         // >0: PEC image embedding, cells = 2*mirror (images last)
  int *cell_box;            // [cells] box index of each cell
  int *box_cell;            // [nbox] cell index or -1
  int box_identity;         // 1: every box holds a cell and cell index == box index
  double2 *eps;             // [cells]
  double2 *diag;            // [3 cells] eps - (eps-1) self[i]
  double2 self[3];
  long long H[3], GH;       // octant extents P/2+1 and their product
  void *spec;               // [6][Hx][Hy][Hz] octant of Ghat/G, transform precision
  double2 *spec64;          // same in FP64 (== spec for FP64 plans; mixed plans keep
                            // both: FP32 for Arnoldi products, FP64 for residuals)
  void *box, *t1, *t2;      // work grids, sized for FP64
  double2 *tw64[3];
  float2 *tw32[3];
  double2 *table;           // build only: 6 entries per sorted offset
  int *table_ok, *offsets;
  long long *slab_start, *row_start;
  double *partials;         // reduction scratch
  unsigned int *ticket;
  size_t device_bytes;
  void *gm_work;            // persistent GMRES workspace (gmres.cu)
  // Pass schedule per transform precision (0 FP32, 1 FP64); tuned[i] != 0
  // once the tuner has measured precision i for this plan.
  n2d_pass_choice sched[2][N2D_VIE_PASSES];
  int tuned[2];
  // planes[i] != 0: passes 0-1 and 3-4 of precision i run as the fused
  // yz-plane kernels (fft_plane.cuh) where the grid allows them.
  int planes[2];
};

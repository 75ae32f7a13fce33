// Wire-wire block of the method-of-moments matrix (matrix.c cmset -> cmww
// with the transposed fill, itrp = 1) on the GPU in FP64, for the NEC-2 wire
// engine with the classic thin-wire kernel in free space or over a perfect
// ground.  The stored matrix is NEC's: entry (row i, column b) = the field of
// basis function b tested on segment i, at cm[i * nrow + b].
//
// Step 1, pair kernel: for every observation segment i and source segment j,
// the source's constant, sine and cosine current fields at i's centre with
// i's radius as the observer radius (efld(x_i, y_i, z_i, b_i, i - j),
// fields.c:38-253; i == j takes eksc's diagonal integral), tested along i
// (cmww, matrix.c:880-887):
//   etk, ets, etc = E_k, E_s, E_c . (cab_i, sab_i, salp_i)
// stored per pair, [i][j][3].
//
// Step 2, gather kernel: entry (i, b) = the sum over the source segments j
// that carry basis b (the caller's trio lists, transposed so that j
// increases) of etk a + ets b + etc c (cmww_basis_value, matrix.c:721-740),
// added in the order cmset's source loop adds them; a load impedance z_j
// enters entry (j, b) right after segment j's term as -(a + c) z_j
// (matrix.c:107-121).  No atomics: every entry is one thread's ordered sum.
#include <math.h>
#include <string.h>
#include "common.cuh"
#include "device_api.h"
#include "nec_wire_field.cuh"
#include "runtime.cuh"

namespace {

using namespace n2c_wire;
using n2c::cadd;
using n2c::cmul;
using n2c::csub;

struct FillArgs {
  const Segment *seg;        // segments (wavelengths)
  int n;
  double rkh;                // lumped-element distance (wavelengths)
  int image;                 // perfect ground
  long long row0, rows;      // observation rows of this chunk
  double2 *pair;             // [rows][n][3]: etk, ets, etc
  const int *sup_first;      // n + 1: basis b's entries sup_first[b] .. sup_first[b+1]-1
  const int *sup_src;        // source segment of each entry (increasing within a basis)
  const double2 *sup_coef;   // 3 per entry: constant, sine, cosine coefficients
  const double2 *loads;      // per segment load impedance, or null
  double2 *out;              // [n][nrow]
  long long nrow;
};

// One thread per (observation i, source j); consecutive threads take
// consecutive sources, so the stores of a warp are contiguous.
__global__ void __launch_bounds__(128) pair_kernel(FillArgs a) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.rows * a.n) return;
  const long long r = t / a.n;
  const int j = (int)(t - r * a.n);
  const int i = (int)(a.row0 + r);
  const Segment &o = a.seg[i];
  const SegmentField f = segment_field(a.seg[j], o.x, o.y, o.z, o.b, a.rkh, a.image != 0, i == j);
  double2 *p = a.pair + 3 * t;
  // etk = exk cab + eyk sab + ezk salp, likewise ets and etc.
  for (int c = 0; c < 3; ++c)
    p[c] = cadd(cadd(cscl(f.e[3 * c], o.cab), cscl(f.e[3 * c + 1], o.sab)), cscl(f.e[3 * c + 2], o.salp));
}

// One thread per entry (i, b) of the chunk's rows, b over the padded row.
__global__ void __launch_bounds__(256) gather_kernel(FillArgs a) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.rows * a.nrow) return;
  const long long r = t / a.nrow, b = t - r * a.nrow;
  const long long i = a.row0 + r;
  double2 acc = cx(0.0, 0.0);
  if (b < a.n) {
    const double2 *p = a.pair + r * a.n * 3;
    for (int k = a.sup_first[b]; k < a.sup_first[b + 1]; ++k) {
      const int j = a.sup_src[k];
      const double2 *e = p + 3 * (long long)j, *c = a.sup_coef + 3 * (long long)k;
      acc = cadd(acc, cadd(cadd(cmul(e[0], c[0]), cmul(e[1], c[1])), cmul(e[2], c[2])));
      if (a.loads && j == i) acc = csub(acc, cmul(cadd(c[0], c[2]), a.loads[j]));
    }
  }
  a.out[i * a.nrow + b] = acc;
}

}  // namespace

extern "C" int n2d_mom_fill(const double *seg_dev, int n, double rkh, int image, const int *sup_first_dev,
                            const int *sup_src_dev, const double *sup_coef_dev, const double *loads_dev,
                            double *out_dev, long long nrow) {
  if (n <= 0) return 1;
  if (nrow < n) { n2c_set_error("MoM fill: row length %lld below the order %d", nrow, n); return 0; }
  FillArgs a;
  memset(&a, 0, sizeof(a));
  a.seg = (const Segment *)seg_dev; a.n = n; a.rkh = rkh; a.image = image;
  a.sup_first = sup_first_dev; a.sup_src = sup_src_dev; a.sup_coef = (const double2 *)sup_coef_dev;
  a.loads = (const double2 *)loads_dev; a.out = (double2 *)out_dev; a.nrow = nrow;
  // Observation rows in chunks whose pair fields take at most 512 MB.
  const long long per_row = (long long)n * 3 * (long long)sizeof(double2);
  long long chunk = (512LL << 20) / per_row;
  if (chunk < 1) chunk = 1;
  if (chunk > n) chunk = n;
  double2 *pair = (double2 *)n2d_alloc_async((size_t)(chunk * per_row));
  if (!pair) return 0;
  a.pair = pair;
  int ok = 1;
  for (long long r0 = 0; r0 < n && ok; r0 += chunk) {
    a.row0 = r0;
    a.rows = n - r0 < chunk ? n - r0 : chunk;
    const long long pairs = a.rows * n, entries = a.rows * nrow;
    const long long pb = (pairs + 127) / 128, gb = (entries + 255) / 256;
    if (pb > 0x7fffffffLL || gb > 0x7fffffffLL) { n2c_set_error("MoM fill grid too large"); ok = 0; break; }
    pair_kernel<<<(unsigned)pb, 128, 0, n2c_stream()>>>(a);
    ok = n2c_check_launch("MoM pair fields");
    if (ok) {
      gather_kernel<<<(unsigned)gb, 256, 0, n2c_stream()>>>(a);
      ok = n2c_check_launch("MoM gather");
    }
  }
  n2d_free_async(pair);
  return ok;
}

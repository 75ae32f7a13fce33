// Wire <-> volume coupling blocks of the hybrid conductor + volume system
// (dielectric_wire.c), on the GPU in FP64.
//
// Volume -> wire rows (dielectric_wire.c:1164-1213): the field of a constant
// current density in cell c, point-tested at the centre of wire segment w
// along the segment: the 3x3 electric N dyad of the cuboid
// (dw_point_cuboid_n_free, dielectric_wire.c:101-138: a 10-point Gauss rule
// per axis over the source cuboid of g = exp(-i k r)/(4 pi r) and its second
// derivatives), plus the mirror cuboid's with the image signs diag(-1,-1,+1)
// over a perfect ground (dielectric_wire.c:193-201), tangent-projected and
// divided by i omega eps0.  One warp per (segment, cell).
//
// Wire -> volume rows (dielectric_wire.c:396-510, 316-354): for every
// conductor unknown, the NEC field of its basis currents (the sine, cosine
// and constant current coefficients per segment that the reference's cabc
// produces from a unit vector) averaged over each cell with a 6-point Gauss
// rule per axis, times -i omega eps0 chi.  The field at a point is NEC-2's
// near-field sum over segments (nefld, fields.c:1123-1380) of the thin-wire
// field of each segment (efld, fields.c:38-253: the lumped current element
// beyond rkh wavelengths, otherwise eksc, fields.c:349-393, with the
// segment-end terms gx, fields.c:581-595, and the adaptive Romberg integral
// intx of gf, calculations.c:497-520 and 734-905), in wavelength units, the
// image segment added over a perfect ground.  The average is linear in the
// basis coefficients, so each segment's three fields are averaged over each
// cell once (one warp per (segment, cell), the lanes taking the 216
// quadrature points) and every unknown's row combines those averages.
//
// The NEC field of a segment is nec_wire_field.cuh's.
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

// The volume kernels of dielectric_wire.c use the full-precision pi.
constexpr double FULL_PI = 3.141592653589793238462643383279502884;

struct WireArgs {
  const Segment *seg;       // segments (wavelengths)
  int nseg;
  double rkh;               // lumped-element distance (wavelengths)
  int image;                // perfect ground
  double wlam;              // wavelength (m)
  const double2 *sources;   // [column][segment][3]: constant, sine, cosine coefficients
  int columns;
  const double *center, *size;   // 3 per cell (m)
  const double2 *chi;       // per cell: eps_r - 1
  long long cells;
  double omega_eps0;        // omega * eps0
  const double *node, *weight;   // 6-point Gauss rule on [-1, 1]
  double2 *out;             // [column][3 cells]
  int *error;
};

// The offset nefld (fields.c:1135-1156) gives a point within 0.9 radius of a
// segment's axis (and within its length): that segment's radius.
__device__ double observation_offset(const WireArgs &a, double xo, double yo, double zo) {
  for (int i = 0; i < a.nseg; ++i) {
    const Segment &g = a.seg[i];
    const double dx = xo - g.x, dy = yo - g.y, dz = zo - g.z;
    double zp = g.cab * dx + g.sab * dy + g.salp * dz;
    if (fabs(zp) > 0.5001 * g.s) continue;
    zp = dx * dx + dy * dy + dz * dz - zp * zp;
    if (zp > 0.9 * g.b * g.b) continue;
    return g.b;
  }
  return 0.0;
}

// Step 1: the cell average of each segment's sine, cosine and constant
// current fields, avg[(segment * cells + cell) * 9 + k].  The field of a
// conductor unknown is linear in its basis coefficients, so every unknown's
// average is a combination of these (step 2), and each segment's field is
// evaluated once per quadrature point instead of once per unknown.  One warp
// per (segment, cell): quadrature point p = (ix * 6 + iy) * 6 + iz to lane
// p % 32, the lanes' sums added in lane order.
__global__ void __launch_bounds__(128) segment_average_kernel(WireArgs a, double2 *avg) {
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= (long long)a.nseg * a.cells) return;
  const int segment = (int)(warp / a.cells);
  const long long cell = warp - (long long)segment * a.cells;
  const double *ctr = a.center + 3 * cell, *sz = a.size + 3 * cell;
  double2 acc[9];
  for (int k = 0; k < 9; ++k) acc[k] = cx(0.0, 0.0);
  for (int p = lane; p < 216; p += 32) {
    const int ix = p / 36, iy = (p / 6) % 6, iz = p % 6;
    const double w = a.weight[ix] * a.weight[iy] * a.weight[iz] / 8.0;
    const double xo = (ctr[0] + 0.5 * sz[0] * a.node[ix]) / a.wlam, yo = (ctr[1] + 0.5 * sz[1] * a.node[iy]) / a.wlam,
                 zo = (ctr[2] + 0.5 * sz[2] * a.node[iz]) / a.wlam;
    const double ax = observation_offset(a, xo, yo, zo);
    const SegmentField f = segment_field(a.seg[segment], xo, yo, zo, ax, a.rkh, a.image != 0);
    for (int k = 0; k < 9; ++k) acc[k] = cadd(acc[k], cscl(f.e[k], w));
  }
  for (int k = 0; k < 9; ++k) {
    double re = acc[k].x, im = acc[k].y;
    for (int o = 16; o > 0; o >>= 1) {
      re += __shfl_xor_sync(0xffffffffu, re, o);
      im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    acc[k] = cx(re, im);
  }
  if (lane == 0) {
    double2 *o = avg + ((long long)segment * a.cells + cell) * 9;
    for (int k = 0; k < 9; ++k) o[k] = acc[k];
  }
}

// Step 2: out[column][3 cell + c] = -i omega eps0 chi_cell sum over segments
// (in order) of the unknown's constant, sine and cosine coefficients times
// the segment's averages; segments whose three coefficients are zero are
// skipped, as nefld skips them.
__global__ void __launch_bounds__(256) combine_kernel(WireArgs a, const double2 *avg) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)a.columns * a.cells * 3) return;
  const int c = (int)(t % 3);
  const long long cc = t / 3, cell = cc % a.cells;
  const int column = (int)(cc / a.cells);
  const double2 *src = a.sources + (long long)column * 3 * a.nseg;
  double2 e = cx(0.0, 0.0);
  for (int i = 0; i < a.nseg; ++i) {
    const double2 ak = src[3 * i], bs = src[3 * i + 1], cs = src[3 * i + 2];
    if (ak.x == 0.0 && ak.y == 0.0 && bs.x == 0.0 && bs.y == 0.0 && cs.x == 0.0 && cs.y == 0.0) continue;
    const double2 *g = avg + ((long long)i * a.cells + cell) * 9;
    e = cadd(e, cadd(cadd(cmul(g[c], ak), cmul(g[3 + c], bs)), cmul(g[6 + c], cs)));
  }
  const double2 k = cmul(cx(0.0, -a.omega_eps0), a.chi[cell]);
  a.out[(long long)column * 3 * a.cells + 3 * cell + c] = cmul(k, e);
}

struct VolumeArgs {
  const double *obs;         // 3 per segment (m): the segment centres
  const double *tangent;     // 3 per segment
  int nseg;
  const double *center, *size;   // 3 per cell (m)
  long long cells;
  double k0, omega_eps0;
  int image;                 // perfect ground: the mirror cell, signs diag(-1,-1,+1)
  const double *node, *weight;   // 10-point Gauss rule on [-1, 1]
  double2 *out;              // [segment][3 cells]
};

// Point-tested N dyad of a cuboid, partial sum of the Gauss points
// p = lane, lane + 32, ... (dw_point_cuboid_n_free).
__device__ void cuboid_dyad(const VolumeArgs &a, const double *obs, const double *ctr, const double *sz, int lane,
                            double2 r[9]) {
  for (int i = 0; i < 9; ++i) r[i] = cx(0.0, 0.0);
  const double k0 = a.k0;
  for (int p = lane; p < 1000; p += 32) {
    const int ix = p / 100, iy = (p / 10) % 10, iz = p % 10;
    const int idx[3] = {ix, iy, iz};
    double d[3], r2 = 0.0, w = 1.0;
    for (int ax = 0; ax < 3; ++ax) {
      const double src = ctr[ax] + 0.5 * sz[ax] * a.node[idx[ax]];
      d[ax] = obs[ax] - src;
      r2 += d[ax] * d[ax];
      w *= 0.5 * sz[ax] * a.weight[idx[ax]];
    }
    const double rad = sqrt(r2);
    double sn, cs;
    sincos(k0 * rad, &sn, &cs);
    const double2 g = cdivr(cx(cs, -sn), 4.0 * FULL_PI * rad);
    const double2 diag = cmul(g, cx(k0 * k0 - 1.0 / r2, -k0 / rad));
    const double2 radial = cmul(g, cx(-k0 * k0 + 3.0 / r2, 3.0 * k0 / rad));
    for (int pp = 0; pp < 3; ++pp)
      for (int q = 0; q < 3; ++q) {
        double2 t = cdivr(cscl(cscl(radial, w), d[pp] * d[q]), r2);
        if (pp == q) t = cadd(cscl(diag, w), t);
        r[3 * pp + q] = cadd(r[3 * pp + q], t);
      }
  }
}

// One warp per (segment, cell).
__global__ void __launch_bounds__(128) volume_to_wire_kernel(VolumeArgs a) {
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= (long long)a.nseg * a.cells) return;
  const int segment = (int)(warp / a.cells);
  const long long cell = warp - (long long)segment * a.cells;
  const double *obs = a.obs + 3 * segment, *ctr = a.center + 3 * cell, *sz = a.size + 3 * cell;
  double2 d[9];
  cuboid_dyad(a, obs, ctr, sz, lane, d);
  if (a.image) {
    const double mirror[3] = {ctr[0], ctr[1], -ctr[2]};
    double2 m[9];
    cuboid_dyad(a, obs, mirror, sz, lane, m);
    for (int pp = 0; pp < 3; ++pp)
      for (int q = 0; q < 3; ++q) d[3 * pp + q] = cadd(d[3 * pp + q], cscl(m[3 * pp + q], q == 2 ? 1.0 : -1.0));
  }
  for (int i = 0; i < 9; ++i) {
    double re = d[i].x, im = d[i].y;
    for (int o = 16; o > 0; o >>= 1) {
      re += __shfl_xor_sync(0xffffffffu, re, o);
      im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    d[i] = cx(re, im);
  }
  if (lane == 0) {
    const double *t = a.tangent + 3 * segment;
    double2 *o = a.out + (long long)segment * 3 * a.cells + 3 * cell;
    for (int q = 0; q < 3; ++q) {
      double2 tested = cx(0.0, 0.0);
      for (int pp = 0; pp < 3; ++pp) tested = cadd(tested, cscl(d[3 * pp + q], t[pp]));
      // tested / (i omega eps0) = -i tested / (omega eps0)
      o[q] = cdivr(cx(tested.y, -tested.x), a.omega_eps0);
    }
  }
}

}  // namespace

extern "C" int n2d_coupling_wire_to_volume(const double *seg_dev, int nseg, double rkh, int image, double wlam,
                                           const double *sources_dev, int columns, const double *center_dev,
                                           const double *size_dev, const double *chi_dev, long long cells,
                                           double omega_eps0, const double *node_dev, const double *weight_dev,
                                           double *out_dev) {
  if (columns <= 0 || cells <= 0 || nseg <= 0) return 1;
  WireArgs a;
  memset(&a, 0, sizeof(a));
  a.seg = (const Segment *)seg_dev; a.nseg = nseg; a.rkh = rkh; a.image = image; a.wlam = wlam;
  a.sources = (const double2 *)sources_dev; a.columns = columns;
  a.center = center_dev; a.size = size_dev; a.chi = (const double2 *)chi_dev; a.cells = cells;
  a.omega_eps0 = omega_eps0; a.node = node_dev; a.weight = weight_dev; a.out = (double2 *)out_dev;
  const long long warps = (long long)nseg * cells, blocks = (warps * 32 + 127) / 128;
  const long long outs = (long long)columns * cells * 3, cblocks = (outs + 255) / 256;
  if (blocks > 0x7fffffffLL || cblocks > 0x7fffffffLL) { n2c_set_error("coupling grid too large"); return 0; }
  double2 *avg = (double2 *)n2d_alloc_async((size_t)warps * 9 * sizeof(double2));
  if (!avg) return 0;
  segment_average_kernel<<<(unsigned)blocks, 128, 0, n2c_stream()>>>(a, avg);
  int ok = n2c_check_launch("segment_average");
  if (ok) {
    combine_kernel<<<(unsigned)cblocks, 256, 0, n2c_stream()>>>(a, avg);
    ok = n2c_check_launch("coupling_combine");
  }
  n2d_free_async(avg);
  return ok;
}

extern "C" int n2d_coupling_volume_to_wire(const double *obs_dev, const double *tangent_dev, int nseg,
                                           const double *center_dev, const double *size_dev, long long cells,
                                           double k0, double omega_eps0, int image, const double *node_dev,
                                           const double *weight_dev, double *out_dev) {
  if (nseg <= 0 || cells <= 0) return 1;
  VolumeArgs a;
  memset(&a, 0, sizeof(a));
  a.obs = obs_dev; a.tangent = tangent_dev; a.nseg = nseg; a.center = center_dev; a.size = size_dev;
  a.cells = cells; a.k0 = k0; a.omega_eps0 = omega_eps0; a.image = image; a.node = node_dev;
  a.weight = weight_dev; a.out = (double2 *)out_dev;
  const long long warps = (long long)nseg * cells;
  const long long blocks = (warps * 32 + 127) / 128;
  if (blocks > 0x7fffffffLL) { n2c_set_error("coupling grid too large"); return 0; }
  volume_to_wire_kernel<<<(unsigned)blocks, 128, 0, n2c_stream()>>>(a);
  return n2c_check_launch("volume_to_wire");
}

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
// The constants are NEC's own (nec2c.h: TP = 6.283185308, ETA = 376.73,
// CONST1 = 4.771341189 i), which the parity with the reference needs.
#include <math.h>
#include <string.h>
#include "common.cuh"
#include "device_api.h"
#include "runtime.cuh"

namespace {

using n2c::cadd;
using n2c::cmul;
using n2c::csub;

constexpr double NEC_TP = 6.283185308;
constexpr double NEC_ETA = 376.73;
constexpr double NEC_PI = 3.141592654;
constexpr double NEC_CONST1 = 4.771341189;   // imaginary part of CONST1
// The volume kernels of dielectric_wire.c use the full-precision pi.
constexpr double FULL_PI = 3.141592653589793238462643383279502884;

__device__ __forceinline__ double2 cx(double re, double im) { return make_double2(re, im); }
__device__ __forceinline__ double2 cscl(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cdivr(double2 a, double d) { return make_double2(a.x / d, a.y / d); }
// i * CONST1 * a
__device__ __forceinline__ double2 mul_const1(double2 a) { return make_double2(-NEC_CONST1 * a.y, NEC_CONST1 * a.x); }

struct Segment {
  double x, y, z, s, b, cab, sab, salp;
};

// Segment end term of the thin-wire kernel at axial distance zz, radius rh
// (gx): gz = exp(-i k r) / r, gzp = -(1 + i k r) gz / r^2.
__device__ __forceinline__ void end_term(double zz, double rh, double xk, double2 &gz, double2 &gzp) {
  const double r2 = zz * zz + rh * rh, r = sqrt(r2), rkz = xk * r;
  double sn, cs;
  sincos(rkz, &sn, &cs);
  gz = cdivr(cx(cs, -sn), r);
  gzp = cdivr(cscl(cmul(cx(1.0, rkz), gz), -1.0), r2);
}

// Integrand of the constant-current term (gf with a non-diagonal pair):
// sin(rk)/rk and cos(rk)/rk at kz = zk, rk = sqrt(rkb2 + (zk - zpk)^2).
__device__ __forceinline__ void filament(double zk, double zpk, double rkb2, double &co, double &si) {
  const double zdk = zk - zpk, rk = sqrt(rkb2 + zdk * zdk);
  double sn, cs;
  sincos(rk, &sn, &cs);
  si = sn / rk;
  co = cs / rk;
}

// Relative differences of two Romberg estimates (test, calculations.c:913-937).
__device__ __forceinline__ void romberg_gap(double f1r, double f2r, double f1i, double f2i, double &tr, double &ti) {
  double den = fabs(f2r);
  tr = fabs(f2i);
  if (den < tr) den = tr;
  if (den < 0.0) den = 0.0;
  if (den < 1.0e-37) { tr = 0.0; ti = 0.0; return; }
  tr = fabs((f1r - f2r) / den);
  ti = fabs((f1i - f2i) / den);
}

// Adaptive Romberg integral of filament() over [el1, el2] (intx with a
// non-diagonal pair): panels of 3- and 5-point Romberg estimates, the step
// halved while the 5-point estimate moves by more than 1e-4 relative (at most
// 65536 panels) and doubled after four accepted panels.
__device__ void romberg_filament(double el1, double el2, double zpk, double rkb2, double &sgr, double &sgi) {
  const int nx = 1, nma = 65536, nts = 4;
  const double rx = 1.0e-4;
  double z = el1;
  const double ze = el2, s = ze - z, ep = s / (10.0 * nma), zend = ze - ep;
  sgr = 0.0;
  sgi = 0.0;
  int ns = nx, nt = 0;
  bool fresh = true;
  double dz = 0.0, dzot = 0.0, g1r, g1i, g3r = 0.0, g3i = 0.0, g5r = 0.0, g5i = 0.0;
  filament(z, zpk, rkb2, g1r, g1i);
  for (int guard = 0; guard < 4 * nma + 64; ++guard) {
    if (fresh) {
      dz = s / (double)ns;
      double zp = z + dz;
      if (zp > ze) {
        dz = ze - z;
        if (fabs(dz) <= ep) return;
      }
      dzot = dz * 0.5;
      filament(z + dzot, zpk, rkb2, g3r, g3i);
      filament(z + dz, zpk, rkb2, g5r, g5i);
    }
    const double t00r = (g1r + g5r) * dzot, t00i = (g1i + g5i) * dzot;
    const double t01r = (t00r + dz * g3r) * 0.5, t01i = (t00i + dz * g3i) * 0.5;
    const double t10r = (4.0 * t01r - t00r) / 3.0, t10i = (4.0 * t01i - t00i) / 3.0;
    double te1r, te1i;
    romberg_gap(t01r, t10r, t01i, t10i, te1r, te1i);
    if (te1i <= rx && te1r <= rx) {
      sgr += t10r;
      sgi += t10i;
      nt += 2;
      z += dz;
      if (z >= zend) return;
      g1r = g5r;
      g1i = g5i;
      if (nt >= nts && ns > nx) { ns /= 2; nt = 1; }
      fresh = true;
      continue;
    }
    double g2r, g2i, g4r, g4i;
    filament(z + dz * 0.25, zpk, rkb2, g2r, g2i);
    filament(z + dz * 0.75, zpk, rkb2, g4r, g4i);
    const double t02r = (t01r + dzot * (g2r + g4r)) * 0.5, t02i = (t01i + dzot * (g2i + g4i)) * 0.5;
    const double t11r = (4.0 * t02r - t01r) / 3.0, t11i = (4.0 * t02i - t01i) / 3.0;
    const double t20r = (16.0 * t11r - t10r) / 15.0, t20i = (16.0 * t11i - t10i) / 15.0;
    double te2r, te2i;
    romberg_gap(t11r, t20r, t11i, t20i, te2r, te2i);
    if ((te2i > rx || te2r > rx) && ns < nma) {
      nt = 0;
      ns *= 2;
      dz = s / (double)ns;
      dzot = dz * 0.5;
      g5r = g3r; g5i = g3i;
      g3r = g2r; g3i = g2i;
      fresh = false;
      continue;
    }
    if (te2i > rx || te2r > rx) nt = 0;   // step size limited: the estimate is kept
    sgr += t20r;
    sgi += t20i;
    nt++;
    z += dz;
    if (z >= zend) return;
    g1r = g5r;
    g1i = g5i;
    if (nt >= nts && ns > nx) { ns /= 2; nt = 1; }
    fresh = true;
  }
}

// Axial and radial fields of the sine, cosine and constant current filaments
// of a segment by the thin-wire approximation (eksc with a non-diagonal
// pair); s segment length, z axial and rh radial observation coordinate.
struct FilamentFields {
  double2 ezs, ers, ezc, erc, ezk, erk;
};
__device__ FilamentFields thin_wire(double s, double z, double rh, double xk) {
  FilamentFields f;
  const double zpk = xk * z, rhk = xk * rh, rkb2 = rhk * rhk, sh = 0.5 * s, shk = xk * sh;
  double ss, cs;
  sincos(shk, &ss, &cs);
  const double z2a = sh - z, z1a = -(sh + z);
  double2 gz1, gp1, gz2, gp2;
  end_term(z1a, rh, xk, gz1, gp1);
  end_term(z2a, rh, xk, gz2, gp2);
  double2 gzp1 = cscl(gp1, z1a), gzp2 = cscl(gp2, z2a);
  f.ezs = mul_const1(csub(cscl(csub(gz2, gz1), cs * xk), cscl(cadd(gzp2, gzp1), ss)));
  f.ezc = cscl(mul_const1(cadd(cscl(cadd(gz2, gz1), ss * xk), cscl(csub(gzp2, gzp1), cs))), -1.0);
  f.erk = mul_const1(cscl(csub(gp2, gp1), rh));
  double cint, sint;
  romberg_filament(-shk, shk, zpk, rkb2, cint, sint);
  f.ezk = cscl(mul_const1(cadd(csub(gzp2, gzp1), cscl(cx(cint, -sint), xk * xk))), -1.0);
  gzp1 = cscl(gzp1, z1a);
  gzp2 = cscl(gzp2, z2a);
  if (rh >= 1.0e-10) {
    f.ers = cscl(mul_const1(cdivr(csub(cscl(cadd(cadd(gzp2, gzp1), cadd(gz2, gz1)), ss),
                                       cscl(csub(cscl(gz2, z2a), cscl(gz1, z1a)), cs * xk)), rh)), -1.0);
    f.erc = cscl(mul_const1(cdivr(cadd(cscl(cadd(csub(gzp2, gzp1), csub(gz2, gz1)), cs),
                                       cscl(cadd(cscl(gz2, z2a), cscl(gz1, z1a)), ss * xk)), rh)), -1.0);
  } else {
    f.ers = cx(0.0, 0.0);
    f.erc = cx(0.0, 0.0);
  }
  return f;
}

// Field at (xi, yi, zi) (wavelengths) of the sine (s), cosine (c) and
// constant (k) currents of segment g (efld with a point observer, NEC-2
// kernel): 9 complex components, x y z of k, s, c.  image: a perfect ground,
// whose mirror segment is added with the opposite sign (frati = 1).
struct SegmentField {
  double2 e[9];   // exk eyk ezk exs eys ezs exc eyc ezc
};
__device__ SegmentField segment_field(const Segment &g, double xi, double yi, double zi, double ai, double rkh,
                                      bool image) {
  SegmentField out;
  const double xij = xi - g.x, yij = yi - g.y;
  double rfl = -1.0;
  for (int ip = 0; ip < (image ? 2 : 1); ++ip) {
    rfl = -rfl;
    const double salpr = g.salp * rfl, zij = zi - rfl * g.z;
    const double zp = xij * g.cab + yij * g.sab + zij * salpr;
    double rhox = xij - g.cab * zp, rhoy = yij - g.sab * zp, rhoz = zij - salpr * zp;
    const double rh = sqrt(rhox * rhox + rhoy * rhoy + rhoz * rhoz + ai * ai);
    if (rh <= 1.e-10) {
      rhox = 0.0; rhoy = 0.0; rhoz = 0.0;
    } else {
      rhox = rhox / rh; rhoy = rhoy / rh; rhoz = rhoz / rh;
    }
    const double r = sqrt(zp * zp + rh * rh);
    double2 tk[3], ts[3], tc[3];
    double2 tezk, terk, tezc, terc;
    if (r >= rkh) {
      // Lumped current element beyond rkh wavelengths.
      double rmag = NEC_TP * r;
      const double cth = zp / r, px = rh / r;
      double sn, cs;
      sincos(rmag, &sn, &cs);
      const double2 txk = cx(cs, -sn);
      const double py = NEC_TP * r * r;
      const double2 tyk = cdivr(cmul(cscl(txk, NEC_ETA * cth), cx(1.0, -1.0 / rmag)), py);
      const double2 tzk = cdivr(cmul(cscl(txk, NEC_ETA * px), cx(1.0, rmag - 1.0 / rmag)), 2.0 * py);
      tezk = csub(cscl(tyk, cth), cscl(tzk, px));
      terk = cadd(cscl(tyk, px), cscl(tzk, cth));
      rmag = sin(NEC_PI * g.s) / NEC_PI;
      tezc = cscl(tezk, rmag);
      terc = cscl(terk, rmag);
      tezk = cscl(tezk, g.s);
      terk = cscl(terk, g.s);
      ts[0] = ts[1] = ts[2] = cx(0.0, 0.0);
    } else {
      const FilamentFields f = thin_wire(g.s, zp, rh, NEC_TP);
      tezk = f.ezk; terk = f.erk; tezc = f.ezc; terc = f.erc;
      ts[0] = cadd(cscl(f.ezs, g.cab), cscl(f.ers, rhox));
      ts[1] = cadd(cscl(f.ezs, g.sab), cscl(f.ers, rhoy));
      ts[2] = cadd(cscl(f.ezs, salpr), cscl(f.ers, rhoz));
    }
    tk[0] = cadd(cscl(tezk, g.cab), cscl(terk, rhox));
    tk[1] = cadd(cscl(tezk, g.sab), cscl(terk, rhoy));
    tk[2] = cadd(cscl(tezk, salpr), cscl(terk, rhoz));
    tc[0] = cadd(cscl(tezc, g.cab), cscl(terc, rhox));
    tc[1] = cadd(cscl(tezc, g.sab), cscl(terc, rhoy));
    tc[2] = cadd(cscl(tezc, salpr), cscl(terc, rhoz));
    if (ip == 1) {
      for (int a = 0; a < 3; ++a) {
        out.e[a] = csub(out.e[a], tk[a]);
        out.e[3 + a] = csub(out.e[3 + a], ts[a]);
        out.e[6 + a] = csub(out.e[6 + a], tc[a]);
      }
    } else {
      for (int a = 0; a < 3; ++a) { out.e[a] = tk[a]; out.e[3 + a] = ts[a]; out.e[6 + a] = tc[a]; }
    }
  }
  return out;
}

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

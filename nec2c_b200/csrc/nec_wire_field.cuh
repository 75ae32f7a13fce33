// NEC-2 thin-wire field of a segment's sine, cosine and constant currents
// on the GPU in FP64 (efld, eksc, gx, gf, intx and test of fields.c and
// calculations.c), shared by the wire <-> volume coupling blocks
// (coupling.cu) and the wire MoM fill (mom_fill.cu).  Lengths in
// wavelengths.
//
// The constants are NEC's own (nec2c.h: TP = 6.283185308, ETA = 376.73,
// PI = 3.141592654, CONST1 = 4.771341189 i), which the parity with the
// reference needs.
#pragma once
#include <math.h>
#include "common.cuh"

namespace n2c_wire {

using n2c::cadd;
using n2c::cmul;
using n2c::csub;

constexpr double NEC_TP = 6.283185308;
constexpr double NEC_ETA = 376.73;
constexpr double NEC_PI = 3.141592654;
constexpr double NEC_CONST1 = 4.771341189;   // imaginary part of CONST1

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

// Integrand of the constant-current term (gf, calculations.c:497-520):
// sin(rk)/rk and cos(rk)/rk at kz = zk, rk = sqrt(rkb2 + (zk - zpk)^2).  For
// the diagonal term (a segment's field on itself) the cosine part is
// (cos(rk) - 1)/rk, whose 1/rk singularity the integral adds analytically;
// below rk = 0.2 it is NEC's three-term series.
template <bool DIAG>
__device__ __forceinline__ void filament(double zk, double zpk, double rkb2, double &co, double &si) {
  const double zdk = zk - zpk, rk = sqrt(rkb2 + zdk * zdk);
  double sn, cs;
  sincos(rk, &sn, &cs);
  si = sn / rk;
  if (!DIAG) {
    co = cs / rk;
  } else if (rk >= 0.2) {
    co = (cs - 1.0) / rk;
  } else {
    const double rks = rk * rk;
    co = ((-1.38888889e-3 * rks + 4.16666667e-2) * rks - 0.5) * rk;
  }
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

// Adaptive Romberg integral of filament() over [el1, el2] (intx,
// calculations.c:734-905): panels of 3- and 5-point Romberg estimates, the
// step halved while the 5-point estimate moves by more than 1e-4 relative
// (at most 65536 panels) and doubled after four accepted panels.  The
// diagonal term integrates [el1, 0] of the symmetric integrand, doubles it
// and adds the integral of the 1/rk singularity, log((sqrt(b^2 + s^2) + s)/b)
// with b = k rh (rhk) and s = -el1.
template <bool DIAG>
__device__ void romberg_filament(double el1, double el2, double zpk, double rkb2, double rhk, double &sgr,
                                 double &sgi) {
  const int nx = 1, nma = 65536, nts = 4;
  const double rx = 1.0e-4;
  double z = el1;
  const double ze = DIAG ? 0.0 : el2, s = ze - z, ep = s / (10.0 * nma), zend = ze - ep;
  sgr = 0.0;
  sgi = 0.0;
  auto finish = [&]() {
    if (DIAG) {
      sgr = 2.0 * (sgr + log((sqrt(rhk * rhk + s * s) + s) / rhk));
      sgi = 2.0 * sgi;
    }
  };
  int ns = nx, nt = 0;
  bool fresh = true;
  double dz = 0.0, dzot = 0.0, g1r, g1i, g3r = 0.0, g3i = 0.0, g5r = 0.0, g5i = 0.0;
  filament<DIAG>(z, zpk, rkb2, g1r, g1i);
  for (int guard = 0; guard < 4 * nma + 64; ++guard) {
    if (fresh) {
      dz = s / (double)ns;
      double zp = z + dz;
      if (zp > ze) {
        dz = ze - z;
        if (fabs(dz) <= ep) { finish(); return; }
      }
      dzot = dz * 0.5;
      filament<DIAG>(z + dzot, zpk, rkb2, g3r, g3i);
      filament<DIAG>(z + dz, zpk, rkb2, g5r, g5i);
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
      if (z >= zend) { finish(); return; }
      g1r = g5r;
      g1i = g5i;
      if (nt >= nts && ns > nx) { ns /= 2; nt = 1; }
      fresh = true;
      continue;
    }
    double g2r, g2i, g4r, g4i;
    filament<DIAG>(z + dz * 0.25, zpk, rkb2, g2r, g2i);
    filament<DIAG>(z + dz * 0.75, zpk, rkb2, g4r, g4i);
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
    if (z >= zend) { finish(); return; }
    g1r = g5r;
    g1i = g5i;
    if (nt >= nts && ns > nx) { ns /= 2; nt = 1; }
    fresh = true;
  }
}

// Axial and radial fields of the sine, cosine and constant current filaments
// of a segment by the thin-wire approximation (eksc, fields.c:349-393); s
// segment length, z axial and rh radial observation coordinate; DIAG: the
// segment's field on itself.
struct FilamentFields {
  double2 ezs, ers, ezc, erc, ezk, erk;
};
template <bool DIAG>
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
  romberg_filament<DIAG>(-shk, shk, zpk, rkb2, rhk, cint, sint);
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
// constant (k) currents of segment g (efld, fields.c:38-253, NEC-2 kernel):
// 9 complex components, x y z of k, s, c.  ai: the observer's radius (0 for
// a point).  image: a perfect ground, whose mirror segment is added with the
// opposite sign (frati = 1).  diag: the observer is the segment's own centre
// (ij = 0: the direct term takes the diagonal integral; the image's never).
struct SegmentField {
  double2 e[9];   // exk eyk ezk exs eys ezs exc eyc ezc
};
__device__ inline SegmentField segment_field(const Segment &g, double xi, double yi, double zi, double ai, double rkh,
                                      bool image, bool diag = false) {
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
      const FilamentFields f = (diag && ip == 0) ? thin_wire<true>(g.s, zp, rh, NEC_TP)
                                                 : thin_wire<false>(g.s, zp, rh, NEC_TP);
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


}  // namespace n2c_wire

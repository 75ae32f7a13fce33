// Volume FFT operator of the nec2c dielectric path on sm_100a.
//
// Replaces the builtin/FFTW plan of vie_fft.c: the Green spectrum build
// (vie_fft.c:338-377, far pairs quadratured on the GPU), the matvec
// y = eps x - (eps-1) gather(IFFT(Ghat FFT(scatter x)))   (vie_fft.c:239-263)
// and the Jacobi preconditioner (vie_fft.c:265-273).
//
// HBM layout (one plan):
//   box  [3][nx][ny][nz]      planar source / field on the lattice box
//   T1   [3][nx][ny][Pz]      after the z transform (x<nx, y<ny only)
//   T2   [3][nx][Py][Pz]      after the y transform (x<nx only)
//   spec [6][Px][Py][Pz]      Ghat / G (xx yy zz xy xz yz), 1/G folded in
// The zero half of the padded source is never stored and the discarded half of
// the inverse transform is never computed past the pass that drops it.
#include <math.h>
#include <string.h>
#include <vector>
#include "common.cuh"
#include "device_api.h"
#include <atomic>
#include <mutex>
#include "fft_passes.cuh"
#include "runtime.cuh"
#include "vie_internal.cuh"
#include "vie_batch.cuh"

using namespace n2c;

// ------------------------------------------------------------ pass schedule
// The passes themselves are launched through fft_passes.cuh.  Each of the
// five matvec passes runs with a tile height and radix split taken from the
// plan's schedule: the heuristic below, or the measured choice of the tuner
// (n2d_vie_tune).

// Lines per tile of a strided pass: as many as fit a ~48 KB tile (four CTAs
// per SM), <= 32.
static int lines_per_tile(int L, int ncomp, size_t elem) {
  size_t per_line = (size_t)L * ncomp * elem;
  int nl = 32;
  while (nl > 1 && (size_t)nl * per_line > 48 * 1024) nl >>= 1;
  return nl;
}

// ceil(2^32 / d) for the device's multiply-high division (0 for d == 1).
static unsigned div_magic(long long d) {
  return d <= 1 ? 0u : (unsigned)((0x100000000ULL + (unsigned long long)d - 1) / (unsigned long long)d);
}

// Lines per tile of a staged z pass: two padded [L][NL+1] buffers within
// ~56 KB (three to four blocks per SM); `unit` keeps NL a multiple of 3 for
// cell tiles.
static int zlines_per_tile(int L, size_t elem, int unit) {
  int nl = 32 * unit;
  while (nl > unit && (size_t)2 * (nl + 1) * L * elem > 56 * 1024) nl -= unit;
  return nl;
}

// Lines per tile of a staged z pass covering `groups` groups of `unit` lines,
// chosen to fill whole waves of resident blocks: among heights from half the
// default up to buffers of 80 KB, the one that leaves the fewest block slots
// of the last wave idle (a grid just past one wave would take two).  Ties go
// to more resident blocks per SM, then to the taller tile.  Cached per shape.
template <typename C>
static int zline_tile(int mode, int L, int unit, long long groups) {
  struct Entry { int mode, L, unit, elem; long long groups; int nl; };
  static Entry cache[32];
  static int used = 0;
  static std::mutex lock;
  {
    std::lock_guard<std::mutex> hold(lock);
    for (int i = 0; i < used; ++i)
      if (cache[i].mode == mode && cache[i].L == L && cache[i].unit == unit && cache[i].elem == (int)sizeof(C) &&
          cache[i].groups == groups)
        return cache[i].nl;
  }
  const int def = zlines_per_tile(L, sizeof(C), unit);
  const int sms = n2c_sm_count();
  int best = def, best_bps = 0;
  double best_eff = -1.0;
  for (int nl = (def / 2 / unit > 0 ? def / 2 / unit : 1) * unit; (size_t)2 * (nl + 1) * L * sizeof(C) <= 80 * 1024;
       nl += unit) {
    const size_t smem = (size_t)2 * (nl + 1) * L * sizeof(C);
    const int bps = fft_zline_occupancy<C>(mode, L, 0, smem);
    if (bps <= 0) continue;
    const long long per = nl / unit, tiles = (groups + per - 1) / per, slots = (long long)sms * bps;
    const long long waves = (tiles + slots - 1) / slots;
    const double eff = (double)tiles / (double)(waves * slots);
    if (eff > best_eff + 0.02 || (eff > best_eff - 0.02 && (bps > best_bps || (bps == best_bps && nl > best)))) {
      if (eff > best_eff) best_eff = eff;
      best = nl;
      best_bps = bps;
    }
  }
  std::lock_guard<std::mutex> hold(lock);
  if (used < 32) cache[used++] = Entry{mode, L, unit, (int)sizeof(C), groups, best};
  return best;
}

// log2(v) for a power of two v > 0, else -1.
static int ilog2_exact(long long v) {
  if (v <= 0 || (v & (v - 1))) return -1;
  int k = 0;
  while ((1LL << k) < v) ++k;
  return k;
}

// Shift forms of the strided passes' index arithmetic (PassArgs::pow2), set
// once NL, I and Pz are final.
template <typename C> static void set_shifts(PassArgs<C> &a) {
  const int nl = ilog2_exact(a.NL), ii = ilog2_exact(a.I), pz = a.Pz ? ilog2_exact(a.Pz) : 0;
  a.pow2 = nl >= 0 && ii >= 0 && pz >= 0;
  a.nl_log2 = nl; a.i_log2 = ii; a.pz_log2 = pz;
}

// One axis transform over a batch of lines.  Element e of line (b, i) lives at
// (b*A + e)*I + i; lines = B*I.  Strided lines (I > 1) take the tile height
// and radix split of `ch` (heuristic height when ch.nl == 0); contiguous lines
// (the spectrum build) always take the heuristic.
template <typename C>
static int axis_pass(int mode, int L, const C *in, C *out, const C *tw, long long B, long long I,
                     long long A_in, long long A_out, int n_in, int n_out, n2d_pass_choice ch = {0, 0}) {
  PassArgs<C> a;
  memset(&a, 0, sizeof(a));
  a.in = in; a.out = out; a.tw = tw;
  a.lines = B * I; a.I = I; a.A_in = A_in; a.A_out = A_out; a.n_in = n_in; a.n_out = n_out;
  a.gate = n2c_gate();
  if (I == 1) {
    a.NL = zline_tile<C>(mode + 5, L, 1, a.lines);
    a.nl_div = div_magic(a.NL);
    a.nout_div = div_magic(a.n_out);
    const long long tiles = (a.lines + a.NL - 1) / a.NL;
    return fft_launch_pass<C>(mode + 5, L, 0, a, (size_t)2 * (a.NL + 1) * L * sizeof(C), tiles);
  }
  a.NL = ch.nl ? ch.nl : lines_per_tile(L, 1, sizeof(C));
  set_shifts(a);
  const long long tiles = (a.lines + a.NL - 1) / a.NL;
  return fft_launch_pass<C>(mode, L, ch.radix, a, (size_t)L * a.NL * sizeof(C), tiles);
}

// Launch description of one pass: its arguments, kernel mode, line length,
// radix variant, dynamic shared memory and tile count.
template <typename C> struct PassPlan {
  PassArgs<C> a;
  int mode, L, variant;
  size_t smem;
  long long tiles;
};

template <typename C>
static void product_plan(const n2d_vie *p, const C *in, C *out, const C *tw, const C *spec, n2d_pass_choice ch,
                         PassPlan<C> *pp) {
  const int L = (int)p->P[0], nx = (int)p->S[0];
  const long long I = p->P[1] * p->P[2];
  PassArgs<C> &a = pp->a;
  memset(&a, 0, sizeof(a));
  a.in = in; a.out = out; a.tw = tw; a.spec = spec;
  a.lines = I; a.I = I; a.A_in = nx; a.A_out = nx; a.n_in = nx; a.n_out = nx;
  a.comp_in = (long long)nx * I; a.comp_out = (long long)nx * I; a.spec_comp = p->GH;
  a.Py = (int)p->P[1]; a.Pz = (int)p->P[2]; a.Hy = (int)p->H[1]; a.Hz = (int)p->H[2];
  a.NL = ch.nl ? ch.nl : lines_per_tile(L, 3, sizeof(C));
  a.gate = n2c_gate();
  set_shifts(a);
  pp->mode = 2; pp->L = L; pp->variant = ch.radix;
  pp->smem = (size_t)3 * L * a.NL * sizeof(C);

  pp->tiles = (a.lines + a.NL - 1) / a.NL;
}

// Strided y pass of the matvec (mode 0 forward, 1 inverse).
template <typename C>
static void strided_plan(int mode, int L, const C *in, C *out, const C *tw, long long B, long long I,
                         long long A_in, long long A_out, int n_in, int n_out, n2d_pass_choice ch, PassPlan<C> *pp) {
  PassArgs<C> &a = pp->a;
  memset(&a, 0, sizeof(a));
  a.in = in; a.out = out; a.tw = tw;
  a.lines = B * I; a.I = I; a.A_in = A_in; a.A_out = A_out; a.n_in = n_in; a.n_out = n_out;
  a.gate = n2c_gate();
  a.NL = ch.nl ? ch.nl : lines_per_tile(L, 1, sizeof(C));
  set_shifts(a);
  pp->mode = mode; pp->L = L; pp->variant = ch.radix;
  pp->smem = (size_t)L * a.NL * sizeof(C);
  pp->tiles = (a.lines + a.NL - 1) / a.NL;
}

// --------------------------------------------------------- scatter / gather
// box[c][b] = z(cell(b))_c, z = x or x ./ diag.  Non-finite z raises *flag.
// With PEC images (mirror > 0) cell m+c is the image of cell c and carries
// diag(-1,-1,+1) times its source (dielectric_fft.c:44-50).
template <typename C>
__global__ void scatter_kernel(const double2 *__restrict__ x, const double2 *__restrict__ diag,
                               const int *__restrict__ box_cell, C *__restrict__ box,
                               long long nbox, long long mirror, int *flag, const int *gate) {
  if (gated_off(gate)) return;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nbox;
       b += (long long)gridDim.x * blockDim.x) {
    long long cell = box_cell[b];
    double sgn[3] = {1, 1, 1};
    if (mirror && cell >= mirror) { cell -= mirror; sgn[0] = -1; sgn[1] = -1; }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double2 v = make_double2(0, 0);
      if (cell >= 0) {
        v = x[3LL * cell + c];
        if (diag) v = cdiv(v, diag[3LL * cell + c]);
        if (flag && !finite2(v)) *flag = 1;
        v.x *= sgn[c]; v.y *= sgn[c];
      }
      box[c * nbox + b] = from_d<C>(v);
    }
  }
}

// y = eps z - (eps-1) field, per cell; optional sum |y|^2 (deterministic).
template <typename C>
__global__ void gather_kernel(const double2 *__restrict__ x, const double2 *__restrict__ diag,
                              const double2 *__restrict__ eps, const int *__restrict__ cell_box,
                              const C *__restrict__ box, long long nbox, long long cells,
                              double2 *__restrict__ y, double *partials, unsigned int *ticket,
                              double *norm_out, int *flag, const int *gate) {
  if (gated_off(gate)) return;
  double acc = 0;
  bool bad = false;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
       c += (long long)gridDim.x * blockDim.x) {
    const double2 e = eps[c], em1 = make_double2(e.x - 1.0, e.y);
    const long long b = cell_box[c];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double2 z = x[3 * c + i];
      if (diag) z = cdiv(z, diag[3 * c + i]);
      const double2 f = to_d(box[i * nbox + b]);
      const double2 v = csub(cmul(e, z), cmul(em1, f));
      y[3 * c + i] = v;
      acc += v.x * v.x + v.y * v.y;
      bad |= !finite2(v);
    }
  }
  if (!norm_out) return;
  if (bad && flag) *flag = 1;
  double2 s = block_sum(make_double2(acc, 0));
  if (threadIdx.x == 0) partials[blockIdx.x] = s.x;
  if (last_block_done(ticket)) {
    double t = 0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) t += partials[i];
    double2 tot = block_sum(make_double2(t, 0));
    if (threadIdx.x == 0) { *norm_out = tot.x; *ticket = 0; }
  }
}

__global__ void precondition_kernel(const double2 *__restrict__ x, const double2 *__restrict__ diag,
                                    double2 *__restrict__ y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = cdiv(x[i], diag[i]);
}

__global__ void eps_kernel(const double2 *__restrict__ eps, double2 s0, double2 s1, double2 s2,
                           double2 *__restrict__ diag, long long cells) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
       c += (long long)gridDim.x * blockDim.x) {
    const double2 e = eps[c], em1 = make_double2(e.x - 1.0, e.y);
    diag[3 * c + 0] = csub(e, cmul(em1, s0));
    diag[3 * c + 1] = csub(e, cmul(em1, s1));
    diag[3 * c + 2] = csub(e, cmul(em1, s2));
  }
}

// ------------------------------------------------------ far-pair quadrature
// Gauss-Legendre nodes/weights on [0,1] for orders 4, 6, 8, 12 (host-computed).
__constant__ double c_gauss_node[4][12];
__constant__ double c_gauss_weight[4][12];

// One order of the difference-coordinate rule (vie_fft.c:299-318) for offset v;
// returns the six independent entries (xx yy zz xy xz yz), block-reduced.
__device__ void far_rule_block(const int v[3], double h, double k, int s, int order,
                               double2 out[6]) {
  double2 acc[6];
#pragma unroll
  for (int e = 0; e < 6; ++e) acc[e] = make_double2(0, 0);
  const int total = order * order * order * 8;
  const double inv4pi = 1.0 / (4.0 * 3.141592653589793238462643383279502884);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int mask = idx & 7, q = idx >> 3;
    const int ia = q / (order * order), ib = (q / order) % order, ic = q % order;
    const double t[3] = {c_gauss_node[s][ia], c_gauss_node[s][ib], c_gauss_node[s][ic]};
    const double wt = h * h * h * c_gauss_weight[s][ia] * c_gauss_weight[s][ib] *
                      c_gauss_weight[s][ic] * (1 - t[0]) * (1 - t[1]) * (1 - t[2]);
    double r[3], r2 = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      r[i] = h * ((double)v[i] + ((mask & (1 << i)) ? -t[i] : t[i]));
      r2 += r[i] * r[i];
    }
    const double rr = sqrt(r2);
    double sn, cs;
    sincos(k * rr, &sn, &cs);
    const double gm = wt * inv4pi / rr;
    const double2 g = make_double2(gm * cs, -gm * sn);   // wt e^{-ikr} / (4 pi r)
    const double2 dterm = make_double2(k * k - 1.0 / r2, -k / rr);
    const double2 rterm = make_double2((-k * k + 3.0 / r2) / r2, (3.0 * k / rr) / r2);
    const double2 diag = cmul(g, dterm), radial = cmul(g, rterm);
    acc[0] = cadd(acc[0], cadd(diag, cscale(radial, r[0] * r[0])));
    acc[1] = cadd(acc[1], cadd(diag, cscale(radial, r[1] * r[1])));
    acc[2] = cadd(acc[2], cadd(diag, cscale(radial, r[2] * r[2])));
    acc[3] = cadd(acc[3], cscale(radial, r[0] * r[1]));
    acc[4] = cadd(acc[4], cscale(radial, r[0] * r[2]));
    acc[5] = cadd(acc[5], cscale(radial, r[1] * r[2]));
  }
#pragma unroll
  for (int e = 0; e < 6; ++e) out[e] = block_sum(acc[e]);
}

static __device__ double cabs_d(double2 a) { return hypot(a.x, a.y); }

// Order ladder 4,6,8,12 with 2e-12 abs + 2e-9 rel acceptance, gap^2 > 4 only
// (vie_fft.c:319-335).  One block per offset.
__global__ void __launch_bounds__(256) far_kernel(const int *__restrict__ offsets, long long count,
                                                  double h, double k, double2 *__restrict__ table,
                                                  int *__restrict__ ok) {
  const long long o = blockIdx.x;
  if (o >= count) return;
  const int v[3] = {offsets[3 * o], offsets[3 * o + 1], offsets[3 * o + 2]};
  double gap2 = 0;
  for (int i = 0; i < 3; ++i) { double g = v[i] > 1 ? (double)v[i] - 1 : 0; gap2 += g * g; }
  if (gap2 <= 4) { if (threadIdx.x == 0) ok[o] = 0; return; }
  const int ladder[4] = {4, 6, 8, 12};
  double2 prev[6], cur[6];
  far_rule_block(v, h, k, 0, ladder[0], prev);
  for (int s = 1; s < 4; ++s) {
    far_rule_block(v, h, k, s, ladder[s], cur);
    bool conv = true;
    for (int e = 0; e < 6; ++e) {
      const double2 d = csub(cur[e], prev[e]);
      if (!finite2(cur[e]) || cabs_d(d) > 2e-12 + 2e-9 * cabs_d(cur[e])) conv = false;
    }
    if (conv) {
      if (threadIdx.x == 0) {
        // Off-diagonal entries vanish where an offset component is zero
        // (vie_fft.c:356-359); symmetric averaging leaves far entries as is.
        cur[3] = (v[0] && v[1]) ? cur[3] : make_double2(0, 0);
        cur[4] = (v[0] && v[2]) ? cur[4] : make_double2(0, 0);
        cur[5] = (v[1] && v[2]) ? cur[5] : make_double2(0, 0);
        for (int e = 0; e < 6; ++e) table[6 * o + e] = cur[e];
        ok[o] = 1;
      }
      return;
    }
    for (int e = 0; e < 6; ++e) prev[e] = cur[e];
  }
  if (threadIdx.x == 0) ok[o] = 0;
}

// ------------------------------------------------------------ spectrum fill
struct FillArgs {
  long long P[3], S[3];         // padded grid, lattice shape
  long long Ss[3];              // shape sorted descending
  const long long *slab_start;  // per a: first table index of slab a
  const long long *row_start;   // per b: first index of row b within a slab
  const double2 *table;         // 6 entries per sorted offset
  double2 *spec;                // 6 x G
  long long G;
};

__device__ __forceinline__ int sym_slot(int i, int j) {
  const int lo = i < j ? i : j, hi = i < j ? j : i;
  if (lo == hi) return lo;
  if (lo == 0) return hi == 1 ? 3 : 4;
  return 5;
}

// Each padded-grid site takes the value the reference's permutation x sign
// loop (vie_fft.c:360-373) writes last: the last matching permutation and,
// for zero components, the negative-sign mask.
__global__ void fill_kernel(FillArgs f) {
  const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < f.G;
       g += (long long)gridDim.x * blockDim.x) {
    long long pos[3];
    pos[2] = g % f.P[2];
    pos[1] = (g / f.P[2]) % f.P[1];
    pos[0] = g / (f.P[2] * f.P[1]);
    long long d[3];
    int sg[3];
    bool inside = true;
    for (int i = 0; i < 3; ++i) {
      if (pos[i] < f.S[i]) { d[i] = pos[i]; sg[i] = pos[i] == 0 ? -1 : 1; }
      else if (pos[i] > f.P[i] - f.S[i]) { d[i] = f.P[i] - pos[i]; sg[i] = -1; }
      else inside = false;
    }
    double2 val[6];
    for (int e = 0; e < 6; ++e) val[e] = make_double2(0, 0);
    if (inside) {
      long long v[3] = {d[0], d[1], d[2]};
      // sort descending
      if (v[0] < v[1]) { long long t = v[0]; v[0] = v[1]; v[1] = t; }
      if (v[1] < v[2]) { long long t = v[1]; v[1] = v[2]; v[2] = t; }
      if (v[0] < v[1]) { long long t = v[0]; v[0] = v[1]; v[1] = t; }
      int q = 0;
      for (int p = 5; p >= 0; --p)
        if (v[perms[p][0]] == d[0] && v[perms[p][1]] == d[1] && v[perms[p][2]] == d[2]) { q = p; break; }
      const long long idx = f.slab_start[v[0]] + f.row_start[v[1]] + v[2];
      const double2 *n = f.table + 6 * idx;
      for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) {
          const double2 src = n[sym_slot(perms[q][i], perms[q][j])];
          const double s = (double)(sg[i] * sg[j]);
          val[sym_slot(i, j)] = make_double2(s * src.x, s * src.y);
        }
    }
    for (int e = 0; e < 6; ++e) f.spec[e * f.G + g] = val[e];
  }
}

// Octant of the full transformed spectrum, scaled: out[s][kx][ky][kz] for
// k <= P/2 per axis.
__global__ void compress_kernel(const double2 *__restrict__ full, double2 *__restrict__ oct,
                                long long Px, long long Py, long long Pz, long long Hx,
                                long long Hy, long long Hz, double scale) {
  const long long GH = Hx * Hy * Hz, G = Px * Py * Pz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 6 * GH;
       i += (long long)gridDim.x * blockDim.x) {
    const long long s = i / GH, r = i - s * GH;
    const long long kz = r % Hz, ky = (r / Hz) % Hy, kx = r / (Hz * Hy);
    const double2 v = full[s * G + (kx * Py + ky) * Pz + kz];
    oct[i] = make_double2(v.x * scale, v.y * scale);
  }
}

// Full 6 x G spectrum from the octant (validation read-back).
__global__ void expand_kernel(const double2 *__restrict__ oct, double2 *__restrict__ full,
                              long long Px, long long Py, long long Pz, long long Hy, long long Hz,
                              long long GH) {
  const long long G = Px * Py * Pz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 6 * G;
       i += (long long)gridDim.x * blockDim.x) {
    const long long s = i / G, r = i - s * G;
    const int kz = (int)(r % Pz), ky = (int)((r / Pz) % Py), kx = (int)(r / (Pz * Py));
    const Fold fx = fold(kx, (int)Px), fy = fold(ky, (int)Py), fz = fold(kz, (int)Pz);
    double sg = 1;
    if (s == 3) sg = fx.sgn * fy.sgn;
    if (s == 4) sg = fx.sgn * fz.sgn;
    if (s == 5) sg = fy.sgn * fz.sgn;
    const double2 v = oct[s * GH + ((long long)fx.idx * Hy + fy.idx) * Hz + fz.idx];
    full[i] = make_double2(sg * v.x, sg * v.y);
  }
}

template <typename C>
__global__ void scale_convert_kernel(const double2 *__restrict__ in, C *__restrict__ out, long long n,
                                     double s) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 v = in[i];
    out[i] = from_d<C>(make_double2(v.x * s, v.y * s));
  }
}

// ------------------------------------------------------------------- plan
static unsigned grid_for(long long n, int threads = 256) {
  long long b = (n + threads - 1) / threads;
  long long cap = (long long)n2c_sm_count() * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

void n2c_gmres_work_free(void *w);
void **n2c_vie_gm_slot(n2d_vie *p) { return &p->gm_work; }

static void free_plan(n2d_vie *p) {
  if (!p) return;
  n2c_gmres_work_free(p->gm_work);
  void *bufs[] = {p->cell_box, p->box_cell, p->eps, p->diag, p->spec64,
                  p->fp32 ? p->spec : nullptr, p->box, p->t1, p->t2,
                  p->tw64[0], p->tw64[1], p->tw64[2], p->tw32[0], p->tw32[1], p->tw32[2],
                  p->table, p->table_ok, p->offsets, p->slab_start, p->row_start, p->partials,
                  p->ticket};
  for (void *b : bufs) n2d_free(b);
  delete p;
}

extern "C" void n2d_vie_destroy(n2d_vie *p) { free_plan(p); }
extern "C" size_t n2d_vie_device_bytes(const n2d_vie *p) { return p ? p->device_bytes : 0; }
extern "C" int n2d_vie_fp32(const n2d_vie *p) { return p ? p->fp32 : 0; }
extern "C" long long n2d_vie_cells(const n2d_vie *p) { return p ? p->cells : 0; }
extern "C" const double *n2d_vie_diag(const n2d_vie *p) { return (const double *)p->diag; }

static void *track(n2d_vie *p, size_t bytes) {
  void *q = n2d_alloc(bytes);
  if (q) p->device_bytes += bytes;
  return q;
}

extern "C" int n2d_vie_create(n2d_vie **out, const long long shape[3], const long long padded[3],
                              long long cells, const int *cell_box, const double *const twiddles[3],
                              int fp32) {
  *out = nullptr;
  n2d_vie *p = new n2d_vie();
  memset(p, 0, sizeof(*p));
  p->fp32 = fp32;
  p->G = 1;
  p->nbox = 1;
  for (int d = 0; d < 3; ++d) {
    p->S[d] = shape[d];
    p->P[d] = padded[d];
    p->G *= padded[d];
    p->nbox *= shape[d];
    if (padded[d] > 1024 || (padded[d] & (padded[d] - 1))) {
      n2c_set_error("padded axis %lld unsupported (power of two <= 1024 required)", padded[d]);
      delete p;
      return 0;
    }
  }
  p->cells = cells;
  const size_t ce = fp32 ? sizeof(float2) : sizeof(double2);
  p->cell_box = (int *)track(p, cells * sizeof(int));
  p->box_cell = (int *)track(p, p->nbox * sizeof(int));
  p->eps = (double2 *)track(p, cells * sizeof(double2));
  p->diag = (double2 *)track(p, 3 * cells * sizeof(double2));
  for (int d = 0; d < 3; ++d) p->H[d] = padded[d] / 2 + 1;
  p->GH = p->H[0] * p->H[1] * p->H[2];
  p->spec64 = (double2 *)track(p, 6 * p->GH * sizeof(double2));
  p->spec = fp32 ? track(p, 6 * p->GH * ce) : (void *)p->spec64;
  const size_t we = sizeof(double2);
  p->box = track(p, 3 * p->nbox * we);
  p->t1 = track(p, 3 * p->S[0] * p->S[1] * p->P[2] * we);
  p->t2 = track(p, 3 * p->S[0] * p->P[1] * p->P[2] * we);
  p->partials = (double *)track(p, 65536 * sizeof(double));
  p->ticket = (unsigned int *)track(p, 64);
  for (int d = 0; d < 3; ++d) {
    p->tw64[d] = (double2 *)track(p, padded[d] * sizeof(double2));
    p->tw32[d] = (float2 *)track(p, padded[d] * sizeof(float2));
  }
  if (!p->cell_box || !p->box_cell || !p->eps || !p->diag || !p->spec || !p->spec64 || !p->box || !p->t1 ||
      !p->t2 || !p->partials || !p->ticket || !p->tw64[0] || !p->tw64[1] || !p->tw64[2] ||
      !p->tw32[0] || !p->tw32[1] || !p->tw32[2]) {
    free_plan(p);
    return 0;
  }
  std::vector<int> inv(p->nbox, -1);
  for (long long c = 0; c < cells; ++c) inv[cell_box[c]] = (int)c;
  // A lattice filled in box order (every box a cell, cell c in box c) lets
  // the z passes index cells directly.
  p->box_identity = cells == p->nbox;
  for (long long c = 0; p->box_identity && c < cells; ++c) p->box_identity = cell_box[c] == c;
  for (int d = 0; d < 3; ++d) {
    std::vector<float2> t32(padded[d]);
    for (long long j = 0; j < padded[d]; ++j)
      t32[j] = make_float2((float)twiddles[d][2 * j], (float)twiddles[d][2 * j + 1]);
    if (!n2d_upload(p->tw64[d], twiddles[d], padded[d] * sizeof(double2)) ||
        !n2d_upload(p->tw32[d], t32.data(), padded[d] * sizeof(float2))) { free_plan(p); return 0; }
    if (!n2d_sync()) { free_plan(p); return 0; }
  }
  if (!n2d_upload(p->cell_box, cell_box, cells * sizeof(int)) ||
      !n2d_upload(p->box_cell, inv.data(), p->nbox * sizeof(int)) ||
      !n2d_memset(p->ticket, 0, 64) || !n2d_sync()) {
    free_plan(p);
    return 0;
  }
  p->planes[0] = p->planes[1] = 1;
  *out = p;
  return 1;
}

extern "C" int n2d_vie_set_gauss(const double *nodes, const double *weights) {
  N2C_CHECK(cudaMemcpyToSymbol(c_gauss_node, nodes, sizeof(double) * 48));
  N2C_CHECK(cudaMemcpyToSymbol(c_gauss_weight, weights, sizeof(double) * 48));
  return 1;
}

extern "C" int n2d_vie_far_tensors(n2d_vie *p, long long count, const int *offsets,
                                   const long long sorted_shape[3], double pitch, double k0,
                                   int *far_ok) {
  // Index tables: slab a starts at slab_start[a]; within a slab, row b starts
  // at row_start[b] = sum_{b'<b} (min(b', S2-1) + 1).
  const long long S0 = sorted_shape[0], S1 = sorted_shape[1], S2 = sorted_shape[2];
  std::vector<long long> row(S1 + 1), slab(S0 + 1);
  row[0] = 0;
  for (long long b = 0; b < S1; ++b) row[b + 1] = row[b] + (b < S2 - 1 ? b : S2 - 1) + 1;
  slab[0] = 0;
  for (long long a = 0; a < S0; ++a) slab[a + 1] = slab[a] + row[(a < S1 - 1 ? a : S1 - 1) + 1];
  if (slab[S0] != count) {
    n2c_set_error("offset enumeration mismatch (%lld vs %lld)", slab[S0], count);
    return 0;
  }
  p->count = count;
  p->table = (double2 *)track(p, 6 * count * sizeof(double2));
  p->table_ok = (int *)track(p, count * sizeof(int));
  p->offsets = (int *)track(p, 3 * count * sizeof(int));
  p->slab_start = (long long *)track(p, (S0 + 1) * sizeof(long long));
  p->row_start = (long long *)track(p, (S1 + 1) * sizeof(long long));
  if (!p->table || !p->table_ok || !p->offsets || !p->slab_start || !p->row_start) return 0;
  if (!n2d_upload(p->offsets, offsets, 3 * count * sizeof(int)) ||
      !n2d_upload(p->slab_start, slab.data(), (S0 + 1) * sizeof(long long)) ||
      !n2d_upload(p->row_start, row.data(), (S1 + 1) * sizeof(long long)))
    return 0;
  for (int d = 0; d < 3; ++d) p->Ss[d] = sorted_shape[d];
  for (long long first = 0; first < count; first += 65535) {
    const long long n = count - first < 65535 ? count - first : 65535;
    far_kernel<<<(unsigned)n, 256, 0, n2c_stream()>>>(p->offsets + 3 * first, n, pitch, k0,
                                                        p->table + 6 * first, p->table_ok + first);
    if (!n2c_check_launch("far_kernel")) return 0;
  }
  return n2d_download(far_ok, p->table_ok, count * sizeof(int));
}

extern "C" int n2d_vie_put_tensors(n2d_vie *p, long long count, const long long *index,
                                   const double *tensors) {
  for (long long i = 0; i < count; ++i)
    if (!n2d_upload(p->table + 6 * index[i], tensors + 12 * i, 6 * sizeof(double2))) return 0;
  return n2d_sync();
}

template <typename C>
static int transform_spectrum(n2d_vie *p, C *spec, const C *const tw[3]) {
  const long long Px = p->P[0], Py = p->P[1], Pz = p->P[2];
  return axis_pass<C>(0, (int)Pz, spec, spec, tw[2], 6 * Px * Py, 1, Pz, Pz, (int)Pz, (int)Pz) &&
         axis_pass<C>(0, (int)Py, spec, spec, tw[1], 6 * Px, Pz, Py, Py, (int)Py, (int)Py) &&
         axis_pass<C>(0, (int)Px, spec, spec, tw[0], 6, Py * Pz, Px, Px, (int)Px, (int)Px);
}

extern "C" int n2d_vie_finish_spectrum(n2d_vie *p) {
  FillArgs f;
  for (int d = 0; d < 3; ++d) { f.P[d] = p->P[d]; f.S[d] = p->S[d]; f.Ss[d] = p->Ss[d]; }
  f.slab_start = p->slab_start; f.row_start = p->row_start; f.table = p->table; f.G = p->G;
  // The spectrum is built and transformed in FP64 on a temporary full grid,
  // then its octant is kept, scaled by 1/G, and for mixed plans also rounded
  // into the FP32 copy.
  double2 *work = (double2 *)n2d_alloc(6 * p->G * sizeof(double2));
  if (!work) return 0;
  f.spec = work;
  fill_kernel<<<grid_for(p->G), 256, 0, n2c_stream()>>>(f);
  int ok = n2c_check_launch("fill_kernel");
  const double2 *tw[3] = {p->tw64[0], p->tw64[1], p->tw64[2]};
  ok = ok && transform_spectrum<double2>(p, work, tw);
  if (ok) {
    compress_kernel<<<grid_for(6 * p->GH), 256, 0, n2c_stream()>>>(
        work, p->spec64, p->P[0], p->P[1], p->P[2], p->H[0], p->H[1], p->H[2], 1.0 / (double)p->G);
    ok = n2c_check_launch("compress");
  }
  if (ok && p->fp32) {
    scale_convert_kernel<float2><<<grid_for(6 * p->GH), 256, 0, n2c_stream()>>>(
        p->spec64, (float2 *)p->spec, 6 * p->GH, 1.0);
    ok = n2c_check_launch("scale_convert");
  }
  ok = ok && n2d_sync();
  n2d_free(work);
  // The offset table is only needed while building.
  n2d_free(p->table); n2d_free(p->table_ok); n2d_free(p->offsets);
  n2d_free(p->slab_start); n2d_free(p->row_start);
  p->device_bytes -= 6 * p->count * sizeof(double2) + p->count * sizeof(int) * 4 +
                     (p->Ss[0] + 1 + p->Ss[1] + 1) * sizeof(long long);
  p->table = nullptr; p->table_ok = nullptr; p->offsets = nullptr;
  p->slab_start = nullptr; p->row_start = nullptr;
  if (ok && n2d_vie_autotune_enabled()) ok = n2d_vie_tune(p, 1);
  return ok;
}

extern "C" int n2d_vie_read_spectrum(n2d_vie *p, double *out) {
  double2 *full = (double2 *)n2d_alloc(6 * p->G * sizeof(double2));
  if (!full) return 0;
  expand_kernel<<<grid_for(6 * p->G), 256, 0, n2c_stream()>>>(p->spec64, full, p->P[0], p->P[1],
                                                              p->P[2], p->H[1], p->H[2], p->GH);
  int ok = n2c_check_launch("expand") && n2d_download(out, full, 6 * p->G * sizeof(double2));
  n2d_free(full);
  return ok;
}

extern "C" int n2d_vie_set_eps(n2d_vie *p, const double *eps, const double *self) {
  if (!n2d_upload(p->eps, eps, p->cells * sizeof(double2))) return 0;
  for (int i = 0; i < 3; ++i) p->self[i] = make_double2(self[2 * i], self[2 * i + 1]);
  eps_kernel<<<grid_for(p->cells), 256, 0, n2c_stream()>>>(p->eps, p->self[0], p->self[1], p->self[2],
                                                           p->diag, p->cells);
  return n2c_check_launch("eps_kernel") && n2d_sync();
}

// z passes with the cell vector as input / output: the forward z pass
// scatters (and preconditions) the cells, the inverse z pass applies
// y = eps z - (eps-1) field and reduces |y|^2.
template <typename C>
static int z_cell_plan(int mode, n2d_vie *p, const C *in, C *out, const C *tw, const double2 *x, double2 *y,
                       int precondition, double *norm, int *flag, n2d_pass_choice ch, PassPlan<C> *pp) {
  const long long nx = p->S[0], ny = p->S[1], nz = p->S[2], Pz = p->P[2];
  PassArgs<C> &a = pp->a;
  memset(&a, 0, sizeof(a));
  a.in = in; a.out = out; a.tw = tw;
  a.lines = 3 * nx * ny; a.I = 1;
  if (mode == 3) { a.A_in = nz; a.A_out = Pz; a.n_in = (int)nz; a.n_out = (int)Pz; }
  else { a.A_in = Pz; a.A_out = nz; a.n_in = (int)Pz; a.n_out = (int)nz; }
  a.NL = ch.nl ? ch.nl : zline_tile<C>(mode == 3 ? 7 : 8, (int)Pz, 3, nx * ny);
  a.nl_div = div_magic(a.NL);
  a.np_div = div_magic(a.NL / 3);
  a.nout_div = div_magic(a.n_out);
  a.gate = n2c_gate();
  a.cx = x; a.cy = y; a.eps = p->eps; a.box_cell = p->box_cell;
  a.box_identity = p->box_identity && !p->mirror;
  a.self0 = p->self[0]; a.self1 = p->self[1]; a.self2 = p->self[2];
  a.nxy = nx * ny; a.mirror = p->mirror; a.precondition = precondition;
  a.flag = flag; a.partials = p->partials; a.ticket = p->ticket; a.norm = norm;
  const int NP = a.NL / 3;
  pp->tiles = (a.nxy + NP - 1) / NP;
  if (norm && pp->tiles > 65536) { n2c_set_error("norm reduction grid too large"); return 0; }
  // Cell tiles take T1 rows of 3 components: T1 is [3][nx*ny][Pz], so the
  // component planes are addressed through lines = comp * nxy + pos.
  pp->mode = mode == 3 ? 7 : 8; pp->L = (int)Pz; pp->variant = ch.radix;
  pp->smem = (size_t)2 * (a.NL + 1) * Pz * sizeof(C);
  return 1;
}

template <typename C> static constexpr int prec_of() { return sizeof(C) == sizeof(float2) ? 0 : 1; }

// Launch description of pass `pass` of the matvec y = A x (numbering of
// n2d_pass_choice) with the tile height and radix split of ch.
template <typename C>
static int pass_plan(n2d_vie *p, int pass, n2d_pass_choice ch, const double2 *x, double2 *y, int precondition,
                     double *norm, int *flag, PassPlan<C> *pp) {
  const long long nx = p->S[0], ny = p->S[1];
  const long long Py = p->P[1], Pz = p->P[2];
  constexpr bool single = sizeof(C) == sizeof(float2);
  C *t1 = (C *)p->t1, *t2 = (C *)p->t2;
  const C *tw[3];
  for (int d = 0; d < 3; ++d) tw[d] = single ? (const C *)p->tw32[d] : (const C *)p->tw64[d];
  const C *spec = single ? (const C *)p->spec : (const C *)p->spec64;
  switch (pass) {
    case 0: return z_cell_plan<C>(3, p, nullptr, t1, tw[2], x, y, precondition, nullptr, flag, ch, pp);
    case 1: strided_plan<C>(0, (int)Py, t1, t2, tw[1], 3 * nx, Pz, ny, Py, (int)ny, (int)Py, ch, pp); return 1;
    case 2: product_plan<C>(p, t2, t2, tw[0], spec, ch, pp); return 1;
    case 3: strided_plan<C>(1, (int)Py, t2, t1, tw[1], 3 * nx, Pz, Py, ny, (int)Py, (int)ny, ch, pp); return 1;
    case 4: return z_cell_plan<C>(4, p, t1, nullptr, tw[2], x, y, precondition, norm, flag, ch, pp);
  }
  n2c_set_error("no FFT pass %d", pass);
  return 0;
}

template <typename C>
static int run_pass(n2d_vie *p, int pass, n2d_pass_choice ch, const double2 *x, double2 *y, int precondition,
                    double *norm, int *flag) {
  PassPlan<C> pp;
  if (!pass_plan<C>(p, pass, ch, x, y, precondition, norm, flag, &pp)) return 0;
  return fft_launch_pass<C>(pp.mode, pp.L, pp.variant, pp.a, pp.smem, pp.tiles);
}

// The fused yz-plane passes apply when the padded y and z axes have the same
// length P = 2Q with Q one the plane kernels are built for, and the inverse
// pass's norm reduction (one partial per CTA, 12 nx CTAs) fits the plan's
// partials.
static bool plane_ok(const n2d_vie *p) {
  return p->P[1] == p->P[2] && plane_supported((int)(p->P[1] / 2)) && p->S[1] <= p->P[1] / 2 &&
         p->S[2] <= p->P[2] / 2 && 12 * p->S[0] <= 65536;
}

template <typename C>
static int apply_planes(n2d_vie *p, const double2 *x, double2 *y, int precondition, double *norm, int *flag) {
  constexpr bool single = sizeof(C) == sizeof(float2);
  PlaneArgs<C> a;
  memset(&a, 0, sizeof(a));
  a.grid = (C *)p->t2;
  a.twy = single ? (const C *)p->tw32[1] : (const C *)p->tw64[1];
  a.twz = single ? (const C *)p->tw32[2] : (const C *)p->tw64[2];
  a.nx = (int)p->S[0]; a.ny = (int)p->S[1]; a.nz = (int)p->S[2];
  a.gate = n2c_gate();
  a.cx = x; a.cy = y; a.eps = p->eps; a.box_cell = p->box_cell;
  a.self0 = p->self[0]; a.self1 = p->self[1]; a.self2 = p->self[2];
  a.mirror = p->mirror; a.precondition = precondition; a.flag = flag;
  a.partials = p->partials; a.ticket = p->ticket; a.norm = norm;
  const int Q = (int)(p->P[1] / 2);
  return fft_plane_launch<C>(false, Q, a, n2c_stream()) &&
         run_pass<C>(p, 2, p->sched[prec_of<C>()][2], x, y, precondition, norm, flag) &&
         fft_plane_launch<C>(true, Q, a, n2c_stream());
}

template <typename C>
static int apply_five(n2d_vie *p, const double2 *x, double2 *y, int precondition, double *norm, int *flag) {
  const n2d_pass_choice *s = p->sched[prec_of<C>()];
  for (int i = 0; i < N2D_VIE_PASSES; ++i)
    if (!run_pass<C>(p, i, s[i], x, y, precondition, norm, flag)) return 0;
  return 1;
}

template <typename C>
static int apply_t(n2d_vie *p, const double2 *x, double2 *y, int precondition, double *norm,
                   int *flag) {
  if (p->planes[prec_of<C>()] && plane_ok(p)) return apply_planes<C>(p, x, y, precondition, norm, flag);
  return apply_five<C>(p, x, y, precondition, norm, flag);
}

extern "C" int n2d_vie_apply(n2d_vie *p, const double *x, double *y, int precondition_input,
                             double *norm, int *flag, int full_precision) {
  if (p->fp32 && !full_precision)
    return apply_t<float2>(p, (const double2 *)x, (double2 *)y, precondition_input, norm, flag);
  return apply_t<double2>(p, (const double2 *)x, (double2 *)y, precondition_input, norm, flag);
}

// ------------------------------------------------------------------- tuner
// The tile height and radix split of each matvec pass are chosen by timing
// candidates on the plan's own grids (CUDA events on the plan's stream; per
// candidate one warm-up launch, then the best of two runs of three launches):
// first the radix split at the heuristic height, then the height at the split
// kept.  A candidate replaces the incumbent only when it is at least 3%
// faster, so timing noise does not move a pass off the heuristic for nothing.
// Choices are cached per (lattice, padded grid, precision) for the process,
// so the plans of a frequency sweep or of many same-sized models are timed
// once.  Every candidate computes the same transform; the split only changes
// the order of the butterflies, hence the rounding.
namespace {

struct TuneEntry {
  long long S[3], P[3];
  int prec;
  n2d_pass_choice c[N2D_VIE_PASSES];
  int planes;
};
std::mutex g_tune_lock;
std::vector<TuneEntry> g_tune_cache;
std::atomic<int> g_autotune{-1};   // -1: NEC2C_CUDA_FFT_AUTOTUNE not read yet

bool tune_key_is(const TuneEntry &e, const n2d_vie *p, int prec) {
  for (int d = 0; d < 3; ++d)
    if (e.S[d] != p->S[d] || e.P[d] != p->P[d]) return false;
  return e.prec == prec;
}

int autotune_enabled() {
  int v = g_autotune.load();
  if (v < 0) {
    const char *env = getenv("NEC2C_CUDA_FFT_AUTOTUNE");
    v = (env && env[0] == '0') ? 0 : 1;
    int expected = -1;
    g_autotune.compare_exchange_strong(expected, v);
    v = g_autotune.load();
  }
  return v;
}

int pass_length(const n2d_vie *p, int pass) {
  return (int)(pass == 0 || pass == 4 ? p->P[2] : pass == 2 ? p->P[0] : p->P[1]);
}

// The height the heuristic gives pass `pass`.
template <typename C>
int heuristic_height(const n2d_vie *p, int pass) {
  switch (pass) {
    case 0: return zline_tile<C>(7, (int)p->P[2], 3, p->S[0] * p->S[1]);
    case 4: return zline_tile<C>(8, (int)p->P[2], 3, p->S[0] * p->S[1]);
    case 2: return lines_per_tile((int)p->P[0], 3, sizeof(C));
  }
  return lines_per_tile((int)p->P[1], 1, sizeof(C));
}

// Heights tried: whole lattice columns (multiples of 3 lines) for the z
// passes, powers of two for the strided passes, each within 100 KB of shared
// memory (two CTAs per SM at least); the z epilogue also keeps its norm
// reduction within the 65,536 partials of the plan.
template <typename C>
std::vector<int> candidate_heights(const n2d_vie *p, int pass) {
  std::vector<int> out;
  const size_t e = sizeof(C), L = (size_t)pass_length(p, pass);
  if (pass == 0 || pass == 4) {
    const long long cols = p->S[0] * p->S[1];
    for (int nl = 3; nl <= 96 && (size_t)2 * (nl + 1) * L * e <= 100 * 1024; nl += 3)
      if (pass == 0 || (cols + nl / 3 - 1) / (nl / 3) <= 65536) out.push_back(nl);
  } else {
    const size_t ncomp = pass == 2 ? 3 : 1;
    for (int nl = 1; nl <= 64; nl *= 2)
      if (L * ncomp * nl * e <= 100 * 1024) out.push_back(nl);
  }
  return out;
}

// Milliseconds of three launches of one candidate (best of two runs), or a
// negative value when the candidate cannot run.
template <typename C>
float time_candidate(n2d_vie *p, int pass, n2d_pass_choice ch, const double2 *x, double2 *y, double *norm,
                     cudaEvent_t e0, cudaEvent_t e1) {
  if (!run_pass<C>(p, pass, ch, x, y, 0, norm, nullptr)) return -1.0f;
  float best = -1.0f;
  for (int trial = 0; trial < 2; ++trial) {
    if (cudaEventRecord(e0, n2c_stream()) != cudaSuccess) return -1.0f;
    for (int r = 0; r < 3; ++r)
      if (!run_pass<C>(p, pass, ch, x, y, 0, norm, nullptr)) return -1.0f;
    float ms = 0;
    if (cudaEventRecord(e1, n2c_stream()) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      return -1.0f;
    if (best < 0 || ms < best) best = ms;
  }
  return best;
}

// Milliseconds of three whole products with the plan's current schedule
// (best of three runs), or a negative value when a product fails.
template <typename C>
float time_product(n2d_vie *p, const double2 *x, double2 *y, double *norm, cudaEvent_t e0, cudaEvent_t e1) {
  if (!apply_t<C>(p, x, y, 0, norm, nullptr)) return -1.0f;
  float best = -1.0f;
  for (int trial = 0; trial < 3; ++trial) {
    if (cudaEventRecord(e0, n2c_stream()) != cudaSuccess) return -1.0f;
    for (int r = 0; r < 3; ++r)
      if (!apply_t<C>(p, x, y, 0, norm, nullptr)) return -1.0f;
    float ms = 0;
    if (cudaEventRecord(e1, n2c_stream()) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      return -1.0f;
    if (best < 0 || ms < best) best = ms;
  }
  return best;
}

template <typename C>
int tune_precision(n2d_vie *p, const double2 *x, double2 *y, double *norm, bool use_cache) {
  const int prec = prec_of<C>();
  if (use_cache) {
    std::lock_guard<std::mutex> hold(g_tune_lock);
    for (const TuneEntry &e : g_tune_cache)
      if (tune_key_is(e, p, prec)) {
        memcpy(p->sched[prec], e.c, sizeof(e.c));
        p->planes[prec] = e.planes;
        p->tuned[prec] = 1;
        return 1;
      }
  }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) { n2c_set_error("tuner: event creation failed"); return 0; }
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    n2c_set_error("tuner: event creation failed");
    return 0;
  }
  n2d_pass_choice chosen[N2D_VIE_PASSES];
  for (int pass = 0; pass < N2D_VIE_PASSES; ++pass) {
    // A heuristic that cannot run here (a z epilogue whose norm reduction
    // would need more than 65,536 partials) stays the fallback; any
    // candidate that runs replaces it.
    n2d_pass_choice best = {heuristic_height<C>(p, pass), 0};
    float bt = time_candidate<C>(p, pass, best, x, y, norm, e0, e1);
    if (bt < 0) {
      best = n2d_pass_choice{0, 0};
      bt = 3.0e38f;
    }
    const int L = pass_length(p, pass);
    for (int v = 1; v < fft_radix_variants(L); ++v) {
      const n2d_pass_choice c = {best.nl, v};
      const float t = time_candidate<C>(p, pass, c, x, y, norm, e0, e1);
      if (t >= 0 && t < 0.97f * bt) { best = c; bt = t; }
    }
    for (int nl : candidate_heights<C>(p, pass)) {
      if (nl == best.nl) continue;
      const n2d_pass_choice c = {nl, best.radix};
      const float t = time_candidate<C>(p, pass, c, x, y, norm, e0, e1);
      if (t >= 0 && t < 0.97f * bt) { best = c; bt = t; }
    }
    chosen[pass] = best;
  }
  memcpy(p->sched[prec], chosen, sizeof(chosen));
  // Whole-product refinement: a pass timed alone (its input warm in L2, no
  // neighbours) can favour a height that loses inside a product, so each
  // pass's neighbouring heights are tried in whole products as well and
  // replace the choice when at least 2% faster.
  {
    p->planes[prec] = 0;   // the five passes (the plane forms are weighed below)
    float tb = time_product<C>(p, x, y, norm, e0, e1);
    for (int pass = 0; tb >= 0 && pass < N2D_VIE_PASSES; ++pass) {
      const std::vector<int> hs = candidate_heights<C>(p, pass);
      int at = -1;
      for (int i = 0; i < (int)hs.size(); ++i)
        if (hs[i] == chosen[pass].nl) at = i;
      if (at < 0) continue;
      const int reach = pass == 0 || pass == 4 ? 2 : 1;
      for (int i = at - reach; i <= at + reach; ++i) {
        if (i < 0 || i >= (int)hs.size() || i == at) continue;
        const n2d_pass_choice keep = p->sched[prec][pass];
        p->sched[prec][pass] = n2d_pass_choice{hs[i], chosen[pass].radix};
        const float t = time_product<C>(p, x, y, norm, e0, e1);
        if (t >= 0 && t < 0.98f * tb) tb = t;
        else p->sched[prec][pass] = keep;
      }
      chosen[pass] = p->sched[prec][pass];
    }
  }
  // Whole products: the five tuned passes against the fused plane passes
  // around the tuned x pass; the planes are kept when at least 3% faster.
  int planes = 0;
  if (plane_ok(p)) {
    p->planes[prec] = 0;
    const float t5 = time_product<C>(p, x, y, norm, e0, e1);
    p->planes[prec] = 1;
    const float t3 = time_product<C>(p, x, y, norm, e0, e1);
    planes = t3 >= 0 && (t5 < 0 || t3 < 0.97f * t5);
  }
  p->planes[prec] = planes;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // A candidate that could not run may have left a launch error behind.
  cudaGetLastError();
  p->tuned[prec] = 1;
  std::lock_guard<std::mutex> hold(g_tune_lock);
  TuneEntry e;
  for (int d = 0; d < 3; ++d) { e.S[d] = p->S[d]; e.P[d] = p->P[d]; }
  e.prec = prec;
  e.planes = planes;
  memcpy(e.c, chosen, sizeof(chosen));
  for (TuneEntry &old : g_tune_cache)
    if (tune_key_is(old, p, prec)) { old = e; return 1; }
  if (g_tune_cache.size() < 4096) g_tune_cache.push_back(e);
  return 1;
}

}  // namespace

extern "C" void n2d_vie_autotune(int enable) { g_autotune.store(enable ? 1 : 0); }
extern "C" int n2d_vie_autotune_enabled(void) { return autotune_enabled(); }

// measure: 0 the heuristic schedule, 1 measured (a cached choice for the same
// shape is reused), 2 measured afresh (the cache entry is replaced).
extern "C" int n2d_vie_tune(n2d_vie *p, int measure) {
  // A captured GMRES cycle bakes the tile heights into its launches.
  n2c_gmres_work_free(p->gm_work);
  p->gm_work = nullptr;
  memset(p->sched, 0, sizeof(p->sched));
  p->tuned[0] = p->tuned[1] = 0;
  p->planes[0] = p->planes[1] = 1;
  if (measure == 0 || p->cells == 0) return 1;
  const size_t vec = 3 * (size_t)p->cells * sizeof(double2);
  double2 *x = (double2 *)n2d_alloc(vec), *y = (double2 *)n2d_alloc(vec);
  double *norm = (double *)n2d_alloc(sizeof(double));
  int ok = x && y && norm && n2d_memset(x, 0, vec);
  ok = ok && (!p->fp32 || tune_precision<float2>(p, x, y, norm, measure == 1));
  ok = ok && tune_precision<double2>(p, x, y, norm, measure == 1);
  ok = ok && n2d_sync();
  n2d_free(x);
  n2d_free(y);
  n2d_free(norm);
  if (!ok) {
    memset(p->sched, 0, sizeof(p->sched));
    p->tuned[0] = p->tuned[1] = 0;
    p->planes[0] = p->planes[1] = 1;
  }
  return ok;
}

// Pins the schedule of precision prec (0 FP32, 1 FP64): pass i runs tiles[i]
// lines per tile with the split whose first radix is r1[i].  Each height and
// split must be one the tuner would try; otherwise nothing changes and 0 is
// returned with the error set.
extern "C" int n2d_vie_set_schedule(n2d_vie *p, int prec, const int *tiles, const int *r1) {
  prec = prec ? 1 : 0;
  n2d_pass_choice c[N2D_VIE_PASSES];
  for (int i = 0; i < N2D_VIE_PASSES; ++i) {
    const int L = pass_length(p, i);
    int v = -1;
    for (int k = 0; k < fft_radix_variants(L); ++k)
      if (fft_radix_r1(L, k) == r1[i]) v = k;
    if (v < 0) {
      n2c_set_error("FFT pass %d: R1 = %d is not a radix split of %d on offer", i, r1[i], L);
      return 0;
    }
    const std::vector<int> ok = prec ? candidate_heights<double2>(p, i) : candidate_heights<float2>(p, i);
    bool found = false;
    for (int nl : ok) found = found || nl == tiles[i];
    if (!found) {
      n2c_set_error("FFT pass %d: %d lines per tile is not a height on offer", i, tiles[i]);
      return 0;
    }
    c[i] = n2d_pass_choice{tiles[i], v};
  }
  n2c_gmres_work_free(p->gm_work);
  p->gm_work = nullptr;
  memcpy(p->sched[prec], c, sizeof(c));
  p->tuned[prec] = 1;
  return 1;
}

// Whether precision prec runs passes 0-1 and 3-4 as the fused plane passes:
// 1 yes, 0 no (the five passes), -1 when the plane passes do not apply to the
// plan's grid.
extern "C" int n2d_vie_planes(n2d_vie *p, int prec) {
  if (!plane_ok(p)) return -1;
  return p->planes[prec ? 1 : 0] ? 1 : 0;
}

// Pins the choice above (the tuner makes it by timing both forms).  Returns 0
// with the error set when the plane passes do not apply.
extern "C" int n2d_vie_set_planes(n2d_vie *p, int prec, int planes) {
  if (planes && !plane_ok(p)) {
    n2c_set_error("the fused plane passes do not apply to this grid (padded y and z must be one length 32, 64 or 128)");
    return 0;
  }
  n2c_gmres_work_free(p->gm_work);
  p->gm_work = nullptr;
  p->planes[prec ? 1 : 0] = planes ? 1 : 0;
  return 1;
}

// Schedule of precision prec (0 FP32, 1 FP64): lines per tile and R1 of the
// radix split of each pass.  Returns 1 when timed or pinned, 0 when
// heuristic.
extern "C" int n2d_vie_schedule(n2d_vie *p, int prec, int *tiles, int *r1) {
  prec = prec ? 1 : 0;
  for (int i = 0; i < N2D_VIE_PASSES; ++i) {
    const n2d_pass_choice c = p->sched[prec][i];
    const int nl = c.nl ? c.nl : (prec ? heuristic_height<double2>(p, i) : heuristic_height<float2>(p, i));
    if (tiles) tiles[i] = nl;
    if (r1) r1[i] = fft_radix_r1(pass_length(p, i), c.radix);
  }
  return p->tuned[prec];
}

extern "C" void n2d_vie_set_mirror(n2d_vie *p, long long physical_cells) {
  if (p->mirror == physical_cells) return;
  p->mirror = physical_cells;
  // A captured GMRES cycle bakes the cell layout into its launches.
  n2c_gmres_work_free(p->gm_work);
  p->gm_work = nullptr;
}

extern "C" int n2d_vie_precondition(n2d_vie *p, const double *x, double *y) {
  const long long n = 3 * (p->mirror ? p->mirror : p->cells);
  precondition_kernel<<<grid_for(n), 256, 0, n2c_stream()>>>((const double2 *)x, p->diag,
                                                              (double2 *)y, n);
  return n2c_check_launch("precondition");
}

// Tile height of pass `pass` in a batch.  A batch fills the GPU with the
// tiles of many plans, so a tile is made as large as a single plan's tile may
// be at most: about 4096 complex elements per component in the strided y
// passes and 2048 in the x product pass (within 48 KB of shared memory), and
// the default z tile of 56 KB (whole lattice columns).  Small plans then
// give each thread several butterflies instead of leaving threads idle.
// scale -1 / +1 halves / doubles that height (within the kernels' limits:
// whole lattice columns up to 96 lines, powers of two up to 64 lines, 100 KB
// of shared memory); the batch tuner picks the scale per pass.
static int batch_height(const n2d_vie *p, int pass, size_t elem, int scale) {
  const int L = pass_length(p, pass);
  if (pass == 0 || pass == 4) {
    const int h = zlines_per_tile(L, elem, 3);
    int nl = scale < 0 ? h / 2 : scale > 0 ? 2 * h : h;
    nl = nl / 3 * 3;
    if (nl < 3) nl = 3;
    if (nl > 96) nl = 96;
    while (nl > 3 && (size_t)2 * (nl + 1) * L * elem > 100 * 1024) nl -= 3;
    return scale == 0 ? h : nl;
  }
  const size_t ncomp = pass == 2 ? 3 : 1;
  const long long target = pass == 2 ? 2048 : 4096;
  int nl = 1;
  while ((long long)nl * 2 * L <= target && (size_t)nl * 2 * L * ncomp * elem <= 48 * 1024) nl *= 2;
  if (scale < 0 && nl > 1) nl /= 2;
  if (scale > 0 && nl < 64 && (size_t)2 * nl * L * ncomp * elem <= 100 * 1024) nl *= 2;
  return nl;
}

// ------------------------------------------------------------ far field
// Radiation amplitude of the volume polarisation current in free space
// (dielectric_solver.c:90-150): for direction d,
//   integral = V prod_a sinc(k d_a h / 2) sum_cells J_cell exp(+i k d.r_cell),
//   amplitude = i k c0 mu0 / (4 pi) ((integral x d) x d),
// with r_cell = origin + h (ix, iy, iz) from the cell's lattice index.  A CTA
// takes RAD_DIRS directions and sums over all cells in a fixed order.
constexpr int RAD_DIRS = 4;

__device__ __forceinline__ double sinc_small(double x) {
  if (fabs(x) < 1.0e-5) { const double x2 = x * x; return 1.0 - x2 / 6.0 + x2 * x2 / 120.0; }
  return sin(x) / x;
}

__global__ void __launch_bounds__(256) radiation_kernel(const double2 *__restrict__ J, const int *__restrict__ cell_box,
                                                        long long cells, long long ny, long long nz, double ox,
                                                        double oy, double oz, double h, double k0,
                                                        const double *__restrict__ dirs, int count,
                                                        double2 *__restrict__ out) {
  const int d0 = blockIdx.x * RAD_DIRS;
  double dx[RAD_DIRS], dy[RAD_DIRS], dz[RAD_DIRS];
#pragma unroll
  for (int r = 0; r < RAD_DIRS; ++r) {
    const int d = d0 + r < count ? d0 + r : count - 1;
    dx[r] = dirs[3 * d]; dy[r] = dirs[3 * d + 1]; dz[r] = dirs[3 * d + 2];
  }
  double2 acc[RAD_DIRS][3];
#pragma unroll
  for (int r = 0; r < RAD_DIRS; ++r)
#pragma unroll
    for (int a = 0; a < 3; ++a) acc[r][a] = make_double2(0, 0);
  const long long nyz = ny * nz;
  for (long long c = threadIdx.x; c < cells; c += blockDim.x) {
    const long long box = cell_box[c], ix = box / nyz, rem = box - ix * nyz, iy = rem / nz, iz = rem - iy * nz;
    const double x = ox + h * (double)ix, y = oy + h * (double)iy, z = oz + h * (double)iz;
    const double2 j0 = J[3 * c], j1 = J[3 * c + 1], j2 = J[3 * c + 2];
#pragma unroll
    for (int r = 0; r < RAD_DIRS; ++r) {
      double sn, cs;
      sincos(k0 * (dx[r] * x + dy[r] * y + dz[r] * z), &sn, &cs);
      const double2 e = make_double2(cs, sn);
      acc[r][0] = cadd(acc[r][0], cmul(j0, e));
      acc[r][1] = cadd(acc[r][1], cmul(j1, e));
      acc[r][2] = cadd(acc[r][2], cmul(j2, e));
    }
  }
  __shared__ double2 red[8][RAD_DIRS * 3];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int r = 0; r < RAD_DIRS; ++r)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double2 v = acc[r][a];
      for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
      }
      if (lane == 0) red[warp][r * 3 + a] = v;
    }
  __syncthreads();
  if (threadIdx.x >= RAD_DIRS || d0 + (int)threadIdx.x >= count) return;
  const int r = threadIdx.x, d = d0 + r;
  double2 in[3];
  for (int a = 0; a < 3; ++a) {
    double2 t = make_double2(0, 0);
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = cadd(t, red[w][r * 3 + a]);
    in[a] = t;
  }
  const double dir[3] = {dx[r], dy[r], dz[r]};
  double scale = h * h * h;
  for (int a = 0; a < 3; ++a) scale *= sinc_small(0.5 * k0 * dir[a] * h);
  for (int a = 0; a < 3; ++a) in[a] = cscale(in[a], scale);
  const double2 cr0 = csub(cscale(in[1], dir[2]), cscale(in[2], dir[1]));
  const double2 cr1 = csub(cscale(in[2], dir[0]), cscale(in[0], dir[2]));
  const double2 cr2 = csub(cscale(in[0], dir[1]), cscale(in[1], dir[0]));
  double2 t[3];
  t[0] = csub(cscale(cr1, dir[2]), cscale(cr2, dir[1]));
  t[1] = csub(cscale(cr2, dir[0]), cscale(cr0, dir[2]));
  t[2] = csub(cscale(cr0, dir[1]), cscale(cr1, dir[0]));
  const double f = k0 * 299792458.0 * 1.25663706212e-6 / (4.0 * 3.141592653589793238462643383279502884);
  for (int a = 0; a < 3; ++a) out[3 * d + a] = make_double2(-f * t[a].y, f * t[a].x);   // i f t
}

// Amplitudes of count directions (dirs: 3 per direction, device) of the
// current J_dev (3 per physical cell) into out_dev (3 per direction).
extern "C" int n2d_vie_radiation(n2d_vie *p, const double *current_dev, const double origin[3], double h,
                                 double k0, const double *dirs_dev, long long count, double *out_dev) {
  if (p->mirror) { n2c_set_error("radiation amplitude: free space only (plan has PEC images)"); return 0; }
  if (count <= 0) return 1;
  const long long blocks = (count + RAD_DIRS - 1) / RAD_DIRS;
  if (blocks > 0x7fffffffLL) { n2c_set_error("too many directions"); return 0; }
  radiation_kernel<<<(unsigned)blocks, 256, 0, n2c_stream()>>>((const double2 *)current_dev, p->cell_box, p->cells,
                                                               p->S[1], p->S[2], origin[0], origin[1], origin[2], h,
                                                               k0, dirs_dev, (int)count, (double2 *)out_dev);
  return n2c_check_launch("radiation");
}

template <typename C>
int n2c_vie_pass_plans(n2d_vie *p, int precondition, double *norm, int *flag, const int *scale, const int *variant,
                       PassArgs<C> args[5], int mode[5], int L[5], int var[5], size_t smem[5], long long tiles[5]) {
  for (int i = 0; i < N2D_VIE_PASSES; ++i) {
    PassPlan<C> pp;
    const int v = variant && variant[i] && fft_radix_variants(pass_length(p, i)) > 1 ? 1 : 0;
    const n2d_pass_choice ch = {batch_height(p, i, sizeof(C), scale ? scale[i] : 0), v};
    if (!pass_plan<C>(p, i, ch, nullptr, nullptr, precondition, norm, flag, &pp)) return 0;
    args[i] = pp.a;
    mode[i] = pp.mode;
    L[i] = pp.L;
    var[i] = v;
    smem[i] = pp.smem;
    tiles[i] = pp.tiles;
  }
  return 1;
}
template int n2c_vie_pass_plans<float2>(n2d_vie *, int, double *, int *, const int *, const int *,
                                        PassArgs<float2> *, int *, int *, int *, size_t *, long long *);
template int n2c_vie_pass_plans<double2>(n2d_vie *, int, double *, int *, const int *, const int *,
                                         PassArgs<double2> *, int *, int *, int *, size_t *, long long *);

/* CPU oracle for the nec2c dielectric solve path: TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference algorithms the CUDA backend replaces.
 * Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU baseline
 * arm, as the checker.  Each function names the reference file:line it follows.
 * Parity of this restatement with the reference is pinned by
 * tests/test_oracle.py against oracle/_ref (the reference compiled from its own
 * sources) and the reference's known-answer vectors.
 */
#include "nec2c_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static const double kPi = 3.141592653589793238462643383279502884;

struct oracle_plan {
  size_t cells, shape[3], padded[3], grid;
  size_t *site;        /* padded-grid index of each cell */
  ocplx *spectrum;     /* 6 x grid: xx yy zz xy xz yz */
  ocplx *work;         /* 6 x grid: 3 source + 3 field components */
  ocplx *twiddle[3];   /* exp(-2 pi i j / P) per axis */
  ocplx *eps;          /* per-cell relative permittivity */
  ocplx self[3];
};

/* Symmetric 3x3 component slot, vie_fft.c:53-54 (tensor_index). */
static int slot(int i, int j)
{
  int lo = i < j ? i : j, hi = i < j ? j : i;
  if(lo == hi) return lo;
  if(lo == 0) return hi == 1 ? 3 : 4;
  return 5;
}

static size_t site_index(const oracle_plan *p, size_t x, size_t y, size_t z)
{ return (x * p->padded[1] + y) * p->padded[2] + z; }

/* One radix-2 decimation-in-time line transform, vie_fft.c:94-115:
   bit-reversal permutation, then butterflies of growing span using the
   forward roots (conjugated for the inverse), then 1/n for the inverse. */
static void line_transform(ocplx *a, size_t n, size_t stride, const ocplx *roots,
                           int inverse)
{
  size_t i, rev = 0;
  for(i = 1; i < n; ++i) {
    size_t bit = n >> 1;
    while(rev & bit) { rev ^= bit; bit >>= 1; }
    rev ^= bit;
    if(i < rev) { ocplx t = a[i*stride]; a[i*stride] = a[rev*stride]; a[rev*stride] = t; }
  }
  for(size_t span = 2; span <= n; span <<= 1) {
    size_t half = span >> 1, step = n / span;
    for(size_t base = 0; base < n; base += span)
      for(size_t k = 0; k < half; ++k) {
        ocplx w = roots[k * step];
        if(inverse) w = conj(w);
        ocplx u = a[(base + k) * stride];
        ocplx v = w * a[(base + k + half) * stride];
        a[(base + k) * stride] = u + v;
        a[(base + k + half) * stride] = u - v;
      }
  }
  if(inverse) for(i = 0; i < n; ++i) a[i*stride] /= (double)n;
}

/* 3-D transform, axis order z, y, x: vie_fft.c:117-126 (fft3_serial). */
static void transform3(oracle_plan *p, ocplx *a, int inverse)
{
  size_t nx = p->padded[0], ny = p->padded[1], nz = p->padded[2], x, y, z;
  for(x = 0; x < nx; ++x) for(y = 0; y < ny; ++y)
    line_transform(a + site_index(p, x, y, 0), nz, 1, p->twiddle[2], inverse);
  for(x = 0; x < nx; ++x) for(z = 0; z < nz; ++z)
    line_transform(a + site_index(p, x, 0, z), ny, nz, p->twiddle[1], inverse);
  for(y = 0; y < ny; ++y) for(z = 0; z < nz; ++z)
    line_transform(a + site_index(p, 0, y, z), nx, ny * nz, p->twiddle[0], inverse);
}

/* Gauss-Legendre nodes on [0,1] by Newton iteration, vie_fft.c:284-298. */
static void gauss_legendre(int n, double *node, double *weight)
{
  for(int i = 0; i < (n + 1) / 2; ++i) {
    double z = cos(kPi * (i + .75) / (n + .5)), previous, slope = 0;
    do {
      double p0 = 1, p1 = 0;
      previous = z;
      for(int j = 1; j <= n; ++j) { double p2 = p1; p1 = p0; p0 = ((2*j - 1) * z * p1 - (j - 1) * p2) / j; }
      slope = n * (z * p0 - p1) / (z * z - 1);
      z = previous - p0 / slope;
    } while(fabs(z - previous) > 2e-15);
    node[i] = (1 - z) / 2; node[n - 1 - i] = (1 + z) / 2;
    weight[i] = weight[n - 1 - i] = 1 / ((1 - z * z) * slope * slope);
  }
}

/* Difference-coordinate Gauss rule with triangular weights, one order:
   vie_fft.c:299-318 (far_order). */
static void far_rule(const size_t offset[3], double h, double k, int order, ocplx out[9])
{
  double node[12], weight[12];
  gauss_legendre(order, node, weight);
  memset(out, 0, 9 * sizeof(ocplx));
  for(int a = 0; a < order; ++a) for(int b = 0; b < order; ++b) for(int c = 0; c < order; ++c) {
    double t[3] = {node[a], node[b], node[c]};
    double wt = h*h*h * weight[a]*weight[b]*weight[c] * (1 - t[0]) * (1 - t[1]) * (1 - t[2]);
    for(int mask = 0; mask < 8; ++mask) {
      double r[3], r2 = 0;
      for(int i = 0; i < 3; ++i) {
        r[i] = h * ((double)offset[i] + ((mask & (1 << i)) ? -t[i] : t[i]));
        r2 += r[i] * r[i];
      }
      double rr = sqrt(r2);
      ocplx g = wt * cexp(-I * k * rr) / (4 * kPi * rr);
      ocplx diag = g * (k*k - I*k/rr - 1/r2);
      ocplx radial = g * (-k*k + 3*I*k/rr + 3/r2) / r2;
      for(int i = 0; i < 3; ++i) for(int j = i; j < 3; ++j)
        out[3*i + j] += (i == j ? diag : 0) + radial * r[i] * r[j];
    }
  }
  for(int i = 0; i < 3; ++i) for(int j = i + 1; j < 3; ++j) out[3*j + i] = out[3*i + j];
}

/* Order ladder 4,6,8,12 with 2e-12 abs + 2e-9 rel acceptance, only for
   gap^2 > 4: vie_fft.c:319-335 (far_kernel). */
int oracle_far_kernel(const size_t v[3], double h, double k, ocplx out[9])
{
  static const int ladder[4] = {4, 6, 8, 12};
  ocplx last[9];
  double gap2 = 0;
  for(int i = 0; i < 3; ++i) { double g = v[i] > 1 ? (double)v[i] - 1 : 0; gap2 += g * g; }
  if(gap2 <= 4) return 0;
  far_rule(v, h, k, ladder[0], last);
  for(int s = 1; s < 4; ++s) {
    int ok = 1;
    far_rule(v, h, k, ladder[s], out);
    for(int e = 0; e < 9; ++e)
      if(!isfinite(creal(out[e])) || !isfinite(cimag(out[e])) ||
         cabs(out[e] - last[e]) > 2e-12 + 2e-9 * cabs(out[e])) ok = 0;
    if(ok) return 1;
    memcpy(last, out, sizeof(last));
  }
  return 0;
}

/* Spectrum build over sorted offsets a>=b>=c with permutation/sign fill,
   then the forward transform of the six components: vie_fft.c:338-377. */
static int build_spectrum(oracle_plan *p, double h, double k, oracle_near_fn near_fn, void *ctx)
{
  static const int perms[6][3] = {{0,1,2},{0,2,1},{1,0,2},{1,2,0},{2,0,1},{2,1,0}};
  size_t top = p->shape[0];
  if(p->shape[1] > top) top = p->shape[1];
  if(p->shape[2] > top) top = p->shape[2];
  for(size_t a = 0; a < top; ++a) for(size_t b = 0; b <= a; ++b) for(size_t c = 0; c <= b; ++c) {
    size_t v[3] = {a, b, c};
    ocplx n[9];
    int used = 0;
    for(int q = 0; q < 6; ++q)
      if(v[perms[q][0]] < p->shape[0] && v[perms[q][1]] < p->shape[1] && v[perms[q][2]] < p->shape[2]) used = 1;
    if(!used) continue;
    if(!oracle_far_kernel(v, h, k, n)) {
      if(!near_fn || !near_fn(ctx, v, h, k, n)) return 0;
    }
    for(int i = 0; i < 3; ++i) for(int j = i + 1; j < 3; ++j) {
      ocplx mean = (n[3*i + j] + n[3*j + i]) * 0.5;
      n[3*i + j] = n[3*j + i] = (v[i] && v[j]) ? mean : 0;
    }
    if(a == 0) for(int i = 0; i < 3; ++i) p->self[i] = n[4*i];
    for(int q = 0; q < 6; ++q) {
      const int *pm = perms[q];
      size_t d[3] = {v[pm[0]], v[pm[1]], v[pm[2]]};
      if(d[0] >= p->shape[0] || d[1] >= p->shape[1] || d[2] >= p->shape[2]) continue;
      for(int mask = 0; mask < 8; ++mask) {
        int sg[3]; size_t pos[3];
        for(int i = 0; i < 3; ++i) {
          sg[i] = (mask & (1 << i)) ? -1 : 1;
          pos[i] = (sg[i] < 0 && d[i]) ? p->padded[i] - d[i] : d[i];
        }
        size_t g = site_index(p, pos[0], pos[1], pos[2]);
        for(int i = 0; i < 3; ++i) for(int j = i; j < 3; ++j)
          p->spectrum[slot(i, j) * p->grid + g] = sg[i] * sg[j] * n[3*pm[i] + pm[j]];
      }
    }
  }
  for(int comp = 0; comp < 6; ++comp) transform3(p, p->spectrum + comp * p->grid, 0);
  return 1;
}

void oracle_plan_destroy(oracle_plan *p)
{
  if(!p) return;
  for(int d = 0; d < 3; ++d) free(p->twiddle[d]);
  free(p->site); free(p->spectrum); free(p->work); free(p->eps); free(p);
}

/* vie_fft.c:378-441 (vie_fft_create), validation and lattice map. */
int oracle_plan_create(oracle_plan **out, const size_t shape[3], size_t cells,
                       const size_t *xyz, double h, double k, double er_re,
                       double er_im, oracle_near_fn near_fn, void *near_ctx)
{
  oracle_plan *p;
  ocplx er = er_re + I * er_im;
  size_t c;
  if(!out) return 0;
  *out = NULL;
  if(!shape || !xyz || !cells || cells > SIZE_MAX / 3 || !isfinite(h) || h <= 0 ||
     !isfinite(k) || k < 0 || !isfinite(creal(er)) || !isfinite(cimag(er)) ||
     creal(er) < 1 || cimag(er) > 0 || !isfinite(k * h) || k * h > 1) return 0;
  p = calloc(1, sizeof(*p));
  if(!p) return 0;
  p->grid = 1;
  for(int d = 0; d < 3; ++d) {
    if(!shape[d] || shape[d] > (1u << 20)) { oracle_plan_destroy(p); return 0; }
    p->shape[d] = shape[d];
    p->padded[d] = 1;
    while(p->padded[d] < 2 * shape[d] - 1) p->padded[d] *= 2;
    p->grid *= p->padded[d];
  }
  p->cells = cells;
  p->site = malloc(cells * sizeof(*p->site));
  p->spectrum = calloc(6 * p->grid, sizeof(ocplx));
  p->work = calloc(6 * p->grid, sizeof(ocplx));
  p->eps = malloc(cells * sizeof(ocplx));
  if(!p->site || !p->spectrum || !p->work || !p->eps) goto fail;
  for(c = 0; c < cells; ++c) {
    size_t pos[3];
    for(int d = 0; d < 3; ++d) { pos[d] = xyz[3*c + d]; if(pos[d] >= shape[d]) goto fail; }
    size_t g = site_index(p, pos[0], pos[1], pos[2]);
    if(creal(p->work[g]) != 0) goto fail;       /* duplicate lattice site */
    p->work[g] = 1; p->site[c] = g;
  }
  memset(p->work, 0, p->grid * sizeof(ocplx));
  for(int d = 0; d < 3; ++d) {
    p->twiddle[d] = malloc(p->padded[d] * sizeof(ocplx));
    if(!p->twiddle[d]) goto fail;
    for(size_t j = 0; j < p->padded[d]; ++j)
      p->twiddle[d][j] = cexp(-2 * kPi * I * (double)j / (double)p->padded[d]);
  }
  if(!build_spectrum(p, h, k, near_fn, near_ctx)) goto fail;
  for(c = 0; c < cells; ++c) if(!oracle_plan_set_permittivity(p, c, er_re, er_im)) goto fail;
  *out = p;
  return 1;
fail:
  oracle_plan_destroy(p);
  return 0;
}

/* vie_fft.c:445-455 (vie_fft_set_permittivity). */
int oracle_plan_set_permittivity(oracle_plan *p, size_t cell, double er_re, double er_im)
{
  ocplx er = er_re + I * er_im;
  if(!p || cell >= p->cells || !isfinite(creal(er)) || !isfinite(cimag(er)) ||
     creal(er) < 1 || cimag(er) > 0) return 0;
  for(int i = 0; i < 3; ++i) {
    ocplx dg = er - (er - 1) * p->self[i];
    if(!isfinite(cabs(dg)) || cabs(dg) < 1e-30) return 0;
  }
  p->eps[cell] = er;
  return 1;
}

size_t oracle_plan_padded(const oracle_plan *p, int axis) { return p->padded[axis]; }
void oracle_plan_spectrum(const oracle_plan *p, ocplx *out)
{ memcpy(out, p->spectrum, 6 * p->grid * sizeof(ocplx)); }
void oracle_plan_self(const oracle_plan *p, ocplx self[3])
{ for(int i = 0; i < 3; ++i) self[i] = p->self[i]; }

/* y = eps x - (eps-1) gather(IFFT(Ghat . FFT(scatter x))): vie_fft.c:239-263. */
int oracle_plan_apply(oracle_plan *p, const ocplx *x, ocplx *y)
{
  size_t G = p->grid;
  ocplx *src = p->work, *dst = p->work + 3 * G;
  memset(p->work, 0, 6 * G * sizeof(ocplx));
  for(size_t c = 0; c < p->cells; ++c)
    for(int i = 0; i < 3; ++i) src[i * G + p->site[c]] = x[3*c + i];
  for(int i = 0; i < 3; ++i) transform3(p, src + i * G, 0);
  for(size_t g = 0; g < 3 * G; ++g) {
    size_t comp = g / G, point = g % G;
    for(int j = 0; j < 3; ++j)
      dst[g] += p->spectrum[slot((int)comp, j) * G + point] * src[j * G + point];
  }
  for(int i = 0; i < 3; ++i) transform3(p, dst + i * G, 1);
  for(size_t c = 0; c < p->cells; ++c)
    for(int i = 0; i < 3; ++i)
      y[3*c + i] = p->eps[c] * x[3*c + i] - (p->eps[c] - 1) * dst[i * G + p->site[c]];
  return 1;
}

/* Jacobi: x / (eps - (eps-1) self[i]): vie_fft.c:265-273. */
int oracle_plan_precondition(oracle_plan *p, const ocplx *x, ocplx *y)
{
  for(size_t c = 0; c < p->cells; ++c)
    for(int i = 0; i < 3; ++i)
      y[3*c + i] = x[3*c + i] / (p->eps[c] - (p->eps[c] - 1) * p->self[i]);
  return 1;
}

/* ---------------------------------------------------------------- hybrid */
struct oracle_hybrid {
  size_t c, v;
  int pec;
  const ocplx *blocks;   /* caller-owned, dielectric_fft.c:34-40 layout */
  oracle_plan *volume;
  ocplx *image;          /* 4 v scratch for the PEC image embedding */
};

int oracle_hybrid_create(oracle_hybrid **out, oracle_plan *volume, size_t c, size_t v,
                         const ocplx *blocks, int pec)
{
  oracle_hybrid *h = calloc(1, sizeof(*h));
  if(!h) return 0;
  h->c = c; h->v = v; h->pec = pec; h->blocks = blocks; h->volume = volume;
  if(pec && v) { h->image = calloc(4 * v, sizeof(ocplx)); if(!h->image) { free(h); return 0; } }
  *out = h;
  return 1;
}

void oracle_hybrid_destroy(oracle_hybrid *h) { if(h) { free(h->image); free(h); } }

/* dielectric_fft.c:41-66: volume (optionally through PEC images), then the
   dense conductor rows [C|B] and the cross block D. */
int oracle_hybrid_apply(oracle_hybrid *h, const ocplx *x, ocplx *y)
{
  size_t c = h->c, v = h->v;
  if(v && h->image) {
    ocplx *in = h->image, *out = in + 2 * v;
    for(size_t i = 0; i < v; ++i) { in[i] = x[c + i]; in[v + i] = (i % 3 == 2 ? 1 : -1) * x[c + i]; }
    if(!oracle_plan_apply(h->volume, in, out)) return 0;
    memcpy(y + c, out, v * sizeof(ocplx));
  } else if(v && !oracle_plan_apply(h->volume, x + c, y + c)) return 0;
  for(size_t i = 0; i < c; ++i) {
    y[i] = 0;
    for(size_t j = 0; j < c + v; ++j) y[i] += h->blocks[i * (c + v) + j] * x[j];
  }
  for(size_t i = 0; i < v; ++i)
    for(size_t j = 0; j < c; ++j) y[c + i] += h->blocks[c * (c + v) + i * c + j] * x[j];
  return 1;
}

/* dielectric_fft.c:67-83. */
int oracle_hybrid_precondition(oracle_hybrid *h, const ocplx *x, ocplx *y)
{
  size_t c = h->c, v = h->v;
  if(v && h->image) {
    ocplx *in = h->image, *out = in + 2 * v;
    memcpy(in, x + c, v * sizeof(ocplx));
    memset(in + v, 0, v * sizeof(ocplx));
    if(!oracle_plan_precondition(h->volume, in, out)) return 0;
    memcpy(y + c, out, v * sizeof(ocplx));
  } else if(v && !oracle_plan_precondition(h->volume, x + c, y + c)) return 0;
  for(size_t i = 0; i < c; ++i) {
    ocplx dg = h->blocks[i * (c + v) + i];
    if(!isfinite(cabs(dg)) || cabs(dg) < DBL_MIN) return 0;
    y[i] = x[i] / dg;
  }
  return 1;
}

/* ------------------------------------------------------------------ GMRES */
enum { ST_CONVERGED, ST_LIMIT, ST_BREAKDOWN, ST_CALLBACK, ST_INVALID, ST_ALLOC, ST_NONFINITE };

/* hypot-accumulated 2-norm with a non-finite check: vie_iterative.c:9-19. */
static double safe_norm(size_t n, const ocplx *x)
{
  double r = 0;
  for(size_t i = 0; i < n; ++i) {
    if(!isfinite(creal(x[i])) || !isfinite(cimag(x[i]))) return NAN;
    r = hypot(r, cabs(x[i]));
  }
  return r;
}

/* vie_iterative.c:50-63. */
static int true_residual(size_t n, oracle_map apply, void *actx, const ocplx *b,
                         const ocplx *x, ocplx *r, oracle_report *rep)
{
  ++rep->operator_applications;
  if(!apply(actx, x, r)) { rep->status = ST_CALLBACK; return 0; }
  for(size_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
  rep->residual_norm = safe_norm(n, r);
  if(!isfinite(rep->residual_norm)) { rep->status = ST_NONFINITE; return 0; }
  return 1;
}

/* Unitary Givens [c s; -conj(s) c]: vie_iterative.c:66-78. */
static void givens(ocplx a, ocplx b, double *c, ocplx *s)
{
  double aa = cabs(a), bb = cabs(b);
  if(bb == 0.0) { *c = 1.0; *s = 0.0; }
  else if(aa == 0.0) { *c = 0.0; *s = conj(b) / bb; }
  else { double len = hypot(aa, bb); *c = aa / len; *s = (a / aa) * (conj(b) / len); }
}

/* Right-preconditioned restarted GMRES with two MGS passes, true residual at
   every restart: vie_iterative.c:80-199. */
int oracle_gmres(size_t n, oracle_map apply, void *actx, oracle_map precondition,
                 void *pctx, const ocplx *b, ocplx *x, size_t restart,
                 size_t maxit, double rtol, double atol, oracle_report *rep)
{
  oracle_report local;
  ocplx *V = NULL, *Z = NULL, *H = NULL, *r = NULL, *w = NULL, *g = NULL, *y = NULL, *s = NULL;
  double *cs = NULL, bnorm, target;
  size_t m, j, k, i;
  int ok = 0;
  if(!rep) rep = &local;
  memset(rep, 0, sizeof(*rep));
  rep->status = ST_INVALID;
  rep->residual_norm = rep->relative_residual = INFINITY;
  if(!apply || n == 0 || !b || !x || b == x || restart == 0 || maxit == 0 ||
     !isfinite(rtol) || rtol < 0 || !isfinite(atol) || atol < 0 || (rtol == 0 && atol == 0))
    return 0;
  m = restart;
  if(m > n) m = n;
  if(m > maxit) m = maxit;
  if(n > SIZE_MAX / 16 / (m + 1)) { rep->status = ST_ALLOC; return 0; }
  V = calloc(n * (m + 1), sizeof(ocplx)); Z = calloc(n * m, sizeof(ocplx));
  H = calloc((m + 1) * m, sizeof(ocplx)); r = calloc(n, sizeof(ocplx));
  w = calloc(n, sizeof(ocplx)); g = calloc(m + 1, sizeof(ocplx));
  y = calloc(m, sizeof(ocplx)); s = calloc(m, sizeof(ocplx)); cs = calloc(m, sizeof(double));
  if(!V || !Z || !H || !r || !w || !g || !y || !s || !cs) { rep->status = ST_ALLOC; goto done; }
  bnorm = safe_norm(n, b);
  target = fmax(atol, rtol * bnorm);
  if(!isfinite(bnorm) || !isfinite(safe_norm(n, x)) || !isfinite(target)) { rep->status = ST_NONFINITE; goto done; }
  if(!true_residual(n, apply, actx, b, x, r, rep)) goto done;
  for(;;) {
    size_t used = 0;
    int broke = 0;
    double beta = rep->residual_norm;
    rep->relative_residual = bnorm > 0 ? beta / bnorm : beta;
    if(beta <= target) { rep->status = ST_CONVERGED; ok = 1; goto done; }
    if(rep->iterations >= maxit) { rep->status = ST_LIMIT; goto done; }
    memset(H, 0, (m + 1) * m * sizeof(ocplx));
    memset(g, 0, (m + 1) * sizeof(ocplx)); g[0] = beta;
    for(i = 0; i < n; ++i) V[i] = r[i] / beta;
    for(j = 0; j < m && rep->iterations < maxit; ++j) {
      double before, after;
      if(precondition) {
        if(!precondition(pctx, V + j*n, Z + j*n)) { rep->status = ST_CALLBACK; goto done; }
      } else memcpy(Z + j*n, V + j*n, n * sizeof(ocplx));
      if(!isfinite(safe_norm(n, Z + j*n))) { rep->status = ST_NONFINITE; goto done; }
      ++rep->operator_applications;
      if(!apply(actx, Z + j*n, w)) { rep->status = ST_CALLBACK; goto done; }
      before = safe_norm(n, w);
      if(!isfinite(before)) { rep->status = ST_NONFINITE; goto done; }
      for(int pass = 0; pass < 2; ++pass)
        for(k = 0; k <= j; ++k) {
          ocplx proj = 0;
          for(i = 0; i < n; ++i) proj += conj(V[k*n + i]) * w[i];
          H[k*m + j] += proj;
          for(i = 0; i < n; ++i) w[i] -= proj * V[k*n + i];
        }
      after = safe_norm(n, w);
      if(!isfinite(after)) { rep->status = ST_NONFINITE; goto done; }
      H[(j+1)*m + j] = after;
      broke = after <= 32 * DBL_EPSILON * before;
      if(!broke) for(i = 0; i < n; ++i) V[(j+1)*n + i] = w[i] / after;
      for(k = 0; k < j; ++k) {
        ocplx h0 = H[k*m + j], h1 = H[(k+1)*m + j];
        H[k*m + j] = cs[k] * h0 + s[k] * h1;
        H[(k+1)*m + j] = -conj(s[k]) * h0 + cs[k] * h1;
      }
      givens(H[j*m + j], H[(j+1)*m + j], &cs[j], &s[j]);
      H[j*m + j] = cs[j] * H[j*m + j] + s[j] * H[(j+1)*m + j];
      H[(j+1)*m + j] = 0;
      g[j+1] = -conj(s[j]) * g[j]; g[j] *= cs[j];
      ++rep->iterations; used = j + 1;
      if(broke || cabs(g[j+1]) <= target) break;
    }
    for(i = used; i-- > 0; ) {
      ocplx val = g[i];
      for(k = i + 1; k < used; ++k) val -= H[i*m + k] * y[k];
      if(cabs(H[i*m + i]) == 0.0) { rep->status = ST_BREAKDOWN; goto done; }
      y[i] = val / H[i*m + i];
    }
    for(j = 0; j < used; ++j) for(i = 0; i < n; ++i) x[i] += Z[j*n + i] * y[j];
    if(!true_residual(n, apply, actx, b, x, r, rep)) goto done;
    rep->relative_residual = bnorm > 0 ? rep->residual_norm / bnorm : rep->residual_norm;
    if(broke && rep->residual_norm > target) { rep->status = ST_BREAKDOWN; goto done; }
    if(rep->residual_norm > target && rep->iterations < maxit) ++rep->restarts;
  }
done:
  free(cs); free(s); free(y); free(g); free(w); free(r); free(H); free(Z); free(V);
  return ok;
}

static int plan_apply_cb(void *c, const ocplx *x, ocplx *y) { return oracle_plan_apply(c, x, y); }
static int plan_prec_cb(void *c, const ocplx *x, ocplx *y) { return oracle_plan_precondition(c, x, y); }
static int hyb_apply_cb(void *c, const ocplx *x, ocplx *y) { return oracle_hybrid_apply(c, x, y); }
static int hyb_prec_cb(void *c, const ocplx *x, ocplx *y) { return oracle_hybrid_precondition(c, x, y); }

int oracle_plan_gmres(oracle_plan *p, const ocplx *b, ocplx *x, size_t restart,
                      size_t maxit, double rtol, double atol, oracle_report *rep)
{
  return oracle_gmres(3 * p->cells, plan_apply_cb, p, plan_prec_cb, p, b, x,
                      restart, maxit, rtol, atol, rep);
}

int oracle_hybrid_gmres(oracle_hybrid *h, const ocplx *b, ocplx *x, size_t restart,
                        size_t maxit, double rtol, double atol, oracle_report *rep)
{
  return oracle_gmres(h->c + h->v, hyb_apply_cb, h, hyb_prec_cb, h, b, x,
                      restart, maxit, rtol, atol, rep);
}

/* -------------------------------------------------------------------- LU */
/* Gauss-Doolittle on NEC's transposed storage: un-transpose, then factor one
   column at a time with pivot = largest |.|^2 (later row wins ties), 1-based
   pivot rows in ip[]: matrix.c:1313-1416 (factr, builtin branch).  Returns 0
   when a pivot is exactly zero (the reference only prints a warning there). */
int oracle_factr(int n, ocplx *a, int *ip, int ndim)
{
  ocplx *col = malloc((size_t)(n > 0 ? n : 1) * sizeof(ocplx));
  int ok = 1;
  if(!col) return 0;
  for(int i = 1; i < n; ++i)
    for(int j = 0; j < i; ++j) {
      ocplx t = a[i + (size_t)j*ndim]; a[i + (size_t)j*ndim] = a[j + (size_t)i*ndim]; a[j + (size_t)i*ndim] = t;
    }
  for(int r = 0; r < n; ++r) {
    for(int k = 0; k < n; ++k) col[k] = a[k + (size_t)r*ndim];
    for(int j = 0; j < r; ++j) {
      int pj = ip[j] - 1;
      ocplx arj = col[pj];
      a[j + (size_t)r*ndim] = arj;
      col[pj] = col[j];
      for(int i = j + 1; i < n; ++i) col[i] -= a[i + (size_t)j*ndim] * arj;
    }
    double best = creal(col[r] * conj(col[r]));
    ip[r] = r + 1;
    for(int i = r + 1; i < n; ++i) {
      double mag = creal(col[i] * conj(col[i]));
      if(mag >= best) { best = mag; ip[r] = i + 1; }
    }
    if(best == 0.0) ok = 0;
    int pr = ip[r] - 1;
    a[r + (size_t)r*ndim] = col[pr];
    col[pr] = col[r];
    if(r + 1 < n) {
      ocplx inv = 1. / a[r + (size_t)r*ndim];
      for(int i = r + 1; i < n; ++i) a[i + (size_t)r*ndim] = col[i] * inv;
    }
  }
  free(col);
  return ok;
}

/* Forward substitution with row interchanges, then back substitution:
   matrix.c:1523-1555 (solve_builtin). */
void oracle_solve(int n, const ocplx *a, const int *ip, ocplx *b, int ndim)
{
  ocplx *tmp = malloc((size_t)(n > 0 ? n : 1) * sizeof(ocplx));
  if(!tmp) return;
  for(int i = 0; i < n; ++i) {
    int pi = ip[i] - 1;
    tmp[i] = b[pi]; b[pi] = b[i];
    for(int j = i + 1; j < n; ++j) b[j] -= a[j + (size_t)i*ndim] * tmp[i];
  }
  for(int k = 0; k < n; ++k) {
    int i = n - k - 1;
    ocplx sum = 0;
    for(int j = i + 1; j < n; ++j) sum += a[i + (size_t)j*ndim] * b[j];
    b[i] = (tmp[i] - sum) / a[i + (size_t)i*ndim];
  }
  free(tmp);
}

/* Row-major elimination with partial pivoting on cabs (strict >, first row
   wins ties), pivot floor 64 eps, RHS eliminated in place:
   dense_backend.c:152-190 (builtin_row_major_solve). */
int oracle_row_major_solve(ocplx *a, ocplx *b, size_t n)
{
  for(size_t k = 0; k < n; ++k) {
    size_t piv = k;
    double big = cabs(a[k*n + k]);
    for(size_t i = k + 1; i < n; ++i) { double c = cabs(a[i*n + k]); if(c > big) { big = c; piv = i; } }
    if(!(big > 64.0 * DBL_EPSILON)) return 0;
    if(piv != k) {
      for(size_t j = k; j < n; ++j) { ocplx t = a[k*n + j]; a[k*n + j] = a[piv*n + j]; a[piv*n + j] = t; }
      ocplx t = b[k]; b[k] = b[piv]; b[piv] = t;
    }
    for(size_t i = k + 1; i < n; ++i) {
      ocplx mul = a[i*n + k] / a[k*n + k];
      a[i*n + k] = mul;
      for(size_t j = k + 1; j < n; ++j) a[i*n + j] -= mul * a[k*n + j];
      b[i] -= mul * b[k];
    }
  }
  for(size_t i = n; i-- > 0; ) {
    ocplx sum = b[i];
    for(size_t j = i + 1; j < n; ++j) sum -= a[i*n + j] * b[j];
    b[i] = sum / a[i*n + i];
  }
  return 1;
}

/* ------------------------------------------------ far-field amplitude */
/* sin(x)/x with its series near 0 (dielectric_solver.c:47-55). */
static double sinc_small(double x)
{
  if(fabs(x) < 1.0e-5) { const double x2 = x * x; return 1.0 - x2 / 6.0 + x2 * x2 / 120.0; }
  return sin(x) / x;
}

/* dielectric_solver.c:90-150 in free space: integral = sum_cells J V
   prod_a sinc(k d_a s_a / 2) exp(+i k d.r), then the transverse part
   (integral x d) x d, times i k c0 mu0 / (4 pi) (c0 = 299792458,
   mu0 = 1.25663706212e-6 as dielectric_solver.c:21-22). */
void oracle_radiation_amplitude(size_t cells, const double *centers, double h, const ocplx *current,
                                double k0, const double direction[3], ocplx out[3])
{
  const double c0 = 299792458.0, mu0 = 1.25663706212e-6, volume = h * h * h;
  ocplx integral[3] = {0, 0, 0}, crossed[3];
  double average = 1.0;
  for(int a = 0; a < 3; ++a) average *= sinc_small(0.5 * k0 * direction[a] * h);
  for(size_t i = 0; i < cells; ++i) {
    const double dot = direction[0] * centers[3 * i] + direction[1] * centers[3 * i + 1] +
                       direction[2] * centers[3 * i + 2];
    const ocplx weight = volume * average * cexp(I * k0 * dot);
    for(int a = 0; a < 3; ++a) integral[a] += current[3 * i + a] * weight;
  }
  crossed[0] = integral[1] * direction[2] - integral[2] * direction[1];
  crossed[1] = integral[2] * direction[0] - integral[0] * direction[2];
  crossed[2] = integral[0] * direction[1] - integral[1] * direction[0];
  out[0] = crossed[1] * direction[2] - crossed[2] * direction[1];
  out[1] = crossed[2] * direction[0] - crossed[0] * direction[2];
  out[2] = crossed[0] * direction[1] - crossed[1] * direction[0];
  for(int a = 0; a < 3; ++a) out[a] *= I * k0 * c0 * mu0 / (4.0 * kPi);
}

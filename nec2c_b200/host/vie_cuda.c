/* Host side of the CUDA volume operator, hybrid system and GMRES (C, like the
 * reference).  Validation, lattice mapping, byte accounting and the near-pair
 * callback follow vie_fft.c / dielectric_fft.c / vie_iterative.c; the device
 * work is done through the device layer (csrc/device_api.h). */
#include <complex.h>
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/nec2c_cuda.h"
#include "../csrc/device_api.h"

static const double kPi = 3.141592653589793238462643383279502884;

enum { ST_CONVERGED, ST_LIMIT, ST_BREAKDOWN, ST_CALLBACK, ST_INVALID, ST_ALLOC, ST_NONFINITE };

static int g_fft_fp32 = 0;

int nec2c_cuda_available(void) { return n2d_device_ok(); }
const char *nec2c_cuda_last_error(void) { return n2d_last_error(); }
void nec2c_cuda_set_stream(void *s) { n2d_set_stream(s); }
int nec2c_cuda_set_device(int device) { return n2d_set_device(device); }
unsigned long long nec2c_cuda_launch_count(void) { return n2d_launch_count(); }

int nec2c_cuda_vie_fft_backend_set(const char *name)
{
  if(!name) { n2c_set_error("FFT backend: null name"); return 0; }
  if(!strcmp(name, "cuda")) g_fft_fp32 = 0;
  else if(!strcmp(name, "cuda-mixed")) g_fft_fp32 = 1;
  else { n2c_set_error("unknown FFT backend '%s' (cuda, cuda-mixed)", name); return 0; }
  return 1;
}
const char *nec2c_cuda_vie_fft_backend_name(void) { return g_fft_fp32 ? "cuda-mixed" : "cuda"; }

struct nec2c_cuda_vie_plan {
  n2d_vie *dev;
  size_t cells, shape[3], padded[3], grids, bytes;
  double pitch, k0;
  double complex *eps;      /* host shadow of the per-cell permittivity */
  double complex self[3];
  int eps_dirty;
  double *x_dev, *y_dev;    /* staging for host-vector products */
};

static int mul_ok(size_t a, size_t b, size_t *out) { if(b && a > SIZE_MAX / b) return 0; *out = a * b; return 1; }
static int add_ok(size_t a, size_t b, size_t *out) { if(a > SIZE_MAX - b) return 0; *out = a + b; return 1; }

/* Gauss-Legendre nodes/weights on [0,1] by Newton iteration (the rule of
   vie_fft.c:284-298), orders 4, 6, 8, 12. */
static void gauss_tables(double nodes[4][12], double weights[4][12])
{
  static const int orders[4] = {4, 6, 8, 12};
  memset(nodes, 0, 48 * sizeof(double)); memset(weights, 0, 48 * sizeof(double));
  for(int s = 0; s < 4; ++s) {
    const int n = orders[s];
    for(int i = 0; i < (n + 1) / 2; ++i) {
      double z = cos(kPi * (i + .75) / (n + .5)), prev, slope = 0;
      do {
        double p0 = 1, p1 = 0;
        prev = z;
        for(int j = 1; j <= n; ++j) { double p2 = p1; p1 = p0; p0 = ((2*j - 1) * z * p1 - (j - 1) * p2) / j; }
        slope = n * (z * p0 - p1) / (z * z - 1);
        z = prev - p0 / slope;
      } while(fabs(z - prev) > 2e-15);
      nodes[s][i] = (1 - z) / 2; nodes[s][n - 1 - i] = (1 + z) / 2;
      weights[s][i] = weights[s][n - 1 - i] = 1 / ((1 - z * z) * slope * slope);
    }
  }
}

static int diag_ok(const double complex self[3], double complex er)
{
  for(int i = 0; i < 3; ++i) {
    double complex d = er - (er - 1) * self[i];
    if(!isfinite(cabs(d)) || cabs(d) < 1e-30) return 0;
  }
  return 1;
}

static int upload_eps(struct nec2c_cuda_vie_plan *p)
{
  double self[6];
  for(int i = 0; i < 3; ++i) { self[2*i] = creal(p->self[i]); self[2*i + 1] = cimag(p->self[i]); }
  if(!n2d_vie_set_eps(p->dev, (const double *)p->eps, self)) return 0;
  p->eps_dirty = 0;
  return 1;
}

void nec2c_cuda_vie_fft_destroy(nec2c_cuda_vie_plan *p)
{
  if(!p) return;
  n2d_vie_destroy(p->dev);
  n2d_free(p->x_dev); n2d_free(p->y_dev);
  free(p->eps);
  free(p);
}

/* vie_fft_create starts its byte count at sizeof(struct vie_fft_plan)
   (vie_fft.c:19-28, :381): seven size_t, an int, five pointers and three
   complex doubles, 160 bytes on LP64 in a build without FFTW (whose three
   plan handles and flag add 32). */
enum { REF_PLAN_STRUCT_BYTES = 160 };

int nec2c_cuda_vie_fft_create(nec2c_cuda_vie_plan **out, const size_t shape[3], size_t cells,
                              const size_t *xyz, double h, double k, double er_re, double er_im,
                              size_t limit, nec2c_cuda_near_tensor_fn near, void *near_ctx)
{
  struct nec2c_cuda_vie_plan *p = NULL;
  double complex er = er_re + I * er_im;
  size_t padded[3], g = 1, bytes = REF_PLAN_STRUCT_BYTES, tmp, root_bytes = 0;
  int *cell_box = NULL, *offsets = NULL, *far_ok = NULL;
  unsigned char *seen = NULL;
  double *tw[3] = {NULL, NULL, NULL}, *near_t = NULL;
  long long *near_i = NULL;
  if(!out) return 0;
  *out = NULL;
  /* vie_fft.c:383-384 */
  if(!shape || !xyz || !cells || cells > SIZE_MAX / 3 || !isfinite(h) || h <= 0 || !isfinite(k) ||
     k < 0 || !isfinite(er_re) || !isfinite(er_im) || er_re < 1 || er_im > 0 || !isfinite(k * h) ||
     k * h > 1) { n2c_set_error("invalid plan arguments"); return 0; }
  for(int d = 0; d < 3; ++d) {
    if(!shape[d] || shape[d] > SIZE_MAX / 2) { n2c_set_error("invalid lattice shape"); return 0; }
    padded[d] = 1;
    while(padded[d] < 2 * shape[d] - 1) {
      if(padded[d] > SIZE_MAX / 2) return 0;
      padded[d] *= 2;
    }
    if(!mul_ok(g, padded[d], &g) || !mul_ok(padded[d], sizeof(double complex), &tmp) ||
       !add_ok(root_bytes, tmp, &root_bytes)) { n2c_set_error("lattice size overflow"); return 0; }
  }
  /* The reference's accounted bytes (vie_fft.c:394-396). */
  if(!mul_ok(g, 12 * sizeof(double complex), &tmp) || !add_ok(bytes, tmp, &bytes) ||
     !mul_ok(cells, sizeof(size_t) + sizeof(double complex), &tmp) || !add_ok(bytes, tmp, &bytes) ||
     !add_ok(bytes, root_bytes, &bytes) || bytes > limit) {
    n2c_set_error("plan exceeds its byte limit");
    return 0;
  }
  if(!n2d_device_ok()) return 0;
  for(int d = 0; d < 3; ++d)
    if(padded[d] > 1024) { n2c_set_error("padded axis %zu exceeds 1024", padded[d]); return 0; }
  p = calloc(1, sizeof(*p));
  if(!p) return 0;
  p->cells = cells; p->grids = g; p->bytes = bytes;
  memcpy(p->shape, shape, sizeof(p->shape)); memcpy(p->padded, padded, sizeof(p->padded));
  p->pitch = h; p->k0 = k;
  p->eps = malloc(cells * sizeof(double complex));
  cell_box = malloc(cells * sizeof(int));
  size_t nbox = shape[0] * shape[1] * shape[2];
  seen = calloc(nbox, 1);
  if(!p->eps || !cell_box || !seen) goto fail;
  /* Lattice map with duplicate rejection (vie_fft.c:416-423). */
  for(size_t c = 0; c < cells; ++c) {
    size_t pos[3];
    for(int d = 0; d < 3; ++d) { pos[d] = xyz[3*c + d]; if(pos[d] >= shape[d]) { n2c_set_error("cell outside lattice"); goto fail; } }
    size_t b = (pos[0] * shape[1] + pos[1]) * shape[2] + pos[2];
    if(seen[b]) { n2c_set_error("duplicate lattice site"); goto fail; }
    seen[b] = 1;
    cell_box[c] = (int)b;
  }
  for(int d = 0; d < 3; ++d) {
    tw[d] = malloc(2 * padded[d] * sizeof(double));
    if(!tw[d]) goto fail;
    for(size_t j = 0; j < padded[d]; ++j) {
      double complex w = cexp(-2 * kPi * I * (double)j / (double)padded[d]);
      tw[d][2*j] = creal(w); tw[d][2*j + 1] = cimag(w);
    }
  }
  {
    long long ls[3] = {(long long)shape[0], (long long)shape[1], (long long)shape[2]};
    long long lp[3] = {(long long)padded[0], (long long)padded[1], (long long)padded[2]};
    const double *twc[3] = {tw[0], tw[1], tw[2]};
    double nodes[4][12], weights[4][12];
    gauss_tables(nodes, weights);
    if(!n2d_vie_set_gauss(&nodes[0][0], &weights[0][0])) goto fail;
    if(!n2d_vie_create(&p->dev, ls, lp, (long long)cells, cell_box, twc, g_fft_fp32)) goto fail;
  }
  /* Sorted displacements a>=b>=c that fit the lattice in some orientation, in
     the reference's enumeration order (vie_fft.c:345-351). */
  {
    long long S[3] = {(long long)shape[0], (long long)shape[1], (long long)shape[2]};
    for(int i = 0; i < 2; ++i) for(int j = 0; j < 2 - i; ++j)
      if(S[j] < S[j + 1]) { long long t = S[j]; S[j] = S[j + 1]; S[j + 1] = t; }
    long long count = 0;
    for(long long a = 0; a < S[0]; ++a)
      for(long long b = 0; b <= a && b < S[1]; ++b)
        count += (b < S[2] ? b : S[2] - 1) + 1;
    offsets = malloc(3 * count * sizeof(int));
    far_ok = malloc(count * sizeof(int));
    if(!offsets || !far_ok) goto fail;
    long long q = 0;
    for(long long a = 0; a < S[0]; ++a)
      for(long long b = 0; b <= a && b < S[1]; ++b)
        for(long long c = 0; c <= b && c < S[2]; ++c) {
          offsets[3*q] = (int)a; offsets[3*q + 1] = (int)b; offsets[3*q + 2] = (int)c; ++q;
        }
    if(!n2d_vie_far_tensors(p->dev, count, offsets, S, h, k, far_ok)) goto fail;
    long long nn = 0;
    for(long long i = 0; i < count; ++i) nn += !far_ok[i];
    near_t = malloc((nn ? nn : 1) * 12 * sizeof(double));
    near_i = malloc((nn ? nn : 1) * sizeof(long long));
    if(!near_t || !near_i) goto fail;
    long long m = 0;
    for(long long i = 0; i < count; ++i) {
      if(far_ok[i]) continue;
      size_t v[3] = {(size_t)offsets[3*i], (size_t)offsets[3*i + 1], (size_t)offsets[3*i + 2]};
      nec2c_cuda_complex n9[9];
      double complex n[9];
      if(!near || !near(near_ctx, v, h, k, n9)) { n2c_set_error("near-pair tensor unavailable"); goto fail; }
      memcpy(n, n9, sizeof(n));
      /* Symmetric off-diagonals, zero where the offset component vanishes
         (vie_fft.c:353-356). */
      double complex xy = (v[0] && v[1]) ? (n[1] + n[3]) * 0.5 : 0;
      double complex xz = (v[0] && v[2]) ? (n[2] + n[6]) * 0.5 : 0;
      double complex yz = (v[1] && v[2]) ? (n[5] + n[7]) * 0.5 : 0;
      double complex six[6] = {n[0], n[4], n[8], xy, xz, yz};
      for(int e = 0; e < 6; ++e) { near_t[12*m + 2*e] = creal(six[e]); near_t[12*m + 2*e + 1] = cimag(six[e]); }
      near_i[m++] = i;
      if(v[0] == 0) for(int d = 0; d < 3; ++d) p->self[d] = n[4*d];   /* offset (0,0,0) */
    }
    if(!n2d_vie_put_tensors(p->dev, m, near_i, near_t)) goto fail;
    if(!n2d_vie_finish_spectrum(p->dev)) goto fail;
  }
  /* Uniform permittivity, validated like vie_fft.c:437. */
  if(!diag_ok(p->self, er)) { n2c_set_error("singular local diagonal"); goto fail; }
  for(size_t c = 0; c < cells; ++c) p->eps[c] = er;
  if(!upload_eps(p)) goto fail;
  p->x_dev = n2d_alloc(3 * cells * 2 * sizeof(double));
  p->y_dev = n2d_alloc(3 * cells * 2 * sizeof(double));
  if(!p->x_dev || !p->y_dev) goto fail;
  for(int d = 0; d < 3; ++d) free(tw[d]);
  free(cell_box); free(seen); free(offsets); free(far_ok); free(near_t); free(near_i);
  *out = p;
  return 1;
fail:
  for(int d = 0; d < 3; ++d) free(tw[d]);
  free(cell_box); free(seen); free(offsets); free(far_ok); free(near_t); free(near_i);
  nec2c_cuda_vie_fft_destroy(p);
  return 0;
}

int nec2c_cuda_vie_fft_set_permittivity(nec2c_cuda_vie_plan *p, size_t cell, double re, double im)
{
  double complex er = re + I * im;
  if(!p || cell >= p->cells) { n2c_set_error("set_permittivity: no plan or cell out of range"); return 0; }
  /* vie_fft.c:448-453: a finite eps with Re >= 1 and Im <= 0, and a Jacobi
     divisor of at least 1e-30 on every axis. */
  if(!isfinite(re) || !isfinite(im) || re < 1 || im > 0) {
    n2c_set_error("set_permittivity: need a finite eps with Re >= 1 and Im <= 0");
    return 0;
  }
  if(!diag_ok(p->self, er)) { n2c_set_error("set_permittivity: Jacobi divisor of cell %zu vanishes", cell); return 0; }
  p->eps[cell] = er;
  p->eps_dirty = 1;
  return 1;
}

size_t nec2c_cuda_vie_fft_bytes(const nec2c_cuda_vie_plan *p) { return p ? p->bytes : 0; }
size_t nec2c_cuda_vie_fft_device_bytes(const nec2c_cuda_vie_plan *p) { return p ? n2d_vie_device_bytes(p->dev) : 0; }
size_t nec2c_cuda_vie_fft_order(const nec2c_cuda_vie_plan *p) { return p ? 3 * p->cells : 0; }

/* Exposed to the hybrid and GMRES code in this layer. */
__attribute__((visibility("hidden"))) n2d_vie *nec2c_cuda_plan_device(nec2c_cuda_vie_plan *p)
{
  if(!p) { n2c_set_error("null plan"); return NULL; }
  if(p->eps_dirty && !upload_eps(p)) return NULL;
  return p->dev;
}

int nec2c_cuda_vie_fft_apply(void *ctx, const nec2c_cuda_complex *x, nec2c_cuda_complex *y)
{
  struct nec2c_cuda_vie_plan *p = ctx;
  size_t bytes;
  if(!nec2c_cuda_plan_device(p)) return 0;
  if(!x || !y) { n2c_set_error("null vector"); return 0; }
  bytes = 3 * p->cells * sizeof(double complex);
  return n2d_upload(p->x_dev, x, bytes) && n2d_vie_apply(p->dev, p->x_dev, p->y_dev, 0, NULL, NULL, 0) &&
         n2d_download(y, p->y_dev, bytes);
}

int nec2c_cuda_vie_fft_precondition(void *ctx, const nec2c_cuda_complex *x, nec2c_cuda_complex *y)
{
  struct nec2c_cuda_vie_plan *p = ctx;
  size_t bytes;
  if(!nec2c_cuda_plan_device(p)) return 0;
  if(!x || !y) { n2c_set_error("null vector"); return 0; }
  bytes = 3 * p->cells * sizeof(double complex);
  return n2d_upload(p->x_dev, x, bytes) && n2d_vie_precondition(p->dev, p->x_dev, p->y_dev) &&
         n2d_download(y, p->y_dev, bytes);
}

int nec2c_cuda_vie_fft_apply_device(nec2c_cuda_vie_plan *p, const void *x_dev, void *y_dev)
{
  if(!nec2c_cuda_plan_device(p)) return 0;
  return n2d_vie_apply(p->dev, x_dev, y_dev, 0, NULL, NULL, 0);
}

int nec2c_cuda_vie_fft_spectrum(nec2c_cuda_vie_plan *p, nec2c_cuda_complex *out)
{
  if(!p || !out) { n2c_set_error("spectrum: null plan or output"); return 0; }
  return n2d_vie_read_spectrum(p->dev, (double *)out);
}

int nec2c_cuda_vie_fft_radiation_device(nec2c_cuda_vie_plan *p, const double origin[3], const void *current_dev,
                                        size_t count, const double *directions, nec2c_cuda_complex *amplitude)
{
  double *dirs, *out;
  int ok;
  if(!p || !origin || !current_dev || (count && (!directions || !amplitude))) {
    n2c_set_error("radiation: null plan, origin, current, directions or output");
    return 0;
  }
  if(count == 0) return 1;
  if(count > (size_t)1 << 28) { n2c_set_error("radiation: too many directions"); return 0; }
  dirs = n2d_alloc(3 * count * sizeof(double));
  out = n2d_alloc(3 * count * 2 * sizeof(double));
  ok = dirs && out && n2d_upload(dirs, directions, 3 * count * sizeof(double)) &&
       n2d_vie_radiation(p->dev, current_dev, origin, p->pitch, p->k0, dirs, (long long)count, out) &&
       n2d_download(amplitude, out, 3 * count * 2 * sizeof(double));
  n2d_free(dirs);
  n2d_free(out);
  return ok;
}

void nec2c_cuda_vie_fft_autotune(int enable) { n2d_vie_autotune(enable); }
int nec2c_cuda_vie_fft_autotune_enabled(void) { return n2d_vie_autotune_enabled(); }

int nec2c_cuda_vie_fft_tune(nec2c_cuda_vie_plan *p, int measure)
{
  if(!p || measure < 0 || measure > 2) { n2c_set_error("tune: bad argument"); return 0; }
  if(!nec2c_cuda_plan_device(p)) return 0;
  return n2d_vie_tune(p->dev, measure);
}

int nec2c_cuda_vie_fft_schedule(nec2c_cuda_vie_plan *p, int fp64, int tiles[5], int r1[5])
{
  if(!p || !tiles || !r1) return -1;
  if(!fp64 && !n2d_vie_fp32(p->dev)) return -1;
  if(!nec2c_cuda_plan_device(p)) return -1;
  return n2d_vie_schedule(p->dev, fp64 ? 1 : 0, tiles, r1);
}

int nec2c_cuda_vie_fft_set_schedule(nec2c_cuda_vie_plan *p, int fp64, const int tiles[5], const int r1[5])
{
  if(!p || !tiles || !r1) { n2c_set_error("set_schedule: bad argument"); return 0; }
  if(!fp64 && !n2d_vie_fp32(p->dev)) { n2c_set_error("set_schedule: the plan has no FP32 transforms"); return 0; }
  if(!nec2c_cuda_plan_device(p)) return 0;
  return n2d_vie_set_schedule(p->dev, fp64 ? 1 : 0, tiles, r1);
}

int nec2c_cuda_vie_fft_planes(nec2c_cuda_vie_plan *p, int fp64)
{
  if(!p) return -1;
  if(!fp64 && !n2d_vie_fp32(p->dev)) return -1;
  if(!nec2c_cuda_plan_device(p)) return -1;
  return n2d_vie_planes(p->dev, fp64 ? 1 : 0);
}

int nec2c_cuda_vie_fft_set_planes(nec2c_cuda_vie_plan *p, int fp64, int planes)
{
  if(!p) { n2c_set_error("set_planes: bad argument"); return 0; }
  if(!fp64 && !n2d_vie_fp32(p->dev)) { n2c_set_error("set_planes: the plan has no FP32 transforms"); return 0; }
  if(!nec2c_cuda_plan_device(p)) return 0;
  return n2d_vie_set_planes(p->dev, fp64 ? 1 : 0, planes);
}

/* ------------------------------------------------------------------ hybrid */
struct nec2c_cuda_hybrid {
  n2d_hybrid *dev;
  nec2c_cuda_vie_plan *volume;
  size_t c, v;
  int blocks_set;
  double *x_dev, *y_dev;
};

int nec2c_cuda_hybrid_create(nec2c_cuda_hybrid **out, nec2c_cuda_vie_plan *volume, size_t c, size_t v,
                             int pec)
{
  struct nec2c_cuda_hybrid *h;
  if(!out) return 0;
  *out = NULL;
  if((v && !volume) || (volume && v != 3 * volume->cells / (pec ? 2 : 1)) || c > SIZE_MAX - v) {
    n2c_set_error("hybrid system does not match its volume plan");
    return 0;
  }
  if(!n2d_device_ok()) return 0;
  h = calloc(1, sizeof(*h));
  if(!h) return 0;
  h->volume = volume; h->c = c; h->v = v;
  if(!n2d_hybrid_create(&h->dev, volume ? volume->dev : NULL, (long long)c, (long long)v, pec)) { free(h); return 0; }
  h->x_dev = n2d_alloc((c + v) * 2 * sizeof(double));
  h->y_dev = n2d_alloc((c + v) * 2 * sizeof(double));
  if(!h->x_dev || !h->y_dev) { nec2c_cuda_hybrid_destroy(h); return 0; }
  *out = h;
  return 1;
}

void nec2c_cuda_hybrid_destroy(nec2c_cuda_hybrid *h)
{
  if(!h) return;
  n2d_hybrid_destroy(h->dev);
  n2d_free(h->x_dev); n2d_free(h->y_dev);
  free(h);
}

int nec2c_cuda_hybrid_set_blocks(nec2c_cuda_hybrid *h, const nec2c_cuda_complex *blocks)
{
  if(!h || !blocks) { n2c_set_error("set_blocks: null system or blocks"); return 0; }
  if(h->volume && !nec2c_cuda_plan_device(h->volume)) return 0;
  if(!n2d_hybrid_upload_blocks(h->dev, (const double *)blocks)) return 0;
  h->blocks_set = 1;
  return 1;
}

size_t nec2c_cuda_hybrid_order(const nec2c_cuda_hybrid *h) { return h ? h->c + h->v : 0; }

/* The volume plan a hybrid system runs on (request server exclusivity). */
const nec2c_cuda_vie_plan *n2c_hybrid_volume_plan(const nec2c_cuda_hybrid *h) { return h ? h->volume : NULL; }

static int hybrid_ready(struct nec2c_cuda_hybrid *h)
{
  if(!h) { n2c_set_error("null hybrid system"); return 0; }
  if(!h->blocks_set) { n2c_set_error("hybrid blocks were never uploaded"); return 0; }
  return !h->volume || nec2c_cuda_plan_device(h->volume) != NULL;
}

int nec2c_cuda_hybrid_apply(void *ctx, const nec2c_cuda_complex *x, nec2c_cuda_complex *y)
{
  struct nec2c_cuda_hybrid *h = ctx;
  size_t bytes;
  if(!hybrid_ready(h)) return 0;
  if(!x || !y) { n2c_set_error("null vector"); return 0; }
  bytes = (h->c + h->v) * sizeof(double complex);
  return n2d_upload(h->x_dev, x, bytes) &&
         n2d_hybrid_apply(h->dev, h->x_dev, h->y_dev, 0, NULL, NULL, 0) && n2d_download(y, h->y_dev, bytes);
}

int nec2c_cuda_hybrid_precondition(void *ctx, const nec2c_cuda_complex *x, nec2c_cuda_complex *y)
{
  struct nec2c_cuda_hybrid *h = ctx;
  size_t bytes;
  if(!hybrid_ready(h)) return 0;
  if(!x || !y) { n2c_set_error("null vector"); return 0; }
  bytes = (h->c + h->v) * sizeof(double complex);
  /* dielectric_fft.c:77-81: a zero or non-finite conductor diagonal fails. */
  if(!n2d_hybrid_precondition_ok(h->dev)) {
    n2c_set_error("hybrid preconditioner: a diagonal entry is zero or not finite");
    return 0;
  }
  return n2d_upload(h->x_dev, x, bytes) &&
         n2d_hybrid_precondition(h->dev, h->x_dev, h->y_dev) && n2d_download(y, h->y_dev, bytes);
}

/* ------------------------------------------------------------------- GMRES */
static int gmres_common(int kind, void *op, size_t n, const void *b, void *x, int device,
                        double *stage_b, double *stage_x,
                        const nec2c_cuda_gmres_options *options, nec2c_cuda_gmres_report *report)
{
  nec2c_cuda_gmres_report local;
  nec2c_cuda_gmres_options defaults = {30, 300, 1e-12, 0.0};
  n2d_gmres_report r;
  if(!report) report = &local;
  memset(report, 0, sizeof(*report));
  report->status = ST_INVALID;
  report->residual_norm = report->relative_residual = INFINITY;
  if(!options) options = &defaults;
  /* vie_iterative.c:97-103 */
  if(!op || n == 0 || !b || !x || (const void *)b == (const void *)x || options->restart == 0 ||
     options->maximum_iterations == 0 || !isfinite(options->relative_tolerance) ||
     options->relative_tolerance < 0 || !isfinite(options->absolute_tolerance) ||
     options->absolute_tolerance < 0 ||
     (options->relative_tolerance == 0 && options->absolute_tolerance == 0))
    return 0;
  if(options->restart == SIZE_MAX || n > (size_t)LLONG_MAX / 64) { report->status = ST_ALLOC; return 0; }
  int ok;
  if(device || !stage_b) {
    ok = (device ? n2d_gmres_dev : n2d_gmres)(kind, op, (long long)n, (const double *)b, (double *)x,
                                              options->restart, options->maximum_iterations,
                                              options->relative_tolerance,
                                              options->absolute_tolerance, &r);
  } else {
    /* Host vectors through the operator's persistent staging buffers; x is
       copied back even when the solve fails (vie_iterative.h:51-53). */
    size_t bytes = n * sizeof(double complex);
    memset(&r, 0, sizeof(r));
    r.status = ST_ALLOC;
    ok = n2d_upload(stage_b, b, bytes) && n2d_upload(stage_x, x, bytes);
    if(ok) {
      ok = n2d_gmres_dev(kind, op, (long long)n, stage_b, stage_x, options->restart,
                         options->maximum_iterations, options->relative_tolerance,
                         options->absolute_tolerance, &r);
      if(!n2d_download(x, stage_x, bytes)) ok = 0;
    }
  }
  report->status = r.status;
  report->iterations = r.iterations;
  report->operator_applications = r.operator_applications;
  report->restarts = r.restarts;
  report->residual_norm = r.residual_norm;
  report->relative_residual = r.relative_residual;
  return ok;
}

int nec2c_cuda_gmres_plan(nec2c_cuda_vie_plan *p, const nec2c_cuda_complex *b, nec2c_cuda_complex *x,
                          const nec2c_cuda_gmres_options *options, nec2c_cuda_gmres_report *report)
{
  n2d_vie *dev = p ? nec2c_cuda_plan_device(p) : NULL;
  return gmres_common(0, dev, p ? 3 * p->cells : 0, b, x, 0, p ? p->x_dev : NULL, p ? p->y_dev : NULL,
                      options, report);
}

int nec2c_cuda_gmres_plan_device(nec2c_cuda_vie_plan *p, const void *b, void *x,
                                 const nec2c_cuda_gmres_options *options, nec2c_cuda_gmres_report *report)
{
  n2d_vie *dev = p ? nec2c_cuda_plan_device(p) : NULL;
  return gmres_common(0, dev, p ? 3 * p->cells : 0, b, x, 1, NULL, NULL, options, report);
}

int nec2c_cuda_gmres_hybrid(nec2c_cuda_hybrid *h, const nec2c_cuda_complex *b, nec2c_cuda_complex *x,
                            const nec2c_cuda_gmres_options *options, nec2c_cuda_gmres_report *report)
{
  if(h && !hybrid_ready(h)) {
    if(report) { memset(report, 0, sizeof(*report)); report->status = ST_CALLBACK; }
    return 0;
  }
  return gmres_common(1, h ? h->dev : NULL, h ? h->c + h->v : 0, b, x, 0, h ? h->x_dev : NULL,
                      h ? h->y_dev : NULL, options, report);
}

int nec2c_cuda_gmres_hybrid_device(nec2c_cuda_hybrid *h, const void *b, void *x,
                                   const nec2c_cuda_gmres_options *options, nec2c_cuda_gmres_report *report)
{
  if(h && !hybrid_ready(h)) {
    if(report) { memset(report, 0, sizeof(*report)); report->status = ST_CALLBACK; }
    return 0;
  }
  return gmres_common(1, h ? h->dev : NULL, h ? h->c + h->v : 0, b, x, 1, NULL, NULL, options, report);
}

/* ------------------------------------------------------- batch of plans */
struct nec2c_cuda_vie_batch {
  n2d_vie_batch *dev;
  size_t count, order;
  nec2c_cuda_vie_plan **plans;    /* volume plan of each system */
  nec2c_cuda_hybrid **hybrids;    /* NULL for a batch of plans */
  size_t *offsets;
  void *b_dev, *x_dev;   /* staging of the host-vector solve */
};

static int batch_ready(nec2c_cuda_vie_batch *b)
{
  for(size_t q = 0; q < b->count; ++q) {
    if(b->hybrids && !hybrid_ready(b->hybrids[q])) return 0;
    if(!nec2c_cuda_plan_device(b->plans[q])) return 0;
  }
  return 1;
}

void nec2c_cuda_vie_batch_destroy(nec2c_cuda_vie_batch *b)
{
  if(!b) return;
  n2d_vie_batch_destroy(b->dev);
  n2d_free(b->b_dev);
  n2d_free(b->x_dev);
  free(b->plans);
  free(b->hybrids);
  free(b->offsets);
  free(b);
}

int nec2c_cuda_vie_batch_create(nec2c_cuda_vie_batch **out, nec2c_cuda_vie_plan *const *plans, size_t count)
{
  nec2c_cuda_vie_batch *b;
  n2d_vie **devs;
  if(!out) return 0;
  *out = NULL;
  if(!plans || count == 0 || count > ((size_t)1 << 20)) { n2c_set_error("batch: bad plan list"); return 0; }
  b = calloc(1, sizeof(*b));
  devs = calloc(count, sizeof(*devs));
  if(!b || !devs) { free(b); free(devs); return 0; }
  b->count = count;
  b->plans = calloc(count, sizeof(*b->plans));
  b->offsets = calloc(count + 1, sizeof(*b->offsets));
  if(!b->plans || !b->offsets) { free(devs); nec2c_cuda_vie_batch_destroy(b); return 0; }
  for(size_t q = 0; q < count; ++q) {
    if(!plans[q]) { n2c_set_error("batch: plan %zu is NULL", q); free(devs); nec2c_cuda_vie_batch_destroy(b); return 0; }
    b->plans[q] = plans[q];
    devs[q] = nec2c_cuda_plan_device(plans[q]);
    if(!devs[q]) { free(devs); nec2c_cuda_vie_batch_destroy(b); return 0; }
  }
  if(!n2d_vie_batch_create(&b->dev, devs, (long long)count)) { free(devs); nec2c_cuda_vie_batch_destroy(b); return 0; }
  free(devs);
  for(size_t q = 0; q <= count; ++q) b->offsets[q] = (size_t)n2d_vie_batch_offset(b->dev, (long long)q);
  b->order = b->offsets[count];
  *out = b;
  return 1;
}

int nec2c_cuda_hybrid_batch_create(nec2c_cuda_vie_batch **out, nec2c_cuda_hybrid *const *systems, size_t count)
{
  nec2c_cuda_vie_batch *b;
  n2d_hybrid **devs;
  if(!out) return 0;
  *out = NULL;
  if(!systems || count == 0 || count > ((size_t)1 << 20)) { n2c_set_error("batch: bad system list"); return 0; }
  b = calloc(1, sizeof(*b));
  devs = calloc(count, sizeof(*devs));
  if(!b || !devs) { free(b); free(devs); return 0; }
  b->count = count;
  b->plans = calloc(count, sizeof(*b->plans));
  b->hybrids = calloc(count, sizeof(*b->hybrids));
  b->offsets = calloc(count + 1, sizeof(*b->offsets));
  if(!b->plans || !b->hybrids || !b->offsets) { free(devs); nec2c_cuda_vie_batch_destroy(b); return 0; }
  for(size_t q = 0; q < count; ++q) {
    nec2c_cuda_hybrid *h = systems[q];
    if(!h || !h->volume) {
      n2c_set_error("batch: system %zu has no volume plan", q);
      free(devs); nec2c_cuda_vie_batch_destroy(b); return 0;
    }
    if(!hybrid_ready(h) || !nec2c_cuda_plan_device(h->volume)) { free(devs); nec2c_cuda_vie_batch_destroy(b); return 0; }
    b->hybrids[q] = h;
    b->plans[q] = h->volume;
    devs[q] = h->dev;
  }
  if(!n2d_hybrid_batch_create(&b->dev, devs, (long long)count)) { free(devs); nec2c_cuda_vie_batch_destroy(b); return 0; }
  free(devs);
  for(size_t q = 0; q <= count; ++q) b->offsets[q] = (size_t)n2d_vie_batch_offset(b->dev, (long long)q);
  b->order = b->offsets[count];
  *out = b;
  return 1;
}

size_t nec2c_cuda_vie_batch_order(const nec2c_cuda_vie_batch *b) { return b ? b->order : 0; }
size_t nec2c_cuda_vie_batch_systems(const nec2c_cuda_vie_batch *b) { return b ? b->count : 0; }

/* The volume plan of system q of a batch (request server exclusivity). */
const nec2c_cuda_vie_plan *n2c_batch_plan(const nec2c_cuda_vie_batch *b, size_t q)
{
  return b && q < b->count ? b->plans[q] : NULL;
}
size_t nec2c_cuda_vie_batch_offset(const nec2c_cuda_vie_batch *b, size_t q)
{
  return b && q <= b->count ? b->offsets[q] : 0;
}

int nec2c_cuda_vie_batch_schedule(const nec2c_cuda_vie_batch *b, int scale[5], int variant[5])
{
  if(!b || !scale || !variant) { n2c_set_error("batch schedule: bad argument"); return 0; }
  n2d_vie_batch_schedule(b->dev, scale, variant);
  return 1;
}

int nec2c_cuda_vie_batch_set_schedule(nec2c_cuda_vie_batch *b, const int scale[5], const int variant[5])
{
  if(!b || !scale || !variant) { n2c_set_error("batch schedule: bad argument"); return 0; }
  return n2d_vie_batch_set_schedule(b->dev, scale, variant);
}

int nec2c_cuda_vie_batch_apply_device(nec2c_cuda_vie_batch *b, const void *x_dev, void *y_dev)
{
  if(!b || !x_dev || !y_dev || x_dev == y_dev) { n2c_set_error("batch apply: bad argument"); return 0; }
  return batch_ready(b) && n2d_vie_batch_apply(b->dev, x_dev, y_dev);
}

static int batch_options_ok(const nec2c_cuda_gmres_options *o)
{
  /* vie_iterative.c:97-103 */
  return o->restart > 0 && o->maximum_iterations > 0 && isfinite(o->relative_tolerance) &&
         o->relative_tolerance >= 0 && isfinite(o->absolute_tolerance) && o->absolute_tolerance >= 0 &&
         !(o->relative_tolerance == 0 && o->absolute_tolerance == 0);
}

static int batch_solve(nec2c_cuda_vie_batch *b, const void *b_dev, void *x_dev, const unsigned char *idle,
                       const nec2c_cuda_gmres_options *options, nec2c_cuda_gmres_report *reports)
{
  nec2c_cuda_gmres_options defaults = {30, 300, 1e-12, 0.0};
  n2d_gmres_report *r;
  int ok;
  for(size_t q = 0; q < b->count; ++q) {
    memset(&reports[q], 0, sizeof(reports[q]));
    reports[q].status = ST_INVALID;
    reports[q].residual_norm = reports[q].relative_residual = INFINITY;
  }
  if(!options) options = &defaults;
  if(!batch_options_ok(options) || b_dev == x_dev) {
    n2c_set_error(b_dev == x_dev ? "batch solve: b and x must differ" : "batch solve: invalid GMRES options");
    return 0;
  }
  r = calloc(b->count, sizeof(*r));
  if(!r) { n2c_set_error("batch solve: out of host memory"); return 0; }
  ok = batch_ready(b) &&
       n2d_gmres_batch_dev(b->dev, b_dev, x_dev, options->restart, options->maximum_iterations,
                           options->relative_tolerance, options->absolute_tolerance, idle, r);
  for(size_t q = 0; q < b->count; ++q) {
    reports[q].status = r[q].status;
    reports[q].iterations = r[q].iterations;
    reports[q].operator_applications = r[q].operator_applications;
    reports[q].restarts = r[q].restarts;
    reports[q].residual_norm = r[q].residual_norm;
    reports[q].relative_residual = r[q].relative_residual;
  }
  free(r);
  return ok;
}

int nec2c_cuda_gmres_batch_device(nec2c_cuda_vie_batch *b, const void *b_dev, void *x_dev,
                                  const nec2c_cuda_gmres_options *options, nec2c_cuda_gmres_report *reports)
{
  if(!b || !b_dev || !x_dev || !reports) { n2c_set_error("batch solve: null batch, vector or reports"); return 0; }
  return batch_solve(b, b_dev, x_dev, NULL, options, reports);
}

/* Host vectors through the batch's staging buffers.  With subset != 0 a
   system whose bv[q] is NULL is idle: its segments are zeroed, it takes no
   part in the solve and its xv[q] is not written. */
static int batch_host(nec2c_cuda_vie_batch *b, const nec2c_cuda_complex *const *bv, nec2c_cuda_complex *const *xv,
                      int subset, const nec2c_cuda_gmres_options *options, nec2c_cuda_gmres_report *reports)
{
  const size_t cpx = sizeof(nec2c_cuda_complex);
  unsigned char *idle = NULL;
  size_t active = 0;
  int ok = 1, whole = 1;
  if(!b || !bv || !xv || !reports) { n2c_set_error("batch solve: null batch, vector list or reports"); return 0; }
  for(size_t q = 0; q < b->count; ++q) {
    if(subset && !bv[q]) continue;
    if(!bv[q] || !xv[q]) { n2c_set_error("batch solve: vector of system %zu is NULL", q); return 0; }
    ++active;
  }
  if(active < b->count) {
    if(active == 0) { n2c_set_error("batch solve: no system to solve"); return 0; }
    idle = calloc(b->count, 1);
    if(!idle) { n2c_set_error("batch solve: out of host memory"); return 0; }
    for(size_t q = 0; q < b->count; ++q) idle[q] = !bv[q];
    whole = 0;
  }
  /* Vectors that lie back to back in host memory (a server batch request's
     concatenated b and x) move in one copy each way. */
  for(size_t q = 1; q < b->count && whole; ++q)
    whole = bv[q] == bv[0] + b->offsets[q] && xv[q] == xv[0] + b->offsets[q];
  if(!b->b_dev) b->b_dev = n2d_alloc(b->order * cpx);
  if(!b->x_dev) b->x_dev = n2d_alloc(b->order * cpx);
  if(!b->b_dev || !b->x_dev) { free(idle); return 0; }
  if(whole) {
    ok = n2d_upload(b->b_dev, bv[0], b->order * cpx) && n2d_upload(b->x_dev, xv[0], b->order * cpx);
  } else {
    if(idle) ok = n2d_memset(b->b_dev, 0, b->order * cpx) && n2d_memset(b->x_dev, 0, b->order * cpx);
    for(size_t q = 0; q < b->count && ok; ++q) {
      const size_t off = b->offsets[q] * cpx, bytes = (b->offsets[q + 1] - b->offsets[q]) * cpx;
      if(idle && idle[q]) continue;
      ok = n2d_upload((char *)b->b_dev + off, bv[q], bytes) && n2d_upload((char *)b->x_dev + off, xv[q], bytes);
    }
  }
  if(!ok) { free(idle); return 0; }
  const int solved = batch_solve(b, b->b_dev, b->x_dev, idle, options, reports);
  /* x is copied back even when a solve fails (vie_iterative.h:51-53). */
  if(whole) {
    if(!n2d_download(xv[0], b->x_dev, b->order * cpx)) ok = 0;
  } else {
    for(size_t q = 0; q < b->count; ++q) {
      const size_t off = b->offsets[q] * cpx, bytes = (b->offsets[q + 1] - b->offsets[q]) * cpx;
      if(idle && idle[q]) continue;
      if(!n2d_download(xv[q], (char *)b->x_dev + off, bytes)) ok = 0;
    }
  }
  free(idle);
  /* A subset solve reports convergence per system only. */
  return subset ? ok : ok && solved;
}

int nec2c_cuda_gmres_batch(nec2c_cuda_vie_batch *b, const nec2c_cuda_complex *const *bv,
                           nec2c_cuda_complex *const *xv, const nec2c_cuda_gmres_options *options,
                           nec2c_cuda_gmres_report *reports)
{
  return batch_host(b, bv, xv, 0, options, reports);
}

/* The request server's merged volume requests: the systems whose bv[q] is
   non-NULL, solved together; the others idle.  Returns 1 when the solve ran
   and every x came back (each system's convergence is in its report), 0
   with the error set otherwise. */
int n2c_gmres_batch_subset(nec2c_cuda_vie_batch *b, const nec2c_cuda_complex *const *bv,
                           nec2c_cuda_complex *const *xv, const nec2c_cuda_gmres_options *options,
                           nec2c_cuda_gmres_report *reports)
{
  return batch_host(b, bv, xv, 1, options, reports);
}

/* Index of a volume request's operator (a plan, or a hybrid system) among a
   batch's systems; (size_t)-1 when it is not one of them. */
size_t n2c_batch_index(const nec2c_cuda_vie_batch *b, const nec2c_cuda_vie_plan *plan,
                       const nec2c_cuda_hybrid *system)
{
  if(!b || (!plan) == (!system)) return (size_t)-1;
  for(size_t q = 0; q < b->count; ++q) {
    if(system && b->hybrids && b->hybrids[q] == system) return q;
    if(plan && !b->hybrids && b->plans[q] == plan) return q;
  }
  return (size_t)-1;
}

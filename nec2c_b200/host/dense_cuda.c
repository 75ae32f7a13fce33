/* Host side of the CUDA dense backend: dense_backend.c's classic factor/solve
 * and row-major solve entry points (C, like the reference).  The factor keeps
 * its device copy (and, for the mixed form, the original matrix) so the
 * solves that follow on the same thread do not re-upload it.  The cache is
 * per thread: the reference keeps one factorisation per process
 * (dense_backend.c:15), and threads that each own a stream (the request
 * server) keep one each. */
#include <complex.h>
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/nec2c_cuda.h"
#include "../csrc/device_api.h"

static int g_dense_mixed = 0;

int nec2c_cuda_dense_backend_set(const char *name)
{
  if(!name) { n2c_set_error("dense backend: null name"); return 0; }
  if(!strcmp(name, "cuda")) g_dense_mixed = 0;
  else if(!strcmp(name, "cuda-mixed")) g_dense_mixed = 1;
  else { n2c_set_error("unknown dense backend '%s' (cuda, cuda-mixed)", name); return 0; }
  return 1;
}
const char *nec2c_cuda_dense_backend_name(void) { return g_dense_mixed ? "cuda-mixed" : "cuda"; }

/* The most recent classic factorisation of this thread, kept on the device. */
static _Thread_local struct {
  const void *host;      /* host matrix the factors were written to */
  size_t order, ld;
  double *lu_dev;        /* FP64 form: row-major LU, leading dim order */
  int *piv_dev;
  float *lu32_dev;       /* split form: FP32 LU, leading dim ld32 (even) */
  size_t ld32;
  double *orig_dev;      /* split form: the FP64 matrix (refinement residuals) */
  double anorm;          /* split form: its infinity norm */
  int mixed;
} g_cache;

static _Thread_local int g_last_refinement = 0;

void nec2c_cuda_dense_release(void)
{
  n2d_free(g_cache.lu_dev); n2d_free(g_cache.piv_dev); n2d_free_async(g_cache.lu32_dev); n2d_free(g_cache.orig_dev);
  memset(&g_cache, 0, sizeof(g_cache));
}

int nec2c_cuda_dense_last_refinement(void) { return g_last_refinement; }

static const size_t CPX = 2 * sizeof(double);

/* Uploads NEC's transposed storage (column-major A^T, leading dim ld), which
   is the algebraic matrix A row-major: the device factors it in that layout
   (leading dim order). */
static double *upload_matrix(const void *matrix, size_t n, size_t ld)
{
  double *a = n2d_alloc(n * n * CPX);
  if(!a) return NULL;
  if(!n2d_upload2d(a, n * CPX, matrix, ld * CPX, n * CPX, n) || !n2d_sync()) { n2d_free(a); return NULL; }
  return a;
}

/* Split-precision factors on the device, with the FP64 original. */
typedef struct {
  float *lu32;
  size_t ld32;
  int *piv;
  const double *orig;
  double anorm;
} split_factors;

/* Refined solve with split-precision factors (the iteration of LAPACK's
   mixed-precision zcgesv): x = 0, r = b; repeat d = LU32 \ r, x += d,
   r = b - A x until every column has ||r||_inf <= ||x||_inf ||A||_inf eps
   sqrt(n), at most 30 steps; otherwise an FP64 factorisation solves it.  b
   (order x count on the device) is replaced by the solution.  Buffers are
   stream-ordered. */
static int solve_refined(size_t n, const split_factors *f, double *b, size_t count, int *steps)
{
  const long long N = (long long)n, K = (long long)count;
  const double cte = f->anorm * DBL_EPSILON * sqrt((double)n);
  double *x = n2d_alloc_async(n * count * CPX), *r = n2d_alloc_async(n * count * CPX);
  double *d = n2d_alloc_async(n * count * CPX);
  unsigned long long *norm = n2d_alloc_async(2 * count * sizeof(unsigned long long));
  double *rn = malloc(2 * count * sizeof(double)), *xn = rn ? rn + count : NULL;
  int ok = x && r && d && norm && rn && xn && n2d_memset(x, 0, n * count * CPX) && n2d_copy_d2d(r, b, n * count * CPX);
  int done = 0, it;
  *steps = 0;
  for(it = 1; ok && it <= 30 && !done; ++it) {
    size_t j;
    ok = n2d_copy_d2d(d, r, n * count * CPX) &&
         n2d_lu_solve32(f->lu32, N, (long long)f->ld32, f->piv, d, N, K) &&
         n2d_add_correction(x, d, N, K, N, norm + count, NULL) &&
         n2d_residual(f->orig, N, N, x, b, r, K, N, norm, NULL) && n2d_read_norms(norm, 2 * K, rn);
    done = ok;
    for(j = 0; ok && j < count; ++j) if(!(rn[j] <= xn[j] * cte)) done = 0;
    if(done) *steps = it;
  }
  if(ok && !done) {
    /* Not converged: FP64 factorisation of a copy of the original. */
    double *a = n2d_alloc_async(n * n * CPX);
    int *piv = n2d_alloc_async(n * sizeof(int)), info = 0;
    ok = a && piv && n2d_copy_d2d(a, f->orig, n * n * CPX) &&
         n2d_lu_factor(a, N, N, piv, 0, 0, &info) && !info && n2d_copy_d2d(x, b, n * count * CPX) &&
         n2d_lu_solve(a, N, N, piv, x, N, K);
    n2d_free_async(a); n2d_free_async(piv);
    *steps = -1;
  }
  ok = ok && n2d_copy_d2d(b, x, n * count * CPX);
  n2d_free_async(x); n2d_free_async(r); n2d_free_async(d); n2d_free_async(norm);
  free(rn);
  return ok;
}

/* Split-precision factorisation of the device matrix a (order n, leading
   dim n), which stays as the refinement original. */
static int split_factor(double *a, size_t n, int *piv, split_factors *f)
{
  const size_t ld32 = n + (n & 1);
  float *lu32 = n2d_alloc_async(n * ld32 * 2 * sizeof(float));
  void *norm = n2d_alloc_async(sizeof(unsigned long long));
  double anorm = 0;
  int info = 0;
  int ok = lu32 && norm && n2d_narrow(a, (long long)n, lu32, (long long)ld32, (long long)n, (long long)n) &&
           n2d_norm_inf(a, (long long)n, (long long)n, norm, &anorm) &&
           n2d_lu_factor32(lu32, (long long)n, (long long)ld32, piv, 0, &info);
  if(ok && info) { n2c_set_error("matrix is singular (pivot %d)", info); ok = 0; }
  n2d_free_async(norm);
  if(!ok) { n2d_free_async(lu32); return 0; }
  f->lu32 = lu32; f->ld32 = ld32; f->piv = piv; f->orig = a; f->anorm = anorm;
  return 1;
}

/* Factor and solve on a private device copy (the host matrix is left as it
   is and no factors are kept): the request server's dense solve.  split
   selects the split-precision form.  Every device buffer is stream-ordered on
   this thread's stream. */
int n2c_dense_solve_private(size_t n, const nec2c_cuda_complex *matrix, size_t ld, nec2c_cuda_complex *rhs,
                            size_t stride, size_t count, int split, int *steps)
{
  double *a, *b;
  int *piv, ok, info = 0;
  split_factors f;
  *steps = 0;
  if(!matrix || !rhs || n == 0 || n > INT_MAX || ld < n || stride < n || count == 0 || count > INT_MAX) return 0;
  a = n2d_alloc_async(n * n * CPX);
  b = n2d_alloc_async(n * count * CPX);
  piv = n2d_alloc_async(n * sizeof(int));
  ok = a && b && piv && n2d_upload2d(a, n * CPX, matrix, ld * CPX, n * CPX, n) &&
       n2d_upload2d(b, n * CPX, rhs, stride * CPX, n * CPX, count);
  if(ok && split) {
    ok = split_factor(a, n, piv, &f) && solve_refined(n, &f, b, count, steps);
    if(f.lu32 && ok) n2d_free_async(f.lu32);
  } else if(ok) {
    ok = n2d_lu_factor(a, (long long)n, (long long)n, piv, 0, 0, &info);
    if(ok && info) { n2c_set_error("matrix is singular (pivot %d)", info); ok = 0; }
    ok = ok && n2d_lu_solve(a, (long long)n, (long long)n, piv, b, (long long)n, (long long)count);
  }
  ok = ok && n2d_download2d(rhs, stride * CPX, b, n * CPX, n * CPX, count);
  n2d_free_async(a); n2d_free_async(b); n2d_free_async(piv);
  return ok;
}

int nec2c_cuda_dense_factor_classic(size_t n, nec2c_cuda_complex *matrix, size_t ld, int *pivots)
{
  int info = 0, ok;
  double *a;
  int *piv;
  /* dense_backend.c:71-81: the LAPACK branch's dimension checks. */
  if(!matrix || !pivots || n == 0 || n > INT_MAX || ld < n || ld > INT_MAX) {
    n2c_set_error("factor: null matrix or pivots, order 0, or leading dimension below the order");
    return 0;
  }
  if(!n2d_device_ok()) return 0;
  nec2c_cuda_dense_release();
  a = upload_matrix(matrix, n, ld);
  piv = n2d_alloc(n * sizeof(int));
  if(!a || !piv) { n2d_free(a); n2d_free(piv); return 0; }
  if(g_dense_mixed) {
    /* Split form: FP32 factors on the device, widened into the host storage;
       the FP64 matrix stays for the refinement. */
    split_factors f;
    double *wide = NULL;
    memset(&f, 0, sizeof(f));
    ok = split_factor(a, n, piv, &f);
    wide = ok ? n2d_alloc(n * n * CPX) : NULL;
    ok = ok && wide && n2d_widen(f.lu32, (long long)f.ld32, wide, (long long)n, (long long)n, (long long)n) &&
         n2d_download2d(matrix, ld * CPX, wide, n * CPX, n * CPX, n) && n2d_download(pivots, piv, n * sizeof(int));
    n2d_free(wide);
    if(!ok) { n2d_free_async(f.lu32); n2d_free(a); n2d_free(piv); return 0; }
    g_cache.host = matrix; g_cache.order = n; g_cache.ld = ld; g_cache.piv_dev = piv; g_cache.mixed = 1;
    g_cache.lu32_dev = f.lu32; g_cache.ld32 = f.ld32; g_cache.orig_dev = a; g_cache.anorm = f.anorm;
    return 1;
  }
  ok = n2d_lu_factor(a, (long long)n, (long long)n, piv, 0, 0, &info);
  ok = ok && n2d_download2d(matrix, ld * CPX, a, n * CPX, n * CPX, n) &&
       n2d_download(pivots, piv, n * sizeof(int));
  if(!ok || info) { n2d_free(a); n2d_free(piv); if(ok && info) n2c_set_error("matrix is singular (pivot %d)", info); return 0; }
  g_cache.host = matrix; g_cache.order = n; g_cache.ld = ld;
  g_cache.lu_dev = a; g_cache.piv_dev = piv; g_cache.mixed = 0;
  return 1;
}

int nec2c_cuda_dense_solve_classic_many(size_t n, const nec2c_cuda_complex *matrix, size_t ld,
                                        const int *pivots, nec2c_cuda_complex *rhs, size_t stride,
                                        size_t count)
{
  double *lu = NULL, *b = NULL;
  int *piv = NULL, own = 0, ok;
  if(count == 0) return 1;
  if(!matrix || !pivots || !rhs || n == 0 || n > INT_MAX || ld < n || ld > INT_MAX || stride < n ||
     count > INT_MAX) {
    n2c_set_error("solve: null matrix, pivots or rhs, order 0, or a leading dimension or stride below the order");
    return 0;
  }
  if(!n2d_device_ok()) return 0;
  const int cached = g_cache.piv_dev && g_cache.host == (const void *)matrix && g_cache.order == n && g_cache.ld == ld;
  b = n2d_alloc(n * count * CPX);
  if(!b || !n2d_upload2d(b, n * CPX, rhs, stride * CPX, n * CPX, count)) { n2d_free(b); return 0; }
  if(cached && g_cache.mixed) {
    split_factors f = {g_cache.lu32_dev, g_cache.ld32, g_cache.piv_dev, g_cache.orig_dev, g_cache.anorm};
    ok = solve_refined(n, &f, b, count, &g_last_refinement) &&
         n2d_download2d(rhs, stride * CPX, b, n * CPX, n * CPX, count);
    n2d_free(b);
    return ok;
  }
  if(cached) {
    lu = g_cache.lu_dev; piv = g_cache.piv_dev;
  } else {
    /* Factors produced earlier (or in another process): upload them as
       stored.  Split-precision factors solved this way carry FP32 accuracy. */
    own = 1;
    lu = n2d_alloc(n * n * CPX);
    piv = n2d_alloc(n * sizeof(int));
    if(!lu || !piv || !n2d_upload2d(lu, n * CPX, matrix, ld * CPX, n * CPX, n) ||
       !n2d_upload(piv, pivots, n * sizeof(int))) { n2d_free(lu); n2d_free(piv); n2d_free(b); return 0; }
  }
  ok = n2d_lu_solve(lu, (long long)n, (long long)n, piv, b, (long long)n, (long long)count) &&
       n2d_download2d(rhs, stride * CPX, b, n * CPX, n * CPX, count);
  n2d_free(b);
  if(own) { n2d_free(lu); n2d_free(piv); }
  return ok;
}

int nec2c_cuda_dense_solve_classic(size_t n, const nec2c_cuda_complex *matrix, size_t ld, const int *pivots,
                                   nec2c_cuda_complex *rhs)
{
  return nec2c_cuda_dense_solve_classic_many(n, matrix, ld, pivots, rhs, n, 1);
}

int nec2c_cuda_dense_solve_row_major(nec2c_cuda_complex *matrix, nec2c_cuda_complex *rhs, size_t n)
{
  double *a, *b = NULL;
  int *piv = NULL, info = 0, ok;
  if(!matrix || !rhs || n == 0 || n > INT_MAX) { n2c_set_error("row-major solve: null matrix or rhs, or order 0"); return 0; }
  if(!n2d_device_ok()) return 0;
  /* The row-major system is the classic storage with leading dimension n. */
  a = upload_matrix(matrix, n, n);
  if(!a) return 0;
  piv = n2d_alloc(n * sizeof(int));
  b = n2d_alloc(n * CPX);
  ok = piv && b && n2d_upload(b, rhs, n * CPX) &&
       n2d_lu_factor(a, (long long)n, (long long)n, piv, 1, 0, &info);
  if(ok && info) { n2c_set_error("pivot %d below 64 eps", info); ok = 0; }
  ok = ok && n2d_lu_solve(a, (long long)n, (long long)n, piv, b, (long long)n, 1) &&
       n2d_download(rhs, b, n * CPX);
  n2d_free(a); n2d_free(b); n2d_free(piv);
  return ok;
}

/* Ragged batch of small systems (orders <= 64) in one launch: factored in
   place (factr's pivots and factors, as nec2c_cuda_dense_factor_classic
   writes them) and solved for one right-hand side each.  Larger orders go
   through the classic factor and solve one after another. */
int nec2c_cuda_dense_solve_batched(size_t count, const size_t *orders, nec2c_cuda_complex *const *matrices,
                                   const size_t *lds, int *const *pivots, nec2c_cuda_complex *const *rhs,
                                   int *status)
{
  size_t i, small = 0, a_total = 0, b_total = 0;
  int all = 1, ok = 1;
  int *order32 = NULL, *info = NULL, *piv_host = NULL;
  double complex *a_host = NULL, *b_host = NULL;
  double *a_dev = NULL, *b_dev = NULL;
  int *piv_dev = NULL, *info_dev = NULL;
  void *desc_dev = NULL;
  if(count == 0) return 1;
  if(!orders || !matrices || !lds || !rhs || !status) return 0;
  if(!n2d_device_ok()) return 0;
  for(i = 0; i < count; ++i) {
    if(orders[i] == 0 || !matrices[i] || !rhs[i] || lds[i] < orders[i]) { n2c_set_error("invalid system %zu", i); return 0; }
    status[i] = 0;
    if(orders[i] <= 64) { small++; a_total += orders[i] * orders[i]; b_total += orders[i]; }
  }
  if(small) {
    size_t k = 0, ao = 0, bo = 0;
    order32 = malloc(small * sizeof(int));
    info = calloc(small, sizeof(int));
    piv_host = malloc(b_total * sizeof(int));
    a_host = malloc(a_total * sizeof(double complex));
    b_host = malloc(b_total * sizeof(double complex));
    ok = order32 && info && piv_host && a_host && b_host;
    for(i = 0; ok && i < count; ++i) {
      const size_t n = orders[i];
      size_t r;
      if(n > 64) continue;
      order32[k++] = (int)n;
      /* NEC storage column r is algebraic row r: copy the first n entries. */
      for(r = 0; r < n; ++r) memcpy(a_host + ao + r * n, matrices[i] + r * lds[i], n * sizeof(double complex));
      memcpy(b_host + bo, rhs[i], n * sizeof(double complex));
      ao += n * n;
      bo += n;
    }
    a_dev = ok ? n2d_alloc_async(a_total * CPX) : NULL;
    b_dev = ok ? n2d_alloc_async(b_total * CPX) : NULL;
    piv_dev = ok ? n2d_alloc_async(b_total * sizeof(int)) : NULL;
    info_dev = ok ? n2d_alloc_async(small * sizeof(int)) : NULL;
    desc_dev = ok ? n2d_alloc_async(n2d_lu_batched_descriptor_bytes((long long)small)) : NULL;
    ok = ok && a_dev && b_dev && piv_dev && info_dev && desc_dev &&
         n2d_upload(a_dev, a_host, a_total * CPX) && n2d_upload(b_dev, b_host, b_total * CPX) &&
         n2d_memset(info_dev, 0, small * sizeof(int)) &&
         n2d_lu_batched(a_dev, b_dev, piv_dev, order32, (long long)small, info_dev, desc_dev) &&
         n2d_download(a_host, a_dev, a_total * CPX) && n2d_download(b_host, b_dev, b_total * CPX) &&
         n2d_download(piv_host, piv_dev, b_total * sizeof(int)) && n2d_download(info, info_dev, small * sizeof(int));
    for(i = 0, k = 0, ao = 0, bo = 0; ok && i < count; ++i) {
      const size_t n = orders[i];
      size_t r;
      if(n > 64) continue;
      for(r = 0; r < n; ++r) memcpy(matrices[i] + r * lds[i], a_host + ao + r * n, n * sizeof(double complex));
      memcpy(rhs[i], b_host + bo, n * sizeof(double complex));
      if(pivots && pivots[i]) memcpy(pivots[i], piv_host + bo, n * sizeof(int));
      status[i] = info[k] == 0;
      if(!status[i]) all = 0;
      ao += n * n;
      bo += n;
      k++;
    }
    n2d_free_async(a_dev); n2d_free_async(b_dev); n2d_free_async(piv_dev); n2d_free_async(info_dev);
    n2d_free_async(desc_dev);
    free(order32); free(info); free(piv_host); free(a_host); free(b_host);
    if(!ok) return 0;
  }
  for(i = 0; i < count; ++i) {
    int *p;
    if(orders[i] <= 64) continue;
    p = (pivots && pivots[i]) ? pivots[i] : malloc(orders[i] * sizeof(int));
    status[i] = p && nec2c_cuda_dense_factor_classic(orders[i], matrices[i], lds[i], p) &&
                nec2c_cuda_dense_solve_classic(orders[i], matrices[i], lds[i], p, rhs[i]);
    if(!(pivots && pivots[i])) free(p);
    if(!status[i]) all = 0;
  }
  return all;
}

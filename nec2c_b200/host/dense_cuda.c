/* Host side of the CUDA dense backend: dense_backend.c's classic factor/solve
 * and row-major solve entry points (C, like the reference).  The factor keeps
 * its device copy (and, for the mixed form, the original matrix) so the
 * solves that follow in the same process do not re-upload it. */
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
  if(!name) return 0;
  if(!strcmp(name, "cuda")) g_dense_mixed = 0;
  else if(!strcmp(name, "cuda-mixed")) g_dense_mixed = 1;
  else return 0;
  return 1;
}
const char *nec2c_cuda_dense_backend_name(void) { return g_dense_mixed ? "cuda-mixed" : "cuda"; }

/* The most recent classic factorisation, kept on the device. */
static struct {
  const void *host;      /* host matrix the factors were written to */
  size_t order, ld;
  double *lu_dev;        /* column-major LU, leading dimension order */
  int *piv_dev;
  double *orig_dev;      /* mixed form: the unfactored matrix (for refinement) */
  int mixed;
} g_cache;

void nec2c_cuda_dense_release(void)
{
  n2d_free(g_cache.lu_dev); n2d_free(g_cache.piv_dev); n2d_free(g_cache.orig_dev);
  memset(&g_cache, 0, sizeof(g_cache));
}

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

int nec2c_cuda_dense_factor_classic(size_t n, nec2c_cuda_complex *matrix, size_t ld, int *pivots)
{
  int info = 0, ok;
  double *a, *orig = NULL;
  int *piv;
  if(!matrix || !pivots || n == 0 || n > INT_MAX || ld < n || ld > INT_MAX) return 0;
  if(!n2d_device_ok()) return 0;
  nec2c_cuda_dense_release();
  a = upload_matrix(matrix, n, ld);
  piv = n2d_alloc(n * sizeof(int));
  if(!a || !piv) { n2d_free(a); n2d_free(piv); return 0; }
  if(g_dense_mixed) {
    orig = n2d_alloc(n * n * CPX);
    if(!orig || !n2d_copy_d2d(orig, a, n * n * CPX)) { n2d_free(a); n2d_free(piv); n2d_free(orig); return 0; }
  }
  ok = n2d_lu_factor(a, (long long)n, (long long)n, piv, 0, g_dense_mixed, &info);
  ok = ok && n2d_download2d(matrix, ld * CPX, a, n * CPX, n * CPX, n) &&
       n2d_download(pivots, piv, n * sizeof(int));
  if(!ok || info) { n2d_free(a); n2d_free(piv); n2d_free(orig); if(ok && info) n2c_set_error("matrix is singular (pivot %d)", info); return 0; }
  g_cache.host = matrix; g_cache.order = n; g_cache.ld = ld;
  g_cache.lu_dev = a; g_cache.piv_dev = piv; g_cache.orig_dev = orig; g_cache.mixed = g_dense_mixed;
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
     count > INT_MAX) return 0;
  if(!n2d_device_ok()) return 0;
  if(g_cache.lu_dev && g_cache.host == (const void *)matrix && g_cache.order == n && g_cache.ld == ld) {
    lu = g_cache.lu_dev; piv = g_cache.piv_dev;
  } else {
    /* Factors produced earlier (or in another process): upload them as stored. */
    own = 1;
    lu = n2d_alloc(n * n * CPX);
    piv = n2d_alloc(n * sizeof(int));
    if(!lu || !piv || !n2d_upload2d(lu, n * CPX, matrix, ld * CPX, n * CPX, n) ||
       !n2d_upload(piv, pivots, n * sizeof(int))) { n2d_free(lu); n2d_free(piv); return 0; }
  }
  b = n2d_alloc(n * count * CPX);
  ok = b && n2d_upload2d(b, n * CPX, rhs, stride * CPX, n * CPX, count) &&
       n2d_lu_solve(lu, (long long)n, (long long)n, piv, b, (long long)n, (long long)count) &&
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
  if(!matrix || !rhs || n == 0 || n > INT_MAX) return 0;
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

/* Host side of the CUDA dense backend: dense_backend.c's classic factor/solve
 * and row-major solve entry points (C, like the reference).  Each factor
 * keeps its device copy (and, for the mixed form, the original matrix) so the
 * solves that follow on the same thread do not re-upload it.  The entries are
 * per thread, since threads that each own a stream (the request server) work
 * independently. */
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

/* Classic factorisations of this thread kept on the device: one entry per
   host storage the factors were written to, so that the solves that follow
   find them whatever the order of calls (netwk factors its network matrix
   between the main matrix's factor and solves, network.c:505-560; factrs
   factors every symmetry block before solves uses them, matrix.c:1424-1435
   and 1683-1701).  An entry is recognised by the storage address, order and
   leading dimension, and checked against the pivots and the diagonal of the
   factors written back; a factorisation written over an entry's storage
   replaces it. */
typedef struct dense_entry {
  struct dense_entry *next;
  const void *host;      /* host storage the factors were written to */
  size_t order, ld;
  double *lu_dev;        /* FP64 form: row-major LU, leading dim order */
  int *piv_dev;
  float *lu32_dev;       /* split form: FP32 LU, leading dim ld32 (even) */
  size_t ld32;
  double *orig_dev;      /* split form: the FP64 matrix (refinement residuals) */
  double anorm;          /* split form: its infinity norm */
  int mixed;
  int *piv_host;         /* pivots and diagonal written back (recognition) */
  nec2c_cuda_complex *diag_host;
  size_t bytes;          /* device bytes held */
  unsigned long long stamp;
} dense_entry;

static _Thread_local dense_entry *g_entries = NULL;
static _Thread_local size_t g_entry_bytes = 0;
static _Thread_local unsigned long long g_entry_clock = 0;
static _Thread_local int g_last_refinement = 0;

static void entry_free(dense_entry *e)
{
  n2d_free(e->lu_dev); n2d_free(e->piv_dev); n2d_free_async(e->lu32_dev); n2d_free(e->orig_dev);
  free(e->piv_host); free(e->diag_host);
  g_entry_bytes -= e->bytes;
  free(e);
}

/* Unlinks and frees every entry for which drop(e, ctx) holds. */
static void entries_drop(int (*drop)(const dense_entry *, const void *), const void *ctx)
{
  dense_entry **pp = &g_entries;
  while(*pp) {
    dense_entry *e = *pp;
    if(drop(e, ctx)) { *pp = e->next; entry_free(e); }
    else pp = &e->next;
  }
}

static int drop_all(const dense_entry *e, const void *ctx) { (void)e; (void)ctx; return 1; }

/* Storage of a factorisation: n columns of n entries, ld apart (NEC's
   transposed storage; factrs's symmetry blocks are row blocks of one matrix,
   matrix.c:1424-1435, so their columns interleave without overlapping). */
typedef struct { const char *base; size_t n, ld; } host_block;

/* 1 when block b (offset d >= 0 elements after a, same leading dimension)
   shares an entry with a. */
static int blocks_overlap_after(size_t d, size_t na, size_t nb, size_t ld)
{
  const size_t q = d / ld, r = d % ld;
  /* b's column j starts at row r of a's column q + j and, when r + nb > ld,
     runs on into a's column q + j + 1 from row 0. */
  if(r < na && q < na) return 1;
  if(r + nb > ld && q + 1 < na) return 1;
  return 0;
}

static int blocks_overlap(const host_block *a, const host_block *b)
{
  const size_t cpx = 2 * sizeof(double);
  const char *alo = a->base, *ahi = alo + ((a->ld * (a->n - 1)) + a->n) * cpx;
  const char *blo = b->base, *bhi = blo + ((b->ld * (b->n - 1)) + b->n) * cpx;
  if(!(alo < bhi && blo < ahi)) return 0;
  if(a->ld != b->ld || ((size_t)(blo > alo ? blo - alo : alo - blo)) % cpx) return 1;  /* conservative */
  if(blo >= alo) return blocks_overlap_after((size_t)(blo - alo) / cpx, a->n, b->n, a->ld);
  return blocks_overlap_after((size_t)(alo - blo) / cpx, b->n, a->n, a->ld);
}

static int drop_overlap(const dense_entry *e, const void *ctx)
{
  const host_block mine = {(const char *)e->host, e->order, e->ld};
  return blocks_overlap(&mine, (const host_block *)ctx);
}

static _Thread_local const dense_entry *g_victim;
static int drop_victim(const dense_entry *e, const void *ctx) { (void)ctx; return e == g_victim; }

void nec2c_cuda_dense_release(void)
{
  entries_drop(drop_all, NULL);
}

int nec2c_cuda_dense_last_refinement(void) { return g_last_refinement; }

/* Keeps the entries of this thread within a quarter of the device's memory,
   dropping the least recently used first (their FP64 factors are uploaded
   again from the host storage when solved; split-precision ones must be
   factored again). */
static void entries_trim(size_t incoming)
{
  size_t free_b = 0, total_b = 0;
  if(!n2d_mem_info(&free_b, &total_b) || total_b == 0) return;
  while(g_entries && g_entry_bytes + incoming > total_b / 4) {
    dense_entry *e, *lru = g_entries;
    for(e = g_entries; e; e = e->next) if(e->stamp < lru->stamp) lru = e;
    g_victim = lru;
    entries_drop(drop_victim, NULL);
  }
}

/* The entry whose factors the host storage holds, or NULL (a stale entry for
   the same storage is dropped). */
static dense_entry *entry_find(const void *matrix, size_t n, size_t ld, const int *pivots)
{
  dense_entry *e;
  for(e = g_entries; e; e = e->next) {
    if(e->host == matrix && e->order == n && e->ld == ld) {
      const nec2c_cuda_complex *m = matrix;
      size_t i;
      int same = !memcmp(e->piv_host, pivots, n * sizeof(int));
      for(i = 0; same && i < n; ++i) same = m[i * ld + i] == e->diag_host[i];
      if(same) { e->stamp = ++g_entry_clock; return e; }
      g_victim = e;
      entries_drop(drop_victim, NULL);
      return NULL;
    }
  }
  return NULL;
}

/* Records a factorisation just written back to the host storage. */
static int entry_add(dense_entry *proto, const nec2c_cuda_complex *matrix, const int *pivots)
{
  size_t i;
  const size_t n = proto->order, ld = proto->ld;
  dense_entry *e = malloc(sizeof(*e));
  if(!e) { n2c_set_error("host allocation failed"); return 0; }
  *e = *proto;
  e->piv_host = malloc(n * sizeof(int));
  e->diag_host = malloc(n * sizeof(nec2c_cuda_complex));
  if(!e->piv_host || !e->diag_host) {
    free(e->piv_host); free(e->diag_host); free(e);
    n2c_set_error("host allocation failed");
    return 0;
  }
  memcpy(e->piv_host, pivots, n * sizeof(int));
  for(i = 0; i < n; ++i) e->diag_host[i] = matrix[i * ld + i];
  e->stamp = ++g_entry_clock;
  e->next = g_entries;
  g_entries = e;
  g_entry_bytes += e->bytes;
  return 1;
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
  {
    /* Factors written over an entry's storage replace it. */
    const host_block blk = {(const char *)matrix, n, ld};
    entries_drop(drop_overlap, &blk);
  }
  entries_trim(n * n * CPX * (g_dense_mixed ? 2 : 1));
  a = upload_matrix(matrix, n, ld);
  piv = n2d_alloc(n * sizeof(int));
  if(!a || !piv) { n2d_free(a); n2d_free(piv); return 0; }
  dense_entry proto;
  memset(&proto, 0, sizeof(proto));
  proto.host = matrix; proto.order = n; proto.ld = ld; proto.piv_dev = piv;
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
    proto.mixed = 1; proto.lu32_dev = f.lu32; proto.ld32 = f.ld32; proto.orig_dev = a; proto.anorm = f.anorm;
    proto.bytes = n * n * CPX + n * f.ld32 * 2 * sizeof(float) + n * sizeof(int);
    if(!entry_add(&proto, matrix, pivots)) { n2d_free_async(f.lu32); n2d_free(a); n2d_free(piv); return 0; }
    return 1;
  }
  ok = n2d_lu_factor(a, (long long)n, (long long)n, piv, 0, 0, &info);
  ok = ok && n2d_download2d(matrix, ld * CPX, a, n * CPX, n * CPX, n) &&
       n2d_download(pivots, piv, n * sizeof(int));
  if(!ok || info) { n2d_free(a); n2d_free(piv); if(ok && info) n2c_set_error("matrix is singular (pivot %d)", info); return 0; }
  proto.lu_dev = a; proto.bytes = n * n * CPX + n * sizeof(int);
  if(!entry_add(&proto, matrix, pivots)) { n2d_free(a); n2d_free(piv); return 0; }
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
  const dense_entry *e = entry_find(matrix, n, ld, pivots);
  if(!e && g_dense_mixed) {
    /* Split-precision factors carry FP32 accuracy; only the refinement
       against the FP64 matrix, which lives with the entry, gives the FP64
       answer.  Without it the solve is refused rather than returned at FP32
       accuracy. */
    n2c_set_error("solve: the split-precision factors of this matrix are not on the device (factored in another "
                  "thread or process, released, or overwritten); factor it again");
    return 0;
  }
  b = n2d_alloc(n * count * CPX);
  if(!b || !n2d_upload2d(b, n * CPX, rhs, stride * CPX, n * CPX, count)) { n2d_free(b); return 0; }
  if(e && e->mixed) {
    split_factors f = {e->lu32_dev, e->ld32, e->piv_dev, e->orig_dev, e->anorm};
    ok = solve_refined(n, &f, b, count, &g_last_refinement) &&
         n2d_download2d(rhs, stride * CPX, b, n * CPX, n * CPX, count);
    n2d_free(b);
    return ok;
  }
  if(e) {
    lu = e->lu_dev; piv = e->piv_dev;
  } else {
    /* FP64 factors produced earlier (in another thread or process, or
       dropped from the device): upload them as stored. */
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
size_t nec2c_cuda_dense_batch_max_order(void)
{
  const long long m = n2d_device_ok() ? n2d_lu_batch_max_order() : 0;
  return m > 0 ? (size_t)m : 0;
}

/* Lockstep batch (FP64 form): count systems in NEC storage on the host are
   uploaded, factored together by n2d_lu_factor_batch and solved together by
   n2d_lu_solve_batch on this thread's stream.  rhs_count[i] right-hand sides
   of rhs[i] (stride[i]) receive the solutions; factors / pivots (either may
   be NULL, or hold NULL entries) receive the factors in NEC storage as
   nec2c_cuda_dense_factor_classic writes them, and the 1-based pivots.
   status[i] is 1 when system i was solved, 0 when it is singular.  Returns 0
   (error set) when the device work itself failed. */
static int lockstep_batch(size_t count, const size_t *order, const nec2c_cuda_complex *const *matrix,
                          const size_t *ld, nec2c_cuda_complex *const *factors, int *const *pivots,
                          nec2c_cuda_complex *const *rhs, const size_t *stride, const size_t *rhs_count, int *status)
{
  double **a = calloc(count, sizeof(*a)), **b = calloc(count, sizeof(*b));
  int **piv = calloc(count, sizeof(*piv)), *info = calloc(count, sizeof(int));
  long long *n = calloc(count, sizeof(long long)), *nr = calloc(count, sizeof(long long));
  size_t i;
  int ok = a && b && piv && info && n && nr;
  if(!ok) n2c_set_error("batched solve: out of host memory");
  for(i = 0; ok && i < count; ++i) {
    const size_t k = order[i];
    status[i] = 0;
    n[i] = (long long)k;
    a[i] = n2d_alloc_async(k * k * CPX);
    b[i] = n2d_alloc_async(k * (rhs_count[i] ? rhs_count[i] : 1) * CPX);
    piv[i] = n2d_alloc_async(k * sizeof(int));
    ok = a[i] && b[i] && piv[i] && n2d_upload2d(a[i], k * CPX, matrix[i], ld[i] * CPX, k * CPX, k) &&
         n2d_upload2d(b[i], k * CPX, rhs[i], stride[i] * CPX, k * CPX, rhs_count[i]);
  }
  ok = ok && n2d_lu_factor_batch(a, n, n, piv, (int)count, 0, info);
  /* Singular systems take no part in the solve. */
  for(i = 0; ok && i < count; ++i) nr[i] = info[i] ? 0 : (long long)rhs_count[i];
  ok = ok && n2d_lu_solve_batch((const double *const *)a, n, n, (const int *const *)piv, b, n, nr, (int)count);
  for(i = 0; ok && i < count; ++i) {
    const size_t k = order[i];
    if(factors && factors[i])
      ok = n2d_download2d(factors[i], ld[i] * CPX, a[i], k * CPX, k * CPX, k);
    if(ok && pivots && pivots[i]) ok = n2d_download(pivots[i], piv[i], k * sizeof(int));
    if(ok && !info[i]) ok = n2d_download2d(rhs[i], stride[i] * CPX, b[i], k * CPX, k * CPX, rhs_count[i]);
    if(ok) status[i] = info[i] == 0;
  }
  if(ok) n2d_sync();
  for(i = 0; a && b && piv && i < count; ++i) { n2d_free_async(a[i]); n2d_free_async(b[i]); n2d_free_async(piv[i]); }
  free(a); free(b); free(piv); free(info); free(n); free(nr);
  return ok;
}

/* The split-precision lockstep batch (the server's merged dense run on a
   split-precision server): each system's FP64 matrix uploaded and kept for the
   refinement residuals, narrowed to FP32 (even leading dimension), the FP32
   copies factored together by n2d_lu_factor32_batch (tensor-core updates),
   then solve_refined's iteration for every system at once: one batched FP32
   solve per step, each system's correction and FP64 residual, one read of all
   the norms, and the systems that meet solve_refined's test leave the loop.
   A system not converged in 30 steps is solved by an FP64 factorisation of
   its original, as solve_refined does.  steps[i] receives its step count
   (-1: the FP64 fallback). */
static int lockstep_batch_split(size_t count, const size_t *order, const nec2c_cuda_complex *const *matrix,
                                const size_t *ld, nec2c_cuda_complex *const *rhs, const size_t *stride,
                                const size_t *rhs_count, int *status, int *steps)
{
  double **a = calloc(count, sizeof(*a)), **b = calloc(count, sizeof(*b)), **x = calloc(count, sizeof(*x));
  double **r = calloc(count, sizeof(*r)), **d = calloc(count, sizeof(*d)), *anorm = calloc(count, sizeof(double));
  float **lu = calloc(count, sizeof(*lu));
  int **piv = calloc(count, sizeof(*piv)), *info = calloc(count, sizeof(int)), *live = calloc(count, sizeof(int));
  long long *n = calloc(count, sizeof(long long)), *ld32 = calloc(count, sizeof(long long));
  long long *nr = calloc(count, sizeof(long long));
  size_t *noff = calloc(count, sizeof(size_t)), ntot = 0, i;
  double *norms = NULL;
  unsigned long long *norm_dev = NULL;
  int ok = a && b && x && r && d && anorm && lu && piv && info && live && n && ld32 && nr && noff, it, left;
  if(!ok) n2c_set_error("batched solve: out of host memory");
  for(i = 0; ok && i < count; ++i) {
    const size_t k = order[i], c = rhs_count[i];
    status[i] = 0; steps[i] = 0;
    n[i] = (long long)k; ld32[i] = (long long)(k + (k & 1));
    noff[i] = ntot; ntot += 2 * c;
    a[i] = n2d_alloc_async(k * k * CPX);
    lu[i] = n2d_alloc_async(k * (size_t)ld32[i] * 2 * sizeof(float));
    piv[i] = n2d_alloc_async(k * sizeof(int));
    b[i] = n2d_alloc_async(k * c * CPX); x[i] = n2d_alloc_async(k * c * CPX);
    r[i] = n2d_alloc_async(k * c * CPX); d[i] = n2d_alloc_async(k * c * CPX);
    ok = a[i] && lu[i] && piv[i] && b[i] && x[i] && r[i] && d[i] &&
         n2d_upload2d(a[i], k * CPX, matrix[i], ld[i] * CPX, k * CPX, k) &&
         n2d_upload2d(b[i], k * CPX, rhs[i], stride[i] * CPX, k * CPX, c) &&
         n2d_narrow(a[i], n[i], lu[i], ld32[i], n[i], n[i]);
  }
  norm_dev = ok ? n2d_alloc_async((ntot > count ? ntot : count) * sizeof(unsigned long long)) : NULL;
  norms = ok ? malloc(ntot * sizeof(double)) : NULL;
  ok = ok && norm_dev && norms;
  /* Every system's ||A||_inf into its own slot, one read for all. */
  for(i = 0; ok && i < count; ++i)
    ok = n2d_norm_inf(a[i], n[i], n[i], (unsigned long long *)norm_dev + noff[i], NULL);
  ok = ok && n2d_read_norms(norm_dev, (long long)ntot, norms);
  for(i = 0; ok && i < count; ++i) anorm[i] = norms[noff[i]];
  ok = ok && n2d_lu_factor32_batch(lu, n, ld32, piv, (int)count, 0, info);
  for(i = 0, left = 0; ok && i < count; ++i) {
    live[i] = !info[i];   /* singular systems take no part */
    left += live[i];
    ok = n2d_memset(x[i], 0, order[i] * rhs_count[i] * CPX) && n2d_copy_d2d(r[i], b[i], order[i] * rhs_count[i] * CPX);
  }
  for(it = 1; ok && it <= 30 && left; ++it) {
    for(i = 0; ok && i < count; ++i) {
      nr[i] = live[i] ? (long long)rhs_count[i] : 0;
      if(live[i]) ok = n2d_copy_d2d(d[i], r[i], order[i] * rhs_count[i] * CPX);
    }
    ok = ok && n2d_lu_solve32_batch((const float *const *)lu, n, ld32, (const int *const *)piv, d, n, nr, (int)count);
    for(i = 0; ok && i < count; ++i) {
      const long long K = (long long)rhs_count[i];
      if(!live[i]) continue;
      ok = n2d_add_correction(x[i], d[i], n[i], K, n[i], norm_dev + noff[i] + rhs_count[i], NULL) &&
           n2d_residual(a[i], n[i], n[i], x[i], b[i], r[i], K, n[i], norm_dev + noff[i], NULL);
    }
    ok = ok && n2d_read_norms(norm_dev, (long long)ntot, norms);
    for(i = 0; ok && i < count; ++i) {
      const double cte = anorm[i] * DBL_EPSILON * sqrt((double)order[i]);
      size_t j;
      int done = live[i];
      if(!live[i]) continue;
      for(j = 0; j < rhs_count[i]; ++j)
        if(!(norms[noff[i] + j] <= norms[noff[i] + rhs_count[i] + j] * cte)) done = 0;
      if(done) { live[i] = 0; left--; steps[i] = it; status[i] = 1; }
    }
  }
  /* Not converged in 30 steps: an FP64 factorisation of the original. */
  for(i = 0; ok && i < count; ++i) {
    const size_t k = order[i], c = rhs_count[i];
    int inf = 0;
    if(!live[i]) continue;
    ok = n2d_lu_factor(a[i], n[i], n[i], piv[i], 0, 0, &inf) && n2d_copy_d2d(x[i], b[i], k * c * CPX) &&
         (inf || n2d_lu_solve(a[i], n[i], n[i], piv[i], x[i], n[i], (long long)c));
    status[i] = ok && !inf;
    steps[i] = -1;
  }
  for(i = 0; ok && i < count; ++i)
    if(status[i]) ok = n2d_download2d(rhs[i], stride[i] * CPX, x[i], order[i] * CPX, order[i] * CPX, rhs_count[i]);
  if(ok) n2d_sync();
  for(i = 0; a && b && x && r && d && lu && piv && i < count; ++i) {
    n2d_free_async(a[i]); n2d_free_async(lu[i]); n2d_free_async(piv[i]);
    n2d_free_async(b[i]); n2d_free_async(x[i]); n2d_free_async(r[i]); n2d_free_async(d[i]);
  }
  n2d_free_async(norm_dev);
  free(a); free(b); free(x); free(r); free(d); free(anorm); free(lu); free(piv); free(info); free(live);
  free(n); free(ld32); free(nr); free(noff); free(norms);
  return ok;
}

/* The request server's merged dense run: the private copies of count
   requests' matrices factored and solved as one lockstep batch, in the FP64
   form or (split) the split-precision form with FP64 refinement. */
int n2c_dense_solve_private_batch(size_t count, const size_t *order, const nec2c_cuda_complex *const *matrix,
                                  const size_t *ld, nec2c_cuda_complex *const *rhs, const size_t *stride,
                                  const size_t *rhs_count, int split, int *status, int *steps)
{
  size_t i;
  for(i = 0; i < count; ++i) {
    status[i] = 0;
    if(!matrix[i] || !rhs[i] || order[i] == 0 || (long long)order[i] > n2d_lu_batch_max_order() || ld[i] < order[i] ||
       stride[i] < order[i] || rhs_count[i] == 0 || rhs_count[i] > 65535) {
      n2c_set_error("merged dense run: invalid request %zu", i);
      return 0;
    }
  }
  if(split) return lockstep_batch_split(count, order, matrix, ld, rhs, stride, rhs_count, status, steps);
  for(i = 0; i < count; ++i) steps[i] = 0;
  return lockstep_batch(count, order, matrix, ld, NULL, NULL, rhs, stride, rhs_count, status);
}

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
  /* FP64 form: the larger systems up to the batch limit in one lockstep
     batch (one launch per kernel and panel step for all of them). */
  if(!g_dense_mixed) {
    size_t k = 0, j;
    const long long cap = n2d_lu_batch_max_order();
    size_t *ord = malloc(count * sizeof(size_t)), *ldv = malloc(count * sizeof(size_t)), *one = malloc(count * sizeof(size_t));
    size_t *idx = malloc(count * sizeof(size_t));
    const nec2c_cuda_complex **mat = malloc(count * sizeof(*mat));
    nec2c_cuda_complex **fac = malloc(count * sizeof(*fac)), **rv = malloc(count * sizeof(*rv));
    int **pv = malloc(count * sizeof(*pv)), *st = malloc(count * sizeof(int));
    ok = ord && ldv && one && idx && mat && fac && rv && pv && st;
    for(i = 0; ok && i < count; ++i) {
      if(orders[i] <= 64 || (long long)orders[i] > cap) continue;
      {
        /* Factors written over an entry's storage replace it. */
        const host_block blk = {(const char *)matrices[i], orders[i], lds[i]};
        entries_drop(drop_overlap, &blk);
      }
      idx[k] = i; ord[k] = orders[i]; ldv[k] = lds[i]; one[k] = 1;
      mat[k] = matrices[i]; fac[k] = matrices[i]; rv[k] = rhs[i]; pv[k] = pivots ? pivots[i] : NULL;
      k++;
    }
    ok = ok && (k == 0 || lockstep_batch(k, ord, mat, ldv, fac, pv, rv, ord, one, st));
    for(j = 0; ok && j < k; ++j) {
      status[idx[j]] = st[j];
      if(!st[j]) all = 0;
    }
    free(ord); free(ldv); free(one); free(idx); free(mat); free(fac); free(rv); free(pv); free(st);
    if(!ok) return 0;
  }
  for(i = 0; i < count; ++i) {
    int *p;
    if(orders[i] <= 64 || (!g_dense_mixed && (long long)orders[i] <= n2d_lu_batch_max_order())) continue;
    p = (pivots && pivots[i]) ? pivots[i] : malloc(orders[i] * sizeof(int));
    status[i] = p && nec2c_cuda_dense_factor_classic(orders[i], matrices[i], lds[i], p) &&
                nec2c_cuda_dense_solve_classic(orders[i], matrices[i], lds[i], p, rhs[i]);
    if(!(pivots && pivots[i])) free(p);
    if(!status[i]) all = 0;
  }
  return all;
}

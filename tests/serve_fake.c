/* Fake device layer for testing the request server's host logic on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY.  tests/test_serve_cpu.py compiles the server's
 * own source (nec2c_b200/host/serve.c) together with this file instead of the
 * CUDA layer.  A fake solve holds the volume plans its request runs on for a
 * fixed time, counts every time a second request reaches a plan that is
 * already held, and copies b into x (x[0] of a dense request's rhs receives
 * the order), so the tests see exclusivity, concurrency and data flow without
 * a GPU.
 */
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../include/nec2c_cuda.h"
#include "../nec2c_b200/csrc/device_api.h"

struct nec2c_cuda_vie_plan {
  size_t order;
  int busy;
};
struct nec2c_cuda_hybrid {
  nec2c_cuda_vie_plan *volume;
  size_t conductors;
};
struct nec2c_cuda_vie_batch {
  size_t count, order;
  nec2c_cuda_vie_plan **plans;
  nec2c_cuda_hybrid **hybrids;   /* NULL for a batch of plans */
  size_t *offsets;
};

static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;
static int g_violations, g_running, g_peak;
static int g_merged_runs, g_merged_peak;   /* merged solves seen; most systems in one */
static int g_dense_runs, g_dense_peak, g_dense_mixed_classes;   /* lockstep dense batches */
static long g_delay_us = 2000;
static size_t g_free_bytes = (size_t)10 << 30;
static __thread char g_error[256];

/* ---- test controls ---- */
void fake_reset(long delay_us, size_t free_bytes)
{
  pthread_mutex_lock(&g_lock);
  g_violations = g_running = g_peak = 0;
  g_merged_runs = g_merged_peak = 0;
  g_dense_runs = g_dense_peak = g_dense_mixed_classes = 0;
  g_delay_us = delay_us;
  g_free_bytes = free_bytes;
  pthread_mutex_unlock(&g_lock);
}
int fake_violations(void) { return g_violations; }
int fake_peak(void) { return g_peak; }

nec2c_cuda_vie_plan *fake_plan(size_t order)
{
  nec2c_cuda_vie_plan *p = calloc(1, sizeof(*p));
  if(p) p->order = order;
  return p;
}
nec2c_cuda_hybrid *fake_hybrid(nec2c_cuda_vie_plan *volume, size_t conductors)
{
  nec2c_cuda_hybrid *h = calloc(1, sizeof(*h));
  if(h) { h->volume = volume; h->conductors = conductors; }
  return h;
}
nec2c_cuda_vie_batch *fake_batch(nec2c_cuda_vie_plan *const *plans, size_t count)
{
  nec2c_cuda_vie_batch *b = calloc(1, sizeof(*b));
  if(!b) return NULL;
  b->count = count;
  b->plans = calloc(count, sizeof(*b->plans));
  b->offsets = calloc(count + 1, sizeof(*b->offsets));
  for(size_t q = 0; q < count; ++q) {
    b->plans[q] = plans[q];
    b->offsets[q + 1] = b->offsets[q] + plans[q]->order;
  }
  b->order = b->offsets[count];
  return b;
}
nec2c_cuda_vie_batch *fake_hybrid_batch(nec2c_cuda_hybrid *const *systems, size_t count)
{
  nec2c_cuda_vie_batch *b = calloc(1, sizeof(*b));
  if(!b) return NULL;
  b->count = count;
  b->plans = calloc(count, sizeof(*b->plans));
  b->hybrids = calloc(count, sizeof(*b->hybrids));
  b->offsets = calloc(count + 1, sizeof(*b->offsets));
  for(size_t q = 0; q < count; ++q) {
    b->hybrids[q] = systems[q];
    b->plans[q] = systems[q]->volume;
    b->offsets[q + 1] = b->offsets[q] + systems[q]->conductors + systems[q]->volume->order;
  }
  b->order = b->offsets[count];
  return b;
}
void fake_release(void *p) { free(p); }

int fake_merged_runs(void) { return g_merged_runs; }
int fake_merged_peak(void) { return g_merged_peak; }

/* Holds the plans for the solve's duration; a plan already held is an
   exclusivity violation. */
static void hold(nec2c_cuda_vie_plan *const *plans, size_t count)
{
  struct timespec t = {g_delay_us / 1000000, (g_delay_us % 1000000) * 1000};
  pthread_mutex_lock(&g_lock);
  for(size_t q = 0; q < count; ++q) {
    if(plans[q]->busy) ++g_violations;
    ++plans[q]->busy;
  }
  if(++g_running > g_peak) g_peak = g_running;
  pthread_mutex_unlock(&g_lock);
  nanosleep(&t, NULL);
  pthread_mutex_lock(&g_lock);
  for(size_t q = 0; q < count; ++q) --plans[q]->busy;
  --g_running;
  pthread_mutex_unlock(&g_lock);
}

static void converged(nec2c_cuda_gmres_report *r, size_t iterations)
{
  memset(r, 0, sizeof(*r));
  r->iterations = iterations;
  r->operator_applications = iterations + 1;
  r->relative_residual = 1e-13;
}

/* ---- the device layer the server calls ---- */
void n2c_set_error(const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
}
const char *nec2c_cuda_last_error(void) { return g_error; }
int n2d_set_device(int device) { return device >= 0; }
int n2d_device_ok(void) { return 1; }
int n2d_mem_info(size_t *free_bytes, size_t *total_bytes)
{
  *free_bytes = *total_bytes = g_free_bytes;
  return 1;
}
static int g_stream_token;
void *n2d_stream_create(void) { return &g_stream_token; }
void n2d_stream_destroy(void *stream) { (void)stream; }
void n2d_set_stream(void *stream) { (void)stream; }
int n2d_sync(void) { return 1; }

int n2c_dense_solve_private(size_t n, const nec2c_cuda_complex *matrix, size_t ld, nec2c_cuda_complex *rhs,
                            size_t stride, size_t count, int split, int *steps)
{
  (void)matrix; (void)ld; (void)stride; (void)count;
  hold(NULL, 0);
  rhs[0] = (double)n;
  *steps = split ? 3 : 0;
  return 1;
}

/* Lockstep dense batches: each member's rhs[0] receives its order, and the
   batch records the size classes it mixed (a class is the power of two
   ceil(order / 256) rounded up) and its device footprint sum. */
static long long g_batch_max_order = 4096;
int fake_dense_runs(void) { return g_dense_runs; }
int fake_dense_peak(void) { return g_dense_peak; }
int fake_dense_mixed_classes(void) { return g_dense_mixed_classes; }
long long n2d_lu_batch_max_order(void) { return g_batch_max_order; }

static size_t fake_class(size_t n)
{
  size_t c = 1;
  while(c * 256 < n) c <<= 1;
  return c;
}

int n2c_dense_solve_private_batch(size_t count, const size_t *order, const nec2c_cuda_complex *const *matrix,
                                  const size_t *ld, nec2c_cuda_complex *const *rhs, const size_t *stride,
                                  const size_t *rhs_count, int split, int *status, int *steps)
{
  (void)matrix; (void)ld; (void)stride; (void)rhs_count;
  for(size_t i = 0; i < count; ++i) steps[i] = split ? 3 : 0;
  pthread_mutex_lock(&g_lock);
  ++g_dense_runs;
  if((int)count > g_dense_peak) g_dense_peak = (int)count;
  for(size_t i = 1; i < count; ++i)
    if(fake_class(order[i]) != fake_class(order[0])) ++g_dense_mixed_classes;
  pthread_mutex_unlock(&g_lock);
  hold(NULL, 0);
  for(size_t i = 0; i < count; ++i) { rhs[i][0] = (double)order[i]; status[i] = 1; }
  return 1;
}

int nec2c_cuda_gmres_plan(nec2c_cuda_vie_plan *p, const nec2c_cuda_complex *b, nec2c_cuda_complex *x,
                          const nec2c_cuda_gmres_options *options, nec2c_cuda_gmres_report *report)
{
  (void)options;
  hold(&p, 1);
  memcpy(x, b, p->order * sizeof(*x));
  converged(report, 7);
  return 1;
}

int nec2c_cuda_gmres_hybrid(nec2c_cuda_hybrid *h, const nec2c_cuda_complex *b, nec2c_cuda_complex *x,
                            const nec2c_cuda_gmres_options *options, nec2c_cuda_gmres_report *report)
{
  (void)options;
  hold(&h->volume, 1);
  memcpy(x, b, (h->conductors + h->volume->order) * sizeof(*x));
  converged(report, 9);
  return 1;
}

int nec2c_cuda_gmres_batch(nec2c_cuda_vie_batch *b, const nec2c_cuda_complex *const *bv,
                           nec2c_cuda_complex *const *xv, const nec2c_cuda_gmres_options *options,
                           nec2c_cuda_gmres_report *reports)
{
  (void)options;
  hold(b->plans, b->count);
  for(size_t q = 0; q < b->count; ++q) {
    memcpy(xv[q], bv[q], b->plans[q]->order * sizeof(*xv[q]));
    converged(&reports[q], q + 1);
  }
  return 1;
}

/* A merged solve: holds only the plans of the systems it solves, copies b
   into x for those (reports: q + 1 iterations), leaves the rest alone. */
int n2c_gmres_batch_subset(nec2c_cuda_vie_batch *b, const nec2c_cuda_complex *const *bv,
                           nec2c_cuda_complex *const *xv, const nec2c_cuda_gmres_options *options,
                           nec2c_cuda_gmres_report *reports)
{
  nec2c_cuda_vie_plan *held[64];
  size_t n = 0;
  (void)options;
  for(size_t q = 0; q < b->count; ++q)
    if(bv[q] && n < 64) held[n++] = b->plans[q];
  pthread_mutex_lock(&g_lock);
  ++g_merged_runs;
  if((int)n > g_merged_peak) g_merged_peak = (int)n;
  pthread_mutex_unlock(&g_lock);
  hold(held, n);
  for(size_t q = 0; q < b->count; ++q) {
    if(!bv[q]) { memset(&reports[q], 0, sizeof(reports[q])); reports[q].status = 4; continue; }
    memcpy(xv[q], bv[q], (b->offsets[q + 1] - b->offsets[q]) * sizeof(*xv[q]));
    converged(&reports[q], q + 1);
  }
  return 1;
}

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

size_t nec2c_cuda_vie_batch_systems(const nec2c_cuda_vie_batch *b) { return b ? b->count : 0; }
size_t nec2c_cuda_vie_batch_order(const nec2c_cuda_vie_batch *b) { return b ? b->order : 0; }
size_t nec2c_cuda_vie_batch_offset(const nec2c_cuda_vie_batch *b, size_t q)
{
  return b && q <= b->count ? b->offsets[q] : 0;
}
size_t nec2c_cuda_vie_fft_order(const nec2c_cuda_vie_plan *p) { return p ? p->order : 0; }
size_t nec2c_cuda_hybrid_order(const nec2c_cuda_hybrid *h) { return h ? h->conductors + h->volume->order : 0; }
const nec2c_cuda_vie_plan *n2c_hybrid_volume_plan(const nec2c_cuda_hybrid *h) { return h ? h->volume : NULL; }
const nec2c_cuda_vie_plan *n2c_batch_plan(const nec2c_cuda_vie_batch *b, size_t q)
{
  return b && q < b->count ? b->plans[q] : NULL;
}

/* Request server: concurrent dense MoM and volume (VIE) solves on one GPU.
 *
 * The reference runs a frequency sweep as fork()ed worker processes
 * (main.c:586-760), as many as the host's memory allows for the estimated
 * per-worker bytes (concurrency.c:118-171: usable memory = available minus a
 * reserve of max(1/5, 1 GiB), jobs = usable / worker bytes).  On the GPU the
 * workers are host threads, each owning a CUDA stream, and the memory they
 * share is device memory: a request is admitted when its device footprint
 * fits the budget left by the requests in flight, so requests that arrive
 * while others run start as soon as a worker and memory free up and their
 * work overlaps on the device.
 *
 * Dense requests factor and solve a private device copy (the split-precision
 * form with FP64 refinement when the server was created with split != 0).
 * Batch requests solve every system of a plan batch at once (a frequency
 * sweep of one model, nec2c_cuda_gmres_batch).
 * Volume requests run GMRES on a plan or hybrid system the caller created and
 * keeps on the device across requests (a frequency's spectrum is built once);
 * a plan is not reentrant (vie_fft.h:6), so two requests that run on the same
 * plan (directly, through a hybrid system or in a batch) never run at the
 * same time.  Admission is FIFO, except that a request that
 * does not fit may be passed by later ones that do, at most `slots` times
 * each before the queue waits for it.
 *
 * Continuous batching: for a batch registered with
 * nec2c_cuda_server_merge_batch, a worker that takes a volume request on one
 * of the batch's systems also takes the queued volume requests on its other
 * systems (same GMRES options) and runs them as one batched solve with the
 * remaining systems idle, so the requests that pile up while the device is
 * busy (frequencies of one model from many callers) share each launch. */
#include <errno.h>
#include <limits.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../include/nec2c_cuda.h"
#include "../csrc/device_api.h"

int n2c_dense_solve_private(size_t n, const nec2c_cuda_complex *matrix, size_t ld, nec2c_cuda_complex *rhs,
                            size_t stride, size_t count, int split, int *steps);
int n2c_dense_solve_private_batch(size_t count, const size_t *order, const nec2c_cuda_complex *const *matrix,
                                  const size_t *ld, nec2c_cuda_complex *const *rhs, const size_t *stride,
                                  const size_t *rhs_count, int split, int *status, int *steps);
const nec2c_cuda_vie_plan *n2c_hybrid_volume_plan(const nec2c_cuda_hybrid *h);
const nec2c_cuda_vie_plan *n2c_batch_plan(const nec2c_cuda_vie_batch *b, size_t q);
size_t n2c_batch_index(const nec2c_cuda_vie_batch *b, const nec2c_cuda_vie_plan *plan,
                       const nec2c_cuda_hybrid *system);
int n2c_gmres_batch_subset(nec2c_cuda_vie_batch *b, const nec2c_cuda_complex *const *bv,
                           nec2c_cuda_complex *const *xv, const nec2c_cuda_gmres_options *options,
                           nec2c_cuda_gmres_report *reports);

/* The batched GMRES restarts after at most this many steps. */
#define MERGE_MAX_RESTART 30

/* What one worker runs: a request, or (batch != NULL, n >= 2) the volume
   requests merged into one solve of that batch, member j on system index[j],
   or (dense, n >= 2) dense requests factored and solved as one lockstep
   batch. */
typedef struct {
  nec2c_cuda_request **member;
  size_t *index, n;
  nec2c_cuda_vie_batch *batch;
  int dense;
} run_t;

struct nec2c_cuda_server {
  int device, slots, split;
  size_t budget, in_use;
  pthread_mutex_t lock;
  pthread_cond_t work, done;
  nec2c_cuda_request **queue;   /* FIFO, [head, head + count) modulo cap */
  size_t head, count, cap;
  run_t *busy;                  /* in flight per worker (n == 0: idle) */
  nec2c_cuda_vie_batch **merge; /* batches whose systems' requests merge */
  size_t merges;
  size_t dense_merge;           /* most dense requests in one lockstep batch (< 2: none) */
  size_t pending;               /* submitted, not finished */
  int stop, started;
  pthread_t *threads;
};

static double now_s(void)
{
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static const size_t CPX = 2 * sizeof(double);

/* Device bytes a request holds while it runs. */
static size_t footprint(const nec2c_cuda_server *s, const nec2c_cuda_request *r)
{
  if(r->kind == NEC2C_CUDA_REQUEST_DENSE) {
    const size_t n = r->order, k = r->rhs_count;
    size_t bytes = n * n * CPX + n * k * CPX + n * sizeof(int) + 4096;
    if(s->split) bytes += n * (n + 1) * 2 * sizeof(float) + 4 * n * 2 * 32 * sizeof(float) + 3 * n * k * CPX;
    return bytes;
  }
  {
    const size_t n = r->kind == NEC2C_CUDA_REQUEST_BATCH ? nec2c_cuda_vie_batch_order(r->batch)
                     : r->plan ? nec2c_cuda_vie_fft_order(r->plan) : nec2c_cuda_hybrid_order(r->system);
    const size_t m = r->options.restart ? r->options.restart : 30;
    return (m + 4) * n * CPX + (r->kind == NEC2C_CUDA_REQUEST_BATCH ? 2 * n * CPX : 0);
  }
}

/* The volume plans a request runs on.  A hybrid system runs its plan's
 * passes on the plan's work grids, and a batch those of every system's plan
 * (one plan appears at most once in a batch), so exclusivity is per plan. */
static size_t request_plans(const nec2c_cuda_request *r)
{
  if(r->kind == NEC2C_CUDA_REQUEST_BATCH) return nec2c_cuda_vie_batch_systems(r->batch);
  return r->kind == NEC2C_CUDA_REQUEST_VOLUME ? 1 : 0;
}

static const nec2c_cuda_vie_plan *request_plan(const nec2c_cuda_request *r, size_t q)
{
  if(r->kind == NEC2C_CUDA_REQUEST_BATCH) return n2c_batch_plan(r->batch, q);
  return r->plan ? r->plan : n2c_hybrid_volume_plan(r->system);
}

/* Every system of the batch at once; the request's report summarises them. */
static int run_batch(nec2c_cuda_request *r)
{
  const size_t k = nec2c_cuda_vie_batch_systems(r->batch);
  size_t q;
  const nec2c_cuda_complex **bv;
  nec2c_cuda_complex **xv;
  int ok;
  bv = malloc((k ? k : 1) * sizeof(*bv));
  xv = malloc((k ? k : 1) * sizeof(*xv));
  if(!bv || !xv) { free(bv); free(xv); n2c_set_error("batch request: out of host memory"); return 0; }
  for(q = 0; q < k; ++q) {
    bv[q] = r->b + nec2c_cuda_vie_batch_offset(r->batch, q);
    xv[q] = r->x + nec2c_cuda_vie_batch_offset(r->batch, q);
  }
  ok = nec2c_cuda_gmres_batch(r->batch, bv, xv, &r->options, r->reports);
  r->report.status = 0;
  for(q = 0; q < k; ++q) {
    const nec2c_cuda_gmres_report *p = &r->reports[q];
    if(p->status != 0 && r->report.status == 0) r->report.status = p->status;
    if(p->iterations > r->report.iterations) r->report.iterations = p->iterations;
    if(p->restarts > r->report.restarts) r->report.restarts = p->restarts;
    r->report.operator_applications += p->operator_applications;
    if(q == 0 || p->relative_residual > r->report.relative_residual) {
      r->report.relative_residual = p->relative_residual;
      r->report.residual_norm = p->residual_norm;
    }
  }
  free(bv); free(xv);
  return ok;
}

/* True when c shares a volume plan with a request in flight. */
static int plan_busy(const nec2c_cuda_server *s, const nec2c_cuda_request *c)
{
  const size_t n = request_plans(c);
  size_t a, b, j;
  int i;
  if(n == 0) return 0;
  for(i = 0; i < s->slots; ++i)
    for(j = 0; j < s->busy[i].n; ++j) {
      const nec2c_cuda_request *r = s->busy[i].member[j];
      const size_t m = request_plans(r);
      for(a = 0; a < n; ++a)
        for(b = 0; b < m; ++b)
          if(request_plan(c, a) == request_plan(r, b)) return 1;
    }
  return 0;
}

/* True when a run in flight uses batch b's own vectors: a batch request on
   it, or volume requests merged into it. */
static int batch_busy(const nec2c_cuda_server *s, const nec2c_cuda_vie_batch *b)
{
  int i;
  for(i = 0; i < s->slots; ++i) {
    const run_t *u = &s->busy[i];
    if(u->n == 0) continue;
    if(u->batch == b || (u->member[0]->kind == NEC2C_CUDA_REQUEST_BATCH && u->member[0]->batch == b)) return 1;
  }
  return 0;
}

static int same_options(const nec2c_cuda_gmres_options *a, const nec2c_cuda_gmres_options *b)
{
  return a->restart == b->restart && a->maximum_iterations == b->maximum_iterations &&
         a->relative_tolerance == b->relative_tolerance && a->absolute_tolerance == b->absolute_tolerance;
}

/* The registered batch holding volume request r's operator (its index in
   *q), or NULL. */
static nec2c_cuda_vie_batch *merge_batch_of(const nec2c_cuda_server *s, const nec2c_cuda_request *r, size_t *q)
{
  size_t i;
  if(r->kind != NEC2C_CUDA_REQUEST_VOLUME || r->options.restart == 0 || r->options.restart > MERGE_MAX_RESTART)
    return NULL;
  for(i = 0; i < s->merges; ++i) {
    const size_t k = n2c_batch_index(s->merge[i], r->plan, r->system);
    if(k != (size_t)-1) { *q = k; return s->merge[i]; }
  }
  return NULL;
}

/* Merged volume requests: one batched solve over their systems. */
static void run_merged(run_t *u)
{
  const size_t k = nec2c_cuda_vie_batch_systems(u->batch);
  const nec2c_cuda_complex **bv = calloc(k, sizeof(*bv));
  nec2c_cuda_complex **xv = calloc(k, sizeof(*xv));
  nec2c_cuda_gmres_report *reps = calloc(k, sizeof(*reps));
  size_t j;
  int ok = bv && xv && reps;
  if(!ok) n2c_set_error("merged requests: out of host memory");
  for(j = 0; ok && j < u->n; ++j) {
    bv[u->index[j]] = u->member[j]->b;
    xv[u->index[j]] = u->member[j]->x;
  }
  if(ok) ok = n2c_gmres_batch_subset(u->batch, bv, xv, &u->member[0]->options, reps);
  for(j = 0; j < u->n; ++j) {
    nec2c_cuda_request *r = u->member[j];
    if(reps) r->report = reps[u->index[j]];
    /* 1 when the system converged and its x came back, as a single solve
       returns 1 only on convergence. */
    r->status = ok && reps && reps[u->index[j]].status == 0;
    r->merged = u->n;
    if(!r->status) {
      const int st = ok ? (int)r->report.status : -1;
      strncpy(r->error, st == 1 ? "GMRES iteration limit" : st == 2 ? "GMRES breakdown" : nec2c_cuda_last_error(),
              sizeof(r->error) - 1);
      r->error[sizeof(r->error) - 1] = 0;
    }
  }
  free(bv); free(xv); free(reps);
}

static void run_request(nec2c_cuda_server *s, nec2c_cuda_request *r)
{
  int steps = 0;
  memset(&r->report, 0, sizeof(r->report));
  r->merged = 1;
  if(r->kind == NEC2C_CUDA_REQUEST_DENSE) {
    r->status = n2c_dense_solve_private(r->order, r->matrix, r->ld, r->rhs, r->rhs_stride, r->rhs_count, s->split,
                                        &steps);
    r->report.status = r->status;
    r->report.iterations = steps < 0 ? 0 : (size_t)steps;
  } else if(r->kind == NEC2C_CUDA_REQUEST_BATCH) {
    r->status = run_batch(r);
  } else if(r->plan) {
    r->status = nec2c_cuda_gmres_plan(r->plan, r->b, r->x, &r->options, &r->report);
  } else {
    r->status = nec2c_cuda_gmres_hybrid(r->system, r->b, r->x, &r->options, &r->report);
  }
  if(!r->status) {
    strncpy(r->error, nec2c_cuda_last_error(), sizeof(r->error) - 1);
    r->error[sizeof(r->error) - 1] = 0;
  }
}

static int fits(const nec2c_cuda_server *s, size_t f)
{
  return s->in_use == 0 || (f <= s->budget && s->in_use + f <= s->budget);
}

/* With the lock held: the queued volume requests that can join r (at queue
   position pick, on system q0 of registered batch b) in one batched solve,
   r first.  Fills u (member / index arrays of b's system count) and marks
   the chosen queue positions in taken; returns the run's footprint, or 0
   when fewer than two requests can merge or the merged run does not fit. */
static size_t gather_merge(const nec2c_cuda_server *s, nec2c_cuda_request *r, size_t pick, size_t q0,
                           nec2c_cuda_vie_batch *b, run_t *u, unsigned char *taken)
{
  const size_t k = nec2c_cuda_vie_batch_systems(b), order = nec2c_cuda_vie_batch_order(b);
  unsigned char *used = calloc(k, 1);
  size_t q, f;
  if(!used) return 0;
  u->n = 0;
  u->member[u->n] = r; u->index[u->n++] = q0; used[q0] = 1; taken[pick] = 1;
  for(q = 0; q < s->count && u->n < k; ++q) {
    nec2c_cuda_request *c = s->queue[(s->head + q) % s->cap];
    size_t qc;
    if(q == pick || c->kind != NEC2C_CUDA_REQUEST_VOLUME || !same_options(&c->options, &r->options)) continue;
    qc = n2c_batch_index(b, c->plan, c->system);
    if(qc == (size_t)-1 || used[qc] || plan_busy(s, c)) continue;
    used[qc] = 1; taken[q] = 1;
    u->member[u->n] = c; u->index[u->n++] = qc;
  }
  free(used);
  /* The batch request's footprint for the whole batch's vectors. */
  f = (r->options.restart + 4) * order * CPX + 2 * order * CPX;
  if(u->n < 2 || !fits(s, f)) {
    for(q = 0; q < s->count; ++q) taken[q] = 0;
    u->n = 0;
    return 0;
  }
  return f;
}

/* Size class of a dense request: the cluster size of its first panel (one
   CTA per 256 rows, rounded up to a power of two), so that the members of a
   lockstep batch, which advances at its largest member's pace, are within a
   factor of two of each other in order. */
static size_t dense_class(size_t n)
{
  size_t c = 1;
  while(c * 256 < n) c <<= 1;
  return c;
}

static int dense_mergeable(const nec2c_cuda_server *s, const nec2c_cuda_request *r)
{
  return r->kind == NEC2C_CUDA_REQUEST_DENSE && s->dense_merge >= 2 && r->order > 0 &&
         (long long)r->order <= n2d_lu_batch_max_order() && r->rhs_count > 0 && r->rhs_count <= 65535 &&
         r->ld >= r->order && r->rhs_stride >= r->order;
}

/* With the lock held: the queued dense requests of r's size class that join
   r (at queue position pick) in one lockstep batch, r first, while their
   summed footprint fits (at most dense_merge).  Fills u and taken; returns
   the run's footprint, or 0 when no other request joins. */
static size_t gather_dense(const nec2c_cuda_server *s, nec2c_cuda_request *r, size_t pick, size_t fp, run_t *u,
                           unsigned char *taken)
{
  const size_t cls = dense_class(r->order);
  size_t q, f = fp;
  u->n = 0;
  u->member[u->n++] = r;
  taken[pick] = 1;
  for(q = 0; q < s->count && u->n < s->dense_merge; ++q) {
    nec2c_cuda_request *c = s->queue[(s->head + q) % s->cap];
    size_t fc;
    if(q == pick || !dense_mergeable(s, c) || dense_class(c->order) != cls) continue;
    fc = footprint(s, c);
    /* Members after the first always fit within the budget (a lone request
       larger than the budget may still run alone). */
    if(s->in_use + f + fc > s->budget) continue;
    f += fc;
    taken[q] = 1;
    u->member[u->n++] = c;
  }
  if(u->n < 2) {
    for(q = 0; q < s->count; ++q) taken[q] = 0;
    u->n = 0;
    return 0;
  }
  return f;
}

/* Merged dense requests: one lockstep factorisation and solve of their
   private matrix copies (the split-precision form with FP64 refinement on a
   split server). */
static void run_dense_merged(const nec2c_cuda_server *s, run_t *u)
{
  const size_t k = u->n;
  size_t *order = calloc(k, sizeof(size_t)), *ld = calloc(k, sizeof(size_t)), *stride = calloc(k, sizeof(size_t));
  size_t *count = calloc(k, sizeof(size_t)), j;
  const nec2c_cuda_complex **mat = calloc(k, sizeof(*mat));
  nec2c_cuda_complex **rhs = calloc(k, sizeof(*rhs));
  int *st = calloc(k, sizeof(int)), *steps = calloc(k, sizeof(int));
  int ok = order && ld && stride && count && mat && rhs && st && steps;
  if(!ok) n2c_set_error("merged dense run: out of host memory");
  for(j = 0; ok && j < k; ++j) {
    const nec2c_cuda_request *r = u->member[j];
    order[j] = r->order; ld[j] = r->ld; stride[j] = r->rhs_stride; count[j] = r->rhs_count;
    mat[j] = r->matrix; rhs[j] = r->rhs;
  }
  if(ok) ok = n2c_dense_solve_private_batch(k, order, mat, ld, rhs, stride, count, s->split, st, steps);
  for(j = 0; j < k; ++j) {
    nec2c_cuda_request *r = u->member[j];
    memset(&r->report, 0, sizeof(r->report));
    r->status = ok && st && st[j];
    r->report.status = r->status;
    r->report.iterations = ok && steps && steps[j] > 0 ? (size_t)steps[j] : 0;
    r->merged = k;
    if(!r->status) {
      strncpy(r->error, ok ? "matrix is singular" : nec2c_cuda_last_error(), sizeof(r->error) - 1);
      r->error[sizeof(r->error) - 1] = 0;
    }
  }
  free(order); free(ld); free(stride); free(count); free(mat); free(rhs); free(st); free(steps);
}

static void *worker(void *arg)
{
  nec2c_cuda_server *s = arg;
  void *stream;
  int slot = -1, i;
  n2d_set_device(s->device);
  stream = n2d_stream_create();
  n2d_set_stream(stream);
  pthread_mutex_lock(&s->lock);
  for(;;) {
    nec2c_cuda_request *r = NULL;
    nec2c_cuda_vie_batch *mb = NULL;
    run_t *u;
    size_t pick = 0, q, fp = 0, q0 = 0, kept, j;
    unsigned char *taken = NULL;
    if(s->stop && s->count == 0) break;
    for(q = 0; q < s->count; ++q) {
      nec2c_cuda_request *c = s->queue[(s->head + q) % s->cap];
      const size_t f = footprint(s, c);
      const int ok = fits(s, f);
      if(ok && !plan_busy(s, c)) { r = c; pick = q; fp = f; break; }
      /* A request that does not fit may be passed only `slots` times. */
      if(!ok && c->skipped >= (unsigned)s->slots) break;
    }
    if(!r) { pthread_cond_wait(&s->work, &s->lock); continue; }
    for(q = 0; q < pick; ++q) {
      nec2c_cuda_request *c = s->queue[(s->head + q) % s->cap];
      if(!fits(s, footprint(s, c))) c->skipped++;
    }
    for(i = 0; i < s->slots; ++i) if(s->busy[i].n == 0) { slot = i; break; }
    if(slot < 0) { pthread_cond_wait(&s->work, &s->lock); continue; }   /* one run per worker: not reached */
    u = &s->busy[slot];
    u->batch = NULL;
    u->dense = 0;
    /* Continuous batching: the queued requests on the other systems of r's
       registered batch join it. */
    mb = merge_batch_of(s, r, &q0);
    if(mb && !batch_busy(s, mb) && s->count > 1 && (taken = calloc(s->count, 1)) != NULL &&
       (u->member = malloc(nec2c_cuda_vie_batch_systems(mb) * sizeof(*u->member))) != NULL &&
       (u->index = malloc(nec2c_cuda_vie_batch_systems(mb) * sizeof(*u->index))) != NULL) {
      const size_t f = gather_merge(s, r, pick, q0, mb, u, taken);
      if(f) { fp = f; u->batch = mb; }
    }
    /* Dense requests of r's size class queued behind it join it in one
       lockstep factorisation. */
    if(!u->batch && dense_mergeable(s, r) && s->count > 1) {
      free(u->member); free(u->index); free(taken);
      u->index = NULL;
      taken = calloc(s->count, 1);
      u->member = malloc(s->dense_merge * sizeof(*u->member));
      if(taken && u->member) {
        const size_t f = gather_dense(s, r, pick, fp, u, taken);
        if(f) { fp = f; u->dense = 1; }
      }
    }
    if(!u->batch && !u->dense) {
      free(u->member); free(u->index);
      u->member = NULL; u->index = NULL;
      free(taken);
      taken = calloc(s->count, 1);
      u->member = malloc(sizeof(*u->member));
      if(!taken || !u->member) {
        /* Out of host memory: fail the request rather than the server. */
        free(taken); free(u->member); u->member = NULL;
        for(q = pick; q + 1 < s->count; ++q)
          s->queue[(s->head + q) % s->cap] = s->queue[(s->head + q + 1) % s->cap];
        s->count--;
        r->status = 0;
        strncpy(r->error, "server: out of host memory", sizeof(r->error) - 1);
        r->finished_s = now_s();
        r->done = 1;
        s->pending--;
        pthread_cond_broadcast(&s->done);
        continue;
      }
      taken[pick] = 1;
      u->member[0] = r;
      u->n = 1;
    }
    /* Take the chosen requests out of the queue, keeping the order of the rest. */
    for(q = 0, kept = 0; q < s->count; ++q)
      if(!taken[q]) s->queue[(s->head + kept++) % s->cap] = s->queue[(s->head + q) % s->cap];
    s->count = kept;
    free(taken);
    s->in_use += fp;
    for(j = 0; j < u->n; ++j) {
      u->member[j]->footprint = j == 0 ? fp : 0;
      u->member[j]->started_s = now_s();
    }
    pthread_mutex_unlock(&s->lock);
    if(u->batch) run_merged(u);
    else if(u->dense) run_dense_merged(s, u);
    else run_request(s, r);
    pthread_mutex_lock(&s->lock);
    s->in_use -= fp;
    for(j = 0; j < u->n; ++j) {
      u->member[j]->finished_s = now_s();
      u->member[j]->done = 1;
      s->pending--;
    }
    u->n = 0;
    u->batch = NULL;
    u->dense = 0;
    free(u->member); free(u->index);
    u->member = NULL; u->index = NULL;
    slot = -1;
    pthread_cond_broadcast(&s->done);
    pthread_cond_broadcast(&s->work);
  }
  pthread_mutex_unlock(&s->lock);
  n2d_sync();
  n2d_set_stream(NULL);
  n2d_stream_destroy(stream);
  return NULL;
}

int nec2c_cuda_server_create(nec2c_cuda_server **out, int device, int slots, size_t device_budget, int split)
{
  nec2c_cuda_server *s;
  int i;
  if(!out) return 0;
  *out = NULL;
  if(slots < 1 || slots > 64) { n2c_set_error("slots must be 1..64"); return 0; }
  if(!n2d_set_device(device) || !n2d_device_ok()) return 0;
  if(device_budget == 0) {
    /* concurrency.c:131-136: keep max(1/5, 1 GiB) of the free memory back. */
    size_t free_b = 0, total_b = 0, reserve;
    if(!n2d_mem_info(&free_b, &total_b)) return 0;
    reserve = free_b / 5 > ((size_t)1 << 30) ? free_b / 5 : ((size_t)1 << 30);
    device_budget = free_b > reserve ? free_b - reserve : free_b / 2;
  }
  s = calloc(1, sizeof(*s));
  if(!s) return 0;
  s->device = device; s->slots = slots; s->split = split != 0; s->budget = device_budget;
  s->cap = 64;
  s->queue = calloc(s->cap, sizeof(*s->queue));
  s->busy = calloc((size_t)slots, sizeof(*s->busy));
  s->threads = calloc((size_t)slots, sizeof(*s->threads));
  if(!s->queue || !s->busy || !s->threads) { free(s->queue); free(s->busy); free(s->threads); free(s); return 0; }
  pthread_mutex_init(&s->lock, NULL);
  pthread_cond_init(&s->work, NULL);
  pthread_cond_init(&s->done, NULL);
  for(i = 0; i < slots; ++i) {
    if(pthread_create(&s->threads[i], NULL, worker, s) != 0) {
      pthread_mutex_lock(&s->lock);
      s->stop = 1;
      pthread_cond_broadcast(&s->work);
      pthread_mutex_unlock(&s->lock);
      while(i-- > 0) pthread_join(s->threads[i], NULL);
      free(s->queue); free(s->busy); free(s->threads); free(s);
      n2c_set_error("worker thread creation failed");
      return 0;
    }
  }
  s->started = slots;
  *out = s;
  return 1;
}

int nec2c_cuda_server_submit(nec2c_cuda_server *s, nec2c_cuda_request *r)
{
  if(!s || !r) { n2c_set_error("submit: null server or request"); return 0; }
  if(r->kind == NEC2C_CUDA_REQUEST_DENSE) {
    if(!r->matrix || !r->rhs || r->order == 0 || r->ld < r->order || r->rhs_count == 0 ||
       r->rhs_stride < r->order) {
      n2c_set_error("submit: dense request needs matrix, rhs, order > 0, ld >= order, rhs_count > 0 and "
                    "rhs_stride >= order");
      return 0;
    }
  } else if(r->kind == NEC2C_CUDA_REQUEST_VOLUME) {
    if((!r->plan) == (!r->system) || !r->b || !r->x) {
      n2c_set_error("submit: volume request needs exactly one of plan / system, and b and x");
      return 0;
    }
  } else if(r->kind == NEC2C_CUDA_REQUEST_BATCH) {
    if(!r->batch || !r->b || !r->x || !r->reports || r->b == (const nec2c_cuda_complex *)r->x) {
      n2c_set_error("submit: batch request needs batch, reports and distinct b and x");
      return 0;
    }
  } else {
    n2c_set_error("submit: unknown request kind %d", r->kind);
    return 0;
  }
  pthread_mutex_lock(&s->lock);
  if(s->stop) { pthread_mutex_unlock(&s->lock); n2c_set_error("submit: server is stopping"); return 0; }
  if(s->count == s->cap) {
    nec2c_cuda_request **q = malloc(2 * s->cap * sizeof(*q));
    size_t i;
    if(!q) { pthread_mutex_unlock(&s->lock); n2c_set_error("submit: out of host memory"); return 0; }
    for(i = 0; i < s->count; ++i) q[i] = s->queue[(s->head + i) % s->cap];
    free(s->queue);
    s->queue = q; s->head = 0; s->cap *= 2;
  }
  r->done = 0; r->status = 0; r->skipped = 0; r->footprint = 0; r->error[0] = 0;
  r->queued_s = now_s(); r->started_s = r->finished_s = 0;
  s->queue[(s->head + s->count) % s->cap] = r;
  s->count++;
  s->pending++;
  pthread_cond_broadcast(&s->work);
  pthread_mutex_unlock(&s->lock);
  return 1;
}

int nec2c_cuda_server_wait(nec2c_cuda_server *s, nec2c_cuda_request *r)
{
  if(!s || !r) return 0;
  pthread_mutex_lock(&s->lock);
  while(!r->done) pthread_cond_wait(&s->done, &s->lock);
  pthread_mutex_unlock(&s->lock);
  return r->status;
}

int nec2c_cuda_server_drain(nec2c_cuda_server *s)
{
  if(!s) return 0;
  pthread_mutex_lock(&s->lock);
  while(s->pending) pthread_cond_wait(&s->done, &s->lock);
  pthread_mutex_unlock(&s->lock);
  return 1;
}

size_t nec2c_cuda_server_budget(const nec2c_cuda_server *s) { return s ? s->budget : 0; }

int nec2c_cuda_server_merge_batch(nec2c_cuda_server *s, nec2c_cuda_vie_batch *b)
{
  nec2c_cuda_vie_batch **m;
  size_t i;
  if(!s || !b) { n2c_set_error("merge batch: null server or batch"); return 0; }
  pthread_mutex_lock(&s->lock);
  for(i = 0; i < s->merges; ++i)
    if(s->merge[i] == b) {
      pthread_mutex_unlock(&s->lock);
      n2c_set_error("merge batch: batch already registered");
      return 0;
    }
  m = realloc(s->merge, (s->merges + 1) * sizeof(*m));
  if(!m) { pthread_mutex_unlock(&s->lock); n2c_set_error("merge batch: out of host memory"); return 0; }
  s->merge = m;
  s->merge[s->merges++] = b;
  pthread_cond_broadcast(&s->work);
  pthread_mutex_unlock(&s->lock);
  return 1;
}

int nec2c_cuda_server_merge_dense(nec2c_cuda_server *s, size_t max_systems)
{
  if(!s) { n2c_set_error("dense merging: null server"); return 0; }
  if(max_systems > 65535) { n2c_set_error("dense merging: at most 65535 systems per batch"); return 0; }
  pthread_mutex_lock(&s->lock);
  s->dense_merge = max_systems;
  pthread_mutex_unlock(&s->lock);
  return 1;
}

void nec2c_cuda_server_destroy(nec2c_cuda_server *s)
{
  int i;
  if(!s) return;
  nec2c_cuda_server_drain(s);
  pthread_mutex_lock(&s->lock);
  s->stop = 1;
  pthread_cond_broadcast(&s->work);
  pthread_mutex_unlock(&s->lock);
  for(i = 0; i < s->started; ++i) pthread_join(s->threads[i], NULL);
  pthread_mutex_destroy(&s->lock);
  pthread_cond_destroy(&s->work);
  pthread_cond_destroy(&s->done);
  free(s->queue); free(s->busy); free(s->threads); free(s->merge);
  free(s);
}

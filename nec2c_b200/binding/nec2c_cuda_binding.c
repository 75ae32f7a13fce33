/* Reference-side binding of the CUDA backend: the `cuda` and `cuda-mixed`
 * values of nec2c's --backend and --fft-backend switches.
 *
 * nec2c (N5HXR/nec2c) selects its dense LU in dense_backend.c and its volume
 * FFT operator in vie_fft.c; dielectric_fft.c builds the hybrid [C B; D V]
 * system over that operator and vie_iterative.c runs GMRES on it.  This file
 * puts the CUDA library behind exactly those interfaces without editing the
 * files that define them: every function below is linked in place of the
 * reference's own with GNU ld's --wrap (a call to f from another object file
 * reaches __wrap_f; __real_f is the reference's f), and it forwards to the
 * reference unless a CUDA backend is selected.  The only source edit the
 * reference needs is the command-line whitelist (main.c:1409-1421 and
 * main.c:1439-1450), which must let "cuda" and "cuda-mixed" through to the
 * setters wrapped here.
 *
 *   dense_backend.c (dense_backend.h:14-37)   -> nec2c_cuda_dense_*
 *   vie_fft.c      (vie_fft.h:8-32)           -> nec2c_cuda_vie_fft_*
 *   dielectric_fft.c prepare / get_operator / free (dielectric_fft.h:10-25)
 *                                              -> nec2c_cuda_hybrid_*
 *   vie_iterative.c vie_gmres (vie_iterative.h:55-57), for the CUDA operators
 *                                              -> nec2c_cuda_gmres_plan / _hybrid
 *   concurrency.c concurrency_plan_for         -> one frequency job at a time
 *   matrix.c cmset (wires, classic kernel, free space or perfect ground, with
 *   the CUDA dense backend selected)           -> nec2c_cuda_mom_fill
 *
 * The two wire <-> volume coupling blocks of dielectric_wire.c are computed
 * by static code the wrapping cannot reach; the drop-in program compiles a
 * copy of that file with three insertions (patch_dielectric_wire.py) that
 * call nec2c_binding_wire_to_volume and nec2c_binding_volume_to_wire below.
 *
 * The certified near-pair Green tensor stays on the CPU: the CUDA plan calls
 * back into the reference's vie_cuboid_n with the options vie_fft.c:344 uses.
 * A GPU solve runs in the nec2c process itself; the reference's forked
 * frequency workers could not use the parent's CUDA context, so with a CUDA
 * backend selected the planner is held to one job (its threads still serve
 * the CPU work around the solve).
 */
#include <complex.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "coated_wire.h"
#include "concurrency.h"
#include "dense_backend.h"
#include "dielectric_fft.h"
#include "shared.h"
#include "vie_fft.h"
#include "vie_iterative.h"
#include "vie_kernel.h"
#include "wire_operator.h"

#include "nec2c_cuda.h"

/* ------------------------------------------------------------ selection */
static int g_dense_cuda = 0;   /* --backend cuda|cuda-mixed */
static int g_fft_cuda = 0;     /* --fft-backend cuda|cuda-mixed */
static int g_fft_last_cuda = 0;

static int is_cuda_name(const char *name) { return name && !strncmp(name, "cuda", 4); }

static void report_failure(const char *what)
{
  fprintf(stderr, "nec2c: CUDA %s failed: %s\n", what, nec2c_cuda_last_error());
}

/* ------------------------------------------------------------ dense LU */
int __real_dense_backend_set(const char *name);
const char *__real_dense_backend_requested_name(void);
const char *__real_dense_backend_name_for_order(size_t order);
int __real_dense_backend_factor_classic(size_t order, complex double *matrix, size_t ld, int *pivots);
int __real_dense_backend_solve_classic(size_t order, const complex double *matrix, size_t ld,
                                       const int *pivots, complex double *rhs);
int __real_dense_backend_solve_classic_many(size_t order, const complex double *matrix, size_t ld,
                                            const int *pivots, complex double *rhs, size_t stride,
                                            size_t count);
int __real_dense_backend_solve_row_major(complex double *matrix, complex double *rhs, size_t order);

/* dense_backend.c:21-34 */
int __wrap_dense_backend_set(const char *name)
{
  if(is_cuda_name(name)) {
    if(!nec2c_cuda_available() || !nec2c_cuda_dense_backend_set(name)) {
      report_failure("dense backend selection");
      return 0;
    }
    g_dense_cuda = 1;
    return 1;
  }
  g_dense_cuda = 0;
  return __real_dense_backend_set(name);
}

const char *__wrap_dense_backend_requested_name(void)
{
  return g_dense_cuda ? nec2c_cuda_dense_backend_name() : __real_dense_backend_requested_name();
}

const char *__wrap_dense_backend_name_for_order(size_t order)
{
  return g_dense_cuda ? nec2c_cuda_dense_backend_name() : __real_dense_backend_name_for_order(order);
}

/* dense_backend.c:84, called by factr (matrix.c:1318). */
int __wrap_dense_backend_factor_classic(size_t order, complex double *matrix, size_t ld, int *pivots)
{
  if(!g_dense_cuda) return __real_dense_backend_factor_classic(order, matrix, ld, pivots);
  if(!nec2c_cuda_dense_factor_classic(order, matrix, ld, pivots)) { report_failure("LU factor"); return 0; }
  return 1;
}

/* dense_backend.c:109, called by solve (matrix.c:1561). */
int __wrap_dense_backend_solve_classic(size_t order, const complex double *matrix, size_t ld,
                                       const int *pivots, complex double *rhs)
{
  if(!g_dense_cuda) return __real_dense_backend_solve_classic(order, matrix, ld, pivots, rhs);
  if(!nec2c_cuda_dense_solve_classic(order, matrix, ld, pivots, rhs)) { report_failure("LU solve"); return 0; }
  return 1;
}

/* dense_backend.c:117, called by solves (matrix.c:1683). */
int __wrap_dense_backend_solve_classic_many(size_t order, const complex double *matrix, size_t ld,
                                            const int *pivots, complex double *rhs, size_t stride,
                                            size_t count)
{
  if(!g_dense_cuda)
    return __real_dense_backend_solve_classic_many(order, matrix, ld, pivots, rhs, stride, count);
  if(!nec2c_cuda_dense_solve_classic_many(order, matrix, ld, pivots, rhs, stride, count)) {
    report_failure("LU solve");
    return 0;
  }
  return 1;
}

/* dense_backend.c:192, called by the -s dense coupled and volume solvers. */
int __wrap_dense_backend_solve_row_major(complex double *matrix, complex double *rhs, size_t order)
{
  if(!g_dense_cuda) return __real_dense_backend_solve_row_major(matrix, rhs, order);
  if(!nec2c_cuda_dense_solve_row_major(matrix, rhs, order)) { report_failure("row-major solve"); return 0; }
  return 1;
}

/* ------------------------------------------------------ volume FFT plan */
int __real_vie_fft_backend_set(const char *name);
const char *__real_vie_fft_backend_requested_name(void);
const char *__real_vie_fft_backend_name(const vie_fft_plan *plan);
const char *__real_vie_fft_backend_last_used_name(void);
void __real_vie_fft_backend_clear_last_used(void);
int __real_vie_fft_create(vie_fft_plan **out, const size_t shape[3], size_t cells, const size_t *xyz,
                          double pitch, double k0, complex double epsilon_r, size_t byte_limit);
int __real_vie_fft_set_permittivity(vie_fft_plan *plan, size_t cell, complex double epsilon_r);
void __real_vie_fft_destroy(vie_fft_plan *plan);
size_t __real_vie_fft_bytes(const vie_fft_plan *plan);
size_t __real_vie_fft_threads(const vie_fft_plan *plan);
void __real_vie_fft_operator(vie_fft_plan *plan, vie_linear_operator *op);

/* CUDA plans handed out as vie_fft_plan pointers (the type is opaque outside
   vie_fft.c, so only the functions below ever look inside). */
static nec2c_cuda_vie_plan **g_plans = NULL;
static size_t g_plan_count = 0, g_plan_capacity = 0;
/* The plan the latest wrapped vie_fft_create built (dielectric_fft.c's
   prepare builds exactly one). */
static nec2c_cuda_vie_plan *g_last_plan = NULL;

static nec2c_cuda_vie_plan *cuda_plan(const vie_fft_plan *plan)
{
  size_t i;
  for(i = 0; plan && i < g_plan_count; ++i)
    if((const void *)g_plans[i] == (const void *)plan) return g_plans[i];
  return NULL;
}

static int plan_register(nec2c_cuda_vie_plan *p)
{
  if(g_plan_count == g_plan_capacity) {
    size_t cap = g_plan_capacity ? 2 * g_plan_capacity : 8;
    nec2c_cuda_vie_plan **grown = realloc(g_plans, cap * sizeof(*grown));
    if(!grown) return 0;
    g_plans = grown;
    g_plan_capacity = cap;
  }
  g_plans[g_plan_count++] = p;
  return 1;
}

static void plan_unregister(nec2c_cuda_vie_plan *p)
{
  size_t i;
  for(i = 0; i < g_plan_count; ++i)
    if(g_plans[i] == p) { g_plans[i] = g_plans[--g_plan_count]; return; }
}

/* vie_fft.c:69-78 */
int __wrap_vie_fft_backend_set(const char *name)
{
  if(is_cuda_name(name)) {
    if(!nec2c_cuda_available() || !nec2c_cuda_vie_fft_backend_set(name)) {
      report_failure("FFT backend selection");
      return 0;
    }
    g_fft_cuda = 1;
    return 1;
  }
  g_fft_cuda = 0;
  return __real_vie_fft_backend_set(name);
}

const char *__wrap_vie_fft_backend_requested_name(void)
{
  return g_fft_cuda ? nec2c_cuda_vie_fft_backend_name() : __real_vie_fft_backend_requested_name();
}

const char *__wrap_vie_fft_backend_name(const vie_fft_plan *plan)
{
  return cuda_plan(plan) ? nec2c_cuda_vie_fft_backend_name() : __real_vie_fft_backend_name(plan);
}

const char *__wrap_vie_fft_backend_last_used_name(void)
{
  return g_fft_last_cuda ? nec2c_cuda_vie_fft_backend_name() : __real_vie_fft_backend_last_used_name();
}

void __wrap_vie_fft_backend_clear_last_used(void)
{
  g_fft_last_cuda = 0;
  __real_vie_fft_backend_clear_last_used();
}

/* The certified near-pair tensor, as vie_fft.c:342-355 computes it: the
   testing cube centred at pitch * offset, the source cube at the origin. */
static int near_tensor(void *context, const size_t offset[3], double pitch, double k0,
                       nec2c_cuda_complex out[9])
{
  vie_cuboid testing = {{pitch * (double)offset[0], pitch * (double)offset[1], pitch * (double)offset[2]},
                        {pitch, pitch, pitch}};
  vie_cuboid source = {{0, 0, 0}, {pitch, pitch, pitch}};
  vie_kernel_options options;
  complex double n[3][3];
  int i, j;
  (void)context;
  vie_kernel_default_options(&options);
  options.relative_tolerance = 5e-7;
  options.absolute_tolerance = 5e-10;
  options.far_order = 16;
  if(!vie_cuboid_n(&testing, &source, k0, &options, n, NULL)) return 0;
  for(i = 0; i < 3; ++i)
    for(j = 0; j < 3; ++j) out[3 * i + j] = n[i][j];
  return 1;
}

/* vie_fft.c:378-441 */
int __wrap_vie_fft_create(vie_fft_plan **out, const size_t shape[3], size_t cells, const size_t *xyz,
                          double pitch, double k0, complex double epsilon_r, size_t byte_limit)
{
  nec2c_cuda_vie_plan *p = NULL;
  if(!g_fft_cuda) {
    g_fft_last_cuda = 0;
    return __real_vie_fft_create(out, shape, cells, xyz, pitch, k0, epsilon_r, byte_limit);
  }
  if(out) *out = NULL;
  if(!out) return 0;
  if(!nec2c_cuda_vie_fft_create(&p, shape, cells, xyz, pitch, k0, creal(epsilon_r), cimag(epsilon_r),
                                byte_limit, near_tensor, NULL)) {
    report_failure("FFT plan");
    return 0;
  }
  if(!plan_register(p)) { nec2c_cuda_vie_fft_destroy(p); return 0; }
  g_last_plan = p;
  g_fft_last_cuda = 1;
  *out = (vie_fft_plan *)(void *)p;
  return 1;
}

/* vie_fft.c:445-455 */
int __wrap_vie_fft_set_permittivity(vie_fft_plan *plan, size_t cell, complex double epsilon_r)
{
  nec2c_cuda_vie_plan *p = cuda_plan(plan);
  if(!p) return __real_vie_fft_set_permittivity(plan, cell, epsilon_r);
  return nec2c_cuda_vie_fft_set_permittivity(p, cell, creal(epsilon_r), cimag(epsilon_r));
}

void __wrap_vie_fft_destroy(vie_fft_plan *plan)
{
  nec2c_cuda_vie_plan *p = cuda_plan(plan);
  if(!p) { __real_vie_fft_destroy(plan); return; }
  plan_unregister(p);
  if(g_last_plan == p) g_last_plan = NULL;
  nec2c_cuda_vie_fft_destroy(p);
}

size_t __wrap_vie_fft_bytes(const vie_fft_plan *plan)
{
  nec2c_cuda_vie_plan *p = cuda_plan(plan);
  return p ? nec2c_cuda_vie_fft_bytes(p) : __real_vie_fft_bytes(plan);
}

size_t __wrap_vie_fft_threads(const vie_fft_plan *plan)
{
  return cuda_plan(plan) ? 1 : __real_vie_fft_threads(plan);
}

/* vie_fft.c:239-273 as callbacks */
void __wrap_vie_fft_operator(vie_fft_plan *plan, vie_linear_operator *op)
{
  nec2c_cuda_vie_plan *p = cuda_plan(plan);
  if(!p) { __real_vie_fft_operator(plan, op); return; }
  op->order = nec2c_cuda_vie_fft_order(p);
  op->apply = nec2c_cuda_vie_fft_apply;
  op->context = p;
  op->precondition = nec2c_cuda_vie_fft_precondition;
  op->precondition_context = p;
}

/* ------------------------------------------------------ hybrid systems */
int __real_dielectric_fft_prepare(dielectric_fft_system **out, const dielectric_model *model,
                                  const dielectric_mesh_result *mesh, size_t conductors, double k0,
                                  size_t extra_bytes, dielectric_diagnostic *diagnostic);
int __real_dielectric_fft_prepare_pec(dielectric_fft_system **out, const dielectric_model *model,
                                      const dielectric_mesh_result *mesh, size_t conductors, double k0,
                                      size_t extra_bytes, dielectric_diagnostic *diagnostic);
void __real_dielectric_fft_free(dielectric_fft_system *system);
void __real_dielectric_fft_get_operator(dielectric_fft_system *system, vie_linear_operator *op);

/* A dielectric_fft_system whose volume plan is a CUDA plan, with the device
   operator made for it when the operator is first asked for. */
typedef struct bound_system {
  struct bound_system *next;
  dielectric_fft_system *system;
  nec2c_cuda_vie_plan *plan;     /* NULL when the system has no cells */
  size_t conductors, volume_unknowns;
  int pec;
  nec2c_cuda_hybrid *hybrid;
} bound_system;
static bound_system *g_systems = NULL;

static bound_system *bound(const dielectric_fft_system *s)
{
  bound_system *b;
  for(b = g_systems; b; b = b->next) if(b->system == s) return b;
  return NULL;
}

/* dielectric_fft.c:89-175: the reference's own lattice inference, PEC image
   embedding and 512 MiB accounting run unchanged; the plan it builds through
   vie_fft_create is the CUDA plan when that backend is selected. */
static int prepare_bound(int pec, dielectric_fft_system **out, const dielectric_model *model,
                         const dielectric_mesh_result *mesh, size_t conductors, double k0, size_t extra,
                         dielectric_diagnostic *diagnostic)
{
  int ok;
  bound_system *b;
  g_last_plan = NULL;
  ok = pec ? __real_dielectric_fft_prepare_pec(out, model, mesh, conductors, k0, extra, diagnostic)
           : __real_dielectric_fft_prepare(out, model, mesh, conductors, k0, extra, diagnostic);
  if(!ok || !g_fft_cuda || !out || !*out) return ok;
  b = calloc(1, sizeof(*b));
  if(!b) { __real_dielectric_fft_free(*out); *out = NULL; return 0; }
  b->system = *out;
  b->plan = mesh->cell_count ? g_last_plan : NULL;
  b->conductors = conductors;
  b->volume_unknowns = 3 * mesh->cell_count;
  b->pec = pec;
  b->next = g_systems;
  g_systems = b;
  return 1;
}

int __wrap_dielectric_fft_prepare(dielectric_fft_system **out, const dielectric_model *model,
                                  const dielectric_mesh_result *mesh, size_t conductors, double k0,
                                  size_t extra_bytes, dielectric_diagnostic *diagnostic)
{
  return prepare_bound(0, out, model, mesh, conductors, k0, extra_bytes, diagnostic);
}

int __wrap_dielectric_fft_prepare_pec(dielectric_fft_system **out, const dielectric_model *model,
                                      const dielectric_mesh_result *mesh, size_t conductors, double k0,
                                      size_t extra_bytes, dielectric_diagnostic *diagnostic)
{
  return prepare_bound(1, out, model, mesh, conductors, k0, extra_bytes, diagnostic);
}

void __wrap_dielectric_fft_free(dielectric_fft_system *s)
{
  bound_system **pp = &g_systems;
  while(*pp) {
    if((*pp)->system == s) {
      bound_system *b = *pp;
      *pp = b->next;
      nec2c_cuda_hybrid_destroy(b->hybrid);
      free(b);
      break;
    }
    pp = &(*pp)->next;
  }
  __real_dielectric_fft_free(s);   /* destroys the plan through vie_fft_destroy */
}

static int failed_operator(void *context, const complex double *x, complex double *y)
{
  (void)context; (void)x; (void)y;
  return 0;
}

/* dielectric_fft.c:84-88.  The callers assemble the conductor and cross
   blocks through dielectric_fft_entry first (dielectric_wire.c:1130-1254)
   and ask for the operator right before GMRES (dielectric_wire.c:1302), so
   the blocks are uploaded here, every time the operator is handed out. */
void __wrap_dielectric_fft_get_operator(dielectric_fft_system *s, vie_linear_operator *op)
{
  bound_system *b = bound(s);
  if(!b) { __real_dielectric_fft_get_operator(s, op); return; }
  if(!b->hybrid &&
     !nec2c_cuda_hybrid_create(&b->hybrid, b->plan, b->conductors, b->volume_unknowns, b->pec)) {
    report_failure("hybrid system");
    b->hybrid = NULL;
  }
  /* Uploaded with no conductors too: the upload also sets the
     preconditioner's volume divisor. */
  static const complex double no_blocks = 0;
  if(b->hybrid && !nec2c_cuda_hybrid_set_blocks(b->hybrid, b->conductors ? dielectric_fft_entry(s, 0, 0)
                                                                         : &no_blocks)) {
    report_failure("hybrid block upload");
    nec2c_cuda_hybrid_destroy(b->hybrid);
    b->hybrid = NULL;
  }
  if(!b->hybrid) {
    /* No device operator: the solve fails (GMRES reports the callback
       failure) rather than running on another path. */
    op->order = b->conductors + b->volume_unknowns;
    op->apply = failed_operator;
    op->context = NULL;
    op->precondition = failed_operator;
    op->precondition_context = NULL;
    return;
  }
  op->order = b->conductors + b->volume_unknowns;
  op->apply = nec2c_cuda_hybrid_apply;
  op->context = b->hybrid;
  op->precondition = nec2c_cuda_hybrid_precondition;
  op->precondition_context = b->hybrid;
}

/* ---------------------------------------------------------------- GMRES */
int __real_vie_gmres(const vie_linear_operator *op, const complex double *rhs, complex double *x,
                     const vie_gmres_options *options, vie_gmres_report *report);

/* vie_iterative.c:80-199: device-resident when the operator is one of the
   CUDA callbacks (options and report have the same layout as the library's). */
static int device_gmres_done(int converged, const vie_gmres_report *report)
{
  /* A failure on the device side (not the iteration itself) says why. */
  if(!converged && report &&
     (report->status == VIE_ITERATIVE_CALLBACK_FAILED || report->status == VIE_ITERATIVE_INVALID_INPUT ||
      report->status == VIE_ITERATIVE_ALLOCATION_FAILED))
    report_failure("GMRES");
  return converged;
}

int __wrap_vie_gmres(const vie_linear_operator *op, const complex double *rhs, complex double *x,
                     const vie_gmres_options *options, vie_gmres_report *report)
{
  if(op && op->apply == nec2c_cuda_hybrid_apply)
    return device_gmres_done(nec2c_cuda_gmres_hybrid(op->context, rhs, x,
                                                     (const nec2c_cuda_gmres_options *)options,
                                                     (nec2c_cuda_gmres_report *)report), report);
  if(op && op->apply == nec2c_cuda_vie_fft_apply)
    return device_gmres_done(nec2c_cuda_gmres_plan(op->context, rhs, x, (const nec2c_cuda_gmres_options *)options,
                                                   (nec2c_cuda_gmres_report *)report), report);
  return __real_vie_gmres(op, rhs, x, options, report);
}

/* ------------------------------------------------------- frequency jobs */
concurrency_plan __real_concurrency_plan_for(size_t frequency_count, size_t estimated_worker_bytes);

/* concurrency.c:118-171 */
concurrency_plan __wrap_concurrency_plan_for(size_t frequency_count, size_t estimated_worker_bytes)
{
  concurrency_plan plan = __real_concurrency_plan_for(frequency_count, estimated_worker_bytes);
  /* The thread count of an automatic plan is recomputed by the caller from
     the job count (main.c:76-89). */
  if(g_dense_cuda || g_fft_cuda) plan.jobs = 1;
  return plan;
}

/* Layout agreement the casts in __wrap_vie_gmres rely on. */
_Static_assert(sizeof(vie_gmres_options) == sizeof(nec2c_cuda_gmres_options), "options layout");
_Static_assert(sizeof(vie_gmres_report) == sizeof(nec2c_cuda_gmres_report), "report layout");

/* ------------------------------------------- wire <-> volume coupling */
static int coupling_ground_ok(void)
{
  return !wire_operator_ground_direct_only() && (gnd.ksymp == 1 || (gnd.ksymp == 2 && gnd.iperf == 1));
}

static int cell_arrays(const dielectric_mesh_result *mesh, double **centers, double **sizes)
{
  size_t c;
  int d;
  *centers = malloc(3 * mesh->cell_count * sizeof(double));
  *sizes = malloc(3 * mesh->cell_count * sizeof(double));
  if(!*centers || !*sizes) { free(*centers); free(*sizes); return 0; }
  for(c = 0; c < mesh->cell_count; ++c)
    for(d = 0; d < 3; ++d) {
      (*centers)[3 * c + d] = mesh->cells[c].center[d];
      (*sizes)[3 * c + d] = mesh->cells[c].size[d];
    }
  return 1;
}

/* dielectric_wire.c:422-510 on the GPU: 1 handled (result allocated with
   calloc, as the reference's serial path allocates it), 0 not a model the
   kernels cover (the reference's own assembly runs), -1 failed.  Covered:
   a CUDA backend selected, wires only, the NEC-2 wire engine with the
   classic thin-wire kernel, free space or a perfect ground. */
int nec2c_binding_wire_to_volume(const dielectric_mesh_result *mesh, size_t nw, size_t np,
    size_t conductor_unknowns, const complex double *sources,
    const complex double *wire_background_basis, const complex double *volume_chi,
    double k0, double omega, complex double **result, int *result_mapped,
    size_t *workers_used, int *fell_back)
{
  nec2c_cuda_wire_model w;
  double *centers = NULL, *sizes = NULL;
  complex double *out;
  (void)k0;
  if(!(g_dense_cuda || g_fft_cuda) || np || wire_background_basis || wire_operator_nec4_basis() ||
     dataj.iexk != 0 || !coupling_ground_ok() || conductor_unknowns != nw || nw != (size_t)data.n)
    return 0;
  if(!mesh->cell_count || !conductor_unknowns) return 0;
  out = calloc(conductor_unknowns * 3 * mesh->cell_count, sizeof(*out));
  if(!out || !cell_arrays(mesh, &centers, &sizes)) { free(out); return -1; }
  w.segments = nw;
  w.x = data.x; w.y = data.y; w.z = data.z; w.length = data.si; w.radius = data.bi;
  w.cab = data.cab; w.sab = data.sab; w.salp = data.salp;
  w.wavelength = data.wlam; w.rkh = dataj.rkh; w.pec_ground = gnd.ksymp == 2;
  if(!nec2c_cuda_coupling_wire_to_volume(&w, conductor_unknowns, sources, mesh->cell_count, centers, sizes,
                                         volume_chi, omega, out)) {
    report_failure("wire-to-volume coupling");
    free(out); free(centers); free(sizes);
    return -1;
  }
  free(centers); free(sizes);
  *result = out;
  *result_mapped = 0;
  *workers_used = 1;
  *fell_back = 0;
  return 1;
}

/* The wire rows of dielectric_wire.c:1164-1213 on the GPU: nw rows of 3 x
   cells values (malloc), or NULL when the model is not covered (a ground
   other than free space or a perfect ground) or the computation failed (the
   reference's loop then runs). */
complex double *nec2c_binding_volume_to_wire(const dielectric_mesh_result *mesh, size_t nw,
    const double *x, const double *y, const double *z, double k0, double omega)
{
  double *centers = NULL, *sizes = NULL, *obs, *tangent;
  complex double *out;
  size_t i;
  if(!(g_dense_cuda || g_fft_cuda) || !coupling_ground_ok() || !nw || !mesh->cell_count) return NULL;
  obs = malloc(6 * nw * sizeof(double));
  out = malloc(nw * 3 * mesh->cell_count * sizeof(*out));
  if(!obs || !out || !cell_arrays(mesh, &centers, &sizes)) { free(obs); free(out); return NULL; }
  tangent = obs + 3 * nw;
  for(i = 0; i < nw; ++i) {
    obs[3 * i] = x[i]; obs[3 * i + 1] = y[i]; obs[3 * i + 2] = z[i];
    tangent[3 * i] = data.cab[i]; tangent[3 * i + 1] = data.sab[i]; tangent[3 * i + 2] = data.salp[i];
  }
  if(!nec2c_cuda_coupling_volume_to_wire(nw, obs, tangent, mesh->cell_count, centers, sizes, k0, omega,
                                         gnd.ksymp == 2, out)) {
    report_failure("volume-to-wire coupling");
    free(out);
    out = NULL;
  }
  free(obs); free(centers); free(sizes);
  return out;
}

/* ------------------------------------------------------- wire MoM fill */
void __real_cmset(int nrow, complex double *cm, double rkhx, int iexkx);

/* A model the GPU fill covers: wires alone, no symmetry, the matrix in core
   (fblock's icase 1), the NEC-2 wire engine with the classic thin-wire
   kernel, no coated segments, free space or a perfect ground. */
static int mom_fill_covered(int nrow, int iexkx)
{
  int j;
  if(!g_dense_cuda || data.n <= 0 || data.m != 0 || data.np != data.n || nrow != data.n ||
     matpar.icase != 1 || matpar.nlast != data.n || iexkx != 0 || wire_operator_nec4_basis() ||
     !coupling_ground_ok())
    return 0;
  for(j = 1; j <= data.n; ++j)
    if(coated_wire_segment_active(j)) return 0;
  return 1;
}

/* cmset (matrix.c:48-195) on the GPU for the models mom_fill_covered
   accepts: the reference's own trio supplies each segment's basis
   functions, nec2c_cuda_mom_fill the matrix with the segment loads.  Other
   models take the reference's cmset.  A GPU failure stops the program, as
   the reference stops on a fill error. */
void __wrap_cmset(int nrow, complex double *cm, double rkhx, int iexkx)
{
  nec2c_cuda_wire_model w;
  size_t *first = NULL, cap = 0, used = 0;
  int *column = NULL;
  complex double *coef = NULL, *loads = NULL;
  int j, i, ok = 1;
  if(!mom_fill_covered(nrow, iexkx)) {
    __real_cmset(nrow, cm, rkhx, iexkx);
    return;
  }
  /* The state cmset leaves behind (matrix.c:54-60). */
  smat.nop = 1;
  dataj.rkh = rkhx;
  dataj.iexk = iexkx;
  first = malloc(((size_t)data.n + 1) * sizeof(*first));
  if(!first) ok = 0;
  for(j = 1; ok && j <= data.n; ++j) {
    first[j - 1] = used;
    wire_operator_trio(j);
    if(used + (size_t)segj.jsno > cap) {
      size_t ncap = 2 * cap + (size_t)segj.jsno + 64;
      int *nc = realloc(column, ncap * sizeof(*column));
      complex double *nf = nc ? realloc(coef, 3 * ncap * sizeof(*coef)) : NULL;
      if(nc) column = nc;
      if(nf) coef = nf;
      if(!nc || !nf) { ok = 0; break; }
      cap = ncap;
    }
    for(i = 0; i < segj.jsno; ++i) {
      column[used] = segj.jco[i] - 1;
      coef[3 * used] = segj.ax[i];
      coef[3 * used + 1] = segj.bx[i];
      coef[3 * used + 2] = segj.cx[i];
      ++used;
    }
  }
  if(ok) first[data.n] = used;
  if(ok && zload.nload != 0) {
    loads = malloc((size_t)data.n * sizeof(*loads));
    if(!loads) ok = 0;
    for(j = 0; ok && j < data.n; ++j) loads[j] = zload.zarray[j];
  }
  if(ok) {
    w.segments = (size_t)data.n;
    w.x = data.x; w.y = data.y; w.z = data.z; w.length = data.si; w.radius = data.bi;
    w.cab = data.cab; w.sab = data.sab; w.salp = data.salp;
    w.wavelength = data.wlam; w.rkh = rkhx; w.pec_ground = gnd.ksymp == 2;
    ok = nec2c_cuda_mom_fill(&w, first, column, coef, loads, cm, (size_t)nrow);
    if(!ok) report_failure("MoM fill");
  } else {
    fprintf(stderr, "nec2c: CUDA MoM fill: out of host memory\n");
  }
  free(first); free(column); free(coef); free(loads);
  if(!ok) stop(-1);
  if(getenv("NEC2C_CUDA_FILL_CHECK")) {
    /* Test hook: the reference's own fill of the same matrix beside the
       GPU's, largest difference relative to the largest entry on stderr. */
    complex double *ref = malloc((size_t)nrow * (size_t)nrow * sizeof(*ref));
    if(ref) {
      double diff = 0.0, big = 0.0;
      size_t e;
      __real_cmset(nrow, ref, rkhx, iexkx);
      for(e = 0; e < (size_t)nrow * (size_t)nrow; ++e) {
        if(cabs(ref[e]) > big) big = cabs(ref[e]);
        if(cabs(ref[e] - cm[e]) > diff) diff = cabs(ref[e] - cm[e]);
      }
      fprintf(stderr, "nec2c: MoM fill check: order %d, largest difference %.3e of largest entry %.6e\n",
              nrow, big > 0 ? diff / big : diff, big);
      free(ref);
    }
  }
}

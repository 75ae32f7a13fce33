/* Thin entry points into the reference nec2c, compiled together with the
 * reference's own unmodified sources into oracle/_ref/libnec2c_ref.so by
 * oracle/Makefile.  TEST INFRASTRUCTURE ONLY: it lets the tests pin the oracle
 * restatement against the real reference on the same inputs, and it backs the
 * benchmark's reference (CPU) arm.  Nothing here is reference code; each
 * function only forwards to the reference routine it names.
 */
#include "nec2c.h"
#include "shared.h"
#include "vie_fft.h"
#include "vie_kernel.h"
#include "vie_ground.h"
#include "vie_iterative.h"
#include "dense_backend.h"
#include "dielectric.h"
#include "dielectric_fft.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* The options vie_fft.c:344 (kernels) uses for near pairs. */
int ref_near_tensor(void *ctx, const size_t offset[3], double h, double k,
                    complex double out[9])
{
  vie_cuboid t = {{0, 0, 0}, {h, h, h}}, s = t;
  vie_kernel_options opt;
  complex double n[3][3];
  (void)ctx;
  vie_kernel_default_options(&opt);
  opt.relative_tolerance = 5e-7; opt.absolute_tolerance = 5e-10; opt.far_order = 16;
  for(int i = 0; i < 3; ++i) t.center[i] = h * (double)offset[i];
  if(!vie_cuboid_n(&t, &s, k, &opt, n, NULL)) return 0;
  memcpy(out, n, sizeof(n));
  return 1;
}

/* Dense pair tensor between two arbitrary lattice cells (tests/vie_fft_test.c
   fixture options). */
int ref_pair_tensor(const double tc[3], const double sc[3], double h, double k,
                    complex double out[9])
{
  vie_cuboid t, s;
  vie_kernel_options opt;
  complex double n[3][3];
  vie_kernel_default_options(&opt);
  opt.relative_tolerance = 5e-7; opt.absolute_tolerance = 5e-10; opt.far_order = 16;
  for(int i = 0; i < 3; ++i) { t.center[i] = tc[i]; s.center[i] = sc[i]; t.size[i] = s.size[i] = h; }
  if(!vie_cuboid_n(&t, &s, k, &opt, n, NULL)) return 0;
  memcpy(out, n, sizeof(n));
  return 1;
}

/* PEC-ground pair tensor, default options (tests/dielectric_fft_test.c:33). */
int ref_pair_tensor_pec(const double tc[3], const double sc[3], double h, double k,
                        complex double out[9])
{
  vie_cuboid t, s;
  complex double n[3][3];
  for(int i = 0; i < 3; ++i) { t.center[i] = tc[i]; s.center[i] = sc[i]; t.size[i] = s.size[i] = h; }
  if(!vie_cuboid_pec_n(&t, &s, k, 0, NULL, n, NULL)) return 0;
  memcpy(out, n, sizeof(n));
  return 1;
}

/* vie_fft plan through the reference's public API. */
int ref_fft_backend_set(const char *name) { return vie_fft_backend_set(name); }

void *ref_fft_create(const size_t shape[3], size_t cells, const size_t *xyz, double h,
                     double k, double er_re, double er_im, size_t limit)
{
  vie_fft_plan *p = NULL;
  if(!vie_fft_create(&p, shape, cells, xyz, h, k, er_re + I * er_im, limit)) return NULL;
  return p;
}
void ref_fft_destroy(void *p) { vie_fft_destroy(p); }
size_t ref_fft_bytes(void *p) { return vie_fft_bytes(p); }
int ref_fft_set_permittivity(void *p, size_t cell, double re, double im)
{ return vie_fft_set_permittivity(p, cell, re + I * im); }
int ref_fft_apply(void *p, const complex double *x, complex double *y)
{ vie_linear_operator op; vie_fft_operator(p, &op); return op.apply(op.context, x, y); }
int ref_fft_precondition(void *p, const complex double *x, complex double *y)
{ vie_linear_operator op; vie_fft_operator(p, &op); return op.precondition(op.precondition_context, x, y); }
int ref_fft_gmres(void *p, const complex double *b, complex double *x, size_t restart,
                  size_t maxit, double rtol, double atol, vie_gmres_report *report)
{
  vie_linear_operator op;
  vie_gmres_options o = {restart, maxit, rtol, atol};
  vie_fft_operator(p, &op);
  return vie_gmres(&op, b, x, &o, report);
}

/* vie_gmres on a dense row-major matrix with Jacobi (vie_iterative.c:228). */
int ref_dense_gmres(const complex double *a, size_t n, const complex double *b,
                    complex double *x, size_t restart, size_t maxit, double rtol,
                    double atol, vie_gmres_report *report)
{
  vie_gmres_options o = {restart, maxit, rtol, atol};
  return vie_dense_gmres(a, n, b, x, &o, report);
}

/* Classic LU: factr / solve on NEC's transposed storage (matrix.c:1313,1557),
   builtin branch. */
static void quiet_output(void) { if(!output_fp) output_fp = fopen("/dev/null", "w"); }
void ref_factr(int n, complex double *a, int *ip, int ndim)
{
  quiet_output();
  dense_backend_set("builtin");
  data.np2m = n;
  factr(n, a, ip, ndim);
}
void ref_solve(int n, complex double *a, int *ip, complex double *b, int ndim)
{
  quiet_output();
  dense_backend_set("builtin");
  data.np2m = n;
  solve(n, a, ip, b, ndim);
}
int ref_row_major_solve(complex double *a, complex double *b, size_t n)
{
  dense_backend_set("builtin");
  return dense_backend_solve_row_major(a, b, n);
}

/* dielectric_radiation_amplitude (dielectric_solver.c:124-150) of cubic cells
   of side h centred at centers[3 i], in free space (gnd.ksymp = 1). */
void dielectric_radiation_amplitude(const dielectric_mesh_result *mesh, const complex double *current,
                                    double k0, const double direction[3], complex double amplitude[3]);
int ref_radiation_amplitude(size_t cells, const double *centers, double h, const complex double *current,
                            double k0, const double direction[3], complex double out[3])
{
  dielectric_mesh_result mesh;
  dielectric_cell *c = calloc(cells ? cells : 1, sizeof(*c));
  int saved = gnd.ksymp;
  if(!c) return 0;
  memset(&mesh, 0, sizeof(mesh));
  for(size_t i = 0; i < cells; ++i)
    for(int a = 0; a < 3; ++a) { c[i].center[a] = centers[3 * i + a]; c[i].size[a] = h; }
  mesh.cells = c;
  mesh.cell_count = cells;
  gnd.ksymp = 1;
  dielectric_radiation_amplitude(&mesh, current, k0, direction, out);
  gnd.ksymp = saved;
  free(c);
  return 1;
}

/* The hybrid [C B; D V] system through the reference's own
   dielectric_fft_prepare(_pec) (dielectric_fft.c:89-175): cubic cells of
   side h centred at centers[3 i], cell i of permittivity eps[i] (one material
   per cell, no conductivity), then the conductor rows [C|B] (row-major,
   c x (c + 3 cells)) and the cross block D (row-major, 3 cells x c) written
   through dielectric_fft_entry as the reference's wire assembly does. */
void *ref_hybrid_create(size_t cells, const double *centers, double h, const complex double *eps,
                        size_t conductors, const complex double *blocks, double k0, int pec)
{
  dielectric_model model;
  dielectric_mesh_result mesh;
  dielectric_diagnostic diagnostic;
  dielectric_material *materials = calloc(cells ? cells : 1, sizeof(*materials));
  dielectric_cell *cell = calloc(cells ? cells : 1, sizeof(*cell));
  dielectric_fft_system *system = NULL;
  const size_t c = conductors, n = conductors + 3 * cells;
  int ok;
  if(!materials || !cell) { free(materials); free(cell); return NULL; }
  memset(&model, 0, sizeof(model));
  memset(&mesh, 0, sizeof(mesh));
  for(size_t i = 0; i < cells; ++i) {
    materials[i].id = (int)i + 1;
    materials[i].epsilon_r = creal(eps[i]);
    materials[i].epsilon_loss = -cimag(eps[i]);
    cell[i].material_id = (int)i + 1;
    for(int a = 0; a < 3; ++a) { cell[i].center[a] = centers[3 * i + a]; cell[i].size[a] = h; }
  }
  model.materials = materials;
  model.material_count = cells;
  mesh.cells = cell;
  mesh.cell_count = cells;
  ok = pec ? dielectric_fft_prepare_pec(&system, &model, &mesh, c, k0, 0, &diagnostic)
           : dielectric_fft_prepare(&system, &model, &mesh, c, k0, 0, &diagnostic);
  free(materials);
  free(cell);
  if(!ok) return NULL;
  for(size_t i = 0; i < n; ++i)
    for(size_t j = 0; j < n; ++j)
      if(i < c || j < c)
        *dielectric_fft_entry(system, i, j) = i < c ? blocks[i * n + j] : blocks[c * n + (i - c) * c + j];
  return system;
}
void ref_hybrid_destroy(void *system) { dielectric_fft_free(system); }
int ref_hybrid_apply(void *system, const complex double *x, complex double *y)
{ vie_linear_operator op; dielectric_fft_get_operator(system, &op); return op.apply(op.context, x, y); }
int ref_hybrid_precondition(void *system, const complex double *x, complex double *y)
{
  vie_linear_operator op;
  dielectric_fft_get_operator(system, &op);
  return op.precondition(op.precondition_context, x, y);
}
int ref_hybrid_gmres(void *system, const complex double *b, complex double *x, size_t restart,
                     size_t maxit, double rtol, double atol, vie_gmres_report *report)
{
  vie_linear_operator op;
  vie_gmres_options o = {restart, maxit, rtol, atol};
  dielectric_fft_get_operator(system, &op);
  return vie_gmres(&op, b, x, &o, report);
}

/* vie_gmres (vie_iterative.c:80-199) on caller callbacks: a NULL
   preconditioner is the identity, as in vie_iterative.h. */
int ref_callback_gmres(size_t n, vie_vector_map apply, void *apply_context, vie_vector_map precondition,
                       void *precondition_context, const complex double *b, complex double *x, size_t restart,
                       size_t maxit, double rtol, double atol, vie_gmres_report *report)
{
  vie_linear_operator op = {n, apply, apply_context, precondition, precondition_context};
  vie_gmres_options o = {restart, maxit, rtol, atol};
  return vie_gmres(&op, b, x, &o, report);
}

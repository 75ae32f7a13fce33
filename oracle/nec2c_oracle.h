/* CPU oracle for the nec2c dielectric solve path: TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithms that the CUDA backend
 * replaces.  Only the test-suite, the smoke check and the benchmark's CPU
 * baseline arm may load it; the product library never links or calls it.
 * Each function names the reference file:line it restates.
 *
 * Parity is pinned two ways (see tests/test_oracle.py):
 *   - against the reference itself, compiled from its own sources into
 *     oracle/_ref/ by oracle/Makefile (identical volume and hybrid operator,
 *     preconditioner, GMRES iterates and statuses, LU factors and far-field
 *     amplitudes on the same inputs);
 *   - against the reference's own known-answer data (tests/dense_backend_test.c
 *     3x3 system, the dense-operator checks of tests/vie_fft_test.c and
 *     tests/dielectric_fft_test.c, tests/m9-fft-skeleton-1e-8.txt integrated
 *     currents).
 */
#ifndef NEC2C_ORACLE_H
#define NEC2C_ORACLE_H
#include <complex.h>
#include <stddef.h>

typedef double complex ocplx;

/* Near-pair Green tensor provider; same contract as the CUDA library's
   nec2c_cuda_near_tensor_fn: 3x3 volume-averaged N tensor of the source cube at
   the origin seen from the testing cube at pitch*offset.  Returns 1 on success. */
typedef int (*oracle_near_fn)(void *ctx, const size_t offset[3], double pitch,
                              double k0, ocplx out[9]);

typedef struct oracle_plan oracle_plan;

/* vie_fft.c:378-441 (vie_fft_create) minus backend selection. */
int oracle_plan_create(oracle_plan **out, const size_t shape[3], size_t cells,
                       const size_t *xyz, double pitch, double k0, double er_re,
                       double er_im, oracle_near_fn near_fn, void *near_ctx);
int oracle_plan_set_permittivity(oracle_plan *p, size_t cell, double er_re, double er_im);
void oracle_plan_destroy(oracle_plan *p);
size_t oracle_plan_padded(const oracle_plan *p, int axis);
/* Copies the 6 x G transformed Green spectrum (xx,yy,zz,xy,xz,yz). */
void oracle_plan_spectrum(const oracle_plan *p, ocplx *out);
void oracle_plan_self(const oracle_plan *p, ocplx self[3]);
/* vie_fft.c:239-263 and vie_fft.c:265-273. */
int oracle_plan_apply(oracle_plan *p, const ocplx *x, ocplx *y);
int oracle_plan_precondition(oracle_plan *p, const ocplx *x, ocplx *y);
/* vie_fft.c:299-335: far-pair quadrature; returns 0 where the reference
   falls back to the certified near-pair kernel. */
int oracle_far_kernel(const size_t offset[3], double pitch, double k0, ocplx out[9]);

/* dielectric_fft.c:41-83: hybrid [C B; D V] operator, optional PEC images. */
typedef struct oracle_hybrid oracle_hybrid;
int oracle_hybrid_create(oracle_hybrid **out, oracle_plan *volume, size_t conductors,
                         size_t volume_unknowns, const ocplx *blocks, int pec);
void oracle_hybrid_destroy(oracle_hybrid *h);
int oracle_hybrid_apply(oracle_hybrid *h, const ocplx *x, ocplx *y);
int oracle_hybrid_precondition(oracle_hybrid *h, const ocplx *x, ocplx *y);

/* vie_iterative.h:9-47 contract. */
typedef int (*oracle_map)(void *ctx, const ocplx *in, ocplx *out);
typedef struct {
  int status;
  size_t iterations, operator_applications, restarts;
  double residual_norm, relative_residual;
} oracle_report;
/* vie_iterative.c:80-199 (vie_gmres). */
int oracle_gmres(size_t n, oracle_map apply, void *actx, oracle_map precondition,
                 void *pctx, const ocplx *b, ocplx *x, size_t restart,
                 size_t max_iterations, double rtol, double atol,
                 oracle_report *report);
/* Convenience wrappers binding the plan / hybrid operator. */
int oracle_plan_gmres(oracle_plan *p, const ocplx *b, ocplx *x, size_t restart,
                      size_t max_iterations, double rtol, double atol,
                      oracle_report *report);
int oracle_hybrid_gmres(oracle_hybrid *h, const ocplx *b, ocplx *x, size_t restart,
                        size_t max_iterations, double rtol, double atol,
                        oracle_report *report);

/* matrix.c:1313-1416 (factr), matrix.c:1523-1555 (solve_builtin). */
int oracle_factr(int n, ocplx *a, int *ip, int ndim);
void oracle_solve(int n, const ocplx *a, const int *ip, ocplx *b, int ndim);
/* dense_backend.c:152-190 (builtin_row_major_solve). */
int oracle_row_major_solve(ocplx *a, ocplx *b, size_t n);

/* Far-field radiation amplitude of the volume polarisation current in free
   space (dielectric_solver.c:90-150): cubic cells of side h centred at
   centers[3 i], current[3 i + c] the c-th component of cell i. */
void oracle_radiation_amplitude(size_t cells, const double *centers, double h, const ocplx *current,
                                double k0, const double direction[3], ocplx out[3]);

#endif

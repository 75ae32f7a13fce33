/* nec2c CUDA backend for NVIDIA B200 (sm_100a): public C ABI.
 *
 * A "cuda" choice behind nec2c's --fft-backend and --backend selection.  Each
 * entry point names the reference interface it replaces (file:line in the
 * N5HXR/nec2c tree).  Conventions follow the reference: int results are 1 for
 * success and 0 for failure unless stated; vectors are complex double arrays
 * in host memory owned by the caller; plans own their device storage.  The
 * library never falls back to a CPU path: without a usable CUDA device every
 * compute entry point fails and nec2c_cuda_last_error() says why.
 */
#ifndef NEC2C_CUDA_H
#define NEC2C_CUDA_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
typedef struct { double re, im; } nec2c_cuda_complex;
#else
#include <complex.h>
typedef double complex nec2c_cuda_complex;
#endif

/* ------------------------------------------------------------ runtime */
/* 1 when a CUDA device of compute capability 10.x is usable. */
int nec2c_cuda_available(void);
/* Text of the last failure on this thread ("" when none). */
const char *nec2c_cuda_last_error(void);
/* Enqueue this thread's work on the given cudaStream_t (NULL: legacy default). */
void nec2c_cuda_set_stream(void *cuda_stream);
/* Selects the CUDA device for this thread's subsequent calls (cudaSetDevice). */
int nec2c_cuda_set_device(int device);
/* Number of kernels this library has launched since it was loaded. */
unsigned long long nec2c_cuda_launch_count(void);

/* ------------------------------------------------- volume FFT operator */
/* Replaces vie_fft_backend_set (vie_fft.h:8) for the names "cuda" (plain FP64
   form) and "cuda-mixed" (FP32 transforms, FP64 vectors and epilogue).
   Returns 0 for any other name. */
int nec2c_cuda_vie_fft_backend_set(const char *name);
const char *nec2c_cuda_vie_fft_backend_name(void);

typedef struct nec2c_cuda_vie_plan nec2c_cuda_vie_plan;

/* Certified near-pair Green tensor (the reference passes vie_cuboid_n with the
   options of vie_fft.c:344): the 3x3 volume-averaged N tensor, row-major, of a
   source cube of edge pitch at the origin seen from the testing cube centred at
   pitch*offset.  Called for the displacements the far-pair quadrature does not
   certify (vie_fft.c:319-335).  Returns 1 on success. */
typedef int (*nec2c_cuda_near_tensor_fn)(void *context, const size_t offset[3], double pitch,
                                         double k0, nec2c_cuda_complex out[9]);

/* Replaces vie_fft_create (vie_fft.h:21-23, vie_fft.c:378-441): same
   validation, padding, byte accounting against byte_limit and failure
   behaviour (*out = NULL, nothing left allocated).  epsilon_r is passed as
   (re, im).  The far-pair quadrature, spectrum fill and transforms run on the
   device; near is called on the host for the remaining displacements. */
int nec2c_cuda_vie_fft_create(nec2c_cuda_vie_plan **out, const size_t shape[3], size_t cells,
                              const size_t *xyz, double pitch, double k0, double epsilon_re,
                              double epsilon_im, size_t byte_limit,
                              nec2c_cuda_near_tensor_fn near, void *near_context);
/* Replaces vie_fft_set_permittivity (vie_fft.h:26, vie_fft.c:445-455). */
int nec2c_cuda_vie_fft_set_permittivity(nec2c_cuda_vie_plan *plan, size_t cell, double epsilon_re,
                                        double epsilon_im);
/* Replaces vie_fft_destroy (vie_fft.h:27). */
void nec2c_cuda_vie_fft_destroy(nec2c_cuda_vie_plan *plan);
/* Replaces vie_fft_bytes (vie_fft.h:28): the reference's accounted bytes. */
size_t nec2c_cuda_vie_fft_bytes(const nec2c_cuda_vie_plan *plan);
/* Device memory the plan holds. */
size_t nec2c_cuda_vie_fft_device_bytes(const nec2c_cuda_vie_plan *plan);
/* Number of unknowns (3 x cells). */
size_t nec2c_cuda_vie_fft_order(const nec2c_cuda_vie_plan *plan);
/* The operator callbacks of vie_fft_operator (vie_fft.h:32): apply is
   vie_fft.c:239-263, precondition vie_fft.c:265-273.  Host vectors of
   3 x cells entries; not reentrant per plan (vie_fft.h:6). */
int nec2c_cuda_vie_fft_apply(void *plan, const nec2c_cuda_complex *x, nec2c_cuda_complex *y);
int nec2c_cuda_vie_fft_precondition(void *plan, const nec2c_cuda_complex *x,
                                    nec2c_cuda_complex *y);
/* Same product on device-resident vectors (no host copies). */
int nec2c_cuda_vie_fft_apply_device(nec2c_cuda_vie_plan *plan, const void *x_dev, void *y_dev);
/* Copies the transformed Green spectrum, 6 x padded-grid complex values in the
   order xx yy zz xy xz yz, each scaled by 1/grid (validation hook). */
int nec2c_cuda_vie_fft_spectrum(nec2c_cuda_vie_plan *plan, nec2c_cuda_complex *out);

/* Far-field radiation amplitude of a volume polarisation current in free
   space, the volume term of dielectric_radiation_amplitude
   (dielectric_solver.c:90-150): for each unit direction d (3 doubles each,
   host), amplitude = i k c0 mu0 / (4 pi) ((I x d) x d) with
   I = sum over cells of J_cell h^3 prod_a sinc(k d_a h / 2) exp(+i k d.r_cell),
   r_cell = origin + h x the cell's lattice index (h, k: the plan's pitch and
   wavenumber).  current_dev holds 3 x cells complex values on the device (a
   solve's x); amplitude receives 3 complex values per direction (host).  Not
   for plans with PEC images (the ground terms are not built). */
int nec2c_cuda_vie_fft_radiation_device(nec2c_cuda_vie_plan *plan, const double origin[3], const void *current_dev,
                                        size_t count, const double *directions, nec2c_cuda_complex *amplitude);

/* FFT pass schedule.  A product runs five line-FFT passes: 0 z forward with
   the cell scatter, 1 y forward, 2 x forward + Green-tensor product + x
   inverse, 3 y inverse, 4 z inverse with the permittivity epilogue.  Each has
   a tile height (lines per CTA) and a radix split L = R1 x R2.  With
   autotuning on (the default; NEC2C_CUDA_FFT_AUTOTUNE=0 in the environment
   turns it off) nec2c_cuda_vie_fft_create times the candidates on the new
   plan and keeps the fastest, cached per grid shape for the process.  The
   reference plans its FFTW transforms with FFTW_ESTIMATE (vie_fft.c:227-235),
   i.e. untimed; this is the measured counterpart.  Every schedule computes
   the same transform; the radix split changes the rounding only. */
void nec2c_cuda_vie_fft_autotune(int enable);
int nec2c_cuda_vie_fft_autotune_enabled(void);
/* Re-plans one plan's schedule: measure = 0 the heuristic, 1 timed (reusing
   a cached choice for the same shape), 2 timed afresh.  Returns 1 on success. */
int nec2c_cuda_vie_fft_tune(nec2c_cuda_vie_plan *plan, int measure);
/* Schedule in use for the FP64 (fp64 != 0) or FP32 transforms: tiles[i]
   lines per tile and r1[i] the first radix of pass i.  Returns 1 when that
   precision was timed or pinned, 0 when it runs the heuristic, -1 on a bad
   argument. */
int nec2c_cuda_vie_fft_schedule(nec2c_cuda_vie_plan *plan, int fp64, int tiles[5], int r1[5]);
/* Pins a schedule, e.g. one read back from an earlier run so that results
   repeat bit for bit across processes.  Heights: whole lattice columns
   (multiples of 3 lines, at most 96) for passes 0 and 4, powers of two up to
   64 for passes 1-3, each within 100 KB of shared memory; r1 one of the
   splits on offer for the pass's length.  Returns 0 (schedule unchanged) on
   anything else. */
int nec2c_cuda_vie_fft_set_schedule(nec2c_cuda_vie_plan *plan, int fp64, const int tiles[5], const int r1[5]);
/* Fused yz-plane passes.  Where the padded y and z axes have one length P of
   32, 64 or 128, passes 0-1 and 3-4 can instead run as two kernels that
   transform a whole lattice plane in shared memory (P = 2Q: each plane is four
   Q x Q transforms of the parity classes of (ky, kz); the inverse sums them in
   a four-CTA cluster), so a product is three launches.  The tuner times both
   forms on a new plan and keeps the plane passes when they are at least 3%
   faster; without autotuning they are used wherever they apply.  planes()
   returns 1 (plane passes), 0 (five passes) or -1 (not applicable, or a bad
   argument); set_planes pins the choice (with the schedule above, for
   results that repeat bit for bit) and returns 0 when not applicable.  The
   forms compute the same product; they round differently. */
int nec2c_cuda_vie_fft_planes(nec2c_cuda_vie_plan *plan, int fp64);
int nec2c_cuda_vie_fft_set_planes(nec2c_cuda_vie_plan *plan, int fp64, int planes);

/* --------------------------------------- hybrid conductor + volume system */
typedef struct nec2c_cuda_hybrid nec2c_cuda_hybrid;
/* Device half of dielectric_fft_prepare / dielectric_fft_prepare_pec
   (dielectric_fft.h:10-18): the [C B; D V] operator over an existing volume
   plan (NULL when there are no cells).  With pec != 0 the plan holds the
   physical cells followed by their images (dielectric_fft.c:137-154) and
   volume_unknowns counts the physical ones only. */
int nec2c_cuda_hybrid_create(nec2c_cuda_hybrid **out, nec2c_cuda_vie_plan *volume,
                             size_t conductors, size_t volume_unknowns, int pec);
void nec2c_cuda_hybrid_destroy(nec2c_cuda_hybrid *system);
/* Uploads the blocks the caller assembled through dielectric_fft_entry
   (dielectric_fft.c:34-40 layout: c rows of c+v, then v rows of c). */
int nec2c_cuda_hybrid_set_blocks(nec2c_cuda_hybrid *system, const nec2c_cuda_complex *blocks);
size_t nec2c_cuda_hybrid_order(const nec2c_cuda_hybrid *system);
/* Operator callbacks of dielectric_fft_get_operator (dielectric_fft.c:41-83). */
int nec2c_cuda_hybrid_apply(void *system, const nec2c_cuda_complex *x, nec2c_cuda_complex *y);
int nec2c_cuda_hybrid_precondition(void *system, const nec2c_cuda_complex *x,
                                   nec2c_cuda_complex *y);

/* --------------------------------------------------------------- GMRES */
/* Same layouts as vie_gmres_options / vie_gmres_report (vie_iterative.h:20-47);
   status uses vie_iterative_status values. */
typedef struct {
  size_t restart;
  size_t maximum_iterations;
  double relative_tolerance;
  double absolute_tolerance;
} nec2c_cuda_gmres_options;
typedef struct {
  int status;
  size_t iterations;
  size_t operator_applications;
  size_t restarts;
  double residual_norm;
  double relative_residual;
} nec2c_cuda_gmres_report;
/* Replaces vie_gmres (vie_iterative.h:55-57) when the operator is a CUDA plan
   or hybrid system: right-preconditioned restarted GMRES, two MGS passes,
   complex Givens, true residual at every restart, run device-resident.  NULL
   options mean the reference defaults {30, 300, 1e-12, 0}.  x is the initial
   guess and is updated even on failure. */
int nec2c_cuda_gmres_plan(nec2c_cuda_vie_plan *plan, const nec2c_cuda_complex *b,
                          nec2c_cuda_complex *x, const nec2c_cuda_gmres_options *options,
                          nec2c_cuda_gmres_report *report);
int nec2c_cuda_gmres_hybrid(nec2c_cuda_hybrid *system, const nec2c_cuda_complex *b,
                            nec2c_cuda_complex *x, const nec2c_cuda_gmres_options *options,
                            nec2c_cuda_gmres_report *report);
/* The same solves on device-resident b and x (complex double, order entries). */
int nec2c_cuda_gmres_plan_device(nec2c_cuda_vie_plan *plan, const void *b_dev, void *x_dev,
                                 const nec2c_cuda_gmres_options *options,
                                 nec2c_cuda_gmres_report *report);
int nec2c_cuda_gmres_hybrid_device(nec2c_cuda_hybrid *system, const void *b_dev, void *x_dev,
                                   const nec2c_cuda_gmres_options *options,
                                   nec2c_cuda_gmres_report *report);

/* ------------------------------------------------- ragged batch of plans */
typedef struct nec2c_cuda_vie_batch nec2c_cuda_vie_batch;
/* Many volume plans (frequencies or geometries with ragged lattices, padded
   axes up to 256, all with the same transform precision, each at most once)
   solved together: every FFT pass of a GMRES step is one launch over all the
   plans, every Gram-Schmidt sweep one launch over all the systems, and the
   steps of a restart cycle run as CUDA graphs of five steps, the cycle ending
   after the graph in which the last system stopped.  The reference solves such a sweep
   one vie_gmres at a time in its frequency workers (main.c:586-760); there is
   no counterpart function.  The plans stay the caller's, must outlive the
   batch and must not be used elsewhere while a batched call runs;
   permittivity changes made to them are picked up by the next call. */
int nec2c_cuda_vie_batch_create(nec2c_cuda_vie_batch **out, nec2c_cuda_vie_plan *const *plans, size_t count);
/* The same for hybrid conductor + volume systems (dielectric_fft.c: wire
   segments beside a dielectric body, each with its volume plan and its blocks
   uploaded): the conductor and cross rows of all systems are one launch each
   as well.  A system's vector is its conductor unknowns, then its volume
   unknowns, as nec2c_cuda_hybrid_apply orders them. */
int nec2c_cuda_hybrid_batch_create(nec2c_cuda_vie_batch **out, nec2c_cuda_hybrid *const *systems, size_t count);
void nec2c_cuda_vie_batch_destroy(nec2c_cuda_vie_batch *batch);
/* Unknowns of the batch (sum of the systems' orders); system q's entries
   start at nec2c_cuda_vie_batch_offset(batch, q). */
size_t nec2c_cuda_vie_batch_order(const nec2c_cuda_vie_batch *batch);
size_t nec2c_cuda_vie_batch_systems(const nec2c_cuda_vie_batch *batch);
size_t nec2c_cuda_vie_batch_offset(const nec2c_cuda_vie_batch *batch, size_t plan);
/* Schedule of the batched FFT passes.  Per pass: scale[i] in -1..1 halves,
   keeps or doubles the batch's tile height, and variant[i] 0/1 picks the
   default or the transposed radix split.  With autotuning on,
   nec2c_cuda_vie_batch_create times the candidates on the batch and keeps the
   fastest.  set_schedule pins a schedule and returns 0 (schedule unchanged)
   when it cannot be built. */
int nec2c_cuda_vie_batch_schedule(const nec2c_cuda_vie_batch *batch, int scale[5], int variant[5]);
int nec2c_cuda_vie_batch_set_schedule(nec2c_cuda_vie_batch *batch, const int scale[5], const int variant[5]);
/* y = A x of every plan (vie_fft.c:239-263 per plan) on device vectors of the
   batch's order. */
int nec2c_cuda_vie_batch_apply_device(nec2c_cuda_vie_batch *batch, const void *x_dev, void *y_dev);
/* vie_gmres (vie_iterative.h:55-57) on every plan at once with the same
   options (restart at most 30): right-preconditioned restarted GMRES, complex
   Givens, true residual at every restart, each system stopping on its own
   test; reports[q] as vie_gmres reports plan q's solve.  The Arnoldi process
   is classical Gram-Schmidt, with a second pass always (FP64 plans) or on a
   tenfold cancellation (FP32 transforms).  b_dev, x_dev: device vectors of
   the batch's order; x is the initial guess and is updated.  Returns 1 when
   every system converged. */
int nec2c_cuda_gmres_batch_device(nec2c_cuda_vie_batch *batch, const void *b_dev, void *x_dev,
                                  const nec2c_cuda_gmres_options *options, nec2c_cuda_gmres_report *reports);
/* The same with host vectors: b[q] and x[q] hold the order of system q. */
int nec2c_cuda_gmres_batch(nec2c_cuda_vie_batch *batch, const nec2c_cuda_complex *const *b,
                           nec2c_cuda_complex *const *x, const nec2c_cuda_gmres_options *options,
                           nec2c_cuda_gmres_report *reports);

/* ------------------------------------------------------------ dense LU */
/* Replaces dense_backend_set (dense_backend.h:14) for "cuda" (FP64 LU) and
   "cuda-mixed" (split-precision tensor-core update plus FP64 refinement in the
   solve).  Returns 0 for any other name. */
int nec2c_cuda_dense_backend_set(const char *name);
const char *nec2c_cuda_dense_backend_name(void);
/* Replaces dense_backend_factor_classic (dense_backend.h:22-23), called by
   factr (matrix.c:1318): factors NEC's transposed storage in place.  That
   storage is the algebraic matrix row-major; the factors are its LU in the
   same layout with 1-based pivots chosen by the builtin factr's rule (largest
   |.|^2, later row on ties), L in the getrf row convention.  Only this
   backend's solves consume them.  Returns 1, or 0 when singular/failed. */
int nec2c_cuda_dense_factor_classic(size_t order, nec2c_cuda_complex *matrix,
                                    size_t leading_dimension, int *pivots);
/* Replaces dense_backend_solve_classic(_many) (dense_backend.h:24-32), called by
   solve (matrix.c:1561) and solves (matrix.c:1683). */
int nec2c_cuda_dense_solve_classic(size_t order, const nec2c_cuda_complex *matrix,
                                   size_t leading_dimension, const int *pivots,
                                   nec2c_cuda_complex *rhs);
int nec2c_cuda_dense_solve_classic_many(size_t order, const nec2c_cuda_complex *matrix,
                                        size_t leading_dimension, const int *pivots,
                                        nec2c_cuda_complex *rhs, size_t rhs_stride,
                                        size_t rhs_count);
/* Replaces dense_backend_solve_row_major (dense_backend.h:36-37): row-major
   system, pivot rule of dense_backend.c:152-190 (largest |.|, first row on
   ties, pivot must exceed 64 eps), solution returned in rhs.  The matrix is
   left unchanged. */
int nec2c_cuda_dense_solve_row_major(nec2c_cuda_complex *matrix, nec2c_cuda_complex *rhs,
                                     size_t order);
/* No single counterpart in the reference: factr + solve (matrix.c:1313-1416,
   1523-1555) of count independent systems (the wire blocks of many
   frequencies or geometries) at once.  Systems of order <= 64 are factored
   and solved together in one launch (one CTA per system).  Under the "cuda"
   backend the larger ones up to nec2c_cuda_dense_batch_max_order() are
   factored in lockstep: each panel step is one launch per kernel for all of
   them (a thread-block cluster per system for the panel), then they are
   solved together; they get the pivots and factors each would get alone.
   The others (larger, or under "cuda-mixed") run through the classic factor
   and solve.  Each matrix is NEC's storage
   (leading dimension lds[i]) and receives its factors as
   nec2c_cuda_dense_factor_classic writes them; pivots[i] (optional) the
   1-based pivots; rhs[i] the solution.  status[i] is 1 when system i was
   solved, 0 when singular or failed; returns 1 when all were solved. */
int nec2c_cuda_dense_solve_batched(size_t count, const size_t *orders, nec2c_cuda_complex *const *matrices,
                                   const size_t *lds, int *const *pivots, nec2c_cuda_complex *const *rhs,
                                   int *status);
/* Largest order the lockstep batch takes on the current device (4096 where
   16-CTA clusters can run, else 2048). */
size_t nec2c_cuda_dense_batch_max_order(void);
/* Drops the device copies kept between a factor and its solves. */
void nec2c_cuda_dense_release(void);
/* No counterpart in the reference (diagnostic of the "cuda-mixed" form):
   refinement steps the last split-precision solve took, -1 when it fell back
   to an FP64 factorisation, 0 before any. */
int nec2c_cuda_dense_last_refinement(void);
/* No counterpart in the reference.  The classic factor above, for callers that
   must not allocate device memory during the call (a process whose GPU memory
   belongs to its own pool allocator, or a loop that cannot absorb cudaMalloc's
   device synchronisation).  matrix_dev and pivots_dev are device pointers the
   caller owns: NEC's storage (the algebraic matrix row-major, leading
   dimension >= order) factored in place, and 1-based pivots written to
   pivots_dev.  It is always the plain FP64 factor: the same pivots and
   factors as nec2c_cuda_dense_factor_classic under the "cuda" backend,
   whichever backend name is selected.  The work runs on this thread's stream
   and the call returns when it is done.  Scratch is one 19 KiB array inside
   the library that each GPU using it holds until exit; calls that overlap on
   the GPU share it and race.  Each call looks up that array's address in the
   current context; the first lookup loads the library's device code, so make
   the first call on a device before any stream capture.  Orders above
   NEC2C_CUDA_STATIC_LU_MAX_ORDER are rejected.  Returns 1, or 0 when
   singular, too large or failed. */
#define NEC2C_CUDA_STATIC_LU_MAX_ORDER 4096
int nec2c_cuda_dense_factor_device_static(size_t order, nec2c_cuda_complex *matrix_dev,
                                          size_t leading_dimension, int *pivots_dev);

/* ------------------------------------------- wire <-> volume coupling */
/* The wires of a NEC model as NEC holds them while a hybrid system is
   assembled (dielectric_wire.c: geometry scaled to wavelengths): segment
   centres, lengths and radii in wavelengths, direction cosines, the
   wavelength in metres, NEC's lumped-element distance rkh (wavelengths, the
   RK card, 1 by default) and whether a perfectly conducting ground plane
   (GN 1) mirrors every segment. */
typedef struct {
  size_t segments;
  const double *x, *y, *z;
  const double *length, *radius;
  const double *cab, *sab, *salp;
  double wavelength;
  double rkh;
  int pec_ground;
} nec2c_cuda_wire_model;
/* Replaces dw_assemble_wire_to_volume (dielectric_wire.c:396-510) for the
   NEC-2 wire engine with the classic thin-wire kernel, in free space or over
   a perfect ground: for each of columns conductor unknowns, whose basis
   currents sources holds (per segment the constant, sine and cosine
   coefficients cabc gives for a unit vector, dw_prepare_conductor_sources),
   the NEC field (nefld/efld, fields.c:38-253, 1123-1380) averaged over each
   cell by a 6-point Gauss rule per axis, times -i omega eps0 chi[cell].
   centers and sizes hold 3 doubles per cell (m); out receives columns rows
   of 3 x cells values (row column, entry 3 cell + component).  Returns 1, or
   0 with the reason in nec2c_cuda_last_error(). */
int nec2c_cuda_coupling_wire_to_volume(const nec2c_cuda_wire_model *wires, size_t columns,
                                       const nec2c_cuda_complex *sources, size_t cells,
                                       const double *centers, const double *sizes,
                                       const nec2c_cuda_complex *chi, double omega, nec2c_cuda_complex *out);
/* Replaces the wire-row loop of dielectric_solve_conductor_coupled
   (dielectric_wire.c:1164-1213) in free space or over a perfect ground: the
   point-tested N dyad of each cell (dw_point_cuboid_n, dielectric_wire.c:
   101-138, 193-201; 10-point Gauss rule per axis) at each segment centre
   (centers_m, metres), projected on the segment direction (tangents) and
   divided by i omega eps0.  out receives segments rows of 3 x cells values.
   Returns 1, or 0 with the reason set. */
int nec2c_cuda_coupling_volume_to_wire(size_t segments, const double *centers_m, const double *tangents,
                                       size_t cells, const double *cell_centers, const double *cell_sizes,
                                       double k0, double omega, int pec_ground, nec2c_cuda_complex *out);

/* ------------------------------------------------------- wire MoM fill */
/* Replaces cmset (matrix.c:48-195) for wires alone (no patches, no symmetry,
   one block in core), the NEC-2 wire engine with the classic thin-wire
   kernel, free space or a perfect ground: the wire-wire interaction matrix
   of cmww (matrix.c:742-966) with the transposed fill cmset uses, plus the
   segment loads (matrix.c:107-121).  wires->wavelength is not used.
   Basis functions per source segment j (the reference's trio):
   basis_first[j] .. basis_first[j+1]-1 index basis_column (0-based, < the
   segment count) and basis_coef (3 per entry: the constant, sine and cosine
   coefficients of that basis function on segment j).  loads: the load
   impedance of every segment as cmset takes it (zload.zarray), or NULL.
   cm receives rows 0 .. segments-1 of nrow values each (nrow >= segments):
   entry (i, b) at cm[i * nrow + b], the field of basis b tested on segment i,
   zeros beyond column segments-1.  Returns 1, or 0 with the reason in
   nec2c_cuda_last_error(). */
int nec2c_cuda_mom_fill(const nec2c_cuda_wire_model *wires, const size_t *basis_first, const int *basis_column,
                        const nec2c_cuda_complex *basis_coef, const nec2c_cuda_complex *loads,
                        nec2c_cuda_complex *cm, size_t nrow);

/* ------------------------------------------------------- request server */
/* No single counterpart in the reference: replaces the fork()ed frequency
   workers (main.c:586-760) and their memory-capped job count
   (concurrency.c:118-171) for a stream of solve requests on one GPU.  Worker
   threads, each with its own CUDA stream, take queued requests as their
   device footprint fits the budget left by the requests in flight; the work
   of requests in flight overlaps on the device.  Dense requests factor and
   solve a private device copy of the matrix (the host matrix is not
   modified; rhs receives the solutions); volume requests run GMRES on a plan
   or hybrid system the caller created and keeps resident across requests.
   Batch requests solve every system of a plan batch at once (a frequency
   sweep of one model).  A plan is not reentrant, and hybrid systems and
   batches run on their plans' work grids, so two requests that reach the
   same plan (directly, through a hybrid system or in a batch) never run at
   the same time. */
enum { NEC2C_CUDA_REQUEST_DENSE = 1, NEC2C_CUDA_REQUEST_VOLUME = 2, NEC2C_CUDA_REQUEST_BATCH = 3 };
typedef struct {
  int kind;
  /* dense: NEC's storage (order x order, leading dimension ld) and
     rhs_count right-hand sides (stride rhs_stride), overwritten with x */
  size_t order, ld, rhs_count, rhs_stride;
  const nec2c_cuda_complex *matrix;
  nec2c_cuda_complex *rhs;
  /* volume: exactly one of plan / system; x is the initial guess and the
     result, as for nec2c_cuda_gmres_plan */
  nec2c_cuda_vie_plan *plan;
  nec2c_cuda_hybrid *system;
  const nec2c_cuda_complex *b;
  nec2c_cuda_complex *x;
  nec2c_cuda_gmres_options options;
  /* filled by the server */
  int status;                      /* 1 solved, 0 failed (error holds why) */
  int done;
  unsigned skipped;
  nec2c_cuda_gmres_report report;  /* volume: GMRES report; dense: iterations = refinement steps */
  size_t footprint;                /* device bytes admitted for it */
  double queued_s, started_s, finished_s;   /* CLOCK_MONOTONIC seconds */
  char error[128];
  /* batch: b and x hold the batch's order of values in batch order (host);
     reports receives one report per system; the request's report holds the
     worst status, the largest iteration and restart counts, the sum of the
     products and the largest relative residual */
  nec2c_cuda_vie_batch *batch;
  nec2c_cuda_gmres_report *reports;
  /* filled by the server: how many volume requests ran together in the
     batched solve this one was merged into (1: it ran alone) */
  size_t merged;
} nec2c_cuda_request;
typedef struct nec2c_cuda_server nec2c_cuda_server;
/* slots worker threads on device; device_budget 0 means the free device
   memory less max(1/5, 1 GiB) (the reserve of concurrency.c:131-136).
   split != 0 selects the split-precision dense form. */
int nec2c_cuda_server_create(nec2c_cuda_server **out, int device, int slots, size_t device_budget, int split);
/* Queues a request (caller-owned until it is done); returns at once. */
int nec2c_cuda_server_submit(nec2c_cuda_server *server, nec2c_cuda_request *request);
/* Blocks until the request is done; returns its status. */
int nec2c_cuda_server_wait(nec2c_cuda_server *server, nec2c_cuda_request *request);
/* Blocks until every submitted request is done. */
int nec2c_cuda_server_drain(nec2c_cuda_server *server);
size_t nec2c_cuda_server_budget(const nec2c_cuda_server *server);
/* Lets the server merge queued volume requests: a worker that takes a volume
   request whose plan (or hybrid system) is one of batch's systems also takes
   every other queued volume request on a system of the same batch with the
   same GMRES options (restart <= 30), and solves them as one batched solve
   in which the batch's other systems stay idle (the batched GMRES, to the
   same tolerances as the single-system solve).  Each request gets its
   own report, x and status; `merged` tells how many ran together.  The
   batch must outlive the server; registering it twice is refused. */
int nec2c_cuda_server_merge_batch(nec2c_cuda_server *server, nec2c_cuda_vie_batch *batch);
/* Lets the server merge queued dense requests: a worker that takes a dense
   request of order up to nec2c_cuda_dense_batch_max_order() also takes the
   queued dense requests of the same size class (orders up to 256, 512, 1024,
   2048 or 4096: the cluster size of the first panel), as many as fit the
   device budget and at most max_systems in all, and factors and solves their
   private matrix copies as one lockstep batch: one launch per kernel and
   panel step for all of them, each system's pivots and factors as its own
   factorisation gives them.  On an FP64 server the batch is the FP64 form; on
   a split-precision server it factors FP32 copies with tensor-core (3xTF32)
   updates and refines every system's solution in FP64 (report.iterations:
   its refinement steps).  Each request gets its own status; `merged` tells
   how many ran together.  max_systems < 2 turns merging off. */
int nec2c_cuda_server_merge_dense(nec2c_cuda_server *server, size_t max_systems);
/* Drains, stops the workers and frees the server. */
void nec2c_cuda_server_destroy(nec2c_cuda_server *server);

#ifdef __cplusplus
}
#endif
#endif

/* Device layer of the nec2c CUDA backend: C-linkage entry points implemented
 * in CUDA C++ (the .cu files of csrc/) and called by the C host layer (the .c
 * files of host/).  Not part of the public ABI (that is include/nec2c_cuda.h).
 * All pointers named *_dev are device pointers; everything else is host
 * memory. */
#ifndef NEC2C_DEVICE_API_H
#define NEC2C_DEVICE_API_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Error text of the last failed call on this thread. */
const char *n2d_last_error(void);
void n2c_set_error(const char *fmt, ...);
/* Stream all work of this thread is enqueued on (NULL = legacy default). */
void n2d_set_stream(void *stream);
void *n2d_get_stream(void);
int n2d_sync(void);
/* Device flag checked by operator kernels (0 = skip the launch's work). */
void n2d_set_gate(const int *gate_dev);
/* Device buffers and copies on the current stream. */
void *n2d_alloc(size_t bytes);
void n2d_free(void *p);
/* Stream-ordered allocation on this thread's stream (pool keeps freed memory;
   no device-wide synchronisation).  Free with n2d_free_async on the same
   stream. */
void *n2d_alloc_async(size_t bytes);
void n2d_free_async(void *p);
/* A new non-blocking stream / its release. */
void *n2d_stream_create(void);
void n2d_stream_destroy(void *stream);
/* cudaMemGetInfo of the current device. */
int n2d_mem_info(size_t *free_bytes, size_t *total_bytes);
int n2d_upload(void *dst_dev, const void *src, size_t bytes);
int n2d_download(void *dst, const void *src_dev, size_t bytes);
int n2d_memset(void *dst_dev, int value, size_t bytes);
int n2d_copy_d2d(void *dst_dev, const void *src_dev, size_t bytes);
/* Pitched copies (cudaMemcpy2D semantics: width bytes per row, rows rows). */
int n2d_upload2d(void *dst_dev, size_t dpitch, const void *src, size_t spitch, size_t width,
                 size_t rows);
int n2d_download2d(void *dst, size_t dpitch, const void *src_dev, size_t spitch, size_t width,
                   size_t rows);
/* 1 when a compute capability 10.x device is present. */
int n2d_device_ok(void);
int n2d_set_device(int device);
/* Kernels this library has launched since load (for the launch-count check). */
unsigned long long n2d_launch_count(void);

/* ---- volume FFT operator (vie_fft.c's plan) ---- */
typedef struct n2d_vie n2d_vie;
/* shape = lattice extent, padded = FFT grid (each a power of two <= 1024,
   >= 2*shape-1); cell_box[c] = (x*shape1 + y)*shape2 + z. */
int n2d_vie_create(n2d_vie **out, const long long shape[3], const long long padded[3],
                   long long cells, const int *cell_box, const double *const twiddles[3],
                   int fp32);
/* Gauss-Legendre nodes / weights on [0,1], orders 4, 6, 8, 12 (4 x 12 each). */
int n2d_vie_set_gauss(const double *nodes, const double *weights);
void n2d_vie_destroy(n2d_vie *p);
size_t n2d_vie_device_bytes(const n2d_vie *p);
int n2d_vie_fp32(const n2d_vie *p);
long long n2d_vie_cells(const n2d_vie *p);
/* Green spectrum.  offsets: sorted displacements a>=b>=c in enumeration order
   (a outer, then b, then c); sorted_shape: shape sorted descending.  The far
   kernel fills what it can and flags (0) the entries that need the caller's
   certified near-pair tensor; put_tensors supplies those (6 complex each, xx yy
   zz xy xz yz, already symmetrised and with the reference's zeroing applied). */
int n2d_vie_far_tensors(n2d_vie *p, long long count, const int *offsets,
                        const long long sorted_shape[3], double pitch, double k0,
                        int *far_ok);
int n2d_vie_put_tensors(n2d_vie *p, long long count, const long long *index,
                        const double *tensors);
int n2d_vie_finish_spectrum(n2d_vie *p);
/* Downloads the transformed spectrum (6 x G, FP64, scaled by 1/G). */
int n2d_vie_read_spectrum(n2d_vie *p, double *out);
/* Per-cell permittivity (2 doubles each) and self terms (3 complex). */
int n2d_vie_set_eps(n2d_vie *p, const double *eps, const double *self);
/* y_dev = A z where z = x_dev (or x_dev ./ diag when precondition_input).
   When norm_dev is non-NULL, the sum of |y|^2 is written there (and a
   non-finite y sets *flag_dev to 1 when flag_dev is non-NULL).  Mixed plans
   transform in FP32 unless full_precision is set (FP64 spectrum and grids). */
int n2d_vie_apply(n2d_vie *p, const double *x_dev, double *y_dev, int precondition_input,
                  double *norm_dev, int *flag_dev, int full_precision);
/* y_dev = x_dev ./ (eps - (eps-1) self). */
int n2d_vie_precondition(n2d_vie *p, const double *x_dev, double *y_dev);
const double *n2d_vie_diag(const n2d_vie *p);
/* PEC image embedding: the plan's cells are physical_cells physical cells
   followed by their images; apply/precondition then act on the physical half. */
void n2d_vie_set_mirror(n2d_vie *p, long long physical_cells);
/* Pass schedule (tile height and radix split of the five matvec passes).
   measure: 0 the heuristic, 1 timed on this plan (a cached choice for the
   same grid shape and precision is reused), 2 timed afresh.  Plans are tuned
   with measure = 1 at the end of n2d_vie_finish_spectrum while autotuning is
   enabled (the default; NEC2C_CUDA_FFT_AUTOTUNE=0 disables it). */
int n2d_vie_tune(n2d_vie *p, int measure);
void n2d_vie_autotune(int enable);
int n2d_vie_autotune_enabled(void);
/* Far-field radiation amplitude (dielectric_solver.c:90-150, free space) of
   the cell current current_dev (3 per cell) for count directions dirs_dev
   (3 per direction) into out_dev (3 complex per direction); cell centres are
   origin + h x lattice index. */
int n2d_vie_radiation(n2d_vie *p, const double *current_dev, const double origin[3], double h, double k0,
                      const double *dirs_dev, long long count, double *out_dev);
/* Lines per tile and R1 (R2 = L / R1) of each pass for precision prec
   (0 FP32, 1 FP64); returns 1 when the schedule was measured. */
int n2d_vie_schedule(n2d_vie *p, int prec, int *tiles, int *r1);
/* Pins a schedule (heights and splits the tuner would try; 0 otherwise). */
int n2d_vie_set_schedule(n2d_vie *p, int prec, const int *tiles, const int *r1);
/* Fused yz-plane passes for precision prec: 1 in use, 0 the five passes, -1
   not applicable to the grid; set returns 0 (error set) when not applicable. */
int n2d_vie_planes(n2d_vie *p, int prec);
int n2d_vie_set_planes(n2d_vie *p, int prec, int planes);

/* ---- hybrid [C B; D V] operator (dielectric_fft.c) ---- */
typedef struct n2d_hybrid n2d_hybrid;
int n2d_hybrid_create(n2d_hybrid **out, n2d_vie *volume, long long conductors,
                      long long volume_unknowns, int pec);
void n2d_hybrid_destroy(n2d_hybrid *h);
/* Uploads the dense blocks (c*(c+v) + v*c complex, dielectric_fft.c:34-40). */
int n2d_hybrid_upload_blocks(n2d_hybrid *h, const double *blocks);
int n2d_hybrid_apply(n2d_hybrid *h, const double *x_dev, double *y_dev, int precondition_input,
                     double *norm_dev, int *flag_dev, int full_precision);
int n2d_hybrid_precondition(n2d_hybrid *h, const double *x_dev, double *y_dev);
long long n2d_hybrid_order(const n2d_hybrid *h);
/* 0 when a conductor diagonal is zero or non-finite (dielectric_fft.c:77-81). */
int n2d_hybrid_precondition_ok(const n2d_hybrid *h);

/* ---- device-resident GMRES (vie_iterative.c) ---- */
typedef struct {
  int status;
  size_t iterations, operator_applications, restarts;
  double residual_norm, relative_residual;
} n2d_gmres_report;
/* kind 0: volume plan, kind 1: hybrid system.  b, x are host vectors. */
int n2d_gmres(int kind, void *op, long long n, const double *b, double *x,
              size_t restart, size_t maximum_iterations, double rtol, double atol,
              n2d_gmres_report *report);
/* Same with device-resident b and x. */
int n2d_gmres_dev(int kind, void *op, long long n, const double *b_dev, double *x_dev,
                  size_t restart, size_t maximum_iterations, double rtol, double atol,
                  n2d_gmres_report *report);

/* ---- ragged batch of volume plans (vie_batch.cu) ---- */
typedef struct n2d_vie_batch n2d_vie_batch;
/* Plans with the same transform precision, padded axes <= 256, each at most
   once; their permittivities must have been uploaded (self terms set). */
int n2d_vie_batch_create(n2d_vie_batch **out, n2d_vie *const *plans, long long count);
/* Hybrid conductor + volume systems (each with a volume plan, blocks
   uploaded) batched the same way. */
int n2d_hybrid_batch_create(n2d_vie_batch **out, n2d_hybrid *const *systems, long long count);
void n2d_vie_batch_destroy(n2d_vie_batch *b);
/* Unknowns of the batch and the offset of plan q's vector in it. */
long long n2d_vie_batch_order(const n2d_vie_batch *b);
long long n2d_vie_batch_offset(const n2d_vie_batch *b, long long q);
/* y = A x of every plan (transform precision, no preconditioning), five
   launches in all. */
int n2d_vie_batch_apply(n2d_vie_batch *b, const double *x_dev, double *y_dev);
/* Schedule of the batched passes (tile height scale -1..1 and radix split 0/1
   per pass), chosen by the batch tuner at creation; pinning rebuilds it. */
void n2d_vie_batch_schedule(const n2d_vie_batch *b, int *scale, int *variant);
int n2d_vie_batch_set_schedule(n2d_vie_batch *b, const int *scale, const int *variant);
/* GMRES(restart <= 30) on every plan in lockstep; reports[q] per system.
   idle (NULL, or one flag per system): systems flagged non-zero take no part
   and their reports stay "invalid".  Returns 1 when every other system
   converged. */
int n2d_gmres_batch_dev(n2d_vie_batch *b, const double *b_dev, double *x_dev, size_t restart,
                        size_t maximum_iterations, double rtol, double atol, const unsigned char *idle,
                        n2d_gmres_report *reports);

/* ---- dense LU (matrix.c factr/solve, dense_backend.c) ---- */
/* Factor order x order in place on the device: the algebraic matrix
   row-major with leading dim ld (NEC's transposed column-major storage),
   partial pivoting.  rule 0: largest |.|^2, later row wins ties (factr);
   rule 1: largest |.|, first row wins, pivot must exceed 64 eps (row-major
   builtin).  pivots_dev receives 1-based pivot rows; *info_host the first
   zero/rejected pivot (1-based) or 0.  precision is ignored (FP64). */
int n2d_lu_factor(double *a_dev, long long order, long long ld, int *pivots_dev, int rule,
                  int precision, int *info_host);
/* Split-precision form: the same factorisation of a complex FP32 matrix
   (float pairs, ld even); panels and triangular solves compute in FP64, the
   trailing update runs on the tensor cores (3xTF32). */
int n2d_lu_factor32(float *a_dev, long long order, long long ld, int *pivots_dev, int rule, int *info_host);
/* Solve with factors from n2d_lu_factor: interchanges + unit-lower forward +
   upper back substitution, for nrhs columns of b_dev (leading dim ldb). */
int n2d_lu_solve(const double *a_dev, long long order, long long ld, const int *pivots_dev,
                 double *b_dev, long long ldb, long long nrhs);
/* The same with FP32 factors (FP64 arithmetic and right-hand sides). */
int n2d_lu_solve32(const float *a_dev, long long order, long long ld, const int *pivots_dev,
                   double *b_dev, long long ldb, long long nrhs);
/* Complex block copies between FP64 and FP32 (rows x cols, leading dims in
   complex elements). */
int n2d_narrow(const double *src_dev, long long lds, float *dst_dev, long long ldd, long long rows, long long cols);
int n2d_widen(const float *src_dev, long long lds, double *dst_dev, long long ldd, long long rows, long long cols);
/* Infinity norm of the row-major complex matrix (max row sum of |Re|+|Im|).
   norm_dev: caller-owned device scratch of 8 bytes per column. */
int n2d_norm_inf(const double *a_dev, long long order, long long ld, void *norm_dev, double *norm_host);
/* (With norm_host NULL the norm stays in norm_dev for n2d_read_norms.) */
/* Refinement step pieces for nrhs columns (leading dim ldb): r = b - A x with
   A row-major (ld), and x += d; each reports per-column infinity norms
   (|Re|+|Im|) of r and of the updated x into rnorm_host / xnorm_host. */
int n2d_residual(const double *a_dev, long long order, long long ld, const double *x_dev,
                 const double *b_dev, double *r_dev, long long nrhs, long long ldb, void *norm_dev,
                 double *rnorm_host);
int n2d_add_correction(double *x_dev, const double *d_dev, long long order, long long nrhs, long long ldb,
                       void *norm_dev, double *xnorm_host);
/* With a NULL host pointer the two above leave their norms on the device;
   this reads count of them back (synchronises). */
int n2d_read_norms(const void *norm_dev, long long count, double *host);
/* Ragged batch of count small systems (orders[i] <= 64) in one launch:
   mats_dev holds the row-major matrices back to back, rhs_dev and piv_dev the
   right-hand sides and pivots (orders[i] entries each), info_dev (count ints,
   zeroed) the first singular column + 1 of each; systems_dev is scratch of
   n2d_lu_batched_descriptor_bytes(count) bytes. */
int n2d_lu_batched(double *mats_dev, double *rhs_dev, int *piv_dev, const int *orders, long long count,
                   int *info_dev, void *systems_dev);
size_t n2d_lu_batched_descriptor_bytes(long long count);
/* Ragged batch of count FP64 factorisations advanced in lockstep (one launch
   per kernel and panel step for all of them): system i is order[i] x order[i]
   at a_dev[i] (leading dim ld[i]), factored exactly as n2d_lu_factor would
   (pivots into ipiv_dev[i]); info_host[i] gets its first zero / rejected
   pivot (1-based) or 0.  Orders up to n2d_lu_batch_max_order(). */
int n2d_lu_factor_batch(double *const *a_dev, const long long *order, const long long *ld, int *const *ipiv_dev,
                        int count, int rule, int *info_host);
long long n2d_lu_batch_max_order(void);
/* The split-precision form of the same (FP32 matrices, even leading dims,
   16-byte aligned; tensor-core 3xTF32 updates), factored as n2d_lu_factor32
   would factor each. */
int n2d_lu_factor32_batch(float *const *a_dev, const long long *order, const long long *ld, int *const *ipiv_dev,
                          int count, int rule, int *info_host);
/* Solves of count factored systems as n2d_lu_solve would, all at once:
   nrhs[i] columns of b_dev[i] (leading dim ldb[i]). */
int n2d_lu_solve_batch(const double *const *a_dev, const long long *order, const long long *ld,
                       const int *const *ipiv_dev, double *const *b_dev, const long long *ldb,
                       const long long *nrhs, int count);
/* The same with FP32 factors (FP64 arithmetic and right-hand sides). */
int n2d_lu_solve32_batch(const float *const *a_dev, const long long *order, const long long *ld,
                         const int *const *ipiv_dev, double *const *b_dev, const long long *ldb,
                         const long long *nrhs, int count);
/* In-place device transpose of an order x order block (leading dims lda/ldb). */
int n2d_transpose(const double *src_dev, long long lds, double *dst_dev, long long ldd,
                  long long rows, long long cols);

/* ---- wire <-> volume coupling blocks (dielectric_wire.c) ---- */
/* seg_dev: 8 doubles per segment (x y z length radius cab sab salp, lengths
   in wavelengths); sources_dev: per column, per segment the constant, sine
   and cosine current coefficients (complex); centers/sizes: 3 doubles per
   cell (m); chi_dev: eps_r - 1 per cell (complex); node/weight: the 6-point
   Gauss rule on [-1, 1].  out_dev: columns x 3 cells complex. */
int n2d_coupling_wire_to_volume(const double *seg_dev, int nseg, double rkh, int image, double wlam,
                                const double *sources_dev, int columns, const double *center_dev,
                                const double *size_dev, const double *chi_dev, long long cells,
                                double omega_eps0, const double *node_dev, const double *weight_dev,
                                double *out_dev);
/* obs/tangent: 3 doubles per segment (m); node/weight: the 10-point Gauss
   rule.  out_dev: segments x 3 cells complex. */
int n2d_coupling_volume_to_wire(const double *obs_dev, const double *tangent_dev, int nseg,
                                const double *center_dev, const double *size_dev, long long cells,
                                double k0, double omega_eps0, int image, const double *node_dev,
                                const double *weight_dev, double *out_dev);

/* ---- wire MoM fill (matrix.c cmset / cmww) ---- */
/* seg_dev: 8 doubles per segment as for the coupling; sup_first_dev: n + 1
   entry offsets per basis column; sup_src_dev: the source segment of each
   entry (increasing within a column); sup_coef_dev: 3 complex coefficients
   per entry; loads_dev: n complex load impedances or NULL.  out_dev: n rows
   of nrow complex values. */
int n2d_mom_fill(const double *seg_dev, int n, double rkh, int image, const int *sup_first_dev,
                 const int *sup_src_dev, const double *sup_coef_dev, const double *loads_dev, double *out_dev,
                 long long nrow);

#ifdef __cplusplus
}
#endif
#endif

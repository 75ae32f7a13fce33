// Hybrid conductor + volume operator [C B; D V] of dielectric_fft.c:41-83 on
// the device: the volume rows come from the FFT plan, the c dense conductor
// rows [C|B] and the v x c cross block D are complex FP64 row-major blocks
// (dielectric_fft.c:34-40 layout), uploaded once after assembly.
#include <float.h>
#include <math.h>
#include <string.h>
#include <vector>
#include "common.cuh"
#include "device_api.h"
#include "runtime.cuh"
#include "vie_internal.cuh"

using namespace n2c;

struct n2d_hybrid {
  n2d_vie *vol;
  long long c, v, n;
  int pec;
  double2 *blocks;   // c*(c+v) then v*c
  double2 *pdiag;    // full preconditioner divisor [diag(C); volume Jacobi]
  double2 *z;        // x or x ./ pdiag of the current product
  int precondition_ok;
  double *partials;
  unsigned int *ticket;
  void *gm_work;     // persistent GMRES workspace (gmres.cu)
};
void n2c_gmres_work_free(void *w);
void **n2c_hybrid_gm_slot(n2d_hybrid *h) { return &h->gm_work; }

// z = x, or x ./ pdiag when the input is preconditioned: both row kernels
// read z, so each division happens once per product.
__global__ void zc_kernel(const double2 *__restrict__ x, const double2 *__restrict__ pdiag, double2 *__restrict__ z,
                          long long n, const int *gate) {
  if (gated_off(gate)) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = pdiag ? cdiv(x[i], pdiag[i]) : x[i];
}

// One block per conductor row: y_i = sum_j [C|B]_ij z_j (dielectric_fft.c:54-66).
__global__ void __launch_bounds__(256) conductor_rows_kernel(const double2 *__restrict__ blocks,
                                                             const double2 *__restrict__ z, long long c, long long n,
                                                             double2 *__restrict__ y, const int *gate) {
  if (gated_off(gate)) return;
  const long long i = blockIdx.x;
  const double2 *row = blocks + i * n;
  double2 acc = make_double2(0, 0);
  for (long long j = threadIdx.x; j < n; j += blockDim.x) acc = cadd(acc, cmul(row[j], z[j]));
  acc = block_sum(acc);
  if (threadIdx.x == 0) y[i] = acc;
}

// One warp per volume row: y_{c+i} += sum_j D_ij z_j over the c conductor
// unknowns (dielectric_fft.c:67-74).
__global__ void cross_rows_kernel(const double2 *__restrict__ D, const double2 *__restrict__ z, long long c,
                                  long long v, double2 *__restrict__ y, const int *gate) {
  if (gated_off(gate)) return;
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= v) return;
  const double2 *row = D + warp * c;
  double2 acc = make_double2(0, 0);
  for (long long j = lane; j < c; j += 32) acc = cadd(acc, cmul(row[j], z[j]));
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
  }
  if (lane == 0) y[c + warp] = cadd(y[c + warp], acc);
}

// Deterministic sum of |y|^2 with a non-finite flag.
__global__ void norm2_kernel(const double2 *__restrict__ y, long long n, double *partials,
                             unsigned int *ticket, double *out, int *flag, const int *gate) {
  if (gated_off(gate)) return;
  double acc = 0;
  bool bad = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 v = y[i];
    acc += v.x * v.x + v.y * v.y;
    bad |= !finite2(v);
  }
  if (bad && flag) *flag = 1;
  double2 s = block_sum(make_double2(acc, 0));
  if (threadIdx.x == 0) partials[blockIdx.x] = s.x;
  if (last_block_done(ticket)) {
    double t = 0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) t += partials[i];
    double2 tot = block_sum(make_double2(t, 0));
    if (threadIdx.x == 0) { *out = tot.x; *ticket = 0; }
  }
}

int n2c_norm2(const double *y, long long n, double *partials, unsigned int *ticket, double *out,
              int *flag) {
  long long blocks = (n + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  if (blocks < 1) blocks = 1;
  norm2_kernel<<<(unsigned)blocks, 256, 0, n2c_stream()>>>((const double2 *)y, n, partials, ticket,
                                                           out, flag, n2c_gate());
  return n2c_check_launch("norm2");
}

__global__ void divide_kernel(const double2 *__restrict__ x, const double2 *__restrict__ d,
                              double2 *__restrict__ y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = cdiv(x[i], d[i]);
}

extern "C" int n2d_hybrid_create(n2d_hybrid **out, n2d_vie *vol, long long c, long long v, int pec) {
  *out = nullptr;
  n2d_hybrid *h = new n2d_hybrid();
  memset(h, 0, sizeof(*h));
  h->vol = vol; h->c = c; h->v = v; h->n = c + v; h->pec = pec;
  const long long nblk = c * (c + v) + v * c;
  h->blocks = (double2 *)n2d_alloc((nblk ? nblk : 1) * sizeof(double2));
  h->pdiag = (double2 *)n2d_alloc((h->n ? h->n : 1) * sizeof(double2));
  h->partials = (double *)n2d_alloc(4096 * sizeof(double));
  h->z = (double2 *)n2d_alloc((h->n ? h->n : 1) * sizeof(double2));
  h->ticket = (unsigned int *)n2d_alloc(64);
  if (!h->blocks || !h->pdiag || !h->partials || !h->z || !h->ticket || !n2d_memset(h->ticket, 0, 64)) {
    n2d_hybrid_destroy(h);
    return 0;
  }
  if (vol && pec) n2d_vie_set_mirror(vol, v / 3);
  *out = h;
  return 1;
}

extern "C" void n2d_hybrid_destroy(n2d_hybrid *h) {
  if (!h) return;
  n2c_gmres_work_free(h->gm_work);
  n2d_free(h->blocks); n2d_free(h->pdiag); n2d_free(h->partials); n2d_free(h->ticket); n2d_free(h->z);
  delete h;
}

extern "C" long long n2d_hybrid_order(const n2d_hybrid *h) { return h->n; }

extern "C" int n2d_hybrid_upload_blocks(n2d_hybrid *h, const double *blocks) {
  const long long c = h->c, v = h->v, nblk = c * (c + v) + v * c;
  if (!n2d_upload(h->blocks, blocks, nblk * sizeof(double2))) return 0;
  // Preconditioner divisor: conductor diagonal (dielectric_fft.c:77-81) then
  // the volume Jacobi divisor of the physical cells.
  std::vector<double2> cd(c ? c : 1);
  h->precondition_ok = 1;
  for (long long i = 0; i < c; ++i) {
    const double re = blocks[2 * (i * (c + v) + i)], im = blocks[2 * (i * (c + v) + i) + 1];
    const double mag = hypot(re, im);
    if (!isfinite(mag) || mag < DBL_MIN) h->precondition_ok = 0;
    cd[i] = make_double2(re, im);
  }
  if (c && !n2d_upload(h->pdiag, cd.data(), c * sizeof(double2))) return 0;
  if (v && !n2d_copy_d2d(h->pdiag + c, n2d_vie_diag(h->vol), v * sizeof(double2))) return 0;
  return n2d_sync();
}

int n2c_hybrid_precondition_ok(const n2d_hybrid *h) { return h->precondition_ok; }
extern "C" int n2d_hybrid_precondition_ok(const n2d_hybrid *h) { return h->precondition_ok; }
const double2 *n2c_hybrid_pdiag(const n2d_hybrid *h) { return h->pdiag; }
n2d_vie *n2c_hybrid_volume(const n2d_hybrid *h) { return h->vol; }
const double2 *n2c_hybrid_blocks(const n2d_hybrid *h) { return h->blocks; }
long long n2c_hybrid_conductors(const n2d_hybrid *h) { return h->c; }

extern "C" int n2d_hybrid_apply(n2d_hybrid *h, const double *x, double *y, int precondition_input,
                                double *norm, int *flag, int full_precision) {
  const long long c = h->c, v = h->v, n = h->n;
  const double2 *pd = precondition_input ? h->pdiag : nullptr;
  if (v && !n2d_vie_apply(h->vol, x + 2 * c, y + 2 * c, precondition_input, nullptr, flag,
                          full_precision))
    return 0;
  if (c) {
    const long long zb = (n + 255) / 256;
    zc_kernel<<<(unsigned)(zb < 4096 ? zb : 4096), 256, 0, n2c_stream()>>>((const double2 *)x, pd, h->z, n,
                                                                            n2c_gate());
    conductor_rows_kernel<<<(unsigned)c, 256, 0, n2c_stream()>>>(h->blocks, h->z, c, n, (double2 *)y, n2c_gate());
    if (!n2c_check_launch("conductor_rows")) return 0;
    if (v) {
      const long long threads = v * 32;
      cross_rows_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, n2c_stream()>>>(h->blocks + c * n, h->z, c, v,
                                                                                      (double2 *)y, n2c_gate());
      if (!n2c_check_launch("cross_rows")) return 0;
    }
  }
  if (norm) return n2c_norm2(y, n, h->partials, h->ticket, norm, flag);
  return 1;
}

extern "C" int n2d_hybrid_precondition(n2d_hybrid *h, const double *x, double *y) {
  const long long n = h->n;
  divide_kernel<<<(unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256, 0,
                  n2c_stream()>>>((const double2 *)x, h->pdiag, (double2 *)y, n);
  return n2c_check_launch("hybrid precondition");
}

// Ragged batch of small dense systems in one launch: the wire blocks of many
// frequencies or geometries (tens of segments each) factored and solved
// together, one CTA per system.  Each system is factr()/solve() of
// matrix.c:1313-1416 / 1523-1555 on NEC's transposed storage (the algebraic
// matrix row-major): partial pivoting with factr's rule (largest |.|^2, later
// row on ties), the row interchange applied to whole rows (L in the getrf
// convention, as the blocked factorisation stores it), the multiplier formed by
// the reciprocal of the pivot, then forward and back substitution of one
// right-hand side.
//
// The matrix lives in shared memory for the whole factorisation (orders up to
// BATCH_MAX), so a column step is one warp-reduced pivot search, a row swap and
// a rank-1 update, with two CTA barriers.
#include <float.h>
#include <math.h>
#include "common.cuh"
#include "device_api.h"
#include "runtime.cuh"

using namespace n2c;

namespace {

constexpr int BATCH_MAX = 64;
constexpr int BT = 256;

struct BatchSystem {
  long long a_off;     // offset of the n x n row-major matrix (complex elements)
  long long b_off;     // offset of the right-hand side
  long long piv_off;   // offset of the pivots
  int n;
};

// Dynamic shared memory: the matrix with row stride lda = nmax + 1, then x.
__global__ void __launch_bounds__(BT) batched_lu_kernel(double2 *mats, double2 *rhs, int *pivs,
                                                        const BatchSystem *systems, int *info, int lda) {
  extern __shared__ double2 sm[];
  double2 *Am = sm, *x = sm + (size_t)lda * (lda - 1);
#define A(i, c) Am[(i) * lda + (c)]
  __shared__ double s_val[BT / 32];
  __shared__ int s_idx[BT / 32];
  __shared__ int s_piv;
  __shared__ bool s_zero;
  const BatchSystem sys = systems[blockIdx.x];
  const int n = sys.n, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double2 *ga = mats + sys.a_off;
  for (int t = tid; t < n * n; t += BT) A(t / n, t % n) = ga[t];
  for (int t = tid; t < n; t += BT) x[t] = rhs[sys.b_off + t];
  int first_zero = 0;
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    // Pivot: largest |A[i][j]|^2 over i >= j, the later row on ties.
    double v = -1.0;
    int idx = -1;
    for (int i = j + tid; i < n; i += BT) {
      const double m = A(i, j).x * A(i, j).x + A(i, j).y * A(i, j).y;
      if (m >= v) { v = m; idx = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, v, o);
      const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
      if (oi >= 0 && (idx < 0 || ov > v || (ov == v && oi > idx))) { v = ov; idx = oi; }
    }
    if (lane == 0) { s_val[warp] = v; s_idx[warp] = idx; }
    __syncthreads();
    if (tid == 0) {
      double bv = -1.0;
      int bi = -1;
      for (int w = 0; w < BT / 32; ++w)
        if (s_idx[w] >= 0 && (bi < 0 || s_val[w] > bv || (s_val[w] == bv && s_idx[w] > bi))) {
          bv = s_val[w];
          bi = s_idx[w];
        }
      s_piv = bi;
      s_zero = !(bv > 0.0);
      pivs[sys.piv_off + j] = bi + 1;
    }
    __syncthreads();
    const int p = s_piv;
    if (p != j) {
      for (int c = tid; c < n; c += BT) { const double2 t = A(j, c); A(j, c) = A(p, c); A(p, c) = t; }
      if (tid == 0) { const double2 t = x[j]; x[j] = x[p]; x[p] = t; }
    }
    __syncthreads();
    if (s_zero) {
      // Singular column: recorded, interchange kept, no elimination.
      if (first_zero == 0) first_zero = j + 1;
      continue;
    }
    const double2 pv = A(j, j);
    const double r = 1.0 / (pv.x * pv.x + pv.y * pv.y);
    const double2 inv = make_double2(pv.x * r, -pv.y * r);
    // Multipliers of column j, then the rank-1 update of rows j+1.. and the
    // right-hand side (thread per element, row-major).
    for (int i = j + 1 + tid; i < n; i += BT) A(i, j) = cmul(A(i, j), inv);
    __syncthreads();
    const int m = n - j - 1;
    for (int t = tid; t < m * (m + 1); t += BT) {
      const int i = j + 1 + t / (m + 1), c = j + 1 + t % (m + 1);
      if (c < n) A(i, c) = csub(A(i, c), cmul(A(i, j), A(j, c)));
      else x[i] = csub(x[i], cmul(A(i, j), x[j]));
    }
    __syncthreads();
  }
  if (tid == 0 && first_zero) info[blockIdx.x] = first_zero;
  // Back substitution (warp 0, column-oriented).
  if (!first_zero && warp == 0) {
    for (int k = n - 1; k >= 0; --k) {
      if (lane == 0) x[k] = cdiv(x[k], A(k, k));
      __syncwarp();
      const double2 xk = x[k];
      for (int i = lane; i < k; i += 32) x[i] = csub(x[i], cmul(A(i, k), xk));
      __syncwarp();
    }
  }
  __syncthreads();
  for (int t = tid; t < n * n; t += BT) ga[t] = A(t / n, t % n);
  for (int t = tid; t < n; t += BT) rhs[sys.b_off + t] = x[t];
#undef A
}

}  // namespace

// count systems of orders n[i] <= 64 packed in one device buffer each (mats:
// row-major n x n blocks back to back, rhs: n each, pivots: n each); info_dev
// (count ints, zeroed by the caller) receives the first singular column + 1.
extern "C" int n2d_lu_batched(double *mats_dev, double *rhs_dev, int *piv_dev, const int *orders, long long count,
                              int *info_dev, void *systems_dev) {
  if (count <= 0) return 1;
  // Offsets on the host, uploaded into the caller-provided descriptor buffer.
  BatchSystem *host = (BatchSystem *)malloc((size_t)count * sizeof(BatchSystem));
  if (!host) { n2c_set_error("out of host memory"); return 0; }
  long long a = 0, b = 0;
  int nmax = 1;
  for (long long i = 0; i < count; ++i) {
    if (orders[i] > nmax) nmax = orders[i];
    if (orders[i] < 1 || orders[i] > BATCH_MAX) {
      free(host);
      n2c_set_error("batched solve: order %d outside 1..%d", orders[i], BATCH_MAX);
      return 0;
    }
    host[i].a_off = a; host[i].b_off = b; host[i].piv_off = b; host[i].n = orders[i];
    a += (long long)orders[i] * orders[i];
    b += orders[i];
  }
  const int ok = n2d_upload(systems_dev, host, (size_t)count * sizeof(BatchSystem));
  free(host);
  if (!ok) return 0;
  if (count > 0x7fffffffLL) { n2c_set_error("batch too large"); return 0; }
  if (nmax > BATCH_MAX) nmax = BATCH_MAX;
  const int lda = nmax + 1;
  const size_t smem = (size_t)lda * lda * sizeof(double2);   // matrix rows, then x
  static const bool configured =
      cudaFuncSetAttribute(batched_lu_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (BATCH_MAX + 1) * (BATCH_MAX + 1) * (int)sizeof(double2)) == cudaSuccess;
  if (!configured) {
    n2c_set_error("batched LU: shared memory configuration failed");
    return 0;
  }
  batched_lu_kernel<<<(unsigned)count, BT, smem, n2c_stream()>>>((double2 *)mats_dev, (double2 *)rhs_dev, piv_dev,
                                                                 (const BatchSystem *)systems_dev, info_dev, lda);
  return n2c_check_launch("batched LU");
}

extern "C" size_t n2d_lu_batched_descriptor_bytes(long long count) { return (size_t)count * sizeof(BatchSystem); }

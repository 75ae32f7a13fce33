// Blocked right-looking complex LU with partial pivoting (FP64) for the wire
// MoM block: factr()/solve() of matrix.c:1313-1416 / 1523-1555 and the
// row-major builtin solve of dense_backend.c:152-190.
//
// Storage convention: column-major LU of the algebraic matrix with 1-based
// pivot rows ip[r] (the same pivot choices as the builtin factr: largest |.|^2,
// later row on ties), U as factr stores it, and L in the getrf convention
// (rows of earlier L columns follow later interchanges).  The builtin keeps L
// columns un-permuted instead; the backend's own solve consumes this storage,
// as the reference's LAPACK branch does with its own.
//
// Per panel of width KB:
//   panel_kernel     cooperative; one row per thread held in registers, one
//                    bounded grid barrier per column (pivot search + exchange)
//   swap_trsm_kernel interchanges + unit-lower solve on the columns right of
//                    the panel, one thread per column
//   swap_left_kernel the panel's interchanges on the L columns to its left
//   gemm_update      A22 -= L21 U12, 64x64 complex tiles, K chunks of 16
#include <float.h>
#include <math.h>
#include <string.h>
#include "common.cuh"
#include "device_api.h"
#include "runtime.cuh"

using namespace n2c;

namespace {

constexpr int KB = 32;        // panel width
constexpr int PT = 256;       // panel threads per block

struct LuBarrier {
  unsigned int count, gen;
  int error;
  int info;                   // first zero / rejected pivot (1-based), 0 = none
};

struct PanelSlot {            // one block's candidate and the row it carries
  double val;
  int idx;
  int pad;
  double2 row[KB];
};

struct PanelArgs {
  double2 *a;
  long long n, ld, k0;
  int kb, rule;
  int *ipiv;
  PanelSlot *slots;           // 2 x gridDim.x
  double2 *rowj;              // 2 x KB: old row j for the exchange
  LuBarrier *bar;
};

__device__ bool lu_barrier(LuBarrier *b) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned int *gen = &b->gen;
    volatile int *err = &b->error;
    if (*err) ok = 0;
    else {
      const unsigned int g = *gen;
      __threadfence();
      if (atomicAdd(&b->count, 1u) == gridDim.x - 1) {
        b->count = 0;
        __threadfence();
        atomicAdd(&b->gen, 1u);
      } else {
        const long long t0 = clock64();
        while (*gen == g) {
          if (*err || clock64() - t0 > (1LL << 32)) { atomicExch(&b->error, 1); ok = 0; break; }
          __nanosleep(32);
        }
      }
      __threadfence();
    }
  }
  __syncthreads();
  return ok != 0;
}

// Candidate order: larger magnitude wins; ties go to the later row for the
// classic rule (factr's ">=") and to the earlier row for the row-major rule
// (dense_backend.c's strict ">").
__device__ __forceinline__ bool better(double v, int i, double w, int k, int rule) {
  if (v != w) return v > w;
  return rule == 0 ? i > k : i < k;
}

__global__ void __launch_bounds__(PT) panel_kernel(PanelArgs p) {
  const long long rows = p.n - p.k0;
  const int tg = blockIdx.x * PT + threadIdx.x;
  const bool have = tg < rows;
  double2 *col0 = p.a + p.k0 + p.k0 * p.ld;   // panel origin
  double2 a[KB];
#pragma unroll
  for (int c = 0; c < KB; ++c)
    a[c] = (have && c < p.kb) ? col0[tg + c * p.ld] : make_double2(0, 0);
  __shared__ double s_val[PT / 32];
  __shared__ int s_idx[PT / 32];
  __shared__ int s_win;
  for (int j = 0; j < p.kb; ++j) {
    // Candidate magnitude of column j in this thread's row.
    double mag = -1.0;
    if (have && tg >= j) {
      double2 z;
#pragma unroll
      for (int c = 0; c < KB; ++c) if (c == j) z = a[c];
      mag = p.rule == 0 ? z.x * z.x + z.y * z.y : hypot(z.x, z.y);
    }
    double bv = mag;
    int bi = have ? tg : -1;
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (oi >= 0 && (bi < 0 || better(ov, oi, bv, bi, p.rule))) { bv = ov; bi = oi; }
    }
    if ((threadIdx.x & 31) == 0) { s_val[threadIdx.x >> 5] = bv; s_idx[threadIdx.x >> 5] = bi; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = s_val[0];
      int i = s_idx[0];
      for (int w = 1; w < PT / 32; ++w)
        if (s_idx[w] >= 0 && (i < 0 || better(s_val[w], s_idx[w], v, i, p.rule))) { v = s_val[w]; i = s_idx[w]; }
      s_win = i;
      PanelSlot *s = p.slots + (j & 1) * gridDim.x + blockIdx.x;
      s->val = v; s->idx = i;
    }
    __syncthreads();
    // The block's winner publishes its row; the owner of row j publishes it too.
    PanelSlot *mine = p.slots + (j & 1) * gridDim.x + blockIdx.x;
    if (have && tg == s_win) {
#pragma unroll
      for (int c = 0; c < KB; ++c) mine->row[c] = a[c];
    }
    if (have && tg == j) {
#pragma unroll
      for (int c = 0; c < KB; ++c) p.rowj[(j & 1) * KB + c] = a[c];
    }
    if (!lu_barrier(p.bar)) return;
    // Global winner, same fixed-order reduction in every block.
    const PanelSlot *slots = p.slots + (j & 1) * gridDim.x;
    double v = slots[0].val;
    int pi = slots[0].idx, pb = 0;
    for (int b = 1; b < (int)gridDim.x; ++b)
      if (slots[b].idx >= 0 && (pi < 0 || better(slots[b].val, slots[b].idx, v, pi, p.rule))) {
        v = slots[b].val; pi = slots[b].idx; pb = b;
      }
    const double2 *prow = slots[pb].row;
    const double2 piv = prow[j];
    const bool zero = p.rule == 0 ? !(v > 0.0) : !(v > 64.0 * DBL_EPSILON);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      p.ipiv[p.k0 + j] = (int)(p.k0 + pi + 1);
      if (zero && p.bar->info == 0) p.bar->info = (int)(p.k0 + j + 1);
    }
    // Exchange rows j and pi across the whole panel.
    if (have && tg == j) {
#pragma unroll
      for (int c = 0; c < KB; ++c) a[c] = prow[c];
    } else if (have && tg == pi) {
#pragma unroll
      for (int c = 0; c < KB; ++c) a[c] = p.rowj[(j & 1) * KB + c];
    }
    if (have && tg > j && !zero) {
      // Multiplier by the reciprocal, as factr does (matrix.c:1393-1398).
      const double2 inv = cdiv(make_double2(1.0, 0.0), piv);
      double2 l;
#pragma unroll
      for (int c = 0; c < KB; ++c) if (c == j) { l = cmul(a[c], inv); a[c] = l; }
#pragma unroll
      for (int c = 0; c < KB; ++c)
        if (c > j && c < p.kb) a[c] = csub(a[c], cmul(l, prow[c]));
    }
  }
#pragma unroll
  for (int c = 0; c < KB; ++c)
    if (have && c < p.kb) col0[tg + c * p.ld] = a[c];
}

// Interchanges ip[k0..k0+kb) then the unit-lower solve U12 = L11^-1 A12, one
// thread per column right of the panel.
__global__ void __launch_bounds__(128) swap_trsm_kernel(double2 *a, long long n, long long ld, long long k0,
                                                        int kb, const int *ipiv) {
  __shared__ double2 L[KB][KB + 1];
  for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
    const int i = t % kb, j = t / kb;
    L[i][j] = a[(k0 + i) + (k0 + j) * ld];
  }
  __syncthreads();
  const long long c = k0 + kb + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= n) return;
  double2 *col = a + c * ld;
  for (int i = 0; i < kb; ++i) {
    const long long pr = ipiv[k0 + i] - 1;
    if (pr != k0 + i) { double2 t = col[k0 + i]; col[k0 + i] = col[pr]; col[pr] = t; }
  }
  double2 x[KB];
#pragma unroll
  for (int i = 0; i < KB; ++i) x[i] = i < kb ? col[k0 + i] : make_double2(0, 0);
#pragma unroll
  for (int i = 1; i < KB; ++i) {
    if (i < kb) {
      double2 s = x[i];
#pragma unroll
      for (int j = 0; j < KB; ++j) if (j < i) s = csub(s, cmul(L[i][j], x[j]));
      x[i] = s;
    }
  }
#pragma unroll
  for (int i = 0; i < KB; ++i) if (i < kb) col[k0 + i] = x[i];
}

// The panel's interchanges applied to the columns left of it.
__global__ void swap_left_kernel(double2 *a, long long ld, long long k0, int kb, const int *ipiv) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= k0) return;
  double2 *col = a + c * ld;
  for (int i = 0; i < kb; ++i) {
    const long long pr = ipiv[k0 + i] - 1;
    if (pr != k0 + i) { double2 t = col[k0 + i]; col[k0 + i] = col[pr]; col[pr] = t; }
  }
}

// C[m x m'] -= A[m x K] B[K x m'] on column-major complex FP64 blocks.
constexpr int GT = 64;   // tile edge
constexpr int GK = 16;   // K chunk
__global__ void __launch_bounds__(256) gemm_update_kernel(double2 *C, const double2 *A, const double2 *B,
                                                          long long M, long long N, int K, long long ld) {
  __shared__ double2 As[GK][GT + 1];
  __shared__ double2 Bs[GK][GT + 1];
  const long long row0 = blockIdx.x * (long long)GT, col0 = blockIdx.y * (long long)GT;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // 16 x 16 threads, 4 x 4 each
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0, 0);
  for (int k0 = 0; k0 < K; k0 += GK) {
    for (int t = threadIdx.x; t < GT * GK; t += 256) {
      const int r = t % GT, k = t / GT;
      const long long gr = row0 + r;
      As[k][r] = (gr < M && k0 + k < K) ? A[gr + (long long)(k0 + k) * ld] : make_double2(0, 0);
      const int kk = t % GK, cc = t / GK;
      const long long gc = col0 + cc;
      Bs[kk][cc] = (gc < N && k0 + kk < K) ? B[(k0 + kk) + gc * ld] : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < GK; ++k) {
      double2 av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[k][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[k][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x = fma(av[i].x, bv[j].x, acc[i][j].x);
          acc[i][j].x = fma(-av[i].y, bv[j].y, acc[i][j].x);
          acc[i][j].y = fma(av[i].x, bv[j].y, acc[i][j].y);
          acc[i][j].y = fma(av[i].y, bv[j].x, acc[i][j].y);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const long long r = row0 + tx + 16 * i, c = col0 + ty + 16 * j;
      if (r < M && c < N) {
        double2 *p = C + r + c * ld;
        *p = csub(*p, acc[i][j]);
      }
    }
}

// Solve with the getrf-convention factors: all interchanges, unit-lower
// forward substitution, then column-oriented back substitution (the same
// system as matrix.c:1523-1555 solves).  One block per RHS.
__global__ void __launch_bounds__(1024) lu_solve_kernel(const double2 *a, long long n, long long ld,
                                                        const int *ipiv, double2 *b, long long ldb) {
  double2 *x = b + blockIdx.x * ldb;
  __shared__ double2 s;
  if (threadIdx.x == 0)
    for (long long i = 0; i < n; ++i) {
      const long long pi = ipiv[i] - 1;
      if (pi != i) { const double2 t = x[pi]; x[pi] = x[i]; x[i] = t; }
    }
  __syncthreads();
  for (long long i = 0; i < n; ++i) {
    if (threadIdx.x == 0) s = x[i];
    __syncthreads();
    const double2 v = s;
    const double2 *col = a + i * ld;
    for (long long j = i + 1 + threadIdx.x; j < n; j += blockDim.x) x[j] = csub(x[j], cmul(col[j], v));
    __syncthreads();
  }
  for (long long j = n - 1; j >= 0; --j) {
    if (threadIdx.x == 0) {
      const double2 v = cdiv(x[j], a[j + j * ld]);
      x[j] = v;
      s = v;
    }
    __syncthreads();
    const double2 v = s;
    const double2 *col = a + j * ld;
    for (long long i = threadIdx.x; i < j; i += blockDim.x) x[i] = csub(x[i], cmul(col[i], v));
    __syncthreads();
  }
}

__global__ void transpose_kernel(const double2 *src, long long lds, double2 *dst, long long ldd,
                                 long long rows, long long cols) {
  __shared__ double2 tile[32][33];
  const long long bx = blockIdx.x * 32LL, by = blockIdx.y * 32LL;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const long long r = bx + threadIdx.x, c = by + k;
    if (r < rows && c < cols) tile[k][threadIdx.x] = src[r + c * lds];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const long long c = by + threadIdx.x, r = bx + k;
    if (r < rows && c < cols) dst[c + r * ldd] = tile[threadIdx.x][k];
  }
}

}  // namespace

extern "C" int n2d_transpose(const double *src, long long lds, double *dst, long long ldd, long long rows,
                             long long cols) {
  dim3 grid((unsigned)((rows + 31) / 32), (unsigned)((cols + 31) / 32)), block(32, 8);
  transpose_kernel<<<grid, block, 0, n2c_stream()>>>((const double2 *)src, lds, (double2 *)dst, ldd, rows, cols);
  return n2c_check_launch("transpose");
}

extern "C" int n2d_lu_factor(double *a_dev, long long n, long long ld, int *ipiv, int rule, int precision,
                             int *info_host) {
  (void)precision;
  *info_host = 0;
  if (n <= 0) return 1;
  double2 *a = (double2 *)a_dev;
  const long long max_blocks = (n + PT - 1) / PT;
  PanelSlot *slots = (PanelSlot *)n2d_alloc(2 * max_blocks * sizeof(PanelSlot));
  double2 *rowj = (double2 *)n2d_alloc(2 * KB * sizeof(double2));
  LuBarrier *bar = (LuBarrier *)n2d_alloc(sizeof(LuBarrier));
  int ok = slots && rowj && bar && n2d_memset(bar, 0, sizeof(LuBarrier));
  for (long long k0 = 0; ok && k0 < n; k0 += KB) {
    const int kb = (int)(n - k0 < KB ? n - k0 : KB);
    PanelArgs p;
    p.a = a; p.n = n; p.ld = ld; p.k0 = k0; p.kb = kb; p.rule = rule; p.ipiv = ipiv;
    p.slots = slots; p.rowj = rowj; p.bar = bar;
    const int blocks = (int)((n - k0 + PT - 1) / PT);
    void *args[] = {&p};
    cudaError_t e = cudaLaunchCooperativeKernel((void *)panel_kernel, blocks, PT, args, 0, n2c_stream());
    if (e != cudaSuccess) { n2c_set_error("panel launch: %s", cudaGetErrorString(e)); ok = 0; break; }
    n2c_count_launch(1);
    if (k0 > 0) {
      swap_left_kernel<<<(unsigned)((k0 + 127) / 128), 128, 0, n2c_stream()>>>(a, ld, k0, kb, ipiv);
      if (!n2c_check_launch("swap_left")) { ok = 0; break; }
    }
    const long long right = n - k0 - kb;
    if (right > 0) {
      swap_trsm_kernel<<<(unsigned)((right + 127) / 128), 128, 0, n2c_stream()>>>(a, n, ld, k0, kb, ipiv);
      if (!n2c_check_launch("swap_trsm")) { ok = 0; break; }
      dim3 grid((unsigned)((right + GT - 1) / GT), (unsigned)((right + GT - 1) / GT));
      gemm_update_kernel<<<grid, 256, 0, n2c_stream()>>>(a + (k0 + kb) + (k0 + kb) * ld, a + (k0 + kb) + k0 * ld,
                                                         a + k0 + (k0 + kb) * ld, right, right, kb, ld);
      if (!n2c_check_launch("gemm_update")) { ok = 0; break; }
    }
  }
  LuBarrier hb;
  memset(&hb, 0, sizeof(hb));
  if (ok && !n2d_download(&hb, bar, sizeof(hb))) ok = 0;
  if (ok && hb.error) { n2c_set_error("LU panel barrier time-out"); ok = 0; }
  *info_host = hb.info;
  n2d_free(slots); n2d_free(rowj); n2d_free(bar);
  return ok;
}

extern "C" int n2d_lu_solve(const double *a_dev, long long n, long long ld, const int *ipiv, double *b_dev,
                            long long ldb, long long nrhs) {
  if (n <= 0 || nrhs <= 0) return 1;
  lu_solve_kernel<<<(unsigned)nrhs, 1024, 0, n2c_stream()>>>((const double2 *)a_dev, n, ld, ipiv,
                                                             (double2 *)b_dev, ldb);
  return n2c_check_launch("lu_solve");
}

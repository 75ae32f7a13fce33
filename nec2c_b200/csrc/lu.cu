// Blocked right-looking complex LU with partial pivoting (FP64) for the wire
// MoM block: factr()/solve() of matrix.c:1313-1416 / 1523-1555 and the
// row-major builtin solve of dense_backend.c:152-190.
//
// Storage: the algebraic matrix A row-major with leading dimension ld, which
// is NEC's transposed column-major storage itself, so the classic entry points
// factor the caller's array as laid out.  The factors are the LU of the
// row-interchanged A in that layout, 1-based pivot rows ip[r] with the builtin
// factr's pivot choice (largest |.|^2, later row on ties), and L in the getrf
// convention (rows of earlier L columns follow later interchanges).  The
// backend's own solve consumes this storage.
//
// Per panel of width KB (32 columns):
//   panel       thread-block cluster of 8 CTAs: panel rows in registers, one
//               hardware cluster barrier per column, candidates and pivot rows
//               exchanged through distributed shared memory (n <= 4096; larger
//               orders use a cooperative grid with a bounded-spin barrier)
//   interchange the panel's row interchanges outside the panel as a gather of
//               the affected rows into scratch and a scatter back (parallel
//               over rows x columns, coalesced)
//   trsm        U12 = L11^-1 A12, one thread per column
//   gemm        A22 -= L21 U12, 64x64 complex tiles, K chunks of 16
#include <cooperative_groups.h>
#include <float.h>
#include <math.h>
#include <string.h>
#include "common.cuh"
#include "device_api.h"
#include "runtime.cuh"

namespace cg = cooperative_groups;
using namespace n2c;

namespace {

constexpr int KB = 32;        // panel width
constexpr int PT = 256;       // panel threads per CTA
constexpr int CS = 8;         // panel cluster size (portable maximum)

struct LuStatus {
  unsigned int count, gen;
  int error;
  int info;                   // first zero / rejected pivot (1-based), 0 = none
  int npairs;                 // affected rows of the last panel's interchanges
  int pad;
};

// Candidate order: larger magnitude wins; ties go to the later row for the
// classic rule (factr's ">=") and to the earlier row for the row-major rule
// (dense_backend.c's strict ">").
__device__ __forceinline__ bool better(double v, int i, double w, int k, int rule) {
  if (v != w) return v > w;
  return rule == 0 ? i > k : i < k;
}

__device__ __forceinline__ double magnitude(double2 z, int rule) {
  return rule == 0 ? z.x * z.x + z.y * z.y : hypot(z.x, z.y);
}

struct PanelArgs {
  double2 *a;
  long long n, ld, k0;
  int kb, rule;
  int *ipiv;
  int *pairs;                 // 2 x 2KB: destination and source rows of the interchanges
  LuStatus *st;
  // cooperative fallback only
  double *gval;               // 2 x grid candidates
  int *gidx;
  double2 *grow;              // 2 x grid x KB candidate rows
  double2 *growj;             // 2 x KB row j
};

// Net effect of the panel's sequential interchanges, computed by one warp:
// row r receives the old content of row src(r) for at most 2 KB rows.  The
// panel's own rows k0..k0+kb-1 are slots 0..kb-1; pivot rows below the panel
// get slots kb.. (matched with a warp ballot).
__device__ void panel_pairs_warp(const PanelArgs &p) {
  __shared__ int rows[2 * KB], src[2 * KB], cnt;
  const int lane = threadIdx.x & 31;
  const int k0 = (int)p.k0, kb = p.kb;
  for (int u = lane; u < 2 * KB; u += 32) { rows[u] = u < kb ? k0 + u : -1; src[u] = rows[u]; }
  if (lane == 0) cnt = kb;
  __syncwarp();
  for (int i = 0; i < kb; ++i) {
    const int q = p.ipiv[k0 + i] - 1;
    int iq;
    if (q < k0 + kb) {
      iq = q - k0;
    } else {
      const int n = cnt;
      const unsigned m0 = __ballot_sync(0xffffffffu, lane < n - kb && rows[kb + lane] == q);
      if (m0) iq = kb + __ffs(m0) - 1;
      else {
        iq = n;
        if (lane == 0) { rows[n] = q; src[n] = q; cnt = n + 1; }
      }
    }
    __syncwarp();
    if (lane == 0) { const int t = src[i]; src[i] = src[iq]; src[iq] = t; }
    __syncwarp();
  }
  if (lane == 0) {
    int np = 0;
    for (int u = 0; u < cnt; ++u)
      if (src[u] != rows[u]) { p.pairs[np] = rows[u]; p.pairs[2 * KB + np] = src[u]; ++np; }
    p.st->npairs = np;
  }
}

// One column step shared by both panel variants: v is this thread's row
// (ROWS rows), g its panel-row indices.  Returns after the exchange and the
// rank-1 update of column j.
template <int ROWS>
__device__ __forceinline__ void apply_column(double2 (&a)[ROWS][KB], const int (&g)[ROWS], const bool (&have)[ROWS],
                                             int j, int pi, const double2 *prow, const double2 *rowj, bool zero,
                                             int kb) {
  const double2 piv = prow[j];
#pragma unroll
  for (int q = 0; q < ROWS; ++q) {
    if (!have[q]) continue;
    if (g[q] == j) {
#pragma unroll
      for (int c = 0; c < KB; ++c) a[q][c] = prow[c];
    } else if (g[q] == pi) {
#pragma unroll
      for (int c = 0; c < KB; ++c) a[q][c] = rowj[c];
    }
    if (g[q] > j && !zero) {
      // Multiplier by the reciprocal, as factr does (matrix.c:1393-1398).
      const double2 inv = cdiv(make_double2(1.0, 0.0), piv);
      double2 l = make_double2(0, 0);
#pragma unroll
      for (int c = 0; c < KB; ++c) if (c == j) { l = cmul(a[q][c], inv); a[q][c] = l; }
#pragma unroll
      for (int c = 0; c < KB; ++c)
        if (c > j && c < kb) a[q][c] = csub(a[q][c], cmul(l, prow[c]));
    }
  }
}

// Block-wide best candidate; returns it in (*v, *i) for every thread.
__device__ __forceinline__ void block_best(double mv, int mi, int rule, double *v, int *i) {
  __shared__ double s_val[32];
  __shared__ int s_idx[32];
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, mv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, mi, o);
    if (oi >= 0 && (mi < 0 || better(ov, oi, mv, mi, rule))) { mv = ov; mi = oi; }
  }
  if ((threadIdx.x & 31) == 0) { s_val[threadIdx.x >> 5] = mv; s_idx[threadIdx.x >> 5] = mi; }
  __syncthreads();
  double bv = s_val[0];
  int bi = s_idx[0];
  for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
    if (s_idx[w] >= 0 && (bi < 0 || better(s_val[w], s_idx[w], bv, bi, rule))) { bv = s_val[w]; bi = s_idx[w]; }
  __syncthreads();
  *v = bv;
  *i = bi;
}

// Cluster panel: CTA r, thread t owns panel row g = r*TPB + t (TPB threads
// per CTA, one row each in registers, up to CS*TPB rows).  Per column every
// CTA pushes its best candidate (value, row index, row) and, from the owner,
// the current row j into the shared memory of all CTAs of the cluster, then
// one cluster barrier makes them visible: the winner and the pivot row are
// then read locally (double-buffered by column parity).
struct ClusterSlot {
  double val[2][CS];
  int idx[2][CS];
  double2 row[2][CS][KB];   // candidate rows, one per CTA
  double2 rowj[2][KB];      // row j
};

template <int TPB>
__global__ void __cluster_dims__(CS, 1, 1) __launch_bounds__(TPB, 1) panel_cluster_kernel(PanelArgs p) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  __shared__ ClusterSlot slot;
  __shared__ double2 mine[KB], minej[KB];
  __shared__ double m_val;
  __shared__ int m_idx;
  const long long rows = p.n - p.k0;
  double2 a[1][KB];
  const int g[1] = {rank * TPB + (int)threadIdx.x};
  const bool have[1] = {g[0] < rows};
  {
    const double2 *row = p.a + (p.k0 + g[0]) * p.ld + p.k0;
#pragma unroll
    for (int c = 0; c < KB; ++c) a[0][c] = (have[0] && c < p.kb) ? row[c] : make_double2(0, 0);
  }
  for (int j = 0; j < p.kb; ++j) {
    const int buf = j & 1;
    double mv = -1.0;
    int mi = -1;
    if (have[0] && g[0] >= j) {
      double2 z = make_double2(0, 0);
#pragma unroll
      for (int c = 0; c < KB; ++c) if (c == j) z = a[0][c];
      mv = magnitude(z, p.rule);
      mi = g[0];
    }
    double bv;
    int bi;
    block_best(mv, mi, p.rule, &bv, &bi);
    if (have[0] && g[0] == bi) {
#pragma unroll
      for (int c = 0; c < KB; ++c) mine[c] = a[0][c];
    }
    const bool jown = j / TPB == rank;
    if (have[0] && g[0] == j) {
#pragma unroll
      for (int c = 0; c < KB; ++c) minej[c] = a[0][c];
    }
    if (threadIdx.x == 0) { m_val = bv; m_idx = bi; }
    __syncthreads();
    // Push to every CTA (including this one): thread t -> (CTA t / 32, entry t % 32).
    for (int t = threadIdx.x; t < CS * KB; t += TPB) {
      const int dest = t / KB, e = t % KB;
      ClusterSlot *rs = cluster.map_shared_rank(&slot, dest);
      rs->row[buf][rank][e] = mine[e];
      if (jown) rs->rowj[buf][e] = minej[e];
      if (e == 0) { rs->val[buf][rank] = m_val; rs->idx[buf][rank] = m_idx; }
    }
    cluster.sync();
    // Global winner in fixed rank order, from local shared memory.
    double v = -2.0;
    int pi = -1, pr = 0;
#pragma unroll
    for (int r = 0; r < CS; ++r) {
      const int ri = slot.idx[buf][r];
      const double rv = slot.val[buf][r];
      if (ri >= 0 && (pi < 0 || better(rv, ri, v, pi, p.rule))) { v = rv; pi = ri; pr = r; }
    }
    const bool zero = p.rule == 0 ? !(v > 0.0) : !(v > 64.0 * DBL_EPSILON);
    if (rank == 0 && threadIdx.x == 0) {
      p.ipiv[p.k0 + j] = (int)(p.k0 + pi + 1);
      if (zero && p.st->info == 0) p.st->info = (int)(p.k0 + j + 1);
    }
    apply_column<1>(a, g, have, j, pi, slot.row[buf][pr], slot.rowj[buf], zero, p.kb);
  }
  cluster.sync();   // no CTA exits while others may still push into it
  if (have[0]) {
    double2 *row = p.a + (p.k0 + g[0]) * p.ld + p.k0;
#pragma unroll
    for (int c = 0; c < KB; ++c) if (c < p.kb) row[c] = a[0][c];
  }
  if (rank == 0 && threadIdx.x < 32) panel_pairs_warp(p);
}

// Cooperative-grid panel for orders beyond the cluster's capacity: one row per
// thread, one bounded-spin grid barrier per column.
__device__ bool lu_barrier(LuStatus *b) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned int *gen = &b->gen;
    volatile int *err = &b->error;
    if (*err) ok = 0;
    else {
      const unsigned int g0 = *gen;
      __threadfence();
      if (atomicAdd(&b->count, 1u) == gridDim.x - 1) {
        b->count = 0;
        __threadfence();
        atomicAdd(&b->gen, 1u);
      } else {
        const long long t0 = clock64();
        while (*gen == g0) {
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

__global__ void __launch_bounds__(PT) panel_grid_kernel(PanelArgs p) {
  const long long rows = p.n - p.k0;
  double2 a[1][KB];
  int g[1] = {(int)(blockIdx.x * PT + threadIdx.x)};
  bool have[1] = {g[0] < rows};
  const double2 *row0 = p.a + (p.k0 + g[0]) * p.ld + p.k0;
#pragma unroll
  for (int c = 0; c < KB; ++c) a[0][c] = (have[0] && c < p.kb) ? row0[c] : make_double2(0, 0);
  __shared__ int s_win;
  for (int j = 0; j < p.kb; ++j) {
    const int buf = j & 1;
    double mv = -1.0;
    int mi = -1;
    if (have[0] && g[0] >= j) {
      double2 z = make_double2(0, 0);
#pragma unroll
      for (int c = 0; c < KB; ++c) if (c == j) z = a[0][c];
      mv = magnitude(z, p.rule);
      mi = g[0];
    }
    double bv;
    int bi;
    block_best(mv, mi, p.rule, &bv, &bi);
    if (threadIdx.x == 0) {
      p.gval[buf * gridDim.x + blockIdx.x] = bv;
      p.gidx[buf * gridDim.x + blockIdx.x] = bi;
      s_win = bi;
    }
    __syncthreads();
    if (have[0] && g[0] == s_win) {
#pragma unroll
      for (int c = 0; c < KB; ++c) p.grow[((long long)buf * gridDim.x + blockIdx.x) * KB + c] = a[0][c];
    }
    if (have[0] && g[0] == j) {
#pragma unroll
      for (int c = 0; c < KB; ++c) p.growj[buf * KB + c] = a[0][c];
    }
    if (!lu_barrier(p.st)) return;
    double v = -2.0;
    int pi = -1, pb = 0;
    for (int b = 0; b < (int)gridDim.x; ++b) {
      const int ri = p.gidx[buf * gridDim.x + b];
      const double rv = p.gval[buf * gridDim.x + b];
      if (ri >= 0 && (pi < 0 || better(rv, ri, v, pi, p.rule))) { v = rv; pi = ri; pb = b; }
    }
    const bool zero = p.rule == 0 ? !(v > 0.0) : !(v > 64.0 * DBL_EPSILON);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      p.ipiv[p.k0 + j] = (int)(p.k0 + pi + 1);
      if (zero && p.st->info == 0) p.st->info = (int)(p.k0 + j + 1);
    }
    __shared__ double2 lp[KB], lj[KB];
    if (threadIdx.x < KB) lp[threadIdx.x] = p.grow[((long long)buf * gridDim.x + pb) * KB + threadIdx.x];
    else if (threadIdx.x < 2 * KB) lj[threadIdx.x - KB] = p.growj[buf * KB + threadIdx.x - KB];
    __syncthreads();
    apply_column<1>(a, g, have, j, pi, lp, lj, zero, p.kb);
    __syncthreads();
  }
  if (!lu_barrier(p.st)) return;
  double2 *row = p.a + (p.k0 + g[0]) * p.ld + p.k0;
#pragma unroll
  for (int c = 0; c < KB; ++c) if (have[0] && c < p.kb) row[c] = a[0][c];
  if (blockIdx.x == 0 && threadIdx.x < 32) panel_pairs_warp(p);
}

// Row interchanges outside the panel columns [k0, k0+kb): gather the source
// rows of the affected pairs into scratch, then scatter them to their
// destinations.  Thread (pair, column), columns consecutive across threads.
__global__ void rows_gather_kernel(const double2 *a, long long n, long long ld, long long k0, int kb,
                                   const int *pairs, const LuStatus *st, double2 *tmp) {
  const int np = st->npairs;
  const long long cols = n - kb;
  const long long total = (long long)np * cols;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long q = t / cols, c0 = t - q * cols;
    const long long c = c0 < k0 ? c0 : c0 + kb;
    tmp[t] = a[(long long)pairs[2 * KB + q] * ld + c];
  }
}

__global__ void rows_scatter_kernel(double2 *a, long long n, long long ld, long long k0, int kb,
                                    const int *pairs, const LuStatus *st, const double2 *tmp) {
  const int np = st->npairs;
  const long long cols = n - kb;
  const long long total = (long long)np * cols;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long q = t / cols, c0 = t - q * cols;
    const long long c = c0 < k0 ? c0 : c0 + kb;
    a[(long long)pairs[q] * ld + c] = tmp[t];
  }
}

// U12 = L11^-1 A12 (unit lower), one thread per column right of the panel.
__global__ void __launch_bounds__(128) trsm_kernel(double2 *a, long long n, long long ld, long long k0, int kb) {
  __shared__ double2 L[KB][KB + 1];
  for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
    const int i = t / kb, j = t % kb;
    L[i][j] = a[(k0 + i) * ld + k0 + j];
  }
  __syncthreads();
  const long long c = k0 + kb + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= n) return;
  double2 x[KB];
#pragma unroll
  for (int i = 0; i < KB; ++i) x[i] = i < kb ? a[(k0 + i) * ld + c] : make_double2(0, 0);
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
  for (int i = 1; i < KB; ++i) if (i < kb) a[(k0 + i) * ld + c] = x[i];
}

// C[M x N] -= A[M x K] B[K x N], row-major complex FP64 blocks (leading dim ld).
constexpr int GT = 64;   // tile edge
constexpr int GK = 16;   // K chunk
__global__ void __launch_bounds__(256) gemm_update_kernel(double2 *C, const double2 *A, const double2 *B,
                                                          long long M, long long N, int K, long long ld) {
  __shared__ double2 As[GK][GT + 1];
  __shared__ double2 Bs[GK][GT + 1];
  const long long row0 = blockIdx.y * (long long)GT, col0 = blockIdx.x * (long long)GT;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // 16 x 16 threads, 4 x 4 each
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0, 0);
  for (int k0 = 0; k0 < K; k0 += GK) {
    for (int t = threadIdx.x; t < GT * GK; t += 256) {
      const int k = t % GK, r = t / GK;
      const long long gr = row0 + r;
      As[k][r] = (gr < M && k0 + k < K) ? A[gr * ld + k0 + k] : make_double2(0, 0);
      const int cc = t % GT, kk = t / GT;
      const long long gc = col0 + cc;
      Bs[kk][cc] = (gc < N && k0 + kk < K) ? B[(long long)(k0 + kk) * ld + gc] : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < GK; ++k) {
      double2 av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[k][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[k][tx + 16 * j];
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
      const long long r = row0 + ty + 16 * i, c = col0 + tx + 16 * j;
      if (r < M && c < N) {
        double2 *q = C + r * ld + c;
        *q = csub(*q, acc[i][j]);
      }
    }
}

// Solve with the row-major getrf-convention factors: all interchanges, unit
// lower forward substitution, upper back substitution (the system
// matrix.c:1523-1555 solves).  One block per RHS; each 32-row step is solved
// by warp 0 and the rows below / above are updated by the whole block with
// contiguous row segments.
__global__ void __launch_bounds__(1024) lu_solve_kernel(const double2 *a, long long n, long long ld,
                                                        const int *ipiv, double2 *b, long long ldb) {
  double2 *x = b + blockIdx.x * ldb;
  __shared__ double2 xs[32];
  if (threadIdx.x == 0)
    for (long long i = 0; i < n; ++i) {
      const long long pi = ipiv[i] - 1;
      if (pi != i) { const double2 t = x[pi]; x[pi] = x[i]; x[i] = t; }
    }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // Forward: L unit lower.
  for (long long j0 = 0; j0 < n; j0 += 32) {
    const int w = (int)(n - j0 < 32 ? n - j0 : 32);
    if (warp == 0) {
      double2 v = lane < w ? x[j0 + lane] : make_double2(0, 0);
      for (int i = 1; i < w; ++i) {
        // Row j0+i of the diagonal block against the solved entries above it.
        const double2 l = lane < i ? a[(j0 + i) * ld + j0 + lane] : make_double2(0, 0);
        double2 s = cmul(l, make_double2(__shfl_sync(0xffffffffu, v.x, lane), __shfl_sync(0xffffffffu, v.y, lane)));
        s = lane < i ? s : make_double2(0, 0);
        for (int o = 16; o > 0; o >>= 1) {
          s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
          s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
        }
        if (lane == i) v = csub(v, s);
      }
      if (lane < w) { x[j0 + lane] = v; xs[lane] = v; }
    }
    __syncthreads();
    for (long long r = j0 + w + warp; r < n; r += nw) {
      double2 s = lane < w ? cmul(a[r * ld + j0 + lane], xs[lane]) : make_double2(0, 0);
      for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      }
      if (lane == 0) x[r] = csub(x[r], s);
    }
    __syncthreads();
  }
  // Backward: U upper.
  for (long long j1 = n; j1 > 0; j1 -= 32) {
    const long long j0 = j1 - 32 > 0 ? j1 - 32 : 0;
    const int w = (int)(j1 - j0);
    if (warp == 0) {
      double2 v = lane < w ? x[j0 + lane] : make_double2(0, 0);
      for (int i = w - 1; i >= 0; --i) {
        const double2 u = (lane > i && lane < w) ? a[(j0 + i) * ld + j0 + lane] : make_double2(0, 0);
        double2 s = cmul(u, v);
        s = (lane > i && lane < w) ? s : make_double2(0, 0);
        for (int o = 16; o > 0; o >>= 1) {
          s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
          s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
        }
        if (lane == i) v = cdiv(csub(v, s), a[(j0 + i) * ld + j0 + i]);
      }
      if (lane < w) { x[j0 + lane] = v; xs[lane] = v; }
    }
    __syncthreads();
    for (long long r = warp; r < j0; r += nw) {
      double2 s = lane < w ? cmul(a[r * ld + j0 + lane], xs[lane]) : make_double2(0, 0);
      for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      }
      if (lane == 0) x[r] = csub(x[r], s);
    }
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

static unsigned blocks_for(long long work) {
  long long b = (work + 255) / 256;
  const long long cap = (long long)n2c_sm_count() * 8;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

extern "C" int n2d_lu_factor(double *a_dev, long long n, long long ld, int *ipiv, int rule, int precision,
                             int *info_host) {
  (void)precision;
  *info_host = 0;
  if (n <= 0) return 1;
  double2 *a = (double2 *)a_dev;
  const long long grid_blocks = (n + PT - 1) / PT;
  // Cluster panel with 256 or 512 threads per CTA (one row each); beyond
  // 8 x 512 rows the cooperative-grid panel.
  const int rows_per_thread = n <= (long long)CS * 256 ? 1 : (n <= (long long)CS * 512 ? 2 : 0);
  LuStatus *st = (LuStatus *)n2d_alloc(sizeof(LuStatus));
  int *pairs = (int *)n2d_alloc(4 * KB * sizeof(int));
  double2 *tmp = (double2 *)n2d_alloc((size_t)2 * KB * n * sizeof(double2));
  double *gval = nullptr;
  int *gidx = nullptr;
  double2 *grow = nullptr, *growj = nullptr;
  if (!rows_per_thread) {
    gval = (double *)n2d_alloc(2 * grid_blocks * sizeof(double));
    gidx = (int *)n2d_alloc(2 * grid_blocks * sizeof(int));
    grow = (double2 *)n2d_alloc(2 * grid_blocks * KB * sizeof(double2));
    growj = (double2 *)n2d_alloc(2 * KB * sizeof(double2));
  }
  int ok = st && pairs && tmp && n2d_memset(st, 0, sizeof(LuStatus)) &&
           (rows_per_thread || (gval && gidx && grow && growj));
  for (long long k0 = 0; ok && k0 < n; k0 += KB) {
    const int kb = (int)(n - k0 < KB ? n - k0 : KB);
    PanelArgs p;
    memset(&p, 0, sizeof(p));
    p.a = a; p.n = n; p.ld = ld; p.k0 = k0; p.kb = kb; p.rule = rule; p.ipiv = ipiv;
    p.pairs = pairs; p.st = st; p.gval = gval; p.gidx = gidx; p.grow = grow; p.growj = growj;
    if (rows_per_thread == 1) {
      panel_cluster_kernel<256><<<CS, 256, 0, n2c_stream()>>>(p);
      if (!n2c_check_launch("panel")) { ok = 0; break; }
    } else if (rows_per_thread == 2) {
      panel_cluster_kernel<512><<<CS, 512, 0, n2c_stream()>>>(p);
      if (!n2c_check_launch("panel")) { ok = 0; break; }
    } else {
      const int blocks = (int)((n - k0 + PT - 1) / PT);
      void *args[] = {&p};
      cudaError_t e = cudaLaunchCooperativeKernel((void *)panel_grid_kernel, blocks, PT, args, 0, n2c_stream());
      if (e != cudaSuccess) { n2c_set_error("panel launch: %s", cudaGetErrorString(e)); ok = 0; break; }
      n2c_count_launch(1);
    }
    if (n > kb) {
      const unsigned gb = blocks_for(2LL * KB * (n - kb));
      rows_gather_kernel<<<gb, 256, 0, n2c_stream()>>>(a, n, ld, k0, kb, pairs, st, tmp);
      rows_scatter_kernel<<<gb, 256, 0, n2c_stream()>>>(a, n, ld, k0, kb, pairs, st, tmp);
      if (!n2c_check_launch("interchanges")) { ok = 0; break; }
      n2c_count_launch(1);
    }
    const long long right = n - k0 - kb;
    if (right > 0) {
      trsm_kernel<<<(unsigned)((right + 127) / 128), 128, 0, n2c_stream()>>>(a, n, ld, k0, kb);
      if (!n2c_check_launch("trsm")) { ok = 0; break; }
      dim3 grid((unsigned)((right + GT - 1) / GT), (unsigned)((right + GT - 1) / GT));
      gemm_update_kernel<<<grid, 256, 0, n2c_stream()>>>(a + (k0 + kb) * ld + (k0 + kb), a + (k0 + kb) * ld + k0,
                                                         a + k0 * ld + (k0 + kb), right, right, kb, ld);
      if (!n2c_check_launch("gemm_update")) { ok = 0; break; }
    }
  }
  LuStatus hs;
  memset(&hs, 0, sizeof(hs));
  if (ok && !n2d_download(&hs, st, sizeof(hs))) ok = 0;
  if (ok && hs.error) { n2c_set_error("LU panel barrier time-out"); ok = 0; }
  *info_host = hs.info;
  n2d_free(st); n2d_free(pairs); n2d_free(tmp);
  n2d_free(gval); n2d_free(gidx); n2d_free(grow); n2d_free(growj);
  return ok;
}

extern "C" int n2d_lu_solve(const double *a_dev, long long n, long long ld, const int *ipiv, double *b_dev,
                            long long ldb, long long nrhs) {
  if (n <= 0 || nrhs <= 0) return 1;
  lu_solve_kernel<<<(unsigned)nrhs, 1024, 0, n2c_stream()>>>((const double2 *)a_dev, n, ld, ipiv,
                                                             (double2 *)b_dev, ldb);
  return n2c_check_launch("lu_solve");
}

// ------------------------------------------------------ allocation-free factor
// A variant of the classic factor for callers that cannot allocate device
// memory when they call in: a host application that hands the GPU's memory to
// its own pool allocator at start-up and forbids allocation afterwards, a
// plug-in living inside such a process, or a loop with a latency budget that
// cudaMalloc's implicit device synchronisation would break.  The caller passes
// the matrix and the pivot array already resident on the device; the panel
// status, the interchange pairs and the row buffer of the interchanges live in
// one array defined in this file instead of being allocated per call.
//
// That array is a module global: every GPU on which the library is loaded
// holds it (4 MiB + 1 KiB) until the process exits, and every call on that
// GPU shares it.  Calls whose work overlaps on the GPU (two streams, two host
// threads) therefore race on it; callers serialise them.  The array keeps the
// previous call's contents; only the panel status needs to start at zero and
// is cleared at the start of every call.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address (cudaGetSymbolAddress; the array's name in host code
// is only a stand-in) and keeps it.  Make that first call before any stream
// capture on the device.
#include <climits>
#include <mutex>
#include "../../include/nec2c_cuda.h"

namespace {
constexpr size_t STATIC_STATUS_OFF = 0;
constexpr size_t STATIC_PAIRS_OFF = 256;
constexpr size_t STATIC_ROWS_OFF = 1024;
constexpr size_t STATIC_SCRATCH_BYTES =
    STATIC_ROWS_OFF + (size_t)2 * KB * NEC2C_CUDA_STATIC_LU_MAX_ORDER * sizeof(double2);
static_assert(sizeof(LuStatus) <= STATIC_PAIRS_OFF - STATIC_STATUS_OFF, "status slot");
static_assert(4 * KB * sizeof(int) <= STATIC_ROWS_OFF - STATIC_PAIRS_OFF, "pairs slot");
constexpr int STATIC_MAX_DEVICES = 64;
std::mutex g_static_lock;
unsigned char *g_static_addr[STATIC_MAX_DEVICES];
}  // namespace

static __device__ __align__(256) unsigned char lu_static_scratch[STATIC_SCRATCH_BYTES];

// Device address of the scratch array on the current device (looked up once
// per device).
static unsigned char *static_scratch() {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { n2c_set_error("cudaGetDevice: %s", cudaGetErrorString(e)); return nullptr; }
  if (dev < 0 || dev >= STATIC_MAX_DEVICES) { n2c_set_error("device %d out of range", dev); return nullptr; }
  std::lock_guard<std::mutex> hold(g_static_lock);
  if (!g_static_addr[dev]) {
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, lu_static_scratch);
    if (e != cudaSuccess || !ptr) {
      n2c_set_error("scratch address on device %d: %s", dev, cudaGetErrorString(e));
      return nullptr;
    }
    g_static_addr[dev] = (unsigned char *)ptr;
  }
  return g_static_addr[dev];
}

extern "C" int nec2c_cuda_dense_factor_device_static(size_t order, nec2c_cuda_complex *matrix_dev,
                                                     size_t leading_dimension, int *pivots_dev) {
  if (!matrix_dev || !pivots_dev || order == 0 || leading_dimension < order ||
      leading_dimension > (size_t)INT_MAX) {
    n2c_set_error("invalid arguments");
    return 0;
  }
  if (order > NEC2C_CUDA_STATIC_LU_MAX_ORDER) {
    n2c_set_error("order %zu exceeds the allocation-free factor's maximum of %d", order,
                  NEC2C_CUDA_STATIC_LU_MAX_ORDER);
    return 0;
  }
  if (!n2d_device_ok()) return 0;
  unsigned char *base = static_scratch();
  if (!base) return 0;
  LuStatus *st = (LuStatus *)(base + STATIC_STATUS_OFF);
  int *pairs = (int *)(base + STATIC_PAIRS_OFF);
  double2 *tmp = (double2 *)(base + STATIC_ROWS_OFF);
  double2 *a = (double2 *)matrix_dev;
  const long long n = (long long)order, ld = (long long)leading_dimension;
  cudaStream_t s = n2c_stream();
  cudaError_t e = cudaMemsetAsync(st, 0, sizeof(LuStatus), s);
  if (e != cudaSuccess) { n2c_set_error("clearing the panel status: %s", cudaGetErrorString(e)); return 0; }
  int ok = 1;
  for (long long k0 = 0; ok && k0 < n; k0 += KB) {
    const int kb = (int)(n - k0 < KB ? n - k0 : KB);
    PanelArgs p;
    memset(&p, 0, sizeof(p));
    p.a = a; p.n = n; p.ld = ld; p.k0 = k0; p.kb = kb; p.rule = 0; p.ipiv = pivots_dev;
    p.pairs = pairs; p.st = st;
    if (n <= (long long)CS * 256) panel_cluster_kernel<256><<<CS, 256, 0, s>>>(p);
    else panel_cluster_kernel<512><<<CS, 512, 0, s>>>(p);
    if (!n2c_check_launch("panel")) { ok = 0; break; }
    if (n > kb) {
      const unsigned gb = blocks_for(2LL * KB * (n - kb));
      rows_gather_kernel<<<gb, 256, 0, s>>>(a, n, ld, k0, kb, pairs, st, tmp);
      rows_scatter_kernel<<<gb, 256, 0, s>>>(a, n, ld, k0, kb, pairs, st, tmp);
      if (!n2c_check_launch("interchanges")) { ok = 0; break; }
      n2c_count_launch(1);
    }
    const long long right = n - k0 - kb;
    if (right > 0) {
      trsm_kernel<<<(unsigned)((right + 127) / 128), 128, 0, s>>>(a, n, ld, k0, kb);
      if (!n2c_check_launch("trsm")) { ok = 0; break; }
      dim3 grid((unsigned)((right + GT - 1) / GT), (unsigned)((right + GT - 1) / GT));
      gemm_update_kernel<<<grid, 256, 0, s>>>(a + (k0 + kb) * ld + (k0 + kb), a + (k0 + kb) * ld + k0,
                                              a + k0 * ld + (k0 + kb), right, right, kb, ld);
      if (!n2c_check_launch("gemm_update")) { ok = 0; break; }
    }
  }
  if (!ok) return 0;
  LuStatus hs;
  memset(&hs, 0, sizeof(hs));
  e = cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) { n2c_set_error("reading the panel status: %s", cudaGetErrorString(e)); return 0; }
  if (hs.error) { n2c_set_error("LU panel barrier time-out"); return 0; }
  if (hs.info) { n2c_set_error("matrix is singular (pivot %d)", hs.info); return 0; }
  return 1;
}

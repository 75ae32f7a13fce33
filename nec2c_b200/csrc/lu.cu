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
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <vector>
#include "common.cuh"
#include "device_api.h"
#include "runtime.cuh"

namespace cg = cooperative_groups;
using namespace n2c;

namespace {

constexpr int KB = 32;        // panel width
constexpr int PT = 256;       // panel threads per CTA

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
  void *a;                    // the matrix: double2 (FP64 form) or float2 (split-precision form)
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
// piv_rel: the panel's pivot rows relative to k0 (shared memory), or null to
// read them from ipiv.
__device__ void panel_pairs_warp(const PanelArgs &p, const int *piv_rel = nullptr) {
  __shared__ int rows[2 * KB], src[2 * KB], cnt;
  const int lane = threadIdx.x & 31;
  const int k0 = (int)p.k0, kb = p.kb;
  for (int u = lane; u < 2 * KB; u += 32) { rows[u] = u < kb ? k0 + u : -1; src[u] = rows[u]; }
  if (lane == 0) cnt = kb;
  __syncwarp();
  for (int i = 0; i < kb; ++i) {
    const int q = piv_rel ? k0 + piv_rel[i] : p.ipiv[k0 + i] - 1;
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

// Cluster panel.  A cluster of CSZ CTAs (256 threads each) keeps the panel in
// registers: CTA r holds panel rows r*256 .. r*256+255; warp w of a CTA holds
// columns 4w..4w+3 and lane L the rows L, L+32, ..., L+224 of them.  Rows are
// never moved while the panel is factored: each row carries its logical
// position (pos), interchanges only exchange positions, and the rows are
// written to their final positions at the end.  Per column j (owned by warp
// wj = j/4):
//   1  warp wj: best candidate of the CTA (rows with pos >= j), published to
//      the CTA through a local mbarrier, and its header pushed to every CTA
//   2  every warp pushes its four elements of that candidate row to every CTA
//      (st.async, counted in transaction bytes on the receiver's mbarrier)
//   3  every warp waits for all CTAs' candidates, picks the winner in rank
//      order and exchanges positions (pivot row -> j, row at j -> old place)
//   4  warp wj forms the multipliers, publishes them through shared memory and
//      a local mbarrier, and updates its own later columns
//   5  warps w > wj apply the rank-1 update to their four columns
// There is no CTA-wide barrier per column; every wait is bounded.  Buffers and
// mbarriers alternate by column parity; reuse is safe because a warp reaches
// column j+2's publication only after every warp of every CTA has pushed
// column j+1, which each did after finishing its reads of column j.
constexpr int CROWS = 256;            // panel rows per CTA
constexpr int CPT = 256;              // threads per CTA (8 warps x 4 columns)
constexpr int CRL = CROWS / 32;       // rows per lane
constexpr int CCW = KB / (CPT / 32);  // columns per warp
constexpr int CMAX = 16;              // largest cluster (non-portable size, opt-in)

struct CandEntry {
  double val;
  int idx, pad;
  double2 row[KB];
};

template <int CSZ>
struct PanelShared {
  CandEntry cand[2][CSZ];             // candidates pushed by every CTA
  double2 mult[2][CROWS];             // multipliers of column j (by physical row)
  double best_val[2];
  int best_idx[2], best_phys[2];      // CTA best: logical index, physical row
  unsigned long long xbar[2], lbar[2], mbar[2];
  int piv[KB];                        // panel-relative pivot rows
  int info;                           // first zero pivot (column + 1), 0 = none
  int fail;
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint32_t cluster_addr(uint32_t local, int rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}
// 16-byte store into a CTA's shared memory (any CTA of the cluster),
// completing 16 transaction bytes on that CTA's mbarrier.
__device__ __forceinline__ void push16(uint32_t dst, uint4 v, uint32_t bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];"
               :: "r"(dst), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(bar) : "memory");
}
__device__ __forceinline__ uint4 as_u4(double2 v) {
  return make_uint4((unsigned)__double2loint(v.x), (unsigned)__double2hiint(v.x), (unsigned)__double2loint(v.y),
                    (unsigned)__double2hiint(v.y));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect(uint32_t bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t bar, unsigned parity) {
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
  return ok != 0;
}
// Bounded wait (about a second at boost clock) that also gives up as soon as
// another warp of the CTA has recorded a failure; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, unsigned parity, const int *fail) {
  if (mbar_test(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_test(bar, parity))
    if (*(volatile const int *)fail || clock64() - t0 > (1LL << 31)) return false;
  return true;
}

// Column j = 4*wj + CC (CC compile-time) for this thread: a[k][c] is row
// L+32k, column 4*warp+c; pos[k] its logical position (panel-relative).
template <int CSZ, int CC, int RULE>
__device__ __forceinline__ bool panel_column(const PanelArgs &p, PanelShared<CSZ> &sh, double2 (&a)[CRL][CCW],
                                             int (&pos)[CRL], int rank, int wj) {
  constexpr unsigned XBYTES = CSZ * sizeof(CandEntry);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j = CCW * wj + CC, buf = j & 1;
  const unsigned par = (unsigned)(j >> 1) & 1u;
  const uint32_t xbar = smem_addr(&sh.xbar[buf]);
  if (threadIdx.x == 0) mbar_expect(xbar, XBYTES);
  // 1: the CTA's best candidate of column j.
  if (warp == wj) {
    double bv = -1.0;
    int bi = -1, bk = 0;
#pragma unroll
    for (int k = 0; k < CRL; ++k) {
      if (pos[k] >= j && pos[k] < p.n - p.k0) {
        const double m = magnitude(a[k][CC], RULE);
        if (bi < 0 || better(m, pos[k], bv, bi, RULE)) { bv = m; bi = pos[k]; bk = k; }
      }
    }
    int bp = bi >= 0 ? lane + 32 * bk : -1;
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      const int op = __shfl_xor_sync(0xffffffffu, bp, o);
      if (oi >= 0 && (bi < 0 || better(ov, oi, bv, bi, RULE))) { bv = ov; bi = oi; bp = op; }
    }
    if (lane < CSZ) {
      const uint4 hdr = make_uint4((unsigned)__double2loint(bv), (unsigned)__double2hiint(bv), (unsigned)bi, 0u);
      push16(cluster_addr(smem_addr(&sh.cand[buf][rank]), lane), hdr, cluster_addr(xbar, lane));
    }
    if (lane == 0) {
      sh.best_val[buf] = bv;
      sh.best_idx[buf] = bi;
      sh.best_phys[buf] = bp;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_addr(&sh.lbar[buf]));
  }
  // 2: every warp pushes its elements of the candidate row.
  if (!mbar_wait(smem_addr(&sh.lbar[buf]), par, &sh.fail)) return false;
  {
    const int bp = sh.best_phys[buf];
    const int hl = bp >= 0 ? (bp & 31) : 0, hk = bp >= 0 ? (bp >> 5) : 0;
    double2 v[CCW];
#pragma unroll
    for (int c = 0; c < CCW; ++c) v[c] = make_double2(0, 0);
    if (lane == hl) {
      switch (hk) {
#define N2C_TAKE(K) case K: _Pragma("unroll") for (int c = 0; c < CCW; ++c) v[c] = a[K][c]; break;
        N2C_TAKE(0) N2C_TAKE(1) N2C_TAKE(2) N2C_TAKE(3) N2C_TAKE(4) N2C_TAKE(5) N2C_TAKE(6) N2C_TAKE(7)
#undef N2C_TAKE
        default: break;
      }
    }
#pragma unroll
    for (int c = 0; c < CCW; ++c) {
      v[c].x = __shfl_sync(0xffffffffu, v[c].x, hl);
      v[c].y = __shfl_sync(0xffffffffu, v[c].y, hl);
    }
    if (lane < CSZ) {
      const uint32_t rb = cluster_addr(xbar, lane);
#pragma unroll
      for (int c = 0; c < CCW; ++c)
        push16(cluster_addr(smem_addr(&sh.cand[buf][rank].row[CCW * warp + c]), lane), as_u4(v[c]), rb);
    }
  }
  // 3: the winner (fixed rank order) and the position exchange.
  if (!mbar_wait(xbar, par, &sh.fail)) return false;
  double v = -2.0;
  int pi = -1;
  if (lane < CSZ) { v = sh.cand[buf][lane].val; pi = sh.cand[buf][lane].idx; }
  int pr = lane;
  for (int o = CSZ >> 1; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, pi, o);
    const int orr = __shfl_xor_sync(0xffffffffu, pr, o);
    if (oi >= 0 && (pi < 0 || better(ov, oi, v, pi, RULE))) { v = ov; pi = oi; pr = orr; }
  }
  v = __shfl_sync(0xffffffffu, v, 0);
  pi = __shfl_sync(0xffffffffu, pi, 0);
  pr = __shfl_sync(0xffffffffu, pr, 0);
  const bool zero = RULE == 0 ? !(v > 0.0) : !(v > 64.0 * DBL_EPSILON);
#pragma unroll
  for (int k = 0; k < CRL; ++k) {
    if (pos[k] == pi) pos[k] = j;
    else if (pos[k] == j) pos[k] = pi;
  }
  if (threadIdx.x == 0) {
    sh.piv[j] = pi;
    if (zero && sh.info == 0) sh.info = j + 1;
  }
  const double2 *prow = sh.cand[buf][pr].row;
  // 4: multipliers (by the reciprocal, as factr does, matrix.c:1393-1398).
  if (warp == wj) {
    double2 l[CRL];
    const double2 pv = prow[j];
    const double r = 1.0 / (pv.x * pv.x + pv.y * pv.y);
    const double2 inv = make_double2(pv.x * r, -pv.y * r);
#pragma unroll
    for (int k = 0; k < CRL; ++k) {
      l[k] = make_double2(0, 0);
      if (!zero && pos[k] > j && pos[k] < p.n - p.k0) { l[k] = cmul(a[k][CC], inv); a[k][CC] = l[k]; }
      sh.mult[buf][lane + 32 * k] = l[k];
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_addr(&sh.mbar[buf]));
    if (!zero) {
#pragma unroll
      for (int c = CC + 1; c < CCW; ++c) {
        const double2 u = prow[CCW * warp + c];
#pragma unroll
        for (int k = 0; k < CRL; ++k)
          if (pos[k] > j && pos[k] < p.n - p.k0) a[k][c] = csub(a[k][c], cmul(l[k], u));
      }
    }
  } else if (warp > wj) {
    // 5: rank-1 update of this warp's columns.
    if (!mbar_wait(smem_addr(&sh.mbar[buf]), par, &sh.fail)) return false;
    if (!zero) {
      double2 u[CCW];
#pragma unroll
      for (int c = 0; c < CCW; ++c) u[c] = prow[CCW * warp + c];
#pragma unroll
      for (int k = 0; k < CRL; ++k) {
        if (!(pos[k] > j && pos[k] < p.n - p.k0)) continue;
        const double2 lk = sh.mult[buf][lane + 32 * k];
#pragma unroll
        for (int c = 0; c < CCW; ++c) a[k][c] = csub(a[k][c], cmul(lk, u[c]));
      }
    }
  }
  return true;
}

template <int CSZ, int RULE, typename S>
__device__ __forceinline__ void panel_cluster_body(const PanelArgs &p) {
  static_assert(sizeof(CandEntry) % 16 == 0 && CSZ <= 32 && CCW == 4 && KB == 32, "panel layout");
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ __align__(16) PanelShared<CSZ> sh;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_addr(&sh.xbar[b]), 1);
      mbar_init(smem_addr(&sh.lbar[b]), 1);
      mbar_init(smem_addr(&sh.mbar[b]), 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    sh.fail = 0;
    sh.info = 0;
    if (rank == 0) p.st->npairs = 0;   // the CTAs append their moved rows at the end
  }
  cluster.sync();
  const long long rows = p.n - p.k0;
  double2 a[CRL][CCW];
  int pos[CRL];
#pragma unroll
  for (int k = 0; k < CRL; ++k) {
    const int g = rank * CROWS + lane + 32 * k;
    pos[k] = g < rows ? g : INT_MAX;
    const S *row = (const S *)p.a + (p.k0 + g) * p.ld + p.k0 + CCW * warp;
#pragma unroll
    for (int c = 0; c < CCW; ++c)
      a[k][c] = (g < rows && CCW * warp + c < p.kb) ? to_d(row[c]) : make_double2(0, 0);
  }
  bool ok = true;
  for (int wj = 0; wj < KB / CCW && ok; ++wj) {
    if (CCW * wj + 0 < p.kb) ok = panel_column<CSZ, 0, RULE>(p, sh, a, pos, rank, wj);
    if (ok && CCW * wj + 1 < p.kb) ok = panel_column<CSZ, 1, RULE>(p, sh, a, pos, rank, wj);
    if (ok && CCW * wj + 2 < p.kb) ok = panel_column<CSZ, 2, RULE>(p, sh, a, pos, rank, wj);
    if (ok && CCW * wj + 3 < p.kb) ok = panel_column<CSZ, 3, RULE>(p, sh, a, pos, rank, wj);
  }
  if (!ok) sh.fail = 1;
  cluster.sync();   // no CTA exits while others may still push into it
  if (sh.fail) {
    if (threadIdx.x == 0) atomicExch(&p.st->error, 1);
    return;
  }
#pragma unroll
  for (int k = 0; k < CRL; ++k) {
    if (pos[k] == INT_MAX) continue;
    S *row = (S *)p.a + (p.k0 + pos[k]) * p.ld + p.k0 + CCW * warp;
#pragma unroll
    for (int c = 0; c < CCW; ++c) if (CCW * warp + c < p.kb) row[c] = from_d<S>(a[k][c]);
  }
  if (rank == 0 && warp == 0) {
    for (int j = lane; j < p.kb; j += 32) p.ipiv[p.k0 + j] = (int)(p.k0 + sh.piv[j] + 1);
    if (lane == 0 && sh.info && p.st->info == 0) p.st->info = (int)(p.k0 + sh.info);
  }
  // Net interchange of the panel: a row now at position pos[k] holds the old
  // row g, so destination k0 + pos[k] takes source k0 + g.  Warp 0 of each
  // CTA appends its moved rows (at most 2 KB over the cluster).
  if (warp == 0) {
    unsigned moved[CRL];
    int total = 0;
#pragma unroll
    for (int k = 0; k < CRL; ++k) {
      const int g = rank * CROWS + lane + 32 * k;
      moved[k] = __ballot_sync(0xffffffffu, pos[k] != INT_MAX && pos[k] != g);
      total += __popc(moved[k]);
    }
    int base = 0;
    if (lane == 0 && total) base = atomicAdd(&p.st->npairs, total);
    base = __shfl_sync(0xffffffffu, base, 0);
    const unsigned below = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < CRL; ++k) {
      if (moved[k] >> lane & 1u) {
        const int at = base + __popc(moved[k] & below);
        p.pairs[at] = (int)(p.k0 + pos[k]);
        p.pairs[2 * KB + at] = (int)(p.k0 + rank * CROWS + lane + 32 * k);
      }
      base += __popc(moved[k]);
    }
  }
}

template <int CSZ, int RULE, typename S>
__global__ void __launch_bounds__(CPT, 1) panel_cluster_kernel(PanelArgs p) {
  panel_cluster_body<CSZ, RULE, S>(p);
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

template <typename S>
__global__ void __launch_bounds__(PT) panel_grid_kernel(PanelArgs p) {
  const long long rows = p.n - p.k0;
  double2 a[1][KB];
  int g[1] = {(int)(blockIdx.x * PT + threadIdx.x)};
  bool have[1] = {g[0] < rows};
  const S *row0 = (const S *)p.a + (p.k0 + g[0]) * p.ld + p.k0;
#pragma unroll
  for (int c = 0; c < KB; ++c) a[0][c] = (have[0] && c < p.kb) ? to_d(row0[c]) : make_double2(0, 0);
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
  S *row = (S *)p.a + (p.k0 + g[0]) * p.ld + p.k0;
#pragma unroll
  for (int c = 0; c < KB; ++c) if (have[0] && c < p.kb) row[c] = from_d<S>(a[0][c]);
  if (blockIdx.x == 0 && threadIdx.x < 32) panel_pairs_warp(p);
}

// Row interchanges outside the panel columns [k0, k0+kb) and, right of the
// panel, U12 = L11^-1 A12 (unit lower).  One warp per column: its lanes gather
// the source rows of the interchange pairs into registers, then scatter them
// (so overlapping pairs need no scratch), then lane i holds row k0+i of the
// column and the forward substitution runs column-oriented, broadcasting x_k
// by shuffle; each x_i subtracts L[i][k] x_k in increasing k, the order of the
// row-oriented sum.
constexpr int SWT = 256;   // threads per block (8 columns)
// For the split-precision form (S = float2) the kernel also writes column c of
// U12, as stored, into the packed real expansion the tensor-core update reads:
// rows 2c', 2c'+1 (c' = c - k0 - kb) of 64 floats, (Re, -Im) and (Im, Re) per
// k, each split into a TF32-representable hi part and the FP32 remainder.
template <typename S>
__device__ __forceinline__ void swap_trsm_body(S *a, long long n, long long ld, long long k0, int kb,
                                               const int *pairs, const LuStatus *st, float *bt_hi, float *bt_lo,
                                               long long blk) {
  __shared__ int dst[2 * KB], src[2 * KB];
  __shared__ double2 L[KB][KB + 1];
  const int np = st->npairs;
  for (int t = threadIdx.x; t < np; t += blockDim.x) { dst[t] = pairs[t]; src[t] = pairs[2 * KB + t]; }
  const long long first = blk * (SWT / 32);
  const long long cols = n - kb;
  const bool any_right = first + SWT / 32 - 1 >= k0;   // some column of this block is right of the panel
  if (any_right) {
    for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
      const int i = t / kb, j = t % kb;
      L[i][j] = to_d(a[(k0 + i) * ld + k0 + j]);
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long c0 = first + (threadIdx.x >> 5);
  if (c0 >= cols) return;
  const long long c = c0 < k0 ? c0 : c0 + kb;
  S v0 = a[0], v1 = a[0];
  if (lane < np) v0 = a[(long long)src[lane] * ld + c];
  if (lane + 32 < np) v1 = a[(long long)src[lane + 32] * ld + c];
  __syncwarp();
  if (lane < np) a[(long long)dst[lane] * ld + c] = v0;
  if (lane + 32 < np) a[(long long)dst[lane + 32] * ld + c] = v1;
  if (c < k0) return;
  __syncwarp();
  double2 x = lane < kb ? to_d(a[(k0 + lane) * ld + c]) : make_double2(0, 0);
#pragma unroll
  for (int k = 0; k < KB - 1; ++k) {
    double2 xk;
    xk.x = __shfl_sync(0xffffffffu, x.x, k);
    xk.y = __shfl_sync(0xffffffffu, x.y, k);
    if (lane > k && lane < kb) x = csub(x, cmul(L[lane][k], xk));
  }
  const S u = from_d<S>(x);
  if (lane >= 1 && lane < kb) a[(k0 + lane) * ld + c] = u;
  if (bt_hi) {
    const long long r2 = 2 * (c - k0 - kb);
    const double2 v = lane < kb ? to_d(u) : make_double2(0, 0);
    const float re = (float)v.x, im = (float)v.y;
    const float e[4] = {re, -im, im, re};   // row 2c' (k: Re, -Im), row 2c'+1 (k: Im, Re)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float h = __uint_as_float(__float_as_uint(e[q]) & 0xFFFFE000u);
      const long long at = (r2 + (q >> 1)) * (2 * KB) + 2 * lane + (q & 1);
      bt_hi[at] = h;
      bt_lo[at] = e[q] - h;
    }
  }
}

template <typename S>
__global__ void __launch_bounds__(SWT) swap_trsm_kernel(S *a, long long n, long long ld, long long k0, int kb,
                                                        const int *pairs, const LuStatus *st, float *bt_hi,
                                                        float *bt_lo) {
  swap_trsm_body<S>(a, n, ld, k0, kb, pairs, st, bt_hi, bt_lo, blockIdx.x);
}

// C[M x N] -= A[M x K] B[K x N], row-major complex FP64 blocks (leading dim ld).
// The K chunks are copied into two shared-memory stages by cp.async, the next
// chunk's copy in flight while the current one is multiplied (a panel's
// K = 32 is two chunks, so both loads go out at once); each C element's
// products are summed in increasing k as before.
constexpr int GT = 64;   // tile edge
constexpr int GK = 16;   // K chunk
constexpr size_t GEMM_STAGE = (size_t)GK * (GT + 1) * sizeof(double2);
constexpr size_t GEMM_SMEM = 4 * GEMM_STAGE;   // A and B, two stages each (66,560 bytes)
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void gemm_update_body(double2 *C, const double2 *A, const double2 *B, long long M,
                                                 long long N, int K, long long ld, long long row0, long long col0) {
  extern __shared__ __align__(16) unsigned char gemm_smem[];
  typedef double2 Stage[GK][GT + 1];
  Stage *As = reinterpret_cast<Stage *>(gemm_smem), *Bs = reinterpret_cast<Stage *>(gemm_smem + 2 * GEMM_STAGE);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // 16 x 16 threads, 4 x 4 each
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0, 0);
  auto stage = [&](int st, int k0) {
    for (int t = threadIdx.x; t < GT * GK; t += 256) {
      const int k = t % GK, r = t / GK;
      const long long gr = row0 + r;
      if (gr < M && k0 + k < K) cp_async16(&As[st][k][r], A + gr * ld + k0 + k);
      else As[st][k][r] = make_double2(0, 0);
      const int cc = t % GT, kk = t / GT;
      const long long gc = col0 + cc;
      if (gc < N && k0 + kk < K) cp_async16(&Bs[st][kk][cc], B + (long long)(k0 + kk) * ld + gc);
      else Bs[st][kk][cc] = make_double2(0, 0);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  const int chunks = (K + GK - 1) / GK;
  if (chunks > 0) stage(0, 0);
  for (int ch = 0; ch < chunks; ++ch) {
    const int st = ch & 1;
    if (ch + 1 < chunks) {
      stage(st ^ 1, (ch + 1) * GK);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < GK; ++k) {
      double2 av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[st][k][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[st][k][tx + 16 * j];
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
__global__ void __launch_bounds__(256, 2) gemm_update_kernel(double2 *C, const double2 *A, const double2 *B,
                                                          long long M, long long N, int K, long long ld) {
  gemm_update_body(C, A, B, M, N, K, ld, blockIdx.y * (long long)GT, blockIdx.x * (long long)GT);
}

// Solve with the row-major getrf-convention factors: all interchanges, unit
// lower forward substitution, upper back substitution (the system
// matrix.c:1523-1555 solves).  One block per RHS; each 32-row step is solved
// by warp 0 and the rows below / above are updated by the whole block with
// contiguous row segments.
// One right-hand side per CTA (512 threads).  Interchanges: the sequential
// swaps of ipiv are composed into an index permutation in shared memory by
// one thread (orders up to SOLVE_PERM_MAX; beyond, the swaps run on x
// directly), then x is gathered through it in registers.  Forward and back
// substitution in blocks of 32 rows: warp 0 solves the diagonal block
// column-oriented (x_k broadcast by shuffle, each later row subtracting its
// L or U entry times x_k), then all warps update the remaining rows (warp per
// row, a 32-wide dot product).
constexpr int SOLVE_THREADS = 512;    // fits beside other work on a busy SM
constexpr int SOLVE_PERM_MAX = 4 * 1024;    // 8 bytes of shared memory per row, 8 values per thread
constexpr int SOLVE_REG = SOLVE_PERM_MAX / SOLVE_THREADS;
template <typename S>
__device__ __forceinline__ void lu_solve_body(const S *a, long long n, long long ld, const int *ipiv, double2 *x) {
  extern __shared__ int perm_smem[];
  __shared__ double2 xs[32];
  if (n <= SOLVE_PERM_MAX) {
    int *idx = perm_smem, *pv = perm_smem + n;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) { idx[i] = (int)i; pv[i] = ipiv[i] - 1; }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int i = 0; i < (int)n; ++i) {
        const int q = pv[i];
        if (q != i) { const int t = idx[q]; idx[q] = idx[i]; idx[i] = t; }
      }
    __syncthreads();
    double2 v[SOLVE_REG];
#pragma unroll
    for (int r = 0; r < SOLVE_REG; ++r) {
      const long long i = threadIdx.x + (long long)r * SOLVE_THREADS;
      if (i < n) v[r] = x[idx[i]];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SOLVE_REG; ++r) {
      const long long i = threadIdx.x + (long long)r * SOLVE_THREADS;
      if (i < n) x[i] = v[r];
    }
  } else if (threadIdx.x == 0) {
    for (long long i = 0; i < n; ++i) {
      const long long pi = ipiv[i] - 1;
      if (pi != i) { const double2 t = x[pi]; x[pi] = x[i]; x[i] = t; }
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // Forward: L unit lower.
  for (long long j0 = 0; j0 < n; j0 += 32) {
    const int w = (int)(n - j0 < 32 ? n - j0 : 32);
    if (warp == 0) {
      double2 v = lane < w ? x[j0 + lane] : make_double2(0, 0);
      for (int k = 0; k < w - 1; ++k) {
        const double2 l = (lane > k && lane < w) ? to_d(a[(j0 + lane) * ld + j0 + k]) : make_double2(0, 0);
        const double2 xk = make_double2(__shfl_sync(0xffffffffu, v.x, k), __shfl_sync(0xffffffffu, v.y, k));
        if (lane > k && lane < w) v = csub(v, cmul(l, xk));
      }
      if (lane < w) { x[j0 + lane] = v; xs[lane] = v; }
    }
    __syncthreads();
    for (long long r = j0 + w + warp; r < n; r += nw) {
      double2 s = lane < w ? cmul(to_d(a[r * ld + j0 + lane]), xs[lane]) : make_double2(0, 0);
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
      for (int k = w - 1; k >= 0; --k) {
        if (lane == k) v = cdiv(v, to_d(a[(j0 + k) * ld + j0 + k]));
        const double2 u = lane < k ? to_d(a[(j0 + lane) * ld + j0 + k]) : make_double2(0, 0);
        const double2 xk = make_double2(__shfl_sync(0xffffffffu, v.x, k), __shfl_sync(0xffffffffu, v.y, k));
        if (lane < k) v = csub(v, cmul(u, xk));
      }
      if (lane < w) { x[j0 + lane] = v; xs[lane] = v; }
    }
    __syncthreads();
    for (long long r = warp; r < j0; r += nw) {
      double2 s = lane < w ? cmul(to_d(a[r * ld + j0 + lane]), xs[lane]) : make_double2(0, 0);
      for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      }
      if (lane == 0) x[r] = csub(x[r], s);
    }
    __syncthreads();
  }
}

template <typename S>
__global__ void __launch_bounds__(SOLVE_THREADS, 2) lu_solve_kernel(const S *a, long long n, long long ld,
                                                                 const int *ipiv, double2 *b, long long ldb) {
  lu_solve_body<S>(a, n, ld, ipiv, b + blockIdx.x * ldb);
}

// ------------------------------------------------ multi-CTA triangular solve
// The same solve spread over SOLVE_CTAS co-resident CTAs (cooperative
// launch), for orders where one CTA's row updates dominate.  Blocks of
// SOLVE_NB = 64 rows.  In each block step CTA 0 solves the diagonal block by
// warp shuffles (two 32-row halves), then every CTA subtracts the block's
// contribution from its share of the rows below (above, backward), a warp
// per row.  CTA 0 itself updates the next block's rows, so the next diagonal
// solve needs no further barrier: one grid barrier per block.  While the
// grid waits at that barrier CTA 0 already holds the next diagonal block and
// the block of the next rows' update in shared memory (loaded before it
// arrives).  The barrier spins are bounded; on time-out the kernel raises
// *error and every CTA leaves at its next barrier.
constexpr int SOLVE_NB = 64;
constexpr int SOLVE_LDS = SOLVE_NB + 1;                  // padded shared row
constexpr int SOLVE_CTAS = 32;
constexpr int SOLVE_COOP_THREADS = 512;
constexpr int SOLVE_COOP_MIN = 256;     // smaller orders keep the one-CTA kernel
constexpr int SOLVE_COOP_RHS = 4;       // right-hand sides solved in turn by one launch
// Shared memory: diagonal block, next rows' block, solved values, inverse
// diagonal (backward sweep).
constexpr size_t SOLVE_COOP_SMEM = (size_t)(2 * SOLVE_NB * SOLVE_LDS + 2 * SOLVE_NB) * sizeof(double2);
// Orders whose interchanges compose in that shared memory (two ints per row).
constexpr int SOLVE_COOP_PERM_MAX = (int)(SOLVE_COOP_SMEM / 8);

struct SolveSync {
  unsigned count, gen;
  int error;
};

__device__ __forceinline__ bool solve_barrier(SolveSync *sy) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned *gen = &sy->gen;
    volatile int *err = &sy->error;
    if (*err) ok = 0;
    else {
      const unsigned g = *gen;
      __threadfence();
      if (atomicAdd(&sy->count, 1u) == gridDim.x - 1) {
        sy->count = 0;
        __threadfence();
        atomicAdd(&sy->gen, 1u);
      } else {
        const long long t0 = clock64();
        while (*gen == g) {
          if (*err || clock64() - t0 > (1LL << 32)) { atomicExch(&sy->error, 1); ok = 0; break; }
          __nanosleep(32);
        }
      }
      __threadfence();
    }
  }
  __syncthreads();
  return ok != 0;
}

// y[r] -= sum_c A[r][c0 + c] xs[c] for rows r of [r0, r1) taken warp by warp
// from `first` with stride `step` (warp indices); four rows per round, their
// loads issued together.
template <typename S>
__device__ __forceinline__ void solve_rows(const S *a, long long ld, double2 *y, long long r0, long long r1,
                                           long long c0, int w, const double2 *xs, long long first, long long step) {
  const int lane = threadIdx.x & 31;
  const double2 x0 = lane < w ? xs[lane] : make_double2(0, 0);
  const double2 x1 = lane + 32 < w ? xs[lane + 32] : make_double2(0, 0);
  for (long long r = r0 + first; r < r1; r += 4 * step) {
    double2 s[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const long long rr = r + u * step;
      s[u] = make_double2(0, 0);
      if (rr < r1) {
        const S *row = a + rr * ld + c0;
        if (lane < w) s[u] = cmul(to_d(row[lane]), x0);
        if (lane + 32 < w) s[u] = cadd(s[u], cmul(to_d(row[lane + 32]), x1));
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      for (int o = 16; o > 0; o >>= 1) {
        s[u].x += __shfl_xor_sync(0xffffffffu, s[u].x, o);
        s[u].y += __shfl_xor_sync(0xffffffffu, s[u].y, o);
      }
      const long long rr = r + u * step;
      if (lane == 0 && rr < r1) y[rr] = csub(y[rr], s[u]);
    }
  }
}

// Loads the rows x cols block of A at (r0, c0) into shared memory (leading
// dim SOLVE_LDS), zero elsewhere in the SOLVE_NB square; each thread issues
// all its loads before it stores (blockDim.x must divide SOLVE_NB^2).
constexpr int SOLVE_PER_THREAD = SOLVE_NB * SOLVE_NB / SOLVE_COOP_THREADS;
template <typename S>
__device__ __forceinline__ void solve_load_block(const S *a, long long ld, long long r0, long long c0, int rows,
                                                 int cols, double2 *dst) {
  double2 v[SOLVE_PER_THREAD];
#pragma unroll
  for (int u = 0; u < SOLVE_PER_THREAD; ++u) {
    const int e = threadIdx.x + u * SOLVE_COOP_THREADS, r = e >> 6, c = e & (SOLVE_NB - 1);
    v[u] = (r < rows && c < cols) ? to_d(a[(r0 + r) * ld + c0 + c]) : make_double2(0, 0);
  }
#pragma unroll
  for (int u = 0; u < SOLVE_PER_THREAD; ++u) {
    const int e = threadIdx.x + u * SOLVE_COOP_THREADS, r = e >> 6, c = e & (SOLVE_NB - 1);
    dst[r * SOLVE_LDS + c] = v[u];
  }
}

__device__ __forceinline__ double2 shfl2(double2 v, int src) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// Warp 0: forward solve of the unit-lower w x w diagonal block dg in place
// on xs (two halves of 32: solve, update the second half, solve).
__device__ __forceinline__ void solve_diag_lower(const double2 *dg, double2 *xs, int w) {
  const int lane = threadIdx.x & 31;
  double2 v0 = lane < w ? xs[lane] : make_double2(0, 0);
  double2 v1 = lane + 32 < w ? xs[lane + 32] : make_double2(0, 0);
  const int w0 = w < 32 ? w : 32;
  for (int c = 0; c < w0 - 1; ++c) {
    const double2 xc = shfl2(v0, c);
    if (lane > c) v0 = csub(v0, cmul(dg[lane * SOLVE_LDS + c], xc));
  }
  if (w > 32) {
    for (int c = 0; c < 32; ++c) v1 = csub(v1, cmul(dg[(lane + 32) * SOLVE_LDS + c], shfl2(v0, c)));
    for (int c = 0; c < w - 33; ++c) {
      const double2 xc = shfl2(v1, c);
      if (lane > c) v1 = csub(v1, cmul(dg[(lane + 32) * SOLVE_LDS + 32 + c], xc));
    }
  }
  if (lane < w) xs[lane] = v0;
  if (lane + 32 < w) xs[lane + 32] = v1;
}

// 1 / U_cc of the diagonal block's rows (threads 0..w-1), so that the
// sequential back substitution multiplies instead of dividing.
__device__ __forceinline__ void solve_diag_inverse(const double2 *dg, double2 *dinv, int w) {
  const int c = threadIdx.x;
  if (c < w) {
    const double2 u = dg[c * SOLVE_LDS + c];
    const double r = 1.0 / (u.x * u.x + u.y * u.y);
    dinv[c] = make_double2(u.x * r, -u.y * r);
  }
}

// Warp 0: backward solve of the upper w x w diagonal block dg in place on xs
// (dinv: the inverse diagonal).
__device__ __forceinline__ void solve_diag_upper(const double2 *dg, const double2 *dinv, double2 *xs, int w) {
  const int lane = threadIdx.x & 31;
  double2 v0 = lane < w ? xs[lane] : make_double2(0, 0);
  double2 v1 = lane + 32 < w ? xs[lane + 32] : make_double2(0, 0);
  if (w > 32) {
    for (int c = w - 33; c >= 0; --c) {
      if (lane == c) v1 = cmul(v1, dinv[c + 32]);
      const double2 xc = shfl2(v1, c);
      if (lane < c) v1 = csub(v1, cmul(dg[(lane + 32) * SOLVE_LDS + c + 32], xc));
    }
    for (int c = 0; c < w - 32; ++c) v0 = csub(v0, cmul(dg[lane * SOLVE_LDS + 32 + c], shfl2(v1, c)));
  }
  const int w0 = w < 32 ? w : 32;
  for (int c = w0 - 1; c >= 0; --c) {
    if (lane == c) v0 = cmul(v0, dinv[c]);
    const double2 xc = shfl2(v0, c);
    if (lane < c) v0 = csub(v0, cmul(dg[lane * SOLVE_LDS + c], xc));
  }
  if (lane < w) xs[lane] = v0;
  if (lane + 32 < w) xs[lane + 32] = v1;
}

// CTA 0's update of the next block's rows from the shared block nb (rows x
// w): y[r0 + r] -= sum_c nb[r][c] xs[c], a warp per row.
__device__ __forceinline__ void solve_next_rows(const double2 *nb, const double2 *xs, double2 *y, long long r0,
                                                int rows, int w) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int r = warp; r < rows; r += 4 * nw) {
    double2 s[4], yv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int rr = r + u * nw;
      s[u] = make_double2(0, 0);
      yv[u] = (lane == 0 && rr < rows) ? y[r0 + rr] : make_double2(0, 0);
      if (rr < rows)
        for (int c = lane; c < w; c += 32) s[u] = cadd(s[u], cmul(nb[rr * SOLVE_LDS + c], xs[c]));
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      for (int o = 16; o > 0; o >>= 1) {
        s[u].x += __shfl_xor_sync(0xffffffffu, s[u].x, o);
        s[u].y += __shfl_xor_sync(0xffffffffu, s[u].y, o);
      }
      const int rr = r + u * nw;
      if (lane == 0 && rr < rows) y[r0 + rr] = csub(yv[u], s[u]);
    }
  }
}

template <typename S>
__device__ __forceinline__ void lu_solve_coop_body(const S *a, long long n, long long ld, const int *ipiv, double2 *b,
                                                   long long ldb, int nrhs, double2 *scratch, SolveSync *sy) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *dg = reinterpret_cast<double2 *>(smem_raw);   // diagonal block
  double2 *nb = dg + SOLVE_NB * SOLVE_LDS;                // next rows' block
  double2 *xs = nb + SOLVE_NB * SOLVE_LDS;                // solved block values
  double2 *dinv = xs + SOLVE_NB;                          // inverse diagonal (backward)
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // Row updates of the other CTAs: warps of CTAs 1.. (CTA 0 takes the next block).
  const long long ow = (long long)(blockIdx.x - 1) * nw + warp, onw = (long long)(gridDim.x - 1) * nw;
  const long long nblk = (n + SOLVE_NB - 1) / SOLVE_NB;
  for (int rhs = 0; rhs < nrhs; ++rhs) {
    double2 *x = b + rhs * ldb;
    // Interchanges, applied in pivot order by CTA 0 into the scratch vector:
    // composed into an index permutation in shared memory (orders up to
    // SOLVE_COOP_PERM_MAX), then gathered; beyond, swapped in place.
    if (blockIdx.x == 0) {
      if (n <= SOLVE_COOP_PERM_MAX) {
        int *idx = reinterpret_cast<int *>(smem_raw), *pv = idx + n;
        for (long long i = threadIdx.x; i < n; i += blockDim.x) { idx[i] = (int)i; pv[i] = ipiv[i] - 1; }
        __syncthreads();
        if (threadIdx.x == 0)
          for (int i = 0; i < (int)n; ++i) {
            const int q = pv[i];
            if (q != i) { const int t = idx[q]; idx[q] = idx[i]; idx[i] = t; }
          }
        __syncthreads();
        for (long long i = threadIdx.x; i < n; i += blockDim.x) scratch[i] = x[idx[i]];
        __syncthreads();
      } else {
        for (long long i = threadIdx.x; i < n; i += blockDim.x) scratch[i] = x[i];
        __syncthreads();
        if (threadIdx.x == 0)
          for (long long i = 0; i < n; ++i) {
            const long long q = ipiv[i] - 1;
            if (q != i) { const double2 t = scratch[q]; scratch[q] = scratch[i]; scratch[i] = t; }
          }
        __syncthreads();
      }
      solve_load_block(a, ld, 0, 0, (int)(n < SOLVE_NB ? n : SOLVE_NB), (int)(n < SOLVE_NB ? n : SOLVE_NB), dg);
    }
    if (!solve_barrier(sy)) return;
    double2 *y = scratch;
    // Forward: L unit lower.  dg holds block k's diagonal on entry.
    for (long long k = 0; k < nblk; ++k) {
      const long long j0 = k * SOLVE_NB;
      const int w = (int)(n - j0 < SOLVE_NB ? n - j0 : SOLVE_NB);
      const long long r1 = j0 + w + SOLVE_NB < n ? j0 + w + SOLVE_NB : n;   // end of the next block
      if (blockIdx.x == 0) {
        for (int r = threadIdx.x; r < w; r += blockDim.x) xs[r] = y[j0 + r];
        __syncthreads();
        if (warp == 0) solve_diag_lower(dg, xs, w);
        __syncthreads();
        for (int r = threadIdx.x; r < w; r += blockDim.x) y[j0 + r] = xs[r];
        // The next rows' block of L and the next diagonal block while the
        // grid gathers.
        if (k + 1 < nblk) {
          const int wn = (int)(r1 - j0 - w);
          solve_load_block(a, ld, j0 + w, j0, wn, w, nb);
          solve_load_block(a, ld, j0 + w, j0 + w, wn, wn, dg);
        }
      }
      if (!solve_barrier(sy)) return;
      if (k + 1 == nblk) break;
      if (blockIdx.x != 0) {
        for (int r = threadIdx.x; r < w; r += blockDim.x) xs[r] = y[j0 + r];
        __syncthreads();
        solve_rows(a, ld, y, r1, n, j0, w, xs, ow, onw);
      } else {
        solve_next_rows(nb, xs, y, j0 + w, (int)(r1 - j0 - w), w);
        __syncthreads();
      }
    }
    // Backward: U upper, non-unit diagonal.
    if (blockIdx.x == 0) {
      const long long j0 = (nblk - 1) * SOLVE_NB;
      const int w = (int)(n - j0);
      solve_load_block(a, ld, j0, j0, w, w, dg);
      __syncthreads();
      solve_diag_inverse(dg, dinv, w);
    }
    if (!solve_barrier(sy)) return;
    for (long long k = nblk - 1; k >= 0; --k) {
      const long long j0 = k * SOLVE_NB;
      const int w = (int)(n - j0 < SOLVE_NB ? n - j0 : SOLVE_NB);
      const long long p0 = j0 - SOLVE_NB > 0 ? j0 - SOLVE_NB : 0;   // rows of the next block up
      if (blockIdx.x == 0) {
        for (int r = threadIdx.x; r < w; r += blockDim.x) xs[r] = y[j0 + r];
        __syncthreads();
        if (warp == 0) solve_diag_upper(dg, dinv, xs, w);
        __syncthreads();
        for (int r = threadIdx.x; r < w; r += blockDim.x) y[j0 + r] = xs[r];
        if (k > 0) {
          solve_load_block(a, ld, p0, j0, (int)(j0 - p0), w, nb);
          solve_load_block(a, ld, p0, p0, (int)(j0 - p0), (int)(j0 - p0), dg);
          __syncthreads();
          solve_diag_inverse(dg, dinv, (int)(j0 - p0));
        }
      }
      if (!solve_barrier(sy)) return;
      if (k == 0) break;
      if (blockIdx.x != 0) {
        for (int r = threadIdx.x; r < w; r += blockDim.x) xs[r] = y[j0 + r];
        __syncthreads();
        solve_rows(a, ld, y, 0, p0, j0, w, xs, ow, onw);
      } else {
        solve_next_rows(nb, xs, y, p0, (int)(j0 - p0), w);
        __syncthreads();
      }
    }
    if (!solve_barrier(sy)) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      x[i] = y[i];
    if (!solve_barrier(sy)) return;
  }
}
template <typename S>
__global__ void __launch_bounds__(SOLVE_COOP_THREADS) lu_solve_coop_kernel(const S *a, long long n, long long ld,
                                                                         const int *ipiv, double2 *b, long long ldb,
                                                                         int nrhs, double2 *scratch,
                                                                         SolveSync *sy) {
  lu_solve_coop_body<S>(a, n, ld, ipiv, b, ldb, nrhs, scratch, sy);
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

// Panel launch: the smallest cluster of 256-thread CTAs that holds the
// panel's rows (16-CTA clusters where the device allows that non-portable
// size), else the cooperative grid panel.
template <int CSZ, typename S>
static cudaError_t launch_cluster_panel(const PanelArgs &p, cudaStream_t s) {
  void (*kernel)(PanelArgs) = p.rule == 0 ? panel_cluster_kernel<CSZ, 0, S> : panel_cluster_kernel<CSZ, 1, S>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CSZ);
  cfg.blockDim = dim3(CPT);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CSZ;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, p);
}

// 1 when 16-CTA clusters of the panel kernel can be resident.
// NEC2C_CUDA_LU_CLUSTER8=1 in the environment (a test switch) limits the
// panel to 8-CTA clusters, so orders above 2048 take the grid panel.
static int cluster16_probe() {
  int state = 0;
  const char *cap = getenv("NEC2C_CUDA_LU_CLUSTER8");
  if (cap && cap[0] == '1') return 0;
  void (*kernels[4])(PanelArgs) = {panel_cluster_kernel<CMAX, 0, double2>, panel_cluster_kernel<CMAX, 1, double2>,
                                   panel_cluster_kernel<CMAX, 0, float2>, panel_cluster_kernel<CMAX, 1, float2>};
  for (auto k : kernels) {
    if (cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
      cudaGetLastError();
      return state;
    }
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CMAX);
  cfg.blockDim = dim3(CPT);
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CMAX;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, panel_cluster_kernel<CMAX, 0, double2>, &cfg) == cudaSuccess && clusters > 0)
    state = 1;
  cudaGetLastError();
  return state;
}

// Probed once per process; the static's initialisation is thread-safe, so
// server workers that factor concurrently all see the probe's result.
static int cluster16_ok() {
  static const int state = cluster16_probe();
  return state;
}

// Largest panel row count the cluster kernel takes on this device.
static long long cluster_rows() { return (long long)CROWS * (cluster16_ok() ? CMAX : 8); }

template <typename S>
static int launch_panel(const PanelArgs &p, long long rows, cudaStream_t s) {
  cudaError_t e;
  if (rows <= cluster_rows()) {
    if (rows <= CROWS) e = launch_cluster_panel<1, S>(p, s);
    else if (rows <= 2 * CROWS) e = launch_cluster_panel<2, S>(p, s);
    else if (rows <= 4 * CROWS) e = launch_cluster_panel<4, S>(p, s);
    else if (rows <= 8 * CROWS) e = launch_cluster_panel<8, S>(p, s);
    else e = launch_cluster_panel<CMAX, S>(p, s);
  } else {
    const int blocks = (int)((rows + PT - 1) / PT);
    void *args[] = {const_cast<PanelArgs *>(&p)};
    e = cudaLaunchCooperativeKernel((void *)panel_grid_kernel<S>, blocks, PT, args, 0, s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    n2c_set_error("panel launch: %s", cudaGetErrorString(e));
    return 0;
  }
  n2c_count_launch(1);
  return 1;
}

// Scratch of one factorisation: status, interchange pairs and, for the grid
// panel, its candidate arrays.
struct FactorScratch {
  LuStatus *st;
  int *pairs;
  float *bt_hi, *bt_lo;       // split-precision form: packed U12 expansion (2n x 64 floats each)
  double *gval;
  int *gidx;
  double2 *grow, *growj;
};

static int grid_blocks_for(long long n) { return (int)((n + PT - 1) / PT); }

// Side stream of this thread (per device) for the look-ahead panel, created
// with the highest priority so its CTAs are dispatched ahead of the trailing
// update's as SMs free up.
struct LookAhead {
  int dev = -1;
  cudaStream_t aux = nullptr;
  cudaEvent_t next = nullptr, panel = nullptr;
  // Released when the owning thread exits.
  ~LookAhead() {
    if (aux) cudaStreamDestroy(aux);
    if (next) cudaEventDestroy(next);
    if (panel) cudaEventDestroy(panel);
    cudaGetLastError();
  }
};
static thread_local LookAhead g_look;

static LookAhead *look_ahead() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return nullptr; }
  LookAhead &l = g_look;
  if (l.dev == dev && l.aux) return &l;
  if (l.aux) {
    cudaStreamDestroy(l.aux);
    cudaEventDestroy(l.next);
    cudaEventDestroy(l.panel);
    l = LookAhead();
  }
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  if (cudaStreamCreateWithPriority(&l.aux, cudaStreamNonBlocking, hi) != cudaSuccess ||
      cudaEventCreateWithFlags(&l.next, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&l.panel, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    n2c_set_error("look-ahead stream set-up failed");
    return nullptr;
  }
  l.dev = dev;
  return &l;
}

// Trailing update of columns [c_first, c_first + cols) for rows below the
// panel: FP64 tiles on the FP64 pipe, or the split-precision form on the
// tensor cores (U12 from the packed expansion).
static int launch_gemm(double2 *a, long long ld, long long k0, int kb, long long c_first, long long cols,
                       long long rows, const FactorScratch &, cudaStream_t s) {
  if (cols <= 0 || rows <= 0) return 1;
  dim3 grid((unsigned)((cols + GT - 1) / GT), (unsigned)((rows + GT - 1) / GT));
  static const bool configured = cudaFuncSetAttribute(gemm_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)GEMM_SMEM) == cudaSuccess;
  if (!configured) {
    cudaGetLastError();
    n2c_set_error("gemm_update: shared memory configuration failed");
    return 0;
  }
  gemm_update_kernel<<<grid, 256, GEMM_SMEM, s>>>(a + (k0 + kb) * ld + c_first, a + (k0 + kb) * ld + k0,
                                          a + k0 * ld + c_first, rows, cols, kb, ld);
  return n2c_check_launch("gemm_update");
}
static int launch_gemm(float2 *a, long long ld, long long k0, int kb, long long c_first, long long cols,
                       long long rows, const FactorScratch &w, cudaStream_t s) {
  if (cols <= 0 || rows <= 0) return 1;
  const long long r2 = 2 * (c_first - k0 - kb);
  return n2c_tc_update((float *)(a + (k0 + kb) * ld + c_first), ld, (const float *)(a + (k0 + kb) * ld + k0), ld,
                       w.bt_hi + r2 * (2 * KB), w.bt_lo + r2 * (2 * KB), rows, cols, &w.st->error, s,
                       n2c_tc_form(rows, cols));
}

// The blocked factorisation; the status must be zero on entry.  Reads the
// status back (synchronising the stream) and sets *info_host.  With look-ahead
// the trailing update of each panel is split: the next panel's columns are
// updated first, then that panel is factored on the side stream while the
// rest of the update runs on the caller's stream (the two touch disjoint
// columns); the next interchange waits for both.
template <typename S>
static int factor_panels(S *a, long long n, long long ld, int *ipiv, int rule, const FactorScratch &w, bool lookahead,
                         int *info_host) {
  cudaStream_t s = n2c_stream();
  LookAhead *la = lookahead && n > KB ? look_ahead() : nullptr;
  if (lookahead && n > KB && !la) return 0;
  auto panel_args = [&](long long k0) {
    PanelArgs p;
    memset(&p, 0, sizeof(p));
    p.a = a; p.n = n; p.ld = ld; p.k0 = k0; p.kb = (int)(n - k0 < KB ? n - k0 : KB); p.rule = rule; p.ipiv = ipiv;
    p.pairs = w.pairs; p.st = w.st; p.gval = w.gval; p.gidx = w.gidx; p.grow = w.grow; p.growj = w.growj;
    return p;
  };
  int ok = launch_panel<S>(panel_args(0), n, s);
  for (long long k0 = 0; ok && k0 < n; k0 += KB) {
    const int kb = (int)(n - k0 < KB ? n - k0 : KB);
    if (n > kb) {
      const unsigned gb = (unsigned)((n - kb + SWT / 32 - 1) / (SWT / 32));
      swap_trsm_kernel<S><<<gb, SWT, 0, s>>>(a, n, ld, k0, kb, w.pairs, w.st, w.bt_hi, w.bt_lo);
      if (!n2c_check_launch("interchanges and triangular solve")) { ok = 0; break; }
    }
    const long long right = n - k0 - kb;
    if (right <= 0) break;
    const long long c1 = k0 + kb;
    // Cooperative grid panels (orders beyond the cluster's rows) need the
    // whole device co-resident: those run in order on the caller's stream.
    if (!la || right > cluster_rows()) {
      if (!launch_gemm(a, ld, k0, kb, c1, right, right, w, s) || !launch_panel<S>(panel_args(c1), right, s)) ok = 0;
      continue;
    }
    const long long nb = right < KB ? right : KB;
    ok = launch_gemm(a, ld, k0, kb, c1, nb, right, w, s);
    if (ok && (cudaEventRecord(la->next, s) != cudaSuccess || cudaStreamWaitEvent(la->aux, la->next, 0) != cudaSuccess)) {
      n2c_set_error("look-ahead event");
      ok = 0;
    }
    ok = ok && launch_panel<S>(panel_args(c1), right, la->aux);
    if (ok && cudaEventRecord(la->panel, la->aux) != cudaSuccess) { n2c_set_error("look-ahead event"); ok = 0; }
    ok = ok && launch_gemm(a, ld, k0, kb, c1 + nb, right - nb, right, w, s);
    if (ok && cudaStreamWaitEvent(s, la->panel, 0) != cudaSuccess) { n2c_set_error("look-ahead event"); ok = 0; }
  }
  if (la && !ok) cudaStreamSynchronize(la->aux);
  LuStatus hs;
  memset(&hs, 0, sizeof(hs));
  cudaError_t e = cudaMemcpyAsync(&hs, w.st, sizeof(hs), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (ok && e != cudaSuccess) { n2c_set_error("reading the panel status: %s", cudaGetErrorString(e)); ok = 0; }
  if (ok && hs.error) { n2c_set_error("LU kernel wait time-out"); ok = 0; }
  *info_host = hs.info;
  return ok;
}

// Scratch allocation around factor_panels (stream-ordered, so factorisations
// on several streams do not synchronise each other); the split-precision form
// also holds the packed U12 expansion.
template <typename S>
static int factor_alloc(S *a, long long n, long long ld, int *ipiv, int rule, int *info_host) {
  *info_host = 0;
  if (n <= 0) return 1;
  const bool split = sizeof(S) == sizeof(float2);
  FactorScratch w;
  memset(&w, 0, sizeof(w));
  w.st = (LuStatus *)n2d_alloc_async(sizeof(LuStatus));
  w.pairs = (int *)n2d_alloc_async(4 * KB * sizeof(int));
  const bool grid = n > cluster_rows();
  const int gb = grid_blocks_for(n);
  if (grid) {
    w.gval = (double *)n2d_alloc_async(2 * gb * sizeof(double));
    w.gidx = (int *)n2d_alloc_async(2 * gb * sizeof(int));
    w.grow = (double2 *)n2d_alloc_async((size_t)2 * gb * KB * sizeof(double2));
    w.growj = (double2 *)n2d_alloc_async(2 * KB * sizeof(double2));
  }
  if (split) {
    w.bt_hi = (float *)n2d_alloc_async((size_t)2 * n * 2 * KB * sizeof(float));
    w.bt_lo = (float *)n2d_alloc_async((size_t)2 * n * 2 * KB * sizeof(float));
  }
  int ok = w.st && w.pairs && n2d_memset(w.st, 0, sizeof(LuStatus)) &&
           (!grid || (w.gval && w.gidx && w.grow && w.growj)) && (!split || (w.bt_hi && w.bt_lo));
  ok = ok && factor_panels(a, n, ld, ipiv, rule, w, true, info_host);
  n2d_free_async(w.st); n2d_free_async(w.pairs);
  n2d_free_async(w.gval); n2d_free_async(w.gidx); n2d_free_async(w.grow); n2d_free_async(w.growj);
  n2d_free_async(w.bt_hi); n2d_free_async(w.bt_lo);
  return ok;
}

extern "C" int n2d_lu_factor(double *a_dev, long long n, long long ld, int *ipiv, int rule, int precision,
                             int *info_host) {
  (void)precision;
  return factor_alloc((double2 *)a_dev, n, ld, ipiv, rule, info_host);
}

extern "C" int n2d_lu_factor32(float *a_dev, long long n, long long ld, int *ipiv, int rule, int *info_host) {
  if (ld & 1) {
    n2c_set_error("split-precision LU needs an even leading dimension");
    return 0;
  }
  return factor_alloc((float2 *)a_dev, n, ld, ipiv, rule, info_host);
}

static size_t solve_smem(long long n) { return n <= SOLVE_PERM_MAX ? (size_t)8 * n : 0; }
template <typename S>
static int solve_configure() {
  static const bool done = cudaFuncSetAttribute(lu_solve_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                8 * SOLVE_PERM_MAX) == cudaSuccess;
  if (!done) {
    n2c_set_error("triangular solve: shared memory configuration failed");
    return 0;
  }
  return 1;
}

// CTAs of the cooperative solve on this device (0: it cannot run).
template <typename S>
static int solve_coop_blocks() {
  int per_sm = 0;
  if (cudaFuncSetAttribute(lu_solve_coop_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SOLVE_COOP_SMEM) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lu_solve_coop_kernel<S>, SOLVE_COOP_THREADS,
                                                    SOLVE_COOP_SMEM) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    return 0;
  }
  return n2c_sm_count() < SOLVE_CTAS ? n2c_sm_count() : SOLVE_CTAS;
}

// Cooperative multi-CTA solve (orders >= SOLVE_COOP_MIN, up to
// SOLVE_COOP_RHS right-hand sides); 0 with the error set on failure, -1 when
// the one-CTA kernel should be used instead.
template <typename S>
static int solve_coop(const S *a, long long n, long long ld, const int *ipiv, double2 *b, long long ldb,
                      long long nrhs) {
  if (n < SOLVE_COOP_MIN || nrhs > SOLVE_COOP_RHS || n > 0x7fffffffLL) return -1;
  static const int blocks = solve_coop_blocks<S>();
  const size_t smem = SOLVE_COOP_SMEM;
  if (blocks < 2) return -1;   // the rows below the next block need a second CTA
  double2 *scratch = (double2 *)n2d_alloc_async((size_t)n * sizeof(double2));
  SolveSync *sy = (SolveSync *)n2d_alloc_async(sizeof(SolveSync) + 16);
  int ok = scratch && sy && cudaMemsetAsync(sy, 0, sizeof(SolveSync), n2c_stream()) == cudaSuccess;
  if (ok) {
    int nr = (int)nrhs;
    void *args[] = {(void *)&a, (void *)&n, (void *)&ld, (void *)&ipiv, (void *)&b, (void *)&ldb, (void *)&nr,
                    (void *)&scratch, (void *)&sy};
    const cudaError_t e = cudaLaunchCooperativeKernel((void *)lu_solve_coop_kernel<S>, blocks, SOLVE_COOP_THREADS,
                                                      args, smem, n2c_stream());
    if (e != cudaSuccess) {
      // Not launchable as a cooperative grid here: the one-CTA kernel solves it.
      cudaGetLastError();
      n2d_free_async(scratch);
      n2d_free_async(sy);
      return -1;
    }
    n2c_count_launch(1);
  }
  int err = 0;
  if (ok && (cudaMemcpyAsync(&err, &sy->error, sizeof(int), cudaMemcpyDeviceToHost, n2c_stream()) != cudaSuccess ||
             cudaStreamSynchronize(n2c_stream()) != cudaSuccess))
    ok = 0;
  if (ok && err) { n2c_set_error("triangular solve: grid barrier time-out"); ok = 0; }
  n2d_free_async(scratch);
  n2d_free_async(sy);
  return ok;
}

extern "C" int n2d_lu_solve(const double *a_dev, long long n, long long ld, const int *ipiv, double *b_dev,
                            long long ldb, long long nrhs) {
  if (n <= 0 || nrhs <= 0) return 1;
  const int c = solve_coop((const double2 *)a_dev, n, ld, ipiv, (double2 *)b_dev, ldb, nrhs);
  if (c >= 0) return c;
  if (!solve_configure<double2>()) return 0;
  lu_solve_kernel<double2><<<(unsigned)nrhs, SOLVE_THREADS, solve_smem(n), n2c_stream()>>>((const double2 *)a_dev, n, ld, ipiv,
                                                             (double2 *)b_dev, ldb);
  return n2c_check_launch("lu_solve");
}

// Solve with FP32 factors (split-precision form); the arithmetic and the
// right-hand sides are FP64.
extern "C" int n2d_lu_solve32(const float *a_dev, long long n, long long ld, const int *ipiv, double *b_dev,
                              long long ldb, long long nrhs) {
  if (n <= 0 || nrhs <= 0) return 1;
  const int c = solve_coop((const float2 *)a_dev, n, ld, ipiv, (double2 *)b_dev, ldb, nrhs);
  if (c >= 0) return c;
  if (!solve_configure<float2>()) return 0;
  lu_solve_kernel<float2><<<(unsigned)nrhs, SOLVE_THREADS, solve_smem(n), n2c_stream()>>>((const float2 *)a_dev, n, ld, ipiv,
                                                                     (double2 *)b_dev, ldb);
  return n2c_check_launch("lu_solve");
}

// ------------------------------------------------ ragged batch of factors
// Many independent FP64 factorisations (orders up to the cluster panel's
// rows) advanced in lockstep: each panel step is one launch of each kernel
// for the whole batch (one cluster per matrix for the panel; the matrix index
// in grid.y or grid.z for the interchanges, the triangular solve and the
// update), so the latency of the pivot chain is paid once per step for every
// matrix and the updates of all of them fill the device together.  A matrix
// whose order has been passed takes no further part (its blocks return at
// once).  The kernel bodies are the single factorisation's, so each matrix
// gets exactly the pivots and factors n2d_lu_factor gives it alone.
namespace {

struct LuBatchEntry {
  void *a;         // double2 (FP64 form) or float2 (split-precision form)
  long long n, ld;
  int *ipiv;
  int *pairs;      // 4 KB ints of this matrix's interchange pairs
  LuStatus *st;
  float *bt_hi, *bt_lo;   // split-precision form: packed U12 expansion (2n x 64 floats each)
};

__device__ __forceinline__ int batch_kb(long long n, long long k0) { return (int)(n - k0 < KB ? n - k0 : KB); }

template <int CSZ, int RULE, typename S>
__global__ void __launch_bounds__(CPT, 1) panel_cluster_batch_kernel(const LuBatchEntry *e, long long k0) {
  const LuBatchEntry m = e[blockIdx.y];   // clusters run along x: one matrix per cluster
  if (m.n <= k0) return;
  PanelArgs p{};
  p.a = m.a; p.n = m.n; p.ld = m.ld; p.k0 = k0; p.kb = batch_kb(m.n, k0); p.rule = RULE;
  p.ipiv = m.ipiv; p.pairs = m.pairs; p.st = m.st;
  panel_cluster_body<CSZ, RULE, S>(p);
}

template <typename S>
__global__ void __launch_bounds__(SWT) swap_trsm_batch_kernel(const LuBatchEntry *e, long long k0) {
  const LuBatchEntry m = e[blockIdx.y];
  if (m.n <= k0) return;
  const int kb = batch_kb(m.n, k0);
  if ((long long)blockIdx.x * (SWT / 32) >= m.n - kb) return;   // no column of this matrix in the block
  swap_trsm_body<S>((S *)m.a, m.n, m.ld, k0, kb, m.pairs, m.st, m.bt_hi, m.bt_lo, blockIdx.x);
}

// part 0: the next panel's columns (look-ahead); part 1: the columns after it.
__global__ void __launch_bounds__(256, 2) gemm_update_batch_kernel(const LuBatchEntry *e, long long k0, int part) {
  const LuBatchEntry m = e[blockIdx.z];
  if (m.n <= k0) return;
  const int kb = batch_kb(m.n, k0);
  const long long right = m.n - k0 - kb;
  const long long nb = right < KB ? right : KB;
  const long long cf = k0 + kb + (part ? nb : 0);
  const long long cols = part ? right - nb : nb;
  const long long row0 = blockIdx.y * (long long)GT, col0 = blockIdx.x * (long long)GT;
  if (right <= 0 || cols <= 0 || row0 >= right || col0 >= cols) return;
  double2 *a = (double2 *)m.a, *below = a + (k0 + kb) * m.ld;
  gemm_update_body(below + cf, below + k0, a + k0 * m.ld + cf, right, cols, kb, m.ld, row0, col0);
}

struct SolveBatchEntry {
  const void *a;      // double2 or float2 factors
  long long n, ld;
  const int *ipiv;
  double2 *b;
  long long ldb;
  int nrhs;
  double2 *scratch;   // cooperative form: n values
  SolveSync *sy;      // cooperative form: this system's barrier
};

// One CTA per (right-hand side, system).
template <typename S>
__global__ void __launch_bounds__(SOLVE_THREADS, 2) lu_solve_batch_kernel(const SolveBatchEntry *e) {
  const SolveBatchEntry m = e[blockIdx.y];
  if ((int)blockIdx.x >= m.nrhs) return;
  lu_solve_body<S>((const S *)m.a, m.n, m.ld, m.ipiv, m.b + blockIdx.x * m.ldb);
}

// gridDim.x co-resident CTAs per system (grid.y = system), each group on its
// own barrier.
template <typename S>
__global__ void __launch_bounds__(SOLVE_COOP_THREADS) lu_solve_coop_batch_kernel(const SolveBatchEntry *e) {
  const SolveBatchEntry m = e[blockIdx.y];
  lu_solve_coop_body<S>((const S *)m.a, m.n, m.ld, m.ipiv, m.b, m.ldb, m.nrhs, m.scratch, m.sy);
}

template <int CSZ, typename S>
static cudaError_t launch_cluster_panel_batch(const LuBatchEntry *e, int count, long long k0, int rule,
                                              cudaStream_t s) {
  void (*kernel)(const LuBatchEntry *, long long) =
      rule == 0 ? panel_cluster_batch_kernel<CSZ, 0, S> : panel_cluster_batch_kernel<CSZ, 1, S>;
  if (CSZ > 8) {
    static const bool opted = cudaFuncSetAttribute(panel_cluster_batch_kernel<CSZ, 0, S>,
                                                   cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess &&
                              cudaFuncSetAttribute(panel_cluster_batch_kernel<CSZ, 1, S>,
                                                   cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
    if (!opted) return cudaErrorInvalidConfiguration;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CSZ, (unsigned)count);
  cfg.blockDim = dim3(CPT);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CSZ;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, e, k0);
}

// The batch's panels at step k0 (rows: the largest panel's row count).
template <typename S>
static int launch_panel_batch(const LuBatchEntry *e, int count, long long k0, long long rows, int rule,
                              cudaStream_t s) {
  cudaError_t err;
  if (rows <= CROWS) err = launch_cluster_panel_batch<1, S>(e, count, k0, rule, s);
  else if (rows <= 2 * CROWS) err = launch_cluster_panel_batch<2, S>(e, count, k0, rule, s);
  else if (rows <= 4 * CROWS) err = launch_cluster_panel_batch<4, S>(e, count, k0, rule, s);
  else if (rows <= 8 * CROWS) err = launch_cluster_panel_batch<8, S>(e, count, k0, rule, s);
  else err = launch_cluster_panel_batch<CMAX, S>(e, count, k0, rule, s);
  if (err != cudaSuccess) {
    cudaGetLastError();
    n2c_set_error("batched panel launch: %s", cudaGetErrorString(err));
    return 0;
  }
  n2c_count_launch(1);
  return 1;
}

}  // namespace

extern "C" long long n2d_lu_batch_max_order(void) { return cluster_rows(); }

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Lockstep factorisation of count matrices of storage S (FP64, or FP32 with
// the tensor-core update); see n2d_lu_factor_batch.
template <typename S>
static int factor_batch(void *const *a_dev, const long long *n, const long long *ld, int *const *ipiv, int count,
                        int rule, int *info) {
  if (count <= 0) return 1;
  constexpr bool split = sizeof(S) == sizeof(float2);
  const long long cap = cluster_rows();
  if (count > 65535) {
    n2c_set_error("batched factor: %d systems (at most 65535)", count);
    return 0;
  }
  long long nmax = 0;
  for (int i = 0; i < count; ++i) {
    info[i] = 0;
    if (!a_dev[i] || !ipiv[i] || n[i] <= 0 || n[i] > cap || ld[i] < n[i] ||
        (split && ((ld[i] & 1) || ((uintptr_t)a_dev[i] & 15)))) {
      n2c_set_error("batched factor: system %d has a null matrix or pivots, an order outside 1..%lld, or a "
                    "leading dimension below its order%s", i, cap,
                    split ? " (split form: even leading dimension, 16-byte aligned matrix)" : "");
      return 0;
    }
    if (n[i] > nmax) nmax = n[i];
  }
  cudaStream_t s = n2c_stream();
  LookAhead *la = nmax > KB ? look_ahead() : nullptr;
  if (nmax > KB && !la) return 0;
  const size_t eb = align256(count * sizeof(LuBatchEntry)), sb = align256(count * sizeof(LuStatus));
  const size_t pb = align256((size_t)count * 4 * KB * sizeof(int)), tb = split ? align256(count * sizeof(N2cTcBatch)) : 0;
  size_t btb = 0;   // split form: packed U12 expansions, 2n x 64 floats, hi and lo, per matrix
  if (split)
    for (int i = 0; i < count; ++i) btb += 2 * align256((size_t)2 * n[i] * 2 * KB * sizeof(float));
  char *dev = (char *)n2d_alloc_async(eb + sb + pb + tb + btb);
  if (!dev) return 0;
  LuBatchEntry *de = (LuBatchEntry *)dev;
  LuStatus *dst = (LuStatus *)(dev + eb);
  int *dpairs = (int *)(dev + eb + sb);
  N2cTcBatch *dtc = split ? (N2cTcBatch *)(dev + eb + sb + pb) : nullptr;
  char *bt = dev + eb + sb + pb + tb;
  std::vector<LuBatchEntry> h((size_t)count);
  std::vector<N2cTcBatch> htc(split ? (size_t)count : 0);
  for (int i = 0; i < count; ++i) {
    h[i] = LuBatchEntry{a_dev[i], n[i], ld[i], ipiv[i], dpairs + (size_t)i * 4 * KB, dst + i, nullptr, nullptr};
    if (split) {
      const size_t one = align256((size_t)2 * n[i] * 2 * KB * sizeof(float));
      h[i].bt_hi = (float *)bt;
      h[i].bt_lo = (float *)(bt + one);
      bt += 2 * one;
      htc[i] = N2cTcBatch{(float2 *)a_dev[i], n[i], ld[i], h[i].bt_hi, h[i].bt_lo};
    }
  }
  int ok = cudaMemsetAsync(dst, 0, count * sizeof(LuStatus), s) == cudaSuccess &&
           cudaMemcpyAsync(de, h.data(), count * sizeof(LuBatchEntry), cudaMemcpyHostToDevice, s) == cudaSuccess &&
           (!split ||
            cudaMemcpyAsync(dtc, htc.data(), count * sizeof(N2cTcBatch), cudaMemcpyHostToDevice, s) == cudaSuccess);
  if (!ok) n2c_set_error("batched factor: descriptor upload failed");
  // The update of panel step k0, part 0 (next panel's columns) or 1 (the rest).
  // Split form, the large part-1 updates of a batch of four or more: when
  // every matrix still updating has a block of at least 1024 x 1024, each
  // matrix's update goes to the persistent TMA-fed kernel in turn (it keeps
  // each CTA's row band of L21 resident instead of restaging it per 32-column
  // tile, and gives C bit for bit what the staged kernel gives); otherwise one
  // batched staged launch.  (Measured: 16 systems of order 2608 factor in
  // 43.7 ms against 47.4 ms; a single system is faster staged.)
  auto persistent_step = [&](long long k0) -> bool {
    if (count < 4) return false;
    bool any = false;
    for (int i = 0; i < count; ++i) {
      if (n[i] <= k0) continue;
      const long long kb = n[i] - k0 < KB ? n[i] - k0 : KB, right = n[i] - k0 - kb;
      const long long nb = right < KB ? right : KB;
      if (right < 1024 || right - nb < 1024) return false;
      any = true;
    }
    return any;
  };
  auto update = [&](long long k0, int part, long long rows, long long cols, cudaStream_t st) -> int {
    if (rows <= 0 || cols <= 0) return 1;
    if (split && part == 1 && persistent_step(k0)) {
      for (int i = 0; i < count; ++i) {
        if (n[i] <= k0) continue;
        const long long kb = n[i] - k0 < KB ? n[i] - k0 : KB, right = n[i] - k0 - kb;
        const long long nb = right < KB ? right : KB, cf = k0 + kb + nb;
        float2 *below = (float2 *)a_dev[i] + (k0 + kb) * ld[i];
        if (!n2c_tc_update((float *)(below + cf), ld[i], (const float *)(below + k0), ld[i],
                           h[i].bt_hi + 2 * nb * (2 * KB), h[i].bt_lo + 2 * nb * (2 * KB), right, right - nb,
                           &dst[i].error, st, N2C_TC_PERSISTENT))
          return 0;
      }
      return 1;
    }
    if (split) return n2c_tc_update_batch(dtc, count, k0, part, rows, cols, &dst[0].error, st);
    static const bool configured = cudaFuncSetAttribute(gemm_update_batch_kernel,
                                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        (int)GEMM_SMEM) == cudaSuccess;
    if (!configured) {
      cudaGetLastError();
      n2c_set_error("batched update: shared memory configuration failed");
      return 0;
    }
    gemm_update_batch_kernel<<<dim3((unsigned)((cols + GT - 1) / GT), (unsigned)((rows + GT - 1) / GT), (unsigned)count),
                               256, GEMM_SMEM, st>>>(de, k0, part);
    return n2c_check_launch("batched update");
  };
  ok = ok && launch_panel_batch<S>(de, count, 0, nmax, rule, s);
  const unsigned gb = (unsigned)((nmax + SWT / 32 - 1) / (SWT / 32));
  for (long long k0 = 0; ok && k0 < nmax; k0 += KB) {
    swap_trsm_batch_kernel<S><<<dim3(gb, (unsigned)count), SWT, 0, s>>>(de, k0);
    if (!n2c_check_launch("batched interchanges and triangular solve")) { ok = 0; break; }
    const long long right = nmax - k0 - (nmax - k0 < KB ? nmax - k0 : KB);
    if (right <= 0) break;
    const long long nb = right < KB ? right : KB, rest = right - nb;
    ok = update(k0, 0, right, nb, s);
    if (ok && (cudaEventRecord(la->next, s) != cudaSuccess || cudaStreamWaitEvent(la->aux, la->next, 0) != cudaSuccess)) {
      n2c_set_error("look-ahead event");
      ok = 0;
    }
    ok = ok && launch_panel_batch<S>(de, count, k0 + KB, right, rule, la->aux);
    if (ok && cudaEventRecord(la->panel, la->aux) != cudaSuccess) { n2c_set_error("look-ahead event"); ok = 0; }
    ok = ok && update(k0, 1, right, rest, s);
    if (ok && cudaStreamWaitEvent(s, la->panel, 0) != cudaSuccess) { n2c_set_error("look-ahead event"); ok = 0; }
  }
  if (la && !ok) cudaStreamSynchronize(la->aux);
  std::vector<LuStatus> hs((size_t)count);
  cudaError_t e = cudaMemcpyAsync(hs.data(), dst, count * sizeof(LuStatus), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (ok && e != cudaSuccess) { n2c_set_error("reading the batch status: %s", cudaGetErrorString(e)); ok = 0; }
  // A panel's or a per-matrix update's time-out lands in its own system's
  // status word; the batched staged update's in the first system's (its
  // launch covers them all).
  for (int i = 0; ok && i < count; ++i) {
    if (hs[i].error) {
      n2c_set_error("LU kernel wait time-out in a batch of %d (status word of system %d)", count, i);
      ok = 0;
    }
    info[i] = hs[i].info;
  }
  n2d_free_async(dev);
  return ok;
}

extern "C" int n2d_lu_factor_batch(double *const *a_dev, const long long *n, const long long *ld, int *const *ipiv,
                                   int count, int rule, int *info) {
  return factor_batch<double2>((void *const *)a_dev, n, ld, ipiv, count, rule, info);
}

extern "C" int n2d_lu_factor32_batch(float *const *a_dev, const long long *n, const long long *ld, int *const *ipiv,
                                     int count, int rule, int *info) {
  return factor_batch<float2>((void *const *)a_dev, n, ld, ipiv, count, rule, info);
}

// Cooperative CTAs per system when `systems` solves share the device.
static int solve_batch_group(int systems) {
  const int sms = n2c_sm_count();
  int g = systems > 0 ? sms / systems : SOLVE_CTAS;
  if (g > SOLVE_CTAS) g = SOLVE_CTAS;
  if (g < 2) g = 2;
  return g;
}

template <typename S>
static int solve_batch(const void *const *a_dev, const long long *n, const long long *ld, const int *const *ipiv,
                       double *const *b_dev, const long long *ldb, const long long *nrhs, int count) {
  if (count <= 0) return 1;
  if (count > 65535) {
    n2c_set_error("batched solve: %d systems (at most 65535)", count);
    return 0;
  }
  cudaStream_t s = n2c_stream();
  std::vector<SolveBatchEntry> one, coop;
  long long one_n = 0, one_rhs = 0, coop_n = 0;
  for (int i = 0; i < count; ++i) {
    if (!a_dev[i] || !ipiv[i] || !b_dev[i] || n[i] <= 0 || n[i] > 0x7fffffffLL || ld[i] < n[i] || ldb[i] < n[i] ||
        nrhs[i] < 0 || nrhs[i] > 65535) {
      n2c_set_error("batched solve: system %d has a null pointer, an order of 0, a leading dimension below its "
                    "order or a right-hand side count outside 0..65535", i);
      return 0;
    }
    if (nrhs[i] == 0) continue;
    SolveBatchEntry m{a_dev[i], n[i], ld[i], ipiv[i], (double2 *)b_dev[i], ldb[i], (int)nrhs[i], nullptr, nullptr};
    if (n[i] >= SOLVE_COOP_MIN && nrhs[i] <= SOLVE_COOP_RHS) {
      coop.push_back(m);
      if (n[i] > coop_n) coop_n = n[i];
    } else {
      one.push_back(m);
      if (n[i] > one_n) one_n = n[i];
      if (nrhs[i] > one_rhs) one_rhs = nrhs[i];
    }
  }
  static const bool attrs =
      cudaFuncSetAttribute(lu_solve_batch_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           8 * SOLVE_PERM_MAX) == cudaSuccess &&
      cudaFuncSetAttribute(lu_solve_coop_batch_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SOLVE_COOP_SMEM) == cudaSuccess;
  if (!attrs) {
    cudaGetLastError();
    n2c_set_error("batched solve: shared memory configuration failed");
    return 0;
  }
  // Cooperative groups: scratch vectors and barriers of every such system.
  const size_t nc = coop.size();
  size_t scratch_bytes = 0;
  for (const SolveBatchEntry &m : coop) scratch_bytes += align256((size_t)m.n * sizeof(double2));
  const size_t eb = align256((one.size() + nc) * sizeof(SolveBatchEntry)), syb = align256(nc * sizeof(SolveSync));
  char *dev = (char *)n2d_alloc_async(eb + syb + scratch_bytes + 256);
  if (!dev) return 0;
  SolveBatchEntry *de = (SolveBatchEntry *)dev;
  SolveSync *dsy = (SolveSync *)(dev + eb);
  char *sp = dev + eb + syb;
  for (size_t i = 0; i < nc; ++i) {
    coop[i].sy = dsy + i;
    coop[i].scratch = (double2 *)sp;
    sp += align256((size_t)coop[i].n * sizeof(double2));
  }
  std::vector<SolveBatchEntry> all(one);
  all.insert(all.end(), coop.begin(), coop.end());
  int ok = (nc == 0 || cudaMemsetAsync(dsy, 0, nc * sizeof(SolveSync), s) == cudaSuccess) &&
           cudaMemcpyAsync(de, all.data(), all.size() * sizeof(SolveBatchEntry), cudaMemcpyHostToDevice, s) ==
               cudaSuccess;
  if (!ok) n2c_set_error("batched solve: descriptor upload failed");
  if (ok && !one.empty()) {
    const size_t smem = (size_t)8 * (one_n < SOLVE_PERM_MAX ? one_n : SOLVE_PERM_MAX);
    lu_solve_batch_kernel<S><<<dim3((unsigned)one_rhs, (unsigned)one.size()), SOLVE_THREADS, smem, s>>>(de);
    ok = n2c_check_launch("batched solve");
  }
  // Cooperative systems in rounds that fit the device at one CTA per SM.
  const int g = solve_batch_group((int)nc);
  const int per_round = n2c_sm_count() / g > 0 ? n2c_sm_count() / g : 1;
  for (size_t i0 = 0; ok && i0 < nc; i0 += (size_t)per_round) {
    const unsigned k = (unsigned)(nc - i0 < (size_t)per_round ? nc - i0 : (size_t)per_round);
    const SolveBatchEntry *first = de + one.size() + i0;
    void *args[] = {(void *)&first};
    const cudaError_t e = cudaLaunchCooperativeKernel((void *)lu_solve_coop_batch_kernel<S>, dim3((unsigned)g, k),
                                                      SOLVE_COOP_THREADS, args, SOLVE_COOP_SMEM, s);
    if (e != cudaSuccess) {
      // Not launchable as one cooperative grid here: one CTA per system.
      cudaGetLastError();
      const size_t smem = (size_t)8 * (coop_n < SOLVE_PERM_MAX ? coop_n : SOLVE_PERM_MAX);
      lu_solve_batch_kernel<S><<<dim3(SOLVE_COOP_RHS, k), SOLVE_THREADS, smem, s>>>(first);
      ok = n2c_check_launch("batched solve");
    } else {
      n2c_count_launch(1);
    }
  }
  if (ok && nc) {
    std::vector<SolveSync> hs(nc);
    if (cudaMemcpyAsync(hs.data(), dsy, nc * sizeof(SolveSync), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      n2c_set_error("batched solve: reading the barrier status failed");
      ok = 0;
    }
    for (size_t i = 0; ok && i < nc; ++i)
      if (hs[i].error) { n2c_set_error("triangular solve: grid barrier time-out (batched)"); ok = 0; }
  }
  n2d_free_async(dev);
  return ok;
}

extern "C" int n2d_lu_solve_batch(const double *const *a_dev, const long long *n, const long long *ld,
                                  const int *const *ipiv, double *const *b_dev, const long long *ldb,
                                  const long long *nrhs, int count) {
  return solve_batch<double2>((const void *const *)a_dev, n, ld, ipiv, b_dev, ldb, nrhs, count);
}

extern "C" int n2d_lu_solve32_batch(const float *const *a_dev, const long long *n, const long long *ld,
                                    const int *const *ipiv, double *const *b_dev, const long long *ldb,
                                    const long long *nrhs, int count) {
  return solve_batch<float2>((const void *const *)a_dev, n, ld, ipiv, b_dev, ldb, nrhs, count);
}

// ------------------------------------------------------ allocation-free factor
// A variant of the classic factor for callers that cannot allocate device
// memory when they call in: a host application that hands the GPU's memory to
// its own pool allocator at start-up and forbids allocation afterwards, a
// plug-in living inside such a process, or a loop with a latency budget that
// cudaMalloc's implicit device synchronisation would break.  The caller passes
// the matrix and the pivot array already resident on the device; the panel
// status, the interchange pairs and the grid panel's candidate arrays live in
// one array defined in this file instead of being allocated per call.
//
// That array is a module global: every GPU on which the library is loaded
// holds it (19 KiB) until the process exits, and every call on that
// GPU shares it.  Calls whose work overlaps on the GPU (two streams, two host
// threads) therefore race on it; callers serialise them.  The array keeps the
// previous call's contents; only the panel status needs to start at zero and
// is cleared at the start of every call.
//
// Set-up: every call looks up the array's device address on the current
// device (cudaGetSymbolAddress; the array's name in host code is only a
// stand-in).  The lookup allocates nothing, and repeating it keeps the address
// right when the module is loaded again (after cudaDeviceReset, or in another
// context on the same device).  The first lookup in a context loads the
// module, so make the first call on a device before any stream capture.
//
// The factor is always the plain FP64 form (factr's pivot rule), whichever
// dense backend name is selected.
#include <climits>
#include "../../include/nec2c_cuda.h"

namespace {
constexpr int STATIC_GRID = (NEC2C_CUDA_STATIC_LU_MAX_ORDER + PT - 1) / PT;   // grid-panel blocks
constexpr size_t STATIC_STATUS_OFF = 0;
constexpr size_t STATIC_PAIRS_OFF = 256;
constexpr size_t STATIC_GVAL_OFF = 1024;
constexpr size_t STATIC_GIDX_OFF = STATIC_GVAL_OFF + 2 * STATIC_GRID * sizeof(double);
constexpr size_t STATIC_GROWJ_OFF = 2048;
constexpr size_t STATIC_GROW_OFF = STATIC_GROWJ_OFF + 2 * KB * sizeof(double2);
constexpr size_t STATIC_SCRATCH_BYTES = STATIC_GROW_OFF + (size_t)2 * STATIC_GRID * KB * sizeof(double2);
static_assert(sizeof(LuStatus) <= STATIC_PAIRS_OFF - STATIC_STATUS_OFF, "status slot");
static_assert(4 * KB * sizeof(int) <= STATIC_GVAL_OFF - STATIC_PAIRS_OFF, "pairs slot");
static_assert(STATIC_GIDX_OFF + 2 * STATIC_GRID * sizeof(int) <= STATIC_GROWJ_OFF, "grid candidates slot");
// The documented size (header, integration notes): 19 KiB.
static_assert(STATIC_SCRATCH_BYTES == 19 * 1024, "scratch array size changed: update its documentation");
}  // namespace

static __device__ __align__(256) unsigned char lu_static_scratch[STATIC_SCRATCH_BYTES];

// Device address of the scratch array in the current context.
static unsigned char *static_scratch() {
  void *ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, lu_static_scratch);
  if (e != cudaSuccess || !ptr) {
    int dev = -1;
    cudaGetDevice(&dev);
    n2c_set_error("scratch address on device %d: %s", dev, cudaGetErrorString(e));
    return nullptr;
  }
  return (unsigned char *)ptr;
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
  FactorScratch w;
  memset(&w, 0, sizeof(w));
  w.st = (LuStatus *)(base + STATIC_STATUS_OFF);
  w.pairs = (int *)(base + STATIC_PAIRS_OFF);
  w.gval = (double *)(base + STATIC_GVAL_OFF);
  w.gidx = (int *)(base + STATIC_GIDX_OFF);
  w.growj = (double2 *)(base + STATIC_GROWJ_OFF);
  w.grow = (double2 *)(base + STATIC_GROW_OFF);
  cudaError_t e = cudaMemsetAsync(w.st, 0, sizeof(LuStatus), n2c_stream());
  if (e != cudaSuccess) { n2c_set_error("clearing the panel status: %s", cudaGetErrorString(e)); return 0; }
  int info = 0;
  if (!factor_panels((double2 *)matrix_dev, (long long)order, (long long)leading_dimension, pivots_dev, 0, w, false,
                     &info))
    return 0;
  if (info) { n2c_set_error("matrix is singular (pivot %d)", info); return 0; }
  return 1;
}

// Ragged batch of volume FFT plans solved together on one GPU.
//
// Many frequencies or geometries, each a plan with its own lattice, padded
// grid (axes up to 256) and spectrum, advance through GMRES(m) in lockstep:
//   - every FFT pass of a product is ONE launch over the tiles of all plans:
//     a CTA finds its plan by binary search over the plans' first tiles and
//     runs the tile body of that plan's line length (fft_engine.cuh);
//   - every Gram-Schmidt sweep, update and norm is one launch over all
//     systems' unknowns: a CTA covers a fixed range of one system, and the
//     last CTA of each system finishes its reduction in a fixed order;
//   - the Arnoldi steps of a restart cycle are captured CUDA graphs of five
//     steps each; between graphs the host reads how many systems are still
//     in the cycle and ends it when none is.
// Each system keeps its own GMRES state (Hessenberg matrix, rotations,
// status) with vie_gmres's per-system semantics (vie_iterative.c:90-200);
// a system that has converged or stopped is gated off and costs nothing.
// The Arnoldi process is classical Gram-Schmidt: the second pass runs on a
// tenfold cancellation for plans with FP32 transforms and always for FP64
// plans (CGS2, as stable as the two MGS passes of vie_iterative.c).
//
// A system is a volume plan or a hybrid conductor + volume system [C B; D V]
// of dielectric_fft.c:41-83 (wire segments beside a dielectric body): its
// conductor rows and cross rows are one launch each over all systems too.
// The batch's vectors are the systems' vectors (conductor unknowns, then 3 x
// cells) concatenated in system order.
#include <stdlib.h>
#include <float.h>
#include <math.h>
#include <string.h>
#include <algorithm>
#include <atomic>
#include <vector>
#include "common.cuh"
#include "device_api.h"
#include "runtime.cuh"
#include "vie_batch.cuh"
#include "vie_internal.cuh"

using namespace n2c;

n2d_vie *n2c_hybrid_volume(const n2d_hybrid *h);
const double2 *n2c_hybrid_pdiag(const n2d_hybrid *h);
const double2 *n2c_hybrid_blocks(const n2d_hybrid *h);
long long n2c_hybrid_conductors(const n2d_hybrid *h);
int n2c_hybrid_precondition_ok(const n2d_hybrid *h);

namespace {

enum { ST_CONVERGED, ST_LIMIT, ST_BREAKDOWN, ST_CALLBACK, ST_INVALID, ST_ALLOC, ST_NONFINITE };
enum { ST_RUNNING = -1 };

constexpr int BMAXM = 30;                         // longest restart cycle of a batch
constexpr int MAX_L = 256;                        // longest padded axis of a batched plan
constexpr double REORTH = 10.0;                   // cancellation factor of the FP32-transform form
constexpr int DOT_E = 4;                          // elements per lane per dots load
constexpr int DOT_GROUP = 32 * DOT_E;             // elements per warp group
constexpr long long DOT_RANGE = 32 * DOT_GROUP;   // elements per dots CTA
constexpr size_t DOT_SMEM = (size_t)DOT_RANGE * sizeof(double2);
constexpr int VEC_THREADS = 256;
constexpr long long VEC_RANGE = 4 * VEC_THREADS;  // elements per vector-kernel CTA

template <typename C> struct BatchDesc {
  PassArgs<C> a;
  long long off;   // first element of the plan's cell vector in the batch vectors
  int L;           // line length of the pass
  int variant;     // radix split (fft_passes.cuh): 0 default, 1 transposed
};

// Conductor blocks of a hybrid system: the c rows [C|B] (c x n) then the
// v x c cross block D, row-major (n = c + v); c == 0 for a volume plan.
struct BHyb {
  const double2 *blocks;
  long long c, n;
};

// Per-system GMRES state (device).
struct BSys {
  int active;      // inner iterations of the current cycle still running
  int running;     // gate of the true-residual product
  int status;      // ST_RUNNING or a final status
  int flag;        // non-finite raised in an Arnoldi product
  int rflag;       // non-finite raised in a residual product or norm
  int used, breakdown, normalize, reorth;
  int m;           // cycle length of this system, min(restart, unknowns)
  long long iterations, max_iterations;
  double target, before_sq, after, beta;
  unsigned ticket;
  int pad;
};

struct BView {
  BSys *sys;
  const long long *off;                 // K + 1 element offsets
  const long long *first_d, *first_v;   // K + 1 first CTAs (dots / vector kernels)
  int K, m;                             // systems; Hessenberg leading dimension
  long long N;
  double2 *V, *w, *r, *H, *g, *sn, *y, *hp;
  double *cs;
  double2 *parts_d;
  double *parts_v, *norms;
  const double2 *const *diag;           // Jacobi divisors of each system
  int always_reorth;
};

__device__ __forceinline__ int find_seg(const long long *first, int count, long long x) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// True in the one CTA that arrives last among `count` CTAs sharing ticket.
__device__ __forceinline__ bool last_of(unsigned *ticket, unsigned count) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == count - 1;
  __syncthreads();
  return last;
}

__device__ __forceinline__ double cabs_(double2 a) { return hypot(a.x, a.y); }

// ------------------------------------------------------- batched FFT passes
template <typename C, int R1, int R2, int MODE>
__device__ __forceinline__ void tile_body(const PassArgs<C> &a, long long tile, unsigned ntiles) {
  if constexpr (MODE == 0) fft_forward_tile<C, R1, R2>(a, tile);
  else if constexpr (MODE == 1) fft_inverse_tile<C, R1, R2>(a, tile, ntiles);
  else if constexpr (MODE == 2) fft_product_tile<C, R1, R2>(a, tile);
  else if constexpr (MODE == 7) fft_zline_tile<C, R1, R2, false, true>(a, tile, ntiles);
  else fft_zline_tile<C, R1, R2, true, true>(a, tile, ntiles);
}

// One pass over the tiles of every plan; x / y are the batch vectors the z
// passes scatter from and gather into.
template <typename C, int MODE>
__global__ void __launch_bounds__(256, MODE <= 1 ? 1 : (MODE == 2 && sizeof(C) != sizeof(float2) ? 2 : 3))
    batch_pass_kernel(const BatchDesc<C> *desc, const long long *first, int count, const double2 *x, double2 *y) {
  pdl_begin();
  const int q = find_seg(first, count, blockIdx.x);
  // A stopped system's tiles leave before its arguments are read.
  const int *gate = desc[q].a.gate;
  if (gate && *(volatile const int *)gate == 0) return;
  PassArgs<C> a = desc[q].a;
  if (MODE >= 7) {
    a.cx = x + desc[q].off;
    a.cy = y + desc[q].off;
  }
  const long long tile = (long long)blockIdx.x - first[q];
  const unsigned ntiles = (unsigned)(first[q + 1] - first[q]);
  if (desc[q].variant) {
    switch (desc[q].L) {
      case 16: tile_body<C, 4, 4, MODE>(a, tile, ntiles); break;
      case 32: tile_body<C, 4, 8, MODE>(a, tile, ntiles); break;
      case 64: tile_body<C, 16, 4, MODE>(a, tile, ntiles); break;
      case 128: tile_body<C, 8, 16, MODE>(a, tile, ntiles); break;
    }
    return;
  }
  switch (desc[q].L) {
    case 1: tile_body<C, 1, 1, MODE>(a, tile, ntiles); break;
    case 2: tile_body<C, 2, 1, MODE>(a, tile, ntiles); break;
    case 4: tile_body<C, 4, 1, MODE>(a, tile, ntiles); break;
    case 8: tile_body<C, 8, 1, MODE>(a, tile, ntiles); break;
    case 16: tile_body<C, 16, 1, MODE>(a, tile, ntiles); break;
    case 32: tile_body<C, 8, 4, MODE>(a, tile, ntiles); break;
    case 64: tile_body<C, 8, 8, MODE>(a, tile, ntiles); break;
    case 128: tile_body<C, 16, 8, MODE>(a, tile, ntiles); break;
    case 256: tile_body<C, 16, 16, MODE>(a, tile, ntiles); break;
  }
}

template <typename C>
void (*batch_kernel(int mode))(const BatchDesc<C> *, const long long *, int, const double2 *, double2 *) {
  switch (mode) {
    case 0: return batch_pass_kernel<C, 0>;
    case 1: return batch_pass_kernel<C, 1>;
    case 2: return batch_pass_kernel<C, 2>;
    case 7: return batch_pass_kernel<C, 7>;
  }
  return batch_pass_kernel<C, 8>;
}

// ---------------------------------------------------------- vector kernels
// CTA (q, t) of a vector kernel covers elements [t VEC_RANGE, (t+1) VEC_RANGE)
// of system q (clipped to the system).
struct VecCta {
  int q;
  long long lo, hi, nctas;
  bool first;
};
__device__ __forceinline__ VecCta vec_cta(const BView &v) {
  VecCta c;
  c.q = find_seg(v.first_v, v.K, blockIdx.x);
  const long long t = (long long)blockIdx.x - v.first_v[c.q];
  c.lo = v.off[c.q] + t * VEC_RANGE;
  c.hi = min(c.lo + VEC_RANGE, v.off[c.q + 1]);
  c.nctas = v.first_v[c.q + 1] - v.first_v[c.q];
  c.first = t == 0;
  return c;
}

// Sum over the vector CTAs of system q of their partials, in CTA order (same
// value in every thread of the calling CTA).
__device__ double sum_parts_v(const BView &v, int q) {
  double t = 0;
  for (long long c = v.first_v[q] + threadIdx.x; c < v.first_v[q + 1]; c += blockDim.x) t += v.parts_v[c];
  return block_sum(make_double2(t, 0)).x;
}

// norms[q] = ||x_q||^2 of every system; a non-finite sum raises rflag.
__global__ void __launch_bounds__(VEC_THREADS) seg_norm_kernel(BView v, const double2 *x, double *norms) {
  const VecCta c = vec_cta(v);
  double sq = 0;
  for (long long i = c.lo + threadIdx.x; i < c.hi; i += VEC_THREADS) sq += x[i].x * x[i].x + x[i].y * x[i].y;
  const double2 bs = block_sum(make_double2(sq, 0));
  if (threadIdx.x == 0) v.parts_v[blockIdx.x] = bs.x;
  BSys *s = v.sys + c.q;
  if (!last_of(&s->ticket, (unsigned)c.nctas)) return;
  const double tot = sum_parts_v(v, c.q);
  if (threadIdx.x == 0) {
    norms[c.q] = tot;
    if (!isfinite(tot)) s->rflag = 1;
    s->ticket = 0;
  }
}

// r = b - r (A x already in r) for the systems whose residual is taken.
__global__ void __launch_bounds__(VEC_THREADS) seg_residual_kernel(BView v, const double2 *rhs) {
  const VecCta c = vec_cta(v);
  if (!v.sys[c.q].running) return;
  for (long long i = c.lo + threadIdx.x; i < c.hi; i += VEC_THREADS) v.r[i] = csub(rhs[i], v.r[i]);
}

// v_0 = r / beta, Hessenberg and right-hand side reset for a new cycle.
__global__ void __launch_bounds__(VEC_THREADS) seg_cycle_start_kernel(BView v) {
  const VecCta c = vec_cta(v);
  const BSys *s = v.sys + c.q;
  if (!s->active) return;
  const double beta = s->beta;
  for (long long i = c.lo + threadIdx.x; i < c.hi; i += VEC_THREADS)
    v.V[i] = make_double2(v.r[i].x / beta, v.r[i].y / beta);
  if (!c.first) return;
  double2 *H = v.H + (long long)c.q * (v.m + 1) * v.m, *g = v.g + (long long)c.q * (v.m + 1);
  for (int i = threadIdx.x; i < (v.m + 1) * v.m; i += VEC_THREADS) H[i] = make_double2(0, 0);
  for (int i = threadIdx.x; i <= v.m; i += VEC_THREADS) g[i] = make_double2(i == 0 ? beta : 0, 0);
}

// Complex unitary Givens [c s; -conj(s) c], vie_iterative.c:66-78.
__device__ void givens(double2 a, double2 b, double *c, double2 *s) {
  const double aa = cabs_(a), bb = cabs_(b);
  if (bb == 0.0) { *c = 1.0; *s = make_double2(0, 0); }
  else if (aa == 0.0) { *c = 0.0; *s = make_double2(b.x / bb, -b.y / bb); }
  else {
    const double len = hypot(aa, bb);
    *c = aa / len;
    const double2 ua = make_double2(a.x / aa, a.y / aa), ub = make_double2(b.x / len, -b.y / len);
    *s = cmul(ua, ub);
  }
}

// Column j of system q finished with h_{j+1,j} = after: previous rotations,
// the new rotation, the residual estimate and the cycle's stop conditions
// (vie_iterative.c:160-177).
__device__ void finish_column(const BView &v, int q, int j, double after) {
  BSys *s = v.sys + q;
  const int m = v.m;
  const double before = sqrt(s->before_sq);
  const bool broke = after <= 32 * DBL_EPSILON * before;
  s->after = after;
  s->reorth = 0;
  if (!isfinite(after)) { s->status = ST_NONFINITE; s->active = 0; return; }
  double2 *H = v.H + (long long)q * (m + 1) * m, *g = v.g + (long long)q * (m + 1), *sn = v.sn + (long long)q * m;
  double *cs = v.cs + (long long)q * m;
  H[(long long)(j + 1) * m + j] = make_double2(after, 0);
  for (int k = 0; k < j; ++k) {
    const double2 h0 = H[(long long)k * m + j], h1 = H[(long long)(k + 1) * m + j];
    H[(long long)k * m + j] = cadd(cscale(h0, cs[k]), cmul(sn[k], h1));
    H[(long long)(k + 1) * m + j] = csub(cscale(h1, cs[k]), cconjmul(sn[k], h0));
  }
  double c;
  double2 sr;
  givens(H[(long long)j * m + j], H[(long long)(j + 1) * m + j], &c, &sr);
  cs[j] = c;
  sn[j] = sr;
  H[(long long)j * m + j] = cadd(cscale(H[(long long)j * m + j], c), cmul(sr, H[(long long)(j + 1) * m + j]));
  H[(long long)(j + 1) * m + j] = make_double2(0, 0);
  const double2 gj = g[j];
  g[j + 1] = make_double2(-(sr.x * gj.x + sr.y * gj.y), -(sr.x * gj.y - sr.y * gj.x));   // -conj(s) g_j
  g[j] = cscale(gj, c);
  s->iterations += 1;
  s->used = j + 1;
  s->breakdown = broke;
  s->normalize = !broke;
  if (broke || cabs_(g[j + 1]) <= s->target || j + 1 >= s->m || s->iterations >= s->max_iterations) s->active = 0;
}

// h = V^H w of pass P for every active system.  CTA (q, t) covers DOT_RANGE
// elements of system q; warp k % kk of each group of kk warps handles basis
// vector k over its element group, the w chunk sits in shared memory.
template <int P>
__global__ void __launch_bounds__(1024) seg_dots_kernel(BView v, int j) {
  const int q = find_seg(v.first_d, v.K, blockIdx.x);
  BSys *s = v.sys + q;
  if (!s->active || (P == 1 && !s->reorth)) return;
  const long long t0 = (long long)blockIdx.x - v.first_d[q];
  if (P == 0 && s->flag) {
    if (t0 == 0 && threadIdx.x == 0) { s->status = ST_NONFINITE; s->active = 0; }
    return;
  }
  const int kk = j + 1, groups = 32 / kk, chunk = groups * DOT_GROUP;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, k = warp % kk, grp = warp / kk;
  const bool act = grp < groups;
  const long long lo = v.off[q] + t0 * DOT_RANGE, hi = min(lo + DOT_RANGE, v.off[q + 1]);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *sw = reinterpret_cast<double2 *>(smem_raw);   // [chunk]
  const double2 *Vk = v.V + (long long)k * v.N;
  const int wper = (chunk + blockDim.x - 1) / blockDim.x;
  double2 acc = make_double2(0, 0), vv[DOT_E], vn[DOT_E], wv[4], wn[4];
  auto load = [&](long long base, double2 (&a)[DOT_E], double2 (&b)[4]) {
    if (act) {
#pragma unroll
      for (int e = 0; e < DOT_E; ++e) {
        const long long i = base + grp * DOT_GROUP + lane + 32 * e;
        a[e] = i < hi ? Vk[i] : make_double2(0, 0);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int tt = threadIdx.x + u * blockDim.x;
      b[u] = (u < wper && tt < chunk && base + tt < hi) ? v.w[base + tt] : make_double2(0, 0);
    }
  };
  load(lo, vv, wv);
  for (long long base = lo; base < hi; base += chunk) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int tt = threadIdx.x + u * blockDim.x;
      if (u < wper && tt < chunk) sw[tt] = wv[u];
    }
    if (base + chunk < hi) load(base + chunk, vn, wn);
    __syncthreads();
    if (act) {
#pragma unroll
      for (int e = 0; e < DOT_E; ++e) acc = cadd(acc, cconjmul(vv[e], sw[grp * DOT_GROUP + lane + 32 * e]));
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < DOT_E; ++e) vv[e] = vn[e];
#pragma unroll
    for (int u = 0; u < 4; ++u) wv[u] = wn[u];
  }
  __shared__ double2 red[32];
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
  }
  if (lane == 0) red[warp] = act ? acc : make_double2(0, 0);
  __syncthreads();
  if (threadIdx.x < kk) {
    double2 tt = make_double2(0, 0);
    for (int gg = 0; gg < groups; ++gg) tt = cadd(tt, red[gg * kk + threadIdx.x]);
    v.parts_d[(long long)blockIdx.x * BMAXM + threadIdx.x] = tt;
  }
  const long long nctas = v.first_d[q + 1] - v.first_d[q];
  if (!last_of(&s->ticket, (unsigned)nctas)) return;
  if (warp < kk) {
    double2 tt = make_double2(0, 0);
    for (long long c = v.first_d[q] + lane; c < v.first_d[q + 1]; c += 32)
      tt = cadd(tt, v.parts_d[c * BMAXM + warp]);
    for (int o = 16; o > 0; o >>= 1) {
      tt.x += __shfl_xor_sync(0xffffffffu, tt.x, o);
      tt.y += __shfl_xor_sync(0xffffffffu, tt.y, o);
    }
    if (lane == 0) {
      const int m = v.m;
      v.hp[((long long)q * 2 + P) * BMAXM + warp] = tt;
      double2 *H = v.H + (long long)q * (m + 1) * m;
      H[(long long)warp * m + j] = cadd(H[(long long)warp * m + j], tt);
    }
  }
  if (threadIdx.x == 0) s->ticket = 0;
}

// w -= V h of pass P and ||w||^2 for every active system; the last CTA of a
// system requests its second pass or finishes its column.
template <int P>
__global__ void __launch_bounds__(VEC_THREADS) seg_update_kernel(BView v, int j) {
  const VecCta c = vec_cta(v);
  BSys *s = v.sys + c.q;
  if (!s->active || (P == 1 && !s->reorth)) return;
  const int kk = j + 1;
  __shared__ double2 hs[BMAXM];
  if (threadIdx.x < kk) hs[threadIdx.x] = v.hp[((long long)c.q * 2 + P) * BMAXM + threadIdx.x];
  __syncthreads();
  double sq = 0;
  for (long long i = c.lo + threadIdx.x; i < c.hi; i += VEC_THREADS) {
    double2 wi = v.w[i];
#pragma unroll 6
    for (int k = 0; k < kk; ++k) wi = csub(wi, cmul(hs[k], v.V[(long long)k * v.N + i]));
    v.w[i] = wi;
    sq += wi.x * wi.x + wi.y * wi.y;
  }
  const double2 bs = block_sum(make_double2(sq, 0));
  if (threadIdx.x == 0) v.parts_v[blockIdx.x] = bs.x;
  if (!last_of(&s->ticket, (unsigned)c.nctas)) return;
  const double tot = sum_parts_v(v, c.q);
  if (threadIdx.x != 0) return;
  s->ticket = 0;
  const double after = sqrt(tot);
  if (P == 0 && isfinite(after) && (v.always_reorth || REORTH * after < sqrt(s->before_sq))) {
    s->reorth = 1;
    return;
  }
  finish_column(v, c.q, j, after);
}

// v_{j+1} = w / ||w|| of every system whose column j was finished without
// breakdown and whose cycle continues.
__global__ void __launch_bounds__(VEC_THREADS) seg_normalize_kernel(BView v, int j) {
  const VecCta c = vec_cta(v);
  const BSys *s = v.sys + c.q;
  if (!s->active || !s->normalize) return;
  const double inv = s->after;
  double2 *vn = v.V + (long long)(j + 1) * v.N;
  for (long long i = c.lo + threadIdx.x; i < c.hi; i += VEC_THREADS)
    vn[i] = make_double2(v.w[i].x / inv, v.w[i].y / inv);
}

// Gate of a kernel run for descriptor set `set` (0 Arnoldi, 1 residual, 2 plain).
__device__ __forceinline__ bool sys_gated(const BSys *s, int set) {
  return set == 0 ? !s->active : set == 1 ? !s->running : false;
}

// Conductor rows per CTA of the conductor-row kernel, and the cross-row
// layout: a system with at most CROSS_PACK conductor unknowns takes
// CROSS_ELEMS / c volume rows per CTA (its D rows are contiguous, so the CTA
// streams one contiguous block of D); a system with more takes 8 rows per
// CTA, a warp per row.
constexpr int COND_ROWS = 4;
constexpr int CROSS_PACK = 64;
constexpr int CROSS_ELEMS = 2048;
__host__ __device__ __forceinline__ long long cross_rows_per_cta(long long c) {
  return c <= CROSS_PACK ? CROSS_ELEMS / c : 8;
}

// z = x of every hybrid system, divided by its preconditioner divisor for
// the Arnoldi set (the conductor and cross rows then read z, computed once).
__global__ void __launch_bounds__(VEC_THREADS) seg_zc_kernel(BView v, const BHyb *hyb, const double2 *x, double2 *z,
                                                             int set) {
  const VecCta c = vec_cta(v);
  if (hyb[c.q].c == 0 || sys_gated(v.sys + c.q, set)) return;
  const double2 *pd = v.diag[c.q];
  const long long base = v.off[c.q];
  for (long long i = c.lo + threadIdx.x; i < c.hi; i += VEC_THREADS)
    z[i] = set == 0 ? cdiv(x[i], pd[i - base]) : x[i];
}

// COND_ROWS conductor rows of one hybrid system per CTA: y_i = sum_j
// [C|B]_ij z_j (dielectric_fft.c:54-66), z read once for all the CTA's rows.
__global__ void __launch_bounds__(256) seg_conductor_kernel(BView v, const BHyb *hyb, const long long *crow,
                                                            const double2 *z, double2 *y, int set) {
  const int q = find_seg(crow, v.K, blockIdx.x);
  if (sys_gated(v.sys + q, set)) return;
  const BHyb hb = hyb[q];
  const long long i0 = ((long long)blockIdx.x - crow[q]) * COND_ROWS;
  const int rows = (int)min((long long)COND_ROWS, hb.c - i0);
  const double2 *zq = z + v.off[q], *row = hb.blocks + i0 * hb.n;
  double2 acc[COND_ROWS];
#pragma unroll
  for (int r = 0; r < COND_ROWS; ++r) acc[r] = make_double2(0, 0);
  for (long long j = threadIdx.x; j < hb.n; j += blockDim.x) {
    const double2 zj = zq[j];
#pragma unroll
    for (int r = 0; r < COND_ROWS; ++r)
      if (r < rows) acc[r] = cadd(acc[r], cmul(row[r * hb.n + j], zj));
  }
  for (int r = 0; r < rows; ++r) {
    const double2 t = block_sum(acc[r]);
    if (threadIdx.x == 0) y[v.off[q] + i0 + r] = t;
  }
}

// Volume rows of one hybrid system per CTA: y_{c+i} += sum_j D_ij z_j over
// its conductor unknowns (dielectric_fft.c:67-74), summed in j order.  With
// few conductor unknowns the CTA's D rows form one contiguous block: it is
// read coalesced into shared memory as products D_ij z_j, then a thread per
// row adds its row up.  With many, a warp per row.
__global__ void __launch_bounds__(256) seg_cross_kernel(BView v, const BHyb *hyb, const long long *xrow,
                                                        const double2 *z, double2 *y, int set) {
  const int q = find_seg(xrow, v.K, blockIdx.x);
  if (sys_gated(v.sys + q, set)) return;
  const BHyb hb = hyb[q];
  const long long c = hb.c, nv = hb.n - c, per = cross_rows_per_cta(c);
  const long long r0 = ((long long)blockIdx.x - xrow[q]) * per;
  const int rows = (int)min(per, nv - r0);
  const double2 *zq = z + v.off[q], *D = hb.blocks + c * hb.n + r0 * c;
  double2 *yq = y + v.off[q] + c + r0;
  __shared__ double2 prod[CROSS_ELEMS];
  __shared__ double2 zc[CROSS_PACK];
  if (c <= CROSS_PACK) {
    for (int j = threadIdx.x; j < c; j += blockDim.x) zc[j] = zq[j];
    __syncthreads();
    const int cc = (int)c, total = rows * cc;
    for (int e = threadIdx.x; e < total; e += blockDim.x) prod[e] = cmul(D[e], zc[e % cc]);
    __syncthreads();
    for (int t = threadIdx.x; t < rows; t += blockDim.x) {
      double2 acc = make_double2(0, 0);
      for (int j = 0; j < cc; ++j) acc = cadd(acc, prod[t * cc + j]);
      yq[t] = cadd(yq[t], acc);
    }
    return;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp >= rows) return;
  const double2 *row = D + (long long)warp * c;
  double2 acc = make_double2(0, 0);
  for (long long j = lane; j < c; j += 32) acc = cadd(acc, cmul(row[j], zq[j]));
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
  }
  if (lane == 0) yq[warp] = cadd(yq[warp], acc);
}

// ||w||^2 of every active system into before_sq (batches with hybrid
// systems, whose conductor rows come after the volume epilogue); a
// non-finite entry raises the system's flag.
__global__ void __launch_bounds__(VEC_THREADS) seg_wnorm_kernel(BView v) {
  const VecCta c = vec_cta(v);
  BSys *s = v.sys + c.q;
  if (!s->active) return;
  double sq = 0;
  bool bad = false;
  for (long long i = c.lo + threadIdx.x; i < c.hi; i += VEC_THREADS) {
    const double2 wi = v.w[i];
    sq += wi.x * wi.x + wi.y * wi.y;
    bad |= !finite2(wi);
  }
  if (bad) s->flag = 1;
  const double2 bs = block_sum(make_double2(sq, 0));
  if (threadIdx.x == 0) v.parts_v[blockIdx.x] = bs.x;
  if (!last_of(&s->ticket, (unsigned)c.nctas)) return;
  const double tot = sum_parts_v(v, c.q);
  if (threadIdx.x == 0) {
    s->before_sq = tot;
    s->ticket = 0;
  }
}

// *out = number of systems still in their cycle.
__global__ void count_active_kernel(BView v, int *out) {
  int c = 0;
  for (int q = threadIdx.x; q < v.K; q += blockDim.x) c += v.sys[q].active != 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  __shared__ int red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    *out = t;
  }
}

// y = H^{-1} g of every running system (vie_iterative.c:179-186), one warp
// per system: the lanes share each row's sum over the solved unknowns, added
// in a fixed order (lane partials, then a butterfly).
__global__ void seg_backsolve_kernel(BView v) {
  const int q = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (q >= v.K) return;
  BSys *s = v.sys + q;
  if (s->status != ST_RUNNING) return;
  const int m = v.m, used = s->used;
  const double2 *H = v.H + (long long)q * (m + 1) * m, *g = v.g + (long long)q * (m + 1);
  double2 *y = v.y + (long long)q * m;
  for (int i = used - 1; i >= 0; --i) {
    double2 part = make_double2(0, 0);
    for (int k = i + 1 + lane; k < used; k += 32) part = cadd(part, cmul(H[(long long)i * m + k], y[k]));
    for (int o = 16; o > 0; o >>= 1) {
      part.x += __shfl_xor_sync(0xffffffffu, part.x, o);
      part.y += __shfl_xor_sync(0xffffffffu, part.y, o);
    }
    const double2 d = H[(long long)i * m + i];
    if (cabs_(d) == 0.0) {
      if (lane == 0) s->status = ST_BREAKDOWN;
      return;
    }
    if (lane == 0) y[i] = cdiv(csub(g[i], part), d);
    __syncwarp();
  }
}

// x += D^-1 (sum_j v_j y_j) of every running system, the divisor applied
// once to the sum.
__global__ void __launch_bounds__(VEC_THREADS) seg_xupdate_kernel(BView v, double2 *x) {
  const VecCta c = vec_cta(v);
  const BSys *s = v.sys + c.q;
  if (s->status != ST_RUNNING) return;
  const int used = s->used;
  const double2 *y = v.y + (long long)c.q * v.m, *diag = v.diag[c.q];
  const long long base = v.off[c.q];
  for (long long i = c.lo + threadIdx.x; i < c.hi; i += VEC_THREADS) {
    double2 acc = make_double2(0, 0);
    for (int jj = 0; jj < used; ++jj) acc = cadd(acc, cmul(v.V[(long long)jj * v.N + i], y[jj]));
    x[i] = cadd(x[i], cdiv(acc, diag[i - base]));
  }
}

}  // namespace

// ------------------------------------------------------------------ host side
// Pass descriptor sets: 0 Arnoldi products (transform precision, Jacobi
// preconditioned input, ||w||^2, gated by each system's cycle), 1 true
// residual products (FP64, gated by the running systems), 2 plain products
// (transform precision, ungated).
struct PassSet {
  void *desc = nullptr;        // BatchDesc<C>[K]
  long long *first = nullptr;  // K + 1 first tiles
  long long tiles = 0;
  size_t smem = 0;
  int mode = 0;
  bool fp32 = false;
};

// Arnoldi steps per captured graph: after each chunk the host reads how many
// systems are still in their cycle and ends the cycle when none is, so the
// steps after the last system's stop test are not launched.
constexpr int CHUNK = 5;
constexpr int MAX_CHUNKS = (BMAXM + CHUNK - 1) / CHUNK;

struct BatchWork {
  int m = 0;
  BView v;
  int *active_count = nullptr;   // device: systems still in the cycle
  cudaGraphExec_t chunk[MAX_CHUNKS] = {};
  unsigned chunk_launches[MAX_CHUNKS] = {};
  bool tried_graph = false;
};

struct n2d_vie_batch {
  int K = 0, fp32 = 0;
  long long N = 0;
  std::vector<n2d_vie *> plans;
  std::vector<n2d_hybrid *> hybrids;          // null for a volume plan
  std::vector<long long> cond, crow, xrow;    // conductor unknowns; row prefixes
  bool any_hybrid = false;
  BHyb *hyb_dev = nullptr;
  long long *crow_dev = nullptr, *xrow_dev = nullptr;   // CTA prefixes of the conductor / cross kernels
  double2 *zbuf = nullptr;                              // z of the hybrid systems (batch order)
  std::vector<long long> off, first_d, first_v;
  long long *off_dev = nullptr, *first_d_dev = nullptr, *first_v_dev = nullptr;
  BSys *sys = nullptr;
  const double2 **diag_dev = nullptr;
  PassSet sets[3][N2D_VIE_PASSES];
  int scale[N2D_VIE_PASSES] = {0, 0, 0, 0, 0};     // tile height scale per pass (batch tuner)
  int variant[N2D_VIE_PASSES] = {0, 0, 0, 0, 0};   // radix split per pass (batch tuner)
  BatchWork *work = nullptr;
};

static void work_free(BatchWork *w) {
  if (!w) return;
  for (cudaGraphExec_t &g : w->chunk)
    if (g) cudaGraphExecDestroy(g);
  BView &v = w->v;
  void *bufs[] = {v.V, v.w, v.r, v.H, v.g, v.sn, v.y, v.hp, v.cs, v.parts_d, v.parts_v, v.norms, w->active_count};
  for (void *q : bufs) n2d_free(q);
  delete w;
}

static void free_set(n2d_vie_batch *b, int set) {
  for (PassSet &ps : b->sets[set]) {
    n2d_free(ps.desc);
    n2d_free(ps.first);
    ps = PassSet();
  }
}

extern "C" void n2d_vie_batch_destroy(n2d_vie_batch *b) {
  if (!b) return;
  work_free(b->work);
  for (int set = 0; set < 3; ++set) free_set(b, set);
  n2d_free(b->off_dev);
  n2d_free(b->first_d_dev);
  n2d_free(b->first_v_dev);
  n2d_free(b->sys);
  n2d_free((void *)b->diag_dev);
  n2d_free(b->hyb_dev);
  n2d_free(b->crow_dev);
  n2d_free(b->xrow_dev);
  n2d_free(b->zbuf);
  delete b;
}

template <typename C>
static int build_set(n2d_vie_batch *b, int set) {
  const int K = b->K;
  std::vector<BatchDesc<C>> desc[N2D_VIE_PASSES];
  std::vector<long long> first[N2D_VIE_PASSES];
  for (int i = 0; i < N2D_VIE_PASSES; ++i) {
    desc[i].resize(K);
    first[i].assign(K + 1, 0);
  }
  for (int q = 0; q < K; ++q) {
    BSys *s = b->sys + q;
    PassArgs<C> args[N2D_VIE_PASSES];
    int mode[N2D_VIE_PASSES], L[N2D_VIE_PASSES], var[N2D_VIE_PASSES];
    size_t smem[N2D_VIE_PASSES];
    long long tiles[N2D_VIE_PASSES];
    const int precondition = set == 0;
    double *norm = set == 0 && !b->any_hybrid ? &s->before_sq : nullptr;
    int *flag = set == 0 ? &s->flag : set == 1 ? &s->rflag : nullptr;
    if (!n2c_vie_pass_plans<C>(b->plans[q], precondition, norm, flag, b->scale, b->variant, args, mode, L, var, smem,
                               tiles))
      return 0;
    for (int i = 0; i < N2D_VIE_PASSES; ++i) {
      args[i].gate = set == 0 ? &s->active : set == 1 ? &s->running : nullptr;
      desc[i][q].a = args[i];
      desc[i][q].off = b->off[q] + b->cond[q];
      desc[i][q].L = L[i];
      desc[i][q].variant = var[i];
      first[i][q + 1] = first[i][q] + tiles[i];
      PassSet &ps = b->sets[set][i];
      ps.mode = mode[i];
      ps.smem = std::max(ps.smem, smem[i]);
    }
  }
  for (int i = 0; i < N2D_VIE_PASSES; ++i) {
    PassSet &ps = b->sets[set][i];
    ps.fp32 = sizeof(C) == sizeof(float2);
    ps.tiles = first[i][K];
    if (ps.tiles > 0x7fffffffLL) { n2c_set_error("batch pass grid too large"); return 0; }
    ps.desc = n2d_alloc(K * sizeof(BatchDesc<C>));
    ps.first = (long long *)n2d_alloc((K + 1) * sizeof(long long));
    if (!ps.desc || !ps.first || !n2d_upload(ps.desc, desc[i].data(), K * sizeof(BatchDesc<C>)) ||
        !n2d_upload(ps.first, first[i].data(), (K + 1) * sizeof(long long)))
      return 0;
  }
  return 1;
}

template <typename C>
static int launch_set_t(const n2d_vie_batch *b, const PassSet &ps, const double2 *x, double2 *y) {
  auto k = batch_kernel<C>(ps.mode);
  static std::atomic<bool> configured[9];   // per mode, set by the first launching thread
  if (!configured[ps.mode].load(std::memory_order_acquire)) {
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess ||
        cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess) {
      n2c_set_error("cannot raise shared memory for the batched FFT pass");
      return 0;
    }
    configured[ps.mode].store(true, std::memory_order_release);
  }
  // Programmatic dependent launch, as for the single-plan passes
  // (NEC2C_CUDA_PDL=0 turns it off).
  static const bool pdl = [] {
    const char *v = getenv("NEC2C_CUDA_PDL");
    return !(v && v[0] == '0');
  }();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)ps.tiles);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = ps.smem;
  cfg.stream = n2c_stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k, (const BatchDesc<C> *)ps.desc, (const long long *)ps.first,
                                           b->K, x, y);
  if (e != cudaSuccess) {
    n2c_set_error("batched fft pass launch: %s", cudaGetErrorString(e));
    return 0;
  }
  return n2c_check_launch("batched fft pass");
}

static BView view_of(const n2d_vie_batch *b);

// y = A x over the whole batch with descriptor set `set`: the volume passes,
// then the conductor and cross rows of the hybrid systems (and, for the
// Arnoldi set, the norm of w, which the volume epilogue cannot take there).
static int batch_apply(const n2d_vie_batch *b, int set, const double2 *x, double2 *y) {
  for (int i = 0; i < N2D_VIE_PASSES; ++i) {
    const PassSet &ps = b->sets[set][i];
    const int ok = ps.fp32 ? launch_set_t<float2>(b, ps, x, y) : launch_set_t<double2>(b, ps, x, y);
    if (!ok) return 0;
  }
  if (!b->any_hybrid) return 1;
  const BView v = view_of(b);
  const long long cctas = b->crow[b->K], xctas = b->xrow[b->K];
  seg_zc_kernel<<<(unsigned)b->first_v[b->K], VEC_THREADS, 0, n2c_stream()>>>(v, b->hyb_dev, x, b->zbuf, set);
  if (cctas)
    seg_conductor_kernel<<<(unsigned)cctas, 256, 0, n2c_stream()>>>(v, b->hyb_dev, b->crow_dev, b->zbuf, y, set);
  if (xctas) seg_cross_kernel<<<(unsigned)xctas, 256, 0, n2c_stream()>>>(v, b->hyb_dev, b->xrow_dev, b->zbuf, y, set);
  if (!n2c_check_launch("batched conductor rows")) return 0;
  if (set == 0) {
    seg_wnorm_kernel<<<(unsigned)b->first_v[b->K], VEC_THREADS, 0, n2c_stream()>>>(v);
    if (!n2c_check_launch("batched norm of w")) return 0;
  }
  return 1;
}

// Batch tuner: per pass, the tile height scale (-1, 0, +1 of the batch
// height) and the radix split, timed on the plain products of this batch
// (CUDA events, best of two runs of three launches after a warm-up); a
// candidate replaces the incumbent only when it is at least 3% faster.
// Scale -1 is not tried for the z epilogue, whose norm reduction must keep
// within 65,536 tiles per plan.
static int tune_batch(n2d_vie_batch *b) {
  double2 *x = (double2 *)n2d_alloc(b->N * sizeof(double2)), *y = (double2 *)n2d_alloc(b->N * sizeof(double2));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int ok = x && y && n2d_memset(x, 0, b->N * sizeof(double2)) && cudaEventCreate(&e0) == cudaSuccess &&
           cudaEventCreate(&e1) == cudaSuccess;
  auto rebuild = [&]() {
    free_set(b, 2);
    return b->fp32 ? build_set<float2>(b, 2) : build_set<double2>(b, 2);
  };
  auto time_pass = [&](int i) -> float {
    const PassSet &ps = b->sets[2][i];
    auto launch = [&]() { return ps.fp32 ? launch_set_t<float2>(b, ps, x, y) : launch_set_t<double2>(b, ps, x, y); };
    if (!launch()) return -1.0f;
    float best = -1.0f;
    for (int trial = 0; trial < 2; ++trial) {
      if (cudaEventRecord(e0, n2c_stream()) != cudaSuccess) return -1.0f;
      for (int r = 0; r < 3; ++r)
        if (!launch()) return -1.0f;
      float ms = 0;
      if (cudaEventRecord(e1, n2c_stream()) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
        return -1.0f;
      if (best < 0 || ms < best) best = ms;
    }
    return best;
  };
  for (int i = 0; i < N2D_VIE_PASSES && ok; ++i) {
    float bt = time_pass(i);
    if (bt < 0) { ok = 0; break; }
    const int cand[5][2] = {{-1, 0}, {1, 0}, {0, 1}, {-1, 1}, {1, 1}};
    int best_s = 0, best_v = 0;
    for (const auto &c : cand) {
      if (i == 4 && c[0] < 0) continue;
      b->scale[i] = c[0];
      b->variant[i] = c[1];
      if (!rebuild()) { ok = 0; break; }
      const float t = time_pass(i);
      if (t >= 0 && t < 0.97f * bt) { bt = t; best_s = c[0]; best_v = c[1]; }
    }
    b->scale[i] = best_s;
    b->variant[i] = best_v;
    if (ok) ok = rebuild();
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaGetLastError();
  n2d_free(x);
  n2d_free(y);
  return ok;
}

static int batch_create(n2d_vie_batch **out, n2d_vie *const *plans, n2d_hybrid *const *hybrids,
                        long long count) {
  *out = nullptr;
  if (count < 1 || count > (1 << 20)) { n2c_set_error("batch of %lld systems", count); return 0; }
  n2d_vie_batch *b = new n2d_vie_batch();
  b->K = (int)count;
  b->off.assign(count + 1, 0);
  b->first_d.assign(count + 1, 0);
  b->first_v.assign(count + 1, 0);
  b->crow.assign(count + 1, 0);
  b->xrow.assign(count + 1, 0);
  std::vector<const double2 *> diag(count);
  std::vector<BHyb> hyb(count);
  for (long long q = 0; q < count; ++q) {
    n2d_hybrid *h = hybrids ? hybrids[q] : nullptr;
    n2d_vie *p = h ? n2c_hybrid_volume(h) : plans[q];
    if (!p || p->cells < 1) { n2c_set_error("batch system %lld has no volume cells", q); delete b; return 0; }
    if (q == 0) b->fp32 = n2d_vie_fp32(p);
    if (n2d_vie_fp32(p) != b->fp32) {
      n2c_set_error("batch plans mix FP32 and FP64 transforms");
      delete b;
      return 0;
    }
    for (int d = 0; d < 3; ++d)
      if (p->P[d] > MAX_L) {
        n2c_set_error("batch system %lld: padded axis %lld exceeds %d", q, p->P[d], MAX_L);
        delete b;
        return 0;
      }
    for (long long r = 0; r < q; ++r)
      if (b->plans[r] == p) { n2c_set_error("plan of system %lld appears twice in the batch", q); delete b; return 0; }
    const long long nv = 3 * (p->mirror ? p->mirror : p->cells);
    const long long c = h ? n2c_hybrid_conductors(h) : 0;
    if (h && n2d_hybrid_order(h) != c + nv) {
      n2c_set_error("batch system %lld: hybrid order does not match its plan", q);
      delete b;
      return 0;
    }
    const long long n = c + nv;
    b->plans.push_back(p);
    b->hybrids.push_back(h);
    b->cond.push_back(c);
    b->any_hybrid = b->any_hybrid || c > 0;
    b->off[q + 1] = b->off[q] + n;
    b->first_d[q + 1] = b->first_d[q] + (n + DOT_RANGE - 1) / DOT_RANGE;
    b->first_v[q + 1] = b->first_v[q] + (n + VEC_RANGE - 1) / VEC_RANGE;
    b->crow[q + 1] = b->crow[q] + (c + COND_ROWS - 1) / COND_ROWS;
    b->xrow[q + 1] = b->xrow[q] + (c ? (nv + cross_rows_per_cta(c) - 1) / cross_rows_per_cta(c) : 0);
    diag[q] = h ? n2c_hybrid_pdiag(h) : (const double2 *)n2d_vie_diag(p);
    hyb[q] = BHyb{h ? n2c_hybrid_blocks(h) : nullptr, c, n};
  }
  b->N = b->off[count];
  if (b->first_v[count] > 0x7fffffffLL || b->crow[count] > 0x7fffffffLL || b->xrow[count] > 0x7fffffffLL) {
    n2c_set_error("batch too large");
    delete b;
    return 0;
  }
  b->off_dev = (long long *)n2d_alloc((count + 1) * sizeof(long long));
  b->first_d_dev = (long long *)n2d_alloc((count + 1) * sizeof(long long));
  b->first_v_dev = (long long *)n2d_alloc((count + 1) * sizeof(long long));
  b->crow_dev = (long long *)n2d_alloc((count + 1) * sizeof(long long));
  b->xrow_dev = (long long *)n2d_alloc((count + 1) * sizeof(long long));
  b->hyb_dev = (BHyb *)n2d_alloc(count * sizeof(BHyb));
  if (b->any_hybrid) b->zbuf = (double2 *)n2d_alloc(b->N * sizeof(double2));
  b->sys = (BSys *)n2d_alloc(count * sizeof(BSys));
  b->diag_dev = (const double2 **)n2d_alloc(count * sizeof(double2 *));
  int ok = b->off_dev && b->first_d_dev && b->first_v_dev && b->crow_dev && b->xrow_dev && b->hyb_dev && b->sys &&
           (b->zbuf || !b->any_hybrid) &&
           b->diag_dev && n2d_upload(b->off_dev, b->off.data(), (count + 1) * sizeof(long long)) &&
           n2d_upload(b->first_d_dev, b->first_d.data(), (count + 1) * sizeof(long long)) &&
           n2d_upload(b->first_v_dev, b->first_v.data(), (count + 1) * sizeof(long long)) &&
           n2d_upload(b->crow_dev, b->crow.data(), (count + 1) * sizeof(long long)) &&
           n2d_upload(b->xrow_dev, b->xrow.data(), (count + 1) * sizeof(long long)) &&
           n2d_upload(b->hyb_dev, hyb.data(), count * sizeof(BHyb)) &&
           n2d_upload((void *)b->diag_dev, diag.data(), count * sizeof(double2 *)) &&
           n2d_memset(b->sys, 0, count * sizeof(BSys));
  if (ok) ok = b->fp32 ? build_set<float2>(b, 2) : build_set<double2>(b, 2);
  if (ok && n2d_vie_autotune_enabled()) ok = tune_batch(b);
  if (ok) ok = b->fp32 ? build_set<float2>(b, 0) : build_set<double2>(b, 0);
  if (ok) ok = build_set<double2>(b, 1);
  if (!ok || !n2d_sync()) { n2d_vie_batch_destroy(b); return 0; }
  *out = b;
  return 1;
}

extern "C" int n2d_vie_batch_create(n2d_vie_batch **out, n2d_vie *const *plans, long long count) {
  return batch_create(out, plans, nullptr, count);
}

extern "C" int n2d_hybrid_batch_create(n2d_vie_batch **out, n2d_hybrid *const *systems, long long count) {
  return batch_create(out, nullptr, systems, count);
}

// Schedule of the batched passes: tile height scale and radix split per pass.
extern "C" void n2d_vie_batch_schedule(const n2d_vie_batch *b, int *scale, int *variant) {
  for (int i = 0; i < N2D_VIE_PASSES; ++i) {
    scale[i] = b->scale[i];
    variant[i] = b->variant[i];
  }
}

// Pins the schedule (scale in -1..1, variant 0 or 1 per pass) and rebuilds the
// descriptor sets; the batch is left as it was when a set cannot be built.
extern "C" int n2d_vie_batch_set_schedule(n2d_vie_batch *b, const int *scale, const int *variant) {
  int old_s[N2D_VIE_PASSES], old_v[N2D_VIE_PASSES];
  for (int i = 0; i < N2D_VIE_PASSES; ++i) {
    if (scale[i] < -1 || scale[i] > 1 || variant[i] < 0 || variant[i] > 1) {
      n2c_set_error("batch schedule of pass %d out of range", i);
      return 0;
    }
    old_s[i] = b->scale[i];
    old_v[i] = b->variant[i];
  }
  auto build_all = [&]() {
    for (int set = 0; set < 3; ++set) free_set(b, set);
    return (b->fp32 ? build_set<float2>(b, 0) : build_set<double2>(b, 0)) && build_set<double2>(b, 1) &&
           (b->fp32 ? build_set<float2>(b, 2) : build_set<double2>(b, 2));
  };
  for (int i = 0; i < N2D_VIE_PASSES; ++i) {
    b->scale[i] = scale[i];
    b->variant[i] = variant[i];
  }
  // Captured cycles bake the tile grids into their launches.
  work_free(b->work);
  b->work = nullptr;
  if (build_all()) return 1;
  for (int i = 0; i < N2D_VIE_PASSES; ++i) {
    b->scale[i] = old_s[i];
    b->variant[i] = old_v[i];
  }
  build_all();
  return 0;
}

extern "C" long long n2d_vie_batch_order(const n2d_vie_batch *b) { return b ? b->N : 0; }
extern "C" long long n2d_vie_batch_offset(const n2d_vie_batch *b, long long q) {
  return b && q >= 0 && q <= b->K ? b->off[q] : -1;
}

extern "C" int n2d_vie_batch_apply(n2d_vie_batch *b, const double *x_dev, double *y_dev) {
  return batch_apply(b, 2, (const double2 *)x_dev, (double2 *)y_dev);
}

// The kernels' view of the batch: its systems and, once a solve has run, the
// GMRES workspace (the products of batch_apply touch only sys, off, the
// maps and the Jacobi divisors, plus parts_v for the norm of w).
static BView view_of(const n2d_vie_batch *b) {
  if (b->work) return b->work->v;
  BView v;
  memset(&v, 0, sizeof(v));
  v.sys = b->sys; v.off = b->off_dev; v.first_d = b->first_d_dev; v.first_v = b->first_v_dev;
  v.K = b->K; v.N = b->N; v.diag = b->diag_dev;
  return v;
}

static BatchWork *work_get(n2d_vie_batch *b, int m) {
  if (b->work && b->work->m == m) return b->work;
  work_free(b->work);
  b->work = nullptr;
  BatchWork *w = new BatchWork();
  w->m = m;
  BView &v = w->v;
  memset(&v, 0, sizeof(v));
  const long long N = b->N, K = b->K;
  v.sys = b->sys; v.off = b->off_dev; v.first_d = b->first_d_dev; v.first_v = b->first_v_dev;
  v.K = b->K; v.m = m; v.N = N; v.diag = b->diag_dev; v.always_reorth = !b->fp32;
  v.V = (double2 *)n2d_alloc((size_t)(m + 1) * N * sizeof(double2));
  v.w = (double2 *)n2d_alloc(N * sizeof(double2));
  v.r = (double2 *)n2d_alloc(N * sizeof(double2));
  v.H = (double2 *)n2d_alloc(K * (m + 1) * m * sizeof(double2));
  v.g = (double2 *)n2d_alloc(K * (m + 1) * sizeof(double2));
  v.sn = (double2 *)n2d_alloc(K * m * sizeof(double2));
  v.y = (double2 *)n2d_alloc(K * m * sizeof(double2));
  v.hp = (double2 *)n2d_alloc(K * 2 * BMAXM * sizeof(double2));
  v.cs = (double *)n2d_alloc(K * m * sizeof(double));
  v.parts_d = (double2 *)n2d_alloc(b->first_d[K] * BMAXM * sizeof(double2));
  v.parts_v = (double *)n2d_alloc(b->first_v[K] * sizeof(double));
  v.norms = (double *)n2d_alloc(2 * K * sizeof(double));
  w->active_count = (int *)n2d_alloc(sizeof(int));
  if (!v.V || !v.w || !v.r || !v.H || !v.g || !v.sn || !v.y || !v.hp || !v.cs || !v.parts_d || !v.parts_v ||
      !v.norms || !w->active_count) {
    work_free(w);
    return nullptr;
  }
  b->work = w;
  return w;
}

// Steps [j0, j1) of a cycle, gated per system, then the count of systems
// still in the cycle, on the current stream.
static int enqueue_steps(n2d_vie_batch *b, BatchWork *w, int j0, int j1) {
  BView &v = w->v;
  const unsigned nd = (unsigned)b->first_d[b->K], nv = (unsigned)b->first_v[b->K];
  for (int j = j0; j < j1; ++j) {
    if (!batch_apply(b, 0, v.V + (long long)j * v.N, v.w)) return 0;
    seg_dots_kernel<0><<<nd, 1024, DOT_SMEM, n2c_stream()>>>(v, j);
    seg_update_kernel<0><<<nv, VEC_THREADS, 0, n2c_stream()>>>(v, j);
    seg_dots_kernel<1><<<nd, 1024, DOT_SMEM, n2c_stream()>>>(v, j);
    seg_update_kernel<1><<<nv, VEC_THREADS, 0, n2c_stream()>>>(v, j);
    seg_normalize_kernel<<<nv, VEC_THREADS, 0, n2c_stream()>>>(v, j);
    if (!n2c_check_launch("batched Gram-Schmidt")) return 0;
    n2c_count_launch(4);
  }
  count_active_kernel<<<1, 256, 0, n2c_stream()>>>(v, w->active_count);
  return n2c_check_launch("active count");
}

// Captures each chunk of steps once into a graph (launched on the caller's
// stream); a chunk that cannot be captured is launched directly.
static void try_capture(n2d_vie_batch *b, BatchWork *w) {
  w->tried_graph = true;
  static thread_local cudaStream_t cap = nullptr;
  if (!cap && cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) { cap = nullptr; return; }
  void *user = n2d_get_stream();
  for (int c = 0; c * CHUNK < w->m; ++c) {
    const unsigned long long before = n2d_launch_count();
    n2d_set_stream(cap);
    cudaGraph_t graph = nullptr;
    int ok = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) ok = enqueue_steps(b, w, c * CHUNK, std::min(w->m, (c + 1) * CHUNK));
    const cudaError_t e = cudaStreamEndCapture(cap, &graph);
    n2d_set_stream(user);
    if (ok && e == cudaSuccess && graph && cudaGraphInstantiate(&w->chunk[c], graph, 0) == cudaSuccess)
      w->chunk_launches[c] = (unsigned)(n2d_launch_count() - before);
    else
      w->chunk[c] = nullptr;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
  }
}

extern "C" int n2d_gmres_batch_dev(n2d_vie_batch *b, const double *b_dev, double *x_dev, size_t restart,
                                   size_t maxit, double rtol, double atol, const unsigned char *idle,
                                   n2d_gmres_report *reps) {
  const int K = b->K;
  for (int q = 0; q < K; ++q) {
    memset(&reps[q], 0, sizeof(reps[q]));
    reps[q].status = ST_INVALID;
    reps[q].residual_norm = reps[q].relative_residual = INFINITY;
  }
  if (restart < 1 || maxit < 1) return 0;
  const int m = (int)std::min<size_t>(std::min<size_t>(restart, maxit), BMAXM);
  if (restart > (size_t)BMAXM && maxit > (size_t)BMAXM) {
    n2c_set_error("batched GMRES restarts after at most %d steps", BMAXM);
    return 0;
  }
  static const bool configured = [] {
    cudaFuncSetAttribute(seg_dots_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DOT_SMEM);
    cudaFuncSetAttribute(seg_dots_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DOT_SMEM);
    return true;
  }();
  (void)configured;
  BatchWork *w = work_get(b, m);
  if (!w) {
    for (int q = 0; q < K; ++q) reps[q].status = ST_ALLOC;
    return 0;
  }
  BView &v = w->v;
  const double2 *rhs = (const double2 *)b_dev;
  double2 *x = (double2 *)x_dev;
  const unsigned nv = (unsigned)b->first_v[K];
  std::vector<BSys> hs(K);
  std::vector<double> bnorm(K), target(K), norms(2 * K);
  std::vector<char> done(K, 0);
  auto put = [&]() { return n2d_upload(b->sys, hs.data(), K * sizeof(BSys)); };
  auto get = [&]() { return n2d_download(hs.data(), b->sys, K * sizeof(BSys)); };
  auto norms_of = [&](const double2 *vec, double *outh) {
    seg_norm_kernel<<<nv, VEC_THREADS, 0, n2c_stream()>>>(v, vec, v.norms);
    return n2c_check_launch("batched norm") && n2d_download(outh, v.norms, K * sizeof(double));
  };
  memset(hs.data(), 0, K * sizeof(BSys));
  for (int q = 0; q < K; ++q) {
    const long long n = b->off[q + 1] - b->off[q];
    hs[q].status = ST_RUNNING;
    hs[q].max_iterations = (long long)maxit;
    hs[q].m = (int)std::min<long long>(m, n);
    // An idle system takes no part: it is done from the start, never
    // active or running, so its tiles leave at their gates.
    if (idle && idle[q]) { done[q] = 1; hs[q].status = ST_INVALID; }
  }
  // ||b|| and ||x|| (finite check) of every system (vie_iterative.c:116-119).
  if (!put() || !norms_of(rhs, norms.data()) || !norms_of(x, norms.data() + K) || !get()) return 0;
  for (int q = 0; q < K; ++q) {
    if (done[q]) continue;
    bnorm[q] = sqrt(norms[q]);
    target[q] = fmax(atol, rtol * bnorm[q]);
    hs[q].target = target[q];
    if (hs[q].rflag || !isfinite(bnorm[q]) || !isfinite(sqrt(norms[K + q])) || !isfinite(target[q])) {
      reps[q].status = ST_NONFINITE;
      hs[q].status = ST_NONFINITE;
      done[q] = 1;
    }
  }
  // True residual r = b - A x (FP64) of the systems still running.
  auto true_residual = [&]() -> int {
    for (int q = 0; q < K; ++q) {
      hs[q].running = !done[q];
      hs[q].rflag = 0;
      hs[q].active = 0;
      if (!done[q]) ++reps[q].operator_applications;
    }
    if (!put() || !batch_apply(b, 1, x, v.r)) return 0;
    seg_residual_kernel<<<nv, VEC_THREADS, 0, n2c_stream()>>>(v, rhs);
    if (!n2c_check_launch("batched residual") || !norms_of(v.r, norms.data()) || !get()) return 0;
    for (int q = 0; q < K; ++q) {
      if (done[q]) continue;
      reps[q].residual_norm = hs[q].rflag ? NAN : sqrt(norms[q]);
      reps[q].relative_residual = bnorm[q] > 0 ? reps[q].residual_norm / bnorm[q] : reps[q].residual_norm;
      if (!isfinite(reps[q].residual_norm)) { reps[q].status = ST_NONFINITE; done[q] = 1; }
    }
    return 1;
  };
  if (!true_residual()) return 0;
  for (;;) {
    int cycling = 0;
    for (int q = 0; q < K; ++q) {
      hs[q].active = 0;
      if (done[q]) continue;
      const double beta = reps[q].residual_norm;
      if (beta <= target[q]) { reps[q].status = ST_CONVERGED; done[q] = 1; continue; }
      if ((long long)reps[q].iterations >= (long long)maxit) { reps[q].status = ST_LIMIT; done[q] = 1; continue; }
      // A hybrid system with a zero or non-finite conductor diagonal cannot be
      // preconditioned (dielectric_fft.c:77-81): it stops as the single
      // system's solve does.
      if (b->hybrids[q] && !n2c_hybrid_precondition_ok(b->hybrids[q])) {
        reps[q].status = ST_CALLBACK;
        done[q] = 1;
        continue;
      }
      hs[q].active = 1; hs[q].beta = beta; hs[q].used = 0; hs[q].breakdown = 0; hs[q].flag = 0;
      hs[q].normalize = 0; hs[q].reorth = 0; hs[q].status = ST_RUNNING;
      hs[q].iterations = (long long)reps[q].iterations;
      ++cycling;
    }
    if (!cycling) break;
    for (int q = 0; q < K; ++q) if (done[q]) hs[q].status = reps[q].status;
    if (!put()) return 0;
    seg_cycle_start_kernel<<<nv, VEC_THREADS, 0, n2c_stream()>>>(v);
    if (!n2c_check_launch("batched cycle start")) return 0;
    if (!w->tried_graph) try_capture(b, w);
    for (int c = 0; c * CHUNK < w->m; ++c) {
      if (w->chunk[c]) {
        if (cudaGraphLaunch(w->chunk[c], (cudaStream_t)n2d_get_stream()) != cudaSuccess) {
          n2c_set_error("batched GMRES graph launch failed");
          return 0;
        }
        n2c_count_launch(w->chunk_launches[c]);
      } else if (!enqueue_steps(b, w, c * CHUNK, std::min(w->m, (c + 1) * CHUNK))) {
        return 0;
      }
      int still = 0;
      if (!n2d_download(&still, w->active_count, sizeof(int))) return 0;
      if (!still) break;
    }
    seg_backsolve_kernel<<<(K + 3) / 4, 128, 0, n2c_stream()>>>(v);
    seg_xupdate_kernel<<<nv, VEC_THREADS, 0, n2c_stream()>>>(v, x);
    if (!n2c_check_launch("batched solution update") || !get()) return 0;
    std::vector<char> cycled(K, 0);
    for (int q = 0; q < K; ++q) {
      if (done[q]) continue;
      cycled[q] = 1;
      reps[q].iterations = (size_t)hs[q].iterations;
      reps[q].operator_applications += (size_t)hs[q].used;
      if (hs[q].status != ST_RUNNING) { reps[q].status = hs[q].status; done[q] = 1; }
    }
    if (!true_residual()) return 0;
    for (int q = 0; q < K; ++q) {
      if (!cycled[q] || done[q]) continue;
      const double rn = reps[q].residual_norm;
      if (hs[q].breakdown && rn > target[q]) { reps[q].status = ST_BREAKDOWN; done[q] = 1; continue; }
      if (rn > target[q] && (long long)reps[q].iterations < (long long)maxit) ++reps[q].restarts;
    }
  }
  int all = 1;
  for (int q = 0; q < K; ++q) all = all && ((idle && idle[q]) || reps[q].status == ST_CONVERGED);
  return all;
}

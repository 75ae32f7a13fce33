// Device-resident restarted GMRES(m) for the volume plan and the hybrid
// system: vie_iterative.c:80-199 (vie_gmres) with the operator, the two-pass
// modified Gram-Schmidt, the Givens least squares and the true residual all on
// the device.  The host reads a small state block once per restart cycle.
//
// Per inner iteration j the host enqueues: the preconditioned matvec
// w = A D^-1 v_j (with ||w||), then one cooperative kernel that runs both MGS
// passes over v_0..v_j with w held in registers, the norm, the Givens update
// and v_{j+1} = w/||w||.  Every kernel first checks the device "active" flag,
// so iterations after convergence cost only a launch.  x += D^-1 (V y) and
// the true residual close the cycle.  Reductions are deterministic (fixed-order
// block partials), so results are bitwise reproducible run to run.
#include <stdlib.h>
#include <float.h>
#include <math.h>
#include <string.h>
#include "common.cuh"
#include "device_api.h"
#include "runtime.cuh"
#include "vie_internal.cuh"

using namespace n2c;

struct n2d_hybrid;
int n2c_hybrid_precondition_ok(const n2d_hybrid *h);
const double2 *n2c_hybrid_pdiag(const n2d_hybrid *h);
int n2c_norm2(const double *y, long long n, double *partials, unsigned int *ticket, double *out,
              int *flag);

enum { ST_CONVERGED, ST_LIMIT, ST_BREAKDOWN, ST_CALLBACK, ST_INVALID, ST_ALLOC, ST_NONFINITE };
enum { ST_RUNNING = -1 };

struct GmState {
  int active;          // inner loop of the current cycle still running
  int status;          // ST_RUNNING or a final status
  int breakdown;
  int used;            // inner iterations done in the current cycle
  int flag;            // non-finite raised by a kernel
  int barrier_error;   // grid barrier gave up (never expected under cooperative launch)
  long long iterations, max_iterations;
  double target, before_sq, residual_sq, after;
  int normalize;       // CGS step produced v_{j+1}
  int reorth;          // CGS: second pass requested for the current column
  long long reorth_count;
  unsigned int bar_count, bar_gen;
};

// Scratch layout of GmBuffers::partials (doubles): [0, 4096) norm partials,
// [4096, 4096 + 2*1024*32) per-block partials of the Arnoldi kernels, then a
// few device scalars.
constexpr long long PART_BLOCKS = 4096;
constexpr long long PART_SCALARS = 4096 + 2 * 1024 * 32;
constexpr long long PART_TOTAL = PART_SCALARS + 64;

struct GmBuffers {
  GmState *st;
  double2 *H, *g, *sn, *y;   // (m+1) x m Hessenberg (row-major), rotations, solution
  double *cs;
  double2 *V, *w, *r, *tmp;  // basis (m+1) x n, work vectors
  double2 *cgs_h;            // 2 x MAXM: CGS2 pass coefficients
  double *partials;          // 2 x grid partials
  unsigned int *ticket;
};

// ---------------------------------------------------------- grid barrier
// Sense-by-generation barrier for a cooperative launch.  The spin is bounded
// (clock budget); on time-out the barrier records an error and every block
// leaves at its next barrier, so the kernel always ends.
__device__ __forceinline__ bool grid_barrier(GmState *st) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned int *gen = &st->bar_gen;
    volatile int *err = &st->barrier_error;
    if (*err) ok = 0;
    else {
      const unsigned int g = *gen;
      __threadfence();
      if (atomicAdd(&st->bar_count, 1u) == gridDim.x - 1) {
        st->bar_count = 0;
        __threadfence();
        atomicAdd(&st->bar_gen, 1u);
      } else {
        const long long t0 = clock64();
        while (*gen == g) {
          if (*err || clock64() - t0 > (1LL << 32)) { atomicExch(&st->barrier_error, 1); ok = 0; break; }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
  }
  __syncthreads();
  return ok != 0;
}

// Fixed-order sum of the grid's block partials (same value in every block).
__device__ __forceinline__ double2 sum_partials(const double2 *partials) {
  double2 t = make_double2(0, 0);
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) t = cadd(t, partials[i]);
  return block_sum(t);
}

__device__ __forceinline__ double cabs_(double2 a) { return hypot(a.x, a.y); }

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

// Both MGS passes, the norm, the Givens update and v_{j+1} for iteration j.
// E = complex elements of w held per thread.
template <int E>
__global__ void __launch_bounds__(512) arnoldi_kernel(GmBuffers b, long long n, int m, int j) {
  GmState *st = b.st;
  if (!st->active) return;
  if (st->flag) {
    if (blockIdx.x == 0 && threadIdx.x == 0) { st->status = ST_NONFINITE; st->active = 0; }
    return;
  }
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long base = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double2 w[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const long long i = base + e * stride;
    w[e] = i < n ? b.w[i] : make_double2(0, 0);
  }
  double2 *part[2] = {(double2 *)(b.partials + PART_BLOCKS), (double2 *)(b.partials + PART_BLOCKS) + gridDim.x};
  int buf = 0;
  // vk holds the basis vector of the current step; vn prefetches the next one
  // while the block waits at the grid barrier.
  double2 vk[E], vn[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const long long i = base + e * stride;
    vk[e] = i < n ? b.V[i] : make_double2(0, 0);
  }
  const int steps = 2 * (j + 1);
  for (int s = 0; s < steps; ++s) {
    const int k = s % (j + 1);
    double2 acc = make_double2(0, 0);
#pragma unroll
    for (int e = 0; e < E; ++e) acc = cadd(acc, cconjmul(vk[e], w[e]));
    acc = block_sum(acc);
    if (threadIdx.x == 0) part[buf][blockIdx.x] = acc;
    const int kn = (s + 1) % (j + 1);
    if (E <= 8 && s + 1 < steps) {
      const double2 *vnext = b.V + (long long)kn * n;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const long long i = base + e * stride;
        vn[e] = i < n ? vnext[i] : make_double2(0, 0);
      }
    }
    if (!grid_barrier(st)) return;
    const double2 proj = sum_partials(part[buf]);
    buf ^= 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) b.H[(long long)k * m + j] = cadd(b.H[(long long)k * m + j], proj);
#pragma unroll
    for (int e = 0; e < E; ++e) w[e] = csub(w[e], cmul(proj, vk[e]));
    if (E <= 8) {
#pragma unroll
      for (int e = 0; e < E; ++e) vk[e] = vn[e];
    } else if (s + 1 < steps) {
      const double2 *vnext = b.V + (long long)kn * n;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const long long i = base + e * stride;
        vk[e] = i < n ? vnext[i] : make_double2(0, 0);
      }
    }
  }
  double sq = 0;
#pragma unroll
  for (int e = 0; e < E; ++e) sq += w[e].x * w[e].x + w[e].y * w[e].y;
  double2 t = block_sum(make_double2(sq, 0));
  if (threadIdx.x == 0) part[buf][blockIdx.x] = t;
  if (!grid_barrier(st)) return;
  const double after = sqrt(sum_partials(part[buf]).x);
  const double before = sqrt(st->before_sq);
  const bool broke = after <= 32 * DBL_EPSILON * before;
  if (isfinite(after) && !broke) {
    double2 *vn = b.V + (long long)(j + 1) * n;
    const double inv = after;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const long long i = base + e * stride;
      if (i < n) vn[i] = make_double2(w[e].x / inv, w[e].y / inv);
    }
  }
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (!isfinite(after)) { st->status = ST_NONFINITE; st->active = 0; return; }
  double2 *H = b.H;
  H[(long long)(j + 1) * m + j] = make_double2(after, 0);
  for (int k = 0; k < j; ++k) {
    const double2 h0 = H[(long long)k * m + j], h1 = H[(long long)(k + 1) * m + j];
    const double2 s = b.sn[k];
    H[(long long)k * m + j] = cadd(cscale(h0, b.cs[k]), cmul(s, h1));
    H[(long long)(k + 1) * m + j] = csub(cscale(h1, b.cs[k]), cconjmul(s, h0));
  }
  double c;
  double2 s;
  givens(H[(long long)j * m + j], H[(long long)(j + 1) * m + j], &c, &s);
  b.cs[j] = c; b.sn[j] = s;
  H[(long long)j * m + j] = cadd(cscale(H[(long long)j * m + j], c), cmul(s, H[(long long)(j + 1) * m + j]));
  H[(long long)(j + 1) * m + j] = make_double2(0, 0);
  const double2 gj = b.g[j];
  b.g[j + 1] = make_double2(-(s.x * gj.x + s.y * gj.y), -(s.x * gj.y - s.y * gj.x));  // -conj(s) g_j
  b.g[j] = cscale(gj, c);
  st->iterations += 1;
  st->used = j + 1;
  st->breakdown = broke;
  if (broke || cabs_(b.g[j + 1]) <= st->target || j + 1 >= m || st->iterations >= st->max_iterations)
    st->active = 0;
}

// ---------------------------------------------------------------- CGS
// Classical Gram-Schmidt with selective reorthogonalisation (mixed form):
//   dots   h = V^H w                          (warp per basis vector)
//   update w -= V h, ||w||^2                   (thread per element)
// and a second dots/update pass only when the projection cancelled more than
// a factor REORTH of the norm (||w_new|| < ||w|| / REORTH).  One CGS pass
// loses orthogonality by about eps (||w|| / ||w_new||)^2, so the basis stays
// orthogonal to ~100 eps per vector; GMRES here needs far less (the restart
// test is an FP64 true residual, so lost orthogonality could only cost
// iterations, not accuracy), and the 1/sqrt(2) threshold of the
// Daniel-Gragg-Kaufman-Stewart criterion would rerun the pass on nearly every
// Arnoldi step.  Both passes add into the Hessenberg column, as the two MGS
// passes of vie_iterative.c do.  Kernel boundaries are the only grid synchronisation; reductions are
// fixed-order block partials finished by the last block (deterministic).
constexpr int MAXM = 30;   // restarts up to MAXM use this path
constexpr int CGS_E = 4;   // elements per lane in the dots kernel
constexpr double REORTH = 10.0;   // cancellation factor that triggers the second pass
constexpr int CGS_GROUP = 32 * CGS_E;   // elements per warp group

// Hessenberg column j finished with h_{j+1,j} = after: previous rotations,
// the new rotation, the residual estimate and the cycle's stop conditions
// (vie_iterative.c:160-177).
__device__ void finish_step(GmBuffers &b, GmState *st, int m, int j, double after) {
  const double before = sqrt(st->before_sq);
  const bool broke = after <= 32 * DBL_EPSILON * before;
  st->after = after;
  st->reorth = 0;
  if (!isfinite(after)) { st->status = ST_NONFINITE; st->active = 0; return; }
  double2 *H = b.H;
  H[(long long)(j + 1) * m + j] = make_double2(after, 0);
  for (int q = 0; q < j; ++q) {
    const double2 h0 = H[(long long)q * m + j], h1 = H[(long long)(q + 1) * m + j];
    const double2 s = b.sn[q];
    H[(long long)q * m + j] = cadd(cscale(h0, b.cs[q]), cmul(s, h1));
    H[(long long)(q + 1) * m + j] = csub(cscale(h1, b.cs[q]), cconjmul(s, h0));
  }
  double c;
  double2 s;
  givens(H[(long long)j * m + j], H[(long long)(j + 1) * m + j], &c, &s);
  b.cs[j] = c; b.sn[j] = s;
  H[(long long)j * m + j] = cadd(cscale(H[(long long)j * m + j], c), cmul(s, H[(long long)(j + 1) * m + j]));
  H[(long long)(j + 1) * m + j] = make_double2(0, 0);
  const double2 gj = b.g[j];
  b.g[j + 1] = make_double2(-(s.x * gj.x + s.y * gj.y), -(s.x * gj.y - s.y * gj.x));
  b.g[j] = cscale(gj, c);
  st->iterations += 1;
  st->used = j + 1;
  st->breakdown = broke;
  st->normalize = !broke;
  if (broke || cabs_(b.g[j + 1]) <= st->target || j + 1 >= m || st->iterations >= st->max_iterations)
    st->active = 0;
}

// h = V^H w for pass P (0: first, 1: reorthogonalisation, run only when
// requested).  Warp q of a 1024-thread block handles basis vector q % kk over
// element group q / kk, reading w directly (each vector's warp reads the same
// w values, so they come from L2 and L1).
template <int P>
__global__ void __launch_bounds__(1024) cgs_dots_kernel(GmBuffers b, long long n, int m, int j) {
  pdl_begin();
  GmState *st = b.st;
  if (!st->active || (P == 1 && !st->reorth)) return;
  if (P == 0 && st->flag) {
    if (blockIdx.x == 0 && threadIdx.x == 0) { st->status = ST_NONFINITE; st->active = 0; }
    return;
  }
  const int kk = j + 1;
  const int groups = 32 / kk;
  const int chunk = groups * CGS_GROUP;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k = warp % kk, grp = warp / kk;
  const bool active = grp < groups;
  double2 acc = make_double2(0, 0);
  const long long stride = (long long)gridDim.x * chunk;
  // Each active warp streams its vector's elements of the group with the
  // matching w values, read straight from global memory (w is read by every
  // vector's warp, so it is served from L2 and L1); the next chunk's loads are
  // issued before the current one is used.  No barrier inside the loop.
  double2 v[CGS_E], vn[CGS_E], wv[CGS_E], wn[CGS_E];
  auto load = [&](long long base, double2 (&vv)[CGS_E], double2 (&ww)[CGS_E]) {
    const double2 *vk = b.V + (long long)k * n;
#pragma unroll
    for (int e = 0; e < CGS_E; ++e) {
      const long long i = base + grp * CGS_GROUP + lane + 32 * e;
      vv[e] = i < n ? vk[i] : make_double2(0, 0);
      ww[e] = i < n ? b.w[i] : make_double2(0, 0);
    }
  };
  long long base = (long long)blockIdx.x * chunk;
  if (active && base < n) {
    load(base, v, wv);
    for (; base < n; base += stride) {
      if (base + stride < n) load(base + stride, vn, wn);
#pragma unroll
      for (int e = 0; e < CGS_E; ++e) acc = cadd(acc, cconjmul(v[e], wv[e]));
#pragma unroll
      for (int e = 0; e < CGS_E; ++e) { v[e] = vn[e]; wv[e] = wn[e]; }
    }
  }
  double2 *parts = (double2 *)(b.partials + PART_BLOCKS);
  __shared__ double2 red[32];
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
  }
  if (lane == 0) red[warp] = active ? acc : make_double2(0, 0);
  __syncthreads();
  if (threadIdx.x < kk) {
    double2 t = make_double2(0, 0);
    for (int g = 0; g < groups; ++g) t = cadd(t, red[g * kk + threadIdx.x]);
    parts[(long long)blockIdx.x * MAXM + threadIdx.x] = t;
  }
  if (!last_block_done(b.ticket)) return;
  // Last block: warp q sums slot q over the blocks in a fixed order.
  if (warp < kk) {
    double2 t = make_double2(0, 0);
    for (unsigned bl = lane; bl < gridDim.x; bl += 32) t = cadd(t, parts[(long long)bl * MAXM + warp]);
    for (int o = 16; o > 0; o >>= 1) {
      t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
      t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
    }
    if (lane == 0) {
      b.cgs_h[P * MAXM + warp] = t;
      b.H[(long long)warp * m + j] = cadd(b.H[(long long)warp * m + j], t);
    }
  }
  if (threadIdx.x == 0) *b.ticket = 0;
}

// w -= V h for pass P and ||w||^2 (thread per element); the last block
// either requests the reorthogonalisation pass or finishes the column.
template <int P>
__global__ void __launch_bounds__(256) cgs_update_kernel(GmBuffers b, long long n, int m, int j) {
  pdl_begin();
  GmState *st = b.st;
  if (!st->active || (P == 1 && !st->reorth)) return;
  const int kk = j + 1;
  __shared__ double2 hs[MAXM];
  if (threadIdx.x < kk) hs[threadIdx.x] = b.cgs_h[P * MAXM + threadIdx.x];
  __syncthreads();
  double sq = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double2 wi = b.w[i];
#pragma unroll 6
    for (int k = 0; k < kk; ++k) wi = csub(wi, cmul(hs[k], b.V[(long long)k * n + i]));
    b.w[i] = wi;
    sq += wi.x * wi.x + wi.y * wi.y;
  }
  const double2 t = block_sum(make_double2(sq, 0));
  if (threadIdx.x == 0) b.partials[blockIdx.x] = t.x;
  if (!last_block_done(b.ticket)) return;
  double tot = 0;
  for (unsigned bl = threadIdx.x; bl < gridDim.x; bl += blockDim.x) tot += b.partials[bl];
  const double2 all = block_sum(make_double2(tot, 0));
  if (threadIdx.x != 0) return;
  *b.ticket = 0;
  const double after = sqrt(all.x);
  if (P == 0 && isfinite(after) && REORTH * after < sqrt(st->before_sq)) {
    st->reorth = 1;
    st->reorth_count += 1;
    return;
  }
  finish_step(b, st, m, j, after);
}

// v_{j+1} = w / ||w|| after a CGS2 step (skipped on breakdown and once the
// cycle has ended: only v_0..v_{used-1} enter the update).
__global__ void normalize_kernel(GmBuffers b, long long n, int j) {
  pdl_begin();
  GmState *st = b.st;
  if (!st->active || !st->normalize) return;
  const double inv = st->after;
  double2 *vn = b.V + (long long)(j + 1) * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    vn[i] = make_double2(b.w[i].x / inv, b.w[i].y / inv);
}

// v_0 = r / beta and the Hessenberg / rotation reset for a new cycle.
__global__ void cycle_start_kernel(GmBuffers b, long long n, int m, double beta) {
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = tid; i < n; i += stride) b.V[i] = make_double2(b.r[i].x / beta, b.r[i].y / beta);
  for (long long i = tid; i < (long long)(m + 1) * m; i += stride) b.H[i] = make_double2(0, 0);
  for (long long i = tid; i <= m; i += stride) b.g[i] = make_double2(i == 0 ? beta : 0, 0);
}

// y = H^{-1} g (back substitution, vie_iterative.c:179-186), one warp: the
// lanes share each row's sum over the solved unknowns, added in a fixed
// order (lane partials, then a butterfly).
__global__ void backsolve_kernel(GmBuffers b, int m) {
  GmState *st = b.st;
  if (st->status != ST_RUNNING) return;
  const int used = st->used, lane = threadIdx.x;
  __shared__ int broke;
  if (lane == 0) broke = 0;
  __syncwarp();
  for (int i = used - 1; i >= 0; --i) {
    double2 part = make_double2(0, 0);
    for (int k = i + 1 + lane; k < used; k += 32) part = cadd(part, cmul(b.H[(long long)i * m + k], b.y[k]));
    for (int o = 16; o > 0; o >>= 1) {
      part.x += __shfl_xor_sync(0xffffffffu, part.x, o);
      part.y += __shfl_xor_sync(0xffffffffu, part.y, o);
    }
    if (lane == 0) {
      const double2 d = b.H[(long long)i * m + i];
      if (cabs_(d) == 0.0) { st->status = ST_BREAKDOWN; broke = 1; }
      else b.y[i] = cdiv(csub(b.g[i], part), d);
    }
    __syncwarp();
    if (broke) return;
  }
}

// x += D^-1 (sum_j v_j y_j): the divisor is applied once to the sum.
__global__ void update_kernel(GmBuffers b, const double2 *__restrict__ pdiag, double2 *__restrict__ x,
                              long long n) {
  if (b.st->status != ST_RUNNING) return;
  const int used = b.st->used;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double2 acc = make_double2(0, 0);
    for (int j = 0; j < used; ++j) acc = cadd(acc, cmul(b.V[(long long)j * n + i], b.y[j]));
    if (pdiag) acc = cdiv(acc, pdiag[i]);
    x[i] = cadd(x[i], acc);
  }
}

// r = b - A x (A x already in r) with ||r||^2 into residual_sq.
__global__ void residual_kernel(const double2 *__restrict__ rhs, double2 *__restrict__ r, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    r[i] = csub(rhs[i], r[i]);
}

// ------------------------------------------------------------------ host side
struct OpView {
  int kind;
  void *op;
  long long n;
  const double2 *pdiag;
  int mixed;          // FP32 transforms: Arnoldi by CGS2 sweeps
};
n2d_vie *n2c_hybrid_volume(const n2d_hybrid *h);

// Arnoldi products use the operator's transform precision; the true residual
// at every restart is always FP64 (full_precision).
static int op_apply(const OpView &o, const double *x, double *y, int precond, double *norm, int *flag,
                    int full_precision) {
  if (o.kind == 0) return n2d_vie_apply((n2d_vie *)o.op, x, y, precond, norm, flag, full_precision);
  return n2d_hybrid_apply((n2d_hybrid *)o.op, x, y, precond, norm, flag, full_precision);
}

template <int E>
static int launch_arnoldi(GmBuffers &b, long long n, int m, int j, int blocks, int threads) {
  void *args[] = {&b, &n, &m, &j};
  cudaError_t e = cudaLaunchCooperativeKernel((void *)arnoldi_kernel<E>, blocks, threads, args, 0,
                                              n2c_stream());
  if (e != cudaSuccess) { n2c_set_error("arnoldi launch: %s", cudaGetErrorString(e)); return 0; }
  n2c_count_launch(1);
  return 1;
}

typedef int (*ArnoldiLauncher)(GmBuffers &, long long, int, int, int, int);

// Among the co-resident shapes (E elements of w per thread, 256 or 512
// threads) pick the one that spreads w over the most SMs, then the smaller E.
static int arnoldi_shape(long long n, int *blocks, int *threads, ArnoldiLauncher *fn) {
  static const int Es[] = {1, 2, 4, 8, 16};
  static const ArnoldiLauncher fns[] = {launch_arnoldi<1>, launch_arnoldi<2>, launch_arnoldi<4>,
                                        launch_arnoldi<8>, launch_arnoldi<16>};
  static const void *kern[] = {(void *)arnoldi_kernel<1>, (void *)arnoldi_kernel<2>,
                               (void *)arnoldi_kernel<4>, (void *)arnoldi_kernel<8>,
                               (void *)arnoldi_kernel<16>};
  const int sms = n2c_sm_count();
  long long best_cover = -1;
  for (int q = 0; q < 5; ++q)
    for (int th = 256; th <= 512; th *= 2) {
      int occ = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern[q], th, 0) != cudaSuccess || occ < 1)
        continue;
      if (occ > 2) occ = 2;
      const long long per_block = (long long)th * Es[q];
      long long bl = (n + per_block - 1) / per_block;
      if (bl < 1) bl = 1;
      if (bl > (long long)sms * occ) continue;
      const long long cover = bl < sms ? bl : sms;
      if (cover > best_cover) {
        best_cover = cover;
        *blocks = (int)bl; *threads = th; *fn = fns[q];
      }
    }
  if (best_cover < 0) {
    n2c_set_error("GMRES order %lld exceeds the device-resident Arnoldi limit", n);
    return 0;
  }
  return 1;
}

static unsigned grid1(long long n) {
  long long b = (n + 255) / 256;
  long long cap = (long long)n2c_sm_count() * 8;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

// Persistent GMRES workspace of one operator: buffers for (n, m) and the
// captured CUDA graph of a restart cycle's inner iterations.
struct GmWork {
  long long n, m;
  int mixed;
  GmBuffers b;
  int blocks, threads;
  ArnoldiLauncher arnoldi;
  cudaGraphExec_t inner;      // null: launch the inner loop directly
  unsigned inner_launches;    // kernels per replay (launch accounting)
  bool tried_graph;
};

static void work_free(GmWork *w) {
  if (!w) return;
  if (w->inner) cudaGraphExecDestroy(w->inner);
  GmBuffers &b = w->b;
  void *bufs[] = {b.st, b.H, b.g, b.sn, b.y, b.cs, b.V, b.w, b.r, b.partials, b.ticket, b.cgs_h};
  for (void *q : bufs) n2d_free(q);
  delete w;
}

void n2c_gmres_work_free(void *w) { work_free((GmWork *)w); }
void **n2c_vie_gm_slot(n2d_vie *p);
void **n2c_hybrid_gm_slot(n2d_hybrid *h);

static GmWork *work_get(const OpView &o, long long m) {
  void **slot = o.kind == 0 ? n2c_vie_gm_slot((n2d_vie *)o.op) : n2c_hybrid_gm_slot((n2d_hybrid *)o.op);
  GmWork *w = (GmWork *)*slot;
  if (w && w->n == o.n && w->m == m && w->mixed == o.mixed) return w;
  work_free(w);
  *slot = nullptr;
  const long long n = o.n;
  w = new GmWork();
  memset(w, 0, sizeof(*w));
  w->n = n; w->m = m; w->mixed = o.mixed;
  const bool use_cgs = o.mixed && m <= MAXM;
  if (!use_cgs && !arnoldi_shape(n, &w->blocks, &w->threads, &w->arnoldi)) { delete w; return nullptr; }
  GmBuffers &b = w->b;
  b.st = (GmState *)n2d_alloc(sizeof(GmState));
  b.H = (double2 *)n2d_alloc((m + 1) * m * sizeof(double2));
  b.g = (double2 *)n2d_alloc((m + 1) * sizeof(double2));
  b.sn = (double2 *)n2d_alloc(m * sizeof(double2));
  b.y = (double2 *)n2d_alloc(m * sizeof(double2));
  b.cs = (double *)n2d_alloc(m * sizeof(double));
  b.V = (double2 *)n2d_alloc((m + 1) * n * sizeof(double2));
  b.w = (double2 *)n2d_alloc(n * sizeof(double2));
  b.r = (double2 *)n2d_alloc(n * sizeof(double2));
  b.partials = (double *)n2d_alloc(PART_TOTAL * sizeof(double));
  b.cgs_h = (double2 *)n2d_alloc(2 * MAXM * sizeof(double2));
  b.ticket = (unsigned int *)n2d_alloc(64);
  if (!b.st || !b.H || !b.g || !b.sn || !b.y || !b.cs || !b.V || !b.w || !b.r || !b.partials || !b.ticket ||
      !b.cgs_h || !n2d_memset(b.ticket, 0, 64)) {
    work_free(w);
    return nullptr;
  }
  *slot = w;
  return w;
}

// Enqueues the m gated inner iterations of a cycle on the current stream.
static int enqueue_inner(const OpView &o, GmWork *w) {
  GmBuffers &b = w->b;
  const long long n = w->n, m = w->m;
  const bool use_cgs = o.mixed && m <= MAXM;
  n2d_set_gate(&b.st->active);
  int ok = 1;
  for (int j = 0; j < m && ok; ++j) {
    ok = op_apply(o, (const double *)(b.V + (long long)j * n), (double *)b.w, o.pdiag != nullptr,
                  &b.st->before_sq, &b.st->flag, 0);
    if (!ok) break;
    if (use_cgs) {
      const unsigned gb = (unsigned)n2c_sm_count();
      const unsigned ub = grid1(n) < 4096 ? grid1(n) : 4096;
      // Programmatic dependent launches when NEC2C_CUDA_PDL_GMRES=1: each
      // sweep's launch overlaps the previous kernel's last wave (the kernels
      // wait for it first).
      static const bool pdl = [] {
        const char *v = getenv("NEC2C_CUDA_PDL_GMRES");
        return v && v[0] == '1';
      }();
      ok = n2c_launch_pdl(pdl, cgs_dots_kernel<0>, dim3(gb), dim3(1024), 0, "cgs dots", b, n, (int)m, j) &&
           n2c_launch_pdl(pdl, cgs_update_kernel<0>, dim3(ub), dim3(256), 0, "cgs update", b, n, (int)m, j) &&
           n2c_launch_pdl(pdl, cgs_dots_kernel<1>, dim3(gb), dim3(1024), 0, "cgs dots", b, n, (int)m, j) &&
           n2c_launch_pdl(pdl, cgs_update_kernel<1>, dim3(ub), dim3(256), 0, "cgs update", b, n, (int)m, j) &&
           n2c_launch_pdl(pdl, normalize_kernel, dim3(grid1(n)), dim3(256), 0, "cgs normalize", b, n, j);
    } else {
      ok = w->arnoldi(b, n, (int)m, j, w->blocks, w->threads);
    }
  }
  n2d_set_gate(nullptr);
  return ok;
}

// Captures the inner loop once into a graph (launched on the caller's stream
// every cycle); falls back to direct launches when capture is unavailable.
static void try_capture(const OpView &o, GmWork *w) {
  w->tried_graph = true;
  static thread_local cudaStream_t cap = nullptr;
  if (!cap && cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) { cap = nullptr; return; }
  void *user = n2d_get_stream();
  const unsigned long long before = n2d_launch_count();
  n2d_set_stream(cap);
  cudaGraph_t graph = nullptr;
  int ok = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) ok = enqueue_inner(o, w);
  cudaError_t e = cudaStreamEndCapture(cap, &graph);
  n2d_set_stream(user);
  if (ok && e == cudaSuccess && graph && cudaGraphInstantiate(&w->inner, graph, 0) == cudaSuccess) {
    w->inner_launches = (unsigned)(n2d_launch_count() - before);
  } else {
    w->inner = nullptr;
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();
}

static int gmres_core(const OpView &o, const double2 *b_dev, double2 *x_dev, size_t restart, size_t maxit,
                      double rtol, double atol, n2d_gmres_report *rep) {
  const long long n = o.n;
  long long m = (long long)restart;
  if (m > n) m = n;
  if (m > (long long)maxit) m = (long long)maxit;
  GmWork *w = work_get(o, m);
  if (!w) { rep->status = ST_ALLOC; return 0; }
  GmBuffers &b = w->b;
  int ok = 0;
  GmState hs;
  double bnorm = 0, target = 0;
  memset(&hs, 0, sizeof(hs));
  hs.status = ST_RUNNING;
  hs.max_iterations = (long long)maxit;
  double *dnorm = b.partials + PART_SCALARS;
  int *dflag = (int *)(b.partials + PART_SCALARS + 8);
  auto read_state = [&]() { return n2d_download(&hs, b.st, sizeof(hs)); };
  // ||b|| and ||x|| (finite check) before anything else (vie_iterative.c:116-119).
  double norms[2];
  if (!n2d_memset(dflag, 0, sizeof(int)) ||
      !n2c_norm2((const double *)b_dev, n, b.partials, b.ticket, dnorm, dflag) ||
      !n2c_norm2((const double *)x_dev, n, b.partials, b.ticket, dnorm + 1, dflag) ||
      !n2d_download(norms, dnorm, sizeof(norms))) { rep->status = ST_ALLOC; return 0; }
  int hflag = 0;
  if (!n2d_download(&hflag, dflag, sizeof(int))) return 0;
  bnorm = sqrt(norms[0]);
  target = fmax(atol, rtol * bnorm);
  if (hflag || !isfinite(bnorm) || !isfinite(sqrt(norms[1])) || !isfinite(target)) {
    rep->status = ST_NONFINITE;
    return 0;
  }
  hs.target = target;
  // True residual r = b - A x (always FP64).
  auto true_residual = [&]() -> int {
    ++rep->operator_applications;
    if (!n2d_memset(dflag, 0, sizeof(int))) return 0;
    if (!op_apply(o, (const double *)x_dev, (double *)b.r, 0, nullptr, dflag, 1)) { rep->status = ST_CALLBACK; return 0; }
    residual_kernel<<<grid1(n), 256, 0, n2c_stream()>>>(b_dev, b.r, n);
    if (!n2c_check_launch("residual")) return 0;
    double sq = 0;
    if (!n2c_norm2((const double *)b.r, n, b.partials, b.ticket, dnorm, dflag) ||
        !n2d_download(&sq, dnorm, sizeof(double)) || !n2d_download(&hflag, dflag, sizeof(int)))
      return 0;
    rep->residual_norm = hflag ? NAN : sqrt(sq);
    if (!isfinite(rep->residual_norm)) { rep->status = ST_NONFINITE; return 0; }
    return 1;
  };
  if (!true_residual()) return 0;
  for (;;) {
    const double beta = rep->residual_norm;
    rep->relative_residual = bnorm > 0 ? beta / bnorm : beta;
    if (beta <= target) { rep->status = ST_CONVERGED; ok = 1; break; }
    if ((long long)rep->iterations >= (long long)maxit) { rep->status = ST_LIMIT; break; }
    if (o.kind == 1 && !n2c_hybrid_precondition_ok((const n2d_hybrid *)o.op)) { rep->status = ST_CALLBACK; break; }
    cycle_start_kernel<<<grid1(n), 256, 0, n2c_stream()>>>(b, n, (int)m, beta);
    if (!n2c_check_launch("cycle_start")) break;
    // The state block carries the running iteration count across cycles.
    hs.iterations = (long long)rep->iterations;
    hs.active = 1; hs.used = 0; hs.breakdown = 0; hs.flag = 0; hs.barrier_error = 0;
    hs.bar_count = 0; hs.bar_gen = 0; hs.normalize = 0; hs.reorth = 0;
    if (!n2d_upload(b.st, &hs, sizeof(hs))) break;
    if (!w->tried_graph) try_capture(o, w);
    bool launch_fail;
    if (w->inner) {
      launch_fail = cudaGraphLaunch(w->inner, (cudaStream_t)n2d_get_stream()) != cudaSuccess;
      n2c_count_launch(w->inner_launches);
    } else {
      launch_fail = !enqueue_inner(o, w);
    }
    if (launch_fail) { rep->status = ST_CALLBACK; break; }
    backsolve_kernel<<<1, 32, 0, n2c_stream()>>>(b, (int)m);
    if (!n2c_check_launch("backsolve")) break;
    update_kernel<<<grid1(n), 256, 0, n2c_stream()>>>(b, o.pdiag, x_dev, n);
    if (!n2c_check_launch("update")) break;
    if (!read_state()) break;
    rep->iterations = (size_t)hs.iterations;
    rep->operator_applications += (size_t)hs.used;
    if (hs.barrier_error) { n2c_set_error("grid barrier time-out in GMRES"); rep->status = ST_CALLBACK; break; }
    if (hs.status != ST_RUNNING) { rep->status = hs.status; break; }
    if (!true_residual()) break;
    rep->relative_residual = bnorm > 0 ? rep->residual_norm / bnorm : rep->residual_norm;
    if (hs.breakdown && rep->residual_norm > target) { rep->status = ST_BREAKDOWN; break; }
    if (rep->residual_norm > target && (long long)rep->iterations < (long long)maxit) ++rep->restarts;
  }
  return ok;
}

static int gmres_setup(int kind, void *op, long long n, OpView *o) {
  o->kind = kind; o->op = op; o->n = n;
  o->pdiag = kind == 0 ? (const double2 *)n2d_vie_diag((n2d_vie *)op)
                       : n2c_hybrid_pdiag((const n2d_hybrid *)op);
  n2d_vie *vol = kind == 0 ? (n2d_vie *)op : n2c_hybrid_volume((const n2d_hybrid *)op);
  o->mixed = vol && n2d_vie_fp32(vol);
  return 1;
}

extern "C" int n2d_gmres_dev(int kind, void *op, long long n, const double *b_dev, double *x_dev,
                             size_t restart, size_t maxit, double rtol, double atol,
                             n2d_gmres_report *rep) {
  OpView o;
  memset(rep, 0, sizeof(*rep));
  rep->status = ST_INVALID;
  rep->residual_norm = rep->relative_residual = INFINITY;
  gmres_setup(kind, op, n, &o);
  return gmres_core(o, (const double2 *)b_dev, (double2 *)x_dev, restart, maxit, rtol, atol, rep);
}

extern "C" int n2d_gmres(int kind, void *op, long long n, const double *b, double *x, size_t restart,
                         size_t maxit, double rtol, double atol, n2d_gmres_report *rep) {
  memset(rep, 0, sizeof(*rep));
  rep->status = ST_ALLOC;
  rep->residual_norm = rep->relative_residual = INFINITY;
  // Stream-ordered staging: a server worker's solve must not synchronise the
  // device (cudaFree would wait for every other worker's work in flight).
  double *bd = (double *)n2d_alloc_async(n * sizeof(double2)), *xd = (double *)n2d_alloc_async(n * sizeof(double2));
  int ok = 0;
  if (bd && xd && n2d_upload(bd, b, n * sizeof(double2)) && n2d_upload(xd, x, n * sizeof(double2))) {
    ok = n2d_gmres_dev(kind, op, n, bd, xd, restart, maxit, rtol, atol, rep);
    // x is updated even on failure (vie_iterative.h:51-53).
    if (!n2d_download(x, xd, n * sizeof(double2))) ok = 0;
  }
  n2d_free_async(bd);
  n2d_free_async(xd);
  return ok;
}

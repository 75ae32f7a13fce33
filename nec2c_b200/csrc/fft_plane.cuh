// Fused yz-plane passes of the matvec: the y and z transforms of one lattice
// plane x in a single kernel, forward (with the cell scatter) and inverse
// (with the permittivity epilogue), so a product takes three launches
// (forward planes, x pass with the spectrum product, inverse planes) instead
// of five, and the grid between the z and y transforms never leaves shared
// memory.
//
// Parity split.  The padded axes are P = 2Q (the reference pads each axis to a
// power of two >= 2n-1, so Q >= n).  With k = 2m + r (r = 0, 1) the P-point
// transform of n <= Q values is two Q-point transforms of twiddled values:
//   X[2m + r] = sum_{j<n} (x[j] W_P^{j r}) W_Q^{j m},
// and the inverse keeps j < n of
//   y[j] = sum_r W_P^{-j r} sum_{m<Q} Y[2m + r] W_Q^{-j m}.
// In the y and z axes together a plane is four Q x Q transforms, one per
// parity pair (ry, rz), each a CTA:
//   forward : CTA (c, x, ry, rz) loads the plane's n_y x n_z cell values of
//             component c, twiddles them by W_Py^{jy ry} W_Pz^{jz rz}, runs the
//             Q x Q transform and writes grid[c][x][2my+ry][2mz+rz];
//   inverse : the four CTAs of a plane form a thread-block cluster; each runs
//             the inverse Q x Q transform of its parity pair, post-twiddles it
//             and keeps it in shared memory; after a cluster barrier each CTA
//             sums a quarter of the plane over the four CTAs' shared memory
//             (distributed shared memory, fixed order, so the result does not
//             depend on timing) and runs the epilogue on it.
// A Q-point transform is the four-step split Q = R1 x R2 of fft_engine.cuh on
// a Q x (Q+1) shared tile ([element][line], odd row pitch: conflict-free
// 8- and 16-byte accesses), using the P-point twiddle table (W_Q^m =
// tw[2m]).  The second step of the first axis writes its result transposed,
// so the second axis again finds its lines in the [element][line] layout.
#pragma once
#include <atomic>
#include <cooperative_groups.h>
#include "fft_passes.cuh"
#include "runtime.cuh"

namespace n2c {

template <typename C>
__device__ __forceinline__ double2 plane_divisor(const PlaneArgs<C> &a, double2 e, int c) {
  const double2 s = c == 0 ? a.self0 : (c == 1 ? a.self1 : a.self2);
  return csub(e, cmul(make_double2(e.x - 1.0, e.y), s));
}

// Step 1 of the Q-point four-step on lines t < Q of tile S ([element][line],
// pitch QP), in place: per (j2, t) the R1-point DFT over elements j2 + R2 j1
// and the twiddle W_Q^{+-j2 k1}; results back into slots j2 + R2 k1.
template <typename C, int R1, int R2, bool INV>
__device__ __forceinline__ void plane_step1(C *S, const C *__restrict__ tw) {
  constexpr int Q = R1 * R2, QP = Q + 1;
  for (int item = threadIdx.x; item < Q * R2; item += blockDim.x) {
    const int j2 = item / Q, t = item - j2 * Q;
    C v[R1];
#pragma unroll
    for (int j1 = 0; j1 < R1; ++j1) v[j1] = S[(j2 + R2 * j1) * QP + t];
    dft_reg<R1, INV, 2 * R2>(v, tw);
    if (j2) {
#pragma unroll
      for (int k1 = 1; k1 < R1; ++k1) {
        const C w = __ldg(&tw[2 * j2 * k1]);
        v[k1] = INV ? cmulc(v[k1], w) : cmul(v[k1], w);
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) S[(j2 + R2 * k1) * QP + t] = v[k1];
  }
  __syncthreads();
}

// Step 2 of the Q-point four-step: per (k1, t) the R2-point DFT over slots
// k1 + ... (as step 1 left them) giving element k = k1 + R1 k2 of line t.
// TRANSPOSE: the results are held in registers across a barrier and written
// back as S[t][k] (the line index becomes the element index).  Otherwise
// each result is handed to sink(t, k, value).
template <typename C, int R1, int R2, bool INV, int THREADS>
struct PlaneStep2 {
  static constexpr int Q = R1 * R2, QP = Q + 1, ITEMS = Q * R1, IPT = (ITEMS + THREADS - 1) / THREADS;
  __device__ __forceinline__ static void transpose(C *S, const C *__restrict__ tw) {
    C w[IPT][R2];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const int item = threadIdx.x + i * THREADS;
      if (item < ITEMS) {
        const int k1 = item / Q, t = item - k1 * Q;
#pragma unroll
        for (int j2 = 0; j2 < R2; ++j2) w[i][j2] = S[(j2 + R2 * k1) * QP + t];
        dft_reg<R2, INV, 2 * R1>(w[i], tw);
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const int item = threadIdx.x + i * THREADS;
      if (item < ITEMS) {
        const int k1 = item / Q, t = item - k1 * Q;
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) S[t * QP + k1 + R1 * k2] = w[i][k2];
      }
    }
    __syncthreads();
  }
  template <typename Sink>
  __device__ __forceinline__ static void emit(const C *S, const C *__restrict__ tw, Sink &&sink) {
    for (int item = threadIdx.x; item < ITEMS; item += THREADS) {
      const int k1 = item / Q, t = item - k1 * Q;
      C w[R2];
#pragma unroll
      for (int j2 = 0; j2 < R2; ++j2) w[j2] = S[(j2 + R2 * k1) * QP + t];
      dft_reg<R2, INV, 2 * R1>(w, tw);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) sink(t, k1 + R1 * k2, w[k2]);
    }
  }
};

// Inverse (unnormalised) Q-point four-step, in two steps on the same tile:
// step A per (k1, t) the R2-point inverse DFT over slots k1 + R1 k2 and the
// twiddle W_Q^{-n1 k1}, results back into slots k1 + R1 n1 (the same slots,
// so it runs in place); step B per (n1, t) the R1-point inverse DFT over
// slots k1 + R1 n1, giving element n = n1 + R2 n2 of line t, written
// transposed (S[t][n]) after a barrier.
template <typename C, int R1, int R2>
__device__ __forceinline__ void plane_inv_stepA(C *S, const C *__restrict__ tw) {
  constexpr int Q = R1 * R2, QP = Q + 1;
  for (int item = threadIdx.x; item < Q * R1; item += blockDim.x) {
    const int k1 = item / Q, t = item - k1 * Q;
    C w[R2];
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) w[k2] = S[(k1 + R1 * k2) * QP + t];
    dft_reg<R2, true, 2 * R1>(w, tw);
    if (k1) {
#pragma unroll
      for (int n1 = 1; n1 < R2; ++n1) w[n1] = cmulc(w[n1], __ldg(&tw[2 * n1 * k1]));
    }
#pragma unroll
    for (int n1 = 0; n1 < R2; ++n1) S[(k1 + R1 * n1) * QP + t] = w[n1];
  }
  __syncthreads();
}

template <typename C, int R1, int R2, int THREADS>
__device__ __forceinline__ void plane_inv_stepB_transpose(C *S, const C *__restrict__ tw) {
  constexpr int Q = R1 * R2, QP = Q + 1, ITEMS = Q * R2, IPT = (ITEMS + THREADS - 1) / THREADS;
  C v[IPT][R1];
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    const int item = threadIdx.x + i * THREADS;
    if (item < ITEMS) {
      const int n1 = item / Q, t = item - n1 * Q;
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) v[i][k1] = S[(k1 + R1 * n1) * QP + t];
      dft_reg<R1, true, 2 * R2>(v[i], tw);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    const int item = threadIdx.x + i * THREADS;
    if (item < ITEMS) {
      const int n1 = item / Q, t = item - n1 * Q;
#pragma unroll
      for (int n2 = 0; n2 < R1; ++n2) S[t * QP + n1 + R2 * n2] = v[i][n2];
    }
  }
  __syncthreads();
}

constexpr int PLANE_THREADS = 256;

// Forward: CTA b = ((c * nx + x) * 4 + ry * 2 + rz).
template <typename C, int R1, int R2>
__global__ void __launch_bounds__(PLANE_THREADS, 3) fft_plane_forward(PlaneArgs<C> a) {
  if (a.gate && *(volatile const int *)a.gate == 0) return;
  constexpr int Q = R1 * R2, QP = Q + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *S = reinterpret_cast<C *>(smem_raw);
  const int par = blockIdx.x & 3, ry = par >> 1, rz = par & 1;
  const int plane = blockIdx.x >> 2, c = plane / a.nx, x = plane - c * a.nx;
  // Load: S[jz][jy] = twiddled cell value (zero outside the lattice).  Each
  // thread takes PER elements, CH at a time with their loads issued together
  // (box index -> cell, then the cell's value and permittivity), so the
  // dependent global loads cost two round trips per chunk, not two per
  // element.
  constexpr int PER = Q * Q / PLANE_THREADS, CH = PER < 4 ? PER : 4;
  static_assert(PER * PLANE_THREADS == Q * Q && PER % CH == 0, "plane tile per thread");
#pragma unroll
  for (int base = 0; base < PER; base += CH) {
    int cell[CH];
#pragma unroll
    for (int i = 0; i < CH; ++i) {
      const int idx = threadIdx.x + (base + i) * PLANE_THREADS, jy = idx / Q, jz = idx - jy * Q;
      cell[i] = (jy < a.ny && jz < a.nz) ? a.box_cell[((long long)x * a.ny + jy) * a.nz + jz] : -1;
    }
    double2 v[CH], e[CH];
    bool neg[CH];
#pragma unroll
    for (int i = 0; i < CH; ++i) {
      neg[i] = false;
      if (cell[i] >= 0) {
        if (a.mirror && cell[i] >= a.mirror) { cell[i] -= (int)a.mirror; neg[i] = c < 2; }
        v[i] = a.cx[3 * (long long)cell[i] + c];
        if (a.precondition) e[i] = a.eps[cell[i]];
      }
    }
#pragma unroll
    for (int i = 0; i < CH; ++i) {
      const int idx = threadIdx.x + (base + i) * PLANE_THREADS, jy = idx / Q, jz = idx - jy * Q;
      C val = czero<C>();
      if (cell[i] >= 0) {
        double2 w = v[i];
        if (a.precondition) w = jacobi_apply<C>(w, plane_divisor(a, e[i], c));
        if (a.flag && !finite2(w)) *a.flag = 1;
        if (neg[i]) w = make_double2(-w.x, -w.y);
        val = from_d<C>(w);
        if (ry && jy) val = cmul(val, __ldg(&a.twy[jy]));
        if (rz && jz) val = cmul(val, __ldg(&a.twz[jz]));
      }
      S[jz * QP + jy] = val;
    }
  }
  __syncthreads();
  plane_step1<C, R1, R2, false>(S, a.twz);                          // z, lines jy
  PlaneStep2<C, R1, R2, false, PLANE_THREADS>::transpose(S, a.twz);  // S[jy][mz]
  plane_step1<C, R1, R2, false>(S, a.twy);                          // y, lines mz
  const int P = 2 * Q;
  C *out = a.grid + ((long long)c * a.nx + x) * P * P;
  PlaneStep2<C, R1, R2, false, PLANE_THREADS>::emit(S, a.twy, [&](int mz, int my, C v) {
    out[(2 * my + ry) * P + 2 * mz + rz] = v;
  });
}

// Inverse with the epilogue: cluster of the four parity CTAs of a plane.
template <typename C, int R1, int R2>
__global__ void __launch_bounds__(PLANE_THREADS, 3) fft_plane_inverse(PlaneArgs<C> a) {
  if (a.gate && *(volatile const int *)a.gate == 0) return;
  namespace cg = cooperative_groups;
  constexpr int Q = R1 * R2, QP = Q + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *S = reinterpret_cast<C *>(smem_raw);
  cg::cluster_group cluster = cg::this_cluster();
  const int par = (int)cluster.block_rank(), ry = par >> 1, rz = par & 1;
  const int plane = blockIdx.x >> 2, c = plane / a.nx, x = plane - c * a.nx;
  const int P = 2 * Q;
  const C *in = a.grid + ((long long)c * a.nx + x) * P * P;
  // Load: S[mz][my] = grid[2my+ry][2mz+rz], CH loads in flight per thread.
  constexpr int PER = Q * Q / PLANE_THREADS, CH = PER < 8 ? PER : 8;
  static_assert(PER * PLANE_THREADS == Q * Q && PER % CH == 0, "plane tile per thread");
#pragma unroll
  for (int base = 0; base < PER; base += CH) {
    C g[CH];
#pragma unroll
    for (int i = 0; i < CH; ++i) {
      const int idx = threadIdx.x + (base + i) * PLANE_THREADS, my = idx / Q, mz = idx - my * Q;
      g[i] = in[(2 * my + ry) * P + 2 * mz + rz];
    }
#pragma unroll
    for (int i = 0; i < CH; ++i) {
      const int idx = threadIdx.x + (base + i) * PLANE_THREADS, my = idx / Q, mz = idx - my * Q;
      S[mz * QP + my] = g[i];
    }
  }
  __syncthreads();
  plane_inv_stepA<C, R1, R2>(S, a.twz);                              // z, lines my
  plane_inv_stepB_transpose<C, R1, R2, PLANE_THREADS>(S, a.twz);     // S[my][jz]
  plane_inv_stepA<C, R1, R2>(S, a.twy);                              // y, lines jz
  plane_inv_stepB_transpose<C, R1, R2, PLANE_THREADS>(S, a.twy);     // S[jz][jy]
  // Post-twiddle W_Py^{-jy ry} W_Pz^{-jz rz} of this parity pair.
  if (ry || rz) {
    for (int idx = threadIdx.x; idx < Q * Q; idx += PLANE_THREADS) {
      const int jz = idx / Q, jy = idx - jz * Q;
      C v = S[jz * QP + jy];
      if (ry && jy) v = cmulc(v, __ldg(&a.twy[jy]));
      if (rz && jz) v = cmulc(v, __ldg(&a.twz[jz]));
      S[jz * QP + jy] = v;
    }
  }
  cluster.sync();
  // This CTA finishes rows jy = par, par + 4, ... of the plane.
  const C *peer[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) peer[r] = cluster.map_shared_rank(S, r);
  double sq = 0;
  const int rows = (a.ny - par + 3) / 4, total = rows * a.nz;
  constexpr int EC = 4;   // outputs per thread whose loads are issued together
  for (int base = threadIdx.x; base < total; base += EC * PLANE_THREADS) {
    int cell[EC], s[EC];
#pragma unroll
    for (int i = 0; i < EC; ++i) {
      const int idx = base + i * PLANE_THREADS;
      cell[i] = -1;
      s[i] = 0;
      if (idx < total) {
        const int r = idx / a.nz, jz = idx - r * a.nz, jy = par + 4 * r;
        const int cl = a.box_cell[((long long)x * a.ny + jy) * a.nz + jz];
        if (cl >= 0 && !(a.mirror && cl >= a.mirror)) cell[i] = cl;
        s[i] = jz * QP + jy;
      }
    }
    double2 ep[EC], z[EC];
    C f[EC];
#pragma unroll
    for (int i = 0; i < EC; ++i) {
      if (cell[i] < 0) continue;
      ep[i] = a.eps[cell[i]];
      z[i] = a.cx[3 * (long long)cell[i] + c];
      f[i] = peer[0][s[i]];
      f[i] = cadd(f[i], peer[1][s[i]]);
      f[i] = cadd(f[i], peer[2][s[i]]);
      f[i] = cadd(f[i], peer[3][s[i]]);
    }
#pragma unroll
    for (int i = 0; i < EC; ++i) {
      if (cell[i] < 0) continue;
      const double2 em1 = make_double2(ep[i].x - 1.0, ep[i].y);
      double2 zz = z[i];
      if (a.precondition) zz = jacobi_apply<C>(zz, plane_divisor(a, ep[i], c));
      const double2 v = csub(cmul(ep[i], zz), cmul(em1, to_d(f[i])));
      a.cy[3 * (long long)cell[i] + c] = v;
      if (a.flag && !finite2(v)) *a.flag = 1;
      sq += v.x * v.x + v.y * v.y;
    }
  }
  cluster.sync();   // peers' shared memory stays alive until every CTA has read it
  if (a.norm) {
    // Deterministic |y|^2: block partials summed in block order by the last block.
    const unsigned ntiles = gridDim.x;
    const double2 bs = block_sum(make_double2(sq, 0));
    if (threadIdx.x == 0) a.partials[blockIdx.x] = bs.x;
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(a.ticket, 1u) == ntiles - 1;
    __syncthreads();
    if (last) {
      double t2 = 0;
      for (unsigned i = threadIdx.x; i < ntiles; i += PLANE_THREADS) t2 += a.partials[i];
      const double2 tot = block_sum(make_double2(t2, 0));
      if (threadIdx.x == 0) { *a.norm = tot.x; *a.ticket = 0; }
    }
  }
}

template <typename C, int R1, int R2>
static int plane_launch_rr(bool inverse, const PlaneArgs<C> &a, cudaStream_t stream) {
  constexpr int Q = R1 * R2;
  const size_t smem = plane_smem<C>(Q);
  void (*k)(PlaneArgs<C>) = inverse ? fft_plane_inverse<C, R1, R2> : fft_plane_forward<C, R1, R2>;
  static std::atomic<bool> configured[2];
  if (!configured[inverse].load(std::memory_order_acquire)) {
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      n2c_set_error("cannot raise shared memory for the plane pass");
      return 0;
    }
    configured[inverse].store(true, std::memory_order_release);
  }
  const unsigned blocks = 12u * (unsigned)a.nx;
  if (!inverse) {
    k<<<blocks, PLANE_THREADS, smem, stream>>>(a);
    return n2c_check_launch("plane forward");
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(PLANE_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 4;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k, a);
  if (e != cudaSuccess) { n2c_set_error("plane inverse launch: %s", cudaGetErrorString(e)); return 0; }
  n2c_count_launch(1);
  return 1;
}

template <typename C>
int fft_plane_launch(bool inverse, int Q, const PlaneArgs<C> &a, cudaStream_t stream) {
  switch (Q) {
    case 16: return plane_launch_rr<C, 4, 4>(inverse, a, stream);
    case 32: return plane_launch_rr<C, 8, 4>(inverse, a, stream);
    case 64: return plane_launch_rr<C, 8, 8>(inverse, a, stream);
  }
  n2c_set_error("no plane pass for Q = %d", Q);
  return 0;
}

}  // namespace n2c

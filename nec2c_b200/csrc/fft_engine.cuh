// Line-FFT engine for the padded Green-convolution grid.
//
// A length-L line (L = R1*R2, powers of two up to 1024) is transformed in two
// register steps with one shared-memory exchange (the "four-step" split):
//   forward : step 1 (per j2)  R1-point DFT over x[j2 + R2*j1], twiddle W^{j2 k1}
//             step 2 (per k1)  R2-point DFT  -> X[k1 + R1*k2]
//   inverse : step A (per k1)  R2-point DFT over X[k1 + R1*k2], twiddle W^{-n1 k1}
//             step B (per n1)  R1-point DFT  -> x[n1 + R2*n2]
// The shared slot of intermediate (j2|n1, k1) is (j2|n1) + R2*k1 in both
// directions, so a forward step 2 can feed an inverse step A in registers with
// no extra exchange (used by the spectrum-product pass).
//
// Tiles hold NL lines (NL a power of two <= 32).  Work items are mapped
// line-fastest so a warp touches 32 consecutive lines: in the strided passes
// (y and x axes) consecutive lines are consecutive addresses, so every global
// access is coalesced.  Shared layout is [slot][line].
#pragma once
#include "common.cuh"

namespace n2c {

template <int R> __host__ __device__ constexpr int bitrev_c(int i) {
  int r = 0;
  for (int b = 1, rb = R >> 1; b < R; b <<= 1, rb >>= 1)
    if (i & b) r |= rb;
  return r;
}

// Bit-reversal permutation of a register array, unrolled at compile time.
template <int R, int I, typename C>
__device__ __forceinline__ void bitrev_perm(C (&a)[R]) {
  if constexpr (I < R) {
    constexpr int J = bitrev_c<R>(I);
    if constexpr (I < J) { C t = a[I]; a[I] = a[J]; a[J] = t; }
    bitrev_perm<R, I + 1>(a);
  }
}

// v * W_SPAN^k (W_SPAN = exp(-2 pi i / SPAN); conjugated when INV) for the
// butterflies of spans up to 16, whose roots are the constants below (cos and
// sin of multiples of pi/8), so a register DFT of up to 16 points reads no
// twiddle table: the quarter-turn factors become swaps, the others one
// complex multiply by a literal.  Larger spans read the table (root
// tw[k * (R / SPAN) * STRIDE]).
template <int SPAN, int K, bool INV, typename C>
__device__ __forceinline__ C root_mul(C v) {
  using R = decltype(v.x);
  constexpr double c8 = 0.92387953251128674, s8 = 0.38268343236508977, h = 0.70710678118654752;
  // Angle index on the 16-point circle: W_SPAN^K = W_16^(K * 16 / SPAN).
  constexpr int m = K * (16 / SPAN);
  C r;
  if constexpr (m == 4) {                        // -i (forward) / +i (inverse)
    if (INV) { r.x = -v.y; r.y = v.x; } else { r.x = v.y; r.y = -v.x; }
    return r;
  } else {
    constexpr double wr = m == 1 ? c8 : m == 2 ? h : m == 3 ? s8 : m == 5 ? -s8 : m == 6 ? -h : -c8;
    constexpr double wi = m == 1 ? -s8 : m == 2 ? -h : m == 3 ? -c8 : m == 5 ? -c8 : m == 6 ? -h : -s8;
    C w;
    w.x = (R)wr;
    w.y = INV ? (R)-wi : (R)wi;
    return cmul(v, w);
  }
}

template <int SPAN, int K, bool INV, typename C>
__device__ __forceinline__ void span_butterflies(C *a, int base) {
  if constexpr (K < SPAN / 2) {
    C u = a[base + K], v = a[base + K + SPAN / 2];
    if constexpr (K != 0) v = root_mul<SPAN, K, INV>(v);
    a[base + K] = cadd(u, v);
    a[base + K + SPAN / 2] = csub(u, v);
    span_butterflies<SPAN, K + 1, INV>(a, base);
  }
}

// Butterflies of one radix-2 stage (span SPAN) and, recursively, the rest.
template <int R, bool INV, int STRIDE, int SPAN, typename C>
__device__ __forceinline__ void dit_stages(C (&a)[R], const C *__restrict__ tw) {
  if constexpr (SPAN <= R) {
    constexpr int HALF = SPAN / 2;
    if constexpr (SPAN <= 16) {
#pragma unroll
      for (int base = 0; base < R; base += SPAN) span_butterflies<SPAN, 0, INV>(a, base);
    } else {
#pragma unroll
      for (int base = 0; base < R; base += SPAN) {
#pragma unroll
        for (int k = 0; k < HALF; ++k) {
          C u = a[base + k], v = a[base + k + HALF];
          if (k != 0) {
            C w = __ldg(&tw[k * (R / SPAN) * STRIDE]);
            if (INV) w.y = -w.y;
            v = cmul(v, w);
          }
          a[base + k] = cadd(u, v);
          a[base + k + HALF] = csub(u, v);
        }
      }
    }
    dit_stages<R, INV, STRIDE, SPAN * 2>(a, tw);
  }
}

// In-register radix-2 DIT DFT of R points (natural-order output).
// tw[m] = exp(-2 pi i m / L); the R-point root W_R^m is tw[m * STRIDE].
template <int R, bool INV, int STRIDE, typename C>
__device__ __forceinline__ void dft_reg(C (&a)[R], const C *__restrict__ tw) {
  bitrev_perm<R, 0>(a);
  dit_stages<R, INV, STRIDE, 2>(a, tw);
}

template <typename C> struct PassArgs {
  const C *in;
  C *out;
  const C *tw;        // exp(-2 pi i m / L), m < L
  const C *spec;      // product pass: 6 spectrum slots (xx yy zz xy xz yz)
  long long lines;    // number of lines (B * I)
  long long I;        // distance between consecutive axis elements (1 = contiguous lines)
  long long A_in, A_out;        // axis extent stored in the input / output array
  int n_in, n_out;    // nonzero inputs (rest is zero padding) / outputs kept
  int NL;             // lines per tile
  // Strided passes: pow2 = 1 when NL and I (and, for the product pass, Pz)
  // are powers of two, whose logarithms follow; the index arithmetic then
  // shifts instead of dividing by runtime values.
  int pow2, nl_log2, i_log2, pz_log2;
  const int *gate;    // skip all work when *gate == 0 (NULL: always run)
  long long comp_in, comp_out;  // product pass: distance between the 3 components
  long long spec_comp;          // product pass: distance between spectrum slots
  int Py, Pz, Hy, Hz;           // product pass: padded y/z extents, octant extents
  // Cell I/O of the z passes (scatter on the forward load, permittivity
  // epilogue on the inverse store).  Lines are (component, x, y) of the box.
  const double2 *cx;            // cell vector x (3 per cell)
  double2 *cy;                  // cell vector y (3 per cell)
  const double2 *eps;           // per-cell permittivity
  const int *box_cell;          // box index -> cell (-1: empty)
  int box_identity;             // z passes: box_cell is the identity (not read)
  double2 self0, self1, self2;  // self terms of the Jacobi divisor
  long long nxy, mirror;        // lines per component; PEC physical cells (0: none)
  int precondition;             // input is v, the operator acts on v ./ diag
  int *flag;                    // non-finite input / output
  double *partials, *norm;      // |y|^2 reduction (norm NULL: none)
  unsigned int *ticket;
  // z passes: reciprocals ceil(2^32 / d) of the tile height NL, the lattice
  // columns per cell tile NP = NL / 3 and n_out, so that the index arithmetic
  // divides by a multiply-high (exact for the indices of a tile); 0 when
  // d == 1.
  unsigned nl_div, np_div, nout_div;
};

// n / d for 0 <= n < 2^32 / d through the reciprocal m = ceil(2^32 / d)
// (m == 0 stands for d == 1).
__device__ __forceinline__ int fdiv(int n, unsigned m) { return m ? (int)__umulhi((unsigned)n, m) : n; }

// z / d with one real division: conj(d) z / |d|^2 (the split-precision form,
// whose transforms are FP32 anyway; the FP64 form divides as C99 does).
__device__ __forceinline__ double2 cdiv_once(double2 z, double2 d) {
  const double r = 1.0 / (d.x * d.x + d.y * d.y);
  return make_double2((z.x * d.x + z.y * d.y) * r, (z.y * d.x - z.x * d.y) * r);
}
template <typename C> __device__ __forceinline__ double2 jacobi_apply(double2 v, double2 d) {
  return sizeof(C) == sizeof(float2) ? cdiv_once(v, d) : cdiv(v, d);
}

template <typename C> __device__ __forceinline__ double2 jacobi_divisor(const PassArgs<C> &a, double2 e, int c) {
  const double2 s = c == 0 ? a.self0 : (c == 1 ? a.self1 : a.self2);
  const double2 em1 = make_double2(e.x - 1.0, e.y);
  return csub(e, cmul(em1, s));
}

// Source value of box element e of line l (scatter with the Jacobi divisor
// and the PEC image sign diag(-1,-1,+1)).
template <typename C>
__device__ __forceinline__ C cell_load(const PassArgs<C> &a, long long l, int e) {
  const long long comp = l / a.nxy, xy = l - comp * a.nxy;
  long long cell = a.box_cell[xy * a.A_in + e];
  if (cell < 0) return czero<C>();
  double sgn = 1;
  if (a.mirror && cell >= a.mirror) { cell -= a.mirror; if (comp < 2) sgn = -1; }
  double2 v = a.cx[3 * cell + comp];
  if (a.precondition) v = cdiv(v, jacobi_divisor(a, a.eps[cell], (int)comp));
  if (a.flag && !finite2(v)) *a.flag = 1;
  return from_d<C>(make_double2(sgn * v.x, sgn * v.y));
}

// Epilogue y = eps z - (eps-1) field of box element e of line l; returns |y|^2.
template <typename C>
__device__ __forceinline__ double cell_store(const PassArgs<C> &a, long long l, int e, C field) {
  const long long comp = l / a.nxy, xy = l - comp * a.nxy;
  const long long cell = a.box_cell[xy * a.A_out + e];
  if (cell < 0 || (a.mirror && cell >= a.mirror)) return 0;
  const double2 ep = a.eps[cell], em1 = make_double2(ep.x - 1.0, ep.y);
  double2 z = a.cx[3 * cell + comp];
  if (a.precondition) z = cdiv(z, jacobi_divisor(a, ep, (int)comp));
  const double2 v = csub(cmul(ep, z), cmul(em1, to_d(field)));
  a.cy[3 * cell + comp] = v;
  if (a.flag && !finite2(v)) *a.flag = 1;
  return v.x * v.x + v.y * v.y;
}

// The transformed Green tensor is even (xx yy zz) or odd (xy: x,y; xz: x,z;
// yz: y,z) in every axis, so only the octant k <= P/2 per axis is stored:
// Ghat(k) = sign * Ghat(fold(k)), fold(k) = min(k, P-k).
struct Fold {
  int idx;     // folded index
  float sgn;   // -1 when k > P/2
};
__device__ __forceinline__ Fold fold(int k, int P) {
  Fold f;
  if (2 * k > P) { f.idx = P - k; f.sgn = -1.f; } else { f.idx = k; f.sgn = 1.f; }
  return f;
}

// x / NL for the strided passes' work items.
template <typename C> __device__ __forceinline__ int div_nl(const PassArgs<C> &a, int x) {
  return a.pow2 ? x >> a.nl_log2 : x / a.NL;
}

template <typename C>
__device__ __forceinline__ void line_base(const PassArgs<C> &a, long long l, long long &bin, long long &bout) {
  const long long b = a.pow2 ? l >> a.i_log2 : l / a.I, i = l - b * a.I;
  bin = b * a.A_in * a.I + i;
  bout = b * a.A_out * a.I + i;
}

// Forward transform of one component per tile (CELLS: loads scatter the cell
// vector, see cell_load).
template <typename C, int R1, int R2, bool CELLS = false>
__device__ __forceinline__ void fft_forward_tile(const PassArgs<C> &a, long long tile) {
  if (a.gate && *(volatile const int *)a.gate == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *S = reinterpret_cast<C *>(smem_raw);
  const int NL = a.NL;
  const long long l0 = tile * NL;
  for (int item = threadIdx.x; item < NL * R2; item += blockDim.x) {
    const int t = item & (NL - 1), j2 = div_nl(a, item);
    const long long l = l0 + t;
    if (l >= a.lines) continue;
    long long bin, bout;
    line_base(a, l, bin, bout);
    C v[R1];
#pragma unroll
    for (int j1 = 0; j1 < R1; ++j1) {
      const int e = j2 + R2 * j1;
      if (CELLS) v[j1] = e < a.n_in ? cell_load(a, l, e) : czero<C>();
      else v[j1] = e < a.n_in ? a.in[bin + (long long)e * a.I] : czero<C>();
    }
    dft_reg<R1, false, R2>(v, a.tw);
#pragma unroll
    for (int k1 = 1; k1 < R1; ++k1)
      if (j2) v[k1] = cmul(v[k1], __ldg(&a.tw[j2 * k1]));
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) S[(j2 + R2 * k1) * NL + t] = v[k1];
  }
  __syncthreads();
  for (int item = threadIdx.x; item < NL * R1; item += blockDim.x) {
    const int t = item & (NL - 1), k1 = div_nl(a, item);
    const long long l = l0 + t;
    if (l >= a.lines) continue;
    long long bin, bout;
    line_base(a, l, bin, bout);
    C w[R2];
#pragma unroll
    for (int j2 = 0; j2 < R2; ++j2) w[j2] = S[(j2 + R2 * k1) * NL + t];
    dft_reg<R2, false, R1>(w, a.tw);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) {
      const int e = k1 + R1 * k2;
      if (e < a.n_out) a.out[bout + (long long)e * a.I] = w[k2];
    }
  }
}
template <typename C, int R1, int R2, bool CELLS = false>
__global__ void __launch_bounds__(256) fft_forward_pass(PassArgs<C> a) {
  pdl_begin();
  fft_forward_tile<C, R1, R2, CELLS>(a, blockIdx.x);
}

// Inverse transform (unnormalised) of one component per tile (CELLS: stores
// run the permittivity epilogue into the cell vector and reduce |y|^2).
template <typename C, int R1, int R2, bool CELLS = false>
__device__ __forceinline__ void fft_inverse_tile(const PassArgs<C> &a, long long tile, unsigned ntiles) {
  if (a.gate && *(volatile const int *)a.gate == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *S = reinterpret_cast<C *>(smem_raw);
  const int NL = a.NL;
  const long long l0 = tile * NL;
  double sq = 0;
  for (int item = threadIdx.x; item < NL * R1; item += blockDim.x) {
    const int t = item & (NL - 1), k1 = div_nl(a, item);
    const long long l = l0 + t;
    if (l >= a.lines) continue;
    long long bin, bout;
    line_base(a, l, bin, bout);
    C w[R2];
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) {
      const int e = k1 + R1 * k2;
      w[k2] = e < a.n_in ? a.in[bin + (long long)e * a.I] : czero<C>();
    }
    dft_reg<R2, true, R1>(w, a.tw);
#pragma unroll
    for (int n1 = 1; n1 < R2; ++n1)
      if (k1) w[n1] = cmulc(w[n1], __ldg(&a.tw[n1 * k1]));
#pragma unroll
    for (int n1 = 0; n1 < R2; ++n1) S[(n1 + R2 * k1) * NL + t] = w[n1];
  }
  __syncthreads();
  for (int item = threadIdx.x; item < NL * R2; item += blockDim.x) {
    const int t = item & (NL - 1), n1 = div_nl(a, item);
    const long long l = l0 + t;
    if (l >= a.lines) continue;
    long long bin, bout;
    line_base(a, l, bin, bout);
    C v[R1];
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) v[k1] = S[(n1 + R2 * k1) * NL + t];
    dft_reg<R1, true, R2>(v, a.tw);
#pragma unroll
    for (int n2 = 0; n2 < R1; ++n2) {
      const int e = n1 + R2 * n2;
      if (e < a.n_out) {
        if (CELLS) sq += cell_store(a, l, e, v[n2]);
        else a.out[bout + (long long)e * a.I] = v[n2];
      }
    }
  }
  if (CELLS && a.norm) {
    // Deterministic |y|^2: block partials summed by the last block.
    const double2 bs = block_sum(make_double2(sq, 0));
    if (threadIdx.x == 0) a.partials[tile] = bs.x;
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(a.ticket, 1u) == ntiles - 1;
    __syncthreads();
    if (last) {
      double t2 = 0;
      for (unsigned i = threadIdx.x; i < ntiles; i += blockDim.x) t2 += a.partials[i];
      const double2 tot = block_sum(make_double2(t2, 0));
      if (threadIdx.x == 0) { *a.norm = tot.x; *a.ticket = 0; }
    }
  }
}
template <typename C, int R1, int R2, bool CELLS = false>
__global__ void __launch_bounds__(256) fft_inverse_pass(PassArgs<C> a) {
  pdl_begin();
  fft_inverse_tile<C, R1, R2, CELLS>(a, blockIdx.x, gridDim.x);
}

// x-axis pass fused with the Green-tensor product: forward x-FFT of the three
// source components, 3x3 symmetric spectrum product per frequency point, and
// the inverse x-FFT, all on one tile of lines.  Lines are the (ky,kz) points
// (I = Py*Pz, one line per inner index, B = 1 per component).
template <typename C, int R1, int R2>
__device__ __forceinline__ void fft_product_tile(const PassArgs<C> &a, long long tile) {
  if (a.gate && *(volatile const int *)a.gate == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *S = reinterpret_cast<C *>(smem_raw);
  const int NL = a.NL, L = R1 * R2;
  const long long l0 = tile * NL;
  for (int item = threadIdx.x; item < 3 * NL * R2; item += blockDim.x) {
    const int c = div_nl(a, item) / R2, rem = item - c * NL * R2;
    const int t = rem & (NL - 1), j2 = div_nl(a, rem);
    const long long l = l0 + t;
    if (l >= a.lines) continue;
    const C *in = a.in + c * a.comp_in + l;
    C v[R1];
#pragma unroll
    for (int j1 = 0; j1 < R1; ++j1) {
      const int e = j2 + R2 * j1;
      v[j1] = e < a.n_in ? in[(long long)e * a.I] : czero<C>();
    }
    dft_reg<R1, false, R2>(v, a.tw);
#pragma unroll
    for (int k1 = 1; k1 < R1; ++k1)
      if (j2) v[k1] = cmul(v[k1], __ldg(&a.tw[j2 * k1]));
    C *Sc = S + c * L * NL;
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) Sc[(j2 + R2 * k1) * NL + t] = v[k1];
  }
  __syncthreads();
  for (int item = threadIdx.x; item < NL * R1; item += blockDim.x) {
    const int t = item & (NL - 1), k1 = div_nl(a, item);
    const long long l = l0 + t;
    if (l >= a.lines) continue;
    C s0[R2], s1[R2], s2[R2];
#pragma unroll
    for (int j2 = 0; j2 < R2; ++j2) {
      const int slot = (j2 + R2 * k1) * NL + t;
      s0[j2] = S[slot]; s1[j2] = S[L * NL + slot]; s2[j2] = S[2 * L * NL + slot];
    }
    dft_reg<R2, false, R1>(s0, a.tw);
    dft_reg<R2, false, R1>(s1, a.tw);
    dft_reg<R2, false, R1>(s2, a.tw);
    const int ky = (int)(a.pow2 ? l >> a.pz_log2 : l / a.Pz), kz = (int)(l - (long long)ky * a.Pz);
    const Fold fy = fold(ky, a.Py), fz = fold(kz, a.Pz);
    const long long yz = (long long)fy.idx * a.Hz + fz.idx;
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) {
      const Fold fx = fold(k1 + R1 * k2, L);
      const long long g = (long long)fx.idx * a.Hy * a.Hz + yz;
      const C gxx = a.spec[g], gyy = a.spec[a.spec_comp + g], gzz = a.spec[2 * a.spec_comp + g];
      const C gxy = cscale(a.spec[3 * a.spec_comp + g], fx.sgn * fy.sgn);
      const C gxz = cscale(a.spec[4 * a.spec_comp + g], fx.sgn * fz.sgn);
      const C gyz = cscale(a.spec[5 * a.spec_comp + g], fy.sgn * fz.sgn);
      const C x0 = s0[k2], x1 = s1[k2], x2 = s2[k2];
      s0[k2] = cadd(cadd(cmul(gxx, x0), cmul(gxy, x1)), cmul(gxz, x2));
      s1[k2] = cadd(cadd(cmul(gxy, x0), cmul(gyy, x1)), cmul(gyz, x2));
      s2[k2] = cadd(cadd(cmul(gxz, x0), cmul(gyz, x1)), cmul(gzz, x2));
    }
    dft_reg<R2, true, R1>(s0, a.tw);
    dft_reg<R2, true, R1>(s1, a.tw);
    dft_reg<R2, true, R1>(s2, a.tw);
#pragma unroll
    for (int n1 = 0; n1 < R2; ++n1) {
      if (k1 && n1) {
        const C w = __ldg(&a.tw[n1 * k1]);
        s0[n1] = cmulc(s0[n1], w); s1[n1] = cmulc(s1[n1], w); s2[n1] = cmulc(s2[n1], w);
      }
      const int slot = (n1 + R2 * k1) * NL + t;
      S[slot] = s0[n1]; S[L * NL + slot] = s1[n1]; S[2 * L * NL + slot] = s2[n1];
    }
  }
  __syncthreads();
  for (int item = threadIdx.x; item < 3 * NL * R2; item += blockDim.x) {
    const int c = div_nl(a, item) / R2, rem = item - c * NL * R2;
    const int t = rem & (NL - 1), n1 = div_nl(a, rem);
    const long long l = l0 + t;
    if (l >= a.lines) continue;
    const C *Sc = S + c * L * NL;
    C v[R1];
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) v[k1] = Sc[(n1 + R2 * k1) * NL + t];
    dft_reg<R1, true, R2>(v, a.tw);
    C *out = a.out + c * a.comp_out + l;
#pragma unroll
    for (int n2 = 0; n2 < R1; ++n2) {
      const int e = n1 + R2 * n2;
      if (e < a.n_out) out[(long long)e * a.I] = v[n2];
    }
  }
}
// Three CTAs per SM in FP32; two in FP64, whose three components of R2
// complex values per thread would otherwise spill.
template <typename C, int R1, int R2>
__global__ void __launch_bounds__(256, 2) fft_product_pass(PassArgs<C> a) {
  pdl_begin();
  fft_product_tile<C, R1, R2>(a, blockIdx.x);
}

}  // namespace n2c

namespace n2c {

// ---------------------------------------------------------------- z lines
// Passes along the contiguous axis.  The tile (NL lines of length L) is
// staged through shared memory with coalesced cooperative loads and stores,
// transformed in place with the four-step split using a second buffer, and
// written back.  Shared layout [slot][line] with a padded row (NL + 1).
//
// CELLS: the tile is NP lattice columns (x, y) x 3 components, line
// t = c * NP + p; loads scatter the cell vector (Jacobi divisor, PEC image
// sign), stores run the permittivity epilogue and reduce |y|^2.  Cell data are
// touched three components at a time, so those accesses are contiguous too.

// Forward four-step on shared memory: input natural order in S, output
// natural order in T.
template <typename C, int R1, int R2>
__device__ __forceinline__ void smem_forward(C *S, C *T, int NL, int NLP, unsigned nlm, const C *__restrict__ tw) {
  for (int item = threadIdx.x; item < NL * R2; item += blockDim.x) {
    const int j2 = fdiv(item, nlm), t = item - j2 * NL;
    C v[R1];
#pragma unroll
    for (int j1 = 0; j1 < R1; ++j1) v[j1] = S[(j2 + R2 * j1) * NLP + t];
    dft_reg<R1, false, R2>(v, tw);
#pragma unroll
    for (int k1 = 1; k1 < R1; ++k1)
      if (j2) v[k1] = cmul(v[k1], __ldg(&tw[j2 * k1]));
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) S[(j2 + R2 * k1) * NLP + t] = v[k1];
  }
  __syncthreads();
  for (int item = threadIdx.x; item < NL * R1; item += blockDim.x) {
    const int k1 = fdiv(item, nlm), t = item - k1 * NL;
    C w[R2];
#pragma unroll
    for (int j2 = 0; j2 < R2; ++j2) w[j2] = S[(j2 + R2 * k1) * NLP + t];
    dft_reg<R2, false, R1>(w, tw);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) T[(k1 + R1 * k2) * NLP + t] = w[k2];
  }
  __syncthreads();
}

// Inverse four-step (unnormalised): input natural order in S, output natural
// order in S (T is scratch).
template <typename C, int R1, int R2>
__device__ __forceinline__ void smem_inverse(C *S, C *T, int NL, int NLP, unsigned nlm, const C *__restrict__ tw) {
  for (int item = threadIdx.x; item < NL * R1; item += blockDim.x) {
    const int k1 = fdiv(item, nlm), t = item - k1 * NL;
    C w[R2];
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) w[k2] = S[(k1 + R1 * k2) * NLP + t];
    dft_reg<R2, true, R1>(w, tw);
#pragma unroll
    for (int n1 = 1; n1 < R2; ++n1)
      if (k1) w[n1] = cmulc(w[n1], __ldg(&tw[n1 * k1]));
#pragma unroll
    for (int n1 = 0; n1 < R2; ++n1) T[(n1 + R2 * k1) * NLP + t] = w[n1];
  }
  __syncthreads();
  for (int item = threadIdx.x; item < NL * R2; item += blockDim.x) {
    const int n1 = fdiv(item, nlm), t = item - n1 * NL;
    C v[R1];
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) v[k1] = T[(n1 + R2 * k1) * NLP + t];
    dft_reg<R1, true, R2>(v, tw);
#pragma unroll
    for (int n2 = 0; n2 < R1; ++n2) S[(n1 + R2 * n2) * NLP + t] = v[n2];
  }
  __syncthreads();
}

// Global line of tile line t: plain tiles hold lines l0 .. l0+NL-1; cell
// tiles hold NP lattice columns of all 3 component planes ([3][nxy][L]).
template <typename C>
__device__ __forceinline__ long long zline_global(const PassArgs<C> &a, bool cells, int NP, int t, long long tile) {
  if (!cells) {
    const long long l = tile * a.NL + t;
    return l < a.lines ? l : -1;
  }
  const int c = fdiv(t, a.np_div), p = t - c * NP;
  const long long pos = tile * NP + p;
  return pos < a.nxy ? c * a.nxy + pos : -1;
}

// CELLS: the forward pass loads from the cell vector and stores T1 rows; the
// inverse pass loads T1 rows and stores through the permittivity epilogue.
template <typename C, int R1, int R2, bool INV, bool CELLS>
__device__ __forceinline__ void fft_zline_tile(const PassArgs<C> &a, long long tile, unsigned ntiles) {
  if (a.gate && *(volatile const int *)a.gate == 0) return;
  constexpr int L = R1 * R2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NL = a.NL, NLP = NL + 1;
  C *S = reinterpret_cast<C *>(smem_raw);
  C *T = S + (size_t)L * NLP;
  const int NP = NL / 3;
  // ---- load
  if (CELLS && !INV) {
    // CH elements per thread with their loads issued together (box index ->
    // cell, then the cell's value and permittivity): two round trips per
    // chunk instead of two per element.
    constexpr int CH = 4;
    const long long p0 = tile * NP;
    const int total = NP * L * 3;
    for (int base = threadIdx.x; base < total; base += CH * blockDim.x) {
      int cell[CH];
#pragma unroll
      for (int i = 0; i < CH; ++i) {
        const int idx = base + i * blockDim.x;
        cell[i] = -1;
        if (idx < total) {
          const int rest = idx / 3, e = rest % L, p = rest / L;
          const long long pos = p0 + p;
          if (e < a.n_in && pos < a.nxy)
            cell[i] = a.box_identity ? (int)(pos * a.A_in + e) : a.box_cell[pos * a.A_in + e];
        }
      }
      double2 v[CH], ep[CH];
      bool neg[CH];
#pragma unroll
      for (int i = 0; i < CH; ++i) {
        neg[i] = false;
        if (cell[i] >= 0) {
          const int c = (base + i * blockDim.x) % 3;
          if (a.mirror && cell[i] >= a.mirror) { cell[i] -= (int)a.mirror; neg[i] = c < 2; }
          v[i] = a.cx[3 * (long long)cell[i] + c];
          if (a.precondition) ep[i] = a.eps[cell[i]];
        }
      }
#pragma unroll
      for (int i = 0; i < CH; ++i) {
        const int idx = base + i * blockDim.x;
        if (idx >= total) continue;
        const int c = idx % 3, rest = idx / 3, e = rest % L, p = rest / L;
        C val = czero<C>();
        if (cell[i] >= 0) {
          double2 w = v[i];
          if (a.precondition) w = jacobi_apply<C>(w, jacobi_divisor(a, ep[i], c));
          if (a.flag && !finite2(w)) *a.flag = 1;
          if (neg[i]) w = make_double2(-w.x, -w.y);
          val = from_d<C>(w);
        }
        S[e * NLP + c * NP + p] = val;
      }
    }
  } else {
#pragma unroll 4
    for (int idx = threadIdx.x; idx < NL * L; idx += blockDim.x) {
      const int t = idx / L, e = idx - t * L;
      const long long l = zline_global(a, CELLS, NP, t, tile);
      S[e * NLP + t] = (e < a.n_in && l >= 0) ? a.in[l * a.A_in + e] : czero<C>();
    }
  }
  __syncthreads();
  C *R = S;
  if (INV) smem_inverse<C, R1, R2>(S, T, NL, NLP, a.nl_div, a.tw);
  else { smem_forward<C, R1, R2>(S, T, NL, NLP, a.nl_div, a.tw); R = T; }
  // ---- store
  if (CELLS && INV) {
    double sq = 0;
    const long long p0 = tile * NP;
    constexpr int CH = 4;   // outputs per thread whose loads are issued together
    const int total = NP * a.n_out * 3;
    for (int base = threadIdx.x; base < total; base += CH * blockDim.x) {
      int cell[CH];
#pragma unroll
      for (int i = 0; i < CH; ++i) {
        const int idx = base + i * blockDim.x;
        cell[i] = -1;
        if (idx < total) {
          const int rest = idx / 3, p = fdiv(rest, a.nout_div), e = rest - p * a.n_out;
          const long long pos = p0 + p;
          if (pos < a.nxy) {
            const int cl = a.box_identity ? (int)(pos * a.A_out + e) : a.box_cell[pos * a.A_out + e];
            if (cl >= 0 && !(a.mirror && cl >= a.mirror)) cell[i] = cl;
          }
        }
      }
      double2 ep[CH], z[CH];
#pragma unroll
      for (int i = 0; i < CH; ++i) {
        if (cell[i] < 0) continue;
        const int c = (base + i * blockDim.x) % 3;
        ep[i] = a.eps[cell[i]];
        z[i] = a.cx[3 * (long long)cell[i] + c];
      }
#pragma unroll
      for (int i = 0; i < CH; ++i) {
        if (cell[i] < 0) continue;
        const int idx = base + i * blockDim.x;
        const int c = idx % 3, rest = idx / 3, p = fdiv(rest, a.nout_div), e = rest - p * a.n_out;
        const double2 em1 = make_double2(ep[i].x - 1.0, ep[i].y);
        double2 zz = z[i];
        if (a.precondition) zz = jacobi_apply<C>(zz, jacobi_divisor(a, ep[i], c));
        const double2 v = csub(cmul(ep[i], zz), cmul(em1, to_d(R[e * NLP + c * NP + p])));
        a.cy[3 * (long long)cell[i] + c] = v;
        if (a.flag && !finite2(v)) *a.flag = 1;
        sq += v.x * v.x + v.y * v.y;
      }
    }
    if (a.norm) {
      const double2 bs = block_sum(make_double2(sq, 0));
      if (threadIdx.x == 0) a.partials[tile] = bs.x;
      __shared__ bool last;
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) last = atomicAdd(a.ticket, 1u) == ntiles - 1;
      __syncthreads();
      if (last) {
        double t2 = 0;
        for (unsigned i = threadIdx.x; i < ntiles; i += blockDim.x) t2 += a.partials[i];
        const double2 tot = block_sum(make_double2(t2, 0));
        if (threadIdx.x == 0) { *a.norm = tot.x; *a.ticket = 0; }
      }
    }
  } else {
    for (int idx = threadIdx.x; idx < NL * a.n_out; idx += blockDim.x) {
      const int t = fdiv(idx, a.nout_div), e = idx - t * a.n_out;
      const long long l = zline_global(a, CELLS, NP, t, tile);
      if (l >= 0) a.out[l * a.A_out + e] = R[e * NLP + t];
    }
  }
}
template <typename C, int R1, int R2, bool INV, bool CELLS>
__global__ void __launch_bounds__(256, 3) fft_zline_pass(PassArgs<C> a) {
  pdl_begin();
  fft_zline_tile<C, R1, R2, INV, CELLS>(a, blockIdx.x, gridDim.x);
}

}  // namespace n2c

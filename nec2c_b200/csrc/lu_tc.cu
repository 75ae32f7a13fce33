// Trailing update of the split-precision LU on the 5th-generation tensor
// cores: C -= A B for complex FP32 blocks, C (M x N) and A (M x KB) row-major
// in the working matrix, B given as the packed real expansion of U12.
//
// A complex product is one real product over interleaved (re, im) values:
// with A read as an M x 2KB real matrix and B expanded to the 2KB x 2N real
// matrix [[Br, Bi], [-Bi, Br]] per (k, n) pair, the real result's columns
// 2n, 2n+1 are Re and Im of the complex C.  The expansion is stored K-major,
// one 2KB-float row per real column (Bt), split into hi and lo parts.
//
// Precision: every operand x is split as x = hi + lo with hi holding the top
// 11 significant bits (TF32-representable, low 13 mantissa bits cleared) and
// lo = x - hi exact in FP32; D = Ahi Bhi + Ahi Blo + Alo Bhi accumulates in
// FP32 in tensor memory (3xTF32), close to an FP32 product.
//
// One CTA per 128-row x 32-complex-column tile (97 KB of shared memory, two
// CTAs per SM beside other work), 256 threads: the threads
// stage A (split on the fly) and Bt (pre-split) into 128B-swizzled shared
// memory, one elected thread issues the 24 tcgen05.mma (8 K-steps x 3
// products, M=128 N=64 K=8), tcgen05.commit signals an mbarrier, and the
// eight warps read the accumulator back (tcgen05.ld: warp w its 32 lanes of
// quarter w%4, half the columns per warpgroup) and update C.
// No cluster, no multicast.
//
// The persistent form below (gemm_tf32x3_tma_kernel) feeds the same products
// by TMA and overlaps them with the C update; n2c_tc_form says which form the
// LU uses (the staged one by default).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdlib.h>
#include <stdint.h>
#include <string.h>
#include "common.cuh"
#include "device_api.h"
#include "runtime.cuh"

namespace {

constexpr int TM = 128;             // tile rows
constexpr int TNC = 32;             // tile complex columns
constexpr int TN = 2 * TNC;         // tile real columns (MMA N)
constexpr int KR = 64;              // real K (2 x panel width 32)
constexpr int ATOM_ROW = 128;       // bytes per swizzle-atom row (32 floats)
constexpr int KATOMS = KR * 4 / ATOM_ROW;   // 2 atoms along K
constexpr int A_BYTES = KATOMS * TM * ATOM_ROW;   // 32 KB
constexpr int B_BYTES = KATOMS * TN * ATOM_ROW;   // 16 KB
constexpr int SMEM_BYTES = 2 * A_BYTES + 2 * B_BYTES + 1024;   // + alignment slack
constexpr int THREADS = 256;      // two warpgroups: staging and epilogue split between them
constexpr uint32_t TMEM_COLS = TN;   // 64 accumulator columns

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of 16-byte chunk c (0..15 along K) of row r in a K-major
// operand region of `rows` rows: K atoms of rows x 128 B, 128B swizzle
// (chunk index XOR row mod 8 within each 1024-byte group of 8 rows).
__device__ __forceinline__ uint32_t swz(int r, int c, int rows) {
  const int atom = c >> 3, cc = c & 7;
  return (uint32_t)(atom * rows * ATOM_ROW + r * ATOM_ROW + ((cc ^ (r & 7)) << 4));
}

// Shared-memory matrix descriptor: K-major, 128B swizzle, 8-row groups 1024 B
// apart, descriptor version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor, kind::tf32: D F32, A and B TF32, both K-major.
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n"
      :: "r"(tmem), "l"(a), "l"(b), "r"(IDESC), "r"(accumulate));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
  return ok != 0;
}

// One 128 x 32-complex tile at (r0, c0) of C (the body of the staged form).
__device__ __forceinline__ void tf32x3_tile(float2 *C, long long ldc, const float2 *A, long long lda,
                                            const float *bt_hi, const float *bt_lo, long long M, long long N,
                                            int *error, long long wait_cycles, long long r0, long long c0) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ uint32_t tmem_base;
  __shared__ __align__(8) unsigned long long done_bar;
  unsigned char *sm = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char *a_hi = sm, *a_lo = sm + A_BYTES, *b_hi = sm + 2 * A_BYTES, *b_lo = sm + 2 * A_BYTES + B_BYTES;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&tmem_base)), "r"(TMEM_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&done_bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // A: TM rows x 16 chunks of 4 floats, split on the fly; loads batched
  // ahead of the shared-memory stores.
  constexpr int AQ = TM * 16 / THREADS;
#pragma unroll
  for (int b = 0; b < AQ; b += 4) {
    float4 v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int q = tid + (b + u) * THREADS, r = q >> 4, c = q & 15;
      v[u] = r0 + r < M ? *reinterpret_cast<const float4 *>(reinterpret_cast<const float *>(A + (r0 + r) * lda) + 4 * c)
                        : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int q = tid + (b + u) * THREADS, r = q >> 4, c = q & 15;
      const float4 h = make_float4(tf32_hi(v[u].x), tf32_hi(v[u].y), tf32_hi(v[u].z), tf32_hi(v[u].w));
      const float4 l = make_float4(v[u].x - h.x, v[u].y - h.y, v[u].z - h.z, v[u].w - h.w);
      const uint32_t off = swz(r, c, TM);
      *reinterpret_cast<float4 *>(a_hi + off) = h;
      *reinterpret_cast<float4 *>(a_lo + off) = l;
    }
  }
  // Bt: TN real rows x 16 chunks, hi and lo as stored.
  constexpr int BQ = TN * 16 / THREADS;
#pragma unroll
  for (int b = 0; b < BQ; b += 4) {
    float4 h[4], l[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int q = tid + (b + u) * THREADS, r = q >> 4, c = q & 15;
      const long long gr = 2 * c0 + r;
      h[u] = l[u] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (gr < 2 * N) {
        h[u] = *reinterpret_cast<const float4 *>(bt_hi + gr * KR + 4 * c);
        l[u] = *reinterpret_cast<const float4 *>(bt_lo + gr * KR + 4 * c);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int q = tid + (b + u) * THREADS, r = q >> 4, c = q & 15;
      const uint32_t off = swz(r, c, TN);
      *reinterpret_cast<float4 *>(b_hi + off) = h[u];
      *reinterpret_cast<float4 *>(b_lo + off) = l[u];
    }
  }
  // Generic-proxy shared-memory writes become visible to the tensor cores.
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  if (tid == 0) {
    const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo), bh = smem_u32(b_hi), bl = smem_u32(b_lo);
    uint32_t acc = 0;
    // 8 K-steps of 8 TF32 values (32 bytes): 4 per swizzle atom.
#pragma unroll
    for (int k = 0; k < KR / 8; ++k) {
      const uint32_t ao = (uint32_t)((k >> 2) * TM * ATOM_ROW + (k & 3) * 32);
      const uint32_t bo = (uint32_t)((k >> 2) * TN * ATOM_ROW + (k & 3) * 32);
      mma_tf32(tmem, sdesc(al + ao), sdesc(bh + bo), acc);
      acc = 1;
      mma_tf32(tmem, sdesc(ah + ao), sdesc(bl + bo), 1);
    }
#pragma unroll
    for (int k = 0; k < KR / 8; ++k) {
      const uint32_t ao = (uint32_t)((k >> 2) * TM * ATOM_ROW + (k & 3) * 32);
      const uint32_t bo = (uint32_t)((k >> 2) * TN * ATOM_ROW + (k & 3) * 32);
      mma_tf32(tmem, sdesc(ah + ao), sdesc(bh + bo), 1);
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(&done_bar)) : "memory");
  }
  // Bounded wait for the products (wait_cycles, about a second at boost
  // clock by default; zero gives up at once and takes the time-out path).
  bool ok = wait_cycles > 0;
  if (ok) {
    const uint32_t bar = smem_u32(&done_bar);
    const long long t0 = clock64();
    while (!mbar_try(bar, 0)) {
      if (clock64() - t0 > wait_cycles) { ok = false; break; }
    }
  }
  // Every thread takes the same path (tcgen05.ld is warp-aligned).
  ok = __syncthreads_and(ok) != 0;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    // Warp w reads tensor-memory lanes 32*(w%4).. (its rows) and the column
    // chunks of its warpgroup: chunks 0..3 for warps 0-3, 4..7 for warps 4-7.
    const int quarter = warp & 3, half = warp >> 2;
    const long long row = r0 + quarter * 32 + lane;
    float4 *crow = reinterpret_cast<float4 *>(C + row * ldc + c0);
#pragma unroll 1
    for (int jj = 0; jj < TN / 64; ++jj) {
      const int j = half * (TN / 64) + jj;   // 32-float chunk = 16 complex = 8 float4
      float4 cv[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const long long col = c0 + j * 16 + 2 * q;
        cv[q] = (row < M && col < N) ? crow[j * 8 + q] : make_float4(0.f, 0.f, 0.f, 0.f);
      }
      uint32_t d[32];
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(j * 32);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14,"
          " %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
            "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
            "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]),
            "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const long long col = c0 + j * 16 + 2 * q;
          float4 v = cv[q];
          v.x -= __uint_as_float(d[4 * q]);
          v.y -= __uint_as_float(d[4 * q + 1]);
          v.z -= __uint_as_float(d[4 * q + 2]);
          v.w -= __uint_as_float(d[4 * q + 3]);
          if (col + 1 < N) crow[j * 8 + q] = v;
          else if (col < N) reinterpret_cast<float2 *>(crow + j * 8 + q)[0] = make_float2(v.x, v.y);
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(error, 1);
    // Give the products in flight another bounded wait before the memory is freed.
    const uint32_t bar = smem_u32(&done_bar);
    const long long t0 = clock64();
    while (!mbar_try(bar, 0) && clock64() - t0 < (1LL << 31)) {
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

__global__ void __launch_bounds__(THREADS, 2)
gemm_tf32x3_kernel(float2 *C, long long ldc, const float2 *A, long long lda, const float *bt_hi, const float *bt_lo,
                   long long M, long long N, int *error, long long wait_cycles) {
  tf32x3_tile(C, ldc, A, lda, bt_hi, bt_lo, M, N, error, wait_cycles, (long long)blockIdx.y * TM,
              (long long)blockIdx.x * TNC);
}

// Lockstep batch (grid.z = matrix): the trailing update of panel step k0 of
// every matrix of a batch of split-precision factorisations, part 0 the next
// panel's 32 columns, part 1 the columns after them.  A matrix whose order is
// passed, or whose update has no tile at this block, leaves before touching
// tensor memory.
__global__ void __launch_bounds__(THREADS, 2)
gemm_tf32x3_batch_kernel(const N2cTcBatch *e, long long k0, int part, int *error, long long wait_cycles) {
  const N2cTcBatch m = e[blockIdx.z];
  if (m.n <= k0) return;
  const long long kb = m.n - k0 < TNC ? m.n - k0 : TNC;
  const long long right = m.n - k0 - kb, nb = right < TNC ? right : TNC;
  const long long cf = k0 + kb + (part ? nb : 0), cols = part ? right - nb : nb;
  const long long r0 = (long long)blockIdx.y * TM, c0 = (long long)blockIdx.x * TNC;
  if (right <= 0 || cols <= 0 || r0 >= right || c0 >= cols) return;
  float2 *below = m.a + (k0 + kb) * m.ld;
  const long long r2 = 2 * (cf - k0 - kb);
  tf32x3_tile(below + cf, m.ld, below + k0, m.ld, m.bt_hi + r2 * KR, m.bt_lo + r2 * KR, right, cols, error,
              wait_cycles, r0, c0);
}


// ------------------------------------------------------------------------
// Persistent, TMA-fed form.  One CTA per SM holds one 128-row band of A (L21)
// in shared memory for all its column tiles, and runs three roles over its
// range of 128-real-column tiles (64 complex columns):
//   warp 0 (one lane)  TMA producer: the packed U12 tile (hi and lo, two
//                      128-byte swizzle atoms each) into a two-stage ring;
//   warp 1 (one lane)  MMA issuer: 24 tcgen05.mma.kind::tf32 (M128 N128 K8)
//                      per tile into one of two TMEM accumulators, then
//                      tcgen05.commit to the stage's "empty" and the
//                      accumulator's "full" mbarrier;
//   warps 4-11         epilogue: warp w reads tensor-memory lane quarter
//                      w % 4 and half the tile's columns (one warpgroup each),
//                      loads its C values before the products are done,
//                      subtracts the accumulator, stores C and arrives on the
//                      accumulator's "empty" mbarrier;
// so the products of tile i + 1 and the TMA of tile i + 2 overlap the C
// update of tile i.  A is loaded once per CTA by TMA as raw FP32 and split in
// place (hi: the TF32-representable top bits, lo: the FP32 remainder).
// Every wait is bounded; a time-out raises *error, every role leaves, the
// copies and products in flight are waited for (bounded) and the tensor
// memory is freed.  No cluster, no multicast.
constexpr int P_TN = 128;                              // tile real columns (MMA N)
constexpr int P_TNC = P_TN / 2;                        // tile complex columns
constexpr int P_A_BYTES = KATOMS * TM * ATOM_ROW;      // 32 KB per part (hi, lo)
constexpr int P_B_BYTES = KATOMS * P_TN * ATOM_ROW;    // 32 KB per part and stage
constexpr int P_STAGES = 2;
constexpr int P_SMEM_BYTES = 2 * P_A_BYTES + P_STAGES * 2 * P_B_BYTES + 1024;
constexpr uint32_t P_TMEM_COLS = 2 * P_TN;             // two accumulators
constexpr uint32_t P_IDESC =
    (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(P_TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
constexpr int P_THREADS = 384;                         // warps 0-1 producer / MMA, 4-11 epilogue
constexpr int P_EPI_WARP0 = 4;                         // warps 4-11: epilogue (two warpgroups)
constexpr int P_EPI_WARPS = 8;
constexpr long long DRAIN_CYCLES = 1LL << 31;          // bounded waits at teardown

__device__ __forceinline__ void mma_tf32_n(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n"
      :: "r"(tmem), "l"(a), "l"(b), "r"(P_IDESC), "r"(accumulate));
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      :: "r"(dst), "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive1(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(bar) : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar) : "memory");
}

// Bounded wait on phase parity; false on time-out or when another role has
// given up (*abort).  limit 0 gives up at once.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, long long limit,
                                                  const volatile int *abort) {
  if (limit <= 0) return false;
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (*abort || clock64() - t0 > limit) return false;
  }
  return true;
}

struct PersistentShared {
  unsigned long long a_full, b_full[P_STAGES], b_empty[P_STAGES], acc_full[2], acc_empty[2];
  uint32_t tmem_base;
  int abort;
  int issued, mma_done;        // B tiles whose TMA was issued; tiles whose products were issued
};

__global__ void __launch_bounds__(P_THREADS, 1)
gemm_tf32x3_tma_kernel(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_bh,
                       const __grid_constant__ CUtensorMap tm_bl, float2 *C, long long ldc, long long M, long long N,
                       int cpb, int *error, long long wait_cycles) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ PersistentShared sh;
  unsigned char *sm = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char *a_hi = sm, *a_lo = sm + P_A_BYTES, *b_base = sm + 2 * P_A_BYTES;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int band = blockIdx.x / cpb, part = blockIdx.x % cpb;
  const long long tiles = (N + P_TNC - 1) / P_TNC;
  const long long t_begin = tiles * part / cpb, t_end = tiles * (part + 1) / cpb;
  const int ntiles = (int)(t_end - t_begin);
  const long long r0 = (long long)band * TM;
  volatile int *abort = &sh.abort;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&sh.tmem_base)), "r"(P_TMEM_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&sh.a_full)) : "memory");
    for (int i = 0; i < P_STAGES; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&sh.b_full[i])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&sh.b_empty[i])) : "memory");
    }
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&sh.acc_full[i])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&sh.acc_empty[i])), "r"(P_EPI_WARPS)
                   : "memory");
    }
    sh.abort = 0;
    sh.issued = 0;
    sh.mma_done = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  // A band, raw FP32, by TMA (two swizzle atoms along K).
  if (tid == 0 && ntiles > 0) {
    const uint32_t bar = smem_u32(&sh.a_full);
    mbar_expect_tx(bar, P_A_BYTES);
    tma_load_2d(smem_u32(a_hi), &tm_a, 0, (int)r0, bar);
    tma_load_2d(smem_u32(a_hi + TM * ATOM_ROW), &tm_a, 32, (int)r0, bar);
  }
  bool ok = ntiles > 0 && mbar_wait_bounded(smem_u32(&sh.a_full), 0, wait_cycles, abort);
  ok = __syncthreads_and(ok) != 0;
  if (ok) {
    // Split in place: 32 KB of FP32 (layout-agnostic).
    float4 *hp = reinterpret_cast<float4 *>(a_hi), *lp = reinterpret_cast<float4 *>(a_lo);
    for (int i = tid; i < P_A_BYTES / 16; i += P_THREADS) {
      const float4 x = hp[i];
      const float4 h = make_float4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z), tf32_hi(x.w));
      hp[i] = h;
      lp[i] = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  } else if (tid == 0 && ntiles > 0) {
    atomicExch(error, 1);
    sh.abort = 1;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sh.tmem_base;

  if (ok && warp == 0 && lane == 0) {
    // ---- producer
    for (int it = 0; it < ntiles && !*abort; ++it) {
      const int st = it % P_STAGES;
      if (it >= P_STAGES &&
          !mbar_wait_bounded(smem_u32(&sh.b_empty[st]), (uint32_t)((it / P_STAGES - 1) & 1), wait_cycles, abort)) {
        atomicExch(error, 1);
        *abort = 1;
        break;
      }
      unsigned char *bh = b_base + st * 2 * P_B_BYTES, *bl = bh + P_B_BYTES;
      const uint32_t bar = smem_u32(&sh.b_full[st]);
      const int y = (int)(2 * (t_begin + it) * P_TNC);
      mbar_expect_tx(bar, 2 * P_B_BYTES);
      tma_load_2d(smem_u32(bh), &tm_bh, 0, y, bar);
      tma_load_2d(smem_u32(bh + P_TN * ATOM_ROW), &tm_bh, 32, y, bar);
      tma_load_2d(smem_u32(bl), &tm_bl, 0, y, bar);
      tma_load_2d(smem_u32(bl + P_TN * ATOM_ROW), &tm_bl, 32, y, bar);
      sh.issued = it + 1;
    }
  } else if (ok && warp == 1 && lane == 0) {
    // ---- MMA issuer
    const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
    for (int it = 0; it < ntiles && !*abort; ++it) {
      const int st = it % P_STAGES, buf = it & 1;
      if (!mbar_wait_bounded(smem_u32(&sh.b_full[st]), (uint32_t)((it / P_STAGES) & 1), wait_cycles, abort) ||
          (it >= 2 &&
           !mbar_wait_bounded(smem_u32(&sh.acc_empty[buf]), (uint32_t)((it / 2 - 1) & 1), wait_cycles, abort))) {
        atomicExch(error, 1);
        *abort = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t bh = smem_u32(b_base + st * 2 * P_B_BYTES), bl = bh + P_B_BYTES;
      const uint32_t d = tmem + (uint32_t)(buf * P_TN);
      uint32_t acc = 0;
#pragma unroll
      for (int k = 0; k < KR / 8; ++k) {
        const uint32_t ao = (uint32_t)((k >> 2) * TM * ATOM_ROW + (k & 3) * 32);
        const uint32_t bo = (uint32_t)((k >> 2) * P_TN * ATOM_ROW + (k & 3) * 32);
        mma_tf32_n(d, sdesc(al + ao), sdesc(bh + bo), acc);
        acc = 1;
        mma_tf32_n(d, sdesc(ah + ao), sdesc(bl + bo), 1);
      }
#pragma unroll
      for (int k = 0; k < KR / 8; ++k) {
        const uint32_t ao = (uint32_t)((k >> 2) * TM * ATOM_ROW + (k & 3) * 32);
        const uint32_t bo = (uint32_t)((k >> 2) * P_TN * ATOM_ROW + (k & 3) * 32);
        mma_tf32_n(d, sdesc(ah + ao), sdesc(bh + bo), 1);
      }
      mma_commit(smem_u32(&sh.b_empty[st]));
      mma_commit(smem_u32(&sh.acc_full[buf]));
      sh.mma_done = it + 1;
    }
  } else if (ok && warp >= P_EPI_WARP0) {
    // ---- epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. (its rows)
    // and the 32-float chunks 2h, 2h + 1 of the accumulator (h its warpgroup).
    const int quarter = warp & 3, half = (warp - P_EPI_WARP0) >> 2;
    const long long row = r0 + quarter * 32 + lane;
    for (int it = 0; it < ntiles; ++it) {
      const int buf = it & 1;
      const long long c0 = (t_begin + it) * P_TNC;
      float4 *crow = reinterpret_cast<float4 *>(C + row * ldc + c0);
      // C of both chunks, loaded while the products may still run.
      float4 cv[2][8];
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) {
        const int j = 2 * half + jj;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const long long col = c0 + j * 16 + 2 * q;
          cv[jj][q] = (row < M && col < N) ? crow[j * 8 + q] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
      bool got = mbar_wait_bounded(smem_u32(&sh.acc_full[buf]), (uint32_t)((it / 2) & 1), wait_cycles, abort);
      got = __all_sync(0xffffffffu, got);
      if (!got) {
        if (lane == 0) { atomicExch(error, 1); *abort = 1; }
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) {   // 32-float chunk = 16 complex = 8 float4
        const int j = 2 * half + jj;
        float4 *cv_j = cv[jj];
        uint32_t d[32];
        const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * P_TN + j * 32);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14,"
            " %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
              "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
              "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]),
              "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < M) {
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const long long col = c0 + j * 16 + 2 * q;
            float4 v = cv_j[q];
            v.x -= __uint_as_float(d[4 * q]);
            v.y -= __uint_as_float(d[4 * q + 1]);
            v.z -= __uint_as_float(d[4 * q + 2]);
            v.w -= __uint_as_float(d[4 * q + 3]);
            if (col + 1 < N) crow[j * 8 + q] = v;
            else if (col < N) reinterpret_cast<float2 *>(crow + j * 8 + q)[0] = make_float2(v.x, v.y);
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive1(smem_u32(&sh.acc_empty[buf]));
    }
  }
  __syncthreads();
  if (tid == 0 && ntiles > 0) {
    // Nothing may still write this CTA's shared or tensor memory: the A copy,
    // the last two B copies and the last products (bounded waits).
    const volatile int never = 0;
    mbar_wait_bounded(smem_u32(&sh.a_full), 0, DRAIN_CYCLES, &never);
    for (int it = sh.issued - P_STAGES < 0 ? 0 : sh.issued - P_STAGES; it < sh.issued; ++it)
      mbar_wait_bounded(smem_u32(&sh.b_full[it % P_STAGES]), (uint32_t)((it / P_STAGES) & 1), DRAIN_CYCLES, &never);
    if (sh.mma_done > 0) {
      const int last = sh.mma_done - 1;
      mbar_wait_bounded(smem_u32(&sh.acc_full[last & 1]), (uint32_t)((last / 2) & 1), DRAIN_CYCLES, &never);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(P_TMEM_COLS) : "memory");
  }
}

}  // namespace

// C (M x N complex FP32, row-major, leading dimension ldc in complex units)
// -= A (M x 32, lda) times the complex 32 x N block whose packed expansion is
// bt_hi + bt_lo (2N rows of 64 floats).  The rows of A and C must start
// 16-byte aligned (lda, ldc even; A, C 16-byte aligned).  error: device int
// set to 1 on a time-out; C is then left as it was.  The wait for the
// products is 2^31 clocks unless NEC2C_CUDA_TC_WAIT_CYCLES (read once) sets
// another limit; 0 makes every launch take the time-out path, which is how the
// tests exercise it.
static long long tc_wait_cycles() {
  const char *v = getenv("NEC2C_CUDA_TC_WAIT_CYCLES");
  if (!v || !*v) return 1LL << 31;
  char *end = nullptr;
  const long long c = strtoll(v, &end, 10);
  return (end && *end == 0 && c >= 0) ? c : 1LL << 31;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda); null when the driver does not offer it.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    cudaGetLastError();
    return (PFN_cuTensorMapEncodeTiled_v12000)f;
  }();
  return fn;
}

// A rows x 64-float K-major operand (row stride `stride` bytes) as a tensor
// map of 32-float x 128-row boxes with the 128-byte swizzle the MMA
// descriptors expect; rows beyond `rows` read as zeros.
static bool encode_operand(CUtensorMap *map, const float *base, long long rows, long long stride) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)KR, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)stride};
  const cuuint32_t box[2] = {32, (cuuint32_t)TM};
  const cuuint32_t estr[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)base, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Streaming multiprocessors of the current device (cached per device).
static int sm_count() {
  static int counts[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!counts[dev]) {
    int c = 0;
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    counts[dev] = c > 0 ? c : 148;
  }
  return counts[dev];
}

// The persistent form: bands of 128 rows, each split into cpb CTAs over its
// column tiles, at most (SMs - 16) CTAs so that the look-ahead panel's
// cluster (up to 16 CTAs) always finds SMs while the update runs.  Returns
// 1 launched, 0 failed (error set), -1 not available here.
static int launch_persistent(float *C, long long ldc, const float *A, long long lda, const float *bt_hi,
                             const float *bt_lo, long long M, long long N, int *error, long long wait_cycles,
                             cudaStream_t s) {
  CUtensorMap ta, tbh, tbl;
  if (!encode_operand(&ta, A, M, lda * (long long)sizeof(float2)) ||
      !encode_operand(&tbh, bt_hi, 2 * N, KR * (long long)sizeof(float)) ||
      !encode_operand(&tbl, bt_lo, 2 * N, KR * (long long)sizeof(float)))
    return -1;
  static const bool configured =
      cudaFuncSetAttribute(gemm_tf32x3_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, P_SMEM_BYTES) ==
      cudaSuccess;
  if (!configured) {
    n2c_set_error("tensor-core update: shared memory configuration failed");
    return 0;
  }
  const long long bands = (M + TM - 1) / TM, tiles = (N + P_TNC - 1) / P_TNC;
  const long long room = sm_count() > 32 ? sm_count() - 16 : sm_count();
  long long cpb = room / bands;
  if (cpb < 1) cpb = 1;
  if (cpb > tiles) cpb = tiles;
  if (bands * cpb > 0x7fffffffLL) { n2c_set_error("tensor-core update grid too large"); return 0; }
  gemm_tf32x3_tma_kernel<<<(unsigned)(bands * cpb), P_THREADS, P_SMEM_BYTES, s>>>(
      ta, tbh, tbl, (float2 *)C, ldc, M, N, (int)cpb, error, wait_cycles);
  return n2c_check_launch("tensor-core update");
}

int n2c_tc_update_batch(const N2cTcBatch *e, int count, long long k0, int part, long long rows_max,
                        long long cols_max, int *error, cudaStream_t s) {
  if (rows_max <= 0 || cols_max <= 0 || count <= 0) return 1;
  static const bool configured =
      cudaFuncSetAttribute(gemm_tf32x3_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES) ==
      cudaSuccess;
  if (!configured) {
    n2c_set_error("batched tensor-core update: shared memory configuration failed");
    return 0;
  }
  static const long long wait_cycles = tc_wait_cycles();
  dim3 grid((unsigned)((cols_max + TNC - 1) / TNC), (unsigned)((rows_max + TM - 1) / TM), (unsigned)count);
  gemm_tf32x3_batch_kernel<<<grid, THREADS, SMEM_BYTES, s>>>(e, k0, part, error, wait_cycles);
  return n2c_check_launch("batched tensor-core update");
}

int n2c_tc_update(float *C, long long ldc, const float *A, long long lda, const float *bt_hi, const float *bt_lo,
                  long long M, long long N, int *error, cudaStream_t s, int form) {
  if (M <= 0 || N <= 0) return 1;
  if ((lda & 1) || (ldc & 1) || ((uintptr_t)A & 15) || ((uintptr_t)C & 15) || ((uintptr_t)bt_hi & 15) ||
      ((uintptr_t)bt_lo & 15)) {
    n2c_set_error("tensor-core update: operand and result rows must start 16-byte aligned");
    return 0;
  }
  static const bool configured =
      cudaFuncSetAttribute(gemm_tf32x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES) ==
      cudaSuccess;
  if (!configured) {
    n2c_set_error("tensor-core update: shared memory configuration failed");
    return 0;
  }
  static const long long wait_cycles = tc_wait_cycles();
  if (form == N2C_TC_PERSISTENT && M <= 0x7fffffffLL && 2 * N <= 0x7fffffffLL) {
    const int r = launch_persistent(C, ldc, A, lda, bt_hi, bt_lo, M, N, error, wait_cycles, s);
    if (r >= 0) return r;
    // r < 0: the tensor-map encoder is not available; the staged form runs.
  }
  dim3 grid((unsigned)((N + TNC - 1) / TNC), (unsigned)((M + TM - 1) / TM));
  gemm_tf32x3_kernel<<<grid, THREADS, SMEM_BYTES, s>>>((float2 *)C, ldc, (const float2 *)A, lda, bt_hi, bt_lo, M, N,
                                                       error, wait_cycles);
  return n2c_check_launch("tensor-core update");
}

// The form the LU's trailing updates take.  The staged form by default: the
// persistent form holds one CTA with 197 KB of shared memory on most SMs for
// the whole update, and the look-ahead panel's cluster then waits for SMs
// of one GPC to free up (measured: order 1984 factor 7.41 ms against
// 7.28 ms, order 3000 12.49 ms against 11.82 ms, although the large updates
// themselves run faster).  NEC2C_CUDA_TC_PERSISTENT=1 (read once) selects
// the persistent form for updates of at least 1024 x 1024.
int n2c_tc_form(long long M, long long N) {
  static const bool persistent = [] {
    const char *v = getenv("NEC2C_CUDA_TC_PERSISTENT");
    return v && v[0] == '1';
  }();
  return persistent && N >= 1024 && M >= 1024 ? N2C_TC_PERSISTENT : N2C_TC_STAGED;
}

extern "C" int n2d_gemm_tf32x3(float *C, long long ldc, const float *A, long long lda, const float *bt_hi,
                               const float *bt_lo, long long M, long long N, int *error) {
  return n2c_tc_update(C, ldc, A, lda, bt_hi, bt_lo, M, N, error, n2c_stream(), N2C_TC_STAGED);
}

extern "C" int n2d_gemm_tf32x3_persistent(float *C, long long ldc, const float *A, long long lda,
                                          const float *bt_hi, const float *bt_lo, long long M, long long N,
                                          int *error) {
  return n2c_tc_update(C, ldc, A, lda, bt_hi, bt_lo, M, N, error, n2c_stream(), N2C_TC_PERSISTENT);
}

// Internal C++ helpers shared by the .cu files of the backend.
#pragma once
#include <cuda_runtime.h>

cudaStream_t n2c_stream();
// Device int that operator kernels check first: when it reads 0 they return
// at once (set by the GMRES driver around its inner iterations; NULL = off).
const int *n2c_gate();
void n2c_count_launch(unsigned n);
// Checks cudaGetLastError after a launch; counts the launch on success.
int n2c_check_launch(const char *what);
int n2c_sm_count();
// Split-precision (3xTF32) tensor-core trailing update of the FP32 LU on
// stream s; see lu_tc.cu.
int n2c_tc_update(float *C, long long ldc, const float *A, long long lda, const float *bt_hi, const float *bt_lo,
                  long long M, long long N, int *error, cudaStream_t s);

// Deterministic block-partial reduction: each block stores its partial in
// partials[blockIdx.x]; the block that arrives last (ticket counter) sums the
// partials in index order and writes the total.  Returns true in that block.
namespace n2c {
__device__ __forceinline__ bool gated_off(const int *gate) { return gate && *(volatile const int *)gate == 0; }
__device__ __forceinline__ bool last_block_done(unsigned int *ticket) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned v = atomicAdd(ticket, 1u);
    last = (v == gridDim.x - 1);
  }
  __syncthreads();
  return last;
}
}  // namespace n2c

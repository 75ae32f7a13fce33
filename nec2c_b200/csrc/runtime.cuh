// Internal C++ helpers shared by the .cu files of the backend.
#pragma once
#include <cuda_runtime.h>

extern "C" void n2c_set_error(const char *fmt, ...);
cudaStream_t n2c_stream();
// Device int that operator kernels check first: when it reads 0 they return
// at once (set by the GMRES driver around its inner iterations; NULL = off).
const int *n2c_gate();
void n2c_count_launch(unsigned n);
// Checks cudaGetLastError after a launch; counts the launch on success.
int n2c_check_launch(const char *what);
int n2c_sm_count();
// Programmatic dependent launch in use (NEC2C_CUDA_PDL=0 turns it off; read
// once).  Kernels launched with it must call pdl_begin() (common.cuh) first.
bool n2c_pdl_enabled();

// Launches k on the current stream, with programmatic stream serialisation
// when enable and n2c_pdl_enabled(); checks and counts the launch like
// n2c_check_launch.
template <typename... KArgs, typename... Args>
int n2c_launch_pdl(bool enable, void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, const char *what,
                   Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = n2c_stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = enable && n2c_pdl_enabled() ? 1 : 0;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
  if (e != cudaSuccess) {
    cudaGetLastError();
    n2c_set_error("%s launch failed: %s", what, cudaGetErrorString(e));
    return 0;
  }
  return n2c_check_launch(what);
}
// Split-precision (3xTF32) tensor-core trailing update of the FP32 LU on
// stream s; see lu_tc.cu.
// form: N2C_TC_STAGED (thread-staged operands, one tile per CTA) or
// N2C_TC_PERSISTENT (TMA-fed, one CTA per SM over a band's tiles).
enum { N2C_TC_STAGED = 0, N2C_TC_PERSISTENT = 1 };
int n2c_tc_update(float *C, long long ldc, const float *A, long long lda, const float *bt_hi, const float *bt_lo,
                  long long M, long long N, int *error, cudaStream_t s, int form);
// The form the LU's trailing update of an M x N block takes.
int n2c_tc_form(long long M, long long N);
// One matrix of a lockstep batch of split-precision factorisations, as the
// batched tensor-core update reads it: the FP32 working matrix (leading dim
// ld complex, even; rows 16-byte aligned) and its packed U12 expansion.
struct N2cTcBatch {
  float2 *a;
  long long n, ld;
  const float *bt_hi, *bt_lo;
};
// The trailing updates of panel step k0 (panel width 32) of count matrices
// (entries e on the device): part 0 the next panel's columns, part 1 the
// rest; rows_max / cols_max bound every matrix's update block.
int n2c_tc_update_batch(const N2cTcBatch *e, int count, long long k0, int part, long long rows_max,
                        long long cols_max, int *error, cudaStream_t s);

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

// Pass descriptions of a volume plan for the batched launches (vie_batch.cu).
#pragma once
#include <stddef.h>
#include "fft_engine.cuh"
#include "vie_internal.cuh"

// The five matvec passes of plan p with the batch's tile heights (large
// tiles: the batch fills the GPU with many plans) and the default radix
// split: arguments (cell vectors left unset: the batched
// launch points them into the batch vectors), kernel mode, line length,
// dynamic shared memory and tiles.  precondition, norm and flag as in
// n2d_vie_apply.  Returns 0 with the error set when a pass cannot be
// described (norm reduction grid too large).
template <typename C>
int n2c_vie_pass_plans(n2d_vie *p, int precondition, double *norm, int *flag, n2c::PassArgs<C> args[5],
                       int mode[5], int L[5], size_t smem[5], long long tiles[5]);

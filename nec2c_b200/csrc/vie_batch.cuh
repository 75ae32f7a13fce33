// Pass descriptions of a volume plan for the batched launches (vie_batch.cu).
#pragma once
#include <stddef.h>
#include "fft_engine.cuh"
#include "vie_internal.cuh"

// The five matvec passes of plan p with the batch's tile heights (large
// tiles: the batch fills the GPU with many plans), scaled per pass by
// 2^scale[i] (-1, 0, +1; NULL: 0), and the default radix split, or the
// transposed one where variant[i] != 0 and the length has one (NULL: none):
// arguments (cell vectors left unset: the batched launch points them into the
// batch vectors), kernel mode, line length, radix variant, dynamic shared
// memory and tiles.  precondition, norm and flag as in n2d_vie_apply.
// Returns 0 with the error set when a pass cannot be described (norm
// reduction grid too large).
template <typename C>
int n2c_vie_pass_plans(n2d_vie *p, int precondition, double *norm, int *flag, const int *scale, const int *variant,
                       n2c::PassArgs<C> args[5], int mode[5], int L[5], int var[5], size_t smem[5], long long tiles[5]);

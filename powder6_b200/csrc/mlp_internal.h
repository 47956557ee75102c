// Device-side entry of the proposal network for the search kernels' host code.
#pragma once
#include <cuda_runtime.h>

#include "p6cuda.h"

namespace p6 {
namespace mlp {
// Inference (bf16 weights) of `rows` inputs at dX into dY, both device memory, on `st`.
p6_status predict_device(p6_mlp *n, const float *dX, int rows, float *dY, cudaStream_t st);
int input_dim(const p6_mlp *n);
int output_dim(const p6_mlp *n);
}  // namespace mlp
}  // namespace p6

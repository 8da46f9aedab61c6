// Launch interface of the escape-probability network kernels (mlp.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace nbx {
namespace mlp {

size_t train_smem_bytes();
// Accumulates the gradient of the mean BCE loss over samples
// [first, first + count) (rows index[i] if index is not null) into grad, and
// the loss into *loss; inv_batch = 1 / batch size.
cudaError_t launch_train(const float* params, const float* features, const float* labels, const uint32_t* index,
                         uint64_t first, uint64_t count, float inv_batch, float* grad, float* loss, cudaStream_t s);
cudaError_t launch_adam(float* params, const float* grad, float* m, float* v, float lr, float beta1, float beta2,
                        float eps, int step, cudaStream_t s);
cudaError_t launch_predict(const float* params, const float* features, uint64_t n, float* out, cudaStream_t s);

}  // namespace mlp
}  // namespace nbx

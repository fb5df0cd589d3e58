// lsm_batch_kernels.h - host launchers of the batch LSM kernels (lsm_batch_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "lsm_batch.cuh"

namespace fo {

constexpr int kBatchSimThreads = 256;
constexpr int kBatchBackwardThreads = 256;
constexpr int kBatchEvalThreads = 256;

cudaError_t launch_batch_simulate(const BatchArgs& a, cudaStream_t stream);
// backward_order holds the n_large problems above 64Ki paths first (clusters of four CTAs on
// `stream`), then the rest (one CTA each, on `side` between fork and join when side is not null).
cudaError_t launch_batch_backward(const BatchArgs& a, uint32_t n_large, cudaStream_t stream, cudaStream_t side,
                                  cudaEvent_t fork, cudaEvent_t join);
cudaError_t launch_batch_diagnose(const BatchArgs& a, uint32_t n_records, cudaStream_t stream);
// max_strikes: strikes of the widest group; max_rows: the largest observation-row count of the
// wave's groups (sizes the staged rules).
cudaError_t launch_batch_evaluate(const BatchArgs& a, uint32_t max_strikes, uint32_t max_rows, cudaStream_t stream);
// One block per (path block, group, strike): the adjoint Greeks variant of the evaluation.
cudaError_t launch_batch_evaluate_greeks(const BatchArgs& a, uint32_t max_strikes, uint32_t max_rows,
                                         cudaStream_t stream);
cudaError_t launch_batch_summarize(const BatchArgs& a, cudaStream_t stream);

}  // namespace fo

// lsm_batch_kernels.h - host interface of the persistent batch LSM kernel (lsm_persistent.cu).
#pragma once

#include <cuda_runtime.h>

#include "lsm_batch.cuh"

namespace fo {

constexpr int kBatchSimThreads = 256;
constexpr int kBatchBackwardThreads = 256;
constexpr int kBatchEvalThreads = 256;

// Launch shape of a persistent batch launch (lsm_persistent.cu). The autotuner picks it per shape
// class; the results do not depend on it.
struct BatchTuning {
    int sim_blocks = 2;   // training-simulation blocks of 256 paths per work item
    int eval_blocks = 1;  // evaluation blocks of 256 paths per work item
    int strikes = 8;      // strikes an evaluation item applies together (1, 2, 4 or 8)
    int ctas_per_sm = 0;  // resident CTAs per SM of the persistent launch (0: as many as fit)
    int phases = 0;       // 1: one kernel per item kind and a summary kernel instead of one launch
};

// Shared memory of the staged fitted rules: `strikes` x rule_rows PolicyRules, or with the Greeks
// one strike's rules and its per-row stopping counts.
size_t persistent_rule_bytes(int strikes, bool greeks, uint32_t rule_rows);
// One persistent launch over the queue q, in two steps so that the second can be captured into a
// CUDA graph: the kernel instance for the launch shape, its dynamic shared memory and its grid
// (resident CTAs, at most one per item), then the launch itself on `stream`.
struct PersistentLaunch {
    const void* kernel;
    size_t smem;
    int grid;
    int pad;
};
cudaError_t prepare_batch_persistent(const BatchArgs& a, const BatchQueue& q, int strikes, uint32_t rule_rows,
                                     bool stage, int ctas_per_sm, PersistentLaunch* out);
cudaError_t enqueue_batch_persistent(const PersistentLaunch& launch, const BatchArgs& a, const BatchQueue& q,
                                     uint32_t rule_rows, bool stage, cudaStream_t stream);
// The same items as kernels of one kind each (simulation, fits, evaluation), run in stream order:
// q[k] is phase k's part of the queue, and a fourth kernel writes every problem's summary. Each is
// launched with enqueue_batch_persistent.
cudaError_t prepare_batch_phases(const BatchArgs& a, const BatchQueue (&q)[3], int strikes, uint32_t rule_rows,
                                 bool stage, PersistentLaunch (&out)[4]);

}  // namespace fo

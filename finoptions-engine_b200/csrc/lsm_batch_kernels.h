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
    int ctas_per_sm = 0;  // resident CTAs per SM (0: as many as fit)
};

// Shared memory of the staged fitted rules: `strikes` x rule_rows PolicyRules, or with the Greeks
// one strike's rules and its per-row stopping counts.
size_t persistent_rule_bytes(int strikes, bool greeks, uint32_t rule_rows);
// One persistent launch over the queue q; *grid_out receives the CTAs launched.
cudaError_t launch_batch_persistent(const BatchArgs& a, const BatchQueue& q, int strikes, uint32_t rule_rows,
                                    bool stage, int ctas_per_sm, cudaStream_t stream, int* grid_out);

}  // namespace fo

// executor.h - the CudaExecutor object behind the C ABI handle and the device / pinned buffers
// it owns. Shared by the single-contract (capi.cu) and batch (lsm_grouped.cu) entry points.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <vector>
#include <mutex>
#include <string>

#include "../../include/finoptions_cuda.h"
#include "host.h"
#include "lsm_batch_kernels.h"

namespace fo {

inline Error cuda_error(cudaError_t e, const char* what) {
    return make_error(FO_ERR_EXECUTION, FO_CODE_CUDA_FAILURE,
                      std::string("CUDA failure in ") + what + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

#define FO_CUDA_TRY(expr, what)                             \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return ::fo::cuda_error(_e, what); \
    } while (0)

// Grow-only device buffer.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    Error reserve(size_t need) {
        if (need <= bytes) return Error{};
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        const size_t grow = std::max(need, size_t(1) << 20);
        cudaError_t e = cudaMalloc(&ptr, grow);
        if (e != cudaSuccess) return cuda_error(e, "cudaMalloc");
        bytes = grow;
        return Error{};
    }
    ~DeviceBuffer() {
        if (ptr) cudaFree(ptr);
    }
};

// Grow-only pinned host buffer.
struct PinnedBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    Error reserve(size_t need) {
        if (need <= bytes) return Error{};
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
        const size_t grow = std::max(need, size_t(1) << 16);
        cudaError_t e = cudaMallocHost(&ptr, grow);
        if (e != cudaSuccess) return cuda_error(e, "cudaMallocHost");
        bytes = grow;
        return Error{};
    }
    ~PinnedBuffer() {
        if (ptr) cudaFreeHost(ptr);
    }
};

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace fo

struct fo_executor {
    int device = 0;
    int sms = 0;
    int backward_blocks_max = 0;
    int backward_max_ppt = 0;
    int eval_blocks_per_sm = 0;
    cudaStream_t stream = nullptr;
    // Higher-priority side stream for work no later kernel reads on the device (the per-row
    // diagnostic), forked after the backward pass and joined before results are read back; null
    // for stack executors, which run it inline.
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    std::mutex mu;
    fo::DeviceBuffer slab;        // training path storage shared by this executor's plans (stream-ordered)
    fo::DeviceBuffer scratch;     // per-call block for one-shot calls
    fo::DeviceBuffer normals;     // caller standard normals of a host-buffer external-normal simulation
    fo::PinnedBuffer staging;     // one-shot upload / download staging
    fo::DeviceBuffer batch;       // batch arena (plans, records, values, outputs)
    fo::PinnedBuffer batch_host;  // batch upload / download staging
    cudaEvent_t batch_marks[FO_BATCH_KERNELS + 1] = {};  // per-kernel timing of batch waves
    double batch_ms[FO_BATCH_KERNELS] = {};              // last batch call, summed over waves
    uint64_t batch_launches = 0;
    uint64_t batch_h2d = 0, batch_d2h = 0;                // bytes copied by the last batch call
    fo::BatchTuning batch_tuning;                         // launch shape when the autotuner is off
    bool batch_autotune = true;                           // pick shapes per class (else batch_tuning)
    std::map<std::string, fo::BatchTuning> batch_tuned;   // autotuned shape per wave class
    fo::BatchTuning batch_tuning_used;                    // shape of the last batch launch
    int batch_tuning_source = 0;                          // 0 set by the caller, 1 cached, 2 tuned now
    uint64_t batch_tuning_runs = 0;                       // launches the last tuning timed
    int batch_grid = 0;                                   // CTAs of the last batch launch
    int batch_strikes = 0;                                // strikes per evaluation item of the last launch
    uint64_t batch_items = 0;                             // work items of the last launch
    // The last batch wave as a captured CUDA graph (table upload, resets, the persistent launch and
    // the read-back), replayed while a wave's launch key (addresses, sizes, launch arguments)
    // repeats; any other key captures again.
    cudaGraphExec_t batch_graph = nullptr;
    std::vector<unsigned char> batch_graph_key;
    uint64_t batch_graph_replays = 0, batch_graph_captures = 0;  // last batch call
    ~fo_executor() {
        if (batch_graph) cudaGraphExecDestroy(batch_graph);
        for (cudaEvent_t& e : batch_marks)
            if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
    }
};

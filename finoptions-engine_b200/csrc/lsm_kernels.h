// lsm_kernels.h - launch interface of the single-contract LSM kernels (host <-> device).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "lsm_device.cuh"

namespace fo {

constexpr int kBackwardThreads = 1024;
constexpr int kEvalThreads = 256;

struct BackwardArgs {
    DevicePlan plan;
    const double* slab;          // stored training rows [rows - first_stored_row, paths]
    double2* partials;           // [2][16][blocks] double-double CTA partials (ping-pong), slot-major
    size_t partial_stride;       // doubles2 per ping-pong half
    FitRecord* records;          // [rows]
    DeviceStatus* status;
    int ppt;                     // paths per thread
    double* values;              // NULL: values and spots on chip (shared memory); else [train paths]
                                 // values in HBM, spots read from the slab (populations beyond the
                                 // on-chip capacity)
};

struct EvalArgs {
    DevicePlan plan;
    const FitRecord* records;
    double2* partials;           // [blocks][2]
    unsigned* counts;            // [rows] stopping counts
    unsigned* itm_counts;        // [rows] active in-the-money paths at unsupported rows
    DeviceStatus* status;
    uint32_t* stops;             // optional [evaluation paths]: the row at which each path stopped
};

// Pathwise adjoint Greeks of the fused evaluation (lsm_greeks.cu).
constexpr int kMaxGreekDividends = 8;
constexpr int kGreekSlots = 32;
enum GreekSlot : int {
    kGreekDelta = 0,     // sum of dP/dS0
    kGreekVega = 1,      // sum of dP/dsigma
    kGreekL0 = 2,        // sum of dP/dL_0 (drift of the first step)
    kGreekTerminal = 3,  // sum of dP/dL_N at expiry stops (discount + last drift)
    kGreekJump = 4,      // [kMaxGreekDividends]: sums of dP/dL at each cash-dividend node
    kGreekDividend = kGreekJump + kMaxGreekDividends,  // [kMaxGreekDividends]: sums of dP/dD_j
};

struct GreeksArgs {
    uint32_t dividends;                         // cash dividends of the schedule, in node order
    uint32_t div_node[kMaxGreekDividends];
    double div_amount[kMaxGreekDividends];
    double sigma;
    const double* sqrt_dt;                      // [intervals]
    const double* dt;                           // [intervals]
    double2* partials;                          // [blocks][kGreekSlots] double-double block sums
};

cudaError_t launch_normals(uint64_t seed, uint32_t domain, uint32_t path_start, uint64_t paths, uint32_t count,
                           double* out, unsigned long long* fail, cudaStream_t stream);
cudaError_t launch_simulate(const DevicePlan& plan, uint64_t paths, uint64_t seed, uint32_t domain, double* out,
                            uint32_t store_first_row, int reconstruct_escrowed, unsigned long long* fail,
                            cudaStream_t stream);
cudaError_t launch_replay(const DevicePlan& plan, uint64_t seed, uint32_t domain, uint32_t path, int want_row,
                          SimFailure* out, cudaStream_t stream);
// External normals ([intervals, paths], time-major): the first non-finite value's index, the
// simulation, and the replay of one failing path.
cudaError_t launch_first_nonfinite(const double* values, uint64_t n, unsigned long long* first, cudaStream_t stream);
cudaError_t launch_simulate_external(const DevicePlan& plan, uint64_t paths, const double* normals, double* out,
                                     unsigned long long* fail, cudaStream_t stream);
cudaError_t launch_replay_external(const DevicePlan& plan, uint64_t paths, const double* normals, uint64_t path,
                                   SimFailure* out, cudaStream_t stream);
int backward_max_blocks(int device);
int backward_max_ppt();
size_t backward_smem_bytes(int ppt);
cudaError_t launch_backward(const BackwardArgs& args, int blocks, int ppt, cudaStream_t stream);
cudaError_t launch_diagnose(const DevicePlan& plan, FitRecord* records, cudaStream_t stream);
size_t evaluate_smem_bytes(uint32_t rows);
cudaError_t launch_evaluate(const EvalArgs& args, int blocks, cudaStream_t stream);
cudaError_t launch_finalize(const double2* partials, int blocks, uint64_t paths, double* out, cudaStream_t stream);
size_t evaluate_greeks_smem_bytes(uint32_t rows);
cudaError_t launch_evaluate_greeks(const EvalArgs& args, const GreeksArgs& greeks, int blocks, cudaStream_t stream);
cudaError_t launch_finalize_greeks(const double2* partials, int blocks, double* out, cudaStream_t stream);

}  // namespace fo

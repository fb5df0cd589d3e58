// wait_harness.cu - test harness: runs the backward kernel's bounded grid wait (lsm_sync.cuh
// wait_arrivals) on an arrival counter that nothing increments, and on one that has already reached
// its target. Built by tests/test_gpu_wait_timeout.py; test infrastructure only.
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../finoptions-engine_b200/csrc/lsm_sync.cuh"

namespace {

// One warp per block waits for `target` arrivals; lane 0 reports the outcome and the time taken.
__global__ void wait_kernel(fo::DeviceStatus* st, unsigned target, unsigned long long limit_ns, int* passed,
                            unsigned long long* elapsed_ns) {
    const unsigned long long t0 = fo::global_timer_ns();
    const bool ok = fo::wait_arrivals(st, target, limit_ns);
    if (threadIdx.x == 0) {
        passed[blockIdx.x] = ok ? 1 : 0;
        elapsed_ns[blockIdx.x] = fo::global_timer_ns() - t0;
    }
}

}  // namespace

// Returns 0 and fills the per-block results and the status word's timeout flag, or the CUDA error.
extern "C" int wait_check(unsigned arrivals, unsigned target, unsigned long long limit_ns, int blocks, int* passed,
                          unsigned long long* elapsed_ns, unsigned* timeout_flag) {
    fo::DeviceStatus* st = nullptr;
    int* d_passed = nullptr;
    unsigned long long* d_elapsed = nullptr;
    cudaError_t e = cudaMalloc(&st, sizeof(fo::DeviceStatus));
    if (e == cudaSuccess) e = cudaMalloc(&d_passed, sizeof(int) * blocks);
    if (e == cudaSuccess) e = cudaMalloc(&d_elapsed, sizeof(unsigned long long) * blocks);
    if (e == cudaSuccess) e = cudaMemset(st, 0, sizeof(fo::DeviceStatus));
    if (e == cudaSuccess)
        e = cudaMemcpy(reinterpret_cast<unsigned char*>(st) + offsetof(fo::DeviceStatus, arrivals), &arrivals,
                       sizeof(unsigned), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        wait_kernel<<<blocks, 32>>>(st, target, limit_ns, d_passed, d_elapsed);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(passed, d_passed, sizeof(int) * blocks, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(elapsed_ns, d_elapsed, sizeof(unsigned long long) * blocks, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(timeout_flag, reinterpret_cast<unsigned char*>(st) + offsetof(fo::DeviceStatus, barrier_timeout),
                       sizeof(unsigned), cudaMemcpyDeviceToHost);
    cudaFree(st);
    cudaFree(d_passed);
    cudaFree(d_elapsed);
    return int(e);
}

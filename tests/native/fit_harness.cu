// GPU harness: the warp-wide regression solve (lsm_fit_warp.cuh) against the one-thread solve
// (fit_continuation, fo_core.cuh) on the same reduced sums. One warp per case; both models start
// from the same byte pattern in shared memory, as the backward kernel's model does, and are copied
// out whole so the test can compare them byte for byte.
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../finoptions-engine_b200/csrc/lsm_fit_warp.cuh"

using namespace fo;

struct FitCase {
    dd sums[kMomentSlots];
    double pivot;
    uint64_t count;
    int degree;
    double rank_tolerance;
    double rank_limit;  // filled by fit_compare from rank_tolerance
};

__global__ void __launch_bounds__(32) compare_kernel(const FitCase* cases, int n, FitModel* one, FitModel* warp) {
    const int c = int(blockIdx.x);
    if (c >= n) return;
    __shared__ dd sums[kMomentSlots];
    __shared__ FitModel m_one, m_warp;
    if (threadIdx.x < kMomentSlots) sums[threadIdx.x] = cases[c].sums[threadIdx.x];
    unsigned char* a = reinterpret_cast<unsigned char*>(&m_one);
    unsigned char* b = reinterpret_cast<unsigned char*>(&m_warp);
    for (unsigned i = threadIdx.x; i < sizeof(FitModel); i += 32) {
        a[i] = 0xA5;
        b[i] = 0xA5;
    }
    __syncwarp();
    const FitCase& q = cases[c];
    if (threadIdx.x == 0) fit_continuation(sums, q.pivot, q.count, q.degree, q.rank_tolerance, &m_one);
    __syncwarp();
    fit_continuation_warp(sums, q.pivot, q.count, q.degree, q.rank_tolerance, q.rank_limit, &m_warp);
    if (threadIdx.x == 0) {
        one[c] = m_one;
        warp[c] = m_warp;
    }
}

extern "C" int fit_model_bytes() { return int(sizeof(FitModel)); }
extern "C" int fit_case_bytes() { return int(sizeof(FitCase)); }

// Runs `n` cases (host arrays); returns 0 or the CUDA error code.
extern "C" int fit_compare(const void* cases, int n, void* one, void* warp) {
    std::vector<FitCase> host(static_cast<const FitCase*>(cases), static_cast<const FitCase*>(cases) + n);
    for (FitCase& q : host) q.rank_limit = rank_limit(q.rank_tolerance);
    FitCase* d_cases = nullptr;
    FitModel *d_one = nullptr, *d_warp = nullptr;
    cudaError_t e = cudaMalloc(&d_cases, sizeof(FitCase) * size_t(n));
    if (e == cudaSuccess) e = cudaMalloc(&d_one, sizeof(FitModel) * size_t(n));
    if (e == cudaSuccess) e = cudaMalloc(&d_warp, sizeof(FitModel) * size_t(n));
    if (e == cudaSuccess) e = cudaMemcpy(d_cases, host.data(), sizeof(FitCase) * size_t(n), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        compare_kernel<<<n, 32>>>(d_cases, n, d_one, d_warp);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(one, d_one, sizeof(FitModel) * size_t(n), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(warp, d_warp, sizeof(FitModel) * size_t(n), cudaMemcpyDeviceToHost);
    cudaFree(d_cases);
    cudaFree(d_one);
    cudaFree(d_warp);
    return int(e);
}

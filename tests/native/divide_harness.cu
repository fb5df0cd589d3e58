// divide_harness.cu - test harness: compares the engine's corrected division (fo_core.cuh divide /
// make_divisor) with IEEE binary64 division on the device, over counter-generated operands.
// Built by tests/test_gpu_divide.py with the engine's flags (-fmad=false); test infrastructure only.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../finoptions-engine_b200/csrc/fo_core.cuh"

namespace {

__device__ uint64_t mix(uint64_t x) {  // SplitMix64 finaliser
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

__device__ double uniform(uint64_t bits) { return double(bits >> 11) * 0x1p-53; }

// Operand families: 0 spot / strike (log-uniform 1e-3..1e5 over 1e-2..1e4), 1 centred predictor /
// scale, 2 divisors with an all-ones significand, 3 numerators just around powers of two.
__device__ void operands(uint64_t i, int family, double* a, double* b) {
    const uint64_t r0 = mix(2 * i), r1 = mix(2 * i + 1);
    switch (family) {
        case 0:
            *a = exp(log(1e-3) + uniform(r0) * (log(1e5) - log(1e-3)));
            *b = exp(log(1e-2) + uniform(r1) * (log(1e4) - log(1e-2)));
            break;
        case 1:
            *a = (uniform(r0) - 0.5) * 8.0;
            *b = exp(log(1e-3) + uniform(r1) * (log(1e2) - log(1e-3)));
            break;
        case 2: {
            const int e = int(r1 % 40) - 20;
            *b = ldexp(2.0 - 0x1p-52, e);
            *a = exp(log(1e-3) + uniform(r0) * (log(1e5) - log(1e-3)));
            break;
        }
        default: {
            const int e = int(r1 % 60) - 30;
            const double base = ldexp(1.0, e);
            *a = nextafter(base, (r0 & 1) ? 1e308 : 0.0) * (1.0 + double(r0 % 7) * 0x1p-50);
            *b = exp(log(1e-2) + uniform(r1 >> 8) * (log(1e4) - log(1e-2)));
            break;
        }
    }
}

__global__ void check(uint64_t n, int family, unsigned long long* mismatches, double* first) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        double a, b;
        operands(i, family, &a, &b);
        const double q = fo::divide(a, fo::make_divisor(b));
        const double ref = a / b;
        if (__double_as_longlong(q) != __double_as_longlong(ref)) {
            if (atomicAdd(mismatches, 1ull) == 0) {
                first[0] = a;
                first[1] = b;
            }
        }
    }
}

}  // namespace

// Returns 0 on success; *mismatches receives the count, first[0..1] the first mismatching pair.
extern "C" int divide_check(uint64_t n, int family, unsigned long long* mismatches, double* first) {
    unsigned long long* d_count = nullptr;
    double* d_first = nullptr;
    if (cudaMalloc(&d_count, sizeof(unsigned long long)) != cudaSuccess) return 1;
    if (cudaMalloc(&d_first, 2 * sizeof(double)) != cudaSuccess) return 1;
    cudaMemset(d_count, 0, sizeof(unsigned long long));
    cudaMemset(d_first, 0, 2 * sizeof(double));
    check<<<148 * 8, 256>>>(n, family, d_count, d_first);
    const cudaError_t e = cudaDeviceSynchronize();
    cudaMemcpy(mismatches, d_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaMemcpy(first, d_first, 2 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_count);
    cudaFree(d_first);
    return e == cudaSuccess ? 0 : 2;
}

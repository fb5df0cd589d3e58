// lsm_sync.cuh - grid synchronisation of the persistent backward kernel: a grid arrival counter
// that each CTA bumps with release semantics once its partial is written, and a bounded warp-wide
// wait on it. Every wait gives up after a time limit and raises status->barrier_timeout, so a CTA
// that never arrives ends the kernel with an error the host reports, not a hang.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "lsm_device.cuh"

namespace fo {

__device__ __forceinline__ unsigned ld_volatile_u32(const unsigned* p) {
    return *(const volatile unsigned*)p;
}

__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void red_release_add_gpu(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned ld_relaxed_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void named_barrier_sync(int id, int threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Grid synchronisation of the backward pass (all CTAs co-resident: cooperative launch). There is
// no grid barrier. When its partial for sync point `seq` is written (cta_reduce_to ends with a CTA
// barrier), thread 0 adds one to the grid's arrival counter with release semantics and moves on
// without waiting for a reply. Warp 0 of every CTA reads the counter until it reaches
// seq * gridDim.x, fences once, and the combine warps read the partials. A partial buffer is
// reused two sync points later: a CTA arrives at seq + 2 only after combining seq + 1, which needs
// every CTA to have arrived at seq + 1, which each does only after it has read the partials of
// seq. A waiting warp gives up after kBarrierTimeoutNs, raising status->barrier_timeout; every CTA
// then leaves at its next wait.
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;
__device__ __forceinline__ void publish_partial(DeviceStatus* st) {
    if (threadIdx.x == 0) red_release_add_gpu(&st->arrivals, 1u);
}

// Warp-wide wait until the arrival counter reaches `target`. Lane 0 reads the counter and every
// decision is taken on its broadcast value, so the lanes leave the loop together however they
// entered it. Returns false (in every lane) once `limit_ns` has passed or another waiter has
// already raised the timeout.
__device__ inline bool wait_arrivals(DeviceStatus* st, unsigned target,
                                     unsigned long long limit_ns = kBarrierTimeoutNs) {
    const int lane = threadIdx.x & 31;
    unsigned spins = 0;
    unsigned long long start = 0;
    __syncwarp();
    for (;;) {
        unsigned seen = 0;
        if (lane == 0) seen = ld_relaxed_gpu(&st->arrivals);
        seen = __shfl_sync(0xffffffffu, seen, 0);
        if (seen >= target) break;
        if ((++spins & 255u) == 0) {
            int give_up = 0;
            if (lane == 0) {
                give_up = ld_volatile_u32(&st->barrier_timeout) != 0;
                const unsigned long long now = global_timer_ns();
                if (start == 0) {
                    start = now;
                } else if (now - start > limit_ns) {
                    atomicExch(&st->barrier_timeout, 1u);
                    give_up = 1;
                }
            }
            if (__shfl_sync(0xffffffffu, give_up, 0)) return false;
        }
    }
    __threadfence();
    return true;
}

}  // namespace fo

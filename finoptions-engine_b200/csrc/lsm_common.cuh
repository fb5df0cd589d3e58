// lsm_common.cuh - device building blocks shared by the single-contract and batch LSM kernels:
// ZIGNOR tables in shared memory, the seeded path simulation with event phases, deterministic
// warp / CTA / grid reductions, the exercise rule and the in-the-money power-sum accumulator.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "lsm_device.cuh"

namespace fo {

static __constant__ uint64_t c_zig_x[257] = FO_ZIG_NORM_X_BITS;
static __constant__ uint64_t c_zig_f[257] = FO_ZIG_NORM_F_BITS;

constexpr unsigned long long kNone = ~0ull;

__device__ __forceinline__ void load_zig_tables(double* sx, double* sf) {
    for (int i = threadIdx.x; i < 257; i += blockDim.x) {
        sx[i] = bits_to_double(c_zig_x[i]);
        sf[i] = bits_to_double(c_zig_f[i]);
    }
    __syncthreads();
}

__device__ __forceinline__ SmemZig make_zig(const double* sx, const double* sf) {
    SmemZig z;
    z.xs = sx;
    z.fs = sf;
    z.rr = bits_to_double(FO_ZIG_NORM_R_BITS);
    return z;
}

// ---------------------------------------------------------------------------------------------
// Seeded path simulation
// ---------------------------------------------------------------------------------------------

struct SimResult {
    int code;  // 0 ok, kNormalBudget, kNormalRejection, 3 non-finite transition
    int interval;
    double spot;
    double normal;
};

// Simulates one path; calls store(row, value) at every observation. Mirrors simulate_one_seeded
// (seeded.rs:399-459) including the terminal-dividend phase order.
template <typename Store>
__device__ __forceinline__ SimResult simulate_path(const DevicePlan& plan, const SmemZig& zig, uint64_t seed,
                                                   uint32_t domain, uint32_t path, Store&& store) {
    PathStream s;
    s.init(seed, domain, path, plan.intervals);
    double spot = plan.sim_start;
    SimResult r{0, 0, 0.0, 0.0};
    if (plan.row_node[0] == 0) store(0, spot);
    for (uint32_t i = 0; i < plan.intervals; ++i) {
        double z = 0.0;
        const int status = zig_sample(s, zig, &z);
        if (status != kNormalOk) {
            r.code = status;
            r.interval = int(i);
            return r;
        }
        const StepCoef c = plan.steps[i];
        const double next = gbm_advance(spot, c.diffusion, c.log_drift, z);
        if (!fo_isfinite(next)) {
            r.code = 3;
            r.interval = int(i);
            r.spot = spot;
            r.normal = z;
            return r;
        }
        spot = next;
        const NodeEvent ev = plan.events[i + 1];
        const bool dividend = (ev.flags & kEventDividend) != 0;
        const bool terminal = (ev.flags & kEventTerminal) != 0;
        if (dividend && terminal) spot = apply_cash_dividend(plan.policy, ev.dividend_amount, spot);
        if (ev.row >= 0) store(ev.row, spot);
        if (dividend && !terminal) spot = apply_cash_dividend(plan.policy, ev.dividend_amount, spot);
    }
    return r;
}

// simulate_path for caller-supplied standard normals: normals[i * paths + path] drives interval i
// (GbmPathPlan::simulate with an external shock matrix, path.rs:139-175). The buffer was checked for
// non-finite values before the launch; only a non-finite transition fails here.
template <typename Store>
__device__ __forceinline__ SimResult simulate_path_external(const DevicePlan& plan, const double* normals,
                                                            uint64_t paths, uint64_t path, Store&& store) {
    double spot = plan.sim_start;
    SimResult r{0, 0, 0.0, 0.0};
    if (plan.row_node[0] == 0) store(0, spot);
    for (uint32_t i = 0; i < plan.intervals; ++i) {
        const double z = normals[uint64_t(i) * paths + path];
        const StepCoef c = plan.steps[i];
        const double next = gbm_advance(spot, c.diffusion, c.log_drift, z);
        if (!fo_isfinite(next)) {
            r.code = 3;
            r.interval = int(i);
            r.spot = spot;
            r.normal = z;
            return r;
        }
        spot = next;
        const NodeEvent ev = plan.events[i + 1];
        const bool dividend = (ev.flags & kEventDividend) != 0;
        const bool terminal = (ev.flags & kEventTerminal) != 0;
        if (dividend && terminal) spot = apply_cash_dividend(plan.policy, ev.dividend_amount, spot);
        if (ev.row >= 0) store(ev.row, spot);
        if (dividend && !terminal) spot = apply_cash_dividend(plan.policy, ev.dividend_amount, spot);
    }
    return r;
}

// ---------------------------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------------------------

constexpr int kSlots = 16;  // T_0..T_8, U_0..U_4, non-finite count, spare
constexpr int kBadSlot = kMomentSlots;  // in-the-money paths with a non-finite predictor or response

__device__ __forceinline__ dd shfl_dd_down(dd v, int off);

// Butterfly "transpose" reduction of S values across a warp: at each stage a lane keeps half of
// its remaining values and adds its partner's copy of that half, so S values need S - 1 + log2
// shuffles instead of 5 S. Lane l ends holding the warp total of value (l % S) (S a power of two
// no larger than 32).
template <int S>
__device__ __forceinline__ double warp_transpose_reduce(double (&v)[S]) {
    const int lane = threadIdx.x & 31;
    double buf[S];
#pragma unroll
    for (int k = 0; k < S; ++k) buf[k] = v[k];
#pragma unroll
    for (int half = S / 2; half >= 1; half >>= 1) {
        // partner offset = half; lanes with (lane & half) keep the upper half.
        const bool upper = (lane & half) != 0;
#pragma unroll
        for (int k = 0; k < half; ++k) {
            const double send = upper ? buf[k] : buf[k + half];
            const double keep = upper ? buf[k + half] : buf[k];
            buf[k] = keep + __shfl_xor_sync(0xffffffffu, send, half);
        }
    }
    double total = buf[0];
#pragma unroll
    for (int off = S; off < 32; off <<= 1) total += __shfl_xor_sync(0xffffffffu, total, off);
    return total;
}

__device__ __forceinline__ dd shfl_dd_down(dd v, int off);

// Warp sums in double, then warp k combines slot k across the CTA's warps with a double-double
// shuffle tree; lane 0 of warp k writes slot k of the CTA partial. Requires S <= warps per CTA.
template <int S>
__device__ __forceinline__ void cta_reduce_to(double (&acc)[S], double* smem /* [32 * S] */, double2* dst,
                                              size_t slot_stride = 1) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    const double total = warp_transpose_reduce<S>(acc);
    // lane l holds value l % S: lanes 0..S-1 publish
    if (lane < S) smem[warp * S + lane] = total;
    __syncthreads();
    if (warp < S) {
        dd v = dd_make(lane < warps ? smem[lane * S + warp] : 0.0);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = dd_add(v, shfl_dd_down(v, off));
        if (lane == 0) dst[size_t(warp) * slot_stride] = make_double2(v.hi, v.lo);
    }
    __syncthreads();
}

__device__ __forceinline__ dd shfl_dd_down(dd v, int off) {
    dd o;
    o.hi = __shfl_down_sync(0xffffffffu, v.hi, off);
    o.lo = __shfl_down_sync(0xffffffffu, v.lo, off);
    return o;
}

// Sums partials[b * S + k] over b in a fixed order; warp k handles slot k. Identical in every CTA.
template <int S>
__device__ __forceinline__ void grid_combine(const double2* partials, int blocks, dd* out /* smem [S] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp < S) {
        // Issue the first eight partials of this lane before adding any, so their L2 latencies
        // overlap; the additions keep the fixed block order.
        constexpr int kBatch = 8;
        double2 v[kBatch];
#pragma unroll
        for (int i = 0; i < kBatch; ++i) {
            const int b = lane + 32 * i;
            v[i] = b < blocks ? __ldcg(&partials[b * S + warp]) : make_double2(0.0, 0.0);
        }
        dd acc = dd_make(0.0);
#pragma unroll
        for (int i = 0; i < kBatch; ++i)
            if (lane + 32 * i < blocks) acc = dd_add(acc, dd{v[i].x, v[i].y});
        for (int b = lane + 32 * kBatch; b < blocks; b += 32) {
            const double2 w = __ldcg(&partials[b * S + warp]);
            acc = dd_add(acc, dd{w.x, w.y});
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc = dd_add(acc, shfl_dd_down(acc, off));
        if (lane == 0) out[warp] = acc;
    }
    __syncthreads();
}

// CTA reduction of S per-thread doubles to double-double totals in shared memory. Warp sums are
// formed in double by the transpose reduction; warp w then combines slots w, w + warps, ... over
// the CTA's warps in double-double in a fixed order, so the totals do not depend on timing.
template <int S>
__device__ __forceinline__ void cta_reduce_dd(double (&acc)[S], double* red /* [32 * S] */, dd* out /* [S] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    const double total = warp_transpose_reduce<S>(acc);
    if (lane < S) red[warp * S + lane] = total;
    __syncthreads();
    for (int slot = warp; slot < S; slot += warps) {
        dd v = dd_make(lane < warps ? red[lane * S + slot] : 0.0);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = dd_add(v, shfl_dd_down(v, off));
        if (lane == 0) out[slot] = v;
    }
    __syncthreads();
}

__device__ __forceinline__ bool exercise_rule(int tie_rule, double intrinsic, double continuation) {
    return tie_rule == 0 ? intrinsic > continuation : intrinsic >= continuation;
}

struct RowSums {
    double acc[kSlots];
};

__device__ __forceinline__ void accumulate_itm(RowSums& r, double x, double y, double pivot) {
    const double t = x - pivot;
    r.acc[0] += 1.0;
    double pw = t;
    r.acc[kPowerSums] += y;
#pragma unroll
    for (int k = 1; k < kPowerSums; ++k) {
        r.acc[k] += pw;
        if (k < kResponseSums) r.acc[kPowerSums + k] = fo_fma(y, pw, r.acc[kPowerSums + k]);
        pw *= t;
    }
}

// The halves of accumulate_itm: count and T_1..T_8 of t = x - pivot (they do not depend on the
// response), and U_0..U_4 of the response y.
__device__ __forceinline__ void accumulate_powers(RowSums& r, double t) {
    r.acc[0] += 1.0;
    double pw = t;
#pragma unroll
    for (int k = 1; k < kPowerSums; ++k) {
        r.acc[k] += pw;
        pw *= t;
    }
}

__device__ __forceinline__ void accumulate_responses(RowSums& r, double t, double y) {
    r.acc[kPowerSums] += y;
    double pw = t;
#pragma unroll
    for (int k = 1; k < kResponseSums; ++k) {
        r.acc[kPowerSums + k] = fo_fma(y, pw, r.acc[kPowerSums + k]);
        pw *= t;
    }
}

}  // namespace fo

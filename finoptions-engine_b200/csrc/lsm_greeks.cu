// lsm_greeks.cu - fused evaluation with pathwise adjoint Greeks for one contract (no reference
// counterpart: the reference obtains sensitivities by bump-and-reprice through price_lsm_call).
//
// The fitted exercise policy is held fixed. Each evaluation path is re-simulated exactly as in
// evaluate_kernel (same Philox stream, ZIGNOR normals and GBM / cash-dividend arithmetic), so the
// price partials are bitwise those of the plain evaluation. While simulating, the path keeps a
// few numbers per segment between cash-dividend nodes; when it stops (exercise or expiry) a short
// backward recurrence over those segments yields its contribution to delta, vega, the
// log-discount sensitivities and the cash-dividend sensitivities.
//
// With payoff P = (S_obs - K) exp(L_n) at the stopping node n and a = dP/dS the adjoint of the
// state, the GBM step S' = S exp(u_i), u_i = sigma sqrt(dt_i) Z_i + log_drift_i, is multiplicative,
// so w = a S is constant along a segment without cash dividends and
//   dP/du_i = w_segment(i),   dP/dsigma = sum_segments w_s sum_{i in s} (Z_i sqrt(dt_i) - sigma dt_i).
// Because log_drift_i = -(L_{i+1} - L_i) - (Q_{i+1} - Q_i) - sigma^2 dt_i / 2, the log-discount
// gradient is w at node 0, the jump of w at each cash-dividend node, and P - w_last at the
// stopping node (exactly -K exp(L_n) for an early exercise, which the host applies from the
// stopping counts). A cash jump S+ = h(S-) maps a+ to a- = a+ h'(S-) and contributes
// -a+ [S- > D] to dP/dD.
#include <cuda_runtime.h>
#include <stdint.h>

#include "lsm_adjoint.cuh"
#include "lsm_common.cuh"
#include "lsm_device.cuh"
#include "lsm_kernels.h"

namespace fo {

struct GreeksEvalRow {
    FitModel model;
    int32_t kind;
    int32_t pad;
    double discount;
};

template <int D>  // == plan.degree
__global__ void __launch_bounds__(kEvalThreads, 4) evaluate_greeks_kernel(EvalArgs a, GreeksArgs gk) {
    extern __shared__ __align__(16) unsigned char greeks_smem_raw[];
    __shared__ double gred[32 * kGreekSlots];
    __shared__ dd gtot[kGreekSlots];
    const DevicePlan& plan = a.plan;
    const uint32_t rows = plan.rows;
    double* sx = reinterpret_cast<double*>(greeks_smem_raw);
    double* sf = sx + 257;
    double* red = sf + 257;                                             // [32 * 2]
    GreeksEvalRow* rules = reinterpret_cast<GreeksEvalRow*>(red + 64);  // [rows]
    unsigned* counts = reinterpret_cast<unsigned*>(rules + rows);       // [rows]
    unsigned* itm_counts = counts + rows;                               // [rows]
    for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) {
        GreeksEvalRow er;
        if (r + 1 < rows) {
            er.model = a.records[r].model;
            er.kind = a.records[r].kind;
        } else {
            er.kind = kRuleNone;
        }
        er.discount = plan.disc_to_origin[r];
        rules[r] = er;
        counts[r] = 0;
        itm_counts[r] = 0;
    }
    load_zig_tables(sx, sf);
    const SmemZig zig = make_zig(sx, sf);
    const double K = plan.strike;
    const Divisor Kd = make_divisor(K);
    const uint64_t P = plan.eval_paths;
    const uint32_t last = rows - 1;
    double sum = 0.0, sumsq = 0.0;
    GreekSums gs;
    gs.reset();
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < P; p += uint64_t(gridDim.x) * blockDim.x) {
        bool active = true;
        double payoff = 0.0;
        PathAdjoint adj;
        adj.reset();
        auto observe = [&](int row, double spot) {
            if (!active) return;
            const GreeksEvalRow& er = rules[row];
            if (uint32_t(row) == last) {
                const double d = spot - K;
                payoff = (d > 0.0 ? d : 0.0) * er.discount;
                if (!fo_isfinite(payoff)) atomicMin(&a.status->eval_terminal_fail, (unsigned long long)p);
                active = false;
                atomicAdd(&counts[row], 1u);
                adj.stop(gs, plan.row_node[row], spot, payoff, er.discount, true, plan.policy, 1.0);
                return;
            }
            if (er.kind == kRuleNoSupport) {
                if (spot > K) atomicAdd(&itm_counts[row], 1u);
                return;
            }
            if (er.kind != kRuleRegression || !(spot > K)) return;
            const double intrinsic = spot - K;
            double continuation;
            if (!predict_continuation_d<D>(er.model, divide(spot, Kd), &continuation)) {
                atomicMin(&a.status->eval_fail, ((unsigned long long)row << 33) | (p << 1));
                return;
            }
            if (exercise_rule(plan.tie_rule, intrinsic, continuation)) {
                payoff = intrinsic * er.discount;
                if (!fo_isfinite(payoff))
                    atomicMin(&a.status->eval_fail, ((unsigned long long)row << 33) | (p << 1) | 1ull);
                active = false;
                atomicAdd(&counts[row], 1u);
                adj.stop(gs, plan.row_node[row], spot, payoff, er.discount, false, plan.policy, 1.0);
            }
        };
        // The path: simulate_path's arithmetic and event phases, with the segment bookkeeping.
        PathStream s;
        s.init(plan.eval_seed, plan.eval_domain, uint32_t(p), plan.intervals);
        double spot = plan.sim_start;
        if (plan.row_node[0] == 0) observe(0, spot);
        bool failed = false;
        for (uint32_t i = 0; i < plan.intervals; ++i) {
            double z = 0.0;
            if (zig_sample(s, zig, &z) != kNormalOk) {
                failed = true;
                break;
            }
            const StepCoef c = plan.steps[i];
            double next = 0.0;
            double g = 1.0;
            if (spot != 0.0) {
                g = fo_exp(fo_fma(c.diffusion, z, c.log_drift));
                next = spot * g;
            }
            if (!fo_isfinite(next)) {
                failed = true;
                break;
            }
            if (active) adj.step(g, z * gk.sqrt_dt[i] - gk.sigma * gk.dt[i]);
            spot = next;
            const uint32_t at = i + 1;
            const NodeEvent ev = plan.events[at];
            const bool dividend = (ev.flags & kEventDividend) != 0;
            const bool terminal = (ev.flags & kEventTerminal) != 0;
            if (dividend && terminal) {
                const double before = spot;
                spot = apply_cash_dividend(plan.policy, ev.dividend_amount, before);
                if (active) adj.cash(at, before, ev.dividend_amount);
            }
            if (ev.row >= 0) observe(ev.row, spot);
            if (dividend && !terminal) {
                const double before = spot;
                spot = apply_cash_dividend(plan.policy, ev.dividend_amount, before);
                if (active) adj.cash(at, before, ev.dividend_amount);
            }
        }
        if (failed) atomicMin(&a.status->eval_sim_fail, (unsigned long long)p);
        sum += payoff;
        sumsq += payoff * payoff;
    }
    // Price partials exactly as evaluate_kernel forms them.
    double acc[2] = {sum, sumsq};
    cta_reduce_to<2>(acc, red, a.partials + size_t(blockIdx.x) * 2);
    for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) {
        if (counts[r]) atomicAdd(&a.counts[r], counts[r]);
        if (itm_counts[r]) atomicAdd(&a.itm_counts[r], itm_counts[r]);
    }
    double gacc[kGreekSlots];
    gs.to_slots(gacc);
    cta_reduce_dd<kGreekSlots>(gacc, gred, gtot);
    if (threadIdx.x < kGreekSlots)
        gk.partials[size_t(blockIdx.x) * kGreekSlots + threadIdx.x] = make_double2(gtot[threadIdx.x].hi, gtot[threadIdx.x].lo);
}

// Sums the Greek partials of every block in a fixed order: warp k handles slot k.
__global__ void __launch_bounds__(32 * kGreekSlots) finalize_greeks_kernel(const double2* partials, int blocks,
                                                                             double* out) {
    __shared__ dd total[kGreekSlots];
    grid_combine<kGreekSlots>(partials, blocks, total);
    if (threadIdx.x < kGreekSlots) out[threadIdx.x] = dd_round(total[threadIdx.x]);
}

size_t evaluate_greeks_smem_bytes(uint32_t rows) {
    return sizeof(double) * (257 * 2 + 64) + sizeof(GreeksEvalRow) * rows + sizeof(unsigned) * 2 * rows;
}

template <int D>
static cudaError_t launch_evaluate_greeks_d(const EvalArgs& args, const GreeksArgs& greeks, int blocks,
                                            cudaStream_t stream) {
    const size_t smem = evaluate_greeks_smem_bytes(args.plan.rows);
    if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(evaluate_greeks_kernel<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    evaluate_greeks_kernel<D><<<blocks, kEvalThreads, smem, stream>>>(args, greeks);
    return cudaGetLastError();
}

cudaError_t launch_evaluate_greeks(const EvalArgs& args, const GreeksArgs& greeks, int blocks, cudaStream_t stream) {
    switch (args.plan.degree) {  // validated to 0..4 on the host
        case 0: return launch_evaluate_greeks_d<0>(args, greeks, blocks, stream);
        case 1: return launch_evaluate_greeks_d<1>(args, greeks, blocks, stream);
        case 2: return launch_evaluate_greeks_d<2>(args, greeks, blocks, stream);
        case 3: return launch_evaluate_greeks_d<3>(args, greeks, blocks, stream);
        default: return launch_evaluate_greeks_d<4>(args, greeks, blocks, stream);
    }
}

cudaError_t launch_finalize_greeks(const double2* partials, int blocks, double* out, cudaStream_t stream) {
    finalize_greeks_kernel<<<1, 32 * kGreekSlots, 0, stream>>>(partials, blocks, out);
    return cudaGetLastError();
}

}  // namespace fo

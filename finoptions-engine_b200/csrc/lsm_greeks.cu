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

__global__ void __launch_bounds__(kEvalThreads, 2) evaluate_greeks_kernel(EvalArgs a, GreeksArgs gk) {
    extern __shared__ unsigned char greeks_smem_raw[];
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
    const uint64_t P = plan.eval_paths;
    const int degree = plan.degree;
    const uint32_t last = rows - 1;
    const int n_div = int(gk.dividends);
    double sum = 0.0, sumsq = 0.0;
    double g_delta = 0.0, g_vega = 0.0, g_l0 = 0.0, g_terminal = 0.0;
    double g_jump[kMaxGreekDividends], g_div[kMaxGreekDividends];
#pragma unroll
    for (int j = 0; j < kMaxGreekDividends; ++j) g_jump[j] = g_div[j] = 0.0;
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < P; p += uint64_t(gridDim.x) * blockDim.x) {
        bool active = true;
        double payoff = 0.0;
        // Segment bookkeeping: seg = cash dividends applied so far; growth[s] = product of the step
        // factors of segment s, sens[s] = its sum of (Z sqrt(dt) - sigma dt); pre[j] = S before cash j.
        int seg = 0;
        double growth[kMaxGreekDividends + 1], sens[kMaxGreekDividends + 1], pre[kMaxGreekDividends];
        growth[0] = 1.0;
        sens[0] = 0.0;
        // Contribution of a path stopping at `row` with observed state s_obs and payoff `pay`.
        auto adjoint = [&](uint32_t row, double s_obs, double pay, bool terminal) {
            if (!(pay > 0.0)) return;
            const double ad = rules[row].discount;  // dP/dS_obs for an in-the-money stop
            int s = seg;
            double a_end = ad, s_end = s_obs;
            if (terminal && s > 0 && gk.div_node[s - 1] == plan.row_node[row]) {
                // Cash jump at expiry precedes the record: S_obs = h(S-).
                const int j = s - 1;
                const bool above = pre[j] > gk.div_amount[j];
                g_div[j] += above ? -ad : 0.0;
                a_end = plan.policy == 0 && !above ? 0.0 : ad;
                s_end = pre[j];
                s = j;
            }
            double w = a_end * s_end;
            if (terminal) g_terminal += pay - w;
            for (;;) {
                g_vega += w * sens[s];
                const double a_start = a_end * growth[s];
                if (s == 0) {
                    g_delta += a_start;
                    g_l0 += w;
                    break;
                }
                const int j = s - 1;  // the cash dividend that opened segment s
                const bool above = pre[j] > gk.div_amount[j];
                g_div[j] += above ? -a_start : 0.0;
                const double a_prev = plan.policy == 0 && !above ? 0.0 : a_start;
                const double w_prev = a_prev * pre[j];
                g_jump[j] += w - w_prev;
                a_end = a_prev;
                w = w_prev;
                s = j;
            }
        };
        auto observe = [&](int row, double spot) {
            if (!active) return;
            const GreeksEvalRow& er = rules[row];
            if (uint32_t(row) == last) {
                const double d = spot - K;
                payoff = (d > 0.0 ? d : 0.0) * er.discount;
                if (!fo_isfinite(payoff)) atomicMin(&a.status->eval_terminal_fail, (unsigned long long)p);
                active = false;
                atomicAdd(&counts[row], 1u);
                adjoint(uint32_t(row), spot, payoff, true);
                return;
            }
            if (er.kind == kRuleNoSupport) {
                if (spot > K) atomicAdd(&itm_counts[row], 1u);
                return;
            }
            if (er.kind != kRuleRegression || !(spot > K)) return;
            const double intrinsic = spot - K;
            double continuation;
            if (!predict_continuation(er.model, degree, spot / K, &continuation)) {
                atomicMin(&a.status->eval_fail, ((unsigned long long)row << 33) | (p << 1));
                return;
            }
            if (exercise_rule(plan.tie_rule, intrinsic, continuation)) {
                payoff = intrinsic * er.discount;
                if (!fo_isfinite(payoff))
                    atomicMin(&a.status->eval_fail, ((unsigned long long)row << 33) | (p << 1) | 1ull);
                active = false;
                atomicAdd(&counts[row], 1u);
                adjoint(uint32_t(row), spot, payoff, false);
            }
        };
        auto cash = [&](const NodeEvent& ev, double* spot) {
            const double before = *spot;
            *spot = apply_cash_dividend(plan.policy, ev.dividend_amount, before);
            if (active && seg < n_div) {
                pre[seg] = before;
                seg += 1;
                growth[seg] = 1.0;
                sens[seg] = 0.0;
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
            if (spot != 0.0) {
                const double g = fo_exp(fo_fma(c.diffusion, z, c.log_drift));
                next = spot * g;
                if (active) growth[seg] *= g;
            }
            if (!fo_isfinite(next)) {
                failed = true;
                break;
            }
            if (active) sens[seg] += z * gk.sqrt_dt[i] - gk.sigma * gk.dt[i];
            spot = next;
            const NodeEvent ev = plan.events[i + 1];
            const bool dividend = (ev.flags & kEventDividend) != 0;
            const bool terminal = (ev.flags & kEventTerminal) != 0;
            if (dividend && terminal) cash(ev, &spot);
            if (ev.row >= 0) observe(ev.row, spot);
            if (dividend && !terminal) cash(ev, &spot);
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
#pragma unroll
    for (int k = 0; k < kGreekSlots; ++k) gacc[k] = 0.0;
    gacc[kGreekDelta] = g_delta;
    gacc[kGreekVega] = g_vega;
    gacc[kGreekL0] = g_l0;
    gacc[kGreekTerminal] = g_terminal;
#pragma unroll
    for (int j = 0; j < kMaxGreekDividends; ++j) {
        gacc[kGreekJump + j] = g_jump[j];
        gacc[kGreekDividend + j] = g_div[j];
    }
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

cudaError_t launch_evaluate_greeks(const EvalArgs& args, const GreeksArgs& greeks, int blocks, cudaStream_t stream) {
    const size_t smem = evaluate_greeks_smem_bytes(args.plan.rows);
    if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(evaluate_greeks_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    evaluate_greeks_kernel<<<blocks, kEvalThreads, smem, stream>>>(args, greeks);
    return cudaGetLastError();
}

cudaError_t launch_finalize_greeks(const double2* partials, int blocks, double* out, cudaStream_t stream) {
    finalize_greeks_kernel<<<1, 32 * kGreekSlots, 0, stream>>>(partials, blocks, out);
    return cudaGetLastError();
}

}  // namespace fo

// lsm_adjoint.cuh - per-path pathwise-adjoint bookkeeping shared by the single-contract and batch
// Greeks kernels (lsm_greeks.cu). With the fitted policy fixed, an evaluation path keeps a few
// numbers per segment between cash-dividend nodes; when it stops, a backward recurrence over the
// segments adds its contributions to delta, vega, the log-discount gradient and the cash-dividend
// gradient (the derivation is in lsm_greeks.cu).
#pragma once

#include <stdint.h>

#include "lsm_kernels.h"

namespace fo {

// Per-thread sums of the per-path adjoint contributions.
struct GreekSums {
    double delta, vega, l0, terminal;
    double jump[kMaxGreekDividends];
    double div[kMaxGreekDividends];
    __device__ void reset() {
        delta = vega = l0 = terminal = 0.0;
#pragma unroll
        for (int j = 0; j < kMaxGreekDividends; ++j) jump[j] = div[j] = 0.0;
    }
    __device__ void to_slots(double (&acc)[kGreekSlots]) const {
#pragma unroll
        for (int k = 0; k < kGreekSlots; ++k) acc[k] = 0.0;
        acc[kGreekDelta] = delta;
        acc[kGreekVega] = vega;
        acc[kGreekL0] = l0;
        acc[kGreekTerminal] = terminal;
#pragma unroll
        for (int j = 0; j < kMaxGreekDividends; ++j) {
            acc[kGreekJump + j] = jump[j];
            acc[kGreekDividend + j] = div[j];
        }
    }
};

// Segment bookkeeping of one evaluation path: seg = cash dividends applied so far; growth[s] =
// product of the step factors of segment s; sens[s] = its sum of dP/du_i-weights for sigma; pre[j]
// = the state before cash j, above[j] = whether that state exceeded the amount, node[j] its node.
struct PathAdjoint {
    int seg;
    double growth[kMaxGreekDividends + 1];
    double sens[kMaxGreekDividends + 1];
    double pre[kMaxGreekDividends];
    bool above[kMaxGreekDividends];
    uint32_t node[kMaxGreekDividends];

    __device__ void reset() {
        seg = 0;
        growth[0] = 1.0;
        sens[0] = 0.0;
    }
    __device__ void step(double g, double sens_term) {
        growth[seg] *= g;
        sens[seg] += sens_term;
    }
    __device__ void cash(uint32_t at, double before, double amount) {
        if (seg >= kMaxGreekDividends) return;
        pre[seg] = before;
        above[seg] = before > amount;
        node[seg] = at;
        seg += 1;
        growth[seg] = 1.0;
        sens[seg] = 0.0;
    }
    // A path stops at `at` with observed state s_obs, payoff pay = (s_obs - K) * ad > 0. Adds its
    // delta, vega (sens scaled by sens_scale), log-discount and dividend contributions.
    __device__ void stop(GreekSums& acc, uint32_t at, double s_obs, double pay, double ad, bool terminal, int policy,
                         double sens_scale) const {
        if (!(pay > 0.0)) return;
        int s = seg;
        double a_end = ad, s_end = s_obs;
        if (terminal && s > 0 && node[s - 1] == at) {
            // Cash at expiry precedes the record: S_obs = h(S-).
            const int j = s - 1;
            acc.div[j] += above[j] ? -ad : 0.0;
            a_end = policy == 0 && !above[j] ? 0.0 : ad;
            s_end = pre[j];
            s = j;
        }
        double w = a_end * s_end;
        if (terminal) acc.terminal += pay - w;
        for (;;) {
            acc.vega += w * sens[s] * sens_scale;
            const double a_start = a_end * growth[s];
            if (s == 0) {
                acc.delta += a_start;
                acc.l0 += w;
                return;
            }
            const int j = s - 1;  // the cash dividend that opened segment s
            acc.div[j] += above[j] ? -a_start : 0.0;
            const double a_prev = policy == 0 && !above[j] ? 0.0 : a_start;
            const double w_prev = a_prev * pre[j];
            acc.jump[j] += w - w_prev;
            a_end = a_prev;
            w = w_prev;
            s = j;
        }
    }
};

}  // namespace fo

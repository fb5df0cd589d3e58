// The regression solve of one exercise row, run by one warp.
//
// fit_near_pivot<D> (fo_core.cuh) holds about 37 doubles live through its recurrence, more than a
// thread of the 64-register backward kernel has, so a one-thread solve spills on the critical
// path of every row. Here the same solve is spread over the 32 lanes of a converged warp:
//
//   * lane k <= 2D shifts power sum k and lane 2D + 1 + k (k <= D) response sum k to moments of
//     z = (x - mean) / scale, each summing its binomial terms j = k..0 in the sequential order;
//   * lane l then holds sigma_l = <p_j, z^l> and lane i the basis coefficient a_i; the three dot
//     products of a step are summed in lane order 0..j by every lane from shuffled products, and
//     the three-term updates read their neighbours' values by shuffle;
//   * the four quotients of a step (alpha, coefficient, norm / n for the rank test, beta) are one
//     division across lanes instead of four in sequence, and the rank test compares norm / n with
//     rank_limit(rank_tolerance) (fo_core.cuh) instead of taking a square root: the same decision.
//
// Every value goes through the same binary64 operations in the same order as the one-thread
// solve, so the fitted model is bit-identical to fit_continuation's, including what it has written
// when it stops at a failure. The one-thread solve runs its divisions as one serial chain; this one
// overlaps each step's four.
#pragma once

#include "fo_core.cuh"

namespace fo {

#ifdef __CUDACC__

constexpr unsigned kWarpLanes = 0xffffffffu;

// Every lane stores its share of *m once, when the solve ends: the one-thread solve's final model
// (arrays zeroed, then norm / coef of the first `columns` steps and alpha / beta of the first
// `steps` taken from lane j = step j).
__device__ __forceinline__ void store_fit(FitModel* m, int lane, double mean, double scale, double inv_scale,
                                          int status, int aux, double aux_value, int columns, int steps,
                                          double norm, double coef, double alpha, double beta) {
    if (lane < kMaxColumns) {
        m->norm[lane] = lane < columns ? norm : 0.0;
        m->coef[lane] = lane < columns ? coef : 0.0;
    }
    if (lane < kMaxDegree) {
        m->alpha[lane] = lane < steps ? alpha : 0.0;
        m->beta[lane] = lane < steps ? beta : 0.0;
    }
    if (lane == 0) {
        m->status = status;
        m->aux = aux;
        m->aux_value = aux_value;
        m->mean = mean;
        m->scale = scale;
        m->inv_scale = (fo_fabs(scale) > 0x1p-960 && fo_fabs(scale) < 0x1p960) ? inv_scale : 0.0;
    }
}

template <int D>
__device__ __noinline__ bool fit_near_pivot_warp(const dd* sums, double pivot, uint64_t count, double spread_limit,
                                                 FitModel* m) {
    static_assert(D >= 1 && D <= kMaxDegree, "degree 0 is solved by one lane");
    constexpr int K = 2 * D + 2;  // moments 0..2D+1 (the last stays zero)
    const int lane = int(threadIdx.x & 31);
    const double n = double(count);
    const double t1 = sums[1].hi + sums[1].lo;
    const double offset = t1 / n;
    const double t2 = sums[2].hi + sums[2].lo;
    const double var = (t2 - t1 * offset) / n;
    if (!(var > 0.0) || !(offset * offset <= var)) return false;
    const double mean = pivot + offset;
    const double scale = fo_sqrt(var);
    const double inv_scale = 1.0 / scale;  // make_divisor(scale).inv in its range; one division for both
    if (!fo_isfinite(mean) || !fo_isfinite(scale) || !(scale > 0.0)) {
        store_fit(m, lane, mean, scale, inv_scale, kFitDegeneratePredictor, 0, scale, 0, 0, 0.0, 0.0, 0.0, 0.0);
        return true;
    }

    // Binomial shift: lane k adds C(k, j) * delta^(k-j) * S_j for j = k..0 (S = T for the power-
    // sum lanes, with T_0 = n, and U for the response lanes), the sequential order, then scales by
    // scale^-k. The loop runs j from 2D down to 0 in every lane, so the sums are read uniformly;
    // a lane adds from j = k on, carrying delta^(k-j) by the same product chain as the one-thread
    // solve. C(k, j) is formed exactly in integers beforehand (constant divisors).
    const double delta = pivot - mean;
    const bool response = lane > 2 * D;
    const int k = response ? lane - (2 * D + 1) : lane;
    const bool shifting = !response || k <= D;
    int binomial[2 * D + 1];
    binomial[0] = 1;
#pragma unroll
    for (int j = 1; j <= 2 * D; ++j) binomial[j] = binomial[j - 1] * (k - j + 1) / j;  // 0 for j > k
    double acc = 0.0, power = 1.0;
#pragma unroll
    for (int j = 2 * D; j >= 0; --j) {
        // Branch-free: a lane adds +0.0 before its first term (its acc is still +0.0, so the sum
        // is unchanged) and its own terms from j = k on.
        const double tj = j == 0 ? n : sums[j].hi + sums[j].lo;
        const double uj = j <= D ? sums[kPowerSums + j].hi + sums[kPowerSums + j].lo : 0.0;
        const bool active = shifting && j <= k;
        const double term = double(binomial[j]) * power * (response ? uj : tj);
        acc += active ? term : 0.0;
        power = active ? power * delta : power;
    }
    double spow = 1.0;
#pragma unroll
    for (int j = 1; j <= 2 * D; ++j) spow = j <= k ? spow * inv_scale : spow;
    const double shifted = acc * spow;
    const double resp = __shfl_sync(kWarpLanes, shifted, lane + 2 * D + 1 < 32 ? lane + 2 * D + 1 : 31);

    // Stieltjes recurrence from the moments (lane l: sigma_l of p_j and p_{j-1}; lane i: a_i).
    // Step j's norm, coefficient, alpha and beta stay in lane j until store_fit.
    double sig_cur = lane < K - 1 ? shifted : 0.0, sig_prev = 0.0;
    double a_cur = lane == 0 ? 1.0 : 0.0, a_prev = 0.0;
    double previous_norm = 1.0;
    double out_norm = 0.0, out_coef = 0.0, out_alpha = 0.0, out_beta = 0.0;
    int status = kFitOk, aux = 0, columns = 0, steps = 0;
#pragma unroll
    for (int j = 0; j <= D; ++j) {
        const double sig_above = __shfl_down_sync(kWarpLanes, sig_cur, 1);
        const double a_below = __shfl_up_sync(kWarpLanes, a_cur, 1);
        const double pn = a_cur * sig_cur, pw = a_cur * sig_above, pp = a_cur * resp;
        double norm = 0.0, proj = 0.0, wp = 0.0;
#pragma unroll
        for (int a = 0; a <= j; ++a) {
            norm += __shfl_sync(kWarpLanes, pn, a);
            wp += __shfl_sync(kWarpLanes, pw, a);
            proj += __shfl_sync(kWarpLanes, pp, a);
        }
        // Lanes 4i .. 4i+3 divide wp, proj, norm, norm by norm, norm, n, previous_norm.
        const int which = lane & 3;
        const double quotient = (which == 0 ? wp : (which == 1 ? proj : norm)) /
                                (which < 2 ? norm : (which == 2 ? n : previous_norm));
        const double alpha = __shfl_sync(kWarpLanes, quotient, 0);
        const double coef = __shfl_sync(kWarpLanes, quotient, 1);
        const double spread = __shfl_sync(kWarpLanes, quotient, 2);
        const double beta = j == 0 ? 0.0 : __shfl_sync(kWarpLanes, quotient, 3);
        // The one-thread solve's checks in its order, decided together (one branch per step).
        const bool sums_finite = fo_isfinite(norm) && fo_isfinite(proj) && fo_isfinite(wp);
        const bool deficient = norm <= 0.0 || spread <= spread_limit;
        const bool kept = sums_finite && !deficient;  // norm and coef of step j are written
        const bool coef_finite = fo_isfinite(coef);
        const bool stepped = kept && coef_finite && j < D && fo_isfinite(alpha) && fo_isfinite(beta);
        const int failed = !sums_finite ? kFitNonFinite
                         : deficient    ? kFitRankDeficient
                         : !coef_finite ? kFitNonFinite
                         : (j < D && !stepped) ? kFitNonFinite
                                               : kFitOk;
        if (lane == j && kept) {
            out_norm = norm;
            out_coef = coef;
        }
        if (lane == j && stepped) {
            out_alpha = alpha;
            out_beta = beta;
        }
        columns = kept ? j + 1 : columns;
        steps = stepped ? j + 1 : steps;
        const double a_next = (lane > 0 ? a_below : 0.0) - alpha * a_cur - beta * a_prev;
        const double sig_next = (lane + 1 < K ? sig_above : 0.0) - alpha * sig_cur - beta * sig_prev;
        if (failed != kFitOk) {
            status = failed;
            aux = j;
            break;
        }
        a_prev = a_cur;
        a_cur = a_next;
        sig_prev = sig_cur;
        sig_cur = sig_next;
        previous_norm = norm;
    }
    store_fit(m, lane, mean, scale, inv_scale, status, aux, 0.0, columns, steps, out_norm, out_coef, out_alpha,
              out_beta);
    return true;
}

// fit_continuation for a converged warp: every lane calls it with the same arguments (spread_limit
// = rank_limit(rank_tolerance)); on return *m is complete and visible to the whole warp. Degree 0
// and the double-double fallback (pivot more than one standard deviation from the mean) run on
// lane 0 as in fit_continuation.
static __device__ __noinline__ void fit_continuation_warp(const dd* sums, double pivot, uint64_t count, int degree,
                                                   double rank_tolerance, double spread_limit, FitModel* m) {
    const bool writer = (threadIdx.x & 31) == 0;
    bool done;
    switch (degree) {
        case 0: done = false; break;
        case 1: done = fit_near_pivot_warp<1>(sums, pivot, count, spread_limit, m); break;
        case 2: done = fit_near_pivot_warp<2>(sums, pivot, count, spread_limit, m); break;
        case 3: done = fit_near_pivot_warp<3>(sums, pivot, count, spread_limit, m); break;
        default: done = fit_near_pivot_warp<4>(sums, pivot, count, spread_limit, m); break;
    }
    if (!done && writer) fit_continuation(sums, pivot, count, degree, rank_tolerance, m);
    __syncwarp();
}

#endif  // __CUDACC__

}  // namespace fo

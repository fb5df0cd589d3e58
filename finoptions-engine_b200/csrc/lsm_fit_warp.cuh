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
// solve, so the fitted model is bit-identical to fit_continuation's. Lane 0 writes the model in
// the order the one-thread solve writes it (partial writes before a failure included). The one-
// thread solve is the latency floor of one serial chain of divisions per step; this one overlaps
// them.
#pragma once

#include "fo_core.cuh"

namespace fo {

#ifdef __CUDACC__

constexpr unsigned kWarpLanes = 0xffffffffu;

template <int D>
__device__ __noinline__ bool fit_near_pivot_warp(const dd* sums, double pivot, uint64_t count, double spread_limit,
                                                 FitModel* m) {
    static_assert(D >= 1 && D <= kMaxDegree, "degree 0 is solved by one lane");
    constexpr int K = 2 * D + 2;  // moments 0..2D+1 (the last stays zero)
    const int lane = int(threadIdx.x & 31);
    const bool writer = lane == 0;
    const double n = double(count);
    const double t1 = sums[1].hi + sums[1].lo;
    const double offset = t1 / n;
    const double t2 = sums[2].hi + sums[2].lo;
    const double var = (t2 - t1 * offset) / n;
    if (!(var > 0.0) || !(offset * offset <= var)) return false;
    const double mean = pivot + offset;
    const double scale = fo_sqrt(var);
    const double inv_scale = 1.0 / scale;  // make_divisor(scale).inv in its range; one division for both
    if (writer) {
#pragma unroll
        for (int j = 0; j < kMaxDegree; ++j) {
            m->alpha[j] = 0.0;
            m->beta[j] = 0.0;
        }
#pragma unroll
        for (int j = 0; j < kMaxColumns; ++j) {
            m->coef[j] = 0.0;
            m->norm[j] = 0.0;
        }
        m->status = kFitOk;
        m->aux = 0;
        m->aux_value = 0.0;
        m->mean = mean;
        m->scale = scale;
        m->inv_scale = (fo_fabs(scale) > 0x1p-960 && fo_fabs(scale) < 0x1p960) ? inv_scale : 0.0;
    }
    if (!fo_isfinite(mean) || !fo_isfinite(scale) || !(scale > 0.0)) {
        if (writer) {
            m->status = kFitDegeneratePredictor;
            m->aux_value = scale;
        }
        return true;
    }

    // Binomial shift: term s of lane k is C(k, s) * delta^s * S_{k-s} (S = T for the power-sum
    // lanes, with T_0 = n, and U for the response lanes), added in s = 0..k order, then scaled by
    // scale^-k. C(k, s) is formed exactly in integers; delta^s and scale^-k by the same product
    // chains as the one-thread solve.
    const double delta = pivot - mean;
    const bool response = lane > 2 * D;
    const int k = response ? lane - (2 * D + 1) : lane;
    const bool shifting = !response || k <= D;
    double acc = 0.0, dpow = 1.0, spow = 1.0;
    int binomial = 1;
#pragma unroll
    for (int s = 0; s <= 2 * D; ++s) {
        if (s > 0) binomial = binomial * (k - s + 1) / s;
        if (shifting && s <= k) {
            const int j = k - s;
            const double sj = response ? sums[kPowerSums + j].hi + sums[kPowerSums + j].lo
                                       : (j == 0 ? n : sums[j].hi + sums[j].lo);
            acc += double(binomial) * dpow * sj;
            if (s > 0) spow *= inv_scale;
        }
        dpow *= delta;
    }
    const double shifted = acc * spow;
    const double resp = __shfl_sync(kWarpLanes, shifted, lane + 2 * D + 1 < 32 ? lane + 2 * D + 1 : 31);

    // Stieltjes recurrence from the moments (lane l: sigma_l of p_j and p_{j-1}; lane i: a_i).
    double sig_cur = lane < K - 1 ? shifted : 0.0, sig_prev = 0.0;
    double a_cur = lane == 0 ? 1.0 : 0.0, a_prev = 0.0;
    double previous_norm = 1.0;
#pragma unroll
    for (int j = 0; j <= D; ++j) {
        const double sig_above = __shfl_down_sync(kWarpLanes, sig_cur, 1);
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
        if (!fo_isfinite(norm) || !fo_isfinite(proj) || !fo_isfinite(wp)) {
            if (writer) {
                m->status = kFitNonFinite;
                m->aux = j;
            }
            return true;
        }
        if (norm <= 0.0 || spread <= spread_limit) {
            if (writer) {
                m->status = kFitRankDeficient;
                m->aux = j;
            }
            return true;
        }
        if (writer) {
            m->norm[j] = norm;
            m->coef[j] = coef;
        }
        if (!fo_isfinite(coef)) {
            if (writer) {
                m->status = kFitNonFinite;
                m->aux = j;
            }
            return true;
        }
        if (j < D) {
            if (!fo_isfinite(alpha) || !fo_isfinite(beta)) {
                if (writer) {
                    m->status = kFitNonFinite;
                    m->aux = j;
                }
                return true;
            }
            if (writer) {
                m->alpha[j] = alpha;
                m->beta[j] = beta;
            }
            const double a_below = __shfl_up_sync(kWarpLanes, a_cur, 1);
            const double a_next = (lane > 0 ? a_below : 0.0) - alpha * a_cur - beta * a_prev;
            const double sig_next = (lane + 1 < K ? sig_above : 0.0) - alpha * sig_cur - beta * sig_prev;
            a_prev = a_cur;
            a_cur = a_next;
            sig_prev = sig_cur;
            sig_cur = sig_next;
            previous_norm = norm;
        }
    }
    return true;
}

// fit_continuation for a converged warp: every lane calls it with the same arguments (spread_limit
// = rank_limit(rank_tolerance)); on return *m is complete and visible to the whole warp. Degree 0
// and the double-double fallback (pivot more than one standard deviation from the mean) run on
// lane 0 as in fit_continuation.
__device__ __noinline__ void fit_continuation_warp(const dd* sums, double pivot, uint64_t count, int degree,
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

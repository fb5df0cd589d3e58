// Host build of the device regression solve (finoptions-engine_b200/csrc/fo_core.cuh) for the CPU
// test suite: reduces in-the-money power sums the way the kernels do (per-thread binary64
// partials, warp trees in binary64, double-double above) and solves with fit_continuation.
#include <cstdint>
#include <vector>

#include "../../finoptions-engine_b200/csrc/fo_core.cuh"

using namespace fo;

extern "C" int harness_fit(const double* x, const double* y, uint64_t n, double pivot, int degree,
                           int paths_per_thread, double* model_out) {
    const uint64_t threads = (n + paths_per_thread - 1) / paths_per_thread;
    std::vector<double> partial(threads * kMomentSlots, 0.0);
    for (uint64_t t = 0; t < threads; ++t) {
        double* acc = &partial[t * kMomentSlots];
        for (int j = 0; j < paths_per_thread; ++j) {
            const uint64_t i = t * paths_per_thread + j;
            if (i >= n) break;
            const double d = x[i] - pivot;
            acc[0] += 1.0;
            acc[kPowerSums] += y[i];
            double pw = d;
            for (int k = 1; k < kPowerSums; ++k) {
                acc[k] += pw;
                if (k < kResponseSums) acc[kPowerSums + k] += y[i] * pw;
                pw *= d;
            }
        }
    }
    dd sums[kMomentSlots];
    for (int k = 0; k < kMomentSlots; ++k) sums[k] = dd_make(0.0);
    for (uint64_t w = 0; w < threads; w += 32) {
        double lane[32][kMomentSlots] = {};
        for (int l = 0; l < 32 && w + l < threads; ++l)
            for (int k = 0; k < kMomentSlots; ++k) lane[l][k] = partial[(w + l) * kMomentSlots + k];
        for (int off = 16; off > 0; off >>= 1)
            for (int l = 0; l < off; ++l)
                for (int k = 0; k < kMomentSlots; ++k) lane[l][k] += lane[l + off][k];
        for (int k = 0; k < kMomentSlots; ++k) sums[k] = dd_add(sums[k], dd_make(lane[0][k]));
    }
    FitModel m;
    fit_continuation(sums, pivot, n, degree, 1e-12, &m);
    model_out[0] = m.mean;
    model_out[1] = m.scale;
    for (int i = 0; i < 4; ++i) model_out[2 + i] = m.alpha[i];
    for (int i = 0; i < 4; ++i) model_out[6 + i] = m.beta[i];
    for (int i = 0; i < 5; ++i) model_out[10 + i] = m.coef[i];
    for (int i = 0; i < 5; ++i) model_out[15 + i] = m.norm[i];
    int rank = 0, aux = 0;
    double condition = 0.0;
    const int diag = m.status == kFitOk ? diagnose_design(m, degree, 1e-12, 1e8, &rank, &condition, &aux) : -1;
    model_out[20] = rank;
    model_out[21] = condition;
    return m.status * 10 + (diag < 0 ? 9 : diag);
}

// rank_limit(tol): the largest q whose correctly rounded square root is at most tol.
extern "C" double harness_rank_limit(double tol) { return rank_limit(tol); }

// predict_continuation_d<D> against predict_continuation(degree = D) on `n` predictors for a model
// given as mean, scale, alpha[4], beta[4], coef[5]: the number of predictions whose bits or
// success differ.
extern "C" int harness_predict_mismatches(const double* model_in, int degree, const double* x, uint64_t n) {
    FitModel m{};
    m.mean = model_in[0];
    m.scale = model_in[1];
    m.inv_scale = make_divisor(m.scale).inv;
    for (int i = 0; i < 4; ++i) m.alpha[i] = model_in[2 + i];
    for (int i = 0; i < 4; ++i) m.beta[i] = model_in[6 + i];
    for (int i = 0; i < 5; ++i) m.coef[i] = model_in[10 + i];
    int bad = 0;
    for (uint64_t i = 0; i < n; ++i) {
        double a = -1.0, b = -2.0;
        const bool ok_a = predict_continuation(m, degree, x[i], &a);
        bool ok_b = false;
        switch (degree) {
            case 0: ok_b = predict_continuation_d<0>(m, x[i], &b); break;
            case 1: ok_b = predict_continuation_d<1>(m, x[i], &b); break;
            case 2: ok_b = predict_continuation_d<2>(m, x[i], &b); break;
            case 3: ok_b = predict_continuation_d<3>(m, x[i], &b); break;
            default: ok_b = predict_continuation_d<4>(m, x[i], &b); break;
        }
        uint64_t ba, bb;
        __builtin_memcpy(&ba, &a, 8);
        __builtin_memcpy(&bb, &b, 8);
        if (ok_a != ok_b || (ok_a && ba != bb)) ++bad;
    }
    return bad;
}

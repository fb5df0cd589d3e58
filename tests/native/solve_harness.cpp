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

// lsm_grouped.cu - grouped and row-addressed LSM batches on the device
// (GroupedBatchLsmCallInputs::price and BatchLsmCallInputs::price,
// crates/finoptions-lsm/src/batch/pricing.rs:191-300, 422-589, 704-1114).
//
// Host side: request validation in the reference's order (lib.rs:1302-1415 parse_batch_lsm_method,
// input.rs try_new, BatchRandomStreams::validate, validate_exercise_mesh_domain), then per group
// the exact union mesh, curves, event schedule and simulation plan (build_path_plan). Groups are
// priced in waves sized to the device memory budget; each wave is one persistent launch that
// drains a queue of simulation, fit and evaluation items (lsm_persistent.cu). The lowest failing
// group is reported with the typed error its serial replay in the reference would raise
// (pricing.rs:452-503); no partial result is returned.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <thread>
#include <utility>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/finoptions_cuda.h"
#include "executor.h"
#include "host.h"
#include "lsm_batch.cuh"
#include "lsm_batch_kernels.h"
#include "lsm_kernels.h"

using namespace fo;

namespace {

constexpr unsigned long long kNone = ~0ull;
// Shared memory the persistent launch may spend on staged fitted rules (with three 80-register
// CTAs per SM, about 57 KB each leaves every CTA resident; more lowers the CTAs per SM).
constexpr size_t kPersistentRuleSmemBytes = 200 * 1024;
constexpr int kPersistentMaxCtasPerSm = 3;  // the persistent kernel's launch bounds
constexpr uint64_t kU32Max = 0xffffffffull;

std::string u(uint64_t v) { return std::to_string(v); }

Error input_error(int32_t code, std::string message) { return make_error(FO_ERR_INPUT, code, std::move(message)); }
Error lsm_error(int32_t code, std::string message) { return make_error(FO_ERR_LSM, code, std::move(message)); }

bool canonical_nonnegative(double v) { return std::isfinite(v) && !(v < 0.0) && !(v == 0.0 && std::signbit(v)); }

uint64_t bits(double x) {
    uint64_t b;
    std::memcpy(&b, &x, sizeof b);
    return b;
}

// f64::total_cmp on the finite, non-negative values the validated batch columns hold.
int total_cmp(double a, double b) {
    if (a < b) return -1;
    if (a > b) return 1;
    const bool sa = std::signbit(a), sb = std::signbit(b);
    if (sa == sb) return 0;
    return sa ? -1 : 1;
}

// BatchLsmError wrappers of row-addressed sources (batch/error.rs).
Error financial_at_row(uint64_t row, const Error& e) {
    Error w = wrap(e, FO_ERR_INPUT, "LSM batch financial input failed at row " + u(row));
    w.row = int64_t(row);
    return w;
}
Error plan_at_row(uint64_t row, const Error& e) {
    Error w = wrap(e, FO_ERR_INPUT, "LSM batch simulation plan failed at row " + u(row));
    w.row = int64_t(row);
    return w;
}
Error estimator_at_row(uint64_t row, const Error& e) {
    Error w = wrap(e, FO_ERR_LSM, "LSM batch estimator failed at row " + u(row));
    w.row = int64_t(row);
    return w;
}

// A grouped request or a row batch seen as groups of strike rows.
struct BatchView {
    const fo_lsm_grouped_request* q;
    bool grouped;
    uint64_t groups() const { return q->n_initial_spots; }
    uint64_t rows() const { return q->n_strikes; }
    uint64_t first_row(uint64_t g) const { return grouped ? q->group_offsets[g] : g; }
    uint64_t end_row(uint64_t g) const { return grouped ? q->group_offsets[g + 1] : g + 1; }
    bool cash() const { return q->dividend_model != FO_MODEL_CONTINUOUS_YIELD; }
    uint64_t cash_rows() const { return q->n_dividend_offsets ? q->n_dividend_offsets - 1 : 0; }
    void cash_row(uint64_t g, const double** times, const double** amounts, uint64_t* n) const {
        const int64_t base = q->dividend_offsets[0];
        const int64_t b = q->dividend_offsets[g] - base, e = q->dividend_offsets[g + 1] - base;
        *times = q->dividend_times + b;
        *amounts = q->dividend_amounts + b;
        *n = uint64_t(e - b);
    }
    uint64_t explicit_rows() const { return q->n_explicit_exercise_offsets ? q->n_explicit_exercise_offsets - 1 : 0; }
    void explicit_row(uint64_t g, const double** times, uint64_t* n) const {
        const int64_t base = q->explicit_exercise_offsets[0];
        const int64_t b = q->explicit_exercise_offsets[g] - base, e = q->explicit_exercise_offsets[g + 1] - base;
        *times = q->explicit_exercise_times + b;
        *n = uint64_t(e - b);
    }
};

// ---- method (parse_batch_lsm_method, lib.rs:1302-1415; BatchLsmCallMethod, input.rs:276-437) ---

Error validate_method(const fo_lsm_grouped_request& q) {
    if (q.polynomial_degree > 4)
        return lsm_error(FO_CODE_UNSUPPORTED_DEGREE,
                         "polynomial degree " + u(q.polynomial_degree) + " is unsupported; the validated maximum degree is 4");
    if (!std::isfinite(q.rank_tolerance) || q.rank_tolerance <= 0.0 || q.rank_tolerance >= 1.0)
        return lsm_error(FO_CODE_INVALID_RANK_TOLERANCE,
                         "rank tolerance must be finite and strictly between 0 and 1; observed " + fmt_f64(q.rank_tolerance));
    const double maximum = 1.0 / q.rank_tolerance;
    if (!std::isfinite(q.condition_limit) || q.condition_limit < 1.0 || q.condition_limit > maximum)
        return lsm_error(FO_CODE_INVALID_CONDITION_LIMIT,
                         "condition limit must be finite, at least 1, and no greater than 1/rank_tolerance (" +
                             fmt_f64(maximum) + "); observed " + fmt_f64(q.condition_limit));
    if (q.tie_rule != FO_TIE_STRICTLY_GREATER && q.tie_rule != FO_TIE_GREATER_OR_EQUAL)
        return input_error(FO_CODE_UNSUPPORTED_ENUM, "unsupported exercise tie rule " + std::to_string(q.tie_rule));
    if (q.insufficient_exercise_support != FO_SUPPORT_FAIL && q.insufficient_exercise_support != FO_SUPPORT_CONTINUE)
        return input_error(FO_CODE_UNSUPPORTED_ENUM, "unsupported insufficient exercise support policy " +
                                                         std::to_string(q.insufficient_exercise_support));
    const bool has_offsets = q.explicit_exercise_offsets != nullptr, has_times = q.explicit_exercise_times != nullptr;
    auto origin_ok = [&]() { return q.origin_exercise == FO_ORIGIN_INCLUDED || q.origin_exercise == FO_ORIGIN_EXCLUDED; };
    switch (q.exercise_mesh) {
        case FO_MESH_UNIFORM:
            if (has_offsets || has_times)
                return input_error(FO_CODE_INVALID_ARGUMENT, "uniform exercise mesh forbids explicit exercise buffers");
            if (!q.has_base_intervals)
                return input_error(FO_CODE_INVALID_ARGUMENT, "uniform exercise mesh requires base_intervals");
            if (!q.has_origin_exercise)
                return input_error(FO_CODE_INVALID_ARGUMENT, "uniform exercise mesh requires origin_exercise");
            if (!origin_ok())
                return input_error(FO_CODE_UNSUPPORTED_ENUM, "unsupported origin exercise convention " +
                                                                 std::to_string(q.origin_exercise));
            if (q.base_intervals == 0)
                return input_error(FO_CODE_EMPTY_BASE_INTERVALS,
                                   "LSM uniform exercise mesh must contain at least one base interval");
            break;
        case FO_MESH_CASH_DIVIDEND_DATES:
            if (q.has_base_intervals || q.has_origin_exercise || has_offsets || has_times)
                return input_error(FO_CODE_INVALID_ARGUMENT,
                                   "cash-dividend-date exercise mesh forbids uniform and explicit mesh fields");
            break;
        case FO_MESH_EXPLICIT_TIMES: {
            if (q.has_base_intervals)
                return input_error(FO_CODE_INVALID_ARGUMENT, "explicit exercise mesh forbids base_intervals");
            if (!q.has_origin_exercise)
                return input_error(FO_CODE_INVALID_ARGUMENT, "explicit exercise mesh requires origin_exercise");
            if (!has_offsets) return input_error(FO_CODE_INVALID_ARGUMENT, "explicit exercise mesh requires exercise offsets");
            if (!has_times) return input_error(FO_CODE_INVALID_ARGUMENT, "explicit exercise mesh requires exercise times");
            Error e = validate_ragged_exercise(q.explicit_exercise_offsets, q.n_explicit_exercise_offsets,
                                               q.explicit_exercise_times, q.n_explicit_exercise_times);
            if (!e.ok()) return e;
            if (!origin_ok())
                return input_error(FO_CODE_UNSUPPORTED_ENUM, "unsupported origin exercise convention " +
                                                                 std::to_string(q.origin_exercise));
            break;
        }
        default:
            return input_error(FO_CODE_UNSUPPORTED_ENUM, "unsupported batched LSM exercise mesh " + std::to_string(q.exercise_mesh));
    }
    auto path_count = [](const char* population, uint64_t n) -> Error {
        if (n == 0 || n > kU32Max)
            return input_error(FO_CODE_BATCH_PATH_COUNT_OUTSIDE_DOMAIN, std::string("batched LSM ") + population +
                                                                             " path count " + u(n) +
                                                                             " exceeds maximum 4294967295");
        return Error{};
    };
    Error e = path_count("training", q.training_paths);
    if (!e.ok()) return e;
    e = path_count("evaluation", q.evaluation_paths);
    if (!e.ok()) return e;
    if (q.evaluation_paths < 2)
        return input_error(FO_CODE_INSUFFICIENT_EVALUATION_PATHS,
                           "batched LSM evaluation requires at least two paths; observed " + u(q.evaluation_paths));
    return Error{};
}

// ---- dividend model and columns (input.rs:502-902) ----------------------------------------------

Error validate_dividend_model(const fo_lsm_grouped_request& q) {
    switch (q.dividend_model) {
        case FO_MODEL_CONTINUOUS_YIELD:
            return Error{};
        case FO_MODEL_CASH_DIVIDENDS:
            if (q.dividend_policy != FO_DIVIDEND_LIQUIDATOR && q.dividend_policy != FO_DIVIDEND_SURVIVOR)
                return input_error(FO_CODE_UNSUPPORTED_ENUM, "unsupported dividend policy " + std::to_string(q.dividend_policy));
            break;
        case FO_MODEL_ESCROWED_CASH_DIVIDENDS:
            if (q.volatility_convention != FO_ESCROWED_PREPAID_FORWARD &&
                q.volatility_convention != FO_ESCROWED_SPOT_MATCHED_AT_ORIGIN)
                return input_error(FO_CODE_UNSUPPORTED_ENUM, "unsupported escrowed volatility convention " +
                                                                 std::to_string(q.volatility_convention));
            break;
        default:
            return input_error(FO_CODE_UNSUPPORTED_ENUM, "unsupported batch dividend model " + std::to_string(q.dividend_model));
    }
    if (q.maturity_boundary != FO_MATURITY_STRICTLY_BEFORE && q.maturity_boundary != FO_MATURITY_AT_OR_BEFORE)
        return input_error(FO_CODE_UNSUPPORTED_CASH_MATURITY_BOUNDARY,
                           "cash-dividend maturity boundary is unsupported by this LSM engine");
    // RaggedCashDividends::try_new; in the LSM batch context its errors surface as InputError.
    Error e = validate_ragged_cash(q.dividend_offsets, q.n_dividend_offsets, q.dividend_times, q.n_dividend_times,
                                   q.dividend_amounts, q.n_dividend_amounts);
    if (!e.ok()) e.kind = FO_ERR_INPUT;
    return e;
}

Error row_count(const char* field, uint64_t expected, uint64_t observed) {
    if (observed != expected)
        return input_error(FO_CODE_ROW_COUNT_MISMATCH, std::string("LSM batch field ") + field + " has " + u(observed) +
                                                           " rows; expected " + u(expected));
    return Error{};
}

Error invalid_row_value(const char* field, uint64_t row, double observed) {
    return input_error(FO_CODE_INVALID_ROW_VALUE, std::string("LSM batch field ") + field + " is invalid at row " + u(row) +
                                                      ": observed " + fmt_f64(observed));
}
Error finite_value(const char* field, uint64_t row, double v) {
    return std::isfinite(v) ? Error{} : invalid_row_value(field, row, v);
}
Error positive_value(const char* field, uint64_t row, double v) {
    return std::isfinite(v) && v > 0.0 ? Error{} : invalid_row_value(field, row, v);
}
Error nonnegative_value(const char* field, uint64_t row, double v) {
    return canonical_nonnegative(v) ? Error{} : invalid_row_value(field, row, v);
}

Error validate_cash_schedule(uint64_t row, double maturity, const double* times, uint64_t n, int32_t boundary) {
    for (uint64_t event = 0; event < n; ++event) {
        const double time = times[event];
        const int c = total_cmp(time, maturity);
        if (c > 0)
            return input_error(FO_CODE_CASH_DIVIDEND_AFTER_MATURITY,
                               "cash dividend at batch row " + u(row) + ", event " + u(event) + ", time " + fmt_f64(time) +
                                   " occurs after maturity " + fmt_f64(maturity));
        if (c == 0 && boundary == FO_MATURITY_STRICTLY_BEFORE)
            return input_error(FO_CODE_CASH_DIVIDEND_AT_EXCLUDED_MATURITY,
                               "cash dividend at batch row " + u(row) + ", event " + u(event) + " equals maturity " +
                                   fmt_f64(maturity) + ", but the declared boundary is strictly-before");
        if (event > 0 && bits(times[event - 1]) == bits(time))
            return input_error(FO_CODE_DUPLICATE_CASH_DIVIDEND_TIME,
                               "cash-dividend batch row " + u(row) + " repeats exact event time " + fmt_f64(time) +
                                   " at event " + u(event) + "; aggregation policy is not declared");
    }
    return Error{};
}

// escrowed_origin_prepaid_cash (input.rs:830-850)
Error escrowed_origin_prepaid_cash(uint64_t row, double rate, const double* times, const double* amounts, uint64_t n,
                                   double* out) {
    double prepaid = 0.0;
    for (uint64_t event = 0; event < n; ++event) {
        const double discounted = amounts[event] * std::exp(-rate * times[event]);
        prepaid += discounted;
        if (!std::isfinite(discounted) || !std::isfinite(prepaid))
            return input_error(FO_CODE_ESCROWED_NON_FINITE_PREPAID_CASH,
                               "escrowed prepaid cash is not finite at batch row " + u(row) + ", event " + u(event) +
                                   ": time=" + fmt_f64(times[event]) + ", amount=" + fmt_f64(amounts[event]) +
                                   ", rate=" + fmt_f64(rate));
    }
    *out = prepaid;
    return Error{};
}

Error validate_escrowed_row(uint64_t row, double s0, double rate, double vol, const double* times, const double* amounts,
                            uint64_t n, int32_t convention) {
    double prepaid = 0.0;
    Error e = escrowed_origin_prepaid_cash(row, rate, times, amounts, n, &prepaid);
    if (!e.ok()) return e;
    const double forward = s0 - prepaid;
    if (!std::isfinite(forward) || forward <= 0.0)
        return input_error(FO_CODE_ESCROWED_NON_POSITIVE_PREPAID_FORWARD,
                           "escrowed prepaid forward must be strictly positive at batch row " + u(row) + "; initial spot is " +
                               fmt_f64(s0) + " and origin prepaid cash is " + fmt_f64(prepaid));
    if (convention == FO_ESCROWED_SPOT_MATCHED_AT_ORIGIN) {
        const double transformed = vol * s0 / forward;
        if (!std::isfinite(transformed) || transformed <= 0.0)
            return input_error(FO_CODE_ESCROWED_INVALID_VOLATILITY,
                               "escrowed spot-matched volatility is invalid at batch row " + u(row) + ": supplied=" +
                                   fmt_f64(vol) + ", initial_spot=" + fmt_f64(s0) + ", prepaid_forward=" + fmt_f64(forward) +
                                   ", transformed=" + fmt_f64(transformed));
    }
    return Error{};
}

// The dividend-model checks of one row (continuous yield, or cash schedule + escrowed row).
Error validate_row_dividends(const BatchView& v, uint64_t g, uint64_t index) {
    const fo_lsm_grouped_request& q = *v.q;
    if (!v.cash()) return nonnegative_value("continuous_dividend_yields", index, q.dividend_yields[g]);
    const double *times, *amounts;
    uint64_t n;
    v.cash_row(g, &times, &amounts, &n);
    Error e = validate_cash_schedule(index, q.maturities[g], times, n, q.maturity_boundary);
    if (!e.ok()) return e;
    if (q.dividend_model == FO_MODEL_ESCROWED_CASH_DIVIDENDS)
        return validate_escrowed_row(index, q.initial_spots[g], q.rates[g], q.volatilities[g], times, amounts, n,
                                     q.volatility_convention);
    return Error{};
}

uint64_t dividend_model_rows(const BatchView& v) {
    return v.cash() ? v.cash_rows() : v.q->n_dividend_yields;
}

// GroupedBatchLsmCallInputs::try_new (input.rs:617-706)
Error validate_grouped_inputs(const BatchView& v) {
    const fo_lsm_grouped_request& q = *v.q;
    const uint64_t groups = q.n_initial_spots;
    if (groups == 0 || q.n_strikes == 0)
        return input_error(FO_CODE_EMPTY_BATCH, "LSM call batch must contain at least one contract");
    Error e = row_count("maturities", groups, q.n_maturities);
    if (e.ok()) e = row_count("constant_continuously_compounded_rates", groups, q.n_rates);
    if (e.ok()) e = row_count("constant_volatilities", groups, q.n_volatilities);
    if (e.ok()) e = row_count("dividend_model", groups, dividend_model_rows(v));
    if (!e.ok()) return e;
    // validate_group_offsets (input.rs:761-796)
    if (q.n_group_offsets != groups + 1)
        return input_error(FO_CODE_GROUP_OFFSET_COUNT_MISMATCH, "LSM grouped batch offsets contain " + u(q.n_group_offsets) +
                                                                    " values; expected " + u(groups + 1));
    if (q.group_offsets[0] != 0)
        return input_error(FO_CODE_GROUP_OFFSETS_DO_NOT_START_AT_ZERO,
                           "LSM grouped batch offsets must start at zero; observed " + u(q.group_offsets[0]));
    for (uint64_t g = 0; g < groups; ++g) {
        if (q.group_offsets[g] >= q.group_offsets[g + 1])
            return input_error(FO_CODE_INVALID_GROUP_RANGE, "LSM grouped batch range " + u(g) +
                                                                " must be nonempty and increasing; observed [" +
                                                                u(q.group_offsets[g]) + ", " + u(q.group_offsets[g + 1]) + ")");
    }
    if (uint64_t(q.group_offsets[groups]) != q.n_strikes)
        return input_error(FO_CODE_GROUP_OFFSET_END_MISMATCH, "LSM grouped batch terminal offset is " +
                                                                  u(q.group_offsets[groups]) + "; expected " +
                                                                  u(q.n_strikes) + " contract rows");
    for (uint64_t r = 0; r < q.n_strikes; ++r) {
        e = positive_value("strikes", r, q.strikes[r]);
        if (!e.ok()) return e;
    }
    for (uint64_t g = 0; g < groups; ++g) {
        e = nonnegative_value("initial_spots", g, q.initial_spots[g]);
        if (e.ok()) e = positive_value("maturities", g, q.maturities[g]);
        if (e.ok()) e = finite_value("constant_continuously_compounded_rates", g, q.rates[g]);
        if (e.ok()) e = positive_value("constant_volatilities", g, q.volatilities[g]);
        if (e.ok()) e = validate_row_dividends(v, g, g);
        if (!e.ok()) return e;
    }
    return Error{};
}

// BatchLsmCallInputs::try_new (input.rs:502-585)
Error validate_row_inputs(const BatchView& v) {
    const fo_lsm_grouped_request& q = *v.q;
    const uint64_t rows = q.n_initial_spots;
    if (rows == 0) return input_error(FO_CODE_EMPTY_BATCH, "LSM call batch must contain at least one contract");
    Error e = row_count("strikes", rows, q.n_strikes);
    if (e.ok()) e = row_count("maturities", rows, q.n_maturities);
    if (e.ok()) e = row_count("constant_continuously_compounded_rates", rows, q.n_rates);
    if (e.ok()) e = row_count("constant_volatilities", rows, q.n_volatilities);
    if (e.ok()) e = row_count("dividend_model", rows, dividend_model_rows(v));
    if (!e.ok()) return e;
    for (uint64_t r = 0; r < rows; ++r) {
        e = nonnegative_value("initial_spots", r, q.initial_spots[r]);
        if (e.ok()) e = positive_value("strikes", r, q.strikes[r]);
        if (e.ok()) e = positive_value("maturities", r, q.maturities[r]);
        if (e.ok()) e = finite_value("constant_continuously_compounded_rates", r, q.rates[r]);
        if (e.ok()) e = positive_value("constant_volatilities", r, q.volatilities[r]);
        if (e.ok()) e = validate_row_dividends(v, r, r);
        if (!e.ok()) return e;
    }
    return Error{};
}

// BatchRandomStreams::validate (input.rs:201-255)
Error validate_streams(const fo_lsm_grouped_request& q, uint64_t rows) {
    auto end = [&](const char* population, uint32_t start, uint64_t* out) -> Error {
        const uint64_t e = uint64_t(start) + rows;
        if (e > kU32Max + 1)
            return input_error(FO_CODE_RANDOM_DOMAIN_RANGE_OVERFLOW, std::string("batched LSM ") + population +
                                                                         " random domains starting at " + u(start) +
                                                                         " cannot address " + u(rows) + " rows");
        *out = e;
        return Error{};
    };
    uint64_t te = 0, ee = 0;
    Error e = end("training", q.training_domain_start, &te);
    if (!e.ok()) return e;
    e = end("evaluation", q.evaluation_domain_start, &ee);
    if (!e.ok()) return e;
    const uint64_t ts = q.training_domain_start, es = q.evaluation_domain_start;
    if (ts < ee && es < te)
        return input_error(FO_CODE_RANDOM_DOMAIN_RANGE_COLLISION, "batched LSM training domains [" + u(ts) + ", " + u(te) +
                                                                      ") overlap evaluation domains [" + u(es) + ", " +
                                                                      u(ee) + ")");
    return Error{};
}

Error cash_mesh_row(uint64_t row, double maturity, double rate, const double* times, uint64_t n) {
    if (rate < 0.0)
        return input_error(FO_CODE_NEGATIVE_RATE_FOR_CASH_MESH,
                           "cash-dividend-date exercise mesh requires a nonnegative continuously compounded rate at batch row " +
                               u(row) + "; observed " + fmt_f64(rate));
    for (uint64_t event = 0; event < n; ++event)
        if (bits(times[event]) == bits(maturity))
            return input_error(FO_CODE_TERMINAL_CASH_FOR_CASH_MESH,
                               "cash-dividend-date exercise mesh does not admit terminal cash at batch row " + u(row) +
                                   ", event " + u(event) + "; event and maturity are " + fmt_f64(maturity));
    return Error{};
}

Error explicit_times_row(uint64_t row, double maturity, const double* times, uint64_t n) {
    for (uint64_t event = 0; event < n; ++event)
        if (times[event] >= maturity)
            return input_error(FO_CODE_EXPLICIT_EXERCISE_AT_OR_AFTER_MATURITY,
                               "explicit exercise time at batch row " + u(row) + ", event " + u(event) + ", time " +
                                   fmt_f64(times[event]) + " must be strictly before maturity " + fmt_f64(maturity));
    return Error{};
}

// validate_exercise_mesh_domain (pricing.rs:356-400 rows, 622-664 groups)
Error validate_mesh_domain(const BatchView& v) {
    const fo_lsm_grouped_request& q = *v.q;
    const uint64_t groups = v.groups();
    if (q.exercise_mesh == FO_MESH_CASH_DIVIDEND_DATES) {
        if (!v.cash())
            return input_error(FO_CODE_CASH_MESH_REQUIRES_CASH_DIVIDENDS,
                               "cash-dividend-date exercise mesh requires a deterministic cash-dividend model");
        for (uint64_t g = 0; g < groups; ++g) {
            const double *times, *amounts;
            uint64_t n;
            v.cash_row(g, &times, &amounts, &n);
            Error e = cash_mesh_row(v.first_row(g), q.maturities[g], q.rates[g], times, n);
            if (!e.ok()) return e;
        }
    } else if (q.exercise_mesh == FO_MESH_EXPLICIT_TIMES) {
        if (v.explicit_rows() != groups) return row_count("explicit_exercise_times", groups, v.explicit_rows());
        for (uint64_t g = 0; g < groups; ++g) {
            const double* times;
            uint64_t n;
            v.explicit_row(g, &times, &n);
            Error e = explicit_times_row(v.first_row(g), q.maturities[g], times, n);
            if (!e.ok()) return e;
        }
    }
    return Error{};
}

// ---- per-group plan (build_path_plan, pricing.rs:704-748) -------------------------------------

uint32_t next_base_node(uint32_t node, uint32_t final_node, bool* done) {
    if (node == final_node) {
        *done = true;
        return node;
    }
    return node + 1;
}

// exact_union_times (pricing.rs:967-1047)
Error exact_union_times(uint64_t row, double maturity, uint32_t base_intervals, const double* cash, uint64_t n_cash,
                        std::vector<double>* out) {
    const uint64_t capacity = uint64_t(base_intervals) + 1 + n_cash;
    if (capacity - 1 > kU32Max)
        return input_error(FO_CODE_CONTRACT_MESH_SHAPE_OVERFLOW, "LSM batch mesh shape overflow at row " + u(row) + " for " +
                                                                     u(base_intervals) + " base intervals and " + u(n_cash) +
                                                                     " cash events");
    std::vector<double>& times = *out;
    times.clear();
    times.reserve(capacity);
    bool base_done = false;
    uint32_t base_node = 0;
    uint64_t event = 0;
    while (!base_done || event < n_cash) {
        double base = 0.0;
        if (!base_done) base = base_node == base_intervals ? maturity : maturity * (double(base_node) / double(base_intervals));
        if (!base_done && event < n_cash) {
            const int c = total_cmp(base, cash[event]);
            if (c < 0) {
                times.push_back(base);
                base_node = next_base_node(base_node, base_intervals, &base_done);
            } else if (c == 0) {
                times.push_back(base);
                base_node = next_base_node(base_node, base_intervals, &base_done);
                event += 1;
            } else {
                times.push_back(cash[event]);
                event += 1;
            }
        } else if (!base_done) {
            times.push_back(base);
            base_node = next_base_node(base_node, base_intervals, &base_done);
        } else {
            times.push_back(cash[event]);
            event += 1;
        }
    }
    return Error{};
}

// exact_explicit_union_times (pricing.rs:1049-1114)
Error exact_explicit_union_times(uint64_t row, double maturity, const double* ex, uint64_t n_ex, const double* cash,
                                 uint64_t n_cash, std::vector<double>* out) {
    const uint64_t capacity = n_ex + n_cash + 2;
    if (capacity - 1 > kU32Max)
        return input_error(FO_CODE_EXPLICIT_CONTRACT_MESH_SHAPE_OVERFLOW,
                           "LSM explicit batch mesh shape overflow at row " + u(row) + " for " + u(n_ex) +
                               " exercise events and " + u(n_cash) + " cash events");
    std::vector<double>& times = *out;
    times.clear();
    times.reserve(capacity);
    times.push_back(0.0);
    uint64_t e = 0, c = 0;
    while (e < n_ex || c < n_cash) {
        double next;
        if (e < n_ex && c < n_cash) {
            const int cmp = total_cmp(ex[e], cash[c]);
            if (cmp < 0) {
                next = ex[e++];
            } else if (cmp == 0) {
                next = ex[e++];
                c++;
            } else {
                next = cash[c++];
            }
        } else if (e < n_ex) {
            next = ex[e++];
        } else {
            next = cash[c++];
        }
        if (next < maturity) times.push_back(next);
    }
    times.push_back(maturity);
    return Error{};
}

// Index of `t` in the strictly increasing grid by total order, or -1.
int64_t find_exact(const std::vector<double>& grid, double t) {
    size_t lo = 0, hi = grid.size();
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        const int c = total_cmp(grid[mid], t);
        if (c == 0) return int64_t(mid);
        if (c < 0) lo = mid + 1;
        else hi = mid;
    }
    return -1;
}

// EscrowedGbmPathPlan prepaid cash by node (path.rs:889-944).
Error escrowed_prepaid_cash(const std::vector<double>& log_discounts, const std::vector<uint32_t>& dividend_nodes,
                            const std::vector<double>& amounts, std::vector<double>* out) {
    const size_t n = log_discounts.size();
    std::vector<double> prepaid(n, 0.0);
    size_t event = dividend_nodes.size();
    const size_t last = n - 1;
    if (event > 0 && dividend_nodes[event - 1] == last) {
        event -= 1;
        prepaid[last] = amounts[event];
    }
    for (size_t node = n - 1; node-- > 0;) {
        const double interval = log_discounts[node + 1] - log_discounts[node];
        const double discounted_future = prepaid[node + 1] * std::exp(interval);
        double same_node_cash = 0.0;
        if (event > 0 && dividend_nodes[event - 1] == node) {
            event -= 1;
            same_node_cash = amounts[event];
        }
        const double value = discounted_future + same_node_cash;
        if (!std::isfinite(value))
            return make_error(FO_ERR_SIMULATION, FO_CODE_NON_FINITE_ESCROWED_PREPAID_CASH,
                              "escrowed-dividend prepaid cash is not finite at node " + u(node) +
                                  "; discounted later cash is " + fmt_f64(discounted_future) + " and same-node cash is " +
                                  fmt_f64(same_node_cash));
        prepaid[node] = value;
    }
    double origin = 0.0;
    for (size_t i = 0; i < dividend_nodes.size(); ++i) {
        const double discounted_future = amounts[i] * std::exp(log_discounts[dividend_nodes[i]]);
        origin += discounted_future;
        if (!std::isfinite(origin))
            return make_error(FO_ERR_SIMULATION, FO_CODE_NON_FINITE_ESCROWED_PREPAID_CASH,
                              "escrowed-dividend prepaid cash is not finite at node 0; discounted later cash is " +
                                  fmt_f64(discounted_future) + " and same-node cash is 0.0");
    }
    prepaid[0] = origin;
    *out = std::move(prepaid);
    return Error{};
}

// Conventions shared by every group of a batch.
struct BatchMethod {
    int32_t mesh = FO_MESH_UNIFORM;
    uint32_t base_intervals = 0;
    int32_t origin = FO_ORIGIN_EXCLUDED;
    bool cash = false;         // cash-dividend schedules (spot or escrowed)
    bool escrowed = false;
    int32_t policy = FO_DIVIDEND_LIQUIDATOR;
    int32_t convention = FO_ESCROWED_PREPAID_FORWARD;
    uint64_t train_seed = 0, eval_seed = 0;
    int32_t degree = 4;
    double rank_tolerance = 1e-12, condition_limit = 1e8;
    int32_t tie_rule = FO_TIE_STRICTLY_GREATER, support = FO_SUPPORT_FAIL;
};

// One group: its market, its schedule and its two populations.
struct GroupSpec {
    uint64_t first_row = 0, end_row = 0;
    double s0 = 0.0, maturity = 0.0, rate = 0.0, vol = 0.0, yield = 0.0;
    const double* cash_times = nullptr;
    const double* cash_amounts = nullptr;
    uint64_t n_cash = 0;
    const double* ex_times = nullptr;  // explicit meshes
    uint64_t n_ex = 0;
    uint64_t train_paths = 0, eval_paths = 0;
    uint32_t train_domain = 0, eval_domain = 0;
};

struct GroupWork {
    HostPlan hp;              // simulation plan + method (strike unused)
    double sigma = 0.0;       // the simulated constant volatility
    uint64_t first_row = 0, end_row = 0;
    Error build;              // build_path_plan failure: the group's error at first_row
    Error fit;                // discount failure raised by the first strike's fit
};

BatchMethod method_of(const fo_lsm_grouped_request& q) {
    BatchMethod m;
    m.mesh = q.exercise_mesh;
    m.base_intervals = q.base_intervals;
    m.origin = q.exercise_mesh == FO_MESH_CASH_DIVIDEND_DATES ? int32_t(FO_ORIGIN_EXCLUDED) : q.origin_exercise;
    m.cash = q.dividend_model != FO_MODEL_CONTINUOUS_YIELD;
    m.escrowed = q.dividend_model == FO_MODEL_ESCROWED_CASH_DIVIDENDS;
    m.policy = q.dividend_model == FO_MODEL_CASH_DIVIDENDS ? q.dividend_policy : int32_t(FO_DIVIDEND_LIQUIDATOR);
    m.convention = q.volatility_convention;
    m.train_seed = q.training_seed;
    m.eval_seed = q.evaluation_seed;
    m.degree = int32_t(q.polynomial_degree);
    m.rank_tolerance = q.rank_tolerance;
    m.condition_limit = q.condition_limit;
    m.tie_rule = q.tie_rule;
    m.support = q.insufficient_exercise_support;
    return m;
}

GroupSpec spec_of(const BatchView& v, uint64_t g) {
    const fo_lsm_grouped_request& q = *v.q;
    GroupSpec s;
    s.first_row = v.first_row(g);
    s.end_row = v.end_row(g);
    s.s0 = q.initial_spots[g];
    s.maturity = q.maturities[g];
    s.rate = q.rates[g];
    s.vol = q.volatilities[g];
    s.yield = v.cash() ? 0.0 : q.dividend_yields[g];
    if (v.cash()) v.cash_row(g, &s.cash_times, &s.cash_amounts, &s.n_cash);
    if (q.exercise_mesh == FO_MESH_EXPLICIT_TIMES) v.explicit_row(g, &s.ex_times, &s.n_ex);
    s.train_paths = q.training_paths;
    s.eval_paths = q.evaluation_paths;
    s.train_domain = uint32_t(uint64_t(q.training_domain_start) + g);
    s.eval_domain = uint32_t(uint64_t(q.evaluation_domain_start) + g);
    return s;
}

Error build_group(const BatchMethod& m, const GroupSpec& gs, GroupWork* w) {
    const uint64_t row = gs.first_row;
    const double maturity = gs.maturity, rate = gs.rate, s0 = gs.s0;
    const double* cash_times = gs.cash_times;
    const double* cash_amounts = gs.cash_amounts;
    const uint64_t n_cash = gs.n_cash;
    // resolve_exercise_mesh (pricing.rs:750-800)
    std::vector<double> times;
    const double* ex_times = nullptr;
    uint64_t n_ex = 0;
    bool all_transition = true;
    int32_t origin = FO_ORIGIN_EXCLUDED;
    Error e;
    if (m.mesh == FO_MESH_UNIFORM) {
        e = exact_union_times(row, maturity, m.base_intervals, cash_times, n_cash, &times);
        origin = m.origin;
    } else if (m.mesh == FO_MESH_CASH_DIVIDEND_DATES) {
        e = cash_mesh_row(row, maturity, rate, cash_times, n_cash);
        if (e.ok()) e = exact_union_times(row, maturity, 1, cash_times, n_cash, &times);
    } else {
        ex_times = gs.ex_times;
        n_ex = gs.n_ex;
        e = explicit_times_row(row, maturity, ex_times, n_ex);
        if (e.ok()) e = exact_explicit_union_times(row, maturity, ex_times, n_ex, cash_times, n_cash, &times);
        all_transition = false;
        origin = m.origin;
    }
    if (!e.ok()) return e;
    e = validate_time_grid(times);
    if (!e.ok()) return financial_at_row(row, e);
    // build_row_curves (pricing.rs:862-893)
    const size_t n = times.size();
    const double yield = gs.yield;
    std::vector<double> log_discounts(n), yields(n);
    for (size_t i = 0; i < n; ++i) {
        log_discounts[i] = i == 0 ? 0.0 : -rate * times[i];
        yields[i] = i == 0 ? 0.0 : yield * times[i];
    }
    e = validate_log_discount_curve(times, log_discounts);
    if (e.ok()) e = validate_cumulative_yield_curve(times, yields);
    if (!e.ok()) return financial_at_row(row, e);
    // build_row_schedule (pricing.rs:895-965)
    std::vector<uint32_t> dividend_nodes;
    std::vector<double> dividend_amounts;
    for (uint64_t event = 0; event < n_cash; ++event) {
        const int64_t node = find_exact(times, cash_times[event]);
        if (node < 0)
            return input_error(FO_CODE_CASH_DIVIDEND_NODE_MISSING, "cash dividend at batch row " + u(row) + ", event " +
                                                                       u(event) + ", time " + fmt_f64(cash_times[event]) +
                                                                       " is absent from its exact union mesh");
        e = validate_cash_dividend(uint32_t(node), cash_amounts[event]);
        if (!e.ok()) return financial_at_row(row, e);
        dividend_nodes.push_back(uint32_t(node));
        dividend_amounts.push_back(cash_amounts[event]);
    }
    std::vector<uint32_t> exercise;
    if (all_transition) {
        const size_t start = origin == FO_ORIGIN_EXCLUDED ? 1 : 0;
        for (size_t node = start; node + 1 < n; ++node) exercise.push_back(uint32_t(node));
    } else {
        if (origin == FO_ORIGIN_INCLUDED) exercise.push_back(0);
        for (uint64_t event = 0; event < n_ex; ++event) {
            const int64_t node = find_exact(times, ex_times[event]);
            if (node < 0)
                return input_error(FO_CODE_EXPLICIT_EXERCISE_NODE_MISSING, "exercise time at batch row " + u(row) +
                                                                               ", event " + u(event) + ", time " +
                                                                               fmt_f64(ex_times[event]) +
                                                                               " is absent from its exact union mesh");
            exercise.push_back(uint32_t(node));
        }
    }
    const uint32_t expiry = uint32_t(n - 1);
    e = validate_event_schedule(times, dividend_nodes, dividend_amounts, exercise, expiry);
    if (!e.ok()) return financial_at_row(row, e);
    // path_volatility (pricing.rs:840-860)
    double volatility = gs.vol;
    const bool escrowed = m.escrowed;
    if (escrowed && m.convention == FO_ESCROWED_SPOT_MATCHED_AT_ORIGIN) {
        double prepaid = 0.0;
        e = escrowed_origin_prepaid_cash(row, rate, cash_times, cash_amounts, n_cash, &prepaid);
        if (!e.ok()) return e;
        volatility = volatility * s0 / (s0 - prepaid);
    }
    e = validate_constant_volatility(volatility);
    if (!e.ok()) return financial_at_row(row, e);
    w->sigma = volatility;
    HostPlan& hp = w->hp;
    if (escrowed) {
        // Risky prepaid forward: no yield, no cash jumps; the prepaid cash is added back per row.
        std::vector<double> prepaid;
        e = escrowed_prepaid_cash(log_discounts, dividend_nodes, dividend_amounts, &prepaid);
        if (!e.ok()) return plan_at_row(row, e);
        const std::vector<double> zero(n, 0.0);
        e = build_gbm_plan(times.data(), n, times.data(), n, log_discounts.data(), n, times.data(), n, zero.data(), n,
                           nullptr, 0, nullptr, 0, exercise.data(), exercise.size(), expiry, volatility,
                           FO_DIVIDEND_LIQUIDATOR, &hp);
        if (!e.ok()) return plan_at_row(row, e);
        hp.escrowed = true;
        for (size_t r = 0; r < hp.row_node.size(); ++r) {
            const uint32_t node = hp.row_node[r];
            hp.escrow_cash[r] = node == expiry ? 0.0 : prepaid[node];
        }
        hp.sim_start = s0 - prepaid[0];
    } else {
        const int32_t policy = m.policy;
        e = build_gbm_plan(times.data(), n, times.data(), n, log_discounts.data(), n, times.data(), n, yields.data(), n,
                           dividend_nodes.data(), dividend_nodes.size(), dividend_amounts.data(), dividend_amounts.size(),
                           exercise.data(), exercise.size(), expiry, volatility, policy, &hp);
        if (!e.ok()) return plan_at_row(row, e);
        hp.sim_start = s0;
    }
    hp.initial_spot = s0;
    hp.strike = 0.0;
    hp.train_paths = gs.train_paths;
    hp.eval_paths = gs.eval_paths;
    hp.train_seed = m.train_seed;
    hp.eval_seed = m.eval_seed;
    hp.train_domain = gs.train_domain;
    hp.eval_domain = gs.eval_domain;
    hp.degree = m.degree;
    hp.rank_tolerance = m.rank_tolerance;
    hp.condition_limit = m.condition_limit;
    hp.tie_rule = m.tie_rule;
    hp.support = m.support;
    // Discounts of the fit (policy.rs:1049-1108): a failure is the first strike's fit error.
    Error fit = finish_discounts(&hp);
    if (!fit.ok()) {
        w->fit = fit;
        hp.disc_from_later.assign(hp.rows(), 1.0);
        hp.disc_to_origin.assign(hp.rows(), 1.0);
        hp.origin_discount = 1.0;
    }
    return Error{};
}

// ---- device layout of one wave ------------------------------------------------------------------

struct WaveLayout {
    size_t groups, problems, items, group_status, problem_status, summaries;  // read-back region: group_status..summaries
    size_t counters;
    size_t greek_sums;                                                  // (read back, Greeks only)
    size_t counts, itm_counts, stop_counts, eval_partials, greek_partials, records, values, slab, replay;
    size_t team_arrive, team_slots;
    size_t out_begin, out_bytes, clear_begin, clear_bytes, total;
};

struct Wave {
    uint64_t g0 = 0, g1 = 0;     // groups [g0, g1)
    uint64_t problems = 0;       // strike rows
    uint64_t records = 0;        // FitRecords (rows per problem)
    uint64_t slab_elems = 0;     // stored training states
    uint64_t value_elems = 0;    // training values of every problem
    uint32_t eval_blocks = 0;    // largest evaluation grid of a group
    uint32_t train_blocks = 0;   // largest training grid of a group
    uint64_t partial_slots = 0;  // evaluation blocks summed over the problems (one partial slot each)
    uint64_t item_bound = 0;     // work items of the persistent launch, at most (one block per item)
    uint64_t team_slots = 0;     // exchange slots (double2) of the teams of large problems
    bool greeks = false;         // adjoint Greeks buffers
};

uint32_t eval_blocks_for(uint64_t eval_paths) {
    return uint32_t((eval_paths + kBatchEvalThreads - 1) / kBatchEvalThreads);
}

// CTAs that fit a problem of `train_paths` paths together (one up to kTeamPaths).
uint32_t team_members(uint64_t train_paths) {
    const uint64_t m = (train_paths + kTeamPaths - 1) / kTeamPaths;
    return uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(m, kMaxTeam)));
}

WaveLayout layout_for(const Wave& w, size_t base) {
    WaveLayout L{};
    size_t off = base;
    auto take = [&](size_t bytes) {
        off = align_up(off, 256);
        const size_t at = off;
        off += bytes;
        return at;
    };
    const uint64_t G = w.g1 - w.g0, P = w.problems;
    L.groups = take(sizeof(BatchGroup) * G);
    L.problems = take(sizeof(BatchProblem) * P);
    L.items = take(sizeof(BatchItem) * std::max<uint64_t>(w.item_bound, 1));
    off = align_up(off, 256);
    L.out_begin = off;
    L.group_status = take(sizeof(GroupStatus) * G);
    L.problem_status = take(sizeof(ProblemStatus) * P);
    L.summaries = take(sizeof(ProblemSummary) * P);
    L.greek_sums = take(w.greeks ? sizeof(double) * kGreekSlots * P : 0);
    off = align_up(off, 256);
    L.out_bytes = off - L.out_begin;
    L.clear_begin = off;
    L.counts = take(sizeof(unsigned) * 2 * P);
    L.itm_counts = take(sizeof(unsigned) * w.records);
    L.stop_counts = take(w.greeks ? sizeof(unsigned) * w.records : 0);
    L.records = take(sizeof(FitRecord) * w.records);
    // next item (one launch), timeout, next item of each phase kernel, sim / bwd / eval done per group
    L.counters = take(sizeof(unsigned) * (3 * G + 5));
    L.team_arrive = take(sizeof(unsigned) * P);
    off = align_up(off, 256);
    L.clear_bytes = off - L.clear_begin;
    L.eval_partials = take(sizeof(double2) * 2 * std::max<uint64_t>(w.partial_slots, 1));
    L.greek_partials = take(w.greeks ? sizeof(double2) * kGreekSlots * w.partial_slots : 0);
    L.replay = take(sizeof(SimFailure));
    L.team_slots = take(sizeof(double2) * std::max<uint64_t>(w.team_slots, 1));
    L.values = take(sizeof(double) * std::max<uint64_t>(w.value_elems, 1));
    L.slab = take(sizeof(double) * std::max<uint64_t>(w.slab_elems, 1));
    L.total = align_up(off, 256);
    return L;
}

// Offsets of one group's plan arrays inside the batch input block (uploaded once per call).
struct InputOffsets {
    size_t steps, events, row_node, disc_from_later, disc_to_origin, escrow_cash;
};

DevicePlan device_plan(const HostPlan& hp, const InputOffsets& o, unsigned char* dev) {
    DevicePlan p{};
    p.intervals = hp.intervals();
    p.rows = hp.rows();
    p.first_stored_row = hp.origin_row ? 1u : 0u;
    p.strike = 0.0;
    p.sim_start = hp.sim_start;
    p.initial_spot = hp.initial_spot;
    p.policy = hp.policy;
    p.escrowed = hp.escrowed ? 1 : 0;
    p.degree = hp.degree;
    p.tie_rule = hp.tie_rule;
    p.support = hp.support;
    p.origin_row = hp.origin_row ? 1 : 0;
    p.rank_tolerance = hp.rank_tolerance;
    p.condition_limit = hp.condition_limit;
    p.rank_limit = rank_limit(hp.rank_tolerance);
    p.train_paths = hp.train_paths;
    p.eval_paths = hp.eval_paths;
    p.train_seed = hp.train_seed;
    p.eval_seed = hp.eval_seed;
    p.train_domain = hp.train_domain;
    p.eval_domain = hp.eval_domain;
    p.steps = reinterpret_cast<const StepCoef*>(dev + o.steps);
    p.events = reinterpret_cast<const NodeEvent*>(dev + o.events);
    p.row_node = reinterpret_cast<const uint32_t*>(dev + o.row_node);
    p.disc_from_later = reinterpret_cast<const double*>(dev + o.disc_from_later);
    p.disc_to_origin = reinterpret_cast<const double*>(dev + o.disc_to_origin);
    p.escrow_cash = reinterpret_cast<const double*>(dev + o.escrow_cash);
    p.origin_discount = hp.origin_discount;
    return p;
}

// ---- failure reports ------------------------------------------------------------------------------

struct BatchRun {
    fo_executor* ex;
    std::vector<GroupWork>* work;
    std::vector<DevicePlan>* plans;
    const std::vector<uint64_t>* slab_of;  // wave-local group -> first slab element
    unsigned char* dev;
    WaveLayout L;
    Wave w;
};

Error replay_path(const BatchRun& run, uint64_t g, bool training, uint64_t path, int want_row, SimFailure* out) {
    const HostPlan& hp = (*run.work)[g].hp;
    auto* d = reinterpret_cast<SimFailure*>(run.dev + run.L.replay);
    FO_CUDA_TRY(launch_replay((*run.plans)[g], training ? hp.train_seed : hp.eval_seed,
                              training ? hp.train_domain : hp.eval_domain, uint32_t(path), want_row, d, run.ex->stream),
                "replay launch");
    FO_CUDA_TRY(cudaMemcpyAsync(out, d, sizeof(SimFailure), cudaMemcpyDeviceToHost, run.ex->stream), "replay copy");
    FO_CUDA_TRY(cudaStreamSynchronize(run.ex->stream), "replay");
    return Error{};
}

Error simulation_failure(const BatchRun& run, uint64_t g, bool training, uint64_t path) {
    SimFailure f{};
    Error e = replay_path(run, g, training, path, -1, &f);
    if (!e.ok()) return e;
    Error out = lsm_error(simulation_failure_code(f.code), std::string("LSM ") + (training ? "training" : "evaluation") +
                                                               " simulation failed: " +
                                                               simulation_failure_message(f.code, uint32_t(f.interval), path,
                                                                                          f.spot, f.normal));
    out.path = int64_t(path);
    return estimator_at_row((*run.work)[g].first_row, out);
}

Error read_record(const BatchRun& run, uint64_t record, FitRecord* out) {
    FO_CUDA_TRY(cudaMemcpy(out, run.dev + run.L.records + record * sizeof(FitRecord), sizeof(FitRecord),
                           cudaMemcpyDeviceToHost),
                "record read");
    return Error{};
}

// The fit error of problem `i` (wave-local) at its first failing backward order.
Error fit_error(const BatchRun& run, uint64_t g, uint64_t row, const BatchProblem& pr, const ProblemStatus& st,
                const ProblemSummary& s) {
    const HostPlan& hp = (*run.work)[g].hp;
    const uint32_t E = hp.rows() - 1;
    const uint32_t order = s.fit_fail_order;
    Error e;
    if (s.fit_fail_kind == kFitFailPayoff) {
        const uint64_t path = st.fit_payoff_fail & kU32Max;
        e = lsm_error(FO_CODE_NON_FINITE_DISCOUNTED_PAYOFF, "LSM evaluation produced non-finite discounted payoff at path " + u(path));
        e.path = int64_t(path);
        return estimator_at_row(row, e);
    }
    const uint32_t r = E - 1 - order;
    const uint32_t node = hp.row_node[r];
    FitRecord rec{};
    Error re = read_record(run, pr.records + r, &rec);
    if (!re.ok()) return re;
    switch (s.fit_fail_kind) {
        case kFitFailNonFinite: {
            const uint64_t path = st.fit_nonfinite & kU32Max;
            e = lsm_error(FO_CODE_NON_FINITE_PREDICTOR, "continuation regression failed at exercise node " + node_str(node) +
                                                            ": regression predictor or response at path " + u(path) +
                                                            " must be finite");
            e.node = node;
            e.path = int64_t(path);
            break;
        }
        case kFitFailFit: e = fit_failure(hp, rec, node); break;
        case kFitFailDiagnostic: e = diag_failure(hp, rec, node); break;
        default: {
            // The stored state of the failing path at the row (time-major group slab).
            const uint64_t path = st.fit_predict_fail & kU32Max;
            const uint64_t elem = (*run.slab_of)[g - run.w.g0] + uint64_t(r - (hp.origin_row ? 1u : 0u)) * hp.train_paths + path;
            double spot = 0.0;
            FO_CUDA_TRY(cudaMemcpy(&spot, run.dev + run.L.slab + elem * sizeof(double), sizeof(double), cudaMemcpyDeviceToHost),
                        "state read");
            e = lsm_error(FO_CODE_NON_FINITE_PREDICTION, "continuation prediction failed at exercise node " + node_str(node) +
                                                             ", path " + u(path) +
                                                             ": polynomial regression produced non-finite prediction for predictor " +
                                                             fmt_f64(spot / pr.strike));
            e.node = node;
            e.path = int64_t(path);
            break;
        }
    }
    return estimator_at_row(row, e);
}

// The evaluation error of a problem, if any, in the reference's order (policy.rs:642-834).
Error evaluation_error(const BatchRun& run, uint64_t g, uint64_t row, const BatchProblem& pr, const ProblemStatus& st,
                       const ProblemSummary& s) {
    if (s.origin_exercised) return Error{};
    const HostPlan& hp = (*run.work)[g].hp;
    const uint64_t eval_row = st.eval_fail != kNone ? (st.eval_fail >> 33) : ~0ull;
    if (s.nosupport_row != 0xffffffffu && !(eval_row < s.nosupport_row)) {
        const uint32_t node = hp.row_node[s.nosupport_row];
        Error e = lsm_error(FO_CODE_EVALUATION_OUTSIDE_TRAINING_SUPPORT,
                            u(s.nosupport_count) + " active evaluation paths are in the money at node " + node_str(node) +
                                ", but training had no in-the-money support");
        e.node = node;
        return estimator_at_row(row, e);
    }
    if (st.eval_fail != kNone) {
        const uint32_t r = uint32_t(st.eval_fail >> 33);
        const uint64_t path = (st.eval_fail >> 1) & kU32Max;
        if (st.eval_fail & 1ull) {
            Error e = lsm_error(FO_CODE_NON_FINITE_DISCOUNTED_PAYOFF,
                                "LSM evaluation produced non-finite discounted payoff at path " + u(path));
            e.path = int64_t(path);
            return estimator_at_row(row, e);
        }
        SimFailure f{};
        Error re = replay_path(run, g, false, path, int(r), &f);
        if (!re.ok()) return re;
        double spot = f.observed;
        if (hp.escrowed) spot = hp.row_node[r] == 0 ? hp.initial_spot : spot + hp.escrow_cash[r];
        const uint32_t node = hp.row_node[r];
        Error e = lsm_error(FO_CODE_NON_FINITE_PREDICTION, "continuation prediction failed at exercise node " + node_str(node) +
                                                               ", path " + u(path) +
                                                               ": polynomial regression produced non-finite prediction for predictor " +
                                                               fmt_f64(spot / pr.strike));
        e.node = node;
        e.path = int64_t(path);
        return estimator_at_row(row, e);
    }
    if (st.eval_terminal_fail != kNone) {
        Error e = lsm_error(FO_CODE_NON_FINITE_DISCOUNTED_PAYOFF,
                            "LSM evaluation produced non-finite discounted payoff at path " + u(st.eval_terminal_fail));
        e.path = int64_t(st.eval_terminal_fail);
        return estimator_at_row(row, e);
    }
    if (!std::isfinite(s.price) || !std::isfinite(s.sample_standard_deviation) || !std::isfinite(s.standard_error)) {
        Error e = lsm_error(FO_CODE_NON_FINITE_DISCOUNTED_PAYOFF, "LSM evaluation produced non-finite discounted payoff at path 0");
        e.path = 0;
        return estimator_at_row(row, e);
    }
    return Error{};
}

// ---- orchestration ----------------------------------------------------------------------------------

size_t memory_budget(const fo_executor* ex) {
    size_t free_bytes = 0, total = 0;
    if (cudaMemGetInfo(&free_bytes, &total) != cudaSuccess) free_bytes = size_t(8) << 30;
    const size_t usable = size_t(double(free_bytes + ex->batch.bytes) * 0.8);
    return std::min<size_t>(usable, size_t(48) << 30);
}

// Request validation in the reference's order (lib.rs:1302-1415, input.rs, pricing.rs:356-400).
Error validate_request(const BatchView& v, const fo_batch_result_columns* out) {
    const fo_lsm_grouped_request& q = *v.q;
    Error e = validate_method(q);
    if (!e.ok()) return e;
    e = validate_dividend_model(q);
    if (!e.ok()) return e;
    e = v.grouped ? validate_grouped_inputs(v) : validate_row_inputs(v);
    if (!e.ok()) return e;
    e = validate_streams(q, v.groups());
    if (!e.ok()) return e;
    e = validate_mesh_domain(v);
    if (!e.ok()) return e;
    if (out && out->rows != v.rows())
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                          "result columns hold " + u(out->rows) + " rows; the batch has " + u(v.rows()));
    return Error{};
}

// Where the adjoint Greeks of a batch go (ragged batches): the caller's columns and, per contract
// row, the index of its first cash event in dividend_sensitivities.
struct GreeksSink {
    fo_ragged_greeks_columns* cols = nullptr;
    std::vector<uint64_t> cash_first;
};

// Writes one problem's Greeks from its slot sums and per-row stopping counts (the host half of
// the adjoint; the per-path half is PathAdjoint in lsm_adjoint.cuh).
void write_greeks(const GreeksSink& sink, uint64_t row, const GroupWork& gw, double strike, const ProblemSummary& ps,
                  const double* sums, const unsigned* stops) {
    const HostPlan& hp = gw.hp;
    fo_ragged_greeks_columns& c = *sink.cols;
    double* dl = c.log_discount_sensitivities + c.log_discount_offsets[row];
    double* dd_out = c.dividend_sensitivities ? c.dividend_sensitivities + sink.cash_first[row] : nullptr;
    const uint64_t nodes = hp.times.size();
    std::vector<uint32_t> div_nodes;
    for (uint32_t node = 1; node < hp.events.size(); ++node)
        if (hp.events[node].flags & kEventDividend) div_nodes.push_back(node);
    for (uint64_t i = 0; i < nodes; ++i) dl[i] = 0.0;
    for (size_t j = 0; j < div_nodes.size() && dd_out; ++j) dd_out[j] = 0.0;
    if (ps.origin_exercised) {
        const double d = hp.initial_spot - strike;
        c.delta[row] = d > 0.0 ? 1.0 : 0.0;
        c.vega[row] = 0.0;
        dl[0] = d > 0.0 ? d : 0.0;
        return;
    }
    const double n = double(hp.eval_paths);
    c.delta[row] = sums[kGreekDelta] / n;
    c.vega[row] = sums[kGreekVega] / n;
    dl[0] += sums[kGreekL0] / n;
    for (size_t j = 0; j < div_nodes.size(); ++j) {
        dl[div_nodes[j]] += sums[kGreekJump + j] / n;
        if (dd_out) dd_out[j] = sums[kGreekDividend + j] / n;
    }
    const uint32_t rows = hp.rows();
    for (uint32_t r = 0; r + 1 < rows; ++r)
        if (stops[r]) dl[hp.row_node[r]] += -strike * hp.disc_to_origin[r] * double(stops[r]) / n;
    dl[hp.row_node[rows - 1]] += sums[kGreekTerminal] / n;
}

// Shape class of a wave for the autotuner: launches of one class share their best launch shape.
template <typename Work, typename WaveT>
std::string tuning_key(const Work& work, const WaveT& w, bool greeks, int degree, uint32_t max_rows,
                       uint32_t max_strikes) {
    uint64_t max_paths = 1;
    for (uint64_t g = w.g0; g < w.g1; ++g) max_paths = std::max<uint64_t>(max_paths, work[g].hp.train_paths);
    auto log2_ceil = [](uint64_t v) {
        int k = 0;
        while ((uint64_t(1) << k) < v && k < 63) ++k;
        return k;
    };
    return std::to_string(greeks) + "/" + std::to_string(degree) + "/" + std::to_string(log2_ceil(max_paths)) + "/" +
           std::to_string((max_rows + 15) / 16) + "/" + std::to_string(max_strikes) + "/" +
           std::to_string(log2_ceil(w.g1 - w.g0));
}

// The autotuner: a coordinate search from the default launch shape over the executor (one persistent
// launch or the phase kernels), the evaluation blocks per item, the simulation blocks per item,
// the strikes per evaluation item and the CTAs per SM, each candidate timed by one launch of the
// wave; a change is kept when it is at least 1% faster.
template <typename Run>
Error autotune_wave(Run& run, bool greeks, int max_strikes, BatchTuning* best, uint64_t* runs) {
    BatchTuning cur;
    float cur_ms = 0.f;
    // The first launch of a wave meets a cold L2 and freshly reserved memory: run the default once
    // untimed, so that it is timed on the same footing as the candidates after it.
    Error e = run(cur, &cur_ms);
    if (e.ok()) e = run(cur, &cur_ms);
    if (!e.ok()) return e;
    *runs = 2;
    auto attempt = [&](BatchTuning cand) -> Error {
        float ms = 0.f;
        Error te = run(cand, &ms);
        if (!te.ok()) return te;
        *runs += 1;
        if (ms < 0.99f * cur_ms) {
            cur = cand;
            cur_ms = ms;
        }
        return Error{};
    };
    {
        BatchTuning c = cur;  // the phase kernels instead of one persistent launch
        c.phases = 1;
        if (!(e = attempt(c)).ok()) return e;
    }
    for (const int eval_blocks : {2, 4}) {
        BatchTuning c = cur;
        c.eval_blocks = eval_blocks;
        if (!(e = attempt(c)).ok()) return e;
    }
    {
        BatchTuning c = cur;
        c.sim_blocks = 8;
        if (!(e = attempt(c)).ok()) return e;
    }
    int widest = 1;
    while (widest < kEvalStrikes && widest < max_strikes) widest *= 2;
    if (!greeks && widest > 1) {
        BatchTuning c = cur;
        c.strikes = widest / 2;
        if (!(e = attempt(c)).ok()) return e;
    }
    if (!cur.phases) {  // CTAs per SM only shape the persistent launch
        BatchTuning c = cur;
        c.ctas_per_sm = 2;
        if (!(e = attempt(c)).ok()) return e;
    }
    *best = cur;
    return Error{};
}

// Prices validated groups: host plans, waves within the memory budget, five kernels per wave,
// the lowest failing group's typed error or the row-aligned result columns (and, with a sink,
// the adjoint Greeks of every row).
Error price_groups(fo_executor* ex, const BatchMethod& m, const std::vector<GroupSpec>& specs, const double* strikes,
                   fo_batch_result_columns* out, const GreeksSink* sink = nullptr) {
    const bool greeks = sink != nullptr;
    // Per-group plans on the host. Only groups before the first one whose plan fails can matter.
    const uint64_t groups = specs.size();
    // Groups plan independently (build_group reads only its inputs), so large batches spread them
    // over host threads; the first failing group in order still bounds what is launched.
    std::vector<GroupWork> work(groups);
    auto build_range = [&](uint64_t lo, uint64_t hi) {
        for (uint64_t g = lo; g < hi; ++g) {
            GroupWork& w = work[g];
            w.first_row = specs[g].first_row;
            w.end_row = specs[g].end_row;
            w.build = build_group(m, specs[g], &w);
        }
    };
    const uint64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const uint64_t threads = std::min<uint64_t>(std::min<uint64_t>(hw, 32), (groups + 63) / 64);
    if (threads <= 1) {
        build_range(0, groups);
    } else {
        std::vector<std::thread> pool;
        pool.reserve(threads);
        for (uint64_t t = 0; t < threads; ++t)
            pool.emplace_back(build_range, groups * t / threads, groups * (t + 1) / threads);
        for (std::thread& th : pool) th.join();
    }
    uint64_t launchable = groups;
    for (uint64_t g = 0; g < groups; ++g) {
        if (!work[g].build.ok()) {
            launchable = g;
            break;
        }
    }

    // Input block: every launchable group's plan arrays.
    std::vector<InputOffsets> offsets(launchable);
    size_t in_bytes = 0;
    auto take = [&](size_t bytes) {
        in_bytes = align_up(in_bytes, 16);
        const size_t at = in_bytes;
        in_bytes += bytes;
        return at;
    };
    for (uint64_t g = 0; g < launchable; ++g) {
        const HostPlan& hp = work[g].hp;
        InputOffsets& o = offsets[g];
        o.steps = take(sizeof(StepCoef) * std::max<size_t>(hp.steps.size(), 1));
        o.events = take(sizeof(NodeEvent) * hp.events.size());
        o.row_node = take(sizeof(uint32_t) * hp.rows());
        o.disc_from_later = take(sizeof(double) * hp.rows());
        o.disc_to_origin = take(sizeof(double) * hp.rows());
        o.escrow_cash = take(sizeof(double) * hp.rows());
    }
    in_bytes = align_up(std::max<size_t>(in_bytes, 16), 256);
    if (greeks && launchable == groups) {
        // Ragged log-discount offsets: one sensitivity per node of each row's mesh.
        int64_t at = 0;
        for (uint64_t g = 0; g < groups; ++g)
            for (uint64_t r = work[g].first_row; r < work[g].end_row; ++r) {
                sink->cols->log_discount_offsets[r] = at;
                at += int64_t(work[g].hp.times.size());
            }
        sink->cols->log_discount_offsets[out->rows] = at;
        if (uint64_t(at) > sink->cols->log_discount_capacity)
            return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                              "log-discount sensitivities need " + u(uint64_t(at)) + " entries; capacity is " +
                                  u(sink->cols->log_discount_capacity));
    }

    // Waves: consecutive groups within the memory budget (and the grid's y extent).
    const size_t budget = memory_budget(ex);
    std::vector<Wave> waves;
    {
        Wave cur;
        size_t bytes = 0;
        for (uint64_t g = 0; g < launchable; ++g) {
            const HostPlan& hp = work[g].hp;
            const uint64_t strikes_g = work[g].end_row - work[g].first_row;
            const uint64_t rows = hp.rows();
            const uint64_t stored = rows - (hp.origin_row ? 1 : 0);
            const uint32_t eval_blocks = eval_blocks_for(hp.eval_paths);
            const uint32_t train_blocks = eval_blocks_for(hp.train_paths);
            const size_t cost = sizeof(double) * (stored + strikes_g) * hp.train_paths +
                                strikes_g * (rows * (sizeof(FitRecord) + 2 * sizeof(unsigned)) +
                                             size_t(eval_blocks) * sizeof(double2) * (2 + (greeks ? kGreekSlots : 0)) +
                                             sizeof(BatchProblem) + sizeof(ProblemStatus) + sizeof(ProblemSummary) +
                                             sizeof(double) * kGreekSlots + sizeof(uint32_t) + 8) +
                                sizeof(BatchGroup) + sizeof(GroupStatus) + 1024;
            if (cur.g1 > cur.g0 && (bytes + cost > budget || cur.g1 - cur.g0 >= 65535)) {
                waves.push_back(cur);
                cur = Wave{};
                cur.g0 = cur.g1 = g;
                bytes = 0;
            }
            cur.g1 = g + 1;
            cur.problems += strikes_g;
            cur.records += strikes_g * rows;
            cur.slab_elems += stored * hp.train_paths;
            cur.value_elems += strikes_g * hp.train_paths;
            cur.eval_blocks = std::max(cur.eval_blocks, eval_blocks);
            cur.train_blocks = std::max(cur.train_blocks, train_blocks);
            cur.partial_slots += strikes_g * eval_blocks;
            const uint32_t members = team_members(hp.train_paths);
            cur.item_bound += train_blocks + strikes_g * members + strikes_g * eval_blocks;
            if (members > 1) cur.team_slots += strikes_g * 2ull * members * kTeamSlots;
            cur.greeks = greeks;
            bytes += cost;
        }
        if (cur.g1 > cur.g0) waves.push_back(cur);
    }
    size_t arena = in_bytes;
    for (const Wave& w : waves) arena = std::max(arena, layout_for(w, in_bytes).total);
    Error e = ex->batch.reserve(arena);
    if (!e.ok()) return e;
    unsigned char* dev = static_cast<unsigned char*>(ex->batch.ptr);
    std::vector<DevicePlan> plans(launchable);
    for (uint64_t g = 0; g < launchable; ++g) plans[g] = device_plan(work[g].hp, offsets[g], dev);

    // Host staging: inputs, then per wave the group / problem / item tables followed by the
    // read-back region. The two never overlap: the autotuner launches a wave several times from the
    // same tables, reading results back between the launches.
    size_t stage = in_bytes;
    for (const Wave& w : waves) {
        const WaveLayout L = layout_for(w, 0);
        stage = std::max(stage, L.out_begin + L.out_bytes + 16);
    }
    e = ex->batch_host.reserve(stage);
    if (!e.ok()) return e;
    unsigned char* host = static_cast<unsigned char*>(ex->batch_host.ptr);
    cudaStream_t s = ex->stream;
    for (cudaEvent_t& mk : ex->batch_marks)
        if (!mk) FO_CUDA_TRY(cudaEventCreate(&mk), "cudaEventCreate");
    for (double& ms : ex->batch_ms) ms = 0.0;
    ex->batch_launches = 0;
    ex->batch_graph_replays = ex->batch_graph_captures = 0;
    ex->batch_h2d = ex->batch_d2h = 0;
    if (launchable > 0) {
        std::memset(host, 0, in_bytes);
        for (uint64_t g = 0; g < launchable; ++g) {
            const HostPlan& hp = work[g].hp;
            const InputOffsets& o = offsets[g];
            std::memcpy(host + o.steps, hp.steps.data(), sizeof(StepCoef) * hp.steps.size());
            std::memcpy(host + o.events, hp.events.data(), sizeof(NodeEvent) * hp.events.size());
            std::memcpy(host + o.row_node, hp.row_node.data(), sizeof(uint32_t) * hp.rows());
            std::memcpy(host + o.disc_from_later, hp.disc_from_later.data(), sizeof(double) * hp.rows());
            std::memcpy(host + o.disc_to_origin, hp.disc_to_origin.data(), sizeof(double) * hp.rows());
            std::memcpy(host + o.escrow_cash, hp.escrow_cash.data(), sizeof(double) * hp.rows());
        }
        FO_CUDA_TRY(cudaMemcpyAsync(dev, host, in_bytes, cudaMemcpyHostToDevice, s), "batch input upload");
        ex->batch_h2d += in_bytes;
        FO_CUDA_TRY(cudaStreamSynchronize(s), "batch input upload");
    }

    std::vector<uint64_t> slab_of;
    for (const Wave& w : waves) {
        const WaveLayout L = layout_for(w, in_bytes);
        // Group and problem tables.
        auto* hg = reinterpret_cast<BatchGroup*>(host + (L.groups - in_bytes));
        auto* hpb = reinterpret_cast<BatchProblem*>(host + (L.problems - in_bytes));
        unsigned char* back = host + (L.out_begin - in_bytes);  // the read-back region, after the tables
        uint64_t slab = 0, record = 0, problem = 0, values = 0, partial = 0, team = 0;
        slab_of.assign(w.g1 - w.g0, 0);
        uint32_t max_rows = 1, max_strikes = 1;
        for (uint64_t g = w.g0; g < w.g1; ++g) {
            const HostPlan& hp = work[g].hp;
            BatchGroup& bg = hg[g - w.g0];
            bg.plan = plans[g];
            bg.slab_offset = slab;
            slab_of[g - w.g0] = slab;
            bg.first_problem = uint32_t(problem);
            bg.problems = uint32_t(work[g].end_row - work[g].first_row);
            bg.sigma = work[g].sigma;
            const uint32_t members = team_members(hp.train_paths);
            bg.fit_items = bg.problems * members;
            max_strikes = std::max(max_strikes, bg.problems);
            for (uint64_t r = work[g].first_row; r < work[g].end_row; ++r) {
                BatchProblem& pb = hpb[problem];
                pb.strike = strikes[r];
                pb.group = uint32_t(g - w.g0);
                pb.records = uint32_t(record);
                pb.values = values;
                pb.skip_fit = work[g].fit.ok() ? 0 : 1;
                pb.partial_base = uint32_t(partial);
                pb.members = members;
                pb.team_base = uint32_t(team);
                if (members > 1) team += 2ull * members * kTeamSlots;
                partial += eval_blocks_for(hp.eval_paths);
                record += hp.rows();
                values += hp.train_paths;
                problem += 1;
            }
            slab += uint64_t(hp.rows() - (hp.origin_row ? 1 : 0)) * hp.train_paths;
            max_rows = std::max<uint32_t>(max_rows, hp.rows());
        }
        // One persistent launch of the wave with launch shape `tune`. Every launch recomputes the
        // whole wave from its inputs (the state it writes is cleared first), so the result does not
        // depend on the shape or on launches before it.
        float phase_ms[3] = {0.f, 0.f, 0.f};  // the phase kernels of the last launch (phase executor)
        auto run_wave = [&](const BatchTuning& tune, float* launch_ms) -> Error {
            // The persistent launch's work queue (lsm_persistent.cu), topologically ordered: every
            // group's training simulation (largest training work first, long fits right after their
            // group's), the other fits (largest paths x rows first, ties in problem order), then the
            // groups' evaluations in the order their last fit was queued. Items cover tune.sim_blocks / tune.eval_blocks blocks of 256
            // paths; an evaluation item applies `eval_strikes` strikes together (all of a group's strikes
            // when they fit, with the Greeks one).
            const uint64_t G = w.g1 - w.g0;
            int eval_strikes = 1;
            if (!greeks)
                while (eval_strikes < kEvalStrikes && eval_strikes < int(max_strikes) && eval_strikes < tune.strikes)
                    eval_strikes *= 2;
            const size_t rule_bytes = persistent_rule_bytes(eval_strikes, greeks, max_rows);
            const bool stage = rule_bytes <= kPersistentRuleSmemBytes;
            if (greeks && !stage)
                return make_error(FO_ERR_EXECUTION, FO_CODE_CAPACITY_EXCEEDED,
                                  "adjoint Greeks of a batch hold at most " +
                                      u(kPersistentRuleSmemBytes / (sizeof(PolicyRule) + 4)) +
                                      " observation rows per contract; observed " + u(max_rows));
            // The items are written straight into their region of the pinned staging buffer, which
            // the wave layout sizes for the finest cut (w.item_bound): no per-call allocation or copy.
            BatchItem* const staged_items = reinterpret_cast<BatchItem*>(host + (L.items - in_bytes));
            uint64_t n_items = 0;
            auto push_item = [&](const BatchItem& it) {
                if (n_items < w.item_bound) staged_items[n_items] = it;
                ++n_items;
            };
            uint32_t phase_items[3] = {0, 0, 0};  // simulation, fit, evaluation items (phase order only)
            {
                const uint32_t sim_step = uint32_t(std::max(1, tune.sim_blocks));
                const uint32_t eval_step = uint32_t(std::max(1, tune.eval_blocks));
                std::vector<uint32_t> gorder(G);
                std::iota(gorder.begin(), gorder.end(), 0u);
                auto train_work = [&](uint32_t gl) {
                    const HostPlan& hp = work[w.g0 + gl].hp;
                    return uint64_t(hp.train_paths) * hp.rows() * (1 + uint64_t(hg[gl].problems));
                };
                std::stable_sort(gorder.begin(), gorder.end(),
                                 [&](uint32_t x, uint32_t y) { return train_work(x) > train_work(y); });
                // Fits by one member's work (its training paths x rows), largest first. A fit that alone
                // is long next to a CTA's share of all fitting work (at least half of it on the largest
                // grid) is queued right after its group's simulation, so it starts early instead of
                // after every group's simulation. A team's members are queued in a row.
                std::vector<std::pair<uint64_t, uint32_t>> fits;
                fits.reserve(w.problems);
                uint64_t fit_work = 0;
                for (uint64_t i = 0; i < w.problems; ++i) {
                    const HostPlan& hp = work[w.g0 + hpb[i].group].hp;
                    const uint64_t member_paths = (hp.train_paths + hpb[i].members - 1) / hpb[i].members;
                    fits.emplace_back(member_paths * hp.rows(), uint32_t(i));
                    fit_work += fits.back().first * hpb[i].members;
                }
                std::stable_sort(fits.begin(), fits.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
                const uint64_t long_fit = fit_work / (2 * uint64_t(std::max(1, ex->sms)) * kPersistentMaxCtasPerSm);
                std::vector<std::vector<uint32_t>> early(G);
                std::vector<uint32_t> late;
                for (const auto& f : fits) {
                    if (f.first >= long_fit) early[hpb[f.second].group].push_back(f.second);
                    else late.push_back(f.second);
                }
                std::vector<uint64_t> last_fit(G, 0);
                uint64_t queued_fits = 0;
                auto queue_fit = [&](uint32_t i) {
                    for (uint32_t m = 0; m < hpb[i].members; ++m)
                        push_item(BatchItem{kItemBackward, i, m, hpb[i].members, 0, {0, 0, 0}});
                    last_fit[hpb[i].group] = queued_fits++;
                };
                // The phase kernels take the items kind by kind: every simulation, then every fit
                // (largest first), then every evaluation.
                for (const uint32_t gl : gorder) {
                    const uint32_t blocks = eval_blocks_for(work[w.g0 + gl].hp.train_paths);
                    for (uint32_t b = 0; b < blocks; b += sim_step)
                        push_item(BatchItem{kItemSimulate, gl, b, std::min(sim_step, blocks - b), 0, {0, 0, 0}});
                    if (!tune.phases)
                        for (const uint32_t i : early[gl]) queue_fit(i);
                }
                phase_items[0] = uint32_t(n_items);
                if (tune.phases) {
                    for (const auto& f : fits) queue_fit(f.second);
                } else {
                    for (const uint32_t i : late) queue_fit(i);
                }
                phase_items[1] = uint32_t(n_items) - phase_items[0];
                std::vector<uint32_t> eorder(G);
                std::iota(eorder.begin(), eorder.end(), 0u);
                std::stable_sort(eorder.begin(), eorder.end(),
                                 [&](uint32_t x, uint32_t y) { return last_fit[x] < last_fit[y]; });
                for (const uint32_t gl : eorder) {
                    const uint32_t blocks = eval_blocks_for(work[w.g0 + gl].hp.eval_paths);
                    const uint32_t chunks = greeks ? hg[gl].problems : (hg[gl].problems + eval_strikes - 1) / eval_strikes;
                    for (uint32_t z = 0; z < chunks; ++z)
                        for (uint32_t b = 0; b < blocks; b += eval_step)
                            push_item(BatchItem{kItemEvaluate, gl, b, std::min(eval_step, blocks - b), z, {0, 0, 0}});
                }
                phase_items[2] = uint32_t(n_items) - phase_items[0] - phase_items[1];
            }
            if (n_items > w.item_bound)
                return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                                  "batch work queue of " + u(n_items) + " items exceeds its bound of " + u(w.item_bound));
            // The group and problem tables and the queue's items (the item region is sized for the
            // finest cut; only the items of this launch shape travel).
            const size_t table_bytes = (L.items - L.groups) + sizeof(BatchItem) * n_items;
            BatchArgs a{};
            a.groups = reinterpret_cast<const BatchGroup*>(dev + L.groups);
            a.problems = reinterpret_cast<const BatchProblem*>(dev + L.problems);
            a.n_groups = uint32_t(G);
            a.n_problems = uint32_t(w.problems);
            a.slab = reinterpret_cast<double*>(dev + L.slab);
            a.values = reinterpret_cast<double*>(dev + L.values);
            a.records = reinterpret_cast<FitRecord*>(dev + L.records);
            a.group_status = reinterpret_cast<GroupStatus*>(dev + L.group_status);
            a.problem_status = reinterpret_cast<ProblemStatus*>(dev + L.problem_status);
            a.counts = reinterpret_cast<unsigned*>(dev + L.counts);
            a.itm_counts = reinterpret_cast<unsigned*>(dev + L.itm_counts);
            a.eval_partials = reinterpret_cast<double2*>(dev + L.eval_partials);
            a.summaries = reinterpret_cast<ProblemSummary*>(dev + L.summaries);
            a.greek_partials = greeks ? reinterpret_cast<double2*>(dev + L.greek_partials) : nullptr;
            a.greek_sums = greeks ? reinterpret_cast<double*>(dev + L.greek_sums) : nullptr;
            a.stop_counts = greeks ? reinterpret_cast<unsigned*>(dev + L.stop_counts) : nullptr;
            a.team_slots = reinterpret_cast<double2*>(dev + L.team_slots);
            a.team_arrive = reinterpret_cast<unsigned*>(dev + L.team_arrive);
            a.train_blocks = w.train_blocks;
            a.eval_blocks = w.eval_blocks;
            a.degree = m.degree;
            a.rank_tolerance = m.rank_tolerance;
            a.condition_limit = m.condition_limit;
            a.tie_rule = m.tie_rule;
            a.support = m.support;
            unsigned* counters = reinterpret_cast<unsigned*>(dev + L.counters);
            BatchQueue q{};
            q.items = reinterpret_cast<const BatchItem*>(dev + L.items);
            q.n_items = uint32_t(n_items);
            q.next = counters;
            q.timeout = counters + 1;
            q.sim_done = counters + 5;
            q.bwd_done = counters + 5 + G;
            q.eval_done = counters + 5 + 2 * G;
            // The phase kernels' parts of the queue (the items are in phase order then).
            BatchQueue qs[3] = {q, q, q};
            {
                uint32_t at = 0;
                for (int k = 0; k < 3; ++k) {
                    qs[k].items = q.items + at;
                    qs[k].n_items = phase_items[k];
                    qs[k].next = counters + 2 + k;
                    at += phase_items[k];
                }
            }
            cudaEvent_t* mark = ex->batch_marks;
            int grid = 0;
            PersistentLaunch launch[4] = {};
            const int n_launches = tune.phases ? 4 : 1;
            if (tune.phases) {
                FO_CUDA_TRY(prepare_batch_phases(a, qs, eval_strikes, max_rows, stage, launch), "batch launch");
                grid = launch[1].grid;
            } else {
                FO_CUDA_TRY(prepare_batch_persistent(a, q, eval_strikes, max_rows, stage, tune.ctas_per_sm, &launch[0]),
                            "batch launch");
                grid = launch[0].grid;
            }
            // The wave's stream work, in order: table upload, status / state resets, the persistent
            // launch between two timing marks, the read-back (results, then the timeout flag into
            // the pinned tail of the read-back region).
            unsigned* timed_out = reinterpret_cast<unsigned*>(back + L.out_bytes);
            auto enqueue = [&]() -> cudaError_t {
                cudaError_t ce = cudaMemcpyAsync(dev + L.groups, host + (L.groups - in_bytes), table_bytes,
                                                 cudaMemcpyHostToDevice, s);
                if (ce == cudaSuccess) ce = cudaMemsetAsync(dev + L.out_begin, 0xff, L.summaries - L.out_begin, s);
                if (ce == cudaSuccess) ce = cudaMemsetAsync(dev + L.clear_begin, 0, L.clear_bytes, s);
                // External record nodes: the marks are recorded when the graph runs (a plain record
                // during capture would only order the captured work).
                if (ce == cudaSuccess) ce = cudaEventRecordWithFlags(mark[0], s, cudaEventRecordExternal);
                for (int k = 0; k < n_launches && ce == cudaSuccess; ++k) {
                    ce = enqueue_batch_persistent(launch[k], a, tune.phases ? qs[k < 3 ? k : 2] : q, max_rows, stage, s);
                    if (ce == cudaSuccess) ce = cudaEventRecordWithFlags(mark[k + 1], s, cudaEventRecordExternal);
                }
                if (ce == cudaSuccess) ce = cudaMemcpyAsync(back, dev + L.out_begin, L.out_bytes, cudaMemcpyDeviceToHost, s);
                if (ce == cudaSuccess)
                    ce = cudaMemcpyAsync(timed_out, q.timeout, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
                return ce;
            };
            // Launch key: everything the captured work depends on.
            std::vector<unsigned char> key;
            auto put = [&](const void* p, size_t n) {
                const auto* c = static_cast<const unsigned char*>(p);
                key.insert(key.end(), c, c + n);
            };
            const void* bases[2] = {dev, host};
            const size_t sizes[8] = {L.groups, L.out_begin, L.out_bytes, L.summaries, L.clear_begin, L.clear_bytes,
                                     table_bytes, in_bytes};
            put(bases, sizeof bases);
            put(sizes, sizeof sizes);
            put(&a, sizeof a);
            put(&q, sizeof q);
            put(qs, sizeof qs);
            put(launch, sizeof launch);
            put(&n_launches, sizeof n_launches);
            const uint32_t extra[2] = {max_rows, stage ? 1u : 0u};
            put(extra, sizeof extra);
            if (!ex->batch_graph || key != ex->batch_graph_key) {
                if (ex->batch_graph) {
                    cudaGraphExecDestroy(ex->batch_graph);
                    ex->batch_graph = nullptr;
                }
                cudaGraph_t graph = nullptr;
                FO_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "batch capture");
                const cudaError_t ce = enqueue();
                const cudaError_t ee = cudaStreamEndCapture(s, &graph);
                FO_CUDA_TRY(ce, "batch capture");
                FO_CUDA_TRY(ee, "batch capture");
                const cudaError_t ie = cudaGraphInstantiate(&ex->batch_graph, graph, 0);
                cudaGraphDestroy(graph);
                FO_CUDA_TRY(ie, "batch graph instantiation");
                ex->batch_graph_key = std::move(key);
                ex->batch_graph_captures += 1;
            } else {
                ex->batch_graph_replays += 1;
            }
            FO_CUDA_TRY(cudaGraphLaunch(ex->batch_graph, s), "batch graph launch");
            ex->batch_h2d += table_bytes;
            ex->batch_launches += 1;
            ex->batch_grid = grid;
            ex->batch_strikes = eval_strikes;
            ex->batch_items = n_items;
            ex->batch_d2h += L.out_bytes + sizeof(unsigned);
            FO_CUDA_TRY(cudaStreamSynchronize(s), "batch pricing");
            FO_CUDA_TRY(cudaEventElapsedTime(launch_ms, mark[0], mark[n_launches]), "event");
            for (int k = 0; k < 3; ++k) phase_ms[k] = 0.f;
            if (tune.phases)  // the summary kernel is counted with the evaluation
                for (int k = 0; k < 3; ++k)
                    FO_CUDA_TRY(cudaEventElapsedTime(&phase_ms[k], mark[k], mark[k == 2 ? 4 : k + 1]), "event");
            if (*timed_out)
                return make_error(FO_ERR_EXECUTION, FO_CODE_BARRIER_TIMEOUT,
                                  "a batch work item waited too long for the items it depends on; the device result was "
                                  "discarded");
            return Error{};
        };
        BatchTuning tune = ex->batch_tuning;
        ex->batch_tuning_source = 0;
        if (ex->batch_autotune) {
            const std::string key = tuning_key(work, w, greeks, m.degree, max_rows, max_strikes);
            const auto found = ex->batch_tuned.find(key);
            if (found != ex->batch_tuned.end()) {
                tune = found->second;
                ex->batch_tuning_source = 1;
            } else {
                Error te = autotune_wave(run_wave, greeks, int(max_strikes), &tune, &ex->batch_tuning_runs);
                if (!te.ok()) return te;
                ex->batch_tuned.emplace(key, tune);
                ex->batch_tuning_source = 2;
            }
        }
        ex->batch_tuning_used = tune;
        {
            float ms = 0.f;
            Error re = run_wave(tune, &ms);
            if (!re.ok()) return re;
            ex->batch_ms[0] += ms;
            for (int k = 0; k < 3; ++k) ex->batch_ms[1 + k] += phase_ms[k];
        }
        const auto* gst = reinterpret_cast<const GroupStatus*>(back + (L.group_status - L.out_begin));
        const auto* pst = reinterpret_cast<const ProblemStatus*>(back + (L.problem_status - L.out_begin));
        const auto* sum = reinterpret_cast<const ProblemSummary*>(back + (L.summaries - L.out_begin));
        const auto* greek_sums = reinterpret_cast<const double*>(back + (L.greek_sums - L.out_begin));
        std::vector<unsigned> stops;
        if (greeks) {
            stops.resize(w.records);
            FO_CUDA_TRY(cudaMemcpy(stops.data(), dev + L.stop_counts, sizeof(unsigned) * w.records, cudaMemcpyDeviceToHost),
                        "stopping counts copy");
            ex->batch_d2h += sizeof(unsigned) * w.records;
        }
        BatchRun run{ex, &work, &plans, &slab_of, dev, L, w};
        // Failure scan in group order (the lowest failing group wins).
        uint64_t i0 = 0;
        uint64_t first_record = 0;
        for (uint64_t g = w.g0; g < w.g1; ++g) {
            const GroupWork& gw = work[g];
            const uint64_t strikes_g = gw.end_row - gw.first_row;
            const GroupStatus& gs = gst[g - w.g0];
            bool failed = gs.train_sim_fail != kNone || !gw.fit.ok() || gs.eval_sim_fail != kNone;
            for (uint64_t k = 0; k < strikes_g && !failed; ++k) {
                const ProblemSummary& ps = sum[i0 + k];
                const ProblemStatus& st = pst[i0 + k];
                failed = ps.fit_fail_order != 0xffffffffu ||
                         (!ps.origin_exercised && (ps.nosupport_row != 0xffffffffu || st.eval_fail != kNone ||
                                                   st.eval_terminal_fail != kNone || !std::isfinite(ps.price) ||
                                                   !std::isfinite(ps.sample_standard_deviation)));
            }
            if (failed) {
                if (gs.train_sim_fail != kNone) return simulation_failure(run, g, true, gs.train_sim_fail);
                if (!gw.fit.ok()) return estimator_at_row(gw.first_row, gw.fit);
                uint64_t rec = first_record;
                for (uint64_t k = 0; k < strikes_g; ++k) {
                    const ProblemSummary& ps = sum[i0 + k];
                    BatchProblem pr{};
                    pr.strike = strikes[gw.first_row + k];
                    pr.records = uint32_t(rec);
                    rec += gw.hp.rows();
                    if (ps.fit_fail_order != 0xffffffffu) return fit_error(run, g, gw.first_row + k, pr, pst[i0 + k], ps);
                }
                if (gs.eval_sim_fail != kNone) return simulation_failure(run, g, false, gs.eval_sim_fail);
                rec = first_record;
                for (uint64_t k = 0; k < strikes_g; ++k) {
                    BatchProblem pr{};
                    pr.strike = strikes[gw.first_row + k];
                    pr.records = uint32_t(rec);
                    rec += gw.hp.rows();
                    Error ee = evaluation_error(run, g, gw.first_row + k, pr, pst[i0 + k], sum[i0 + k]);
                    if (!ee.ok()) return ee;
                }
                return make_error(FO_ERR_LSM, FO_CODE_INVALID_ARGUMENT,
                                  "parallel LSM batch reported row " + u(gw.first_row) +
                                      " as failed, but deterministic serial replay succeeded");
            }
            for (uint64_t k = 0; k < strikes_g; ++k) {
                const ProblemSummary& ps = sum[i0 + k];
                const uint64_t r = gw.first_row + k;
                out->prices[r] = ps.price;
                out->sample_standard_deviations[r] = ps.sample_standard_deviation;
                out->standard_errors[r] = ps.standard_error;
                out->origin_decisions_fitted[r] = uint8_t(ps.origin_fitted);
                out->origin_exercised[r] = uint8_t(ps.origin_exercised);
                out->regression_nodes[r] = ps.regression_nodes;
                out->no_training_support_nodes[r] = ps.no_support_nodes;
                out->insufficient_exercise_support_nodes[r] = ps.insufficient_nodes;
                out->minimum_in_the_money_training_paths[r] = ps.minimum_itm;
                out->maximum_regression_condition_numbers[r] = ps.maximum_condition;
                out->early_exercise_paths[r] = ps.early_paths;
                out->expiry_paths[r] = ps.expiry_paths;
                if (greeks)
                    write_greeks(*sink, r, gw, strikes[r], ps, greek_sums + (i0 + k) * kGreekSlots,
                                 stops.data() + first_record + k * gw.hp.rows());
            }
            i0 += strikes_g;
            first_record += strikes_g * gw.hp.rows();
        }
    }
    if (launchable < groups) return work[launchable].build;
    return Error{};
}

Error price_batch(fo_executor* ex, const BatchView& v, fo_batch_result_columns* out) {
    Error e = validate_request(v, out);
    if (!e.ok()) return e;
    std::vector<GroupSpec> specs(v.groups());
    for (uint64_t g = 0; g < specs.size(); ++g) specs[g] = spec_of(v, g);
    return price_groups(ex, method_of(*v.q), specs, v.q->strikes, out);
}

// ---- ragged batches (per-contract path counts; no reference counterpart) -----------------------

Error validate_ragged(const fo_lsm_ragged_request& q, const fo_batch_result_columns* out) {
    // The regression method first, as parse_batch_lsm_method does for the batch routes.
    fo_lsm_grouped_request m{};
    m.polynomial_degree = q.polynomial_degree;
    m.rank_tolerance = q.rank_tolerance;
    m.condition_limit = q.condition_limit;
    m.tie_rule = q.tie_rule;
    m.insufficient_exercise_support = q.insufficient_exercise_support;
    m.exercise_mesh = FO_MESH_CASH_DIVIDEND_DATES;  // no mesh fields to check here
    m.training_paths = 1;
    m.evaluation_paths = 2;
    Error e = validate_method(m);
    if (!e.ok()) return e;
    const uint64_t rows = q.rows;
    if (rows == 0) return input_error(FO_CODE_EMPTY_BATCH, "LSM call batch must contain at least one contract");
    if (!q.initial_spots || !q.strikes || !q.maturities || !q.rates || !q.volatilities || !q.exercise_offsets ||
        (!q.exercise_times && q.n_exercise_times) || !q.training_paths || !q.evaluation_paths)
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                          "ragged batch columns (spots, strikes, maturities, rates, volatilities, exercise offsets, "
                          "path counts) must not be NULL");
    if (q.origin_exercise != FO_ORIGIN_INCLUDED && q.origin_exercise != FO_ORIGIN_EXCLUDED)
        return input_error(FO_CODE_UNSUPPORTED_ENUM, "unsupported origin exercise convention " + std::to_string(q.origin_exercise));
    e = validate_ragged_exercise(q.exercise_offsets, q.n_exercise_offsets, q.exercise_times, q.n_exercise_times);
    if (!e.ok()) return e;
    if (q.n_exercise_offsets != rows + 1) return row_count("exercise_times", rows, q.n_exercise_offsets - 1);
    const bool cash = q.dividend_offsets != nullptr;
    if (cash) {
        if (q.dividend_policy != FO_DIVIDEND_LIQUIDATOR && q.dividend_policy != FO_DIVIDEND_SURVIVOR)
            return input_error(FO_CODE_UNSUPPORTED_ENUM, "unsupported dividend policy " + std::to_string(q.dividend_policy));
        if (q.maturity_boundary != FO_MATURITY_STRICTLY_BEFORE && q.maturity_boundary != FO_MATURITY_AT_OR_BEFORE)
            return input_error(FO_CODE_UNSUPPORTED_CASH_MATURITY_BOUNDARY,
                               "cash-dividend maturity boundary is unsupported by this LSM engine");
        e = validate_ragged_cash(q.dividend_offsets, q.n_dividend_offsets, q.dividend_times, q.n_dividend_events,
                                 q.dividend_amounts, q.n_dividend_events);
        if (!e.ok()) {
            e.kind = FO_ERR_INPUT;
            return e;
        }
        if (q.n_dividend_offsets != rows + 1) return row_count("dividend_model", rows, q.n_dividend_offsets - 1);
    }
    auto path_count = [](const char* population, uint64_t row, uint64_t n, uint64_t minimum) -> Error {
        if (n < minimum || n > kU32Max)
            return input_error(FO_CODE_BATCH_PATH_COUNT_OUTSIDE_DOMAIN,
                               std::string("batched LSM ") + population + " path count " + u(n) + " at row " + u(row) +
                                   " is outside [" + u(minimum) + ", 4294967295]");
        return Error{};
    };
    const int64_t ex_base = q.exercise_offsets[0];
    const int64_t cash_base = cash ? q.dividend_offsets[0] : 0;
    for (uint64_t r = 0; r < rows; ++r) {
        e = nonnegative_value("initial_spots", r, q.initial_spots[r]);
        if (e.ok()) e = positive_value("strikes", r, q.strikes[r]);
        if (e.ok()) e = positive_value("maturities", r, q.maturities[r]);
        if (e.ok()) e = finite_value("constant_continuously_compounded_rates", r, q.rates[r]);
        if (e.ok()) e = positive_value("constant_volatilities", r, q.volatilities[r]);
        if (e.ok() && q.dividend_yields) e = nonnegative_value("continuous_dividend_yields", r, q.dividend_yields[r]);
        if (e.ok() && cash) {
            const int64_t b = q.dividend_offsets[r] - cash_base, en = q.dividend_offsets[r + 1] - cash_base;
            e = validate_cash_schedule(r, q.maturities[r], q.dividend_times + b, uint64_t(en - b), q.maturity_boundary);
        }
        if (e.ok()) {
            const int64_t b = q.exercise_offsets[r] - ex_base, en = q.exercise_offsets[r + 1] - ex_base;
            e = explicit_times_row(r, q.maturities[r], q.exercise_times + b, uint64_t(en - b));
        }
        if (e.ok()) e = path_count("training", r, q.training_paths[r], 1);
        if (e.ok()) e = path_count("evaluation", r, q.evaluation_paths[r], 2);
        if (!e.ok()) return e;
    }
    fo_lsm_grouped_request streams{};
    streams.training_domain_start = q.training_domain_start;
    streams.evaluation_domain_start = q.evaluation_domain_start;
    e = validate_streams(streams, rows);
    if (!e.ok()) return e;
    if (out && out->rows != rows)
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                          "result columns hold " + u(out->rows) + " rows; the batch has " + u(rows));
    return Error{};
}

Error price_ragged(fo_executor* ex, const fo_lsm_ragged_request& q, fo_batch_result_columns* out,
                   fo_ragged_greeks_columns* greeks) {
    Error e = validate_ragged(q, out);
    if (!e.ok()) return e;
    GreeksSink sink;
    if (greeks) {
        if (!greeks->delta || !greeks->vega || !greeks->log_discount_sensitivities || !greeks->log_discount_offsets ||
            (q.n_dividend_events && !greeks->dividend_sensitivities))
            return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "every requested Greeks column must be provided");
        sink.cols = greeks;
        sink.cash_first.assign(q.rows, 0);
        for (uint64_t r = 0; r < q.rows && q.dividend_offsets; ++r) {
            sink.cash_first[r] = uint64_t(q.dividend_offsets[r] - q.dividend_offsets[0]);
            const uint64_t events = uint64_t(q.dividend_offsets[r + 1] - q.dividend_offsets[r]);
            if (events > uint64_t(kMaxGreekDividends))
                return make_error(FO_ERR_EXECUTION, FO_CODE_CAPACITY_EXCEEDED,
                                  "adjoint Greeks support at most " + std::to_string(kMaxGreekDividends) +
                                      " cash dividends per contract; row " + u(r) + " has " + u(events));
        }
    }
    BatchMethod m;
    m.mesh = FO_MESH_EXPLICIT_TIMES;
    m.origin = q.origin_exercise;
    m.cash = q.dividend_offsets != nullptr;
    m.policy = m.cash ? q.dividend_policy : int32_t(FO_DIVIDEND_LIQUIDATOR);
    m.train_seed = q.training_seed;
    m.eval_seed = q.evaluation_seed;
    m.degree = int32_t(q.polynomial_degree);
    m.rank_tolerance = q.rank_tolerance;
    m.condition_limit = q.condition_limit;
    m.tie_rule = q.tie_rule;
    m.support = q.insufficient_exercise_support;
    std::vector<GroupSpec> specs(q.rows);
    const int64_t ex_base = q.exercise_offsets[0];
    const int64_t cash_base = m.cash ? q.dividend_offsets[0] : 0;
    for (uint64_t r = 0; r < q.rows; ++r) {
        GroupSpec& s = specs[r];
        s.first_row = r;
        s.end_row = r + 1;
        s.s0 = q.initial_spots[r];
        s.maturity = q.maturities[r];
        s.rate = q.rates[r];
        s.vol = q.volatilities[r];
        s.yield = q.dividend_yields ? q.dividend_yields[r] : 0.0;
        if (m.cash) {
            const int64_t b = q.dividend_offsets[r] - cash_base, en = q.dividend_offsets[r + 1] - cash_base;
            s.cash_times = q.dividend_times + b;
            s.cash_amounts = q.dividend_amounts + b;
            s.n_cash = uint64_t(en - b);
        }
        const int64_t b = q.exercise_offsets[r] - ex_base, en = q.exercise_offsets[r + 1] - ex_base;
        s.ex_times = q.exercise_times + b;
        s.n_ex = uint64_t(en - b);
        s.train_paths = q.training_paths[r];
        s.eval_paths = q.evaluation_paths[r];
        s.train_domain = uint32_t(uint64_t(q.training_domain_start) + r);
        s.eval_domain = uint32_t(uint64_t(q.evaluation_domain_start) + r);
    }
    return price_groups(ex, m, specs, q.strikes, out, greeks ? &sink : nullptr);
}

int finish(fo_error* err, const Error& e) {
    if (!e.ok()) write_error(err, e);
    return e.kind;
}

Error check_columns(const fo_batch_result_columns* out) {
    if (!out || !out->prices || !out->sample_standard_deviations || !out->standard_errors || !out->origin_decisions_fitted ||
        !out->origin_exercised || !out->regression_nodes || !out->no_training_support_nodes ||
        !out->insufficient_exercise_support_nodes || !out->minimum_in_the_money_training_paths ||
        !out->maximum_regression_condition_numbers || !out->early_exercise_paths || !out->expiry_paths)
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "every batch result column must be provided");
    return Error{};
}

int entry(fo_executor* ex, const fo_lsm_grouped_request* request, fo_batch_result_columns* out, fo_error* err,
          bool grouped) {
    if (!ex || !request)
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "executor and request must not be NULL"));
    Error e = check_columns(out);
    if (!e.ok()) return finish(err, e);
    if (grouped && !request->group_offsets && request->n_group_offsets)
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "group offsets must not be NULL"));
    if (!grouped && request->group_offsets)
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                                      "a row-addressed batch takes no group offsets"));
    std::lock_guard<std::mutex> lock(ex->mu);
    cudaError_t ce = cudaSetDevice(ex->device);
    if (ce != cudaSuccess) return finish(err, cuda_error(ce, "cudaSetDevice"));
    BatchView v{request, grouped};
    try {
        return finish(err, price_batch(ex, v, out));
    } catch (const std::bad_alloc&) {
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_CAPACITY_EXCEEDED, "host memory exhausted"));
    }
}

}  // namespace

extern "C" {

int fo_price_lsm_grouped_f64(fo_executor* executor, const fo_lsm_grouped_request* request, fo_batch_result_columns* out,
                             fo_error* err) {
    return entry(executor, request, out, err, true);
}

int fo_price_lsm_batch_f64(fo_executor* executor, const fo_lsm_grouped_request* request, fo_batch_result_columns* out,
                           fo_error* err) {
    return entry(executor, request, out, err, false);
}

int fo_price_lsm_ragged_f64(fo_executor* executor, const fo_lsm_ragged_request* request, fo_batch_result_columns* out,
                            fo_ragged_greeks_columns* greeks, fo_error* err) {
    if (!executor || !request)
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "executor and request must not be NULL"));
    Error e = check_columns(out);
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(executor->mu);
    cudaError_t ce = cudaSetDevice(executor->device);
    if (ce != cudaSuccess) return finish(err, cuda_error(ce, "cudaSetDevice"));
    try {
        return finish(err, price_ragged(executor, *request, out, greeks));
    } catch (const std::bad_alloc&) {
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_CAPACITY_EXCEEDED, "host memory exhausted"));
    }
}

int fo_validate_lsm_grouped_f64(const fo_lsm_grouped_request* request, int32_t grouped, fo_error* err) {
    if (!request)
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "request must not be NULL"));
    if (grouped && !request->group_offsets && request->n_group_offsets)
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "group offsets must not be NULL"));
    if (!grouped && request->group_offsets)
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                                      "a row-addressed batch takes no group offsets"));
    try {
        return finish(err, validate_request(BatchView{request, grouped != 0}, nullptr));
    } catch (const std::bad_alloc&) {
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_CAPACITY_EXCEEDED, "host memory exhausted"));
    }
}

int fo_validate_lsm_ragged_f64(const fo_lsm_ragged_request* request, fo_error* err) {
    if (!request)
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "request must not be NULL"));
    try {
        return finish(err, validate_ragged(*request, nullptr));
    } catch (const std::bad_alloc&) {
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_CAPACITY_EXCEEDED, "host memory exhausted"));
    }
}

int fo_executor_set_batch_tuning(fo_executor* executor, int32_t autotune, const fo_batch_tuning* fixed, fo_error* err) {
    if (!executor)
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "executor must not be NULL"));
    std::lock_guard<std::mutex> lock(executor->mu);
    if (autotune) {
        executor->batch_autotune = true;
        return FO_OK;
    }
    if (!fixed)
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                                      "a fixed batch launch shape must be given when the autotuner is off"));
    const bool valid = fixed->sim_blocks >= 1 && fixed->sim_blocks <= 64 && fixed->eval_blocks >= 1 &&
                       fixed->eval_blocks <= 64 && (fixed->strikes == 1 || fixed->strikes == 2 ||
                                                    fixed->strikes == 4 || fixed->strikes == 8) &&
                       fixed->ctas_per_sm >= 0 && fixed->ctas_per_sm <= 8 && (fixed->phases == 0 || fixed->phases == 1);
    if (!valid)
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                                      "batch launch shape outside its range: blocks per item 1..64, strikes per "
                                      "evaluation item 1, 2, 4 or 8, CTAs per SM 0..8, phases 0 or 1"));
    executor->batch_autotune = false;
    executor->batch_tuning.sim_blocks = fixed->sim_blocks;
    executor->batch_tuning.eval_blocks = fixed->eval_blocks;
    executor->batch_tuning.strikes = fixed->strikes;
    executor->batch_tuning.ctas_per_sm = fixed->ctas_per_sm;
    executor->batch_tuning.phases = fixed->phases;
    return FO_OK;
}

int fo_executor_batch_launch(fo_executor* executor, fo_batch_launch_info* out) {
    if (!executor || !out) return FO_ERR_EXECUTION;
    std::lock_guard<std::mutex> lock(executor->mu);
    const BatchTuning& t = executor->batch_tuning_used;
    out->tuning.sim_blocks = t.sim_blocks;
    out->tuning.eval_blocks = t.eval_blocks;
    out->tuning.strikes = executor->batch_strikes;
    out->tuning.ctas_per_sm = t.ctas_per_sm;
    out->tuning.phases = t.phases;
    out->source = executor->batch_tuning_source;
    out->grid = executor->batch_grid;
    out->items = executor->batch_items;
    out->tuning_launches = executor->batch_tuning_source == 2 ? executor->batch_tuning_runs : 0;
    out->graph_replays = executor->batch_graph_replays;
    out->graph_captures = executor->batch_graph_captures;
    return FO_OK;
}

int fo_executor_batch_kernel_ms(fo_executor* executor, double* kernel_ms, uint64_t capacity, uint64_t* launches) {
    if (!executor) return FO_ERR_EXECUTION;
    std::lock_guard<std::mutex> lock(executor->mu);
    for (uint64_t k = 0; kernel_ms && k < capacity && k < FO_BATCH_KERNELS; ++k) kernel_ms[k] = executor->batch_ms[k];
    if (launches) *launches = executor->batch_launches;
    return FO_OK;
}

int fo_executor_batch_transfer_bytes(fo_executor* executor, uint64_t* h2d_bytes, uint64_t* d2h_bytes) {
    if (!executor) return FO_ERR_EXECUTION;
    std::lock_guard<std::mutex> lock(executor->mu);
    if (h2d_bytes) *h2d_bytes = executor->batch_h2d;
    if (d2h_bytes) *d2h_bytes = executor->batch_d2h;
    return FO_OK;
}

}  // extern "C"

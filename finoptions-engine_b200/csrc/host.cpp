// host.cpp - request validation, typed error messages and single-contract plan construction.
//
// Validation restates the reference's constructors in the order the reference applies them, so a
// malformed request fails with the same typed error and message:
//   TimeGrid::try_new                        crates/finoptions-core/src/time.rs:40-74
//   LogDiscountCurve::try_new                crates/finoptions-core/src/curve.rs:24-61
//   CumulativeDividendYieldCurve::try_new    crates/finoptions-core/src/yield_curve.rs:28-81
//   CashDividend::try_new                    crates/finoptions-core/src/dividend.rs:30-40
//   EventSchedule::try_new                   crates/finoptions-core/src/event.rs:42-105
//   parse_event_schedule / parse_gbm_model   crates/finoptions-python/src/lib.rs:671-829
//   GbmPathPlan::try_new / GbmStep::try_new  crates/finoptions-sim/src/{path.rs:55-99,step.rs:27-57}
//   PolynomialDegree / RegressionSpec        crates/finoptions-lsm/src/regression.rs:24-89
//   LsmCallEstimator::try_new / price_seeded crates/finoptions-lsm/src/policy.rs:135-336
#include "host.h"

#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace fo {

Error make_error(int32_t kind, int32_t code, std::string message) {
    Error e;
    e.kind = kind;
    e.code = code;
    e.message = std::move(message);
    return e;
}

void write_error(fo_error* out, const Error& e) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->kind = e.kind;
    out->code = e.code;
    out->row = e.row;
    out->group = e.group;
    out->node = e.node;
    out->path = e.path;
    std::snprintf(out->message, sizeof(out->message), "%s", e.message.c_str());
}

Error wrap(const Error& e, int32_t kind, const std::string& prefix) {
    Error w = e;
    w.kind = kind;
    w.message = prefix + ": " + e.message;
    return w;
}

std::string fmt_f64(double x) {
    if (std::isnan(x)) return "NaN";
    if (std::isinf(x)) return x > 0 ? "inf" : "-inf";
    if (x == 0.0) return std::signbit(x) ? "-0.0" : "0.0";
    char buf[64];
    auto res = std::to_chars(buf, buf + sizeof(buf), x, std::chars_format::scientific);
    std::string sci(buf, res.ptr);
    // sci: [-]d[.ddd]e[+-]XX
    const bool negative = sci[0] == '-';
    if (negative) sci.erase(0, 1);
    const size_t epos = sci.find('e');
    std::string mant = sci.substr(0, epos);
    const int exp10 = std::stoi(sci.substr(epos + 1));
    std::string digits;
    for (char c : mant)
        if (c != '.') digits.push_back(c);
    const double a = std::fabs(x);
    std::string out;
    if (a >= 1e-4 && a < 1e16) {
        const int point = exp10 + 1;  // digits before the decimal point
        if (point <= 0) {
            out = "0." + std::string(size_t(-point), '0') + digits;
        } else if (size_t(point) >= digits.size()) {
            out = digits + std::string(size_t(point) - digits.size(), '0') + ".0";
        } else {
            out = digits.substr(0, size_t(point)) + "." + digits.substr(size_t(point));
        }
    } else {
        out = digits.substr(0, 1);
        if (digits.size() > 1) out += "." + digits.substr(1);
        out += "e" + std::to_string(exp10);
    }
    return negative ? "-" + out : out;
}

static std::string u(uint64_t v) { return std::to_string(v); }

static bool canonical_nonnegative(double v) { return std::isfinite(v) && !(v < 0.0) && !(v == 0.0 && std::signbit(v)); }

// ---- core types --------------------------------------------------------------------------------

Error validate_time_grid(const std::vector<double>& times) {
    if (times.empty()) return make_error(FO_ERR_INPUT, FO_CODE_EMPTY_TIME_GRID, "time grid must contain at least the valuation node");
    const double origin = times[0];
    if (!std::isfinite(origin))
        return make_error(FO_ERR_INPUT, FO_CODE_NON_FINITE_TIME, "time at node 0 must be finite; observed " + fmt_f64(origin));
    if (!(origin == 0.0 && !std::signbit(origin)))
        return make_error(FO_ERR_INPUT, FO_CODE_INVALID_TIME_ORIGIN,
                          "time grid must begin at exactly 0.0; observed " + fmt_f64(origin));
    if (times.size() - 1 > 0xffffffffull)
        return make_error(FO_ERR_INPUT, FO_CODE_TOO_MANY_NODES,
                          "time grid contains " + u(times.size()) + " nodes, exceeding the supported node-ID domain");
    for (size_t i = 1; i < times.size(); ++i) {
        if (!std::isfinite(times[i]))
            return make_error(FO_ERR_INPUT, FO_CODE_NON_FINITE_TIME,
                              "time at node " + u(i) + " must be finite; observed " + fmt_f64(times[i]));
        if (times[i] <= times[i - 1])
            return make_error(FO_ERR_INPUT, FO_CODE_NON_INCREASING_TIME,
                              "time grid must be strictly increasing; node " + u(i - 1) + " is " + fmt_f64(times[i - 1]) +
                                  " and node " + u(i) + " is " + fmt_f64(times[i]));
    }
    return Error{};
}

Error validate_log_discount_curve(const std::vector<double>& times, const std::vector<double>& values) {
    Error e = validate_time_grid(times);
    if (!e.ok()) return e;
    if (values.size() != times.size())
        return make_error(FO_ERR_INPUT, FO_CODE_CURVE_LENGTH_MISMATCH,
                          "log-discount curve has " + u(values.size()) + " nodes; time grid requires " + u(times.size()));
    if (!(values[0] == 0.0 && !std::signbit(values[0])) || !std::isfinite(values[0]))
        return make_error(FO_ERR_INPUT, FO_CODE_INVALID_DISCOUNT_ORIGIN,
                          "log discount at node 0 must be exactly 0.0; observed " + fmt_f64(values[0]));
    for (size_t i = 0; i < values.size(); ++i) {
        if (!std::isfinite(values[i]))
            return make_error(FO_ERR_INPUT, FO_CODE_NON_FINITE_LOG_DISCOUNT,
                              "log discount at node " + u(i) + " must be finite; observed " + fmt_f64(values[i]));
        if (i == 0) continue;
        const double interval = values[i] - values[i - 1];
        const double discount = std::exp(interval);
        if (!std::isfinite(discount) || discount <= 0.0)
            return make_error(FO_ERR_INPUT, FO_CODE_UNREPRESENTABLE_INTERVAL_DISCOUNT,
                              "discount factor from node " + u(i - 1) + " to " + u(i) +
                                  " is not finite and positive; interval log discount is " + fmt_f64(interval));
    }
    return Error{};
}

Error validate_cumulative_yield_curve(const std::vector<double>& times, const std::vector<double>& values) {
    Error e = validate_time_grid(times);
    if (!e.ok()) return e;
    if (values.size() != times.size())
        return make_error(FO_ERR_INPUT, FO_CODE_DIVIDEND_YIELD_CURVE_LENGTH_MISMATCH,
                          "cumulative dividend-yield curve has " + u(values.size()) + " nodes; time grid requires " +
                              u(times.size()));
    if (!(values[0] == 0.0 && !std::signbit(values[0])) || !std::isfinite(values[0]))
        return make_error(FO_ERR_INPUT, FO_CODE_INVALID_CUMULATIVE_DIVIDEND_YIELD_ORIGIN,
                          "cumulative dividend yield at node 0 must be exactly 0.0; observed " + fmt_f64(values[0]));
    for (size_t i = 0; i < values.size(); ++i) {
        if (!canonical_nonnegative(values[i]))
            return make_error(FO_ERR_INPUT, FO_CODE_INVALID_CUMULATIVE_DIVIDEND_YIELD,
                              "cumulative dividend yield at node " + u(i) +
                                  " must be finite and canonically nonnegative; observed " + fmt_f64(values[i]));
        if (i == 0) continue;
        if (values[i] < values[i - 1])
            return make_error(FO_ERR_INPUT, FO_CODE_DECREASING_CUMULATIVE_DIVIDEND_YIELD,
                              "cumulative dividend yield must be nondecreasing; node " + u(i - 1) + " is " +
                                  fmt_f64(values[i - 1]) + " and node " + u(i) + " is " + fmt_f64(values[i]));
        const double interval = values[i] - values[i - 1];
        const double factor = std::exp(-interval);
        if (!std::isfinite(factor) || factor <= 0.0)
            return make_error(FO_ERR_INPUT, FO_CODE_UNREPRESENTABLE_INTERVAL_DIVIDEND_YIELD,
                              "continuous dividend-yield factor from node " + u(i - 1) + " to " + u(i) +
                                  " is not finite and positive; integrated interval yield is " + fmt_f64(interval));
    }
    return Error{};
}

Error validate_cash_dividend(uint32_t node, double amount) {
    if (!canonical_nonnegative(amount))
        return make_error(FO_ERR_INPUT, FO_CODE_INVALID_CASH_DIVIDEND,
                          "cash dividend at node " + u(node) + " must be finite and nonnegative; observed " + fmt_f64(amount));
    return Error{};
}

Error validate_constant_volatility(double sigma) {
    if (!std::isfinite(sigma) || sigma <= 0.0)
        return make_error(FO_ERR_INPUT, FO_CODE_INVALID_CONSTANT_VOLATILITY,
                          "constant annualized volatility must be finite and strictly positive; observed " + fmt_f64(sigma));
    return Error{};
}

static Error node_out_of_bounds(uint64_t node, size_t nodes) {
    return make_error(FO_ERR_INPUT, FO_CODE_NODE_OUT_OF_BOUNDS,
                      "node " + u(node) + " is outside a time grid containing " + u(nodes) + " nodes");
}

Error validate_event_schedule(const std::vector<double>& times, const std::vector<uint32_t>& dividend_nodes,
                              const std::vector<double>& dividend_amounts, const std::vector<uint32_t>& exercise_nodes,
                              uint32_t expiry) {
    if (dividend_nodes.size() != dividend_amounts.size())
        return make_error(FO_ERR_INPUT, FO_CODE_DIVIDEND_COLUMN_LENGTH_MISMATCH,
                          "event schedule has " + u(dividend_nodes.size()) + " dividend nodes but " +
                              u(dividend_amounts.size()) + " dividend amounts");
    Error e = validate_time_grid(times);
    if (!e.ok()) return e;
    const size_t n = times.size();
    for (size_t i = 0; i < dividend_nodes.size(); ++i) {
        if (dividend_nodes[i] >= n) return node_out_of_bounds(dividend_nodes[i], n);
        e = validate_cash_dividend(dividend_nodes[i], dividend_amounts[i]);
        if (!e.ok()) return e;
    }
    for (uint32_t node : exercise_nodes)
        if (node >= n) return node_out_of_bounds(node, n);
    if (expiry >= n) return node_out_of_bounds(expiry, n);
    const uint32_t expected = uint32_t(n - 1);
    if (expected == 0 || expiry != expected)
        return make_error(FO_ERR_INPUT, FO_CODE_INVALID_EXPIRY_NODE,
                          "expiry must be the final non-origin node " + u(expected) + "; observed node " + u(expiry));
    for (size_t i = 0; i < dividend_nodes.size(); ++i) {
        const uint32_t node = dividend_nodes[i];
        if (node == 0 || node > expiry)
            return make_error(FO_ERR_INPUT, FO_CODE_INVALID_DIVIDEND_NODE,
                              "cash dividend at node " + u(node) +
                                  " must occur strictly after valuation and no later than expiry node " + u(expiry));
        if (i > 0) {
            const uint32_t previous = dividend_nodes[i - 1];
            if (previous == node)
                return make_error(FO_ERR_INPUT, FO_CODE_DUPLICATE_DIVIDEND_NODE, "cash-dividend schedule repeats node " + u(node));
            if (previous > node)
                return make_error(FO_ERR_INPUT, FO_CODE_UNORDERED_DIVIDEND_NODE,
                                  "cash-dividend nodes must be strictly increasing; observed node " + u(node) + " after " +
                                      u(previous));
        }
    }
    for (size_t i = 0; i < exercise_nodes.size(); ++i) {
        const uint32_t node = exercise_nodes[i];
        if (node >= expiry)
            return make_error(FO_ERR_INPUT, FO_CODE_INVALID_EXERCISE_NODE,
                              "exercise opportunity at node " + u(node) + " must occur before expiry node " + u(expiry));
        if (i > 0) {
            const uint32_t previous = exercise_nodes[i - 1];
            if (previous == node)
                return make_error(FO_ERR_INPUT, FO_CODE_DUPLICATE_EXERCISE_NODE, "exercise schedule repeats node " + u(node));
            if (previous > node)
                return make_error(FO_ERR_INPUT, FO_CODE_UNORDERED_EXERCISE_NODE,
                                  "exercise nodes must be strictly increasing; observed node " + u(node) + " after " +
                                      u(previous));
        }
    }
    return Error{};
}

// Ragged Arrow-style views (crates/finoptions-batch/src/{view.rs,exercise.rs}).
static Error validate_offsets(const int64_t* offsets, uint64_t n_offsets, uint64_t n_events, uint64_t* base) {
    if (n_offsets < 2)
        return make_error(FO_ERR_BATCH, FO_CODE_INSUFFICIENT_OFFSETS,
                          "ragged offsets must contain at least two values; observed " + u(n_offsets));
    for (uint64_t i = 0; i < n_offsets; ++i) {
        if (offsets[i] < 0)
            return make_error(FO_ERR_BATCH, FO_CODE_NEGATIVE_OFFSET,
                              "ragged offset " + u(i) + " must be nonnegative; observed " + std::to_string(offsets[i]));
        if (i > 0 && offsets[i - 1] > offsets[i])
            return make_error(FO_ERR_BATCH, FO_CODE_DECREASING_OFFSET,
                              "ragged offsets must be nondecreasing; offset " + u(i - 1) + " is " +
                                  std::to_string(offsets[i - 1]) + " and offset " + u(i) + " is " + std::to_string(offsets[i]));
    }
    const uint64_t first = uint64_t(offsets[0]), last = uint64_t(offsets[n_offsets - 1]);
    if (last - first != n_events)
        return make_error(FO_ERR_BATCH, FO_CODE_OFFSET_SPAN_MISMATCH,
                          "ragged offset span [" + u(first) + ", " + u(last) + ") contains " + u(last - first) +
                              " events but child buffers contain " + u(n_events));
    *base = first;
    return Error{};
}

Error validate_ragged_cash(const int64_t* offsets, uint64_t n_offsets, const double* times, uint64_t n_times,
                           const double* amounts, uint64_t n_amounts) {
    if (n_offsets < 2)
        return make_error(FO_ERR_BATCH, FO_CODE_INSUFFICIENT_OFFSETS,
                          "ragged offsets must contain at least two values; observed " + u(n_offsets));
    if (n_times != n_amounts)
        return make_error(FO_ERR_BATCH, FO_CODE_EVENT_COLUMN_LENGTH_MISMATCH,
                          "event-time buffer has " + u(n_times) + " values but cash-amount buffer has " + u(n_amounts));
    uint64_t base = 0;
    Error e = validate_offsets(offsets, n_offsets, n_times, &base);
    if (!e.ok()) return e;
    for (uint64_t row = 0; row + 1 < n_offsets; ++row) {
        const uint64_t b = uint64_t(offsets[row]) - base, end = uint64_t(offsets[row + 1]) - base;
        for (uint64_t k = b; k < end; ++k) {
            const uint64_t event = k - b;
            const double t = times[k], a = amounts[k];
            if (!std::isfinite(t) || t <= 0.0)
                return make_error(FO_ERR_BATCH, FO_CODE_INVALID_EVENT_TIME,
                                  "cash-dividend time at row " + u(row) + ", event " + u(event) +
                                      " must be finite and strictly positive; observed " + fmt_f64(t));
            if (event > 0 && times[k - 1] > t)
                return make_error(FO_ERR_BATCH, FO_CODE_DECREASING_EVENT_TIME,
                                  "cash-dividend times must be nondecreasing; row " + u(row) + ", event " + u(event) + " is " +
                                      fmt_f64(t) + " after " + fmt_f64(times[k - 1]));
            if (!canonical_nonnegative(a))
                return make_error(FO_ERR_BATCH, FO_CODE_INVALID_CASH_AMOUNT,
                                  "cash-dividend amount at row " + u(row) + ", event " + u(event) +
                                      " must be finite, nonnegative, and canonical; observed " + fmt_f64(a));
        }
    }
    return Error{};
}

Error validate_ragged_exercise(const int64_t* offsets, uint64_t n_offsets, const double* times, uint64_t n_times) {
    uint64_t base = 0;
    Error e = validate_offsets(offsets, n_offsets, n_times, &base);
    if (!e.ok()) return e;
    for (uint64_t row = 0; row + 1 < n_offsets; ++row) {
        const uint64_t b = uint64_t(offsets[row]) - base, end = uint64_t(offsets[row + 1]) - base;
        for (uint64_t k = b; k < end; ++k) {
            const uint64_t event = k - b;
            const double t = times[k];
            if (!std::isfinite(t) || t <= 0.0)
                return make_error(FO_ERR_BATCH, FO_CODE_INVALID_EXERCISE_TIME,
                                  "exercise time at row " + u(row) + ", event " + u(event) +
                                      " must be finite and strictly positive; observed " + fmt_f64(t));
            if (event > 0 && times[k - 1] >= t)
                return make_error(FO_ERR_BATCH, FO_CODE_NON_INCREASING_EXERCISE_TIME,
                                  "exercise times must be strictly increasing; row " + u(row) + ", event " + u(event) +
                                      " is " + fmt_f64(t) + " after " + fmt_f64(times[k - 1]));
        }
    }
    return Error{};
}

// ---- plans -------------------------------------------------------------------------------------

template <typename T>
static std::vector<T> vec(const T* p, uint64_t n) {
    return p ? std::vector<T>(p, p + n) : std::vector<T>();
}

Error build_gbm_plan(const double* schedule_times, uint64_t n_schedule, const double* curve_times, uint64_t n_curve,
                     const double* log_discounts, uint64_t n_ld, const double* yield_times, uint64_t n_yt,
                     const double* yields, uint64_t n_y, const uint32_t* dividend_nodes, uint64_t n_dn,
                     const double* dividend_amounts, uint64_t n_da, const uint32_t* exercise_nodes, uint64_t n_ex,
                     uint32_t expiry, double volatility, int32_t policy, HostPlan* plan) {
    const auto times = vec(schedule_times, n_schedule);
    const auto dn = vec(dividend_nodes, n_dn);
    const auto da = vec(dividend_amounts, n_da);
    const auto ex = vec(exercise_nodes, n_ex);
    Error e = validate_event_schedule(times, dn, da, ex, expiry);
    if (!e.ok()) return e;
    const auto ct = vec(curve_times, n_curve);
    const auto ld = vec(log_discounts, n_ld);
    e = validate_log_discount_curve(ct, ld);
    if (!e.ok()) return e;
    const auto yt = vec(yield_times, n_yt);
    const auto y = vec(yields, n_y);
    e = validate_cumulative_yield_curve(yt, y);
    if (!e.ok()) return e;
    e = validate_constant_volatility(volatility);
    if (!e.ok()) return e;
    if (policy != FO_DIVIDEND_LIQUIDATOR && policy != FO_DIVIDEND_SURVIVOR)
        return make_error(FO_ERR_INPUT, FO_CODE_UNSUPPORTED_ENUM, "unsupported dividend policy " + std::to_string(policy));
    // GbmPathPlan::try_new compares grids by value (TimeGrid: PartialEq on the f64 slice).
    auto same = [](const std::vector<double>& a, const std::vector<double>& b) {
        if (a.size() != b.size()) return false;
        for (size_t i = 0; i < a.size(); ++i)
            if (!(a[i] == b[i])) return false;
        return true;
    };
    if (!same(times, ct))
        return make_error(FO_ERR_SIMULATION, FO_CODE_TIME_GRID_MISMATCH,
                          "discount curve and event schedule must use the identical time grid");
    if (!same(times, yt))
        return make_error(FO_ERR_SIMULATION, FO_CODE_DIVIDEND_YIELD_TIME_GRID_MISMATCH,
                          "continuous dividend-yield curve and event schedule must use the identical time grid");
    const size_t n = times.size();
    plan->times = times;
    plan->log_discounts = ld;
    plan->steps.resize(n - 1);
    for (size_t to = 1; to < n; ++to) {
        // GbmStep::try_new (step.rs:44-51)
        const double dt = times[to] - times[to - 1];
        const double interval_log_discount = ld[to] - ld[to - 1];
        const double interval_yield = y[to] - y[to - 1];
        const double variance = std::fma(volatility, volatility, 0.0) * dt;
        const double log_drift = -interval_log_discount - interval_yield - 0.5 * variance;
        plan->steps[to - 1] = StepCoef{log_drift, std::sqrt(variance)};
    }
    plan->events.assign(n, NodeEvent{0.0, -1, 0});
    for (size_t i = 0; i < dn.size(); ++i) {
        plan->events[dn[i]].flags |= kEventDividend;
        plan->events[dn[i]].dividend_amount = da[i];
    }
    plan->row_node = ex;
    plan->row_node.push_back(expiry);
    for (size_t r = 0; r < plan->row_node.size(); ++r) {
        const uint32_t node = plan->row_node[r];
        if (node > 0) plan->events[node].row = int32_t(r);
    }
    plan->events[expiry].flags |= kEventTerminal;
    plan->policy = policy;
    plan->origin_row = plan->row_node[0] == 0;
    plan->escrowed = false;
    plan->escrow_cash.assign(plan->row_node.size(), 0.0);
    return Error{};
}

static Error lsm_error(int32_t code, std::string message) { return make_error(FO_ERR_LSM, code, std::move(message)); }

Error finish_discounts(HostPlan* plan) {
    const size_t rows = plan->row_node.size();
    plan->disc_from_later.assign(rows, 1.0);
    plan->disc_to_origin.assign(rows, 1.0);
    const auto& L = plan->log_discounts;
    uint32_t later = plan->row_node[rows - 1];
    // Backward over exercise rows, skipping the origin (policy.rs:242-264, 1049-1108).
    for (size_t r = rows - 1; r-- > 0;) {
        const uint32_t node = plan->row_node[r];
        if (node == 0) continue;
        const double log_discount = L[later] - L[node];
        const double d = std::exp(log_discount);
        if (!std::isfinite(d) || d <= 0.0) {
            Error e = lsm_error(FO_CODE_UNREPRESENTABLE_OBSERVATION_DISCOUNT,
                                "discount factor from observation node " + u(node) + " to " + u(later) +
                                    " is not finite and positive; log discount is " + fmt_f64(log_discount));
            return e;
        }
        plan->disc_from_later[r] = d;
        later = node;
    }
    {
        const double d = std::exp(L[later]);
        if (!std::isfinite(d) || d <= 0.0)
            return lsm_error(FO_CODE_UNREPRESENTABLE_OBSERVATION_DISCOUNT,
                             "discount factor from observation node 0 to " + u(later) +
                                 " is not finite and positive; log discount is " + fmt_f64(L[later]));
        plan->origin_discount = d;
    }
    for (size_t r = 0; r < rows; ++r) {
        const uint32_t node = plan->row_node[r];
        const double d = std::exp(L[node]);
        if (!std::isfinite(d) || d <= 0.0)
            return lsm_error(FO_CODE_UNREPRESENTABLE_OBSERVATION_DISCOUNT,
                             "discount factor from observation node 0 to " + u(node) +
                                 " is not finite and positive; log discount is " + fmt_f64(L[node]));
        plan->disc_to_origin[r] = d;
    }
    return Error{};
}

Error build_call_plan(const fo_lsm_call_request& q, HostPlan* plan) {
    Error e = build_gbm_plan(q.schedule_times, q.n_schedule_times, q.curve_times, q.n_curve_times, q.log_discounts,
                             q.n_log_discounts, q.dividend_yield_times, q.n_dividend_yield_times,
                             q.cumulative_dividend_yields, q.n_cumulative_dividend_yields, q.dividend_nodes,
                             q.n_dividend_nodes, q.dividend_amounts, q.n_dividend_amounts, q.exercise_nodes,
                             q.n_exercise_nodes, q.expiry_node, q.annualized_volatility, q.dividend_policy, plan);
    if (!e.ok()) return e;
    // PolynomialDegree / PolynomialRegressionSpec (mapped to LsmError at lib.rs:1211-1214)
    if (q.polynomial_degree > 4)
        return lsm_error(FO_CODE_UNSUPPORTED_DEGREE, "polynomial degree " + u(q.polynomial_degree) +
                                                         " is unsupported; the validated maximum degree is 4");
    if (!std::isfinite(q.rank_tolerance) || q.rank_tolerance <= 0.0 || q.rank_tolerance >= 1.0)
        return lsm_error(FO_CODE_INVALID_RANK_TOLERANCE,
                         "rank tolerance must be finite and strictly between 0 and 1; observed " + fmt_f64(q.rank_tolerance));
    const double maximum = 1.0 / q.rank_tolerance;
    if (!std::isfinite(q.condition_limit) || q.condition_limit < 1.0 || q.condition_limit > maximum)
        return lsm_error(FO_CODE_INVALID_CONDITION_LIMIT,
                         "condition limit must be finite, at least 1, and no greater than 1/rank_tolerance (" +
                             fmt_f64(maximum) + "); observed " + fmt_f64(q.condition_limit));
    if (q.tie_rule != FO_TIE_STRICTLY_GREATER && q.tie_rule != FO_TIE_GREATER_OR_EQUAL)
        return make_error(FO_ERR_INPUT, FO_CODE_UNSUPPORTED_ENUM, "unsupported exercise tie rule " + std::to_string(q.tie_rule));
    if (q.insufficient_exercise_support != FO_SUPPORT_FAIL && q.insufficient_exercise_support != FO_SUPPORT_CONTINUE)
        return make_error(FO_ERR_INPUT, FO_CODE_UNSUPPORTED_ENUM,
                          "unsupported insufficient exercise support policy " + std::to_string(q.insufficient_exercise_support));
    if (!std::isfinite(q.strike) || q.strike <= 0.0)
        return lsm_error(FO_CODE_INVALID_STRIKE, "call strike must be finite and strictly positive; observed " + fmt_f64(q.strike));
    // price_seeded (policy.rs:306-336)
    if (q.training_domain == q.evaluation_domain)
        return lsm_error(FO_CODE_RANDOM_DOMAIN_COLLISION, "LSM training and evaluation random domains must differ; both use domain " +
                                                             u(q.training_domain));
    // validate_seeded (seeded.rs:384-397) for the training then the evaluation population.
    const double s0 = q.initial_spot;
    const bool spot_ok = std::isfinite(s0) && !(s0 < 0.0) && !(s0 == 0.0 && std::signbit(s0));
    auto check_paths = [&](uint64_t paths, const char* role) -> Error {
        if (!spot_ok)
            return make_error(FO_ERR_LSM, FO_CODE_INVALID_INITIAL_SPOT,
                              std::string("LSM ") + role +
                                  " simulation failed: initial spot must be finite, nonnegative, and canonical; observed " +
                                  fmt_f64(s0));
        if (paths == 0)
            return make_error(FO_ERR_LSM, FO_CODE_EMPTY_PATH_SET,
                              std::string("LSM ") + role + " simulation failed: simulation path count must be positive");
        if (paths > 0xffffffffull)
            return make_error(FO_ERR_LSM, FO_CODE_RANDOM_PATH_NAMESPACE_OVERFLOW,
                              std::string("LSM ") + role + " simulation failed: seeded simulation supports at most 4294967295 "
                                                           "paths in one random domain; observed " + u(paths));
        return Error{};
    };
    e = check_paths(q.training_paths, "training");
    if (!e.ok()) return e;
    e = finish_discounts(plan);
    if (!e.ok()) return e;
    plan->sim_start = s0;
    plan->initial_spot = s0;
    plan->strike = q.strike;
    plan->train_paths = q.training_paths;
    plan->eval_paths = q.evaluation_paths;
    plan->train_seed = q.training_seed;
    plan->eval_seed = q.evaluation_seed;
    plan->train_domain = q.training_domain;
    plan->eval_domain = q.evaluation_domain;
    plan->degree = int32_t(q.polynomial_degree);
    plan->rank_tolerance = q.rank_tolerance;
    plan->condition_limit = q.condition_limit;
    plan->tie_rule = q.tie_rule;
    plan->support = q.insufficient_exercise_support;
    // The evaluation population's own checks are deferred until after the fit in the reference
    // (its simulation starts after fitting); they are raised in that order by the caller.
    return Error{};
}

int32_t simulation_failure_code(int code) {
    switch (code) {
        case kNormalBudget: return FO_CODE_RANDOM_NORMAL_BUDGET_EXHAUSTED;
        case kNormalRejection: return FO_CODE_RANDOM_NORMAL_REJECTION_LIMIT;
        default: return FO_CODE_NON_FINITE_PATH_TRANSITION;
    }
}

std::string simulation_failure_message(int code, uint32_t interval, uint64_t path, double spot, double normal) {
    switch (code) {
        case kNormalBudget:
            return "random-normal budget exhausted at interval " + u(interval) + ", path " + u(path) +
                   "; this indicates an internal estimator-contract violation";
        case kNormalRejection:
            return "random-normal rejection limit reached at interval " + u(interval) + ", path " + u(path) +
                   "; no variate or fallback was produced";
        default:
            return "GBM path transition from node " + u(interval) + " to " + u(uint64_t(interval) + 1) + " at path " + u(path) +
                   " produced non-finite spot from state " + fmt_f64(spot) + " and variate " + fmt_f64(normal);
    }
}

// ---- fit failures (RegressionError Display wrapped in LsmError::RegressionAtNode) ------------

std::string node_str(uint32_t node) { return std::to_string(node); }

Error fit_failure(const HostPlan& hp, const FitRecord& rec, uint32_t node) {
    const int d = hp.degree;
    const std::string prefix = "continuation regression failed at exercise node " + node_str(node) + ": ";
    if (rec.itm < uint64_t(d + 1)) {
        Error e = make_error(FO_ERR_LSM, FO_CODE_INSUFFICIENT_OBSERVATIONS,
                             prefix + "regression has " + std::to_string(rec.itm) + " observations but degree " +
                                 std::to_string(d) + " requires at least " + std::to_string(d + 1));
        e.node = node;
        return e;
    }
    Error e;
    switch (rec.model.status) {
        case kFitDegeneratePredictor:
            e = make_error(FO_ERR_LSM, FO_CODE_DEGENERATE_PREDICTOR,
                           prefix + "degree " + std::to_string(d) + " regression predictor scale is degenerate; observed " +
                               fmt_f64(rec.model.aux_value));
            break;
        case kFitRankDeficient:
            e = make_error(FO_ERR_LSM, FO_CODE_RANK_DEFICIENT,
                           prefix + "degree " + std::to_string(d) + " polynomial design has numerical rank " +
                               std::to_string(rec.model.aux) + " of " + std::to_string(d + 1) + " at rank tolerance " +
                               fmt_f64(hp.rank_tolerance));
            break;
        case kFitNonFinite:
            e = make_error(FO_ERR_LSM, FO_CODE_NON_FINITE_FIT,
                           prefix + "polynomial regression produced non-finite arithmetic at basis degree " +
                               std::to_string(rec.model.aux));
            break;
        default:
            e = make_error(FO_ERR_LSM, FO_CODE_NON_FINITE_PREDICTOR,
                           prefix + "regression population contains a non-finite predictor or response");
            break;
    }
    e.node = node;
    return e;
}

Error diag_failure(const HostPlan& hp, const FitRecord& rec, uint32_t node) {
    const int d = hp.degree;
    const std::string prefix = "continuation regression failed at exercise node " + node_str(node) + ": ";
    Error e;
    switch (rec.diag_status) {
        case kDiagRankDeficient:
            e = make_error(FO_ERR_LSM, FO_CODE_RANK_DEFICIENT,
                           prefix + "degree " + std::to_string(d) + " polynomial design has numerical rank " +
                               std::to_string(rec.diag_rank) + " of " + std::to_string(d + 1) + " at rank tolerance " +
                               fmt_f64(hp.rank_tolerance));
            break;
        case kDiagConditionExceeded:
            e = make_error(FO_ERR_LSM, FO_CODE_CONDITION_LIMIT_EXCEEDED,
                           prefix + "degree " + std::to_string(d) + " polynomial design condition number " +
                               fmt_f64(rec.diag_condition) + " exceeds configured limit " + fmt_f64(hp.condition_limit));
            break;
        case kDiagNotConverged:
            e = make_error(FO_ERR_LSM, FO_CODE_CONDITION_DIAGNOSTIC_DID_NOT_CONVERGE,
                           prefix + "polynomial condition diagnostic did not converge for " + std::to_string(d + 1) +
                               " columns after 32 sweeps");
            break;
        default:
            e = make_error(FO_ERR_LSM, FO_CODE_NON_FINITE_FIT,
                           prefix + "polynomial regression produced non-finite arithmetic at basis degree " +
                               std::to_string(rec.diag_aux));
            break;
    }
    e.node = node;
    return e;
}

}  // namespace fo

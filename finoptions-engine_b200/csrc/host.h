// host.h - host-side request validation, typed errors and plan construction.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/finoptions_cuda.h"
#include "lsm_device.cuh"

namespace fo {

// Typed failure carried through the host layer and written into fo_error at the ABI.
struct Error {
    int32_t kind = FO_OK;
    int32_t code = FO_CODE_NONE;
    int64_t row = -1, group = -1, node = -1, path = -1;
    std::string message;
    bool ok() const { return kind == FO_OK; }
};

Error make_error(int32_t kind, int32_t code, std::string message);
void write_error(fo_error* out, const Error& e);
// Wraps e's message as "<prefix>: <message>" keeping its code and indices.
Error wrap(const Error& e, int32_t kind, const std::string& prefix);

// Rust `{:?}` rendering of an f64 (shortest round-trip digits; exponent form outside [1e-4, 1e16)).
std::string fmt_f64(double x);

// ---- validated financial inputs (crates/finoptions-core) ------------------------------------

Error validate_time_grid(const std::vector<double>& times);
Error validate_log_discount_curve(const std::vector<double>& times, const std::vector<double>& values);
Error validate_cumulative_yield_curve(const std::vector<double>& times, const std::vector<double>& values);
Error validate_cash_dividend(uint32_t node, double amount);
Error validate_constant_volatility(double sigma);
Error validate_event_schedule(const std::vector<double>& times, const std::vector<uint32_t>& dividend_nodes,
                              const std::vector<double>& dividend_amounts, const std::vector<uint32_t>& exercise_nodes,
                              uint32_t expiry);
Error validate_ragged_cash(const int64_t* offsets, uint64_t n_offsets, const double* times, uint64_t n_times,
                           const double* amounts, uint64_t n_amounts);
Error validate_ragged_exercise(const int64_t* offsets, uint64_t n_offsets, const double* times, uint64_t n_times);

// ---- single-contract plan -------------------------------------------------------------------

struct HostPlan {
    // schedule
    std::vector<double> times;
    std::vector<double> log_discounts;
    std::vector<StepCoef> steps;
    std::vector<NodeEvent> events;        // [intervals + 1]
    std::vector<uint32_t> row_node;       // observation nodes
    std::vector<double> disc_from_later;  // [rows]
    std::vector<double> disc_to_origin;   // [rows]
    std::vector<double> escrow_cash;      // [rows]
    double origin_discount = 1.0;
    bool origin_row = false;
    bool escrowed = false;
    int32_t policy = FO_DIVIDEND_LIQUIDATOR;
    double sim_start = 0.0;
    double initial_spot = 0.0;
    double strike = 0.0;
    // method
    uint64_t train_paths = 0, eval_paths = 0;
    uint64_t train_seed = 0, eval_seed = 0;
    uint32_t train_domain = 0, eval_domain = 0;
    int32_t degree = 4;
    double rank_tolerance = 1e-12, condition_limit = 1e8;
    int32_t tie_rule = FO_TIE_STRICTLY_GREATER;
    int32_t support = FO_SUPPORT_FAIL;

    uint32_t intervals() const { return uint32_t(steps.size()); }
    uint32_t rows() const { return uint32_t(row_node.size()); }
};

// Schedule + curves + volatility + policy -> transition plan (parse_gbm_model,
// crates/finoptions-python/src/lib.rs:723-829, and GbmPathPlan::try_new, path.rs:55-99).
Error build_gbm_plan(const double* schedule_times, uint64_t n_schedule, const double* curve_times, uint64_t n_curve,
                     const double* log_discounts, uint64_t n_ld, const double* yield_times, uint64_t n_yt,
                     const double* yields, uint64_t n_y, const uint32_t* dividend_nodes, uint64_t n_dn,
                     const double* dividend_amounts, uint64_t n_da, const uint32_t* exercise_nodes, uint64_t n_ex,
                     uint32_t expiry, double volatility, int32_t policy, HostPlan* plan);

// Full host-side validation of a single-contract request (price_lsm_call_seeded_f64 and
// LsmCallEstimator::price_seeded up to the first simulation).
Error build_call_plan(const fo_lsm_call_request& q, HostPlan* plan);

// Fills the observation discounts once rows and log discounts are known (policy.rs:1049-1108).
Error finish_discounts(HostPlan* plan);

// Messages for simulation failures (SimulationError Display).
std::string simulation_failure_message(int code, uint32_t interval, uint64_t path, double spot, double normal);
int32_t simulation_failure_code(int code);

// Typed errors of a failed backward row: the regression itself (fit_failure) or its rank /
// condition diagnostic (diag_failure), at exercise node `node`.
std::string node_str(uint32_t node);
Error fit_failure(const HostPlan& hp, const FitRecord& rec, uint32_t node);
Error diag_failure(const HostPlan& hp, const FitRecord& rec, uint32_t node);

}  // namespace fo

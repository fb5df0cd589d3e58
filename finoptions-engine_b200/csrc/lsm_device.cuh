// lsm_device.cuh - device-side data layout shared by the LSM kernels and the host plan builder.
#pragma once

#include <stdint.h>

#include "fo_core.cuh"

namespace fo {

// Per-interval transition coefficients (GbmStep, crates/finoptions-sim/src/step.rs:27-57),
// computed on the host exactly as the reference does.
struct StepCoef {
    double log_drift;
    double diffusion;
};

// Event phases at grid node n >= 1 (crates/finoptions-sim/src/path.rs:422-472): the observation
// row recorded at the node (-1 if none) and an optional cash dividend. At the terminal
// observation the cash jump precedes the record; elsewhere the record precedes the jump.
struct NodeEvent {
    double dividend_amount;
    int32_t row;
    int32_t flags;  // bit 0: dividend at node, bit 1: terminal observation
};

constexpr int32_t kEventDividend = 1;
constexpr int32_t kEventTerminal = 2;

// Rule of one exercise row once fitted (policy.rs:89-95).
enum RuleKind : int32_t {
    kRuleNone = 0,         // row 0 at the origin when not exercising, or a skipped row
    kRuleOrigin = 1,       // common origin decision
    kRuleNoSupport = 2,    // no in-the-money training path (Fail policy)
    kRuleContinue = 3,     // declared continuation without regression
    kRuleRegression = 4,
    kRuleFitFailed = 5,    // the fit raised a typed error; evaluation must not run
};

// What the backward pass records for one exercise row.
struct FitRecord {
    FitModel model;
    int32_t kind;            // RuleKind
    int32_t origin_exercise; // origin decision
    uint64_t itm;            // in-the-money training paths
    double origin_continuation;
    double pivot;
    // diagnostic (filled by the diagnose kernel for regression rows)
    int32_t diag_status;
    int32_t diag_rank;
    double diag_condition;
    int32_t diag_aux;
    int32_t pad;
};

// Device status words. Path-addressed failures keep the lowest key with atomicMin so the host
// reports the same failure the reference's serial order would (seeded.rs:171-186).
// The first kStatusNoneBytes bytes start as all-ones ("none"); the rest start at zero.
struct DeviceStatus {
    unsigned long long train_sim_fail;   // path (all-ones: none)
    unsigned long long eval_sim_fail;    // path
    unsigned long long fit_payoff_fail;  // (order << 32) | path: non-finite discounted value
    unsigned long long fit_predict_fail; // (order << 32) | path: non-finite prediction
    unsigned long long eval_fail;        // (row << 33) | (path << 1) | type (0 predict, 1 payoff)
    unsigned long long eval_terminal_fail;  // path: non-finite terminal payoff
    unsigned long long fit_nonfinite;    // (order << 32) | path: non-finite ITM predictor/response
    unsigned int fit_failed_order;       // first backward order whose fit failed
    unsigned int barrier_timeout;        // zero-initialised: a grid wait timed out
    unsigned int arrivals;               // zero-initialised: backward CTA partials published so far
};
constexpr size_t kStatusNoneBytes = 7 * sizeof(unsigned long long) + sizeof(unsigned int);

// Failure replay record for one path (filled by the replay kernel): the failure, if any, and
// the state observed at one requested row.
struct SimFailure {
    int32_t code;      // 0 none, kNormalBudget, kNormalRejection, or 3 = non-finite transition
    int32_t interval;
    double spot;
    double normal;
    double observed;   // state recorded at the requested row
};

// One contract's device-resident plan (pointers into one device allocation).
struct DevicePlan {
    uint32_t intervals;
    uint32_t rows;             // observation rows (exercise rows + expiry)
    uint32_t first_stored_row; // 1 when row 0 is the origin (constant S0, not stored)
    uint32_t pad0;
    double strike;
    double sim_start;          // S0, or the prepaid forward S0 - PV(cash) for escrowed plans
    double initial_spot;       // S0
    int32_t policy;
    int32_t escrowed;
    int32_t degree;
    int32_t tie_rule;
    int32_t support;
    int32_t origin_row;        // 1 when row 0 is node 0 (common origin decision)
    double rank_tolerance;
    double condition_limit;
    double rank_limit;         // rank_limit(rank_tolerance): the warp solve's rank test
    uint64_t train_paths, eval_paths;
    uint64_t train_seed, eval_seed;
    uint32_t train_domain, eval_domain;
    const StepCoef* steps;     // [intervals]
    const NodeEvent* events;   // [intervals + 1] (index by node; node 0 unused)
    const uint32_t* row_node;  // [rows]
    const double* disc_from_later;  // [rows]: exp(L[later] - L[node]) for positive exercise rows
    const double* disc_to_origin;   // [rows]: exp(L[node])
    const double* escrow_cash;      // [rows]: prepaid cash added to observations (escrowed)
    double origin_discount;    // exp(L[last processed node]) applied before the origin mean
};

// Device tables for ZIGNOR, held in shared memory.
struct SmemZig {
    const double* xs;
    const double* fs;
    double rr;
    FO_D double x(int i) const { return xs[i]; }
    FO_D double f(int i) const { return fs[i]; }
    FO_D double r() const { return rr; }
};

}  // namespace fo

// lsm_oracle.cpp - CPU restatement of finoptions-engine's Longstaff-Schwartz hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the parity oracle for the B200 engine: only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and only as the checker or as
// the timed CPU baseline. The product library never links or calls it.
//
// It restates, in plain C++ with the same operation order, the reference's CpuExecutor path:
//   Philox4x32-10 streams        crates/finoptions-sim/src/random/philox.rs:9-114
//   ZIGNOR normals               crates/finoptions-sim/src/random/normal.rs:33-109
//   exact GBM step               crates/finoptions-sim/src/step.rs:27-95
//   event-aligned path plan      crates/finoptions-sim/src/path.rs:55-99, 422-472, 618-944
//   fused seeded simulation      crates/finoptions-sim/src/path/seeded.rs:38-77, 147-196, 384-459
//   moment kernels               crates/finoptions-runtime/src/lib.rs:59-170
//   Stieltjes regression + SVD   crates/finoptions-lsm/src/regression.rs:197-850
//   policy fit / evaluation      crates/finoptions-lsm/src/policy.rs:215-926, 1049-1122
//   grouped batch                crates/finoptions-lsm/src/batch/{input,pricing}.rs
// Rust's f64::exp/ln/sqrt/hypot resolve to glibc on x86-64 Linux and mul_add to a correctly
// rounded fma; this file uses std::exp/log/sqrt/hypot/fma and is compiled with
// -ffp-contract=off, so it is expected to reproduce the reference bit for bit. It is pinned
// against the reference's own known-answer vectors in tests/test_oracle_*.py.
//
// Validation is restated only where the numeric path depends on it; the product library owns
// the full typed-error surface.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "../include/finoptions_cuda.h"
#include "../finoptions-engine_b200/csrc/zignor_tables.h"

namespace {

// ---------------------------------------------------------------------------------------------
// Error record (kind/code/indices; messages are the product's job).
// ---------------------------------------------------------------------------------------------

enum OracleCode : int32_t {
    ORC_OK = 0,
    ORC_BUDGET_EXHAUSTED = 1,
    ORC_REJECTION_LIMIT = 2,
    ORC_NON_FINITE_PATH_TRANSITION = 3,
    ORC_NON_FINITE_NORMAL_BUFFER = 4,
    ORC_INSUFFICIENT_OBSERVATIONS = 10,
    ORC_NON_FINITE_PREDICTOR = 11,
    ORC_NON_FINITE_RESPONSE = 12,
    ORC_DEGENERATE_PREDICTOR = 13,
    ORC_RANK_DEFICIENT = 14,
    ORC_CONDITION_LIMIT_EXCEEDED = 15,
    ORC_CONDITION_DID_NOT_CONVERGE = 16,
    ORC_NON_FINITE_FIT = 17,
    ORC_NON_FINITE_PREDICTION = 18,
    ORC_NON_FINITE_DISCOUNTED_PAYOFF = 20,
    ORC_EVALUATION_OUTSIDE_TRAINING_SUPPORT = 21,
    ORC_RANDOM_DOMAIN_COLLISION = 22,
    ORC_UNREPRESENTABLE_DISCOUNT = 23,
    ORC_INVALID_INPUT = 30,
    ORC_ESCROWED_NON_POSITIVE_FORWARD = 31,
    ORC_ESCROWED_NON_FINITE = 32,
    ORC_MESH_NODE_MISSING = 33,
};

struct Failure {
    int32_t code = ORC_OK;
    int64_t row = -1, node = -1, path = -1, interval = -1;
    int64_t a = -1, b = -1;  // auxiliary integers (e.g. rank / columns, itm / required)
    double x = 0.0;          // auxiliary value (e.g. condition number, scale)
    bool ok() const { return code == ORC_OK; }
};

Failure fail(int32_t code) {
    Failure f;
    f.code = code;
    return f;
}

void write_error(fo_error* err, const Failure& f, int32_t kind) {
    if (!err) return;
    std::memset(err, 0, sizeof(*err));
    err->kind = kind;
    err->code = f.code;
    err->row = f.row;
    err->group = -1;
    err->node = f.node;
    err->path = f.path;
    std::snprintf(err->message, sizeof(err->message),
                  "oracle failure code=%d row=%lld node=%lld path=%lld interval=%lld a=%lld b=%lld x=%.17g",
                  f.code, (long long)f.row, (long long)f.node, (long long)f.path,
                  (long long)f.interval, (long long)f.a, (long long)f.b, f.x);
}

double from_bits(uint64_t bits) {
    double value;
    std::memcpy(&value, &bits, sizeof(value));
    return value;
}
uint64_t to_bits(double value) {
    uint64_t bits;
    std::memcpy(&bits, &value, sizeof(bits));
    return bits;
}

// ---------------------------------------------------------------------------------------------
// Philox4x32-10 (philox.rs:3-40) and the path-local stream (philox.rs:52-114).
// ---------------------------------------------------------------------------------------------

constexpr uint32_t kMul0 = 0xd2511f53u;
constexpr uint32_t kMul1 = 0xcd9e8d57u;
constexpr uint32_t kKeyBump0 = 0x9e3779b9u;
constexpr uint32_t kKeyBump1 = 0xbb67ae85u;

void philox_round(uint32_t c[4], const uint32_t k[2]) {
    const uint64_t p0 = uint64_t(kMul0) * c[0];
    const uint64_t p1 = uint64_t(kMul1) * c[2];
    const uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
    const uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
    const uint32_t n0 = hi1 ^ c[1] ^ k[0];
    const uint32_t n2 = hi0 ^ c[3] ^ k[1];
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
}

void philox4x32_10(const uint32_t counter[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c[4] = {counter[0], counter[1], counter[2], counter[3]};
    uint32_t k[2] = {key_in[0], key_in[1]};
    philox_round(c, k);
    for (int round = 1; round < 10; ++round) {
        k[0] += kKeyBump0;
        k[1] += kKeyBump1;
        philox_round(c, k);
    }
    std::memcpy(out, c, sizeof(c));
}

struct PathStream {
    uint32_t key[2];
    uint32_t domain;
    uint32_t path;
    uint64_t next_block = 0;
    uint32_t remaining_normals;
    uint32_t buffer[4] = {0, 0, 0, 0};
    uint32_t position = 4;

    PathStream(uint64_t seed, uint32_t domain_, uint32_t path_, uint32_t budget)
        : key{uint32_t(seed), uint32_t(seed >> 32)}, domain(domain_), path(path_),
          remaining_normals(budget) {}

    void refill() {
        const uint32_t counter[4] = {uint32_t(next_block), uint32_t(next_block >> 32), path, domain};
        philox4x32_10(counter, key, buffer);
        position = 0;
        next_block += 1;
    }
    uint32_t next_u32() {
        if (position == 4) refill();
        return buffer[position++];
    }
    bool begin_normal() {
        if (remaining_normals == 0) return false;
        remaining_normals -= 1;
        return true;
    }
    uint64_t next_u64() {
        const uint64_t low = next_u32();
        const uint64_t high = next_u32();
        return low | (high << 32);
    }
};

// ---------------------------------------------------------------------------------------------
// ZIGNOR (normal.rs:9-109).
// ---------------------------------------------------------------------------------------------

constexpr uint64_t kZigX[257] = FO_ZIG_NORM_X_BITS;
constexpr uint64_t kZigF[257] = FO_ZIG_NORM_F_BITS;
constexpr size_t kMaxRejectionIterations = 1048576;
constexpr uint64_t kFractionMask = (uint64_t(1) << 52) - 1;
constexpr uint64_t kExponent0 = uint64_t(1023) << 52;
constexpr uint64_t kExponent1 = uint64_t(1024) << 52;

double zig_x(size_t i) { return from_bits(kZigX[i]); }
double zig_f(size_t i) { return from_bits(kZigF[i]); }
double zig_r() { return from_bits(FO_ZIG_NORM_R_BITS); }

double symmetric_unit(uint64_t bits) {
    return from_bits(((bits >> 12) & kFractionMask) | kExponent1) - 3.0;
}
double open_unit(PathStream& s) {
    const uint64_t bits = s.next_u64();
    const uint64_t fraction = (bits >> 12) & kFractionMask;
    const double epsilon = std::numeric_limits<double>::epsilon();
    return from_bits(fraction | kExponent0) - (1.0 - epsilon / 2.0);
}
double standard_unit(PathStream& s) {
    return double(s.next_u64() >> 11) * (1.0 / 9007199254740992.0);
}

int sample_tail(PathStream& s, double signed_unit, double* out) {
    const double r = zig_r();
    for (size_t it = 0; it < kMaxRejectionIterations; ++it) {
        const double x = std::log(open_unit(s)) / r;
        const double y = std::log(open_unit(s));
        if (-2.0 * y >= x * x) {
            *out = signed_unit < 0.0 ? x - r : r - x;
            return ORC_OK;
        }
    }
    return ORC_REJECTION_LIMIT;
}

int sample_rejected(PathStream& s, size_t index, double unit, double value, double* out) {
    for (size_t it = 0; it < kMaxRejectionIterations; ++it) {
        if (index == 0) return sample_tail(s, unit, out);
        const double ordinate = zig_f(index + 1) + (zig_f(index) - zig_f(index + 1)) * standard_unit(s);
        if (ordinate < std::exp(-0.5 * value * value)) {
            *out = value;
            return ORC_OK;
        }
        const uint64_t bits = s.next_u64();
        index = size_t(bits & 0xff);
        unit = symmetric_unit(bits);
        value = unit * zig_x(index);
        if (std::fabs(value) < zig_x(index + 1)) {
            *out = value;
            return ORC_OK;
        }
    }
    return ORC_REJECTION_LIMIT;
}

int sample_standard_normal(PathStream& s, double* out) {
    if (!s.begin_normal()) return ORC_BUDGET_EXHAUSTED;
    const uint64_t bits = s.next_u64();
    const size_t index = size_t(bits & 0xff);
    const double unit = symmetric_unit(bits);
    const double value = unit * zig_x(index);
    if (std::fabs(value) < zig_x(index + 1)) {
        *out = value;
        return ORC_OK;
    }
    return sample_rejected(s, index, unit, value, out);
}

// ---------------------------------------------------------------------------------------------
// Path plan (path.rs:55-99) and steps (step.rs:27-57).
// ---------------------------------------------------------------------------------------------

struct Step {
    double log_drift;
    double diffusion;
};

struct Plan {
    std::vector<double> times;
    std::vector<double> log_discounts;
    std::vector<Step> steps;                  // intervals
    std::vector<int8_t> has_dividend;         // by node
    std::vector<double> dividend_amount;      // by node
    std::vector<uint32_t> observation_nodes;  // exercise nodes followed by expiry
    int32_t policy = FO_DIVIDEND_LIQUIDATOR;
    // Escrowed model (path.rs:618-944): observations are risky prepaid forward + prepaid cash.
    bool escrowed = false;
    std::vector<double> prepaid_cash;         // by node
    size_t intervals() const { return steps.size(); }
    size_t rows() const { return observation_nodes.size(); }
    bool is_terminal_observation(uint32_t node) const { return observation_nodes.back() == node; }
};

Plan build_spot_plan(const std::vector<double>& times, const std::vector<double>& log_discounts,
                     const std::vector<double>& cumulative_yields, double volatility,
                     const std::vector<uint32_t>& dividend_nodes,
                     const std::vector<double>& dividend_amounts,
                     const std::vector<uint32_t>& exercise_nodes, uint32_t expiry, int32_t policy) {
    Plan plan;
    plan.times = times;
    plan.log_discounts = log_discounts;
    const size_t n = times.size();
    for (size_t to = 1; to < n; ++to) {
        const double dt = times[to] - times[to - 1];
        const double interval_log_discount = log_discounts[to] - log_discounts[to - 1];
        const double interval_yield = cumulative_yields[to] - cumulative_yields[to - 1];
        const double variance = std::fma(volatility, volatility, 0.0) * dt;
        const double log_drift = -interval_log_discount - interval_yield - 0.5 * variance;
        plan.steps.push_back(Step{log_drift, std::sqrt(variance)});
    }
    plan.has_dividend.assign(n, 0);
    plan.dividend_amount.assign(n, 0.0);
    for (size_t i = 0; i < dividend_nodes.size(); ++i) {
        plan.has_dividend[dividend_nodes[i]] = 1;
        plan.dividend_amount[dividend_nodes[i]] = dividend_amounts[i];
    }
    plan.observation_nodes = exercise_nodes;
    plan.observation_nodes.push_back(expiry);
    plan.policy = policy;
    return plan;
}

double apply_dividend(int32_t policy, double amount, double spot) {
    if (policy == FO_DIVIDEND_LIQUIDATOR) return std::max(spot - amount, 0.0);
    return spot > amount ? spot - amount : spot;
}

// Escrowed plan: prepaid cash by node (path.rs:889-944), risky plan without dividends.
Failure build_escrowed_plan(const std::vector<double>& times, const std::vector<double>& log_discounts,
                            double volatility, const std::vector<uint32_t>& dividend_nodes,
                            const std::vector<double>& dividend_amounts,
                            const std::vector<uint32_t>& exercise_nodes, uint32_t expiry, Plan* out) {
    const size_t n = times.size();
    std::vector<double> prepaid(n, 0.0);
    size_t event = dividend_nodes.size();
    const size_t last = n - 1;
    if (event > 0 && dividend_nodes[event - 1] == last) {
        event -= 1;
        prepaid[last] = dividend_amounts[event];
    }
    for (size_t node = n - 1; node-- > 0;) {
        const double interval_log_discount = log_discounts[node + 1] - log_discounts[node];
        const double discounted_future = prepaid[node + 1] * std::exp(interval_log_discount);
        double same_node_cash = 0.0;
        if (event > 0 && dividend_nodes[event - 1] == node) {
            event -= 1;
            same_node_cash = dividend_amounts[event];
        }
        const double value = discounted_future + same_node_cash;
        if (!std::isfinite(value)) {
            Failure f = fail(ORC_ESCROWED_NON_FINITE);
            f.node = int64_t(node);
            return f;
        }
        prepaid[node] = value;
    }
    double origin = 0.0;
    for (size_t i = 0; i < dividend_nodes.size(); ++i) {
        origin += dividend_amounts[i] * std::exp(log_discounts[dividend_nodes[i]]);
        if (!std::isfinite(origin)) {
            Failure f = fail(ORC_ESCROWED_NON_FINITE);
            f.node = 0;
            return f;
        }
    }
    prepaid[0] = origin;
    const std::vector<double> zero_yield(n, 0.0);
    *out = build_spot_plan(times, log_discounts, zero_yield, volatility, {}, {}, exercise_nodes,
                           expiry, FO_DIVIDEND_LIQUIDATOR);
    out->escrowed = true;
    out->prepaid_cash = prepaid;
    return Failure{};
}

// ---------------------------------------------------------------------------------------------
// Seeded simulation (seeded.rs:384-474).
// ---------------------------------------------------------------------------------------------

// One path; `obs` receives rows() pre-event states (path-major slice).
// `normals`, when given, replaces the Philox stream: the variate of interval i is
// normals[i * stride + path] (GbmPathPlan::simulate_with, path.rs:139-175).
Failure simulate_one(const Plan& plan, double initial_spot, uint32_t path, uint64_t seed,
                     uint32_t domain, double* obs, const double* normals = nullptr, uint64_t stride = 0) {
    const uint32_t budget = uint32_t(plan.times.size() - 1);
    PathStream stream(seed, domain, path, budget);
    double spot = initial_spot;
    size_t observation = 0;
    if (plan.observation_nodes[0] == 0) {
        obs[0] = spot;
        observation = 1;
    }
    for (size_t interval = 0; interval < plan.steps.size(); ++interval) {
        double normal = 0.0;
        const int status = normals ? ORC_OK : sample_standard_normal(stream, &normal);
        if (normals) normal = normals[interval * stride + path];
        if (status != ORC_OK) {
            Failure f = fail(status);
            f.interval = int64_t(interval);
            f.path = path;
            return f;
        }
        const Step step = plan.steps[interval];
        const double before = spot;
        double next = 0.0;
        if (before != 0.0) next = before * std::exp(std::fma(step.diffusion, normal, step.log_drift));
        if (!std::isfinite(next)) {
            Failure f = fail(ORC_NON_FINITE_PATH_TRANSITION);
            f.interval = int64_t(interval);
            f.node = int64_t(interval + 1);
            f.path = path;
            f.x = before;
            return f;
        }
        spot = next;
        const uint32_t node = uint32_t(interval + 1);
        const bool dividend = plan.has_dividend[node] != 0;
        const bool terminal = dividend && plan.is_terminal_observation(node);
        if (terminal) spot = apply_dividend(plan.policy, plan.dividend_amount[node], spot);
        if (observation < plan.rows() && plan.observation_nodes[observation] == node) {
            obs[observation] = spot;
            observation += 1;
        }
        if (dividend && !terminal) spot = apply_dividend(plan.policy, plan.dividend_amount[node], spot);
    }
    return Failure{};
}

// Escrowed reconstruction of one path's observations (path.rs:840-877).
Failure reconstruct_escrowed(const Plan& plan, double initial_spot, uint32_t path, double* obs) {
    const size_t last = plan.times.size() - 1;
    for (size_t row = 0; row < plan.rows(); ++row) {
        const uint32_t node = plan.observation_nodes[row];
        if (node == 0) {
            obs[row] = initial_spot;
            continue;
        }
        const double cash = node == last ? 0.0 : plan.prepaid_cash[node];
        const double stock = obs[row] + cash;
        if (!std::isfinite(stock)) {
            Failure f = fail(ORC_ESCROWED_NON_FINITE);
            f.node = node;
            f.path = path;
            return f;
        }
        obs[row] = stock;
    }
    return Failure{};
}

// Time-major [rows, paths] simulation, path-parallel over `threads` workers with the lowest
// failing path reported (seeded.rs:147-196). Escrowed plans start at S0 - prepaid[0].
Failure simulate(const Plan& plan, double initial_spot, uint64_t paths, uint64_t seed,
                 uint32_t domain, int threads, std::vector<double>* time_major, const double* normals = nullptr) {
    const size_t rows = plan.rows();
    double start = initial_spot;
    if (plan.escrowed) {
        start = initial_spot - plan.prepaid_cash[0];
        if (!std::isfinite(start) || start <= 0.0) return fail(ORC_ESCROWED_NON_POSITIVE_FORWARD);
    }
    time_major->assign(rows * paths, 0.0);
    std::atomic<uint64_t> first_failure{UINT64_MAX};
    auto worker = [&](uint64_t begin, uint64_t end) {
        std::vector<double> obs(rows);
        for (uint64_t p = begin; p < end; ++p) {
            if (p > first_failure.load(std::memory_order_relaxed)) return;
            Failure f = simulate_one(plan, start, uint32_t(p), seed, domain, obs.data(), normals, paths);
            if (f.ok() && plan.escrowed) f = reconstruct_escrowed(plan, initial_spot, uint32_t(p), obs.data());
            if (!f.ok()) {
                uint64_t cur = first_failure.load();
                while (p < cur && !first_failure.compare_exchange_weak(cur, p)) {}
                return;
            }
            for (size_t r = 0; r < rows; ++r) (*time_major)[r * paths + p] = obs[r];
        }
    };
    const int workers = std::max(1, std::min<int>(threads, int(std::min<uint64_t>(paths, 1u << 20))));
    if (workers == 1) {
        worker(0, paths);
    } else {
        std::vector<std::thread> pool;
        const uint64_t chunk = (paths + workers - 1) / workers;
        for (int w = 0; w < workers; ++w) {
            const uint64_t b = uint64_t(w) * chunk, e = std::min<uint64_t>(paths, b + chunk);
            if (b < e) pool.emplace_back(worker, b, e);
        }
        for (auto& t : pool) t.join();
    }
    const uint64_t failed = first_failure.load();
    if (failed != UINT64_MAX) {
        std::vector<double> obs(rows);
        Failure f = simulate_one(plan, start, uint32_t(failed), seed, domain, obs.data(), normals, paths);
        if (f.ok() && plan.escrowed) f = reconstruct_escrowed(plan, initial_spot, uint32_t(failed), obs.data());
        return f;
    }
    return Failure{};
}

// ---------------------------------------------------------------------------------------------
// Regression (regression.rs:197-850, runtime/src/lib.rs:59-170).
// ---------------------------------------------------------------------------------------------

constexpr int kMaxDegree = 4;
constexpr int kMaxColumns = kMaxDegree + 1;
constexpr int kJacobiMaxSweeps = 32;

struct Spec {
    int degree;
    double rank_tolerance;
    double condition_limit;
};

struct Model {
    int degree = 0;
    double mean = 0.0, scale = 1.0;
    double alphas[kMaxDegree] = {0, 0, 0, 0};
    double betas[kMaxDegree] = {0, 0, 0, 0};
    double coefficients[kMaxColumns] = {0, 0, 0, 0, 0};
    double norms[kMaxColumns] = {0, 0, 0, 0, 0};
    uint64_t observations = 0;
    int rank = 0;
    double condition_number = 0.0;
};

// polynomial_moments_f64 (runtime/src/lib.rs:84-95)
void moments(const double* z, const double* y, const double* basis, size_t n, double out[3]) {
    double norm = 0.0, projection = 0.0, weighted = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double sq = basis[i] * basis[i];
        norm += sq;
        projection = std::fma(y[i], basis[i], projection);
        weighted = std::fma(z[i], sq, weighted);
    }
    out[0] = norm;
    out[1] = projection;
    out[2] = weighted;
}

// polynomial_recurrence_moments_f64 (runtime/src/lib.rs:145-157)
void recurrence_moments(const double* z, const double* y, const double* previous, const double* current,
                        double* next, size_t n, double alpha, double beta, double out[3]) {
    double norm = 0.0, projection = 0.0, weighted = 0.0;
    for (size_t i = 0; i < n; ++i) {
        next[i] = std::fma(z[i] - alpha, current[i], -beta * previous[i]);
        const double sq = next[i] * next[i];
        norm += sq;
        projection = std::fma(y[i], next[i], projection);
        weighted = std::fma(z[i], sq, weighted);
    }
    out[0] = norm;
    out[1] = projection;
    out[2] = weighted;
}

Failure rank_deficient(int degree, int rank) {
    Failure f = fail(ORC_RANK_DEFICIENT);
    f.a = rank;
    f.b = degree + 1;
    return f;
}

// one_sided_jacobi_singular_values_for (regression.rs:766-850)
Failure jacobi_singular_values(double m[kMaxColumns * kMaxColumns], int columns, double sv[kMaxColumns]) {
    const double tolerance = 16.0 * std::numeric_limits<double>::epsilon();
    bool converged = false;
    for (int sweep = 0; sweep < kJacobiMaxSweeps; ++sweep) {
        converged = true;
        for (int left = 0; left + 1 < columns; ++left) {
            for (int right = left + 1; right < columns; ++right) {
                double ln = 0.0, rn = 0.0, cross = 0.0;
                for (int row = 0; row < columns; ++row) {
                    const double lv = m[left * kMaxColumns + row];
                    const double rv = m[right * kMaxColumns + row];
                    ln = std::fma(lv, lv, ln);
                    rn = std::fma(rv, rv, rn);
                    cross = std::fma(lv, rv, cross);
                }
                if (!std::isfinite(ln) || !std::isfinite(rn) || !std::isfinite(cross) || ln <= 0.0 || rn <= 0.0) {
                    Failure f = fail(ORC_NON_FINITE_FIT);
                    f.a = right;
                    return f;
                }
                if (std::fabs(cross) <= tolerance * std::sqrt(ln * rn)) continue;
                converged = false;
                const double zeta = (rn - ln) / (2.0 * cross);
                double tangent = 1.0;
                if (zeta != 0.0) tangent = std::copysign(1.0, zeta) / (std::fabs(zeta) + std::hypot(zeta, 1.0));
                const double cosine = 1.0 / std::sqrt(std::fma(tangent, tangent, 1.0));
                const double sine = cosine * tangent;
                for (int row = 0; row < columns; ++row) {
                    const int li = left * kMaxColumns + row, ri = right * kMaxColumns + row;
                    const double lv = m[li], rv = m[ri];
                    m[li] = std::fma(cosine, lv, -sine * rv);
                    m[ri] = std::fma(sine, lv, cosine * rv);
                }
            }
        }
        if (converged) break;
    }
    if (!converged) {
        Failure f = fail(ORC_CONDITION_DID_NOT_CONVERGE);
        f.a = columns;
        return f;
    }
    for (int c = 0; c < kMaxColumns; ++c) sv[c] = 0.0;
    for (int c = 0; c < columns; ++c) {
        double sq = 0.0;
        for (int row = 0; row < columns; ++row) {
            const double v = m[c * kMaxColumns + row];
            sq += v * v;
        }
        sv[c] = std::sqrt(sq);
    }
    std::sort(sv, sv + columns, [](double a, double b) { return a > b; });
    return Failure{};
}

// orthonormal_basis_transform + diagnose_design (regression.rs:540-577, 711-750)
Failure diagnose(Model* model, const Spec& spec) {
    const int degree = spec.degree, columns = degree + 1;
    double transform[kMaxColumns * kMaxColumns] = {};
    double previous[kMaxColumns] = {}, current[kMaxColumns] = {};
    current[0] = 1.0;
    for (int j = 0; j <= degree; ++j) {
        const double inverse_norm = 1.0 / std::sqrt(model->norms[j]);
        if (!std::isfinite(inverse_norm)) {
            Failure f = fail(ORC_NON_FINITE_FIT);
            f.a = j;
            return f;
        }
        for (int k = 0; k <= j; ++k) transform[j * kMaxColumns + k] = current[k] * inverse_norm;
        if (j == degree) break;
        double next[kMaxColumns] = {};
        for (int k = 0; k <= j; ++k) {
            next[k + 1] += current[k];
            next[k] -= model->alphas[j] * current[k];
            next[k] -= model->betas[j] * previous[k];
        }
        for (double v : next) {
            if (!std::isfinite(v)) {
                Failure f = fail(ORC_NON_FINITE_FIT);
                f.a = j + 1;
                return f;
            }
        }
        std::memcpy(previous, current, sizeof(current));
        std::memcpy(current, next, sizeof(next));
    }
    double sv[kMaxColumns];
    Failure f = jacobi_singular_values(transform, columns, sv);
    if (!f.ok()) return f;
    const double largest = sv[0];
    const double threshold = spec.rank_tolerance * largest;
    int rank = 0;
    for (int c = 0; c < columns; ++c) rank += sv[c] > threshold ? 1 : 0;
    if (rank < columns) return rank_deficient(degree, rank);
    const double condition = largest / sv[columns - 1];
    if (!std::isfinite(condition)) {
        Failure g = fail(ORC_NON_FINITE_FIT);
        g.a = degree;
        return g;
    }
    if (condition > spec.condition_limit) {
        Failure g = fail(ORC_CONDITION_LIMIT_EXCEEDED);
        g.x = condition;
        return g;
    }
    model->rank = rank;
    model->condition_number = condition;
    return Failure{};
}

// RegressionWorkspace::fit_population (regression.rs:369-523) over an ITM population whose
// Welford location was accumulated in source order (regression.rs:279-297, 315-325).
Failure fit_population(const std::vector<double>& x, const std::vector<double>& y, const Spec& spec,
                       Model* model) {
    const size_t n = x.size();
    const int degree = spec.degree, columns = degree + 1;
    if (n < size_t(columns)) {
        Failure f = fail(ORC_INSUFFICIENT_OBSERVATIONS);
        f.a = int64_t(n);
        f.b = columns;
        return f;
    }
    // Welford over finite predictors in population order; non-finite checks (regression.rs:614-627).
    double count = 0.0, mean = 0.0, m2 = 0.0;
    int64_t bad_x = -1, bad_y = -1;
    for (size_t i = 0; i < n; ++i) {
        if (!std::isfinite(x[i])) {
            if (bad_x < 0) bad_x = int64_t(i);
        } else if (degree != 0) {
            count += 1.0;
            const double delta = x[i] - mean;
            mean += delta / count;
            m2 = std::fma(delta, x[i] - mean, m2);
        }
        if (!std::isfinite(y[i]) && bad_y < 0) bad_y = int64_t(i);
    }
    if (bad_x >= 0) {
        Failure f = fail(ORC_NON_FINITE_PREDICTOR);
        f.a = bad_x;
        return f;
    }
    if (bad_y >= 0) {
        Failure f = fail(ORC_NON_FINITE_RESPONSE);
        f.a = bad_y;
        return f;
    }
    double location = 0.0, scale = 1.0;
    if (degree != 0) {
        scale = std::sqrt(m2 / count);
        if (!std::isfinite(mean) || !std::isfinite(scale) || scale <= 0.0) {
            Failure f = fail(ORC_DEGENERATE_PREDICTOR);
            f.x = scale;
            return f;
        }
        location = mean;
    }
    std::vector<double> z(n), previous(n, 0.0), current(n, 1.0), next(n, 0.0);
    for (size_t i = 0; i < n; ++i) z[i] = degree == 0 ? 0.0 : (x[i] - location) / scale;

    Model out;
    out.degree = degree;
    out.mean = location;
    out.scale = scale;
    double previous_norm = 1.0;
    double pending[3];
    moments(z.data(), y.data(), current.data(), n, pending);
    for (int j = 0; j <= degree; ++j) {
        const double norm = pending[0], projection = pending[1], weighted = pending[2];
        if (!std::isfinite(norm) || !std::isfinite(projection) || !std::isfinite(weighted)) {
            Failure f = fail(ORC_NON_FINITE_FIT);
            f.a = j;
            return f;
        }
        if (norm <= 0.0) return rank_deficient(degree, j);
        const double relative_pivot = std::sqrt(norm / double(uint32_t(n)));
        if (relative_pivot <= spec.rank_tolerance) return rank_deficient(degree, j);
        out.norms[j] = norm;
        out.coefficients[j] = projection / norm;
        if (!std::isfinite(out.coefficients[j])) {
            Failure f = fail(ORC_NON_FINITE_FIT);
            f.a = j;
            return f;
        }
        if (j < degree) {
            out.alphas[j] = weighted / norm;
            out.betas[j] = j == 0 ? 0.0 : norm / previous_norm;
            if (!std::isfinite(out.alphas[j]) || !std::isfinite(out.betas[j])) {
                Failure f = fail(ORC_NON_FINITE_FIT);
                f.a = j;
                return f;
            }
            recurrence_moments(z.data(), y.data(), previous.data(), current.data(), next.data(), n,
                               out.alphas[j], out.betas[j], pending);
            if (!std::isfinite(pending[0]) || !std::isfinite(pending[1]) || !std::isfinite(pending[2])) {
                Failure f = fail(ORC_NON_FINITE_FIT);
                f.a = j + 1;
                return f;
            }
            previous_norm = norm;
            std::swap(previous, current);
            std::swap(current, next);
        }
    }
    out.observations = n;
    Failure f = diagnose(&out, spec);
    if (!f.ok()) return f;
    *model = out;
    return Failure{};
}

// PolynomialModel::predict_for (regression.rs:197-224)
bool predict(const Model& m, double predictor, double* out) {
    if (!std::isfinite(predictor)) return false;
    const double z = m.degree == 0 ? 0.0 : (predictor - m.mean) / m.scale;
    double prediction = m.coefficients[0];
    double previous = 0.0, current = 1.0;
    for (int j = 0; j < m.degree; ++j) {
        const double next = std::fma(z - m.alphas[j], current, -m.betas[j] * previous);
        prediction = std::fma(m.coefficients[j + 1], next, prediction);
        previous = current;
        current = next;
    }
    if (!std::isfinite(prediction)) return false;
    *out = prediction;
    return true;
}

// ---------------------------------------------------------------------------------------------
// Policy fit and evaluation (policy.rs:215-926).
// ---------------------------------------------------------------------------------------------

enum RuleKind { RULE_ORIGIN, RULE_NO_SUPPORT, RULE_CONTINUE, RULE_REGRESSION };

struct Rule {
    RuleKind kind = RULE_CONTINUE;
    bool exercise = false;
    Model model;
};

struct Estimator {
    double strike;
    Spec spec;
    int32_t tie_rule;
    int32_t support;
};

bool should_exercise(int32_t tie, double intrinsic, double continuation) {
    return tie == FO_TIE_STRICTLY_GREATER ? intrinsic > continuation : intrinsic >= continuation;
}

double call_intrinsic(double spot, double strike) { return std::max(spot - strike, 0.0); }

bool checked_discount(double log_discount, double* out) {
    const double d = std::exp(log_discount);
    if (!std::isfinite(d) || d <= 0.0) return false;
    *out = d;
    return true;
}

struct Fitted {
    std::vector<Rule> rules;                        // one per exercise row
    std::vector<fo_lsm_node_diagnostic> diagnostics;
    std::vector<double> discount_to_origin;         // per observation row
};

Failure fit_policy(const Estimator& est, const Plan& plan, const std::vector<double>& training,
                   uint64_t paths, double initial_spot, Fitted* fitted) {
    const size_t rows = plan.rows();
    const size_t exercise_rows = rows - 1;
    const double* terminal = training.data() + exercise_rows * paths;
    std::vector<double> values(paths);
    for (uint64_t p = 0; p < paths; ++p) values[p] = call_intrinsic(terminal[p], est.strike);
    std::vector<Rule> reversed_rules;
    std::vector<fo_lsm_node_diagnostic> reversed_diags;
    uint32_t later = plan.observation_nodes[exercise_rows];
    const uint32_t required = uint32_t(est.spec.degree + 1);
    std::vector<double> px, py;
    std::vector<uint64_t> src;
    for (size_t row = exercise_rows; row-- > 0;) {
        const uint32_t node = plan.observation_nodes[row];
        if (node == 0) continue;
        double discount;
        if (!checked_discount(plan.log_discounts[later] - plan.log_discounts[node], &discount)) {
            Failure f = fail(ORC_UNREPRESENTABLE_DISCOUNT);
            f.node = node;
            return f;
        }
        for (uint64_t p = 0; p < paths; ++p) {
            values[p] *= discount;
            if (!std::isfinite(values[p])) {
                Failure f = fail(ORC_NON_FINITE_DISCOUNTED_PAYOFF);
                f.path = int64_t(p);
                return f;
            }
        }
        const double* spots = training.data() + row * paths;
        px.clear();
        py.clear();
        src.clear();
        for (uint64_t p = 0; p < paths; ++p) {
            if (spots[p] > est.strike) {
                px.push_back(spots[p] / est.strike);
                py.push_back(values[p]);
                src.push_back(p);
            }
        }
        fo_lsm_node_diagnostic d{};
        d.node = node;
        Rule rule;
        if (px.empty()) {
            if (est.support == FO_SUPPORT_CONTINUE) {
                rule.kind = RULE_CONTINUE;
                d.kind = FO_DIAG_INSUFFICIENT_SUPPORT;
                d.in_the_money_paths = 0;
                d.columns = required;
            } else {
                rule.kind = RULE_NO_SUPPORT;
                d.kind = FO_DIAG_NO_IN_THE_MONEY_PATHS;
            }
        } else if (px.size() < required && est.support == FO_SUPPORT_CONTINUE) {
            rule.kind = RULE_CONTINUE;
            d.kind = FO_DIAG_INSUFFICIENT_SUPPORT;
            d.in_the_money_paths = uint32_t(px.size());
            d.columns = required;
        } else {
            Model model;
            Failure f = fit_population(px, py, est.spec, &model);
            if (!f.ok()) {
                f.node = node;
                return f;
            }
            for (size_t i = 0; i < px.size(); ++i) {
                const uint64_t p = src[i];
                const double intrinsic = spots[p] - est.strike;
                double continuation;
                if (!predict(model, px[i], &continuation)) {
                    Failure g = fail(ORC_NON_FINITE_PREDICTION);
                    g.node = node;
                    g.path = int64_t(p);
                    return g;
                }
                if (should_exercise(est.tie_rule, intrinsic, continuation)) values[p] = intrinsic;
            }
            rule.kind = RULE_REGRESSION;
            rule.model = model;
            d.kind = FO_DIAG_REGRESSION;
            d.in_the_money_paths = uint32_t(px.size());
            d.observations = model.observations;
            d.columns = required;
            d.rank = uint64_t(model.rank);
            d.condition_number = model.condition_number;
            d.predictor_mean = model.mean;
            d.predictor_scale = model.scale;
        }
        reversed_rules.push_back(rule);
        reversed_diags.push_back(d);
        later = node;
    }
    double to_origin;
    if (!checked_discount(plan.log_discounts[later], &to_origin)) {
        Failure f = fail(ORC_UNREPRESENTABLE_DISCOUNT);
        f.node = later;
        return f;
    }
    for (uint64_t p = 0; p < paths; ++p) {
        values[p] *= to_origin;
        if (!std::isfinite(values[p])) {
            Failure f = fail(ORC_NON_FINITE_DISCOUNTED_PAYOFF);
            f.path = int64_t(p);
            return f;
        }
    }
    if (plan.observation_nodes[0] == 0) {
        // online_mean (policy.rs:1110-1122)
        uint32_t count = 0;
        double mean = 0.0;
        for (uint64_t p = 0; p < paths; ++p) {
            count += 1;
            mean += (values[p] - mean) / double(count);
        }
        const double intrinsic = call_intrinsic(initial_spot, est.strike);
        Rule rule;
        rule.kind = RULE_ORIGIN;
        rule.exercise = should_exercise(est.tie_rule, intrinsic, mean);
        fo_lsm_node_diagnostic d{};
        d.node = 0;
        d.kind = FO_DIAG_ORIGIN_DECISION;
        d.exercise = rule.exercise ? 1 : 0;
        d.estimated_continuation = mean;
        reversed_rules.push_back(rule);
        reversed_diags.push_back(d);
    }
    std::reverse(reversed_rules.begin(), reversed_rules.end());
    std::reverse(reversed_diags.begin(), reversed_diags.end());
    fitted->rules = reversed_rules;
    fitted->diagnostics = reversed_diags;
    fitted->discount_to_origin.resize(rows);
    for (size_t r = 0; r < rows; ++r) {
        if (!checked_discount(plan.log_discounts[plan.observation_nodes[r]], &fitted->discount_to_origin[r])) {
            Failure f = fail(ORC_UNREPRESENTABLE_DISCOUNT);
            f.node = plan.observation_nodes[r];
            return f;
        }
    }
    return Failure{};
}

struct Evaluation {
    double price = 0.0;
    uint32_t paths = 0;
    bool has_sd = false;
    double sd = 0.0, se = 0.0;
    std::vector<uint32_t> counts;
};

// payoffs_out / stops_out (optional, `paths` entries each) receive every path's discounted payoff
// and the observation row at which it stopped: the per-path record finite-difference checks use to
// find the paths whose stopping row a bump moved.
Failure evaluate(const Estimator& est, const Plan& plan, const Fitted& fitted,
                 const std::vector<double>& evaluation, uint64_t paths, double initial_spot,
                 Evaluation* out, double* payoffs_out = nullptr, uint32_t* stops_out = nullptr) {
    const size_t rows = plan.rows();
    out->paths = uint32_t(paths);
    out->counts.assign(rows, 0);
    if (!fitted.rules.empty() && fitted.rules[0].kind == RULE_ORIGIN && fitted.rules[0].exercise) {
        out->counts[0] = uint32_t(paths);
        out->price = call_intrinsic(initial_spot, est.strike);
        out->has_sd = true;
        out->sd = 0.0;
        out->se = 0.0;
        for (uint64_t p = 0; p < paths; ++p) {
            if (payoffs_out) payoffs_out[p] = out->price;
            if (stops_out) stops_out[p] = 0;
        }
        return Failure{};
    }
    std::vector<uint8_t> active(paths, 1);
    std::vector<double> payoffs(paths, 0.0);
    for (size_t row = 0; row < fitted.rules.size(); ++row) {
        const Rule& rule = fitted.rules[row];
        const double* spots = evaluation.data() + row * paths;
        if (rule.kind == RULE_NO_SUPPORT) {
            uint64_t itm = 0;
            for (uint64_t p = 0; p < paths; ++p) itm += (active[p] && spots[p] > est.strike) ? 1 : 0;
            if (itm > 0) {
                Failure f = fail(ORC_EVALUATION_OUTSIDE_TRAINING_SUPPORT);
                f.node = plan.observation_nodes[row];
                f.a = int64_t(itm);
                return f;
            }
        } else if (rule.kind == RULE_REGRESSION) {
            const double discount = fitted.discount_to_origin[row];
            uint32_t count = 0;
            for (uint64_t p = 0; p < paths; ++p) {
                if (!active[p] || spots[p] <= est.strike) continue;
                const double intrinsic = spots[p] - est.strike;
                double continuation;
                if (!predict(rule.model, spots[p] / est.strike, &continuation)) {
                    Failure f = fail(ORC_NON_FINITE_PREDICTION);
                    f.node = plan.observation_nodes[row];
                    f.path = int64_t(p);
                    return f;
                }
                if (should_exercise(est.tie_rule, intrinsic, continuation)) {
                    const double payoff = intrinsic * discount;
                    if (!std::isfinite(payoff)) {
                        Failure f = fail(ORC_NON_FINITE_DISCOUNTED_PAYOFF);
                        f.path = int64_t(p);
                        return f;
                    }
                    payoffs[p] = payoff;
                    active[p] = 0;
                    if (stops_out) stops_out[p] = uint32_t(row);
                    count += 1;
                }
            }
            out->counts[row] = count;
        }
    }
    const size_t terminal_row = rows - 1;
    const double terminal_discount = fitted.discount_to_origin[terminal_row];
    const double* terminal = evaluation.data() + terminal_row * paths;
    uint32_t terminal_count = 0;
    for (uint64_t p = 0; p < paths; ++p) {
        if (!active[p]) continue;
        const double payoff = call_intrinsic(terminal[p], est.strike) * terminal_discount;
        if (!std::isfinite(payoff)) {
            Failure f = fail(ORC_NON_FINITE_DISCOUNTED_PAYOFF);
            f.path = int64_t(p);
            return f;
        }
        payoffs[p] = payoff;
        active[p] = 0;
        if (stops_out) stops_out[p] = uint32_t(terminal_row);
        terminal_count += 1;
    }
    out->counts[terminal_row] = terminal_count;
    if (payoffs_out) std::copy(payoffs.begin(), payoffs.end(), payoffs_out);
    // LsmEvaluation::from_path_payoffs (policy.rs:891-926)
    uint32_t count = 0;
    double mean = 0.0, m2 = 0.0;
    for (uint64_t p = 0; p < paths; ++p) {
        count += 1;
        const double delta = payoffs[p] - mean;
        mean += delta / double(count);
        m2 = std::fma(delta, payoffs[p] - mean, m2);
    }
    out->price = mean;
    if (paths > 1) {
        const double sd = std::sqrt(m2 / double(uint32_t(paths - 1)));
        const double se = sd / std::sqrt(double(uint32_t(paths)));
        if (!std::isfinite(sd) || !std::isfinite(se)) {
            Failure f = fail(ORC_NON_FINITE_DISCOUNTED_PAYOFF);
            f.path = 0;
            return f;
        }
        out->has_sd = true;
        out->sd = sd;
        out->se = se;
    }
    return Failure{};
}

// The payoffs of evaluation paths whose stopping rows are given (frozen_stops[p], e.g. the rows a
// base market's policy chose): (S_row - K) exp(L_row) at an early row, max(S_T - K, 0) exp(L_T) at
// expiry. With every decision frozen, a central difference of this price over a bumped market is
// the pathwise derivative that a fixed-policy adjoint forms (the exercise indicators held fixed).
Failure evaluate_frozen(const Estimator& est, const Plan& plan, const Fitted& fitted,
                        const std::vector<double>& evaluation, uint64_t paths, const uint32_t* frozen_stops,
                        Evaluation* out, double* payoffs_out, uint32_t* stops_out) {
    const size_t rows = plan.rows();
    out->paths = uint32_t(paths);
    out->counts.assign(rows, 0);
    std::vector<double> payoffs(paths, 0.0);
    for (uint64_t p = 0; p < paths; ++p) {
        const uint32_t row = frozen_stops[p];
        if (row >= rows) return fail(ORC_INVALID_INPUT);
        const double spot = evaluation[row * paths + p];
        const double intrinsic = row + 1 == rows ? call_intrinsic(spot, est.strike) : spot - est.strike;
        payoffs[p] = intrinsic * fitted.discount_to_origin[row];
        out->counts[row] += 1;
        if (stops_out) stops_out[p] = row;
    }
    uint32_t count = 0;
    double mean = 0.0, m2 = 0.0;
    for (uint64_t p = 0; p < paths; ++p) {
        count += 1;
        const double delta = payoffs[p] - mean;
        mean += delta / double(count);
        m2 = std::fma(delta, payoffs[p] - mean, m2);
    }
    out->price = mean;
    out->has_sd = paths > 1;
    out->sd = paths > 1 ? std::sqrt(m2 / double(uint32_t(paths - 1))) : 0.0;
    out->se = paths > 1 ? out->sd / std::sqrt(double(uint32_t(paths))) : 0.0;
    if (payoffs_out) std::copy(payoffs.begin(), payoffs.end(), payoffs_out);
    return Failure{};
}

enum Stage { STAGE_TRAINING_SIM = 1, STAGE_FIT = 2, STAGE_EVALUATION_SIM = 3, STAGE_EVALUATION = 4 };

// LsmCallEstimator::price_seeded (policy.rs:306-336).
Failure price_seeded(const Estimator& est, const Plan& plan, double initial_spot, uint64_t training_paths,
                     uint64_t evaluation_paths, uint64_t training_seed, uint32_t training_domain,
                     uint64_t evaluation_seed, uint32_t evaluation_domain, int threads, Fitted* fitted,
                     Evaluation* evaluation, int* stage) {
    if (training_domain == evaluation_domain) {
        *stage = 0;
        Failure f = fail(ORC_RANDOM_DOMAIN_COLLISION);
        f.a = training_domain;
        return f;
    }
    std::vector<double> paths;
    Failure f = simulate(plan, initial_spot, training_paths, training_seed, training_domain, threads, &paths);
    if (!f.ok()) {
        *stage = STAGE_TRAINING_SIM;
        return f;
    }
    f = fit_policy(est, plan, paths, training_paths, initial_spot, fitted);
    if (!f.ok()) {
        *stage = STAGE_FIT;
        return f;
    }
    paths.clear();
    paths.shrink_to_fit();
    f = simulate(plan, initial_spot, evaluation_paths, evaluation_seed, evaluation_domain, threads, &paths);
    if (!f.ok()) {
        *stage = STAGE_EVALUATION_SIM;
        return f;
    }
    f = evaluate(est, plan, *fitted, paths, evaluation_paths, initial_spot, evaluation);
    if (!f.ok()) *stage = STAGE_EVALUATION;
    return f;
}

template <typename T>
std::vector<T> to_vec(const T* data, uint64_t n) {
    return data ? std::vector<T>(data, data + n) : std::vector<T>();
}

// ---------------------------------------------------------------------------------------------
// Grouped batches (batch/pricing.rs:422-589, 704-1114).
// ---------------------------------------------------------------------------------------------

uint32_t next_base_node_or(uint32_t node, uint32_t final_node, bool* done) {
    if (node == final_node) {
        *done = true;
        return node;
    }
    return node + 1;
}

// exact_union_times (pricing.rs:967-1047)
std::vector<double> exact_union_times(double maturity, uint32_t base_intervals, const double* cash, size_t n_cash) {
    std::vector<double> times;
    bool base_done = false;
    uint32_t base_node = 0;
    size_t event = 0;
    auto total_cmp = [](double a, double b) {
        // total order on finite, non-negative times is the numeric order with -0 < +0
        if (a < b) return -1;
        if (a > b) return 1;
        const bool sa = std::signbit(a), sb = std::signbit(b);
        if (sa == sb) return 0;
        return sa ? -1 : 1;
    };
    while (!base_done || event < n_cash) {
        bool have_base = !base_done;
        double base = 0.0;
        if (have_base) {
            base = base_node == base_intervals ? maturity
                                               : maturity * (double(base_node) / double(base_intervals));
        }
        const bool have_cash = event < n_cash;
        if (have_base && have_cash) {
            const int c = total_cmp(base, cash[event]);
            if (c < 0) {
                times.push_back(base);
                base_node = next_base_node_or(base_node, base_intervals, &base_done);
            } else if (c == 0) {
                times.push_back(base);
                base_node = next_base_node_or(base_node, base_intervals, &base_done);
                event += 1;
            } else {
                times.push_back(cash[event]);
                event += 1;
            }
        } else if (have_base) {
            times.push_back(base);
            base_node = next_base_node_or(base_node, base_intervals, &base_done);
        } else if (have_cash) {
            times.push_back(cash[event]);
            event += 1;
        } else {
            break;
        }
    }
    return times;
}

// exact_explicit_union_times (pricing.rs:1049-1114)
std::vector<double> exact_explicit_union_times(double maturity, const double* ex, size_t n_ex,
                                               const double* cash, size_t n_cash) {
    std::vector<double> times{0.0};
    size_t e = 0, c = 0;
    while (e < n_ex || c < n_cash) {
        double next;
        if (e < n_ex && c < n_cash) {
            if (ex[e] < cash[c]) {
                next = ex[e++];
            } else if (ex[e] == cash[c]) {
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
    return times;
}

int64_t find_exact(const std::vector<double>& grid, double t) {
    auto it = std::lower_bound(grid.begin(), grid.end(), t);
    if (it != grid.end() && to_bits(*it) == to_bits(t)) return int64_t(it - grid.begin());
    return -1;
}

struct GroupOutput {
    double price, sd, se;
    uint8_t origin_fitted, origin_exercised;
    uint32_t regression_nodes, no_support_nodes, insufficient_nodes, min_itm;
    double max_condition;
    uint32_t early, expiry;
};

// price_group_into for one group (pricing.rs:505-589, 704-748, 862-965).
Failure price_group(const fo_lsm_grouped_request* q, uint64_t group, uint64_t first_row,
                    uint64_t end_row, int threads, GroupOutput* outputs) {
    const double maturity = q->maturities[group];
    const double rate = q->rates[group];
    const double s0 = q->initial_spots[group];
    std::vector<double> cash_times, cash_amounts;
    if (q->dividend_model != FO_MODEL_CONTINUOUS_YIELD) {
        const int64_t base = q->dividend_offsets[0];
        const int64_t b = q->dividend_offsets[group] - base, e = q->dividend_offsets[group + 1] - base;
        cash_times.assign(q->dividend_times + b, q->dividend_times + e);
        cash_amounts.assign(q->dividend_amounts + b, q->dividend_amounts + e);
    }
    const double q_yield = q->dividend_model == FO_MODEL_CONTINUOUS_YIELD ? q->dividend_yields[group] : 0.0;
    std::vector<double> times;
    std::vector<uint32_t> exercise;
    if (q->exercise_mesh == FO_MESH_UNIFORM) {
        times = exact_union_times(maturity, q->base_intervals, cash_times.data(), cash_times.size());
        const size_t start = q->origin_exercise == FO_ORIGIN_EXCLUDED ? 1 : 0;
        for (size_t n = start; n + 1 < times.size(); ++n) exercise.push_back(uint32_t(n));
    } else if (q->exercise_mesh == FO_MESH_CASH_DIVIDEND_DATES) {
        times = exact_union_times(maturity, 1, cash_times.data(), cash_times.size());
        for (size_t n = 1; n + 1 < times.size(); ++n) exercise.push_back(uint32_t(n));
    } else {
        const int64_t base = q->explicit_exercise_offsets[0];
        const int64_t b = q->explicit_exercise_offsets[group] - base;
        const int64_t e = q->explicit_exercise_offsets[group + 1] - base;
        const double* ex = q->explicit_exercise_times + b;
        times = exact_explicit_union_times(maturity, ex, size_t(e - b), cash_times.data(), cash_times.size());
        if (q->origin_exercise == FO_ORIGIN_INCLUDED) exercise.push_back(0);
        for (int64_t i = 0; i < e - b; ++i) {
            const int64_t node = find_exact(times, ex[i]);
            if (node < 0) {
                Failure f = fail(ORC_MESH_NODE_MISSING);
                f.row = int64_t(first_row);
                return f;
            }
            exercise.push_back(uint32_t(node));
        }
    }
    const size_t n = times.size();
    std::vector<double> log_discounts(n), yields(n);
    for (size_t i = 0; i < n; ++i) {
        log_discounts[i] = i == 0 ? 0.0 : -rate * times[i];
        yields[i] = i == 0 ? 0.0 : q_yield * times[i];
    }
    std::vector<uint32_t> div_nodes;
    for (size_t i = 0; i < cash_times.size(); ++i) {
        const int64_t node = find_exact(times, cash_times[i]);
        if (node < 0) {
            Failure f = fail(ORC_MESH_NODE_MISSING);
            f.row = int64_t(first_row);
            return f;
        }
        div_nodes.push_back(uint32_t(node));
    }
    double volatility = q->volatilities[group];
    Plan plan;
    if (q->dividend_model == FO_MODEL_ESCROWED_CASH_DIVIDENDS) {
        if (q->volatility_convention == FO_ESCROWED_SPOT_MATCHED_AT_ORIGIN) {
            double prepaid = 0.0;
            for (size_t i = 0; i < cash_times.size(); ++i) prepaid += cash_amounts[i] * std::exp(-rate * cash_times[i]);
            volatility = volatility * s0 / (s0 - prepaid);
        }
        Failure f = build_escrowed_plan(times, log_discounts, volatility, div_nodes, cash_amounts, exercise,
                                        uint32_t(n - 1), &plan);
        if (!f.ok()) {
            f.row = int64_t(first_row);
            return f;
        }
    } else {
        plan = build_spot_plan(times, log_discounts, yields, volatility, div_nodes, cash_amounts, exercise,
                               uint32_t(n - 1),
                               q->dividend_model == FO_MODEL_CASH_DIVIDENDS ? q->dividend_policy
                                                                            : FO_DIVIDEND_LIQUIDATOR);
    }
    const uint32_t training_domain = uint32_t(q->training_domain_start + group);
    const uint32_t evaluation_domain = uint32_t(q->evaluation_domain_start + group);
    std::vector<double> training;
    Failure f = simulate(plan, s0, q->training_paths, q->training_seed, training_domain, threads, &training);
    if (!f.ok()) {
        f.row = int64_t(first_row);
        return f;
    }
    Spec spec{int(q->polynomial_degree), q->rank_tolerance, q->condition_limit};
    std::vector<Fitted> policies(end_row - first_row);
    for (uint64_t r = first_row; r < end_row; ++r) {
        Estimator est{q->strikes[r], spec, q->tie_rule, q->insufficient_exercise_support};
        f = fit_policy(est, plan, training, q->training_paths, s0, &policies[r - first_row]);
        if (!f.ok()) {
            f.row = int64_t(r);
            return f;
        }
    }
    training.clear();
    training.shrink_to_fit();
    std::vector<double> evaluation;
    f = simulate(plan, s0, q->evaluation_paths, q->evaluation_seed, evaluation_domain, threads, &evaluation);
    if (!f.ok()) {
        f.row = int64_t(first_row);
        return f;
    }
    for (uint64_t r = first_row; r < end_row; ++r) {
        Estimator est{q->strikes[r], spec, q->tie_rule, q->insufficient_exercise_support};
        const Fitted& fitted = policies[r - first_row];
        Evaluation ev;
        f = evaluate(est, plan, fitted, evaluation, q->evaluation_paths, s0, &ev);
        if (!f.ok()) {
            f.row = int64_t(r);
            return f;
        }
        // BatchLsmCallRowResult::try_from_parts (pricing.rs:1130-1230)
        GroupOutput o{};
        o.price = ev.price;
        o.sd = ev.sd;
        o.se = ev.se;
        uint32_t min_itm = UINT32_MAX;
        for (const auto& d : fitted.diagnostics) {
            switch (d.kind) {
                case FO_DIAG_ORIGIN_DECISION:
                    o.origin_fitted = 1;
                    o.origin_exercised = uint8_t(d.exercise);
                    break;
                case FO_DIAG_NO_IN_THE_MONEY_PATHS: o.no_support_nodes += 1; break;
                case FO_DIAG_INSUFFICIENT_SUPPORT: o.insufficient_nodes += 1; break;
                case FO_DIAG_REGRESSION:
                    o.regression_nodes += 1;
                    min_itm = std::min(min_itm, d.in_the_money_paths);
                    o.max_condition = std::max(o.max_condition, d.condition_number);
                    break;
                default: break;
            }
        }
        o.min_itm = o.regression_nodes == 0 ? 0 : min_itm;
        uint64_t early = 0;
        for (size_t i = 0; i + 1 < ev.counts.size(); ++i) early += ev.counts[i];
        o.early = uint32_t(early);
        o.expiry = ev.counts.back();
        outputs[r - first_row] = o;
    }
    return Failure{};
}

}  // namespace

// =============================================================================================
// Exported C entry points (ctypes). Prefix orc_ keeps them apart from the product's fo_ ABI.
// =============================================================================================

extern "C" {

void orc_philox4x32_10(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4]) {
    philox4x32_10(counter, key, out);
}

// k-th normal of each path: out[p * count + k]; returns the oracle code of the first failure.
int orc_sample_normals(uint64_t seed, uint32_t domain, uint32_t path_start, uint64_t paths, uint32_t count,
                       double* out) {
    for (uint64_t p = 0; p < paths; ++p) {
        PathStream stream(seed, domain, uint32_t(path_start + p), count);
        for (uint32_t k = 0; k < count; ++k) {
            const int status = sample_standard_normal(stream, &out[p * count + k]);
            if (status != ORC_OK) return status;
        }
    }
    return ORC_OK;
}

// Exhaust a budget: returns the status of normal number `count + 1` from a stream of budget `count`.
int orc_normal_after_budget(uint64_t seed, uint32_t domain, uint32_t path, uint32_t count) {
    PathStream stream(seed, domain, path, count);
    double v;
    for (uint32_t k = 0; k < count; ++k) sample_standard_normal(stream, &v);
    return sample_standard_normal(stream, &v);
}

void orc_moments(const double* z, const double* y, const double* basis, uint64_t n, double out[3]) {
    moments(z, y, basis, n, out);
}

void orc_recurrence_moments(const double* z, const double* y, const double* previous, const double* current,
                            double* next, uint64_t n, double alpha, double beta, double out[3]) {
    recurrence_moments(z, y, previous, current, next, n, alpha, beta, out);
}

double orc_apply_dividend(int32_t policy, double amount, double spot) { return apply_dividend(policy, amount, spot); }

// Regression fit on explicit columns; model_out = [mean, scale, alphas[4], betas[4], coefficients[5],
// norms[5], rank, condition] (21 doubles). Returns oracle code.
int orc_fit_regression(const double* x, const double* y, uint64_t n, uint32_t degree, double rank_tolerance,
                       double condition_limit, double* model_out, int64_t* aux) {
    std::vector<double> xs(x, x + n), ys(y, y + n);
    Model m;
    Spec spec{int(degree), rank_tolerance, condition_limit};
    Failure f = fit_population(xs, ys, spec, &m);
    if (aux) {
        aux[0] = f.a;
        aux[1] = f.b;
    }
    if (!f.ok()) return f.code;
    model_out[0] = m.mean;
    model_out[1] = m.scale;
    for (int i = 0; i < 4; ++i) model_out[2 + i] = m.alphas[i];
    for (int i = 0; i < 4; ++i) model_out[6 + i] = m.betas[i];
    for (int i = 0; i < 5; ++i) model_out[10 + i] = m.coefficients[i];
    for (int i = 0; i < 5; ++i) model_out[15 + i] = m.norms[i];
    model_out[20] = m.rank;
    model_out[21] = m.condition_number;
    return ORC_OK;
}

// Predictions of a fitted model_out (layout above) at `n` predictors.
int orc_predict(const double* model_in, uint32_t degree, const double* x, uint64_t n, double* out) {
    Model m;
    m.degree = int(degree);
    m.mean = model_in[0];
    m.scale = model_in[1];
    for (int i = 0; i < 4; ++i) m.alphas[i] = model_in[2 + i];
    for (int i = 0; i < 4; ++i) m.betas[i] = model_in[6 + i];
    for (int i = 0; i < 5; ++i) m.coefficients[i] = model_in[10 + i];
    for (uint64_t i = 0; i < n; ++i) {
        if (!predict(m, x[i], &out[i])) return ORC_NON_FINITE_PREDICTION;
    }
    return ORC_OK;
}

static Plan plan_from_gbm(const double* times, uint64_t n_times, const double* log_discounts,
                          const double* cumulative_yields, const uint32_t* dividend_nodes,
                          const double* dividend_amounts, uint64_t n_dividends, const uint32_t* exercise_nodes,
                          uint64_t n_exercise, uint32_t expiry, double volatility, int32_t policy) {
    return build_spot_plan(to_vec(times, n_times), to_vec(log_discounts, n_times), to_vec(cumulative_yields, n_times),
                           volatility, to_vec(dividend_nodes, n_dividends), to_vec(dividend_amounts, n_dividends),
                           to_vec(exercise_nodes, n_exercise), expiry, policy);
}

int orc_simulate_gbm_seeded(const fo_gbm_seeded_request* q, int32_t threads, double* states, uint64_t out_len,
                            fo_error* err) {
    Plan plan = plan_from_gbm(q->schedule_times, q->n_schedule_times, q->log_discounts,
                              q->cumulative_dividend_yields, q->dividend_nodes, q->dividend_amounts,
                              q->n_dividend_nodes, q->exercise_nodes, q->n_exercise_nodes, q->expiry_node,
                              q->annualized_volatility, q->dividend_policy);
    if (out_len != plan.rows() * q->paths) {
        write_error(err, fail(ORC_INVALID_INPUT), FO_ERR_INPUT);
        return FO_ERR_INPUT;
    }
    std::vector<double> tm;
    Failure f = simulate(plan, q->initial_spot, q->paths, q->seed, q->domain, threads, &tm);
    if (!f.ok()) {
        write_error(err, f, FO_ERR_SIMULATION);
        return FO_ERR_SIMULATION;
    }
    std::memcpy(states, tm.data(), tm.size() * sizeof(double));
    return FO_OK;
}

// simulate_gbm_f64 over the oracle: `normals` is [intervals][paths]. Every variate is checked
// before any path is stepped (GbmPathPlan::validate_execution, path.rs:558-603); the first
// non-finite one fails with its interval and path.
int orc_simulate_gbm(const fo_gbm_seeded_request* q, const double* normals, int32_t threads, double* states,
                     uint64_t out_len, fo_error* err) {
    Plan plan = plan_from_gbm(q->schedule_times, q->n_schedule_times, q->log_discounts,
                              q->cumulative_dividend_yields, q->dividend_nodes, q->dividend_amounts,
                              q->n_dividend_nodes, q->exercise_nodes, q->n_exercise_nodes, q->expiry_node,
                              q->annualized_volatility, q->dividend_policy);
    const uint64_t paths = q->paths;
    if (paths == 0 || out_len != plan.rows() * paths) {
        write_error(err, fail(ORC_INVALID_INPUT), FO_ERR_INPUT);
        return FO_ERR_INPUT;
    }
    const uint64_t n = plan.steps.size() * paths;
    for (uint64_t i = 0; i < n; ++i)
        if (!std::isfinite(normals[i])) {
            Failure f = fail(ORC_NON_FINITE_NORMAL_BUFFER);
            f.interval = int64_t(i / paths);
            f.path = int64_t(i % paths);
            f.x = normals[i];
            write_error(err, f, FO_ERR_SIMULATION);
            return FO_ERR_SIMULATION;
        }
    std::vector<double> tm;
    Failure f = simulate(plan, q->initial_spot, paths, 0, 0, threads, &tm, normals);
    if (!f.ok()) {
        write_error(err, f, FO_ERR_SIMULATION);
        return FO_ERR_SIMULATION;
    }
    std::memcpy(states, tm.data(), tm.size() * sizeof(double));
    return FO_OK;
}

// price_lsm_call_seeded_f64 over the oracle. `stage_out` receives the failing stage (1 training
// simulation, 2 fit, 3 evaluation simulation, 4 evaluation, 0 request).
int orc_price_lsm_call(const fo_lsm_call_request* q, int32_t threads, fo_lsm_call_result* result, fo_error* err,
                       int32_t* stage_out) {
    Plan plan = plan_from_gbm(q->schedule_times, q->n_schedule_times, q->log_discounts,
                              q->cumulative_dividend_yields, q->dividend_nodes, q->dividend_amounts,
                              q->n_dividend_nodes, q->exercise_nodes, q->n_exercise_nodes, q->expiry_node,
                              q->annualized_volatility, q->dividend_policy);
    Estimator est{q->strike, Spec{int(q->polynomial_degree), q->rank_tolerance, q->condition_limit}, q->tie_rule,
                  q->insufficient_exercise_support};
    Fitted fitted;
    Evaluation ev;
    int stage = 0;
    Failure f = price_seeded(est, plan, q->initial_spot, q->training_paths, q->evaluation_paths, q->training_seed,
                             q->training_domain, q->evaluation_seed, q->evaluation_domain, threads, &fitted, &ev,
                             &stage);
    if (stage_out) *stage_out = stage;
    if (!f.ok()) {
        write_error(err, f, FO_ERR_LSM);
        return FO_ERR_LSM;
    }
    result->price = ev.price;
    result->paths = ev.paths;
    result->has_sample_standard_deviation = ev.has_sd;
    result->sample_standard_deviation = ev.sd;
    result->has_standard_error = ev.has_sd;
    result->standard_error = ev.se;
    result->n_observations = plan.rows();
    for (size_t r = 0; r < plan.rows() && r < result->observation_capacity; ++r) {
        result->observation_nodes[r] = plan.observation_nodes[r];
        result->exercise_counts[r] = ev.counts[r];
    }
    result->n_diagnostics = fitted.diagnostics.size();
    for (size_t i = 0; i < fitted.diagnostics.size() && i < result->diagnostics_capacity; ++i)
        result->diagnostics[i] = fitted.diagnostics[i];
    return FO_OK;
}

// One contract on a list of markets with common random numbers: the reference's
// bump-and-reprice (two price_lsm_call calls on identical streams, policy.rs:306-336) when
// refit != 0, and the fixed-policy revaluation of FittedLsmCallPolicy::evaluate (policy.rs:642-834)
// when refit == 0 - the policy is fitted once on `base` (training simulation and fit with the base
// market) and every market's evaluation paths are stopped by it, discounted with the market's own
// curve. Every market keeps the base's schedule, nodes, strike, path counts, streams and method;
// its spot, log discounts, cumulative yields, cash amounts and volatility may differ.
// frozen_stops (optional, refit == 0 only, [evaluation_paths]) fixes every path's stopping row
// instead of applying the policy (evaluate_frozen).
// prices[m] receives market m's price; payoffs / stops (optional, [n_markets][evaluation_paths])
// every path's discounted payoff and stopping row. Markets run in parallel over `threads` workers,
// each market's simulations on threads / workers threads; the lowest failing market's failure is
// reported.
int orc_price_lsm_call_markets(const fo_lsm_call_request* base, const fo_lsm_call_request* markets,
                               uint64_t n_markets, int32_t refit, const uint32_t* frozen_stops, int32_t threads,
                               double* prices, double* payoffs, uint32_t* stops, fo_error* err) {
    auto plan_of = [](const fo_lsm_call_request* q) {
        return plan_from_gbm(q->schedule_times, q->n_schedule_times, q->log_discounts, q->cumulative_dividend_yields,
                             q->dividend_nodes, q->dividend_amounts, q->n_dividend_nodes, q->exercise_nodes,
                             q->n_exercise_nodes, q->expiry_node, q->annualized_volatility, q->dividend_policy);
    };
    const Estimator est{base->strike, Spec{int(base->polynomial_degree), base->rank_tolerance, base->condition_limit},
                        base->tie_rule, base->insufficient_exercise_support};
    const uint64_t paths = base->evaluation_paths;
    Fitted base_fit;
    if (!refit) {
        const Plan plan = plan_of(base);
        std::vector<double> training;
        Failure f = simulate(plan, base->initial_spot, base->training_paths, base->training_seed,
                             base->training_domain, threads, &training);
        if (f.ok()) f = fit_policy(est, plan, training, base->training_paths, base->initial_spot, &base_fit);
        if (!f.ok()) {
            write_error(err, f, FO_ERR_LSM);
            return FO_ERR_LSM;
        }
    }
    const int workers = std::max(1, std::min<int>(threads, int(std::min<uint64_t>(n_markets, 256))));
    const int sim_threads = std::max(1, threads / workers);
    std::vector<Failure> failures(n_markets);
    std::atomic<uint64_t> next{0};
    auto worker = [&]() {
        for (uint64_t m = next.fetch_add(1); m < n_markets; m = next.fetch_add(1)) {
            const fo_lsm_call_request* q = markets + m;
            const Plan plan = plan_of(q);
            Fitted fitted;
            Evaluation ev;
            Failure f;
            if (refit) {
                std::vector<double> training;
                f = simulate(plan, q->initial_spot, q->training_paths, q->training_seed, q->training_domain,
                             sim_threads, &training);
                if (f.ok()) f = fit_policy(est, plan, training, q->training_paths, q->initial_spot, &fitted);
            } else {
                fitted.rules = base_fit.rules;
                fitted.diagnostics = base_fit.diagnostics;
                fitted.discount_to_origin.resize(plan.rows());
                for (size_t r = 0; r < plan.rows() && f.ok(); ++r) {
                    if (!checked_discount(plan.log_discounts[plan.observation_nodes[r]], &fitted.discount_to_origin[r])) {
                        f = fail(ORC_UNREPRESENTABLE_DISCOUNT);
                        f.node = plan.observation_nodes[r];
                    }
                }
            }
            std::vector<double> evaluation;
            if (f.ok())
                f = simulate(plan, q->initial_spot, q->evaluation_paths, q->evaluation_seed, q->evaluation_domain,
                             sim_threads, &evaluation);
            double* pay_m = payoffs ? payoffs + m * paths : nullptr;
            uint32_t* stop_m = stops ? stops + m * paths : nullptr;
            if (f.ok() && frozen_stops && !refit)
                f = evaluate_frozen(est, plan, fitted, evaluation, paths, frozen_stops, &ev, pay_m, stop_m);
            else if (f.ok())
                f = evaluate(est, plan, fitted, evaluation, paths, q->initial_spot, &ev, pay_m, stop_m);
            failures[m] = f;
            prices[m] = f.ok() ? ev.price : std::nan("");
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < workers; ++w) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    for (uint64_t m = 0; m < n_markets; ++m) {
        if (!failures[m].ok()) {
            write_error(err, failures[m], FO_ERR_LSM);
            return FO_ERR_LSM;
        }
    }
    return FO_OK;
}

// Grouped batch over the oracle: groups run in parallel over `threads` workers (each group's
// simulation serial), lowest failing group reported (pricing.rs:452-503). With NULL group offsets
// the request is a row batch: group g is contract row g, with domains start + g. Inputs are
// assumed valid; the product library owns request validation.
int orc_price_lsm_grouped(const fo_lsm_grouped_request* q, int32_t threads, fo_batch_result_columns* out,
                          fo_error* err) {
    const uint64_t groups = q->n_initial_spots;
    std::vector<GroupOutput> rows(q->n_strikes);
    std::vector<Failure> failures(groups);
    std::atomic<uint64_t> next{0};
    std::atomic<uint64_t> first_failure{UINT64_MAX};
    auto worker = [&]() {
        for (;;) {
            const uint64_t g = next.fetch_add(1);
            if (g >= groups) return;
            if (g > first_failure.load()) continue;
            // Row batches (no offsets) are groups of one contract (pricing.rs:191-300).
            const uint64_t b = q->group_offsets ? q->group_offsets[g] : g;
            const uint64_t e = q->group_offsets ? q->group_offsets[g + 1] : g + 1;
            Failure f = price_group(q, g, b, e, 1, rows.data() + b);
            if (!f.ok()) {
                failures[g] = f;
                uint64_t cur = first_failure.load();
                while (g < cur && !first_failure.compare_exchange_weak(cur, g)) {}
            }
        }
    };
    const int workers = std::max(1, std::min<int>(threads, int(groups)));
    if (workers == 1) {
        worker();
    } else {
        std::vector<std::thread> pool;
        for (int w = 0; w < workers; ++w) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
    }
    const uint64_t failed = first_failure.load();
    if (failed != UINT64_MAX) {
        Failure f = failures[failed];
        write_error(err, f, FO_ERR_LSM);
        if (err) err->group = int64_t(failed);
        return FO_ERR_LSM;
    }
    for (uint64_t r = 0; r < q->n_strikes; ++r) {
        const GroupOutput& o = rows[r];
        out->prices[r] = o.price;
        out->sample_standard_deviations[r] = o.sd;
        out->standard_errors[r] = o.se;
        out->origin_decisions_fitted[r] = o.origin_fitted;
        out->origin_exercised[r] = o.origin_exercised;
        out->regression_nodes[r] = o.regression_nodes;
        out->no_training_support_nodes[r] = o.no_support_nodes;
        out->insufficient_exercise_support_nodes[r] = o.insufficient_nodes;
        out->minimum_in_the_money_training_paths[r] = o.min_itm;
        out->maximum_regression_condition_numbers[r] = o.max_condition;
        out->early_exercise_paths[r] = o.early;
        out->expiry_paths[r] = o.expiry;
    }
    return FO_OK;
}

// Union meshes for tests: writes up to `capacity` times, returns the count.
uint64_t orc_exact_union_times(double maturity, uint32_t base_intervals, const double* cash, uint64_t n_cash,
                               double* out, uint64_t capacity) {
    auto t = exact_union_times(maturity, base_intervals, cash, n_cash);
    for (size_t i = 0; i < t.size() && i < capacity; ++i) out[i] = t[i];
    return t.size();
}

uint64_t orc_exact_explicit_union_times(double maturity, const double* ex, uint64_t n_ex, const double* cash,
                                        uint64_t n_cash, double* out, uint64_t capacity) {
    auto t = exact_explicit_union_times(maturity, ex, n_ex, cash, n_cash);
    for (size_t i = 0; i < t.size() && i < capacity; ++i) out[i] = t[i];
    return t.size();
}

}  // extern "C"

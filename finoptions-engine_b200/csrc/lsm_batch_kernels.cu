// lsm_batch_kernels.cu - sm_100a kernels of grouped and row-addressed LSM batches
// (crates/finoptions-lsm/src/batch/pricing.rs:505-589 for one group; 191-300 for row batches).
//
//   batch_simulate_kernel   training paths of every group of the wave, one thread per path, stored
//                           time-major per group [rows, paths] with coalesced row stores.
//   batch_backward_kernel   one CTA per (group, strike) problem: backward induction over the
//                           group's stored rows with the problem's values in HBM, one CTA-wide
//                           deterministic reduction of in-the-money power sums per row, the
//                           regression solve by one thread (policy.rs:215-296, 471-601).
//   batch_diagnose_kernel   rank / condition diagnostic of every regression row of every problem
//                           (regression.rs:540-577).
//   batch_evaluate_kernel   re-simulates each group's evaluation paths once and applies the fixed
//                           policies of up to kEvalStrikes strikes on the fly (policy.rs:642-834).
//   batch_summarize_kernel  per problem: price / SE from the evaluation partials, the row-result
//                           columns (pricing.rs:1130-1230) and the first failing backward row.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "lsm_adjoint.cuh"
#include "lsm_batch.cuh"
#include "lsm_batch_kernels.h"
#include "lsm_common.cuh"

namespace fo {

__device__ __forceinline__ bool sim_failed(const unsigned long long* word) {
    return *(const volatile unsigned long long*)word != kNone;
}

// ---------------------------------------------------------------------------------------------
// Training simulation of every group of the wave.
// ---------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(kBatchSimThreads, 6) batch_simulate_kernel(BatchArgs a) {
    __shared__ double sx[257], sf[257];
    load_zig_tables(sx, sf);
    const SmemZig zig = make_zig(sx, sf);
    const BatchGroup& g = a.groups[blockIdx.y];
    const uint64_t P = g.plan.train_paths;
    const uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const DevicePlan plan = g.plan;
    const uint32_t fsr = plan.first_stored_row;
    double* out = a.slab + g.slab_offset;
    const bool escrowed = plan.escrowed != 0;
    auto store = [&](int row, double value) {
        if (uint32_t(row) < fsr) return;
        // Escrowed observations: origin -> S0; otherwise prepaid forward + prepaid cash.
        if (escrowed) value = plan.row_node[row] == 0 ? plan.initial_spot : value + plan.escrow_cash[row];
        out[uint64_t(row - fsr) * P + p] = value;
    };
    const SimResult r = simulate_path(plan, zig, plan.train_seed, plan.train_domain, uint32_t(p), store);
    if (r.code != 0) atomicMin(&a.group_status[blockIdx.y].train_sim_fail, (unsigned long long)p);
}

// ---------------------------------------------------------------------------------------------
// Backward induction, one CTA per problem.
// ---------------------------------------------------------------------------------------------

struct BatchBackwardSmem {
    double red[32 * kSlots];
    dd total[kSlots];
    dd exchange[kSlots];  // this CTA's totals, read by the other CTAs of its cluster
    FitModel model;
    int kind;
};

// Sums slots 0..S-1 of the CTA totals over the CTAs of the cluster in rank order (double-double),
// leaving the same cluster totals in every CTA. Called by every thread after cta_reduce_dd.
template <int S, int C>
__device__ __forceinline__ void cluster_combine(BatchBackwardSmem& sm) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    if (threadIdx.x < S) sm.exchange[threadIdx.x] = sm.total[threadIdx.x];
    cluster.sync();
    if (threadIdx.x < S) {
        dd acc = cluster.map_shared_rank(&sm, 0)->exchange[threadIdx.x];
#pragma unroll
        for (int r = 1; r < C; ++r) acc = dd_add(acc, cluster.map_shared_rank(&sm, r)->exchange[threadIdx.x]);
        sm.total[threadIdx.x] = acc;
    }
    cluster.sync();  // remote reads done before any CTA writes its exchange slots again
}

// kLoads: paths a thread loads together before computing on them (the loads of one batch are
// independent of each other and of the previous batch's stores, so several memory round trips
// overlap). kMinBlocks: resident CTAs per SM the register budget is cut for. kCluster: CTAs that
// share one problem (a thread-block cluster): CTA rank c takes the path blocks c, c + kCluster, ...
// of kLoads x blockDim paths, and the row sums are combined across the cluster through
// distributed shared memory. Problems of up to 64Ki paths run alone in a CTA with two loads at three
// CTAs per SM; larger ones, whose single CTA would be a long tail, in clusters of four with four
// loads at two CTAs per SM.
template <int kLoads, int kMinBlocks, int kCluster, int D>  // D == a.degree
__global__ void __launch_bounds__(kBatchBackwardThreads, kMinBlocks) batch_backward_kernel(BatchArgs a) {
    constexpr int kBackwardBatch = kLoads;
    __shared__ BatchBackwardSmem sm;
    const unsigned rank = kCluster > 1 ? cooperative_groups::this_cluster().block_rank() : 0u;
    // Problems are dispatched largest first (paths x rows), so the longest ones do not start last.
    const uint32_t pi = a.backward_order[blockIdx.x / kCluster];
    const BatchProblem pr = a.problems[pi];
    if (pr.skip_fit) return;
    if (sim_failed(&a.group_status[pr.group].train_sim_fail)) return;
    const BatchGroup& g = a.groups[pr.group];
    const DevicePlan plan = g.plan;
    ProblemStatus* st = a.problem_status + pi;
    FitRecord* records = a.records + pr.records;
    double* __restrict__ values = a.values + pr.values;
    const double* __restrict__ slab = a.slab + g.slab_offset;
    const uint64_t P = plan.train_paths;
    const unsigned T = blockDim.x;
    const uint64_t stride = uint64_t(T) * kBackwardBatch;
    const uint64_t first = uint64_t(rank) * stride + threadIdx.x;  // this thread's first path block
    const uint64_t step = stride * kCluster;
    const double K = pr.strike;
    const Divisor Kd = make_divisor(K);
    const int degree = a.degree;
    const uint32_t E = plan.rows - 1;
    const uint32_t fsr = plan.first_stored_row;
    const int lowest = plan.origin_row ? 1 : 0;
    auto row_ptr = [&](uint32_t row) { return slab + uint64_t(row - fsr) * P; };
    {
        const double* __restrict__ terminal = row_ptr(E);
        for (uint64_t base = first; base < P; base += step) {
            double s[kBackwardBatch];
#pragma unroll
            for (int u = 0; u < kBackwardBatch; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                s[u] = p < P ? __ldg(&terminal[p]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kBackwardBatch; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                const double d = s[u] - K;
                if (p < P) values[p] = d > 0.0 ? d : 0.0;
            }
        }
    }
    uint32_t order = 0;
    int row = int(E) - 1;
    double pivot = 1.0;
    RowSums sums;
#pragma unroll
    for (int k = 0; k < kSlots; ++k) sums.acc[k] = 0.0;
    if (row >= lowest) {
        // Discount into the first fitted row and locate its in-the-money mean (the moment pivot).
        const double disc = plan.disc_from_later[row];
        const double* __restrict__ srow = row_ptr(uint32_t(row));
        double loc[2] = {0.0, 0.0};
        for (uint64_t base = first; base < P; base += step) {
            double v[kBackwardBatch], s[kBackwardBatch];
#pragma unroll
            for (int u = 0; u < kBackwardBatch; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                v[u] = p < P ? values[p] : 0.0;
                s[u] = p < P ? __ldg(&srow[p]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kBackwardBatch; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                if (p >= P) continue;
                v[u] *= disc;
                values[p] = v[u];
                if (!fo_isfinite(v[u])) atomicMin(&st->fit_payoff_fail, ((unsigned long long)order << 32) | p);
                if (s[u] > K) {
                    const double x = divide(s[u], Kd);
                    if (fo_isfinite(x)) {
                        loc[0] += 1.0;
                        loc[1] += x;
                    }
                }
            }
        }
        cta_reduce_dd<2>(loc, sm.red, sm.total);
        if constexpr (kCluster > 1) cluster_combine<2, kCluster>(sm);
        if (sm.total[0].hi > 0.0) pivot = dd_round(dd_div(sm.total[1], sm.total[0]));
        for (uint64_t base = first; base < P; base += step) {
            double v[kBackwardBatch], s[kBackwardBatch];
#pragma unroll
            for (int u = 0; u < kBackwardBatch; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                v[u] = p < P ? values[p] : 0.0;
                s[u] = p < P ? __ldg(&srow[p]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kBackwardBatch; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                if (p >= P || !(s[u] > K)) continue;
                const double x = divide(s[u], Kd);
                if (!fo_isfinite(x) || !fo_isfinite(v[u])) {
                    sums.acc[kBadSlot] += 1.0;
                    atomicMin(&st->fit_nonfinite, ((unsigned long long)order << 32) | p);
                } else {
                    accumulate_itm(sums, x, v[u], pivot);
                }
            }
        }
    }
    for (; row >= lowest; --row, ++order) {
        cta_reduce_dd<kSlots>(sums.acc, sm.red, sm.total);
        if constexpr (kCluster > 1) cluster_combine<kSlots, kCluster>(sm);
        if (threadIdx.x == 0) {
            const uint64_t itm = uint64_t(sm.total[0].hi);
            const uint64_t bad = uint64_t(sm.total[kBadSlot].hi);
            const uint64_t population = itm + bad;
            const uint32_t required = uint32_t(degree + 1);
            int kind;
            if (population == 0) {
                kind = a.support == 1 ? kRuleContinue : kRuleNoSupport;
            } else if (population < required && a.support == 1) {
                kind = kRuleContinue;
            } else if (population < required || bad > 0) {
                kind = kRuleFitFailed;  // InsufficientObservations / non-finite population
            } else {
                fit_continuation(sm.total, pivot, itm, degree, a.rank_tolerance, &sm.model);
                kind = sm.model.status == kFitOk ? kRuleRegression : kRuleFitFailed;
            }
            sm.kind = kind;
            if (rank == 0) {  // every CTA of a cluster fits the same model; one writes the record
                FitRecord& rec = records[row];
                rec.kind = kind;
                rec.itm = population;
                rec.pivot = pivot;
                rec.model = sm.model;
                rec.origin_exercise = 0;
                rec.origin_continuation = 0.0;
                rec.diag_status = -1;
            }
        }
        __syncthreads();
        const int kind = sm.kind;
        if (kind == kRuleFitFailed) return;  // the problem's fit raised; the host reports it
        const bool regression = kind == kRuleRegression;
        if (regression) pivot = sm.model.mean;
        const bool stage_next = row - 1 >= lowest;
        const double disc = stage_next ? plan.disc_from_later[row - 1] : 1.0;
        const double* __restrict__ cur = row_ptr(uint32_t(row));
        const double* __restrict__ nxt = stage_next ? row_ptr(uint32_t(row - 1)) : cur;
#pragma unroll
        for (int k = 0; k < kSlots; ++k) sums.acc[k] = 0.0;
        for (uint64_t base = first; base < P; base += step) {
            double v[kBackwardBatch], sc[kBackwardBatch], sn[kBackwardBatch];
#pragma unroll
            for (int u = 0; u < kBackwardBatch; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                const bool in = p < P;
                v[u] = in ? values[p] : 0.0;
                sc[u] = in && regression ? __ldg(&cur[p]) : 0.0;
                sn[u] = in && stage_next ? __ldg(&nxt[p]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kBackwardBatch; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                if (p >= P) continue;
                if (regression && sc[u] > K) {
                    const double intrinsic = sc[u] - K;
                    double continuation;
                    if (!predict_continuation_d<D>(sm.model, divide(sc[u], Kd), &continuation)) {
                        atomicMin(&st->fit_predict_fail, ((unsigned long long)order << 32) | p);
                    } else if (exercise_rule(a.tie_rule, intrinsic, continuation)) {
                        v[u] = intrinsic;
                    }
                }
                if (stage_next) {
                    v[u] *= disc;
                    if (!fo_isfinite(v[u]))
                        atomicMin(&st->fit_payoff_fail, ((unsigned long long)(order + 1) << 32) | p);
                    if (sn[u] > K) {
                        const double x = divide(sn[u], Kd);
                        if (!fo_isfinite(x) || !fo_isfinite(v[u])) {
                            sums.acc[kBadSlot] += 1.0;
                            atomicMin(&st->fit_nonfinite, ((unsigned long long)(order + 1) << 32) | p);
                        } else {
                            accumulate_itm(sums, x, v[u], pivot);
                        }
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kBackwardBatch; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                if (p < P) values[p] = v[u];
            }
        }
    }
    // Common origin decision (policy.rs:265-281): mean of the values discounted to the origin.
    if (plan.origin_row) {
        double acc[2] = {0.0, 0.0};
        for (uint64_t base = first; base < P; base += step) {
            double v[kBackwardBatch];
#pragma unroll
            for (int u = 0; u < kBackwardBatch; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                v[u] = p < P ? values[p] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kBackwardBatch; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                if (p >= P) continue;
                const double w = v[u] * plan.origin_discount;
                if (!fo_isfinite(w)) atomicMin(&st->fit_payoff_fail, ((unsigned long long)order << 32) | p);
                acc[0] += 1.0;
                acc[1] += w;
            }
        }
        cta_reduce_dd<2>(acc, sm.red, sm.total);
        if constexpr (kCluster > 1) cluster_combine<2, kCluster>(sm);
        if (threadIdx.x == 0 && rank == 0) {
            const double mean = dd_round(dd_div(sm.total[1], sm.total[0]));
            const double intrinsic = plan.initial_spot - K > 0.0 ? plan.initial_spot - K : 0.0;
            FitRecord& rec = records[0];
            rec.kind = kRuleOrigin;
            rec.origin_exercise = exercise_rule(a.tie_rule, intrinsic, mean) ? 1 : 0;
            rec.origin_continuation = mean;
            rec.itm = 0;
            rec.diag_status = -1;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Diagnostics of every regression row.
// ---------------------------------------------------------------------------------------------

__global__ void batch_diagnose_kernel(BatchArgs a, uint32_t n_records) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_records) return;
    FitRecord& rec = a.records[i];
    if (rec.kind != kRuleRegression) return;
    int rank = 0, aux = 0;
    double condition = 0.0;
    rec.diag_status = diagnose_design(rec.model, a.degree, a.rank_tolerance, a.condition_limit, &rank, &condition, &aux);
    rec.diag_rank = rank;
    rec.diag_condition = condition;
    rec.diag_aux = aux;
}

// ---------------------------------------------------------------------------------------------
// Fused evaluation: one evaluation path per thread, up to kEvalStrikes policies applied on the fly.
// ---------------------------------------------------------------------------------------------

// S: strikes per block (1, 2, 4 or 8; the launcher picks the smallest that covers the widest
// group, so row and ragged batches run the one-strike body). kStaged: the group's fitted rules are
// copied into shared memory ([strike][row]) before the paths run; otherwise each lookup reads the
// FitRecord from HBM / L2.
template <int S, bool kStaged, int D>  // D == a.degree
__global__ void __launch_bounds__(kBatchEvalThreads, S <= 1 ? 4 : 3) batch_evaluate_kernel(BatchArgs a, uint32_t rule_rows) {
    __shared__ double sx[257], sf[257];
    __shared__ double red[32 * 2 * S];
    __shared__ dd tot[2 * S];
    __shared__ unsigned cnt[2 * S];
    __shared__ double strikes[S];
    __shared__ double inv_strikes[S];
    __shared__ uint32_t rbase[S];
    __shared__ uint32_t pbase[S];
    extern __shared__ PolicyRule staged[];  // [S][rule_rows] when kStaged
    const BatchGroup& g = a.groups[blockIdx.y];
    const uint32_t first = g.first_problem + blockIdx.z * S;
    const int ns = min(S, int(g.problems) - int(blockIdx.z) * S);
    if (ns <= 0) return;  // uniform over the block
    if (uint64_t(blockIdx.x) * blockDim.x >= g.plan.eval_paths) return;  // beyond this group's paths
    if (sim_failed(&a.group_status[blockIdx.y].train_sim_fail)) return;
    load_zig_tables(sx, sf);
    const SmemZig zig = make_zig(sx, sf);
    if (threadIdx.x < 2 * S) cnt[threadIdx.x] = 0;
    if (threadIdx.x < S) {
        const bool live = int(threadIdx.x) < ns;
        strikes[threadIdx.x] = live ? a.problems[first + threadIdx.x].strike : 1.0;
        inv_strikes[threadIdx.x] = make_divisor(strikes[threadIdx.x]).inv;
        rbase[threadIdx.x] = live ? a.problems[first + threadIdx.x].records : 0u;
        pbase[threadIdx.x] = live ? a.problems[first + threadIdx.x].partial_base : 0u;
    }
    __syncthreads();
    const DevicePlan plan = g.plan;
    const uint32_t rows = plan.rows;
    if (kStaged) {
        for (uint32_t i = threadIdx.x; i < uint32_t(ns) * rows; i += blockDim.x) {
            const uint32_t k = i / rows, r = i % rows;
            const FitRecord& rec = a.records[rbase[k] + r];
            PolicyRule& rule = staged[k * rule_rows + r];
            rule.kind = rec.kind;
            rule.mean = rec.model.mean;
            rule.scale = rec.model.scale;
            rule.inv_scale = rec.model.inv_scale;
#pragma unroll
            for (int j = 0; j < kMaxDegree; ++j) {
                rule.alpha[j] = rec.model.alpha[j];
                rule.beta[j] = rec.model.beta[j];
            }
#pragma unroll
            for (int j = 0; j < kMaxColumns; ++j) rule.coef[j] = rec.model.coef[j];
        }
        __syncthreads();
    }
    const uint64_t P = plan.eval_paths;
    const uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t last = rows - 1;
    double payoff[S];
#pragma unroll
    for (int k = 0; k < S; ++k) payoff[k] = 0.0;
    unsigned active = p < P ? ((1u << ns) - 1u) : 0u;
    auto observe = [&](int row, double spot) {
        if (!active) return;
        if (plan.escrowed) spot = plan.row_node[row] == 0 ? plan.initial_spot : spot + plan.escrow_cash[row];
        const double disc = plan.disc_to_origin[row];
        if (uint32_t(row) == last) {
#pragma unroll
            for (int k = 0; k < S; ++k) {
                if (!((active >> k) & 1u)) continue;
                const double d = spot - strikes[k];
                payoff[k] = (d > 0.0 ? d : 0.0) * disc;
                if (!fo_isfinite(payoff[k])) atomicMin(&a.problem_status[first + k].eval_terminal_fail, (unsigned long long)p);
                atomicAdd(&cnt[2 * k + 1], 1u);
            }
            active = 0u;
            return;
        }
        // Two strikes per iteration: the fully unrolled eight-strike body stalled on instruction fetch.
#pragma unroll 2
        for (int k = 0; k < S; ++k) {
            if (!((active >> k) & 1u)) continue;
            const double K = strikes[k];
            const int kind = kStaged ? staged[k * rule_rows + row].kind : a.records[rbase[k] + row].kind;
            if (kind == kRuleNoSupport) {
                if (spot > K) atomicAdd(&a.itm_counts[rbase[k] + row], 1u);
                continue;
            }
            if (kind != kRuleRegression || !(spot > K)) continue;
            const double intrinsic = spot - K;
            double continuation;
            const bool ok = kStaged ? predict_continuation_d<D>(staged[k * rule_rows + row], divide(spot, Divisor{K, inv_strikes[k]}), &continuation)
                                    : predict_continuation_d<D>(a.records[rbase[k] + row].model, divide(spot, Divisor{K, inv_strikes[k]}), &continuation);
            if (!ok) {
                atomicMin(&a.problem_status[first + k].eval_fail, ((unsigned long long)row << 33) | (p << 1));
                continue;
            }
            if (exercise_rule(a.tie_rule, intrinsic, continuation)) {
                payoff[k] = intrinsic * disc;
                if (!fo_isfinite(payoff[k]))
                    atomicMin(&a.problem_status[first + k].eval_fail, ((unsigned long long)row << 33) | (p << 1) | 1ull);
                active &= ~(1u << k);
                atomicAdd(&cnt[2 * k], 1u);
            }
        }
    };
    if (p < P) {
        const SimResult r = simulate_path(plan, zig, plan.eval_seed, plan.eval_domain, uint32_t(p), observe);
        if (r.code != 0) atomicMin(&a.group_status[blockIdx.y].eval_sim_fail, (unsigned long long)p);
    }
    double acc[2 * S];
#pragma unroll
    for (int k = 0; k < S; ++k) {
        acc[2 * k] = payoff[k];
        acc[2 * k + 1] = payoff[k] * payoff[k];
    }
    cta_reduce_dd<2 * S>(acc, red, tot);
    if (int(threadIdx.x) < 2 * ns) {
        const uint32_t k = threadIdx.x >> 1, which = threadIdx.x & 1u;
        a.eval_partials[(size_t(pbase[k]) + blockIdx.x) * 2 + which] = make_double2(tot[threadIdx.x].hi, tot[threadIdx.x].lo);
        if (cnt[threadIdx.x]) atomicAdd(&a.counts[size_t(first + k) * 2 + which], cnt[threadIdx.x]);
    }
}

// ---------------------------------------------------------------------------------------------
// Fused evaluation with pathwise adjoint Greeks: one strike per block (grid z = strike in group).
// ---------------------------------------------------------------------------------------------

template <int D>  // == a.degree
__global__ void __launch_bounds__(kBatchEvalThreads, 4) batch_evaluate_greeks_kernel(BatchArgs a, uint32_t rule_rows) {
    __shared__ double sx[257], sf[257];
    __shared__ double red[32 * 2];
    __shared__ dd tot[2];
    __shared__ double gred[32 * kGreekSlots];
    __shared__ dd gtot[kGreekSlots];
    __shared__ unsigned cnt[2];
    extern __shared__ __align__(16) unsigned char batch_greeks_smem[];  // PolicyRule[rule_rows], unsigned stops[rule_rows]
    const BatchGroup& g = a.groups[blockIdx.y];
    const uint32_t k = blockIdx.z;
    if (k >= g.problems) return;                                          // uniform over the block
    if (uint64_t(blockIdx.x) * blockDim.x >= g.plan.eval_paths) return;   // beyond this group's paths
    if (sim_failed(&a.group_status[blockIdx.y].train_sim_fail)) return;
    const uint32_t problem = g.first_problem + k;
    const BatchProblem pr = a.problems[problem];
    PolicyRule* rules = reinterpret_cast<PolicyRule*>(batch_greeks_smem);
    unsigned* stops = reinterpret_cast<unsigned*>(rules + rule_rows);
    load_zig_tables(sx, sf);
    const SmemZig zig = make_zig(sx, sf);
    const DevicePlan plan = g.plan;
    const uint32_t rows = plan.rows;
    for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) {
        const FitRecord& rec = a.records[pr.records + r];
        PolicyRule& rule = rules[r];
        rule.kind = rec.kind;
        rule.mean = rec.model.mean;
        rule.scale = rec.model.scale;
            rule.inv_scale = rec.model.inv_scale;
#pragma unroll
        for (int j = 0; j < kMaxDegree; ++j) {
            rule.alpha[j] = rec.model.alpha[j];
            rule.beta[j] = rec.model.beta[j];
        }
#pragma unroll
        for (int j = 0; j < kMaxColumns; ++j) rule.coef[j] = rec.model.coef[j];
        stops[r] = 0;
    }
    if (threadIdx.x < 2) cnt[threadIdx.x] = 0;
    __syncthreads();
    const double K = pr.strike;
    const Divisor Kd = make_divisor(K);
    const uint64_t P = plan.eval_paths;
    const uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t last = rows - 1;
    const double sens_scale = 1.0 / g.sigma;  // (Z diffusion - diffusion^2) / sigma = Z sqrt(dt) - sigma dt
    double payoff = 0.0;
    bool active = p < P;
    GreekSums gs;
    gs.reset();
    PathAdjoint adj;
    adj.reset();
    auto observe = [&](int row, double spot) {
        if (!active) return;
        const double disc = plan.disc_to_origin[row];
        if (uint32_t(row) == last) {
            const double d = spot - K;
            payoff = (d > 0.0 ? d : 0.0) * disc;
            if (!fo_isfinite(payoff)) atomicMin(&a.problem_status[problem].eval_terminal_fail, (unsigned long long)p);
            atomicAdd(&cnt[1], 1u);
            adj.stop(gs, plan.row_node[row], spot, payoff, disc, true, plan.policy, sens_scale);
            active = false;
            return;
        }
        const PolicyRule& rule = rules[row];
        if (rule.kind == kRuleNoSupport) {
            if (spot > K) atomicAdd(&a.itm_counts[pr.records + row], 1u);
            return;
        }
        if (rule.kind != kRuleRegression || !(spot > K)) return;
        const double intrinsic = spot - K;
        double continuation;
        if (!predict_continuation_d<D>(rule, divide(spot, Kd), &continuation)) {
            atomicMin(&a.problem_status[problem].eval_fail, ((unsigned long long)row << 33) | (p << 1));
            return;
        }
        if (exercise_rule(a.tie_rule, intrinsic, continuation)) {
            payoff = intrinsic * disc;
            if (!fo_isfinite(payoff))
                atomicMin(&a.problem_status[problem].eval_fail, ((unsigned long long)row << 33) | (p << 1) | 1ull);
            atomicAdd(&cnt[0], 1u);
            atomicAdd(&stops[row], 1u);
            adj.stop(gs, plan.row_node[row], spot, payoff, disc, false, plan.policy, sens_scale);
            active = false;
        }
    };
    if (p < P) {
        // simulate_path's arithmetic and event phases, with the segment bookkeeping.
        PathStream s;
        s.init(plan.eval_seed, plan.eval_domain, uint32_t(p), plan.intervals);
        double spot = plan.sim_start;
        if (plan.row_node[0] == 0) observe(0, spot);
        bool failed = false;
        for (uint32_t i = 0; i < plan.intervals; ++i) {
            double z = 0.0;
            if (zig_sample(s, zig, &z) != kNormalOk) {
                failed = true;
                break;
            }
            const StepCoef c = plan.steps[i];
            double next = 0.0, growth = 1.0;
            if (spot != 0.0) {
                growth = fo_exp(fo_fma(c.diffusion, z, c.log_drift));
                next = spot * growth;
            }
            if (!fo_isfinite(next)) {
                failed = true;
                break;
            }
            if (active) adj.step(growth, z * c.diffusion - c.diffusion * c.diffusion);
            spot = next;
            const uint32_t at = i + 1;
            const NodeEvent ev = plan.events[at];
            const bool dividend = (ev.flags & kEventDividend) != 0;
            const bool terminal = (ev.flags & kEventTerminal) != 0;
            if (dividend && terminal) {
                const double before = spot;
                spot = apply_cash_dividend(plan.policy, ev.dividend_amount, before);
                if (active) adj.cash(at, before, ev.dividend_amount);
            }
            if (ev.row >= 0) observe(ev.row, spot);
            if (dividend && !terminal) {
                const double before = spot;
                spot = apply_cash_dividend(plan.policy, ev.dividend_amount, before);
                if (active) adj.cash(at, before, ev.dividend_amount);
            }
        }
        if (failed) atomicMin(&a.group_status[blockIdx.y].eval_sim_fail, (unsigned long long)p);
    }
    double acc[2] = {payoff, payoff * payoff};
    cta_reduce_dd<2>(acc, red, tot);
    if (threadIdx.x < 2) {
        a.eval_partials[(size_t(pr.partial_base) + blockIdx.x) * 2 + threadIdx.x] =
            make_double2(tot[threadIdx.x].hi, tot[threadIdx.x].lo);
        if (cnt[threadIdx.x]) atomicAdd(&a.counts[size_t(problem) * 2 + threadIdx.x], cnt[threadIdx.x]);
    }
    for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x)
        if (stops[r]) atomicAdd(&a.stop_counts[pr.records + r], stops[r]);
    double gacc[kGreekSlots];
    gs.to_slots(gacc);
    cta_reduce_dd<kGreekSlots>(gacc, gred, gtot);
    if (threadIdx.x < kGreekSlots)
        a.greek_partials[(size_t(pr.partial_base) + blockIdx.x) * kGreekSlots + threadIdx.x] =
            make_double2(gtot[threadIdx.x].hi, gtot[threadIdx.x].lo);
}

// ---------------------------------------------------------------------------------------------
// Per-problem summary.
// ---------------------------------------------------------------------------------------------

__global__ void batch_summarize_kernel(BatchArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_problems) return;
    const BatchProblem pr = a.problems[i];
    const BatchGroup& g = a.groups[pr.group];
    const uint32_t rows = g.plan.rows;
    const uint32_t E = rows - 1;
    const uint32_t lowest = g.plan.origin_row ? 1u : 0u;
    const FitRecord* rec = a.records + pr.records;
    const ProblemStatus st = a.problem_status[i];
    ProblemSummary s{};
    // First failure of the backward pass in the reference's order: the discount into the row,
    // then its population, regression, diagnostic and update (policy.rs:215-296).
    s.fit_fail_order = 0xffffffffu;
    s.fit_fail_kind = kFitFailNone;
    if (!pr.skip_fit) {
        const uint32_t fitted = E > lowest ? E - lowest : 0u;
        for (uint32_t order = 0; order <= fitted; ++order) {
            const unsigned long long lo = (unsigned long long)order << 32, hi = lo | 0xffffffffull;
            int kind = kFitFailNone;
            if (st.fit_payoff_fail >= lo && st.fit_payoff_fail <= hi) {
                kind = kFitFailPayoff;
            } else if (order < fitted) {
                const FitRecord& r = rec[E - 1 - order];
                if (st.fit_nonfinite >= lo && st.fit_nonfinite <= hi) kind = kFitFailNonFinite;
                else if (r.kind == kRuleFitFailed) kind = kFitFailFit;
                else if (r.kind == kRuleRegression && r.diag_status != kDiagOk) kind = kFitFailDiagnostic;
                else if (st.fit_predict_fail >= lo && st.fit_predict_fail <= hi) kind = kFitFailPredict;
            }
            if (kind != kFitFailNone) {
                s.fit_fail_order = order;
                s.fit_fail_kind = kind;
                break;
            }
        }
    }
    uint32_t min_itm = 0xffffffffu;
    double max_condition = 0.0;
    s.nosupport_row = 0xffffffffu;
    for (uint32_t r = 0; r < E; ++r) {
        switch (rec[r].kind) {
            case kRuleOrigin:
                s.origin_fitted = 1;
                s.origin_exercised = uint32_t(rec[r].origin_exercise);
                break;
            case kRuleNoSupport:
                s.no_support_nodes += 1;
                if (s.nosupport_row == 0xffffffffu && a.itm_counts[pr.records + r] > 0) {
                    s.nosupport_row = r;
                    s.nosupport_count = a.itm_counts[pr.records + r];
                }
                break;
            case kRuleContinue: s.insufficient_nodes += 1; break;
            case kRuleRegression: {
                s.regression_nodes += 1;
                const uint32_t itm = uint32_t(rec[r].itm);
                min_itm = itm < min_itm ? itm : min_itm;
                max_condition = fmax(max_condition, rec[r].diag_condition);
                break;
            }
            default: break;
        }
    }
    s.minimum_itm = s.regression_nodes == 0 ? 0u : min_itm;
    s.maximum_condition = max_condition;
    if (s.origin_exercised) {
        // LsmEvaluation::deterministic (policy.rs:657-669): every path stops at the origin.
        const double d = g.plan.initial_spot - pr.strike;
        s.price = d > 0.0 ? d : 0.0;
        s.sample_standard_deviation = 0.0;
        s.standard_error = 0.0;
        s.early_paths = uint32_t(g.plan.eval_paths);
        s.expiry_paths = 0;
    } else {
        dd sum = dd_make(0.0), sumsq = dd_make(0.0);
        const uint64_t n = g.plan.eval_paths;
        const uint32_t blocks = uint32_t((n + kBatchEvalThreads - 1) / kBatchEvalThreads);
        const double2* part = a.eval_partials + size_t(pr.partial_base) * 2;
        for (uint32_t b = 0; b < blocks; ++b) {
            sum = dd_add(sum, dd{part[2 * b].x, part[2 * b].y});
            sumsq = dd_add(sumsq, dd{part[2 * b + 1].x, part[2 * b + 1].y});
        }
        const dd mean = dd_div(sum, dd_make(double(n)));
        dd m2 = dd_sub(sumsq, dd_mul(sum, mean));
        if (m2.hi < 0.0) m2 = dd_make(0.0);
        s.price = dd_round(mean);
        const double sd = n > 1 ? dd_round(dd_sqrt(dd_div(m2, dd_make(double(n - 1))))) : 0.0;
        s.sample_standard_deviation = sd;
        s.standard_error = n > 1 ? sd / sqrt(double(n)) : 0.0;
        s.early_paths = a.counts[size_t(i) * 2];
        s.expiry_paths = a.counts[size_t(i) * 2 + 1];
        if (a.greek_partials) {
            // Greek slot sums over the problem's blocks in a fixed order.
            const double2* gp = a.greek_partials + size_t(pr.partial_base) * kGreekSlots;
            for (int slot = 0; slot < kGreekSlots; ++slot) {
                dd acc = dd_make(0.0);
                for (uint32_t b = 0; b < blocks; ++b) acc = dd_add(acc, dd{gp[size_t(b) * kGreekSlots + slot].x,
                                                                           gp[size_t(b) * kGreekSlots + slot].y});
                a.greek_sums[size_t(i) * kGreekSlots + slot] = dd_round(acc);
            }
        }
    }
    a.summaries[i] = s;
}

// ---------------------------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------------------------

cudaError_t launch_batch_simulate(const BatchArgs& a, cudaStream_t stream) {
    batch_simulate_kernel<<<dim3(a.train_blocks, a.n_groups), kBatchSimThreads, 0, stream>>>(a);
    return cudaGetLastError();
}

template <int D>
static cudaError_t launch_batch_backward_d(const BatchArgs& a, uint32_t n_large, cudaStream_t stream, cudaStream_t side,
                                          cudaEvent_t fork, cudaEvent_t join) {
    // backward_order lists the problems above 64Ki paths first (clusters of four CTAs), then the
    // rest (one CTA each); the two launches run side by side when a second stream is given.
    constexpr int kCluster = 4;
    const uint32_t n_small = a.n_problems - n_large;
    cudaStream_t small_stream = side ? side : stream;
    if (n_small > 0 && side) {
        cudaError_t e = cudaEventRecord(fork, stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(side, fork, 0);
        if (e != cudaSuccess) return e;
    }
    if (n_large > 0) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(n_large * kCluster);
        cfg.blockDim = dim3(kBatchBackwardThreads);
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kCluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaError_t e = cudaLaunchKernelEx(&cfg, batch_backward_kernel<4, 2, kCluster, D>, a);
        if (e != cudaSuccess) return e;
    }
    if (n_small > 0) {
        BatchArgs s = a;
        s.backward_order = a.backward_order + n_large;
        batch_backward_kernel<2, 3, 1, D><<<n_small, kBatchBackwardThreads, 0, small_stream>>>(s);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (side) {
            e = cudaEventRecord(join, side);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, join, 0);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

cudaError_t launch_batch_backward(const BatchArgs& a, uint32_t n_large, cudaStream_t stream, cudaStream_t side,
                                  cudaEvent_t fork, cudaEvent_t join) {
    switch (a.degree) {  // validated to 0..4 on the host
        case 0: return launch_batch_backward_d<0>(a, n_large, stream, side, fork, join);
        case 1: return launch_batch_backward_d<1>(a, n_large, stream, side, fork, join);
        case 2: return launch_batch_backward_d<2>(a, n_large, stream, side, fork, join);
        case 3: return launch_batch_backward_d<3>(a, n_large, stream, side, fork, join);
        default: return launch_batch_backward_d<4>(a, n_large, stream, side, fork, join);
    }
}

cudaError_t launch_batch_diagnose(const BatchArgs& a, uint32_t n_records, cudaStream_t stream) {
    batch_diagnose_kernel<<<(n_records + 127) / 128, 128, 0, stream>>>(a, n_records);
    return cudaGetLastError();
}

template <int S, int D>
cudaError_t launch_batch_evaluate_width(const BatchArgs& a, uint32_t max_strikes, uint32_t max_rows, cudaStream_t stream) {
    const dim3 grid(a.eval_blocks, a.n_groups, (max_strikes + S - 1) / S);
    const size_t smem = sizeof(PolicyRule) * S * max_rows;
    if (smem <= kEvalRuleSmemBytes) {
        cudaError_t e = cudaFuncSetAttribute(batch_evaluate_kernel<S, true, D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(kEvalRuleSmemBytes));
        if (e != cudaSuccess) return e;
        batch_evaluate_kernel<S, true, D><<<grid, kBatchEvalThreads, smem, stream>>>(a, max_rows);
    } else {
        batch_evaluate_kernel<S, false, D><<<grid, kBatchEvalThreads, 0, stream>>>(a, max_rows);
    }
    return cudaGetLastError();
}

template <int D>
static cudaError_t launch_batch_evaluate_d(const BatchArgs& a, uint32_t max_strikes, uint32_t max_rows,
                                           cudaStream_t stream) {
    if (max_strikes <= 1) return launch_batch_evaluate_width<1, D>(a, max_strikes, max_rows, stream);
    if (max_strikes <= 2) return launch_batch_evaluate_width<2, D>(a, max_strikes, max_rows, stream);
    if (max_strikes <= 4) return launch_batch_evaluate_width<4, D>(a, max_strikes, max_rows, stream);
    return launch_batch_evaluate_width<kEvalStrikes, D>(a, max_strikes, max_rows, stream);
}

cudaError_t launch_batch_evaluate(const BatchArgs& a, uint32_t max_strikes, uint32_t max_rows, cudaStream_t stream) {
    switch (a.degree) {  // validated to 0..4 on the host
        case 0: return launch_batch_evaluate_d<0>(a, max_strikes, max_rows, stream);
        case 1: return launch_batch_evaluate_d<1>(a, max_strikes, max_rows, stream);
        case 2: return launch_batch_evaluate_d<2>(a, max_strikes, max_rows, stream);
        case 3: return launch_batch_evaluate_d<3>(a, max_strikes, max_rows, stream);
        default: return launch_batch_evaluate_d<4>(a, max_strikes, max_rows, stream);
    }
}

template <int D>
static cudaError_t launch_batch_evaluate_greeks_d(const BatchArgs& a, uint32_t max_strikes, uint32_t max_rows,
                                                  cudaStream_t stream) {
    const dim3 grid(a.eval_blocks, a.n_groups, max_strikes);
    const size_t smem = (sizeof(PolicyRule) + sizeof(unsigned)) * max_rows;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(batch_evaluate_greeks_kernel<D>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    batch_evaluate_greeks_kernel<D><<<grid, kBatchEvalThreads, smem, stream>>>(a, max_rows);
    return cudaGetLastError();
}

cudaError_t launch_batch_evaluate_greeks(const BatchArgs& a, uint32_t max_strikes, uint32_t max_rows,
                                         cudaStream_t stream) {
    switch (a.degree) {  // validated to 0..4 on the host
        case 0: return launch_batch_evaluate_greeks_d<0>(a, max_strikes, max_rows, stream);
        case 1: return launch_batch_evaluate_greeks_d<1>(a, max_strikes, max_rows, stream);
        case 2: return launch_batch_evaluate_greeks_d<2>(a, max_strikes, max_rows, stream);
        case 3: return launch_batch_evaluate_greeks_d<3>(a, max_strikes, max_rows, stream);
        default: return launch_batch_evaluate_greeks_d<4>(a, max_strikes, max_rows, stream);
    }
}

cudaError_t launch_batch_summarize(const BatchArgs& a, cudaStream_t stream) {
    batch_summarize_kernel<<<(a.n_problems + 127) / 128, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace fo

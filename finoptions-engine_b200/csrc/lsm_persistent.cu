// lsm_persistent.cu - grouped, row-addressed and ragged LSM batches as one persistent launch per
// wave (crates/finoptions-lsm/src/batch/pricing.rs:452-589 for the work of one group).
//
// A wave's work is a queue of items (lsm_batch.cuh): the training simulation of a group's path
// blocks, the backward fit of one (group, strike) problem, the evaluation of a group's path blocks
// for a chunk of its strikes. The host orders it topologically and largest work first: every
// group's simulation, then every problem's fit (largest training paths x rows first), then the
// evaluations in the order their groups' fits were queued. Resident CTAs take items from the queue
// in order; a fit waits until its group's training paths are stored, an evaluation until its
// group's fits are done, each wait bounded in time. The CTA that finishes a group's last
// evaluation item writes that group's summaries, so the launch ends with every result written.
//
// Work items run the same arithmetic, in the same order, as pricing a group alone: a problem's fit
// is one CTA over its paths in a fixed thread-to-path assignment, and evaluation partials are
// kept per 256-path block. The results therefore do not depend on the queue order, the paths per
// item or the grid size the autotuner picks.
//
// Data written by one CTA and read by another inside the launch (stored paths, fitted records,
// partials, status words) is read through L2 (ld.global.cg): L1 is not coherent across SMs.
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "lsm_adjoint.cuh"
#include "lsm_batch.cuh"
#include "lsm_batch_kernels.h"
#include "lsm_common.cuh"
#include "lsm_fit_warp.cuh"
#include "lsm_sync.cuh"

namespace fo {

namespace {

constexpr int kPersistentThreads = 256;
constexpr int kPersistentLoads = 2;  // paths a backward thread loads together
// The fit kernel of the phase executor runs four CTAs per SM (64 registers a thread): a thread loads
// one path at a time and reads the row's model from shared memory per path. Resident warps hide the
// latency better there than paths in flight per thread (measured on the grouped batch).
constexpr int kFitKernelLoads = 1;
// A dependency wait gives up after this long: one problem's fit on one CTA can take seconds for
// populations of millions of paths, so the limit is well above any fit's duration.
constexpr unsigned long long kDependencyTimeoutNs = 20000000000ull;

__device__ __forceinline__ unsigned long long ld_l2_u64(const unsigned long long* p) { return __ldcg(p); }

__device__ __forceinline__ bool status_failed(const unsigned long long* word) { return ld_l2_u64(word) != kNone; }

// Thread 0 waits (time-bounded) until *counter reaches target; every thread returns whether it did.
// The pause between polls doubles from 64 ns up to max_pause: dependency waits keep their polls of
// L2 rare, a team's per-row exchange polls often.
__device__ bool wait_for(const unsigned* counter, unsigned target, unsigned* timeout, int* flag,
                         unsigned max_pause = 4096) {
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned pause = 64;
        unsigned long long start = 0;
        while (ld_relaxed_gpu(counter) < target) {
            if (ld_volatile_u32(timeout) != 0) {
                ok = 0;
                break;
            }
            const unsigned long long now = global_timer_ns();
            if (start == 0) {
                start = now;
            } else if (now - start > kDependencyTimeoutNs) {
                atomicExch(timeout, 1u);
                ok = 0;
                break;
            }
            __nanosleep(pause);
            pause = pause < max_pause ? 2 * pause : pause;
        }
        __threadfence();  // acquire: the items counted are visible to this CTA's reads below
        *flag = ok;
    }
    __syncthreads();
    return *flag != 0;
}

// Every thread's writes of the item are made visible device-wide, then thread 0 adds n.
// Returns (in thread 0) the counter's value before the addition.
__device__ __forceinline__ unsigned signal_done(unsigned* counter, unsigned n) {
    __threadfence();
    __syncthreads();
    unsigned before = 0;
    if (threadIdx.x == 0) before = atomicAdd(counter, n);
    return before;
}

// The part of a fitted record the evaluation reads: the model's first sixteen doubles are mean,
// scale, inv_scale, alpha[4], beta[4], coef[5] - PolicyRule's layout. The record is 16-byte aligned
// (16-byte loads); a staged PolicyRule only 8-byte aligned (8-byte stores). Records written by other
// CTAs of the same launch are read through L2; kReadOnly (a later kernel) may use the read-only path.
template <bool kReadOnly = false>
__device__ __forceinline__ void load_rule(const FitRecord& rec, PolicyRule* out) {
    static_assert(offsetof(FitModel, mean) == 0 && offsetof(FitModel, coef) + sizeof(double) * kMaxColumns == 128,
                  "FitModel starts with the sixteen doubles of a PolicyRule");
    static_assert(offsetof(PolicyRule, coef) + sizeof(double) * kMaxColumns == 128, "PolicyRule layout");
    static_assert(alignof(FitRecord) >= 16, "records load as 16-byte words");
    const double2* src = reinterpret_cast<const double2*>(&rec.model);
    double* dst = reinterpret_cast<double*>(out);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const double2 v = kReadOnly ? __ldg(src + i) : __ldcg(src + i);
        dst[2 * i] = v.x;
        dst[2 * i + 1] = v.y;
    }
    out->kind = kReadOnly ? __ldg(&rec.kind) : __ldcg(&rec.kind);
}

__device__ __forceinline__ uint32_t blocks_of(uint64_t paths) {
    return uint32_t((paths + kPersistentThreads - 1) / kPersistentThreads);
}

// ---- training simulation ------------------------------------------------------------------------

__device__ void simulate_item(const BatchArgs& a, uint32_t gi, uint32_t first, uint32_t count, const SmemZig& zig) {
    const BatchGroup& g = a.groups[gi];
    const DevicePlan plan = g.plan;  // a local copy: its fields stay in registers (no reloads across stores)
    const uint64_t P = plan.train_paths;
    const uint32_t fsr = plan.first_stored_row;
    double* out = a.slab + g.slab_offset;
    const bool escrowed = plan.escrowed != 0;
    for (uint32_t b = first; b < first + count; ++b) {
        const uint64_t p = uint64_t(b) * kPersistentThreads + threadIdx.x;
        if (p >= P) continue;
        auto store = [&](int row, double value) {
            if (uint32_t(row) < fsr) return;
            // Escrowed observations: origin -> S0; otherwise prepaid forward + prepaid cash.
            if (escrowed) value = plan.row_node[row] == 0 ? plan.initial_spot : value + plan.escrow_cash[row];
            out[uint64_t(row - fsr) * P + p] = value;
        };
        const SimResult r = simulate_path(plan, zig, plan.train_seed, plan.train_domain, uint32_t(p), store);
        if (r.code != 0) atomicMin(&a.group_status[gi].train_sim_fail, (unsigned long long)p);
    }
}

// ---- backward fit of one problem ----------------------------------------------------------------

// The CTAs that fit one problem together. Member m owns the contiguous paths [lo, hi).
struct Team {
    uint32_t member, members;
    double2* slots;    // [2][members][kSlots]
    unsigned* arrive;  // arrivals at this problem's exchanges
    unsigned round;    // exchanges this member has made
    unsigned* timeout;
    int* flag;
};

// Every member publishes its CTA totals of a reduction (S double-double slots) and sums all members'
// in member order, so each member ends with the same totals. Consecutive exchanges alternate between
// two buffers: a member overwrites one only after every member has arrived at the exchange in
// between, that is, has finished reading it. False when a wait gave up (the timeout flag is set).
static_assert(kTeamSlots == kSlots, "a member's exchange holds one row reduction");

template <int S, bool kTeam>
__device__ bool team_exchange(Team& t, dd* total /* shared [S] */) {
    if constexpr (!kTeam) return true;
    if (t.members == 1) return true;
    const unsigned parity = t.round & 1u;
    if (threadIdx.x < S)
        t.slots[(size_t(parity) * t.members + t.member) * kSlots + threadIdx.x] =
            make_double2(total[threadIdx.x].hi, total[threadIdx.x].lo);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(t.arrive, 1u);
    t.round += 1;
    if (!wait_for(t.arrive, t.members * t.round, t.timeout, t.flag, 256)) return false;
    if (threadIdx.x < S) {
        const double2* column = t.slots + size_t(parity) * t.members * kSlots + threadIdx.x;
        dd acc = dd_make(0.0);
        for (uint32_t m = 0; m < t.members; ++m) {
            const double2 v = __ldcg(column + size_t(m) * kSlots);
            acc = dd_add(acc, dd{v.x, v.y});
        }
        total[threadIdx.x] = acc;
    }
    __syncthreads();
    return true;
}

struct BackwardItemSmem {
    double red[32 * kSlots];
    dd total[kSlots];
    FitModel model;
    double new_pivot;  // the row's own mean, when its sums are taken again about it
    int kind;
    int recenter;
};

// Backward induction of one problem over the group's stored rows with the problem's values in HBM
// (policy.rs:215-296, 471-601): per row one deterministic reduction of in-the-money power sums and
// the regression solve by one warp. A problem of up to kTeamPaths paths is one CTA's; a larger one
// is split over a team of CTAs (this one is member `member` of `members`), each owning a contiguous
// range of paths, whose CTA sums are exchanged in member order before every decision, so that every
// member fits the same model; member 0 writes the records. Thread t owns paths lo + t + m * 256
// (m = 0, 1, ...), loading kPersistentLoads of them together (kFitKernelLoads in the fit kernel).
// The order of a thread's paths, and so every sum, does not depend on that count. False when a team
// exchange gave up.
// A stored training state. The persistent launch reads rows that other CTAs of the same launch wrote,
// so through L2 (the SM's L1 is not coherent with other SMs' writes); the fit kernel of the phase
// executor runs after the simulation kernel has finished, so its reads may use the read-only path.
template <bool kReadOnly>
__device__ __forceinline__ double load_slab(const double* p) {
    if constexpr (kReadOnly) return __ldg(p);
    else return __ldcg(p);
}

template <int D, bool kReadOnlySlab, bool kTeam>
__device__ bool backward_item(const BatchArgs& a, uint32_t pi, uint32_t member, uint32_t members, unsigned* timeout,
                              int* flag, BackwardItemSmem& sm) {
    constexpr int kL = kReadOnlySlab ? kFitKernelLoads : kPersistentLoads;
    const BatchProblem pr = a.problems[pi];
    if (pr.skip_fit) return true;
    if (status_failed(&a.group_status[pr.group].train_sim_fail)) return true;
    const BatchGroup& g = a.groups[pr.group];
    const DevicePlan plan = g.plan;  // a local copy: its fields stay in registers (no reloads across stores)
    ProblemStatus* st = a.problem_status + pi;
    FitRecord* records = a.records + pr.records;
    // Restrict-qualified: this problem's values are its own, and the slab is only read here, so the
    // loads of several paths may be issued together, ahead of the stores.
    double* __restrict__ values = a.values + pr.values;
    const double* __restrict__ slab = a.slab + g.slab_offset;
    const uint64_t P = plan.train_paths;
    const unsigned T = blockDim.x;
    const uint64_t step = uint64_t(T) * kL;
    // This member's paths [lo, hi): contiguous ranges of a multiple of 256 paths, in member order.
    const uint64_t span = members == 1 ? P : ((P + members - 1) / members + 255) / 256 * 256;
    const uint64_t lo = members == 1 ? 0 : (uint64_t(member) * span < P ? uint64_t(member) * span : P);
    const uint64_t hi = members == 1 ? P : (lo + span < P ? lo + span : P);
    const uint64_t first = lo + threadIdx.x;
    Team team{member, members, a.team_slots + pr.team_base, a.team_arrive + pi, 0u, timeout, flag};
    const bool writer = member == 0;
    const double K = pr.strike;
    const Divisor Kd = make_divisor(K);
    const int degree = a.degree;
    const uint32_t E = plan.rows - 1;
    const uint32_t fsr = plan.first_stored_row;
    const int lowest = plan.origin_row ? 1 : 0;
    auto row_ptr = [&](uint32_t row) { return slab + uint64_t(row - fsr) * P; };
    {
        const double* terminal = row_ptr(E);
        for (uint64_t base = first; base < hi; base += step) {
            double s[kL];
#pragma unroll
            for (int u = 0; u < kL; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                s[u] = p < hi ? load_slab<kReadOnlySlab>(&terminal[p]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kL; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                const double d = s[u] - K;
                if (p < hi) values[p] = d > 0.0 ? d : 0.0;
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
        const double* srow = row_ptr(uint32_t(row));
        double loc[2] = {0.0, 0.0};
        for (uint64_t base = first; base < hi; base += step) {
            double v[kL], s[kL];
#pragma unroll
            for (int u = 0; u < kL; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                v[u] = p < hi ? values[p] : 0.0;
                s[u] = p < hi ? load_slab<kReadOnlySlab>(&srow[p]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kL; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                if (p >= hi) continue;
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
        if (!team_exchange<2, kTeam>(team, sm.total)) return false;
        if (sm.total[0].hi > 0.0) pivot = dd_round(dd_div(sm.total[1], sm.total[0]));
        for (uint64_t base = first; base < hi; base += step) {
            double v[kL], s[kL];
#pragma unroll
            for (int u = 0; u < kL; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                v[u] = p < hi ? values[p] : 0.0;
                s[u] = p < hi ? load_slab<kReadOnlySlab>(&srow[p]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kL; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                if (p >= hi || !(s[u] > K)) continue;
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
        if (!team_exchange<kSlots, kTeam>(team, sm.total)) return false;
        if (threadIdx.x == 0) {
            const uint64_t itm = uint64_t(sm.total[0].hi);
            double mean = pivot;
            sm.recenter = degree > 0 && itm >= uint64_t(degree + 1) && sm.total[kBadSlot].hi == 0.0 &&
                                  pivot_too_far(sm.total, pivot, itm, &mean)
                              ? 1
                              : 0;
            sm.new_pivot = mean;
        }
        __syncthreads();
        if (sm.recenter) {
            // The pivot lay more than a standard deviation from the row's in-the-money mean: take
            // the row's sums again about that mean (values[] holds the row's discounted values).
            pivot = sm.new_pivot;
            const double* cur = row_ptr(uint32_t(row));
#pragma unroll
            for (int k = 0; k < kSlots; ++k) sums.acc[k] = 0.0;
            for (uint64_t base = first; base < hi; base += step) {
                double v[kL], s[kL];
#pragma unroll
                for (int u = 0; u < kL; ++u) {
                    const uint64_t p = base + uint64_t(u) * T;
                    v[u] = p < hi ? values[p] : 0.0;
                    s[u] = p < hi ? load_slab<kReadOnlySlab>(&cur[p]) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < kL; ++u) {
                    const uint64_t p = base + uint64_t(u) * T;
                    if (p >= hi || !(s[u] > K)) continue;
                    const double x = divide(s[u], Kd);
                    if (!fo_isfinite(x) || !fo_isfinite(v[u])) sums.acc[kBadSlot] += 1.0;
                    else accumulate_itm(sums, x, v[u], pivot);
                }
            }
            cta_reduce_dd<kSlots>(sums.acc, sm.red, sm.total);
            if (!team_exchange<kSlots, kTeam>(team, sm.total)) return false;
        }
        if (threadIdx.x < 32) {
            // Warp 0 decides the row and fits it (the lane-parallel solve, bit-identical to the
            // one-thread one), then writes the row's record, the model as 16-byte words by lanes.
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
                fit_continuation_warp(sm.total, pivot, itm, degree, a.rank_tolerance, plan.rank_limit, &sm.model);
                kind = sm.model.status == kFitOk ? kRuleRegression : kRuleFitFailed;
            }
            FitRecord& rec = records[row];
            constexpr int kModelWords = int(sizeof(FitModel) / sizeof(double2));
            static_assert(sizeof(FitModel) % sizeof(double2) == 0, "FitModel is 16-byte aligned");
            if (writer && threadIdx.x < kModelWords)
                reinterpret_cast<double2*>(&rec.model)[threadIdx.x] =
                    reinterpret_cast<const double2*>(&sm.model)[threadIdx.x];
            if (threadIdx.x == 0) sm.kind = kind;
            if (writer && threadIdx.x == 0) {
                rec.kind = kind;
                rec.itm = population;
                rec.pivot = pivot;
                rec.origin_exercise = 0;
                rec.origin_continuation = 0.0;
                rec.diag_status = -1;
            }
        }
        __syncthreads();
        const int kind = sm.kind;
        if (kind == kRuleFitFailed) return true;  // the problem's fit raised; the host reports it
        const bool regression = kind == kRuleRegression;
        if (regression) pivot = sm.model.mean;
        const bool stage_next = row - 1 >= lowest;
        const double disc = stage_next ? plan.disc_from_later[row - 1] : 1.0;
        const double* cur = row_ptr(uint32_t(row));
        const double* nxt = stage_next ? row_ptr(uint32_t(row - 1)) : cur;
#pragma unroll
        for (int k = 0; k < kSlots; ++k) sums.acc[k] = 0.0;
        // The fit kernel fetches the next step's value and spots before the current step's
        // arithmetic, so their latency overlaps it (one path per thread and step); the persistent
        // launch, at two paths per step and the heaviest kind's register budget, fetches in place.
        constexpr bool kAhead = kReadOnlySlab;
        double fv[kL], fsc[kL], fsn[kL];
        auto fetch = [&](uint64_t at) {
#pragma unroll
            for (int u = 0; u < kL; ++u) {
                const uint64_t p = at + uint64_t(u) * T;
                const bool in = p < hi;
                fv[u] = in ? values[p] : 0.0;
                fsc[u] = in && regression ? load_slab<kReadOnlySlab>(&cur[p]) : 0.0;
                fsn[u] = in && stage_next ? load_slab<kReadOnlySlab>(&nxt[p]) : 0.0;
            }
        };
        if constexpr (kAhead) fetch(first);
        for (uint64_t base = first; base < hi; base += step) {
            if constexpr (!kAhead) fetch(base);
            double v[kL], sc[kL], sn[kL];
#pragma unroll
            for (int u = 0; u < kL; ++u) {
                v[u] = fv[u];
                sc[u] = fsc[u];
                sn[u] = fsn[u];
            }
            if constexpr (kAhead) fetch(base + step);
#pragma unroll
            for (int u = 0; u < kL; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                if (p >= hi) continue;
                if (regression && sc[u] > K) {
                    const double intrinsic = sc[u] - K;
                    double continuation;
                    if (!predict_continuation_shared<D>(&sm.model, divide(sc[u], Kd), &continuation)) {
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
            for (int u = 0; u < kL; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                if (p < hi) values[p] = v[u];
            }
        }
    }
    // Common origin decision (policy.rs:265-281): mean of the values discounted to the origin.
    if (plan.origin_row) {
        double acc[2] = {0.0, 0.0};
        for (uint64_t base = first; base < hi; base += step) {
            double v[kL];
#pragma unroll
            for (int u = 0; u < kL; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                v[u] = p < hi ? values[p] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kL; ++u) {
                const uint64_t p = base + uint64_t(u) * T;
                if (p >= hi) continue;
                const double w = v[u] * plan.origin_discount;
                if (!fo_isfinite(w)) atomicMin(&st->fit_payoff_fail, ((unsigned long long)order << 32) | p);
                acc[0] += 1.0;
                acc[1] += w;
            }
        }
        cta_reduce_dd<2>(acc, sm.red, sm.total);
        if (!team_exchange<2, kTeam>(team, sm.total)) return false;
        if (writer && threadIdx.x == 0) {
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
    return true;
}

// Rank / condition diagnostic of every regression row of problem pi (regression.rs:540-577); the
// records were written by this CTA.
__device__ void diagnose_problem(const BatchArgs& a, uint32_t pi) {
    const BatchProblem pr = a.problems[pi];
    const uint32_t rows = a.groups[pr.group].plan.rows;
    for (uint32_t r = threadIdx.x; r + 1 < rows; r += blockDim.x) {
        FitRecord& rec = a.records[pr.records + r];
        if (rec.kind != kRuleRegression) continue;
        int rank = 0, aux = 0;
        double condition = 0.0;
        rec.diag_status = diagnose_design(rec.model, a.degree, a.rank_tolerance, a.condition_limit, &rank, &condition,
                                          &aux);
        rec.diag_rank = rank;
        rec.diag_condition = condition;
        rec.diag_aux = aux;
    }
}

// ---- evaluation -----------------------------------------------------------------------------------

// CTA sums of S (payoff, squared payoff) pairs as double-double totals: every pair is summed across
// its warp by the same two-value transpose whatever S is, then over the warps in a fixed order, so a
// strike's block totals do not depend on how many strikes an item evaluates together.
template <int S>
__device__ void cta_reduce_pairs(double (&acc)[2 * S], double* red /* [32 * 2S] */, dd* out /* [2S] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < S; ++k) {
        double pair[2] = {acc[2 * k], acc[2 * k + 1]};
        const double total = warp_transpose_reduce<2>(pair);
        if (lane < 2) red[warp * 2 * S + 2 * k + lane] = total;
    }
    __syncthreads();
    for (int slot = warp; slot < 2 * S; slot += warps) {
        dd v = dd_make(lane < warps ? red[lane * 2 * S + slot] : 0.0);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = dd_add(v, shfl_dd_down(v, off));
        if (lane == 0) out[slot] = v;
    }
    __syncthreads();
}

// Shared memory of one evaluation item: S strikes evaluated together by every thread.
template <int S>
struct EvalSmem {
    double red[32 * 2 * S];
    dd tot[2 * S];
    unsigned cnt[2 * S];
    double strikes[S];
    double inv_strikes[S];
    uint32_t rbase[S];
    uint32_t pbase[S];
    uint32_t problem[S];
};

// Evaluation blocks [first, first + count) of group gi for strike chunk z: each thread
// re-simulates one evaluation path per block and applies up to S fitted policies on the fly
// (policy.rs:642-834); per (problem, block) double-double partials and stopping counts.
// kStaged: the rules were staged in shared memory (read there with shared-memory loads); otherwise
// each lookup reads the FitRecord through L2.
template <int S, int D, bool kStaged, bool kReadOnly>
__device__ void evaluate_item(const BatchArgs& a, uint32_t gi, uint32_t first, uint32_t count, uint32_t z,
                              const SmemZig& zig, EvalSmem<S>& sm, PolicyRule* staged, uint32_t rule_rows) {
    const BatchGroup& g = a.groups[gi];
    const uint32_t p0 = g.first_problem + z * S;
    const int ns = min(S, int(g.problems) - int(z) * S);
    if (ns <= 0 || status_failed(&a.group_status[gi].train_sim_fail)) return;  // uniform over the CTA
    const DevicePlan plan = g.plan;  // a local copy: its fields stay in registers (no reloads across stores)
    const uint32_t rows = plan.rows;
    if (threadIdx.x < S) {
        const bool live = int(threadIdx.x) < ns;
        const BatchProblem pr = a.problems[live ? p0 + threadIdx.x : p0];
        sm.strikes[threadIdx.x] = live ? pr.strike : 1.0;
        sm.inv_strikes[threadIdx.x] = make_divisor(sm.strikes[threadIdx.x]).inv;
        sm.rbase[threadIdx.x] = live ? pr.records : 0u;
        sm.pbase[threadIdx.x] = live ? pr.partial_base : 0u;
        sm.problem[threadIdx.x] = live ? p0 + threadIdx.x : p0;
    }
    __syncthreads();
    if constexpr (kStaged) {
        for (uint32_t i = threadIdx.x; i < uint32_t(ns) * rows; i += blockDim.x) {
            const uint32_t k = i / rows, r = i % rows;
            load_rule<kReadOnly>(a.records[sm.rbase[k] + r], &staged[k * rule_rows + r]);
        }
        __syncthreads();
    }
    const uint64_t P = plan.eval_paths;
    const uint32_t last = rows - 1;
    for (uint32_t b = first; b < first + count; ++b) {
        if (threadIdx.x < 2 * S) sm.cnt[threadIdx.x] = 0;
        __syncthreads();
        const uint64_t p = uint64_t(b) * kPersistentThreads + threadIdx.x;
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
                    const double d = spot - sm.strikes[k];
                    payoff[k] = (d > 0.0 ? d : 0.0) * disc;
                    if (!fo_isfinite(payoff[k]))
                        atomicMin(&a.problem_status[sm.problem[k]].eval_terminal_fail, (unsigned long long)p);
                    atomicAdd(&sm.cnt[2 * k + 1], 1u);
                }
                active = 0u;
                return;
            }
            // Four strikes per unrolled step (measured on the grouped batch: 185 ms for the
            // evaluation phase against 194 unrolled by two, 209 by one and 204 fully).
#pragma unroll 4
            for (int k = 0; k < S; ++k) {
                if (!((active >> k) & 1u)) continue;
                const double K = sm.strikes[k];
                PolicyRule loaded;
                if constexpr (!kStaged) load_rule<kReadOnly>(a.records[sm.rbase[k] + row], &loaded);
                const PolicyRule& rule = kStaged ? staged[k * rule_rows + row] : loaded;
                if (rule.kind == kRuleNoSupport) {
                    if (spot > K) atomicAdd(&a.itm_counts[sm.rbase[k] + row], 1u);
                    continue;
                }
                if (rule.kind != kRuleRegression || !(spot > K)) continue;
                const double intrinsic = spot - K;
                double continuation;
                if (!predict_continuation_d<D>(rule, divide(spot, Divisor{K, sm.inv_strikes[k]}), &continuation)) {
                    atomicMin(&a.problem_status[sm.problem[k]].eval_fail, ((unsigned long long)row << 33) | (p << 1));
                    continue;
                }
                if (exercise_rule(a.tie_rule, intrinsic, continuation)) {
                    payoff[k] = intrinsic * disc;
                    if (!fo_isfinite(payoff[k]))
                        atomicMin(&a.problem_status[sm.problem[k]].eval_fail,
                                  ((unsigned long long)row << 33) | (p << 1) | 1ull);
                    active &= ~(1u << k);
                    atomicAdd(&sm.cnt[2 * k], 1u);
                }
            }
        };
        if (p < P) {
            const SimResult r = simulate_path(plan, zig, plan.eval_seed, plan.eval_domain, uint32_t(p), observe);
            if (r.code != 0) atomicMin(&a.group_status[gi].eval_sim_fail, (unsigned long long)p);
        }
        double acc[2 * S];
#pragma unroll
        for (int k = 0; k < S; ++k) {
            acc[2 * k] = payoff[k];
            acc[2 * k + 1] = payoff[k] * payoff[k];
        }
        cta_reduce_pairs<S>(acc, sm.red, sm.tot);
        if (int(threadIdx.x) < 2 * ns) {
            const uint32_t k = threadIdx.x >> 1, which = threadIdx.x & 1u;
            a.eval_partials[(size_t(sm.pbase[k]) + b) * 2 + which] = make_double2(sm.tot[threadIdx.x].hi,
                                                                                  sm.tot[threadIdx.x].lo);
            if (sm.cnt[threadIdx.x]) atomicAdd(&a.counts[size_t(sm.problem[k]) * 2 + which], sm.cnt[threadIdx.x]);
        }
    }
}

struct GreeksEvalSmem {
    double red[32 * 2];
    dd tot[2];
    double gred[32 * kGreekSlots];
    dd gtot[kGreekSlots];
    unsigned cnt[2];
};

// The adjoint variant: evaluation blocks [first, first + count) of group gi for its strike k alone,
// with the pathwise Greeks (lsm_adjoint.cuh) summed per block in double-double.
template <int D, bool kReadOnly>
__device__ void evaluate_greeks_item(const BatchArgs& a, uint32_t gi, uint32_t first, uint32_t count, uint32_t k,
                                     const SmemZig& zig, GreeksEvalSmem& sm, PolicyRule* rules, unsigned* stops) {
    const BatchGroup& g = a.groups[gi];
    if (k >= g.problems || status_failed(&a.group_status[gi].train_sim_fail)) return;  // uniform over the CTA
    const uint32_t problem = g.first_problem + k;
    const BatchProblem pr = a.problems[problem];
    const DevicePlan plan = g.plan;  // a local copy: its fields stay in registers (no reloads across stores)
    const uint32_t rows = plan.rows;
    for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) load_rule<kReadOnly>(a.records[pr.records + r], &rules[r]);
    const double K = pr.strike;
    const Divisor Kd = make_divisor(K);
    const uint64_t P = plan.eval_paths;
    const uint32_t last = rows - 1;
    const double sens_scale = 1.0 / g.sigma;  // (Z diffusion - diffusion^2) / sigma = Z sqrt(dt) - sigma dt
    for (uint32_t b = first; b < first + count; ++b) {
        for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) stops[r] = 0;
        if (threadIdx.x < 2) sm.cnt[threadIdx.x] = 0;
        __syncthreads();
        const uint64_t p = uint64_t(b) * kPersistentThreads + threadIdx.x;
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
                atomicAdd(&sm.cnt[1], 1u);
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
                atomicAdd(&sm.cnt[0], 1u);
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
                double zn = 0.0;
                if (zig_sample(s, zig, &zn) != kNormalOk) {
                    failed = true;
                    break;
                }
                const StepCoef c = plan.steps[i];
                double next = 0.0, growth = 1.0;
                if (spot != 0.0) {
                    growth = fo_exp(fo_fma(c.diffusion, zn, c.log_drift));
                    next = spot * growth;
                }
                if (!fo_isfinite(next)) {
                    failed = true;
                    break;
                }
                if (active) adj.step(growth, zn * c.diffusion - c.diffusion * c.diffusion);
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
            if (failed) atomicMin(&a.group_status[gi].eval_sim_fail, (unsigned long long)p);
        }
        double acc[2] = {payoff, payoff * payoff};
        cta_reduce_pairs<1>(acc, sm.red, sm.tot);
        if (threadIdx.x < 2) {
            a.eval_partials[(size_t(pr.partial_base) + b) * 2 + threadIdx.x] =
                make_double2(sm.tot[threadIdx.x].hi, sm.tot[threadIdx.x].lo);
            if (sm.cnt[threadIdx.x]) atomicAdd(&a.counts[size_t(problem) * 2 + threadIdx.x], sm.cnt[threadIdx.x]);
        }
        for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x)
            if (stops[r]) atomicAdd(&a.stop_counts[pr.records + r], stops[r]);
        double gacc[kGreekSlots];
        gs.to_slots(gacc);
        cta_reduce_dd<kGreekSlots>(gacc, sm.gred, sm.gtot);
        if (threadIdx.x < kGreekSlots)
            a.greek_partials[(size_t(pr.partial_base) + b) * kGreekSlots + threadIdx.x] =
                make_double2(sm.gtot[threadIdx.x].hi, sm.gtot[threadIdx.x].lo);
    }
}

// ---- per-problem summary ----------------------------------------------------------------------------

// The summary of problem i (its twelve result columns, try_from_parts pricing.rs:1130-1230, and its
// first failing backward row), written by one warp once its group's evaluation is complete: lanes
// 0 / 1 sum the price partials over the blocks in block order, with the Greeks lane s sums Greek
// slot s the same way, and lane 0 scans the records.
__device__ void summarize_problem(const BatchArgs& a, uint32_t i, int lane) {
    const BatchProblem pr = a.problems[i];
    const BatchGroup& g = a.groups[pr.group];
    const uint64_t n = g.plan.eval_paths;
    const uint32_t blocks = blocks_of(n);
    const double2* part = a.eval_partials + size_t(pr.partial_base) * 2;
    // Price partial sums: lane 0 the payoffs, lane 1 their squares, each in block order.
    dd slot_sum = dd_make(0.0);
    if (lane < 2)
        for (uint32_t b = 0; b < blocks; ++b) {
            const double2 v = __ldcg(&part[2 * b + lane]);
            slot_sum = dd_add(slot_sum, dd{v.x, v.y});
        }
    dd sum, sumsq;
    sum.hi = __shfl_sync(0xffffffffu, slot_sum.hi, 0);
    sum.lo = __shfl_sync(0xffffffffu, slot_sum.lo, 0);
    sumsq.hi = __shfl_sync(0xffffffffu, slot_sum.hi, 1);
    sumsq.lo = __shfl_sync(0xffffffffu, slot_sum.lo, 1);
    if (a.greek_partials && lane < kGreekSlots) {
        const double2* gp = a.greek_partials + size_t(pr.partial_base) * kGreekSlots;
        dd acc = dd_make(0.0);
        for (uint32_t b = 0; b < blocks; ++b) {
            const double2 v = __ldcg(&gp[size_t(b) * kGreekSlots + lane]);
            acc = dd_add(acc, dd{v.x, v.y});
        }
        a.greek_sums[size_t(i) * kGreekSlots + lane] = dd_round(acc);
    }
    if (lane != 0) return;
    const uint32_t rows = g.plan.rows;
    const uint32_t E = rows - 1;
    const uint32_t lowest = g.plan.origin_row ? 1u : 0u;
    const FitRecord* rec = a.records + pr.records;
    ProblemStatus st;
    st.fit_payoff_fail = ld_l2_u64(&a.problem_status[i].fit_payoff_fail);
    st.fit_predict_fail = ld_l2_u64(&a.problem_status[i].fit_predict_fail);
    st.fit_nonfinite = ld_l2_u64(&a.problem_status[i].fit_nonfinite);
    st.eval_fail = ld_l2_u64(&a.problem_status[i].eval_fail);
    st.eval_terminal_fail = ld_l2_u64(&a.problem_status[i].eval_terminal_fail);
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
                const int rkind = __ldcg(&r.kind);
                if (st.fit_nonfinite >= lo && st.fit_nonfinite <= hi) kind = kFitFailNonFinite;
                else if (rkind == kRuleFitFailed) kind = kFitFailFit;
                else if (rkind == kRuleRegression && __ldcg(&r.diag_status) != kDiagOk) kind = kFitFailDiagnostic;
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
        const int kind = __ldcg(&rec[r].kind);
        switch (kind) {
            case kRuleOrigin:
                s.origin_fitted = 1;
                s.origin_exercised = uint32_t(__ldcg(&rec[r].origin_exercise));
                break;
            case kRuleNoSupport: {
                s.no_support_nodes += 1;
                const unsigned itm = __ldcg(&a.itm_counts[pr.records + r]);
                if (s.nosupport_row == 0xffffffffu && itm > 0) {
                    s.nosupport_row = r;
                    s.nosupport_count = itm;
                }
                break;
            }
            case kRuleContinue: s.insufficient_nodes += 1; break;
            case kRuleRegression: {
                s.regression_nodes += 1;
                const uint32_t itm = uint32_t(__ldcg(reinterpret_cast<const unsigned long long*>(&rec[r].itm)));
                min_itm = itm < min_itm ? itm : min_itm;
                max_condition = fmax(max_condition, __ldcg(&rec[r].diag_condition));
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
        s.early_paths = uint32_t(n);
        s.expiry_paths = 0;
    } else {
        const dd mean = dd_div(sum, dd_make(double(n)));
        dd m2 = dd_sub(sumsq, dd_mul(sum, mean));
        if (m2.hi < 0.0) m2 = dd_make(0.0);
        s.price = dd_round(mean);
        const double sd = n > 1 ? dd_round(dd_sqrt(dd_div(m2, dd_make(double(n - 1))))) : 0.0;
        s.sample_standard_deviation = sd;
        s.standard_error = n > 1 ? sd / sqrt(double(n)) : 0.0;
        s.early_paths = __ldcg(&a.counts[size_t(i) * 2]);
        s.expiry_paths = __ldcg(&a.counts[size_t(i) * 2 + 1]);
    }
    a.summaries[i] = s;
}

}  // namespace

// ---- the persistent kernel ------------------------------------------------------------------------

// Executors of the work items. kPhaseAll is the persistent launch: one kernel drains the whole queue,
// items of every kind waiting on the counters. The other phases run the items of one kind as a
// queue-draining kernel of their own, launched in stream order (simulation, fits, evaluation), so
// that each kind gets the register budget and CTAs per SM that suit it; their dependency waits are
// then already met. Both run the same item functions, so they give the same results, bit for bit.
enum BatchPhase : int { kPhaseAll = 0, kPhaseSimulate = 1, kPhaseFit = 2, kPhaseEvaluate = 3 };

// Shared memory of the items a kernel runs: all kinds for the persistent launch, one kind each for
// the phase kernels (less static shared memory leaves more of the SM's L1).
template <int S>
union AllItemsSmem {
    BackwardItemSmem bwd;
    EvalSmem<S> eval;
    GreeksEvalSmem greeks;
};
struct NoItemSmem {};
struct FitItemSmem {
    BackwardItemSmem bwd;
};
template <int S>
struct EvalItemSmem {
    EvalSmem<S> eval;
};
struct GreeksItemSmem {
    GreeksEvalSmem greeks;
};
template <int kPhase, int S, bool kGreeks>
struct PhaseSmem {
    using type = AllItemsSmem<S>;
};
template <int S, bool kGreeks>
struct PhaseSmem<1, S, kGreeks> {
    using type = NoItemSmem;
};
template <int S, bool kGreeks>
struct PhaseSmem<2, S, kGreeks> {
    using type = FitItemSmem;
};
template <int S>
struct PhaseSmem<3, S, false> {
    using type = EvalItemSmem<S>;
};
template <int S>
struct PhaseSmem<3, S, true> {
    using type = GreeksItemSmem;
};

template <int kPhase, int S, bool kGreeks>
struct PhaseOccupancy {
    // Resident CTAs per SM the register budget is cut for.
    static constexpr int value = kPhase == kPhaseSimulate                              ? 6
                                 : kPhase == kPhaseFit                                   ? 4
                                 : kPhase == kPhaseEvaluate && (S == 1 || kGreeks)       ? 4
                                                                                         : 3;
};

// S: strikes an evaluation item applies together (kGreeks: one, with the adjoint). The dynamic
// shared memory holds the staged rules (S x rule_rows PolicyRules, plus per-row stopping counts with
// the Greeks) when stage_rules is set.
template <int kPhase, int S, bool kGreeks, int D>
__global__ void __launch_bounds__(kPersistentThreads, (PhaseOccupancy<kPhase, S, kGreeks>::value))
    batch_persistent_kernel(BatchArgs a, BatchQueue q, uint32_t rule_rows, int stage_rules) {
    constexpr bool kSim = kPhase == kPhaseAll || kPhase == kPhaseSimulate;
    constexpr bool kFit = kPhase == kPhaseAll || kPhase == kPhaseFit;
    constexpr bool kEval = kPhase == kPhaseAll || kPhase == kPhaseEvaluate;
    __shared__ double sx[257], sf[257];
    __shared__ BatchItem item;
    __shared__ int flag;
    __shared__ typename PhaseSmem<kPhase, S, kGreeks>::type sm;
    extern __shared__ __align__(16) unsigned char persistent_dyn[];
    PolicyRule* staged = reinterpret_cast<PolicyRule*>(persistent_dyn);
    if constexpr (kSim || kEval) load_zig_tables(sx, sf);
    const SmemZig zig = make_zig(sx, sf);
    for (;;) {
        __syncthreads();  // the previous item is done with the shared memory
        if (threadIdx.x == 0) {
            const unsigned i = atomicAdd(q.next, 1u);
            if (i < q.n_items) {
                item = q.items[i];
            } else {
                item.kind = kItemNone;
            }
        }
        __syncthreads();
        const BatchItem it = item;
        if (it.kind == kItemNone) return;
        if (it.kind == kItemSimulate) {
            if constexpr (kSim) {
                simulate_item(a, it.index, it.first, it.count, zig);
                signal_done(&q.sim_done[it.index], it.count);
            }
        } else if (it.kind == kItemBackward) {
            if constexpr (kFit) {
                const uint32_t gi = a.problems[it.index].group;
                const uint32_t sim_blocks = blocks_of(a.groups[gi].plan.train_paths);
                // The fit kernel runs after the simulation kernel: its dependencies are met.
                if (kPhase == kPhaseFit || wait_for(&q.sim_done[gi], sim_blocks, q.timeout, &flag)) {
                    // Lone CTAs run a copy of the fit without the team exchanges (fewer live registers).
                    const bool done =
                        it.count == 1
                            ? backward_item<D, kPhase == kPhaseFit, false>(a, it.index, 0, 1, q.timeout, &flag, sm.bwd)
                            : backward_item<D, kPhase == kPhaseFit, true>(a, it.index, it.first, it.count, q.timeout,
                                                                          &flag, sm.bwd);
                    __syncthreads();
                    if (done && it.first == 0) diagnose_problem(a, it.index);  // member 0 wrote the records
                }
                signal_done(&q.bwd_done[gi], 1u);
            }
        } else if constexpr (kEval) {
            const uint32_t gi = it.index;
            const BatchGroup& g = a.groups[gi];
            if (kPhase == kPhaseEvaluate || wait_for(&q.bwd_done[gi], g.fit_items, q.timeout, &flag)) {
                if constexpr (kGreeks) {
                    unsigned* stops = reinterpret_cast<unsigned*>(staged + rule_rows);
                    evaluate_greeks_item<D, kPhase == kPhaseEvaluate>(a, gi, it.first, it.count, it.chunk, zig,
                                                                      sm.greeks, staged, stops);
                } else {
                    constexpr bool kRO = kPhase == kPhaseEvaluate;
                    if (stage_rules)
                        evaluate_item<S, D, true, kRO>(a, gi, it.first, it.count, it.chunk, zig, sm.eval, staged,
                                                       rule_rows);
                    else
                        evaluate_item<S, D, false, kRO>(a, gi, it.first, it.count, it.chunk, zig, sm.eval, staged,
                                                        rule_rows);
                }
            }
            // The item that completes the group's evaluation writes the group's summaries (in the
            // phase executor a summary kernel follows the evaluation kernel instead).
            if constexpr (kPhase == kPhaseEvaluate) continue;
            const uint32_t chunks = kGreeks ? g.problems : (g.problems + S - 1) / S;
            const unsigned units = blocks_of(g.plan.eval_paths) * chunks;
            const unsigned before = signal_done(&q.eval_done[gi], it.count);
            if (threadIdx.x == 0) flag = before + it.count == units;
            __syncthreads();
            if (flag) {
                __threadfence();
                const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
                for (uint32_t k = warp; k < g.problems; k += blockDim.x >> 5)
                    summarize_problem(a, g.first_problem + k, lane);
            }
        }
    }
}

// The phase executor's last kernel: every problem's summary, one warp per problem, once every
// evaluation partial is written (the evaluation kernel has finished).
__global__ void __launch_bounds__(kPersistentThreads) batch_summarize_kernel(BatchArgs a, BatchQueue, uint32_t, int) {
    const uint32_t warps = kPersistentThreads / 32;
    const uint32_t i = blockIdx.x * warps + (threadIdx.x >> 5);
    if (i < a.n_problems) summarize_problem(a, i, int(threadIdx.x & 31));
}

// ---- launcher ---------------------------------------------------------------------------------------

size_t persistent_rule_bytes(int strikes, bool greeks, uint32_t rule_rows) {
    return greeks ? (sizeof(PolicyRule) + sizeof(unsigned)) * rule_rows : sizeof(PolicyRule) * size_t(strikes) * rule_rows;
}

template <int kPhase, int S, bool kGreeks, int D>
static cudaError_t prepare_persistent_d(const BatchQueue& q, uint32_t rule_rows, bool stage, int ctas_per_sm,
                                        PersistentLaunch* out) {
    auto kernel = batch_persistent_kernel<kPhase, S, kGreeks, D>;
    const bool rules = stage && (kPhase == kPhaseAll || kPhase == kPhaseEvaluate);
    const size_t smem = rules ? persistent_rule_bytes(S, kGreeks, rule_rows) : 0;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPersistentThreads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int device = 0, sms = 0;
    e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    const int cap = kPhase == kPhaseAll && ctas_per_sm > 0 && ctas_per_sm < per_sm ? ctas_per_sm : per_sm;
    const int resident = cap * sms;
    out->kernel = reinterpret_cast<const void*>(kernel);
    out->grid = int(q.n_items) < resident ? int(q.n_items) : resident;
    out->smem = smem;
    return cudaSuccess;
}

template <int kPhase, int S, bool kGreeks>
static cudaError_t prepare_persistent_s(int degree, const BatchQueue& q, uint32_t rule_rows, bool stage,
                                        int ctas_per_sm, PersistentLaunch* out) {
    switch (degree) {  // validated to 0..4 on the host
        case 0: return prepare_persistent_d<kPhase, S, kGreeks, 0>(q, rule_rows, stage, ctas_per_sm, out);
        case 1: return prepare_persistent_d<kPhase, S, kGreeks, 1>(q, rule_rows, stage, ctas_per_sm, out);
        case 2: return prepare_persistent_d<kPhase, S, kGreeks, 2>(q, rule_rows, stage, ctas_per_sm, out);
        case 3: return prepare_persistent_d<kPhase, S, kGreeks, 3>(q, rule_rows, stage, ctas_per_sm, out);
        default: return prepare_persistent_d<kPhase, S, kGreeks, 4>(q, rule_rows, stage, ctas_per_sm, out);
    }
}

template <int kPhase>
static cudaError_t prepare_phase(const BatchArgs& a, const BatchQueue& q, int strikes, uint32_t rule_rows, bool stage,
                                 int ctas_per_sm, PersistentLaunch* out) {
    *out = PersistentLaunch{};
    if (a.greek_partials)
        return prepare_persistent_s<kPhase, 1, true>(a.degree, q, rule_rows, stage, ctas_per_sm, out);
    if constexpr (kPhase == kPhaseSimulate || kPhase == kPhaseFit) {
        // No evaluation code: one instance serves every evaluation width.
        return prepare_persistent_s<kPhase, 1, false>(a.degree, q, rule_rows, stage, ctas_per_sm, out);
    } else {
        switch (strikes) {
            case 1: return prepare_persistent_s<kPhase, 1, false>(a.degree, q, rule_rows, stage, ctas_per_sm, out);
            case 2: return prepare_persistent_s<kPhase, 2, false>(a.degree, q, rule_rows, stage, ctas_per_sm, out);
            case 4: return prepare_persistent_s<kPhase, 4, false>(a.degree, q, rule_rows, stage, ctas_per_sm, out);
            default:
                return prepare_persistent_s<kPhase, kEvalStrikes, false>(a.degree, q, rule_rows, stage, ctas_per_sm,
                                                                         out);
        }
    }
}

cudaError_t prepare_batch_persistent(const BatchArgs& a, const BatchQueue& q, int strikes, uint32_t rule_rows,
                                     bool stage, int ctas_per_sm, PersistentLaunch* out) {
    return prepare_phase<kPhaseAll>(a, q, strikes, rule_rows, stage, ctas_per_sm, out);
}

cudaError_t prepare_batch_phases(const BatchArgs& a, const BatchQueue (&q)[3], int strikes, uint32_t rule_rows,
                                 bool stage, PersistentLaunch (&out)[4]) {
    cudaError_t e = prepare_phase<kPhaseSimulate>(a, q[0], strikes, rule_rows, stage, 0, &out[0]);
    if (e == cudaSuccess) e = prepare_phase<kPhaseFit>(a, q[1], strikes, rule_rows, stage, 0, &out[1]);
    if (e == cudaSuccess) e = prepare_phase<kPhaseEvaluate>(a, q[2], strikes, rule_rows, stage, 0, &out[2]);
    const uint32_t warps = kPersistentThreads / 32;
    out[3] = PersistentLaunch{reinterpret_cast<const void*>(batch_summarize_kernel), 0,
                              int((a.n_problems + warps - 1) / warps), 0};
    return e;
}

cudaError_t enqueue_batch_persistent(const PersistentLaunch& launch, const BatchArgs& a, const BatchQueue& q,
                                     uint32_t rule_rows, bool stage, cudaStream_t stream) {
    if (launch.grid <= 0) return cudaSuccess;
    BatchArgs args = a;
    BatchQueue queue = q;
    uint32_t rows = rule_rows;
    int stage_rules = stage ? 1 : 0;
    void* params[4] = {&args, &queue, &rows, &stage_rules};
    return cudaLaunchKernel(launch.kernel, dim3(unsigned(launch.grid)), dim3(kPersistentThreads), params, launch.smem,
                            stream);
}

}  // namespace fo

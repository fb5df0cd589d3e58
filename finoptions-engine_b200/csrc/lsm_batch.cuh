// lsm_batch.cuh - device layout of grouped and row-addressed LSM batches
// (crates/finoptions-lsm/src/batch/pricing.rs:422-589, 191-300).
//
// A batch is a list of groups; a group owns one training and one evaluation path population
// (one simulation plan, one random domain per role) shared by its strike rows. Each (group,
// strike) pair is a "problem": its own backward policy fit over the group's stored training rows
// and its own fixed-policy evaluation on the group's evaluation paths. A row-addressed batch is
// the special case of one strike per group.
#pragma once

#include <stdint.h>

#include "lsm_device.cuh"

namespace fo {

// One group of the launched wave. `plan` points into the batch input block; its strike field is
// unused (strikes live on the problems).
struct BatchGroup {
    DevicePlan plan;
    uint64_t slab_offset;    // first element of the group's stored training rows in the wave slab
    uint32_t first_problem;  // wave-local index of the group's first strike problem
    uint32_t problems;       // strike rows in the group
    double sigma;            // the plan's constant volatility (adjoint vega)
    uint32_t fit_items;      // backward work items of the group (team members summed over its problems)
    uint32_t pad;
};

// One (group, strike) problem of the launched wave.
struct BatchProblem {
    double strike;
    uint32_t group;          // wave-local group index
    uint32_t records;        // index of its first FitRecord (one per observation row)
    uint64_t values;         // first element of its training values (train_paths doubles)
    int32_t skip_fit;        // 1: the host already failed this problem's fit (no backward pass)
    uint32_t partial_base;   // first of its evaluation blocks' partial slots (one per block)
    uint32_t members;        // CTAs that fit it together (1: one CTA)
    uint32_t team_base;      // first of its team's exchange slots (2 x members x kTeamSlots double2)
};

// Training paths one member of a team fits: problems with more are split over several CTAs, whose
// CTA sums are exchanged once per row (at most kMaxTeam members; the queue holds them in a row).
constexpr uint64_t kTeamPaths = 32768;
constexpr uint32_t kMaxTeam = 64;
constexpr int kTeamSlots = 16;  // double2 slots of one member's exchange (the row reduction's sums)

// Failure keys; every word starts as all-ones ("none") and keeps the lowest key with atomicMin.
struct GroupStatus {
    unsigned long long train_sim_fail;  // lowest failing training path
    unsigned long long eval_sim_fail;   // lowest failing evaluation path
};

struct ProblemStatus {
    unsigned long long fit_payoff_fail;     // (order << 32) | path: non-finite discounted value
    unsigned long long fit_predict_fail;    // (order << 32) | path: non-finite prediction
    unsigned long long fit_nonfinite;       // (order << 32) | path: non-finite ITM predictor/response
    unsigned long long eval_fail;           // (row << 33) | (path << 1) | type (0 predict, 1 payoff)
    unsigned long long eval_terminal_fail;  // path: non-finite terminal payoff
};

// Per-problem outputs: the twelve result columns (BatchLsmCallRowResult::try_from_parts,
// pricing.rs:1130-1230) and what the host needs to report the problem's first failure.
struct ProblemSummary {
    double price;
    double sample_standard_deviation;
    double standard_error;
    double maximum_condition;
    uint32_t regression_nodes;
    uint32_t no_support_nodes;
    uint32_t insufficient_nodes;
    uint32_t minimum_itm;
    uint32_t early_paths;
    uint32_t expiry_paths;
    uint32_t origin_fitted;
    uint32_t origin_exercised;
    uint32_t fit_fail_order;   // first failing backward order (all-ones: none)
    int32_t fit_fail_kind;     // kFitFail*
    uint32_t nosupport_row;    // first unsupported row reached by in-the-money evaluation paths
    uint32_t nosupport_count;  // those paths
};

enum FitFailKind : int32_t {
    kFitFailNone = 0,
    kFitFailPayoff = 1,     // non-finite discounted value (order = row being staged)
    kFitFailNonFinite = 2,  // non-finite in-the-money predictor or response
    kFitFailFit = 3,        // the regression itself failed (FitRecord.model.status / population)
    kFitFailDiagnostic = 4, // rank / condition diagnostic failed
    kFitFailPredict = 5,    // non-finite continuation prediction in the update
};

// Strikes evaluated together by one evaluation thread (groups with more run several passes).
constexpr int kEvalStrikes = 8;

// The part of a fitted row the evaluation reads, staged in shared memory per (strike, row).
struct PolicyRule {
    double mean, scale, inv_scale;
    double alpha[kMaxDegree];
    double beta[kMaxDegree];
    double coef[kMaxColumns];
    int32_t kind;
    int32_t pad;
};

// Shared memory the evaluation may spend on staged rules; larger groups read them from HBM.
constexpr size_t kEvalRuleSmemBytes = 96 * 1024;

// ---- persistent launch ------------------------------------------------------------------------
// One launch prices a whole wave: its CTAs take work items from a queue in order until it is empty.
// The queue is topologically ordered (every item depends only on items before it), so every item a
// CTA waits on has already been taken by a running CTA, and the waits end.
enum BatchItemKind : uint32_t {
    kItemNone = 0,
    kItemSimulate = 1,  // training paths of blocks [first, first + count) of group `index`
    kItemBackward = 2,  // backward fit of problem `index` by team member `first` of `count`
    kItemEvaluate = 3,  // evaluation blocks [first, first + count) of group `index`, strike chunk `chunk`
};

struct BatchItem {
    uint32_t kind;
    uint32_t index;
    uint32_t first;
    uint32_t count;
    uint32_t chunk;
    uint32_t pad[3];
};

// Dependency counters of one launch, all zeroed before it: a group's backward items wait until
// sim_done[g] reaches its training blocks, its evaluation items until bwd_done[g] reaches its
// fit items; the item that brings eval_done[g] to the group's evaluation units writes the group's
// summaries. A wait gives up after a time limit and raises *timeout (no item ever waits forever).
// The members of a team are consecutive items and wait only on each other and on earlier items,
// and a team has at most kMaxTeam members (fewer than the launch's CTAs), so its waits end too.
struct BatchQueue {
    const BatchItem* items;
    uint32_t n_items;
    unsigned* next;
    unsigned* sim_done;
    unsigned* bwd_done;
    unsigned* eval_done;
    unsigned* timeout;
};

struct BatchArgs {
    const BatchGroup* groups;
    const BatchProblem* problems;
    uint32_t n_groups;
    uint32_t n_problems;
    double* slab;
    double* values;
    FitRecord* records;
    GroupStatus* group_status;
    ProblemStatus* problem_status;
    unsigned* counts;          // [problems * 2]: early, expiry
    unsigned* itm_counts;      // [records]: in-the-money evaluation paths at unsupported rows
    double2* eval_partials;    // [evaluation blocks of all problems][2]: (sum, sum of squares), double-double
    ProblemSummary* summaries; // [problems]
    // Adjoint Greeks (ragged batches): per-block slot partials, per-problem slot sums, per-record
    // stopping counts. greek_partials is NULL when the batch prices without Greeks.
    double2* greek_partials;   // [evaluation blocks of all problems][kGreekSlots]
    double* greek_sums;        // [problems][kGreekSlots]
    unsigned* stop_counts;     // [records]
    double2* team_slots;       // exchange slots of the teams (BatchProblem::team_base)
    unsigned* team_arrive;     // [problems]: arrivals at the team's exchanges
    uint32_t train_blocks;     // training-simulation blocks of the largest group (grid x)
    uint32_t eval_blocks;      // evaluation blocks of the largest group (grid x, partials stride)
    int32_t degree;
    double rank_tolerance;
    double condition_limit;
    int32_t tie_rule;
    int32_t support;
};

}  // namespace fo

// capi.cu - the C ABI (include/finoptions_cuda.h): executor, device arena, single-contract plans
// and the simulation exports. Host orchestration of LsmCallEstimator::price_seeded
// (crates/finoptions-lsm/src/policy.rs:306-336) over the kernels in lsm_kernels.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/finoptions_cuda.h"
#include "executor.h"
#include "host.h"
#include "lsm_kernels.h"

#ifndef FO_PACKAGE_VERSION
#define FO_PACKAGE_VERSION "0.1.0"
#endif

using namespace fo;

namespace {

constexpr unsigned long long kNone = ~0ull;

}  // namespace

// Layout of a plan's device block. Everything the host reads back is contiguous at `out`.
struct PlanLayout {
    size_t steps, events, row_node, disc_from_later, disc_to_origin, escrow_cash;  // inputs
    size_t sqrt_dt, dt;       // per-interval sqrt(dt) and dt for the adjoint vega
    size_t greek_partials;    // eval_blocks * kGreekSlots double2
    size_t greek_out;         // kGreekSlots doubles (read back)
    size_t partials;          // backward partials: 2 * blocks * 16 double2
    size_t eval_partials;     // eval partials: eval_blocks * 2 double2
    size_t out;               // start of the read-back region
    size_t status, result, records, counts, itm_counts, replay;
    size_t out_bytes;
    size_t total;
    size_t inputs_bytes;
};

struct fo_lsm_call_plan {
    fo_executor* ex = nullptr;
    HostPlan hp;
    Error eval_error;          // deferred evaluation-population validation failure
    bool run_eval = true;
    int backward_blocks = 0;
    int ppt = 0;
    bool backward_hbm = false;   // the backward pass keeps its values in HBM (after the slab)
    int eval_blocks = 0;
    uint32_t first_stored_row = 0;
    PlanLayout lay{};
    DeviceBuffer own_block;    // used when the plan was created through the public API
    void* d_block = nullptr;
    double* d_slab = nullptr;
    PinnedBuffer own_staging;
    void* h_out = nullptr;
    DevicePlan dp{};
    bool launched = false;
    // Per-kernel timing marks (created on first timed launch): [0..4] on the plan's stream around
    // simulate, backward, evaluate and finalize; [5], [6] around the diagnostic on whichever stream
    // runs it; [8], [9] bracket a timed series.
    cudaEvent_t marks[10] = {};
    bool timing = false;
    bool fitted = false;         // a launch has left a fitted policy in the device records
    bool greeks = false;         // evaluation also forms the pathwise adjoint Greeks
    double sigma = 0.0;          // constant volatility of the request
    GreeksArgs gk{};
    ~fo_lsm_call_plan() {
        for (cudaEvent_t& e : marks)
            if (e) cudaEventDestroy(e);
    }
};

namespace {

Error open_device(int device, fo_executor* ex) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= 0)
        return make_error(FO_ERR_EXECUTION, FO_CODE_NO_DEVICE,
                          "no CUDA device is available for CudaExecutor; there is no CPU fallback");
    if (device < 0 || device >= count)
        return make_error(FO_ERR_EXECUTION, FO_CODE_NO_DEVICE,
                          "CUDA device " + std::to_string(device) + " does not exist; " + std::to_string(count) +
                              " device(s) are visible");
    cudaDeviceProp prop{};
    FO_CUDA_TRY(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    // The library holds sm_100a code only: another 10.x part would fail at its first launch.
    if (prop.major != 10 || prop.minor != 0)
        return make_error(FO_ERR_EXECUTION, FO_CODE_UNSUPPORTED_DEVICE,
                          std::string("CudaExecutor requires an sm_100 (Blackwell B200) device; device ") +
                              std::to_string(device) + " is " + prop.name + " (sm_" + std::to_string(prop.major) +
                              std::to_string(prop.minor) + ")");
    FO_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    if (!prop.cooperativeLaunch)
        return make_error(FO_ERR_EXECUTION, FO_CODE_UNSUPPORTED_DEVICE, "device does not support cooperative launches");
    ex->device = device;
    ex->sms = prop.multiProcessorCount;
    FO_CUDA_TRY(cudaStreamCreateWithFlags(&ex->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    int least = 0, greatest = 0;
    FO_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest), "cudaDeviceGetStreamPriorityRange");
    FO_CUDA_TRY(cudaStreamCreateWithPriority(&ex->side, cudaStreamNonBlocking, greatest), "cudaStreamCreate");
    FO_CUDA_TRY(cudaEventCreateWithFlags(&ex->fork, cudaEventDisableTiming), "cudaEventCreate");
    FO_CUDA_TRY(cudaEventCreateWithFlags(&ex->join, cudaEventDisableTiming), "cudaEventCreate");
    ex->backward_blocks_max = backward_max_blocks(device);
    ex->backward_max_ppt = backward_max_ppt();
    ex->eval_blocks_per_sm = 8;
    return Error{};
}

// Chooses the persistent grid (at most one CTA per SM) and the paths per thread of the backward
// pass. Populations up to the on-chip capacity (148 SMs x 1024 threads x the paths per thread
// whose values and two spot rows fit in shared memory) keep them on chip; larger ones (*hbm) keep
// the values in HBM and read the spots from the stored rows, on the whole grid.
Error choose_backward_shape(const fo_executor* ex, uint64_t paths, int* blocks, int* ppt, bool* hbm) {
    const uint64_t threads = kBackwardThreads;
    const uint64_t max_blocks = uint64_t(ex->backward_blocks_max);
    const uint64_t max_ppt = uint64_t(ex->backward_max_ppt);
    uint64_t per_thread = (paths + max_blocks * threads - 1) / (max_blocks * threads);
    if (per_thread == 0) per_thread = 1;
    *hbm = per_thread > max_ppt;
    if (per_thread > uint64_t(INT32_MAX))
        return make_error(FO_ERR_EXECUTION, FO_CODE_CAPACITY_EXCEEDED,
                          "training population of " + std::to_string(paths) + " paths is too large for one device");
    *ppt = int(per_thread);
    *blocks = int(std::max<uint64_t>(1, (paths + threads * per_thread - 1) / (threads * per_thread)));
    return Error{};
}

PlanLayout layout_for(const HostPlan& hp, int backward_blocks, int eval_blocks) {
    PlanLayout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        off = align_up(off, 256);
        const size_t at = off;
        off += bytes;
        return at;
    };
    const size_t rows = hp.rows();
    L.steps = take(sizeof(StepCoef) * std::max<size_t>(hp.intervals(), 1));
    L.events = take(sizeof(NodeEvent) * (hp.intervals() + 1));
    L.row_node = take(sizeof(uint32_t) * rows);
    L.disc_from_later = take(sizeof(double) * rows);
    L.disc_to_origin = take(sizeof(double) * rows);
    L.escrow_cash = take(sizeof(double) * rows);
    L.sqrt_dt = take(sizeof(double) * std::max<size_t>(hp.intervals(), 1));
    L.dt = take(sizeof(double) * std::max<size_t>(hp.intervals(), 1));
    L.inputs_bytes = off;
    L.partials = take(sizeof(double2) * 2 * size_t(backward_blocks) * 16);
    L.eval_partials = take(sizeof(double2) * size_t(eval_blocks) * 2);
    L.greek_partials = take(sizeof(double2) * size_t(eval_blocks) * kGreekSlots);
    off = align_up(off, 256);
    L.out = off;
    L.status = take(sizeof(DeviceStatus));
    L.result = take(sizeof(double) * 4);
    L.records = take(sizeof(FitRecord) * rows);
    L.counts = take(sizeof(unsigned) * rows);
    L.itm_counts = take(sizeof(unsigned) * rows);
    L.replay = take(sizeof(SimFailure));
    L.greek_out = take(sizeof(double) * kGreekSlots);
    L.out_bytes = align_up(off, 256) - L.out;
    L.total = align_up(off, 256);
    return L;
}

// Packs the plan arrays in the same layout as the device block's input region.
void pack_inputs(const HostPlan& hp, const PlanLayout& L, unsigned char* host) {
    std::memset(host, 0, L.inputs_bytes);
    std::memcpy(host + L.steps, hp.steps.data(), sizeof(StepCoef) * hp.steps.size());
    std::memcpy(host + L.events, hp.events.data(), sizeof(NodeEvent) * hp.events.size());
    std::memcpy(host + L.row_node, hp.row_node.data(), sizeof(uint32_t) * hp.row_node.size());
    std::memcpy(host + L.disc_from_later, hp.disc_from_later.data(), sizeof(double) * hp.rows());
    std::memcpy(host + L.disc_to_origin, hp.disc_to_origin.data(), sizeof(double) * hp.rows());
    std::memcpy(host + L.escrow_cash, hp.escrow_cash.data(), sizeof(double) * hp.rows());
    auto* sqrt_dt = reinterpret_cast<double*>(host + L.sqrt_dt);
    auto* dt = reinterpret_cast<double*>(host + L.dt);
    for (uint32_t i = 0; i < hp.intervals(); ++i) {
        dt[i] = hp.times[i + 1] - hp.times[i];
        sqrt_dt[i] = std::sqrt(dt[i]);
    }
}

DevicePlan device_plan(const HostPlan& hp, const PlanLayout& L, unsigned char* dev, uint32_t first_stored_row) {
    DevicePlan p{};
    p.intervals = hp.intervals();
    p.rows = hp.rows();
    p.first_stored_row = first_stored_row;
    p.strike = hp.strike;
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
    p.steps = reinterpret_cast<const StepCoef*>(dev + L.steps);
    p.events = reinterpret_cast<const NodeEvent*>(dev + L.events);
    p.row_node = reinterpret_cast<const uint32_t*>(dev + L.row_node);
    p.disc_from_later = reinterpret_cast<const double*>(dev + L.disc_from_later);
    p.disc_to_origin = reinterpret_cast<const double*>(dev + L.disc_to_origin);
    p.escrow_cash = reinterpret_cast<const double*>(dev + L.escrow_cash);
    p.origin_discount = hp.origin_discount;
    return p;
}

// The adjoint's view of the plan: cash dividends in node order, volatility, device arrays.
void fill_greeks_args(fo_lsm_call_plan* plan) {
    GreeksArgs& g = plan->gk;
    g = GreeksArgs{};
    const HostPlan& hp = plan->hp;
    for (uint32_t node = 1; node < hp.events.size(); ++node) {
        if (!(hp.events[node].flags & kEventDividend)) continue;
        if (g.dividends < uint32_t(kMaxGreekDividends)) {
            g.div_node[g.dividends] = node;
            g.div_amount[g.dividends] = hp.events[node].dividend_amount;
        }
        g.dividends += 1;
    }
    g.sigma = plan->sigma;
    unsigned char* dev = static_cast<unsigned char*>(plan->d_block);
    g.sqrt_dt = reinterpret_cast<const double*>(dev + plan->lay.sqrt_dt);
    g.dt = reinterpret_cast<const double*>(dev + plan->lay.dt);
    g.partials = reinterpret_cast<double2*>(dev + plan->lay.greek_partials);
}

Error plan_create(fo_executor* ex, const fo_lsm_call_request& q, bool own_memory, fo_lsm_call_plan** out) {
    auto plan = std::make_unique<fo_lsm_call_plan>();
    plan->ex = ex;
    Error e = build_call_plan(q, &plan->hp);
    if (!e.ok()) return e;
    HostPlan& hp = plan->hp;
    // Evaluation population checks run after the fit in the reference (policy.rs:330-333).
    if (q.evaluation_paths == 0) {
        plan->eval_error = make_error(FO_ERR_LSM, FO_CODE_EMPTY_PATH_SET,
                                      "LSM evaluation simulation failed: simulation path count must be positive");
    } else if (q.evaluation_paths > 0xffffffffull) {
        plan->eval_error = make_error(FO_ERR_LSM, FO_CODE_RANDOM_PATH_NAMESPACE_OVERFLOW,
                                      "LSM evaluation simulation failed: seeded simulation supports at most 4294967295 "
                                      "paths in one random domain; observed " + std::to_string(q.evaluation_paths));
    }
    plan->run_eval = plan->eval_error.ok();
    e = choose_backward_shape(ex, hp.train_paths, &plan->backward_blocks, &plan->ppt, &plan->backward_hbm);
    if (!e.ok()) return e;
    const uint64_t eval_threads = kEvalThreads;
    const uint64_t eval_needed = plan->run_eval ? (hp.eval_paths + eval_threads - 1) / eval_threads : 1;
    plan->eval_blocks = int(std::max<uint64_t>(1, std::min<uint64_t>(eval_needed, uint64_t(ex->sms) * ex->eval_blocks_per_sm)));
    plan->first_stored_row = hp.origin_row ? 1u : 0u;
    plan->lay = layout_for(hp, plan->backward_blocks, plan->eval_blocks);
    const PlanLayout& L = plan->lay;
    // device memory: plan block + slab
    if (own_memory) {
        e = plan->own_block.reserve(L.total);
        if (!e.ok()) return e;
        plan->d_block = plan->own_block.ptr;
        e = plan->own_staging.reserve(std::max(L.inputs_bytes, L.out_bytes));
        if (!e.ok()) return e;
        plan->h_out = plan->own_staging.ptr;
    } else {
        e = ex->scratch.reserve(L.total);
        if (!e.ok()) return e;
        plan->d_block = ex->scratch.ptr;
        e = ex->staging.reserve(std::max(L.inputs_bytes, L.out_bytes));
        if (!e.ok()) return e;
        plan->h_out = ex->staging.ptr;
    }
    const uint64_t stored_rows = hp.rows() - plan->first_stored_row;
    const size_t slab_bytes = sizeof(double) * stored_rows * hp.train_paths +
                              (plan->backward_hbm ? sizeof(double) * hp.train_paths : 0);
    e = ex->slab.reserve(std::max<size_t>(slab_bytes, 8));
    if (!e.ok()) {
        if (e.code == FO_CODE_CUDA_FAILURE)
            return make_error(FO_ERR_EXECUTION, FO_CODE_CAPACITY_EXCEEDED,
                              "training paths need " + std::to_string(slab_bytes) +
                                  " bytes of device memory (paths x stored rows x 8 bytes), more than the device can "
                                  "allocate: " + e.message);
        return e;
    }
    plan->d_slab = static_cast<double*>(ex->slab.ptr);
    unsigned char* dev = static_cast<unsigned char*>(plan->d_block);
    plan->dp = device_plan(hp, L, dev, plan->first_stored_row);
    plan->sigma = q.annualized_volatility;
    fill_greeks_args(plan.get());
    // upload inputs once
    pack_inputs(hp, L, static_cast<unsigned char*>(plan->h_out));
    FO_CUDA_TRY(cudaMemcpyAsync(dev, plan->h_out, L.inputs_bytes, cudaMemcpyHostToDevice, ex->stream), "plan upload");
    // A plan of its own may be packed again (revaluation) while this copy is pending, so it waits
    // here. A one-shot plan borrows the executor's staging, which nothing rewrites before the
    // call's read-back has synchronised the stream: its kernels simply queue behind the copy.
    if (own_memory) FO_CUDA_TRY(cudaStreamSynchronize(ex->stream), "plan upload");
    *out = plan.release();
    return Error{};
}

cudaError_t launch_evaluation(const fo_lsm_call_plan* plan, const EvalArgs& a) {
    return plan->greeks ? launch_evaluate_greeks(a, plan->gk, plan->eval_blocks, plan->ex->stream)
                        : launch_evaluate(a, plan->eval_blocks, plan->ex->stream);
}

Error plan_launch(fo_lsm_call_plan* plan) {
    fo_executor* ex = plan->ex;
    const PlanLayout& L = plan->lay;
    unsigned char* dev = static_cast<unsigned char*>(plan->d_block);
    cudaStream_t s = ex->stream;
    auto* status = reinterpret_cast<DeviceStatus*>(dev + L.status);
    auto* records = reinterpret_cast<FitRecord*>(dev + L.records);
    FO_CUDA_TRY(cudaMemsetAsync(dev + L.out, 0, L.out_bytes, s), "reset");
    FO_CUDA_TRY(cudaMemsetAsync(status, 0xff, kStatusNoneBytes, s), "reset");
    auto mark = [&](int i) -> cudaError_t { return plan->timing ? cudaEventRecord(plan->marks[i], s) : cudaSuccess; };
    FO_CUDA_TRY(mark(0), "event");
    // K1 training simulation
    FO_CUDA_TRY(launch_simulate(plan->dp, plan->hp.train_paths, plan->hp.train_seed, plan->hp.train_domain, plan->d_slab,
                                plan->first_stored_row, plan->hp.escrowed ? 1 : 0, &status->train_sim_fail, s),
                "training simulation launch");
    FO_CUDA_TRY(mark(1), "event");
    // K2 backward induction
    BackwardArgs b{};
    b.plan = plan->dp;
    b.slab = plan->d_slab;
    b.partials = reinterpret_cast<double2*>(dev + L.partials);
    b.partial_stride = size_t(plan->backward_blocks) * 16;
    b.records = records;
    b.status = status;
    b.ppt = plan->ppt;
    b.values = plan->backward_hbm
                   ? plan->d_slab + uint64_t(plan->hp.rows() - plan->first_stored_row) * plan->hp.train_paths
                   : nullptr;
    FO_CUDA_TRY(launch_backward(b, plan->backward_blocks, plan->ppt, s), "backward launch");
    FO_CUDA_TRY(mark(2), "event");
    // K3 diagnostics: nothing on the device reads them, so they run on the side stream next to
    // the evaluation (inline for a stack executor).
    cudaStream_t ds = ex->side ? ex->side : s;
    if (ex->side) {
        FO_CUDA_TRY(cudaEventRecord(ex->fork, s), "event");
        FO_CUDA_TRY(cudaStreamWaitEvent(ex->side, ex->fork, 0), "event");
    }
    if (plan->timing) FO_CUDA_TRY(cudaEventRecord(plan->marks[5], ds), "event");
    FO_CUDA_TRY(launch_diagnose(plan->dp, records, ds), "diagnose launch");
    if (plan->timing) FO_CUDA_TRY(cudaEventRecord(plan->marks[6], ds), "event");
    if (ex->side) FO_CUDA_TRY(cudaEventRecord(ex->join, ex->side), "event");
    if (plan->run_eval) {
        EvalArgs a{};
        a.plan = plan->dp;
        a.records = records;
        a.partials = reinterpret_cast<double2*>(dev + L.eval_partials);
        a.counts = reinterpret_cast<unsigned*>(dev + L.counts);
        a.itm_counts = reinterpret_cast<unsigned*>(dev + L.itm_counts);
        a.status = status;
        FO_CUDA_TRY(launch_evaluation(plan, a), "evaluation launch");
        FO_CUDA_TRY(mark(3), "event");
        FO_CUDA_TRY(launch_finalize(a.partials, plan->eval_blocks, plan->hp.eval_paths,
                                    reinterpret_cast<double*>(dev + L.result), s),
                    "finalize launch");
        if (plan->greeks)
            FO_CUDA_TRY(launch_finalize_greeks(plan->gk.partials, plan->eval_blocks,
                                               reinterpret_cast<double*>(dev + L.greek_out), s),
                        "Greeks finalize launch");
        FO_CUDA_TRY(mark(4), "event");
    }
    if (ex->side) FO_CUDA_TRY(cudaStreamWaitEvent(s, ex->join, 0), "event");
    plan->launched = true;
    plan->fitted = true;
    return Error{};
}

// Timed kernel segments of one launch (the Greeks finalize shares the last segment).
uint64_t kernels_per_launch(const fo_lsm_call_plan* plan) { return plan->run_eval ? 5 : 3; }

Error plan_time_launches(fo_lsm_call_plan* plan, uint32_t iterations, double* elapsed_ms, double* kernel_ms,
                         uint64_t capacity) {
    cudaStream_t s = plan->ex->stream;
    for (cudaEvent_t& e : plan->marks)
        if (!e) FO_CUDA_TRY(cudaEventCreate(&e), "cudaEventCreate");
    const uint64_t kernels = kernels_per_launch(plan);
    std::vector<double> sums(kernels, 0.0);
    cudaEvent_t begin = plan->marks[8], end = plan->marks[9];
    // Segments in the order simulate, backward, diagnose, evaluate, finalize. The diagnostic runs
    // beside the evaluation on the side stream, so the evaluation starts where the backward pass
    // ends; inline, it starts where the diagnostic ends.
    const bool side = plan->ex->side != nullptr;
    const std::pair<int, int> segments[5] = {{0, 1}, {1, 2}, {5, 6}, {side ? 2 : 6, 3}, {3, 4}};
    FO_CUDA_TRY(cudaEventRecord(begin, s), "event");
    double total = 0.0;
    for (uint32_t i = 0; i < iterations; ++i) {
        plan->timing = kernel_ms != nullptr;
        Error e = plan_launch(plan);
        plan->timing = false;
        if (!e.ok()) return e;
        if (kernel_ms) {
            FO_CUDA_TRY(cudaEventSynchronize(plan->marks[plan->run_eval ? 4 : 2]), "event");
            FO_CUDA_TRY(cudaEventSynchronize(plan->marks[6]), "event");
            for (uint64_t k = 0; k < kernels; ++k) {
                float ms = 0.f;
                FO_CUDA_TRY(cudaEventElapsedTime(&ms, plan->marks[segments[k].first], plan->marks[segments[k].second]),
                            "event");
                sums[k] += ms;
            }
        }
    }
    FO_CUDA_TRY(cudaEventRecord(end, s), "event");
    FO_CUDA_TRY(cudaEventSynchronize(end), "event");
    float ms = 0.f;
    FO_CUDA_TRY(cudaEventElapsedTime(&ms, begin, end), "event");
    total = ms;
    *elapsed_ms = total;
    for (uint64_t k = 0; kernel_ms && k < kernels && k < capacity; ++k) kernel_ms[k] = sums[k];
    return Error{};
}

Error replay(fo_lsm_call_plan* plan, bool training, uint64_t path, int want_row, SimFailure* out) {
    fo_executor* ex = plan->ex;
    unsigned char* dev = static_cast<unsigned char*>(plan->d_block);
    auto* d_replay = reinterpret_cast<SimFailure*>(dev + plan->lay.replay);
    const HostPlan& hp = plan->hp;
    FO_CUDA_TRY(launch_replay(plan->dp, training ? hp.train_seed : hp.eval_seed, training ? hp.train_domain : hp.eval_domain,
                              uint32_t(path), want_row, d_replay, ex->stream),
                "replay launch");
    FO_CUDA_TRY(cudaMemcpyAsync(out, d_replay, sizeof(SimFailure), cudaMemcpyDeviceToHost, ex->stream), "replay copy");
    FO_CUDA_TRY(cudaStreamSynchronize(ex->stream), "replay");
    return Error{};
}

Error simulation_error(fo_lsm_call_plan* plan, bool training, uint64_t path) {
    SimFailure f{};
    Error e = replay(plan, training, path, -1, &f);
    if (!e.ok()) return e;
    const std::string role = training ? "training" : "evaluation";
    Error out = make_error(FO_ERR_LSM, simulation_failure_code(f.code),
                           "LSM " + role + " simulation failed: " +
                               simulation_failure_message(f.code, uint32_t(f.interval), path, f.spot, f.normal));
    out.path = int64_t(path);
    return out;
}

Error plan_collect(fo_lsm_call_plan* plan, fo_lsm_call_result* result) {
    if (!plan->launched)
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "plan was collected before it was launched");
    fo_executor* ex = plan->ex;
    const PlanLayout& L = plan->lay;
    const HostPlan& hp = plan->hp;
    unsigned char* dev = static_cast<unsigned char*>(plan->d_block);
    unsigned char* host = static_cast<unsigned char*>(plan->h_out);
    FO_CUDA_TRY(cudaMemcpyAsync(host, dev + L.out, L.out_bytes, cudaMemcpyDeviceToHost, ex->stream), "result copy");
    FO_CUDA_TRY(cudaStreamSynchronize(ex->stream), "pricing");
    plan->launched = false;
    const auto* status = reinterpret_cast<const DeviceStatus*>(host + (L.status - L.out));
    const auto* res = reinterpret_cast<const double*>(host + (L.result - L.out));
    const auto* records = reinterpret_cast<const FitRecord*>(host + (L.records - L.out));
    const auto* counts = reinterpret_cast<const unsigned*>(host + (L.counts - L.out));
    const auto* itm_counts = reinterpret_cast<const unsigned*>(host + (L.itm_counts - L.out));
    const uint32_t rows = hp.rows();
    const uint32_t E = rows - 1;
    if (status->barrier_timeout)
        return make_error(FO_ERR_EXECUTION, FO_CODE_BARRIER_TIMEOUT,
                          "backward-induction grid synchronisation timed out; the device result was discarded");
    if (status->train_sim_fail != kNone) return simulation_error(plan, true, status->train_sim_fail);
    // Fit failures in backward order: discount, population, regression, diagnostic, update.
    const uint32_t lowest = hp.origin_row ? 1u : 0u;
    const uint32_t fitted_rows = E > lowest ? E - lowest : 0;
    for (uint32_t order = 0; order <= fitted_rows; ++order) {
        const unsigned long long lo = (unsigned long long)order << 32, hi = lo | 0xffffffffull;
        if (status->fit_payoff_fail >= lo && status->fit_payoff_fail <= hi) {
            Error e = make_error(FO_ERR_LSM, FO_CODE_NON_FINITE_DISCOUNTED_PAYOFF,
                                 "LSM evaluation produced non-finite discounted payoff at path " +
                                     std::to_string(status->fit_payoff_fail & 0xffffffffull));
            e.path = int64_t(status->fit_payoff_fail & 0xffffffffull);
            return e;
        }
        if (order == fitted_rows) break;
        const uint32_t row = E - 1 - order;
        const uint32_t node = hp.row_node[row];
        const FitRecord& rec = records[row];
        if (status->fit_nonfinite >= lo && status->fit_nonfinite <= hi) {
            Error e = make_error(FO_ERR_LSM, FO_CODE_NON_FINITE_PREDICTOR,
                                 "continuation regression failed at exercise node " + node_str(node) +
                                     ": regression predictor or response at path " +
                                     std::to_string(status->fit_nonfinite & 0xffffffffull) + " must be finite");
            e.node = node;
            e.path = int64_t(status->fit_nonfinite & 0xffffffffull);
            return e;
        }
        if (rec.kind == kRuleFitFailed) return fit_failure(hp, rec, node);
        if (rec.kind == kRuleRegression && rec.diag_status != kDiagOk) return diag_failure(hp, rec, node);
        if (status->fit_predict_fail >= lo && status->fit_predict_fail <= hi) {
            const uint64_t path = status->fit_predict_fail & 0xffffffffull;
            double spot = 0.0;
            cudaMemcpy(&spot, plan->d_slab + uint64_t(row - plan->first_stored_row) * hp.train_paths + path,
                       sizeof(double), cudaMemcpyDeviceToHost);
            Error e = make_error(FO_ERR_LSM, FO_CODE_NON_FINITE_PREDICTION,
                                 "continuation prediction failed at exercise node " + node_str(node) + ", path " +
                                     std::to_string(path) + ": polynomial regression produced non-finite prediction for predictor " +
                                     fmt_f64(spot / hp.strike));
            e.node = node;
            e.path = int64_t(path);
            return e;
        }
    }
    if (!plan->run_eval) return plan->eval_error;
    if (status->eval_sim_fail != kNone) return simulation_error(plan, false, status->eval_sim_fail);
    // Assemble diagnostics (policy.rs:39-65) in row order.
    result->paths = uint32_t(hp.eval_paths);
    result->n_observations = rows;
    result->n_diagnostics = 0;
    const bool origin = hp.origin_row;
    const bool origin_exercise = origin && records[0].kind == kRuleOrigin && records[0].origin_exercise;
    for (uint32_t r = 0; r < E; ++r) {
        const FitRecord& rec = records[r];
        fo_lsm_node_diagnostic d{};
        d.node = hp.row_node[r];
        switch (rec.kind) {
            case kRuleOrigin:
                d.kind = FO_DIAG_ORIGIN_DECISION;
                d.exercise = rec.origin_exercise;
                d.estimated_continuation = rec.origin_continuation;
                break;
            case kRuleNoSupport: d.kind = FO_DIAG_NO_IN_THE_MONEY_PATHS; break;
            case kRuleContinue:
                d.kind = FO_DIAG_INSUFFICIENT_SUPPORT;
                d.in_the_money_paths = uint32_t(rec.itm);
                d.columns = uint64_t(hp.degree + 1);
                break;
            case kRuleRegression:
                d.kind = FO_DIAG_REGRESSION;
                d.in_the_money_paths = uint32_t(rec.itm);
                d.observations = rec.itm;
                d.columns = uint64_t(hp.degree + 1);
                d.rank = uint64_t(rec.diag_rank);
                d.condition_number = rec.diag_condition;
                d.predictor_mean = rec.model.mean;
                d.predictor_scale = rec.model.scale;
                break;
            default:
                return make_error(FO_ERR_EXECUTION, FO_CODE_CUDA_FAILURE,
                                  "backward pass left exercise row " + std::to_string(r) + " unfitted");
        }
        if (result->diagnostics && result->n_diagnostics < result->diagnostics_capacity)
            result->diagnostics[result->n_diagnostics] = d;
        result->n_diagnostics += 1;
    }
    for (uint32_t r = 0; r < rows && result->observation_nodes && r < result->observation_capacity; ++r)
        result->observation_nodes[r] = hp.row_node[r];
    if (origin_exercise) {
        // LsmEvaluation::deterministic (policy.rs:657-669)
        for (uint32_t r = 0; r < rows && result->exercise_counts && r < result->observation_capacity; ++r)
            result->exercise_counts[r] = r == 0 ? uint32_t(hp.eval_paths) : 0u;
        const double d = hp.initial_spot - hp.strike;
        result->price = d > 0.0 ? d : 0.0;
        result->has_sample_standard_deviation = 1;
        result->sample_standard_deviation = 0.0;
        result->has_standard_error = 1;
        result->standard_error = 0.0;
        return Error{};
    }
    // Evaluation failures in row order: prediction/payoff (key) or unsupported in-the-money paths.
    const uint64_t eval_row = status->eval_fail != kNone ? (status->eval_fail >> 33) : ~0ull;
    for (uint32_t r = 0; r < E; ++r) {
        if (records[r].kind == kRuleNoSupport && itm_counts[r] > 0) {
            if (eval_row < r) break;
            Error e = make_error(FO_ERR_LSM, FO_CODE_EVALUATION_OUTSIDE_TRAINING_SUPPORT,
                                 std::to_string(itm_counts[r]) + " active evaluation paths are in the money at node " +
                                     node_str(hp.row_node[r]) + ", but training had no in-the-money support");
            e.node = hp.row_node[r];
            return e;
        }
    }
    if (status->eval_fail != kNone) {
        const uint32_t r = uint32_t(status->eval_fail >> 33);
        const uint64_t path = (status->eval_fail >> 1) & 0xffffffffull;
        if (status->eval_fail & 1ull) {
            Error e = make_error(FO_ERR_LSM, FO_CODE_NON_FINITE_DISCOUNTED_PAYOFF,
                                 "LSM evaluation produced non-finite discounted payoff at path " + std::to_string(path));
            e.path = int64_t(path);
            return e;
        }
        SimFailure f{};
        Error re = replay(plan, false, path, int(r), &f);
        if (!re.ok()) return re;
        Error e = make_error(FO_ERR_LSM, FO_CODE_NON_FINITE_PREDICTION,
                             "continuation prediction failed at exercise node " + node_str(hp.row_node[r]) + ", path " +
                                 std::to_string(path) + ": polynomial regression produced non-finite prediction for predictor " +
                                 fmt_f64(f.observed / hp.strike));
        e.node = hp.row_node[r];
        e.path = int64_t(path);
        return e;
    }
    if (status->eval_terminal_fail != kNone) {
        Error e = make_error(FO_ERR_LSM, FO_CODE_NON_FINITE_DISCOUNTED_PAYOFF,
                             "LSM evaluation produced non-finite discounted payoff at path " +
                                 std::to_string(status->eval_terminal_fail));
        e.path = int64_t(status->eval_terminal_fail);
        return e;
    }
    for (uint32_t r = 0; r < rows && result->exercise_counts && r < result->observation_capacity; ++r)
        result->exercise_counts[r] = counts[r];
    result->price = res[0];
    if (hp.eval_paths > 1) {
        if (!std::isfinite(res[2]) || !std::isfinite(res[3])) {
            Error e = make_error(FO_ERR_LSM, FO_CODE_NON_FINITE_DISCOUNTED_PAYOFF,
                                 "LSM evaluation produced non-finite discounted payoff at path 0");
            e.path = 0;
            return e;
        }
        result->has_sample_standard_deviation = 1;
        result->sample_standard_deviation = res[2];
        result->has_standard_error = 1;
        result->standard_error = res[3];
    } else {
        result->has_sample_standard_deviation = 0;
        result->has_standard_error = 0;
        result->sample_standard_deviation = 0.0;
        result->standard_error = 0.0;
    }
    return Error{};
}

// Pathwise adjoint Greeks of the last collected launch (lsm_greeks.cu for the per-path terms).
Error plan_greeks(const fo_lsm_call_plan* plan, fo_lsm_call_greeks* g) {
    if (!plan->greeks)
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "the plan does not form adjoint Greeks");
    const HostPlan& hp = plan->hp;
    const PlanLayout& L = plan->lay;
    const auto* host = static_cast<const unsigned char*>(plan->h_out);
    const auto* out = reinterpret_cast<const double*>(host + (L.greek_out - L.out));
    const auto* counts = reinterpret_cast<const unsigned*>(host + (L.counts - L.out));
    const auto* records = reinterpret_cast<const FitRecord*>(host + (L.records - L.out));
    const uint64_t nodes = hp.times.size();
    const uint32_t n_div = plan->gk.dividends;
    if ((nodes && (!g->log_discount_sensitivities || g->log_discount_capacity < nodes)) ||
        (n_div && (!g->dividend_sensitivities || g->dividend_capacity < n_div)))
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                          "Greeks buffers must hold " + std::to_string(nodes) + " log-discount and " +
                              std::to_string(n_div) + " dividend sensitivities");
    for (uint64_t i = 0; i < nodes; ++i) g->log_discount_sensitivities[i] = 0.0;
    for (uint32_t j = 0; j < n_div; ++j) g->dividend_sensitivities[j] = 0.0;
    const double K = hp.strike;
    if (hp.origin_row && records[0].kind == kRuleOrigin && records[0].origin_exercise) {
        // Deterministic origin exercise (policy.rs:657-669): price = max(S0 - K, 0) at node 0.
        const double d = hp.initial_spot - K;
        g->delta = d > 0.0 ? 1.0 : 0.0;
        g->vega = 0.0;
        g->log_discount_sensitivities[0] = d > 0.0 ? d : 0.0;
        return Error{};
    }
    const double n = double(hp.eval_paths);
    g->delta = out[kGreekDelta] / n;
    g->vega = out[kGreekVega] / n;
    double* dl = g->log_discount_sensitivities;
    dl[0] += out[kGreekL0] / n;
    for (uint32_t j = 0; j < n_div; ++j) {
        dl[plan->gk.div_node[j]] += out[kGreekJump + j] / n;
        g->dividend_sensitivities[j] = out[kGreekDividend + j] / n;
    }
    // Early exercise at row r contributes exactly -K exp(L_node) per stopped path.
    const uint32_t rows = hp.rows();
    for (uint32_t r = 0; r + 1 < rows; ++r)
        if (counts[r]) dl[hp.row_node[r]] += -K * hp.disc_to_origin[r] * double(counts[r]) / n;
    dl[hp.row_node[rows - 1]] += out[kGreekTerminal] / n;
    return Error{};
}

// Re-values the plan's fitted policy on another market of the same contract shape: only the
// initial spot, log discounts, cumulative yields, cash amounts and volatility may change.
Error plan_revalue(fo_lsm_call_plan* plan, const fo_lsm_call_request& q, fo_lsm_call_result* result) {
    if (!plan->fitted)
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "the plan has no fitted policy; launch it first");
    HostPlan next;
    Error e = build_call_plan(q, &next);
    if (!e.ok()) return e;
    const HostPlan& hp = plan->hp;
    bool same = next.times.size() == hp.times.size() && next.row_node == hp.row_node &&
                next.train_paths == hp.train_paths && next.eval_paths == hp.eval_paths &&
                next.train_seed == hp.train_seed && next.eval_seed == hp.eval_seed &&
                next.train_domain == hp.train_domain && next.eval_domain == hp.eval_domain &&
                next.strike == hp.strike && next.degree == hp.degree && next.tie_rule == hp.tie_rule &&
                next.support == hp.support && next.policy == hp.policy;
    for (size_t i = 0; same && i < hp.times.size(); ++i)
        same = next.times[i] == hp.times[i] && (next.events[i].flags & kEventDividend) == (hp.events[i].flags & kEventDividend);
    if (!same)
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                          "a revaluation market must keep the plan's schedule, dividend nodes, strike, paths, streams "
                          "and method");
    plan->hp = std::move(next);
    plan->sigma = q.annualized_volatility;
    const PlanLayout& L = plan->lay;
    unsigned char* dev = static_cast<unsigned char*>(plan->d_block);
    plan->dp = device_plan(plan->hp, L, dev, plan->first_stored_row);
    fill_greeks_args(plan);
    fo_executor* ex = plan->ex;
    cudaStream_t s = ex->stream;
    pack_inputs(plan->hp, L, static_cast<unsigned char*>(plan->h_out));
    FO_CUDA_TRY(cudaMemcpyAsync(dev, plan->h_out, L.inputs_bytes, cudaMemcpyHostToDevice, s), "revaluation upload");
    auto* status = reinterpret_cast<DeviceStatus*>(dev + L.status);
    FO_CUDA_TRY(cudaMemsetAsync(&status->eval_sim_fail, 0xff, sizeof(unsigned long long), s), "reset");
    FO_CUDA_TRY(cudaMemsetAsync(&status->eval_fail, 0xff, 2 * sizeof(unsigned long long), s), "reset");
    FO_CUDA_TRY(cudaMemsetAsync(dev + L.result, 0, sizeof(double) * 4, s), "reset");
    FO_CUDA_TRY(cudaMemsetAsync(dev + L.counts, 0, sizeof(unsigned) * plan->hp.rows(), s), "reset");
    FO_CUDA_TRY(cudaMemsetAsync(dev + L.itm_counts, 0, sizeof(unsigned) * plan->hp.rows(), s), "reset");
    FO_CUDA_TRY(cudaMemsetAsync(dev + L.greek_out, 0, sizeof(double) * kGreekSlots, s), "reset");
    if (plan->run_eval) {
        EvalArgs a{};
        a.plan = plan->dp;
        a.records = reinterpret_cast<const FitRecord*>(dev + L.records);
        a.partials = reinterpret_cast<double2*>(dev + L.eval_partials);
        a.counts = reinterpret_cast<unsigned*>(dev + L.counts);
        a.itm_counts = reinterpret_cast<unsigned*>(dev + L.itm_counts);
        a.status = status;
        FO_CUDA_TRY(launch_evaluation(plan, a), "revaluation launch");
        FO_CUDA_TRY(launch_finalize(a.partials, plan->eval_blocks, plan->hp.eval_paths,
                                    reinterpret_cast<double*>(dev + L.result), s),
                    "finalize launch");
        if (plan->greeks)
            FO_CUDA_TRY(launch_finalize_greeks(plan->gk.partials, plan->eval_blocks,
                                               reinterpret_cast<double*>(dev + L.greek_out), s),
                        "Greeks finalize launch");
    }
    plan->launched = true;
    return plan_collect(plan, result);
}

// Re-runs the evaluation of the plan's fitted policy on its current market with every path's
// stopping row recorded, and copies those rows to the host: the per-path record that counts the
// decisions in which two implementations differ.
Error plan_stopping_rows(fo_lsm_call_plan* plan, uint32_t* rows_out, uint64_t capacity) {
    if (!plan->fitted)
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, "the plan has no fitted policy; launch it first");
    if (!plan->run_eval) return plan->eval_error;
    const uint64_t n = plan->hp.eval_paths;
    if (!rows_out || capacity < n)
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                          "stopping rows need " + std::to_string(n) + " entries; capacity is " + std::to_string(capacity));
    fo_executor* ex = plan->ex;
    cudaStream_t s = ex->stream;
    const PlanLayout& L = plan->lay;
    unsigned char* dev = static_cast<unsigned char*>(plan->d_block);
    FitRecord origin{};
    FO_CUDA_TRY(cudaMemcpyAsync(&origin, dev + L.records, sizeof(FitRecord), cudaMemcpyDeviceToHost, s), "record copy");
    FO_CUDA_TRY(cudaStreamSynchronize(s), "record copy");
    if (plan->hp.origin_row && origin.kind == kRuleOrigin && origin.origin_exercise) {
        // LsmEvaluation::deterministic (policy.rs:657-669): every path stops at the origin row.
        std::fill(rows_out, rows_out + n, 0u);
        return Error{};
    }
    DeviceBuffer stops;
    Error e = stops.reserve(sizeof(uint32_t) * n);
    if (!e.ok()) return e;
    auto* status = reinterpret_cast<DeviceStatus*>(dev + L.status);
    FO_CUDA_TRY(cudaMemsetAsync(&status->eval_sim_fail, 0xff, sizeof(unsigned long long), s), "reset");
    FO_CUDA_TRY(cudaMemsetAsync(&status->eval_fail, 0xff, 2 * sizeof(unsigned long long), s), "reset");
    FO_CUDA_TRY(cudaMemsetAsync(dev + L.counts, 0, sizeof(unsigned) * plan->hp.rows(), s), "reset");
    FO_CUDA_TRY(cudaMemsetAsync(dev + L.itm_counts, 0, sizeof(unsigned) * plan->hp.rows(), s), "reset");
    EvalArgs a{};
    a.plan = plan->dp;
    a.records = reinterpret_cast<const FitRecord*>(dev + L.records);
    a.partials = reinterpret_cast<double2*>(dev + L.eval_partials);
    a.counts = reinterpret_cast<unsigned*>(dev + L.counts);
    a.itm_counts = reinterpret_cast<unsigned*>(dev + L.itm_counts);
    a.status = status;
    a.stops = static_cast<uint32_t*>(stops.ptr);
    FO_CUDA_TRY(launch_evaluate(a, plan->eval_blocks, s), "stopping-row evaluation launch");
    DeviceStatus st{};
    FO_CUDA_TRY(cudaMemcpyAsync(rows_out, stops.ptr, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s), "stops copy");
    FO_CUDA_TRY(cudaMemcpyAsync(&st, status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, s), "status copy");
    FO_CUDA_TRY(cudaStreamSynchronize(s), "stopping-row evaluation");
    if (st.eval_sim_fail != kNone || st.eval_fail != kNone || st.eval_terminal_fail != kNone)
        return make_error(FO_ERR_LSM, FO_CODE_INVALID_ARGUMENT,
                          "the plan's evaluation fails on its current market; price it for the typed error");
    return Error{};
}

Error enable_greeks(fo_lsm_call_plan* plan, bool enabled) {
    if (enabled && plan->gk.dividends > uint32_t(kMaxGreekDividends))
        return make_error(FO_ERR_EXECUTION, FO_CODE_CAPACITY_EXCEEDED,
                          "adjoint Greeks support at most " + std::to_string(kMaxGreekDividends) +
                              " cash dividends per contract; observed " + std::to_string(plan->gk.dividends));
    plan->greeks = enabled;
    return Error{};
}

// simulate_gbm_seeded_f64 (normals == NULL: the path's Philox stream from (seed, domain)) and
// simulate_gbm_f64 (normals: a caller matrix [intervals, paths], time-major) over K1; checks in the
// reference's order (GbmPathPlan::simulate / simulate_seeded, path.rs:139-175, 533-615,
// seeded.rs:384-397) with its messages. Buffers live on the device when *_on_device, else on the
// host. Returns with the states written and the executor's stream idle.
Error simulate_gbm(fo_executor* executor, const fo_gbm_seeded_request& q, const double* normals, uint64_t normal_rows,
                   bool normals_on_device, double* states, uint64_t out_len, bool states_on_device) {
    const bool external = normals != nullptr;
    HostPlan hp;
    Error e = build_gbm_plan(q.schedule_times, q.n_schedule_times, q.curve_times, q.n_curve_times, q.log_discounts,
                             q.n_log_discounts, q.dividend_yield_times, q.n_dividend_yield_times,
                             q.cumulative_dividend_yields, q.n_cumulative_dividend_yields, q.dividend_nodes,
                             q.n_dividend_nodes, q.dividend_amounts, q.n_dividend_amounts, q.exercise_nodes,
                             q.n_exercise_nodes, q.expiry_node, q.annualized_volatility, q.dividend_policy, &hp);
    if (!e.ok()) return e;
    const uint64_t paths = q.paths;
    const uint64_t intervals = hp.intervals();
    const double s0 = q.initial_spot;
    auto bad_spot = [&] {
        return make_error(FO_ERR_SIMULATION, FO_CODE_INVALID_INITIAL_SPOT,
                          "initial spot must be finite, nonnegative, and canonical; observed " + fmt_f64(s0));
    };
    const bool spot_ok = std::isfinite(s0) && s0 >= 0.0 && !(s0 == 0.0 && std::signbit(s0));
    if (external) {
        // simulate_gbm_f64 (lib.rs:1000-1008) checks the matrix's interval rows after the plan;
        // GbmPathPlan::validate_execution (path.rs:558-603) then the spot, the path count and the
        // finiteness of every variate.
        if (normal_rows != intervals)
            return make_error(FO_ERR_SIMULATION, FO_CODE_BUFFER_LENGTH_MISMATCH,
                              "normal interval-row buffer length mismatch: expected " + std::to_string(intervals) +
                                  ", observed " + std::to_string(normal_rows));
        if (!spot_ok) return bad_spot();
        if (paths == 0)
            return make_error(FO_ERR_SIMULATION, FO_CODE_EMPTY_PATH_SET, "simulation path count must be positive");
    } else {
        if (paths == 0)
            return make_error(FO_ERR_SIMULATION, FO_CODE_EMPTY_PATH_SET, "simulation path count must be positive");
        if (!spot_ok) return bad_spot();
        if (paths > 0xffffffffull)
            return make_error(FO_ERR_SIMULATION, FO_CODE_RANDOM_PATH_NAMESPACE_OVERFLOW,
                              "seeded simulation supports at most 4294967295 paths in one random domain; observed " +
                                  std::to_string(paths));
    }
    const uint64_t n_normals = external ? intervals * paths : 0;
    const uint64_t rows = hp.rows();
    if (!states || out_len != rows * paths)
        return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                          "states buffer must hold exactly " + std::to_string(rows * paths) + " values");
    hp.sim_start = s0;
    hp.initial_spot = s0;
    hp.disc_from_later.assign(rows, 1.0);
    hp.disc_to_origin.assign(rows, 1.0);
    PlanLayout L = layout_for(hp, 1, 1);
    e = executor->scratch.reserve(L.total);
    if (e.ok()) e = executor->staging.reserve(std::max(L.inputs_bytes, L.out_bytes));
    if (e.ok() && !states_on_device) e = executor->slab.reserve(sizeof(double) * rows * paths);
    if (e.ok() && external && !normals_on_device) e = executor->normals.reserve(sizeof(double) * n_normals);
    if (!e.ok()) return e;
    unsigned char* dev = static_cast<unsigned char*>(executor->scratch.ptr);
    pack_inputs(hp, L, static_cast<unsigned char*>(executor->staging.ptr));
    cudaStream_t s = executor->stream;
    DevicePlan dp = device_plan(hp, L, dev, 0);
    auto* status = reinterpret_cast<DeviceStatus*>(dev + L.status);
    double* out = states_on_device ? states : static_cast<double*>(executor->slab.ptr);
    const double* d_normals = normals;
    FO_CUDA_TRY(cudaMemcpyAsync(dev, executor->staging.ptr, L.inputs_bytes, cudaMemcpyHostToDevice, s), "upload");
    FO_CUDA_TRY(cudaMemsetAsync(status, 0xff, kStatusNoneBytes, s), "reset");
    if (external) {
        if (!normals_on_device) {
            FO_CUDA_TRY(cudaMemcpyAsync(executor->normals.ptr, normals, sizeof(double) * n_normals,
                                        cudaMemcpyHostToDevice, s),
                        "normals upload");
            d_normals = static_cast<const double*>(executor->normals.ptr);
        }
        // Every variate is checked before any path is computed (path.rs:596-603).
        unsigned long long first = 0;
        FO_CUDA_TRY(launch_first_nonfinite(d_normals, n_normals, &status->eval_sim_fail, s), "normals check");
        FO_CUDA_TRY(cudaMemcpyAsync(&first, &status->eval_sim_fail, sizeof(first), cudaMemcpyDeviceToHost, s), "status");
        FO_CUDA_TRY(cudaStreamSynchronize(s), "normals check");
        if (first != kNone) {
            double observed = 0.0;
            FO_CUDA_TRY(cudaMemcpyAsync(&observed, d_normals + first, sizeof(double), cudaMemcpyDeviceToHost, s),
                        "normal copy");
            FO_CUDA_TRY(cudaStreamSynchronize(s), "normal copy");
            Error ne = make_error(FO_ERR_SIMULATION, FO_CODE_NON_FINITE_NORMAL_BUFFER,
                                  "standard-normal buffer contains a non-finite value at interval " +
                                      std::to_string(first / paths) + ", path " + std::to_string(first % paths) + ": " +
                                      fmt_f64(observed));
            ne.path = int64_t(first % paths);
            return ne;
        }
        FO_CUDA_TRY(launch_simulate_external(dp, paths, d_normals, out, &status->train_sim_fail, s), "simulation launch");
    } else {
        FO_CUDA_TRY(launch_simulate(dp, paths, q.seed, q.domain, out, 0, 0, &status->train_sim_fail, s),
                    "simulation launch");
    }
    unsigned long long fail = 0;
    FO_CUDA_TRY(cudaMemcpyAsync(&fail, &status->train_sim_fail, sizeof(fail), cudaMemcpyDeviceToHost, s), "status");
    FO_CUDA_TRY(cudaStreamSynchronize(s), "simulation");
    if (fail != kNone) {
        auto* d_replay = reinterpret_cast<SimFailure*>(dev + L.replay);
        SimFailure f{};
        if (external)
            FO_CUDA_TRY(launch_replay_external(dp, paths, d_normals, fail, d_replay, s), "replay");
        else
            FO_CUDA_TRY(launch_replay(dp, q.seed, q.domain, uint32_t(fail), -1, d_replay, s), "replay");
        FO_CUDA_TRY(cudaMemcpyAsync(&f, d_replay, sizeof(f), cudaMemcpyDeviceToHost, s), "replay copy");
        FO_CUDA_TRY(cudaStreamSynchronize(s), "replay");
        Error se = make_error(FO_ERR_SIMULATION, simulation_failure_code(f.code),
                              simulation_failure_message(f.code, uint32_t(f.interval), fail, f.spot, f.normal));
        se.path = int64_t(fail);
        return se;
    }
    if (!states_on_device) {
        FO_CUDA_TRY(cudaMemcpyAsync(states, out, sizeof(double) * rows * paths, cudaMemcpyDeviceToHost, s), "states copy");
        FO_CUDA_TRY(cudaStreamSynchronize(s), "states copy");
    }
    return Error{};
}

// The standalone simulation exports classify failures as the reference's Python boundary does
// (IntoPySimulationError, crates/finoptions-python/src/lib.rs:277-292): non-finite transitions and
// exhausted or rejected random draws stay SimulationErrors, every other simulation failure (spot,
// path count, buffer lengths, non-finite normals, escrowed forwards) is an InputError.
Error simulation_entry_error(Error e) {
    if (e.kind == FO_ERR_SIMULATION && e.code != FO_CODE_NON_FINITE_PATH_TRANSITION &&
        e.code != FO_CODE_RANDOM_NORMAL_BUDGET_EXHAUSTED && e.code != FO_CODE_RANDOM_NORMAL_REJECTION_LIMIT)
        e.kind = FO_ERR_INPUT;
    return e;
}

int finish(fo_error* err, const Error& e) {
    if (!e.ok()) write_error(err, e);
    return e.kind;
}

Error require(const void* p, const char* what) {
    if (!p) return make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT, std::string(what) + " must not be NULL");
    return Error{};
}

}  // namespace

// =============================================================================================
// extern "C"
// =============================================================================================

extern "C" {

int fo_cuda_executor_create(int32_t device, fo_executor** out, fo_error* err) {
    Error e = require(out, "executor output");
    if (!e.ok()) return finish(err, e);
    auto ex = std::make_unique<fo_executor>();
    e = open_device(device, ex.get());
    if (!e.ok()) return finish(err, e);
    *out = ex.release();
    return FO_OK;
}

void fo_executor_destroy(fo_executor* executor) {
    if (!executor) return;
    cudaSetDevice(executor->device);
    if (executor->stream) {
        cudaStreamSynchronize(executor->stream);
        cudaStreamDestroy(executor->stream);
    }
    if (executor->side) {
        cudaStreamSynchronize(executor->side);
        cudaStreamDestroy(executor->side);
    }
    delete executor;
}

int fo_executor_device(const fo_executor* executor, int32_t* device) {
    if (!executor || !device) return FO_ERR_EXECUTION;
    *device = executor->device;
    return FO_OK;
}

int fo_lsm_call_plan_create(fo_executor* executor, const fo_lsm_call_request* request, fo_lsm_call_plan** out,
                            fo_error* err) {
    Error e = require(executor, "executor");
    if (e.ok()) e = require(request, "request");
    if (e.ok()) e = require(out, "plan output");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(executor->mu);
    cudaSetDevice(executor->device);
    return finish(err, plan_create(executor, *request, true, out));
}

int fo_lsm_call_plan_launch(fo_lsm_call_plan* plan, fo_error* err) {
    Error e = require(plan, "plan");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(plan->ex->mu);
    cudaSetDevice(plan->ex->device);
    return finish(err, plan_launch(plan));
}

int fo_lsm_call_plan_collect(fo_lsm_call_plan* plan, fo_lsm_call_result* result, fo_error* err) {
    Error e = require(plan, "plan");
    if (e.ok()) e = require(result, "result");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(plan->ex->mu);
    cudaSetDevice(plan->ex->device);
    return finish(err, plan_collect(plan, result));
}

int fo_lsm_call_plan_time_launches(fo_lsm_call_plan* plan, uint32_t iterations, double* elapsed_ms, double* kernel_ms,
                                   uint64_t kernel_capacity, fo_error* err) {
    Error e = require(plan, "plan");
    if (e.ok()) e = require(elapsed_ms, "elapsed_ms");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(plan->ex->mu);
    cudaSetDevice(plan->ex->device);
    return finish(err, plan_time_launches(plan, iterations, elapsed_ms, kernel_ms, kernel_capacity));
}

int fo_lsm_call_plan_transfer_bytes(const fo_lsm_call_plan* plan, uint64_t* h2d_bytes, uint64_t* d2h_bytes) {
    if (!plan || !h2d_bytes || !d2h_bytes) return FO_ERR_EXECUTION;
    *h2d_bytes = plan->lay.inputs_bytes;
    *d2h_bytes = plan->lay.out_bytes;
    return FO_OK;
}

int fo_lsm_call_plan_kernel_count(const fo_lsm_call_plan* plan, uint64_t* kernels) {
    if (!plan || !kernels) return FO_ERR_EXECUTION;
    *kernels = kernels_per_launch(plan);
    return FO_OK;
}

int fo_lsm_call_plan_stream(const fo_lsm_call_plan* plan, void** stream) {
    if (!plan || !stream) return FO_ERR_EXECUTION;
    *stream = plan->ex->stream;
    return FO_OK;
}

void fo_lsm_call_plan_destroy(fo_lsm_call_plan* plan) {
    if (!plan) return;
    {
        std::lock_guard<std::mutex> lock(plan->ex->mu);
        cudaSetDevice(plan->ex->device);
        cudaStreamSynchronize(plan->ex->stream);
    }
    delete plan;
}

int fo_price_lsm_call_f64(fo_executor* executor, const fo_lsm_call_request* request, fo_lsm_call_result* result,
                          fo_error* err) {
    Error e = require(executor, "executor");
    if (e.ok()) e = require(request, "request");
    if (e.ok()) e = require(result, "result");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(executor->mu);
    cudaSetDevice(executor->device);
    fo_lsm_call_plan* raw = nullptr;
    e = plan_create(executor, *request, false, &raw);
    if (!e.ok()) return finish(err, e);
    std::unique_ptr<fo_lsm_call_plan> plan(raw);
    e = plan_launch(plan.get());
    if (e.ok()) e = plan_collect(plan.get(), result);
    else cudaStreamSynchronize(executor->stream);  // the input upload may still read the staging
    return finish(err, e);
}

int fo_price_lsm_call_greeks_f64(fo_executor* executor, const fo_lsm_call_request* request, fo_lsm_call_result* result,
                                 fo_lsm_call_greeks* greeks, fo_error* err) {
    Error e = require(executor, "executor");
    if (e.ok()) e = require(request, "request");
    if (e.ok()) e = require(result, "result");
    if (e.ok()) e = require(greeks, "greeks");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(executor->mu);
    cudaSetDevice(executor->device);
    fo_lsm_call_plan* raw = nullptr;
    e = plan_create(executor, *request, false, &raw);
    if (!e.ok()) return finish(err, e);
    std::unique_ptr<fo_lsm_call_plan> plan(raw);
    e = enable_greeks(plan.get(), true);
    if (e.ok()) e = plan_launch(plan.get());
    if (e.ok()) e = plan_collect(plan.get(), result);
    else cudaStreamSynchronize(executor->stream);  // the input upload may still read the staging
    if (e.ok()) e = plan_greeks(plan.get(), greeks);
    return finish(err, e);
}

int fo_lsm_call_plan_set_greeks(fo_lsm_call_plan* plan, int32_t enabled, fo_error* err) {
    Error e = require(plan, "plan");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(plan->ex->mu);
    return finish(err, enable_greeks(plan, enabled != 0));
}

int fo_lsm_call_plan_greeks(fo_lsm_call_plan* plan, fo_lsm_call_greeks* greeks, fo_error* err) {
    Error e = require(plan, "plan");
    if (e.ok()) e = require(greeks, "greeks");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(plan->ex->mu);
    return finish(err, plan_greeks(plan, greeks));
}

int fo_lsm_call_plan_stopping_rows(fo_lsm_call_plan* plan, uint32_t* rows, uint64_t capacity, fo_error* err) {
    Error e = require(plan, "plan");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(plan->ex->mu);
    cudaSetDevice(plan->ex->device);
    return finish(err, plan_stopping_rows(plan, rows, capacity));
}

int fo_lsm_call_plan_revalue_f64(fo_lsm_call_plan* plan, const fo_lsm_call_request* market, fo_lsm_call_result* result,
                                 fo_error* err) {
    Error e = require(plan, "plan");
    if (e.ok()) e = require(market, "market");
    if (e.ok()) e = require(result, "result");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(plan->ex->mu);
    cudaSetDevice(plan->ex->device);
    return finish(err, plan_revalue(plan, *market, result));
}

int fo_simulate_gbm_seeded_f64(fo_executor* executor, const fo_gbm_seeded_request* q, double* states, uint64_t out_len,
                               fo_error* err) {
    Error e = require(executor, "executor");
    if (e.ok()) e = require(q, "request");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(executor->mu);
    cudaSetDevice(executor->device);
    return finish(err, simulation_entry_error(simulate_gbm(executor, *q, nullptr, 0, false, states, out_len, false)));
}

int fo_simulate_gbm_f64(fo_executor* executor, const fo_gbm_seeded_request* q, const double* normals,
                        uint64_t normal_rows, double* states, uint64_t out_len, fo_error* err) {
    Error e = require(executor, "executor");
    if (e.ok()) e = require(q, "request");
    if (e.ok()) e = require(normals, "normals");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(executor->mu);
    cudaSetDevice(executor->device);
    return finish(err, simulation_entry_error(simulate_gbm(executor, *q, normals, normal_rows, false, states, out_len, false)));
}

int fo_simulate_gbm_device_f64(fo_executor* executor, const fo_gbm_seeded_request* q, const double* device_normals,
                               uint64_t normal_rows, double* device_states, uint64_t out_len, fo_error* err) {
    Error e = require(executor, "executor");
    if (e.ok()) e = require(q, "request");
    if (!e.ok()) return finish(err, e);
    std::lock_guard<std::mutex> lock(executor->mu);
    cudaSetDevice(executor->device);
    return finish(err, simulation_entry_error(simulate_gbm(executor, *q, device_normals, normal_rows, true, device_states, out_len, true)));
}

int fo_sample_standard_normals_f64(fo_executor* executor, uint64_t seed, uint32_t domain, uint32_t path_start,
                                   uint64_t paths, uint32_t normals_per_path, double* out, uint64_t out_len,
                                   fo_error* err) {
    Error e = require(executor, "executor");
    if (e.ok()) e = require(out, "output");
    if (!e.ok()) return finish(err, e);
    if (out_len != paths * uint64_t(normals_per_path) || uint64_t(path_start) + paths > (1ull << 32))
        return finish(err, make_error(FO_ERR_EXECUTION, FO_CODE_INVALID_ARGUMENT,
                                      "normal buffer must hold paths * normals_per_path values within the u32 path domain"));
    std::lock_guard<std::mutex> lock(executor->mu);
    cudaSetDevice(executor->device);
    const size_t bytes = sizeof(double) * out_len + 256;
    e = executor->slab.reserve(bytes);
    if (!e.ok()) return finish(err, e);
    cudaStream_t s = executor->stream;
    auto run = [&]() -> Error {
        auto* fail = reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(executor->slab.ptr) + sizeof(double) * out_len);
        FO_CUDA_TRY(cudaMemsetAsync(fail, 0xff, sizeof(unsigned long long), s), "reset");
        FO_CUDA_TRY(launch_normals(seed, domain, path_start, paths, normals_per_path, static_cast<double*>(executor->slab.ptr),
                                   fail, s),
                    "normals launch");
        unsigned long long f = 0;
        FO_CUDA_TRY(cudaMemcpyAsync(&f, fail, sizeof(f), cudaMemcpyDeviceToHost, s), "status");
        FO_CUDA_TRY(cudaStreamSynchronize(s), "normals");
        if (f != kNone) {
            Error se = make_error(FO_ERR_SIMULATION, FO_CODE_RANDOM_NORMAL_REJECTION_LIMIT,
                                  "standard-normal generation failed at path " + std::to_string(uint64_t(path_start) + f));
            se.path = int64_t(path_start + f);
            return se;
        }
        FO_CUDA_TRY(cudaMemcpy(out, executor->slab.ptr, sizeof(double) * out_len, cudaMemcpyDeviceToHost), "copy");
        return Error{};
    };
    return finish(err, run());
}

int fo_build_info(char* buf, uint64_t capacity) {
    if (!buf || capacity == 0) return FO_ERR_EXECUTION;
    int runtime = 0;
    cudaRuntimeGetVersion(&runtime);
    std::snprintf(buf, capacity, "%s;nvcc %d.%d;sm_100a;cudart %d", FO_PACKAGE_VERSION, __CUDACC_VER_MAJOR__,
                  __CUDACC_VER_MINOR__, runtime);
    return FO_OK;
}

// ---- host-only validation -----------------------------------------------------------------------

int fo_validate_cash_dividend_amount(double amount, fo_error* err) { return finish(err, validate_cash_dividend(1, amount)); }

int fo_validate_constant_volatility(double sigma, fo_error* err) { return finish(err, validate_constant_volatility(sigma)); }

int fo_validate_event_schedule(const double* times, uint64_t n_times, const uint32_t* dividend_nodes,
                               uint64_t n_dividend_nodes, const double* dividend_amounts, uint64_t n_dividend_amounts,
                               const uint32_t* exercise_nodes, uint64_t n_exercise_nodes, uint32_t expiry_node,
                               fo_error* err) {
    std::vector<double> t(times, times + n_times);
    std::vector<uint32_t> dn(dividend_nodes, dividend_nodes + n_dividend_nodes);
    std::vector<double> da(dividend_amounts, dividend_amounts + n_dividend_amounts);
    std::vector<uint32_t> ex(exercise_nodes, exercise_nodes + n_exercise_nodes);
    return finish(err, validate_event_schedule(t, dn, da, ex, expiry_node));
}

int fo_validate_log_discount_curve(const double* times, uint64_t n_times, const double* log_discounts, uint64_t n,
                                   fo_error* err) {
    std::vector<double> t(times, times + n_times), v(log_discounts, log_discounts + n);
    return finish(err, validate_log_discount_curve(t, v));
}

int fo_validate_cumulative_dividend_yield_curve(const double* times, uint64_t n_times, const double* yields, uint64_t n,
                                                fo_error* err) {
    std::vector<double> t(times, times + n_times), v(yields, yields + n);
    return finish(err, validate_cumulative_yield_curve(t, v));
}

int fo_validate_ragged_cash_dividends(const int64_t* offsets, uint64_t n_offsets, const double* times, uint64_t n_times,
                                      const double* amounts, uint64_t n_amounts, fo_error* err) {
    return finish(err, validate_ragged_cash(offsets, n_offsets, times, n_times, amounts, n_amounts));
}

int fo_validate_ragged_exercise_times(const int64_t* offsets, uint64_t n_offsets, const double* times, uint64_t n_times,
                                      fo_error* err) {
    return finish(err, validate_ragged_exercise(offsets, n_offsets, times, n_times));
}

int fo_validate_lsm_call_request(const fo_lsm_call_request* request, fo_error* err) {
    Error e = require(request, "request");
    if (!e.ok()) return finish(err, e);
    HostPlan hp;
    return finish(err, build_call_plan(*request, &hp));
}

}  // extern "C"

// =============================================================================================
// Allocation-free pricing: the whole pass (plan inputs, training-path slab, partials, status and
// results) runs in one file-scope device array, so a call makes no device allocation. For callers
// whose device memory belongs to another allocator (a framework's caching allocator or a pool
// reserved at start-up that forbids further driver allocations), and for latency-critical callers
// that cannot absorb cudaMalloc/cudaFree's implicit device-wide synchronisation. Every GPU that
// loads this library holds the array until the process exits.
// =============================================================================================

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[FO_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;

// What the allocation-free entry needs to know about a device, looked up on its first call there
// (with the device current) and kept: the array's device address - in host code the symbol is only
// a host-side stand-in, never a device address - and the launch shapes.
struct NoallocDevice {
    bool ready = false;
    unsigned char* scratch = nullptr;
    int sms = 0;
    int backward_blocks_max = 0;
    int backward_max_ppt = 0;
};
NoallocDevice g_noalloc_devices[256];

Error noalloc_device(int device, NoallocDevice* out) {
    if (device < 0 || device >= 256)
        return make_error(FO_ERR_EXECUTION, FO_CODE_NO_DEVICE, "device ordinal outside the supported range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoallocDevice& d = g_noalloc_devices[device];
    if (!d.ready) {
        int major = 0, minor = 0, cooperative = 0;
        FO_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device), "cudaDeviceGetAttribute");
        FO_CUDA_TRY(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device), "cudaDeviceGetAttribute");
        FO_CUDA_TRY(cudaDeviceGetAttribute(&cooperative, cudaDevAttrCooperativeLaunch, device), "cudaDeviceGetAttribute");
        if (major != 10 || minor != 0)
            return make_error(FO_ERR_EXECUTION, FO_CODE_UNSUPPORTED_DEVICE,
                              "allocation-free pricing requires an sm_100 (Blackwell B200) device; device " +
                                  std::to_string(device) + " is sm_" + std::to_string(major) + std::to_string(minor));
        if (!cooperative)
            return make_error(FO_ERR_EXECUTION, FO_CODE_UNSUPPORTED_DEVICE, "device does not support cooperative launches");
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress of the allocation-free scratch");
        FO_CUDA_TRY(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
        d.scratch = static_cast<unsigned char*>(p);
        d.backward_blocks_max = backward_max_blocks(device);
        d.backward_max_ppt = backward_max_ppt();
        d.ready = true;
    }
    *out = d;
    return Error{};
}

Error price_noalloc(const fo_lsm_call_request& q, cudaStream_t stream, fo_lsm_call_result* result) {
    int device = 0;
    FO_CUDA_TRY(cudaGetDevice(&device), "cudaGetDevice");
    NoallocDevice dev_info;
    Error e = noalloc_device(device, &dev_info);
    if (!e.ok()) return e;
    unsigned char* scratch = dev_info.scratch;
    // A stack executor carries the caller's stream and the device's launch shapes; it owns no
    // memory and creates nothing.
    fo_executor shadow;
    shadow.device = device;
    shadow.sms = dev_info.sms;
    shadow.stream = stream;
    shadow.backward_blocks_max = dev_info.backward_blocks_max;
    shadow.backward_max_ppt = dev_info.backward_max_ppt;
    shadow.eval_blocks_per_sm = 8;
    fo_lsm_call_plan plan;
    plan.ex = &shadow;
    e = build_call_plan(q, &plan.hp);
    if (!e.ok()) return e;
    const HostPlan& hp = plan.hp;
    if (q.evaluation_paths == 0) {
        plan.eval_error = make_error(FO_ERR_LSM, FO_CODE_EMPTY_PATH_SET,
                                     "LSM evaluation simulation failed: simulation path count must be positive");
    } else if (q.evaluation_paths > 0xffffffffull) {
        plan.eval_error = make_error(FO_ERR_LSM, FO_CODE_RANDOM_PATH_NAMESPACE_OVERFLOW,
                                     "LSM evaluation simulation failed: seeded simulation supports at most 4294967295 "
                                     "paths in one random domain; observed " + std::to_string(q.evaluation_paths));
    }
    plan.run_eval = plan.eval_error.ok();
    e = choose_backward_shape(&shadow, hp.train_paths, &plan.backward_blocks, &plan.ppt, &plan.backward_hbm);
    if (!e.ok()) return e;
    const uint64_t eval_needed = plan.run_eval ? (hp.eval_paths + kEvalThreads - 1) / kEvalThreads : 1;
    plan.eval_blocks = int(std::max<uint64_t>(1, std::min<uint64_t>(eval_needed, uint64_t(shadow.sms) * 8)));
    plan.first_stored_row = hp.origin_row ? 1u : 0u;
    plan.lay = layout_for(hp, plan.backward_blocks, plan.eval_blocks);
    const PlanLayout& L = plan.lay;
    const uint64_t stored_rows = hp.rows() - plan.first_stored_row;
    const uint64_t slab_bytes = uint64_t(sizeof(double)) * stored_rows * hp.train_paths +
                                (plan.backward_hbm ? uint64_t(sizeof(double)) * hp.train_paths : 0);
    const uint64_t needed = uint64_t(L.total) + slab_bytes;
    if (needed > FO_NOALLOC_SCRATCH_BYTES)
        return make_error(FO_ERR_EXECUTION, FO_CODE_CAPACITY_EXCEEDED,
                          "request needs " + std::to_string(needed) +
                              " bytes of device scratch; the allocation-free entry point holds at most " +
                              std::to_string(uint64_t(FO_NOALLOC_SCRATCH_BYTES)) +
                              " bytes (training paths x stored rows x 8 bytes plus the plan block)");
    std::vector<unsigned char> host(std::max(L.inputs_bytes, L.out_bytes));
    plan.d_block = scratch;
    plan.d_slab = reinterpret_cast<double*>(scratch + L.total);
    plan.h_out = host.data();
    plan.dp = device_plan(hp, L, scratch, plan.first_stored_row);
    pack_inputs(hp, L, host.data());
    FO_CUDA_TRY(cudaMemcpyAsync(scratch, host.data(), L.inputs_bytes, cudaMemcpyHostToDevice, stream), "plan upload");
    e = plan_launch(&plan);  // clears the status and result region before the kernels run
    if (!e.ok()) return e;
    return plan_collect(&plan, result);
}

}  // namespace

extern "C" int fo_price_lsm_call_f64_noalloc(const fo_lsm_call_request* request, void* cuda_stream,
                                             fo_lsm_call_result* result, fo_error* err) {
    Error e = require(request, "request");
    if (e.ok()) e = require(result, "result");
    if (!e.ok()) return finish(err, e);
    return finish(err, price_noalloc(*request, static_cast<cudaStream_t>(cuda_stream), result));
}

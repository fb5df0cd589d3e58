// lsm_kernels.cu - sm_100a kernels of the single-contract LSM path.
//
//   K1 simulate_kernel     Philox -> ZIGNOR -> GBM -> event phases, one thread per path; stores the
//                          observed rows time-major [rows, paths] with coalesced row stores
//                          (path/seeded.rs:399-474 fused with the transpose).
//   K2 backward_kernel     persistent cooperative kernel: backward induction over exercise rows
//                          with every thread's discounted values held in shared memory; one grid-wide
//                          reduction of in-the-money power sums per row, then each CTA solves the
//                          continuation regression redundantly and applies the exercise rule
//                          (policy.rs:215-296, 471-601).
//   K3 diagnose_kernel     rank / condition diagnostic per fitted row, off the critical path
//                          (regression.rs:540-577).
//   K4 evaluate_kernel     re-simulates the evaluation population and applies the fixed policy on
//                          the fly: no path storage (policy.rs:642-834).
//   K5 finalize_kernel     price / standard error from the CTA partials (policy.rs:891-926).
//   replay_kernel          re-runs one failing path to recover the typed failure details.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "lsm_common.cuh"
#include "lsm_device.cuh"
#include "lsm_fit_warp.cuh"
#include "lsm_kernels.h"
#include "lsm_sync.cuh"

namespace fo {

// Asynchronous 8-byte global -> shared copies (cp.async): issued before a row's reduction, barrier
// and solve, waited for just before the pass that reads them.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

constexpr int kCombineWarps = kSlots;  // warps 0..15 wait for and combine the CTA partials
constexpr int kCombineThreads = kCombineWarps * 32;

// Run by the combine warps only (they meet at named barrier 1). Warp 0 waits for every CTA's arrival;
// then warp k < S sums slot k of the partials over the CTAs in block order (double-double, the
// same fixed order in every CTA). The partials are slot-major, [k][block], so a warp's loads are
// contiguous: every CTA reads every CTA's partials, and the block-major layout made each lane's
// load a separate sector. *wait_failed is 1 when the wait timed out (out is not written).
template <int S>
__device__ __forceinline__ void combine_published(const double2* partials, unsigned seq, DeviceStatus* st, dd* out,
                                                  int* wait_failed) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int blocks = int(gridDim.x);
    if (warp == 0) {
        const bool ok = wait_arrivals(st, seq * unsigned(blocks));
        if (lane == 0) *wait_failed = ok ? 0 : 1;
    }
    named_barrier_sync(1, kCombineThreads);
    if (*wait_failed) return;
    if (warp < S) {
        constexpr int kBatch = 8;  // first eight partials of the lane in flight together
        double2 v[kBatch];
#pragma unroll
        for (int i = 0; i < kBatch; ++i) {
            const int b = lane + 32 * i;
            v[i] = b < blocks ? __ldcg(&partials[warp * blocks + b]) : make_double2(0.0, 0.0);
        }
        dd acc = dd_make(0.0);
#pragma unroll
        for (int i = 0; i < kBatch; ++i)
            if (lane + 32 * i < blocks) acc = dd_add(acc, dd{v[i].x, v[i].y});
        for (int b = lane + 32 * kBatch; b < blocks; b += 32) {
            const double2 w = __ldcg(&partials[warp * blocks + b]);
            acc = dd_add(acc, dd{w.x, w.y});
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc = dd_add(acc, shfl_dd_down(acc, off));
        if (lane == 0) out[warp] = acc;
    }
    named_barrier_sync(1, kCombineThreads);
}

// ---------------------------------------------------------------------------------------------
// Normals export
// ---------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(256) normals_kernel(uint64_t seed, uint32_t domain, uint32_t path_start,
                                                      uint64_t paths, uint32_t count, double* out,
                                                      unsigned long long* fail) {
    __shared__ double sx[257], sf[257];
    load_zig_tables(sx, sf);
    const SmemZig zig = make_zig(sx, sf);
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < paths;
         p += uint64_t(gridDim.x) * blockDim.x) {
        PathStream s;
        s.init(seed, domain, uint32_t(path_start + p), count);
        for (uint32_t k = 0; k < count; ++k) {
            double z = 0.0;
            const int status = zig_sample(s, zig, &z);
            if (status != kNormalOk) {
                atomicMin(fail, (unsigned long long)p);
                break;
            }
            out[p * count + k] = z;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// K1: seeded simulation with time-major row stores.
// ---------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(256) simulate_kernel(DevicePlan plan, uint64_t paths, uint64_t seed,
                                                       uint32_t domain, double* out, uint32_t store_first_row,
                                                       int reconstruct_escrowed, unsigned long long* fail) {
    __shared__ double sx[257], sf[257];
    load_zig_tables(sx, sf);
    const SmemZig zig = make_zig(sx, sf);
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < paths;
         p += uint64_t(gridDim.x) * blockDim.x) {
        auto store = [&](int row, double value) {
            if (uint32_t(row) < store_first_row) return;
            if (reconstruct_escrowed) {
                // Escrowed observations: origin -> S0; otherwise prepaid forward + prepaid cash.
                value = plan.row_node[row] == 0 ? plan.initial_spot : value + plan.escrow_cash[row];
            }
            out[uint64_t(row - store_first_row) * paths + p] = value;
        };
        const SimResult r = simulate_path(plan, zig, seed, domain, uint32_t(p), store);
        if (r.code != 0) atomicMin(fail, (unsigned long long)p);
    }
}

// External normals: the lowest index of a non-finite value in the [intervals, paths] buffer.
__global__ void __launch_bounds__(256) first_nonfinite_kernel(const double* values, uint64_t n,
                                                              unsigned long long* first) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        if (!fo_isfinite(values[i])) atomicMin(first, (unsigned long long)i);
}

// K1 driven by caller normals: one thread per path, time-major [rows, paths] stores.
__global__ void __launch_bounds__(256) simulate_external_kernel(DevicePlan plan, uint64_t paths, const double* normals,
                                                                double* out, unsigned long long* fail) {
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < paths;
         p += uint64_t(gridDim.x) * blockDim.x) {
        const SimResult r = simulate_path_external(plan, normals, paths, p,
                                                   [&](int row, double value) { out[uint64_t(row) * paths + p] = value; });
        if (r.code != 0) atomicMin(fail, (unsigned long long)p);
    }
}

__global__ void replay_external_kernel(DevicePlan plan, uint64_t paths, const double* normals, uint64_t path,
                                       SimFailure* out) {
    if (threadIdx.x != 0) return;
    const SimResult r = simulate_path_external(plan, normals, paths, path, [](int, double) {});
    out->code = r.code;
    out->interval = r.interval;
    out->spot = r.spot;
    out->normal = r.normal;
    out->observed = 0.0;
}

// Re-runs one path serially to recover the typed failure details and the state at `want_row`.
__global__ void replay_kernel(DevicePlan plan, uint64_t seed, uint32_t domain, uint32_t path, int want_row,
                              SimFailure* out) {
    __shared__ double sx[257], sf[257];
    load_zig_tables(sx, sf);
    if (threadIdx.x != 0) return;
    const SmemZig zig = make_zig(sx, sf);
    double observed = 0.0;
    const SimResult r = simulate_path(plan, zig, seed, domain, path, [&](int row, double v) {
        if (row == want_row) observed = v;
    });
    out->code = r.code;
    out->interval = r.interval;
    out->spot = r.spot;
    out->normal = r.normal;
    out->observed = observed;
}

// ---------------------------------------------------------------------------------------------
// K2: persistent backward induction.
// ---------------------------------------------------------------------------------------------

struct BackwardSmem {
    double red[32 * kSlots];
    dd total[kSlots];
    FitModel model;
    double new_pivot;  // the row's own mean, when its sums are taken again about it
    int kind;
    int wait_failed;
};

// Decision of warp 0 that the row's sums must be taken again about its own mean (pivot_too_far)
// before it is fitted; not a rule kind of any record.
constexpr int kRecenterRow = -1;

// This thread's in-the-money paths of the row being decided, summed about `pivot` and reduced over
// the CTA into dst (the classification of each path is the main pass's). Out of line: it runs only
// when the pivot lies far from the row's mean, and keeps the backward loop's registers untouched.
template <bool kHbm>
__device__ __noinline__ void recenter_partial(const double* values_smem, const double* values_hbm,
                                              const double* spots_smem, const double* row_spots, uint64_t P,
                                              uint64_t gtid, uint64_t nthreads, int ppt, double K, Divisor Kd,
                                              double pivot, double* red, double2* dst, unsigned blocks) {
    RowSums s;
#pragma unroll
    for (int k = 0; k < kSlots; ++k) s.acc[k] = 0.0;
    for (int j = 0; j < ppt; ++j) {
        const uint64_t p = gtid + uint64_t(j) * nthreads;
        if (p >= P) break;
        const double sp = kHbm ? __ldcg(&row_spots[p]) : spots_smem[j * blockDim.x + threadIdx.x];
        if (!(sp > K)) continue;
        const double x = divide(sp, Kd);
        const double y = kHbm ? values_hbm[p] : values_smem[j * blockDim.x + threadIdx.x];
        if (!fo_isfinite(x) || !fo_isfinite(y)) s.acc[kBadSlot] += 1.0;
        else accumulate_itm(s, x, y, pivot);
    }
    cta_reduce_to<kSlots>(s.acc, red, dst, blocks);
}

// Each thread owns paths gtid + j * nthreads (j < ppt). When the population fits on chip
// (kHbm false), their discounted values, the current row's spots and the staged row's spots live
// in this CTA's shared memory ([j * blockDim + tid]) for the whole backward pass, so the only HBM
// traffic is one read of each stored row. Larger populations (kHbm true) keep each path's value in
// HBM at a.values[p] and read the spots straight from the stored rows; the arithmetic and its order
// are the same, so a path's decisions do not depend on where its value lives.
//
// Per exercise row k the CTA reduces its in-the-money power sums of row k and publishes them;
// then the warps split. Warps 0..15 wait for every CTA's partial, combine them and warp 0 fits
// row k's continuation (lsm_fit_warp.cuh). Meanwhile warps 16..31 take row k-1, whose spots were prefetched with
// cp.async: its in-the-money test and the power sums T_0..T_8 of its moneyness do not depend on
// row k's exercise decision, so they are accumulated while the grid synchronises and the fit
// runs. After a CTA barrier every thread applies row k's exercise rule to its paths, discounts
// them to row k-1 (policy.rs:1049-1063) and adds the response sums U_0..U_4, which need the
// decided values. Row k-1's sums are taken about the mean of the latest fitted row available when
// its staging starts (two rows later than row k-1); any pivot near the in-the-money mean serves.
template <int D, bool kHbm>  // D == plan.degree (launch_backward dispatches on it)
__global__ void __launch_bounds__(kBackwardThreads, 1) backward_kernel(BackwardArgs a) {
    __shared__ BackwardSmem sm;
    extern __shared__ double backward_dyn[];
    const DevicePlan& plan = a.plan;
    if (*(const volatile unsigned long long*)&a.status->train_sim_fail != kNone)
        return;  // training simulation failed: every CTA reads the same word and leaves
    const int ppt = a.ppt;
    const int T = blockDim.x;
    const int warp = threadIdx.x >> 5;
    const bool stager = warp >= kCombineWarps;
    const int stage_threads = T - kCombineThreads;
    const int stage_tid = int(threadIdx.x) - kCombineThreads;
    // On chip: values, the spots of the row being decided, and the spots of the row being staged
    // (filled by cp.async while the current row is reduced and solved); the two spot buffers
    // alternate.
    double* values = backward_dyn;
    double* spots = backward_dyn + size_t(ppt) * T;
    double* spots_next = backward_dyn + 2 * size_t(ppt) * T;
    const uint64_t P = plan.train_paths;
    const uint64_t nthreads = uint64_t(gridDim.x) * T;
    const uint64_t block_first = uint64_t(blockIdx.x) * T;
    const uint64_t gtid = block_first + threadIdx.x;
    const double K = plan.strike;
    const Divisor Kd = make_divisor(K);
    const int degree = plan.degree;
    const uint32_t rows = plan.rows;
    const uint32_t E = rows - 1;
    const uint32_t fsr = plan.first_stored_row;
    const int lowest = plan.origin_row ? 1 : 0;
    auto row_ptr = [&](uint32_t row) { return a.slab + uint64_t(row - fsr) * P; };
    // Value of this thread's j-th path (p = gtid + j * nthreads < P): shared memory or HBM.
    auto value = [&](int j) -> double& {
        if constexpr (kHbm) return a.values[gtid + uint64_t(j) * nthreads];
        else return values[j * T + threadIdx.x];
    };
    {
        const double* terminal = row_ptr(E);
#pragma unroll 4
        for (int j = 0; j < ppt; ++j) {
            const uint64_t p = gtid + uint64_t(j) * nthreads;
            double v = 0.0;
            if (p < P) {
                const double d = __ldcs(&terminal[p]) - K;
                v = d > 0.0 ? d : 0.0;
            }
            if (!kHbm || p < P) value(j) = v;
        }
    }
    double2* parts = a.partials;
    int parity = 0;
    unsigned seq = 0;
    uint32_t order = 0;
    int row = int(E) - 1;
    double fit_pivot = 1.0;    // pivot of the sums being reduced
    double latest_mean = 1.0;  // mean of the latest fitted row: pivot of the row staged next
    RowSums sums;
#pragma unroll
    for (int k = 0; k < kSlots; ++k) sums.acc[k] = 0.0;
    if (row >= lowest) {
        // Stage the first fitted row and locate its in-the-money mean (the moment pivot).
        const double disc = plan.disc_from_later[row];
        const double* srow = row_ptr(uint32_t(row));
        double loc[2] = {0.0, 0.0};
#pragma unroll 4
        for (int j = 0; j < ppt; ++j) {
            const uint64_t p = gtid + uint64_t(j) * nthreads;
            double sp = 0.0, x = 0.0;
            if (p < P) {
                sp = __ldcs(&srow[p]);
                const double v = value(j) * disc;
                value(j) = v;
                if (!fo_isfinite(v)) atomicMin(&a.status->fit_payoff_fail, ((unsigned long long)order << 32) | p);
                if (sp > K) {
                    x = divide(sp, Kd);
                    if (fo_isfinite(x)) {
                        loc[0] += 1.0;
                        loc[1] += x;
                    }
                }
            }
            if constexpr (!kHbm) spots[j * T + threadIdx.x] = sp;
        }
        cta_reduce_to<2>(loc, sm.red, parts + size_t(parity) * a.partial_stride + blockIdx.x, gridDim.x);
        publish_partial(a.status);
        ++seq;
        if (!stager)
            combine_published<2>(parts + size_t(parity) * a.partial_stride, seq, a.status, sm.total,
                                 &sm.wait_failed);
        __syncthreads();
        if (sm.wait_failed) return;
        parity ^= 1;
        if (sm.total[0].hi > 0.0) fit_pivot = dd_round(dd_div(sm.total[1], sm.total[0]));
        latest_mean = fit_pivot;
        for (int j = 0; j < ppt; ++j) {
            const uint64_t p = gtid + uint64_t(j) * nthreads;
            if (kHbm && p >= P) break;
            const double sp = kHbm ? __ldcg(&srow[p]) : spots[j * T + threadIdx.x];
            if (sp > K) {
                const double x = divide(sp, Kd), y = value(j);
                if (!fo_isfinite(x) || !fo_isfinite(y)) {
                    sums.acc[kBadSlot] += 1.0;
                    atomicMin(&a.status->fit_nonfinite, ((unsigned long long)order << 32) | p);
                } else {
                    accumulate_itm(sums, x, y, fit_pivot);
                }
            }
        }
    }
    for (; row >= lowest; --row, ++order) {
        const bool stage_next = row - 1 >= lowest;
        const double stage_pivot = latest_mean;
        cta_reduce_to<kSlots>(sums.acc, sm.red, parts + size_t(parity) * a.partial_stride + blockIdx.x, gridDim.x);
        publish_partial(a.status);
        ++seq;
#pragma unroll
        for (int k = 0; k < kSlots; ++k) sums.acc[k] = 0.0;
        if (!kHbm && stage_next && stager) {
            // Load the next row's spots for the positions this thread stages (after the release
            // above, which would otherwise wait for these loads).
            const double* srow = row_ptr(uint32_t(row - 1));
            for (int j = 0; j < ppt; ++j) {
                for (int t = stage_tid; t < T; t += stage_threads) {
                    const uint64_t p = block_first + uint64_t(t) + uint64_t(j) * nthreads;
                    if (p < P) cp_async8(&spots_next[j * T + t], &srow[p]);
                }
            }
            cp_async_commit();
        }
        // Warp 0 decides the row from the combined totals (the same in every lane and every CTA) and
        // fits it, or first asks for the row's sums about its own mean (once per row).
        auto decide_row = [&](bool allow_recenter) {
            const uint64_t itm = uint64_t(sm.total[0].hi);
            const uint64_t bad = uint64_t(sm.total[kBadSlot].hi);
            const uint64_t population = itm + bad;
            const uint32_t required = uint32_t(degree + 1);
            int kind;
            double mean = fit_pivot;
            if (population == 0) {
                kind = plan.support == 1 ? kRuleContinue : kRuleNoSupport;
            } else if (population < required && plan.support == 1) {
                kind = kRuleContinue;
            } else if (population < required || bad > 0) {
                kind = kRuleFitFailed;  // InsufficientObservations / non-finite population
            } else if (allow_recenter && degree > 0 && pivot_too_far(sm.total, fit_pivot, itm, &mean)) {
                kind = kRecenterRow;
                if (threadIdx.x == 0) sm.new_pivot = mean;
            } else {
                fit_continuation_warp(sm.total, fit_pivot, itm, degree, plan.rank_tolerance, plan.rank_limit,
                                      &sm.model);
                kind = sm.model.status == kFitOk ? kRuleRegression : kRuleFitFailed;
            }
            if (threadIdx.x == 0) sm.kind = kind;
            if (blockIdx.x == 0 && kind != kRecenterRow) {
                // CTA 0 writes the row's record; the model goes out as twelve 16-byte words from
                // as many lanes (a one-thread copy made CTA 0 the last to arrive at the next sync).
                FitRecord& rec = a.records[row];
                constexpr int kModelWords = int(sizeof(FitModel) / sizeof(double2));
                static_assert(sizeof(FitModel) % sizeof(double2) == 0, "FitModel is 16-byte aligned");
                if (threadIdx.x < kModelWords)
                    reinterpret_cast<double2*>(&rec.model)[threadIdx.x] =
                        reinterpret_cast<const double2*>(&sm.model)[threadIdx.x];
                if (threadIdx.x == 0) {
                    rec.kind = kind;
                    rec.itm = population;
                    rec.pivot = fit_pivot;
                    rec.origin_exercise = 0;
                    rec.origin_continuation = 0.0;
                    rec.diag_status = -1;
                    if (kind == kRuleFitFailed) atomicMin(&a.status->fit_failed_order, order);
                }
            }
        };
        if (!stager) {
            combine_published<kSlots>(parts + size_t(parity) * a.partial_stride, seq, a.status, sm.total,
                                      &sm.wait_failed);
            if (threadIdx.x < 32 && !sm.wait_failed) decide_row(true);
        } else if (stage_next) {
            // Row k-1: in-the-money test and power sums, independent of row k's decision.
            const double* srow = row_ptr(uint32_t(row - 1));
            if constexpr (!kHbm) cp_async_wait_all();
            for (int j = 0; j < ppt; ++j) {
                for (int t = stage_tid; t < T; t += stage_threads) {
                    const uint64_t p = block_first + uint64_t(t) + uint64_t(j) * nthreads;
                    if (p >= P) continue;
                    const double sp = kHbm ? __ldcg(&srow[p]) : spots_next[j * T + t];
                    if (sp > K) {
                        const double x = divide(sp, Kd);
                        if (!fo_isfinite(x)) {
                            sums.acc[kBadSlot] += 1.0;
                            atomicMin(&a.status->fit_nonfinite, ((unsigned long long)(order + 1) << 32) | p);
                        } else {
                            accumulate_powers(sums, x - stage_pivot);
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (sm.wait_failed) return;
        if (sm.kind == kRecenterRow) {
            // One more grid exchange: every CTA sums the row about its mean and warp 0 fits it.
            fit_pivot = sm.new_pivot;
            parity ^= 1;
            recenter_partial<kHbm>(values, a.values, spots, row_ptr(uint32_t(row)), P, gtid, nthreads, ppt, K, Kd,
                                   fit_pivot, sm.red, parts + size_t(parity) * a.partial_stride + blockIdx.x,
                                   gridDim.x);
            publish_partial(a.status);
            ++seq;
            if (!stager) {
                combine_published<kSlots>(parts + size_t(parity) * a.partial_stride, seq, a.status, sm.total,
                                          &sm.wait_failed);
                if (threadIdx.x < 32 && !sm.wait_failed) decide_row(false);
            }
            __syncthreads();
            if (sm.wait_failed) return;
        }
        const int kind = sm.kind;
        if (kind == kRuleFitFailed) return;  // identical decision in every CTA
        const bool regression = kind == kRuleRegression;
        const FitModel& model = sm.model;  // read from shared memory
        const double disc = stage_next ? plan.disc_from_later[row - 1] : 1.0;
        const double* cur_row = row_ptr(uint32_t(row));
        const double* next_row = stage_next ? row_ptr(uint32_t(row - 1)) : cur_row;
#pragma unroll 2
        for (int j = 0; j < ppt; ++j) {
            const uint64_t p = gtid + uint64_t(j) * nthreads;
            const int at = j * T + threadIdx.x;
            if (p >= P) continue;
            double v = value(j);
            if (regression) {
                const double sp = kHbm ? __ldcg(&cur_row[p]) : spots[at];
                if (sp > K) {
                    const double intrinsic = sp - K;
                    double continuation;
                    if (!predict_continuation_d<D>(model, divide(sp, Kd), &continuation)) {
                        atomicMin(&a.status->fit_predict_fail, ((unsigned long long)order << 32) | p);
                    } else if (exercise_rule(plan.tie_rule, intrinsic, continuation)) {
                        v = intrinsic;
                    }
                }
            }
            if (stage_next) {
                const double sp = kHbm ? __ldcg(&next_row[p]) : spots_next[at];
                v *= disc;
                if (!fo_isfinite(v))
                    atomicMin(&a.status->fit_payoff_fail, ((unsigned long long)(order + 1) << 32) | p);
                if (sp > K) {
                    const double x = divide(sp, Kd);
                    if (fo_isfinite(x)) {  // a non-finite x was counted by the staging warps
                        if (!fo_isfinite(v)) {
                            // excluded from the regression: move the path from the count to the bad slot
                            sums.acc[0] -= 1.0;
                            sums.acc[kBadSlot] += 1.0;
                            atomicMin(&a.status->fit_nonfinite, ((unsigned long long)(order + 1) << 32) | p);
                        } else {
                            accumulate_responses(sums, x - stage_pivot, v);
                        }
                    }
                }
            }
            value(j) = v;
        }
        double* swap = spots;
        spots = spots_next;
        spots_next = swap;
        fit_pivot = stage_pivot;
        if (regression) latest_mean = model.mean;
        // Consecutive exchanges use alternate partial buffers: a CTA overwrites a buffer only after
        // every CTA has arrived at the exchange in between, that is, has finished reading it.
        parity ^= 1;
    }
    // Common origin decision (policy.rs:265-281): mean of values discounted to the origin.
    if (plan.origin_row) {
        double acc[2] = {0.0, 0.0};
        for (int j = 0; j < ppt; ++j) {
            const uint64_t p = gtid + uint64_t(j) * nthreads;
            if (p < P) {
                const double w = value(j) * plan.origin_discount;
                if (!fo_isfinite(w))
                    atomicMin(&a.status->fit_payoff_fail, ((unsigned long long)order << 32) | p);
                acc[0] += 1.0;
                acc[1] += w;
            }
        }
        cta_reduce_to<2>(acc, sm.red, parts + size_t(parity) * a.partial_stride + blockIdx.x, gridDim.x);
        publish_partial(a.status);
        ++seq;
        if (!stager)
            combine_published<2>(parts + size_t(parity) * a.partial_stride, seq, a.status, sm.total,
                                 &sm.wait_failed);
        if (blockIdx.x == 0 && threadIdx.x == 0 && !sm.wait_failed) {
            const double mean = dd_round(dd_div(sm.total[1], sm.total[0]));
            const double intrinsic = plan.initial_spot - K > 0.0 ? plan.initial_spot - K : 0.0;
            FitRecord& rec = a.records[0];
            rec.kind = kRuleOrigin;
            rec.origin_exercise = exercise_rule(plan.tie_rule, intrinsic, mean) ? 1 : 0;
            rec.origin_continuation = mean;
            rec.itm = 0;
            rec.diag_status = -1;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// K3: diagnostics for regression rows.
// ---------------------------------------------------------------------------------------------

__global__ void diagnose_kernel(DevicePlan plan, FitRecord* records) {
    const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row + 1 >= plan.rows) return;
    FitRecord& rec = records[row];
    if (rec.kind != kRuleRegression) return;
    int rank = 0, aux = 0;
    double condition = 0.0;
    rec.diag_status = diagnose_design(rec.model, plan.degree, plan.rank_tolerance, plan.condition_limit, &rank,
                                      &condition, &aux);
    rec.diag_rank = rank;
    rec.diag_condition = condition;
    rec.diag_aux = aux;
}

// ---------------------------------------------------------------------------------------------
// K4: fused re-simulation + fixed-policy evaluation.
// ---------------------------------------------------------------------------------------------

struct EvalRow {
    FitModel model;
    int32_t kind;
    int32_t pad;
    double discount;
};

template <int D>
__global__ void __launch_bounds__(kEvalThreads, 4) evaluate_kernel(EvalArgs a) {
    extern __shared__ __align__(16) unsigned char eval_smem_raw[];
    const DevicePlan& plan = a.plan;
    const uint32_t rows = plan.rows;
    double* sx = reinterpret_cast<double*>(eval_smem_raw);
    double* sf = sx + 257;
    double* red = sf + 257;                                      // [32 * 2]
    EvalRow* rules = reinterpret_cast<EvalRow*>(red + 64);       // [rows]
    unsigned* counts = reinterpret_cast<unsigned*>(rules + rows);    // [rows]
    unsigned* itm_counts = counts + rows;                            // [rows]
    for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) {
        EvalRow er;
        if (r + 1 < rows) {
            er.model = a.records[r].model;
            er.kind = a.records[r].kind;
        } else {
            er.kind = kRuleNone;
        }
        er.discount = plan.disc_to_origin[r];
        rules[r] = er;
        counts[r] = 0;
        itm_counts[r] = 0;
    }
    load_zig_tables(sx, sf);
    const SmemZig zig = make_zig(sx, sf);
    const double K = plan.strike;
    const Divisor Kd = make_divisor(K);
    const uint64_t P = plan.eval_paths;
    double sum = 0.0, sumsq = 0.0;
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < P; p += uint64_t(gridDim.x) * blockDim.x) {
        bool active = true;
        double payoff = 0.0;
        auto observe = [&](int row, double spot) {
            if (!active) return;
            const EvalRow& er = rules[row];
            if (uint32_t(row) + 1 == rows) {
                const double d = spot - K;
                payoff = (d > 0.0 ? d : 0.0) * er.discount;
                if (!fo_isfinite(payoff)) atomicMin(&a.status->eval_terminal_fail, (unsigned long long)p);
                active = false;
                atomicAdd(&counts[row], 1u);
                if (a.stops) a.stops[p] = uint32_t(row);
                return;
            }
            if (er.kind == kRuleNoSupport) {
                if (spot > K) atomicAdd(&itm_counts[row], 1u);
                return;
            }
            if (er.kind != kRuleRegression || !(spot > K)) return;
            const double intrinsic = spot - K;
            double continuation;
            if (!predict_continuation_d<D>(er.model, divide(spot, Kd), &continuation)) {
                atomicMin(&a.status->eval_fail, ((unsigned long long)row << 33) | (p << 1));
                return;
            }
            if (exercise_rule(plan.tie_rule, intrinsic, continuation)) {
                payoff = intrinsic * er.discount;
                if (!fo_isfinite(payoff))
                    atomicMin(&a.status->eval_fail, ((unsigned long long)row << 33) | (p << 1) | 1ull);
                active = false;
                atomicAdd(&counts[row], 1u);
                if (a.stops) a.stops[p] = uint32_t(row);
            }
        };
        const SimResult r = simulate_path(plan, zig, plan.eval_seed, plan.eval_domain, uint32_t(p), observe);
        if (r.code != 0) atomicMin(&a.status->eval_sim_fail, (unsigned long long)p);
        sum += payoff;
        sumsq += payoff * payoff;
    }
    double acc[2] = {sum, sumsq};
    cta_reduce_to<2>(acc, red, a.partials + size_t(blockIdx.x) * 2);
    for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) {
        if (counts[r]) atomicAdd(&a.counts[r], counts[r]);
        if (itm_counts[r]) atomicAdd(&a.itm_counts[r], itm_counts[r]);
    }
}

// ---------------------------------------------------------------------------------------------
// K5: price and standard error.
// ---------------------------------------------------------------------------------------------

__global__ void finalize_kernel(const double2* partials, int blocks, uint64_t paths, double* out) {
    __shared__ dd total[2];
    grid_combine<2>(partials, blocks, total);
    if (threadIdx.x == 0) {
        const dd n = dd_make(double(paths));
        const dd mean = dd_div(total[0], n);
        // M2 = sum x^2 - (sum x)^2 / n
        dd m2 = dd_sub(total[1], dd_mul(total[0], mean));
        if (m2.hi < 0.0) m2 = dd_make(0.0);
        out[0] = dd_round(mean);
        out[1] = dd_round(m2);
        if (paths > 1) {
            const dd var = dd_div(m2, dd_make(double(paths - 1)));
            const double sd = dd_round(dd_sqrt(var));
            out[2] = sd;
            out[3] = sd / sqrt(double(paths));
        } else {
            out[2] = 0.0;
            out[3] = 0.0;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Host-callable launchers
// ---------------------------------------------------------------------------------------------

cudaError_t launch_normals(uint64_t seed, uint32_t domain, uint32_t path_start, uint64_t paths, uint32_t count,
                           double* out, unsigned long long* fail, cudaStream_t stream) {
    const int threads = 256;
    const uint64_t blocks = (paths + threads - 1) / threads;
    normals_kernel<<<unsigned(blocks < 65535 * 16 ? blocks : 65535 * 16), threads, 0, stream>>>(
        seed, domain, path_start, paths, count, out, fail);
    return cudaGetLastError();
}

cudaError_t launch_simulate(const DevicePlan& plan, uint64_t paths, uint64_t seed, uint32_t domain, double* out,
                            uint32_t store_first_row, int reconstruct_escrowed, unsigned long long* fail,
                            cudaStream_t stream) {
    const int threads = 256;
    uint64_t blocks = (paths + threads - 1) / threads;
    if (blocks > (1u << 20)) blocks = 1u << 20;
    simulate_kernel<<<unsigned(blocks), threads, 0, stream>>>(plan, paths, seed, domain, out, store_first_row,
                                                               reconstruct_escrowed, fail);
    return cudaGetLastError();
}

cudaError_t launch_first_nonfinite(const double* values, uint64_t n, unsigned long long* first, cudaStream_t stream) {
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148u * 16u);
    first_nonfinite_kernel<<<unsigned(std::max<uint64_t>(blocks, 1)), 256, 0, stream>>>(values, n, first);
    return cudaGetLastError();
}

cudaError_t launch_simulate_external(const DevicePlan& plan, uint64_t paths, const double* normals, double* out,
                                     unsigned long long* fail, cudaStream_t stream) {
    uint64_t blocks = (paths + 255) / 256;
    if (blocks > (1u << 20)) blocks = 1u << 20;
    simulate_external_kernel<<<unsigned(blocks), 256, 0, stream>>>(plan, paths, normals, out, fail);
    return cudaGetLastError();
}

cudaError_t launch_replay_external(const DevicePlan& plan, uint64_t paths, const double* normals, uint64_t path,
                                   SimFailure* out, cudaStream_t stream) {
    replay_external_kernel<<<1, 32, 0, stream>>>(plan, paths, normals, path, out);
    return cudaGetLastError();
}

cudaError_t launch_replay(const DevicePlan& plan, uint64_t seed, uint32_t domain, uint32_t path, int want_row,
                          SimFailure* out, cudaStream_t stream) {
    replay_kernel<<<1, 32, 0, stream>>>(plan, seed, domain, path, want_row, out);
    return cudaGetLastError();
}

size_t backward_smem_bytes(int ppt) { return sizeof(double) * 3 * size_t(ppt) * kBackwardThreads; }

int backward_max_ppt() {
    // Dynamic shared memory available next to the kernel's static shared memory.
    cudaFuncAttributes attr{};
    cudaFuncGetAttributes(&attr, backward_kernel<kMaxDegree, false>);  // every degree has the same static shared memory
    int optin = 0, device = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    const size_t avail = size_t(optin) > attr.sharedSizeBytes ? size_t(optin) - attr.sharedSizeBytes : 0;
    return int(avail / (sizeof(double) * 3 * kBackwardThreads));
}

int backward_max_blocks(int device) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return sms;  // one 1024-thread CTA per SM; the dynamic shared memory keeps it at one
}

template <int D, bool kHbm>
static cudaError_t launch_backward_d(const BackwardArgs& args, int blocks, int ppt, cudaStream_t stream) {
    const size_t smem = kHbm ? 0 : backward_smem_bytes(ppt);
    cudaError_t e = cudaFuncSetAttribute(backward_kernel<D, kHbm>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, backward_kernel<D, kHbm>, kBackwardThreads, smem);
    if (e != cudaSuccess) return e;
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (per_sm < 1 || blocks > per_sm * sms) return cudaErrorCooperativeLaunchTooLarge;
    void* params[] = {const_cast<BackwardArgs*>(&args)};
    return cudaLaunchCooperativeKernel((const void*)backward_kernel<D, kHbm>, dim3(blocks), dim3(kBackwardThreads),
                                       params, smem, stream);
}

template <bool kHbm>
static cudaError_t launch_backward_storage(const BackwardArgs& args, int blocks, int ppt, cudaStream_t stream) {
    switch (args.plan.degree) {  // validated to 0..4 on the host
        case 0: return launch_backward_d<0, kHbm>(args, blocks, ppt, stream);
        case 1: return launch_backward_d<1, kHbm>(args, blocks, ppt, stream);
        case 2: return launch_backward_d<2, kHbm>(args, blocks, ppt, stream);
        case 3: return launch_backward_d<3, kHbm>(args, blocks, ppt, stream);
        default: return launch_backward_d<4, kHbm>(args, blocks, ppt, stream);
    }
}

cudaError_t launch_backward(const BackwardArgs& args, int blocks, int ppt, cudaStream_t stream) {
    return args.values ? launch_backward_storage<true>(args, blocks, ppt, stream)
                       : launch_backward_storage<false>(args, blocks, ppt, stream);
}

cudaError_t launch_diagnose(const DevicePlan& plan, FitRecord* records, cudaStream_t stream) {
    const unsigned rows = plan.rows;
    diagnose_kernel<<<(rows + 63) / 64, 64, 0, stream>>>(plan, records);
    return cudaGetLastError();
}

size_t evaluate_smem_bytes(uint32_t rows) {
    return sizeof(double) * (257 * 2 + 64) + sizeof(EvalRow) * rows + sizeof(unsigned) * 2 * rows;
}

template <int D>
static cudaError_t launch_evaluate_d(const EvalArgs& args, int blocks, size_t smem, cudaStream_t stream) {
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(evaluate_kernel<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    evaluate_kernel<D><<<blocks, kEvalThreads, smem, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_evaluate(const EvalArgs& args, int blocks, cudaStream_t stream) {
    const size_t smem = evaluate_smem_bytes(args.plan.rows);
    switch (args.plan.degree) {  // validated to 0..4 on the host
        case 0: return launch_evaluate_d<0>(args, blocks, smem, stream);
        case 1: return launch_evaluate_d<1>(args, blocks, smem, stream);
        case 2: return launch_evaluate_d<2>(args, blocks, smem, stream);
        case 3: return launch_evaluate_d<3>(args, blocks, smem, stream);
        default: return launch_evaluate_d<4>(args, blocks, smem, stream);
    }
}

cudaError_t launch_finalize(const double2* partials, int blocks, uint64_t paths, double* out, cudaStream_t stream) {
    finalize_kernel<<<1, 64, 0, stream>>>(partials, blocks, paths, out);
    return cudaGetLastError();
}

}  // namespace fo

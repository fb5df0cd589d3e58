/*
 * finoptions_cuda.h - C ABI of the B200 Longstaff-Schwartz engine.
 *
 * Plain C types only: pointers, sizes, enums and caller-owned buffers. Every entry point returns
 * an fo_status and, on failure, fills the caller's fo_error with the failure category, the
 * row/group/node/path it concerns and a message worded like the reference's typed errors.
 * No partial result is ever written on failure.
 *
 * Reference interfaces each entry replaces (paths inside jorgensandhaug/finoptions-engine):
 *   fo_cuda_executor_create      - CpuExecutor construction, crates/finoptions-python/src/lib.rs:167-186
 *                                   and crates/finoptions-runtime/src/lib.rs:341-443 (the new
 *                                   CudaExecutor sits beside CpuExecutor; explicit, fail-fast,
 *                                   no CPU fallback)
 *   fo_price_lsm_call_f64        - price_lsm_call_seeded_f64, crates/finoptions-python/src/lib.rs:1169-1241
 *   fo_price_lsm_grouped_f64     - price_lsm_call_grouped_batch_{continuous_yield,cash_dividends,
 *                                   escrowed_cash_dividends}_f64, crates/finoptions-python/src/lib.rs:1884-2100
 *   fo_price_lsm_batch_f64       - price_lsm_call_batch_*_f64 (row-addressed batch; one contract per
 *                                   group), crates/finoptions-lsm/src/batch/pricing.rs:191-300
 *   fo_simulate_gbm_seeded_f64   - simulate_gbm_seeded_f64, crates/finoptions-python/src/lib.rs:1019-1058
 *   fo_sample_standard_normals_f64 - PhiloxPathStream + sample_standard_normal,
 *                                   crates/finoptions-sim/src/random/{philox,normal}.rs
 *   fo_build_info                - build_info, crates/finoptions-python/src/lib.rs:400-404
 */
#ifndef FINOPTIONS_CUDA_H
#define FINOPTIONS_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FO_ABI_VERSION 1

/* ---- status / error ------------------------------------------------------------------------ */

typedef enum fo_status {
    FO_OK = 0,
    FO_ERR_INPUT = 1,      /* InputError(ValueError): request/validation failures            */
    FO_ERR_LSM = 2,        /* LsmError(RuntimeError): simulation/regression/support/evaluation */
    FO_ERR_SIMULATION = 3, /* SimulationError(RuntimeError)                                  */
    FO_ERR_EXECUTION = 4,  /* ExecutionError(RuntimeError): device/executor failures         */
    FO_ERR_BATCH = 5       /* BatchError(ValueError): ragged-view structure failures         */
} fo_status;

#define FO_ERROR_MESSAGE_CAPACITY 1024

typedef struct fo_error {
    int32_t kind;  /* fo_status of the failure                                    */
    int32_t code;  /* fo_error_code: the typed reference error it corresponds to   */
    int64_t row;   /* contract row, -1 when not applicable                         */
    int64_t group; /* strike group, -1 when not applicable                         */
    int64_t node;  /* grid node, -1 when not applicable                            */
    int64_t path;  /* path index, -1 when not applicable                           */
    char message[FO_ERROR_MESSAGE_CAPACITY];
} fo_error;

/* fo_error.code: which typed reference error a failure corresponds to. */
typedef enum fo_error_code {
    FO_CODE_NONE = 0,
    /* InputError (crates/finoptions-core/src/error.rs) */
    FO_CODE_EMPTY_TIME_GRID = 100,
    FO_CODE_INVALID_TIME_ORIGIN,
    FO_CODE_NON_FINITE_TIME,
    FO_CODE_NON_INCREASING_TIME,
    FO_CODE_TOO_MANY_NODES,
    FO_CODE_NODE_OUT_OF_BOUNDS,
    FO_CODE_CURVE_LENGTH_MISMATCH,
    FO_CODE_INVALID_DISCOUNT_ORIGIN,
    FO_CODE_NON_FINITE_LOG_DISCOUNT,
    FO_CODE_UNREPRESENTABLE_INTERVAL_DISCOUNT,
    FO_CODE_DIVIDEND_YIELD_CURVE_LENGTH_MISMATCH,
    FO_CODE_INVALID_CUMULATIVE_DIVIDEND_YIELD_ORIGIN,
    FO_CODE_INVALID_CUMULATIVE_DIVIDEND_YIELD,
    FO_CODE_DECREASING_CUMULATIVE_DIVIDEND_YIELD,
    FO_CODE_UNREPRESENTABLE_INTERVAL_DIVIDEND_YIELD,
    FO_CODE_INVALID_CASH_DIVIDEND,
    FO_CODE_INVALID_EXPIRY_NODE,
    FO_CODE_DUPLICATE_DIVIDEND_NODE,
    FO_CODE_UNORDERED_DIVIDEND_NODE,
    FO_CODE_INVALID_DIVIDEND_NODE,
    FO_CODE_DUPLICATE_EXERCISE_NODE,
    FO_CODE_UNORDERED_EXERCISE_NODE,
    FO_CODE_INVALID_EXERCISE_NODE,
    FO_CODE_DIVIDEND_COLUMN_LENGTH_MISMATCH,
    FO_CODE_INVALID_CONSTANT_VOLATILITY,
    FO_CODE_UNSUPPORTED_ENUM,
    /* SimulationError (crates/finoptions-sim/src/error.rs) */
    FO_CODE_TIME_GRID_MISMATCH = 200,
    FO_CODE_DIVIDEND_YIELD_TIME_GRID_MISMATCH,
    FO_CODE_EMPTY_PATH_SET,
    FO_CODE_RANDOM_PATH_NAMESPACE_OVERFLOW,
    FO_CODE_INVALID_INITIAL_SPOT,
    FO_CODE_NON_POSITIVE_ESCROWED_PREPAID_FORWARD,
    FO_CODE_NON_FINITE_ESCROWED_PREPAID_CASH,
    FO_CODE_NON_FINITE_ESCROWED_OBSERVATION,
    FO_CODE_RANDOM_NORMAL_BUDGET_EXHAUSTED,
    FO_CODE_RANDOM_NORMAL_REJECTION_LIMIT,
    FO_CODE_NON_FINITE_PATH_TRANSITION,
    FO_CODE_SHAPE_OVERFLOW,
    FO_CODE_BUFFER_LENGTH_MISMATCH,
    FO_CODE_NON_FINITE_NORMAL_BUFFER,
    /* RegressionError (crates/finoptions-lsm/src/error.rs:1-160) */
    FO_CODE_UNSUPPORTED_DEGREE = 300,
    FO_CODE_INVALID_RANK_TOLERANCE,
    FO_CODE_INVALID_CONDITION_LIMIT,
    FO_CODE_INSUFFICIENT_OBSERVATIONS,
    FO_CODE_NON_FINITE_PREDICTOR,
    FO_CODE_NON_FINITE_RESPONSE,
    FO_CODE_DEGENERATE_PREDICTOR,
    FO_CODE_RANK_DEFICIENT,
    FO_CODE_CONDITION_LIMIT_EXCEEDED,
    FO_CODE_CONDITION_DIAGNOSTIC_DID_NOT_CONVERGE,
    FO_CODE_NON_FINITE_FIT,
    FO_CODE_NON_FINITE_PREDICTION,
    /* LsmError (crates/finoptions-lsm/src/error.rs:160-319) */
    FO_CODE_INVALID_STRIKE = 400,
    FO_CODE_LSM_INVALID_INITIAL_SPOT,
    FO_CODE_PATH_COUNT_OUTSIDE_DOMAIN,
    FO_CODE_UNREPRESENTABLE_OBSERVATION_DISCOUNT,
    FO_CODE_EVALUATION_OUTSIDE_TRAINING_SUPPORT,
    FO_CODE_NON_FINITE_DISCOUNTED_PAYOFF,
    FO_CODE_RANDOM_DOMAIN_COLLISION,
    /* BatchLsmError (crates/finoptions-lsm/src/batch/error.rs) */
    FO_CODE_EMPTY_BATCH = 500,
    FO_CODE_ROW_COUNT_MISMATCH,
    FO_CODE_GROUP_OFFSET_COUNT_MISMATCH,
    FO_CODE_GROUP_OFFSETS_DO_NOT_START_AT_ZERO,
    FO_CODE_INVALID_GROUP_RANGE,
    FO_CODE_GROUP_OFFSET_END_MISMATCH,
    FO_CODE_INVALID_ROW_VALUE,
    FO_CODE_EMPTY_BASE_INTERVALS,
    FO_CODE_CASH_MESH_REQUIRES_CASH_DIVIDENDS,
    FO_CODE_NEGATIVE_RATE_FOR_CASH_MESH,
    FO_CODE_TERMINAL_CASH_FOR_CASH_MESH,
    FO_CODE_EXPLICIT_EXERCISE_AT_OR_AFTER_MATURITY,
    FO_CODE_INSUFFICIENT_EVALUATION_PATHS,
    FO_CODE_BATCH_PATH_COUNT_OUTSIDE_DOMAIN,
    FO_CODE_RANDOM_DOMAIN_RANGE_OVERFLOW,
    FO_CODE_RANDOM_DOMAIN_RANGE_COLLISION,
    FO_CODE_CASH_DIVIDEND_AFTER_MATURITY,
    FO_CODE_CASH_DIVIDEND_AT_EXCLUDED_MATURITY,
    FO_CODE_UNSUPPORTED_CASH_MATURITY_BOUNDARY,
    FO_CODE_DUPLICATE_CASH_DIVIDEND_TIME,
    FO_CODE_ESCROWED_NON_FINITE_PREPAID_CASH,
    FO_CODE_ESCROWED_NON_POSITIVE_PREPAID_FORWARD,
    FO_CODE_ESCROWED_INVALID_VOLATILITY,
    FO_CODE_CONTRACT_MESH_SHAPE_OVERFLOW,
    FO_CODE_EXPLICIT_CONTRACT_MESH_SHAPE_OVERFLOW,
    FO_CODE_CASH_DIVIDEND_NODE_MISSING,
    FO_CODE_EXPLICIT_EXERCISE_NODE_MISSING,
    FO_CODE_STOPPING_COUNT_MISMATCH,
    FO_CODE_MISSING_SAMPLING_DIAGNOSTIC,
    /* BatchError (crates/finoptions-batch/src/error.rs) */
    FO_CODE_INSUFFICIENT_OFFSETS = 600,
    FO_CODE_EVENT_COLUMN_LENGTH_MISMATCH,
    FO_CODE_NEGATIVE_OFFSET,
    FO_CODE_DECREASING_OFFSET,
    FO_CODE_OFFSET_SPAN_MISMATCH,
    FO_CODE_OFFSET_INDEX_OVERFLOW,
    FO_CODE_INVALID_EVENT_TIME,
    FO_CODE_DECREASING_EVENT_TIME,
    FO_CODE_INVALID_CASH_AMOUNT,
    FO_CODE_INVALID_EXERCISE_TIME,
    FO_CODE_NON_INCREASING_EXERCISE_TIME,
    /* ExecutionError (device / executor) */
    FO_CODE_NO_DEVICE = 700,
    FO_CODE_UNSUPPORTED_DEVICE,
    FO_CODE_CUDA_FAILURE,
    FO_CODE_BARRIER_TIMEOUT,
    FO_CODE_CAPACITY_EXCEEDED,
    FO_CODE_INVALID_ARGUMENT
} fo_error_code;

/* ---- enums mirroring the reference's string enums (lib.rs:514-556) ------------------------ */

typedef enum fo_dividend_policy {
    FO_DIVIDEND_LIQUIDATOR = 0, /* "liquidator": max(S - D, 0)      (dividend.rs:69-70) */
    FO_DIVIDEND_SURVIVOR = 1    /* "survivor": S > D ? S - D : S    (dividend.rs:71-77) */
} fo_dividend_policy;

typedef enum fo_tie_rule {
    FO_TIE_STRICTLY_GREATER = 0, /* exercise iff intrinsic >  continuation (policy.rs:21-26) */
    FO_TIE_GREATER_OR_EQUAL = 1  /* exercise iff intrinsic >= continuation                   */
} fo_tie_rule;

typedef enum fo_insufficient_support {
    FO_SUPPORT_FAIL = 0,    /* "fail"     (policy.rs:31-37) */
    FO_SUPPORT_CONTINUE = 1 /* "continue"                   */
} fo_insufficient_support;

typedef enum fo_dividend_model {
    FO_MODEL_CONTINUOUS_YIELD = 0,
    FO_MODEL_CASH_DIVIDENDS = 1,
    FO_MODEL_ESCROWED_CASH_DIVIDENDS = 2
} fo_dividend_model;

typedef enum fo_maturity_boundary {
    FO_MATURITY_STRICTLY_BEFORE = 0,
    FO_MATURITY_AT_OR_BEFORE = 1
} fo_maturity_boundary;

typedef enum fo_escrowed_volatility {
    FO_ESCROWED_PREPAID_FORWARD = 0,
    FO_ESCROWED_SPOT_MATCHED_AT_ORIGIN = 1
} fo_escrowed_volatility;

typedef enum fo_exercise_mesh {
    FO_MESH_UNIFORM = 0,
    FO_MESH_CASH_DIVIDEND_DATES = 1,
    FO_MESH_EXPLICIT_TIMES = 2
} fo_exercise_mesh;

typedef enum fo_origin_exercise {
    FO_ORIGIN_EXCLUDED = 0,
    FO_ORIGIN_INCLUDED = 1
} fo_origin_exercise;

typedef enum fo_diag_kind {
    FO_DIAG_ORIGIN_DECISION = 0,        /* ExerciseFitDiagnostics::OriginDecision        */
    FO_DIAG_NO_IN_THE_MONEY_PATHS = 1,  /* ExerciseFitDiagnostics::NoInTheMoneyPaths     */
    FO_DIAG_INSUFFICIENT_SUPPORT = 2,   /* ExerciseFitDiagnostics::InsufficientExerciseSupport */
    FO_DIAG_REGRESSION = 3              /* ExerciseFitDiagnostics::Regression            */
} fo_diag_kind;

/* ---- executor ----------------------------------------------------------------------------- */

typedef struct fo_executor fo_executor;

/* Opens an sm_100 device. Fails with FO_ERR_EXECUTION when the device is absent or is not a
 * compute-capability-10.x part; there is no CPU fallback. The executor owns one CUDA stream and a
 * growable device arena; calls on one executor are serialised. */
int fo_cuda_executor_create(int32_t device, fo_executor** out, fo_error* err);
void fo_executor_destroy(fo_executor* executor);
int fo_executor_device(const fo_executor* executor, int32_t* device);

/* ---- single contract: price_lsm_call ------------------------------------------------------ */

/* Field-for-field image of price_lsm_call_seeded_f64's arguments (lib.rs:1170-1197). */
typedef struct fo_lsm_call_request {
    double initial_spot;
    double strike;
    const double* schedule_times;             uint64_t n_schedule_times;
    const double* curve_times;                uint64_t n_curve_times;
    const double* log_discounts;              uint64_t n_log_discounts;
    const double* dividend_yield_times;       uint64_t n_dividend_yield_times;
    const double* cumulative_dividend_yields; uint64_t n_cumulative_dividend_yields;
    const uint32_t* dividend_nodes;           uint64_t n_dividend_nodes;
    const double* dividend_amounts;           uint64_t n_dividend_amounts;
    const uint32_t* exercise_nodes;           uint64_t n_exercise_nodes;
    uint32_t expiry_node;
    double annualized_volatility;
    int32_t dividend_policy;                  /* fo_dividend_policy */
    uint64_t training_paths;
    uint64_t evaluation_paths;
    uint64_t training_seed;
    uint32_t training_domain;
    uint64_t evaluation_seed;
    uint32_t evaluation_domain;
    uint32_t polynomial_degree;
    double rank_tolerance;
    double condition_limit;
    int32_t tie_rule;                         /* fo_tie_rule */
    int32_t insufficient_exercise_support;    /* fo_insufficient_support */
} fo_lsm_call_request;

/* One ExerciseNodeDiagnostics (policy.rs:39-87), flattened like NativeExerciseDiagnostic
 * (lib.rs:1060-1072). For FO_DIAG_INSUFFICIENT_SUPPORT, `columns` carries required_paths. */
typedef struct fo_lsm_node_diagnostic {
    uint32_t node;
    int32_t kind;                  /* fo_diag_kind */
    int32_t exercise;              /* origin decision only */
    double estimated_continuation; /* origin decision only */
    uint32_t in_the_money_paths;
    uint64_t observations;
    uint64_t columns;
    uint64_t rank;
    double condition_number;
    double predictor_mean;
    double predictor_scale;
} fo_lsm_node_diagnostic;

/* NativeLsmResult (lib.rs:1074-1082). The caller owns every array: observation_nodes and
 * exercise_counts need n_exercise_nodes + 1 entries, diagnostics n_exercise_nodes entries. */
typedef struct fo_lsm_call_result {
    double price;
    uint32_t paths;
    int32_t has_sample_standard_deviation;
    double sample_standard_deviation;
    int32_t has_standard_error;
    double standard_error;
    uint32_t* observation_nodes;         uint64_t observation_capacity;
    uint32_t* exercise_counts;           /* same capacity as observation_nodes */
    uint64_t n_observations;             /* written */
    fo_lsm_node_diagnostic* diagnostics; uint64_t diagnostics_capacity;
    uint64_t n_diagnostics;              /* written */
} fo_lsm_call_result;

int fo_price_lsm_call_f64(fo_executor* executor, const fo_lsm_call_request* request,
                          fo_lsm_call_result* result, fo_error* err);

/* Split form of fo_price_lsm_call_f64 for callers that keep a contract resident on the device:
 * create validates the request and uploads the plan once; launch enqueues the whole pricing pass
 * (simulation, backward fit, evaluation) on the executor's stream without synchronising and
 * without host transfers; collect waits, downloads and assembles the result or the typed error. */
typedef struct fo_lsm_call_plan fo_lsm_call_plan;
int fo_lsm_call_plan_create(fo_executor* executor, const fo_lsm_call_request* request,
                            fo_lsm_call_plan** out, fo_error* err);
int fo_lsm_call_plan_launch(fo_lsm_call_plan* plan, fo_error* err);
int fo_lsm_call_plan_collect(fo_lsm_call_plan* plan, fo_lsm_call_result* result, fo_error* err);
/* Enqueues `iterations` launches of the plan bracketed by CUDA events on the plan's stream, waits
 * for them, and returns the elapsed device time in milliseconds. When kernel_ms is not NULL it
 * receives, per kernel of one launch (in launch order, at most kernel_capacity entries), the device
 * time summed over the iterations. Results stay on the device; collect reads the last launch. */
int fo_lsm_call_plan_time_launches(fo_lsm_call_plan* plan, uint32_t iterations, double* elapsed_ms,
                                   double* kernel_ms, uint64_t kernel_capacity, fo_error* err);
/* Bytes one fo_price_lsm_call_f64 of this request copies host->device and device->host. */
int fo_lsm_call_plan_transfer_bytes(const fo_lsm_call_plan* plan, uint64_t* h2d_bytes, uint64_t* d2h_bytes);
/* Number of kernels one launch enqueues (for launch accounting). */
int fo_lsm_call_plan_kernel_count(const fo_lsm_call_plan* plan, uint64_t* kernels);
/* The cudaStream_t (as void*) the plan's kernels run on. */
int fo_lsm_call_plan_stream(const fo_lsm_call_plan* plan, void** stream);
void fo_lsm_call_plan_destroy(fo_lsm_call_plan* plan);

/* ---- pathwise adjoint Greeks ----------------------------------------------------------------
 * No counterpart in the reference, which obtains sensitivities by bump-and-reprice through
 * price_lsm_call_seeded_f64. The fitted exercise policy is held fixed and the evaluation paths are
 * differentiated pathwise in the same pass that prices them (the price and standard error are the
 * plain entry's, bit for bit): delta = dP/dS0, vega = dP/dsigma, dP/dL_i for every schedule node i
 * (L the log discounts) and dP/dD_j for every cash dividend j in node order. At most
 * FO_MAX_GREEK_DIVIDENDS cash dividends per contract. */
#define FO_MAX_GREEK_DIVIDENDS 8
typedef struct fo_lsm_call_greeks {
    double delta;
    double vega;
    double* log_discount_sensitivities;  uint64_t log_discount_capacity;  /* one per schedule node */
    double* dividend_sensitivities;      uint64_t dividend_capacity;      /* one per cash dividend */
} fo_lsm_call_greeks;

int fo_price_lsm_call_greeks_f64(fo_executor* executor, const fo_lsm_call_request* request,
                                 fo_lsm_call_result* result, fo_lsm_call_greeks* greeks, fo_error* err);
/* Resident-plan form: enable the Greeks on a plan, then read them after a successful collect. */
int fo_lsm_call_plan_set_greeks(fo_lsm_call_plan* plan, int32_t enabled, fo_error* err);
int fo_lsm_call_plan_greeks(fo_lsm_call_plan* plan, fo_lsm_call_greeks* greeks, fo_error* err);
/* Re-values the plan's last fitted policy on `market` without refitting: the market must keep the
 * plan's schedule times, exercise and dividend nodes, strike, path counts, streams and method;
 * the initial spot, log discounts, cumulative yields, cash amounts and volatility may change.
 * (Fixed-policy finite differences and scenario revaluation.) Greeks, when enabled, follow. */
int fo_lsm_call_plan_revalue_f64(fo_lsm_call_plan* plan, const fo_lsm_call_request* market,
                                 fo_lsm_call_result* result, fo_error* err);

/* Every evaluation path's stopping observation row under the plan's fitted policy on its current
 * market (rows[p] for evaluation path p; capacity >= evaluation paths). No counterpart in the
 * reference: a diagnostic that counts, path by path, the exercise decisions in which this engine
 * and another implementation of the same contract differ. It re-runs the evaluation pass. */
int fo_lsm_call_plan_stopping_rows(fo_lsm_call_plan* plan, uint32_t* rows, uint64_t capacity, fo_error* err);

/* Allocation-free variant of fo_price_lsm_call_f64. It has no counterpart in the reference.
 *
 * For callers that cannot allocate device memory: code whose device memory belongs to another
 * allocator (a framework's caching allocator, or a pool reserved at start-up that forbids further
 * driver allocations) and latency-critical code that cannot absorb cudaMalloc / cudaFree's implicit
 * device-wide synchronisation. The call prices on the calling thread's current device and on
 * `cuda_stream` (NULL: the legacy default stream), makes no cudaMalloc, cudaFree or other device
 * allocation, and keeps everything it needs on the device (plan inputs, the training-path slab of
 * training_paths x stored rows x 8 bytes, partials, status, results) in one file-scope device
 * array of FO_NOALLOC_SCRATCH_BYTES (64 MiB) that every GPU loading this library holds until the
 * process exits. Requests that need more return FO_ERR_EXECUTION / FO_CODE_CAPACITY_EXCEEDED.
 * The first call on a device looks up the array's device address and the device's launch shapes
 * (kept for later calls); make that first call before any stream capture. Every call shares the one array and clears what must start at zero itself;
 * calls that overlap on the GPU (two streams, or two threads) race on it and must be serialised
 * by the caller. The call synchronises `cuda_stream` before returning. */
#define FO_NOALLOC_SCRATCH_BYTES (64ull << 20)
int fo_price_lsm_call_f64_noalloc(const fo_lsm_call_request* request, void* cuda_stream,
                                  fo_lsm_call_result* result, fo_error* err);

/* ---- grouped / row batches ------------------------------------------------------------------ */

/* Arguments of price_lsm_call_grouped_batch_*_f64 (lib.rs:1884-2100) with the dividend model and
 * the mesh as tags. Optional buffers are NULL when absent. */
typedef struct fo_lsm_grouped_request {
    const uint32_t* group_offsets;    uint64_t n_group_offsets;
    const double* initial_spots;      uint64_t n_initial_spots;  /* one per group */
    const double* strikes;            uint64_t n_strikes;        /* one per contract row */
    const double* maturities;         uint64_t n_maturities;
    const double* rates;              uint64_t n_rates;
    const double* volatilities;       uint64_t n_volatilities;
    int32_t dividend_model;           /* fo_dividend_model */
    const double* dividend_yields;    uint64_t n_dividend_yields;   /* continuous yield */
    const int64_t* dividend_offsets;  uint64_t n_dividend_offsets;  /* cash / escrowed */
    const double* dividend_times;     uint64_t n_dividend_times;
    const double* dividend_amounts;   uint64_t n_dividend_amounts;
    int32_t dividend_policy;          /* cash dividends */
    int32_t maturity_boundary;        /* cash / escrowed */
    int32_t volatility_convention;    /* escrowed */
    int32_t exercise_mesh;            /* fo_exercise_mesh */
    int32_t has_base_intervals;       uint32_t base_intervals;
    int32_t has_origin_exercise;      int32_t origin_exercise;
    const int64_t* explicit_exercise_offsets; uint64_t n_explicit_exercise_offsets;
    const double* explicit_exercise_times;    uint64_t n_explicit_exercise_times;
    uint64_t training_paths;
    uint64_t evaluation_paths;
    uint64_t training_seed;
    uint32_t training_domain_start;
    uint64_t evaluation_seed;
    uint32_t evaluation_domain_start;
    uint32_t polynomial_degree;
    double rank_tolerance;
    double condition_limit;
    int32_t tie_rule;
    int32_t insufficient_exercise_support;
} fo_lsm_grouped_request;

/* NativeBatchLsmResult (lib.rs:1417-1430): twelve caller-owned row-aligned columns. */
typedef struct fo_batch_result_columns {
    uint64_t rows;
    double* prices;
    double* sample_standard_deviations;
    double* standard_errors;
    uint8_t* origin_decisions_fitted;
    uint8_t* origin_exercised;
    uint32_t* regression_nodes;
    uint32_t* no_training_support_nodes;
    uint32_t* insufficient_exercise_support_nodes;
    uint32_t* minimum_in_the_money_training_paths;
    double* maximum_regression_condition_numbers;
    uint32_t* early_exercise_paths;
    uint32_t* expiry_paths;
} fo_batch_result_columns;

int fo_price_lsm_grouped_f64(fo_executor* executor, const fo_lsm_grouped_request* request,
                             fo_batch_result_columns* out, fo_error* err);

/* Row-addressed batch (price_lsm_call_batch): every column (spots, strikes, maturities, rates,
 * volatilities, dividend rows, explicit schedules) has one entry per contract and group_offsets
 * must be NULL; row r uses domains training_domain_start + r and evaluation_domain_start + r. */
int fo_price_lsm_batch_f64(fo_executor* executor, const fo_lsm_grouped_request* request,
                           fo_batch_result_columns* out, fo_error* err);

/* ---- ragged batches --------------------------------------------------------------------------
 * Independent contracts with their own path counts: no counterpart in the reference, whose batch
 * methods take one training and one evaluation path count per request (input.rs:259-267). Row r
 * is priced like a one-row explicit-mesh batch with domains training_domain_start + r and
 * evaluation_domain_start + r: its own exercise times (strictly inside (0, maturity)), a
 * continuous yield and/or a cash-dividend schedule (exact times merged into the mesh), and its
 * own training / evaluation path counts. */
typedef struct fo_lsm_ragged_request {
    uint64_t rows;
    const double* initial_spots;      /* each column: one entry per contract */
    const double* strikes;
    const double* maturities;
    const double* rates;              /* constant continuously compounded rate: L(t) = -r t */
    const double* volatilities;
    const double* dividend_yields;    /* continuous yields, NULL for none */
    const int64_t* dividend_offsets;  uint64_t n_dividend_offsets;  /* rows + 1, NULL for none */
    const double* dividend_times;     const double* dividend_amounts;  uint64_t n_dividend_events;
    int32_t dividend_policy;          /* fo_dividend_policy of the cash jumps */
    int32_t maturity_boundary;        /* fo_maturity_boundary of the cash schedules */
    const int64_t* exercise_offsets;  uint64_t n_exercise_offsets;  /* rows + 1 */
    const double* exercise_times;     uint64_t n_exercise_times;
    int32_t origin_exercise;          /* fo_origin_exercise */
    const uint64_t* training_paths;   /* per contract */
    const uint64_t* evaluation_paths; /* per contract */
    uint64_t training_seed;
    uint32_t training_domain_start;
    uint64_t evaluation_seed;
    uint32_t evaluation_domain_start;
    uint32_t polynomial_degree;
    double rank_tolerance;
    double condition_limit;
    int32_t tie_rule;
    int32_t insufficient_exercise_support;
} fo_lsm_ragged_request;

/* Per-contract adjoint Greeks of a ragged batch (fixed fitted policies, as fo_lsm_call_greeks):
 * delta and vega per row; dP/dL per node of row r's union mesh at
 * log_discount_sensitivities[log_discount_offsets[r] .. log_discount_offsets[r + 1]) (offsets
 * written by the call; node i of the mesh is 0, the merged exercise / cash times, maturity);
 * dP/dD per cash event, aligned with dividend_times. */
typedef struct fo_ragged_greeks_columns {
    double* delta;
    double* vega;
    double* log_discount_sensitivities;  uint64_t log_discount_capacity;
    int64_t* log_discount_offsets;       /* rows + 1 */
    double* dividend_sensitivities;      /* n_dividend_events */
} fo_ragged_greeks_columns;

/* greeks may be NULL (prices only). */
int fo_price_lsm_ragged_f64(fo_executor* executor, const fo_lsm_ragged_request* request,
                            fo_batch_result_columns* out, fo_ragged_greeks_columns* greeks, fo_error* err);

/* Device time of the executor's last grouped / row / ragged batch call (no counterpart in the
 * reference; a measurement hook). A batch runs as one captured graph per wave (a wave: the groups
 * that fit the device memory budget together) holding either one persistent launch or the phase
 * kernels (fo_batch_tuning.phases): kernel_ms[0] receives the milliseconds of the wave's launches
 * summed over the call's waves; with the phase kernels kernel_ms[1..3] receive the simulation, fit
 * and evaluation (with the summary) kernels' shares (zero otherwise); *launches receives the number
 * of waves. Timed with CUDA events recorded by the graph on the executor's stream. */
#define FO_BATCH_KERNELS 5
int fo_executor_batch_kernel_ms(fo_executor* executor, double* kernel_ms, uint64_t capacity, uint64_t* launches);
/* Host->device and device->host bytes the executor's last batch call copied. */
int fo_executor_batch_transfer_bytes(fo_executor* executor, uint64_t* h2d_bytes, uint64_t* d2h_bytes);

/* ---- batch launch shape (no counterpart in the reference) ------------------------------------
 * A batch wave is one persistent launch whose CTAs take work items from a queue: the training
 * simulation of a block range of one group, the backward fit of one (group, strike) problem, the
 * evaluation of a block range of one group for a chunk of its strikes. Its shape: */
typedef struct fo_batch_tuning {
    int32_t sim_blocks;   /* training-simulation blocks (256 paths each) per work item, 1..64     */
    int32_t eval_blocks;  /* evaluation blocks (256 paths each) per work item, 1..64              */
    int32_t strikes;      /* strikes an evaluation item applies together: 1, 2, 4 or 8            */
    int32_t ctas_per_sm;  /* resident CTAs per SM, 0..8 (0: as many as the registers allow)       */
    int32_t phases;       /* 0: one persistent launch drains every item; 1: one kernel per item    */
                          /* kind (simulation, fits, evaluation) and a summary kernel, each with  */
                          /* its own occupancy                                                    */
} fo_batch_tuning;

/* autotune != 0 (the default): the executor picks the shape per class of wave (path counts, rows,
 * strikes per group, group count, degree, Greeks) by timing a few candidates on the first wave of
 * the class, and keeps the fastest for later waves of the class. autotune == 0: every launch takes
 * *fixed. Every shape gives the same results, bit for bit. */
int fo_executor_set_batch_tuning(fo_executor* executor, int32_t autotune, const fo_batch_tuning* fixed, fo_error* err);

typedef struct fo_batch_launch_info {
    fo_batch_tuning tuning;    /* shape of the last launch (strikes: as launched)          */
    int32_t source;            /* 0: fixed by the caller, 1: tuned earlier, 2: tuned now   */
    int32_t grid;              /* CTAs launched                                            */
    uint64_t items;            /* work items of the last launch                            */
    uint64_t tuning_launches;  /* launches the tuner timed (source 2)                      */
    uint64_t graph_replays;    /* waves of the last call replayed from the captured graph  */
    uint64_t graph_captures;   /* waves of the last call captured (a new launch key)       */
} fo_batch_launch_info;
int fo_executor_batch_launch(fo_executor* executor, fo_batch_launch_info* out);

/* ---- simulation exports --------------------------------------------------------------------- */

typedef struct fo_gbm_seeded_request {
    double initial_spot;
    const double* schedule_times;             uint64_t n_schedule_times;
    const double* curve_times;                uint64_t n_curve_times;
    const double* log_discounts;              uint64_t n_log_discounts;
    const double* dividend_yield_times;       uint64_t n_dividend_yield_times;
    const double* cumulative_dividend_yields; uint64_t n_cumulative_dividend_yields;
    const uint32_t* dividend_nodes;           uint64_t n_dividend_nodes;
    const double* dividend_amounts;           uint64_t n_dividend_amounts;
    const uint32_t* exercise_nodes;           uint64_t n_exercise_nodes;
    uint32_t expiry_node;
    double annualized_volatility;
    int32_t dividend_policy;
    uint64_t paths;
    uint64_t seed;
    uint32_t domain;
} fo_gbm_seeded_request;

/* Time-major [n_exercise_nodes + 1, paths] pre-event states at every exercise node followed by
 * the post-event expiry state (path.rs:948-1024). `states` holds out_len doubles, exactly
 * (n_exercise_nodes + 1) * paths. The three simulation exports return FO_ERR_SIMULATION only for
 * a non-finite path transition or an exhausted / rejected random draw; every other simulation
 * failure (spot, path count, buffer lengths, non-finite normals, escrowed forwards) is
 * FO_ERR_INPUT, as the reference's Python boundary classifies them (lib.rs:277-292). */
int fo_simulate_gbm_seeded_f64(fo_executor* executor, const fo_gbm_seeded_request* request,
                               double* states, uint64_t out_len, fo_error* err);

/* simulate_gbm_f64 (crates/finoptions-python/src/lib.rs:969-1018): the same paths driven by the
 * caller's standard normals instead of Philox streams. normals holds normal_rows x request->paths
 * values, time-major ([interval][path]), and normal_rows must equal the schedule's intervals; the
 * request's seed and domain are not read. Checks run in the reference's order: the plan, the
 * interval rows, the initial spot, the path count, then every normal for finiteness before any path
 * is computed (SimulationError with the interval and path of the first bad value, as
 * GbmPathPlan::validate_execution, path.rs:558-603). */
int fo_simulate_gbm_f64(fo_executor* executor, const fo_gbm_seeded_request* request, const double* normals,
                        uint64_t normal_rows, double* states, uint64_t out_len, fo_error* err);
/* Device-resident form of both simulation exports (no counterpart in the reference): states and
 * normals are device pointers on the executor's device (e.g. a torch tensor's storage); normals ==
 * NULL simulates the request's Philox streams (fo_simulate_gbm_seeded_f64), otherwise the caller's
 * normals (fo_simulate_gbm_f64). Nothing is copied to the host; the call returns once the states
 * are written. */
int fo_simulate_gbm_device_f64(fo_executor* executor, const fo_gbm_seeded_request* request,
                               const double* device_normals, uint64_t normal_rows, double* device_states,
                               uint64_t out_len, fo_error* err);

/* Path-local standard normals: out[p * normals_per_path + k] is the k-th ZIGNOR normal of path
 * path_start + p in namespace (seed, domain), with a normal budget of normals_per_path. */
int fo_sample_standard_normals_f64(fo_executor* executor, uint64_t seed, uint32_t domain,
                                   uint32_t path_start, uint64_t paths, uint32_t normals_per_path,
                                   double* out, uint64_t out_len, fo_error* err);

/* ---- host-only validation (no device needed) ------------------------------------------------ */

/* The reference's validate_* functions (crates/finoptions-python/src/lib.rs:405-473) used by the
 * Python model constructors. They return FO_ERR_INPUT (or FO_ERR_BATCH for ragged buffers) with
 * the reference's message on failure. */
int fo_validate_cash_dividend_amount(double amount, fo_error* err);
int fo_validate_constant_volatility(double annualized_decimal, fo_error* err);
int fo_validate_event_schedule(const double* times, uint64_t n_times, const uint32_t* dividend_nodes,
                               uint64_t n_dividend_nodes, const double* dividend_amounts,
                               uint64_t n_dividend_amounts, const uint32_t* exercise_nodes,
                               uint64_t n_exercise_nodes, uint32_t expiry_node, fo_error* err);
int fo_validate_log_discount_curve(const double* times, uint64_t n_times, const double* log_discounts,
                                   uint64_t n_log_discounts, fo_error* err);
int fo_validate_cumulative_dividend_yield_curve(const double* times, uint64_t n_times,
                                                const double* cumulative_yields, uint64_t n_yields,
                                                fo_error* err);
int fo_validate_ragged_cash_dividends(const int64_t* offsets, uint64_t n_offsets, const double* times,
                                      uint64_t n_times, const double* amounts, uint64_t n_amounts,
                                      fo_error* err);
int fo_validate_ragged_exercise_times(const int64_t* offsets, uint64_t n_offsets, const double* times,
                                      uint64_t n_times, fo_error* err);
/* Runs every host-side check fo_price_lsm_call_f64 performs before touching a device. */
int fo_validate_lsm_call_request(const fo_lsm_call_request* request, fo_error* err);
/* Every check fo_price_lsm_grouped_f64 (grouped != 0) or fo_price_lsm_batch_f64 (grouped == 0)
 * makes on the whole request before planning any group, in the reference's order (the method,
 * lib.rs:1302-1415; the columns, input.rs:502-706; the stream domain ranges over every group,
 * input.rs:201-255; the mesh domain, pricing.rs:356-400, 622-664), with the same errors. A caller
 * that prices a batch in shards runs it on the whole request first. */
int fo_validate_lsm_grouped_f64(const fo_lsm_grouped_request* request, int32_t grouped, fo_error* err);
/* The same for fo_price_lsm_ragged_f64. */
int fo_validate_lsm_ragged_f64(const fo_lsm_ragged_request* request, fo_error* err);

/* ---- build identity ------------------------------------------------------------------------- */

/* Writes "package_version;nvcc_version;arch" into buf (NUL-terminated, truncated to capacity). */
int fo_build_info(char* buf, uint64_t capacity);

#ifdef __cplusplus
}
#endif

#endif /* FINOPTIONS_CUDA_H */

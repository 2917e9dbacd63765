/*
 * montepath_cuda.h -- C ABI of the B200-native Monte Carlo pricing backend.
 *
 * This is the drop-in boundary that replaces montepath's `NvidiaCudaBackend`
 * (crates/mc-core/src/backend/cuda.rs:40-203), whose `execute` today delegates
 * to a chunked CPU fallback (crates/mc-core/src/backend/mod.rs:457-540).  Each
 * entry point below names the reference interface it stands in for.
 *
 * Conventions
 *  - Every function returns an `int` status (mpc_status_t); validation errors
 *    are reported as codes, never by aborting, and the device never traps.
 *  - All structs are plain-old-data with explicit padding so that ctypes /
 *    cgo / Rust `#[repr(C)]` mirrors can be written field by field.
 *  - Requests and results live in caller-owned host memory.  Device buffers
 *    are owned by the context (a byte-budgeted pool).
 *  - No function takes or returns a framework (torch) type.
 */
#ifndef MONTEPATH_CUDA_H
#define MONTEPATH_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPC_ABI_VERSION 1

#define MPC_MAX_ASSETS 8
#define MPC_MAX_EXERCISE_DATES 64
#define MPC_MAX_LEVELS 16

/* Status codes.  Mirror of BackendError (crates/mc-core/src/backend/mod.rs:186-194)
 * plus the documented error codes of docs/backend-contract.md:280-300. */
typedef enum mpc_status {
  MPC_OK = 0,
  MPC_E_INVALID_CONFIG = 1, /* config rejected (the CPU path panics via assert!, cpu.rs:5010-5153) */
  MPC_E_UNSUPPORTED = 2,    /* BackendError::UnsupportedFeature */
  MPC_E_NO_DEVICE = 3,      /* BackendError::UnknownDevice / B_DEVICE_UNAVAILABLE */
  MPC_E_OOM_BUDGET = 4,     /* B_OUT_OF_MEMORY: request exceeds the HBM byte budget */
  MPC_E_TIMEOUT = 5,        /* a bounded device or host wait ran out */
  MPC_E_CUDA = 6,           /* B_EXECUTION_FAILED: a CUDA runtime call failed */
  MPC_E_BUSY = 7,           /* serving: ticket not finished yet */
  MPC_E_NOT_FOUND = 8,      /* serving: unknown ticket */
  MPC_E_CANCELLED = 9       /* serving: request cancelled before completion */
} mpc_status_t;

/* Workload families: PricingWorkloadFamily of the reference plus the
 * extensions the B200 backend adds (up-and-out barrier). */
typedef enum mpc_workload {
  MPC_WORKLOAD_EUROPEAN_CALL = 0,         /* cpu.rs:3009-3026, 3191-3262 */
  MPC_WORKLOAD_ARITHMETIC_ASIAN_CALL = 1, /* cpu.rs:3264-3281 */
  MPC_WORKLOAD_DOWN_AND_OUT_CALL = 2,     /* cpu.rs:3753-3769 */
  MPC_WORKLOAD_UP_AND_OUT_CALL = 3,       /* extension: mirror of down-and-out */
  MPC_WORKLOAD_LOOKBACK_CALL = 4,         /* cpu.rs:3771-3783 */
  MPC_WORKLOAD_BASKET_CALL = 5,           /* cpu.rs:4022-4034 (2 assets); d assets = extension */
  MPC_WORKLOAD_AMERICAN_PUT = 6,          /* cpu.rs:3947-3981 */
  MPC_WORKLOAD_BERMUDAN_PUT = 7,          /* cpu.rs:3983-4020 */
  MPC_WORKLOAD_ASIAN_MLMC = 8             /* cpu.rs:3283-3293, 3352-3423 */
} mpc_workload_t;

typedef enum mpc_model {
  MPC_MODEL_GBM = 0,
  MPC_MODEL_HESTON = 1, /* cpu.rs:8632-8686 */
  MPC_MODEL_MERTON = 2  /* cpu.rs:3151-3189 (terminal); stepwise = extension */
} mpc_model_t;

/* EuropeanCallMethod (cpu.rs:3013-3026): Auto == terminal distribution. */
typedef enum mpc_method {
  MPC_METHOD_AUTO = 0,
  MPC_METHOD_TERMINAL = 1,
  MPC_METHOD_STEPWISE = 2
} mpc_method_t;

/* MonteCarloTechnique */
typedef enum mpc_technique {
  MPC_TECHNIQUE_STANDARD = 0,
  MPC_TECHNIQUE_ANTITHETIC = 1,
  MPC_TECHNIQUE_CONTROL_VARIATE = 2
} mpc_technique_t;

/* SamplingMethod (cpu.rs:5790-5836) plus the stateless counter-hash stream of
 * the Metal kernel (cpu.rs:5626-5652, european_call_stepwise_v1.metal:6-28). */
typedef enum mpc_sampling {
  MPC_SAMPLING_PSEUDORANDOM = 0,       /* replay of MonteCarloRng (xorshift64*), cpu.rs:2955-3007 */
  MPC_SAMPLING_RANDOMIZED_HALTON = 1,  /* cpu.rs:5686-5722 */
  MPC_SAMPLING_LATIN_HYPERCUBE = 2,    /* cpu.rs:5724-5788 */
  MPC_SAMPLING_SCRAMBLED_SOBOL = 3,    /* cpu.rs:5393-5432, 5654-5684 */
  MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE = 4, /* cpu.rs:5838-5981 */
  MPC_SAMPLING_COUNTER_HASH = 5        /* cpu.rs:5626-5652 */
} mpc_sampling_t;

typedef enum mpc_precision {
  MPC_PRECISION_FP64_PLAIN = 0, /* one request per launch, FP64, materialised normals */
  MPC_PRECISION_FP32_PATH = 1   /* fused FP32 path arithmetic, FP64 accumulation */
} mpc_precision_t;

/*
 * One pricing request.  Replaces BackendExecutionInput
 * (crates/mc-core/src/backend/mod.rs:179-184) and the per-workload config
 * structs of cpu.rs:1297-1815.  Field names follow the Rust configs.
 * Fill with mpc_request_defaults() first; it mirrors the Rust `Default` impls.
 */
typedef struct mpc_request {
  int32_t workload;  /* mpc_workload_t */
  int32_t model;     /* mpc_model_t */
  int32_t method;    /* mpc_method_t (European only) */
  int32_t technique; /* mpc_technique_t */
  int32_t sampling;  /* mpc_sampling_t */
  int32_t precision; /* mpc_precision_t */
  uint64_t n_paths;
  uint32_t n_steps;
  /* Number of independent seed chunks of the reference's CPU thread split
   * (cpu.rs:6232-6276, 8912-8924).  0 or 1 = one sequential stream.  Unlike
   * the reference, 0 never means "host core count": results must not depend
   * on the machine. */
  uint32_t n_threads;
  uint64_t seed;
  double s0, k, r, sigma, t;
  double barrier; /* down-and-out / up-and-out level */
  /* Heston (HestonEuropeanCallConfig, cpu.rs:1431-1446) */
  double v0, kappa, theta, vol_of_vol, rho;
  /* Merton (MertonJumpDiffusionCallConfig, cpu.rs:1470-1482) */
  double jump_intensity, jump_mean, jump_volatility;
  /* Basket (BasketCallConfig, cpu.rs:1713-1729, generalised to d assets):
   * spots[i], sigmas[i], weights[i]; corr is row-major d x d.  For d == 2 the
   * reference parameterisation (rho = corr[1]) is used exactly. */
  uint32_t n_assets;
  uint32_t _pad0;
  double spots[MPC_MAX_ASSETS];
  double sigmas[MPC_MAX_ASSETS];
  double weights[MPC_MAX_ASSETS];
  double corr[MPC_MAX_ASSETS * MPC_MAX_ASSETS];
  /* LSM (AmericanPutConfig / BermudanPutConfig, cpu.rs:1754-1790) */
  uint32_t basis_degree;
  uint32_t n_exercise; /* Bermudan: number of entries in exercise_steps */
  uint32_t exercise_steps[MPC_MAX_EXERCISE_DATES];
  /* MLMC (ArithmeticAsianMlmcConfig, cpu.rs:1535-1568; tolerance config
   * cpu.rs:1611-1630).  target_stderr > 0 runs the tolerance solver first. */
  uint32_t base_steps, levels, refinement_factor, scramble_replicates;
  uint64_t paths_per_level[MPC_MAX_LEVELS];
  double target_stderr;
  uint64_t pilot_paths_per_level, min_step_updates, max_step_updates;
  /* Launch hints (0 = let the autotuner choose).  block_size: 0, 128, 256 or
   * 512 threads per block of the fused launch (other values return
   * MPC_E_UNSUPPORTED); paths_per_thread: 1..64 units per thread per tile,
   * i.e. tiles of block_size * paths_per_thread paths (the tile partition and
   * the block fix the order of the sums, so a hint changes results at
   * rounding level only). */
  uint32_t block_size, paths_per_thread;
  uint64_t _reserved[4];
} mpc_request_t;

/* Result.  Replaces RunOutput (crates/mc-core/src/backend/mod.rs:172-177) and
 * carries the richer LSM (cpu.rs:1818-1847) and MLMC (cpu.rs:1571-1591) fields. */
typedef struct mpc_result {
  double price;
  double stderr;
  double runtime_ms;   /* device time of this request (CUDA events) */
  uint64_t n_samples;  /* paths, or antithetic pairs (blocks) */
  uint64_t path_steps; /* simulated path-steps (a basket step counts once) */
  /* Raw FP64 moments of the estimator: count, sum p, sum p^2, sum c, sum c^2, sum p*c. */
  double moments[6];
  /* LSM */
  uint64_t early_exercise_count;
  uint64_t maturity_exercise_count;
  uint32_t regression_steps;
  uint32_t basis_degree;
  /* MLMC */
  uint32_t n_levels;
  uint32_t target_met;
  uint32_t max_step_updates_hit;
  uint32_t _pad0;
  double estimated_stderr;
  uint64_t total_paths;
  uint64_t total_step_updates;
  double level_mean[MPC_MAX_LEVELS];
  double level_variance[MPC_MAX_LEVELS];
  uint64_t level_paths[MPC_MAX_LEVELS];
  uint64_t level_fine_steps[MPC_MAX_LEVELS];
  /* Serving timestamps, ms on the server clock (0 outside serving). */
  double t_enqueue_ms, t_admit_ms, t_complete_ms;
  int32_t status;
  uint32_t warnings; /* bit set of MPC_WARN_* */
} mpc_result_t;

#define MPC_WARN_BASIS_DEGREE_CLAMPED 0x1u
#define MPC_WARN_THREADS_IGNORED 0x2u
#define MPC_WARN_SCHEDULE_NORMALISED 0x4u
#define MPC_WARN_INTRINSIC_FLOOR 0x8u

/* Greeks.  Greek / GreekEstimator / GreekEstimate / GreekReport of the
 * reference (crates/mc-core/src/runtime/cpu.rs:138-192). */
typedef enum mpc_greek {
  MPC_GREEK_DELTA = 0,
  MPC_GREEK_DELTA2 = 1, /* basket: second spot */
  MPC_GREEK_VEGA = 2,   /* Heston: sensitivity to sqrt(v0), theta held fixed */
  MPC_GREEK_VEGA2 = 3,  /* basket: second volatility */
  MPC_GREEK_RHO = 4,
  MPC_GREEK_THETA = 5   /* conventional calendar theta (minus d price / d maturity) */
} mpc_greek_t;

typedef enum mpc_greek_estimator {
  MPC_GREEKS_BUMP_AND_REVALUE = 0, /* central common-random-number differences, cpu.rs:4938-4983 */
  MPC_GREEKS_PATHWISE = 1,         /* terminal-GBM European call, cpu.rs:4670-4765 */
  MPC_GREEKS_LIKELIHOOD_RATIO = 2  /* terminal-GBM European call, cpu.rs:4767-4869 */
} mpc_greek_estimator_t;

#define MPC_MAX_GREEKS 6

typedef struct mpc_greek_estimate {
  int32_t greek;     /* mpc_greek_t */
  int32_t estimator; /* mpc_greek_estimator_t */
  double value;
  double stderr;           /* bump: independent-leg propagation; single pass: sample standard error */
  double bump_size;        /* effective half-width of the central difference (0 for single pass) */
  double base_price;
  double bumped_up_price;   /* bump only */
  double bumped_down_price; /* bump only */
} mpc_greek_estimate_t;

typedef struct mpc_greek_report {
  int32_t workload;  /* mpc_workload_t */
  int32_t estimator; /* mpc_greek_estimator_t */
  uint64_t paths;
  uint32_t steps;
  uint32_t n_estimates;
  uint64_t seed;
  double base_price;
  double base_stderr;
  double runtime_ms; /* device time of all launches of the report */
  mpc_greek_estimate_t estimates[MPC_MAX_GREEKS];
  uint32_t warnings; /* bit set of MPC_GREEK_WARN_* */
  int32_t status;
} mpc_greek_report_t;

/* The reference's report warnings, as flags. */
#define MPC_GREEK_WARN_ESTIMATOR_UNSUPPORTED 0x1u /* no estimates: the estimator is not offered for this workload */
#define MPC_GREEK_WARN_PSEUDORANDOM_SHOCKS 0x2u   /* single-pass estimators draw the pseudorandom stream whatever the sampling */
#define MPC_GREEK_WARN_TECHNIQUE_IGNORED 0x4u     /* single-pass estimators ignore the variance-reduction technique */

/* Cost estimate of one request on the GPU: CostEstimate of the reference
 * (crates/mc-core/src/backend/mod.rs:55-63) for NvidiaCudaBackend::estimate_cost
 * (cuda.rs:121-152), from device rates measured per kernel family, sampler and
 * precision on a B200 (148 SMs) and scaled by the SM count given. */
typedef struct mpc_cost {
  double estimated_compile_ms;  /* first call of a shape: lookup tables, autotuner, buffers */
  double estimated_runtime_ms;  /* device time of the request's launches */
  double estimated_total_ms;    /* compile + runtime + per-call overhead */
  double estimated_peak_memory_mb;
  double path_steps_per_sec;    /* modelled device rate */
  uint64_t path_steps;
  char confidence[16];          /* "measured": a measured rate; "derived": scaled from one */
} mpc_cost_t;

typedef struct mpc_device_info {
  int32_t index;
  int32_t sm_count;
  int32_t cc_major, cc_minor;
  uint64_t total_memory_bytes;
  uint64_t free_memory_bytes;
  int32_t clock_khz;
  int32_t l2_bytes;
  char name[96];
} mpc_device_info_t;

typedef struct mpc_options {
  int32_t device;           /* CUDA device ordinal */
  int32_t deterministic;    /* reductions always run in fixed tile order, so results
                               are deterministic for 0 and 1 alike */
  uint64_t hbm_budget_bytes; /* 0 = 64 GiB */
  uint32_t default_block_size; /* 0 (autotuner), 128, 256 or 512: block size of fused
                                  launches when a request gives no hint and mpc_prepare
                                  has not tuned its kind (other values: MPC_E_UNSUPPORTED) */
  uint32_t _pad0;
} mpc_options_t;

/* Reply of mpc_supports: replaces SupportReport (backend/mod.rs) for the CUDA backend. */
typedef struct mpc_support {
  int32_t supported;      /* 1 = runs natively on the GPU */
  int32_t reason;         /* mpc_status_t when not supported */
  uint64_t estimated_bytes;
  char message[160];
} mpc_support_t;

/* What mpc_prepare settled on (CompiledArtifact, backend/mod.rs:407-427). */
typedef struct mpc_artifact {
  int32_t kernel_family;
  uint32_t block_size;
  uint32_t paths_per_thread;
  uint32_t tiles;
  uint64_t bytes;
  char name[96];
} mpc_artifact_t;

typedef struct mpc_context mpc_context_t;
typedef struct mpc_server mpc_server_t;

typedef struct mpc_server_options {
  uint64_t hbm_budget_bytes; /* admission budget (0 = 64 GiB) */
  uint32_t max_slots;        /* live requests on the device at once (0 = 256) */
  uint32_t wave_tiles;       /* tiles per scheduling wave (0 = auto) */
  uint32_t mode;             /* 0 = continuous batching in host-scheduled waves, 1 = plain FIFO, one request
                                per launch in FP64, 2 = continuous batching in a resident device loop */
  uint32_t reserve_sms;      /* mode 2: SMs the loop leaves free for Longstaff-Schwartz and the other
                                host-batched launches, which then run beside it (0 = 32) */
} mpc_server_options_t;

typedef struct mpc_server_stats {
  uint64_t submitted, admitted, completed, rejected, cancelled;
  uint64_t waves;
  uint64_t live_bytes, peak_bytes;
  double p50_ms, p99_ms, mean_ms, max_ms;
  double busy_ms, wall_ms;
  uint64_t path_steps;
} mpc_server_stats_t;

/* ----- library and devices -------------------------------------------- */
int mpc_abi_version(void);
/* Sizes of the ABI structs, for binding self-checks (ctypes, cgo). */
size_t mpc_struct_size(int which); /* 0 request, 1 result, 2 device_info, 3 options, 4 support, 5 artifact, 6 server_options, 7 server_stats, 8 greek_report, 9 cost */
const char* mpc_status_string(int status);

/* Replaces NvidiaCudaBackend::discover_devices' nvidia-smi parsing (cuda.rs:205-241). */
int mpc_device_count(int* count);
int mpc_device_info(int index, mpc_device_info_t* info);

/* ----- requests (host-only, no device needed) --------------------------- */
/* Fills the Rust `Default` values of the workload's config (cpu.rs:1311-1815). */
int mpc_request_defaults(mpc_request_t* req, int workload);
/* Config validation (validate_*_config, cpu.rs:5010-5153) returning a code. */
int mpc_validate(const mpc_request_t* req, char* message, size_t message_len);
/* NvidiaCudaBackend::supports (cuda.rs:68-119). */
int mpc_supports(const mpc_request_t* req, mpc_support_t* out);
/* Device bytes a request holds while it runs (estimate_gpu_bytes_per_path, backend/mod.rs:399-405). */
int mpc_estimate_bytes(const mpc_request_t* req, uint64_t* bytes);
/* NvidiaCudaBackend::estimate_cost (cuda.rs:121-152) from the measured cost
 * model (host only).  sm_count 0 = 148. */
int mpc_estimate_cost(const mpc_request_t* req, int sm_count, mpc_cost_t* out);
/* The same estimate from rates measured on this context's device by
 * mpc_calibrate_cost (confidence "calibrated"); before any calibration, the
 * built-in rates scaled by the device's SM count. */
int mpc_estimate_cost_ctx(mpc_context_t* ctx, const mpc_request_t* req, mpc_cost_t* out);
/* Measures this device's rates for the cost model: one request of 1,048,576
 * paths x 64 steps (1 step for terminal workloads) per model row, sampler
 * column (pseudorandom, counter hash, scrambled Sobol, Halton) and
 * precision, priced twice, the second call's device time kept (the terminal
 * GBM row is priced at 4,194,304 paths too, which separates a per-call
 * intercept from its per-path rate).  Replaces the
 * single-B200 table that cuda.rs:121-152's estimate would otherwise read;
 * combinations the backend does not run, or past the context's byte budget,
 * keep the built-in rate.  `seconds` (optional) receives the wall time it
 * took.  Returns MPC_E_CUDA if a pricing call fails on the device. */
int mpc_calibrate_cost(mpc_context_t* ctx, double* seconds);

/* ----- context ---------------------------------------------------------- */
int mpc_create(const mpc_options_t* options, mpc_context_t** out);
int mpc_destroy(mpc_context_t* ctx);
const char* mpc_last_error_message(const mpc_context_t* ctx);

/* NvidiaCudaBackend::compile (cuda.rs:155-185): launch shape chosen by the autotuner. */
int mpc_prepare(mpc_context_t* ctx, const mpc_request_t* req, mpc_artifact_t* out);
/* NvidiaCudaBackend::execute (cuda.rs:187-193): prices one request on the GPU. */
int mpc_price(mpc_context_t* ctx, const mpc_request_t* req, mpc_result_t* out);
/* Prices n requests: the FP32-path requests in one persistent launch per
 * (sampler, family) group, the FP64-plain requests one launch sequence each,
 * LSM and MLMC requests in shared launches.  When a fused batch of the same
 * shape (sizes, launch shapes, buffers) comes twice in a row, the second call
 * captures its copy/launch sequence in a CUDA graph and later calls of that
 * shape replay the graph (one launch call). */
int mpc_price_batch(mpc_context_t* ctx, const mpc_request_t* reqs, size_t n, mpc_result_t* out);
/* Greeks of one request: european_call_greeks_cpu, arithmetic_asian_call_greeks_cpu,
 * down_and_out_call_greeks_cpu, lookback_call_greeks_cpu, basket_call_greeks_cpu,
 * heston_european_call_greeks_cpu (cpu.rs:4036-4356).
 *  - BUMP_AND_REVALUE: the base request and an up and a down bump per Greek
 *    (spot 1% (min 0.01), volatility 5% (min 0.005), rate 0.001, maturity
 *    min(1/365, T/4)), all with the request's seed, priced in one batch (one
 *    persistent launch on the FP32 path).
 *  - PATHWISE / LIKELIHOOD_RATIO: European call only; one pass over the
 *    pseudorandom terminal shocks of the request's seed (the reference's
 *    MonteCarloRng stream) on the device, base price from the request itself.
 *    Other workloads return MPC_OK with no estimates and
 *    MPC_GREEK_WARN_ESTIMATOR_UNSUPPORTED, as the reference does.
 *  - Merton, LSM and MLMC requests: MPC_E_UNSUPPORTED (the reference has no
 *    Greeks for them). */
int mpc_greeks(mpc_context_t* ctx, const mpc_request_t* req, int estimator, mpc_greek_report_t* out);
/* Per-path discounted payoffs of a (small) request, for same-normals parity
 * checks (the per-path output of mc_cuda_european_call_stepwise_v1).  Writes
 * n_samples doubles (pairs: the block estimate) to host memory. */
int mpc_price_paths(mpc_context_t* ctx, const mpc_request_t* req, double* host_payoffs, uint64_t capacity);

/* Device sampler output, row-major [point][dim] in host memory.
 * precision FP64_PLAIN writes doubles, FP32_PATH floats.
 * Replaces generate_standard_normals_cpu (cpu.rs:5343-5379) and, for
 * COUNTER_HASH, generate_stepwise_stateless_normals_f32 (cpu.rs:5435-5454). */
int mpc_generate_normals(mpc_context_t* ctx, int sampling, uint64_t seed, uint64_t n_points,
                         uint32_t dimensions, int precision, void* host_out);
/* Raw 32-bit counter hashes (hash_u32 of cpu.rs:5645-5652) for lanes 0/1 of
 * (seed, path, step): out[2*(path*n_steps+step)+lane]. */
int mpc_counter_hash_u32(mpc_context_t* ctx, uint32_t seed, uint32_t n_paths, uint32_t n_steps,
                         uint32_t* host_out);
/* xorshift64* outputs of MonteCarloRng::next_u64 (cpu.rs:2975-2983) starting
 * `offset` draws into the stream of `seed`, generated on the device by jump-ahead. */
int mpc_xorshift_u64(mpc_context_t* ctx, uint64_t seed, uint64_t offset, uint64_t count,
                     uint64_t* host_out);

/* The reference kernel contract mc_cuda_european_call_stepwise_v1
 * (crates/mc-core/src/backend/kernels/european_call_stepwise_v1.cu:1-28 and
 * the GpuKernelContract of cuda.rs:247-310): DEVICE pointers, normals
 * path-major [n_paths][n_steps] f64, payoffs [n_paths] f64.  `stream` is a
 * cudaStream_t (NULL = legacy default stream).  Asynchronous. */
int mpc_european_call_stepwise_v1(const double* normals, double* payoffs, int32_t n_paths,
                                  int32_t n_steps, double log_s0, double strike, double drift_dt,
                                  double vol_dt, double discount, void* stream);

/* Writes and reads a buffer larger than L2 on the context stream (timing hygiene). */
int mpc_flush_l2(mpc_context_t* ctx);
/* Device time (ms) of the last mpc_price / mpc_price_batch and the number of
 * kernels it launched. */
int mpc_last_timing(const mpc_context_t* ctx, double* device_ms, uint64_t* kernel_launches);
/* Host<->device bytes the last mpc_price / mpc_price_batch copied (no reference counterpart: diagnostics). */
int mpc_last_transfer(const mpc_context_t* ctx, uint64_t* h2d_bytes, uint64_t* d2h_bytes);
/* Measured FP32 FMA (TFLOP/s) and MUFU (Tops/s) throughput of the device, the
 * roofline denominators of the compute-bound fused kernels (no reference counterpart). */
int mpc_measure_peaks(mpc_context_t* ctx, double* fp32_tflops, double* sfu_tops);

/* Prices one FP32-path request like mpc_price, but allocates nothing: no
 * context, no cudaMalloc/cudaFree, no pinned host buffers.  It is meant for
 * callers that cannot let a library allocate device memory -- a service whose
 * own allocator reserves the GPU's memory at start-up, or a latency-critical
 * path where cudaMalloc/cudaFree (which can synchronise the device) are
 * forbidden.  It has no counterpart in the reference.
 *  - Runs on the current device and `stream` (a cudaStream_t, NULL = legacy
 *    default stream) and returns after the result is on the host.
 *  - Device buffers are file-scope static arrays of fixed size (about 0.7 MB
 *    per GPU, held until the process exits): at most 16,777,216 paths (or
 *    antithetic pairs) per request; larger requests return MPC_E_OOM_BUDGET.
 *  - Samplers: pseudorandom, counter_hash, scrambled_sobol; path-payoff
 *    workloads only (not LSM, MLMC or FP64-plain requests: MPC_E_UNSUPPORTED).
 *  - A paths_per_thread hint is honoured when it is a power of two up to 16
 *    whose tiles (256 * hint paths) number at most 4,096; any other hint
 *    returns MPC_E_UNSUPPORTED.  Without a hint the tile is the smallest
 *    power-of-two multiple of 256 paths that fits 4,096 tiles.
 *  - Serves device ordinals 0-63.
 *  - The first call on a device resolves the arrays' device addresses and
 *    uploads the lookup tables (set-up); make that first call before any
 *    stream capture.
 *  - All calls share the same arrays: calls that overlap on the GPU (other
 *    streams, other host threads) race and must be serialised by the caller.
 *  - error_message (optional) receives the reason for a non-zero status. */
int mpc_price_fused_noalloc(const mpc_request_t* req, mpc_result_t* out, void* stream, char* error_message,
                            size_t error_message_len);

/* ----- serving ------------------------------------------------------------ */
int mpc_server_start(mpc_context_t* ctx, const mpc_server_options_t* options, mpc_server_t** out);
int mpc_submit(mpc_server_t* server, const mpc_request_t* req, uint64_t* ticket);
int mpc_poll(mpc_server_t* server, uint64_t ticket, mpc_result_t* out);
int mpc_wait(mpc_server_t* server, uint64_t ticket, int64_t timeout_ms, mpc_result_t* out);
int mpc_cancel(mpc_server_t* server, uint64_t ticket);
int mpc_server_stats(mpc_server_t* server, mpc_server_stats_t* out);
int mpc_server_stop(mpc_server_t* server);

#ifdef __cplusplus
}
#endif

#endif /* MONTEPATH_CUDA_H */

// mpc_types.h -- host/device shared data layout of the B200 Monte Carlo backend.
#pragma once

#include <stdint.h>

#define MPC_SOBOL_TABLE_DIMS 256
// The device lookup table (32-bit words) holds two layouts of the Sobol
// nibble products: [dim][q][v] (words 0 .. MPC_SOBOL_NIBBLE_WORDS) for
// per-sample lookups, and from MPC_SOBOL_NIBBLE_WORDS on the bit-reversed
// transpose [16 q + v][dim] that the fused kernels stage into shared memory
// rows; then, from MPC_ICDF_OFFSET, the FP32 inverse-normal segments of the
// fused Sobol path (4 cubic coefficients per segment).
#define MPC_SOBOL_NIBBLE_WORDS (MPC_SOBOL_TABLE_DIMS * 8 * 16)
#define MPC_ICDF_SEGMENTS (23 * 32)
#define MPC_ICDF_OFFSET (2 * MPC_SOBOL_NIBBLE_WORDS)
#define MPC_SOBOL_TABLE_WORDS (MPC_ICDF_OFFSET + 4 * MPC_ICDF_SEGMENTS)
// Moments per tile / request: count, sum p, sum p^2, sum c, sum c^2, sum p*c (+2 pad).
#define MPC_MOMENTS 8

namespace mpc {

// Brownian bridge: the device walks the bisection tree with a stack of at
// most kBridgeDepth values, which holds every program of up to
// kBridgeMaxSteps steps (tree depth 16 plus W(T)).
constexpr uint32_t kBridgeDepth = 20;
constexpr uint32_t kBridgeMaxSteps = 65536;

// Scenario (bump-and-revalue) kernel: up to kMaxScen legs share every normal;
// kScenFields float parameters per leg, stored [field][kMaxScen].
constexpr int kMaxScen = 9;
constexpr int kScenFields = 6;

// Basket bump legs (base, then up and down for two spots, two volatilities,
// the rate and the maturity).  The basket payoff reads only terminal values,
// and each leg's log return of asset a is affine in the same correlated
// normal sum, x_a = (r - sigma_a^2 / 2) T + sigma_a sqrt(dt) W_a, so the
// legs share W and differ only in these per-leg constants (float, read from
// the kernel's parameter bank).
constexpr int kBasketScen = 13;
struct BasketScen {
  float log_drift[kBasketScen][8];  // (r - sigma_a^2 / 2) T
  float step_vol[kBasketScen][8];   // sigma_a sqrt(dt)
  float wspot[kBasketScen][8];      // weight_a * spot_a
  float discount[kBasketScen];      // exp(-r T)
};

// Kernel families: the model-specific loop a tile runs.
enum Family : int32_t {
  FAM_GBM_STEP = 0,
  FAM_GBM_TERMINAL = 1,
  FAM_HESTON = 2,
  FAM_MERTON_STEP = 3,
  FAM_MERTON_TERMINAL = 4,
  FAM_BASKET = 5,
  FAM_MLMC_LEVEL = 6,
  FAM_GBM_BRIDGE = 7,  // GBM stepwise driven through the Brownian bridge (bridge Sobol)
  FAM_COUNT = 8        // number of families above
};

// Device samplers.
enum Sampler : int32_t {
  SMP_XORSHIFT = 0,  // replay of MonteCarloRng
  SMP_HALTON = 1,
  SMP_LHS = 2,
  SMP_SOBOL = 3,
  SMP_COUNTER = 5,
};

struct LhsDim {
  uint64_t multiplier, offset, jitter_seed;
};

// Everything a tile needs to simulate units of one request.  Built on the
// host (double precision constants); FP32 kernels round them once per tile.
struct alignas(16) DevReq {
  int32_t family, workload, technique, sampling;
  uint32_t n_steps;        // model steps (fine steps for an MLMC level)
  uint32_t n_assets;
  uint64_t n_paths;        // simulated paths
  uint64_t n_units;        // paths, or antithetic pairs
  uint64_t normals_per_unit;
  uint64_t seed;
  uint32_t seed32;
  uint32_t n_chunks;       // reference CPU chunk split (1 = one stream)
  uint64_t chunk_base, chunk_rem;
  // GBM / payoff
  double s0, k, barrier, log_s0, log_barrier, discount, drift_dt, vol_dt, cv_expectation;
  // Heston
  double v0, kappa, theta, xi, rho, rho_perp, dt, sqrt_dt, rate;
  // Merton
  double jump_mean, jump_vol, lam_dt;
  double lam_p0;   // exp(-lam_dt): no jump while u <= lam_p0
  float lam_p0_f;  // largest float <= lam_p0 (exact FP32 test of the same event)
  uint32_t _pad_m;
  // FP32 Sobol steps: with the Poisson uniform u = (m + 1/2) 2^-23 (m the
  // top 23 bits of the scrambled sample), m >= pois_m[k] exactly when u
  // exceeds the (k+1)-term cumulative sum of sample_poisson (cpu.rs:932-953),
  // i.e. when the jump count is at least k + 1, k = 0..3
  uint32_t pois_m[4];
  // Basket: lower Cholesky factor and per-asset step constants
  double chol[64], b_drift[8], b_vol[8], spots[8], weights[8];
  // MLMC level
  uint32_t level, refinement;
  uint64_t coarse_steps;
  double f_drift, f_vol, c_drift, c_vol, inv_sqrt_m, inv_fine, inv_coarse;
  // Brownian-bridge path construction (GBM stepwise with bridge Sobol): a
  // program of 2 n_steps - 1 events in the reference's depth-first order;
  // event e is an op (a midpoint, weights and stddev in bridge_ops) when bit
  // e of bridge_events is set, else a leaf (one step increment).
  const double* bridge_ops;       // [n_steps - 1][3]: left weight, right weight, stddev
  const uint32_t* bridge_events;  // [(2 n_steps - 1 + 31) / 32]
  double bridge_sqrt_t, bridge_inv_sqrt_dt;
  uint32_t bridge;                // 1: normals come through the bridge
  uint32_t n_scen;                // scenario kernel: legs in `scen` (0 elsewhere)
  const float* scen;              // scenario kernel: [kScenFields][kMaxScen] leg parameters
  // samplers
  const uint32_t* halton_primes;
  const double* halton_shifts;
  const LhsDim* lhs;
  // tiling and outputs
  uint32_t tile_units;     // units per tile
  uint32_t n_tiles;
  double* partials;        // [n_tiles][MPC_MOMENTS]
  double* moments;         // [MPC_MOMENTS] final, written by the last tile
  uint32_t* tiles_done;    // completion counter for the last-tile finalize
  double* per_unit;        // optional [n_units] payoffs (parity checks)
  uint32_t cv;             // record control variate moments
  uint32_t anti;           // antithetic pairs
};

struct Tile {
  uint32_t req;
  uint32_t tile;
};

}  // namespace mpc

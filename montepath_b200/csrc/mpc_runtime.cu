// mpc_runtime.cu -- host runtime of the B200 Monte Carlo backend behind the
// C ABI of include/montepath_cuda.h.
//
// It replaces NvidiaCudaBackend (crates/mc-core/src/backend/cuda.rs:40-203):
// device discovery, support reports, request validation with status codes,
// launch-shape selection, and execution of every pricing family on the GPU.
// There is no CPU fallback: a request the device path cannot run is
// rejected with MPC_E_UNSUPPORTED.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "mpc_device.cuh"
#include "mpc_launch.h"
#include "mpc_runtime.h"
#include "sobol_directions.h"

using namespace mpc;

namespace mpc {

int fail(mpc_context* ctx, int status, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return status;
}

int cuda_fail(mpc_context* ctx, cudaError_t err, const char* what) {
  std::string msg = std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")";
  if (ctx) ctx->last_error = msg;
  return err == cudaErrorMemoryAllocation ? MPC_E_OOM_BUDGET : MPC_E_CUDA;
}

#define MPC_CUDA(ctx, call)                                   \
  do {                                                        \
    cudaError_t _e = (call);                                  \
    if (_e != cudaSuccess) return cuda_fail((ctx), _e, #call); \
  } while (0)

int scratch(mpc_context* ctx, const std::string& name, size_t bytes, void** out) {
  if (bytes == 0) bytes = 16;
  DevBuf& b = ctx->bufs[name];
  if (b.bytes >= bytes) {
    *out = b.ptr;
    return MPC_OK;
  }
  size_t grow = std::max(bytes, b.bytes + b.bytes / 2);
  grow = (grow + 255) & ~size_t(255);
  uint64_t after = ctx->live_bytes - b.bytes + grow;
  if (after > ctx->budget) {
    grow = (bytes + 255) & ~size_t(255);
    after = ctx->live_bytes - b.bytes + grow;
    if (after > ctx->budget)
      return fail(ctx, MPC_E_OOM_BUDGET,
                  "request needs " + std::to_string(bytes) + " device bytes for '" + name +
                      "', beyond the HBM budget of " + std::to_string(ctx->budget) + " bytes");
  }
  if (b.ptr) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(b.ptr);
    ctx->live_bytes -= b.bytes;
    b.ptr = nullptr;
    b.bytes = 0;
  }
  void* p = nullptr;
  cudaError_t err = cudaMalloc(&p, grow);
  if (err != cudaSuccess) return cuda_fail(ctx, err, ("cudaMalloc " + name).c_str());
  // Zero-fill on the context stream and wait for it: the context stream is
  // non-blocking, so a fill on the legacy stream would not be ordered before
  // the caller's copies into the new buffer and could overwrite them.
  err = cudaMemsetAsync(p, 0, grow, ctx->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
  if (err != cudaSuccess) {
    cudaFree(p);
    return cuda_fail(ctx, err, ("zero-fill " + name).c_str());
  }
  b.ptr = p;
  b.bytes = grow;
  ctx->live_bytes += grow;
  ctx->peak_bytes = std::max(ctx->peak_bytes, ctx->live_bytes);
  *out = p;
  return MPC_OK;
}

static int pinned_staging(mpc_context* ctx, size_t bytes, void** out) {
  if (ctx->pinned_bytes < bytes) {
    if (ctx->pinned) {
      cudaStreamSynchronize(ctx->stream);
      cudaFreeHost(ctx->pinned);
    }
    size_t grow = std::max(bytes, ctx->pinned_bytes * 2);
    cudaError_t err = cudaHostAlloc(&ctx->pinned, grow, cudaHostAllocDefault);
    if (err != cudaSuccess) {
      ctx->pinned = nullptr;
      ctx->pinned_bytes = 0;
      return cuda_fail(ctx, err, "cudaHostAlloc");
    }
    ctx->pinned_bytes = grow;
  }
  *out = ctx->pinned;
  return MPC_OK;
}

// ------------------------------------------------------------ validation ---
static bool finite(double x) { return std::isfinite(x); }

static int invalid(std::string* msg, const std::string& m) {
  if (msg) *msg = m;
  return MPC_E_INVALID_CONFIG;
}
static int unsupported(std::string* msg, const std::string& m) {
  if (msg) *msg = m;
  return MPC_E_UNSUPPORTED;
}

static bool is_lsm(int w) { return w == MPC_WORKLOAD_AMERICAN_PUT || w == MPC_WORKLOAD_BERMUDAN_PUT; }

// Lower Cholesky factor; returns false if the matrix is not a valid correlation matrix.
static bool cholesky(const double* corr, uint32_t d, double* L) {
  std::memset(L, 0, sizeof(double) * 64);
  if (d == 2) {  // exactly the reference's rho / sqrt(1 - rho^2) split (cpu.rs:7622-7630)
    if (corr[1] < -1.0 || corr[1] > 1.0) return false;
    L[0] = 1.0;
    L[2] = corr[1];
    L[3] = std::sqrt(std::max(1.0 - corr[1] * corr[1], 0.0));
    return true;
  }
  for (uint32_t i = 0; i < d; ++i) {
    if (std::fabs(corr[i * d + i] - 1.0) > 1e-12) return false;
    for (uint32_t j = 0; j < d; ++j)
      if (std::fabs(corr[i * d + j] - corr[j * d + i]) > 1e-12) return false;
  }
  for (uint32_t i = 0; i < d; ++i) {
    for (uint32_t j = 0; j <= i; ++j) {
      double s = corr[i * d + j];
      for (uint32_t k = 0; k < j; ++k) s -= L[i * d + k] * L[j * d + k];
      if (i == j) {
        if (s < -1e-12) return false;
        L[i * d + i] = std::sqrt(std::max(s, 0.0));
      } else {
        L[i * d + j] = L[j * d + j] > 0.0 ? s / L[j * d + j] : 0.0;
      }
    }
  }
  return true;
}

// Mirrors the reference's config asserts (cpu.rs:5010-5153 and the per-entry
// asserts such as cpu.rs:3014-3016) as status codes, plus the device limits.
int validate(const mpc_request_t& r, std::string* msg) {
  if (r.workload < 0 || r.workload > MPC_WORKLOAD_ASIAN_MLMC) return invalid(msg, "unknown workload");
  if (r.model < 0 || r.model > MPC_MODEL_MERTON) return invalid(msg, "unknown model");
  if (r.technique < 0 || r.technique > MPC_TECHNIQUE_CONTROL_VARIATE) return invalid(msg, "unknown technique");
  if (r.sampling < 0 || r.sampling > MPC_SAMPLING_COUNTER_HASH) return invalid(msg, "unknown sampling");
  if (r.precision != MPC_PRECISION_FP64_PLAIN && r.precision != MPC_PRECISION_FP32_PATH)
    return invalid(msg, "unknown precision");
  if (r.method < 0 || r.method > MPC_METHOD_STEPWISE) return invalid(msg, "unknown method");
  // launch hints: the kernels are built for 256-thread blocks
  if (r.block_size != 0 && r.block_size != 128 && r.block_size != 256 && r.block_size != 512)
    return unsupported(msg, "block_size: the fused kernels run 128-, 256- or 512-thread blocks (0 = autotuner)");
  if (r.paths_per_thread > 64) return invalid(msg, "paths_per_thread must be 0 (autotuner) to 64");
  for (double x : {r.s0, r.k, r.r, r.sigma, r.t})
    if (!finite(x)) return invalid(msg, "market parameters must be finite");
  if (r.workload == MPC_WORKLOAD_ASIAN_MLMC) {
    if (!(r.s0 > 0.0) || !(r.k > 0.0) || !(r.t > 0.0)) return invalid(msg, "s0, k and t must be > 0");
    if (!(r.sigma >= 0.0)) return invalid(msg, "sigma must be >= 0");
    if (r.base_steps == 0) return invalid(msg, "base_steps must be > 0");
    if (r.levels == 0 || r.levels > MPC_MAX_LEVELS) return invalid(msg, "levels must be in 1..=16");
    if (r.refinement_factor < 2) return invalid(msg, "refinement_factor must be >= 2");
    if (r.refinement_factor > 64) return unsupported(msg, "refinement_factor above 64 is not supported");
    if (r.scramble_replicates == 0) return invalid(msg, "scramble_replicates must be > 0");
    uint64_t fine = r.base_steps;
    for (uint32_t l = 1; l < r.levels; ++l) {
      fine *= r.refinement_factor;
      if (fine > (1u << 20)) return unsupported(msg, "finest MLMC level exceeds 2^20 steps");
    }
    if (r.target_stderr > 0.0) {
      if (!finite(r.target_stderr)) return invalid(msg, "target_stderr must be finite");
      if (r.pilot_paths_per_level < 2) return invalid(msg, "pilot_paths_per_level must be > 1");
      if (r.min_step_updates == 0) return invalid(msg, "min_step_updates must be > 0");
      if (r.max_step_updates < r.min_step_updates) return invalid(msg, "max_step_updates must be >= min_step_updates");
    } else {
      for (uint32_t l = 0; l < r.levels; ++l)
        if (r.paths_per_level[l] == 0) return invalid(msg, "paths_per_level values must be > 0");
    }
    if (r.technique != MPC_TECHNIQUE_STANDARD) return unsupported(msg, "MLMC supports the standard technique only");
    if (r.sampling == MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE)
      return unsupported(msg, "Brownian-bridge sampling is not implemented for MLMC levels");
    return MPC_OK;
  }
  if (r.n_paths == 0) return invalid(msg, "n_paths must be > 0");
  if (r.n_paths > (1ull << 32)) return unsupported(msg, "n_paths above 2^32 is not supported");
  if (r.n_steps == 0) return invalid(msg, "n_steps must be > 0");
  if (!(r.t > 0.0)) return invalid(msg, "t must be > 0");
  if (r.sampling == MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE && r.n_steps > kBridgeMaxSteps)
    return unsupported(msg, "Brownian-bridge sampling supports at most 65,536 steps");
  if (is_lsm(r.workload)) {
    if (r.n_steps < 2) return invalid(msg, "n_steps must be >= 2 for LSM regression");
    if (r.n_steps > 511) return unsupported(msg, "LSM supports at most 511 steps");
    if (!(r.s0 > 0.0) || !(r.k > 0.0)) return invalid(msg, "s0 and k must be > 0");
    if (!(r.sigma >= 0.0)) return invalid(msg, "sigma must be >= 0");
    if (r.basis_degree == 0) return invalid(msg, "basis_degree must be > 0");
    if (r.workload == MPC_WORKLOAD_BERMUDAN_PUT) {
      if (r.n_exercise == 0) return invalid(msg, "exercise_steps must include at least one exercise date");
      if (r.n_exercise > MPC_MAX_EXERCISE_DATES) return invalid(msg, "at most 64 exercise dates");
      for (uint32_t i = 0; i < r.n_exercise; ++i)
        if (r.exercise_steps[i] == 0 || r.exercise_steps[i] > r.n_steps)
          return invalid(msg, "exercise_steps must be in 1..=n_steps");
    }
    if (r.sampling != MPC_SAMPLING_PSEUDORANDOM && r.sampling != MPC_SAMPLING_COUNTER_HASH)
      return unsupported(msg, "LSM paths use the pseudorandom or counter-hash stream");
    if (r.technique != MPC_TECHNIQUE_STANDARD) return unsupported(msg, "LSM supports the standard technique only");
    if (r.n_paths > 8ull * 148 * 8 * 256) return unsupported(msg, "LSM path count exceeds the co-resident capacity");
    return MPC_OK;
  }
  if (r.workload == MPC_WORKLOAD_BASKET_CALL) {
    if (r.n_assets < 1 || r.n_assets > MPC_MAX_ASSETS) return invalid(msg, "n_assets must be in 1..=8");
    for (uint32_t a = 0; a < r.n_assets; ++a) {
      if (!(r.spots[a] > 0.0)) return invalid(msg, "basket spots must be > 0");
      if (!(r.sigmas[a] >= 0.0)) return invalid(msg, "basket sigmas must be >= 0");
      if (!finite(r.weights[a])) return invalid(msg, "basket weights must be finite");
    }
    if (!(r.k >= 0.0)) return invalid(msg, "k must be >= 0");
    double L[64];
    if (!cholesky(r.corr, r.n_assets, L)) return invalid(msg, "corr must be a valid correlation matrix");
    if (r.model != MPC_MODEL_GBM) return unsupported(msg, "baskets are simulated under GBM");
  } else {
    if (!(r.s0 > 0.0)) return invalid(msg, "s0 must be > 0");
    if (!(r.k >= 0.0)) return invalid(msg, "k must be >= 0");
    if (!(r.sigma >= 0.0)) return invalid(msg, "sigma must be >= 0");
  }
  if (r.workload == MPC_WORKLOAD_DOWN_AND_OUT_CALL || r.workload == MPC_WORKLOAD_UP_AND_OUT_CALL) {
    if (!(r.barrier > 0.0)) return invalid(msg, "barrier must be > 0");
  }
  if (r.model == MPC_MODEL_HESTON) {
    if (r.workload != MPC_WORKLOAD_EUROPEAN_CALL) return unsupported(msg, "Heston prices European calls");
    if (!(r.v0 >= 0.0) || !(r.kappa >= 0.0) || !(r.theta >= 0.0) || !(r.vol_of_vol >= 0.0))
      return invalid(msg, "v0, kappa, theta and vol_of_vol must be >= 0");
    if (!(r.rho >= -1.0 && r.rho <= 1.0)) return invalid(msg, "rho must be in [-1, 1]");
  }
  if (r.model == MPC_MODEL_MERTON) {
    if (r.workload != MPC_WORKLOAD_EUROPEAN_CALL) return unsupported(msg, "Merton prices European calls");
    if (!(r.k > 0.0)) return invalid(msg, "k must be > 0");
    if (!(r.jump_intensity >= 0.0)) return invalid(msg, "jump_intensity must be >= 0");
    if (!(r.jump_volatility >= 0.0)) return invalid(msg, "jump_volatility must be >= 0");
    if (!finite(r.jump_mean)) return invalid(msg, "jump_mean must be finite");
    if (r.sampling == MPC_SAMPLING_PSEUDORANDOM && r.method == MPC_METHOD_STEPWISE)
      return unsupported(msg,
                         "stepwise Merton draws a variable number of normals per step from one sequential "
                         "stream; the pseudorandom stream replay covers the reference's terminal Merton "
                         "(method auto/terminal); use scrambled_sobol, randomized_halton, latin_hypercube or "
                         "counter_hash for stepwise Merton");
    if (r.sampling == MPC_SAMPLING_PSEUDORANDOM && r.technique != MPC_TECHNIQUE_STANDARD)
      return unsupported(msg, "the reference's pseudorandom Merton estimator is the standard technique");
    if (r.sampling == MPC_SAMPLING_PSEUDORANDOM && r.n_paths > (1ull << 30))
      return unsupported(msg, "pseudorandom Merton supports at most 2^30 paths per request");
    if (r.technique == MPC_TECHNIQUE_ANTITHETIC) return unsupported(msg, "Merton supports standard and control variate");
  }
  uint64_t dims_per_unit = r.n_steps;
  if (r.model == MPC_MODEL_HESTON) dims_per_unit = 2ull * r.n_steps;
  if (r.model == MPC_MODEL_MERTON) dims_per_unit = 3ull * (r.method == MPC_METHOD_STEPWISE ? r.n_steps : 1);
  if (r.workload == MPC_WORKLOAD_BASKET_CALL)
    dims_per_unit = uint64_t(r.n_assets) * (r.method == MPC_METHOD_STEPWISE ? r.n_steps : 1);
  if (dims_per_unit > (1ull << 20)) return unsupported(msg, "more than 2^20 sample dimensions per path");
  if (r.sampling == MPC_SAMPLING_RANDOMIZED_HALTON && dims_per_unit > 8192)
    return unsupported(msg, "randomized Halton supports at most 8192 dimensions");
  if (r.sampling == MPC_SAMPLING_LATIN_HYPERCUBE && dims_per_unit > 8192)
    return unsupported(msg, "Latin hypercube supports at most 8192 dimensions");
  return MPC_OK;
}

// The reference's own Merton: terminal, pseudorandom (mpc_merton.cu).
bool merton_stream_request(const mpc_request_t& r) {
  return r.workload == MPC_WORKLOAD_EUROPEAN_CALL && r.model == MPC_MODEL_MERTON &&
         r.sampling == MPC_SAMPLING_PSEUDORANDOM && r.method != MPC_METHOD_STEPWISE;
}

uint64_t estimate_bytes(const mpc_request_t& r) {
  // Fused: tile partials only.  Plain: materialised samples + payoff buffers.
  if (r.workload == MPC_WORKLOAD_ASIAN_MLMC) {
    uint64_t total = 0, fine = r.base_steps;
    for (uint32_t l = 0; l < r.levels && l < MPC_MAX_LEVELS; ++l) {
      uint64_t paths = r.target_stderr > 0.0 ? std::max<uint64_t>(r.pilot_paths_per_level, 1) : r.paths_per_level[l];
      if (r.precision == MPC_PRECISION_FP64_PLAIN) total = std::max(total, paths * fine * 8 + paths * 16);
      total += (paths / 256 + 1) * 64;
      fine *= std::max<uint32_t>(r.refinement_factor, 1);
    }
    return total + 4096;
  }
  uint64_t units = r.technique == MPC_TECHNIQUE_ANTITHETIC ? (r.n_paths + 1) / 2 : r.n_paths;
  if (is_lsm(r.workload)) {
    uint64_t elem = r.precision == MPC_PRECISION_FP64_PLAIN ? 8 : 4;
    // path matrix, one row of 16-double slots per exercise date for up to
    // 512 blocks (one block per SM), estimator partials and counters
    return r.n_paths * r.n_steps * elem + uint64_t(std::max<uint32_t>(r.n_steps, 1)) * 512 * 16 * 8 + 512 * 4 * 8 + 4096;
  }
  uint64_t dims = r.n_steps;
  if (r.model == MPC_MODEL_HESTON) dims = 2ull * r.n_steps;
  if (r.model == MPC_MODEL_MERTON) dims = 3ull * (r.method == MPC_METHOD_STEPWISE ? r.n_steps : 1);
  if (r.workload == MPC_WORKLOAD_BASKET_CALL) dims = uint64_t(r.n_assets) * (r.method == MPC_METHOD_STEPWISE ? r.n_steps : 1);
  if (r.workload == MPC_WORKLOAD_EUROPEAN_CALL && r.model == MPC_MODEL_GBM && r.method != MPC_METHOD_STEPWISE)
    dims = 1;
  uint64_t partials = (units / 256 + 1) * 64 + 1024;
  if (merton_stream_request(r)) {
    // stream outputs and jump bits (3 positions per path + spare segments),
    // segment maps and states, path starts, payoffs
    const uint64_t positions = 3 * r.n_paths + 64 * (2 + std::max<uint64_t>(r.n_threads, 1)) + 64;
    return positions * 8 + positions / 32 * 4 + positions / 64 * (18 + 1 + 8) + r.n_paths * 16 + partials;
  }
  if (r.precision == MPC_PRECISION_FP64_PLAIN) return units * dims * 8 + units * 16 + partials;
  return partials + 2048;
}

// --------------------------------------------------------------- prepare ---
static int sampler_of(int sampling) {
  switch (sampling) {
    case MPC_SAMPLING_PSEUDORANDOM:
      return SMP_XORSHIFT;
    case MPC_SAMPLING_RANDOMIZED_HALTON:
      return SMP_HALTON;
    case MPC_SAMPLING_LATIN_HYPERCUBE:
      return SMP_LHS;
    case MPC_SAMPLING_COUNTER_HASH:
      return SMP_COUNTER;
    default:
      return SMP_SOBOL;
  }
}

// BrownianBridgePlan::new (cpu.rs:5923-5962) flattened into the event
// program the device walks: the reference's interval stack is replayed and
// every pop becomes an event -- an op (midpoint of an interval longer than
// one step, consuming the next input dimension) or a leaf (one step).  Ops
// carry the reference's weights and stddev, computed the same way.  Returns
// false if the walk would need a deeper stack than the device holds.
static bool build_bridge_program(Prepared* p, uint32_t n, double maturity) {
  const double dt = maturity / double(n);
  p->bridge_ops.clear();
  p->bridge_events.assign((2ull * n - 1 + 31) / 32, 0u);
  std::vector<std::pair<uint32_t, uint32_t>> intervals{{0u, n}};
  uint32_t event = 0, depth = 1, max_depth = 1;  // depth: values on the device stack (starts with W(T))
  while (!intervals.empty()) {
    const auto [left, right] = intervals.back();
    intervals.pop_back();
    if (right <= left + 1) {  // leaf: pops one value
      ++event;
      --depth;
      continue;
    }
    const uint32_t mid = (left + right) / 2;
    const double t_left = double(left) * dt, t_mid = double(mid) * dt, t_right = double(right) * dt;
    const double denom = t_right - t_left;
    p->bridge_ops.push_back((t_right - t_mid) / denom);
    p->bridge_ops.push_back((t_mid - t_left) / denom);
    p->bridge_ops.push_back(std::sqrt((t_mid - t_left) * (t_right - t_mid) / denom));
    p->bridge_events[event >> 5] |= 1u << (event & 31);
    ++event;
    max_depth = std::max(max_depth, ++depth);  // op: pushes the midpoint
    intervals.push_back({mid, right});
    intervals.push_back({left, mid});
  }
  p->q.bridge_sqrt_t = std::sqrt(maturity);
  p->q.bridge_inv_sqrt_dt = 1.0 / std::sqrt(dt);
  return event == 2 * n - 1 && depth == 0 && max_depth <= kBridgeDepth && p->bridge_ops.size() == 3ull * (n - 1);
}

static std::vector<uint32_t> first_primes(size_t n) {
  std::vector<uint32_t> primes;
  uint32_t c = 2;
  while (primes.size() < n) {
    uint32_t lim = uint32_t(std::sqrt(double(c)));
    bool prime = true;
    for (uint32_t p : primes) {
      if (p > lim) break;
      if (c % p == 0) {
        prime = false;
        break;
      }
    }
    if (prime) primes.push_back(c);
    ++c;
  }
  return primes;
}

static double open01_u64(uint64_t v) {
  return std::max(double(v >> 11) * (1.0 / 9007199254740992.0), 2.2250738585072014e-308);
}

static uint64_t gcd64(uint64_t a, uint64_t b) {
  while (b) {
    uint64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// Sampler tables of a structured sampler: RandomizedHalton::new (cpu.rs:5692-5704)
// and LatinHypercube::new (cpu.rs:5737-5761).
static void build_sampler_tables(Prepared* p, uint64_t seed, uint64_t n_paths, uint64_t dims) {
  if (p->sampler == SMP_HALTON) {
    size_t count = std::max<size_t>(dims, 2);
    p->halton_primes = first_primes(count);
    p->halton_shifts.resize(count);
    for (size_t d = 0; d < count; ++d)
      p->halton_shifts[d] = open01_u64(splitmix64(seed + uint64_t(d) * 0x9E3779B97F4A7C15ull));
  } else if (p->sampler == SMP_LHS) {
    size_t count = std::max<size_t>(dims, 1);
    p->lhs.resize(count);
    for (size_t d = 0; d < count; ++d) {
      uint64_t mixed = splitmix64(seed ^ (uint64_t(d) * 0x9E3779B97F4A7C15ull) ^ 0xD1B54A32D192ED03ull);
      uint64_t modulus = std::max<uint64_t>(n_paths, 1), c = 1;
      if (modulus > 1) {  // coprime_multiplier (cpu.rs:5983-6002)
        c = std::max<uint64_t>(mixed % modulus, 1);
        if (c % 2 == 0) c += 1;
        while (gcd64(c, modulus) != 1) {
          c += 2;
          if (c >= modulus) c = 1;
        }
      }
      p->lhs[d].multiplier = c;
      p->lhs[d].offset = n_paths == 0 ? 0 : splitmix64(mixed ^ 0xA24BAED4963EE407ull) % n_paths;
      p->lhs[d].jitter_seed = splitmix64(mixed ^ 0x9FB21C651E98DF25ull);
    }
  }
}

int prepare(mpc_context* ctx, const mpc_request_t& r, Prepared* p, std::string* msg) {
  int st = validate(r, msg);
  if (st != MPC_OK) return st;
  *p = Prepared();
  DevReq& q = p->q;
  std::memset(&q, 0, sizeof(q));
  p->sampler = sampler_of(r.sampling);
  p->ppt_hint = r.paths_per_thread;
  p->block_hint = r.block_size;
  p->plain = r.precision == MPC_PRECISION_FP64_PLAIN;
  p->lsm = is_lsm(r.workload);
  p->mlmc = r.workload == MPC_WORKLOAD_ASIAN_MLMC;
  q.workload = r.workload;
  q.technique = r.technique;
  q.sampling = r.sampling;
  q.seed = r.seed;
  q.seed32 = uint32_t(r.seed);
  q.anti = r.technique == MPC_TECHNIQUE_ANTITHETIC;
  q.cv = r.technique == MPC_TECHNIQUE_CONTROL_VARIATE;
  q.n_paths = r.n_paths;
  q.n_units = q.anti ? (r.n_paths + 1) / 2 : r.n_paths;
  q.s0 = r.s0;
  q.k = r.k;
  q.barrier = r.barrier;
  q.log_s0 = std::log(r.s0 > 0 ? r.s0 : 1.0);
  q.log_barrier = r.barrier > 0.0 ? std::log(r.barrier) : -INFINITY;
  q.discount = std::exp(-r.r * r.t);
  q.cv_expectation = r.s0;
  q.n_chunks = 1;
  if (p->lsm || p->mlmc) return MPC_OK;  // driven by their own runners
  bool chunkable = true;
  if (r.workload == MPC_WORKLOAD_BASKET_CALL) {
    q.family = FAM_BASKET;
    const bool step = r.method == MPC_METHOD_STEPWISE;
    q.n_steps = step ? r.n_steps : 1;
    q.n_assets = r.n_assets;
    double dt = r.t / double(q.n_steps);
    cholesky(r.corr, r.n_assets, q.chol);
    double expectation = 0.0;
    for (uint32_t a = 0; a < r.n_assets; ++a) {
      q.b_drift[a] = (r.r - 0.5 * r.sigmas[a] * r.sigmas[a]) * dt;
      q.b_vol[a] = r.sigmas[a] * std::sqrt(dt);
      q.spots[a] = r.spots[a];
      q.weights[a] = r.weights[a];
      expectation += r.weights[a] * r.spots[a];  // basket_control_expectation (cpu.rs:7637-7639)
    }
    q.cv_expectation = expectation;
    q.normals_per_unit = uint64_t(r.n_assets) * q.n_steps;
    chunkable = false;  // the reference basket runs one stream (cpu.rs:7503-7518)
    p->path_steps = r.n_paths * q.n_steps;
  } else if (r.model == MPC_MODEL_HESTON) {
    q.family = FAM_HESTON;
    q.n_steps = r.n_steps;
    q.v0 = r.v0;
    q.kappa = r.kappa;
    q.theta = r.theta;
    q.xi = r.vol_of_vol;
    q.rho = r.rho;
    q.rho_perp = std::sqrt(std::max(1.0 - r.rho * r.rho, 0.0));
    q.dt = r.t / double(r.n_steps);
    q.sqrt_dt = std::sqrt(r.t / double(r.n_steps));
    q.rate = r.r;
    q.normals_per_unit = 2ull * r.n_steps;
    p->path_steps = r.n_paths * r.n_steps;
  } else if (r.model == MPC_MODEL_MERTON) {
    const bool step = r.method == MPC_METHOD_STEPWISE;
    q.family = step ? FAM_MERTON_STEP : FAM_MERTON_TERMINAL;
    q.n_steps = step ? r.n_steps : 1;
    double kj = r.jump_intensity * (std::exp(r.jump_mean + 0.5 * r.jump_volatility * r.jump_volatility) - 1.0);
    double dt = r.t / double(q.n_steps);
    q.drift_dt = (r.r - kj - 0.5 * r.sigma * r.sigma) * dt;
    q.vol_dt = r.sigma * std::sqrt(dt);
    q.lam_dt = r.jump_intensity * dt;
    q.lam_p0 = std::exp(-q.lam_dt);
    q.lam_p0_f = float(q.lam_p0);
    if (double(q.lam_p0_f) > q.lam_p0) q.lam_p0_f = std::nextafter(q.lam_p0_f, 0.0f);
    {  // the cumulative sums of sample_poisson in its own order of operations
      double prob = q.lam_p0, cum = q.lam_p0;
      for (int k = 0; k < 4; ++k) {
        if (k > 0) {
          prob *= q.lam_dt / double(k);
          cum += prob;
        }
        const double c = cum * 8388608.0 - 0.5;  // exact: u > cum  <=>  m > c
        q.pois_m[k] = c < 0.0 ? 0u : (c >= 8388607.0 ? 8388608u : uint32_t(std::floor(c)) + 1u);
      }
    }
    q.jump_mean = r.jump_mean;
    q.jump_vol = r.jump_volatility;
    q.normals_per_unit = 3ull * q.n_steps;
    p->path_steps = r.n_paths * q.n_steps;
  } else if (r.workload == MPC_WORKLOAD_EUROPEAN_CALL && r.method != MPC_METHOD_STEPWISE) {
    q.family = FAM_GBM_TERMINAL;  // EuropeanCallMethod::Auto == terminal (cpu.rs:3020-3025)
    q.n_steps = 1;
    q.drift_dt = (r.r - 0.5 * r.sigma * r.sigma) * r.t;
    q.vol_dt = r.sigma * std::sqrt(r.t);
    q.normals_per_unit = 1;
    chunkable = !q.anti;  // simulate_terminal_antithetic is single-stream (cpu.rs:7785-7805)
    p->path_steps = r.n_paths;
  } else {
    q.family = FAM_GBM_STEP;
    q.n_steps = r.n_steps;
    double dt = r.t / double(r.n_steps);
    q.drift_dt = (r.r - 0.5 * r.sigma * r.sigma) * dt;
    q.vol_dt = r.sigma * std::sqrt(dt);
    q.normals_per_unit = r.n_steps;
    // simulate_stepwise_antithetic (European) is single-stream (cpu.rs:7807-7835)
    if (r.workload == MPC_WORKLOAD_EUROPEAN_CALL && q.anti) chunkable = false;
    p->path_steps = r.n_paths * r.n_steps;
    // the bridge applies to the stepwise GBM workloads (cpu.rs:7113-7501); the
    // other families read bridge Sobol as plain Sobol, as the reference does
    if (r.sampling == MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE) {
      if (!build_bridge_program(p, r.n_steps, r.t)) {
        if (msg) *msg = "Brownian-bridge program exceeds the device stack";
        return MPC_E_UNSUPPORTED;
      }
      q.bridge = 1;
      q.family = FAM_GBM_BRIDGE;
    }
  }
  p->family = q.family;
  p->cv_expectation = q.cv_expectation;
  const uint64_t threads = r.n_threads <= 1 ? 1 : r.n_threads;
  if (p->sampler == SMP_XORSHIFT && chunkable && threads > 1 && q.n_units >= threads * 2000) {
    q.n_chunks = uint32_t(threads);
    q.chunk_base = q.n_units / threads;
    q.chunk_rem = q.n_units % threads;
  }
  build_sampler_tables(p, r.seed, r.n_paths, q.normals_per_unit);
  (void)ctx;
  return MPC_OK;
}

uint64_t block_key(const Prepared& p) {
  const int steps_bucket = 32 - __builtin_clz(std::max<uint32_t>(p.q.n_steps, 1));
  return (uint64_t(uint32_t(p.family)) << 48) | (uint64_t(p.sampler) << 40) | uint64_t(steps_bucket);
}

// Autotuner: the block size is the request's hint, else the one mpc_prepare
// measured for the request's kind (family, sampler, step bucket), else the
// context default; paths-per-thread is the hint, else picked so that a
// request spreads over at least four waves of resident blocks.  Cached per
// context.
Shape choose_shape(mpc_context* ctx, const Prepared& p) {
  std::lock_guard<std::mutex> lock(ctx->tuner.mu);
  uint32_t block = p.block_hint;
  if (!block) {
    auto bt = ctx->tuner.block.find(block_key(p));
    block = bt != ctx->tuner.block.end() ? bt->second : ctx->tuner.default_block;
  }
  if (p.ppt_hint) {  // the caller's paths-per-thread hint, not cached
    Shape s;
    s.block = block;
    s.ppt = p.ppt_hint;
    return s;
  }
  const int steps_bucket = 32 - __builtin_clz(std::max<uint32_t>(p.q.n_steps, 1));
  const int size_bucket = 64 - __builtin_clzll(std::max<uint64_t>(p.q.n_units, 1));
  const uint64_t key = (uint64_t(uint32_t(p.family)) << 48) | (uint64_t(p.sampler) << 40) |
                       (uint64_t(block) << 16) | (uint64_t(steps_bucket) << 8) | uint64_t(size_bucket);
  auto it = ctx->tuner.cache.find(key);
  if (it != ctx->tuner.cache.end()) {
    ++ctx->tuner.hits;
    return it->second;
  }
  ++ctx->tuner.misses;
  Shape s;
  s.block = block;
  int occ = std::max(1, fused_max_blocks_per_sm(p.family, p.sampler, int(block)));
  uint64_t resident = uint64_t(ctx->sm_count) * occ * block;
  // About four tiles per resident thread, except for the pseudorandom
  // stream, whose later units in a thread's tile start by one table jump
  // instead of a full seek: there fewer, longer tiles pay (1,048,576 GBM
  // paths x 64 steps: 0.244 ms at 1 unit per thread and tile, 0.172 ms at 4)
  const uint64_t tiles_per_thread = p.sampler == SMP_XORSHIFT ? 1 : 4;
  uint64_t want = p.q.n_units / std::max<uint64_t>(resident * tiles_per_thread, 1);
  uint32_t ppt = 1;
  while (ppt < 8 && uint64_t(ppt) * 2 <= want) ppt *= 2;
  s.ppt = ppt;
  ctx->tuner.cache[key] = s;
  return s;
}

static void summarize(double n, double sum, double sq, double* price, double* se) {
  double mean = sum / n;
  double var = (sq / n) - mean * mean;
  *price = mean;
  *se = std::sqrt(std::max(var, 0.0)) / std::sqrt(n);
}

// summarize_payoffs / summarize_block_estimates / summarize_control_variate (cpu.rs:7641-7771).
void summarize_moments(const Prepared& p, const double* m, mpc_result_t* out) {
  const double n = m[0];
  for (int i = 0; i < 6; ++i) out->moments[i] = m[i];
  out->n_samples = uint64_t(n);
  if (p.q.cv) {
    double pm = m[1] / n, cm = m[3] / n;
    double cvar = (m[4] / n) - cm * cm;
    if (cvar <= 2.220446049250313e-16) {
      summarize(n, m[1], m[2], &out->price, &out->stderr);
      return;
    }
    double cov = (m[5] / n) - pm * cm;
    double beta = cov / cvar;
    double e = p.cv_expectation;
    double adj = pm - beta * (cm - e);
    double adj_sq = (m[2] / n) - (2.0 * beta) * ((m[5] / n) - e * pm) +
                    (beta * beta) * ((m[4] / n) - (2.0 * e * cm) + (e * e));
    double var = std::max(adj_sq - adj * adj, 0.0);
    out->price = adj;
    out->stderr = std::sqrt(var) / std::sqrt(n);
    return;
  }
  summarize(n, m[1], m[2], &out->price, &out->stderr);
}

// Uploads the sampler tables of `reqs` into one aux buffer and points the descriptors at them.
static int upload_aux(mpc_context* ctx, std::vector<Prepared*>& reqs) {
  size_t bytes = 0;
  for (Prepared* p : reqs) {
    bytes += p->halton_primes.size() * 4 + 16;
    bytes += p->halton_shifts.size() * 8 + 16;
    bytes += p->lhs.size() * sizeof(LhsDim) + 16;
    bytes += p->bridge_ops.size() * 8 + p->bridge_events.size() * 4 + 32;
  }
  bool any = false;  // per-request tables to place
  for (Prepared* p : reqs) any = any || !p->halton_primes.empty() || !p->lhs.empty() || p->q.bridge;
  if (!any) return MPC_OK;
  void* d_aux = nullptr;
  int st = scratch(ctx, "aux", bytes, &d_aux);
  if (st != MPC_OK) return st;
  std::vector<uint8_t> host(bytes);
  size_t off = 0;
  auto place = [&](const void* src, size_t n) -> void* {
    off = (off + 15) & ~size_t(15);
    std::memcpy(host.data() + off, src, n);
    void* dev = static_cast<uint8_t*>(d_aux) + off;
    off += n;
    return dev;
  };
  for (Prepared* p : reqs) {
    if (!p->halton_primes.empty()) {
      p->q.halton_primes = static_cast<const uint32_t*>(place(p->halton_primes.data(), p->halton_primes.size() * 4));
      p->q.halton_shifts = static_cast<const double*>(place(p->halton_shifts.data(), p->halton_shifts.size() * 8));
    }
    if (!p->lhs.empty()) p->q.lhs = static_cast<const LhsDim*>(place(p->lhs.data(), p->lhs.size() * sizeof(LhsDim)));
    if (p->q.bridge) {  // a one-step program has a leaf event and no op
      if (!p->bridge_ops.empty())
        p->q.bridge_ops = static_cast<const double*>(place(p->bridge_ops.data(), p->bridge_ops.size() * 8));
      p->q.bridge_events =
          static_cast<const uint32_t*>(place(p->bridge_events.data(), p->bridge_events.size() * 4));
    }
  }
  MPC_CUDA(ctx, cudaMemcpyAsync(d_aux, host.data(), off, cudaMemcpyHostToDevice, ctx->stream));
  MPC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return MPC_OK;
}

// ------------------------------------------------------------ fused path ---
int run_fused(mpc_context* ctx, std::vector<Prepared*>& reqs, std::vector<mpc_result_t*>& outs,
              double* per_unit_host, uint64_t per_unit_cap) {
  const size_t n = reqs.size();
  if (n == 0) return MPC_OK;
  int st = upload_aux(ctx, reqs);
  if (st != MPC_OK) return st;
  // tiles: each request split into tiles of block * ppt units
  std::vector<uint32_t> tile_base(n), block_of(n);
  uint64_t total_tiles = 0;
  for (size_t i = 0; i < n; ++i) {
    Shape s = choose_shape(ctx, *reqs[i]);
    DevReq& q = reqs[i]->q;
    block_of[i] = s.block;
    q.tile_units = s.block * s.ppt;
    q.n_tiles = uint32_t((q.n_units + q.tile_units - 1) / q.tile_units);
    tile_base[i] = uint32_t(total_tiles);
    total_tiles += q.n_tiles;
  }
  if (total_tiles > (1ull << 31)) return fail(ctx, MPC_E_UNSUPPORTED, "batch too large (tiles)");
  // device buffers
  void *d_reqs, *d_tiles, *d_part, *d_mom, *d_done, *d_counter, *d_unit = nullptr;
  size_t groups = 0;
  if ((st = scratch(ctx, "reqs", n * sizeof(DevReq), &d_reqs))) return st;
  if ((st = scratch(ctx, "tiles", total_tiles * sizeof(Tile), &d_tiles))) return st;
  if ((st = scratch(ctx, "partials", total_tiles * MPC_MOMENTS * sizeof(double), &d_part))) return st;
  if ((st = scratch(ctx, "moments", n * MPC_MOMENTS * sizeof(double), &d_mom))) return st;
  if ((st = scratch(ctx, "done", n * sizeof(uint32_t), &d_done))) return st;
  if ((st = scratch(ctx, "counter", 64 * sizeof(uint32_t), &d_counter))) return st;
  if (per_unit_host) {  // the kernel writes every unit of request 0; the copy-out is clipped to the capacity
    if ((st = scratch(ctx, "per_unit", reqs[0]->q.n_units * sizeof(double), &d_unit))) return st;
  }
  for (size_t i = 0; i < n; ++i) {
    DevReq& q = reqs[i]->q;
    q.partials = static_cast<double*>(d_part) + size_t(tile_base[i]) * MPC_MOMENTS;
    q.moments = static_cast<double*>(d_mom) + i * MPC_MOMENTS;
    q.tiles_done = static_cast<uint32_t*>(d_done) + i;
    q.per_unit = (per_unit_host && i == 0) ? static_cast<double*>(d_unit) : nullptr;
  }
  // Launch groups: one persistent launch of the specialised kernel instance
  // per (sampler, family) pair present in the batch (a heterogeneous book of
  // GBM payoffs and baskets is two launches); within a group tiles are
  // ordered by per-tile cost, longest first.
  struct Group {
    int sampler, family;
    uint32_t block;
    std::vector<size_t> members;
  };
  const bool split_families = true;
  std::vector<Group> gl;
  for (size_t i = 0; i < n; ++i) {
    Group* g = nullptr;
    for (Group& x : gl)
      if (x.sampler == reqs[i]->sampler && x.block == block_of[i] &&
          (!split_families || x.family == reqs[i]->family))
        g = &x;
    if (!g) {
      gl.push_back({reqs[i]->sampler, reqs[i]->family, block_of[i], {}});
      g = &gl.back();
    }
    if (g->family != reqs[i]->family) g->family = -1;
    g->members.push_back(i);
  }
  groups = gl.size();
  if (groups > 64) return fail(ctx, MPC_E_UNSUPPORTED, "too many sampler groups");
  size_t desc_bytes = n * sizeof(DevReq);
  size_t tile_bytes = total_tiles * sizeof(Tile);
  size_t mom_bytes = n * MPC_MOMENTS * sizeof(double);
  void* pin = nullptr;
  if ((st = pinned_staging(ctx, desc_bytes + tile_bytes + mom_bytes + 256, &pin))) return st;
  uint8_t* hp = static_cast<uint8_t*>(pin);
  for (size_t i = 0; i < n; ++i) std::memcpy(hp + i * sizeof(DevReq), &reqs[i]->q, sizeof(DevReq));
  Tile* ht = reinterpret_cast<Tile*>(hp + desc_bytes);
  std::vector<uint32_t> group_first(groups), group_count(groups);
  uint64_t cursor = 0;
  for (size_t g = 0; g < groups; ++g) {
    std::vector<size_t> order = gl[g].members;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
      return double(reqs[a]->q.normals_per_unit + reqs[a]->q.n_steps) * reqs[a]->q.tile_units >
             double(reqs[b]->q.normals_per_unit + reqs[b]->q.n_steps) * reqs[b]->q.tile_units;
    });
    group_first[g] = uint32_t(cursor);
    for (size_t i : order)
      for (uint32_t t = 0; t < reqs[i]->q.n_tiles; ++t) ht[cursor++] = Tile{uint32_t(i), t};
    group_count[g] = uint32_t(cursor - group_first[g]);
  }
  double* hm = reinterpret_cast<double*>(hp + desc_bytes + tile_bytes);
  std::vector<uint64_t> grids(groups);
  for (size_t g = 0; g < groups; ++g) {
    int occ = std::max(1, fused_max_blocks_per_sm(gl[g].family, gl[g].sampler, int(gl[g].block)));
    grids[g] = std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(ctx->sm_count) * occ, group_count[g]));
  }
  // The sequence between the events: descriptors and tile list in, counters
  // zeroed, one launch per group, moments out.
  auto enqueue = [&]() -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(d_reqs, hp, desc_bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_tiles, ht, tile_bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_counter, 0, groups * sizeof(uint32_t), ctx->stream);
    if (e == cudaSuccess && groups > 1) e = cudaEventRecord(ctx->ev_fork, ctx->stream);
    bool used[mpc_context::kSideStreams] = {};
    for (size_t g = 0; g < groups && e == cudaSuccess; ++g) {
      cudaStream_t st = ctx->stream;
      if (g > 0) {
        const int k = int((g - 1) % mpc_context::kSideStreams);
        st = ctx->side[k];
        if (!used[k]) {
          used[k] = true;
          e = cudaStreamWaitEvent(st, ctx->ev_fork, 0);
          if (e != cudaSuccess) break;
        }
      }
      e = launch_fused(static_cast<DevReq*>(d_reqs), static_cast<Tile*>(d_tiles) + group_first[g], group_count[g],
                       static_cast<uint32_t*>(d_counter) + g, gl[g].family, gl[g].sampler, ctx->tabs, int(grids[g]),
                       int(gl[g].block), st);
    }
    for (int k = 0; k < mpc_context::kSideStreams; ++k) {  // join every forked stream, also after an error
      if (!used[k]) continue;
      const cudaError_t ej = cudaEventRecord(ctx->ev_join[k], ctx->side[k]);
      const cudaError_t ew = ej == cudaSuccess ? cudaStreamWaitEvent(ctx->stream, ctx->ev_join[k], 0) : ej;
      if (e == cudaSuccess) e = ew;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hm, d_mom, mom_bytes, cudaMemcpyDeviceToHost, ctx->stream);
    return e;
  };
  // everything the sequence bakes in: addresses, sizes, launch shapes
  std::vector<uint64_t> key = {uint64_t(uintptr_t(hp)), uint64_t(uintptr_t(d_reqs)), uint64_t(uintptr_t(d_tiles)),
                               uint64_t(uintptr_t(d_counter)), uint64_t(uintptr_t(d_mom)),
                               uint64_t(uintptr_t(ctx->tabs.sobol)), desc_bytes, tile_bytes, mom_bytes, groups};
  for (size_t g = 0; g < groups; ++g)
    key.insert(key.end(), {uint64_t(int64_t(gl[g].family)), uint64_t(gl[g].sampler), uint64_t(gl[g].block), grids[g],
                           group_first[g], group_count[g]});
  uint64_t launches_before = kernel_launch_count();
  bool replay = ctx->graph_exec && key == ctx->graph_key;
  if (!replay && key == ctx->last_batch_key) {  // second time in a row: capture (host only), then replay
    if (ctx->graph_exec) {
      cudaGraphExecDestroy(ctx->graph_exec);
      ctx->graph_exec = nullptr;
      ctx->graph_key.clear();
    }
    cudaGraph_t graph = nullptr;
    MPC_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const uint64_t counted = kernel_launch_count();
    const cudaError_t e = enqueue();
    const cudaError_t e_end = cudaStreamEndCapture(ctx->stream, &graph);
    if (e != cudaSuccess || e_end != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return cuda_fail(ctx, e != cudaSuccess ? e : e_end, "capture of the fused batch");
    }
    const uint64_t kernels = kernel_launch_count() - counted;
    discount_captured_launches(kernels);  // captured, not run: the replay below counts them
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e_inst = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e_inst != cudaSuccess) return cuda_fail(ctx, e_inst, "cudaGraphInstantiate");
    ctx->graph_exec = exec;
    ctx->graph_key = key;
    ctx->graph_kernels = kernels;
    replay = true;
  }
  MPC_CUDA(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));  // device time excludes capture on the host
  if (replay) {
    MPC_CUDA(ctx, cudaGraphLaunch(ctx->graph_exec, ctx->stream));
    count_graph_launches(ctx->graph_kernels);
    ++ctx->graph_replays;
  } else {
    const cudaError_t e = enqueue();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "fused pricing batch");
  }
  ctx->last_batch_key = key;
  MPC_CUDA(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  MPC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
  ctx->last_ms = ms;
  ctx->last_launches = kernel_launch_count() - launches_before;
  ctx->last_h2d = desc_bytes + tile_bytes;
  ctx->last_d2h = mom_bytes;
  for (size_t i = 0; i < n; ++i) {
    summarize_moments(*reqs[i], hm + i * MPC_MOMENTS, outs[i]);
    outs[i]->path_steps = reqs[i]->path_steps;
    outs[i]->runtime_ms = ms;
  }
  if (per_unit_host) {
    uint64_t count = std::min<uint64_t>(per_unit_cap, reqs[0]->q.n_units);
    MPC_CUDA(ctx, cudaMemcpy(per_unit_host, d_unit, count * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return MPC_OK;
}

// ------------------------------------------------------------ plain path ---
static int run_plain(mpc_context* ctx, Prepared* p, mpc_result_t* out, double* per_unit_host,
                     uint64_t per_unit_cap) {
  std::vector<Prepared*> one{p};
  int st = upload_aux(ctx, one);
  if (st != MPC_OK) return st;
  DevReq& q = p->q;
  const uint64_t units = q.n_units, dims = q.normals_per_unit;
  void *d_buf, *d_pay, *d_ctl = nullptr, *d_req, *d_part, *d_mom, *d_done;
  if ((st = scratch(ctx, "plain_buf", units * dims * sizeof(double), &d_buf))) return st;
  if ((st = scratch(ctx, "plain_pay", units * sizeof(double), &d_pay))) return st;
  if (q.cv && (st = scratch(ctx, "plain_ctl", units * sizeof(double), &d_ctl))) return st;
  q.tile_units = 2048;
  q.n_tiles = uint32_t((units + q.tile_units - 1) / q.tile_units);
  if ((st = scratch(ctx, "plain_req", sizeof(DevReq), &d_req))) return st;
  if ((st = scratch(ctx, "plain_part", size_t(q.n_tiles) * MPC_MOMENTS * sizeof(double), &d_part))) return st;
  if ((st = scratch(ctx, "plain_mom", MPC_MOMENTS * sizeof(double), &d_mom))) return st;
  if ((st = scratch(ctx, "plain_done", 16, &d_done))) return st;
  q.partials = static_cast<double*>(d_part);
  q.moments = static_cast<double*>(d_mom);
  q.tiles_done = static_cast<uint32_t*>(d_done);
  q.per_unit = nullptr;
  void* pin = nullptr;
  if ((st = pinned_staging(ctx, sizeof(DevReq) + MPC_MOMENTS * sizeof(double), &pin))) return st;
  std::memcpy(pin, &q, sizeof(DevReq));
  double* hm = reinterpret_cast<double*>(static_cast<uint8_t*>(pin) + sizeof(DevReq));
  uint64_t launches_before = kernel_launch_count();
  MPC_CUDA(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
  MPC_CUDA(ctx, cudaMemcpyAsync(d_req, pin, sizeof(DevReq), cudaMemcpyHostToDevice, ctx->stream));
  MPC_CUDA(ctx, cudaMemsetAsync(d_done, 0, 16, ctx->stream));
  cudaError_t e = launch_plain_generate(q, static_cast<double*>(d_buf), p->sampler, ctx->tabs, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "plain sample generation");
  e = launch_plain_simulate(q, static_cast<DevReq*>(d_req), static_cast<double*>(d_buf), static_cast<double*>(d_pay),
                            static_cast<double*>(d_ctl), ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "plain path simulation");
  e = launch_plain_reduce(static_cast<DevReq*>(d_req), static_cast<double*>(d_pay), static_cast<double*>(d_ctl), units,
                          q.n_tiles, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "plain reduction");
  MPC_CUDA(ctx, cudaMemcpyAsync(hm, d_mom, MPC_MOMENTS * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  MPC_CUDA(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  MPC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
  ctx->last_ms = ms;
  ctx->last_launches = kernel_launch_count() - launches_before;
  ctx->last_h2d = sizeof(DevReq);
  ctx->last_d2h = MPC_MOMENTS * sizeof(double);
  summarize_moments(*p, hm, out);
  out->path_steps = p->path_steps;
  out->runtime_ms = ms;
  if (per_unit_host) {
    uint64_t count = std::min<uint64_t>(per_unit_cap, units);
    MPC_CUDA(ctx, cudaMemcpy(per_unit_host, d_pay, count * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return MPC_OK;
}

// The reference's terminal pseudorandom Merton: each chunk's MonteCarloRng
// stream replayed on the device (mpc_merton.cu), payoffs reduced like the
// plain path.  Both precisions run this FP64 pipeline: its cost is the stream
// replay, and it reproduces the reference's per-path payoffs.
static int run_merton_stream(mpc_context* ctx, Prepared* p, mpc_result_t* out, double* per_unit_host,
                             uint64_t per_unit_cap) {
  DevReq& q = p->q;
  const uint64_t n = q.n_paths;
  MertonStreamArgs a{};
  a.n_paths = n;
  a.n_chunks = q.n_chunks <= 1 ? 1 : q.n_chunks;
  a.chunk_base = q.chunk_base;
  a.chunk_rem = q.chunk_rem;
  a.seed = q.seed;
  a.cv = q.cv;
  const uint64_t max_chunk = a.n_chunks <= 1 ? n : q.chunk_base + (q.chunk_rem ? 1 : 0);
  const uint64_t positions = 3 * max_chunk + 8;  // a path reads at most 3 positions past its start
  a.n_segs = (positions + kMertonSegment - 1) / kMertonSegment;
  a.qpad = (a.n_segs + 1) * kMertonSegment;  // one spare segment: the last one reads 2 bits past its end
  a.mean = q.lam_dt;                         // lambda T (terminal: dt = T)
  a.p0 = q.lam_p0;                           // exp(-lambda T), as sample_poisson computes it
  a.log_s0 = q.log_s0;
  a.drift_t = q.drift_dt;
  a.vol_t = q.vol_dt;
  a.jump_mean = q.jump_mean;
  a.jump_vol = q.jump_vol;
  a.k = q.k;
  a.discount = q.discount;
  const uint64_t chunks = a.n_chunks, segs = a.n_segs * chunks;
  void *d_x, *d_bits, *d_maps, *d_state, *d_before, *d_starts = nullptr, *d_pay, *d_ctl = nullptr;
  void *d_req, *d_part, *d_mom, *d_done;
  int st;
  if ((st = scratch(ctx, "merton_x", chunks * a.qpad * sizeof(uint64_t), &d_x))) return st;
  if ((st = scratch(ctx, "merton_bits", chunks * a.qpad / 32 * sizeof(uint32_t), &d_bits))) return st;
  if ((st = scratch(ctx, "merton_maps", segs * 9 * sizeof(uint16_t), &d_maps))) return st;
  if ((st = scratch(ctx, "merton_state", segs, &d_state))) return st;
  if ((st = scratch(ctx, "merton_before", segs * sizeof(uint64_t), &d_before))) return st;
  if (a.mean != 0.0 && (st = scratch(ctx, "merton_starts", n * sizeof(uint64_t), &d_starts))) return st;
  if ((st = scratch(ctx, "plain_pay", n * sizeof(double), &d_pay))) return st;
  if (q.cv && (st = scratch(ctx, "plain_ctl", n * sizeof(double), &d_ctl))) return st;
  a.x = static_cast<uint64_t*>(d_x);
  a.bits = static_cast<uint32_t*>(d_bits);
  a.maps = static_cast<uint16_t*>(d_maps);
  a.seg_state = static_cast<uint8_t*>(d_state);
  a.seg_before = static_cast<unsigned long long*>(d_before);
  a.starts = static_cast<uint64_t*>(d_starts);
  a.payoff = static_cast<double*>(d_pay);
  a.control = static_cast<double*>(d_ctl);
  q.tile_units = 2048;
  q.n_tiles = uint32_t((n + q.tile_units - 1) / q.tile_units);
  if ((st = scratch(ctx, "plain_req", sizeof(DevReq), &d_req))) return st;
  if ((st = scratch(ctx, "plain_part", size_t(q.n_tiles) * MPC_MOMENTS * sizeof(double), &d_part))) return st;
  if ((st = scratch(ctx, "plain_mom", MPC_MOMENTS * sizeof(double), &d_mom))) return st;
  if ((st = scratch(ctx, "plain_done", 16, &d_done))) return st;
  q.partials = static_cast<double*>(d_part);
  q.moments = static_cast<double*>(d_mom);
  q.tiles_done = static_cast<uint32_t*>(d_done);
  q.per_unit = nullptr;
  void* pin = nullptr;
  if ((st = pinned_staging(ctx, sizeof(DevReq) + MPC_MOMENTS * sizeof(double), &pin))) return st;
  std::memcpy(pin, &q, sizeof(DevReq));
  double* hm = reinterpret_cast<double*>(static_cast<uint8_t*>(pin) + sizeof(DevReq));
  uint64_t launches_before = kernel_launch_count();
  MPC_CUDA(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
  MPC_CUDA(ctx, cudaMemcpyAsync(d_req, pin, sizeof(DevReq), cudaMemcpyHostToDevice, ctx->stream));
  MPC_CUDA(ctx, cudaMemsetAsync(d_done, 0, 16, ctx->stream));
  cudaError_t e = launch_merton_stream(a, ctx->tabs, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "Merton stream replay");
  e = launch_plain_reduce(static_cast<DevReq*>(d_req), a.payoff, a.control, n, q.n_tiles, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "Merton reduction");
  MPC_CUDA(ctx, cudaMemcpyAsync(hm, d_mom, MPC_MOMENTS * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  MPC_CUDA(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  MPC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
  ctx->last_ms = ms;
  ctx->last_launches = kernel_launch_count() - launches_before;
  ctx->last_h2d = sizeof(DevReq);
  ctx->last_d2h = MPC_MOMENTS * sizeof(double);
  summarize_moments(*p, hm, out);
  out->path_steps = p->path_steps;
  out->runtime_ms = ms;
  if (per_unit_host) {
    uint64_t count = std::min<uint64_t>(per_unit_cap, n);
    MPC_CUDA(ctx, cudaMemcpy(per_unit_host, d_pay, count * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return MPC_OK;
}

// ------------------------------------------------------------------- LSM ---
static double powi(double a, int b) {  // f64::powi as compiler-rt __powidf2
  bool recip = b < 0;
  double r = 1.0;
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? 1.0 / r : r;
}

// Exercise schedule: every step (American, cpu.rs:3950) or the normalised
// Bermudan dates (normalize_bermudan_exercise_schedule, cpu.rs:5155-5183).
static std::vector<uint32_t> lsm_schedule(const mpc_request_t& r, bool* normalised) {
  std::vector<uint32_t> sched;
  *normalised = false;
  if (r.workload == MPC_WORKLOAD_AMERICAN_PUT) {
    for (uint32_t s = 1; s <= r.n_steps; ++s) sched.push_back(s);
    return sched;
  }
  std::vector<uint32_t> in(r.exercise_steps, r.exercise_steps + r.n_exercise);
  sched = in;
  std::sort(sched.begin(), sched.end());
  sched.erase(std::unique(sched.begin(), sched.end()), sched.end());
  if (sched != in) *normalised = true;
  if (std::find(sched.begin(), sched.end(), r.n_steps) == sched.end()) {
    sched.push_back(r.n_steps);
    *normalised = true;
  }
  return sched;
}

// Longstaff-Schwartz for a batch of requests (price_put_lsm_cpu,
// cpu.rs:3813-3945): requests are packed into cooperative launches, each
// request owning enough co-resident blocks for <= 8 paths per thread.
int run_lsm_batch(mpc_context* ctx, const std::vector<const mpc_request_t*>& reqs,
                  const std::vector<mpc_result_t*>& outs) {
  struct Job {
    size_t index;
    std::vector<uint32_t> sched;
    std::vector<double> disc_pow;
    std::vector<uint64_t> stride_tab;  // pseudorandom sampler: nibble table of the per-thread path stride jump
    std::vector<uint8_t> blob;         // host copy of the job's schedule, discount powers and stride table
    bool normalised;
    uint32_t degree, blocks;
    int fp64, sampler;
    LsmArgs args;
  };
  // regression rounds of a schedule (one per date before maturity; at least one slot row)
  auto lsm_rounds = [](size_t n_sched) -> uint64_t { return n_sched > 1 ? uint64_t(n_sched - 1) : 1ull; };
  std::vector<Job> jobs(reqs.size());
  for (size_t i = 0; i < reqs.size(); ++i) {
    const mpc_request_t& r = *reqs[i];
    Job& j = jobs[i];
    j.index = i;
    j.sched = lsm_schedule(r, &j.normalised);
    j.degree = std::min<uint32_t>(std::max<uint32_t>(r.basis_degree, 1), 3);
    j.fp64 = r.precision == MPC_PRECISION_FP64_PLAIN;
    j.sampler = sampler_of(r.sampling);
    const double dt = r.t / double(r.n_steps);
    const double disc_step = std::exp(-r.r * dt);
    j.disc_pow.resize(r.n_steps + 1);
    for (uint32_t k = 0; k <= r.n_steps; ++k) j.disc_pow[k] = powi(disc_step, int(k));
    const uint32_t cap = lsm_capacity(j.fp64, j.sampler);
    const uint64_t per_block_max = uint64_t(kLsmThreads) * kLsmPathsPerThreadMax;
    const uint64_t need = (r.n_paths + per_block_max - 1) / per_block_max;
    if (cap == 0 || need > cap)
      return fail(ctx, MPC_E_UNSUPPORTED, "LSM path count exceeds the co-resident capacity of the device");
    // about four paths per thread, at most one block per SM for one job (the
    // capacity is one 512-thread block per SM)
    uint64_t want = (r.n_paths + 4 * kLsmThreads - 1) / (4 * kLsmThreads);
    want = std::min<uint64_t>(want, std::min<uint64_t>(cap, 2ull * uint64_t(ctx->sm_count)));
    if (ctx->lsm_block_cap) {  // a caller that keeps only part of the device free for LSM launches
      if (need > ctx->lsm_block_cap)
        return fail(ctx, MPC_E_UNSUPPORTED, "LSM request needs more blocks than the SMs kept free for it");
      want = std::min<uint64_t>(want, ctx->lsm_block_cap);
    }
    j.blocks = uint32_t(std::max<uint64_t>(need, want));
    if (j.sampler == SMP_XORSHIFT)
      j.stride_tab = xorshift_jump_table(uint64_t(j.blocks) * kLsmThreads * uint64_t(r.n_steps));
    LsmArgs& a = j.args;
    std::memset(&a, 0, sizeof(a));
    a.n_paths = r.n_paths;
    a.n_steps = r.n_steps;
    a.n_sched = uint32_t(j.sched.size());
    a.degree = j.degree;
    a.sampler = uint32_t(j.sampler);
    a.seed = r.seed;
    a.seed32 = uint32_t(r.seed);
    a.fp64 = j.fp64;
    a.s0 = r.s0;
    a.k = r.k;
    a.drift = (r.r - 0.5 * r.sigma * r.sigma) * dt;
    a.vol = r.sigma * std::sqrt(dt);
    a.disc_step = disc_step;
    a.timeout_ns = 2000000000ull;
  }
  // launches: jobs of the same (fp64, sampler), packed under the capacity
  std::vector<bool> done(jobs.size(), false);
  double total_ms = 0.0;
  uint64_t launches_before = kernel_launch_count(), h2d = 0, d2h = 0;
  for (size_t first = 0; first < jobs.size(); ++first) {
    if (done[first]) continue;
    const int fp64 = jobs[first].fp64, sampler = jobs[first].sampler;
    const uint32_t cap = ctx->lsm_block_cap ? std::min(lsm_capacity(fp64, sampler), ctx->lsm_block_cap)
                                            : lsm_capacity(fp64, sampler);
    std::vector<size_t> group;
    uint32_t blocks = 0;
    for (size_t i = first; i < jobs.size(); ++i) {
      if (done[i] || jobs[i].fp64 != fp64 || jobs[i].sampler != sampler) continue;
      if (blocks + jobs[i].blocks > cap) continue;
      group.push_back(i);
      blocks += jobs[i].blocks;
      done[i] = true;
    }
    // device arena layout per job: paths | sched | disc | partials (one slot row per date) | final | out | counters
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    std::vector<size_t> offs;
    size_t bytes = align(group.size() * sizeof(LsmArgs));
    for (size_t i : group) {
      const Job& j = jobs[i];
      offs.push_back(bytes);
      const size_t elem = j.fp64 ? 8 : 4;
      bytes += align(j.args.n_paths * j.args.n_steps * elem) + align(j.sched.size() * 4) +
               align(j.disc_pow.size() * 8) + align(256 * 8) + align(lsm_rounds(j.sched.size()) * j.blocks * 16 * 8) +
               align(j.blocks * 4ull * 8) +
               align(8 * 8) + align(kLsmCounterBytes);
    }
    void* arena = nullptr;
    int st = scratch(ctx, "lsm_arena", bytes, &arena);
    if (st != MPC_OK) return st;
    std::vector<uint8_t> host(align(group.size() * sizeof(LsmArgs)));
    uint8_t* base = static_cast<uint8_t*>(arena);
    uint32_t block_first = 0;
    for (size_t g = 0; g < group.size(); ++g) {
      Job& j = jobs[group[g]];
      const size_t elem = j.fp64 ? 8 : 4;
      size_t o = offs[g];
      LsmArgs& a = j.args;
      a.paths = base + o;
      o += align(a.n_paths * a.n_steps * elem);
      {  // schedule | discount powers | stream stride table: one host-to-device copy
        const size_t sched_b = align(j.sched.size() * 4), disc_b = align(j.disc_pow.size() * 8);
        std::vector<uint8_t> blob(sched_b + disc_b + 256 * 8, 0);
        std::memcpy(blob.data(), j.sched.data(), j.sched.size() * 4);
        std::memcpy(blob.data() + sched_b, j.disc_pow.data(), j.disc_pow.size() * 8);
        if (!j.stride_tab.empty()) std::memcpy(blob.data() + sched_b + disc_b, j.stride_tab.data(), 256 * 8);
        a.sched = reinterpret_cast<const uint32_t*>(base + o);
        a.disc_pow = reinterpret_cast<const double*>(base + o + sched_b);
        a.stride_jump = j.stride_tab.empty() ? nullptr : reinterpret_cast<const uint64_t*>(base + o + sched_b + disc_b);
        j.blob.swap(blob);  // kept alive until the stream synchronises below
        MPC_CUDA(ctx, cudaMemcpyAsync(base + o, j.blob.data(), j.blob.size(), cudaMemcpyHostToDevice, ctx->stream));
        h2d += j.blob.size();
        o += sched_b + disc_b + align(256 * 8);
      }
      a.partials = reinterpret_cast<double*>(base + o);
      // one slot row per exercise date, all marked empty (every byte 0xFF)
      MPC_CUDA(ctx, cudaMemsetAsync(a.partials, 0xFF, lsm_rounds(j.sched.size()) * j.blocks * 16 * 8, ctx->stream));
      o += align(lsm_rounds(j.sched.size()) * j.blocks * 16 * 8);
      a.final_partials = reinterpret_cast<double*>(base + o);
      o += align(j.blocks * 4ull * 8);
      a.out = reinterpret_cast<double*>(base + o);
      o += align(8 * 8);
      // counters (zeroed per launch): block-done counter at 16, error code
      // at 32, failed index at 40
      a.barrier = reinterpret_cast<unsigned*>(base + o);
      a.done = a.barrier + 4;
      a.error = reinterpret_cast<int*>(a.barrier + 8);
      a.diag = reinterpret_cast<unsigned long long*>(a.barrier + 10);
      MPC_CUDA(ctx, cudaMemsetAsync(a.barrier, 0, kLsmCounterBytes, ctx->stream));
      a.paths_len = a.n_paths * a.n_steps;
      a.partials_len = uint32_t(lsm_rounds(j.sched.size()) * j.blocks * 16u);
      a.final_len = j.blocks * 4u;
      a.block_first = block_first;
      a.n_blocks = j.blocks;
      block_first += j.blocks;
      std::memcpy(host.data() + g * sizeof(LsmArgs), &a, sizeof(LsmArgs));
    }
    MPC_CUDA(ctx, cudaMemcpyAsync(base, host.data(), group.size() * sizeof(LsmArgs), cudaMemcpyHostToDevice,
                                  ctx->stream));
    h2d += group.size() * sizeof(LsmArgs);
    MPC_CUDA(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
    cudaError_t e = launch_lsm_batch(reinterpret_cast<const LsmArgs*>(base), uint32_t(group.size()), block_first,
                                     fp64, sampler, ctx->tabs, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "LSM cooperative launch");
    // pinned results: per job 8 doubles of output, then per job 16 bytes of
    // {error code, pad, failed index} copied from the counters at byte 32
    void* pin = nullptr;
    if ((st = pinned_staging(ctx, group.size() * 80, &pin))) return st;
    double* hout = static_cast<double*>(pin);
    uint8_t* hdiag = reinterpret_cast<uint8_t*>(hout + group.size() * 8);
    for (size_t g = 0; g < group.size(); ++g) {
      const LsmArgs& a = jobs[group[g]].args;
      MPC_CUDA(ctx, cudaMemcpyAsync(hout + g * 8, a.out, 8 * 8, cudaMemcpyDeviceToHost, ctx->stream));
      MPC_CUDA(ctx, cudaMemcpyAsync(hdiag + g * 16, a.error, 16, cudaMemcpyDeviceToHost, ctx->stream));
      d2h += 8 * 8 + 16;
    }
    MPC_CUDA(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
    MPC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
    total_ms += ms;
    for (size_t g = 0; g < group.size(); ++g) {
      const Job& j = jobs[group[g]];
      const mpc_request_t& r = *reqs[j.index];
      mpc_result_t* out = outs[j.index];
      const double* h = hout + g * 8;
      int code = 0;
      unsigned long long bad = 0;
      std::memcpy(&code, hdiag + g * 16, sizeof(code));
      std::memcpy(&bad, hdiag + g * 16 + 8, sizeof(bad));
      if (code == kLsmErrTimeout) {
        out->status = MPC_E_TIMEOUT;
        return fail(ctx, MPC_E_TIMEOUT, "LSM block barrier timed out");
      }
      if (code != 0) {
        static const char* what[] = {"", "", "path matrix", "regression partials", "estimator partials",
                                     "exercise date", "exercise discount", "job block range", "path coverage"};
        out->status = MPC_E_CUDA;
        return fail(ctx, MPC_E_CUDA,
                    std::string("LSM kernel self-check failed: ") + (code < 9 ? what[code] : "unknown") +
                        " index " + std::to_string(bad));
      }
      double price, se;
      summarize(h[0], h[1], h[2], &price, &se);
      uint32_t warnings = 0;
      if (r.workload == MPC_WORKLOAD_AMERICAN_PUT) {  // intrinsic floor (cpu.rs:3919-3925)
        double intrinsic = std::max(r.k - r.s0, 0.0);
        if (intrinsic > price) {
          price = intrinsic;
          se = 0.0;
          warnings |= MPC_WARN_INTRINSIC_FLOOR;
        }
      }
      if (r.basis_degree != j.degree) warnings |= MPC_WARN_BASIS_DEGREE_CLAMPED;
      if (j.normalised) warnings |= MPC_WARN_SCHEDULE_NORMALISED;
      if (r.n_threads > 1) warnings |= MPC_WARN_THREADS_IGNORED;
      out->price = price;
      out->stderr = se;
      out->n_samples = r.n_paths;
      out->path_steps = r.n_paths * r.n_steps;
      out->moments[0] = h[0];
      out->moments[1] = h[1];
      out->moments[2] = h[2];
      out->early_exercise_count = uint64_t(h[3]);
      out->maturity_exercise_count = uint64_t(h[4]);
      out->regression_steps = uint32_t(h[5]);
      out->basis_degree = j.degree;
      out->warnings |= warnings;
      out->runtime_ms = ms;
      out->status = MPC_OK;
    }
  }
  ctx->last_ms = total_ms;
  ctx->last_launches = kernel_launch_count() - launches_before;
  ctx->last_h2d = h2d;
  ctx->last_d2h = d2h;
  return MPC_OK;
}

static int run_lsm(mpc_context* ctx, const mpc_request_t& r, mpc_result_t* out) {
  return run_lsm_batch(ctx, {&r}, {out});
}

// ------------------------------------------------------------------ MLMC ---
uint64_t fine_steps(const mpc_request_t& r, uint32_t level) {
  uint64_t s = r.base_steps;
  for (uint32_t l = 0; l < level; ++l) s *= r.refinement_factor;
  return s;
}

// One MLMC level as a pricing unit family (simulate_asian_mlmc_level, cpu.rs:6641-6773).
void level_request(const mpc_request_t& r, uint64_t seed, uint32_t level, uint64_t paths, Prepared* p) {
  *p = Prepared();
  DevReq& q = p->q;
  std::memset(&q, 0, sizeof(q));
  const uint64_t fine = fine_steps(r, level);
  const uint64_t level_seed = derive_chunk_seed(seed, level);
  p->sampler = sampler_of(r.sampling);
  p->family = FAM_MLMC_LEVEL;
  p->plain = r.precision == MPC_PRECISION_FP64_PLAIN;
  q.family = FAM_MLMC_LEVEL;
  q.workload = MPC_WORKLOAD_ASIAN_MLMC;
  q.seed = level_seed;
  q.seed32 = uint32_t(level_seed);
  q.n_chunks = 1;
  q.n_paths = paths;
  q.n_units = paths;
  q.n_steps = uint32_t(fine);
  q.normals_per_unit = fine;
  q.level = level;
  q.refinement = r.refinement_factor;
  q.s0 = r.s0;
  q.k = r.k;
  q.log_s0 = std::log(r.s0);
  q.discount = std::exp(-r.r * r.t);
  double fdt = r.t / double(fine);
  q.f_drift = (r.r - 0.5 * r.sigma * r.sigma) * fdt;
  q.f_vol = r.sigma * std::sqrt(fdt);
  q.inv_fine = 1.0 / double(fine);
  if (level > 0) {
    q.coarse_steps = fine / r.refinement_factor;
    double cdt = r.t / double(q.coarse_steps);
    q.c_drift = (r.r - 0.5 * r.sigma * r.sigma) * cdt;
    q.c_vol = r.sigma * std::sqrt(cdt);
    q.inv_sqrt_m = 1.0 / std::sqrt(double(r.refinement_factor));
    q.inv_coarse = 1.0 / double(q.coarse_steps);
  }
  p->path_steps = paths * (fine + (level > 0 ? fine / r.refinement_factor : 0));
  build_sampler_tables(p, level_seed, paths, fine);
}

// Prices a list of level requests (any mix of MLMC requests, replicates and
// levels): FP32 entries in one fused batch, FP64-plain entries one launch
// sequence each.  Returns per entry (mean, population variance).
static int run_level_list(mpc_context* ctx, std::vector<Prepared>& preps, std::vector<double>* mean,
                          std::vector<double>* var, double* device_ms) {
  std::vector<mpc_result_t> res(preps.size());
  std::vector<Prepared*> fused;
  std::vector<mpc_result_t*> fused_out;
  for (size_t i = 0; i < preps.size(); ++i) {
    std::memset(&res[i], 0, sizeof(res[i]));
    if (preps[i].plain) {
      int st = run_plain(ctx, &preps[i], &res[i], nullptr, 0);
      if (st != MPC_OK) return st;
      *device_ms += ctx->last_ms;
    } else {
      fused.push_back(&preps[i]);
      fused_out.push_back(&res[i]);
    }
  }
  if (!fused.empty()) {
    int st = run_fused(ctx, fused, fused_out, nullptr, 0);
    if (st != MPC_OK) return st;
    *device_ms += ctx->last_ms;
  }
  mean->assign(preps.size(), 0.0);
  var->assign(preps.size(), 0.0);
  for (size_t i = 0; i < preps.size(); ++i) {
    double nn = res[i].moments[0];
    double m = res[i].moments[1] / nn;
    (*mean)[i] = m;
    (*var)[i] = (res[i].moments[2] / nn) - m * m;
  }
  return MPC_OK;
}

// arithmetic_asian_call_price_mlmc_{single,replicated}_cpu (cpu.rs:3612-3751)
// with solve_arithmetic_asian_mlmc_tolerance_cpu (cpu.rs:3352-3423) when
// target_stderr > 0, for a batch of requests: every pilot level of every
// request runs in one fused launch, then every level of every replicate.
// Level variances and the allocation are FP64 on the host.
uint64_t mlmc_replicates(const mpc_request_t& r) {
  const bool pseudo = r.sampling == MPC_SAMPLING_PSEUDORANDOM || r.sampling == MPC_SAMPLING_COUNTER_HASH;
  return pseudo ? 1 : std::max<uint32_t>(r.scramble_replicates, 1);
}

static uint64_t level_cost(const mpc_request_t& r, uint32_t l) {
  return fine_steps(r, l) + (l == 0 ? 0 : fine_steps(r, l) / r.refinement_factor);
}

// solve_arithmetic_asian_mlmc_tolerance_cpu's allocation (cpu.rs:3352-3423,
// 3539-3565) from the pilot level variances: fills r.paths_per_level and the
// solver fields of `out`.
void mlmc_allocate(mpc_request_t& r, const double* pilot_var, mpc_result_t* out) {
  const uint32_t L = r.levels;
  const uint64_t reps = mlmc_replicates(r);
  std::vector<double> var(L);
  for (uint32_t l = 0; l < L; ++l) var[l] = std::max(pilot_var[l], 1.0e-18);
  auto allocate = [&](double target_variance, bool by_budget, uint64_t budget, std::vector<uint64_t>& paths) {
    double denom = 0.0;
    for (uint32_t l = 0; l < L; ++l) denom += std::sqrt(var[l] * double(level_cost(r, l)));
    uint64_t total = 0;
    for (uint32_t l = 0; l < L; ++l) {
      double w = std::sqrt(var[l] / double(level_cost(r, l)));
      double raw = by_budget ? std::ceil(double(budget) * w / denom) : std::ceil(denom * w / target_variance);
      paths[l] = std::max<uint64_t>(uint64_t(raw), 2);
      total += paths[l] * level_cost(r, l);
    }
    return total;
  };
  auto est_se = [&](const std::vector<uint64_t>& paths) {
    double v = 0.0;
    for (uint32_t l = 0; l < L; ++l) v += var[l] / double(paths[l]);
    return std::sqrt(v / double(reps));
  };
  std::vector<uint64_t> paths(L);
  uint64_t updates = allocate(r.target_stderr * r.target_stderr * double(reps), false, 0, paths) * reps;
  double est = est_se(paths);
  if (updates < r.min_step_updates) {
    uint64_t per = std::max<uint64_t>((r.min_step_updates + reps - 1) / reps, 1);
    updates = allocate(0, true, per, paths) * reps;
    est = est_se(paths);
  }
  bool hit = false;
  if (updates > r.max_step_updates) {
    hit = true;
    uint64_t per = std::max<uint64_t>(r.max_step_updates / reps, 1);
    updates = allocate(0, true, per, paths) * reps;
    est = est_se(paths);
  }
  for (uint32_t l = 0; l < L; ++l) r.paths_per_level[l] = paths[l];
  out->estimated_stderr = est;
  out->target_met = (est <= r.target_stderr && updates <= r.max_step_updates) ? 1 : 0;
  out->max_step_updates_hit = hit ? 1 : 0;
}

// The estimator of arithmetic_asian_call_price_mlmc_{single,replicated}_cpu
// (cpu.rs:3612-3751) from the main-phase level results, ordered replicate by
// replicate, level by level.
void mlmc_finish(const mpc_request_t& r, const double* mm, double* mv, double device_ms, mpc_result_t* out) {
  const uint32_t L = r.levels;
  const uint64_t reps = mlmc_replicates(r);
  std::vector<double> rep_price(reps);
  double single_se = 0.0;
  uint64_t total_paths = 0, total_updates = 0;
  for (uint64_t rep = 0; rep < reps; ++rep) {
    double price = 0.0, varc = 0.0;
    for (uint32_t l = 0; l < L; ++l) {
      const size_t e = rep * L + l;
      mv[e] = std::max(mv[e], 0.0);
      price += mm[e];
      varc += mv[e] / double(r.paths_per_level[l]);
      total_paths += r.paths_per_level[l];
      total_updates += r.paths_per_level[l] * level_cost(r, l);
    }
    rep_price[rep] = price;
    single_se = std::sqrt(varc);
  }
  double price = 0.0;
  for (double p : rep_price) price += p;
  price /= double(reps);
  double se = single_se;
  if (reps > 1) {
    double sv = 0.0;
    for (double p : rep_price) sv += (p - price) * (p - price);
    sv /= double(reps - 1);
    se = std::sqrt(sv / double(reps));
  }
  out->price = price;
  out->stderr = se;
  out->n_levels = L;
  out->total_paths = total_paths;
  out->total_step_updates = total_updates;
  out->path_steps = total_updates;
  for (uint32_t l = 0; l < L; ++l) {
    double mean = 0.0;
    for (uint64_t rep = 0; rep < reps; ++rep) mean += mm[rep * L + l];
    mean /= double(reps);
    double var = mv[l];
    if (reps > 1) {
      var = 0.0;
      for (uint64_t rep = 0; rep < reps; ++rep) {
        double d = mm[rep * L + l] - mean;
        var += d * d;
      }
      var /= double(reps - 1);
    }
    out->level_mean[l] = mean;
    out->level_variance[l] = var;
    out->level_paths[l] = r.paths_per_level[l] * reps;
    out->level_fine_steps[l] = fine_steps(r, l);
  }
  out->runtime_ms = device_ms;
  out->status = MPC_OK;
}

// arithmetic_asian_call_price_mlmc_{single,replicated}_cpu (cpu.rs:3612-3751)
// with solve_arithmetic_asian_mlmc_tolerance_cpu (cpu.rs:3352-3423) when
// target_stderr > 0, for a batch of requests: every pilot level of every
// request runs in one fused launch, then every level of every replicate.
// Level variances and the allocation are FP64 on the host.
int run_mlmc_batch(mpc_context* ctx, const std::vector<const mpc_request_t*>& reqs,
                   const std::vector<mpc_result_t*>& outs) {
  std::vector<mpc_request_t> jobs;
  for (const mpc_request_t* rq : reqs) jobs.push_back(*rq);
  double device_ms = 0.0;
  uint64_t launches_before = kernel_launch_count();
  // pilot phase for the tolerance solver
  std::vector<Prepared> pilot;
  std::vector<size_t> pilot_first(jobs.size(), 0);
  for (size_t i = 0; i < jobs.size(); ++i) {
    pilot_first[i] = pilot.size();
    if (jobs[i].target_stderr <= 0.0) continue;
    for (uint32_t l = 0; l < jobs[i].levels; ++l) {
      pilot.emplace_back();
      level_request(jobs[i], jobs[i].seed, l, jobs[i].pilot_paths_per_level, &pilot.back());
    }
  }
  if (!pilot.empty()) {
    std::vector<double> pm, pv;
    int st = run_level_list(ctx, pilot, &pm, &pv, &device_ms);
    if (st != MPC_OK) return st;
    for (size_t i = 0; i < jobs.size(); ++i)
      if (jobs[i].target_stderr > 0.0) mlmc_allocate(jobs[i], pv.data() + pilot_first[i], outs[i]);
  }
  // main phase: every level of every replicate of every request
  std::vector<Prepared> mains;
  std::vector<size_t> main_first(jobs.size(), 0);
  for (size_t i = 0; i < jobs.size(); ++i) {
    const mpc_request_t& r = jobs[i];
    const uint64_t reps = mlmc_replicates(r);
    main_first[i] = mains.size();
    for (uint64_t rep = 0; rep < reps; ++rep) {
      uint64_t seed = reps > 1 ? derive_chunk_seed(r.seed, rep) : r.seed;
      for (uint32_t l = 0; l < r.levels; ++l) {
        mains.emplace_back();
        level_request(r, seed, l, r.paths_per_level[l], &mains.back());
      }
    }
  }
  std::vector<double> mm, mv;
  int st = run_level_list(ctx, mains, &mm, &mv, &device_ms);
  if (st != MPC_OK) return st;
  for (size_t i = 0; i < jobs.size(); ++i)
    mlmc_finish(jobs[i], mm.data() + main_first[i], mv.data() + main_first[i], device_ms, outs[i]);
  ctx->last_ms = device_ms;
  ctx->last_launches = kernel_launch_count() - launches_before;
  return MPC_OK;
}

static int run_mlmc(mpc_context* ctx, const mpc_request_t& r, mpc_result_t* out) {
  return run_mlmc_batch(ctx, {&r}, {out});
}

static int price_one(mpc_context* ctx, const mpc_request_t* req, mpc_result_t* out, double* per_unit,
                     uint64_t cap) {
  std::memset(out, 0, sizeof(*out));
  std::string msg;
  int st = validate(*req, &msg);
  if (st != MPC_OK) {
    out->status = st;
    return fail(ctx, st, msg);
  }
  if (req->workload == MPC_WORKLOAD_ASIAN_MLMC) {
    st = run_mlmc(ctx, *req, out);
  } else if (is_lsm(req->workload)) {
    st = run_lsm(ctx, *req, out);
  } else {
    Prepared p;
    st = prepare(ctx, *req, &p, &msg);
    if (st != MPC_OK) {
      out->status = st;
      return fail(ctx, st, msg);
    }
    if (merton_stream_request(*req)) {
      st = run_merton_stream(ctx, &p, out, per_unit, cap);
    } else if (p.plain) {
      st = run_plain(ctx, &p, out, per_unit, cap);
    } else {
      std::vector<Prepared*> pp{&p};
      std::vector<mpc_result_t*> oo{out};
      st = run_fused(ctx, pp, oo, per_unit, cap);
    }
  }
  out->status = st;
  return st;
}

// ----------------------------------------------------------- device setup ---
// Inverse standard normal CDF to full FP64 accuracy on the host: Acklam's
// rational as the start, then Halley steps on Phi(x) - p with erfc (the
// refinement Acklam publishes with the rational).
static double inverse_normal_refined(double p) {
  const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                       1.383577518672690e+02,  -3.066479806614716e+01, 2.506628277459239e+00};
  const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                       6.680131188771972e+01,  -1.328068155288572e+01};
  const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                       -2.549732539343734e+00, 4.374664141464968e+00,  2.938163982698783e+00};
  const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00, 3.754408661907416e+00};
  const double lo = 0.02425;
  double x;
  if (p < lo || p > 1.0 - lo) {
    const double q = std::sqrt(-2.0 * std::log(p < lo ? p : 1.0 - p));
    x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
        ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    if (p > 1.0 - lo) x = -x;
  } else {
    const double q = p - 0.5, r = q * q;
    x = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
        (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
  }
  for (int it = 0; it < 2; ++it) {
    const double e = 0.5 * std::erfc(-x / std::sqrt(2.0)) - p;
    const double u = e * std::sqrt(2.0 * M_PI) * std::exp(0.5 * x * x);
    x -= u / (1.0 + 0.5 * x * u);
  }
  return x;
}

// FP32 inverse-normal segments of the fused Sobol path.  The argument
// v = min(u, 1 - u) of a 23-bit midpoint uniform lies in [2^-24, 1/2); each
// binade [2^e, 2^(e+1)), e = -24 .. -2, is cut into 32 equal segments, and a
// segment's cubic in t in [0, 1) (the position inside the segment)
// interpolates Phi^-1(v) at the 4 Chebyshev nodes.  Max error over all 2^23
// uniforms: 4.5e-7.  The kernels evaluate it at t / 32 (the segment's 18
// mantissa bits read as a float in [0, 1/32) without a shift), so
// coefficient k is stored times 32^k: a power-of-two scaling that every
// Horner step carries exactly, so the values equal those of the cubic in t.
static void build_icdf_segments(uint32_t* out) {
  for (int e = 0; e < 23; ++e)
    for (int s = 0; s < 32; ++s) {
      const double lo = std::ldexp(1.0 + s / 32.0, e - 24), hi = std::ldexp(1.0 + (s + 1) / 32.0, e - 24);
      double t[4], f[4];
      for (int k = 0; k < 4; ++k) {
        t[k] = 0.5 - 0.5 * std::cos(M_PI * (2 * k + 1) / 8.0);
        f[k] = inverse_normal_refined(lo + t[k] * (hi - lo));
      }
      for (int j = 1; j < 4; ++j)  // Newton divided differences
        for (int k = 3; k >= j; --k) f[k] = (f[k] - f[k - 1]) / (t[k] - t[k - j]);
      double poly[4] = {f[3], 0.0, 0.0, 0.0};  // Newton form -> monomials in t
      for (int j = 2; j >= 0; --j) {
        double next[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < 3; ++k) {
          next[k + 1] += poly[k];
          next[k] -= poly[k] * t[j];
        }
        next[0] += f[j];
        for (int k = 0; k < 4; ++k) poly[k] = next[k];
      }
      for (int k = 0; k < 4; ++k) {
        const float c = std::ldexp((float)poly[k], 5 * k);
        std::memcpy(&out[(e * 32 + s) * 4 + k], &c, sizeof(c));
      }
    }
}

// Nibble table [q][v] of T^k, T the xorshift64* state transition: entry
// (q, v) is T^k applied to the nibble value v placed at bit 4q, so a state x
// jumps k draws with 16 lookups (gf2_apply).  The images of the 64 basis
// vectors come from the T^(2^b) nibble tables (16 lookups per set bit of k
// each); tables are kept per k (a request shape needs the same one every
// call), at most 256 of them.
std::vector<uint64_t> xorshift_jump_table(uint64_t k) {
  static std::mutex mu;
  static std::unordered_map<uint64_t, std::vector<uint64_t>> cache;
  static std::vector<uint64_t> powers;  // [64][16][16]: T^(2^b)
  std::lock_guard<std::mutex> lock(mu);
  auto hit = cache.find(k);
  if (hit != cache.end()) return hit->second;
  if (powers.empty()) {
    std::vector<uint32_t> sob;
    build_tables(sob, powers);
  }
  std::vector<uint64_t> cols(64);
  for (int i = 0; i < 64; ++i) {
    uint64_t x = 1ull << i;
    for (uint64_t kk = k; kk; kk &= kk - 1) {
      const uint64_t* t = &powers[size_t(__builtin_ctzll(kk)) * 256];
      uint64_t y = 0;
      for (int q = 0; q < 16; ++q) y ^= t[q * 16 + ((x >> (4 * q)) & 0xF)];
      x = y;
    }
    cols[i] = x;
  }
  std::vector<uint64_t> tab(256, 0ull);
  for (int q = 0; q < 16; ++q)
    for (int v = 0; v < 16; ++v)
      for (int j = 0; j < 4; ++j)
        if ((v >> j) & 1) tab[q * 16 + v] ^= cols[4 * q + j];
  if (cache.size() >= 256) cache.clear();
  cache.emplace(k, tab);
  return tab;
}

void build_tables(std::vector<uint32_t>& sob, std::vector<uint64_t>& jump) {
  sob.assign(size_t(MPC_SOBOL_TABLE_WORDS), 0u);
  build_icdf_segments(&sob[MPC_ICDF_OFFSET]);
  auto reverse = [](uint32_t x) {
    uint32_t r = 0;
    for (int b = 0; b < 32; ++b) r |= ((x >> b) & 1u) << (31 - b);
    return r;
  };
  for (int d = 0; d < MPC_SOBOL_TABLE_DIMS; ++d)
    for (int q = 0; q < 8; ++q)
      for (int v = 0; v < 16; ++v) {
        uint32_t x = 0;
        for (int j = 0; j < 4; ++j)
          if ((v >> j) & 1) x ^= kSobolDirections[d][4 * q + j];
        sob[(size_t(d) * 8 + q) * 16 + v] = x;
        sob[MPC_SOBOL_NIBBLE_WORDS + size_t(q * 16 + v) * MPC_SOBOL_TABLE_DIMS + d] = reverse(x);
      }
  // Columns of the xorshift64* transition T (image of each basis vector), then T^(2^b).
  auto step = [](uint64_t x) {
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    return x;
  };
  std::vector<uint64_t> M(64), N(64);
  for (int i = 0; i < 64; ++i) M[i] = step(1ull << i);
  auto apply = [](const std::vector<uint64_t>& m, uint64_t x) {
    uint64_t y = 0;
    for (int i = 0; i < 64; ++i)
      if ((x >> i) & 1) y ^= m[i];
    return y;
  };
  jump.assign(64 * 256, 0ull);
  for (int b = 0; b < 64; ++b) {
    for (int q = 0; q < 16; ++q)
      for (int v = 0; v < 16; ++v) {
        uint64_t y = 0;
        for (int j = 0; j < 4; ++j)
          if ((v >> j) & 1) y ^= M[4 * q + j];
        jump[size_t(b) * 256 + q * 16 + v] = y;
      }
    for (int i = 0; i < 64; ++i) N[i] = apply(M, M[i]);  // M <- M * M
    M.swap(N);
  }
}

}  // namespace mpc

// ======================================================= C entry points ====
extern "C" {

// ------------------------------------------------------------ cost model ---
// Device rates in units per second (path-steps for stepwise families, paths
// for terminal ones), steady-state CUDA-event time of one request of
// 1,048,576 paths x 64 steps on a B200 (148 SMs, 1965 MHz), per sampler
// {pseudorandom, counter hash, scrambled Sobol, Halton/LHS}.
namespace {
struct RateRow {
  double fp32[4], fp64[4];
};
// Rows of the rate table; the bridge row has one rate per precision (all
// columns alike).
enum CostRow : int {
  ROW_GBM_STEP,
  ROW_ASIAN,
  ROW_GBM_TERMINAL,
  ROW_HESTON,
  ROW_MERTON_STEP,
  ROW_MERTON_TERMINAL,
  ROW_BASKET2,
  ROW_BRIDGE,
  ROW_COUNT
};
const RateRow kRates[ROW_COUNT] = {
    {{3.72e11, 3.25e11, 3.85e11, 9.05e10}, {1.31e11, 1.35e11, 5.96e10, 5.38e10}},  // GBM stepwise
    {{3.48e11, 2.93e11, 3.50e11, 8.84e10}, {1.12e11, 1.16e11, 5.59e10, 5.02e10}},  // arithmetic Asian
    {{5.4e10, 1.83e10, 1.53e10, 1.11e10}, {7.38e9, 2.45e10, 1.98e10, 1.12e10}},    // GBM terminal (pseudorandom FP32: + kTerminalFixedMs)
    {{2.51e11, 1.93e11, 2.23e11, 5.37e10}, {7.09e10, 6.85e10, 3.02e10, 3.14e10}},  // Heston
    {{1.05e11, 1.05e11, 1.97e11, 4.30e10}, {4.16e10, 4.16e10, 2.65e10, 2.63e10}},  // Merton stepwise
    {{1.70e10, 1.70e10, 1.44e10, 7.09e9}, {1.83e10, 1.83e10, 1.30e10, 6.60e9}},    // Merton terminal
    {{5.46e9, 1.53e10, 1.28e10, 7.74e9}, {5.49e9, 1.58e10, 1.13e10, 6.77e9}},      // 2-asset basket
    {{1.41e11, 1.41e11, 1.41e11, 1.41e11}, {4.59e10, 4.59e10, 4.59e10, 4.59e10}},  // GBM stepwise, bridge
};
// FP32 pseudorandom terminal GBM: each thread's first path of a tile takes a
// full stream seek and its later paths one table jump each, so the time has
// an intercept (about one full seek per resident thread, scaled down for
// requests with fewer paths than resident threads) beside the per-path
// rate (fit to 2,097,152 and 4,194,304 paths on a B200: 0.082 and 0.119 ms).
const double kTerminalFixedMs = 0.046;
const double kLsmFixedMs = 0.22, kLsmRate = 1.7e11; // 49 cross-block date rounds, then path-steps
                                                      // (fit to 524,288 paths x 50 dates, FP32: 0.37 ms)
const double kCallOverheadMs = 0.035;               // events, copies, one launch
const double kFirstCallMs = 2.0;                    // tables and buffers of a new shape
const int kCostColumns = 4;
const int kCalibrationSampling[kCostColumns] = {MPC_SAMPLING_PSEUDORANDOM, MPC_SAMPLING_COUNTER_HASH,
                                                MPC_SAMPLING_SCRAMBLED_SOBOL, MPC_SAMPLING_RANDOMIZED_HALTON};

int rate_column(int sampling) {
  switch (sampling) {
    case MPC_SAMPLING_PSEUDORANDOM:
      return 0;
    case MPC_SAMPLING_COUNTER_HASH:
      return 1;
    case MPC_SAMPLING_SCRAMBLED_SOBOL:
    case MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE:
      return 2;
    default:
      return 3;
  }
}

// Units per second of (row, precision, column): the context's calibrated
// rate when it has one, else the built-in B200 rate scaled by SM count.
struct RateSource {
  const std::vector<double>* calibrated;  // [row][2][kCostColumns] or null
  double scale;
  const std::vector<double>* fixed = nullptr;  // calibrated intercepts (ms), same layout, or null
  double at(int row, bool fp64, int col) const {
    if (calibrated && !calibrated->empty()) {
      const double v = (*calibrated)[(size_t(row) * 2 + (fp64 ? 1 : 0)) * kCostColumns + col];
      if (v > 0.0) return v;
    }
    return (fp64 ? kRates[row].fp64[col] : kRates[row].fp32[col]) * scale;
  }
  // per-call intercept of the terminal GBM row (ms)
  double fixed_at(int row, bool fp64, int col) const {
    if (calibrated && !calibrated->empty() && fixed && !fixed->empty()) {
      const double r = (*calibrated)[(size_t(row) * 2 + (fp64 ? 1 : 0)) * kCostColumns + col];
      if (r > 0.0) return (*fixed)[(size_t(row) * 2 + (fp64 ? 1 : 0)) * kCostColumns + col];
    }
    return row == ROW_GBM_TERMINAL && !fp64 && col == 0 ? kTerminalFixedMs : 0.0;
  }
  bool measured_here() const { return calibrated && !calibrated->empty(); }
};

int estimate_cost_with(const mpc_request_t* req, const RateSource& rates, mpc_cost_t* out) {
  if (!req || !out) return MPC_E_INVALID_CONFIG;
  std::memset(out, 0, sizeof(*out));
  std::string msg;
  int st = validate(*req, &msg);
  if (st != MPC_OK) return st;
  const mpc_request_t& r = *req;
  const bool fp64 = r.precision == MPC_PRECISION_FP64_PLAIN;
  const int col = rate_column(r.sampling);
  auto pick = [&](int row) { return rates.at(row, fp64, col); };
  double units = double(r.n_paths) * double(r.n_steps), rate = 0.0, fixed_ms = 0.0;
  const char* confidence = rates.measured_here() ? "calibrated" : "measured";
  if (is_lsm(r.workload)) {
    rate = kLsmRate * rates.scale;
    fixed_ms = kLsmFixedMs * double(std::max<uint32_t>(r.n_steps, 2) - 1) / 49.0;
    if (r.workload == MPC_WORKLOAD_BERMUDAN_PUT) fixed_ms *= double(std::max<uint32_t>(r.n_exercise, 1)) / 49.0;
    confidence = "derived";
  } else if (r.workload == MPC_WORKLOAD_ASIAN_MLMC) {
    // the level budget bounds the work: explicit paths per level, else the solver's cap
    double updates = 0.0;
    uint64_t fine = r.base_steps;
    for (uint32_t l = 0; l < r.levels; ++l, fine *= std::max<uint32_t>(r.refinement_factor, 2))
      updates += double(r.paths_per_level[l]) * double(fine) * (l ? 1.5 : 1.0);
    if (r.target_stderr > 0.0) updates = double(r.max_step_updates);
    units = updates;
    rate = pick(ROW_ASIAN);
    fixed_ms = 2.0 * kCallOverheadMs * double(std::max<uint32_t>(r.levels, 1));
    confidence = "derived";
  } else if (r.workload == MPC_WORKLOAD_BASKET_CALL) {
    units = double(r.n_paths) * double(std::max<uint32_t>(r.n_steps, 1)) * double(std::max<uint32_t>(r.n_assets, 2)) / 2.0;
    rate = pick(ROW_BASKET2);
    if (r.n_assets > 2 || r.n_steps > 1) confidence = "derived";
  } else if (r.model == MPC_MODEL_HESTON) {
    rate = pick(ROW_HESTON);
  } else if (r.model == MPC_MODEL_MERTON) {
    if (r.method == MPC_METHOD_STEPWISE) {
      rate = pick(ROW_MERTON_STEP);
    } else {
      units = double(r.n_paths);
      rate = pick(ROW_MERTON_TERMINAL);
    }
  } else if (r.workload == MPC_WORKLOAD_EUROPEAN_CALL && r.method != MPC_METHOD_STEPWISE) {
    units = double(r.n_paths);
    rate = pick(ROW_GBM_TERMINAL);
    // the intercept is one full seek per thread that has a path: it reaches
    // its full size once every resident thread (2,048 per SM) has one
    fixed_ms = rates.fixed_at(ROW_GBM_TERMINAL, fp64, col) * std::min(1.0, units / (2048.0 * 148.0 * rates.scale));
  } else if (r.sampling == MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE) {
    rate = pick(ROW_BRIDGE);
  } else {
    rate = pick(r.workload == MPC_WORKLOAD_ARITHMETIC_ASIAN_CALL ? ROW_ASIAN : ROW_GBM_STEP);
  }
  if (r.technique == MPC_TECHNIQUE_ANTITHETIC) rate *= 1.6;  // one draw drives two paths
  uint64_t bytes = 0;
  mpc_estimate_bytes(req, &bytes);
  out->estimated_compile_ms = kFirstCallMs;
  out->estimated_runtime_ms = fixed_ms + units / rate * 1e3;
  out->estimated_total_ms = out->estimated_runtime_ms + kCallOverheadMs + out->estimated_compile_ms;
  out->estimated_peak_memory_mb = double(bytes) / (1024.0 * 1024.0);
  out->path_steps_per_sec = rate;
  out->path_steps = uint64_t(units);
  std::snprintf(out->confidence, sizeof(out->confidence), "%s", confidence);
  return MPC_OK;
}

// The request a calibration cell times: 1,048,576 paths x 64 steps (one
// step for the terminal rows), the standard technique.
mpc_request_t calibration_request(int row, bool fp64, int col) {
  mpc_request_t r;
  int workload = MPC_WORKLOAD_EUROPEAN_CALL;
  if (row == ROW_ASIAN) workload = MPC_WORKLOAD_ARITHMETIC_ASIAN_CALL;
  if (row == ROW_BASKET2) workload = MPC_WORKLOAD_BASKET_CALL;
  mpc_request_defaults(&r, workload);
  r.n_paths = 1u << 20;
  r.n_steps = 64;
  r.seed = 1;
  r.technique = MPC_TECHNIQUE_STANDARD;
  r.precision = fp64 ? MPC_PRECISION_FP64_PLAIN : MPC_PRECISION_FP32_PATH;
  r.sampling = row == ROW_BRIDGE ? MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE : kCalibrationSampling[col];
  switch (row) {
    case ROW_GBM_STEP:
    case ROW_BRIDGE:
      r.method = MPC_METHOD_STEPWISE;
      break;
    case ROW_GBM_TERMINAL:
      r.method = MPC_METHOD_TERMINAL;
      break;
    case ROW_HESTON:
      r.model = MPC_MODEL_HESTON;
      r.method = MPC_METHOD_STEPWISE;
      break;
    case ROW_MERTON_STEP:
      r.model = MPC_MODEL_MERTON;
      r.method = MPC_METHOD_STEPWISE;
      break;
    case ROW_MERTON_TERMINAL:
      r.model = MPC_MODEL_MERTON;
      r.method = MPC_METHOD_TERMINAL;
      break;
    case ROW_BASKET2:
      r.method = MPC_METHOD_TERMINAL;
      break;
    default:
      break;
  }
  return r;
}
}  // namespace

int mpc_estimate_cost(const mpc_request_t* req, int sm_count, mpc_cost_t* out) {
  const RateSource rates{nullptr, double(sm_count > 0 ? sm_count : 148) / 148.0};
  return estimate_cost_with(req, rates, out);
}

int mpc_estimate_cost_ctx(mpc_context_t* ctx, const mpc_request_t* req, mpc_cost_t* out) {
  if (!ctx) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  const RateSource rates{&ctx->cost_rates, double(ctx->sm_count) / 148.0, &ctx->cost_fixed};
  return estimate_cost_with(req, rates, out);
}

int mpc_calibrate_cost(mpc_context_t* ctx, double* seconds) {
  if (!ctx) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<double> rates(size_t(ROW_COUNT) * 2 * kCostColumns, 0.0);
  std::vector<double> fixed(rates.size(), 0.0);
  const RateSource builtin{nullptr, double(ctx->sm_count) / 148.0};
  for (int row = 0; row < ROW_COUNT; ++row) {
    for (int p = 0; p < 2; ++p) {
      for (int col = 0; col < kCostColumns; ++col) {
        double* cell = &rates[(size_t(row) * 2 + p) * kCostColumns + col];
        if (row == ROW_BRIDGE && col > 0) {  // one bridge rate per precision
          *cell = rates[(size_t(row) * 2 + p) * kCostColumns];
          continue;
        }
        const mpc_request_t r = calibration_request(row, p == 1, col);
        mpc_cost_t units;
        if (estimate_cost_with(&r, builtin, &units) != MPC_OK) continue;
        mpc_result_t res;
        // first call: tables and buffers of the shape; second: steady state.
        // A combination the backend does not run, or one past the context's
        // byte budget, keeps the built-in rate; a CUDA failure ends the
        // calibration with its status.
        int st = mpc_price(ctx, &r, &res);
        if (st == MPC_OK) st = mpc_price(ctx, &r, &res);
        if (st == MPC_E_CUDA || st == MPC_E_NO_DEVICE) return st;
        if (st != MPC_OK) continue;
        if (!(ctx->last_ms > 0.0)) continue;
        *cell = double(units.path_steps) / (ctx->last_ms * 1e-3);
        if (row == ROW_GBM_TERMINAL) {
          // terminal paths: a second size separates the intercept from the rate
          const double t1 = ctx->last_ms;
          mpc_request_t r4 = r;
          r4.n_paths = 4 * r.n_paths;
          st = mpc_price(ctx, &r4, &res);
          if (st == MPC_OK) st = mpc_price(ctx, &r4, &res);
          if (st == MPC_E_CUDA || st == MPC_E_NO_DEVICE) return st;
          if (st == MPC_OK && ctx->last_ms > t1) {
            const double per_path_ms = (ctx->last_ms - t1) / double(r4.n_paths - r.n_paths);
            *cell = 1.0 / (per_path_ms * 1e-3);  // paths per second
            fixed[(size_t(row) * 2 + p) * kCostColumns + col] = std::max(0.0, t1 - per_path_ms * double(r.n_paths));
          }
        }
      }
    }
  }
  ctx->cost_rates = rates;
  ctx->cost_fixed = fixed;
  ctx->last_error.clear();  // messages of the skipped combinations
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return MPC_OK;
}

int mpc_abi_version(void) { return MPC_ABI_VERSION; }

size_t mpc_struct_size(int which) {
  switch (which) {
    case 0:
      return sizeof(mpc_request_t);
    case 1:
      return sizeof(mpc_result_t);
    case 2:
      return sizeof(mpc_device_info_t);
    case 3:
      return sizeof(mpc_options_t);
    case 4:
      return sizeof(mpc_support_t);
    case 5:
      return sizeof(mpc_artifact_t);
    case 6:
      return sizeof(mpc_server_options_t);
    case 7:
      return sizeof(mpc_server_stats_t);
    case 8:
      return sizeof(mpc_greek_report_t);
    case 9:
      return sizeof(mpc_cost_t);
    default:
      return 0;
  }
}

const char* mpc_status_string(int status) {
  switch (status) {
    case MPC_OK:
      return "MPC_OK";
    case MPC_E_INVALID_CONFIG:
      return "MPC_E_INVALID_CONFIG";
    case MPC_E_UNSUPPORTED:
      return "MPC_E_UNSUPPORTED";
    case MPC_E_NO_DEVICE:
      return "MPC_E_NO_DEVICE";
    case MPC_E_OOM_BUDGET:
      return "MPC_E_OOM_BUDGET";
    case MPC_E_TIMEOUT:
      return "MPC_E_TIMEOUT";
    case MPC_E_CUDA:
      return "MPC_E_CUDA";
    case MPC_E_BUSY:
      return "MPC_E_BUSY";
    case MPC_E_NOT_FOUND:
      return "MPC_E_NOT_FOUND";
    case MPC_E_CANCELLED:
      return "MPC_E_CANCELLED";
    default:
      return "MPC_E_UNKNOWN";
  }
}

int mpc_device_count(int* count) {
  if (!count) return MPC_E_INVALID_CONFIG;
  int n = 0;
  cudaError_t err = cudaGetDeviceCount(&n);
  if (err != cudaSuccess) {
    *count = 0;
    return MPC_E_NO_DEVICE;
  }
  *count = n;
  return MPC_OK;
}

int mpc_device_info(int index, mpc_device_info_t* info) {
  if (!info) return MPC_E_INVALID_CONFIG;
  std::memset(info, 0, sizeof(*info));
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || index < 0 || index >= n) return MPC_E_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, index) != cudaSuccess) return MPC_E_NO_DEVICE;
  info->index = index;
  info->sm_count = prop.multiProcessorCount;
  info->cc_major = prop.major;
  info->cc_minor = prop.minor;
  info->total_memory_bytes = prop.totalGlobalMem;
  int clk = 0;
  cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, index);
  info->clock_khz = clk;
  info->l2_bytes = prop.l2CacheSize;
  int cur = 0;
  cudaGetDevice(&cur);
  size_t free_b = 0, total_b = 0;
  if (cudaSetDevice(index) == cudaSuccess && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
    info->free_memory_bytes = free_b;
  cudaSetDevice(cur);
  // the device name, cut to the ABI field (cudaDeviceProp holds up to 256 bytes)
  std::snprintf(info->name, sizeof(info->name), "%.*s", int(sizeof(info->name) - 1), prop.name);
  return MPC_OK;
}

// Rust `Default` impls of the configs (cpu.rs:1311-1815).
int mpc_request_defaults(mpc_request_t* r, int workload) {
  if (!r) return MPC_E_INVALID_CONFIG;
  std::memset(r, 0, sizeof(*r));
  r->workload = workload;
  r->model = MPC_MODEL_GBM;
  r->method = MPC_METHOD_AUTO;
  r->technique = MPC_TECHNIQUE_STANDARD;
  r->sampling = MPC_SAMPLING_PSEUDORANDOM;
  r->precision = MPC_PRECISION_FP32_PATH;
  r->n_paths = 100000;
  r->n_steps = 252;
  r->seed = 42;
  r->s0 = 100.0;
  r->k = 100.0;
  r->r = 0.03;
  r->sigma = 0.2;
  r->t = 1.0;
  r->v0 = 0.04;
  r->kappa = 1.5;
  r->theta = 0.04;
  r->vol_of_vol = 0.3;
  r->rho = -0.6;
  r->jump_intensity = 0.4;
  r->jump_mean = -0.08;
  r->jump_volatility = 0.25;
  r->n_assets = 2;
  r->spots[0] = 100.0;
  r->spots[1] = 95.0;
  r->sigmas[0] = 0.2;
  r->sigmas[1] = 0.25;
  r->weights[0] = 0.5;
  r->weights[1] = 0.5;
  r->corr[0] = 1.0;
  r->corr[1] = 0.35;
  r->corr[2] = 0.35;
  r->corr[3] = 1.0;
  r->basis_degree = 2;
  r->base_steps = 16;
  r->levels = 4;
  r->refinement_factor = 2;
  r->scramble_replicates = 1;
  r->paths_per_level[0] = 50000;
  r->paths_per_level[1] = 25000;
  r->paths_per_level[2] = 12500;
  r->paths_per_level[3] = 6250;
  r->pilot_paths_per_level = 2048;
  r->min_step_updates = 100000;
  r->max_step_updates = 10000000;
  switch (workload) {
    case MPC_WORKLOAD_DOWN_AND_OUT_CALL:
      r->barrier = 80.0;
      break;
    case MPC_WORKLOAD_UP_AND_OUT_CALL:
      r->barrier = 120.0;
      break;
    case MPC_WORKLOAD_AMERICAN_PUT:
      r->n_steps = 64;
      break;
    case MPC_WORKLOAD_BERMUDAN_PUT:
      r->n_steps = 64;
      r->n_exercise = 4;
      r->exercise_steps[0] = 16;
      r->exercise_steps[1] = 32;
      r->exercise_steps[2] = 48;
      r->exercise_steps[3] = 64;
      break;
    case MPC_WORKLOAD_BASKET_CALL:
      r->method = MPC_METHOD_TERMINAL;
      r->n_steps = 1;
      break;
    default:
      break;
  }
  if (workload < 0 || workload > MPC_WORKLOAD_ASIAN_MLMC) return MPC_E_INVALID_CONFIG;
  return MPC_OK;
}

int mpc_validate(const mpc_request_t* req, char* message, size_t message_len) {
  if (!req) return MPC_E_INVALID_CONFIG;
  std::string msg;
  int st = validate(*req, &msg);
  if (message && message_len) std::snprintf(message, message_len, "%s", msg.c_str());
  return st;
}

int mpc_supports(const mpc_request_t* req, mpc_support_t* out) {
  if (!req || !out) return MPC_E_INVALID_CONFIG;
  std::memset(out, 0, sizeof(*out));
  std::string msg;
  int st = validate(*req, &msg);
  out->supported = st == MPC_OK ? 1 : 0;
  out->reason = st;
  out->estimated_bytes = estimate_bytes(*req);
  std::snprintf(out->message, sizeof(out->message), "%s",
                st == MPC_OK ? "native CUDA execution on sm_100a" : msg.c_str());
  return MPC_OK;
}

int mpc_estimate_bytes(const mpc_request_t* req, uint64_t* bytes) {
  if (!req || !bytes) return MPC_E_INVALID_CONFIG;
  *bytes = estimate_bytes(*req);
  return MPC_OK;
}

int mpc_create(const mpc_options_t* options, mpc_context_t** out) {
  if (!out) return MPC_E_INVALID_CONFIG;
  *out = nullptr;
  // the kernels run 256-thread blocks
  if (options && options->default_block_size != 0 && options->default_block_size != 128 &&
      options->default_block_size != 256 && options->default_block_size != 512)
    return MPC_E_UNSUPPORTED;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return MPC_E_NO_DEVICE;
  mpc_context* ctx = new mpc_context();
  ctx->device = options ? options->device : 0;
  if (ctx->device < 0 || ctx->device >= n) {
    delete ctx;
    return MPC_E_NO_DEVICE;
  }
  ctx->budget = (options && options->hbm_budget_bytes) ? options->hbm_budget_bytes : (64ull << 30);
  if (options && options->default_block_size) ctx->tuner.default_block = options->default_block_size;
  auto bail = [&](cudaError_t e, const char* what) {
    std::fprintf(stderr, "montepath_cuda: %s failed: %s\n", what, cudaGetErrorString(e));
    delete ctx;
    return e == cudaErrorMemoryAllocation ? MPC_E_OOM_BUDGET : MPC_E_CUDA;
  };
  cudaError_t e;
  if ((e = cudaSetDevice(ctx->device)) != cudaSuccess) return bail(e, "cudaSetDevice");
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device);
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(e, "cudaStreamCreate");
  for (int i = 0; i < mpc_context::kSideStreams; ++i) {
    if ((e = cudaStreamCreateWithFlags(&ctx->side[i], cudaStreamNonBlocking)) != cudaSuccess)
      return bail(e, "cudaStreamCreate");
    cudaEventCreateWithFlags(&ctx->ev_join[i], cudaEventDisableTiming);
  }
  cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
  cudaEventCreate(&ctx->ev_start);
  cudaEventCreate(&ctx->ev_stop);
  std::vector<uint32_t> sob;
  std::vector<uint64_t> jump;
  build_tables(sob, jump);
  if ((e = cudaMalloc(&ctx->d_sobol, sob.size() * 4)) != cudaSuccess) return bail(e, "cudaMalloc tables");
  if ((e = cudaMalloc(&ctx->d_jump, jump.size() * 8)) != cudaSuccess) return bail(e, "cudaMalloc tables");
  cudaMemcpy(ctx->d_sobol, sob.data(), sob.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(ctx->d_jump, jump.data(), jump.size() * 8, cudaMemcpyHostToDevice);
  ctx->live_bytes = sob.size() * 4 + jump.size() * 8;
  ctx->tabs.sobol = static_cast<const uint32_t*>(ctx->d_sobol);
  ctx->tabs.jump = static_cast<const uint64_t*>(ctx->d_jump);
  *out = ctx;
  return MPC_OK;
}

int mpc_destroy(mpc_context_t* ctx) {
  if (!ctx) return MPC_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  for (auto& kv : ctx->bufs)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  if (ctx->d_sobol) cudaFree(ctx->d_sobol);
  if (ctx->d_jump) cudaFree(ctx->d_jump);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  for (int i = 0; i < mpc_context::kSideStreams; ++i) {
    if (ctx->side[i]) {
      cudaStreamSynchronize(ctx->side[i]);
      cudaStreamDestroy(ctx->side[i]);
    }
    if (ctx->ev_join[i]) cudaEventDestroy(ctx->ev_join[i]);
  }
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return MPC_OK;
}

const char* mpc_last_error_message(const mpc_context_t* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

namespace mpc {
// Measures the fused launch of a request's kind (family, sampler, step
// bucket) at 128, 256 and 512 threads per block, on the request itself (its
// first 4,194,304 units at most: a probe much shorter than the request
// misjudges the tail of the launch), and keeps the fastest for the kind; 256
// is kept unless another size is more than 1% faster (the best of three
// timed runs each), so the choice does not flip on timing noise.  Once per
// kind and context.
static int tune_block(mpc_context* ctx, const Prepared& p0) {
  const uint64_t key = block_key(p0);
  {
    std::lock_guard<std::mutex> lock(ctx->tuner.mu);
    if (ctx->tuner.block.count(key)) return MPC_OK;
  }
  const uint32_t cands[3] = {128, 256, 512};
  double ms[3];
  for (int c = 0; c < 3; ++c) {
    ms[c] = 1e300;
    const int occ = fused_max_blocks_per_sm(p0.family, p0.sampler, int(cands[c]));
    if (occ < 1) continue;
    Prepared p = p0;
    p.block_hint = cands[c];
    const uint64_t probe = std::min<uint64_t>(p.q.n_units, 1ull << 22);
    p.q.n_units = probe;
    p.q.n_paths = p.q.anti ? std::min<uint64_t>(p0.q.n_paths, 2 * probe) : probe;
    for (int rep = 0; rep < 4; ++rep) {
      std::vector<Prepared*> one{&p};
      mpc_result_t r;
      std::vector<mpc_result_t*> outs{&r};
      const int st = run_fused(ctx, one, outs, nullptr, 0);
      if (st != MPC_OK) return st;
      if (rep > 0) ms[c] = std::min(ms[c], ctx->last_ms);  // the first run warms up
    }
  }
  int best = 1;
  for (int c = 0; c < 3; ++c)
    if (ms[c] < ms[best]) best = c;
  if (ms[1] <= 1.01 * ms[best]) best = 1;
  std::lock_guard<std::mutex> lock(ctx->tuner.mu);
  ctx->tuner.block[key] = cands[best];
  ctx->tuner.measured++;
  return MPC_OK;
}
}  // namespace mpc

int mpc_prepare(mpc_context_t* ctx, const mpc_request_t* req, mpc_artifact_t* out) {
  if (!ctx || !req || !out) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  std::memset(out, 0, sizeof(*out));
  std::string msg;
  if (req->workload == MPC_WORKLOAD_ASIAN_MLMC || is_lsm(req->workload)) {
    int st = validate(*req, &msg);
    if (st != MPC_OK) return fail(ctx, st, msg);
    out->kernel_family = is_lsm(req->workload) ? 100 : FAM_MLMC_LEVEL;
    out->block_size = 256;
    out->paths_per_thread = 1;
    out->bytes = estimate_bytes(*req);
    std::snprintf(out->name, sizeof(out->name), "%s", is_lsm(req->workload) ? "lsm_cooperative" : "mlmc_levels");
    return MPC_OK;
  }
  Prepared p;
  int st = prepare(ctx, *req, &p, &msg);
  if (st != MPC_OK) return fail(ctx, st, msg);
  if (!p.plain && !p.block_hint && !merton_stream_request(*req)) {  // the autotuner measures the request's kind
    st = tune_block(ctx, p);
    if (st != MPC_OK) return st;
  }
  Shape s = choose_shape(ctx, p);
  out->kernel_family = p.family;
  out->block_size = s.block;
  out->paths_per_thread = s.ppt;
  out->tiles = uint32_t((p.q.n_units + s.block * s.ppt - 1) / (s.block * s.ppt));
  out->bytes = estimate_bytes(*req);
  std::snprintf(out->name, sizeof(out->name), "%s_family%d_sampler%d", p.plain ? "plain_fp64" : "fused_fp32",
                p.family, p.sampler);
  return MPC_OK;
}

int mpc_price(mpc_context_t* ctx, const mpc_request_t* req, mpc_result_t* out) {
  if (!ctx || !req || !out) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  return price_one(ctx, req, out, nullptr, 0);
}

int mpc_price_paths(mpc_context_t* ctx, const mpc_request_t* req, double* host_payoffs, uint64_t capacity) {
  if (!ctx || !req || !host_payoffs) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  if (req->workload == MPC_WORKLOAD_ASIAN_MLMC || is_lsm(req->workload))
    return fail(ctx, MPC_E_UNSUPPORTED, "per-path payoffs are available for path-payoff workloads");
  mpc_result_t tmp;
  return price_one(ctx, req, &tmp, host_payoffs, capacity);
}

int mpc_price_batch(mpc_context_t* ctx, const mpc_request_t* reqs, size_t n, mpc_result_t* out) {
  if (!ctx || (!reqs && n) || (!out && n)) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  std::vector<Prepared> preps(n);
  std::vector<Prepared*> fused;
  std::vector<mpc_result_t*> fused_out;
  std::vector<const mpc_request_t*> lsm, mlmc;
  std::vector<mpc_result_t*> lsm_out, mlmc_out;
  int first_error = MPC_OK;
  double total_ms = 0.0;
  uint64_t launches_before = kernel_launch_count();
  for (size_t i = 0; i < n; ++i) {
    std::memset(&out[i], 0, sizeof(out[i]));
    std::string msg;
    int st = validate(reqs[i], &msg);
    if (st == MPC_OK && reqs[i].workload != MPC_WORKLOAD_ASIAN_MLMC && !is_lsm(reqs[i].workload)) {
      st = prepare(ctx, reqs[i], &preps[i], &msg);
      if (st == MPC_OK && !preps[i].plain && !merton_stream_request(reqs[i])) {
        fused.push_back(&preps[i]);
        fused_out.push_back(&out[i]);
        continue;
      }
    }
    if (st != MPC_OK) {
      out[i].status = st;
      if (first_error == MPC_OK) {
        first_error = st;
        ctx->last_error = msg;
      }
      continue;
    }
    if (is_lsm(reqs[i].workload)) {
      lsm.push_back(&reqs[i]);
      lsm_out.push_back(&out[i]);
      continue;
    }
    if (reqs[i].workload == MPC_WORKLOAD_ASIAN_MLMC) {
      mlmc.push_back(&reqs[i]);
      mlmc_out.push_back(&out[i]);
      continue;
    }
    // FP64-plain requests and the pseudorandom Merton replay run one launch sequence each
    st = price_one(ctx, &reqs[i], &out[i], nullptr, 0);
    total_ms += ctx->last_ms;
    if (st != MPC_OK && first_error == MPC_OK) first_error = st;
  }
  if (!lsm.empty()) {  // packed into shared cooperative launches
    int st = run_lsm_batch(ctx, lsm, lsm_out);
    total_ms += ctx->last_ms;
    if (st != MPC_OK) {
      for (mpc_result_t* o : lsm_out) o->status = st;
      if (first_error == MPC_OK) first_error = st;
    }
  }
  if (!mlmc.empty()) {  // all pilot levels in one launch, all main levels in another
    int st = run_mlmc_batch(ctx, mlmc, mlmc_out);
    total_ms += ctx->last_ms;
    if (st != MPC_OK) {
      for (mpc_result_t* o : mlmc_out) o->status = st;
      if (first_error == MPC_OK) first_error = st;
    }
  }
  if (!fused.empty()) {
    int st = run_fused(ctx, fused, fused_out, nullptr, 0);
    total_ms += ctx->last_ms;
    for (mpc_result_t* o : fused_out) o->status = st;
    if (st != MPC_OK && first_error == MPC_OK) first_error = st;
  }
  ctx->last_ms = total_ms;
  ctx->last_launches = kernel_launch_count() - launches_before;
  return first_error;
}

int mpc_generate_normals(mpc_context_t* ctx, int sampling, uint64_t seed, uint64_t n_points, uint32_t dimensions,
                         int precision, void* host_out) {
  if (!ctx || !host_out || n_points == 0 || dimensions == 0) return MPC_E_INVALID_CONFIG;
  if (sampling == MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE)
    return fail(ctx, MPC_E_UNSUPPORTED, "bridge ordering applies to paths, not raw normals");
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  Prepared p;
  DevReq& q = p.q;
  std::memset(&q, 0, sizeof(q));
  p.sampler = sampler_of(sampling);
  q.seed = seed;
  q.seed32 = uint32_t(seed);
  q.n_paths = n_points;
  q.n_units = n_points;
  q.n_chunks = 1;
  q.normals_per_unit = dimensions;  // the reference generator is one stream over point-major normals
  build_sampler_tables(&p, seed, n_points, dimensions);
  std::vector<Prepared*> one{&p};
  int st = upload_aux(ctx, one);
  if (st != MPC_OK) return st;
  const size_t elem = precision == MPC_PRECISION_FP32_PATH ? 4 : 8;
  void* d_out = nullptr;
  if ((st = scratch(ctx, "gen_out", n_points * dimensions * elem, &d_out))) return st;
  cudaError_t e = launch_generate_normals(q, p.sampler, precision == MPC_PRECISION_FP32_PATH, d_out, n_points,
                                          dimensions, ctx->tabs, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "generate normals");
  MPC_CUDA(ctx, cudaMemcpyAsync(host_out, d_out, n_points * dimensions * elem, cudaMemcpyDeviceToHost, ctx->stream));
  MPC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return MPC_OK;
}

int mpc_counter_hash_u32(mpc_context_t* ctx, uint32_t seed, uint32_t n_paths, uint32_t n_steps, uint32_t* host_out) {
  if (!ctx || !host_out) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  size_t bytes = size_t(n_paths) * n_steps * 2 * 4;
  void* d = nullptr;
  int st = scratch(ctx, "gen_out", bytes, &d);
  if (st != MPC_OK) return st;
  cudaError_t e = launch_counter_hash(seed, n_paths, n_steps, static_cast<uint32_t*>(d), ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "counter hash");
  MPC_CUDA(ctx, cudaMemcpyAsync(host_out, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  MPC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return MPC_OK;
}

int mpc_xorshift_u64(mpc_context_t* ctx, uint64_t seed, uint64_t offset, uint64_t count, uint64_t* host_out) {
  if (!ctx || !host_out) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  void* d = nullptr;
  int st = scratch(ctx, "gen_out", count * 8, &d);
  if (st != MPC_OK) return st;
  cudaError_t e = launch_xorshift(seed, offset, count, static_cast<uint64_t*>(d), ctx->tabs, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "xorshift stream");
  MPC_CUDA(ctx, cudaMemcpyAsync(host_out, d, count * 8, cudaMemcpyDeviceToHost, ctx->stream));
  MPC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return MPC_OK;
}

int mpc_european_call_stepwise_v1(const double* normals, double* payoffs, int32_t n_paths, int32_t n_steps,
                                  double log_s0, double strike, double drift_dt, double vol_dt, double discount,
                                  void* stream) {
  if (n_paths < 0 || n_steps < 0 || (n_paths > 0 && (!normals || !payoffs))) return MPC_E_INVALID_CONFIG;
  cudaError_t e = launch_european_call_stepwise_v1(normals, payoffs, n_paths, n_steps, log_s0, strike, drift_dt,
                                                   vol_dt, discount, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? MPC_OK : MPC_E_CUDA;
}

int mpc_flush_l2(mpc_context_t* ctx) {
  if (!ctx) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  void* d = nullptr;
  const size_t bytes = 256ull << 20;  // twice the 126 MB L2
  int st = scratch(ctx, "flush", bytes, &d);
  if (st != MPC_OK) return st;
  cudaError_t e = launch_flush(d, bytes, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "flush");
  MPC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return MPC_OK;
}

int mpc_last_timing(const mpc_context_t* ctx, double* device_ms, uint64_t* kernel_launches) {
  if (!ctx) return MPC_E_INVALID_CONFIG;
  if (device_ms) *device_ms = ctx->last_ms;
  if (kernel_launches) *kernel_launches = ctx->last_launches;
  return MPC_OK;
}

int mpc_last_transfer(const mpc_context_t* ctx, uint64_t* h2d_bytes, uint64_t* d2h_bytes) {
  if (!ctx) return MPC_E_INVALID_CONFIG;
  if (h2d_bytes) *h2d_bytes = ctx->last_h2d;
  if (d2h_bytes) *d2h_bytes = ctx->last_d2h;
  return MPC_OK;
}

}  // extern "C"

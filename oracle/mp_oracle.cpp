// mp_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// FP64 CPU restatement of montepath's Monte Carlo pricing hot path
// (crates/mc-core/src/runtime/cpu.rs of the reference).  It is the checker
// the CUDA backend is compared against and the timed CPU baseline of
// bench.py; nothing in the product links it.  Every function cites the
// reference lines it follows.  Where the B200 backend extends the reference
// (Heston/Merton with structured samplers, stepwise Merton, up-and-out
// barriers, d-asset baskets, LSM with other samplers) the extension is built
// so that it reduces to the reference semantics in a checkable limit.
//
// Pinning: the analytic functions are checked against the reference's
// fixture registry (benchmarks/reference-fixtures.json); the integer
// generators against independent restatements and known answers; the
// unscrambled Sobol core against SciPy.  The scrambled Sobol generator
// restates the published algorithm of the `sobol_burley = "0.5"` crate
// (Burley 2020, "Practical Hash-based Owen Scrambling", JCGT 9(4)); the crate
// is not vendored, so bit parity with it is unpinned.
//
// Build: oracle/Makefile (gcc, -ffp-contract=off so that a*b+c rounds twice,
// as Rust does).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <thread>
#include <vector>

#include "../include/montepath_cuda.h"
#include "../montepath_b200/csrc/sobol_directions.h"

namespace orc {

static const double kPi = 3.14159265358979323846;
static const double kMinPositive = 2.2250738585072014e-308;  // f64::MIN_POSITIVE
static const double kEps = 2.220446049250313e-16;            // f64::EPSILON

// ---------------------------------------------------------------- RNGs ----

// MonteCarloRng: xorshift64* with a cached Box-Muller normal (cpu.rs:2955-3007).
struct McRng {
  uint64_t state;
  bool has_cached = false;
  double cached = 0.0;
  explicit McRng(uint64_t seed) : state(seed == 0 ? 0x9E3779B97F4A7C15ull : seed) {}
  uint64_t next_u64() {  // cpu.rs:2975-2983
    uint64_t x = state;
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    state = x;
    return x * 0x2545F4914F6CDD1Dull;
  }
  double next_f64_open01() {  // cpu.rs:2985-2990
    uint64_t raw = next_u64() >> 11;
    double value = double(raw) * (1.0 / double(1ull << 53));
    return std::max(value, kMinPositive);
  }
  double standard_normal() {  // cpu.rs:2992-3006
    if (has_cached) {
      has_cached = false;
      return cached;
    }
    double u1 = next_f64_open01();
    double u2 = next_f64_open01();
    double radius = std::sqrt(-2.0 * std::log(u1));
    double theta = 2.0 * kPi * u2;
    double z0 = radius * std::cos(theta);
    double z1 = radius * std::sin(theta);
    cached = z1;
    has_cached = true;
    return z0;
  }
};

// splitmix64 / derive_chunk_seed (cpu.rs:8922-8932).
uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  uint64_t z = x;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
uint64_t derive_chunk_seed(uint64_t base, uint64_t idx) {
  return splitmix64(base + idx * 0x9E3779B97F4A7C15ull);
}
// open01_from_u64 (cpu.rs:6104-6107)
double open01_from_u64(uint64_t v) {
  uint64_t top = v >> 11;
  return std::max(double(top) * (1.0 / double(1ull << 53)), kMinPositive);
}

// Counter-hash normals of the Metal kernel (cpu.rs:5626-5652).
uint32_t hash_u32(uint32_t x) {
  x += 0x9E3779B9u;
  x ^= x >> 16;
  x *= 0x85EBCA6Bu;
  x ^= x >> 13;
  x *= 0xC2B2AE35u;
  return x ^ (x >> 16);
}
uint32_t counter_mix(uint32_t seed, uint32_t path, uint32_t step, uint32_t lane) {
  return seed ^ (path * 747796405u) ^ (step * 2891336453u) ^ (lane * 277803737u);
}
float stateless_open01_f32(uint32_t seed, uint32_t path, uint32_t step, uint32_t lane) {
  uint32_t h = hash_u32(counter_mix(seed, path, step, lane));
  double v = (double(h) + 1.0) / 4294967297.0;
  return float(std::max(v, double(std::numeric_limits<float>::min())));
}
float stateless_standard_normal_f32(uint32_t seed, uint32_t path, uint32_t step) {
  float u1 = stateless_open01_f32(seed, path, step, 0);
  float u2 = stateless_open01_f32(seed, path, step, 1);
  float radius = std::sqrt(-2.0f * std::log(u1));
  float theta = 2.0f * float(kPi) * u2;
  return radius * std::cos(theta);
}

// Acklam rational inverse normal CDF (cpu.rs:6012-6061).
double inverse_standard_normal(double p) {
  static const double A[6] = {-3.969683028665376e1, 2.209460984245205e2, -2.759285104469687e2,
                              1.38357751867269e2,   -3.066479806614716e1, 2.506628277459239};
  static const double B[5] = {-5.447609879822406e1, 1.615858368580409e2, -1.556989798598866e2,
                              6.680131188771972e1, -1.328068155288572e1};
  static const double C[6] = {-7.784894002430293e-3, -3.223964580411365e-1, -2.400758277161838,
                              -2.549732539343734,   4.374664141464968,    2.938163982698783};
  static const double D[4] = {7.784695709041462e-3, 3.224671290700398e-1, 2.445134137142996,
                              3.754408661907416};
  const double p_low = 0.02425, p_high = 1.0 - p_low;
  p = std::min(std::max(p, kMinPositive), 1.0 - kEps);
  if (p < p_low) {
    double q = std::sqrt(-2.0 * std::log(p));
    return (((((C[0] * q + C[1]) * q + C[2]) * q + C[3]) * q + C[4]) * q + C[5]) /
           ((((D[0] * q + D[1]) * q + D[2]) * q + D[3]) * q + 1.0);
  }
  if (p <= p_high) {
    double q = p - 0.5;
    double r = q * q;
    return (((((A[0] * r + A[1]) * r + A[2]) * r + A[3]) * r + A[4]) * r + A[5]) * q /
           (((((B[0] * r + B[1]) * r + B[2]) * r + B[3]) * r + B[4]) * r + 1.0);
  }
  double q = std::sqrt(-2.0 * std::log(1.0 - p));
  return -(((((C[0] * q + C[1]) * q + C[2]) * q + C[3]) * q + C[4]) * q + C[5]) /
         ((((D[0] * q + D[1]) * q + D[2]) * q + D[3]) * q + 1.0);
}

// ------------------------------------------------------------- Halton -----
// halton / halton_with_shift / first_n_primes (cpu.rs:6063-6102).
double halton(uint64_t index, uint32_t base) {
  double f = 1.0 / double(base);
  double value = 0.0;
  while (index > 0) {
    value += f * double(index % base);
    index /= base;
    f /= double(base);
  }
  return std::max(value, kMinPositive);
}
double halton_with_shift(uint64_t index, uint32_t base, double shift) {
  double shifted = halton(index, base) + shift;
  return shifted - std::floor(shifted);
}
std::vector<uint32_t> first_n_primes(size_t n) {
  std::vector<uint32_t> primes;
  uint32_t candidate = 2;
  while (primes.size() < n) {
    uint32_t limit = uint32_t(std::sqrt(double(candidate)));
    bool prime = true;
    for (uint32_t p : primes) {
      if (p > limit) break;
      if (candidate % p == 0) {
        prime = false;
        break;
      }
    }
    if (prime) primes.push_back(candidate);
    ++candidate;
  }
  return primes;
}

// -------------------------------------------------------------- Sobol -----
// Restatement of Burley 2020 hash-based Owen scrambling, the algorithm of
// the `sobol_burley` crate the reference calls at cpu.rs:5399-5431.
uint32_t reverse_bits32(uint32_t x) {
  x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
  x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
  x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
  x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
  return (x >> 16) | (x << 16);
}
uint32_t lk_permute(uint32_t x, uint32_t seed) {
  x += seed;
  x ^= x * 0x6c50b47cu;
  x ^= x * 0xb82f1e52u;
  x ^= x * 0xc7afe638u;
  x ^= x * 0x8d22f6e6u;
  return x;
}
uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) {
  return reverse_bits32(lk_permute(reverse_bits32(x), seed));
}
uint32_t hash_combine(uint32_t seed, uint32_t v) {
  return seed ^ (v + 0x9e3779b9u + (seed << 6) + (seed >> 2));
}
uint32_t sobol_u32(uint32_t index, uint32_t dim) {
  uint32_t x = 0;
  for (int b = 0; b < 32; ++b)
    if ((index >> b) & 1u) x ^= kSobolDirections[dim][b];
  return x;
}
uint32_t sobol_owen_u32(uint32_t index, uint32_t dim, uint32_t seed) {
  uint32_t shuffled = nested_uniform_scramble(index, seed);
  uint32_t x = sobol_u32(shuffled, dim);
  return nested_uniform_scramble(x, hash_combine(seed, dim));
}
// 23-bit midpoint uniform in (0,1): exact in f32 and f64, never 0 or 1.
double sobol_unit(uint32_t x) { return (double(x >> 9) + 0.5) * (1.0 / 8388608.0); }

// ScrambledSobol::standard_normal point/dimension split (cpu.rs:5654-5684):
// points in blocks of 2^16 with a per-block seed, dimensions wrapped every
// MPC_SOBOL_DIMS with a seed offset.
const uint32_t kSobolBlock = 1u << 16;
uint32_t sobol_point_u32(uint64_t point, uint64_t normal_index, uint32_t seed32) {
  uint64_t block = point / kSobolBlock;
  uint32_t local = uint32_t(point % kSobolBlock);
  uint32_t dim = uint32_t(normal_index % MPC_SOBOL_DIMS);
  uint32_t seed = seed32 + uint32_t(normal_index / MPC_SOBOL_DIMS) + uint32_t(block) * 0x9E3779B9u;
  return sobol_owen_u32(local, dim, seed);
}

// ------------------------------------------------------------ Samplers ----
// StructuredNormalSampler (cpu.rs:5790-5836): randomized Halton, Latin
// hypercube and scrambled Sobol, per (point, dimension).
struct Sampler {
  int kind = MPC_SAMPLING_PSEUDORANDOM;
  uint32_t seed32 = 0;
  uint64_t n_paths = 0;
  std::vector<uint32_t> primes;
  std::vector<double> shifts;
  struct Lhs {
    uint64_t multiplier, offset, jitter_seed;
  };
  std::vector<Lhs> lhs;

  static uint64_t gcd(uint64_t a, uint64_t b) {
    while (b) {
      uint64_t t = a % b;
      a = b;
      b = t;
    }
    return a;
  }
  // coprime_multiplier (cpu.rs:5983-6002)
  static uint64_t coprime_multiplier(uint64_t seed, uint64_t modulus) {
    if (modulus <= 1) return 1;
    uint64_t c = std::max<uint64_t>(seed % modulus, 1);
    if (c % 2 == 0) c += 1;
    while (gcd(c, modulus) != 1) {
      c += 2;
      if (c >= modulus) c = 1;
    }
    return c;
  }

  Sampler(int method, uint64_t seed, uint64_t n_paths_, size_t dims) : kind(method), n_paths(n_paths_) {
    seed32 = uint32_t(seed);
    if (method == MPC_SAMPLING_RANDOMIZED_HALTON) {  // RandomizedHalton::new, cpu.rs:5692-5704
      size_t count = std::max<size_t>(dims, 2);
      primes = first_n_primes(count);
      for (size_t d = 0; d < count; ++d)
        shifts.push_back(open01_from_u64(splitmix64(seed + uint64_t(d) * 0x9E3779B97F4A7C15ull)));
    } else if (method == MPC_SAMPLING_LATIN_HYPERCUBE) {  // LatinHypercube::new, cpu.rs:5737-5761
      size_t count = std::max<size_t>(dims, 1);
      for (size_t d = 0; d < count; ++d) {
        uint64_t mixed =
            splitmix64(seed ^ (uint64_t(d) * 0x9E3779B97F4A7C15ull) ^ 0xD1B54A32D192ED03ull);
        Lhs p;
        p.multiplier = coprime_multiplier(mixed, std::max<uint64_t>(n_paths, 1));
        p.offset = n_paths == 0 ? 0 : splitmix64(mixed ^ 0xA24BAED4963EE407ull) % n_paths;
        p.jitter_seed = splitmix64(mixed ^ 0x9FB21C651E98DF25ull);
        lhs.push_back(p);
      }
    }
  }
  double uniform(uint64_t point, uint64_t dim) const {
    switch (kind) {
      case MPC_SAMPLING_RANDOMIZED_HALTON:  // cpu.rs:5706-5712
        return halton_with_shift(point + 1, primes[dim], shifts[dim]);
      case MPC_SAMPLING_LATIN_HYPERCUBE: {  // cpu.rs:5764-5780
        const Lhs& p = lhs[dim];
        uint64_t stratum = n_paths == 0 ? 0 : (p.multiplier * point + p.offset) % n_paths;
        double jitter = open01_from_u64(splitmix64(p.jitter_seed ^ (point * 0xBF58476D1CE4E5B9ull)));
        double u = (double(stratum) + jitter) / double(n_paths);
        return std::min(std::max(u, kMinPositive), 1.0 - kEps);
      }
      default:
        return sobol_unit(sobol_point_u32(point, dim, seed32));
    }
  }
  double normal(uint64_t point, uint64_t dim) const { return inverse_standard_normal(uniform(point, dim)); }
};

// BrownianBridgePlan (cpu.rs:5886-5981).
struct BridgePlan {
  struct Op {
    size_t left, mid, right;
    double lw, rw, sd;
    size_t normal_index;
  };
  size_t n_steps;
  double maturity_sqrt, inv_sqrt_dt;
  std::vector<Op> ops;
  BridgePlan(size_t n, double maturity) : n_steps(n) {
    double dt = maturity / double(n);
    std::vector<std::pair<size_t, size_t>> stack{{0, n}};
    size_t normal_index = 1;
    while (!stack.empty()) {
      auto [l, r] = stack.back();
      stack.pop_back();
      if (r <= l + 1) continue;
      size_t mid = (l + r) / 2;
      double tl = double(l) * dt, tm = double(mid) * dt, tr = double(r) * dt;
      double denom = tr - tl;
      ops.push_back({l, mid, r, (tr - tm) / denom, (tm - tl) / denom,
                     std::sqrt((tm - tl) * (tr - tm) / denom), normal_index});
      ++normal_index;
      stack.push_back({mid, r});
      stack.push_back({l, mid});
    }
    maturity_sqrt = std::sqrt(maturity);
    inv_sqrt_dt = 1.0 / std::sqrt(dt);
  }
  void increments(const std::vector<double>& in, std::vector<double>& out) const {
    std::vector<double> w(n_steps + 1, 0.0);
    w[n_steps] = maturity_sqrt * in[0];
    for (const Op& op : ops) w[op.mid] = op.lw * w[op.left] + op.rw * w[op.right] + op.sd * in[op.normal_index];
    out.resize(n_steps);
    for (size_t s = 1; s <= n_steps; ++s) out[s - 1] = (w[s] - w[s - 1]) * inv_sqrt_dt;
  }
};

// ---------------------------------------------------------- Estimators ----
// ControlVariateMoments (cpu.rs:6202-6230) doubling as the plain (sum, sq_sum) pair.
struct Moments {
  uint64_t n = 0;
  double s = 0, s2 = 0, c = 0, c2 = 0, pc = 0;
  void add(double p) {
    ++n;
    s += p;
    s2 += p * p;
  }
  void add_cv(double p, double ctl) {
    ++n;
    s += p;
    s2 += p * p;
    c += ctl;
    c2 += ctl * ctl;
    pc += p * ctl;
  }
  void merge(const Moments& o) {
    n += o.n;
    s += o.s;
    s2 += o.s2;
    c += o.c;
    c2 += o.c2;
    pc += o.pc;
  }
};
// summarize_payoffs / summarize_block_estimates (cpu.rs:7641-7665).
void summarize(uint64_t count, double sum, double sq, double* price, double* stderr_) {
  double n = double(count);
  double mean = sum / n;
  double var = (sq / n) - mean * mean;
  *price = mean;
  *stderr_ = std::sqrt(std::max(var, 0.0)) / std::sqrt(n);
}
// summarize_control_variate (cpu.rs:7738-7771).
void summarize_cv(const Moments& m, double expectation, double* price, double* stderr_) {
  double n = double(m.n);
  double pm = m.s / n, cm = m.c / n;
  double cvar = (m.c2 / n) - cm * cm;
  if (cvar <= kEps) {
    summarize(m.n, m.s, m.s2, price, stderr_);
    return;
  }
  double cov = (m.pc / n) - pm * cm;
  double beta = cov / cvar;
  double adj = pm - beta * (cm - expectation);
  double adj_sq = (m.s2 / n) - (2.0 * beta) * ((m.pc / n) - expectation * pm) +
                  (beta * beta) * ((m.c2 / n) - (2.0 * expectation * cm) + (expectation * expectation));
  double var = std::max(adj_sq - adj * adj, 0.0);
  *price = adj;
  *stderr_ = std::sqrt(var) / std::sqrt(n);
}

// Runs `fn(seed, first_unit, units, out)` either as one stream or split into
// the reference's deterministic chunks (cpu.rs:6232-6276: derive_chunk_seed
// per chunk, base + (idx < remainder) units, merged in spawn order).
Moments run_chunked(const mpc_request_t& r, uint64_t units, bool chunkable,
                    const std::function<Moments(uint64_t, uint64_t, uint64_t)>& fn) {
  uint64_t threads = r.n_threads <= 1 ? 1 : r.n_threads;
  if (!chunkable || threads <= 1 || units < threads * 2000) return fn(r.seed, 0, units);
  std::vector<Moments> parts(threads);
  std::vector<std::thread> pool;
  uint64_t base = units / threads, rem = units % threads, first = 0;
  for (uint64_t idx = 0; idx < threads; ++idx) {
    uint64_t count = base + (idx < rem ? 1 : 0);
    uint64_t seed = derive_chunk_seed(r.seed, idx);
    pool.emplace_back([&parts, &fn, idx, seed, first, count] { parts[idx] = fn(seed, first, count); });
    first += count;
  }
  Moments total;
  for (uint64_t idx = 0; idx < threads; ++idx) {
    pool[idx].join();
    total.merge(parts[idx]);
  }
  return total;
}

// ------------------------------------------------------- GBM payoffs -------
// Path observers for the GBM payoff family: European (cpu.rs:6443-6507),
// arithmetic Asian (cpu.rs:6561-6591), down-and-out (cpu.rs:7973-8009),
// up-and-out (mirror, extension), fixed-strike lookback (cpu.rs:8324-8354).
struct GbmObs {
  int workload;
  double k, barrier, s0;
  double log_s, sum = 0.0, max_s;
  bool knocked;
  size_t steps = 0;
  GbmObs(int w, double k_, double b, double s0_)
      : workload(w), k(k_), barrier(b), s0(s0_), log_s(std::log(s0_)), max_s(s0_) {
    knocked = (w == MPC_WORKLOAD_DOWN_AND_OUT_CALL && s0 <= b) || (w == MPC_WORKLOAD_UP_AND_OUT_CALL && s0 >= b);
  }
  void step(double increment) {
    log_s += increment;
    ++steps;
    switch (workload) {
      case MPC_WORKLOAD_ARITHMETIC_ASIAN_CALL:
        sum += std::exp(log_s);
        break;
      case MPC_WORKLOAD_DOWN_AND_OUT_CALL:
        if (std::exp(log_s) <= barrier) knocked = true;
        break;
      case MPC_WORKLOAD_UP_AND_OUT_CALL:
        if (std::exp(log_s) >= barrier) knocked = true;
        break;
      case MPC_WORKLOAD_LOOKBACK_CALL:
        max_s = std::max(max_s, std::exp(log_s));
        break;
      default:
        break;
    }
  }
  double payoff(double discount) const {
    switch (workload) {
      case MPC_WORKLOAD_ARITHMETIC_ASIAN_CALL:
        return std::max(sum / double(steps) - k, 0.0) * discount;
      case MPC_WORKLOAD_DOWN_AND_OUT_CALL:
      case MPC_WORKLOAD_UP_AND_OUT_CALL:
        return knocked ? 0.0 : std::max(std::exp(log_s) - k, 0.0) * discount;
      case MPC_WORKLOAD_LOOKBACK_CALL:
        return std::max(max_s - k, 0.0) * discount;
      default:
        return std::max(std::exp(log_s) - k, 0.0) * discount;
    }
  }
  double control(double discount) const { return discount * std::exp(log_s); }
};

struct Out {  // optional per-unit output (per path, or per antithetic pair)
  double* values = nullptr;
  uint64_t capacity = 0;
  // Point window for the threaded timing harness: structured and counter-hash
  // loops simulate points [point0, point0 + point_count) (0 = all).
  uint64_t point0 = 0, point_count = 0;
  void put(uint64_t i, double v) const {
    if (values && i - point0 < capacity) values[i - point0] = v;
  }
  uint64_t last(uint64_t units) const { return point_count ? point0 + point_count : units; }
};

// f64::powi: repeated squaring as in compiler-rt's __powidf2.
double powi(double a, int b) {
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

// GBM stepwise, all payoffs, all techniques and samplers: the
// simulate_*_stepwise_* family (cpu.rs:6443-6591, 7113-7501, 7885-8630).
void price_gbm_stepwise(const mpc_request_t& r, mpc_result_t* res, const Out& out) {
  const uint64_t n = r.n_paths, steps = r.n_steps;
  const double dt = r.t / double(steps);
  const double drift_dt = (r.r - 0.5 * r.sigma * r.sigma) * dt;
  const double vol_dt = r.sigma * std::sqrt(dt);
  const double discount = std::exp(-r.r * r.t);
  const int w = r.workload;
  const bool european = w == MPC_WORKLOAD_EUROPEAN_CALL;
  Moments m;
  double price, se;
  if (r.sampling == MPC_SAMPLING_PSEUDORANDOM) {
    if (r.technique == MPC_TECHNIQUE_ANTITHETIC) {
      // European: single stream (cpu.rs:7807-7835); the others chunk by pairs (cpu.rs:6982-7020).
      uint64_t pairs = (n + 1) / 2;
      m = run_chunked(r, pairs, !european, [&](uint64_t seed, uint64_t first, uint64_t count) {
        McRng rng(seed);
        Moments mm;
        for (uint64_t i = 0; i < count; ++i) {
          GbmObs a(w, r.k, r.barrier, r.s0), b(w, r.k, r.barrier, r.s0);
          for (uint64_t s = 0; s < steps; ++s) {
            double z = rng.standard_normal();
            a.step(drift_dt + vol_dt * z);
            b.step(drift_dt - vol_dt * z);
          }
          double block = 0.5 * (a.payoff(discount) + b.payoff(discount));
          mm.add(block);
          out.put(first + i, block);
        }
        return mm;
      });
      summarize(pairs, m.s, m.s2, &price, &se);
    } else {
      bool cv = r.technique == MPC_TECHNIQUE_CONTROL_VARIATE;
      m = run_chunked(r, n, true, [&](uint64_t seed, uint64_t first, uint64_t count) {
        McRng rng(seed);
        Moments mm;
        for (uint64_t i = 0; i < count; ++i) {
          GbmObs a(w, r.k, r.barrier, r.s0);
          for (uint64_t s = 0; s < steps; ++s) {
            double z = rng.standard_normal();
            a.step(drift_dt + vol_dt * z);
          }
          double p = a.payoff(discount);
          if (cv)
            mm.add_cv(p, a.control(discount));
          else
            mm.add(p);
          out.put(first + i, p);
        }
        return mm;
      });
      if (cv)
        summarize_cv(m, r.s0, &price, &se);
      else
        summarize(n, m.s, m.s2, &price, &se);
    }
  } else if (r.sampling == MPC_SAMPLING_COUNTER_HASH) {
    // Stateless counter-hash normals (FP32 values, cpu.rs:5435-5454) fed to the FP64 path.
    uint32_t seed32 = uint32_t(r.seed);
    bool cv = r.technique == MPC_TECHNIQUE_CONTROL_VARIATE;
    bool anti = r.technique == MPC_TECHNIQUE_ANTITHETIC;
    uint64_t units = anti ? (n + 1) / 2 : n;
    for (uint64_t i = out.point0; i < out.last(units); ++i) {
      GbmObs a(w, r.k, r.barrier, r.s0), b(w, r.k, r.barrier, r.s0);
      for (uint64_t s = 0; s < steps; ++s) {
        double z = double(stateless_standard_normal_f32(seed32, uint32_t(i), uint32_t(s)));
        a.step(drift_dt + vol_dt * z);
        if (anti) b.step(drift_dt - vol_dt * z);
      }
      double p = anti ? 0.5 * (a.payoff(discount) + b.payoff(discount)) : a.payoff(discount);
      if (cv)
        m.add_cv(p, a.control(discount));
      else
        m.add(p);
      out.put(i, p);
    }
    if (cv)
      summarize_cv(m, r.s0, &price, &se);
    else
      summarize(units, m.s, m.s2, &price, &se);
  } else {
    // Structured samplers (simulate_stepwise_qmc and siblings, cpu.rs:7113-7501).
    Sampler sampler(r.sampling == MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE ? MPC_SAMPLING_SCRAMBLED_SOBOL : r.sampling,
                    r.seed, n, steps);
    bool bridge = r.sampling == MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE;
    BridgePlan plan(bridge ? steps : 1, r.t);
    bool anti = r.technique == MPC_TECHNIQUE_ANTITHETIC;
    bool cv = r.technique == MPC_TECHNIQUE_CONTROL_VARIATE;
    uint64_t units = anti ? (n + 1) / 2 : n;
    std::vector<double> normals(steps), inc;
    for (uint64_t i = out.point0; i < out.last(units); ++i) {
      for (uint64_t s = 0; s < steps; ++s) normals[s] = sampler.normal(i, s);
      const std::vector<double>* zs = &normals;
      if (bridge) {
        plan.increments(normals, inc);
        zs = &inc;
      }
      GbmObs a(w, r.k, r.barrier, r.s0), b(w, r.k, r.barrier, r.s0);
      for (uint64_t s = 0; s < steps; ++s) {
        a.step(drift_dt + vol_dt * (*zs)[s]);
        if (anti) b.step(drift_dt - vol_dt * (*zs)[s]);
      }
      double p = anti ? 0.5 * (a.payoff(discount) + b.payoff(discount)) : a.payoff(discount);
      if (cv)
        m.add_cv(p, a.control(discount));
      else
        m.add(p);
      out.put(i, p);
    }
    if (cv)
      summarize_cv(m, r.s0, &price, &se);
    else
      summarize(units, m.s, m.s2, &price, &se);
  }
  res->price = price;
  res->stderr = se;
  res->n_samples = m.n;
  res->path_steps = n * steps;
  double mom[6] = {double(m.n), m.s, m.s2, m.c, m.c2, m.pc};
  std::memcpy(res->moments, mom, sizeof mom);
}

// GBM terminal European (cpu.rs:3191-3226, 6360-6406, 7063-7111, 7773-7807).
void price_gbm_terminal(const mpc_request_t& r, mpc_result_t* res, const Out& out) {
  const uint64_t n = r.n_paths;
  const double drift_t = (r.r - 0.5 * r.sigma * r.sigma) * r.t;
  const double vol_t = r.sigma * std::sqrt(r.t);
  const double discount = std::exp(-r.r * r.t);
  auto payoff = [&](double z) {  // european_call_payoff_from_shock, cpu.rs:7773-7783
    double st = r.s0 * std::exp(drift_t + vol_t * z);
    return std::max(st - r.k, 0.0) * discount;
  };
  Moments m;
  double price, se;
  bool anti = r.technique == MPC_TECHNIQUE_ANTITHETIC;
  bool cv = r.technique == MPC_TECHNIQUE_CONTROL_VARIATE;
  uint64_t units = anti ? (n + 1) / 2 : n;
  if (r.sampling == MPC_SAMPLING_PSEUDORANDOM) {
    m = run_chunked(r, units, !anti, [&](uint64_t seed, uint64_t first, uint64_t count) {
      McRng rng(seed);
      Moments mm;
      for (uint64_t i = 0; i < count; ++i) {
        double z = rng.standard_normal();
        double p;
        if (anti) {
          p = 0.5 * (payoff(z) + payoff(-z));
          mm.add(p);
        } else if (cv) {
          double st = r.s0 * std::exp(drift_t + vol_t * z);
          p = std::max(st - r.k, 0.0) * discount;
          mm.add_cv(p, discount * st);
        } else {
          p = payoff(z);
          mm.add(p);
        }
        out.put(first + i, p);
      }
      return mm;
    });
  } else {
    Sampler sampler(r.sampling == MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE ? MPC_SAMPLING_SCRAMBLED_SOBOL : r.sampling,
                    r.seed, n, 1);
    for (uint64_t i = 0; i < units; ++i) {
      double z = r.sampling == MPC_SAMPLING_COUNTER_HASH
                     ? double(stateless_standard_normal_f32(uint32_t(r.seed), uint32_t(i), 0))
                     : sampler.normal(i, 0);
      double p;
      if (anti) {
        p = 0.5 * (payoff(z) + payoff(-z));
        m.add(p);
      } else if (cv) {
        double st = r.s0 * std::exp(drift_t + vol_t * z);
        p = std::max(st - r.k, 0.0) * discount;
        m.add_cv(p, discount * st);
      } else {
        p = payoff(z);
        m.add(p);
      }
      out.put(i, p);
    }
  }
  if (cv)
    summarize_cv(m, r.s0, &price, &se);
  else
    summarize(units, m.s, m.s2, &price, &se);
  res->price = price;
  res->stderr = se;
  res->n_samples = m.n;
  res->path_steps = n;
  double mom[6] = {double(m.n), m.s, m.s2, m.c, m.c2, m.pc};
  std::memcpy(res->moments, mom, sizeof mom);
}

// ------------------------------------------------------------- Heston -----
// HestonStepParams / heston_path_terminal (cpu.rs:8632-8686): per step
// z_var, z_independent; variance floored after every step.
struct HestonP {
  double log_s0, k, v0, kappa, theta, xi, rho, rho_perp, dt, sqrt_dt, r, discount;
  uint64_t steps;
};
HestonP heston_params(const mpc_request_t& r) {
  HestonP p;
  p.log_s0 = std::log(r.s0);
  p.k = r.k;
  p.v0 = r.v0;
  p.kappa = r.kappa;
  p.theta = r.theta;
  p.xi = r.vol_of_vol;
  p.rho = r.rho;
  p.rho_perp = std::sqrt(std::max(1.0 - r.rho * r.rho, 0.0));
  p.dt = r.t / double(r.n_steps);
  p.sqrt_dt = std::sqrt(r.t / double(r.n_steps));
  p.steps = r.n_steps;
  p.r = r.r;
  p.discount = std::exp(-r.r * r.t);
  return p;
}
struct HestonState {
  double log_s, v;
  void step(const HestonP& p, double z_var, double z_ind) {
    double vp = std::max(v, 0.0);
    double z_price = p.rho * z_var + p.rho_perp * z_ind;
    log_s += (p.r - 0.5 * vp) * p.dt + std::sqrt(vp) * p.sqrt_dt * z_price;
    v = v + p.kappa * (p.theta - vp) * p.dt + p.xi * std::sqrt(vp) * p.sqrt_dt * z_var;
    v = std::max(v, 0.0);
  }
};

void price_heston(const mpc_request_t& r, mpc_result_t* res, const Out& out) {
  HestonP p = heston_params(r);
  const uint64_t n = r.n_paths;
  bool anti = r.technique == MPC_TECHNIQUE_ANTITHETIC;
  bool cv = r.technique == MPC_TECHNIQUE_CONTROL_VARIATE;
  uint64_t units = anti ? (n + 1) / 2 : n;
  auto finish = [&](const HestonState& s, double* ctl) {
    double st = std::exp(s.log_s);
    if (ctl) *ctl = st * p.discount;
    return std::max(st - p.k, 0.0) * p.discount;
  };
  Moments m;
  if (r.sampling == MPC_SAMPLING_PSEUDORANDOM) {
    // simulate_heston_{,antithetic_,control_variate_}chunk (cpu.rs:8700-8778), chunked (cpu.rs:8780-8881).
    m = run_chunked(r, units, true, [&](uint64_t seed, uint64_t first, uint64_t count) {
      McRng rng(seed);
      Moments mm;
      for (uint64_t i = 0; i < count; ++i) {
        HestonState a{p.log_s0, p.v0}, b{p.log_s0, p.v0};
        for (uint64_t s = 0; s < p.steps; ++s) {
          double zv = rng.standard_normal();
          double zi = rng.standard_normal();
          a.step(p, zv, zi);
          if (anti) b.step(p, -zv, -zi);
        }
        double ctl = 0.0, v;
        if (anti) {
          v = 0.5 * (finish(a, nullptr) + finish(b, nullptr));
          mm.add(v);
        } else if (cv) {
          v = finish(a, &ctl);
          mm.add_cv(v, ctl);
        } else {
          v = finish(a, nullptr);
          mm.add(v);
        }
        out.put(first + i, v);
      }
      return mm;
    });
  } else {
    // Extension: structured / counter-hash inputs, dims 2 per step (z_var, z_independent).
    Sampler sampler(r.sampling, r.seed, n, 2 * size_t(p.steps));
    uint32_t seed32 = uint32_t(r.seed);
    for (uint64_t i = out.point0; i < out.last(units); ++i) {
      HestonState a{p.log_s0, p.v0}, b{p.log_s0, p.v0};
      for (uint64_t s = 0; s < p.steps; ++s) {
        double zv, zi;
        if (r.sampling == MPC_SAMPLING_COUNTER_HASH) {
          zv = stateless_standard_normal_f32(seed32, uint32_t(i), uint32_t(2 * s));
          zi = stateless_standard_normal_f32(seed32, uint32_t(i), uint32_t(2 * s + 1));
        } else {
          zv = sampler.normal(i, 2 * s);
          zi = sampler.normal(i, 2 * s + 1);
        }
        a.step(p, zv, zi);
        if (anti) b.step(p, -zv, -zi);
      }
      double ctl = 0.0, v;
      if (anti) {
        v = 0.5 * (finish(a, nullptr) + finish(b, nullptr));
        m.add(v);
      } else if (cv) {
        v = finish(a, &ctl);
        m.add_cv(v, ctl);
      } else {
        v = finish(a, nullptr);
        m.add(v);
      }
      out.put(i, v);
    }
  }
  double price, se;
  if (cv)
    summarize_cv(m, r.s0, &price, &se);
  else
    summarize(units, m.s, m.s2, &price, &se);
  res->price = price;
  res->stderr = se;
  res->n_samples = m.n;
  res->path_steps = n * p.steps;
  double mom[6] = {double(m.n), m.s, m.s2, m.c, m.c2, m.pc};
  std::memcpy(res->moments, mom, sizeof mom);
}

// ------------------------------------------------------------- Merton -----
// sample_poisson by sequential inversion (cpu.rs:932-953), with the uniform supplied.
uint64_t poisson_inverse(double u, double mean) {
  if (mean == 0.0) return 0;
  double prob = std::exp(-mean), cum = prob;
  uint64_t k = 0;
  while (u > cum && k < 4095) {
    ++k;
    prob *= mean / double(k);
    cum += prob;
  }
  return k;
}

void price_merton(const mpc_request_t& r, mpc_result_t* res, const Out& out) {
  const uint64_t n = r.n_paths;
  const double kappa_j = r.jump_intensity * (std::exp(r.jump_mean + 0.5 * r.jump_volatility * r.jump_volatility) - 1.0);
  const double discount = std::exp(-r.r * r.t);
  const double log_s0 = std::log(r.s0);
  Moments m;
  const bool stepwise = r.method == MPC_METHOD_STEPWISE;
  if (!stepwise) {
    // Terminal (cpu.rs:3151-3189, 6408-6441).
    const double drift_t = (r.r - kappa_j - 0.5 * r.sigma * r.sigma) * r.t;
    const double dvol_t = r.sigma * std::sqrt(r.t);
    const double jump_mean_t = r.jump_intensity * r.t;
    auto terminal = [&](double z, uint64_t count, double zj) {
      double jump = count == 0 ? 0.0
                               : double(count) * r.jump_mean + r.jump_volatility * std::sqrt(double(count)) * zj;
      double st = std::exp(log_s0 + drift_t + dvol_t * z + jump);
      return std::max(st - r.k, 0.0) * discount;
    };
    if (r.sampling == MPC_SAMPLING_PSEUDORANDOM) {
      m = run_chunked(r, n, true, [&](uint64_t seed, uint64_t first, uint64_t count) {
        McRng rng(seed);
        Moments mm;
        for (uint64_t i = 0; i < count; ++i) {
          double z = rng.standard_normal();
          // sample_poisson draws its uniform straight from next_f64_open01 (cpu.rs:941).
          uint64_t jumps = 0;
          if (jump_mean_t != 0.0) jumps = poisson_inverse(rng.next_f64_open01(), jump_mean_t);
          double zj = jumps == 0 ? 0.0 : rng.standard_normal();
          double v = terminal(z, jumps, zj);
          mm.add(v);
          out.put(first + i, v);
        }
        return mm;
      });
    } else {
      Sampler sampler(r.sampling, r.seed, n, 3);
      for (uint64_t i = 0; i < n; ++i) {
        double z = sampler.normal(i, 0);
        uint64_t jumps = poisson_inverse(sampler.uniform(i, 1), jump_mean_t);
        double zj = jumps == 0 ? 0.0 : sampler.normal(i, 2);
        double v = terminal(z, jumps, zj);
        m.add(v);
        out.put(i, v);
      }
    }
    res->path_steps = n;
  } else {
    // Extension: stepwise Merton with a Poisson count per step, dims (z, u, z_J) per step.
    const uint64_t steps = r.n_steps;
    const double dt = r.t / double(steps);
    const double drift_dt = (r.r - kappa_j - 0.5 * r.sigma * r.sigma) * dt;
    const double vol_dt = r.sigma * std::sqrt(dt);
    const double lam_dt = r.jump_intensity * dt;
    Sampler sampler(r.sampling, r.seed, n, 3 * size_t(steps));
    auto path = [&](auto&& normal, auto&& uniform) {
      double log_s = log_s0;
      for (uint64_t s = 0; s < steps; ++s) {
        double z = normal(3 * s);
        uint64_t jumps = poisson_inverse(uniform(3 * s + 1), lam_dt);
        log_s += drift_dt + vol_dt * z;
        if (jumps > 0)
          log_s += double(jumps) * r.jump_mean + r.jump_volatility * std::sqrt(double(jumps)) * normal(3 * s + 2);
      }
      return std::max(std::exp(log_s) - r.k, 0.0) * discount;
    };
    if (r.sampling == MPC_SAMPLING_PSEUDORANDOM) {
      m = run_chunked(r, n, true, [&](uint64_t seed, uint64_t first, uint64_t count) {
        McRng rng(seed);
        Moments mm;
        for (uint64_t i = 0; i < count; ++i) {
          // sequential stream: the jump normal is drawn only when a jump occurs
          double log_s = log_s0;
          for (uint64_t s = 0; s < steps; ++s) {
            double z = rng.standard_normal();
            uint64_t jumps = lam_dt == 0.0 ? 0 : poisson_inverse(rng.next_f64_open01(), lam_dt);
            log_s += drift_dt + vol_dt * z;
            if (jumps > 0)
              log_s += double(jumps) * r.jump_mean +
                       r.jump_volatility * std::sqrt(double(jumps)) * rng.standard_normal();
          }
          double v = std::max(std::exp(log_s) - r.k, 0.0) * discount;
          mm.add(v);
          out.put(first + i, v);
        }
        return mm;
      });
    } else if (r.sampling == MPC_SAMPLING_COUNTER_HASH) {
      uint32_t seed32 = uint32_t(r.seed);
      for (uint64_t i = out.point0; i < out.last(n); ++i) {
        double v = path(
            [&](uint64_t d) { return double(stateless_standard_normal_f32(seed32, uint32_t(i), uint32_t(d))); },
            [&](uint64_t d) { return double(stateless_open01_f32(seed32, uint32_t(i), uint32_t(d), 0)); });
        m.add(v);
        out.put(i, v);
      }
    } else {
      for (uint64_t i = out.point0; i < out.last(n); ++i) {
        double v = path([&](uint64_t d) { return sampler.normal(i, d); },
                        [&](uint64_t d) { return sampler.uniform(i, d); });
        m.add(v);
        out.put(i, v);
      }
    }
    res->path_steps = n * steps;
  }
  double price, se;
  summarize(n, m.s, m.s2, &price, &se);
  res->price = price;
  res->stderr = se;
  res->n_samples = m.n;
  double mom[6] = {double(m.n), m.s, m.s2, m.c, m.c2, m.pc};
  std::memcpy(res->moments, mom, sizeof mom);
}

// ------------------------------------------------------------- Basket -----
// Cholesky factor of the correlation matrix (lower, row-major).  For d == 2
// it is [[1,0],[rho, sqrt(1-rho^2)]], i.e. exactly the reference's
// z2 = rho z1 + sqrt(1-rho^2) z2' (cpu.rs:7622-7630).
bool cholesky(const double* corr, uint32_t d, double* L) {
  std::memset(L, 0, sizeof(double) * d * d);
  if (d == 2) {
    L[0] = 1.0;
    L[2] = corr[1];
    L[3] = std::sqrt(std::max(1.0 - corr[1] * corr[1], 0.0));
    return true;
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

void price_basket(const mpc_request_t& r, mpc_result_t* res, const Out& out) {
  const uint32_t d = r.n_assets;
  double L[MPC_MAX_ASSETS * MPC_MAX_ASSETS];
  cholesky(r.corr, d, L);
  const double discount = std::exp(-r.r * r.t);
  const bool stepwise = r.method == MPC_METHOD_STEPWISE;
  const uint64_t steps = stepwise ? r.n_steps : 1;
  const double dt = r.t / double(steps);
  double drift[MPC_MAX_ASSETS], vol[MPC_MAX_ASSETS], expectation = 0.0;
  for (uint32_t a = 0; a < d; ++a) {
    // BasketTerminalParams (cpu.rs:7601-7614) per step of length dt.
    drift[a] = (r.r - 0.5 * r.sigmas[a] * r.sigmas[a]) * dt;
    vol[a] = r.sigmas[a] * std::sqrt(dt);
    expectation += r.weights[a] * r.spots[a];  // basket_control_expectation, cpu.rs:7637-7639
  }
  const uint64_t n = r.n_paths;
  bool anti = r.technique == MPC_TECHNIQUE_ANTITHETIC;
  bool cv = r.technique == MPC_TECHNIQUE_CONTROL_VARIATE;
  uint64_t units = anti ? (n + 1) / 2 : n;
  // basket_terminal_payoff (cpu.rs:7616-7635), generalised to d assets and n steps.
  auto simulate = [&](const double* zs, double sign, double* ctl) {
    double x[MPC_MAX_ASSETS] = {0};
    for (uint64_t s = 0; s < steps; ++s) {
      const double* z = zs + s * d;
      for (uint32_t a = 0; a < d; ++a) {
        double zc = 0.0;
        if (d == 2 && a == 1)
          zc = r.corr[1] * (sign * z[0]) + L[3] * (sign * z[1]);
        else
          for (uint32_t b = 0; b <= a; ++b) zc += L[a * d + b] * (sign * z[b]);
        x[a] += drift[a] + vol[a] * zc;
      }
    }
    double basket = 0.0;
    for (uint32_t a = 0; a < d; ++a) basket += r.weights[a] * (r.spots[a] * std::exp(x[a]));
    if (ctl) *ctl = basket * discount;
    return std::max(basket - r.k, 0.0) * discount;
  };
  std::vector<double> zs(steps * d);
  Moments m;
  McRng rng(r.seed);  // the reference basket uses one stream, no chunking (cpu.rs:7503-7518)
  Sampler sampler(r.sampling, r.seed, n, steps * d);
  for (uint64_t i = 0; i < units; ++i) {
    for (uint64_t j = 0; j < steps * d; ++j) {
      if (r.sampling == MPC_SAMPLING_PSEUDORANDOM)
        zs[j] = rng.standard_normal();
      else if (r.sampling == MPC_SAMPLING_COUNTER_HASH)
        zs[j] = stateless_standard_normal_f32(uint32_t(r.seed), uint32_t(i), uint32_t(j));
      else
        zs[j] = sampler.normal(i, j);
    }
    double ctl = 0.0, v;
    if (anti) {
      v = 0.5 * (simulate(zs.data(), 1.0, nullptr) + simulate(zs.data(), -1.0, nullptr));
      m.add(v);
    } else if (cv) {
      v = simulate(zs.data(), 1.0, &ctl);
      m.add_cv(v, ctl);
    } else {
      v = simulate(zs.data(), 1.0, nullptr);
      m.add(v);
    }
    out.put(i, v);
  }
  double price, se;
  if (cv)
    summarize_cv(m, expectation, &price, &se);
  else
    summarize(units, m.s, m.s2, &price, &se);
  res->price = price;
  res->stderr = se;
  res->n_samples = m.n;
  res->path_steps = n * steps;
  double mom[6] = {double(m.n), m.s, m.s2, m.c, m.c2, m.pc};
  std::memcpy(res->moments, mom, sizeof mom);
}

// ---------------------------------------------------------------- LSM -----
// laguerre_lsm_basis (cpu.rs:7667-7682)
void laguerre(double x, int degree, double* b) {
  double x2 = x * x, x3 = x2 * x;
  b[0] = 1.0;
  b[1] = degree >= 1 ? 1.0 - x : 0.0;
  b[2] = degree >= 2 ? 1.0 - 2.0 * x + 0.5 * x2 : 0.0;
  b[3] = degree >= 3 ? 1.0 - 3.0 * x + 1.5 * x2 - x3 / 6.0 : 0.0;
}
// solve_lsm_normal_equations: Gauss-Jordan with partial pivoting, pivot
// threshold 1e-12 (cpu.rs:7684-7736).
bool solve_normal_equations(double a[4][4], double rhs[4], int dim) {
  for (int piv = 0; piv < dim; ++piv) {
    int best = piv;
    double best_abs = std::fabs(a[piv][piv]);
    for (int row = piv + 1; row < dim; ++row) {
      double c = std::fabs(a[row][piv]);
      if (c > best_abs) {
        best = row;
        best_abs = c;
      }
    }
    if (best_abs <= 1e-12) return false;
    if (best != piv) {
      for (int c = 0; c < 4; ++c) std::swap(a[piv][c], a[best][c]);
      std::swap(rhs[piv], rhs[best]);
    }
    double pv = a[piv][piv];
    for (int c = piv; c < dim; ++c) a[piv][c] /= pv;
    rhs[piv] /= pv;
    for (int row = 0; row < dim; ++row) {
      if (row == piv) continue;
      double f = a[row][piv];
      if (f == 0.0) continue;
      for (int c = piv; c < dim; ++c) a[row][c] -= f * a[piv][c];
      rhs[row] -= f * rhs[piv];
    }
  }
  return true;
}

// Exercise schedule: every step for American (cpu.rs:3950), sorted, deduped
// and maturity-appended for Bermudan (normalize_bermudan_exercise_schedule, cpu.rs:5155-5183).
std::vector<uint32_t> lsm_schedule(const mpc_request_t& r, bool* normalised) {
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

// price_put_lsm_cpu (cpu.rs:3813-3945).  Paths come from one sequential
// MonteCarloRng stream (reference), or from the counter-hash stream (extension).
void price_lsm(const mpc_request_t& r, mpc_result_t* res, const Out& out) {
  const int degree = std::min<int>(std::max<int>(int(r.basis_degree), 1), 3);
  const int coeffs = degree + 1;
  const uint64_t n = r.n_paths, steps = r.n_steps, len = steps + 1;
  const double dt = r.t / double(steps);
  const double drift = (r.r - 0.5 * r.sigma * r.sigma) * dt;
  const double vol_dt = r.sigma * std::sqrt(dt);
  const double disc_step = std::exp(-r.r * dt);
  bool normalised = false;
  std::vector<uint32_t> sched = lsm_schedule(r, &normalised);
  std::vector<double> paths(n * len);
  McRng rng(r.seed);
  for (uint64_t i = 0; i < n; ++i) {
    double s = r.s0;
    paths[i * len] = s;
    for (uint64_t st = 1; st <= steps; ++st) {
      double z = r.sampling == MPC_SAMPLING_COUNTER_HASH
                     ? double(stateless_standard_normal_f32(uint32_t(r.seed), uint32_t(i), uint32_t(st - 1)))
                     : rng.standard_normal();
      s *= std::exp(drift + vol_dt * z);
      paths[i * len + st] = s;
    }
  }
  std::vector<double> cash(n);
  std::vector<uint64_t> ex(n, steps);
  for (uint64_t i = 0; i < n; ++i) cash[i] = std::max(r.k - paths[i * len + steps], 0.0);
  uint32_t regressions = 0;
  const double kk = std::max(r.k, kMinPositive);
  for (int si = int(sched.size()) - 2; si >= 0; --si) {
    uint64_t step = sched[si];
    double ata[4][4] = {{0}}, atb[4] = {0};
    uint64_t itm = 0;
    for (uint64_t i = 0; i < n; ++i) {
      double s = paths[i * len + step];
      double imm = std::max(r.k - s, 0.0);
      if (imm <= 0.0) continue;
      double cont = cash[i] * powi(disc_step, int(ex[i] - step));
      double b[4];
      laguerre(s / kk, degree, b);
      for (int row = 0; row < coeffs; ++row) {
        atb[row] += b[row] * cont;
        for (int col = 0; col < coeffs; ++col) ata[row][col] += b[row] * b[col];
      }
      ++itm;
    }
    if (itm < uint64_t(coeffs)) continue;
    if (!solve_normal_equations(ata, atb, coeffs)) continue;
    ++regressions;
    for (uint64_t i = 0; i < n; ++i) {
      double s = paths[i * len + step];
      double imm = std::max(r.k - s, 0.0);
      if (imm <= 0.0) continue;
      double b[4];
      laguerre(s / kk, degree, b);
      double cont = 0.0;
      for (int j = 0; j < coeffs; ++j) cont += atb[j] * b[j];
      if (imm > std::max(cont, 0.0)) {
        cash[i] = imm;
        ex[i] = step;
      }
    }
  }
  double sum = 0.0, sq = 0.0;
  uint64_t early = 0, maturity = 0;
  for (uint64_t i = 0; i < n; ++i) {
    double v = cash[i] * powi(disc_step, int(ex[i]));
    sum += v;
    sq += v * v;
    out.put(i, v);
    if (ex[i] < steps)
      ++early;
    else if (cash[i] > 0.0)
      ++maturity;
  }
  double price, se;
  summarize(n, sum, sq, &price, &se);
  uint32_t warnings = 0;
  if (r.workload == MPC_WORKLOAD_AMERICAN_PUT) {
    double intrinsic = std::max(r.k - r.s0, 0.0);
    if (intrinsic > price) {
      price = intrinsic;
      se = 0.0;
      warnings |= MPC_WARN_INTRINSIC_FLOOR;
    }
  }
  if (int(r.basis_degree) != degree) warnings |= MPC_WARN_BASIS_DEGREE_CLAMPED;
  if (normalised) warnings |= MPC_WARN_SCHEDULE_NORMALISED;
  res->price = price;
  res->stderr = se;
  res->n_samples = n;
  res->path_steps = n * steps;
  res->early_exercise_count = early;
  res->maturity_exercise_count = maturity;
  res->regression_steps = regressions;
  res->basis_degree = uint32_t(degree);
  res->warnings |= warnings;
  double mom[6] = {double(n), sum, sq, 0, 0, 0};
  std::memcpy(res->moments, mom, sizeof mom);
}

// -------------------------------------------------------------- MLMC ------
uint64_t mlmc_fine_steps(uint64_t base, uint64_t m, uint64_t level) {  // cpu.rs:6631-6639
  uint64_t s = base;
  for (uint64_t l = 0; l < level; ++l) s *= m;
  return s;
}

// simulate_asian_mlmc_level / _structured_level / coupled differences
// (cpu.rs:6641-6894): level 0 is the plain Asian payoff with base steps;
// level l couples a fine path (M normals per coarse step) with a coarse path
// driven by sum(z)/sqrt(M).
Moments mlmc_level(const mpc_request_t& r, uint64_t seed, uint64_t level, uint64_t paths) {
  const uint64_t fine = mlmc_fine_steps(r.base_steps, r.refinement_factor, level);
  const uint64_t level_seed = derive_chunk_seed(seed, level);
  const double discount = std::exp(-r.r * r.t);
  const double ls0 = std::log(r.s0);
  Moments m;
  McRng rng(level_seed);
  Sampler sampler(r.sampling, level_seed, paths, fine);
  std::vector<double> zs(fine);
  for (uint64_t i = 0; i < paths; ++i) {
    for (uint64_t j = 0; j < fine; ++j)
      zs[j] = r.sampling == MPC_SAMPLING_PSEUDORANDOM
                  ? rng.standard_normal()
                  : (r.sampling == MPC_SAMPLING_COUNTER_HASH
                         ? double(stateless_standard_normal_f32(uint32_t(level_seed), uint32_t(i), uint32_t(j)))
                         : sampler.normal(i, j));
    double v;
    if (level == 0) {
      double dt = r.t / double(fine);
      double drift = (r.r - 0.5 * r.sigma * r.sigma) * dt, vol = r.sigma * std::sqrt(dt);
      double ls = ls0, sum = 0.0;
      for (uint64_t j = 0; j < fine; ++j) {
        ls += drift + vol * zs[j];
        sum += std::exp(ls);
      }
      v = std::max(sum / double(fine) - r.k, 0.0) * discount;
    } else {
      const uint64_t M = r.refinement_factor, coarse = fine / M;
      double fdt = r.t / double(fine), cdt = r.t / double(coarse);
      double fdrift = (r.r - 0.5 * r.sigma * r.sigma) * fdt, fvol = r.sigma * std::sqrt(fdt);
      double cdrift = (r.r - 0.5 * r.sigma * r.sigma) * cdt, cvol = r.sigma * std::sqrt(cdt);
      double sqrt_m = std::sqrt(double(M));
      double fl = ls0, cl = ls0, fs = 0.0, cs = 0.0;
      uint64_t j = 0;
      for (uint64_t c = 0; c < coarse; ++c) {
        double zsum = 0.0;
        for (uint64_t q = 0; q < M; ++q) {
          double z = zs[j++];
          zsum += z;
          fl += fdrift + fvol * z;
          fs += std::exp(fl);
        }
        double zc = zsum / sqrt_m;
        cl += cdrift + cvol * zc;
        cs += std::exp(cl);
      }
      double pf = std::max(fs / double(coarse * M) - r.k, 0.0) * discount;
      double pc = std::max(cs / double(coarse) - r.k, 0.0) * discount;
      v = pf - pc;
    }
    m.add(v);
  }
  return m;
}

// arithmetic_asian_call_price_mlmc_single_cpu / _replicated_cpu
// (cpu.rs:3612-3751) with the tolerance solver of cpu.rs:3352-3423,
// 3539-3610 when target_stderr > 0.
void price_mlmc(const mpc_request_t& r_in, mpc_result_t* res) {
  mpc_request_t r = r_in;
  const uint64_t L = r.levels;
  bool pseudo = r.sampling == MPC_SAMPLING_PSEUDORANDOM || r.sampling == MPC_SAMPLING_COUNTER_HASH;
  uint64_t reps = pseudo ? 1 : std::max<uint32_t>(r.scramble_replicates, 1);
  if (r.target_stderr > 0.0) {
    auto cost = [&](uint64_t l) {
      uint64_t f = mlmc_fine_steps(r.base_steps, r.refinement_factor, l);
      return f + (l == 0 ? 0 : f / r.refinement_factor);
    };
    std::vector<double> pilot_var(L);
    for (uint64_t l = 0; l < L; ++l) {  // measure_arithmetic_asian_mlmc_pilot_levels, cpu.rs:3567-3598
      Moments m = mlmc_level(r, r.seed, l, r.pilot_paths_per_level);
      double nn = double(r.pilot_paths_per_level), mean = m.s / nn;
      pilot_var[l] = std::max((m.s2 / nn) - mean * mean, 1.0e-18);
    }
    auto allocate = [&](double target_variance, bool by_budget, uint64_t budget, std::vector<uint64_t>& paths) {
      double denom = 0.0;
      for (uint64_t l = 0; l < L; ++l) denom += std::sqrt(pilot_var[l] * double(cost(l)));
      uint64_t total = 0;
      for (uint64_t l = 0; l < L; ++l) {
        double weight = std::sqrt(pilot_var[l] / double(cost(l)));
        double raw = by_budget ? std::ceil(double(budget) * weight / denom) : std::ceil(denom * weight / target_variance);
        paths[l] = std::max<uint64_t>(uint64_t(raw), 2);
        total += paths[l] * cost(l);
      }
      return total;
    };
    auto est_se = [&](const std::vector<uint64_t>& paths) {
      double v = 0.0;
      for (uint64_t l = 0; l < L; ++l) v += pilot_var[l] / double(paths[l]);
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
    for (uint64_t l = 0; l < L; ++l) r.paths_per_level[l] = paths[l];
    res->estimated_stderr = est;
    res->target_met = (est <= r.target_stderr && updates <= r.max_step_updates) ? 1 : 0;
    res->max_step_updates_hit = hit ? 1 : 0;
  }
  std::vector<double> rep_price(reps);
  std::vector<std::vector<double>> lmean(reps, std::vector<double>(L)), lvar(reps, std::vector<double>(L));
  double single_se = 0.0;
  uint64_t total_paths = 0, total_updates = 0;
  for (uint64_t rep = 0; rep < reps; ++rep) {
    uint64_t seed = reps > 1 ? derive_chunk_seed(r.seed, rep) : r.seed;
    double price = 0.0, varc = 0.0;
    for (uint64_t l = 0; l < L; ++l) {
      uint64_t paths = r.paths_per_level[l];
      uint64_t fine = mlmc_fine_steps(r.base_steps, r.refinement_factor, l);
      Moments m = mlmc_level(r, seed, l, paths);
      double nn = double(paths), mean = m.s / nn;
      double var = std::max((m.s2 / nn) - mean * mean, 0.0);
      price += mean;
      varc += var / nn;
      lmean[rep][l] = mean;
      lvar[rep][l] = var;
      total_paths += paths;
      total_updates += paths * (fine + (l == 0 ? 0 : fine / r.refinement_factor));
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
  res->price = price;
  res->stderr = se;
  res->n_levels = uint32_t(L);
  res->total_paths = total_paths;
  res->total_step_updates = total_updates;
  res->path_steps = total_updates;
  for (uint64_t l = 0; l < L && l < MPC_MAX_LEVELS; ++l) {
    double mean = 0.0;
    for (uint64_t rep = 0; rep < reps; ++rep) mean += lmean[rep][l];
    mean /= double(reps);
    double var = lvar[0][l];
    if (reps > 1) {
      var = 0.0;
      for (uint64_t rep = 0; rep < reps; ++rep) var += (lmean[rep][l] - mean) * (lmean[rep][l] - mean);
      var /= double(reps - 1);
    }
    res->level_mean[l] = mean;
    res->level_variance[l] = var;
    res->level_paths[l] = r.paths_per_level[l] * reps;
    res->level_fine_steps[l] = mlmc_fine_steps(r.base_steps, r.refinement_factor, l);
  }
}

// ------------------------------------------------------------ Analytic ----
// standard_normal_cdf with Abramowitz-Stegun 7.1.26 erf (cpu.rs:896-909).
double norm_cdf_as(double x) {
  double sign = x < 0.0 ? -1.0 : 1.0;
  double z = std::fabs(x) / std::sqrt(2.0);
  double t = 1.0 / (1.0 + 0.3275911 * z);
  double poly = (((((1.061405429 * t + -1.453152027) * t) + 1.421413741) * t + -0.284496736) * t + 0.254829592) * t;
  double erf_approx = 1.0 - poly * std::exp(-z * z);
  return 0.5 * (1.0 + sign * erf_approx);
}
double norm_cdf_exact(double x) { return 0.5 * std::erfc(-x / std::sqrt(2.0)); }

// black_scholes_european_call_price (cpu.rs:839-860); exact=1 uses erfc.
double bs_call(double s0, double k, double r, double sigma, double t, int exact) {
  if (k == 0.0) return s0;
  if (t == 0.0) return std::max(s0 - k, 0.0);
  if (sigma == 0.0) return std::max(s0 - k * std::exp(-r * t), 0.0);
  double st = std::sqrt(t);
  double d1 = (std::log(s0 / k) + (r + 0.5 * sigma * sigma) * t) / (sigma * st);
  double d2 = d1 - sigma * st;
  auto N = exact ? norm_cdf_exact : norm_cdf_as;
  return s0 * N(d1) - k * std::exp(-r * t) * N(d2);
}

// discounted_lognormal_call_price (cpu.rs:912-930)
double lognormal_call(double log_mean, double log_var, double k, double r, double t, int exact) {
  if (log_var == 0.0) return std::exp(-r * t) * std::max(std::exp(log_mean) - k, 0.0);
  double sd = std::sqrt(log_var);
  double d2 = (log_mean - std::log(k)) / sd;
  double d1 = d2 + sd;
  auto N = exact ? norm_cdf_exact : norm_cdf_as;
  return std::exp(-r * t) * (std::exp(log_mean + 0.5 * log_var) * N(d1) - k * N(d2));
}

// merton_jump_diffusion_call_reference_price (cpu.rs:3110-3149)
double merton_series(double s0, double k, double r, double sigma, double lam, double mj, double sj, double t,
                     int max_terms, double tail_tol, int exact) {
  double lam_t = lam * t;
  if (lam_t == 0.0) return bs_call(s0, k, r, sigma, t, exact);
  double comp = lam * (std::exp(mj + 0.5 * sj * sj) - 1.0);
  double base = std::log(s0) + (r - comp - 0.5 * sigma * sigma) * t;
  double w = std::exp(-lam_t), cum = 0.0, price = 0.0;
  for (int n = 0; n < max_terms; ++n) {
    double lm = base + double(n) * mj;
    double lv = sigma * sigma * t + double(n) * sj * sj;
    price += w * lognormal_call(lm, lv, k, r, t, exact);
    cum += w;
    if (std::max(1.0 - cum, 0.0) <= tail_tol) break;
    w *= lam_t / double(n + 1);
  }
  return price;
}

// binomial_put_reference_price, CRR tree with an exercise mask (cpu.rs:5244-5305).
double crr_put(double s0, double k, double r, double sigma, double t, int ref_steps, const uint32_t* ex,
               int n_ex) {
  int N = ref_steps;
  if (N < 1) return std::max(k - s0, 0.0);
  double dt = t / double(N);
  double u = std::exp(sigma * std::sqrt(dt)), d = 1.0 / u;
  double growth = std::exp(r * dt);
  double p = (growth - d) / (u - d);
  double disc = std::exp(-r * dt);
  std::vector<double> v(N + 1);
  std::vector<char> mask(N + 1, 0);
  if (ex == nullptr) {
    for (int s = 0; s <= N; ++s) mask[s] = 1;
  } else {
    for (int i = 0; i < n_ex; ++i)
      if (int(ex[i]) <= N) mask[ex[i]] = 1;
  }
  mask[N] = 1;
  for (int dn = 0; dn <= N; ++dn) {
    double st = s0 * powi(u, N - dn) * powi(d, dn);
    v[dn] = std::max(k - st, 0.0);
  }
  for (int step = N - 1; step >= 0; --step) {
    for (int dn = 0; dn <= step; ++dn) {
      double cont = disc * (p * v[dn] + (1.0 - p) * v[dn + 1]);
      if (mask[step]) {
        double st = s0 * powi(u, step - dn) * powi(d, dn);
        v[dn] = std::max(cont, k - st);
      } else {
        v[dn] = cont;
      }
    }
  }
  return v[0];
}

// Heston (1993) semi-analytic call via the Lewis (2001) single integral and
// the Albrecher et al. (2007) "little trap" characteristic function.  The
// reference has no closed-form Heston; this is the backend's own yardstick.
double heston_call(double s0, double k, double r, double v0, double kappa, double theta, double xi, double rho,
                   double t) {
  using cd = std::complex<double>;
  const cd I(0.0, 1.0);
  if (xi < 1e-10) {  // deterministic variance: BS with integrated variance
    double vbar = kappa > 1e-12 ? theta + (v0 - theta) * (1.0 - std::exp(-kappa * t)) / (kappa * t) : v0;
    return bs_call(s0, k, r, std::sqrt(std::max(vbar, 0.0)), t, 1);
  }
  // characteristic function of X = ln(S_T/S_0) - r T
  auto cf = [&](cd u) {
    cd a = kappa - rho * xi * I * u;
    cd d = std::sqrt(a * a + xi * xi * (I * u + u * u));
    cd g = (a - d) / (a + d);
    cd e = std::exp(-d * t);
    cd C = kappa * theta / (xi * xi) * ((a - d) * t - 2.0 * std::log((1.0 - g * e) / (1.0 - g)));
    cd D = (a - d) / (xi * xi) * (1.0 - e) / (1.0 - g * e);
    return std::exp(C + D * v0);
  };
  double x = std::log(s0 / k) + r * t;
  // integrand Re[e^{i u x} cf(u - i/2)] / (u^2 + 1/4) on (0, inf), u = tan-mapped.
  auto f = [&](double u) {
    cd val = std::exp(I * u * x) * cf(cd(u, -0.5));
    return val.real() / (u * u + 0.25);
  };
  // Gauss-Legendre on [0, U] in panels.
  static const double gx[8] = {-0.9602898564975363, -0.7966664774136267, -0.5255324099163290, -0.1834346424956498,
                               0.1834346424956498,  0.5255324099163290,  0.7966664774136267,  0.9602898564975363};
  static const double gw[8] = {0.1012285362903763, 0.2223810344533745, 0.3137066458778873, 0.3626837833783620,
                               0.3626837833783620, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763};
  double integral = 0.0;
  const double U = 400.0;
  const int panels = 4000;
  double h = U / panels;
  for (int pnl = 0; pnl < panels; ++pnl) {
    double a = pnl * h, mid = a + 0.5 * h;
    for (int q = 0; q < 8; ++q) integral += gw[q] * 0.5 * h * f(mid + 0.5 * h * gx[q]);
  }
  return s0 - std::sqrt(s0 * k) * std::exp(-r * t / 2.0) / kPi * integral;
}

int price(const mpc_request_t& r, mpc_result_t* res, const Out& out) {
  std::memset(res, 0, sizeof(*res));
  switch (r.workload) {
    case MPC_WORKLOAD_AMERICAN_PUT:
    case MPC_WORKLOAD_BERMUDAN_PUT:
      price_lsm(r, res, out);
      return 0;
    case MPC_WORKLOAD_ASIAN_MLMC:
      price_mlmc(r, res);
      return 0;
    case MPC_WORKLOAD_BASKET_CALL:
      price_basket(r, res, out);
      return 0;
    default:
      break;
  }
  if (r.model == MPC_MODEL_HESTON) {
    price_heston(r, res, out);
    return 0;
  }
  if (r.model == MPC_MODEL_MERTON) {
    price_merton(r, res, out);
    return 0;
  }
  if (r.workload == MPC_WORKLOAD_EUROPEAN_CALL && r.method != MPC_METHOD_STEPWISE) {
    price_gbm_terminal(r, res, out);
    return 0;
  }
  price_gbm_stepwise(r, res, out);
  return 0;
}

// ---------------------------------------------- same-normals FP32 paths ----
// european/asian/down_and_out/lookback_call_price_mc_stepwise_from_f32_normals
// (cpu.rs:5457-5623): FP32 path arithmetic, FP64 accumulation, path-major normals.
void price_from_f32_normals(const mpc_request_t& r, const float* normals, mpc_result_t* res, double* per_path) {
  std::memset(res, 0, sizeof(*res));
  const float log_s0 = float(std::log(r.s0));
  const float strike = float(r.k);
  const float barrier = float(r.barrier);
  const float dt = float(r.t / double(r.n_steps));
  const float drift_dt = float(r.r - 0.5 * r.sigma * r.sigma) * dt;
  const float vol_dt = float(r.sigma) * std::sqrt(dt);
  const float discount = float(std::exp(-r.r * r.t));
  const float inv_steps = 1.0f / float(r.n_steps);
  double sum = 0.0, sq = 0.0;
  for (uint64_t i = 0; i < r.n_paths; ++i) {
    float ls = log_s0, asum = 0.0f, max_s = float(r.s0);
    bool knocked = (r.workload == MPC_WORKLOAD_DOWN_AND_OUT_CALL && r.s0 <= r.barrier) ||
                   (r.workload == MPC_WORKLOAD_UP_AND_OUT_CALL && r.s0 >= r.barrier);
    const float* z = normals + i * r.n_steps;
    for (uint32_t s = 0; s < r.n_steps; ++s) {
      float inc = drift_dt + vol_dt * z[s];
      ls += inc;
      switch (r.workload) {
        case MPC_WORKLOAD_ARITHMETIC_ASIAN_CALL:
          asum += std::exp(ls);
          break;
        case MPC_WORKLOAD_DOWN_AND_OUT_CALL:
          if (std::exp(ls) <= barrier) knocked = true;
          break;
        case MPC_WORKLOAD_UP_AND_OUT_CALL:
          if (std::exp(ls) >= barrier) knocked = true;
          break;
        case MPC_WORKLOAD_LOOKBACK_CALL:
          max_s = std::max(max_s, std::exp(ls));
          break;
        default:
          break;
      }
    }
    float pf;
    switch (r.workload) {
      case MPC_WORKLOAD_ARITHMETIC_ASIAN_CALL:
        pf = std::max(asum * inv_steps - strike, 0.0f) * discount;
        break;
      case MPC_WORKLOAD_LOOKBACK_CALL:
        pf = std::max(max_s - strike, 0.0f) * discount;
        break;
      case MPC_WORKLOAD_DOWN_AND_OUT_CALL:
      case MPC_WORKLOAD_UP_AND_OUT_CALL:
        pf = knocked ? 0.0f : std::max(std::exp(ls) - strike, 0.0f) * discount;
        break;
      default:
        pf = std::max(std::exp(ls) - strike, 0.0f) * discount;
    }
    double p = double(pf);
    sum += p;
    sq += p * p;
    if (per_path) per_path[i] = p;
  }
  summarize(r.n_paths, sum, sq, &res->price, &res->stderr);
  res->n_samples = r.n_paths;
  res->path_steps = r.n_paths * r.n_steps;
  double mom[6] = {double(r.n_paths), sum, sq, 0, 0, 0};
  std::memcpy(res->moments, mom, sizeof mom);
}

// --------------------------------------------------------------- Greeks ---
// Bump sizes and floors (cpu.rs:4985-5008).
static double bump_spot(double spot) { return std::max(std::fabs(spot) * 0.01, 0.01); }
static double bump_volatility(double vol) { return std::max(std::fabs(vol) * 0.05, 0.005); }
static double bump_rate() { return 0.001; }
static double bump_maturity(double t) { return std::min(1.0 / 365.0, t * 0.25); }
static double parameter_floor(int greek) { return greek == MPC_GREEK_RHO ? -1.0 : kMinPositive; }

// MomentAccumulator::mean_stderr (cpu.rs:4846-4869): (n - 1) sample variance.
struct GreekMoments {
  double sum = 0.0, sq = 0.0;
  uint64_t count = 0;
  void record(double v) {
    sum += v;
    sq += v * v;
    ++count;
  }
  void mean_stderr(double* mean, double* se) const {
    if (count == 0) {
      *mean = *se = 0.0;
      return;
    }
    const double n = double(count);
    *mean = sum / n;
    const double var = count > 1 ? std::max((sq - sum * sum / n) / (n - 1.0), 0.0) : 0.0;
    *se = std::sqrt(var / n);
  }
};

// One bumped parameter of the bump-and-revalue recipe.
struct BumpSpec {
  int greek;
  double center, bump;
  bool reverse;
  std::function<void(mpc_request_t&, double)> set;
};

// The Greeks a workload offers and how each parameter is bumped
// (european_call_bump_greeks_cpu, cpu.rs:4409-4482; Asian, barrier and
// lookback cpu.rs:4047-4323; basket_call_bump_greeks_cpu, cpu.rs:4484-4590;
// heston_call_bump_greeks_cpu, cpu.rs:4592-4668).  Empty = no Greeks.
static std::vector<BumpSpec> bump_specs(const mpc_request_t& r) {
  std::vector<BumpSpec> v;
  const auto rho = BumpSpec{MPC_GREEK_RHO, r.r, bump_rate(), false, [](mpc_request_t& q, double x) { q.r = x; }};
  const auto theta =
      BumpSpec{MPC_GREEK_THETA, r.t, bump_maturity(r.t), true, [](mpc_request_t& q, double x) { q.t = x; }};
  switch (r.workload) {
    case MPC_WORKLOAD_BASKET_CALL:
      v.push_back({MPC_GREEK_DELTA, r.spots[0], bump_spot(r.spots[0]), false,
                   [](mpc_request_t& q, double x) { q.spots[0] = x; }});
      v.push_back({MPC_GREEK_DELTA2, r.spots[1], bump_spot(r.spots[1]), false,
                   [](mpc_request_t& q, double x) { q.spots[1] = x; }});
      v.push_back({MPC_GREEK_VEGA, r.sigmas[0], bump_volatility(r.sigmas[0]), false,
                   [](mpc_request_t& q, double x) { q.sigmas[0] = x; }});
      v.push_back({MPC_GREEK_VEGA2, r.sigmas[1], bump_volatility(r.sigmas[1]), false,
                   [](mpc_request_t& q, double x) { q.sigmas[1] = x; }});
      v.push_back(rho);
      v.push_back(theta);
      return v;
    case MPC_WORKLOAD_EUROPEAN_CALL:
      if (r.model == MPC_MODEL_MERTON) return v;
      if (r.model == MPC_MODEL_HESTON) {
        const double sv = std::sqrt(std::max(r.v0, 0.0));
        v.push_back({MPC_GREEK_DELTA, r.s0, bump_spot(r.s0), false, [](mpc_request_t& q, double x) { q.s0 = x; }});
        v.push_back({MPC_GREEK_VEGA, sv, bump_volatility(sv), false, [](mpc_request_t& q, double x) {
                       const double c = std::max(x, 0.0);
                       q.v0 = c * c;
                     }});
        v.push_back(rho);
        v.push_back(theta);
        return v;
      }
      [[fallthrough]];
    case MPC_WORKLOAD_ARITHMETIC_ASIAN_CALL:
    case MPC_WORKLOAD_DOWN_AND_OUT_CALL:
    case MPC_WORKLOAD_UP_AND_OUT_CALL:
    case MPC_WORKLOAD_LOOKBACK_CALL:
      if (r.model != MPC_MODEL_GBM) return v;
      v.push_back({MPC_GREEK_DELTA, r.s0, bump_spot(r.s0), false, [](mpc_request_t& q, double x) { q.s0 = x; }});
      v.push_back({MPC_GREEK_VEGA, r.sigma, bump_volatility(r.sigma), false,
                   [](mpc_request_t& q, double x) { q.sigma = x; }});
      v.push_back(rho);
      v.push_back(theta);
      return v;
    default:
      return v;
  }
}

// european_call_pathwise_greeks_cpu / european_call_likelihood_ratio_greeks_cpu
// (cpu.rs:4670-4869): one pass over the terminal shocks of MonteCarloRng(seed).
static void single_pass(const mpc_request_t& r, int estimator, GreekMoments m[4]) {
  McRng rng(r.seed);
  const double sqrt_t = std::sqrt(r.t);
  const double drift_t = (r.r - 0.5 * r.sigma * r.sigma) * r.t;
  const double vol_t = r.sigma * sqrt_t;
  const double discount = std::exp(-r.r * r.t);
  for (uint64_t i = 0; i < r.n_paths; ++i) {
    const double z = rng.standard_normal();
    const double st = r.s0 * std::exp(drift_t + vol_t * z);
    if (estimator == MPC_GREEKS_PATHWISE) {
      const double intrinsic = st - r.k;
      const bool active = intrinsic > 0.0;
      const double payoff = std::max(intrinsic, 0.0);
      const double dpay = discount * payoff;
      m[0].record(active ? discount * st / r.s0 : 0.0);
      m[1].record(active ? discount * st * (-r.sigma * r.t + sqrt_t * z) : 0.0);
      m[2].record(active ? discount * (r.t * st - r.t * payoff) : -r.t * dpay);
      const double dst_dt = st * (r.r - 0.5 * r.sigma * r.sigma + r.sigma * z / (2.0 * sqrt_t));
      const double dmat = active ? discount * (dst_dt - r.r * payoff) : -r.r * dpay;
      m[3].record(-dmat);
    } else {
      const double dpay = discount * std::max(st - r.k, 0.0);
      m[0].record(dpay * z / (r.s0 * r.sigma * sqrt_t));
      const double vega_score = (z * z - 1.0) / r.sigma - sqrt_t * z;
      m[1].record(dpay * vega_score);
      m[2].record(dpay * (z / (r.sigma * sqrt_t) - r.t));
    }
  }
}

// GreekReport of one request (european_call_greeks_cpu and siblings,
// cpu.rs:4036-4356; push_bump_estimate cpu.rs:4938-4983).
int greeks(const mpc_request_t& r, int estimator, mpc_greek_report_t* out) {
  std::memset(out, 0, sizeof(*out));
  out->workload = r.workload;
  out->estimator = estimator;
  out->paths = r.n_paths;
  out->steps = r.workload == MPC_WORKLOAD_BASKET_CALL ? 2u : r.n_steps;
  out->seed = r.seed;
  const std::vector<BumpSpec> specs = bump_specs(r);
  if (specs.empty()) return MPC_E_UNSUPPORTED;
  mpc_result_t base;
  price(r, &base, Out{});
  out->base_price = base.price;
  out->base_stderr = base.stderr;
  if (estimator == MPC_GREEKS_BUMP_AND_REVALUE) {
    for (const BumpSpec& b : specs) {
      mpc_request_t up = r, down = r;
      const double lo = std::max(b.center - b.bump, parameter_floor(b.greek));
      b.set(up, b.center + b.bump);
      b.set(down, lo);
      mpc_result_t ru, rd;
      price(up, &ru, Out{});
      price(down, &rd, Out{});
      const double eff = ((b.center + b.bump) - lo) * 0.5;
      const double raw = eff > 0.0 ? (ru.price - rd.price) / (2.0 * eff) : 0.0;
      mpc_greek_estimate_t& e = out->estimates[out->n_estimates++];
      e.greek = b.greek;
      e.estimator = estimator;
      e.value = b.reverse ? -raw : raw;
      e.stderr = eff > 0.0 ? std::sqrt(ru.stderr * ru.stderr + rd.stderr * rd.stderr) / (2.0 * eff) : 0.0;
      e.bump_size = eff;
      e.base_price = base.price;
      e.bumped_up_price = ru.price;
      e.bumped_down_price = rd.price;
    }
    return 0;
  }
  const bool terminal_gbm_call = r.workload == MPC_WORKLOAD_EUROPEAN_CALL && r.model == MPC_MODEL_GBM;
  if (!terminal_gbm_call) {
    out->warnings |= MPC_GREEK_WARN_ESTIMATOR_UNSUPPORTED;
    return 0;
  }
  if (r.n_paths == 0 || !(r.s0 > 0.0) || !(r.sigma > 0.0) || !(r.t > 0.0)) return MPC_E_INVALID_CONFIG;
  GreekMoments m[4];
  single_pass(r, estimator, m);
  const int greeks_pw[4] = {MPC_GREEK_DELTA, MPC_GREEK_VEGA, MPC_GREEK_RHO, MPC_GREEK_THETA};
  const int count = estimator == MPC_GREEKS_PATHWISE ? 4 : 3;
  for (int g = 0; g < count; ++g) {
    mpc_greek_estimate_t& e = out->estimates[out->n_estimates++];
    e.greek = greeks_pw[g];
    e.estimator = estimator;
    m[g].mean_stderr(&e.value, &e.stderr);
    e.base_price = base.price;
  }
  if (r.sampling != MPC_SAMPLING_PSEUDORANDOM) out->warnings |= MPC_GREEK_WARN_PSEUDORANDOM_SHOCKS;
  if (r.technique != MPC_TECHNIQUE_STANDARD) out->warnings |= MPC_GREEK_WARN_TECHNIQUE_IGNORED;
  return 0;
}

}  // namespace orc

// ====================================================== C entry points ====
extern "C" {

uint64_t or_splitmix64(uint64_t x) { return orc::splitmix64(x); }
uint64_t or_derive_chunk_seed(uint64_t seed, uint64_t idx) { return orc::derive_chunk_seed(seed, idx); }

void or_xorshift_u64(uint64_t seed, uint64_t count, uint64_t* out) {
  orc::McRng rng(seed);
  for (uint64_t i = 0; i < count; ++i) out[i] = rng.next_u64();
}
void or_pseudorandom_normals(uint64_t seed, uint64_t count, double* out) {
  orc::McRng rng(seed);
  for (uint64_t i = 0; i < count; ++i) out[i] = rng.standard_normal();
}
uint32_t or_hash_u32(uint32_t x) { return orc::hash_u32(x); }
uint32_t or_counter_hash(uint32_t seed, uint32_t path, uint32_t step, uint32_t lane) {
  return orc::hash_u32(orc::counter_mix(seed, path, step, lane));
}
float or_counter_uniform_f32(uint32_t seed, uint32_t path, uint32_t step, uint32_t lane) {
  return orc::stateless_open01_f32(seed, path, step, lane);
}
// generate_stepwise_stateless_normals_f32 (cpu.rs:5435-5454), path-major.
void or_stateless_normals_f32(uint64_t seed, uint64_t n_paths, uint64_t n_steps, float* out) {
  for (uint64_t p = 0; p < n_paths; ++p)
    for (uint64_t s = 0; s < n_steps; ++s)
      out[p * n_steps + s] = orc::stateless_standard_normal_f32(uint32_t(seed), uint32_t(p), uint32_t(s));
}
double or_inverse_normal(double p) { return orc::inverse_standard_normal(p); }
uint32_t or_sobol_unscrambled(uint32_t index, uint32_t dim) { return orc::sobol_u32(index, dim); }
uint32_t or_sobol_owen(uint32_t index, uint32_t dim, uint32_t seed) { return orc::sobol_owen_u32(index, dim, seed); }
uint32_t or_sobol_point(uint64_t point, uint64_t dim, uint32_t seed) { return orc::sobol_point_u32(point, dim, seed); }
double or_halton(uint64_t index, uint32_t base) { return orc::halton(index, base); }

// generate_standard_normals_cpu (cpu.rs:5343-5379), row-major [point][dim];
// COUNTER_HASH gives the stateless FP32 normals widened to f64.
void or_generate_normals(int sampling, uint64_t seed, uint64_t n_points, uint64_t dims, double* out) {
  if (sampling == MPC_SAMPLING_PSEUDORANDOM) {
    orc::McRng rng(seed);
    for (uint64_t i = 0; i < n_points * dims; ++i) out[i] = rng.standard_normal();
    return;
  }
  if (sampling == MPC_SAMPLING_COUNTER_HASH) {
    for (uint64_t p = 0; p < n_points; ++p)
      for (uint64_t d = 0; d < dims; ++d)
        out[p * dims + d] = orc::stateless_standard_normal_f32(uint32_t(seed), uint32_t(p), uint32_t(d));
    return;
  }
  int kind = sampling == MPC_SAMPLING_SCRAMBLED_SOBOL_BRIDGE ? MPC_SAMPLING_SCRAMBLED_SOBOL : sampling;
  orc::Sampler s(kind, seed, n_points, dims);
  for (uint64_t p = 0; p < n_points; ++p)
    for (uint64_t d = 0; d < dims; ++d) out[p * dims + d] = s.normal(p, d);
}
void or_generate_uniforms(int sampling, uint64_t seed, uint64_t n_points, uint64_t dims, double* out) {
  orc::Sampler s(sampling, seed, n_points, dims);
  for (uint64_t p = 0; p < n_points; ++p)
    for (uint64_t d = 0; d < dims; ++d) out[p * dims + d] = s.uniform(p, d);
}

int or_price(const mpc_request_t* req, mpc_result_t* res) { return orc::price(*req, res, orc::Out{}); }

// The reference configs' Default values (cpu.rs:1311-1327 EuropeanCallConfig,
// 1448-1466 Heston, 1484-1500 Merton, 1517-1533 Asian, 1551-1568 MLMC,
// 1620-1630 MLMC tolerance, 1660-1678 down-and-out, 1694-1710 lookback,
// 1731-1751 basket, 1767-1781 American put, 1799-1815 Bermudan put), folded
// into one request: the fields a workload's config does not have are the
// values of the config that has them.  The up-and-out barrier (120) has no
// reference config.  The oracle's own copy, so that a caller of the oracle
// (the CPU reference arm of the benchmark) needs nothing from the CUDA library.
int or_request_defaults(mpc_request_t* r, int workload) {
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
  const uint64_t ppl[4] = {50000, 25000, 12500, 6250};
  for (int i = 0; i < 4; ++i) r->paths_per_level[i] = ppl[i];
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
      for (int i = 0; i < 4; ++i) r->exercise_steps[i] = 16u * uint32_t(i + 1);
      break;
    case MPC_WORKLOAD_BASKET_CALL:
      r->method = MPC_METHOD_TERMINAL;
      r->n_steps = 1;
      break;
    default:
      break;
  }
  return (workload < 0 || workload > MPC_WORKLOAD_ASIAN_MLMC) ? MPC_E_INVALID_CONFIG : MPC_OK;
}
int or_greeks(const mpc_request_t* req, int estimator, mpc_greek_report_t* out) {
  return orc::greeks(*req, estimator, out);
}
int or_price_paths(const mpc_request_t* req, mpc_result_t* res, double* values, uint64_t capacity) {
  orc::Out out;
  out.values = values;
  out.capacity = capacity;
  return orc::price(*req, res, out);
}
void or_price_from_f32_normals(const mpc_request_t* req, const float* normals, mpc_result_t* res,
                               double* per_path) {
  orc::price_from_f32_normals(*req, normals, res, per_path);
}

// Throughput harness for the CPU baseline: splits the points of a structured
// or counter-hash request into `threads` contiguous windows priced
// concurrently and merged in window order.  Only the floating-point
// summation order differs from the single-thread oracle.
int or_price_threaded(const mpc_request_t* req, int threads, mpc_result_t* res) {
  bool windowed = req->sampling != MPC_SAMPLING_PSEUDORANDOM && req->technique != MPC_TECHNIQUE_CONTROL_VARIATE &&
                  req->workload != MPC_WORKLOAD_AMERICAN_PUT && req->workload != MPC_WORKLOAD_BERMUDAN_PUT &&
                  req->workload != MPC_WORKLOAD_ASIAN_MLMC && req->workload != MPC_WORKLOAD_BASKET_CALL;
  if (threads <= 1 || !windowed || req->n_paths < uint64_t(threads) * 64) return or_price(req, res);
  const uint64_t units = req->technique == MPC_TECHNIQUE_ANTITHETIC ? (req->n_paths + 1) / 2 : req->n_paths;
  std::vector<orc::Moments> parts(threads);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    uint64_t first = units * uint64_t(t) / uint64_t(threads), last = units * uint64_t(t + 1) / uint64_t(threads);
    pool.emplace_back([&parts, req, t, first, last] {
      orc::Out out;
      out.point0 = first;
      out.point_count = last - first;
      mpc_result_t rr;
      orc::price(*req, &rr, out);
      parts[t].n = last - first;
      parts[t].s = rr.moments[1];
      parts[t].s2 = rr.moments[2];
    });
  }
  orc::Moments total;
  for (int t = 0; t < threads; ++t) {
    pool[t].join();
    total.merge(parts[t]);
  }
  std::memset(res, 0, sizeof(*res));
  orc::summarize(total.n, total.s, total.s2, &res->price, &res->stderr);
  res->n_samples = total.n;
  res->moments[0] = double(total.n);
  res->moments[1] = total.s;
  res->moments[2] = total.s2;
  return 0;
}

double or_bs_call(double s0, double k, double r, double sigma, double t, int exact) {
  return orc::bs_call(s0, k, r, sigma, t, exact);
}
// black_scholes_european_put_price (cpu.rs:862-865)
double or_bs_put(double s0, double k, double r, double sigma, double t, int exact) {
  return orc::bs_call(s0, k, r, sigma, t, exact) + k * std::exp(-r * t) - s0;
}
// black_scholes_european_call_greeks (cpu.rs:867-893): out = price, delta, vega, rho, theta.
// exact = 1 evaluates the normal CDF with erfc instead of the A&S 7.1.26 erf.
void or_bs_greeks(double s0, double k, double r, double sigma, double t, int exact, double* out) {
  auto N = exact ? orc::norm_cdf_exact : orc::norm_cdf_as;
  double st = std::sqrt(t);
  double d1 = (std::log(s0 / k) + (r + 0.5 * sigma * sigma) * t) / (sigma * st);
  double d2 = d1 - sigma * st;
  double disc = std::exp(-r * t);
  double pdf = std::exp(-0.5 * d1 * d1) / std::sqrt(2.0 * orc::kPi);
  out[0] = s0 * N(d1) - k * disc * N(d2);
  out[1] = N(d1);
  out[2] = s0 * pdf * st;
  out[3] = k * t * disc * N(d2);
  out[4] = -(s0 * pdf * sigma) / (2.0 * st) - r * k * disc * N(d2);
}
double or_merton_series(double s0, double k, double r, double sigma, double lam, double mj, double sj, double t,
                        int max_terms, double tail_tol, int exact) {
  return orc::merton_series(s0, k, r, sigma, lam, mj, sj, t, max_terms, tail_tol, exact);
}
double or_crr_put(double s0, double k, double r, double sigma, double t, int ref_steps, const uint32_t* ex,
                  int n_ex) {
  return orc::crr_put(s0, k, r, sigma, t, ref_steps, ex, n_ex);
}
double or_heston_call(double s0, double k, double r, double v0, double kappa, double theta, double xi, double rho,
                      double t) {
  return orc::heston_call(s0, k, r, v0, kappa, theta, xi, rho, t);
}

}  // extern "C"

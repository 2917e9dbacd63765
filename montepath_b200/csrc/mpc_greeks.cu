// mpc_greeks.cu -- Greeks of one pricing request (mpc_greeks).
//
// Restates the reference's Greek reports (crates/mc-core/src/runtime/cpu.rs:
// european_call_greeks_cpu and siblings 4036-4356, bump recipe 4938-5008,
// single-pass estimators 4670-4869) on the device:
//  - bump-and-revalue: the base request plus an up and a down bump per Greek,
//    all with the request's seed (common random numbers).  FP32 requests
//    with xorshift, Sobol or counter-hash samples (any technique; a basket
//    with the standard one) price all 9 legs (13 for a basket) in one
//    scenario launch that draws each normal once for every leg; the others
//    price their legs with one mpc_price_batch call;
//  - pathwise / likelihood ratio: one kernel pass over the pseudorandom
//    terminal shocks of the request's seed, sums in FP64.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/montepath_cuda.h"
#include "mpc_launch.h"
#include "mpc_runtime.h"

namespace mpc {
namespace {

// Bump sizes and floors (bump_spot / bump_volatility / bump_rate /
// bump_maturity / parameter_floor, cpu.rs:4985-5008).
double bump_spot(double spot) { return std::max(std::fabs(spot) * 0.01, 0.01); }
double bump_volatility(double vol) { return std::max(std::fabs(vol) * 0.05, 0.005); }
double bump_rate() { return 0.001; }
double bump_maturity(double t) { return std::min(1.0 / 365.0, t * 0.25); }
double parameter_floor(int greek) { return greek == MPC_GREEK_RHO ? -1.0 : 2.2250738585072014e-308; }

// The parameter a bump moves.
enum Param { P_S0, P_SIGMA, P_R, P_T, P_SPOT0, P_SPOT1, P_SIGMA0, P_SIGMA1, P_SQRT_V0 };

struct Bump {
  int greek;
  Param param;
  double center, bump;
  bool reverse;  // theta: minus the maturity derivative
};

void set_param(mpc_request_t& q, Param p, double x) {
  switch (p) {
    case P_S0: q.s0 = x; break;
    case P_SIGMA: q.sigma = x; break;
    case P_R: q.r = x; break;
    case P_T: q.t = x; break;
    case P_SPOT0: q.spots[0] = x; break;
    case P_SPOT1: q.spots[1] = x; break;
    case P_SIGMA0: q.sigmas[0] = x; break;
    case P_SIGMA1: q.sigmas[1] = x; break;
    case P_SQRT_V0: {  // Heston vega moves sqrt(v0), theta fixed (cpu.rs:4610-4626)
      const double c = std::max(x, 0.0);
      q.v0 = c * c;
      break;
    }
  }
}

// The Greeks each workload reports (cpu.rs:4047-4356, 4409-4668); empty when
// the reference has no Greeks for it (Merton, LSM, MLMC).
std::vector<Bump> bumps_of(const mpc_request_t& r) {
  std::vector<Bump> v;
  const Bump rho{MPC_GREEK_RHO, P_R, r.r, bump_rate(), false};
  const Bump theta{MPC_GREEK_THETA, P_T, r.t, bump_maturity(r.t), true};
  switch (r.workload) {
    case MPC_WORKLOAD_BASKET_CALL:
      v = {{MPC_GREEK_DELTA, P_SPOT0, r.spots[0], bump_spot(r.spots[0]), false},
           {MPC_GREEK_DELTA2, P_SPOT1, r.spots[1], bump_spot(r.spots[1]), false},
           {MPC_GREEK_VEGA, P_SIGMA0, r.sigmas[0], bump_volatility(r.sigmas[0]), false},
           {MPC_GREEK_VEGA2, P_SIGMA1, r.sigmas[1], bump_volatility(r.sigmas[1]), false},
           rho,
           theta};
      return v;
    case MPC_WORKLOAD_EUROPEAN_CALL:
      if (r.model == MPC_MODEL_HESTON) {
        const double sv = std::sqrt(std::max(r.v0, 0.0));
        v = {{MPC_GREEK_DELTA, P_S0, r.s0, bump_spot(r.s0), false},
             {MPC_GREEK_VEGA, P_SQRT_V0, sv, bump_volatility(sv), false},
             rho,
             theta};
        return v;
      }
      [[fallthrough]];
    case MPC_WORKLOAD_ARITHMETIC_ASIAN_CALL:
    case MPC_WORKLOAD_DOWN_AND_OUT_CALL:
    case MPC_WORKLOAD_UP_AND_OUT_CALL:
    case MPC_WORKLOAD_LOOKBACK_CALL:
      if (r.model != MPC_MODEL_GBM) return v;
      v = {{MPC_GREEK_DELTA, P_S0, r.s0, bump_spot(r.s0), false},
           {MPC_GREEK_VEGA, P_SIGMA, r.sigma, bump_volatility(r.sigma), false},
           rho,
           theta};
      return v;
    default:
      return v;
  }
}

// push_bump_estimate (cpu.rs:4938-4983) for one bump from the priced legs.
void bump_estimate(const Bump& b, const mpc_result_t& base, const mpc_result_t& up, const mpc_result_t& down,
                   mpc_greek_estimate_t* e) {
  const double lo = std::max(b.center - b.bump, parameter_floor(b.greek));
  const double eff = ((b.center + b.bump) - lo) * 0.5;
  const double raw = eff > 0.0 ? (up.price - down.price) / (2.0 * eff) : 0.0;
  e->greek = b.greek;
  e->estimator = MPC_GREEKS_BUMP_AND_REVALUE;
  e->value = b.reverse ? -raw : raw;
  e->stderr = eff > 0.0 ? std::sqrt(up.stderr * up.stderr + down.stderr * down.stderr) / (2.0 * eff) : 0.0;
  e->bump_size = eff;
  e->base_price = base.price;
  e->bumped_up_price = up.price;
  e->bumped_down_price = down.price;
}

// MomentAccumulator::mean_stderr (cpu.rs:4846-4869): (n - 1) sample variance.
void mean_stderr(double sum, double sq, uint64_t count, double* mean, double* se) {
  if (count == 0) {
    *mean = *se = 0.0;
    return;
  }
  const double n = double(count);
  *mean = sum / n;
  const double var = count > 1 ? std::max((sq - sum * sum / n) / (n - 1.0), 0.0) : 0.0;
  *se = std::sqrt(var / n);
}

// Whether the legs of a bump report can share their normals in one
// scenario launch: FP32 path, a family the scenario kernel runs (any
// technique; a basket with the standard one), a sampler whose normals depend
// only on (point, dimension).
bool scenario_eligible(const Prepared& p, const mpc_request_t& r, size_t legs) {
  if (r.precision != MPC_PRECISION_FP32_PATH) return false;
  if (p.q.bridge) return false;
  if (p.family == FAM_BASKET) {
    if (legs > size_t(kBasketScen) || r.technique != MPC_TECHNIQUE_STANDARD) return false;
  } else {
    if (legs > size_t(kMaxScen)) return false;
    if (p.family != FAM_GBM_STEP && p.family != FAM_GBM_TERMINAL && p.family != FAM_HESTON) return false;
  }
  return p.sampler == SMP_XORSHIFT || p.sampler == SMP_SOBOL || p.sampler == SMP_COUNTER;
}

// Per-leg constants of the basket scenario kernel; legs past the last are
// copies of the base leg (computed, never reported).
BasketScen basket_legs(const std::vector<Prepared>& preps) {
  BasketScen b{};
  for (int s = 0; s < kBasketScen; ++s) {
    const DevReq& q = preps[s < int(preps.size()) ? s : 0].q;
    for (uint32_t a = 0; a < q.n_assets; ++a) {
      b.log_drift[s][a] = float(q.b_drift[a] * double(q.n_steps));
      b.step_vol[s][a] = float(q.b_vol[a]);
      b.wspot[s][a] = float(q.weights[a] * q.spots[a]);
    }
    b.discount[s] = float(q.discount);
  }
  return b;
}

// Prices every leg (same seed, same dimensions) in one scenario launch.
int run_scenario_legs(mpc_context* ctx, const std::vector<mpc_request_t>& legs, std::vector<mpc_result_t>& res) {
  std::vector<Prepared> preps(legs.size());
  std::string msg;
  for (size_t i = 0; i < legs.size(); ++i) {
    const int st = prepare(ctx, legs[i], &preps[i], &msg);
    if (st != MPC_OK) return fail(ctx, st, msg);
  }
  const Prepared& base = preps[0];
  const int n_scen = int(legs.size());
  const bool basket = base.family == FAM_BASKET;
  const int slots = basket ? kBasketScen : kMaxScen;  // legs per tile partial
  const int technique = legs[0].technique;
  const int nm = basket ? 2 : scenario_moments(technique);  // moments per leg
  float scen[kScenFields * kMaxScen];
  for (int s = 0; s < kMaxScen && !basket; ++s) {
    const DevReq& q = preps[s < n_scen ? s : 0].q;
    float f[kScenFields];
    if (base.family == FAM_HESTON) {
      const float v[kScenFields] = {float(q.log_s0), float(q.v0), float(q.rate), float(q.dt), float(q.sqrt_dt),
                                    float(q.discount)};
      std::memcpy(f, v, sizeof(f));
    } else {
      const bool ko = (q.workload == MPC_WORKLOAD_DOWN_AND_OUT_CALL && q.s0 <= q.barrier) ||
                      (q.workload == MPC_WORKLOAD_UP_AND_OUT_CALL && q.s0 >= q.barrier);
      const float v[kScenFields] = {float(q.log_s0),   float(q.s0),       float(q.drift_dt),
                                    float(q.vol_dt),   float(q.discount), ko ? 1.0f : 0.0f};
      std::memcpy(f, v, sizeof(f));
    }
    for (int k = 0; k < kScenFields; ++k) scen[k * kMaxScen + s] = f[k];
  }
  DevReq q = base.q;
  q.n_scen = uint32_t(n_scen);
  q.tile_units = 256;
  const uint64_t n_tiles = (q.n_units + q.tile_units - 1) / q.tile_units;
  if (n_tiles > (1ull << 31)) return fail(ctx, MPC_E_UNSUPPORTED, "too many tiles for one scenario launch");
  q.n_tiles = uint32_t(n_tiles);
  // device layout: descriptor | leg parameters | partials | moments | counters (done, tile counter)
  const size_t o_scen = 256 * ((sizeof(DevReq) + 255) / 256);
  const size_t o_part = o_scen + 256;
  const size_t o_mom = o_part + ((n_tiles * slots * nm * sizeof(double) + 255) / 256) * 256;
  const size_t o_cnt = o_mom + ((size_t(slots) * nm * sizeof(double) + 255) / 256) * 256;
  void* d = nullptr;
  int st = scratch(ctx, "scenarios", o_cnt + 256, &d);
  if (st != MPC_OK) return st;
  uint8_t* base_ptr = static_cast<uint8_t*>(d);
  q.scen = reinterpret_cast<const float*>(base_ptr + o_scen);
  q.partials = reinterpret_cast<double*>(base_ptr + o_part);
  q.moments = reinterpret_cast<double*>(base_ptr + o_mom);
  q.tiles_done = reinterpret_cast<uint32_t*>(base_ptr + o_cnt);
  q.per_unit = nullptr;
  uint32_t* counter = q.tiles_done + 1;
  double host_mom[kBasketScen * 5];
  static_assert(kBasketScen >= kMaxScen, "moments buffer");
  auto fin = [&](cudaError_t e, const char* what) { return e == cudaSuccess ? MPC_OK : cuda_fail(ctx, e, what); };
  if ((st = fin(cudaMemsetAsync(q.tiles_done, 0, 2 * sizeof(uint32_t), ctx->stream), "memset counters"))) return st;
  if ((st = fin(cudaMemcpyAsync(base_ptr, &q, sizeof(q), cudaMemcpyHostToDevice, ctx->stream), "descriptor"))) return st;
  if (!basket && (st = fin(cudaMemcpyAsync(base_ptr + o_scen, scen, sizeof(scen), cudaMemcpyHostToDevice, ctx->stream),
                           "leg parameters")))
    return st;
  const int occ = std::max(1, basket ? basket_scenario_max_blocks_per_sm(base.sampler)
                                     : scenario_max_blocks_per_sm(base.family, base.sampler, technique));
  const int grid = int(std::min<uint64_t>(n_tiles, uint64_t(ctx->sm_count) * occ));
  if ((st = fin(cudaEventRecord(ctx->ev_start, ctx->stream), "event"))) return st;
  const DevReq* d_req = reinterpret_cast<const DevReq*>(base_ptr);
  const cudaError_t launched =
      basket ? launch_basket_scenarios(d_req, q.n_tiles, counter, base.sampler, basket_legs(preps), ctx->tabs, grid,
                                       ctx->stream)
             : launch_scenarios(d_req, q.n_tiles, counter, base.family, base.sampler, technique, ctx->tabs, grid,
                                ctx->stream);
  if ((st = fin(launched, "scenario kernel"))) return st;
  if ((st = fin(cudaEventRecord(ctx->ev_stop, ctx->stream), "event"))) return st;
  if ((st = fin(cudaMemcpyAsync(host_mom, q.moments, size_t(slots) * nm * sizeof(double), cudaMemcpyDeviceToHost,
                                ctx->stream),
                "moments")))
    return st;
  if ((st = fin(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize"))) return st;
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
  ctx->last_ms = ms;
  res.assign(legs.size(), mpc_result_t{});
  for (int s = 0; s < n_scen; ++s) {
    // the fused path's moments layout (count, sum p, sum p^2, sum c, sum c^2,
    // sum p c), summarised by the request's own estimator (cpu.rs:7641-7771)
    double m[MPC_MOMENTS] = {double(q.n_units), 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < nm; ++k) m[1 + k] = host_mom[s * nm + k];
    summarize_moments(preps[s], m, &res[s]);
    res[s].path_steps = preps[s].path_steps;
    res[s].runtime_ms = ms;
    res[s].status = MPC_OK;
  }
  return MPC_OK;
}

}  // namespace
}  // namespace mpc

using namespace mpc;

#define GREEKS_CUDA(call)                                             \
  do {                                                                \
    cudaError_t _e = (call);                                          \
    if (_e != cudaSuccess) return finish(cuda_fail(ctx, _e, #call)); \
  } while (0)

extern "C" int mpc_greeks(mpc_context_t* ctx, const mpc_request_t* req, int estimator, mpc_greek_report_t* out) {
  if (!ctx || !req || !out) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  const mpc_request_t& r = *req;
  std::memset(out, 0, sizeof(*out));
  out->workload = r.workload;
  out->estimator = estimator;
  out->paths = r.n_paths;
  out->steps = r.workload == MPC_WORKLOAD_BASKET_CALL ? 2u : r.n_steps;
  out->seed = r.seed;
  auto finish = [&](int st) {
    out->status = st;
    return st;
  };
  if (estimator < MPC_GREEKS_BUMP_AND_REVALUE || estimator > MPC_GREEKS_LIKELIHOOD_RATIO)
    return finish(fail(ctx, MPC_E_INVALID_CONFIG, "unknown Greek estimator"));
  const std::vector<Bump> bumps = bumps_of(r);
  if (bumps.empty())
    return finish(fail(ctx, MPC_E_UNSUPPORTED, "no Greeks for this workload/model (the reference offers none)"));

  if (estimator == MPC_GREEKS_BUMP_AND_REVALUE) {
    // base, then (up, down) per Greek, every request with the same seed
    std::vector<mpc_request_t> reqs(1 + 2 * bumps.size(), r);
    for (size_t i = 0; i < bumps.size(); ++i) {
      const Bump& b = bumps[i];
      set_param(reqs[1 + 2 * i], b.param, b.center + b.bump);
      set_param(reqs[2 + 2 * i], b.param, std::max(b.center - b.bump, parameter_floor(b.greek)));
    }
    std::vector<mpc_result_t> res(reqs.size());
    Prepared base_prep;
    std::string msg;
    int st = prepare(ctx, r, &base_prep, &msg);
    if (st != MPC_OK) return finish(fail(ctx, st, msg));
    if (scenario_eligible(base_prep, r, reqs.size()))  // all legs share each normal: one launch
      st = run_scenario_legs(ctx, reqs, res);
    else
      st = mpc_price_batch(ctx, reqs.data(), reqs.size(), res.data());
    out->runtime_ms = ctx->last_ms;
    if (st != MPC_OK) return finish(st);
    out->base_price = res[0].price;
    out->base_stderr = res[0].stderr;
    for (size_t i = 0; i < bumps.size(); ++i)
      bump_estimate(bumps[i], res[0], res[1 + 2 * i], res[2 + 2 * i], &out->estimates[out->n_estimates++]);
    return finish(MPC_OK);
  }

  // single-pass estimators: the base price is the request's own price
  mpc_result_t base;
  int st = mpc_price(ctx, req, &base);
  if (st != MPC_OK) return finish(st);
  double total_ms = ctx->last_ms;
  out->base_price = base.price;
  out->base_stderr = base.stderr;
  const bool terminal_gbm_call = r.workload == MPC_WORKLOAD_EUROPEAN_CALL && r.model == MPC_MODEL_GBM;
  if (!terminal_gbm_call) {  // unsupported_greek_report (cpu.rs:4917-4936)
    out->warnings |= MPC_GREEK_WARN_ESTIMATOR_UNSUPPORTED;
    out->runtime_ms = total_ms;
    return finish(MPC_OK);
  }
  if (!(r.s0 > 0.0) || !(r.sigma > 0.0) || !(r.t > 0.0))  // cpu.rs:4671-4674
    return finish(fail(ctx, MPC_E_INVALID_CONFIG, "single-pass Greeks need s0 > 0, sigma > 0 and t > 0"));
  GreekArgs a{};
  a.seed = r.seed;
  a.n_paths = r.n_paths;
  a.s0 = r.s0;
  a.k = r.k;
  a.r = r.r;
  a.sigma = r.sigma;
  a.t = r.t;
  a.sqrt_t = std::sqrt(r.t);
  a.drift_t = (r.r - 0.5 * r.sigma * r.sigma) * r.t;
  a.vol_t = r.sigma * a.sqrt_t;
  a.discount = std::exp(-r.r * r.t);
  a.estimator = estimator;
  a.fp64 = r.precision == MPC_PRECISION_FP64_PLAIN ? 1 : 0;
  const uint64_t want = (r.n_paths + 255) / 256;
  const uint32_t grid = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(want, uint64_t(ctx->sm_count) * 8)));
  void* d = nullptr;
  // partials [grid][8] | totals [8] | counter
  if ((st = scratch(ctx, "greeks", (size_t(grid) * 8 + 8) * sizeof(double) + 64, &d)) != MPC_OK) return finish(st);
  a.partials = static_cast<double*>(d);
  a.out = a.partials + size_t(grid) * 8;
  a.done = reinterpret_cast<unsigned*>(a.out + 8);
  double host[8];
  GREEKS_CUDA(cudaMemsetAsync(a.done, 0, sizeof(unsigned), ctx->stream));
  GREEKS_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
  cudaError_t e = launch_greeks_single_pass(a, grid, ctx->tabs, ctx->stream);
  if (e != cudaSuccess) return finish(cuda_fail(ctx, e, "single-pass Greeks kernel"));
  GREEKS_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
  GREEKS_CUDA(cudaMemcpyAsync(host, a.out, sizeof(host), cudaMemcpyDeviceToHost, ctx->stream));
  GREEKS_CUDA(cudaStreamSynchronize(ctx->stream));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
  out->runtime_ms = total_ms + ms;
  const int names[4] = {MPC_GREEK_DELTA, MPC_GREEK_VEGA, MPC_GREEK_RHO, MPC_GREEK_THETA};
  const int count = estimator == MPC_GREEKS_PATHWISE ? 4 : 3;
  for (int g = 0; g < count; ++g) {
    mpc_greek_estimate_t& est = out->estimates[out->n_estimates++];
    est.greek = names[g];
    est.estimator = estimator;
    mean_stderr(host[2 * g], host[2 * g + 1], r.n_paths, &est.value, &est.stderr);
    est.base_price = base.price;
  }
  if (r.sampling != MPC_SAMPLING_PSEUDORANDOM) out->warnings |= MPC_GREEK_WARN_PSEUDORANDOM_SHOCKS;
  if (r.technique != MPC_TECHNIQUE_STANDARD) out->warnings |= MPC_GREEK_WARN_TECHNIQUE_IGNORED;
  return finish(MPC_OK);
}

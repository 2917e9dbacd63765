// mpc_runtime.h -- internal host runtime shared by mpc_runtime.cu and mpc_server.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/montepath_cuda.h"
#include "mpc_launch.h"
#include "mpc_types.h"

namespace mpc {

// A growable device allocation charged against the context's HBM budget.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

// Launch shape chosen for one request (autotuner output).
struct Shape {
  uint32_t block = 256;
  uint32_t ppt = 1;  // units per thread per tile
};

// Host view of a request prepared for the device.
struct Prepared {
  DevReq q{};
  int sampler = 0;
  int family = 0;
  bool plain = false;     // FP64 plain pipeline
  bool lsm = false;
  bool mlmc = false;
  uint32_t ppt_hint = 0;  // request's paths_per_thread (0: autotuner)
  uint32_t block_hint = 0;  // request's block_size (0: autotuner)
  double cv_expectation = 0.0;
  std::vector<uint32_t> halton_primes;
  std::vector<double> halton_shifts;
  std::vector<LhsDim> lhs;
  std::vector<double> bridge_ops;
  std::vector<uint32_t> bridge_events;
  uint64_t path_steps = 0;
};

struct Autotuner {
  std::mutex mu;
  std::map<uint64_t, Shape> cache;     // key: family | sampler | steps bucket | size bucket | block
  std::map<uint64_t, uint32_t> block;  // measured block size per family | sampler | steps bucket
  uint64_t hits = 0, misses = 0, measured = 0;
  uint32_t default_block = 256;        // block of untuned kinds (context option)
};

}  // namespace mpc

struct mpc_context {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  // Concurrent group launches of a batch: group 0 runs on `stream`, group g
  // on side[(g - 1) % kSideStreams], forked after the tile counters are reset
  // and joined before the moments are copied out, so one family's blocks
  // start on the SMs another family's tail leaves idle.
  static constexpr int kSideStreams = 3;
  cudaStream_t side[kSideStreams] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kSideStreams] = {};
  mpc::DeviceTables tabs{};
  void* d_sobol = nullptr;
  void* d_jump = nullptr;
  uint64_t budget = 0;
  uint64_t live_bytes = 0;
  uint64_t peak_bytes = 0;
  std::string last_error;
  std::recursive_mutex mu;
  double last_ms = 0.0;
  uint64_t last_launches = 0;
  uint64_t last_h2d = 0, last_d2h = 0;
  std::map<std::string, mpc::DevBuf> bufs;  // named scratch buffers
  void* pinned = nullptr;                   // pinned staging for descriptors and results
  size_t pinned_bytes = 0;
  mpc::Autotuner tuner;
  // CUDA graph of the fused batch sequence (copies in, launches, copy out):
  // captured when the same batch shape comes twice in a row, replayed while
  // it repeats.  The key holds every address, size and launch shape the graph
  // bakes in.
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<uint64_t> graph_key;      // key of graph_exec
  std::vector<uint64_t> last_batch_key;  // key of the previous fused batch
  uint64_t graph_kernels = 0;           // kernels in graph_exec
  uint64_t graph_replays = 0;
  // Cost-model rates measured on this device by mpc_calibrate_cost, units
  // per second as [row][fp32, fp64][sampler column]; empty until then.
  std::vector<double> cost_rates;
  std::vector<double> cost_fixed;  // calibrated per-call intercepts in ms, same layout (terminal GBM row)
  // At most this many blocks per LSM launch (0 = the device's co-resident
  // capacity): set by a device-loop server that keeps only some SMs free.
  uint32_t lsm_block_cap = 0;
};

namespace mpc {

int fail(mpc_context* ctx, int status, const std::string& msg);
int cuda_fail(mpc_context* ctx, cudaError_t err, const char* what);
// Returns a device buffer of at least `bytes` for `name`, growing it under the budget.
int scratch(mpc_context* ctx, const std::string& name, size_t bytes, void** out);
int validate(const mpc_request_t& r, std::string* msg);
int prepare(mpc_context* ctx, const mpc_request_t& r, Prepared* p, std::string* msg);
uint64_t estimate_bytes(const mpc_request_t& r);
// The reference's terminal pseudorandom Merton, priced by the stream replay
// (its own launch sequence, not a fused tile family).
bool merton_stream_request(const mpc_request_t& r);
Shape choose_shape(mpc_context* ctx, const Prepared& p);
// Key of the measured block size of a request kind.
uint64_t block_key(const Prepared& p);
void summarize_moments(const Prepared& p, const double* m, mpc_result_t* out);
// Longstaff-Schwartz and MLMC requests of a batch, packed into shared launches.
int run_lsm_batch(mpc_context* ctx, const std::vector<const mpc_request_t*>& reqs,
                  const std::vector<mpc_result_t*>& outs);
int run_mlmc_batch(mpc_context* ctx, const std::vector<const mpc_request_t*>& reqs,
                   const std::vector<mpc_result_t*>& outs);
// MLMC pieces shared by the batch runner and the serving loop: fine steps of
// a level, one level as a fused request, replicates of a request, the
// tolerance solver's allocation from pilot variances and the estimator from
// the main-phase level results (means and population variances, replicate by
// replicate, level by level).
uint64_t fine_steps(const mpc_request_t& r, uint32_t level);
void level_request(const mpc_request_t& r, uint64_t seed, uint32_t level, uint64_t paths, Prepared* p);
uint64_t mlmc_replicates(const mpc_request_t& r);
void mlmc_allocate(mpc_request_t& r, const double* pilot_var, mpc_result_t* out);
void mlmc_finish(const mpc_request_t& r, const double* mean, double* var, double device_ms, mpc_result_t* out);
// Host copies of the device lookup tables: Sobol nibble tables [256][8][16]
// and xorshift64* jump-ahead nibble tables [64][16][16].
void build_tables(std::vector<uint32_t>& sob, std::vector<uint64_t>& jump);
// Nibble table [16][16] of the xorshift64* jump by k draws (for gf2_apply).
std::vector<uint64_t> xorshift_jump_table(uint64_t k);
// Fused FP32 requests: one persistent launch per (sampler, family) group on the context stream.
int run_fused(mpc_context* ctx, std::vector<Prepared*>& reqs, std::vector<mpc_result_t*>& outs,
              double* per_unit_host, uint64_t per_unit_cap);

}  // namespace mpc

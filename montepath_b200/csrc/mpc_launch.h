// mpc_launch.h -- host-side launch wrappers of the kernels in mpc_kernels.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/montepath_cuda.h"
#include "mpc_types.h"

namespace mpc {

struct DeviceTables {
  const uint32_t* sobol;  // [256][8][16] nibble tables
  const uint64_t* jump;   // [64][16][16] xorshift jump nibble tables
};

// Fused FP32 path: one persistent launch over a tile work list.  All
// requests in `reqs` must share `sampler`; `family` < 0 lets each tile switch
// on its request's family (mixed batches).
cudaError_t launch_fused(const DevReq* d_reqs, const Tile* d_tiles, uint32_t n_tiles, uint32_t* d_tile_counter,
                         int family, int sampler, const DeviceTables& tabs, int grid, int block,
                         cudaStream_t stream);
int fused_max_blocks_per_sm(int family, int sampler, int block);

// Resident serving loop (mpc_server mode 2): one persistent launch that
// takes pricing work as the host publishes it.  The host copies entries into
// a ring in device memory and then advances `tail` (the doorbell, also in
// device memory, copied after the entries on the same stream, so the loop's
// polls stay in L2 and never cross PCIe); every block claims tiles
// of the oldest entry that still has some (a 64-bit compare-and-swap on the
// slot's claim word, generation << 32 | next tile, so a claim can never land
// on a slot's later request), runs them through the fused tile body of the
// entry's sampler (xorshift, counter hash or Sobol; any family), and the
// block that finishes a request's last tile writes its moments into mapped
// host memory and then the request's generation into done[slot].  Blocks
// leave when the host sets stop or pause, or after idle_ns without work;
// every wait is a bounded poll.
struct LoopEntry {
  uint32_t slot, gen, n_tiles, pos;  // pos: absolute ring position (detects a reused ring entry)
};
struct LoopArgs {
  const DevReq* slots;           // device [max_slots]: slot descriptors
  unsigned long long* claim;     // device [max_slots]: gen << 32 | next tile
  const LoopEntry* ring;         // device [ring_cap]
  const uint32_t* doorbell;      // device, 16-byte aligned: [0] tail (entries published), [1] stop, [2] pause
  uint32_t* done;                // mapped host [max_slots]: generation finished last
  uint32_t ring_cap, max_slots;
  uint64_t idle_ns;
  uint32_t reserve_sms;          // blocks that start on an SM with %smid below this leave at once
  uint32_t _pad;
};
cudaError_t launch_serve_loop(const LoopArgs& a, const DeviceTables& tabs, int grid, cudaStream_t stream);
int serve_loop_blocks_per_sm();

// FP64 plain path: materialise samples, simulate into a payoff buffer, reduce.
cudaError_t launch_plain_generate(const DevReq& q, double* d_buf, int sampler, const DeviceTables& tabs,
                                  cudaStream_t stream);
cudaError_t launch_plain_simulate(const DevReq& q, const DevReq* d_req, const double* d_buf, double* d_payoff,
                                  double* d_control, cudaStream_t stream);
cudaError_t launch_plain_reduce(const DevReq* d_req, const double* d_payoff, const double* d_control,
                                uint64_t n_units, uint32_t n_tiles, cudaStream_t stream);

// Reference kernel contract mc_cuda_european_call_stepwise_v1.
cudaError_t launch_european_call_stepwise_v1(const double* normals, double* payoffs, int32_t n_paths,
                                             int32_t n_steps, double log_s0, double strike, double drift_dt,
                                             double vol_dt, double discount, cudaStream_t stream);

// Longstaff-Schwartz: one cooperative launch (paths, backward induction, estimator).
struct LsmArgs {
  uint64_t n_paths;
  uint32_t n_steps, n_sched, degree, sampler;
  uint64_t seed;
  uint32_t seed32, fp64;
  double s0, k, drift, vol, disc_step;
  const uint32_t* sched;     // exercise dates (ascending, ends with n_steps)
  const double* disc_pow;    // disc_step^j, j = 0..n_steps
  const uint64_t* stride_jump;  // pseudorandom sampler: nibble table [16][16] of T^(grid threads x n_steps),
                                // the stream jump between a thread's successive paths
  void* paths;               // [n_steps][n_paths] float or double
  double* partials;          // [rounds][grid][16], every slot empty (all bits set) at launch
  double* final_partials;    // [grid][4]
  double* out;               // [8]: n, sum, sumsq, early, maturity, regressions, -, -
  unsigned* barrier;         // counter area (kLsmCounterBytes)
  unsigned* done;            // last-block counter
  int* error;                // first failure: kLsmErr* code (0 = none)
  unsigned long long* diag;  // offending index of a failed self-check
  uint64_t timeout_ns;
  uint32_t block_first;      // this job's blocks in the batched launch
  uint32_t n_blocks;
  uint64_t paths_len;        // elements allocated for `paths`
  uint32_t partials_len;     // elements allocated for `partials`
  uint32_t final_len;        // elements allocated for `final_partials`
};
// Failure codes written to LsmArgs::error.  Every indexed global or shared
// access of the kernel is checked against its allocation; a failed check
// records its code and index, skips the access and makes every block of the
// job leave at the next barrier.
enum : int {
  kLsmErrTimeout = 1,
  kLsmErrPaths = 2,
  kLsmErrPartials = 3,
  kLsmErrFinal = 4,
  kLsmErrSched = 5,
  kLsmErrDisc = 6,
  kLsmErrJob = 7,
  kLsmErrCoverage = 8,
};
// Several LSM requests in one cooperative launch: job j owns blocks
// [block_first, block_first + n_blocks) and synchronises only them.  All jobs
// of a launch share precision (fp64) and sampler.
cudaError_t launch_lsm_batch(const LsmArgs* d_jobs, uint32_t n_jobs, uint32_t total_blocks, int fp64, int sampler,
                             const DeviceTables& tabs, cudaStream_t stream);
// Co-resident LSM blocks on the device for (fp64, sampler); 0 if the kernel cannot launch.
uint32_t lsm_capacity(int fp64, int sampler);
constexpr uint32_t kLsmPathsPerThreadMax = 8;
constexpr uint32_t kLsmThreads = 512;
// Counter area of an LSM job (zeroed per launch): the last-block counter at
// uint 4, the error code at uint 8 and its index at uint 10.
constexpr size_t kLsmCounterBytes = 256;

// Bump-and-revalue legs sharing every normal: one request d_req (GBM step,
// GBM terminal or Heston; xorshift, Sobol or counter-hash samples; any
// technique) whose q.scen holds the legs' parameters; with NM =
// scenario_moments(technique), q.partials must hold [n_tiles][kMaxScen][NM]
// doubles and q.moments [kMaxScen][NM]: sum p, sum p^2 (pair averages for
// antithetic requests), then for control variates sum c, sum c^2, sum p c.
constexpr int scenario_moments(int technique) { return technique == MPC_TECHNIQUE_CONTROL_VARIATE ? 5 : 2; }
cudaError_t launch_scenarios(const DevReq* d_req, uint32_t n_tiles, uint32_t* d_counter, int family, int sampler,
                             int technique, const DeviceTables& tabs, int grid, cudaStream_t stream);
int scenario_max_blocks_per_sm(int family, int sampler, int technique);

// Basket bump legs sharing every normal: one basket request d_req
// (xorshift, Sobol or counter-hash samples); q.partials must hold
// [n_tiles][kBasketScen][2] doubles and q.moments [kBasketScen][2].
cudaError_t launch_basket_scenarios(const DevReq* d_req, uint32_t n_tiles, uint32_t* d_counter, int sampler,
                                    const BasketScen& legs, const DeviceTables& tabs, int grid, cudaStream_t stream);
int basket_scenario_max_blocks_per_sm(int sampler);

// Single-pass Greek estimators of the terminal-GBM European call
// (pathwise: delta, vega, rho, theta; likelihood ratio: delta, vega, rho)
// over the pseudorandom terminal shocks of one MonteCarloRng stream.
struct GreekArgs {
  uint64_t seed, n_paths;
  double s0, k, r, sigma, t;
  double sqrt_t, drift_t, vol_t, discount;
  int32_t estimator;  // mpc_greek_estimator_t (PATHWISE or LIKELIHOOD_RATIO)
  int32_t fp64;       // 1: FP64 shocks and arithmetic; 0: FP32 path arithmetic
  double* partials;   // [grid][8]: sum and sum of squares of 4 estimators
  double* out;        // [8] totals in block order
  unsigned* done;     // last-block counter (zero before the launch, zero after)
};
cudaError_t launch_greeks_single_pass(const GreekArgs& a, uint32_t grid, const DeviceTables& tabs,
                                      cudaStream_t stream);

// The reference's Merton estimator (terminal, pseudorandom): each chunk's
// sequential MonteCarloRng stream is replayed and the variable number of
// draws per path resolved by a parallel chain over 64-position segments
// (mpc_merton.cu).  Per chunk, qpad stream positions (a multiple of
// kMertonSegment, at least 3 per path plus one spare segment) and n_segs =
// qpad / kMertonSegment - 1 segments.
constexpr uint32_t kMertonSegment = 64;
struct MertonStreamArgs {
  uint64_t n_paths;             // all chunks
  uint32_t n_chunks, cv;        // chunk count (1 = one stream); record controls
  uint64_t chunk_base, chunk_rem;  // the reference's split of n_paths
  uint64_t seed;                // request seed (chunk seeds derived from it)
  uint64_t qpad, n_segs;
  double mean, p0;              // lambda T and exp(-lambda T)
  double log_s0, drift_t, vol_t, jump_mean, jump_vol, k, discount;
  uint64_t* x;                  // [n_chunks][qpad] stream outputs
  uint32_t* bits;               // [n_chunks][qpad / 32] jump bits
  uint16_t* maps;               // [n_chunks][n_segs][9] segment maps
  uint8_t* seg_state;           // [n_chunks][n_segs] entry state
  unsigned long long* seg_before;  // [n_chunks][n_segs] paths before the segment
  uint64_t* starts;             // [n_paths] path start states
  double* payoff;               // [n_paths]
  double* control;              // [n_paths] or null
};
cudaError_t launch_merton_stream(const MertonStreamArgs& a, const DeviceTables& tabs, cudaStream_t stream);

// Device generators for the ABI's sampler entry points.
cudaError_t launch_generate_normals(const DevReq& q, int sampler, int fp32, void* d_out, uint64_t n_points,
                                    uint32_t dims, const DeviceTables& tabs, cudaStream_t stream);
cudaError_t launch_counter_hash(uint32_t seed, uint32_t n_paths, uint32_t n_steps, uint32_t* d_out,
                                cudaStream_t stream);
cudaError_t launch_xorshift(uint64_t seed, uint64_t offset, uint64_t count, uint64_t* d_out,
                            const DeviceTables& tabs, cudaStream_t stream);
cudaError_t launch_flush(void* d_buf, size_t bytes, cudaStream_t stream);

// Kernel launches issued by the wrappers above since process start.
uint64_t kernel_launch_count();
// Adds the kernels of a replayed CUDA graph to the count.
void count_graph_launches(uint64_t kernels);
// Takes back the counts of launches that were only captured into a graph.
void discount_captured_launches(uint64_t kernels);

}  // namespace mpc

// mpc_server.cu -- serving loop of the B200 Monte Carlo backend.
//
// Continuous batching (mode 0): submitted requests wait in a FIFO queue and
// are admitted into device slots while slots and the HBM byte budget allow
// (the analogue of plan_gpu_chunking / estimate_gpu_bytes_per_path,
// crates/mc-core/src/backend/mod.rs:372-405).  Each scheduling wave takes a
// bounded number of tiles from all live FP32-path requests, oldest first,
// and runs them in one persistent launch of the fused kernel; requests that
// arrive meanwhile join the next wave.  A request's tile partials stay
// resident in its slot across waves and the block that completes its last
// tile writes its moments, so a result is the same alone and in any mix.
// LSM and MLMC requests admitted between waves run batched: every LSM
// request in shared cooperative launches, every MLMC request in one pilot
// and one main launch.
//
// Plain mode (mode 1): one request per launch sequence, FP64, strictly FIFO
// -- the baseline continuous batching is compared against.
//
// Device-loop mode (mode 2): a persistent kernel stays resident on the GPU
// and takes work as it arrives (serve_loop_kernel, mpc_kernels.cu).  The
// host thread admits requests under the HBM budget, writes each admitted
// FP32-path request (or MLMC level) into a device slot, publishes it as an
// entry of a ring in mapped host memory and advances the ring's tail; the
// device blocks claim the tiles of the oldest published entries, so a
// request that arrives while others run starts on the next free block, with
// no launch.  The block that finishes a request's last tile writes its
// moments into mapped host memory and then the slot's generation into
// done[slot], which the host thread polls.  MLMC requests run their pilot
// levels, then (after the host's allocation) their main levels, through the
// loop.  Longstaff-Schwartz requests (cooperative launches with grid
// barriers) and requests with per-request sampler tables are batched on the
// host: the loop is paused (its blocks leave after their current tile), the
// batch runs, and the loop is relaunched.  The loop's blocks also leave after
// an idle period; the host relaunches it when work is published again.
//
// Host waiting is on CUDA events, condition variables and short sleeps with
// timeouts; the device loop's waits are bounded polls.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "mpc_device.cuh"
#include "mpc_launch.h"
#include "mpc_runtime.h"

using namespace mpc;

namespace {

using Clock = std::chrono::steady_clock;

struct Ticket {
  uint64_t id = 0;
  mpc_request_t req{};
  mpc_result_t res{};
  Prepared prep;
  int state = 0;  // 0 queued, 1 live, 2 done, 3 cancelled
  int slot = -1;
  uint64_t bytes = 0;
  uint32_t next_tile = 0;
  uint32_t tiles_finished = 0;
  bool uploaded = false;
  double t_enqueue = 0, t_admit = 0, t_complete = 0;
  // device-loop mode
  int route = 0;                  // 1 device loop, 2 host batch
  int phase = 0;                  // MLMC: 1 pilot levels, 2 main levels
  uint32_t jobs_left = 0;         // loop jobs of the current phase not yet finished
  mpc_request_t work{};           // MLMC: the request with the solver's allocation
  std::vector<double> lvl_mean, lvl_var;
  double t_batch = 0;             // host batch: when it joined the batch list
};

// One unit of device-loop work: a fused request, or one MLMC level (of one
// replicate) of a request's current phase.
struct LoopJob {
  uint64_t ticket = 0;
  uint32_t index = 0;  // MLMC: replicate * levels + level (the phase's order)
  Prepared prep;
  int slot = -1;
  uint32_t gen = 0;
};

}  // namespace

struct mpc_server {
  mpc_context* ctx = nullptr;
  mpc_server_options_t opt{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> queue;
  std::map<uint64_t, Ticket> tickets;
  std::vector<int64_t> slot_owner;  // ticket id per slot or -1
  std::vector<uint8_t> dirty;       // slot descriptor changed since the last upload
  uint64_t next_id = 1;
  bool stop = false;
  std::thread worker;
  Clock::time_point t0;
  mpc_server_stats_t stats{};
  std::vector<double> latencies;
  uint64_t live_bytes = 0;
  // device slot table
  DevReq* d_slots = nullptr;
  double* d_partials = nullptr;
  double* d_moments = nullptr;
  uint32_t* d_done = nullptr;
  Tile* d_tiles = nullptr;
  uint32_t* d_counter = nullptr;
  cudaStream_t stream = nullptr;
  DevReq* h_slots = nullptr;  // pinned mirror
  Tile* h_tiles = nullptr;
  double* h_moments = nullptr;
  uint32_t max_tiles_per_slot = 16384;
  uint32_t wave_tiles = 0;
  double busy_ms = 0.0;
  // device-loop mode (mode 2)
  cudaStream_t loop_stream = nullptr, upload_stream = nullptr;
  LoopEntry* h_ring = nullptr;       // pinned staging of new ring entries
  LoopEntry* d_ring = nullptr;       // device ring
  uint32_t* h_ctl = nullptr;         // pinned staging of the doorbell: [0] tail, [1] stop, [2] pause
  uint32_t* d_ctl = nullptr;         // device doorbell
  uint32_t* h_fin = nullptr;         // mapped [slots]: generation finished last per slot
  uint32_t* d_fin = nullptr;
  double* h_mom = nullptr;           // mapped [slots][MPC_MOMENTS]: finished moments
  double* d_mom = nullptr;
  unsigned long long* d_claim = nullptr;  // device [slots]
  unsigned long long* h_claim = nullptr;  // pinned staging
  uint32_t ring_cap = 0, ring_tail = 0, next_gen = 1;
  std::vector<uint32_t> ring_gen;    // generation published at each ring entry
  std::vector<LoopJob> pending;      // waiting for a slot
  std::map<int, LoopJob> running;    // by slot
  std::vector<int> free_slots;
  std::vector<uint64_t> host_batch;  // tickets for the next host batch
  int loop_grid = 0;
  bool loop_launched = false;
  uint64_t live_requests = 0;        // admitted, not finished (at most max_slots)
};

namespace {

double now_ms(const mpc_server* s) {
  return std::chrono::duration<double, std::milli>(Clock::now() - s->t0).count();
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  double pos = q * double(v.size() - 1);
  size_t lo = size_t(pos);
  size_t hi = std::min(lo + 1, v.size() - 1);
  double f = pos - double(lo);
  return v[lo] * (1.0 - f) + v[hi] * f;
}

void complete(mpc_server* s, Ticket& t, int status) {
  if (t.state == 1 && s->live_requests > 0) s->live_requests--;
  t.res.status = status;
  t.t_complete = now_ms(s);
  t.res.t_enqueue_ms = t.t_enqueue;
  t.res.t_admit_ms = t.t_admit;
  t.res.t_complete_ms = t.t_complete;
  t.state = 2;
  if (t.slot >= 0) s->slot_owner[t.slot] = -1;
  t.slot = -1;
  s->live_bytes -= std::min(s->live_bytes, t.bytes);
  t.bytes = 0;
  if (status == MPC_OK) {
    s->stats.completed++;
    s->stats.path_steps += t.res.path_steps;
    s->latencies.push_back(t.t_complete - t.t_enqueue);
  } else {
    s->stats.rejected++;
  }
}

// Tile size of a slot request: the autotuner's shape, doubled until the work
// list fits the slot's partials, up to 2^16 units (a fused tile stays inside
// one 2^16-point Sobol block).  False when the request needs more tiles than
// a slot holds even then (over 2^30 units): it runs as its own batch.
bool shape_for_slot(const mpc_server* s, Prepared* p) {
  Shape sh = choose_shape(s->ctx, *p);
  p->q.tile_units = sh.block * sh.ppt;
  while ((p->q.n_units + p->q.tile_units - 1) / p->q.tile_units > s->max_tiles_per_slot &&
         p->q.tile_units < 65536u)
    p->q.tile_units *= 2;
  p->q.n_tiles = uint32_t((p->q.n_units + p->q.tile_units - 1) / p->q.tile_units);
  return p->q.n_tiles <= s->max_tiles_per_slot;
}

bool fused_eligible(const Ticket& t) {
  return !t.prep.plain && !t.prep.lsm && !t.prep.mlmc && t.req.workload != MPC_WORKLOAD_ASIAN_MLMC &&
         t.req.workload != MPC_WORKLOAD_AMERICAN_PUT && t.req.workload != MPC_WORKLOAD_BERMUDAN_PUT;
}

// Admits queued requests into free slots within the byte budget (FIFO: a
// request that does not fit blocks the ones behind it, so big requests are
// not starved).
void admit(mpc_server* s) {
  while (!s->queue.empty()) {
    Ticket& t = s->tickets[s->queue.front()];
    if (t.state == 3) {
      s->queue.pop_front();
      continue;
    }
    uint64_t need = estimate_bytes(t.req);
    if (need > s->opt.hbm_budget_bytes) {  // can never fit
      s->queue.pop_front();
      t.res.status = MPC_E_OOM_BUDGET;
      complete(s, t, MPC_E_OOM_BUDGET);
      continue;
    }
    if (s->live_bytes + need > s->opt.hbm_budget_bytes) break;
    int slot = -1;
    for (size_t i = 0; i < s->slot_owner.size(); ++i)
      if (s->slot_owner[i] < 0) {
        slot = int(i);
        break;
      }
    if (slot < 0) break;
    s->queue.pop_front();
    s->slot_owner[slot] = int64_t(t.id);
    t.slot = slot;
    t.state = 1;
    t.bytes = need;
    t.t_admit = now_ms(s);
    s->live_bytes += need;
    s->stats.admitted++;
    s->stats.peak_bytes = std::max(s->stats.peak_bytes, s->live_bytes);
  }
}

// LSM and MLMC requests admitted so far run together: all LSM requests in
// shared cooperative launches, all MLMC requests as one pilot launch and one
// main launch.  Returns the number of requests completed.
int run_batched_families(mpc_server* s, std::unique_lock<std::mutex>& lk) {
  std::vector<uint64_t> lsm_ids, mlmc_ids;
  for (size_t i = 0; i < s->slot_owner.size(); ++i) {
    if (s->slot_owner[i] < 0) continue;
    const Ticket& t = s->tickets[uint64_t(s->slot_owner[i])];
    if (fused_eligible(t)) continue;
    if (t.req.workload == MPC_WORKLOAD_ASIAN_MLMC)
      mlmc_ids.push_back(t.id);
    else if (t.req.workload == MPC_WORKLOAD_AMERICAN_PUT || t.req.workload == MPC_WORKLOAD_BERMUDAN_PUT)
      lsm_ids.push_back(t.id);
    else
      mlmc_ids.push_back(t.id);  // structured-table samplers: priced whole through mpc_price_batch
  }
  if (lsm_ids.empty() && mlmc_ids.empty()) return 0;
  std::vector<mpc_request_t> lsm_req, other_req;
  for (uint64_t id : lsm_ids) lsm_req.push_back(s->tickets[id].req);
  for (uint64_t id : mlmc_ids) other_req.push_back(s->tickets[id].req);
  lk.unlock();
  std::vector<mpc_result_t> lsm_res(lsm_req.size()), other_res(other_req.size());
  int st_lsm = MPC_OK, st_other = MPC_OK;
  {
    std::lock_guard<std::recursive_mutex> g(s->ctx->mu);
    cudaSetDevice(s->ctx->device);
    if (!lsm_req.empty()) {
      st_lsm = mpc_price_batch(s->ctx, lsm_req.data(), lsm_req.size(), lsm_res.data());
      s->busy_ms += s->ctx->last_ms;
    }
    if (!other_req.empty()) {
      st_other = mpc_price_batch(s->ctx, other_req.data(), other_req.size(), other_res.data());
      s->busy_ms += s->ctx->last_ms;
    }
  }
  lk.lock();
  for (size_t i = 0; i < lsm_ids.size(); ++i) {
    Ticket& t = s->tickets[lsm_ids[i]];
    t.res = lsm_res[i];
    complete(s, t, lsm_res[i].status != MPC_OK ? lsm_res[i].status : st_lsm);
  }
  for (size_t i = 0; i < mlmc_ids.size(); ++i) {
    Ticket& t = s->tickets[mlmc_ids[i]];
    t.res = other_res[i];
    complete(s, t, other_res[i].status != MPC_OK ? other_res[i].status : st_other);
  }
  s->stats.waves++;
  return int(lsm_ids.size() + mlmc_ids.size());
}

// Runs one wave: up to wave_tiles tiles from live fused requests, oldest first.
int run_wave(mpc_server* s, std::unique_lock<std::mutex>& lk) {
  std::vector<uint64_t> live;
  for (size_t i = 0; i < s->slot_owner.size(); ++i)
    if (s->slot_owner[i] >= 0) live.push_back(uint64_t(s->slot_owner[i]));
  std::sort(live.begin(), live.end());
  // fused wave
  std::vector<Tile> tiles;
  std::vector<uint64_t> finishing;
  uint32_t budget = s->wave_tiles;
  bool any = true;
  while (budget > 0 && any) {
    any = false;
    for (uint64_t id : live) {  // round-robin quanta of 8 tiles, oldest first
      Ticket& t = s->tickets[id];
      if (!fused_eligible(t) || t.next_tile >= t.prep.q.n_tiles) continue;
      uint32_t take = std::min<uint32_t>(std::min<uint32_t>(8, budget), t.prep.q.n_tiles - t.next_tile);
      for (uint32_t j = 0; j < take; ++j) tiles.push_back(Tile{uint32_t(t.slot), t.next_tile + j});
      t.next_tile += take;
      budget -= take;
      any = true;
      if (t.next_tile >= t.prep.q.n_tiles) finishing.push_back(id);
      if (budget == 0) break;
    }
  }
  if (tiles.empty()) return 0;
  // all live fused requests share one sampler per launch: group the wave by sampler
  std::map<int, std::vector<Tile>> by_sampler;
  std::map<int, int> family_of;
  for (const Tile& tl : tiles) {
    const Ticket& t = s->tickets[uint64_t(s->slot_owner[tl.req])];
    by_sampler[t.prep.sampler].push_back(tl);
    auto it = family_of.find(t.prep.sampler);
    if (it == family_of.end())
      family_of[t.prep.sampler] = t.prep.family;
    else if (it->second != t.prep.family)
      it->second = -1;
  }
  size_t off = 0;
  for (auto& kv : by_sampler) {
    std::memcpy(s->h_tiles + off, kv.second.data(), kv.second.size() * sizeof(Tile));
    off += kv.second.size();
  }
  lk.unlock();
  int status = MPC_OK;
  {
    std::lock_guard<std::recursive_mutex> g(s->ctx->mu);
    cudaSetDevice(s->ctx->device);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s->stream);
    for (size_t i = 0; i < s->dirty.size(); ++i)
      if (s->dirty[i]) {
        cudaMemcpyAsync(s->d_slots + i, s->h_slots + i, sizeof(DevReq), cudaMemcpyHostToDevice, s->stream);
        s->dirty[i] = 0;
      }
    cudaMemcpyAsync(s->d_tiles, s->h_tiles, off * sizeof(Tile), cudaMemcpyHostToDevice, s->stream);
    cudaMemsetAsync(s->d_counter, 0, 64 * sizeof(uint32_t), s->stream);
    size_t first = 0, g_idx = 0;
    for (auto& kv : by_sampler) {
      int fam = family_of[kv.first];
      int occ = std::max(1, fused_max_blocks_per_sm(fam, kv.first, 256));
      uint64_t grid = std::min<uint64_t>(uint64_t(s->ctx->sm_count) * occ, kv.second.size());
      cudaError_t e = launch_fused(s->d_slots, s->d_tiles + first, uint32_t(kv.second.size()), s->d_counter + g_idx,
                                   fam, kv.first, s->ctx->tabs, int(std::max<uint64_t>(grid, 1)), 256, s->stream);
      if (e != cudaSuccess) status = MPC_E_CUDA;
      first += kv.second.size();
      ++g_idx;
    }
    cudaMemcpyAsync(s->h_moments, s->d_moments, s->slot_owner.size() * MPC_MOMENTS * sizeof(double),
                    cudaMemcpyDeviceToHost, s->stream);
    cudaEventRecord(e1, s->stream);
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) status = MPC_E_CUDA;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    s->busy_ms += ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  lk.lock();
  s->stats.waves++;
  for (uint64_t id : finishing) {
    Ticket& t = s->tickets[id];
    const double* m = s->h_moments + size_t(t.slot) * MPC_MOMENTS;
    summarize_moments(t.prep, m, &t.res);
    t.res.path_steps = t.prep.path_steps;
    t.res.runtime_ms = 0.0;
    complete(s, t, status);
  }
  return 1;
}

void serve_device_loop(mpc_server* s);

void serve(mpc_server* s) {
  cudaSetDevice(s->ctx->device);
  if (s->opt.mode == 2) {
    serve_device_loop(s);
    return;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    if (s->opt.mode == 1) {
      // plain FIFO: one FP64 request per launch sequence
      if (s->queue.empty()) {
        s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
        continue;
      }
      uint64_t id = s->queue.front();
      s->queue.pop_front();
      Ticket& t = s->tickets[id];
      if (t.state == 3) continue;
      t.state = 1;
      t.t_admit = now_ms(s);
      s->stats.admitted++;
      mpc_request_t req = t.req;
      req.precision = MPC_PRECISION_FP64_PLAIN;
      lk.unlock();
      mpc_result_t res;
      int st;
      {
        std::lock_guard<std::recursive_mutex> g(s->ctx->mu);
        st = mpc_price(s->ctx, &req, &res);
        s->busy_ms += s->ctx->last_ms;
      }
      lk.lock();
      Ticket& t2 = s->tickets[id];
      t2.res = res;
      complete(s, t2, st);
      s->stats.waves++;
      s->cv_done.notify_all();
      continue;
    }
    admit(s);
    // refresh the pinned slot table for newly admitted requests
    for (size_t i = 0; i < s->slot_owner.size(); ++i) {
      if (s->slot_owner[i] < 0) continue;
      Ticket& t = s->tickets[uint64_t(s->slot_owner[i])];
      if (!fused_eligible(t) || t.next_tile != 0 || t.uploaded) continue;
      t.uploaded = true;
      s->dirty[i] = 1;
      DevReq q = t.prep.q;
      q.partials = s->d_partials + i * size_t(s->max_tiles_per_slot) * MPC_MOMENTS;
      q.moments = s->d_moments + i * MPC_MOMENTS;
      q.tiles_done = s->d_done + i;
      q.per_unit = nullptr;
      s->h_slots[i] = q;
    }
    int ran = run_batched_families(s, lk);
    if (ran) s->cv_done.notify_all();
    ran += run_wave(s, lk);
    s->cv_done.notify_all();
    if (!ran) s->cv_work.wait_for(lk, std::chrono::milliseconds(20));
  }
}

// ------------------------------------------------------ device-loop mode ---
bool loop_sampler(const Prepared& p) {
  return p.sampler == SMP_XORSHIFT || p.sampler == SMP_COUNTER || p.sampler == SMP_SOBOL;
}

// A finished loop job: level mean and population variance from its moments.
void level_stats(const double* m, double* mean, double* var) {
  const double n = m[0];
  *mean = m[1] / n;
  *var = (m[2] / n) - (*mean) * (*mean);
}

// Queues the loop jobs of an MLMC phase: pilot levels at pilot_paths_per_level
// (phase 1) or every level of every replicate at the allocation (phase 2).
// False when a level needs more tiles than a slot holds (over 2^30 paths).
bool queue_mlmc_phase(mpc_server* s, Ticket& t, int phase) {
  const mpc_request_t& r = t.work;
  t.phase = phase;
  const uint64_t reps = phase == 1 ? 1 : mlmc_replicates(r);
  const uint32_t L = r.levels;
  t.lvl_mean.assign(reps * L, 0.0);
  t.lvl_var.assign(reps * L, 0.0);
  std::vector<LoopJob> jobs;
  for (uint64_t rep = 0; rep < reps; ++rep) {
    const uint64_t seed = reps > 1 ? derive_chunk_seed(r.seed, rep) : r.seed;
    for (uint32_t l = 0; l < L; ++l) {
      LoopJob j;
      j.ticket = t.id;
      j.index = uint32_t(rep * L + l);
      level_request(r, seed, l, phase == 1 ? r.pilot_paths_per_level : r.paths_per_level[l], &j.prep);
      if (!shape_for_slot(s, &j.prep)) return false;
      jobs.push_back(std::move(j));
    }
  }
  t.jobs_left = uint32_t(jobs.size());
  for (LoopJob& j : jobs) s->pending.push_back(std::move(j));
  return true;
}

// Admission under the HBM budget (FIFO); routes each admitted request to the
// device loop or to the host batch.
void admit_loop(mpc_server* s) {
  while (!s->queue.empty()) {
    Ticket& t = s->tickets[s->queue.front()];
    if (t.state == 3) {
      s->queue.pop_front();
      continue;
    }
    uint64_t need = estimate_bytes(t.req);
    if (need > s->opt.hbm_budget_bytes) {
      s->queue.pop_front();
      complete(s, t, MPC_E_OOM_BUDGET);
      continue;
    }
    if (s->live_bytes + need > s->opt.hbm_budget_bytes) break;
    if (s->live_requests >= s->slot_owner.size()) break;  // max_slots live requests
    s->queue.pop_front();
    t.state = 1;
    t.bytes = need;
    t.t_admit = now_ms(s);
    s->live_bytes += need;
    s->live_requests++;
    s->stats.admitted++;
    s->stats.peak_bytes = std::max(s->stats.peak_bytes, s->live_bytes);
    const bool mlmc = t.req.workload == MPC_WORKLOAD_ASIAN_MLMC;
    const int smp = mlmc ? (t.req.sampling == MPC_SAMPLING_PSEUDORANDOM ? SMP_XORSHIFT
                            : t.req.sampling == MPC_SAMPLING_COUNTER_HASH ? SMP_COUNTER
                            : t.req.sampling == MPC_SAMPLING_SCRAMBLED_SOBOL ? SMP_SOBOL : -1)
                         : t.prep.sampler;
    if (mlmc && t.req.precision == MPC_PRECISION_FP32_PATH && smp >= 0) {
      t.route = 1;
      t.work = t.req;
      if (!queue_mlmc_phase(s, t, t.req.target_stderr > 0.0 ? 1 : 2)) complete(s, t, MPC_E_UNSUPPORTED);
    } else if (!mlmc && fused_eligible(t) && loop_sampler(t.prep)) {
      t.route = 1;
      t.jobs_left = 1;
      LoopJob j;
      j.ticket = t.id;
      j.prep = t.prep;
      s->pending.push_back(std::move(j));
    } else {
      t.route = 2;
      t.t_batch = now_ms(s);
      s->host_batch.push_back(t.id);
    }
  }
}

// Writes pending jobs into free slots and publishes them on the ring.
// Returns the number published.
int publish(mpc_server* s) {
  std::vector<int> slots;
  size_t i = 0;
  while (i < s->pending.size() && !s->free_slots.empty()) {
    // the ring entry about to be reused must belong to a finished job
    const uint32_t pos = s->ring_tail + uint32_t(slots.size());
    const uint32_t old_gen = s->ring_gen[pos % s->ring_cap];
    bool old_live = false;
    for (const auto& kv : s->running)
      if (kv.second.gen == old_gen) old_live = true;
    if (old_live) break;
    LoopJob j = std::move(s->pending[i]);
    ++i;
    const int slot = s->free_slots.back();
    s->free_slots.pop_back();
    j.slot = slot;
    j.gen = s->next_gen++;
    if (s->next_gen == 0) s->next_gen = 1;
    DevReq q = j.prep.q;
    // the loop kernel picks the tile body from the descriptor's sampling (MLMC
    // level descriptors leave it unset)
    q.sampling = j.prep.sampler == SMP_XORSHIFT  ? MPC_SAMPLING_PSEUDORANDOM
                 : j.prep.sampler == SMP_COUNTER ? MPC_SAMPLING_COUNTER_HASH
                                                 : MPC_SAMPLING_SCRAMBLED_SOBOL;
    q.partials = s->d_partials + size_t(slot) * s->max_tiles_per_slot * MPC_MOMENTS;
    q.moments = s->d_mom + size_t(slot) * MPC_MOMENTS;
    q.tiles_done = s->d_done + slot;
    q.per_unit = nullptr;
    s->h_slots[slot] = q;
    s->h_claim[slot] = (unsigned long long)j.gen << 32;
    slots.push_back(slot);
    s->running[slot] = std::move(j);
  }
  s->pending.erase(s->pending.begin(), s->pending.begin() + long(i));
  if (slots.empty()) return 0;
  cudaError_t e = cudaSuccess;
  for (int slot : slots) {
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s->d_slots + slot, s->h_slots + slot, sizeof(DevReq), cudaMemcpyHostToDevice,
                          s->upload_stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s->d_claim + slot, s->h_claim + slot, sizeof(unsigned long long), cudaMemcpyHostToDevice,
                          s->upload_stream);
  }
  // entries after their slots, the doorbell after the entries: one stream, in order
  for (int slot : slots) {
    const LoopJob& j = s->running[slot];
    const uint32_t pos = s->ring_tail++;
    LoopEntry& en = s->h_ring[pos % s->ring_cap];
    en.slot = uint32_t(slot);
    en.gen = j.gen;
    en.n_tiles = j.prep.q.n_tiles;
    en.pos = pos;
    s->ring_gen[pos % s->ring_cap] = j.gen;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s->d_ring + pos % s->ring_cap, &en, sizeof(LoopEntry), cudaMemcpyHostToDevice,
                          s->upload_stream);
  }
  s->h_ctl[0] = s->ring_tail;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_ctl, s->h_ctl, sizeof(uint32_t), cudaMemcpyHostToDevice, s->upload_stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->upload_stream);  // staging reusable
  if (e != cudaSuccess) return -1;
  return int(slots.size());
}

// Writes doorbell word `index` (1 stop, 2 pause) on the device.
void set_control(mpc_server* s, int index, uint32_t value) {
  s->h_ctl[index] = value;
  cudaMemcpyAsync(s->d_ctl + index, s->h_ctl + index, sizeof(uint32_t), cudaMemcpyHostToDevice, s->upload_stream);
  cudaStreamSynchronize(s->upload_stream);
}

// (Re)launches the resident loop when it is not running and work is published.
int ensure_loop(mpc_server* s) {
  if (s->running.empty()) return MPC_OK;
  if (s->loop_launched && cudaStreamQuery(s->loop_stream) == cudaErrorNotReady) return MPC_OK;
  LoopArgs a{};
  a.slots = s->d_slots;
  a.claim = s->d_claim;
  a.ring = s->d_ring;
  a.doorbell = s->d_ctl;
  a.done = s->d_fin;
  a.ring_cap = s->ring_cap;
  a.max_slots = uint32_t(s->slot_owner.size());
  a.idle_ns = 20ull * 1000 * 1000;  // blocks leave after 20 ms without work
  a.reserve_sms = s->opt.reserve_sms;
  cudaError_t e = launch_serve_loop(a, s->ctx->tabs, s->loop_grid, s->loop_stream);
  s->loop_launched = true;
  s->stats.waves++;
  return e == cudaSuccess ? MPC_OK : MPC_E_CUDA;
}

// Finished loop jobs: fused requests complete; MLMC phases advance.
int reap(mpc_server* s) {
  int n = 0;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  for (auto it = s->running.begin(); it != s->running.end();) {
    const int slot = it->first;
    LoopJob& j = it->second;
    if (reinterpret_cast<volatile uint32_t*>(s->h_fin)[slot] != j.gen) {
      ++it;
      continue;
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    double m[MPC_MOMENTS];
    for (int k = 0; k < MPC_MOMENTS; ++k) m[k] = reinterpret_cast<volatile double*>(s->h_mom)[slot * MPC_MOMENTS + k];
    Ticket& t = s->tickets[j.ticket];
    if (t.req.workload == MPC_WORKLOAD_ASIAN_MLMC) {
      level_stats(m, &t.lvl_mean[j.index], &t.lvl_var[j.index]);
      if (--t.jobs_left == 0) {
        if (t.phase == 1) {
          mlmc_allocate(t.work, t.lvl_var.data(), &t.res);
          if (!queue_mlmc_phase(s, t, 2)) complete(s, t, MPC_E_UNSUPPORTED);
        } else {
          const double est = t.res.estimated_stderr;
          const uint32_t met = t.res.target_met, hit = t.res.max_step_updates_hit;
          mlmc_finish(t.work, t.lvl_mean.data(), t.lvl_var.data(), 0.0, &t.res);
          t.res.estimated_stderr = est;
          t.res.target_met = met;
          t.res.max_step_updates_hit = hit;
          complete(s, t, MPC_OK);
        }
      }
    } else {
      summarize_moments(j.prep, m, &t.res);
      t.res.path_steps = j.prep.path_steps;
      t.res.runtime_ms = 0.0;
      complete(s, t, MPC_OK);
    }
    s->free_slots.push_back(slot);
    it = s->running.erase(it);
    ++n;
  }
  return n;
}

// Host batch, beside the running loop: Longstaff-Schwartz requests run one
// cooperative launch each on the SMs the loop keeps free (at most
// reserve_sms blocks per launch); the other requests (per-request sampler
// tables, FP64 plain, the Merton stream replay) are ordinary launches.  An
// LSM request that needs more blocks than the free SMs hold pauses the loop
// (its blocks leave after their current tile) for its own launch.
int run_host_batch(mpc_server* s, std::unique_lock<std::mutex>& lk) {
  std::vector<uint64_t> ids;
  ids.swap(s->host_batch);
  std::vector<std::pair<uint64_t, mpc_request_t>> lsm_fit, lsm_big, other;
  const uint64_t per_block_max = uint64_t(kLsmThreads) * kLsmPathsPerThreadMax;
  for (uint64_t id : ids) {
    const Ticket& t = s->tickets[id];
    if (t.req.workload == MPC_WORKLOAD_AMERICAN_PUT || t.req.workload == MPC_WORKLOAD_BERMUDAN_PUT) {
      const uint64_t need = (t.req.n_paths + per_block_max - 1) / per_block_max;
      (need <= s->opt.reserve_sms ? lsm_fit : lsm_big).push_back({id, t.req});
    } else {
      other.push_back({id, t.req});
    }
  }
  lk.unlock();
  std::vector<std::pair<uint64_t, mpc_result_t>> done;
  auto price = [&](const std::vector<std::pair<uint64_t, mpc_request_t>>& list, bool one_by_one, uint32_t cap) {
    if (list.empty()) return;
    std::lock_guard<std::recursive_mutex> g(s->ctx->mu);
    cudaSetDevice(s->ctx->device);
    s->ctx->lsm_block_cap = cap;
    const size_t step = one_by_one ? 1 : list.size();
    for (size_t i = 0; i < list.size(); i += step) {
      std::vector<mpc_request_t> reqs;
      for (size_t k = i; k < std::min(list.size(), i + step); ++k) reqs.push_back(list[k].second);
      std::vector<mpc_result_t> res(reqs.size());
      int st = mpc_price_batch(s->ctx, reqs.data(), reqs.size(), res.data());
      s->busy_ms += s->ctx->last_ms;
      for (size_t k = 0; k < reqs.size(); ++k) {
        if (res[k].status == MPC_OK && st != MPC_OK) res[k].status = st;
        done.push_back({list[i + k].first, res[k]});
      }
    }
    s->ctx->lsm_block_cap = 0;
  };
  price(other, false, 0);
  price(lsm_fit, true, s->opt.reserve_sms);
  if (!lsm_big.empty()) {
    set_control(s, 2, 1);  // pause: the loop's blocks leave after their current tile
    cudaStreamSynchronize(s->loop_stream);
    set_control(s, 2, 0);
    price(lsm_big, false, 0);
  }
  lk.lock();
  for (auto& d : done) {
    Ticket& t = s->tickets[d.first];
    t.res = d.second;
    complete(s, t, d.second.status);
  }
  if (!lsm_big.empty()) s->loop_launched = false;  // the paused loop has left; relaunch on the next pass
  return int(ids.size());
}

void fail_running(mpc_server* s, int status) {
  for (auto& kv : s->running) {
    Ticket& t = s->tickets[kv.second.ticket];
    if (t.state != 2) complete(s, t, status);
  }
  for (LoopJob& j : s->pending) {
    Ticket& t = s->tickets[j.ticket];
    if (t.state != 2) complete(s, t, status);
  }
  s->running.clear();
  s->pending.clear();
  s->free_slots.clear();
  for (int i = int(s->slot_owner.size()) - 1; i >= 0; --i) s->free_slots.push_back(i);
}

void serve_device_loop(mpc_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    admit_loop(s);
    int progress = 0;
    const int pub = publish(s);
    if (pub < 0 || ensure_loop(s) != MPC_OK) {
      fail_running(s, MPC_E_CUDA);
      progress = 1;
    } else {
      progress += pub;
    }
    const int finished = reap(s);
    progress += finished;
    // host-batched requests run beside the loop as soon as they are admitted
    if (!s->host_batch.empty()) progress += run_host_batch(s, lk);
    if (finished || progress) s->cv_done.notify_all();
    if (progress || !s->running.empty()) {
      // poll the finished flags while work runs; let submitters and waiters
      // take the lock between passes
      lk.unlock();
      std::this_thread::yield();
      lk.lock();
    } else if (s->running.empty() && s->pending.empty() && s->host_batch.empty() && s->queue.empty()) {
      s->cv_work.wait_for(lk, std::chrono::milliseconds(20));
    } else {
      s->cv_work.wait_for(lk, std::chrono::microseconds(20));
    }
  }
  lk.unlock();
  set_control(s, 1, 1);  // stop
  cudaStreamSynchronize(s->loop_stream);
}

}  // namespace

extern "C" {

int mpc_server_start(mpc_context_t* ctx, const mpc_server_options_t* options, mpc_server_t** out) {
  if (!ctx || !out) return MPC_E_INVALID_CONFIG;
  mpc_server* s = new mpc_server();
  s->ctx = ctx;
  if (options) s->opt = *options;
  if (s->opt.hbm_budget_bytes == 0) s->opt.hbm_budget_bytes = 64ull << 30;
  if (s->opt.max_slots == 0) s->opt.max_slots = 256;
  s->opt.max_slots = std::min<uint32_t>(s->opt.max_slots, 1024);
  s->slot_owner.assign(s->opt.max_slots, -1);
  s->dirty.assign(s->opt.max_slots, 0);
  s->t0 = Clock::now();
  cudaSetDevice(ctx->device);
  const size_t slots = s->opt.max_slots;
  int occ = std::max(1, fused_max_blocks_per_sm(FAM_GBM_STEP, SMP_COUNTER, 256));
  s->wave_tiles = s->opt.wave_tiles ? s->opt.wave_tiles : uint32_t(ctx->sm_count * occ * 2);
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&s->d_slots, slots * sizeof(DevReq));
  if (e == cudaSuccess) e = cudaMalloc(&s->d_partials, slots * s->max_tiles_per_slot * MPC_MOMENTS * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&s->d_moments, slots * MPC_MOMENTS * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&s->d_done, slots * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&s->d_tiles, size_t(s->wave_tiles) * sizeof(Tile));
  if (e == cudaSuccess) e = cudaMalloc(&s->d_counter, 64 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaHostAlloc(&s->h_slots, slots * sizeof(DevReq), cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaHostAlloc(&s->h_tiles, size_t(s->wave_tiles) * sizeof(Tile), cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaHostAlloc(&s->h_moments, slots * MPC_MOMENTS * sizeof(double), cudaHostAllocDefault);
  // zeroed on the server stream (non-blocking, so not ordered after the legacy stream)
  if (e == cudaSuccess) e = cudaMemsetAsync(s->d_done, 0, slots * sizeof(uint32_t), s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) {
    ctx->last_error = std::string("server allocation: ") + cudaGetErrorString(e);
    mpc_server_stop(s);
    return e == cudaErrorMemoryAllocation ? MPC_E_OOM_BUDGET : MPC_E_CUDA;
  }
  std::memset(s->h_slots, 0, slots * sizeof(DevReq));
  if (s->opt.mode == 2) {
    if (s->opt.reserve_sms == 0) s->opt.reserve_sms = 32;
    s->opt.reserve_sms = std::min<uint32_t>(s->opt.reserve_sms, uint32_t(ctx->sm_count) - 1);
    s->ring_cap = uint32_t(4 * slots);
    s->ring_gen.assign(s->ring_cap, 0);
    for (int i = int(slots) - 1; i >= 0; --i) s->free_slots.push_back(i);
    const unsigned mapped = cudaHostAllocMapped;
    e = cudaStreamCreateWithFlags(&s->loop_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->upload_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaHostAlloc(&s->h_ring, s->ring_cap * sizeof(LoopEntry), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(&s->h_ctl, 64 * sizeof(uint32_t), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_ring, s->ring_cap * sizeof(LoopEntry));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_ctl, 64 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaHostAlloc(&s->h_fin, slots * sizeof(uint32_t), mapped);
    if (e == cudaSuccess) e = cudaHostAlloc(&s->h_mom, slots * MPC_MOMENTS * sizeof(double), mapped);
    if (e == cudaSuccess) e = cudaHostAlloc(&s->h_claim, slots * sizeof(unsigned long long), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_claim, slots * sizeof(unsigned long long));
    if (e == cudaSuccess) {
      std::memset(s->h_ring, 0xFF, s->ring_cap * sizeof(LoopEntry));
      std::memset(s->h_ctl, 0, 64 * sizeof(uint32_t));
      std::memset(s->h_fin, 0, slots * sizeof(uint32_t));
      std::memset(s->h_mom, 0, slots * MPC_MOMENTS * sizeof(double));
      e = cudaMemcpyAsync(s->d_ring, s->h_ring, s->ring_cap * sizeof(LoopEntry), cudaMemcpyHostToDevice, s->stream);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_ctl, 0, 64 * sizeof(uint32_t), s->stream);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&s->d_fin, s->h_fin, 0);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&s->d_mom, s->h_mom, 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_claim, 0, slots * sizeof(unsigned long long), s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    const int per_sm = serve_loop_blocks_per_sm();
    s->loop_grid = ctx->sm_count * std::max(per_sm, 1);
    if (e != cudaSuccess || per_sm < 1) {
      ctx->last_error = std::string("device-loop server set-up: ") +
                        (e != cudaSuccess ? cudaGetErrorString(e) : "the loop kernel cannot be resident");
      mpc_server_stop(s);
      return MPC_E_CUDA;
    }
  }
  s->worker = std::thread(serve, s);
  *out = s;
  return MPC_OK;
}

int mpc_submit(mpc_server_t* s, const mpc_request_t* req, uint64_t* ticket) {
  if (!s || !req || !ticket) return MPC_E_INVALID_CONFIG;
  std::string msg;
  int st = validate(*req, &msg);
  Ticket t;
  t.req = *req;
  std::memset(&t.res, 0, sizeof(t.res));
  if (st == MPC_OK && req->workload != MPC_WORKLOAD_ASIAN_MLMC && req->workload != MPC_WORKLOAD_AMERICAN_PUT &&
      req->workload != MPC_WORKLOAD_BERMUDAN_PUT) {
    st = prepare(s->ctx, *req, &t.prep, &msg);
    if (st == MPC_OK && !t.prep.plain && s->opt.mode != 1) {
      if (!t.prep.halton_primes.empty() || !t.prep.lhs.empty() || t.prep.q.bridge || merton_stream_request(*req))
        t.prep.plain = true;  // per-request tables or the Merton stream replay: their own launches
      else if (!shape_for_slot(s, &t.prep))
        t.prep.plain = true;  // too many tiles for a slot: priced as its own batch
    }
  } else if (st == MPC_OK) {
    t.prep.lsm = req->workload != MPC_WORKLOAD_ASIAN_MLMC;
    t.prep.mlmc = req->workload == MPC_WORKLOAD_ASIAN_MLMC;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  t.id = s->next_id++;
  t.t_enqueue = now_ms(s);
  s->stats.submitted++;
  *ticket = t.id;
  if (st != MPC_OK) {
    t.res.status = st;
    t.state = 2;
    t.t_complete = t.t_enqueue;
    s->stats.rejected++;
    s->tickets[t.id] = t;
    return st;
  }
  s->tickets[t.id] = t;
  s->queue.push_back(t.id);
  s->cv_work.notify_one();
  return MPC_OK;
}

int mpc_poll(mpc_server_t* s, uint64_t ticket, mpc_result_t* out) {
  if (!s || !out) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return MPC_E_NOT_FOUND;
  if (it->second.state == 3) return MPC_E_CANCELLED;
  if (it->second.state != 2) return MPC_E_BUSY;
  *out = it->second.res;
  return it->second.res.status;
}

int mpc_wait(mpc_server_t* s, uint64_t ticket, int64_t timeout_ms, mpc_result_t* out) {
  if (!s || !out) return MPC_E_INVALID_CONFIG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto deadline = Clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 3600000 : timeout_ms);
  for (;;) {
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return MPC_E_NOT_FOUND;
    if (it->second.state == 3) return MPC_E_CANCELLED;
    if (it->second.state == 2) {
      *out = it->second.res;
      return it->second.res.status;
    }
    if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
      auto it2 = s->tickets.find(ticket);
      if (it2 != s->tickets.end() && it2->second.state == 2) {
        *out = it2->second.res;
        return it2->second.res.status;
      }
      return MPC_E_TIMEOUT;
    }
  }
}

int mpc_cancel(mpc_server_t* s, uint64_t ticket) {
  if (!s) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return MPC_E_NOT_FOUND;
  if (it->second.state != 0) return MPC_E_BUSY;  // only queued requests can be cancelled
  it->second.state = 3;
  s->stats.cancelled++;
  s->cv_done.notify_all();
  return MPC_OK;
}

int mpc_server_stats(mpc_server_t* s, mpc_server_stats_t* out) {
  if (!s || !out) return MPC_E_INVALID_CONFIG;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->live_bytes = s->live_bytes;
  out->p50_ms = percentile(s->latencies, 0.50);
  out->p99_ms = percentile(s->latencies, 0.99);
  double sum = 0, mx = 0;
  for (double v : s->latencies) {
    sum += v;
    mx = std::max(mx, v);
  }
  out->mean_ms = s->latencies.empty() ? 0.0 : sum / double(s->latencies.size());
  out->max_ms = mx;
  out->busy_ms = s->busy_ms;
  out->wall_ms = now_ms(s);
  return MPC_OK;
}

int mpc_server_stop(mpc_server_t* s) {
  if (!s) return MPC_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->ctx->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  cudaFree(s->d_slots);
  cudaFree(s->d_partials);
  cudaFree(s->d_moments);
  cudaFree(s->d_done);
  cudaFree(s->d_tiles);
  cudaFree(s->d_counter);
  if (s->h_slots) cudaFreeHost(s->h_slots);
  if (s->h_tiles) cudaFreeHost(s->h_tiles);
  if (s->h_moments) cudaFreeHost(s->h_moments);
  if (s->loop_stream) {
    if (s->h_ctl && s->d_ctl && s->upload_stream) set_control(s, 1, 1);  // stop a loop still resident
    cudaStreamSynchronize(s->loop_stream);
    cudaStreamDestroy(s->loop_stream);
  }
  cudaFree(s->d_ring);
  cudaFree(s->d_ctl);
  if (s->upload_stream) cudaStreamDestroy(s->upload_stream);
  if (s->h_ring) cudaFreeHost(s->h_ring);
  if (s->h_ctl) cudaFreeHost(s->h_ctl);
  if (s->h_fin) cudaFreeHost(s->h_fin);
  if (s->h_mom) cudaFreeHost(s->h_mom);
  if (s->h_claim) cudaFreeHost(s->h_claim);
  cudaFree(s->d_claim);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return MPC_OK;
}

}  // extern "C"

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
// All waiting is host-side on CUDA events and condition variables with
// timeouts; no device code spins.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

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

void serve(mpc_server* s) {
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
    if (st == MPC_OK && !t.prep.plain && s->opt.mode == 0) {
      if (!t.prep.halton_primes.empty() || !t.prep.lhs.empty() || t.prep.q.bridge)
        t.prep.plain = true;  // samplers with per-request tables run as their own launch
      else {
        Shape sh = choose_shape(s->ctx, t.prep);
        t.prep.q.tile_units = sh.block * sh.ppt;
        while ((t.prep.q.n_units + t.prep.q.tile_units - 1) / t.prep.q.tile_units > s->max_tiles_per_slot)
          t.prep.q.tile_units *= 2;
        t.prep.q.n_tiles = uint32_t((t.prep.q.n_units + t.prep.q.tile_units - 1) / t.prep.q.tile_units);
      }
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
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return MPC_OK;
}

}  // extern "C"

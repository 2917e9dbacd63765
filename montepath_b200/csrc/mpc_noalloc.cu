// mpc_noalloc.cu -- pricing entry point that allocates no memory.
//
// Some callers cannot let a library allocate device memory: a pricing
// service that reserves the GPU's memory for its own allocator at start-up
// (a cudaMalloc from a library would fail or break its accounting), or a
// latency-critical path where cudaMalloc / cudaFree, which can synchronise
// the device, are not allowed.  mpc_price_fused_noalloc serves them: it runs
// the fused FP32-path pricing kernel of mpc_price with every device buffer it
// needs -- the request descriptor, the tile work list, the per-tile moment
// partials, the completion counters and the lookup tables -- in file-scope
// static __device__ arrays of fixed size.  Each GPU that loads the library
// holds these arrays (about 0.7 MB) until the process exits.

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "mpc_launch.h"
#include "mpc_runtime.h"
#include "mpc_types.h"

namespace {

// Capacity of the scratch: at most kNoAllocMaxTiles tiles of at most
// 256 * kNoAllocMaxPpt units (paths, or antithetic pairs) each.
constexpr uint32_t kNoAllocMaxTiles = 4096;
constexpr uint32_t kNoAllocMaxPpt = 16;
constexpr uint64_t kNoAllocMaxUnits = uint64_t(kNoAllocMaxTiles) * 256 * kNoAllocMaxPpt;  // 16,777,216

struct NoAllocScratch {
  mpc::DevReq req;                                   // request descriptor
  double moments[MPC_MOMENTS];                       // final moments
  uint32_t tiles_done;                               // last-tile counter (reset by the kernel)
  uint32_t tile_counter;                             // work-list cursor (cleared every call)
  uint32_t _pad[2];
  mpc::Tile tiles[kNoAllocMaxTiles];                 // work list
  double partials[kNoAllocMaxTiles * MPC_MOMENTS];  // per-tile moments
};

// The scratch and the read-only tables.  In host code these names are
// host-side stand-ins, not device addresses; device addresses come from
// cudaGetSymbolAddress in setup_device().
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;
static __device__ __align__(256) uint32_t g_noalloc_sobol[MPC_SOBOL_TABLE_WORDS];
static __device__ __align__(256) uint64_t g_noalloc_jump[64 * 256];

struct DeviceState {
  bool ready = false;
  NoAllocScratch* scratch = nullptr;
  mpc::DeviceTables tabs{};
  int sm_count = 0;
};

// One slot per device ordinal in storage that never moves: a call in flight on
// one device keeps a valid DeviceState* while another device is set up.
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_mu;
DeviceState g_devices[kNoAllocMaxDevices];

void write_message(char* out, size_t len, const std::string& msg) {
  if (out && len) std::snprintf(out, len, "%s", msg.c_str());
}

// Once per device, with that device current: resolves the device addresses
// of the static arrays and uploads the lookup tables.
int setup_device(int device, DeviceState** out, std::string* msg) {
  if (device < 0 || device >= kNoAllocMaxDevices) {
    *msg = "device ordinal " + std::to_string(device) + " is beyond the " + std::to_string(kNoAllocMaxDevices) +
           " devices the no-allocation entry point serves";
    return MPC_E_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceState& st = g_devices[device];
  if (!st.ready) {
    void* scratch = nullptr;
    void* sobol = nullptr;
    void* jump = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
    if (e == cudaSuccess) e = cudaGetSymbolAddress(&sobol, g_noalloc_sobol);
    if (e == cudaSuccess) e = cudaGetSymbolAddress(&jump, g_noalloc_jump);
    if (e != cudaSuccess) {
      *msg = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return MPC_E_CUDA;
    }
    std::vector<uint32_t> sob;
    std::vector<uint64_t> jmp;
    mpc::build_tables(sob, jmp);
    e = cudaMemcpyToSymbol(g_noalloc_sobol, sob.data(), sob.size() * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_noalloc_jump, jmp.data(), jmp.size() * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMemset(scratch, 0, sizeof(NoAllocScratch));
    // the work list of a single request is always tiles 0, 1, 2, ... of request 0
    std::vector<mpc::Tile> tiles(kNoAllocMaxTiles);
    for (uint32_t t = 0; t < kNoAllocMaxTiles; ++t) tiles[t] = mpc::Tile{0u, t};
    if (e == cudaSuccess)
      e = cudaMemcpy(static_cast<NoAllocScratch*>(scratch)->tiles, tiles.data(), tiles.size() * sizeof(mpc::Tile),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      *msg = std::string("table upload: ") + cudaGetErrorString(e);
      return MPC_E_CUDA;
    }
    cudaDeviceGetAttribute(&st.sm_count, cudaDevAttrMultiProcessorCount, device);
    st.scratch = static_cast<NoAllocScratch*>(scratch);
    st.tabs.sobol = static_cast<const uint32_t*>(sobol);
    st.tabs.jump = static_cast<const uint64_t*>(jump);
    st.ready = true;
  }
  *out = &st;
  return MPC_OK;
}

}  // namespace

extern "C" int mpc_price_fused_noalloc(const mpc_request_t* req, mpc_result_t* out, void* stream,
                                       char* error_message, size_t error_message_len) {
  if (!req || !out) return MPC_E_INVALID_CONFIG;
  std::memset(out, 0, sizeof(*out));
  auto reject = [&](int status, const std::string& msg) {
    write_message(error_message, error_message_len, msg);
    out->status = status;
    return status;
  };
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return reject(MPC_E_NO_DEVICE, "no CUDA device");
  std::string msg;
  mpc::Prepared p;
  int st = mpc::prepare(nullptr, *req, &p, &msg);
  if (st != MPC_OK) return reject(st, msg);
  if (p.plain || p.lsm || p.mlmc)
    return reject(MPC_E_UNSUPPORTED, "the no-allocation entry point prices FP32-path path-payoff requests only");
  if (p.sampler != mpc::SMP_XORSHIFT && p.sampler != mpc::SMP_COUNTER && p.sampler != mpc::SMP_SOBOL)
    return reject(MPC_E_UNSUPPORTED,
                  "the no-allocation entry point supports pseudorandom, counter_hash and scrambled_sobol sampling");
  if (p.q.bridge)  // the bridge program lives in a per-request device table
    return reject(MPC_E_UNSUPPORTED, "the no-allocation entry point does not run Brownian-bridge paths");
  if (p.q.n_units > kNoAllocMaxUnits)
    return reject(MPC_E_OOM_BUDGET, "request has " + std::to_string(p.q.n_units) +
                                        " paths (or antithetic pairs); the no-allocation scratch holds at most " +
                                        std::to_string(kNoAllocMaxUnits));
  DeviceState* ds = nullptr;
  if ((st = setup_device(device, &ds, &msg)) != MPC_OK) return reject(st, msg);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Tiles of 256 * ppt units: the request's paths_per_thread hint when it is a
  // power of two whose work list fits the scratch, else (no hint) the smallest
  // power of two that fits.
  uint32_t ppt = 1;
  if (req->paths_per_thread != 0) {
    ppt = req->paths_per_thread;
    const bool pow2 = (ppt & (ppt - 1)) == 0;
    if (!pow2 || ppt > kNoAllocMaxPpt ||
        (p.q.n_units + 256ull * ppt - 1) / (256ull * ppt) > kNoAllocMaxTiles)
      return reject(MPC_E_UNSUPPORTED, "paths_per_thread hint " + std::to_string(ppt) +
                                           " is not a power of two up to " + std::to_string(kNoAllocMaxPpt) +
                                           " whose tiles of 256 * hint paths fit the " +
                                           std::to_string(kNoAllocMaxTiles) + "-tile scratch");
  } else {
    while ((p.q.n_units + 256ull * ppt - 1) / (256ull * ppt) > kNoAllocMaxTiles) ppt *= 2;
  }
  mpc::DevReq q = p.q;
  q.tile_units = 256 * ppt;
  q.n_tiles = uint32_t((q.n_units + q.tile_units - 1) / q.tile_units);
  q.partials = ds->scratch->partials;
  q.moments = ds->scratch->moments;
  q.tiles_done = &ds->scratch->tiles_done;
  q.per_unit = nullptr;
  // The scratch keeps the previous call's contents: the counters must start at zero.
  cudaError_t e = cudaMemsetAsync(&ds->scratch->tiles_done, 0, 2 * sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&ds->scratch->req, &q, sizeof(q), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return reject(MPC_E_CUDA, std::string("upload: ") + cudaGetErrorString(e));
  const int occ = std::max(1, mpc::fused_max_blocks_per_sm(p.family, p.sampler, 256));
  const int grid = int(std::min<uint64_t>(uint64_t(ds->sm_count) * occ, q.n_tiles));
  e = mpc::launch_fused(&ds->scratch->req, ds->scratch->tiles, q.n_tiles, &ds->scratch->tile_counter, p.family,
                        p.sampler, ds->tabs, std::max(grid, 1), 256, s);
  if (e != cudaSuccess) return reject(MPC_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  double moments[MPC_MOMENTS];
  e = cudaMemcpyAsync(moments, ds->scratch->moments, sizeof(moments), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return reject(MPC_E_CUDA, std::string("execution: ") + cudaGetErrorString(e));
  mpc::summarize_moments(p, moments, out);
  out->path_steps = p.path_steps;
  out->status = MPC_OK;
  return MPC_OK;
}

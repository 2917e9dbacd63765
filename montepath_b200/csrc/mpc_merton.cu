// mpc_merton.cu -- the reference's Merton jump-diffusion estimator on the
// device: terminal sampling from one sequential MonteCarloRng stream per
// chunk (simulate_merton_jump_diffusion_chunk, crates/mc-core/src/runtime/
// cpu.rs:6408-6441; chunk split cpu.rs:6154-6199).
//
// Each path draws a Box-Muller normal (two stream outputs, or none when the
// stream holds a cached normal), one uniform for the Poisson jump count
// (sample_poisson, cpu.rs:932-953) and, only when the count is positive, a
// second normal.  Where a path starts in the stream therefore depends on the
// jump counts of every earlier path of its chunk.  With the stream position p
// of a path start and the cache state c (NONE, or a cached sine branch of the
// pair drawn 2 or 3 positions back), a path starting at (p, NONE) reads its
// Poisson uniform at p + 2 and moves to (p + 3, NONE) after a jump or
// (p + 3, CACHE3) without one; a path starting at (p, CACHE) reads it at p
// and moves to (p + 3, CACHE2) or (p + 1, NONE).  Path starts advance by one
// or three positions and depend only on one "jump" bit per position, so the
// chain of path starts is found in parallel:
//
//   1. fill:    every stream output x[q] (GF(2) jump-ahead to a 64-position
//               run, then sequential xorshift64*) and the bit
//               J[q] = (open01(x[q]) > exp(-lambda T)), i.e. "sample_poisson
//               would return k > 0 from this uniform";
//   2. maps:    for each 64-position segment and each of its 9 possible entry
//               states (first path start at offset 0, 1 or 2, cache state),
//               the exit state into the next segment and the number of path
//               starts inside, walking the jump bits in registers;
//   3. scan:    per chunk, the segment maps composed from the chunk's first
//               path (position 0, no cache): every segment's true entry state
//               and the number of paths before it;
//   4. emit:    every segment re-walked from its true entry, writing each
//               path's start state at its path index;
//   5. payoff:  one thread per path: its normals, exact jump count and
//               discounted payoff in FP64, rounding every product and sum
//               separately as the reference does (no FMA contraction).
//
// The payoffs then go through the plain FP64 tile reduction.  With
// lambda T == 0, sample_poisson draws no uniform, so paths alternate between
// the cosine and sine branch of consecutive pairs and need no chain.

#include <cuda_runtime.h>
#include <stdint.h>

#include "mpc_device.cuh"
#include "mpc_launch.h"

namespace mpc {

namespace {

constexpr uint32_t kSeg = kMertonSegment;  // positions per segment (two 32-bit jump words)
constexpr int kScanThreads = 512;

enum : uint32_t { CS_NONE = 0, CS_CACHE2 = 1, CS_CACHE3 = 2 };

__device__ __forceinline__ uint64_t chunk_seed(const MertonStreamArgs& a, uint32_t c) {
  uint64_t s = a.n_chunks <= 1 ? a.seed : derive_chunk_seed(a.seed, c);
  return s == 0 ? 0x9E3779B97F4A7C15ull : s;  // MonteCarloRng::new (cpu.rs:2961-2970)
}

__device__ __forceinline__ uint64_t chunk_paths(const MertonStreamArgs& a, uint32_t c) {
  if (a.n_chunks <= 1) return a.n_paths;
  return a.chunk_base + (c < a.chunk_rem ? 1 : 0);
}

__device__ __forceinline__ uint64_t chunk_first_path(const MertonStreamArgs& a, uint32_t c) {
  if (a.n_chunks <= 1) return 0;
  return uint64_t(c) * a.chunk_base + (c < a.chunk_rem ? c : a.chunk_rem);
}

__device__ __forceinline__ double open01(uint64_t x) {  // next_f64_open01 (cpu.rs:2985-2990)
  double v = (double)(x >> 11) * (1.0 / 9007199254740992.0);
  return fmax(v, 2.2250738585072014e-308);
}

// One path-start transition; `bit(q)` is the jump bit at relative position q.
template <typename Bit>
__device__ __forceinline__ void advance(uint32_t& p, uint32_t& cs, Bit bit) {
  if (cs == CS_NONE) {
    const bool j = bit(p + 2);
    p += 3;
    cs = j ? CS_NONE : CS_CACHE3;
  } else {
    const bool j = bit(p);
    if (j) {
      p += 3;
      cs = CS_CACHE2;
    } else {
      p += 1;
      cs = CS_NONE;
    }
  }
}

// 1. Stream outputs and jump bits, 64 consecutive positions per thread.
__global__ void __launch_bounds__(256) merton_fill_kernel(MertonStreamArgs a, const uint64_t* __restrict__ nibble) {
  const uint64_t runs_per_chunk = a.qpad / kSeg;
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= runs_per_chunk * a.n_chunks) return;
  const uint32_t c = uint32_t(t / runs_per_chunk);
  const uint64_t run = t - uint64_t(c) * runs_per_chunk;
  XorshiftStream s;
  s.state = xorshift_jump(nibble, chunk_seed(a, c), run * kSeg);
  s.has_cached = false;
  const uint64_t base = uint64_t(c) * a.qpad + run * kSeg;
  uint32_t w0 = 0, w1 = 0;
#pragma unroll 4
  for (uint32_t i = 0; i < kSeg; ++i) {
    const uint64_t x = s.next_u64();
    a.x[base + i] = x;
    const uint32_t j = open01(x) > a.p0 ? 1u : 0u;  // sample_poisson's first `u > cumulative`
    if (i < 32)
      w0 |= j << i;
    else
      w1 |= j << (i - 32);
  }
  const uint64_t wbase = (uint64_t(c) * a.qpad + run * kSeg) / 32;
  a.bits[wbase] = w0;
  a.bits[wbase + 1] = w1;
}

// 2. Segment maps: entry e = offset * 3 + cache state -> (count << 4) | exit.
__global__ void __launch_bounds__(256) merton_maps_kernel(MertonStreamArgs a) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t per_chunk = a.n_segs * 9;
  if (t >= per_chunk * a.n_chunks) return;
  const uint32_t c = uint32_t(t / per_chunk);
  const uint64_t rem = t - uint64_t(c) * per_chunk;
  const uint64_t seg = rem / 9;
  const uint32_t e = uint32_t(rem - seg * 9);
  const uint32_t* w = a.bits + (uint64_t(c) * a.qpad + seg * kSeg) / 32;
  const uint32_t b0 = w[0], b1 = w[1], b2 = w[2];  // positions 0..95 of the segment
  auto bit = [&](uint32_t q) -> bool {
    const uint32_t word = q < 32 ? b0 : (q < 64 ? b1 : b2);
    return (word >> (q & 31)) & 1u;
  };
  uint32_t p = e / 3, cs = e % 3, count = 0;
  while (p < kSeg) {
    advance(p, cs, bit);
    ++count;
  }
  a.maps[(uint64_t(c) * a.n_segs + seg) * 9 + e] = uint16_t((count << 4) | ((p - kSeg) * 3 + cs));
}

// 3. Per chunk (one block): each thread composes a contiguous range of
// segment maps for all 9 entries, thread 0 chains the ranges from the chunk's
// first path, then each thread walks its range from its true entry state.
__global__ void __launch_bounds__(kScanThreads) merton_scan_kernel(MertonStreamArgs a) {
  __shared__ uint8_t s_exit[kScanThreads][9];
  __shared__ uint32_t s_count[kScanThreads][9];
  __shared__ uint8_t s_entry[kScanThreads];
  __shared__ unsigned long long s_before[kScanThreads];
  const uint32_t c = blockIdx.x;
  const uint64_t n_segs = a.n_segs;
  const uint64_t per = (n_segs + kScanThreads - 1) / kScanThreads;
  const uint64_t first = min(n_segs, uint64_t(threadIdx.x) * per);
  const uint64_t last = min(n_segs, first + per);
  const uint16_t* maps = a.maps + uint64_t(c) * n_segs * 9;
  for (uint32_t e = 0; e < 9; ++e) {
    uint32_t st = e, cnt = 0;
    for (uint64_t s = first; s < last; ++s) {
      const uint16_t m = maps[s * 9 + st];
      cnt += m >> 4;
      st = m & 15u;
    }
    s_exit[threadIdx.x][e] = uint8_t(st);
    s_count[threadIdx.x][e] = cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t st = 0;  // position 0, no cached normal
    unsigned long long before = 0;
    for (int t = 0; t < kScanThreads; ++t) {
      s_entry[t] = uint8_t(st);
      s_before[t] = before;
      before += s_count[t][st];
      st = s_exit[t][st];
    }
  }
  __syncthreads();
  uint32_t st = s_entry[threadIdx.x];
  unsigned long long before = s_before[threadIdx.x];
  for (uint64_t s = first; s < last; ++s) {
    a.seg_state[uint64_t(c) * n_segs + s] = uint8_t(st);
    a.seg_before[uint64_t(c) * n_segs + s] = before;
    const uint16_t m = maps[s * 9 + st];
    before += m >> 4;
    st = m & 15u;
  }
}

// 4. Path starts: (relative position << 2) | cache state, at each path's index.
__global__ void __launch_bounds__(256) merton_emit_kernel(MertonStreamArgs a) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= a.n_segs * a.n_chunks) return;
  const uint32_t c = uint32_t(t / a.n_segs);
  const uint64_t seg = t - uint64_t(c) * a.n_segs;
  const uint32_t* w = a.bits + (uint64_t(c) * a.qpad + seg * kSeg) / 32;
  const uint32_t b0 = w[0], b1 = w[1], b2 = w[2];
  auto bit = [&](uint32_t q) -> bool {
    const uint32_t word = q < 32 ? b0 : (q < 64 ? b1 : b2);
    return (word >> (q & 31)) & 1u;
  };
  const uint32_t e = a.seg_state[t];
  uint64_t idx = a.seg_before[t];
  const uint64_t n_c = chunk_paths(a, c), out0 = chunk_first_path(a, c);
  uint32_t p = e / 3, cs = e % 3;
  while (p < kSeg) {
    if (idx < n_c) a.starts[out0 + idx] = ((seg * kSeg + p) << 2) | cs;
    advance(p, cs, bit);
    ++idx;
  }
}

struct Pair {
  double cos_branch, sin_branch;
};
// Box-Muller of the pair at positions (i, i + 1) (cpu.rs:2992-3006).
__device__ __forceinline__ Pair box_muller(const uint64_t* __restrict__ x, uint64_t i) {
  const double u1 = open01(x[i]);
  const double u2 = open01(x[i + 1]);
  const double radius = sqrt(__dmul_rn(-2.0, log(u1)));
  const double theta = __dmul_rn(6.283185307179586, u2);  // 2.0 * PI * u2
  double s, c;
  sincos(theta, &s, &c);
  return Pair{__dmul_rn(radius, c), __dmul_rn(radius, s)};
}

// sample_poisson (cpu.rs:932-953) from its uniform, with exp(-mean) from the host.
__device__ __forceinline__ uint32_t poisson_count(double u, double mean, double p0) {
  double prob = p0, cum = p0;
  uint32_t k = 0;
  while (u > cum && k < 4095) {
    ++k;
    prob = __dmul_rn(prob, __ddiv_rn(mean, (double)k));
    cum = __dadd_rn(cum, prob);
  }
  return k;
}

// 5. Payoffs (cpu.rs:6420-6437).
__global__ void __launch_bounds__(256) merton_payoff_kernel(MertonStreamArgs a) {
  const uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= a.n_paths) return;
  uint32_t c = 0;
  uint64_t i = g;
  if (a.n_chunks > 1) {
    const uint64_t big = a.chunk_rem * (a.chunk_base + 1);
    if (g < big) {
      c = uint32_t(g / (a.chunk_base + 1));
      i = g - uint64_t(c) * (a.chunk_base + 1);
    } else {
      c = uint32_t(a.chunk_rem + (g - big) / a.chunk_base);
      i = g - big - uint64_t(c - a.chunk_rem) * a.chunk_base;
    }
  }
  const uint64_t* x = a.x + uint64_t(c) * a.qpad;
  double z, zj = 0.0;
  uint32_t jumps = 0;
  if (a.mean == 0.0) {
    // no Poisson uniform: path i takes the cosine (even i) or cached sine (odd i) of pair i / 2
    const Pair pr = box_muller(x, 2 * (i / 2));
    z = (i & 1) ? pr.sin_branch : pr.cos_branch;
  } else {
    const uint64_t st = a.starts[g];
    const uint64_t p = st >> 2;
    const uint32_t cs = uint32_t(st & 3);
    if (cs == CS_NONE) {
      const Pair pr = box_muller(x, p);
      z = pr.cos_branch;
      jumps = poisson_count(open01(x[p + 2]), a.mean, a.p0);
      if (jumps > 0) zj = pr.sin_branch;  // the cached normal
    } else {
      z = box_muller(x, p - (cs == CS_CACHE2 ? 2 : 3)).sin_branch;
      jumps = poisson_count(open01(x[p]), a.mean, a.p0);
      if (jumps > 0) zj = box_muller(x, p + 1).cos_branch;
    }
  }
  const double diffusion = __dmul_rn(a.vol_t, z);
  double jump = 0.0;
  if (jumps > 0) {
    const double n = (double)jumps;
    jump = __dadd_rn(__dmul_rn(n, a.jump_mean), __dmul_rn(__dmul_rn(a.jump_vol, sqrt(n)), zj));
  }
  const double log_st = __dadd_rn(__dadd_rn(__dadd_rn(a.log_s0, a.drift_t), diffusion), jump);
  const double s_t = exp(log_st);
  a.payoff[g] = __dmul_rn(fmax(__dsub_rn(s_t, a.k), 0.0), a.discount);
  if (a.control) a.control[g] = __dmul_rn(a.discount, s_t);
}

}  // namespace

cudaError_t launch_merton_stream(const MertonStreamArgs& a, const DeviceTables& tabs, cudaStream_t stream) {
  uint32_t launches = 0;
  if (a.mean != 0.0) {
    const uint64_t runs = a.qpad / kSeg * a.n_chunks;
    merton_fill_kernel<<<uint32_t((runs + 255) / 256), 256, 0, stream>>>(a, tabs.jump);
    const uint64_t maps = a.n_segs * 9 * a.n_chunks;
    merton_maps_kernel<<<uint32_t((maps + 255) / 256), 256, 0, stream>>>(a);
    merton_scan_kernel<<<a.n_chunks, kScanThreads, 0, stream>>>(a);
    const uint64_t segs = a.n_segs * a.n_chunks;
    merton_emit_kernel<<<uint32_t((segs + 255) / 256), 256, 0, stream>>>(a);
    launches += 4;
  } else {
    const uint64_t runs = a.qpad / kSeg * a.n_chunks;
    merton_fill_kernel<<<uint32_t((runs + 255) / 256), 256, 0, stream>>>(a, tabs.jump);
    launches += 1;
  }
  merton_payoff_kernel<<<uint32_t((a.n_paths + 255) / 256), 256, 0, stream>>>(a);
  launches += 1;
  count_graph_launches(launches);  // adds to the launch count
  return cudaGetLastError();
}

}  // namespace mpc

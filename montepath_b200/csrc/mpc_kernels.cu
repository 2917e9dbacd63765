// mpc_kernels.cu -- sm_100a kernels of the B200 Monte Carlo pricing backend.
//
// Fused path (FP32 path arithmetic, FP64 accumulation): samples are generated
// in registers, stepped through the model, turned into a payoff and reduced
// warp -> block -> tile partial; the block that completes a request's last
// tile sums the tile partials in tile order (deterministic, independent of
// which requests share the launch).  One persistent kernel walks a tile work
// list, so a single request, a heterogeneous book and a serving wave all use
// the same launch.
//
// Plain path (FP64, one request per launch sequence): samples materialised
// in HBM, a stepping kernel writing per-path payoffs (the contract of the
// reference's mc_cuda_european_call_stepwise_v1), and a reduction kernel.
//
// Longstaff-Schwartz: one cooperative launch.  Paths are written date-major,
// each date's ITM basis moments are reduced block -> grid (FP64), every block
// solves the 4x4 normal equations redundantly after a bounded grid barrier,
// and exercise decisions are applied in registers.

#include <atomic>
#include <mutex>
#include <set>
#include <utility>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/montepath_cuda.h"
#include "mpc_device.cuh"
#include "mpc_launch.h"
#include "mpc_types.h"

namespace mpc {

static std::atomic<uint64_t> g_launches{0};
uint64_t kernel_launch_count() { return g_launches.load(); }
void count_graph_launches(uint64_t kernels) { g_launches.fetch_add(kernels); }
void discount_captured_launches(uint64_t kernels) { g_launches.fetch_sub(kernels); }
static inline void count_launch() { g_launches.fetch_add(1); }

enum Workload : int32_t {
  W_EURO = 0,
  W_ASIAN = 1,
  W_DAO = 2,
  W_UAO = 3,
  W_LOOKBACK = 4,
};

struct SrcCtx {
  const uint32_t* sobol;  // device lookup table (MPC_SOBOL_TABLE_WORDS words)
  const uint64_t* jump;
  uint32_t* win;          // shared-memory window of Sobol table rows (fused kernel), null elsewhere
  const float4* icdf;     // shared-memory copy of the inverse-normal segments (fused kernel)
};

// Dimensions of the Sobol table rows staged in shared memory at a time, and
// the row stride in words: kSobolWindow + 4 is 4 mod 32, so the 16 rows one
// warp touches with a 128-bit load fall into two wavefronts.  The window
// holds the 48 rows of the index's three low nibbles and one constant row:
// a bit of the Owen-shuffled index depends only on the point's bits at and
// above it (and the seed), so bits 12..31 of the shuffled index are the same
// for every point of one aligned 4,096-point group, and the XOR of their five
// nibble rows is one word per dimension.  The points a block runs together
// (one iteration of a tile: at most 512 consecutive aligned units, the tile's
// idle threads repeating the iteration's first unit) lie in one such group.
// The output scramble's seed of a dimension, hash_combine(seed_g, dim),
// depends on the block's seed and the dimension alone, so a last row holds
// it for the window's dimensions: a quad reads its four seeds with one load.
constexpr uint32_t kSobolWindow = 64;
constexpr uint32_t kSobolRowStride = kSobolWindow + 4;
constexpr uint32_t kSobolLowNibbles = 3;                        // nibble positions 0..2 staged per point
constexpr uint32_t kSobolLowRows = 16 * kSobolLowNibbles;       // 48 rows
constexpr uint32_t kSobolConstRow = kSobolLowRows;              // XOR of the upper nibble rows
constexpr uint32_t kSobolSeedRow = kSobolLowRows + 1;           // output-scramble seed per dimension
constexpr uint32_t kSobolWindowWords = (kSobolLowRows + 2) * kSobolRowStride;  // 13,600 bytes

// Phi^-1(u) for a 23-bit midpoint uniform u from the segment table: v =
// min(u, 1 - u) (exact) selects binade and one of 32 segments from its
// exponent and top mantissa bits, the remaining 18 mantissa bits give the
// position t in [0, 1/32) in the segment (they sit below 1.0's exponent as
// they are, so no shift is needed), and the segment's cubic gives Phi^-1(v).
// Defined for v in [2^-24, 1/2), which every 23-bit midpoint uniform meets.
__device__ __forceinline__ float icdf_segments(const float4* __restrict__ seg, float u) {
  const float v = fminf(u, 1.0f - u);
  const uint32_t bits = __float_as_uint(v);
  const uint32_t idx = (bits >> 18) - (103u << 5);  // (exponent - 103) * 32 + top 5 mantissa bits
  const float t = __int_as_float((bits & 0x3FFFFu) | 0x3F800000u) - 1.0f;
  const float4 c = seg[idx];
  const float p = fmaf(fmaf(fmaf(c.w, t, c.z), t, c.y), t, c.x);
  return u < 0.5f ? p : -p;
}
// icdf_segments(seg, sobol_unit_f32_bits(x)) from the Sobol sample's bits.
// With m = x >> 9 the uniform is u = (m + 0.5) 2^-23, and its mirror 1 - u
// is the same expression of the 23-bit complement of m, so
// v = min(u, 1 - u) is built from x ^ (x >> 31, arithmetic): the complement
// exactly when bit 31 (u > 1/2) is set, which also gives the result's sign.
// Equal bit for bit to the two-step form, with no compare or select.
__device__ __forceinline__ float icdf_sobol_bits(const float4* __restrict__ seg, uint32_t x) {
  const uint32_t xm = x ^ (uint32_t)((int32_t)x >> 31);
  const float v = __fsub_rn(__uint_as_float((xm >> 9) + 0x3F800000u), 0.99999994f);
  const uint32_t bits = __float_as_uint(v);
  const uint32_t idx = (bits >> 18) - (103u << 5);
  const float t = __int_as_float((bits & 0x3FFFFu) | 0x3F800000u) - 1.0f;
  const float4 c = seg[idx];
  const float p = fmaf(fmaf(fmaf(c.w, t, c.z), t, c.y), t, c.x);
  return __uint_as_float(__float_as_uint(p) ^ (x & 0x80000000u));
}
// Two samples at once: the floating-point steps as packed FP32 pairs
// (FADD2 / FFMA2, each lane rounded exactly as the scalar operation), so the
// pair equals two icdf_sobol_bits calls bit for bit.
__device__ __forceinline__ float2 icdf_sobol_bits2(const float4* __restrict__ seg, uint32_t xa, uint32_t xb) {
  const uint32_t ma = xa ^ (uint32_t)((int32_t)xa >> 31), mb = xb ^ (uint32_t)((int32_t)xb >> 31);
  const float2 v = __fadd2_rn(make_float2(__uint_as_float((ma >> 9) + 0x3F800000u), __uint_as_float((mb >> 9) + 0x3F800000u)),
                              make_float2(-0.99999994f, -0.99999994f));
  const uint32_t ba = __float_as_uint(v.x), bb = __float_as_uint(v.y);
  const float4 ca = seg[(ba >> 18) - (103u << 5)], cb = seg[(bb >> 18) - (103u << 5)];
  const float2 t = __fadd2_rn(make_float2(__int_as_float((ba & 0x3FFFFu) | 0x3F800000u),
                                          __int_as_float((bb & 0x3FFFFu) | 0x3F800000u)),
                              make_float2(-1.0f, -1.0f));
  float2 p = __ffma2_rn(make_float2(ca.w, cb.w), t, make_float2(ca.z, cb.z));
  p = __ffma2_rn(p, t, make_float2(ca.y, cb.y));
  p = __ffma2_rn(p, t, make_float2(ca.x, cb.x));
  return make_float2(__uint_as_float(__float_as_uint(p.x) ^ (xa & 0x80000000u)),
                     __uint_as_float(__float_as_uint(p.y) ^ (xb & 0x80000000u)));
}

// ------------------------------------------------------------- sources ----
// A Source yields the samples of one unit (path or antithetic pair) by
// dimension index.  n32/n64: standard normal in FP32 / FP64; u64: the raw
// uniform (Merton's Poisson dimension).  Models announce each step's
// dimensions with at_step(first, count) before sampling them; every thread
// of a block makes the same at_step calls, which lets the Sobol source stage
// its tables block-synchronously.
template <int S>
struct Source;

template <>
struct Source<SMP_COUNTER> {
  uint32_t seed, unit;
  template <bool FP64>
  __device__ __forceinline__ void begin(const DevReq& q, const SrcCtx&, uint64_t u) {
    seed = q.seed32;
    unit = (uint32_t)u;
  }
  __device__ __forceinline__ void at_step(uint32_t, uint32_t) {}
  __device__ __forceinline__ float n32(uint32_t d) { return counter_normal_f32(seed, unit, d); }
  __device__ __forceinline__ double n64(uint32_t d) { return (double)counter_normal_f32(seed, unit, d); }
  __device__ __forceinline__ double u64(uint32_t d) {
    return (double)counter_open01(hash_u32(counter_mix(seed, unit, d, 0u)));
  }
  __device__ __forceinline__ float u32(uint32_t d) { return counter_open01(hash_u32(counter_mix(seed, unit, d, 0u))); }
};

// Scrambled Sobol with the per-point work hoisted: the Owen-shuffled index
// and its nibble offsets depend only on (point, dimension group of 256), so
// they are recomputed when a path crosses into the next group; per
// dimension only the 8 table lookups and the output scramble remain.  The
// values equal sobol_point() bit for bit.  Reads the [dim][q][v] layout from
// global memory (generators and the FP64 plain path).
template <>
struct Source<SMP_SOBOL> {
  const uint32_t* table;
  uint32_t local, block_seed, group, seed_g, combine_g;
  uint32_t off[8];
  template <bool FP64>
  __device__ __forceinline__ void begin(const DevReq& q, const SrcCtx& c, uint64_t u) {
    table = c.sobol;
    local = (uint32_t)(u & 0xFFFFu);
    block_seed = q.seed32 + (uint32_t)(u >> 16) * 0x9E3779B9u;
    group = 0xFFFFFFFFu;
  }
  __device__ __forceinline__ void at_step(uint32_t, uint32_t) {}
  __device__ __forceinline__ uint32_t sample(uint32_t d) {
    const uint32_t g = d / MPC_SOBOL_TABLE_DIMS;
    if (g != group) {
      group = g;
      seed_g = block_seed + g;
      const uint32_t shuffled = nested_uniform_scramble(local, seed_g);
#pragma unroll
      for (int q = 0; q < 8; ++q) off[q] = q * 16 + ((shuffled >> (4 * q)) & 0xFu);
      combine_g = 0x9e3779b9u + (seed_g << 6) + (seed_g >> 2);
    }
    const uint32_t dim = d & (MPC_SOBOL_TABLE_DIMS - 1);
    const uint32_t* td = table + dim * 128;
    uint32_t x = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) x ^= __ldg(td + off[q]);
    return nested_uniform_scramble(x, seed_g ^ (dim + combine_g));  // hash_combine(seed_g, dim)
  }
  __device__ __forceinline__ float n32(uint32_t d) { return normcdfinvf(sobol_unit_f32(sample(d))); }
  __device__ __forceinline__ float u32(uint32_t d) { return sobol_unit_f32(sample(d)); }
  __device__ __forceinline__ double n64(uint32_t d) { return icdf_f64(sobol_unit_f64(sample(d))); }
  __device__ __forceinline__ double u64(uint32_t d) { return sobol_unit_f64(sample(d)); }
};

template <>
struct Source<SMP_HALTON> {
  uint64_t index;
  const uint32_t* primes;
  const double* shifts;
  template <bool FP64>
  __device__ __forceinline__ void begin(const DevReq& q, const SrcCtx&, uint64_t u) {
    index = u + 1;
    primes = q.halton_primes;
    shifts = q.halton_shifts;
  }
  __device__ __forceinline__ void at_step(uint32_t, uint32_t) {}
  __device__ __forceinline__ double u64(uint32_t d) { return halton_shifted(index, __ldg(primes + d), __ldg(shifts + d)); }
  __device__ __forceinline__ double n64(uint32_t d) { return icdf_f64(u64(d)); }
  __device__ __forceinline__ float n32(uint32_t d) {
    float u = fminf(fmaxf((float)u64(d), 5.9604645e-08f), 0.99999994f);
    return normcdfinvf(u);
  }
  __device__ __forceinline__ float u32(uint32_t d) { return (float)u64(d); }
};

template <>
struct Source<SMP_LHS> {
  uint64_t point, n_paths;
  const LhsDim* dims;
  template <bool FP64>
  __device__ __forceinline__ void begin(const DevReq& q, const SrcCtx&, uint64_t u) {
    point = u;
    n_paths = q.n_paths;
    dims = q.lhs;
  }
  __device__ __forceinline__ void at_step(uint32_t, uint32_t) {}
  __device__ __forceinline__ double u64(uint32_t d) {
    LhsDim ld;
    ld.multiplier = __ldg(&dims[d].multiplier);
    ld.offset = __ldg(&dims[d].offset);
    ld.jitter_seed = __ldg(&dims[d].jitter_seed);
    return lhs_uniform(ld, point, n_paths);
  }
  __device__ __forceinline__ double n64(uint32_t d) { return icdf_f64(u64(d)); }
  __device__ __forceinline__ float n32(uint32_t d) {
    float u = fminf(fmaxf((float)u64(d), 5.9604645e-08f), 0.99999994f);
    return normcdfinvf(u);
  }
  __device__ __forceinline__ float u32(uint32_t d) { return (float)u64(d); }
};

template <>
struct Source<SMP_XORSHIFT> {
  XorshiftStream st;
  template <bool FP64>
  __device__ __forceinline__ void begin(const DevReq& q, const SrcCtx& c, uint64_t u) {
    uint64_t seed, local;
    chunk_of(q, u, &seed, &local);
    st.seek(c.jump, seed, local * q.normals_per_unit, !FP64);
  }
  __device__ __forceinline__ void at_step(uint32_t, uint32_t) {}
  // Sequential stream: dimensions must be requested in increasing order.
  __device__ __forceinline__ float n32(uint32_t) { return st.normal_f32(); }
  __device__ __forceinline__ double n64(uint32_t) { return st.normal_f64(); }
  __device__ __forceinline__ double u64(uint32_t) { return st.next_open01(); }
  __device__ __forceinline__ float u32(uint32_t) { return st.next_open01_f32(); }
};

// ------------------------------------------------ fused FP32 sources ---
// The fused kernels draw their samples through FusedSource<SMP>::type:
// the generic sources except for scrambled Sobol and the counter hash.

// Scrambled Sobol for the fused kernels, bit-identical to Source<SMP_SOBOL>.
// A block-synchronous window in shared memory holds, for each table row
// r = 16 q + v of the three low nibble positions, the bit-reversed nibble
// products of kSobolWindow consecutive dimensions, the constant row of the
// upper positions and the output-scramble seeds, so one 128-bit load per row
// serves four dimensions: a quad of dimensions costs 5 shared loads and 12
// XORs instead of 32 loads.  XOR commutes with bit reversal, so the quad
// holds brev(x) and the output scramble skips its first reversal.
struct SobolQuad {
  const uint32_t* rows_global;  // [128][256] bit-reversed rows
  uint32_t* win;                // [kSobolLowRows + 2][kSobolRowStride] shared-memory window
  const float4* icdf;           // inverse-normal segments in shared memory
  uint32_t win_first;           // first dimension in the window (multiple of 4)
  uint32_t local, block_seed, group, quad;
  uint32_t rows[kSobolLowNibbles];  // window word offset of this point's row per low nibble position
  uint32_t x0, x1, x2, x3;      // reversed products of the dimensions of `quad`
  uint32_t s0, s1, s2, s3;      // their output-scramble seeds
  template <bool FP64>
  __device__ __forceinline__ void begin(const DevReq& q, const SrcCtx& c, uint64_t u) {
    rows_global = c.sobol + MPC_SOBOL_NIBBLE_WORDS;
    win = c.win;
    icdf = c.icdf;
    win_first = 0xFFFFFFFFu;
    local = (uint32_t)(u & 0xFFFFu);
    block_seed = q.seed32 + (uint32_t)(u >> 16) * 0x9E3779B9u;
    group = 0xFFFFFFFFu;
    quad = 0xFFFFFFFFu;
  }
  // Block-synchronous: restages the window at d0 rounded down to a multiple
  // of 4 when [d0, d0 + count) is not inside it.  Requires
  // count <= kSobolWindow - 3 so that the step fits the aligned window, and
  // every point the block runs together in one aligned 4,096-point group, so
  // that the constant row is theirs.  The low
  // rows are 16-byte asynchronous global-to-shared transfers (four dimensions
  // of one row each; an aligned quad never crosses the 256-dimension wrap),
  // all in flight at once while the constant row is computed, then one wait.
  __device__ __forceinline__ void at_step(uint32_t d0, uint32_t count) {
    if (win_first != 0xFFFFFFFFu && d0 >= win_first && d0 + count <= win_first + kSobolWindow) return;
    __syncthreads();
    const uint32_t w0 = d0 & ~3u;
    constexpr uint32_t kQuadsPerRow = kSobolWindow / 4;
    const uint32_t win_s = (uint32_t)__cvta_generic_to_shared(win);
    for (uint32_t i = threadIdx.x; i < kSobolLowRows * kQuadsPerRow; i += blockDim.x) {
      const uint32_t row = i / kQuadsPerRow, j = 4 * (i % kQuadsPerRow);
      const uint32_t* src = rows_global + row * MPC_SOBOL_TABLE_DIMS + ((w0 + j) & (MPC_SOBOL_TABLE_DIMS - 1));
      const uint32_t dst = win_s + 4u * (row * kSobolRowStride + j);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
    }
    for (uint32_t j = threadIdx.x; j < kSobolWindow; j += blockDim.x) {
      const uint32_t d = w0 + j;
      const uint32_t sg = block_seed + d / MPC_SOBOL_TABLE_DIMS;
      // bits 12..31 of the shuffled index of this block's points (its bits
      // below 12 do not reach them)
      const uint32_t hi = nested_uniform_scramble(local & 0xF000u, sg);
      const uint32_t dm = d & (MPC_SOBOL_TABLE_DIMS - 1);
      uint32_t c = 0;
#pragma unroll
      for (int k = kSobolLowNibbles; k < 8; ++k)
        c ^= __ldg(rows_global + (16u * k + ((hi >> (4 * k)) & 0xFu)) * MPC_SOBOL_TABLE_DIMS + dm);
      win[kSobolConstRow * kSobolRowStride + j] = c;
      win[kSobolSeedRow * kSobolRowStride + j] = hash_combine(sg, dm);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    win_first = w0;
  }
  // Loads the quad of dimensions [d0, d0 + 4), d0 a multiple of 4 inside
  // the window (the chunked model loops call it directly).
  __device__ __forceinline__ void quad_load(uint32_t d0) {
    const uint32_t g = d0 / MPC_SOBOL_TABLE_DIMS;
    if (g != group) {
      group = g;
      const uint32_t shuffled = nested_uniform_scramble(local, block_seed + g);
#pragma unroll
      for (int k = 0; k < (int)kSobolLowNibbles; ++k) rows[k] = (16u * k + ((shuffled >> (4 * k)) & 0xFu)) * kSobolRowStride;
    }
    quad = d0 >> 2;
    const uint32_t* base = win + (d0 - win_first);
    const uint4 sd = *reinterpret_cast<const uint4*>(base + kSobolSeedRow * kSobolRowStride);
    s0 = sd.x;
    s1 = sd.y;
    s2 = sd.z;
    s3 = sd.w;
    uint4 a = *reinterpret_cast<const uint4*>(base + kSobolConstRow * kSobolRowStride);
#pragma unroll
    for (int k = 0; k < (int)kSobolLowNibbles; ++k) {
      const uint4 b = *reinterpret_cast<const uint4*>(base + rows[k]);
      a.x ^= b.x;
      a.y ^= b.y;
      a.z ^= b.z;
      a.w ^= b.w;
    }
    x0 = a.x;
    x1 = a.y;
    x2 = a.z;
    x3 = a.w;
  }
  // Scrambled value of dimension d0 + K of the quad loaded at d0.
  template <int K>
  __device__ __forceinline__ uint32_t take(uint32_t) const {
    return __brev(lk_permute(K == 0 ? x0 : K == 1 ? x1 : K == 2 ? x2 : x3, K == 0 ? s0 : K == 1 ? s1 : K == 2 ? s2 : s3));
  }
  template <int K>
  __device__ __forceinline__ float take_u(uint32_t d0) const {
    return sobol_unit_f32_bits(take<K>(d0));
  }
  template <int K>
  __device__ __forceinline__ float take_n(uint32_t d0) const {
    return icdf_sobol_bits(icdf, take<K>(d0));
  }
  template <int K0, int K1>
  __device__ __forceinline__ float2 take_n2(uint32_t d0) const {
    return icdf_sobol_bits2(icdf, take<K0>(d0), take<K1>(d0));
  }
  __device__ __forceinline__ uint32_t sample(uint32_t d) {
    if ((d >> 2) != quad) quad_load(d & ~3u);
    const uint32_t k = d & 3u;
    return __brev(lk_permute((k & 2u) ? ((k & 1u) ? x3 : x2) : ((k & 1u) ? x1 : x0),
                             (k & 2u) ? ((k & 1u) ? s3 : s2) : ((k & 1u) ? s1 : s0)));
  }
  __device__ __forceinline__ float u32(uint32_t d) { return sobol_unit_f32_bits(sample(d)); }
  __device__ __forceinline__ float n32(uint32_t d) { return icdf_sobol_bits(icdf, sample(d)); }
  __device__ __forceinline__ double u64(uint32_t d) { return sobol_unit_f64(sample(d)); }
  __device__ __forceinline__ double n64(uint32_t d) { return icdf_f64(u64(d)); }
};

// Counter-hash normals for the fused kernels: the reference's u32 hashes
// with the short FP32 transform (counter_normal_fast).
template <bool HWCOS>
struct CounterFastT {
  uint32_t seed, unit;
  template <bool FP64>
  __device__ __forceinline__ void begin(const DevReq& q, const SrcCtx&, uint64_t u) {
    seed = q.seed32;
    unit = (uint32_t)u;
  }
  __device__ __forceinline__ void at_step(uint32_t, uint32_t) {}
  __device__ __forceinline__ float n32(uint32_t d) { return counter_normal_fast<HWCOS>(seed, unit, d); }
  __device__ __forceinline__ float u32(uint32_t d) {
    return counter_open01_fast(hash_u32(counter_mix(seed, unit, d, 0u)));
  }
  __device__ __forceinline__ double n64(uint32_t d) { return (double)counter_normal_f32(seed, unit, d); }
  __device__ __forceinline__ double u64(uint32_t d) {
    return (double)counter_open01(hash_u32(counter_mix(seed, unit, d, 0u)));
  }
};

// Sources with the explicit-quad interface (quad_load / take_n / take_u).
template <class S>
constexpr bool kQuadSource = false;
template <>
constexpr bool kQuadSource<SobolQuad> = true;

template <int SMP>
struct FusedSource {
  using type = Source<SMP>;
};
template <>
struct FusedSource<SMP_SOBOL> {
  using type = SobolQuad;
};
template <>
struct FusedSource<SMP_COUNTER> {
  using type = CounterFastT<false>;
};
// Per family: the single-asset GBM families (one normal per step, the MUFU
// pipe about a third busy) take the hardware cosine; the others keep the
// polynomial.
template <int FAM, int SMP>
struct FusedUnitSource {
  using type = typename FusedSource<SMP>::type;
};
template <int FAM>
struct FusedUnitSource<FAM, SMP_COUNTER> {
  using type = CounterFastT<FAM == FAM_GBM_STEP || FAM == FAM_GBM_TERMINAL>;
};

// Reads materialised samples [dim][unit] (FP64 plain path).
struct BufSource {
  const double* buf;
  uint64_t n_units, unit;
  __device__ __forceinline__ void at_step(uint32_t, uint32_t) {}
  __device__ __forceinline__ double n64(uint32_t d) { return buf[(uint64_t)d * n_units + unit]; }
  __device__ __forceinline__ double u64(uint32_t d) { return buf[(uint64_t)d * n_units + unit]; }
  __device__ __forceinline__ float n32(uint32_t d) { return (float)n64(d); }
  __device__ __forceinline__ float u32(uint32_t d) { return (float)u64(d); }
};

template <class Real, class Src>
__device__ __forceinline__ Real normal(Src& s, uint32_t d) {
  if constexpr (sizeof(Real) == 4)
    return s.n32(d);
  else
    return s.n64(d);
}

template <class Real>
__device__ __forceinline__ Real ex(Real x) {
  if constexpr (sizeof(Real) == 4)
    return __expf(x);
  else
    return exp(x);
}
__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
template <class Real>
__device__ __forceinline__ Real sq_root(Real x) {
  if constexpr (sizeof(Real) == 4)
    return sqrt_approx(x);
  else
    return sqrt(x);
}

// sample_poisson by inversion with the uniform supplied (cpu.rs:932-953),
// entered only when u > exp(-mean) (at least one jump); p0 = exp(-mean) is
// precomputed on the host.
__device__ __forceinline__ uint32_t poisson_tail(double u, double mean, double p0) {
  double prob = p0, cum = p0;
  uint32_t k = 0;
  while (u > cum && k < 4095u) {
    ++k;
    prob *= mean / (double)k;
    cum += prob;
  }
  return k;
}

// ------------------------------------------------------- Brownian bridge ---
// fill_step_normals_from_inputs (cpu.rs:5964-5981) as a streaming walk: the
// reference fills w[0..n] op by op and then differences it; here the same
// ops run in the same (depth-first) order, but only the right endpoints still
// needed stay on a small stack, and each leaf yields the next step's
// increment (w[s] - w[s-1]) / sqrt(dt) at once.  Input dimensions are drawn in
// increasing order (0 = W(T), then one per op), every thread of a request
// runs the same event sequence, so block-synchronous sources stay in lockstep.
// FP64 keeps the reference's two-rounding products and left-to-right sums.
template <class Real>
struct BridgeWalk {
  Real stack[kBridgeDepth];
  Real w_left;
  uint32_t sp, ev, op, dim;

  __device__ __forceinline__ static Real mid(Real lw, Real wl, Real rw, Real wr, Real sd, Real z) {
    if constexpr (sizeof(Real) == 8)
      return __dadd_rn(__dadd_rn(__dmul_rn(lw, wl), __dmul_rn(rw, wr)), __dmul_rn(sd, z));
    else
      return lw * wl + rw * wr + sd * z;
  }
  template <class Src>
  __device__ __forceinline__ void begin(const DevReq& q, Src& src) {
    src.at_step(0, 1);
    const Real z0 = normal<Real>(src, 0);
    if constexpr (sizeof(Real) == 8)
      stack[0] = __dmul_rn(q.bridge_sqrt_t, z0);
    else
      stack[0] = (Real)q.bridge_sqrt_t * z0;
    sp = 1;
    w_left = (Real)0;
    ev = 0;
    op = 0;
    dim = 1;
  }
  // The increment of the next step (the host checked the program: it ends
  // every op run with a leaf and never needs more than kBridgeDepth values).
  template <class Src>
  __device__ __forceinline__ Real next(const DevReq& q, Src& src) {
    for (;;) {
      const uint32_t is_op = (__ldg(q.bridge_events + (ev >> 5)) >> (ev & 31)) & 1u;
      ++ev;
      if (!is_op) break;
      const double* o = q.bridge_ops + 3 * op;
      ++op;
      src.at_step(dim, 1);
      const Real z = normal<Real>(src, dim);
      ++dim;
      const Real wr = stack[sp - 1];
      stack[sp] = mid((Real)__ldg(o), w_left, (Real)__ldg(o + 1), wr, (Real)__ldg(o + 2), z);
      ++sp;
    }
    --sp;
    const Real wr = stack[sp];
    Real inc;
    if constexpr (sizeof(Real) == 8)
      inc = __dmul_rn(__dsub_rn(wr, w_left), q.bridge_inv_sqrt_dt);
    else
      inc = (wr - w_left) * (Real)q.bridge_inv_sqrt_dt;
    w_left = wr;
    return inc;
  }
};

// ------------------------------------------------------------- models -----
// GBM stepwise with the payoff observer of workload W (cpu.rs:6443-6591,
// 7973-8009, 8324-8354; up-and-out mirrors down-and-out).  FP32 compares the
// barrier in log space; FP64 compares exp(log S) with the barrier as the
// reference does.
template <class Real, int W, class Src, bool BRIDGE = false>
__device__ __forceinline__ void unit_gbm_step(const DevReq& q, Src& src, double& pay, double& ctl) {
  const Real drift = (Real)q.drift_dt, vol = (Real)q.vol_dt, kk = (Real)q.k, disc = (Real)q.discount;
  const Real lbar = (Real)q.log_barrier, bar = (Real)q.barrier;
  const bool anti = q.anti != 0;
  Real ls0 = (Real)q.log_s0, ls1 = ls0;
  Real acc0 = (W == W_LOOKBACK) ? (Real)q.s0 : (Real)0, acc1 = acc0;
  bool ko0 = (W == W_DAO && q.s0 <= q.barrier) || (W == W_UAO && q.s0 >= q.barrier), ko1 = ko0;
  const uint32_t n = q.n_steps;
  auto advance = [&](const Real z) {
    ls0 += drift + vol * z;
    if (anti) ls1 += drift - vol * z;
    if constexpr (W == W_ASIAN) {
      acc0 += ex<Real>(ls0);
      if (anti) acc1 += ex<Real>(ls1);
    } else if constexpr (W == W_LOOKBACK) {
      acc0 = acc0 > ex<Real>(ls0) ? acc0 : ex<Real>(ls0);
      if (anti) acc1 = acc1 > ex<Real>(ls1) ? acc1 : ex<Real>(ls1);
    } else if constexpr (W == W_DAO) {
      if constexpr (sizeof(Real) == 4) {
        ko0 |= ls0 <= lbar;
        if (anti) ko1 |= ls1 <= lbar;
      } else {
        ko0 |= ex<Real>(ls0) <= bar;
        if (anti) ko1 |= ex<Real>(ls1) <= bar;
      }
    } else if constexpr (W == W_UAO) {
      if constexpr (sizeof(Real) == 4) {
        ko0 |= ls0 >= lbar;
        if (anti) ko1 |= ls1 >= lbar;
      } else {
        ko0 |= ex<Real>(ls0) >= bar;
        if (anti) ko1 |= ex<Real>(ls1) >= bar;
      }
    }
  };
  uint32_t s = 0;
  if constexpr (BRIDGE) {  // increments from the Brownian bridge over the inputs
    BridgeWalk<Real> bw;
    bw.begin(q, src);
    for (; s < n; ++s) advance(bw.next(q, src));
  } else if constexpr (kQuadSource<Src>) {
    for (; s + 4 <= n; s += 4) {  // four steps per quad of dimensions
      src.at_step(s, 4);
      src.quad_load(s);
      const float2 z01 = src.template take_n2<0, 1>(s), z23 = src.template take_n2<2, 3>(s);
      advance(z01.x);
      advance(z01.y);
      advance(z23.x);
      advance(z23.y);
    }
  }
  for (; s < n; ++s) {
    src.at_step(s, 1);
    advance(normal<Real>(src, s));
  }
  auto payoff = [&](Real ls, Real acc, bool ko) -> Real {
    Real v;
    if constexpr (W == W_ASIAN) {
      if constexpr (sizeof(Real) == 4)
        v = acc * (Real)(1.0 / (double)n) - kk;
      else
        v = acc / (Real)n - kk;
    } else if constexpr (W == W_LOOKBACK) {
      v = acc - kk;
    } else {
      v = ex<Real>(ls) - kk;
      if (ko) v = 0;
    }
    return (v > (Real)0 ? v : (Real)0) * disc;
  };
  Real p0 = payoff(ls0, acc0, ko0);
  if (anti) {
    Real p1 = payoff(ls1, acc1, ko1);
    pay = 0.5 * ((double)p0 + (double)p1);
  } else {
    pay = (double)p0;
  }
  ctl = (double)(disc * ex<Real>(ls0));
}

// GBM terminal European (european_call_payoff_from_shock, cpu.rs:7773-7783).
template <class Real, class Src>
__device__ __forceinline__ void unit_gbm_terminal(const DevReq& q, Src& src, double& pay, double& ctl) {
  src.at_step(0, 1);
  const Real z = normal<Real>(src, 0);
  const Real s0 = (Real)q.s0, drift = (Real)q.drift_dt, vol = (Real)q.vol_dt, kk = (Real)q.k,
             disc = (Real)q.discount;
  Real st = s0 * ex<Real>(drift + vol * z);
  Real p = (st - kk > (Real)0 ? st - kk : (Real)0) * disc;
  if (q.anti) {
    Real sb = s0 * ex<Real>(drift + vol * (-z));
    Real pb = (sb - kk > (Real)0 ? sb - kk : (Real)0) * disc;
    pay = 0.5 * ((double)p + (double)pb);
  } else {
    pay = (double)p;
  }
  ctl = (double)(disc * st);
}

// Heston Euler with the variance floored after every step (heston_path_terminal, cpu.rs:8667-8686).
template <class Real, class Src>
__device__ __forceinline__ void unit_heston(const DevReq& q, Src& src, double& pay, double& ctl) {
  const Real kappa = (Real)q.kappa, theta = (Real)q.theta, xi = (Real)q.xi, rho = (Real)q.rho,
             rho_perp = (Real)q.rho_perp, dt = (Real)q.dt, sqdt = (Real)q.sqrt_dt, rate = (Real)q.rate;
  const bool anti = q.anti != 0;
  Real ls0 = (Real)q.log_s0, ls1 = ls0, v0 = (Real)q.v0, v1 = v0;
  const uint32_t n = q.n_steps;
  // FP32 path: the same update with the step constants folded on the host
  // (rate dt, dt / 2, kappa dt, kappa theta dt, xi sqrt(dt)) and FMAs; the
  // variance is floored after every step and starts >= 0 (validated), so it
  // needs no floor before use.  The FP64 path keeps the reference's form.
  // (Rearranged into fewer instructions -- the drift of all steps folded into
  // the start, 1 - kappa dt, rho sqrt(dt) -- it measured 2.5% slower: two
  // dependent FMAs on the log-price per step instead of one add.)
  const float c_rdt = (float)(q.rate * q.dt), c_hdt = (float)(0.5 * q.dt), c_kdt = (float)(q.kappa * q.dt),
              c_ktdt = (float)(q.kappa * q.theta * q.dt), c_xsq = (float)(q.xi * q.sqrt_dt);
  auto step_f32 = [&](float& ls, float& v, const float zv, const float zi) {
    const float sv = sqrt_approx(v);
    const float zp = fmaf(rho, zv, rho_perp * zi);
    ls += fmaf(sv * sqdt, zp, fmaf(-c_hdt, v, c_rdt));
    const float vn = fmaf(c_xsq * sv, zv, v + fmaf(-c_kdt, v, c_ktdt));
    v = vn > 0.0f ? vn : 0.0f;
  };
  auto step = [&](const Real zv, const Real zi) {
    if constexpr (sizeof(Real) == 4) {
      step_f32(ls0, v0, zv, zi);
      if (anti) step_f32(ls1, v1, -zv, -zi);
      return;
    }
    {
      Real vp = v0 > (Real)0 ? v0 : (Real)0;
      Real sv = sq_root<Real>(vp);
      Real zp = rho * zv + rho_perp * zi;
      ls0 += (rate - (Real)0.5 * vp) * dt + sv * sqdt * zp;
      v0 = v0 + kappa * (theta - vp) * dt + xi * sv * sqdt * zv;
      v0 = v0 > (Real)0 ? v0 : (Real)0;
    }
    if (anti) {
      Real vp = v1 > (Real)0 ? v1 : (Real)0;
      Real sv = sq_root<Real>(vp);
      Real zp = rho * (-zv) + rho_perp * (-zi);
      ls1 += (rate - (Real)0.5 * vp) * dt + sv * sqdt * zp;
      v1 = v1 + kappa * (theta - vp) * dt + xi * sv * sqdt * (-zv);
      v1 = v1 > (Real)0 ? v1 : (Real)0;
    }
  };
  uint32_t s = 0;
  if constexpr (kQuadSource<Src>) {
    for (; s + 2 <= n; s += 2) {  // two steps per quad: dimensions 2s .. 2s + 3
      const uint32_t d0 = 2 * s;
      src.at_step(d0, 4);
      src.quad_load(d0);
      const float2 z01 = src.template take_n2<0, 1>(d0), z23 = src.template take_n2<2, 3>(d0);
      step(z01.x, z01.y);
      step(z23.x, z23.y);
    }
  }
  for (; s < n; ++s) {
    src.at_step(2 * s, 2);
    const Real zv = normal<Real>(src, 2 * s);
    const Real zi = normal<Real>(src, 2 * s + 1);
    step(zv, zi);
  }
  const Real kk = (Real)q.k, disc = (Real)q.discount;
  Real st = ex<Real>(ls0);
  Real p = (st - kk > (Real)0 ? st - kk : (Real)0) * disc;
  if (anti) {
    Real sb = ex<Real>(ls1);
    Real pb = (sb - kk > (Real)0 ? sb - kk : (Real)0) * disc;
    pay = 0.5 * ((double)p + (double)pb);
  } else {
    pay = (double)p;
  }
  ctl = (double)(st * disc);
}

// Merton: stepwise extension (z, u, z_J per step) and the reference terminal
// form (cpu.rs:6408-6441) with dims (z, u, z_J).
template <class Real, bool STEP, class Src>
__device__ __forceinline__ void unit_merton(const DevReq& q, Src& src, double& pay, double& ctl) {
  const Real drift = (Real)q.drift_dt, vol = (Real)q.vol_dt, jm = (Real)q.jump_mean, jv = (Real)q.jump_vol;
  Real ls = (Real)q.log_s0;
  const uint32_t n = STEP ? q.n_steps : 1;
  uint32_t s0 = 0;
  // The FP32 Sobol path adds the deterministic drift of all n steps to the
  // start (only the terminal log-price is read), so a step is one FMA.
  if constexpr (kQuadSource<Src>) ls = (float)(q.log_s0 + q.drift_dt * (double)n);
  if constexpr (kQuadSource<Src>) {
    // four steps per three quads: step k of the chunk uses dimensions
    // d0 + 3k (z), d0 + 3k + 1 (Poisson uniform), d0 + 3k + 2 (jump normal)
    // xu: the scrambled 32-bit Poisson sample; its top 23 bits against the
    // integer thresholds give the jump count of sample_poisson exactly (the
    // FP64 inversion only from four jumps on)
    // (xu >> 9) >= m0 exactly when xu >= m0 << 9 (m0 < 2^23): the shift
    // leaves the common no-jump case
    const uint32_t pois_x0 = q.pois_m[0] << 9;
    auto step = [&](const float z, const uint32_t xu, auto&& jump_normal) {
      ls = fmaf(vol, z, ls);
      if (xu >= pois_x0) {
        const uint32_t mu = xu >> 9;
        uint32_t jumps = 1u + (mu >= q.pois_m[1] ? 1u : 0u) + (mu >= q.pois_m[2] ? 1u : 0u) + (mu >= q.pois_m[3] ? 1u : 0u);
        if (jumps == 4u) jumps = poisson_tail((double)sobol_unit_f32_bits(xu), q.lam_dt, q.lam_p0);
        ls += (Real)jumps * jm + jv * sq_root<Real>((Real)jumps) * jump_normal();
      }
    };
    for (; s0 + 4 <= n; s0 += 4) {
      const uint32_t d0 = 3 * s0;
      src.at_step(d0, 12);
      src.quad_load(d0);
      const float z0 = src.template take_n<0>(d0);
      const uint32_t u0 = src.template take<1>(d0);
      step(z0, u0, [&] { return src.template take_n<2>(d0); });
      const float z1 = src.template take_n<3>(d0);
      src.quad_load(d0 + 4);
      const uint32_t u1 = src.template take<0>(d0 + 4);
      step(z1, u1, [&] { return src.template take_n<1>(d0 + 4); });
      const float z2 = src.template take_n<2>(d0 + 4);
      const uint32_t u2 = src.template take<3>(d0 + 4);
      src.quad_load(d0 + 8);
      step(z2, u2, [&] { return src.template take_n<0>(d0 + 8); });
      step(src.template take_n<1>(d0 + 8), src.template take<2>(d0 + 8),
           [&] { return src.template take_n<3>(d0 + 8); });
    }
  }
  for (uint32_t s = s0; s < n; ++s) {
    src.at_step(3 * s, 3);
    const Real z = normal<Real>(src, 3 * s);
    uint32_t jumps;
    if constexpr (sizeof(Real) == 4) {
      const float u = src.u32(3 * s + 1);
      jumps = u <= q.lam_p0_f ? 0u : poisson_tail((double)u, q.lam_dt, q.lam_p0);
    } else {
      const double u = src.u64(3 * s + 1);
      jumps = u <= q.lam_p0 ? 0u : poisson_tail(u, q.lam_dt, q.lam_p0);
    }
    if constexpr (kQuadSource<Src>)
      ls = fmaf(vol, z, ls);
    else
      ls += drift + vol * z;
    if (jumps > 0) {
      const Real zj = normal<Real>(src, 3 * s + 2);
      ls += (Real)jumps * jm + jv * sq_root<Real>((Real)jumps) * zj;
    }
  }
  const Real kk = (Real)q.k, disc = (Real)q.discount;
  Real st = ex<Real>(ls);
  pay = (double)((st - kk > (Real)0 ? st - kk : (Real)0) * disc);
  ctl = (double)(st * disc);
}

// d-asset basket, terminal or stepwise (basket_terminal_payoff, cpu.rs:7616-7635),
// for a compile-time asset count D: the Cholesky factor and per-asset step
// constants are converted to Real once per unit and kept in registers, and
// every asset loop unrolls without predicates.
template <class Real, int D, class Src>
__device__ __forceinline__ void unit_basket_d(const DevReq& q, Src& src, double& pay, double& ctl) {
  const uint32_t n = q.n_steps;
  const bool anti = q.anti != 0;
  Real L[D][D], dr[D], vo[D], x0[D], x1[D];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    dr[a] = (Real)q.b_drift[a];
    vo[a] = (Real)q.b_vol[a];
    x0[a] = x1[a] = (Real)0;
#pragma unroll
    for (int b = 0; b <= a; ++b) L[a][b] = (Real)q.chol[a * D + b];
  }
  uint32_t dim = 0;
  for (uint32_t s = 0; s < n; ++s) {
    Real z[D];
    src.at_step(dim, D);
#pragma unroll
    for (int a = 0; a < D; ++a) z[a] = normal<Real>(src, dim + a);
    dim += D;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      Real zc = (Real)0;
#pragma unroll
      for (int b = 0; b <= a; ++b) zc += L[a][b] * z[b];
      x0[a] += dr[a] + vo[a] * zc;
      if (anti) x1[a] += dr[a] + vo[a] * (-zc);
    }
  }
  Real b0 = 0, b1 = 0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    b0 += (Real)q.weights[a] * ((Real)q.spots[a] * ex<Real>(x0[a]));
    if (anti) b1 += (Real)q.weights[a] * ((Real)q.spots[a] * ex<Real>(x1[a]));
  }
  const Real kk = (Real)q.k, disc = (Real)q.discount;
  Real p = (b0 - kk > (Real)0 ? b0 - kk : (Real)0) * disc;
  if (anti) {
    Real pb = (b1 - kk > (Real)0 ? b1 - kk : (Real)0) * disc;
    pay = 0.5 * ((double)p + (double)pb);
  } else {
    pay = (double)p;
  }
  ctl = (double)(b0 * disc);
}

template <class Real, class Src>
__device__ __forceinline__ void unit_basket(const DevReq& q, Src& src, double& pay, double& ctl) {
  switch (q.n_assets) {
    case 1:
      unit_basket_d<Real, 1>(q, src, pay, ctl);
      break;
    case 2:
      unit_basket_d<Real, 2>(q, src, pay, ctl);
      break;
    case 3:
      unit_basket_d<Real, 3>(q, src, pay, ctl);
      break;
    case 4:
      unit_basket_d<Real, 4>(q, src, pay, ctl);
      break;
    case 5:
      unit_basket_d<Real, 5>(q, src, pay, ctl);
      break;
    case 6:
      unit_basket_d<Real, 6>(q, src, pay, ctl);
      break;
    case 7:
      unit_basket_d<Real, 7>(q, src, pay, ctl);
      break;
    default:
      unit_basket_d<Real, 8>(q, src, pay, ctl);
      break;
  }
}

// Coupled MLMC level of the arithmetic Asian (cpu.rs:6641-6894): level 0 is
// the plain Asian with the base steps; level l couples M fine normals per
// coarse step with a coarse path driven by sum(z)/sqrt(M).
template <class Real, class Src>
__device__ __forceinline__ void unit_mlmc(const DevReq& q, Src& src, double& pay, double& ctl) {
  const Real kk = (Real)q.k, disc = (Real)q.discount;
  ctl = 0.0;
  if (q.level == 0) {
    const Real drift = (Real)q.f_drift, vol = (Real)q.f_vol;
    Real ls = (Real)q.log_s0, acc = 0;
    for (uint32_t s = 0; s < q.n_steps; ++s) {
      src.at_step(s, 1);
      ls += drift + vol * normal<Real>(src, s);
      acc += ex<Real>(ls);
    }
    Real avg;
    if constexpr (sizeof(Real) == 4)
      avg = acc * (Real)q.inv_fine;
    else
      avg = acc / (Real)q.n_steps;
    pay = (double)((avg - kk > (Real)0 ? avg - kk : (Real)0) * disc);
    return;
  }
  const Real fd = (Real)q.f_drift, fv = (Real)q.f_vol, cd = (Real)q.c_drift, cv = (Real)q.c_vol;
  const uint32_t M = q.refinement;
  Real fl = (Real)q.log_s0, cl = fl, fs = 0, cs = 0;
  uint32_t j = 0;
  for (uint64_t c = 0; c < q.coarse_steps; ++c) {
    Real zsum = 0;
    for (uint32_t m = 0; m < M; ++m) {
      src.at_step(j, 1);  // one dimension at a time: M may exceed what a window step holds
      const Real z = normal<Real>(src, j++);
      zsum += z;
      fl += fd + fv * z;
      fs += ex<Real>(fl);
    }
    Real zc;
    if constexpr (sizeof(Real) == 4)
      zc = zsum * (Real)q.inv_sqrt_m;
    else
      zc = zsum / sqrt((double)M);
    cl += cd + cv * zc;
    cs += ex<Real>(cl);
  }
  Real fa, ca;
  if constexpr (sizeof(Real) == 4) {
    fa = fs * (Real)q.inv_fine;
    ca = cs * (Real)q.inv_coarse;
  } else {
    fa = fs / (Real)q.n_steps;
    ca = cs / (Real)q.coarse_steps;
  }
  Real pf = (fa - kk > (Real)0 ? fa - kk : (Real)0) * disc;
  Real pc = (ca - kk > (Real)0 ? ca - kk : (Real)0) * disc;
  pay = (double)pf - (double)pc;
}

template <class Real, int FAM, class Src>
__device__ __forceinline__ void run_family(const DevReq& q, Src& src, double& p, double& c) {
  if constexpr (FAM == FAM_GBM_BRIDGE) {
    switch (q.workload) {
      case W_ASIAN:
        unit_gbm_step<Real, W_ASIAN, Src, true>(q, src, p, c);
        break;
      case W_DAO:
        unit_gbm_step<Real, W_DAO, Src, true>(q, src, p, c);
        break;
      case W_UAO:
        unit_gbm_step<Real, W_UAO, Src, true>(q, src, p, c);
        break;
      case W_LOOKBACK:
        unit_gbm_step<Real, W_LOOKBACK, Src, true>(q, src, p, c);
        break;
      default:
        unit_gbm_step<Real, W_EURO, Src, true>(q, src, p, c);
        break;
    }
  } else if constexpr (FAM == FAM_GBM_STEP) {
    switch (q.workload) {
      case W_ASIAN:
        unit_gbm_step<Real, W_ASIAN>(q, src, p, c);
        break;
      case W_DAO:
        unit_gbm_step<Real, W_DAO>(q, src, p, c);
        break;
      case W_UAO:
        unit_gbm_step<Real, W_UAO>(q, src, p, c);
        break;
      case W_LOOKBACK:
        unit_gbm_step<Real, W_LOOKBACK>(q, src, p, c);
        break;
      default:
        unit_gbm_step<Real, W_EURO>(q, src, p, c);
        break;
    }
  } else if constexpr (FAM == FAM_GBM_TERMINAL) {
    unit_gbm_terminal<Real>(q, src, p, c);
  } else if constexpr (FAM == FAM_HESTON) {
    unit_heston<Real>(q, src, p, c);
  } else if constexpr (FAM == FAM_MERTON_STEP) {
    unit_merton<Real, true>(q, src, p, c);
  } else if constexpr (FAM == FAM_MERTON_TERMINAL) {
    unit_merton<Real, false>(q, src, p, c);
  } else if constexpr (FAM == FAM_BASKET) {
    unit_basket<Real>(q, src, p, c);
  } else {
    unit_mlmc<Real>(q, src, p, c);
  }
}

template <int FAM, int SMP>
__device__ __forceinline__ void fused_unit(const DevReq& q, const SrcCtx& ctx, uint64_t u, double& p, double& c) {
  typename FusedUnitSource<FAM, SMP>::type src;
  src.template begin<false>(q, ctx, u);
  run_family<float, FAM>(q, src, p, c);
}

template <int SMP>
__device__ __forceinline__ void fused_unit_any(const DevReq& q, const SrcCtx& ctx, uint64_t u, double& p,
                                               double& c) {
  switch (q.family) {
    case FAM_GBM_STEP:
      fused_unit<FAM_GBM_STEP, SMP>(q, ctx, u, p, c);
      break;
    case FAM_GBM_TERMINAL:
      fused_unit<FAM_GBM_TERMINAL, SMP>(q, ctx, u, p, c);
      break;
    case FAM_HESTON:
      fused_unit<FAM_HESTON, SMP>(q, ctx, u, p, c);
      break;
    case FAM_BASKET:
      fused_unit<FAM_BASKET, SMP>(q, ctx, u, p, c);
      break;
    case FAM_MLMC_LEVEL:
      fused_unit<FAM_MLMC_LEVEL, SMP>(q, ctx, u, p, c);
      break;
    case FAM_GBM_BRIDGE:
      if constexpr (SMP == SMP_SOBOL)
        fused_unit<FAM_GBM_BRIDGE, SMP>(q, ctx, u, p, c);
      else
        p = c = 0.0;
      break;
    default:
      if constexpr (SMP != SMP_XORSHIFT) {
        if (q.family == FAM_MERTON_STEP)
          fused_unit<FAM_MERTON_STEP, SMP>(q, ctx, u, p, c);
        else
          fused_unit<FAM_MERTON_TERMINAL, SMP>(q, ctx, u, p, c);
      } else {
        p = c = 0.0;
      }
      break;
  }
}

// ----------------------------------------------------- block reduction ----
constexpr int kFusedBlock = 256;
constexpr int kWarps = kFusedBlock / 32;
// The fused pricing kernel runs 128-, 256- or 512-thread blocks (the
// autotuner's choice); its launch bounds are written for 512 threads.
constexpr int kMaxFusedBlock = 512;
constexpr int kMaxWarps = kMaxFusedBlock / 32;

// Reduces v[0..4] over the block in a fixed order; result valid in thread 0.
// The leading barrier keeps a previous call's reader of `red` safe, so calls
// may follow each other directly.
__device__ __forceinline__ void block_reduce5(double v[5], double (*red)[5]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 5; ++i) v[i] = warp_sum(v[i]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < 5; ++i) red[warp][i] = v[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int warps = (blockDim.x + 31) >> 5;
    for (int i = 0; i < 5; ++i) {
      double s = 0.0;
      for (int w = 0; w < warps; ++w) s += red[w][i];
      v[i] = s;
    }
  }
}

// Sums the request's tile partials in tile order (strided per thread, then a
// fixed block tree) into q.moments.  Called by the block that finished the
// request's last tile.
__device__ void finalize_request(DevReq& q, double (*red)[5]) {
  double acc[5] = {0, 0, 0, 0, 0};
  double cnt = 0.0;
  for (uint32_t t = threadIdx.x; t < q.n_tiles; t += blockDim.x) {
    const double* pt = q.partials + (size_t)t * MPC_MOMENTS;
    cnt += __ldcg(pt + 0);
#pragma unroll
    for (int i = 0; i < 5; ++i) acc[i] += __ldcg(pt + 1 + i);
  }
  double v[5] = {acc[0], acc[1], acc[2], acc[3], acc[4]};
  block_reduce5(v, red);
  double c6[5] = {cnt, 0, 0, 0, 0};
  block_reduce5(c6, red);
  if (threadIdx.x == 0) {
    q.moments[0] = c6[0];
    for (int i = 0; i < 5; ++i) q.moments[1 + i] = v[i];
    q.moments[6] = 0.0;
    q.moments[7] = 0.0;
    *q.tiles_done = 0u;  // reusable without a memset
  }
}

// --------------------------------------------------------- fused kernel ---
// Resident blocks per SM the register allocation must allow: the
// family-switching instance is the widest; the GBM and terminal families
// with the counter-hash generator are long serial chains that want more warps.
constexpr int fused_min_blocks(int fam, int smp) {
  return fam < 0 ? 2 : ((fam == FAM_GBM_STEP || fam == FAM_GBM_TERMINAL) && smp == SMP_COUNTER ? 6 : 4);
}
// The same resident threads per SM (hence the same register budget per
// thread) expressed in 512-thread blocks, for the launch bounds.
constexpr int fused_min_blocks512(int fam, int smp) { return fused_min_blocks(fam, smp) * kFusedBlock / kMaxFusedBlock; }

// One tile of request `sq`: its units through the model, the block's moment
// sums written as the tile's partial, and *s_last (shared) set when this was
// the request's last tile to finish.  Ends with the block synchronised.
// gf2_apply with the nibble table in shared memory.
__device__ __forceinline__ uint64_t gf2_apply_shared(const uint64_t* table, uint64_t x) {
  uint64_t y = 0;
#pragma unroll
  for (int q = 0; q < 16; ++q) y ^= table[q * 16 + ((x >> (4 * q)) & 0xF)];
  return y;
}

// A unit of a single-family fused kernel whose pseudorandom stream is
// already positioned: `aligned` is the chunk stream's state after
// 2 * (idx / 2) draws, idx the unit's first normal in its chunk.
template <int FAM>
__device__ __forceinline__ void fused_unit_stream(const DevReq& q, uint64_t aligned, uint64_t idx, double& p, double& c) {
  Source<SMP_XORSHIFT> src;
  src.st.seek_aligned(aligned, idx, true);
  run_family<float, FAM>(q, src, p, c);
}

template <int FAM, int SMP>
__device__ __forceinline__ void fused_tile(const DevReq& sq, const SrcCtx& ctx, uint32_t tile, double (*red)[5],
                                           int* s_last) {
  const uint64_t first = (uint64_t)tile * sq.tile_units;
  const uint64_t last = min(first + (uint64_t)sq.tile_units, sq.n_units);
  double v[5] = {0, 0, 0, 0, 0};
  const bool cv = sq.cv != 0;
  double* per_unit = sq.per_unit;
  // Every thread runs the same number of units so that block-synchronous
  // sources stay in lockstep; a thread past the tile end repeats the first
  // unit and discards it.
  const uint32_t iters = (uint32_t)((last - first + blockDim.x - 1) / blockDim.x);
  // Pseudorandom streams in a single-family kernel: a thread's units of one
  // tile lie blockDim units apart, so inside one chunk the next unit's
  // stream starts one jump of T^(blockDim x normals per unit) draws later
  // (blockDim is even, so the pair alignment carries over).  The block
  // tabulates that jump in shared memory for the tile (the images of the 64
  // basis vectors, then the nibble table), and each unit after a thread's
  // first in the tile takes 16 lookups instead of a full seek.
  constexpr bool kStride = SMP == SMP_XORSHIFT && FAM >= 0;
  uint64_t* stride_tab = nullptr;
  if constexpr (kStride) {
    __shared__ uint64_t s_cols[64];
    __shared__ uint64_t s_stride[256];
    stride_tab = s_stride;
    if (iters > 1) {
      const uint64_t delta = (uint64_t)blockDim.x * sq.normals_per_unit;
      for (uint32_t i = threadIdx.x; i < 64; i += blockDim.x) s_cols[i] = xorshift_jump(ctx.jump, 1ull << i, delta);
      __syncthreads();
      for (uint32_t e = threadIdx.x; e < 256; e += blockDim.x) {
        uint64_t y = 0;
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j)
          if ((e >> j) & 1u) y ^= s_cols[4 * (e >> 4) + j];
        s_stride[e] = y;
      }
      __syncthreads();
    }
  }
  uint64_t aligned = 0, prev_seed = 0;
  bool chained = false;  // `aligned` holds this thread's previous unit's start in the same tile
  for (uint32_t it = 0; it < iters; ++it) {
    uint64_t u = first + threadIdx.x + (uint64_t)it * blockDim.x;
    const bool valid = u < last;
    if (!valid) u = first + (uint64_t)it * blockDim.x;  // the iteration's first unit: same Sobol index bits 12..31
    double p, c;
    if constexpr (kStride) {
      uint64_t seed, local;
      chunk_of(sq, u, &seed, &local);
      const uint64_t idx = local * sq.normals_per_unit;
      if (chained && valid && seed == prev_seed)
        aligned = gf2_apply_shared(stride_tab, aligned);
      else
        aligned = xorshift_jump(ctx.jump, XorshiftStream::first_state(seed), 2 * (idx >> 1));
      chained = valid;
      prev_seed = seed;
      fused_unit_stream<FAM>(sq, aligned, idx, p, c);
    } else if constexpr (FAM >= 0)
      fused_unit<FAM, SMP>(sq, ctx, u, p, c);
    else
      fused_unit_any<SMP>(sq, ctx, u, p, c);
    if (!valid) continue;
    v[0] += p;
    v[1] += p * p;
    if (cv) {
      v[2] += c;
      v[3] += c * c;
      v[4] += p * c;
    }
    if (per_unit) per_unit[u] = p;
  }
  block_reduce5(v, red);
  if (threadIdx.x == 0) {
    double* pt = sq.partials + (size_t)tile * MPC_MOMENTS;
    pt[0] = (double)(last - first);
    for (int i = 0; i < 5; ++i) pt[1 + i] = v[i];
    __threadfence();
    *s_last = (atomicAdd(sq.tiles_done, 1u) == sq.n_tiles - 1) ? 1 : 0;
  }
  __syncthreads();
}

// FAM >= 0: every request in the list has that family; FAM < 0: switch per tile.
template <int FAM, int SMP>
__global__ void __launch_bounds__(kMaxFusedBlock, fused_min_blocks512(FAM, SMP)) fused_kernel(const DevReq* __restrict__ reqs,
                                                            const Tile* __restrict__ tiles, uint32_t n_tiles,
                                                            uint32_t* __restrict__ counter, SrcCtx ctx) {
  extern __shared__ __align__(16) uint32_t sobol_window[];
  if constexpr (SMP == SMP_SOBOL) {
    // window rows, then the inverse-normal segments (staged once per launch)
    float4* seg = reinterpret_cast<float4*>(sobol_window + kSobolWindowWords);
    const float4* src = reinterpret_cast<const float4*>(ctx.sobol + MPC_ICDF_OFFSET);
    for (uint32_t i = threadIdx.x; i < MPC_ICDF_SEGMENTS; i += blockDim.x) seg[i] = src[i];
    ctx.win = sobol_window;
    ctx.icdf = seg;
  } else {
    ctx.win = nullptr;
    ctx.icdf = nullptr;
  }
  __shared__ DevReq sq;
  __shared__ double red[kMaxWarps][5];
  __shared__ uint32_t s_tile;
  __shared__ int s_last;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    if (t >= n_tiles) break;
    const Tile tl = tiles[t];
    {  // stage the request descriptor in shared memory
      const uint4* src = reinterpret_cast<const uint4*>(reqs + tl.req);
      uint4* dst = reinterpret_cast<uint4*>(&sq);
      for (uint32_t i = threadIdx.x; i < sizeof(DevReq) / sizeof(uint4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    fused_tile<FAM, SMP>(sq, ctx, tl.tile, red, &s_last);
    if (s_last) {
      __threadfence();
      finalize_request(sq, red);
    }
    __syncthreads();
  }
}

template <int SMP>
constexpr size_t fused_dynamic_smem() {
  return SMP == SMP_SOBOL ? kSobolWindowWords * sizeof(uint32_t) + MPC_ICDF_SEGMENTS * sizeof(float4) : 0;
}

template <int FAM, int SMP>
static cudaError_t launch_fused_t(const DevReq* reqs, const Tile* tiles, uint32_t n_tiles, uint32_t* counter,
                                  const SrcCtx& ctx, int grid, int block, cudaStream_t stream) {
  fused_kernel<FAM, SMP><<<grid, block, fused_dynamic_smem<SMP>(), stream>>>(reqs, tiles, n_tiles, counter, ctx);
  count_launch();
  return cudaGetLastError();
}

template <int SMP>
static cudaError_t launch_fused_s(int family, const DevReq* reqs, const Tile* tiles, uint32_t n_tiles,
                                  uint32_t* counter, const SrcCtx& ctx, int grid, int block, cudaStream_t stream) {
  switch (family) {
    case FAM_GBM_STEP:
      return launch_fused_t<FAM_GBM_STEP, SMP>(reqs, tiles, n_tiles, counter, ctx, grid, block, stream);
    case FAM_GBM_TERMINAL:
      return launch_fused_t<FAM_GBM_TERMINAL, SMP>(reqs, tiles, n_tiles, counter, ctx, grid, block, stream);
    case FAM_HESTON:
      return launch_fused_t<FAM_HESTON, SMP>(reqs, tiles, n_tiles, counter, ctx, grid, block, stream);
    case FAM_BASKET:
      return launch_fused_t<FAM_BASKET, SMP>(reqs, tiles, n_tiles, counter, ctx, grid, block, stream);
    case FAM_MLMC_LEVEL:
      return launch_fused_t<FAM_MLMC_LEVEL, SMP>(reqs, tiles, n_tiles, counter, ctx, grid, block, stream);
    case FAM_GBM_BRIDGE:
      if constexpr (SMP == SMP_SOBOL)
        return launch_fused_t<FAM_GBM_BRIDGE, SMP>(reqs, tiles, n_tiles, counter, ctx, grid, block, stream);
      return cudaErrorInvalidValue;
    case FAM_MERTON_STEP:
      if constexpr (SMP != SMP_XORSHIFT)
        return launch_fused_t<FAM_MERTON_STEP, SMP>(reqs, tiles, n_tiles, counter, ctx, grid, block, stream);
      return cudaErrorInvalidValue;
    case FAM_MERTON_TERMINAL:
      if constexpr (SMP != SMP_XORSHIFT)
        return launch_fused_t<FAM_MERTON_TERMINAL, SMP>(reqs, tiles, n_tiles, counter, ctx, grid, block, stream);
      return cudaErrorInvalidValue;
    default:
      return launch_fused_t<-1, SMP>(reqs, tiles, n_tiles, counter, ctx, grid, block, stream);
  }
}

cudaError_t launch_fused(const DevReq* d_reqs, const Tile* d_tiles, uint32_t n_tiles, uint32_t* d_tile_counter,
                         int family, int sampler, const DeviceTables& tabs, int grid, int block,
                         cudaStream_t stream) {
  SrcCtx ctx{tabs.sobol, tabs.jump, nullptr};
  if (block != 128 && block != 256 && block != kMaxFusedBlock) return cudaErrorInvalidValue;
  switch (sampler) {
    case SMP_XORSHIFT:
      return launch_fused_s<SMP_XORSHIFT>(family, d_reqs, d_tiles, n_tiles, d_tile_counter, ctx, grid, block, stream);
    case SMP_HALTON:
      return launch_fused_s<SMP_HALTON>(family, d_reqs, d_tiles, n_tiles, d_tile_counter, ctx, grid, block, stream);
    case SMP_LHS:
      return launch_fused_s<SMP_LHS>(family, d_reqs, d_tiles, n_tiles, d_tile_counter, ctx, grid, block, stream);
    case SMP_SOBOL:
      return launch_fused_s<SMP_SOBOL>(family, d_reqs, d_tiles, n_tiles, d_tile_counter, ctx, grid, block, stream);
    case SMP_COUNTER:
      return launch_fused_s<SMP_COUNTER>(family, d_reqs, d_tiles, n_tiles, d_tile_counter, ctx, grid, block, stream);
    default:
      return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------- resident serving loop ---
__device__ __forceinline__ void st_release_sys(uint32_t* p, uint32_t v) {
  asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t loop_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ LoopEntry loop_entry(const LoopArgs& a, uint32_t pos) {
  const LoopEntry* ep = a.ring + (pos % a.ring_cap);
  LoopEntry e;
  asm volatile("ld.relaxed.gpu.global.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(e.slot), "=r"(e.gen), "=r"(e.n_tiles), "=r"(e.pos)
               : "l"(ep)
               : "memory");
  return e;
}

// 0: the entry at `pos` has no tile left to claim (its claim word has moved
// past its last tile or on to a later request of the slot, or the ring entry
// was reused by a later request, which happens only after it finished);
// otherwise its claim word.
__device__ __forceinline__ unsigned long long loop_open(const LoopArgs& a, const LoopEntry& e, uint32_t pos) {
  if (e.pos != pos || e.slot >= a.max_slots) return 0ull;
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(a.claim + e.slot) : "memory");
  if ((uint32_t)(v >> 32) != e.gen || (uint32_t)v >= e.n_tiles) return 0ull;
  return v;
}

// Thread 0: the next tile to run, or 0 when the block should leave (stop,
// pause, or idle_ns without claimable work).  The live entries are the ring
// positions [cursor, tail) after the exhausted front ones are skipped; each
// claim starts its scan at a position that rotates per block and per claim,
// so concurrent requests share the blocks tile by tile (a large request does
// not hold back the small ones behind it).  The doorbell, ring and claim
// words are device memory read through L2; an idle poll is followed by a
// sleep that doubles up to 4 us.
__device__ __forceinline__ int loop_claim(const LoopArgs& a, uint32_t& cursor, uint32_t& turn, uint32_t* slot,
                                          uint32_t* tile, uint32_t* gen) {
  uint64_t idle_since = 0;
  uint32_t nap = 500;
  for (;;) {
    uint32_t db[4];  // tail, stop, pause and a padding word, read in one load
    asm volatile("ld.acquire.gpu.global.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(db[0]), "=r"(db[1]), "=r"(db[2]), "=r"(db[3])
                 : "l"(a.doorbell)
                 : "memory");
    const uint32_t tail = db[0];
    if (db[1] | db[2]) return 0;  // stop or pause
    while (cursor != tail && loop_open(a, loop_entry(a, cursor), cursor) == 0ull) ++cursor;
    const uint32_t live = tail - cursor;
    const uint32_t first = live ? turn++ % live : 0u;
    for (uint32_t k = 0; k < live; ++k) {
      const uint32_t pos = cursor + (first + k) % live;
      const LoopEntry e = loop_entry(a, pos);
      unsigned long long v = loop_open(a, e, pos);
      for (int tries = 0; v != 0ull && tries < 64; ++tries) {  // bounded: contention leaves the entry for the next pass
        const unsigned long long w = atomicCAS(a.claim + e.slot, v, v + 1ull);
        if (w == v) {
          *slot = e.slot;
          *tile = (uint32_t)v;
          *gen = e.gen;
          return 1;
        }
        v = ((uint32_t)(w >> 32) == e.gen && (uint32_t)w < e.n_tiles) ? w : 0ull;
      }
    }
    const uint64_t now = loop_ns();
    if (idle_since == 0)
      idle_since = now;
    else if (now - idle_since > a.idle_ns)
      return 0;
    __nanosleep(nap);
    nap = nap < 4000u ? 2u * nap : 4000u;
  }
}

// The loop's tile body per sampler, kept out of line so that each sampler's
// register allocation stands on its own.
template <int SMP>
__device__ __noinline__ void loop_tile(const DevReq& sq, const SrcCtx& ctx, uint32_t tile, double (*red)[5],
                                       int* s_last) {
  fused_tile<-1, SMP>(sq, ctx, tile, red, s_last);
}

__global__ void __launch_bounds__(kFusedBlock, 2) serve_loop_kernel(LoopArgs a, SrcCtx ctx) {
  extern __shared__ __align__(16) uint32_t sobol_window[];
  {  // SMs kept free for the host-batched launches
    uint32_t smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    if (smid < a.reserve_sms) return;
  }
  {  // Sobol window rows, then the inverse-normal segments (staged once per launch)
    float4* seg = reinterpret_cast<float4*>(sobol_window + kSobolWindowWords);
    const float4* src = reinterpret_cast<const float4*>(ctx.sobol + MPC_ICDF_OFFSET);
    for (uint32_t i = threadIdx.x; i < MPC_ICDF_SEGMENTS; i += blockDim.x) seg[i] = src[i];
    ctx.win = sobol_window;
    ctx.icdf = seg;
  }
  __shared__ DevReq sq;
  __shared__ double red[kWarps][5];
  __shared__ uint32_t s_slot, s_tile, s_gen, s_go;
  __shared__ int s_last;
  uint32_t cursor = 0;            // thread 0: ring entries before it have no tile left to claim
  uint32_t turn = blockIdx.x;     // thread 0: rotation of the scan start
  for (;;) {
    if (threadIdx.x == 0) s_go = loop_claim(a, cursor, turn, &s_slot, &s_tile, &s_gen);
    __syncthreads();
    if (!s_go) break;
    {  // the slot's descriptor, through L2 (the host rewrites slots between requests)
      const uint4* src = reinterpret_cast<const uint4*>(a.slots + s_slot);
      uint4* dst = reinterpret_cast<uint4*>(&sq);
      for (uint32_t i = threadIdx.x; i < sizeof(DevReq) / sizeof(uint4); i += blockDim.x) dst[i] = __ldcg(src + i);
    }
    __syncthreads();
    switch (sq.sampling) {
      case MPC_SAMPLING_PSEUDORANDOM:
        loop_tile<SMP_XORSHIFT>(sq, ctx, s_tile, red, &s_last);
        break;
      case MPC_SAMPLING_COUNTER_HASH:
        loop_tile<SMP_COUNTER>(sq, ctx, s_tile, red, &s_last);
        break;
      default:  // scrambled Sobol (the host publishes no other sampler)
        loop_tile<SMP_SOBOL>(sq, ctx, s_tile, red, &s_last);
        break;
    }
    if (s_last) {
      __threadfence();
      finalize_request(sq, red);  // moments go to mapped host memory
      if (threadIdx.x == 0) {
        __threadfence_system();
        st_release_sys(a.done + s_slot, s_gen);
      }
    }
    __syncthreads();
  }
}

constexpr size_t kLoopSmem = kSobolWindowWords * sizeof(uint32_t) + MPC_ICDF_SEGMENTS * sizeof(float4);

cudaError_t launch_serve_loop(const LoopArgs& a, const DeviceTables& tabs, int grid, cudaStream_t stream) {
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(serve_loop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kLoopSmem));
  });
  SrcCtx ctx{tabs.sobol, tabs.jump, nullptr, nullptr};
  serve_loop_kernel<<<grid, kFusedBlock, kLoopSmem, stream>>>(a, ctx);
  count_launch();
  return cudaGetLastError();
}

int serve_loop_blocks_per_sm() {
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(serve_loop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kLoopSmem));
  });
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, serve_loop_kernel, kFusedBlock, kLoopSmem);
  return n;
}

template <int FAM, int SMP>
static int occ_t(int block) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fused_kernel<FAM, SMP>, block, fused_dynamic_smem<SMP>());
  return n;
}
template <int SMP>
static int occ_s(int family, int block) {
  switch (family) {
    case FAM_GBM_STEP:
      return occ_t<FAM_GBM_STEP, SMP>(block);
    case FAM_GBM_TERMINAL:
      return occ_t<FAM_GBM_TERMINAL, SMP>(block);
    case FAM_HESTON:
      return occ_t<FAM_HESTON, SMP>(block);
    case FAM_BASKET:
      return occ_t<FAM_BASKET, SMP>(block);
    case FAM_MLMC_LEVEL:
      return occ_t<FAM_MLMC_LEVEL, SMP>(block);
    case FAM_GBM_BRIDGE:
      if constexpr (SMP == SMP_SOBOL) return occ_t<FAM_GBM_BRIDGE, SMP>(block);
      return 1;
    case FAM_MERTON_STEP:
      if constexpr (SMP != SMP_XORSHIFT) return occ_t<FAM_MERTON_STEP, SMP>(block);
      return 1;
    case FAM_MERTON_TERMINAL:
      if constexpr (SMP != SMP_XORSHIFT) return occ_t<FAM_MERTON_TERMINAL, SMP>(block);
      return 1;
    default:
      return occ_t<-1, SMP>(block);
  }
}
int fused_max_blocks_per_sm(int family, int sampler, int block) {
  switch (sampler) {
    case SMP_XORSHIFT:
      return occ_s<SMP_XORSHIFT>(family, block);
    case SMP_HALTON:
      return occ_s<SMP_HALTON>(family, block);
    case SMP_LHS:
      return occ_s<SMP_LHS>(family, block);
    case SMP_SOBOL:
      return occ_s<SMP_SOBOL>(family, block);
    default:
      return occ_s<SMP_COUNTER>(family, block);
  }
}

// Raises a kernel's dynamic shared memory limit to `bytes` once per device
// (the attribute is per device).  Kernels whose Sobol window and
// inverse-normal table (46,592 bytes) plus their static shared memory pass
// the 48 KB default need it before their first launch and occupancy query.
static cudaError_t allow_dynamic_smem(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({fn, dev})) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) done.insert({fn, dev});
  return e;
}

// ------------------------------------------------ scenario (bump) kernel ---
// Bump-and-revalue Greeks with common random numbers: every leg of the
// recipe (base, then up and down per Greek) has the same seed, so every leg
// sees the same normals.  Here one thread draws each normal once and advances
// all legs' paths with it; each leg keeps its own FP32 state and payoff, with
// the same arithmetic as the single-request unit of its family.  Per unit the
// legs' payoffs are warp-summed (FP64 sum and sum of squares) into per-warp
// shared slots; per tile the slots are summed in warp order into tile
// partials [tile][leg][NM], and the last tile sums those in tile order.
// TECH follows the request's technique: antithetic legs also run the mirrored
// path (-z) and record the pair average, as unit_* does; control-variate legs
// also record the discounted terminal price c with sum c, sum c^2 and sum p c
// (NM = 5 moments per leg instead of 2).
// Scenario parameters, struct of arrays [field][kMaxScen] (float):
//   GBM:    log_s0, s0, drift_dt, vol_dt, discount, knocked-out-at-start (0/1)
//   Heston: log_s0, v0, rate, dt, sqrt_dt, discount
constexpr int kScenStd = MPC_TECHNIQUE_STANDARD, kScenAnti = MPC_TECHNIQUE_ANTITHETIC,
              kScenCv = MPC_TECHNIQUE_CONTROL_VARIATE;

template <int W, int TECH, class Src>
__device__ __forceinline__ void scen_gbm_step(const DevReq& q, Src& src, const float* __restrict__ sp, int n_scen,
                                              float pay[kMaxScen], float pay2[kMaxScen], float ctl[kMaxScen]) {
  constexpr bool ANTI = TECH == kScenAnti;
  float ls[kMaxScen], acc[kMaxScen], drift[kMaxScen], vol[kMaxScen];
  float ls2[kMaxScen], acc2[kMaxScen];  // mirrored paths (antithetic)
  bool ko[kMaxScen], ko2[kMaxScen];
#pragma unroll
  for (int s = 0; s < kMaxScen; ++s) {
    ls[s] = __ldg(sp + 0 * kMaxScen + s);
    acc[s] = (W == W_LOOKBACK) ? __ldg(sp + 1 * kMaxScen + s) : 0.0f;
    drift[s] = __ldg(sp + 2 * kMaxScen + s);
    vol[s] = __ldg(sp + 3 * kMaxScen + s);
    ko[s] = __ldg(sp + 5 * kMaxScen + s) != 0.0f;
    if constexpr (ANTI) {
      ls2[s] = ls[s];
      acc2[s] = acc[s];
      ko2[s] = ko[s];
    }
  }
  const float lbar = (float)q.log_barrier;
  const uint32_t n = q.n_steps;
  for (uint32_t st = 0; st < n; ++st) {
    src.at_step(st, 1);
    const float z = normal<float>(src, st);
#pragma unroll
    for (int s = 0; s < kMaxScen; ++s) {
      if (s >= n_scen) break;
      ls[s] += drift[s] + vol[s] * z;
      if constexpr (W == W_ASIAN) acc[s] += __expf(ls[s]);
      else if constexpr (W == W_LOOKBACK) acc[s] = acc[s] > __expf(ls[s]) ? acc[s] : __expf(ls[s]);
      else if constexpr (W == W_DAO) ko[s] |= ls[s] <= lbar;
      else if constexpr (W == W_UAO) ko[s] |= ls[s] >= lbar;
      if constexpr (ANTI) {
        ls2[s] += drift[s] - vol[s] * z;
        if constexpr (W == W_ASIAN) acc2[s] += __expf(ls2[s]);
        else if constexpr (W == W_LOOKBACK) acc2[s] = acc2[s] > __expf(ls2[s]) ? acc2[s] : __expf(ls2[s]);
        else if constexpr (W == W_DAO) ko2[s] |= ls2[s] <= lbar;
        else if constexpr (W == W_UAO) ko2[s] |= ls2[s] >= lbar;
      }
    }
  }
  const float kk = (float)q.k, inv_n = (float)(1.0 / (double)n);
  auto payoff = [&](float l, float a, bool out, float disc) {
    float v;
    if constexpr (W == W_ASIAN) v = a * inv_n - kk;
    else if constexpr (W == W_LOOKBACK) v = a - kk;
    else {
      v = __expf(l) - kk;
      if (out) v = 0.0f;
    }
    return (v > 0.0f ? v : 0.0f) * disc;
  };
#pragma unroll
  for (int s = 0; s < kMaxScen; ++s) {
    const float disc = __ldg(sp + 4 * kMaxScen + s);
    pay[s] = payoff(ls[s], acc[s], ko[s], disc);
    if constexpr (ANTI) pay2[s] = payoff(ls2[s], acc2[s], ko2[s], disc);
    if constexpr (TECH == kScenCv) ctl[s] = disc * __expf(ls[s]);
  }
}

template <int TECH, class Src>
__device__ __forceinline__ void scen_gbm_terminal(const DevReq& q, Src& src, const float* __restrict__ sp, int n_scen,
                                                  float pay[kMaxScen], float pay2[kMaxScen], float ctl[kMaxScen]) {
  src.at_step(0, 1);
  const float z = normal<float>(src, 0);
  const float kk = (float)q.k;
#pragma unroll
  for (int s = 0; s < kMaxScen; ++s) {
    const float s0 = __ldg(sp + 1 * kMaxScen + s), drift = __ldg(sp + 2 * kMaxScen + s),
                vol = __ldg(sp + 3 * kMaxScen + s), disc = __ldg(sp + 4 * kMaxScen + s);
    const float st = s0 * __expf(drift + vol * z);
    pay[s] = (st - kk > 0.0f ? st - kk : 0.0f) * disc;
    if constexpr (TECH == kScenAnti) {
      const float sb = s0 * __expf(drift + vol * (-z));
      pay2[s] = (sb - kk > 0.0f ? sb - kk : 0.0f) * disc;
    }
    if constexpr (TECH == kScenCv) ctl[s] = disc * st;
  }
  (void)n_scen;
}

template <int TECH, class Src>
__device__ __forceinline__ void scen_heston(const DevReq& q, Src& src, const float* __restrict__ sp, int n_scen,
                                            float pay[kMaxScen], float pay2[kMaxScen], float ctl[kMaxScen]) {
  constexpr bool ANTI = TECH == kScenAnti;
  const float kappa = (float)q.kappa, theta = (float)q.theta, xi = (float)q.xi, rho = (float)q.rho,
              rho_perp = (float)q.rho_perp;
  float ls[kMaxScen], v[kMaxScen], rate[kMaxScen], dt[kMaxScen], sqdt[kMaxScen];
  float ls2[kMaxScen], v2[kMaxScen];  // mirrored paths (antithetic)
#pragma unroll
  for (int s = 0; s < kMaxScen; ++s) {
    ls[s] = __ldg(sp + 0 * kMaxScen + s);
    v[s] = __ldg(sp + 1 * kMaxScen + s);
    rate[s] = __ldg(sp + 2 * kMaxScen + s);
    dt[s] = __ldg(sp + 3 * kMaxScen + s);
    sqdt[s] = __ldg(sp + 4 * kMaxScen + s);
    if constexpr (ANTI) {
      ls2[s] = ls[s];
      v2[s] = v[s];
    }
  }
  auto step = [&](float& l, float& var, int s, float zp, float zv) {
    const float vp = var > 0.0f ? var : 0.0f;
    const float sv = sqrt_approx(vp);
    l += (rate[s] - 0.5f * vp) * dt[s] + sv * sqdt[s] * zp;
    var = var + kappa * (theta - vp) * dt[s] + xi * sv * sqdt[s] * zv;
    var = var > 0.0f ? var : 0.0f;
  };
  const uint32_t n = q.n_steps;
  for (uint32_t st = 0; st < n; ++st) {
    src.at_step(2 * st, 2);
    const float zv = normal<float>(src, 2 * st);
    const float zi = normal<float>(src, 2 * st + 1);
    const float zp = rho * zv + rho_perp * zi;
#pragma unroll
    for (int s = 0; s < kMaxScen; ++s) {
      if (s >= n_scen) break;
      step(ls[s], v[s], s, zp, zv);
      if constexpr (ANTI) step(ls2[s], v2[s], s, rho * (-zv) + rho_perp * (-zi), -zv);
    }
  }
  const float kk = (float)q.k;
#pragma unroll
  for (int s = 0; s < kMaxScen; ++s) {
    const float disc = __ldg(sp + 5 * kMaxScen + s);
    const float stv = __expf(ls[s]);
    pay[s] = (stv - kk > 0.0f ? stv - kk : 0.0f) * disc;
    if constexpr (ANTI) {
      const float sb = __expf(ls2[s]);
      pay2[s] = (sb - kk > 0.0f ? sb - kk : 0.0f) * disc;
    }
    if constexpr (TECH == kScenCv) ctl[s] = stv * disc;
  }
}

template <int FAM, int TECH, class Src>
__device__ __forceinline__ void scen_unit(const DevReq& q, Src& src, int n_scen, float pay[kMaxScen],
                                          float pay2[kMaxScen], float ctl[kMaxScen]) {
  const float* sp = q.scen;
  if constexpr (FAM == FAM_HESTON) {
    scen_heston<TECH>(q, src, sp, n_scen, pay, pay2, ctl);
  } else if constexpr (FAM == FAM_GBM_TERMINAL) {
    scen_gbm_terminal<TECH>(q, src, sp, n_scen, pay, pay2, ctl);
  } else {
    switch (q.workload) {
      case W_ASIAN:
        scen_gbm_step<W_ASIAN, TECH>(q, src, sp, n_scen, pay, pay2, ctl);
        break;
      case W_DAO:
        scen_gbm_step<W_DAO, TECH>(q, src, sp, n_scen, pay, pay2, ctl);
        break;
      case W_UAO:
        scen_gbm_step<W_UAO, TECH>(q, src, sp, n_scen, pay, pay2, ctl);
        break;
      case W_LOOKBACK:
        scen_gbm_step<W_LOOKBACK, TECH>(q, src, sp, n_scen, pay, pay2, ctl);
        break;
      default:
        scen_gbm_step<W_EURO, TECH>(q, src, sp, n_scen, pay, pay2, ctl);
        break;
    }
  }
}

// One request (reqs[0]) split into n_tiles tiles of q.tile_units units.
template <int FAM, int SMP, int TECH>
__global__ void __launch_bounds__(kFusedBlock, 2) scenario_kernel(const DevReq* __restrict__ reqs, uint32_t n_tiles,
                                                                 uint32_t* __restrict__ counter, SrcCtx ctx) {
  constexpr int NM = TECH == kScenCv ? 5 : 2;  // moments per leg
  extern __shared__ __align__(16) uint32_t sobol_window[];
  if constexpr (SMP == SMP_SOBOL) {
    float4* seg = reinterpret_cast<float4*>(sobol_window + kSobolWindowWords);
    const float4* src = reinterpret_cast<const float4*>(ctx.sobol + MPC_ICDF_OFFSET);
    for (uint32_t i = threadIdx.x; i < MPC_ICDF_SEGMENTS; i += blockDim.x) seg[i] = src[i];
    ctx.win = sobol_window;
    ctx.icdf = seg;
  } else {
    ctx.win = nullptr;
    ctx.icdf = nullptr;
  }
  __shared__ DevReq sq;
  __shared__ double slots[kWarps][kMaxScen][NM];
  __shared__ uint32_t s_tile;
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    if (t >= n_tiles) break;
    {
      const uint4* src = reinterpret_cast<const uint4*>(reqs);
      uint4* dst = reinterpret_cast<uint4*>(&sq);
      for (uint32_t i = threadIdx.x; i < sizeof(DevReq) / sizeof(uint4); i += blockDim.x) dst[i] = src[i];
    }
    for (uint32_t i = threadIdx.x; i < kWarps * kMaxScen * NM; i += blockDim.x) (&slots[0][0][0])[i] = 0.0;
    __syncthreads();
    const int n_scen = (int)sq.n_scen;
    const uint64_t first = (uint64_t)t * sq.tile_units;
    const uint64_t last = min(first + (uint64_t)sq.tile_units, sq.n_units);
    const uint32_t iters = (uint32_t)((last - first + blockDim.x - 1) / blockDim.x);
    for (uint32_t it = 0; it < iters; ++it) {
      uint64_t u = first + threadIdx.x + (uint64_t)it * blockDim.x;
      const bool valid = u < last;
      if (!valid) u = first + (uint64_t)it * blockDim.x;  // lockstep for block-synchronous sources; discarded below
      typename FusedUnitSource<FAM, SMP>::type src;  // the samples fused_unit<FAM, SMP> draws
      src.template begin<false>(sq, ctx, u);
      float pay[kMaxScen], pay2[kMaxScen], ctl[kMaxScen];
      scen_unit<FAM, TECH>(sq, src, n_scen, pay, pay2, ctl);
#pragma unroll
      for (int s = 0; s < kMaxScen; ++s) {
        if (s >= n_scen) break;
        double p = (double)pay[s];
        if constexpr (TECH == kScenAnti) p = 0.5 * ((double)pay[s] + (double)pay2[s]);
        if (!valid) p = 0.0;
        const double a = warp_sum(p), b = warp_sum(p * p);
        if constexpr (TECH == kScenCv) {
          const double c = valid ? (double)ctl[s] : 0.0;
          const double cs = warp_sum(c), cc = warp_sum(c * c), pc = warp_sum(p * c);
          if (lane == 0) {
            slots[warp][s][2] += cs;
            slots[warp][s][3] += cc;
            slots[warp][s][4] += pc;
          }
        }
        if (lane == 0) {
          slots[warp][s][0] += a;
          slots[warp][s][1] += b;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x < (uint32_t)(NM * n_scen)) {
      const int s = threadIdx.x / NM, k = threadIdx.x % NM;
      double sum = 0.0;
      for (int w = 0; w < kWarps; ++w) sum += slots[w][s][k];
      sq.partials[((size_t)t * kMaxScen + s) * NM + k] = sum;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(sq.tiles_done, 1u) == n_tiles - 1) ? 1 : 0;
    __syncthreads();
    if (s_last) {
      __threadfence();
      if (threadIdx.x < (uint32_t)(NM * n_scen)) {
        const int s = threadIdx.x / NM, k = threadIdx.x % NM;
        double sum = 0.0;
        for (uint32_t tt = 0; tt < n_tiles; ++tt) sum += __ldcg(sq.partials + ((size_t)tt * kMaxScen + s) * NM + k);
        sq.moments[s * NM + k] = sum;
      }
      if (threadIdx.x == 0) *sq.tiles_done = 0u;
    }
    __syncthreads();
  }
}

using ScenarioKernel = void (*)(const DevReq*, uint32_t, uint32_t*, SrcCtx);
template <int SMP, int TECH>
static ScenarioKernel scenario_kernel_of(int family) {
  switch (family) {
    case FAM_GBM_STEP:
      return scenario_kernel<FAM_GBM_STEP, SMP, TECH>;
    case FAM_GBM_TERMINAL:
      return scenario_kernel<FAM_GBM_TERMINAL, SMP, TECH>;
    case FAM_HESTON:
      return scenario_kernel<FAM_HESTON, SMP, TECH>;
    default:
      return nullptr;
  }
}

template <int SMP, int TECH>
static cudaError_t launch_scen_t(int family, const DevReq* d_req, uint32_t n_tiles, uint32_t* counter,
                                 const SrcCtx& ctx, int grid, cudaStream_t stream) {
  const size_t smem = fused_dynamic_smem<SMP>();
  const ScenarioKernel kernel = scenario_kernel_of<SMP, TECH>(family);
  if (!kernel) return cudaErrorInvalidValue;
  const cudaError_t e = allow_dynamic_smem((const void*)kernel, smem);
  if (e != cudaSuccess) return e;
  kernel<<<grid, kFusedBlock, smem, stream>>>(d_req, n_tiles, counter, ctx);
  count_launch();
  return cudaGetLastError();
}

template <int SMP>
static cudaError_t launch_scen_s(int family, int technique, const DevReq* d_req, uint32_t n_tiles,
                                 uint32_t* counter, const SrcCtx& ctx, int grid, cudaStream_t stream) {
  switch (technique) {
    case kScenStd:
      return launch_scen_t<SMP, kScenStd>(family, d_req, n_tiles, counter, ctx, grid, stream);
    case kScenAnti:
      return launch_scen_t<SMP, kScenAnti>(family, d_req, n_tiles, counter, ctx, grid, stream);
    case kScenCv:
      return launch_scen_t<SMP, kScenCv>(family, d_req, n_tiles, counter, ctx, grid, stream);
    default:
      return cudaErrorInvalidValue;
  }
}

template <int SMP, int TECH>
static int scen_occ_t(int family) {
  int n = 0;
  const size_t smem = fused_dynamic_smem<SMP>();
  const ScenarioKernel kernel = scenario_kernel_of<SMP, TECH>(family);
  if (!kernel || allow_dynamic_smem((const void*)kernel, smem) != cudaSuccess) return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kFusedBlock, smem);
  return n;
}

template <int SMP>
static int scen_occ_s(int family, int technique) {
  if (technique == kScenAnti) return scen_occ_t<SMP, kScenAnti>(family);
  if (technique == kScenCv) return scen_occ_t<SMP, kScenCv>(family);
  return scen_occ_t<SMP, kScenStd>(family);
}

int scenario_max_blocks_per_sm(int family, int sampler, int technique) {
  if (sampler == SMP_XORSHIFT) return scen_occ_s<SMP_XORSHIFT>(family, technique);
  if (sampler == SMP_SOBOL) return scen_occ_s<SMP_SOBOL>(family, technique);
  if (sampler == SMP_COUNTER) return scen_occ_s<SMP_COUNTER>(family, technique);
  return 0;
}

cudaError_t launch_scenarios(const DevReq* d_req, uint32_t n_tiles, uint32_t* d_counter, int family, int sampler,
                             int technique, const DeviceTables& tabs, int grid, cudaStream_t stream) {
  SrcCtx ctx{tabs.sobol, tabs.jump, nullptr};
  switch (sampler) {
    case SMP_XORSHIFT:
      return launch_scen_s<SMP_XORSHIFT>(family, technique, d_req, n_tiles, d_counter, ctx, grid, stream);
    case SMP_SOBOL:
      return launch_scen_s<SMP_SOBOL>(family, technique, d_req, n_tiles, d_counter, ctx, grid, stream);
    case SMP_COUNTER:
      return launch_scen_s<SMP_COUNTER>(family, technique, d_req, n_tiles, d_counter, ctx, grid, stream);
    default:
      return cudaErrorInvalidValue;
  }
}

// ------------------------------------------- basket scenario (bump) kernel ---
// Bump legs of a d-asset basket with common random numbers.  A path draws
// its n_steps x D normals once and keeps only the per-asset sums Z_a; the
// correlated sums are W = L Z (L the Cholesky factor), and leg s prices
//   basket_s = sum_a wspot[s][a] exp(log_drift[s][a] + step_vol[s][a] W_a)
// (basket_terminal_payoff, cpu.rs:7616-7635, with the stepwise log return
// sum_steps (drift_dt + vol_dt zc) regrouped as T drift + vol_dt W).  The
// moment reduction is that of scenario_kernel: per-warp FP64 slots, tile
// partials in warp order, the last tile sums the partials in tile order.
template <int D, class Src>
__device__ __forceinline__ void scen_basket_d(const DevReq& q, Src& src, const BasketScen& legs,
                                              float pay[kBasketScen]) {
  float zs[D];
#pragma unroll
  for (int a = 0; a < D; ++a) zs[a] = 0.0f;
  const uint32_t n = q.n_steps;
  uint32_t dim = 0;
  for (uint32_t st = 0; st < n; ++st) {
    src.at_step(dim, D);
#pragma unroll
    for (int a = 0; a < D; ++a) zs[a] += normal<float>(src, dim + a);
    dim += D;
  }
  float w[D];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    float acc = 0.0f;
#pragma unroll
    for (int b = 0; b <= a; ++b) acc += (float)q.chol[a * D + b] * zs[b];
    w[a] = acc;
  }
  const float kk = (float)q.k;
#pragma unroll
  for (int s = 0; s < kBasketScen; ++s) {
    float basket = 0.0f;
#pragma unroll
    for (int a = 0; a < D; ++a) basket += legs.wspot[s][a] * __expf(legs.log_drift[s][a] + legs.step_vol[s][a] * w[a]);
    pay[s] = (basket - kk > 0.0f ? basket - kk : 0.0f) * legs.discount[s];
  }
}

template <class Src>
__device__ __forceinline__ void scen_basket(const DevReq& q, Src& src, const BasketScen& legs,
                                            float pay[kBasketScen]) {
  switch (q.n_assets) {
    case 1:
      scen_basket_d<1>(q, src, legs, pay);
      break;
    case 2:
      scen_basket_d<2>(q, src, legs, pay);
      break;
    case 3:
      scen_basket_d<3>(q, src, legs, pay);
      break;
    case 4:
      scen_basket_d<4>(q, src, legs, pay);
      break;
    case 5:
      scen_basket_d<5>(q, src, legs, pay);
      break;
    case 6:
      scen_basket_d<6>(q, src, legs, pay);
      break;
    case 7:
      scen_basket_d<7>(q, src, legs, pay);
      break;
    default:
      scen_basket_d<8>(q, src, legs, pay);
      break;
  }
}

// One basket request (reqs[0]) split into n_tiles tiles of q.tile_units units.
template <int SMP>
__global__ void __launch_bounds__(kFusedBlock, 2) basket_scenario_kernel(const DevReq* __restrict__ reqs,
                                                                        uint32_t n_tiles,
                                                                        uint32_t* __restrict__ counter,
                                                                        SrcCtx ctx, const BasketScen legs) {
  extern __shared__ __align__(16) uint32_t sobol_window[];
  if constexpr (SMP == SMP_SOBOL) {
    float4* seg = reinterpret_cast<float4*>(sobol_window + kSobolWindowWords);
    const float4* src = reinterpret_cast<const float4*>(ctx.sobol + MPC_ICDF_OFFSET);
    for (uint32_t i = threadIdx.x; i < MPC_ICDF_SEGMENTS; i += blockDim.x) seg[i] = src[i];
    ctx.win = sobol_window;
    ctx.icdf = seg;
  } else {
    ctx.win = nullptr;
    ctx.icdf = nullptr;
  }
  __shared__ DevReq sq;
  __shared__ double slots[kWarps][kBasketScen][2];
  __shared__ uint32_t s_tile;
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    if (t >= n_tiles) break;
    {
      const uint4* src = reinterpret_cast<const uint4*>(reqs);
      uint4* dst = reinterpret_cast<uint4*>(&sq);
      for (uint32_t i = threadIdx.x; i < sizeof(DevReq) / sizeof(uint4); i += blockDim.x) dst[i] = src[i];
    }
    for (uint32_t i = threadIdx.x; i < kWarps * kBasketScen * 2; i += blockDim.x) (&slots[0][0][0])[i] = 0.0;
    __syncthreads();
    const uint64_t first = (uint64_t)t * sq.tile_units;
    const uint64_t last = min(first + (uint64_t)sq.tile_units, sq.n_units);
    const uint32_t iters = (uint32_t)((last - first + blockDim.x - 1) / blockDim.x);
    for (uint32_t it = 0; it < iters; ++it) {
      uint64_t u = first + threadIdx.x + (uint64_t)it * blockDim.x;
      const bool valid = u < last;
      if (!valid) u = first + (uint64_t)it * blockDim.x;  // lockstep for block-synchronous sources; discarded below
      typename FusedUnitSource<FAM_BASKET, SMP>::type src;  // the samples fused_unit<FAM_BASKET, SMP> draws
      src.template begin<false>(sq, ctx, u);
      float pay[kBasketScen];
      scen_basket(sq, src, legs, pay);
#pragma unroll
      for (int s = 0; s < kBasketScen; ++s) {
        const double p = valid ? (double)pay[s] : 0.0;
        const double a = warp_sum(p), b = warp_sum(p * p);
        if (lane == 0) {
          slots[warp][s][0] += a;
          slots[warp][s][1] += b;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x < (uint32_t)(2 * kBasketScen)) {
      const int s = threadIdx.x >> 1, k = threadIdx.x & 1;
      double sum = 0.0;
      for (int w = 0; w < kWarps; ++w) sum += slots[w][s][k];
      sq.partials[((size_t)t * kBasketScen + s) * 2 + k] = sum;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(sq.tiles_done, 1u) == n_tiles - 1) ? 1 : 0;
    __syncthreads();
    if (s_last) {
      __threadfence();
      if (threadIdx.x < (uint32_t)(2 * kBasketScen)) {
        const int s = threadIdx.x >> 1, k = threadIdx.x & 1;
        double sum = 0.0;
        for (uint32_t tt = 0; tt < n_tiles; ++tt)
          sum += __ldcg(sq.partials + ((size_t)tt * kBasketScen + s) * 2 + k);
        sq.moments[s * 2 + k] = sum;
      }
      if (threadIdx.x == 0) *sq.tiles_done = 0u;
    }
    __syncthreads();
  }
}

template <int SMP>
static cudaError_t launch_basket_scen_s(const DevReq* d_req, uint32_t n_tiles, uint32_t* counter, const SrcCtx& ctx,
                                        const BasketScen& legs, int grid, cudaStream_t stream) {
  const cudaError_t e = allow_dynamic_smem((const void*)basket_scenario_kernel<SMP>, fused_dynamic_smem<SMP>());
  if (e != cudaSuccess) return e;
  basket_scenario_kernel<SMP><<<grid, kFusedBlock, fused_dynamic_smem<SMP>(), stream>>>(d_req, n_tiles, counter, ctx,
                                                                                        legs);
  count_launch();
  return cudaGetLastError();
}

template <int SMP>
static int basket_scen_occ() {
  int n = 0;
  if (allow_dynamic_smem((const void*)basket_scenario_kernel<SMP>, fused_dynamic_smem<SMP>()) != cudaSuccess)
    return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, basket_scenario_kernel<SMP>, kFusedBlock, fused_dynamic_smem<SMP>());
  return n;
}

int basket_scenario_max_blocks_per_sm(int sampler) {
  if (sampler == SMP_XORSHIFT) return basket_scen_occ<SMP_XORSHIFT>();
  if (sampler == SMP_SOBOL) return basket_scen_occ<SMP_SOBOL>();
  if (sampler == SMP_COUNTER) return basket_scen_occ<SMP_COUNTER>();
  return 0;
}

cudaError_t launch_basket_scenarios(const DevReq* d_req, uint32_t n_tiles, uint32_t* d_counter, int sampler,
                                    const BasketScen& legs, const DeviceTables& tabs, int grid, cudaStream_t stream) {
  SrcCtx ctx{tabs.sobol, tabs.jump, nullptr};
  switch (sampler) {
    case SMP_XORSHIFT:
      return launch_basket_scen_s<SMP_XORSHIFT>(d_req, n_tiles, d_counter, ctx, legs, grid, stream);
    case SMP_SOBOL:
      return launch_basket_scen_s<SMP_SOBOL>(d_req, n_tiles, d_counter, ctx, legs, grid, stream);
    case SMP_COUNTER:
      return launch_basket_scen_s<SMP_COUNTER>(d_req, n_tiles, d_counter, ctx, legs, grid, stream);
    default:
      return cudaErrorInvalidValue;
  }
}

// ------------------------------------------------------ FP64 plain path ---
__device__ __forceinline__ bool is_uniform_dim(const DevReq& q, uint32_t d) {
  return (q.family == FAM_MERTON_STEP || q.family == FAM_MERTON_TERMINAL) && (d % 3u) == 1u;
}

template <int SMP>
__global__ void __launch_bounds__(256) plain_generate_kernel(DevReq q, double* __restrict__ buf, SrcCtx ctx) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint32_t dims = (uint32_t)q.normals_per_unit;
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < q.n_units; u += stride) {
    Source<SMP> src;
    src.template begin<true>(q, ctx, u);
    for (uint32_t d = 0; d < dims; ++d) buf[(uint64_t)d * q.n_units + u] = is_uniform_dim(q, d) ? src.u64(d) : src.n64(d);
  }
}

cudaError_t launch_plain_generate(const DevReq& q, double* d_buf, int sampler, const DeviceTables& tabs,
                                  cudaStream_t stream) {
  SrcCtx ctx{tabs.sobol, tabs.jump, nullptr};
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  uint64_t want = (q.n_units + 255) / 256;
  int grid = (int)(want < (uint64_t)sms * 8 ? want : (uint64_t)sms * 8);
  if (grid < 1) grid = 1;
  switch (sampler) {
    case SMP_XORSHIFT:
      plain_generate_kernel<SMP_XORSHIFT><<<grid, 256, 0, stream>>>(q, d_buf, ctx);
      break;
    case SMP_HALTON:
      plain_generate_kernel<SMP_HALTON><<<grid, 256, 0, stream>>>(q, d_buf, ctx);
      break;
    case SMP_LHS:
      plain_generate_kernel<SMP_LHS><<<grid, 256, 0, stream>>>(q, d_buf, ctx);
      break;
    case SMP_SOBOL:
      plain_generate_kernel<SMP_SOBOL><<<grid, 256, 0, stream>>>(q, d_buf, ctx);
      break;
    case SMP_COUNTER:
      plain_generate_kernel<SMP_COUNTER><<<grid, 256, 0, stream>>>(q, d_buf, ctx);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  count_launch();
  return cudaGetLastError();
}

template <int FAM>
__global__ void __launch_bounds__(256) plain_simulate_kernel(const DevReq* __restrict__ qp,
                                                             const double* __restrict__ buf,
                                                             double* __restrict__ payoff,
                                                             double* __restrict__ control) {
  const DevReq& q = *qp;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < q.n_units; u += stride) {
    BufSource src{buf, q.n_units, u};
    double p, c;
    run_family<double, FAM>(q, src, p, c);
    payoff[u] = p;
    if (control) control[u] = c;
  }
}

cudaError_t launch_plain_simulate(const DevReq& q, const DevReq* d_req, const double* d_buf, double* d_payoff,
                                  double* d_control, cudaStream_t stream) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  uint64_t want = (q.n_units + 255) / 256;
  int grid = (int)(want < (uint64_t)sms * 8 ? want : (uint64_t)sms * 8);
  if (grid < 1) grid = 1;
  switch (q.family) {
    case FAM_GBM_STEP:
      plain_simulate_kernel<FAM_GBM_STEP><<<grid, 256, 0, stream>>>(d_req, d_buf, d_payoff, d_control);
      break;
    case FAM_GBM_TERMINAL:
      plain_simulate_kernel<FAM_GBM_TERMINAL><<<grid, 256, 0, stream>>>(d_req, d_buf, d_payoff, d_control);
      break;
    case FAM_HESTON:
      plain_simulate_kernel<FAM_HESTON><<<grid, 256, 0, stream>>>(d_req, d_buf, d_payoff, d_control);
      break;
    case FAM_MERTON_STEP:
      plain_simulate_kernel<FAM_MERTON_STEP><<<grid, 256, 0, stream>>>(d_req, d_buf, d_payoff, d_control);
      break;
    case FAM_MERTON_TERMINAL:
      plain_simulate_kernel<FAM_MERTON_TERMINAL><<<grid, 256, 0, stream>>>(d_req, d_buf, d_payoff, d_control);
      break;
    case FAM_BASKET:
      plain_simulate_kernel<FAM_BASKET><<<grid, 256, 0, stream>>>(d_req, d_buf, d_payoff, d_control);
      break;
    case FAM_GBM_BRIDGE:
      plain_simulate_kernel<FAM_GBM_BRIDGE><<<grid, 256, 0, stream>>>(d_req, d_buf, d_payoff, d_control);
      break;
    default:
      plain_simulate_kernel<FAM_MLMC_LEVEL><<<grid, 256, 0, stream>>>(d_req, d_buf, d_payoff, d_control);
      break;
  }
  count_launch();
  return cudaGetLastError();
}

// Deterministic FP64 reduction of the payoff (and control) buffers in tiles
// of q.tile_units, finalized by the last tile.
__global__ void __launch_bounds__(kFusedBlock) plain_reduce_kernel(DevReq* __restrict__ qp,
                                                                   const double* __restrict__ payoff,
                                                                   const double* __restrict__ control) {
  __shared__ double red[kWarps][5];
  __shared__ int s_last;
  DevReq& q = *qp;
  for (uint32_t t = blockIdx.x; t < q.n_tiles; t += gridDim.x) {
    const uint64_t first = (uint64_t)t * q.tile_units;
    const uint64_t last = min(first + (uint64_t)q.tile_units, q.n_units);
    double v[5] = {0, 0, 0, 0, 0};
    for (uint64_t u = first + threadIdx.x; u < last; u += blockDim.x) {
      const double p = payoff[u];
      v[0] += p;
      v[1] += p * p;
      if (control) {
        const double c = control[u];
        v[2] += c;
        v[3] += c * c;
        v[4] += p * c;
      }
    }
    block_reduce5(v, red);
    if (threadIdx.x == 0) {
      double* pt = q.partials + (size_t)t * MPC_MOMENTS;
      pt[0] = (double)(last - first);
      for (int i = 0; i < 5; ++i) pt[1 + i] = v[i];
      __threadfence();
      s_last = (atomicAdd(q.tiles_done, 1u) == q.n_tiles - 1) ? 1 : 0;
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      finalize_request(q, red);
    }
    __syncthreads();
  }
}

cudaError_t launch_plain_reduce(const DevReq* d_req, const double* d_payoff, const double* d_control,
                                uint64_t n_units, uint32_t n_tiles, cudaStream_t stream) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int grid = (int)(n_tiles < (uint32_t)sms * 4 ? n_tiles : (uint32_t)sms * 4);
  if (grid < 1) grid = 1;
  plain_reduce_kernel<<<grid, kFusedBlock, 0, stream>>>(const_cast<DevReq*>(d_req), d_payoff, d_control);
  count_launch();
  return cudaGetLastError();
}

// ---------------------------------------- reference v1 kernel contract ----
// Same buffers and scalars as mc_cuda_european_call_stepwise_v1
// (european_call_stepwise_v1.cu:1-28): path-major FP64 normals, one path per
// thread, per-path discounted payoff.  Index arithmetic in 64 bits.
__global__ void __launch_bounds__(256) european_call_stepwise_v1_kernel(const double* __restrict__ normals,
                                                                       double* __restrict__ payoffs,
                                                                       int32_t n_paths, int32_t n_steps,
                                                                       double log_s0, double strike,
                                                                       double drift_dt, double vol_dt,
                                                                       double discount) {
  const int64_t path = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (path >= n_paths) return;
  double ls = log_s0;
  const double* z = normals + path * (int64_t)n_steps;
  for (int32_t s = 0; s < n_steps; ++s) ls += drift_dt + vol_dt * z[s];
  const double st = exp(ls);
  payoffs[path] = st > strike ? (st - strike) * discount : 0.0;
}

cudaError_t launch_european_call_stepwise_v1(const double* normals, double* payoffs, int32_t n_paths,
                                             int32_t n_steps, double log_s0, double strike, double drift_dt,
                                             double vol_dt, double discount, cudaStream_t stream) {
  if (n_paths <= 0) return cudaSuccess;
  int grid = (int)((n_paths + 255) / 256);
  european_call_stepwise_v1_kernel<<<grid, 256, 0, stream>>>(normals, payoffs, n_paths, n_steps, log_s0, strike,
                                                              drift_dt, vol_dt, discount);
  count_launch();
  return cudaGetLastError();
}

// ------------------------------------------------------------------ LSM ---
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <class Real>
__device__ __forceinline__ void laguerre4(Real x, Real b[4]) {
  // laguerre_lsm_basis (cpu.rs:7667-7682); degrees above `degree` are unused
  const Real x2 = x * x, x3 = x2 * x;
  b[0] = (Real)1;
  b[1] = (Real)1 - x;
  b[2] = (Real)1 - (Real)2 * x + (Real)0.5 * x2;
  b[3] = (Real)1 - (Real)3 * x + (Real)1.5 * x2 - x3 / (Real)6;
}

// solve_lsm_normal_equations (cpu.rs:7684-7736) for a compile-time size:
// Gauss-Jordan with partial pivoting in FP64, the reference's operations in
// its order, with every index static (the pivot row swap is a predicated exchange), so the
// system stays in registers.
template <int DIM, bool RECIP = false>
__device__ __forceinline__ bool solve_fixed(double a[4][4], double rhs[4]) {
#pragma unroll
  for (int piv = 0; piv < DIM; ++piv) {
    int best = piv;
    double best_abs = fabs(a[piv][piv]);
#pragma unroll
    for (int row = piv + 1; row < DIM; ++row) {
      const double c = fabs(a[row][piv]);
      if (c > best_abs) {
        best = row;
        best_abs = c;
      }
    }
    if (best_abs <= 1e-12) return false;
#pragma unroll
    for (int row = piv + 1; row < DIM; ++row) {
      if (row == best) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const double t = a[piv][c];
          a[piv][c] = a[row][c];
          a[row][c] = t;
        }
        const double t = rhs[piv];
        rhs[piv] = rhs[row];
        rhs[row] = t;
      }
    }
    const double pv = a[piv][piv];
    if constexpr (RECIP) {
      const double ip = 1.0 / pv;
#pragma unroll
      for (int c = piv; c < DIM; ++c) a[piv][c] *= ip;
      rhs[piv] *= ip;
    } else {
#pragma unroll
      for (int c = piv; c < DIM; ++c) a[piv][c] /= pv;
      rhs[piv] /= pv;
    }
#pragma unroll
    for (int row = 0; row < DIM; ++row) {
      if (row == piv) continue;
      const double f = a[row][piv];
      if (f == 0.0) continue;
#pragma unroll
      for (int c = piv; c < DIM; ++c) a[row][c] -= f * a[piv][c];
      rhs[row] -= f * rhs[piv];
    }
  }
  return true;
}


constexpr int kLsmBlock = (int)kLsmThreads;

constexpr int kLsmMaxP = (int)kLsmPathsPerThreadMax;
constexpr int kLsmMom = 15;  // 10 unique A^T A, 4 A^T b, ITM count

// Records the first failed self-check of an LSM job (code and index).
__device__ __noinline__ void lsm_report(const LsmArgs& a, int code, uint64_t index) {
  if (atomicCAS(a.error, 0, code) == 0) *a.diag = (unsigned long long)index;
}
__device__ __forceinline__ bool lsm_ok(const LsmArgs& a, uint64_t index, uint64_t len, int code) {
  if (index < len) return true;
  lsm_report(a, code, index);
  return false;
}

// Warp sums of 16 values per lane by reduce-scatter: in each of four rounds a
// lane keeps half of its values and adds the partner's copy of that half
// (partner lane ^ 16, ^ 8, ^ 4, ^ 2), then lanes l and l ^ 1 add their last
// value.  Lane l ends with the warp sum of value brev4(l >> 1) (lanes l and
// l ^ 1 hold the same bits): 16 double shuffles instead of 80 for 16 separate
// butterflies, in a fixed order.
template <class T>
__device__ __forceinline__ T warp_reduce_scatter16(T (&v)[16]) {
  const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int o = 16 >> r, c = 8 >> r;
    const bool up = (lane & (uint32_t)o) != 0;
#pragma unroll
    for (int i = 0; i < c; ++i) {
      const T send = up ? v[i] : v[i + c];
      const T keep = up ? v[i + c] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}
__device__ __forceinline__ uint32_t reduce_scatter16_index(uint32_t lane) {
  return (((lane >> 4) & 1u) << 3) | (((lane >> 3) & 1u) << 2) | (((lane >> 2) & 1u) << 1) | ((lane >> 1) & 1u);
}

// One exercise date's regression across the job's blocks (round = the date's
// position in the backward pass).  Every block writes its 15 moments to its
// own slot row partials[round][lb] with relaxed stores; the host marks every
// slot empty (all bits set) before the launch and no slot is written twice,
// so the data is its own arrival flag: each block reads every block's slots
// of the round at once and re-reads (bounded) only those still empty, with no
// fence, counter or separate poll between the write and the read.  Then every
// block sums the partials itself in the same fixed order (thread t: moment
// t % 16 over blocks t / 16, t / 16 + 32, ...; the lane groups' sums by
// shuffles, then a fixed shuffle tree per moment over the 16 warps) and solves
// the normal equations in thread 0: the same operations on the same data, so
// every block holds the same coefficients, with no publication round trip
// after the solve.  The FP32 path scales each pivot row by the pivot's
// reciprocal instead of dividing every entry (the FP64 path divides, as the
// reference does).  The wait is bounded: after timeout_ns the block records
// kLsmErrTimeout and every block of the job leaves at its next check.
// Returns false when the job's error flag is set.
// Empty marker of a date's partial slot (all bits set); the host fills the
// partials with it before the launch, and a written value never equals it.
constexpr unsigned long long kLsmEmpty = 0xFFFFFFFFFFFFFFFFull;
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const double* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_f64(double* p, double x) {
  unsigned long long v = (unsigned long long)__double_as_longlong(x);
  if (v == kLsmEmpty) v = 0x7FF8000000000001ull;  // a NaN with the marker's bits: keep it a NaN
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
template <bool RECIP>
__device__ __forceinline__ bool lsm_gather_solve(const LsmArgs& a, uint32_t nb, uint32_t lb, uint32_t round,
                                                 int coeffs, double* fold, double* s_mom, double* s_beta, int* s_ok) {
  __shared__ int s_bad;
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  const uint64_t base_at = (uint64_t)round * nb * 16;
  const uint32_t mom = threadIdx.x & 15u, lane_grp = threadIdx.x >> 4, n_grp = blockDim.x >> 4;
  double acc = 0.0;
  if (mom < (uint32_t)kLsmMom && lsm_ok(a, base_at + (uint64_t)nb * 16 - 1, a.partials_len, kLsmErrPartials)) {
    // every load of the thread's blocks issued at once; the slots still empty
    // are read again (bounded) until their blocks have written them; then
    // the values are summed in block order
    constexpr int kBatch = 8;
    const uint64_t start = global_ns();
    for (uint32_t blk0 = lane_grp; blk0 < nb; blk0 += kBatch * n_grp) {
      unsigned long long v[kBatch];
#pragma unroll
      for (int i = 0; i < kBatch; ++i) {
        const uint32_t blk = blk0 + (uint32_t)i * n_grp;
        v[i] = blk < nb ? ld_relaxed_u64(a.partials + base_at + (size_t)blk * 16 + mom) : 0ull;
      }
      for (;;) {
        bool pending = false;
#pragma unroll
        for (int i = 0; i < kBatch; ++i) {
          if (v[i] != kLsmEmpty) continue;
          pending = true;
          v[i] = ld_relaxed_u64(a.partials + base_at + (size_t)(blk0 + (uint32_t)i * n_grp) * 16 + mom);
        }
        if (!pending) break;
        if (*((volatile int*)a.error) != 0) {
          s_bad = 1;
          break;
        }
        if (global_ns() - start > a.timeout_ns) {
          atomicCAS(a.error, 0, kLsmErrTimeout);
          s_bad = 1;
          break;
        }
      }
#pragma unroll
      for (int i = 0; i < kBatch; ++i) acc += __longlong_as_double((long long)v[i]);
    }
  }
  __syncthreads();
  if (s_bad) return false;
  acc += __shfl_xor_sync(0xffffffffu, acc, 16);  // the warp's two lane groups
  if ((threadIdx.x & 31u) < 16u) fold[(threadIdx.x >> 5) * 17 + mom] = acc;
  __syncthreads();
  if (threadIdx.x < 256u) {  // 16 warps (512-thread blocks): moment t / 16 over warp t % 16
    const uint32_t mo = threadIdx.x >> 4, w = threadIdx.x & 15u;
    double t = mo < (uint32_t)kLsmMom ? fold[w * 17 + mo] : 0.0;
    t += __shfl_xor_sync(0xffffffffu, t, 8);
    t += __shfl_xor_sync(0xffffffffu, t, 4);
    t += __shfl_xor_sync(0xffffffffu, t, 2);
    t += __shfl_xor_sync(0xffffffffu, t, 1);
    if (w == 0 && mo < (uint32_t)kLsmMom) s_mom[mo] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ata[4][4], atb[4];
    int idx = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = r; c < 4; ++c) {
        ata[r][c] = s_mom[idx];
        ata[c][r] = s_mom[idx];
        ++idx;
      }
#pragma unroll
    for (int r = 0; r < 4; ++r) atb[r] = s_mom[10 + r];
    // the reference zeroes rows/columns beyond the basis degree
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (r < coeffs) continue;
      atb[r] = 0.0;
#pragma unroll
      for (int c = 0; c < 4; ++c) ata[r][c] = ata[c][r] = 0.0;
    }
    int ok = s_mom[14] >= (double)coeffs ? 1 : 0;
    if (ok) ok = (coeffs == 2 ? solve_fixed<2, RECIP>(ata, atb) : coeffs == 3 ? solve_fixed<3, RECIP>(ata, atb) : solve_fixed<4, RECIP>(ata, atb)) ? 1 : 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) s_beta[r] = (ok && r < coeffs) ? atb[r] : 0.0;
    *s_ok = ok;
  }
  __syncthreads();
  return true;
}

// One 512-thread block per SM: the same warps per SM as two 256-thread
// blocks, but half the block partials to fold per date (the per-date
// cross-block round is this kernel's critical path).
template <class Real, int SMP>
__global__ void __launch_bounds__(kLsmBlock, 1) lsm_kernel(const LsmArgs* __restrict__ jobs, uint32_t n_jobs, SrcCtx ctx) {
  __shared__ double red[kLsmBlock / 32][5];
  __shared__ double s_mom[16];
  __shared__ double s_beta[4];
  __shared__ int s_ok;
  __shared__ uint32_t s_job;
  __shared__ double s_red15[kLsmBlock / 32][17];
  __shared__ double s_fold[kLsmBlock];  // 16 lanes x 16 moments of the last block's fold
  __shared__ Real s_disc[512];
  if (threadIdx.x == 0) {
    uint32_t j = 0;
    while (j + 1 < n_jobs && blockIdx.x >= jobs[j + 1].block_first) ++j;
    s_job = j;
  }
  __syncthreads();
  const LsmArgs a = jobs[s_job];
  const uint32_t nb = a.n_blocks;             // blocks of this job
  const uint32_t lb = blockIdx.x - a.block_first;  // block index within the job
  const uint64_t n = a.n_paths;
  const uint32_t steps = a.n_steps;
  // launch-shape invariants: this block belongs to the job, the job's blocks
  // cover every path with <= kLsmMaxP paths per thread, the dates fit s_disc
  if (blockIdx.x < a.block_first || lb >= nb) {
    if (threadIdx.x == 0) lsm_report(a, kLsmErrJob, blockIdx.x);
    return;
  }
  if ((uint64_t)nb * blockDim.x * kLsmMaxP < n || steps >= 512 || a.n_sched == 0 || a.n_sched > steps) {
    if (threadIdx.x == 0) lsm_report(a, kLsmErrCoverage, n);
    return;
  }
  for (uint32_t j = threadIdx.x; j <= steps; j += blockDim.x) s_disc[j] = (Real)a.disc_pow[j];
  __syncthreads();
  const uint64_t nthreads = (uint64_t)nb * blockDim.x;
  const uint64_t gtid = (uint64_t)lb * blockDim.x + threadIdx.x;
  Real* paths = reinterpret_cast<Real*>(a.paths);
  const Real k = (Real)a.k, drift = (Real)a.drift, vol = (Real)a.vol, inv_k = (Real)(1.0 / fmax(a.k, 2.2250738585072014e-308));
  const int coeffs = (int)a.degree + 1;
  Real cash[kLsmMaxP];
  uint32_t exd[kLsmMaxP];
  DevReq q;  // sampler view of the request
  q.seed = a.seed;
  q.seed32 = a.seed32;
  q.n_chunks = 1;
  q.normals_per_unit = steps;
  // Pseudorandom sampler: a thread's paths lie nthreads paths apart, so the
  // stream state at each path start after the first is one jump of
  // T^(nthreads x steps) draws (nthreads is even, so the pair alignment of
  // the start carries over), 16 table lookups instead of a full seek.
  uint64_t aligned = 0;
#pragma unroll
  for (int j = 0; j < kLsmMaxP; ++j) {
    const uint64_t path = gtid + (uint64_t)j * nthreads;
    cash[j] = 0;
    exd[j] = steps;
    if (path >= n) continue;
    Source<SMP> src;
    if constexpr (SMP == SMP_XORSHIFT) {
      const uint64_t idx = path * steps;
      aligned = (j == 0 || a.stride_jump == nullptr)
                    ? xorshift_jump(ctx.jump, XorshiftStream::first_state(a.seed), 2 * (idx >> 1))
                    : gf2_apply(a.stride_jump, aligned);
      src.st.seek_aligned(aligned, idx, sizeof(Real) == 4);
    } else {
      src.template begin<sizeof(Real) == 8>(q, ctx, path);
    }
    Real s = (Real)a.s0;
    for (uint32_t st = 1; st <= steps; ++st) {
      const Real z = normal<Real>(src, st - 1);
      s *= ex<Real>(drift + vol * z);  // multiplicative update as cpu.rs:3829-3830
      const uint64_t idx = (uint64_t)(st - 1) * n + path;
      if (lsm_ok(a, idx, a.paths_len, kLsmErrPaths)) paths[idx] = s;
    }
    cash[j] = k - s > (Real)0 ? k - s : (Real)0;
  }
  uint32_t regressions = 0, round = 0;
  // The path values of a date are loaded one date ahead, before the
  // cross-block wait of the current date, so their latency hides behind it.
  Real sv_next[kLsmMaxP];
  auto load_date = [&](int si_load) {
    const uint32_t step_load = a.sched[si_load];
#pragma unroll
    for (int j = 0; j < kLsmMaxP; ++j) {
      const uint64_t path = gtid + (uint64_t)j * nthreads;
      sv_next[j] = (Real)0;
      if (path >= n || step_load == 0 || step_load > steps) continue;
      const uint64_t at = (uint64_t)(step_load - 1) * n + path;
      if (lsm_ok(a, at, a.paths_len, kLsmErrPaths)) sv_next[j] = __ldcg(paths + at);
    }
  };
  if (a.n_sched >= 2) load_date((int)a.n_sched - 2);
  for (int si = (int)a.n_sched - 2; si >= 0; --si) {
    const uint32_t step = a.sched[si];
    if (step == 0 || step > steps) {
      if (threadIdx.x == 0) lsm_report(a, kLsmErrSched, step);
    }
    double m[kLsmMom];
#pragma unroll
    for (int i = 0; i < kLsmMom; ++i) m[i] = 0.0;
    // FP32 path: each thread sums its own <= kLsmMaxP paths in FP32 and the
    // warp sums them in FP32; FP64 takes over from the warp sums (block,
    // cross-block)
    float mf[kLsmMom];
#pragma unroll
    for (int i = 0; i < kLsmMom; ++i) mf[i] = 0.0f;
    Real sv[kLsmMaxP];
#pragma unroll
    for (int j = 0; j < kLsmMaxP; ++j) sv[j] = sv_next[j];
#pragma unroll
    for (int j = 0; j < kLsmMaxP; ++j) {
      const uint64_t path = gtid + (uint64_t)j * nthreads;
      if (path >= n || step == 0 || step > steps) continue;
      const Real s = sv[j];
      const Real imm = k - s;
      if (!(imm > (Real)0)) continue;
      if (exd[j] < step || exd[j] > steps) {
        lsm_report(a, kLsmErrDisc, exd[j]);
        continue;
      }
      const Real cont = cash[j] * s_disc[exd[j] - step];
      Real b[4];
      laguerre4<Real>(s * inv_k, b);
      int idx = 0;
      if constexpr (sizeof(Real) == 4) {
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = r; c < 4; ++c) {
            mf[idx] = fmaf(b[r], b[c], mf[idx]);
            ++idx;
          }
#pragma unroll
        for (int r = 0; r < 4; ++r) mf[10 + r] = fmaf(b[r], cont, mf[10 + r]);
        mf[14] += 1.0f;
      } else {
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = r; c < 4; ++c) m[idx++] += (double)(b[r] * b[c]);
#pragma unroll
        for (int r = 0; r < 4; ++r) m[10 + r] += (double)(b[r] * cont);
        m[14] += 1.0;
      }
    }
    // block reduction of the 15 moments: warp sums by reduce-scatter (the
    // FP32 path reduces the thread sums in FP32 across the warp, and FP64
    // takes over from the warp sums), then a fixed tree folds the warps
    const uint64_t part_at = ((uint64_t)round * nb + lb) * 16;
    {
      double w;
      if constexpr (sizeof(Real) == 4) {
        float mv[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) mv[i] = i < kLsmMom ? mf[i] : 0.0f;
        w = (double)warp_reduce_scatter16(mv);
      } else {
        double mv[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) mv[i] = i < kLsmMom ? m[i] : 0.0;
        w = warp_reduce_scatter16(mv);
      }
      const uint32_t lane = threadIdx.x & 31u;
      if ((lane & 1u) == 0) s_red15[threadIdx.x >> 5][reduce_scatter16_index(lane)] = w;
    }
    __syncthreads();
    if (threadIdx.x < 256u) {
      // moment m = t / 16 over the 16 warps w = t % 16: a shuffle tree per
      // 16-lane group
      const uint32_t mo = threadIdx.x >> 4, w = threadIdx.x & 15u;
      double t = mo < (uint32_t)kLsmMom ? s_red15[w][mo] : 0.0;
      t += __shfl_xor_sync(0xffffffffu, t, 8);
      t += __shfl_xor_sync(0xffffffffu, t, 4);
      t += __shfl_xor_sync(0xffffffffu, t, 2);
      t += __shfl_xor_sync(0xffffffffu, t, 1);
      // the slot's own value marks its arrival (lsm_gather_solve)
      if (w == 0 && mo < (uint32_t)kLsmMom && lsm_ok(a, part_at + mo, a.partials_len, kLsmErrPartials))
        st_relaxed_f64(a.partials + part_at + mo, t);
    }
    if (si > 0) load_date(si - 1);  // next date's values, in flight during the wait
    // Every block waits (bounded) for all blocks' partials of this date, then
    // sums them in block order and solves the normal equations itself.
    if (!lsm_gather_solve<sizeof(Real) == 4>(a, nb, lb, round++, coeffs, s_fold, s_mom, s_beta, &s_ok)) return;
    if (s_ok) {
      ++regressions;
      const Real b0 = (Real)s_beta[0], b1 = (Real)s_beta[1], b2 = (Real)s_beta[2], b3 = (Real)s_beta[3];
#pragma unroll
      for (int j = 0; j < kLsmMaxP; ++j) {
        const uint64_t path = gtid + (uint64_t)j * nthreads;
        if (path >= n) continue;
        const Real imm = k - sv[j];
        if (!(imm > (Real)0)) continue;
        Real b[4];
        laguerre4<Real>(sv[j] * inv_k, b);
        Real cont = b0 * b[0] + b1 * b[1];
        if (coeffs > 2) cont += b2 * b[2];
        if (coeffs > 3) cont += b3 * b[3];
        if (imm > (cont > (Real)0 ? cont : (Real)0)) {
          cash[j] = imm;
          exd[j] = step;
        }
      }
    }
  }
  // estimator: discounted cashflows, exercise counts
  double v[5] = {0, 0, 0, 0, 0};
#pragma unroll
  for (int j = 0; j < kLsmMaxP; ++j) {
    const uint64_t path = gtid + (uint64_t)j * nthreads;
    if (path >= n) continue;
    if (exd[j] > steps) {
      lsm_report(a, kLsmErrDisc, exd[j]);
      continue;
    }
    const double d = (double)cash[j] * a.disc_pow[exd[j]];
    v[0] += d;
    v[1] += d * d;
    if (exd[j] < steps)
      v[2] += 1.0;
    else if (cash[j] > (Real)0)
      v[3] += 1.0;
  }
  block_reduce5(v, red);
  if (threadIdx.x == 0) {
    double* fp = a.final_partials + (size_t)lb * 4;
    if (lsm_ok(a, (uint64_t)lb * 4 + 3, a.final_len, kLsmErrFinal))
      for (int i = 0; i < 4; ++i) fp[i] = v[i];
    __threadfence();
    s_ok = atomicAdd(a.done, 1u) == nb - 1;
  }
  __syncthreads();
  if (s_ok) {
    __threadfence();
    double acc[5] = {0, 0, 0, 0, 0};
    for (uint32_t blk = threadIdx.x; blk < nb; blk += blockDim.x) {
      if (!lsm_ok(a, (uint64_t)blk * 4 + 3, a.final_len, kLsmErrFinal)) break;
      for (int i = 0; i < 4; ++i) acc[i] += __ldcg(a.final_partials + (size_t)blk * 4 + i);
    }
    block_reduce5(acc, red);
    if (threadIdx.x != 0) return;
    a.out[0] = (double)n;
    a.out[1] = acc[0];
    a.out[2] = acc[1];
    a.out[3] = acc[2];
    a.out[4] = acc[3];
    a.out[5] = (double)regressions;
    *a.done = 0u;
  }
}

template <class Real, int SMP>
static uint32_t lsm_capacity_t() {
  int dev = 0, sms = 148, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lsm_kernel<Real, SMP>, kLsmBlock, 0);
  return per_sm > 0 ? (uint32_t)(sms * per_sm) : 0u;
}

uint32_t lsm_capacity(int fp64, int sampler) {
  if (fp64) return sampler == SMP_COUNTER ? lsm_capacity_t<double, SMP_COUNTER>() : lsm_capacity_t<double, SMP_XORSHIFT>();
  return sampler == SMP_COUNTER ? lsm_capacity_t<float, SMP_COUNTER>() : lsm_capacity_t<float, SMP_XORSHIFT>();
}

template <class Real, int SMP>
static cudaError_t launch_lsm_t(const LsmArgs* jobs, uint32_t n_jobs, uint32_t total_blocks, const SrcCtx& ctx,
                                cudaStream_t stream) {
  if (total_blocks == 0 || total_blocks > lsm_capacity_t<Real, SMP>()) return cudaErrorInvalidValue;
  const LsmArgs* j = jobs;
  uint32_t nj = n_jobs;
  SrcCtx c = ctx;
  void* params[] = {&j, &nj, &c};
  cudaError_t err = cudaLaunchCooperativeKernel((const void*)lsm_kernel<Real, SMP>, dim3(total_blocks),
                                                dim3(kLsmBlock), params, 0, stream);
  count_launch();
  return err;
}

cudaError_t launch_lsm_batch(const LsmArgs* d_jobs, uint32_t n_jobs, uint32_t total_blocks, int fp64, int sampler,
                             const DeviceTables& tabs, cudaStream_t stream) {
  SrcCtx ctx{tabs.sobol, tabs.jump, nullptr};
  if (fp64) {
    if (sampler == SMP_COUNTER) return launch_lsm_t<double, SMP_COUNTER>(d_jobs, n_jobs, total_blocks, ctx, stream);
    return launch_lsm_t<double, SMP_XORSHIFT>(d_jobs, n_jobs, total_blocks, ctx, stream);
  }
  if (sampler == SMP_COUNTER) return launch_lsm_t<float, SMP_COUNTER>(d_jobs, n_jobs, total_blocks, ctx, stream);
  return launch_lsm_t<float, SMP_XORSHIFT>(d_jobs, n_jobs, total_blocks, ctx, stream);
}

// ------------------------------------------------------ single-pass Greeks ---
// european_call_pathwise_greeks_cpu / european_call_likelihood_ratio_greeks_cpu
// (cpu.rs:4670-4869): path i draws normal i of MonteCarloRng(seed) (one
// sequential stream, replayed by jump-ahead), prices the terminal GBM state
// and records the per-path estimators; sums and sums of squares in FP64,
// combined in block order by the last block.
template <class Real>
__global__ void __launch_bounds__(256) greeks_single_pass_kernel(GreekArgs a, const uint64_t* __restrict__ jump) {
  __shared__ double red[kWarps][5];
  __shared__ int s_last;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const Real s0 = (Real)a.s0, k = (Real)a.k, r = (Real)a.r, sigma = (Real)a.sigma, t = (Real)a.t;
  const Real sqrt_t = (Real)a.sqrt_t, drift_t = (Real)a.drift_t, vol_t = (Real)a.vol_t, disc = (Real)a.discount;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n_paths; i += stride) {
    XorshiftStream st;
    st.seek(jump, a.seed, i, sizeof(Real) == 4);
    const Real z = sizeof(Real) == 4 ? (Real)st.normal_f32() : (Real)st.normal_f64();
    const Real s = s0 * ex<Real>(drift_t + vol_t * z);
    Real g[4];
    if (a.estimator == MPC_GREEKS_PATHWISE) {
      const Real intrinsic = s - k;
      const bool active = intrinsic > (Real)0;
      const Real payoff = intrinsic > (Real)0 ? intrinsic : (Real)0;
      const Real dpay = disc * payoff;
      g[0] = active ? disc * s / s0 : (Real)0;
      g[1] = active ? disc * s * (-sigma * t + sqrt_t * z) : (Real)0;
      g[2] = active ? disc * (t * s - t * payoff) : -t * dpay;
      const Real dst_dt = s * (r - (Real)0.5 * sigma * sigma + sigma * z / ((Real)2 * sqrt_t));
      g[3] = -(active ? disc * (dst_dt - r * payoff) : -r * dpay);
    } else {
      const Real dpay = disc * (s - k > (Real)0 ? s - k : (Real)0);
      g[0] = dpay * z / (s0 * sigma * sqrt_t);
      g[1] = dpay * ((z * z - (Real)1) / sigma - sqrt_t * z);
      g[2] = dpay * (z / (sigma * sqrt_t) - t);
      g[3] = (Real)0;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const double v = (double)g[j];
      acc[2 * j] += v;
      acc[2 * j + 1] += v * v;
    }
  }
  double v0[5] = {acc[0], acc[1], acc[2], acc[3], acc[4]};
  double v1[5] = {acc[5], acc[6], acc[7], 0.0, 0.0};
  block_reduce5(v0, red);
  block_reduce5(v1, red);
  if (threadIdx.x == 0) {
    double* pt = a.partials + (size_t)blockIdx.x * 8;
    for (int j = 0; j < 5; ++j) pt[j] = v0[j];
    for (int j = 0; j < 3; ++j) pt[5 + j] = v1[j];
    __threadfence();
    s_last = atomicAdd(a.done, 1u) == gridDim.x - 1 ? 1 : 0;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x < 8) {
    double sum = 0.0;
    for (uint32_t b = 0; b < gridDim.x; ++b) sum += __ldcg(a.partials + (size_t)b * 8 + threadIdx.x);
    a.out[threadIdx.x] = sum;
  }
  if (threadIdx.x == 0) *a.done = 0u;
}

cudaError_t launch_greeks_single_pass(const GreekArgs& a, uint32_t grid, const DeviceTables& tabs,
                                      cudaStream_t stream) {
  if (a.fp64)
    greeks_single_pass_kernel<double><<<grid, 256, 0, stream>>>(a, tabs.jump);
  else
    greeks_single_pass_kernel<float><<<grid, 256, 0, stream>>>(a, tabs.jump);
  count_launch();
  return cudaGetLastError();
}

// ------------------------------------------------------------ generators ---
template <int SMP>
__global__ void __launch_bounds__(256) generate_kernel(DevReq q, int fp32, void* out, uint64_t n_points,
                                                       uint32_t dims, SrcCtx ctx) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_points; p += stride) {
    Source<SMP> src;
    if (fp32) {
      src.template begin<false>(q, ctx, p);
      float* o = reinterpret_cast<float*>(out) + p * dims;
      for (uint32_t d = 0; d < dims; ++d) o[d] = src.n32(d);
    } else {
      src.template begin<true>(q, ctx, p);
      double* o = reinterpret_cast<double*>(out) + p * dims;
      for (uint32_t d = 0; d < dims; ++d) o[d] = src.n64(d);
    }
  }
}

cudaError_t launch_generate_normals(const DevReq& q, int sampler, int fp32, void* d_out, uint64_t n_points,
                                    uint32_t dims, const DeviceTables& tabs, cudaStream_t stream) {
  SrcCtx ctx{tabs.sobol, tabs.jump, nullptr};
  uint64_t want = (n_points + 255) / 256;
  int grid = (int)(want < 4096 ? want : 4096);
  if (grid < 1) grid = 1;
  switch (sampler) {
    case SMP_XORSHIFT:
      generate_kernel<SMP_XORSHIFT><<<grid, 256, 0, stream>>>(q, fp32, d_out, n_points, dims, ctx);
      break;
    case SMP_HALTON:
      generate_kernel<SMP_HALTON><<<grid, 256, 0, stream>>>(q, fp32, d_out, n_points, dims, ctx);
      break;
    case SMP_LHS:
      generate_kernel<SMP_LHS><<<grid, 256, 0, stream>>>(q, fp32, d_out, n_points, dims, ctx);
      break;
    case SMP_SOBOL:
      generate_kernel<SMP_SOBOL><<<grid, 256, 0, stream>>>(q, fp32, d_out, n_points, dims, ctx);
      break;
    case SMP_COUNTER:
      generate_kernel<SMP_COUNTER><<<grid, 256, 0, stream>>>(q, fp32, d_out, n_points, dims, ctx);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  count_launch();
  return cudaGetLastError();
}

__global__ void counter_hash_kernel(uint32_t seed, uint32_t n_paths, uint32_t n_steps, uint32_t* out) {
  const uint64_t total = (uint64_t)n_paths * n_steps;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t path = (uint32_t)(i / n_steps), step = (uint32_t)(i % n_steps);
    out[2 * i] = hash_u32(counter_mix(seed, path, step, 0u));
    out[2 * i + 1] = hash_u32(counter_mix(seed, path, step, 1u));
  }
}

cudaError_t launch_counter_hash(uint32_t seed, uint32_t n_paths, uint32_t n_steps, uint32_t* d_out,
                                cudaStream_t stream) {
  uint64_t total = (uint64_t)n_paths * n_steps;
  int grid = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
  if (grid < 1) grid = 1;
  counter_hash_kernel<<<grid, 256, 0, stream>>>(seed, n_paths, n_steps, d_out);
  count_launch();
  return cudaGetLastError();
}

// Each thread emits 64 consecutive draws after one jump.
__global__ void xorshift_kernel(uint64_t seed, uint64_t offset, uint64_t count, uint64_t* out, const uint64_t* jump) {
  const uint64_t chunk = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t first = chunk * 64;
  if (first >= count) return;
  XorshiftStream st;
  uint64_t s0 = seed == 0 ? 0x9E3779B97F4A7C15ull : seed;
  st.state = xorshift_jump(jump, s0, offset + first);
  st.has_cached = false;
  const uint64_t last = first + 64 < count ? first + 64 : count;
  for (uint64_t i = first; i < last; ++i) out[i] = st.next_u64();
}

cudaError_t launch_xorshift(uint64_t seed, uint64_t offset, uint64_t count, uint64_t* d_out,
                            const DeviceTables& tabs, cudaStream_t stream) {
  uint64_t chunks = (count + 63) / 64;
  int grid = (int)((chunks + 255) / 256);
  if (grid < 1) grid = 1;
  xorshift_kernel<<<grid, 256, 0, stream>>>(seed, offset, count, d_out, tabs.jump);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_flush(void* d_buf, size_t bytes, cudaStream_t stream) {
  count_launch();
  return cudaMemsetAsync(d_buf, (int)(g_launches.load() & 0xFF), bytes, stream);
}

}  // namespace mpc

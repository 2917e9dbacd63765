// mpc_device.cuh -- device-side generators, inverse CDF and reductions of the
// B200 Monte Carlo backend.  Everything here is evaluated in registers inside
// the fused pricing kernels; no sample is materialised unless the request is
// an FP64-plain one.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mpc_types.h"

namespace mpc {

// ----------------------------------------------------------- xorshift64* --
// MonteCarloRng (crates/mc-core/src/runtime/cpu.rs:2955-3007) replayed on the
// device.  The state transition x -> x^(x>>12), ^(x<<25), ^(x>>27) is linear
// over GF(2), so T^k is a 64x64 bit matrix.  The host tabulates
// T^(2^b) for b = 0..63 in nibble form: jump[b][q][v] = T^(2^b) applied to
// the nibble value v placed at bit position 4q.  Jumping k draws ahead costs
// popcount(k) * 16 table lookups.
struct JumpTables {
  const uint64_t* nibble;  // [64][16][16]
};

__device__ __forceinline__ uint64_t gf2_apply(const uint64_t* __restrict__ table, uint64_t x) {
  uint64_t y = 0;
#pragma unroll
  for (int q = 0; q < 16; ++q) y ^= __ldg(table + q * 16 + ((x >> (4 * q)) & 0xF));
  return y;
}

__device__ __forceinline__ uint64_t xorshift_jump(const uint64_t* __restrict__ nibble, uint64_t state,
                                                  uint64_t k) {
  while (k) {
    int b = __ffsll((long long)k) - 1;
    state = gf2_apply(nibble + (size_t)b * 256, state);
    k &= k - 1;
  }
  return state;
}

// Sequential MonteCarloRng positioned at an arbitrary normal index.
__device__ __forceinline__ float neg2_log_fast(float u);

struct XorshiftStream {
  uint64_t state;
  double cached;
  bool has_cached;

  __device__ __forceinline__ uint64_t next_u64() {
    uint64_t x = state;
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    state = x;
    return x * 0x2545F4914F6CDD1Dull;
  }
  __device__ __forceinline__ double next_open01() {
    uint64_t raw = next_u64() >> 11;
    double v = (double)raw * (1.0 / 9007199254740992.0);
    return fmax(v, 2.2250738585072014e-308);
  }
  // The same uniform rounded to FP32: (float)((double)(raw >> 11) * 2^-53)
  // is one rounding of the 53-bit integer, which the direct conversion does
  // too (the scale is an exact power of two; raw = 0 gives 0 either way).
  __device__ __forceinline__ float next_open01_f32() {
    return __ull2float_rn(next_u64() >> 11) * 1.1102230246251565e-16f;
  }
  // Box-Muller in FP64 (cpu.rs:2992-3006): returns cos branch, caches sin branch.
  __device__ __forceinline__ double normal_f64() {
    if (has_cached) {
      has_cached = false;
      return cached;
    }
    double u1 = next_open01();
    double u2 = next_open01();
    double radius = sqrt(-2.0 * log(u1));
    double s, c;
    sincos(6.283185307179586 * u2, &s, &c);
    cached = radius * s;
    has_cached = true;
    return radius * c;
  }
  // Same draw with the Box-Muller transform evaluated in FP32: the integer
  // stream and the uniforms (rounded to f32) are the reference's.
  __device__ __forceinline__ float normal_f32() {
    if (has_cached) {
      has_cached = false;
      return (float)cached;
    }
    // FP32 path: the stream's uniforms with the short Box-Muller of the
    // counter-hash normals (atanh series near 1 / hardware log2, approximate
    // square root) and the hardware sine and cosine of 2 pi (u2 - 1/2) in
    // [-pi, pi], where their documented error is 2^-21.4 absolute:
    // sin / cos (2 pi u2) = -sin / -cos (2 pi (u2 - 1/2)).
    const float u1 = next_open01_f32();
    const float u2 = next_open01_f32();
    float radius;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(radius) : "f"(neg2_log_fast(u1)));
    float s, c;
    __sincosf(6.28318548f * (u2 - 0.5f), &s, &c);
    cached = (double)(radius * -s);
    has_cached = true;
    return radius * -c;
  }
  // First state of the stream of `seed` (MonteCarloRng replaces seed 0).
  __device__ __forceinline__ static uint64_t first_state(uint64_t seed) { return seed == 0 ? 0x9E3779B97F4A7C15ull : seed; }
  // Starts from `aligned`, the state after 2 * (normal_index / 2) draws, so
  // that the next normal is normal number `normal_index` (an odd index first
  // draws the pair and keeps its second normal).
  __device__ __forceinline__ void seek_aligned(uint64_t aligned, uint64_t normal_index, bool fp32) {
    state = aligned;
    has_cached = false;
    if (normal_index & 1) {
      if (fp32)
        (void)normal_f32();
      else
        (void)normal_f64();
    }
  }
  // Position the stream of `seed` so that the next normal is normal number
  // `normal_index` of the sequential stream.
  __device__ __forceinline__ void seek(const uint64_t* __restrict__ nibble, uint64_t seed,
                                       uint64_t normal_index, bool fp32) {
    seek_aligned(xorshift_jump(nibble, first_state(seed), 2 * (normal_index >> 1)), normal_index, fp32);
  }
};

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  uint64_t z = x;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// derive_chunk_seed (cpu.rs:8922-8924)
__host__ __device__ __forceinline__ uint64_t derive_chunk_seed(uint64_t base, uint64_t idx) {
  return splitmix64(base + idx * 0x9E3779B97F4A7C15ull);
}

// The reference's CPU thread split (cpu.rs:6232-6276): `chunks` streams of
// base or base+1 units, the first `rem` chunks one larger.  Maps a global
// unit index to (chunk seed, index inside the chunk).
__device__ __forceinline__ void chunk_of(const DevReq& q, uint64_t unit, uint64_t* seed, uint64_t* local) {
  if (q.n_chunks <= 1) {
    *seed = q.seed;
    *local = unit;
    return;
  }
  uint64_t big = q.chunk_rem * (q.chunk_base + 1);
  uint64_t c;
  if (unit < big) {
    c = unit / (q.chunk_base + 1);
    *local = unit - c * (q.chunk_base + 1);
  } else {
    c = q.chunk_rem + (unit - big) / q.chunk_base;
    *local = unit - big - (c - q.chunk_rem) * q.chunk_base;
  }
  *seed = derive_chunk_seed(q.seed, c);
}

// --------------------------------------------------------- counter hash ---
// hash_u32 / stateless_open01_f32 / stateless_standard_normal_f32
// (cpu.rs:5626-5652, european_call_stepwise_v1.metal:6-28).
__host__ __device__ __forceinline__ uint32_t hash_u32(uint32_t x) {
  x += 0x9E3779B9u;
  x ^= x >> 16;
  x *= 0x85EBCA6Bu;
  x ^= x >> 13;
  x *= 0xC2B2AE35u;
  return x ^ (x >> 16);
}
__host__ __device__ __forceinline__ uint32_t counter_mix(uint32_t seed, uint32_t path, uint32_t step,
                                                         uint32_t lane) {
  return seed ^ (path * 747796405u) ^ (step * 2891336453u) ^ (lane * 277803737u);
}
// f32((h + 1) / 4294967297.0): the quotient lies within one unit of 2^-32
// below (h+1)/2^32, so the correctly rounded f64 quotient rounds to the same
// f32 as (h+1)/2^32 rounded to nearest with ties toward zero.  Evaluated
// exactly in integer arithmetic, no FP64 division.
__device__ __forceinline__ float counter_open01(uint32_t h) {
  if (h == 0xFFFFFFFFu) return 1.0f;
  uint32_t m = h + 1u;
  int bits = 32 - __clz(m);
  if (bits <= 24) return (float)m * 2.3283064365386963e-10f;  // exact
  int s = bits - 24;
  uint32_t q = m >> s;
  uint32_t rem = m & ((1u << s) - 1u);
  uint32_t half = 1u << (s - 1);
  if (rem > half) q += 1u;  // ties go down
  return __uint2float_rn(q) * __int_as_float((127 + s - 32) << 23);
}
__device__ __forceinline__ float counter_normal_f32(uint32_t seed, uint32_t path, uint32_t step) {
  float u1 = counter_open01(hash_u32(counter_mix(seed, path, step, 0u)));
  float u2 = counter_open01(hash_u32(counter_mix(seed, path, step, 1u)));
  float radius = sqrtf(-2.0f * logf(u1));
  float theta = 2.0f * 3.14159265358979323846f * u2;
  return radius * cosf(theta);
}

// --- fused FP32 form of the counter-hash normal --------------------------
// Same u32 hashes as counter_normal_f32; the transform is evaluated with
// short instruction sequences (about 3x fewer instructions than the libm
// form) and stays within about 1e-5 absolute of it.
//
// (h + 1) / 2^32 rounded to nearest-even in one conversion.  counter_open01
// rounds ties toward zero; the two differ by one ulp at exact ties only.
__device__ __forceinline__ float counter_open01_fast(uint32_t h) {
  return h == 0xFFFFFFFFu ? 1.0f : __uint2float_rn(h + 1u) * 2.3283064365386963e-10f;
}
// -2 ln(u), u in (0, 1].  Above 15/16, 4 atanh(s) with s = e / (2 - e) and
// e = 1 - u (exact there), three series terms (truncation < 2e-10 relative);
// below, the hardware log2, whose absolute error is small against |ln u|.
__device__ __forceinline__ float neg2_log_fast(float u) {
  const float e = 1.0f - u;
  const float s = __fdividef(e, 2.0f - e), s2 = s * s;
  const float near1 = 4.0f * s * fmaf(s2, fmaf(s2, 0.2f, 0.33333334f), 1.0f);
  const float far = -1.3862943611198906f * __log2f(u);
  return u > 0.9375f ? near1 : far;
}
// cos(2 pi u) for u in [0, 1] as -cos(2 pi t), t = u - 1/2, by a degree-8
// polynomial in t^2 (Chebyshev least-squares fit rounded to float32,
// reproduced by fit_cos2pi.py; max error 3.3e-7).
__device__ __forceinline__ float cos_2pi_fast(float u) {
  const float t = u - 0.5f, x = t * t;
  float p = 2.437560558e-01f;
  p = fmaf(p, x, -1.696802378e+00f);
  p = fmaf(p, x, 7.899099350e+00f);
  p = fmaf(p, x, -2.642559624e+01f);
  p = fmaf(p, x, 6.024458313e+01f);
  p = fmaf(p, x, -8.545681763e+01f);
  p = fmaf(p, x, 6.493939209e+01f);
  p = fmaf(p, x, -1.973920822e+01f);
  p = fmaf(p, x, 1.0f);
  return -p;
}
// The same as -cos(2 pi t) with CUDA's fast cosine on t in [-1/2, 1/2]: its
// documented absolute error bound on [-pi, pi] (2^-21.41) matches the fit
// above, for one multiply and one MUFU operation instead of nine FMAs.
__device__ __forceinline__ float cos_2pi_hw(float u) {
  return -__cosf(6.28318548f * (u - 0.5f));
}
// Box-Muller cosine branch of the counter-hash uniforms; HWCOS picks the
// hardware cosine (for kernels with room on the MUFU pipe) over the
// polynomial (for kernels already bound by it, such as multi-asset baskets).
template <bool HWCOS = false>
__device__ __forceinline__ float counter_normal_fast(uint32_t seed, uint32_t path, uint32_t step) {
  const float u1 = counter_open01_fast(hash_u32(counter_mix(seed, path, step, 0u)));
  const float u2 = counter_open01_fast(hash_u32(counter_mix(seed, path, step, 1u)));
  float radius;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(radius) : "f"(neg2_log_fast(u1)));
  return radius * (HWCOS ? cos_2pi_hw(u2) : cos_2pi_fast(u2));
}

// ---------------------------------------------------------------- Sobol ---
// Burley 2020 hash-based Owen scrambling (the algorithm of the `sobol_burley`
// crate called at cpu.rs:5399-5431): Owen-shuffled index, Sobol matrix
// product, Owen-scrambled output.  The matrix product uses per-dimension
// nibble tables sob[dim][q][v] = XOR of V[dim][4q + j] over the bits j of v,
// 8 lookups per sample instead of 32 conditional XORs.
__host__ __device__ __forceinline__ uint32_t lk_permute(uint32_t x, uint32_t seed) {
  x += seed;
  x ^= x * 0x6c50b47cu;
  x ^= x * 0xb82f1e52u;
  x ^= x * 0xc7afe638u;
  x ^= x * 0x8d22f6e6u;
  return x;
}
__device__ __forceinline__ uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) {
  return __brev(lk_permute(__brev(x), seed));
}
__host__ __device__ __forceinline__ uint32_t hash_combine(uint32_t seed, uint32_t v) {
  return seed ^ (v + 0x9e3779b9u + (seed << 6) + (seed >> 2));
}
__device__ __forceinline__ uint32_t sobol_product(const uint32_t* __restrict__ table_dim, uint32_t index) {
  // table_dim: 8 x 16 words for this dimension (bit 0 of the index = MSB direction)
  uint32_t x = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) x ^= table_dim[q * 16 + ((index >> (4 * q)) & 0xFu)];
  return x;
}
// Sobol sample of (point, normal_index) with the reference's block and
// dimension-wrap seeding (ScrambledSobol::standard_normal, cpu.rs:5665-5677).
__device__ __forceinline__ uint32_t sobol_point(const uint32_t* __restrict__ table, uint64_t point,
                                                uint32_t normal_index, uint32_t seed32) {
  uint32_t block = (uint32_t)(point >> 16);
  uint32_t local = (uint32_t)(point & 0xFFFFu);
  uint32_t dim = normal_index & (MPC_SOBOL_TABLE_DIMS - 1);
  uint32_t seed = seed32 + (normal_index / MPC_SOBOL_TABLE_DIMS) + block * 0x9E3779B9u;
  uint32_t shuffled = nested_uniform_scramble(local, seed);
  uint32_t x = sobol_product(table + dim * 128, shuffled);
  return nested_uniform_scramble(x, hash_combine(seed, dim));
}
// 23-bit midpoint uniform: exact in both precisions, never 0 or 1.
__device__ __forceinline__ float sobol_unit_f32(uint32_t x) {
  return ((float)(x >> 9) + 0.5f) * 1.1920928955078125e-07f;
}
// The same value assembled from bits: 1 + (x >> 9) 2^-23 in [1, 2) minus
// (1 - 2^-24); the difference is exact (Sterbenz), so no conversion is needed.
// (x >> 9) has no bit in common with the exponent, so + equals | here and
// lets the shift and the add issue as one instruction.
__device__ __forceinline__ float sobol_unit_f32_bits(uint32_t x) {
  return __fsub_rn(__int_as_float((x >> 9) + 0x3F800000u), 0.99999994f);
}
__device__ __forceinline__ double sobol_unit_f64(uint32_t x) {
  return ((double)(x >> 9) + 0.5) * 1.1920928955078125e-07;
}

// ------------------------------------------------------- Acklam inverse ---
// inverse_standard_normal (cpu.rs:6012-6061): the reference rational in FP64.
// The FP32 path calls CUDA's normcdfinvf: the rational's 1.15e-9 relative
// error is far below what FP32 resolves, so only the exact inverse matters there.
__device__ __forceinline__ double icdf_f64(double p) {
  const double a0 = -3.969683028665376e1, a1 = 2.209460984245205e2, a2 = -2.759285104469687e2,
               a3 = 1.38357751867269e2, a4 = -3.066479806614716e1, a5 = 2.506628277459239;
  const double b0 = -5.447609879822406e1, b1 = 1.615858368580409e2, b2 = -1.556989798598866e2,
               b3 = 6.680131188771972e1, b4 = -1.328068155288572e1;
  const double c0 = -7.784894002430293e-3, c1 = -3.223964580411365e-1, c2 = -2.400758277161838,
               c3 = -2.549732539343734, c4 = 4.374664141464968, c5 = 2.938163982698783;
  const double d0 = 7.784695709041462e-3, d1 = 3.224671290700398e-1, d2 = 2.445134137142996,
               d3 = 3.754408661907416;
  // Every product and sum is rounded separately (no FMA contraction), as the
  // CPU reference evaluates it, so both give the same bits up to log().
  p = fmin(fmax(p, 2.2250738585072014e-308), 1.0 - 2.220446049250313e-16);
  auto mad = [](double acc, double x, double c) { return __dadd_rn(__dmul_rn(acc, x), c); };
  if (p < 0.02425) {
    double q = sqrt(__dmul_rn(-2.0, log(p)));
    double num = mad(mad(mad(mad(mad(c0, q, c1), q, c2), q, c3), q, c4), q, c5);
    double den = mad(mad(mad(mad(d0, q, d1), q, d2), q, d3), q, 1.0);
    return num / den;
  }
  if (p <= 1.0 - 0.02425) {
    double q = __dadd_rn(p, -0.5);
    double r = __dmul_rn(q, q);
    double num = __dmul_rn(mad(mad(mad(mad(mad(a0, r, a1), r, a2), r, a3), r, a4), r, a5), q);
    double den = mad(mad(mad(mad(mad(b0, r, b1), r, b2), r, b3), r, b4), r, 1.0);
    return num / den;
  }
  double q = sqrt(__dmul_rn(-2.0, log(__dadd_rn(1.0, -p))));
  double num = mad(mad(mad(mad(mad(c0, q, c1), q, c2), q, c3), q, c4), q, c5);
  double den = mad(mad(mad(mad(d0, q, d1), q, d2), q, d3), q, 1.0);
  return -num / den;
}

// --------------------------------------------------------------- Halton ---
// halton / halton_with_shift (cpu.rs:6063-6077), evaluated in FP64 exactly as
// the reference (IEEE division and accumulation order).
__device__ __forceinline__ double halton_shifted(uint64_t index, uint32_t base, double shift) {
  double f = 1.0 / (double)base;
  double value = 0.0;
  while (index > 0) {
    uint64_t next = index / base;
    value += f * (double)(index - next * base);
    index = next;
    f /= (double)base;
  }
  value = fmax(value, 2.2250738585072014e-308);
  double shifted = value + shift;
  return shifted - floor(shifted);
}

__device__ __forceinline__ double open01_from_u64(uint64_t v) {
  return fmax((double)(v >> 11) * (1.0 / 9007199254740992.0), 2.2250738585072014e-308);
}
// LatinHypercube::standard_normal's uniform (cpu.rs:5764-5780).
__device__ __forceinline__ double lhs_uniform(const LhsDim& d, uint64_t point, uint64_t n_paths) {
  uint64_t stratum = (d.multiplier * point + d.offset) % n_paths;
  double jitter = open01_from_u64(splitmix64(d.jitter_seed ^ (point * 0xBF58476D1CE4E5B9ull)));
  double u = ((double)stratum + jitter) / (double)n_paths;
  return fmin(fmax(u, 2.2250738585072014e-308), 1.0 - 2.220446049250313e-16);
}

// ------------------------------------------------------------- reductions -
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}

}  // namespace mpc

// Seeded white noise of the fluctuating inflow: a counter-based stream, so
// that every face node draws independent deviates without per-node state and
// a run repeats bit for bit for a given seed.  The uniform deviates come from
// the SplitMix64 output function (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014) applied to a key built from
// the seed, the application count and the face node; the normal deviates
// from the Box-Muller transform.  The CPU oracle restates the same integer
// steps, so the uniform deviates agree bit for bit; the normal deviates agree
// to the rounding of log and sincospi.
#pragma once
#include <cstdint>

namespace cfk {

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Uniform deviate in (0, 1] number n of face node `node` at application `call`.
__host__ __device__ __forceinline__ double noise_uniform(uint64_t seed, uint64_t call, uint64_t node, uint64_t n) {
  const uint64_t key = splitmix64(seed ^ splitmix64((call << 24) ^ node));
  const uint64_t r = splitmix64(key + n * 0x9E3779B97F4A7C15ull);
  return (double)((r >> 11) + 1) * 0x1.0p-53;
}

// Normal deviates 2 m and 2 m + 1 of a face node (Box-Muller of uniforms 2 m, 2 m + 1).
__device__ __forceinline__ void noise_normal_pair(uint64_t seed, uint64_t call, uint64_t node, uint64_t m,
                                                  double &n0, double &n1) {
  const double u1 = noise_uniform(seed, call, node, 2 * m), u2 = noise_uniform(seed, call, node, 2 * m + 1);
  const double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  n0 = r * c;
  n1 = r * s;
}

}  // namespace cfk

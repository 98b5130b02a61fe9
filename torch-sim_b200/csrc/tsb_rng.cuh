// Counter-based normal random numbers: Philox4x32-10 (Salmon, Moraes, Dror,
// Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11) followed by the
// Box-Muller transform.  Stateless: (key, counter) -> 4 normals, so every atom
// and step draws an independent stream without any RNG state in memory.
#pragma once

#include <stdint.h>

namespace tsb {

struct U4 {
  uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox_round(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
  uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
  return U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
}

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;  // Weyl key increments
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    c = philox_round(c, k0, k1);
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// uniform in (0, 1]
__device__ __forceinline__ double u01_open0(uint32_t v) {
  return ((double)v + 1.0) * 2.3283064365386963e-10;
}

// Four standard normals for (seed, atom, counter).
__device__ inline void normal4(uint64_t seed, uint64_t atom, uint64_t counter, double *z) {
  U4 c{(uint32_t)atom, (uint32_t)(atom >> 32), (uint32_t)counter, (uint32_t)(counter >> 32)};
  U4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double two_pi = 6.283185307179586;
  double r1 = sqrt(-2.0 * log(u01_open0(r.x)));
  double r2 = sqrt(-2.0 * log(u01_open0(r.z)));
  double s1, c1, s2, c2;
  sincos(two_pi * (r.y * 2.3283064365386963e-10), &s1, &c1);
  sincos(two_pi * (r.w * 2.3283064365386963e-10), &s2, &c2);
  z[0] = r1 * c1;
  z[1] = r1 * s1;
  z[2] = r2 * c2;
  z[3] = r2 * s2;
}

}  // namespace tsb

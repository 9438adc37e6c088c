// Counter-based Gaussian samples: Philox-4x32-10 (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11) followed by the
// Box-Muller transform.  Pair j of a stream keyed by `seed` is a pure
// function of (seed, j), so any thread can produce any sample.
#pragma once
#include <cstdint>

namespace mb {

__device__ __forceinline__ void philox_round(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
  const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
  const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
  c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
}

// Samples 2j and 2j+1 of the N(0,1) stream keyed by seed.
__device__ __forceinline__ void gaussian_pair(uint64_t seed, uint64_t j, double& z0, double& z1) {
  uint32_t c[4] = {uint32_t(j), uint32_t(j >> 32), 0u, 0u};
  uint32_t k0 = uint32_t(seed), k1 = uint32_t(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    philox_round(c, k0, k1);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  // two 53-bit uniforms in (0, 1)
  const uint64_t b1 = ((uint64_t(c[0]) << 32) | c[1]) >> 11;
  const uint64_t b2 = ((uint64_t(c[2]) << 32) | c[3]) >> 11;
  const double u1 = (double(b1) + 0.5) * 0x1.0p-53;
  const double u2 = (double(b2) + 0.5) * 0x1.0p-53;
  const double r = sqrt(-2.0 * log(u1));
  double sn, cs;
  sincospi(2.0 * u2, &sn, &cs);
  z0 = r * cs;
  z1 = r * sn;
}

}  // namespace mb

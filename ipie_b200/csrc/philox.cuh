// Philox4x32-10 counter-based generator and its uniform conversion, shared by
// the device draws of the throughput mode (auxiliary fields, population control).
#pragma once

namespace ipie_b200 {

// Philox4x32-10 counter-based generator: Salmon, Moraes, Dror & Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11.  Round function
// and constants as published there.
struct U4 {
  unsigned x, y, z, w;
};
__device__ __forceinline__ U4 philox_round(U4 c, unsigned k0, unsigned k1) {
  const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  unsigned hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
  unsigned hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
  return U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
}
__device__ __forceinline__ U4 philox10(U4 c, unsigned k0, unsigned k1) {
  const unsigned W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    c = philox_round(c, k0, k1);
    k0 += W0;
    k1 += W1;
  }
  return c;
}
// 53-bit uniform in (0, 1].
__device__ __forceinline__ double u53(unsigned a, unsigned b) {
  unsigned long long v = ((unsigned long long)(a >> 5) << 26) | (b >> 6);
  return ((double)v + 1.0) * (1.0 / 9007199254740992.0);
}

}  // namespace ipie_b200

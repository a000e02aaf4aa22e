// Device helpers for composite string indices (shared by the contraction and
// reorder kernels).
#pragma once
#include <cstdint>

#include "device_types.hpp"

namespace gccu {

// composite index -> component indices, first component fastest
__device__ __forceinline__ void decomp(const int32_t* rad, int n, int64_t x, int32_t* comp) {
  for (int q = 0; q < n; ++q) {
    int32_t r = rad[q];
    comp[q] = (int32_t)(x % r);
    x /= r;
  }
}

// address part of the components that merge two spaces (map lookups); cA
// holds the component indices of space spA, cB those of the other space
__device__ __forceinline__ bool mapped(const OpndDesc& od, int spA, const int32_t* cA,
                                       const int32_t* cB, int64_t& off, double& sg) {
  for (int j = 0; j < od.ncomp; ++j) {
    const int32_t* mp = od.map[j];
    if (!mp) continue;
    int i1 = od.sp1[j] == spA ? cA[od.ci1[j]] : cB[od.ci1[j]];
    int i2 = od.sp2[j] == spA ? cA[od.ci2[j]] : cB[od.ci2[j]];
    int v = __ldg(mp + (int64_t)i2 * od.n1[j] + i1);
    if (v == 0) return false;
    if (v < 0) {
      sg = -sg;
      v = -v;
    }
    off += (int64_t)(v - 1) * od.ldim[j];
  }
  return true;
}

// address part of the components taken from one space only
__device__ __forceinline__ int64_t direct(const OpndDesc& od, int spA, const int32_t* cA,
                                          const int32_t* cB) {
  int64_t off = 0;
  for (int j = 0; j < od.ncomp; ++j) {
    if (od.map[j]) continue;
    const bool one = od.sp1[j] != kNone;
    const int sp = one ? od.sp1[j] : od.sp2[j];
    const int ci = one ? od.ci1[j] : od.ci2[j];
    off += (int64_t)(sp == spA ? cA[ci] : cB[ci]) * od.ldim[j];
  }
  return off;
}

}  // namespace gccu

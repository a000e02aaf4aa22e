// Singlet spin projection of ME lists (spin_prj_blk,
// contract/spin_prj_blk.f:254-400).
//
// k_spin_prj  one thread per skeleton element of one skeleton distribution
//             (grid.y): the element of every spin case of the element's
//             spatial configuration is found through the pattern maps of
//             the skeleton's component strings (spprjmap,
//             strings/set_spprjmap_kernel.f:60-130) and the case's
//             distribution offset and leading dimensions; the values (with
//             the sign -1 for every second appearance of an element whose
//             paired orbitals make two cases coincide) are projected with
//             C C^T and written back in case order.  A skeleton element whose
//             alternating cases do not all exist (a skeleton string that is
//             not of the reference spin pattern) is skipped: its
//             configuration is handled by the element that is.  Every element
//             of the class belongs to exactly one configuration, so the
//             threads write disjoint elements and the projection runs in
//             place.  HBM-bound: each element is read and written once, the
//             maps and case tables stay in L1/L2.
#include <algorithm>

#include "kernels.hpp"

namespace gccu {
namespace {

constexpr int kSpinPrjThreads = 128;

// address of case k's element for the skeleton strings sc / sa, -1 if the
// case does not exist for them
__device__ __forceinline__ int64_t case_element(const SpinPrjDesc& d, const SpinPrjCase& K,
                                                const int32_t* sc, const int32_t* sa) {
  if (K.off < 0) return -1;
  int64_t p = K.off;
  for (int i = 0; i < d.nc; ++i) {
    int64_t s = sc[i];
    const int m = K.mc[i];
    if (m != 0) {
      const int v = d.mapc[i] ? __ldg(d.mapc[i] + s * d.nmc[i] + m - 1) : (int)s + 1;
      if (v == 0) return -1;
      s = (v < 0 ? -v : v) - 1;
    }
    p += s * K.ldc[i];
  }
  for (int i = 0; i < d.na; ++i) {
    int64_t s = sa[i];
    const int m = K.ma[i];
    if (m != 0) {
      const int v = d.mapa[i] ? __ldg(d.mapa[i] + s * d.nma[i] + m - 1) : (int)s + 1;
      if (v == 0) return -1;
      s = (v < 0 ? -v : v) - 1;
    }
    p += s * K.lda[i];
  }
  return p;
}

template <int MC>
__global__ void __launch_bounds__(kSpinPrjThreads)
    k_spin_prj(const SpinPrjDesc* __restrict__ ds, double* __restrict__ x) {
  const SpinPrjDesc& d = ds[blockIdx.y];
  const int64_t n = d.lenc * d.lena;
  const int ncase = d.ncase, ncoup = d.ncoup;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    int32_t sc[kDevMaxComp], sa[kDevMaxComp];
    int64_t ia = e / d.lenc, ic = e - ia * d.lenc;
    for (int i = 0; i < d.nc; ++i) {
      sc[i] = (int32_t)(ic % d.lc[i]);
      ic /= d.lc[i];
    }
    for (int i = 0; i < d.na; ++i) {
      sa[i] = (int32_t)(ia % d.la[i]);
      ia /= d.la[i];
    }
    // skeleton strings of a non-reference pattern: nothing to do here
    bool skip = false;
    for (int j = 0; j < d.nomni && !skip; ++j)
      skip = case_element(d, d.cases[d.omni[j]], sc, sa) < 0;
    if (skip) continue;
    int64_t idx[MC];
    double val[MC];
    for (int k = 0; k < ncase; ++k) {
      idx[k] = case_element(d, d.cases[k], sc, sa);
      val[k] = 0.0;
      if (idx[k] < 0) continue;
      int cnt = 0;
      for (int j = 0; j <= k; ++j) cnt += idx[j] == idx[k];
      const double ps = (__popc(cnt - 1) & 1) ? -1.0 : 1.0;
      val[k] = x[idx[k]] * ps;
    }
    // C^T v, then C (C^T v): summed in case order, then in path order
    double ov[MC == 2 ? 1 : MC == 6 ? 2 : MC == 20 ? 5 : kSpinPrjMaxCoup];
    for (int q = 0; q < ncoup; ++q) {
      double s = 0.0;
      for (int k = 0; k < ncase; ++k) s += __ldg(d.coeff + k * ncoup + q) * val[k];
      ov[q] = s;
    }
    for (int k = 0; k < ncase; ++k) {
      if (idx[k] < 0) continue;
      double s = 0.0;
      for (int q = 0; q < ncoup; ++q) s += __ldg(d.coeff + k * ncoup + q) * ov[q];
      int cnt = 0;
      for (int j = 0; j <= k; ++j) cnt += idx[j] == idx[k];
      x[idx[k]] = (__popc(cnt - 1) & 1) ? -s : s;
    }
  }
}

template <int MC>
void launch_t(const SpinPrjDesc* d, int64_t n, double* x, int64_t maxlen, cudaStream_t s) {
  for (int64_t b = 0; b < n; b += 65535) {
    dim3 grid((unsigned)std::min<int64_t>((maxlen + kSpinPrjThreads - 1) / kSpinPrjThreads, 2048),
              (unsigned)std::min<int64_t>(n - b, 65535));
    k_spin_prj<MC><<<grid, kSpinPrjThreads, 0, s>>>(d + b, x);
  }
}

}  // namespace

void launch_spin_prj(const SpinPrjDesc* d, int64_t n, int maxcase, double* x, int64_t maxlen,
                     cudaStream_t s) {
  if (n == 0 || maxlen == 0) return;
  if (maxcase <= 2) launch_t<2>(d, n, x, maxlen, s);
  else if (maxcase <= 6) launch_t<6>(d, n, x, maxlen, s);
  else if (maxcase <= 20) launch_t<20>(d, n, x, maxlen, s);
  else launch_t<kSpinPrjMaxCases>(d, n, x, maxlen, s);
}

}  // namespace gccu

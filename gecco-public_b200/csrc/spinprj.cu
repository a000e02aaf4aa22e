// Singlet spin projection of ME lists (spin_prj_blk,
// contract/spin_prj_blk.f:254-400).
//
// k_spin_prj<MC>  one thread per (thread-side tuple, loop-side tuple) pair
//                 of one skeleton distribution (grid.y), kSpinPrjLoop
//                 loop-side tuples per thread: the elements of the MC spin
//                 cases of the pair's spatial configuration are at the sums
//                 of the two sides' partial offsets (planned on the host with
//                 the reference's pattern maps, strings/set_spprjmap_kernel.f
//                 :60-130); their values, with the sign -1 for every second
//                 appearance of an element that two cases share (paired
//                 orbitals), are projected with C C^T (C: the singlet
//                 coupling coefficients, staged in shared memory) and written
//                 back in case order.  Only skeleton strings of the reference
//                 spin pattern are listed, so every spatial configuration of
//                 the class is handled by exactly one thread: the threads
//                 write disjoint elements and the projection runs in place.
//                 HBM-bound: each element read and written once; the offset
//                 tables are O(square root) of the class and stay in L2.
#include <algorithm>

#include "kernels.hpp"

namespace gccu {
namespace {

template <int MC>
__global__ void __launch_bounds__(kSpinPrjThreads)
    k_spin_prj(const SpinPrjDesc* __restrict__ ds, double* __restrict__ x) {
  constexpr int NP = spin_prj_paths(MC);
  constexpr int UNR = MC <= 20 ? MC : 1;
  __shared__ double cs[MC * NP];
  const SpinPrjDesc d = ds[blockIdx.y];
  for (int i = threadIdx.x; i < MC * NP; i += blockDim.x) cs[i] = d.coeff[i];
  __syncthreads();
  const int64_t tchunks = (d.nt + kSpinPrjThreads - 1) / kSpinPrjThreads;
  const int64_t nb = spin_prj_blocks(d.nt, d.nl);
  for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
    const int64_t lb = b / tchunks;
    const int64_t it = (b - lb * tchunks) * kSpinPrjThreads + threadIdx.x;
    if (it >= d.nt) continue;
    int64_t pt[MC];
#pragma unroll UNR
    for (int k = 0; k < MC; ++k) pt[k] = __ldg(d.pt + k * d.nt + it);
    const int64_t l1 = min(d.nl, (lb + 1) * kSpinPrjLoop);
    for (int64_t il = lb * kSpinPrjLoop; il < l1; ++il) {
      int64_t idx[MC];
      double val[MC];
#pragma unroll UNR
      for (int k = 0; k < MC; ++k) {
        const int64_t l = __ldg(d.pl + k * d.nl + il);
        idx[k] = (pt[k] < 0 || l < 0) ? -1 : pt[k] + l;
      }
#pragma unroll UNR
      for (int k = 0; k < MC; ++k) {
        int cnt = 0;
#pragma unroll UNR
        for (int j = 0; j < k; ++j) cnt += idx[j] == idx[k];
        const double v = idx[k] < 0 ? 0.0 : x[idx[k]];
        val[k] = (__popc(cnt) & 1) ? -v : v;
      }
      // C^T v, then C (C^T v): summed in case order, then in path order
      double ov[NP];
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        double s = 0.0;
#pragma unroll UNR
        for (int k = 0; k < MC; ++k) s += cs[k * NP + q] * val[k];
        ov[q] = s;
      }
#pragma unroll UNR
      for (int k = 0; k < MC; ++k) {
        if (idx[k] < 0) continue;
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < NP; ++q) s += cs[k * NP + q] * ov[q];
        int cnt = 0;
#pragma unroll UNR
        for (int j = 0; j < k; ++j) cnt += idx[j] == idx[k];
        x[idx[k]] = (__popc(cnt) & 1) ? -s : s;
      }
    }
  }
}

template <int MC>
void launch_t(const SpinPrjDesc* d, int64_t n, double* x, int64_t maxblocks, cudaStream_t s) {
  for (int64_t b = 0; b < n; b += 65535) {
    dim3 grid((unsigned)std::min<int64_t>(maxblocks, 4096),
              (unsigned)std::min<int64_t>(n - b, 65535));
    k_spin_prj<MC><<<grid, kSpinPrjThreads, 0, s>>>(d + b, x);
  }
}

}  // namespace

void launch_spin_prj(const SpinPrjDesc* d, int64_t n, int ncase, double* x, int64_t maxblocks,
                     cudaStream_t s) {
  if (n == 0 || maxblocks == 0) return;
  switch (ncase) {
    case 2: launch_t<2>(d, n, x, maxblocks, s); break;
    case 6: launch_t<6>(d, n, x, maxblocks, s); break;
    case 20: launch_t<20>(d, n, x, maxblocks, s); break;
    default: launch_t<kSpinPrjMaxCases>(d, n, x, maxblocks, s); break;
  }
}

}  // namespace gccu

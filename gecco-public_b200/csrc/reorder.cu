// Reorder of a joined operator class (reo_blk_wmaps_c,
// contract/reo_blk_wmaps_c.f:537-840): every element of the original class
// is added, with the string-map signs, to the element of the reordered class
// that holds the same strings with the shifted strings on their new vertex.
// Several (I0, K) splittings can land on one reordered element, so the
// update is atomic.  Bandwidth-bound: 8 bytes read and one 8-byte atomic per
// element plus cached map reads.
#include "index.cuh"
#include "kernels.hpp"

namespace gccu {
namespace {

constexpr int kReoThreads = 256;

// grid: x = element blocks, y = distribution case
__global__ void __launch_bounds__(kReoThreads)
    k_reorder(const ReoItem* __restrict__ items, const double* __restrict__ ori,
              double* __restrict__ reo, double alpha) {
  const ReoItem& it = items[blockIdx.y];
  const int64_t n = it.N0 * it.NK;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    int32_t c0[kDevMaxComp], ck[kDevMaxComp];
    decomp(it.rad[0], it.nsp[0], e % it.N0, c0);
    decomp(it.rad[1], it.nsp[1], e / it.N0, ck);
    double sg = 1.0;
    int64_t oo = direct(it.ori, kEx1, c0, ck), orr = direct(it.reo, kEx1, c0, ck);
    if (!mapped(it.ori, kEx1, c0, ck, oo, sg)) continue;
    if (!mapped(it.reo, kEx1, c0, ck, orr, sg)) continue;
    const double x = __ldg(ori + it.base_ori + oo);
    if (x != 0.0) atomicAdd(reo + it.base_reo + orr, alpha * sg * x);
  }
}

}  // namespace

void launch_reorder(const ReoItem* items, int64_t nitems, int64_t maxlen, const double* ori,
                    double* reo, double alpha, cudaStream_t s) {
  if (nitems == 0 || maxlen == 0) return;
  int64_t bx = (maxlen + kReoThreads - 1) / kReoThreads;
  if (bx > 2048) bx = 2048;
  dim3 grid((unsigned)bx, (unsigned)nitems);
  k_reorder<<<grid, kReoThreads, 0, s>>>(items, ori, reo, alpha);
}

}  // namespace gccu

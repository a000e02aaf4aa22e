// Block contractions with a thin column side (at most 32 columns, a long
// row side): one streaming pass over the long operand.
//
// k_thin      one CTA per (256 rows, contraction range) of one block
//             contraction (the device tile list), one thread per row: the
//             thin operand's slice of the range (at most kThinMaxElems
//             elements) is staged once in shared memory, the thread walks
//             its row of the long operand over the range, eight indices at a
//             time with their loads issued together, and keeps its N sums in
//             registers (FP64 FMA); N = 1 reads the thin operand directly.  A
//             long operand whose strings merge an external and a contracted
//             component is read through its gather description (the signed
//             string-map gather of collect_block_impr,
//             contract/collect_block_impr.f:397) in place, so no dense panel
//             is written and read back (the k_pack + k_gemm<128,32> route of
//             these items).  Results without map lookups only; the update is
//             plain where the tile is the only writer (scatter_block,
//             contract/scatter_block.f:163), atomic otherwise.
#include <cstdio>

#include "kernels.hpp"

namespace gccu {
namespace {

constexpr int kThinThreads = kGemmThinM;  // one thread per row of a tile
constexpr int kThinBatch = 8;             // contraction indices per load batch

template <int NC>
__global__ void __launch_bounds__(kThinThreads)
    k_thin(const GemmDesc* __restrict__ descs, const TileDesc* __restrict__ tiles,
           const PackJob* __restrict__ gathers, double alpha) {
  extern __shared__ __align__(16) double bs[];  // thin operand [k][NC] (NC > 1)
  const TileDesc td = tiles[blockIdx.x];
  const GemmDesc& d = descs[td.item];
  const int tid = threadIdx.x;
  const int64_t M = d.M, N = d.N, K = d.K;
  const int64_t kb = td.k0, ke = td.k1 < K ? td.k1 : K;  // contraction range of the tile
  const double* __restrict__ B = d.b;
  const int64_t* __restrict__ bco = d.bco;
  const int64_t* __restrict__ bko = d.bko;
  if constexpr (NC > 1) {
    for (int64_t i = tid; i < (ke - kb) * NC; i += kThinThreads) {
      const int64_t k = kb + i / NC, c = i % NC;
      bs[i] = c < N ? __ldg(B + __ldg(bco + c) + __ldg(bko + k)) : 0.0;
    }
    __syncthreads();
  }
  const int64_t r = td.m0 + tid;
  if (r >= M) return;
  double acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = 0.0;
  const int64_t bc0 = NC == 1 ? __ldg(bco) : 0;
  // the thin operand's element k (NC = 1: read directly, the same address
  // for the whole warp)
  auto fma_k = [&](int64_t k, double a) {
    if constexpr (NC == 1) {
      acc[0] = fma(a, __ldg(B + bc0 + __ldg(bko + k)), acc[0]);
    } else {
      const double2* brow = reinterpret_cast<const double2*>(bs + (k - kb) * NC);
#pragma unroll
      for (int c = 0; c < NC / 2; ++c) {
        const double2 bv = brow[c];
        acc[2 * c] = fma(a, bv.x, acc[2 * c]);
        acc[2 * c + 1] = fma(a, bv.y, acc[2 * c + 1]);
      }
    }
  };
  if (d.ga == 0) {  // long operand read through its offset tables
    const double* __restrict__ A = d.a;
    const int64_t rof = __ldg(d.aro + r);
    const int64_t akstep = d.akstep;
    const int64_t ak0 = akstep ? __ldg(d.ako) : 0;
    for (int64_t k0 = kb; k0 < ke; k0 += kThinBatch) {
      double v[kThinBatch];
#pragma unroll
      for (int e = 0; e < kThinBatch; ++e) {
        const int64_t k = k0 + e;
        v[e] = k < ke ? __ldg(A + rof + (akstep ? ak0 + k * akstep : __ldg(d.ako + k))) : 0.0;
      }
#pragma unroll
      for (int e = 0; e < kThinBatch; ++e)
        if (k0 + e < ke) fma_k(k0 + e, v[e]);
    }
  } else {  // map-addressed long operand: its gather description
    const PackJob& G = gathers[d.ga - 1];
    const double* __restrict__ src = G.src;
    const int nm = G.nm;
    const int64_t R = G.R;
    const int64_t rof = __ldg(G.roff + r);
    int32_t ir[kTcGatherMaps];
#pragma unroll
    for (int m = 0; m < kTcGatherMaps; ++m)
      ir[m] = m < nm ? (int32_t)__ldg(G.rmi + (int64_t)m * R + r) : 0;
    for (int64_t k0 = kb; k0 < ke; k0 += kThinBatch) {
      int64_t off[kThinBatch];
      bool ok[kThinBatch], neg[kThinBatch];
#pragma unroll
      for (int e = 0; e < kThinBatch; ++e) {
        const int64_t k = k0 + e;
        ok[e] = k < ke;
        off[e] = ok[e] ? rof + __ldg(G.koff + k) : 0;
        neg[e] = false;
      }
#pragma unroll
      for (int m = 0; m < kTcGatherMaps; ++m) {
        if (m >= nm) break;
        const bool r1 = G.row_is_1[m] != 0;
        const int32_t* __restrict__ mp = G.map[m];
        const int64_t n1 = G.n1[m], ld = G.ldim[m];
        int w[kThinBatch];
#pragma unroll
        for (int e = 0; e < kThinBatch; ++e) {
          const int32_t ik = ok[e] ? (int32_t)__ldg(G.kmi + (int64_t)m * K + k0 + e) : 0;
          w[e] = ok[e] ? __ldg(mp + (int64_t)(r1 ? ik : ir[m]) * n1 + (r1 ? ir[m] : ik)) : 1;
        }
#pragma unroll
        for (int e = 0; e < kThinBatch; ++e) {
          int x = w[e];
          if (x == 0) ok[e] = false;
          if (x < 0) {
            neg[e] = !neg[e];
            x = -x;
          }
          off[e] += (int64_t)(x - 1) * ld;
        }
      }
      double v[kThinBatch];
#pragma unroll
      for (int e = 0; e < kThinBatch; ++e) {
        const double x = ok[e] ? __ldg(src + off[e]) : 0.0;
        v[e] = neg[e] ? -x : x;
      }
#pragma unroll
      for (int e = 0; e < kThinBatch; ++e)
        if (k0 + e < ke) fma_k(k0 + e, v[e]);
    }
  }
  const double f = alpha * d.fac;
  double* __restrict__ X = d.c;
  const int64_t ro = __ldg(d.cro + r);
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (c >= N) break;
    double* p = X + ro + __ldg(d.cco + c);
    if (d.exclusive)
      *p += f * acc[c];
    else
      atomicAdd(p, f * acc[c]);
  }
}

template <int NC>
void launch_thin_t(const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles,
                   const PackJob* gathers, int64_t kmax, double alpha, cudaStream_t s) {
  // kmax: the longest contraction range of a tile, kmax * NC <= kThinMaxElems
  const size_t smem = NC > 1 ? (size_t)kmax * NC * sizeof(double) : 0;
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_thin<NC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kThinMaxElems * sizeof(double)));
    configured = true;
  }
  k_thin<NC><<<(unsigned)ntiles, kThinThreads, smem, s>>>(descs, tiles, gathers, alpha);
}

}  // namespace

int thin_columns(int64_t N) { return N <= 1 ? 1 : (int)((N + 7) / 8 * 8); }

void launch_thin(int nc, const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles,
                 const PackJob* gathers, int64_t kmax, double alpha, cudaStream_t s) {
  if (ntiles == 0) return;
  switch (nc) {
    case 1: launch_thin_t<1>(descs, tiles, ntiles, gathers, kmax, alpha, s); break;
    case 8: launch_thin_t<8>(descs, tiles, ntiles, gathers, kmax, alpha, s); break;
    case 16: launch_thin_t<16>(descs, tiles, ntiles, gathers, kmax, alpha, s); break;
    case 24: launch_thin_t<24>(descs, tiles, ntiles, gathers, kmax, alpha, s); break;
    default: launch_thin_t<32>(descs, tiles, ntiles, gathers, kmax, alpha, s); break;
  }
}

}  // namespace gccu

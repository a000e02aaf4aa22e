// Block contractions as grouped FP64 tensor-core GEMMs (sm_100a).
//
// k_pack      gathers an operand whose strings merge a contraction and an
//             external component (string-map lookups, signed) into a dense
//             panel, once per call (collect_block_impr,
//             contract/collect_block_impr.f:217-399).
// k_gemm      all block contractions of one [CONTR] in one launch: per output
//             tile a register-prefetched, double-buffered shared-memory
//             pipeline over the contraction index feeds FP64 MMA
//             (mma.sync m8n8k4 f64; tcgen05 has no f64 kind); the epilogue
//             scales by the factor and scatter-adds with the string-map signs
//             into the result (scatter_block, contract/scatter_block.f:163).
//             Operand elements are addressed through per-row and per-k offset
//             tables, so direct operands are read in place from the ME lists.
#include <cstdio>

#include "kernels.hpp"

namespace gccu {
namespace {

constexpr int BK = 16;
constexpr int PAD = 8;

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

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

// ---------------------------------------------------------------------------
__global__ void k_pack(const PackJob* __restrict__ jobs) {
  const PackJob& J = jobs[blockIdx.y];
  const int64_t n = J.R * J.K;
  const OpndDesc& od = J.op;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = e % J.R, k = e / J.R;
    int32_t rc[kDevMaxComp], kc[kDevMaxComp];
    decomp(J.rad[J.rowspace], J.nsp[J.rowspace], r, rc);
    decomp(J.rad[kCnt], J.nsp[kCnt], k, kc);
    int64_t off = 0;
    double sg = 1.0;
    bool ok = true;
    for (int j = 0; j < od.ncomp && ok; ++j) {
      if (od.map[j]) continue;
      int sp = od.sp1[j] != kNone ? od.sp1[j] : od.sp2[j];
      int ci = od.sp1[j] != kNone ? od.ci1[j] : od.ci2[j];
      off += (int64_t)(sp == kCnt ? kc[ci] : rc[ci]) * od.ldim[j];
    }
    ok = mapped(od, J.rowspace, rc, kc, off, sg);
    J.dst[e] = ok ? sg * J.src[off] : 0.0;
  }
}

// ---------------------------------------------------------------------------
template <int BM, int BN, int WARPS_M, int WARPS_N>
struct Cfg {
  static constexpr int NT = 32 * WARPS_M * WARPS_N;
  static constexpr int WTM = BM / WARPS_M, WTN = BN / WARPS_N;
  static constexpr int MT = WTM / 8, NTL = WTN / 8;
  static constexpr int ELA = BM * BK / NT, ELB = BN * BK / NT;
};

template <int BM, int BN>
struct __align__(16) GemmSmem {
  double As[2][BK][BM + PAD];
  double Bs[2][BK][BN + PAD];
  int64_t aro[BM], bco[BN], cro[BM], cco[BN];
  int32_t rc[BM][kDevMaxComp];
  int32_t cc[BN][kDevMaxComp];
  GemmDesc d;
};

// element (row r, k-slot kk) handled by thread t in slot e of a R x BK tile
template <int R, int NT>
__device__ __forceinline__ void slot(int fastk, int t, int e, int& r, int& kk) {
  if (fastk) {
    kk = t % BK;
    r = t / BK + (NT / BK) * e;
  } else {
    r = t % R;
    kk = t / R + (NT / R) * e;
  }
}

template <int R, int NT, int EL>
__device__ __forceinline__ void load_tile(const double* __restrict__ x,
                                          const int64_t* __restrict__ kofs,
                                          const int64_t* rofs_s, int fastk, int t, int64_t k0,
                                          int64_t k1, int64_t rows, double (&v)[EL]) {
#pragma unroll
  for (int e = 0; e < EL; ++e) {
    int r, kk;
    slot<R, NT>(fastk, t, e, r, kk);
    int64_t k = k0 + kk;
    v[e] = (r < rows && k < k1) ? __ldg(x + rofs_s[r] + __ldg(kofs + k)) : 0.0;
  }
}

template <int R, int NT, int EL>
__device__ __forceinline__ void store_tile(double (*S)[R + PAD], int fastk, int t,
                                           const double (&v)[EL]) {
#pragma unroll
  for (int e = 0; e < EL; ++e) {
    int r, kk;
    slot<R, NT>(fastk, t, e, r, kk);
    S[kk][r] = v[e];
  }
}

template <int BM, int BN, int WARPS_M, int WARPS_N>
__global__ void __launch_bounds__(Cfg<BM, BN, WARPS_M, WARPS_N>::NT)
    k_gemm(const GemmDesc* __restrict__ descs, const TileDesc* __restrict__ tiles,
           double alpha) {
  using C = Cfg<BM, BN, WARPS_M, WARPS_N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GemmSmem<BM, BN>& S = *reinterpret_cast<GemmSmem<BM, BN>*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const TileDesc td = tiles[blockIdx.x];
  {
    const int* src = reinterpret_cast<const int*>(descs + td.item);
    int* dst = reinterpret_cast<int*>(&S.d);
    for (int i = tid; i < (int)(sizeof(GemmDesc) / sizeof(int)); i += C::NT) dst[i] = src[i];
  }
  __syncthreads();
  const GemmDesc& d = S.d;
  const int64_t rows = d.M - td.m0, cols = d.N - td.n0;
  const int colspace = d.rowspace == kEx1 ? kEx2 : kEx1;
  for (int i = tid; i < BM; i += C::NT) {
    if (i < rows) {
      S.aro[i] = d.aro[td.m0 + i];
      S.cro[i] = d.cro[td.m0 + i];
      if (d.cmapped) decomp(d.rad[d.rowspace], d.nsp[d.rowspace], td.m0 + i, S.rc[i]);
    }
  }
  for (int i = tid; i < BN; i += C::NT) {
    if (i < cols) {
      S.bco[i] = d.bco[td.n0 + i];
      S.cco[i] = d.cco[td.n0 + i];
      if (d.cmapped) decomp(d.rad[colspace], d.nsp[colspace], td.n0 + i, S.cc[i]);
    }
  }
  __syncthreads();
  const double* __restrict__ A = d.a;
  const double* __restrict__ B = d.b;
  const int afast = d.afast, bfast = d.bfast;
  const int wm = warp / WARPS_N, wn = warp % WARPS_N;
  double acc[C::MT][C::NTL][2];
#pragma unroll
  for (int i = 0; i < C::MT; ++i)
#pragma unroll
    for (int j = 0; j < C::NTL; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int64_t nk = (td.k1 - td.k0 + BK - 1) / BK;
  double va[C::ELA], vb[C::ELB];
  load_tile<BM, C::NT, C::ELA>(A, d.ako, S.aro, afast, tid, td.k0, td.k1, rows, va);
  load_tile<BN, C::NT, C::ELB>(B, d.bko, S.bco, bfast, tid, td.k0, td.k1, cols, vb);
  store_tile<BM, C::NT, C::ELA>(S.As[0], afast, tid, va);
  store_tile<BN, C::NT, C::ELB>(S.Bs[0], bfast, tid, vb);
  __syncthreads();
  for (int64_t kt = 0; kt < nk; ++kt) {
    const int buf = (int)(kt & 1);
    const bool more = kt + 1 < nk;
    if (more) {
      int64_t k0 = td.k0 + (kt + 1) * BK;
      load_tile<BM, C::NT, C::ELA>(A, d.ako, S.aro, afast, tid, k0, td.k1, rows, va);
      load_tile<BN, C::NT, C::ELB>(B, d.bko, S.bco, bfast, tid, k0, td.k1, cols, vb);
    }
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      double a[C::MT], b[C::NTL];
#pragma unroll
      for (int i = 0; i < C::MT; ++i)
        a[i] = S.As[buf][k4 + (lane & 3)][wm * C::WTM + i * 8 + (lane >> 2)];
#pragma unroll
      for (int j = 0; j < C::NTL; ++j)
        b[j] = S.Bs[buf][k4 + (lane & 3)][wn * C::WTN + j * 8 + (lane >> 2)];
#pragma unroll
      for (int i = 0; i < C::MT; ++i)
#pragma unroll
        for (int j = 0; j < C::NTL; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    if (more) {
      store_tile<BM, C::NT, C::ELA>(S.As[buf ^ 1], afast, tid, va);
      store_tile<BN, C::NT, C::ELB>(S.Bs[buf ^ 1], bfast, tid, vb);
    }
    __syncthreads();
  }
  // signed scatter-add (items and contraction splits may overlap: atomics)
  const double f = alpha * d.fac;
  double* __restrict__ X = d.c;
#pragma unroll
  for (int i = 0; i < C::MT; ++i)
#pragma unroll
    for (int j = 0; j < C::NTL; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = wm * C::WTM + i * 8 + (lane >> 2);
        const int col = wn * C::WTN + j * 8 + 2 * (lane & 3) + h;
        const double v = acc[i][j][h];
        if (row >= rows || col >= cols || v == 0.0) continue;
        int64_t off = S.cro[row] + S.cco[col];
        double sg = 1.0;
        if (d.cmapped && !mapped(d.cmap, d.rowspace, S.rc[row], S.cc[col], off, sg)) continue;
        atomicAdd(X + off, f * sg * v);
      }
}

template <int BM, int BN, int WM, int WN>
void launch_gemm_cfg(const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles, double alpha,
                     cudaStream_t s) {
  using C = Cfg<BM, BN, WM, WN>;
  const size_t smem = sizeof(GemmSmem<BM, BN>);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_gemm<BM, BN, WM, WN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    configured = true;
  }
  k_gemm<BM, BN, WM, WN><<<(unsigned)ntiles, C::NT, smem, s>>>(descs, tiles, alpha);
}

}  // namespace

void launch_pack(const PackJob* jobs, int64_t njobs, int64_t maxlen, cudaStream_t s) {
  if (njobs == 0 || maxlen == 0) return;
  int64_t bx = (maxlen + 255) / 256;
  if (bx > 4096) bx = 4096;
  dim3 grid((unsigned)bx, (unsigned)njobs);
  k_pack<<<grid, 256, 0, s>>>(jobs);
}

void launch_gemm(int kind, const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles,
                 double alpha, cudaStream_t s) {
  if (ntiles == 0) return;
  if (kind == kGemmRegular)
    launch_gemm_cfg<kGemmRegularM, kGemmRegularN, 4, 2>(descs, tiles, ntiles, alpha, s);
  else
    launch_gemm_cfg<kGemmSkinnyM, kGemmSkinnyN, 4, 1>(descs, tiles, ntiles, alpha, s);
}

}  // namespace gccu

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
//             The grid is the device tile list (CTA b takes tile b): the block
//             scheduler hands tiles of uneven length to SMs as they free up.
//             A persistent variant with a static round-robin of the tiles over
//             the resident CTAs took 15% longer on the o24/v200 ladder
//             (95 ms against 82 ms), so this kernel is not persistent.
#include <cstdio>

#include "index.cuh"
#include "kernels.hpp"

namespace gccu {
namespace {

constexpr int BK = 16;
// row pitch of the staged tiles: BM + 4 doubles = 8 words mod 32, so the four
// contraction rows of a 64-bit fragment load (one 16-lane phase: 4 rows x 4
// doubles) fall on 32 distinct banks (BM + 8 put rows 0 and 2 on the same ones)
constexpr int PAD = 4;

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// ---------------------------------------------------------------------------
// grid: x = blocks of (256/F) * kPackPasses slow-dimension indices, y =
// blocks of F fast-dimension indices, z = job.  The fast index's table
// entries are read once per thread, the slow one's (the same for the threads
// of a row of the block) once per pass.
constexpr int kPackThreads = 256, kPackPasses = 8;
__global__ void __launch_bounds__(kPackThreads) k_pack(const PackJob* __restrict__ jobs) {
  const PackJob& J = jobs[blockIdx.z];
  const int F = J.F, S = kPackThreads / F;
  const bool kf = J.kfast != 0;
  const int64_t nf = kf ? J.K : J.R, ns = kf ? J.R : J.K;
  const int64_t f = (int64_t)blockIdx.y * F + threadIdx.x % F;
  const int64_t s0 = (int64_t)blockIdx.x * S * kPackPasses + threadIdx.x / F;
  if (f >= nf || s0 >= ns) return;
  const int64_t* __restrict__ soff = kf ? J.roff : J.koff;
  const int64_t* __restrict__ smi = kf ? J.rmi : J.kmi;
  const int64_t* __restrict__ fmi = kf ? J.kmi : J.rmi;
  const int64_t foff = __ldg((kf ? J.koff : J.roff) + f);
  const int nm = J.nm;
  int32_t fi[kDevMaxComp];
  for (int m = 0; m < nm; ++m) fi[m] = (int32_t)__ldg(fmi + m * nf + f);
  const double* __restrict__ src = J.src;
  double* __restrict__ dst = J.dst;
  for (int p = 0; p < kPackPasses; ++p) {
    const int64_t s = s0 + (int64_t)p * S;
    if (s >= ns) break;
    int64_t off = foff + __ldg(soff + s);
    bool neg = false, ok = true;
    for (int m = 0; m < nm; ++m) {
      const int32_t si = (int32_t)__ldg(smi + m * ns + s);
      const int32_t ir = kf ? si : fi[m], ik = kf ? fi[m] : si;
      const int32_t i1 = J.row_is_1[m] ? ir : ik, i2 = J.row_is_1[m] ? ik : ir;
      int32_t v = __ldg(J.map[m] + (int64_t)i2 * J.n1[m] + i1);
      if (v == 0) {
        ok = false;
        break;
      }
      if (v < 0) {
        neg = !neg;
        v = -v;
      }
      off += (int64_t)(v - 1) * J.ldim[m];
    }
    const int64_t r = kf ? s : f, k = kf ? f : s;
    double x = ok ? __ldg(src + off) : 0.0;
    dst[J.dkfast ? r * J.K + k : k * J.R + r] = neg ? -x : x;
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

// element (row r, k-slot kk) handled by thread t in slot e of a R x BK tile.
// Operand contiguous along k: a warp covers 8 rows x 4 consecutive k per slot
// (32-byte sectors in global memory, distinct shared-memory banks for the
// transposed store); contiguous along rows: a warp covers 32 consecutive rows.
template <int R, int NT>
__device__ __forceinline__ void slot(int fastk, int t, int e, int& r, int& kk) {
  if (fastk) {
    const int lane = t & 31, g = (t >> 5) + (NT / 32) * e;  // group of 4 k x 8 rows
    kk = 4 * (g % (BK / 4)) + (lane & 3);
    r = 8 * (g / (BK / 4)) + (lane >> 2);
  } else {
    r = t % R;
    kk = t / R + (NT / R) * e;
  }
}

// k offset of contraction index k: kbase + k * kstep when the operand's
// table is affine (no dependent table load), else the table entry
template <int R, int NT, int EL>
__device__ __forceinline__ void load_tile(const double* __restrict__ x,
                                          const int64_t* __restrict__ kofs, int64_t kbase,
                                          int64_t kstep, const int64_t* rofs_s, int fastk, int t,
                                          int64_t k0, int64_t k1, int64_t rows, double (&v)[EL]) {
  if (kstep) {
    const double* __restrict__ xk = x + kbase + k0 * kstep;
#pragma unroll
    for (int e = 0; e < EL; ++e) {
      int r, kk;
      slot<R, NT>(fastk, t, e, r, kk);
      v[e] = (r < rows && k0 + kk < k1) ? __ldg(xk + rofs_s[r] + kk * kstep) : 0.0;
    }
  } else {
#pragma unroll
    for (int e = 0; e < EL; ++e) {
      int r, kk;
      slot<R, NT>(fastk, t, e, r, kk);
      const int64_t k = k0 + kk;
      v[e] = (r < rows && k < k1) ? __ldg(x + rofs_s[r] + __ldg(kofs + k)) : 0.0;
    }
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

// resident CTAs per SM the register budget is held to (two 256-thread
// tiles, three 128-thread tiles, four thin ones)
template <int NT, int BN>
constexpr int kGemmMinBlocks = NT >= 256 ? 2 : BN <= 8 ? 4 : 3;

template <int BM, int BN, int WARPS_M, int WARPS_N>
__global__ void __launch_bounds__(Cfg<BM, BN, WARPS_M, WARPS_N>::NT,
                                  kGemmMinBlocks<Cfg<BM, BN, WARPS_M, WARPS_N>::NT, BN>)
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
  const int64_t akstep = d.akstep, bkstep = d.bkstep;
  const int64_t ak0 = akstep ? __ldg(d.ako) : 0, bk0 = bkstep ? __ldg(d.bko) : 0;
  double va[C::ELA], vb[C::ELB];
  load_tile<BM, C::NT, C::ELA>(A, d.ako, ak0, akstep, S.aro, afast, tid, td.k0, td.k1, rows, va);
  load_tile<BN, C::NT, C::ELB>(B, d.bko, bk0, bkstep, S.bco, bfast, tid, td.k0, td.k1, cols, vb);
  store_tile<BM, C::NT, C::ELA>(S.As[0], afast, tid, va);
  store_tile<BN, C::NT, C::ELB>(S.Bs[0], bfast, tid, vb);
  __syncthreads();
  for (int64_t kt = 0; kt < nk; ++kt) {
    const int buf = (int)(kt & 1);
    const bool more = kt + 1 < nk;
    if (more) {
      int64_t k0 = td.k0 + (kt + 1) * BK;
      load_tile<BM, C::NT, C::ELA>(A, d.ako, ak0, akstep, S.aro, afast, tid, k0, td.k1, rows, va);
      load_tile<BN, C::NT, C::ELB>(B, d.bko, bk0, bkstep, S.bco, bfast, tid, k0, td.k1, cols, vb);
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
  if (d.exclusive && !d.cmapped) {
    // sole writer, no map lookups: the read-modify-writes of one row group
    // of the thread's elements with their loads in flight together
#pragma unroll
    for (int i = 0; i < C::MT; ++i) {
      const int row = wm * C::WTM + i * 8 + (lane >> 2);
      const int64_t ro = row < rows ? S.cro[row] : -1;
      int64_t off[C::NTL][2];
      double old[C::NTL][2];
#pragma unroll
      for (int j = 0; j < C::NTL; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int col = wn * C::WTN + j * 8 + 2 * (lane & 3) + h;
          off[j][h] = (ro >= 0 && col < cols) ? ro + S.cco[col] : -1;
          old[j][h] = off[j][h] >= 0 ? X[off[j][h]] : 0.0;
        }
#pragma unroll
      for (int j = 0; j < C::NTL; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h)
          if (off[j][h] >= 0) X[off[j][h]] = old[j][h] + f * acc[i][j][h];
    }
    return;
  }
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
        if (d.exclusive)
          X[off] += f * sg * v;
        else
          atomicAdd(X + off, f * sg * v);
      }
}

// Items with at most 16 result elements (energies, thin intermediates): a
// block reduces a chunk of the contraction index for all M*N elements.
constexpr int kSmallThreads = 256;
__global__ void __launch_bounds__(kSmallThreads)
    k_small(const GemmDesc* __restrict__ descs, const TileDesc* __restrict__ tiles, double alpha) {
  const TileDesc td = tiles[blockIdx.x];
  const GemmDesc& d = descs[td.item];
  const int M = (int)d.M, N = (int)d.N;
  double acc[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) acc[i] = 0.0;
  int64_t ar[16], bc[16];
  for (int r = 0; r < M; ++r) ar[r] = d.aro[r];
  for (int c = 0; c < N; ++c) bc[c] = d.bco[c];
  for (int64_t k = td.k0 + threadIdx.x; k < td.k1; k += kSmallThreads) {
    const int64_t ak = __ldg(d.ako + k), bk = __ldg(d.bko + k);
    double bv[16];
    for (int c = 0; c < N; ++c) bv[c] = __ldg(d.b + bc[c] + bk);
    for (int r = 0; r < M; ++r) {
      const double av = __ldg(d.a + ar[r] + ak);
      for (int c = 0; c < N; ++c) acc[r * N + c] += av * bv[c];
    }
  }
  __shared__ double red[kSmallThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int e = 0; e < M * N; ++e) {
    double v = acc[e];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < kSmallThreads / 32; ++w) s += red[w];
      const int r = e / N, c = e % N;
      int64_t off = d.cro[r] + d.cco[c];
      double sg = 1.0;
      bool ok = true;
      if (d.cmapped) {
        int32_t rc[kDevMaxComp], cc[kDevMaxComp];
        const int colspace = d.rowspace == kEx1 ? kEx2 : kEx1;
        decomp(d.rad[d.rowspace], d.nsp[d.rowspace], r, rc);
        decomp(d.rad[colspace], d.nsp[colspace], c, cc);
        ok = mapped(d.cmap, d.rowspace, rc, cc, off, sg);
      }
      if (ok && s != 0.0) atomicAdd(d.c + off, alpha * d.fac * sg * s);
    }
    __syncthreads();
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

void pack_geometry(const PackJob& j, int64_t& gx, int64_t& gy) {
  const int64_t nf = j.kfast ? j.K : j.R, ns = j.kfast ? j.R : j.K;
  const int64_t span = (int64_t)(kPackThreads / j.F) * kPackPasses;
  gx = (ns + span - 1) / span;
  gy = (nf + j.F - 1) / j.F;
}

void launch_pack(const PackJob* jobs, int64_t njobs, int64_t gx, int64_t gy, cudaStream_t s) {
  if (njobs == 0 || gx == 0 || gy == 0) return;
  dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)njobs);
  k_pack<<<grid, kPackThreads, 0, s>>>(jobs);
}

void launch_gemm(int kind, const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles,
                 double alpha, int* err, int64_t wait_limit, cudaStream_t s) {
  if (ntiles == 0) return;
  if (kind == kGemmTc) {
    launch_gemm_tc(descs, tiles, ntiles, alpha, err, wait_limit, s);
    return;
  }
  if (kind == kGemmRegular)
    launch_gemm_cfg<kGemmRegularM, kGemmRegularN, 4, 2>(descs, tiles, ntiles, alpha, s);
  else if (kind == kGemmMedium)
    launch_gemm_cfg<kGemmMediumM, kGemmMediumN, 4, 1>(descs, tiles, ntiles, alpha, s);
  else if (kind == kGemmSkinny)
    launch_gemm_cfg<kGemmSkinnyM, kGemmSkinnyN, 4, 1>(descs, tiles, ntiles, alpha, s);
  else
    k_small<<<(unsigned)ntiles, kSmallThreads, 0, s>>>(descs, tiles, alpha);
}

}  // namespace gccu

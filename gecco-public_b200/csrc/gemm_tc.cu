// Block contractions on the 5th-generation tensor cores (tcgen05, sm_100a)
// in split TF32: every FP64 operand element x is split into x_hi = tf32(x) and
// x_lo = tf32(x - x_hi); a tile product is accumulated in TMEM (FP32) as
//   A_hi B_hi + A_hi B_lo + A_lo B_hi,
// which keeps about 21 bits of each product (the omitted A_lo B_lo term is
// below 2^-22 relative).  Contraction ranges are at most kTcChunk long, and
// their partial sums are added in FP64 to the result (the scatter epilogue of
// scatter_block, contract/scatter_block.f:163), so the FP32 accumulation
// error does not grow with the full contraction length.
//
// One CTA per 128 x BN output tile, 1024 threads (32 warps: the gathers are
// latency-bound, so many warps in flight matter more than per-thread
// batching).  Per 32-wide slice of the
// contraction index all threads gather the FP64 operand elements through the
// offset tables (the same tables as the FP64 kernel), split them and store
// them to shared memory in the K-major core-matrix layout the tensor core
// reads (8 rows x 16 bytes per core matrix, no swizzle); one thread then
// issues the 12 MMAs of the slice (4 K-steps x 3 products) and commits them to
// the slice's mbarrier.  Two slices are in flight: the loads of slice t+1
// overlap the MMAs of slice t.  The accumulator is read back with tcgen05.ld
// (one TMEM lane per output row) and scattered with the map signs.
//
// Every wait on an mbarrier is bounded; on time-out the kernel records the
// failure in *err, stops issuing work, waits (bounded) for the MMAs it has
// issued, frees its TMEM and returns.
#include <cstdio>

#include "index.cuh"
#include "kernels.hpp"

namespace gccu {
namespace {

constexpr int TBM = 128;    // tile rows = TMEM lanes
constexpr int TBK = 32;     // contraction indices per slice
constexpr int TNT = 1024;   // threads: latency of the gathers is hidden by warps
constexpr int NW = TNT / 32;
constexpr int kTcStages = 2;
constexpr long kWaitLimit = 1L << 22;

template <int BN>
struct __align__(1024) TcSmem {
  float a[kTcStages][2][TBM * TBK];  // [stage][hi/lo][core-matrix layout]
  float b[kTcStages][2][BN * TBK];
  int64_t aro[TBM], bco[BN], cro[TBM], cco[BN];
  int32_t rc[TBM][kDevMaxComp];
  int32_t cc[BN][kDevMaxComp];
  GemmDesc d;
  alignas(8) uint64_t bar[kTcStages];
  uint32_t tmem_base;
  int failed;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major, no-swizzle shared-memory matrix descriptor: core matrices of 8
// rows x 16 bytes; lbo = byte distance of the next core matrix along K,
// sbo = along the rows; version 1 (sm_100)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)(lbo >> 4) << 16) |
         ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}

// instruction descriptor: D f32, A/B tf32, both K-major, M x N
template <int M, int N>
__device__ __forceinline__ uint32_t idesc_tf32() {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
      :
      : "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(bar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(bar), "r"(count) : "memory");
}

// bounded wait for the completion of phase `parity`; false on time-out
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// x -> (tf32(xf), tf32(xf - tf32(xf))) with xf = f32(x), as f32 bit patterns:
// one FP64 conversion per element, the rest on the FP32 pipe; hi + lo keeps
// the 24 bits of xf to within 2^-22 relative
__device__ __forceinline__ void split_tf32(double x, float& hi, float& lo) {
  const float xf = (float)x;
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(xf));
  hi = __uint_as_float(h);
  const float r = xf - hi;  // exact in f32
  uint32_t l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(r));
  lo = __uint_as_float(l);
}

// Operand slice of R rows x 32 contraction indices.  Group g (one per warp
// and unit i, g = warp + NW i) is the core matrix (kg, rg) = rows 8rg..8rg+7
// x indices 4kg..4kg+3; lane -> row 8rg + lane/4, index 4kg + lane%4, which is
// also its float offset within the group's 32 floats.  A warp's load covers
// 8 rows x 4 consecutive indices (coalesced whichever way the operand is
// stored); a thread's row is the same in all its units (its offset stays in
// a register).  The k offset comes from k0 + step*k when the operand's table
// is affine, else from the slice's 32 table values (one per lane, kreg) by
// shuffle.  Elements outside the item are not loaded (zero).
template <int R>
struct Unit {
  static constexpr int NU = R * TBK / (32 * NW);  // elements per thread and slice
  static __device__ __forceinline__ int rg(int warp, int i) { return (warp + NW * i) % (R / 8); }
  static __device__ __forceinline__ int kg(int warp, int i) { return (warp + NW * i) / (R / 8); }
};

template <int R>
__device__ __forceinline__ void gather(const double* __restrict__ x, int64_t kreg, int64_t kbase,
                                       int64_t kstep, int64_t roff, bool rok, int warp, int lane,
                                       int64_t kvalid, double (&v)[Unit<R>::NU]) {
#pragma unroll
  for (int i = 0; i < Unit<R>::NU; ++i) {
    const int kk = 4 * Unit<R>::kg(warp, i) + (lane & 3);
    const int64_t ko = kstep ? kbase + kk * kstep : __shfl_sync(0xffffffffu, kreg, kk);
    double val = 0.0;
    if (rok && kk < kvalid) val = __ldg(x + roff + ko);
    v[i] = val;
  }
}

template <int R>
__device__ __forceinline__ void store_split(float* hi, float* lo, int warp, int lane,
                                            const double (&v)[Unit<R>::NU]) {
#pragma unroll
  for (int i = 0; i < Unit<R>::NU; ++i) {
    const int g = warp + NW * i;
    float h, l;
    split_tf32(v[i], h, l);
    hi[32 * g + lane] = h;
    lo[32 * g + lane] = l;
  }
}

template <int BN>
__global__ void __launch_bounds__(TNT, 1)
    k_gemm_tc(const GemmDesc* __restrict__ descs, const TileDesc* __restrict__ tiles,
              double alpha, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  TcSmem<BN>& S = *reinterpret_cast<TcSmem<BN>*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const TileDesc td = tiles[blockIdx.x];
  {
    const int* src = reinterpret_cast<const int*>(descs + td.item);
    int* dst = reinterpret_cast<int*>(&S.d);
    for (int i = tid; i < (int)(sizeof(GemmDesc) / sizeof(int)); i += TNT) dst[i] = src[i];
  }
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) mbar_init(smem_u32(&S.bar[s]), 1);
    S.failed = 0;
  }
  if (warp == 0) {  // TMEM: BN f32 columns x 128 lanes
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(&S.tmem_base)), "r"((uint32_t)BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  const GemmDesc& d = S.d;
  const int64_t rows = d.M - td.m0, cols = d.N - td.n0;
  const int colspace = d.rowspace == kEx1 ? kEx2 : kEx1;
  for (int i = tid; i < TBM; i += TNT)
    if (i < rows) {
      S.aro[i] = d.aro[td.m0 + i];
      S.cro[i] = d.cro[td.m0 + i];
      if (d.cmapped) decomp(d.rad[d.rowspace], d.nsp[d.rowspace], td.m0 + i, S.rc[i]);
    }
  for (int i = tid; i < BN; i += TNT)
    if (i < cols) {
      S.bco[i] = d.bco[td.n0 + i];
      S.cco[i] = d.cco[td.n0 + i];
      if (d.cmapped) decomp(d.rad[colspace], d.nsp[colspace], td.n0 + i, S.cc[i]);
    }
  __syncthreads();

  static_assert(Unit<TBM>::NU >= 1 && Unit<BN>::NU >= 1, "tile too small for the threads");
  // the row of this thread in each operand tile (the same in all its units)
  static_assert(NW % (TBM / 8) == 0 && NW % (BN / 8) == 0,
                "a thread's row must be the same in all its units");
  const int ra = 8 * Unit<TBM>::rg(warp, 0) + (lane >> 2);
  const int rb = 8 * Unit<BN>::rg(warp, 0) + (lane >> 2);
  const bool rok_a = ra < rows, rok_b = rb < cols;
  const int64_t roff_a = rok_a ? S.aro[ra] : 0, roff_b = rok_b ? S.bco[rb] : 0;
  const uint32_t kIdesc = idesc_tf32<TBM, BN>();
  const int64_t nk = (td.k1 - td.k0 + TBK - 1) / TBK;
  bool ok = true;
  int64_t last = -1;  // last slice whose MMAs were committed
  // k offsets of a slice, one per lane (prefetched a slice ahead)
  auto kfetch = [&](const int64_t* tab, int64_t step, int64_t t) -> int64_t {
    const int64_t k = td.k0 + t * TBK + lane;
    return (!step && t < nk && k < td.k1) ? __ldg(tab + k) : 0;
  };
  const int64_t akstep = d.akstep, bkstep = d.bkstep;
  const int64_t ak0 = akstep ? __ldg(d.ako + td.k0) : 0, bk0 = bkstep ? __ldg(d.bko + td.k0) : 0;
  int64_t ka = kfetch(d.ako, akstep, 0), kb = kfetch(d.bko, bkstep, 0);
  for (int64_t t = 0; t < nk && ok; ++t) {
    const int s = (int)(t & 1);
    if (t >= kTcStages) {  // the MMAs that read this stage two slices ago are done
      if (!mbar_wait(smem_u32(&S.bar[s]), (uint32_t)(((t - kTcStages) >> 1) & 1))) {
        atomicExch(&S.failed, 1);
      }
    }
    __syncthreads();
    if (S.failed) {
      ok = false;
      break;
    }
    const int64_t kvalid = td.k1 - (td.k0 + t * TBK);
    {
      double va[Unit<TBM>::NU], vb[Unit<BN>::NU];
      gather<TBM>(d.a, ka, ak0 + t * TBK * akstep, akstep, roff_a, rok_a, warp, lane, kvalid, va);
      gather<BN>(d.b, kb, bk0 + t * TBK * bkstep, bkstep, roff_b, rok_b, warp, lane, kvalid, vb);
      ka = kfetch(d.ako, akstep, t + 1);  // next slice's offsets, in flight during the stores
      kb = kfetch(d.bko, bkstep, t + 1);
      store_split<TBM>(S.a[s][0], S.a[s][1], warp, lane, va);
      store_split<BN>(S.b[s][0], S.b[s][1], warp, lane, vb);
    }
    // generic-proxy stores -> visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t ah = smem_u32(S.a[s][0]), al = smem_u32(S.a[s][1]);
      const uint32_t bh = smem_u32(S.b[s][0]), bl = smem_u32(S.b[s][1]);
      constexpr uint32_t kA = (TBM / 8) * 128, kB = (BN / 8) * 128;  // next core matrix along K
#pragma unroll
      for (int j = 0; j < TBK / 8; ++j) {  // K = 8 per MMA = two core matrices
        const uint32_t oa = 2 * j * kA, ob = 2 * j * kB;
        const uint64_t dah = smem_desc(ah + oa, kA, 128), dal = smem_desc(al + oa, kA, 128);
        const uint64_t dbh = smem_desc(bh + ob, kB, 128), dbl = smem_desc(bl + ob, kB, 128);
        mma_tf32(tmem, dah, dbh, kIdesc, (t > 0 || j > 0) ? 1u : 0u);
        mma_tf32(tmem, dah, dbl, kIdesc, 1u);
        mma_tf32(tmem, dal, dbh, kIdesc, 1u);
      }
      mma_commit(smem_u32(&S.bar[s]));
    }
    last = t;
  }
  // wait for the last committed slice (a commit covers all earlier MMAs)
  if (last >= 0 && !mbar_wait(smem_u32(&S.bar[last & 1]), (uint32_t)((last >> 1) & 1)))
    ok = false;
  tc_fence_after();
  if (!ok && tid == 0) atomicExch(err, 1);
  if (ok && last >= 0) {
    // epilogue: warp w reads TMEM lanes 32(w%4).. (its rows) and column block w/4
    const int row = 32 * (warp & 3) + lane;
    const int c0 = (warp >> 2) * (BN / (NW / 4));
    const double f = alpha * d.fac;
    double* __restrict__ X = d.c;
    for (int cb = 0; cb < BN / (NW / 4); cb += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(c0 + cb), v);
      if (row >= rows) continue;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int col = c0 + cb + i;
        if (col >= cols || v[i] == 0.0f) continue;
        int64_t off = S.cro[row] + S.cco[col];
        double sg = 1.0;
        if (d.cmapped && !mapped(d.cmap, d.rowspace, S.rc[row], S.cc[col], off, sg)) continue;
        const double val = f * sg * (double)v[i];
        if (d.exclusive)
          X[off] += val;
        else
          atomicAdd(X + off, val);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(tmem), "r"((uint32_t)BN)
                 : "memory");
}

// one CTA per SM (the TMEM allocation of BN <= 256 columns never waits)
static_assert(sizeof(TcSmem<kGemmTcN>) <= 227 * 1024, "tensor-core tile exceeds shared memory");
static_assert(kGemmTcN <= 256 && kGemmTcN % 16 == 0, "UMMA N must be a multiple of 16 up to 256");

template <int BN>
void launch_tc_cfg(const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles, double alpha,
                   int* err, cudaStream_t s) {
  const size_t smem = sizeof(TcSmem<BN>);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_gemm_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    configured = true;
  }
  k_gemm_tc<BN><<<(unsigned)ntiles, TNT, smem, s>>>(descs, tiles, alpha, err);
}

}  // namespace

void launch_gemm_tc(const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles, double alpha,
                    int* err, cudaStream_t s) {
  if (ntiles == 0) return;
  launch_tc_cfg<kGemmTcN>(descs, tiles, ntiles, alpha, err, s);
}

}  // namespace gccu

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
// Two kernels.  k_split_tc reads each operand of each item once, through the
// item's offset tables or, for an operand whose strings merge an external
// and a contracted component, through its gather description (the signed
// string-map gather of collect_block_impr, contract/collect_block_impr.f:397),
// splits it and writes both halves as panels in the K-major core-matrix order
// the tensor core reads (8 rows x 16 bytes per core matrix, no swizzle).
// k_gemm_tc is persistent: one CTA per SM walks the tiles (128 rows x tn
// columns, tn <= 256 chosen per item, one contraction chunk) blockIdx.x,
// +gridDim.x, ... with warp roles.  One thread streams the panel slices of its tiles into a
// 4-stage shared-memory ring with bulk asynchronous copies (cp.async.bulk,
// completion counted in bytes on an mbarrier); one thread issues the MMAs of
// each stage (2 K-steps x 3 products) into one of two TMEM accumulators and
// commits them to the stage's release barrier and, after a tile's last stage,
// to the accumulator's full barrier; eight epilogue warps read a finished
// accumulator back with tcgen05.ld (one TMEM lane per output row), release it
// and scatter it with the map signs while the MMAs of the next tile run in
// the other accumulator.
//
// Every wait on an mbarrier is bounded (the pipeline waits by a runtime
// limit, gccu_set_wait_limit); on time-out the kernel records the failure in
// *err, stops issuing work, waits (bounded by the fixed default limit) for
// the copies and MMAs it has issued, frees its TMEM and returns.
#include <cstdio>

#include "index.cuh"
#include "kernels.hpp"

namespace gccu {

// split-TF32 operand panels of the running contraction (set_tc_workspace)
__device__ float* g_tc_ws;

namespace {

constexpr int TBM = kGemmTcM;  // tile rows = TMEM lanes
constexpr int TBN = kGemmTcN;  // widest tile (columns) = TMEM columns per accumulator
constexpr int SK = (int)kTcSlice;  // contraction indices per panel slice
constexpr int BK = 16;         // contraction indices per pipeline stage
constexpr int NST = 4;         // pipeline stages
// threads: warp 0 producer, warp 1 MMA issuer, warps 2-3 idle, warps 4-11
// epilogue (warp w reads TMEM lanes 32(w%4).., two warps per lane quarter)
constexpr int TNT = 384;
constexpr int kEpiWarp0 = 4, kEpiWarps = 8, kEpiThreads = 32 * kEpiWarps;
// polls of one pipeline wait before it gives up: the default of the
// runtime limit (gccu_set_wait_limit) and the fixed limit of the clean-up
// waits at the end, which only wait for work already issued
constexpr long kWaitLimit = kTcWaitLimitDefault;
constexpr int kTcols = 32;  // columns per pass of the column-major epilogue

struct __align__(1024) TcSmem {
  float a[NST][2][TBM * BK];  // [stage][hi/lo][k/4][row][k%4]
  float b[NST][2][TBN * BK];
  float t[TBM][kTcols + 1];   // column-major epilogue staging
  int64_t cro[TBM], cco[TBN];
  int32_t rc[TBM][kDevMaxComp];
  int32_t cc[TBN][kDevMaxComp];
  GemmDesc d;  // descriptor of the tile in the epilogue
  alignas(8) uint64_t full[NST], empty[NST], accf[2], acce[2], done;
  int64_t issued, consumed;  // stages whose copies were issued / whose MMAs were issued
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
__device__ __forceinline__ uint32_t idesc_tf32(int M, int N) {
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

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" : : "r"(bar) : "memory");
}

// barrier among the epilogue warps only
__device__ __forceinline__ void epi_sync() {
  asm volatile("bar.sync 1, %0;" : : "n"(kEpiThreads) : "memory");
}

// one arrival that also expects `bytes` of asynchronous copies in this phase
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :
               : "r"(bar), "r"(bytes)
               : "memory");
}

// bulk asynchronous copy global -> this CTA's shared memory, counted on bar
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :
      : "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// bounded wait for the completion of phase `parity`: at most `limit` polls;
// false on time-out or when another role of the CTA has failed
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity,
                                          const volatile int* failed, long limit = kWaitLimit) {
  for (long it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (failed && (it & 255) == 255 && *failed) return false;
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

// ---- split pre-pass -------------------------------------------------------
// One block per 128 rows x kSplitGroup consecutive 32-index slices of one
// operand (the rows' offsets and map indices loaded once), one slice after
// the other.  A 128-row x 32-index chunk is read
// coalesced along the operand's contiguous direction (contraction index when
// kfast, else row), split, staged in shared memory in the panel order (each
// k/4 plane padded by 4 floats so that neither read direction conflicts on
// banks) and written out as 16-byte stores, consecutive threads on
// consecutive rows.  A map-addressed operand is read through its gather
// description (the signed string-map gather of collect_block_impr,
// contract/collect_block_impr.f:397, without a dense FP64 panel): the chunk's
// string indices of both sides are staged in shared memory, the element
// offset adds (|map_m[i2 * n1 + i1]| - 1) * ldim_m per map component.
//
// The same kernel makes the int8-slice panels of precision mode 2 in two
// launches over the same chunks: OUT = 1 stages the chunk's values and
// raises the rows' maxima of |x| (atomic maximum on the FP64 bit pattern,
// which orders non-negative values like the values), OUT = 2 cuts every
// element into its IS bytes under its row's scale 127 / m and writes 16-byte
// vectors (16 contraction indices of one row and slice).
constexpr int kSplitThreads = 256;
constexpr int kSplitPitch = 128 * 4 + 4;  // floats per k/4 plane of a staged chunk
constexpr int kValPitch = SK + 1;         // doubles per row of a staged chunk (OUT > 0)
constexpr int kSplitGroup = (int)kTcSplitGroup;  // 32-index slices per block
union SplitStage {
  float sh[2][8 * kSplitPitch];  // split-TF32 planes (OUT = 0)
  double v[128][kValPitch];      // values (OUT = 1, 2)
};

// row maxima of an operand panel (precision mode 2)
__device__ __forceinline__ double* panel_max(const GemmDesc& d, bool row_op) {
  return row_op ? (d.ma_ptr ? d.ma_ptr : reinterpret_cast<double*>(g_tc_ws + d.ma))
                : (d.mb_ptr ? d.mb_ptr : reinterpret_cast<double*>(g_tc_ws + d.mb));
}

template <int OUT, int IS = 1>
__global__ void __launch_bounds__(kSplitThreads, 4)
    k_split_tc(const GemmDesc* __restrict__ descs, const SplitJob* __restrict__ jobs,
               int64_t njobs, const PackJob* __restrict__ gathers) {
  __shared__ __align__(16) SplitStage U;
  float(&sh)[2][8 * kSplitPitch] = U.sh;
  __shared__ double inv_s[128];  // OUT = 2: 127 / row maximum (0 for a zero row)
  __shared__ int64_t ro[128];
  __shared__ int64_t ko[SK];
  __shared__ int32_t rmi_s[kTcGatherMaps][128], kmi_s[kTcGatherMaps][SK];
  __shared__ PackJob G;
  const int tid = threadIdx.x;
  const int64_t blk = blockIdx.x;
  int64_t lo = 0, hi = njobs - 1;  // last job with cstart <= blk
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (jobs[mid].cstart <= blk) lo = mid;
    else hi = mid - 1;
  }
  const SplitJob J = jobs[lo];
  const GemmDesc& d = descs[J.desc];
  const bool row_op = J.op == 0;
  const bool gat = J.gather >= 0;  // block-uniform
  const int64_t R = row_op ? d.M : d.N, K = d.K;
  const int TR = row_op ? TBM : d.tn;
  const PackJob* gp = gat ? gathers + J.gather : nullptr;
  const double* __restrict__ x = gat ? gp->src : row_op ? d.a : d.b;
  const int64_t* rtab = gat ? gp->roff : row_op ? d.aro : d.bco;
  const int64_t* ktab = gat ? gp->koff : row_op ? d.ako : d.bko;
  const int kfast = gat ? gp->kfast : row_op ? d.afast : d.bfast;
  const int64_t nsl = (K + SK - 1) / SK, ngrp = (nsl + kSplitGroup - 1) / kSplitGroup;
  const int64_t c = blk - J.cstart;  // block = row chunk * ngrp + slice group
  const int64_t rc = c / ngrp, r0 = rc * 128;
  const int64_t sl0 = (c % ngrp) * kSplitGroup;
  const int64_t sl1 = sl0 + kSplitGroup < nsl ? sl0 + kSplitGroup : nsl;
  // the chunk's rows: offsets, map string indices and (OUT = 2) scales, once
  // for the block's slices
  if (tid < 128) ro[tid] = r0 + tid < R ? __ldg(rtab + r0 + tid) : -1;
  if constexpr (OUT == 2) {
    if (tid < 128) {
      const double m = r0 + tid < R ? panel_max(d, row_op)[r0 + tid] : 0.0;
      inv_s[tid] = m > 0.0 ? 127.0 / m : 0.0;
    }
  }
  // int8 slicing of a gathered operand whose chunks the row-maxima pass kept
  const bool staged = OUT == 2 && J.stage >= 0;
  if (gat && !staged) {
    const int nw = (int)(sizeof(PackJob) / sizeof(int));
    for (int i = tid; i < nw; i += kSplitThreads)
      reinterpret_cast<int*>(&G)[i] = reinterpret_cast<const int*>(gp)[i];
    const int nm = gp->nm;
    for (int i = tid; i < nm * 128; i += kSplitThreads) {
      const int m = i >> 7, r = i & 127;
      if (r0 + r < R) rmi_s[m][r] = (int32_t)__ldg(gp->rmi + (int64_t)m * R + r0 + r);
    }
  }
  // a 128-row chunk may span two row bands when TR is not a multiple of 128
  const int64_t padded = (R + TR - 1) / TR * TR;
  double mrow = 0.0;  // OUT = 1: this thread's half row, over the block's slices
  for (int64_t sl = sl0; sl < sl1; ++sl) {
    const int64_t k0 = sl * SK;
    double* const stg = J.stage >= 0 ? reinterpret_cast<double*>(g_tc_ws + J.stage) +
                                           (rc * nsl + sl) * (128 * SK)
                                     : nullptr;
    if (tid >= 128 && tid < 128 + SK)
      ko[tid - 128] = k0 + (tid - 128) < K ? __ldg(ktab + k0 + tid - 128) : -1;
    if (gat && !staged) {
      const int nm = gp->nm;
      for (int i = tid; i < nm * SK; i += kSplitThreads) {
        const int m = i / SK, k = i % SK;
        if (k0 + k < K) kmi_s[m][k] = (int32_t)__ldg(gp->kmi + (int64_t)m * K + k0 + k);
      }
    }
    __syncthreads();
    // element (local row r, local index k) of a direct operand
    auto direct = [&](int r, int k) -> double {
      const int64_t rof = ro[r], kof = ko[k];
      return (rof >= 0 && kof >= 0) ? __ldg(x + rof + kof) : 0.0;
    };
    // staging of one chunk of a direct operand: thread mappings per read
    // direction, the element function a template argument so that the loads
    // stay independent (no map branch between them)
    auto stage = [&](auto&& elem) {
      if (kfast) {  // warp: 16 rows, lane: contraction index
        const int warp = tid >> 5, lane = tid & 31;
#pragma unroll 8
        for (int i = 0; i < 16; ++i) {
          const int r = warp * 16 + i;
          const double v = elem(r, lane);
          if constexpr (OUT == 0) {
            float h, l;
            split_tf32(v, h, l);
            sh[0][(lane >> 2) * kSplitPitch + 4 * r + (lane & 3)] = h;
            sh[1][(lane >> 2) * kSplitPitch + 4 * r + (lane & 3)] = l;
          } else {
            U.v[r][lane] = v;
          }
        }
      } else {  // thread: one row, 16 contraction indices
        const int r = tid & 127, kh = tid >> 7;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if constexpr (OUT == 0) {
            float4 h4, l4;
            float* hp = &h4.x;
            float* lp = &l4.x;
#pragma unroll
            for (int e = 0; e < 4; ++e) split_tf32(elem(r, 16 * kh + 4 * q + e), hp[e], lp[e]);
            *reinterpret_cast<float4*>(&sh[0][(4 * kh + q) * kSplitPitch + 4 * r]) = h4;
            *reinterpret_cast<float4*>(&sh[1][(4 * kh + q) * kSplitPitch + 4 * r]) = l4;
          } else {
#pragma unroll
            for (int e = 0; e < 4; ++e) U.v[r][16 * kh + 4 * q + e] = elem(r, 16 * kh + 4 * q + e);
          }
        }
      }
    };
    // map-addressed operand: eight elements at a time, their map lookups of
    // each component issued together, then their value loads, so that the
    // dependent loads of different elements overlap (rows or indices outside
    // the block have ro / ko < 0 and load nothing)
    auto gather8 = [&](const int (&rr)[8], const int (&kk)[8], double (&val)[8]) {
      int64_t off[8];
      bool ok[8], neg[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int64_t rof = ro[rr[e]], kof = ko[kk[e]];
        ok[e] = rof >= 0 && kof >= 0;
        off[e] = ok[e] ? rof + kof : 0;
        neg[e] = false;
      }
      for (int m = 0; m < G.nm; ++m) {
        const bool r1 = G.row_is_1[m] != 0;
        const int32_t* __restrict__ mp = G.map[m];
        const int64_t n1 = G.n1[m], ld = G.ldim[m];
        int v[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int32_t ir = rmi_s[m][rr[e]], ik = kmi_s[m][kk[e]];
          v[e] = ok[e] ? __ldg(mp + (int64_t)(r1 ? ik : ir) * n1 + (r1 ? ir : ik)) : 1;
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          int w = v[e];
          if (w == 0) ok[e] = false;
          if (w < 0) {
            neg[e] = !neg[e];
            w = -w;
          }
          off[e] += (int64_t)(w - 1) * ld;
        }
      }
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const double x0 = ok[e] ? __ldg(x + off[e]) : 0.0;
        val[e] = neg[e] ? -x0 : x0;
      }
    };
    auto stage_mapped = [&]() {
      if (kfast) {  // warp: 16 rows, lane: contraction index
        const int warp = tid >> 5, lane = tid & 31;
#pragma unroll 1
        for (int i0 = 0; i0 < 16; i0 += 8) {
          int rr[8], kk[8];
          double v[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            rr[e] = warp * 16 + i0 + e;
            kk[e] = lane;
          }
          gather8(rr, kk, v);
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            if constexpr (OUT == 0) {
              float h, l;
              split_tf32(v[e], h, l);
              sh[0][(lane >> 2) * kSplitPitch + 4 * rr[e] + (lane & 3)] = h;
              sh[1][(lane >> 2) * kSplitPitch + 4 * rr[e] + (lane & 3)] = l;
            } else {
              U.v[rr[e]][lane] = v[e];
            }
          }
        }
      } else {  // thread: one row, 16 contraction indices
        const int r = tid & 127, kh = tid >> 7;
#pragma unroll 1
        for (int q0 = 0; q0 < 4; q0 += 2) {
          int rr[8], kk[8];
          double v[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            rr[e] = r;
            kk[e] = 16 * kh + 4 * q0 + e;
          }
          gather8(rr, kk, v);
          if constexpr (OUT == 0) {
#pragma unroll
            for (int qq = 0; qq < 2; ++qq) {
              float4 h4, l4;
              float* hp = &h4.x;
              float* lp = &l4.x;
#pragma unroll
              for (int e = 0; e < 4; ++e) split_tf32(v[4 * qq + e], hp[e], lp[e]);
              *reinterpret_cast<float4*>(&sh[0][(4 * kh + q0 + qq) * kSplitPitch + 4 * r]) = h4;
              *reinterpret_cast<float4*>(&sh[1][(4 * kh + q0 + qq) * kSplitPitch + 4 * r]) = l4;
            }
          } else {
#pragma unroll
            for (int e = 0; e < 8; ++e) U.v[r][kk[e]] = v[e];
          }
        }
      }
    };
    if (staged) {
      for (int i = tid; i < 128 * SK; i += kSplitThreads) U.v[i / SK][i % SK] = stg[i];
    } else if (gat) {
      stage_mapped();
    } else {
        stage(direct);
    }
    __syncthreads();
    if constexpr (OUT == 1) {  // rows' maxima: each thread half a row of the chunk
      if (stg)  // the gathered chunk, kept for the slicing pass
        for (int i = tid; i < 128 * SK; i += kSplitThreads) stg[i] = U.v[i / SK][i % SK];
      const int r = tid & 127, kh = tid >> 7;
#pragma unroll
      for (int j = 0; j < 16; ++j) mrow = fmax(mrow, fabs(U.v[r][16 * kh + j]));
    } else if constexpr (OUT == 2) {  // slices: thread = one row x 16 indices (one plane)
      const int r = tid & 127, kh = tid >> 7;
      const int64_t row = r0 + r;
      if (row < padded) {
        const double inv = inv_s[r];
        uint32_t w[IS][4];
#pragma unroll
        for (int s = 0; s < IS; ++s)
#pragma unroll
          for (int q = 0; q < 4; ++q) w[s][q] = 0u;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          double u = U.v[r][16 * kh + j] * inv;  // |u| <= 127
#pragma unroll
          for (int s = 0; s < IS; ++s) {
            const int a = __double2int_rn(u);  // |a| <= 127, then <= 64
            w[s][j >> 2] |= (uint32_t)(a & 0xff) << (8 * (j & 3));
            u = (u - (double)a) * 128.0;  // exact
          }
        }
        uint8_t* const panel = reinterpret_cast<uint8_t*>(
            row_op ? (d.pa_ptr ? d.pa_ptr : g_tc_ws + d.pa)
                   : (d.pb_ptr ? d.pb_ptr : g_tc_ws + d.pb));
        const int64_t band = row / TR, rr = row % TR;
        uint8_t* base = panel + ((band * nsl + sl) * IS * 2 + kh) * TR * 16 + rr * 16;
#pragma unroll
        for (int s = 0; s < IS; ++s)
          *reinterpret_cast<uint4*>(base + (int64_t)s * 2 * TR * 16) =
              make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
      }
    } else {  // split TF32: the staged planes as 16-byte vectors
      float* const panel = row_op ? (d.pa_ptr ? d.pa_ptr : g_tc_ws + d.pa)
                                  : (d.pb_ptr ? d.pb_ptr : g_tc_ws + d.pb);
      float* __restrict__ base = panel + sl * 2 * TR * SK;
#pragma unroll
      for (int i = 0; i < 2 * 8 * 128 / kSplitThreads; ++i) {
        const int u = tid + kSplitThreads * i;
        const int plane = u >> 10, kq = (u >> 7) & 7, r = u & 127;
        const int64_t row = r0 + r;
        if (row >= padded) continue;
        const int64_t band = row / TR, rr = row % TR;
        const float4 v = *reinterpret_cast<const float4*>(&sh[plane][kq * kSplitPitch + 4 * r]);
        *reinterpret_cast<float4*>(base + band * nsl * 2 * TR * SK + plane * TR * SK +
                                   kq * TR * 4 + rr * 4) = v;
      }
    }
    __syncthreads();  // the staging buffers are reused by the next slice
  }
  if constexpr (OUT == 1) {
    const int r = tid & 127;
    if (mrow > 0.0 && r0 + r < R)
      atomicMax(reinterpret_cast<unsigned long long*>(panel_max(d, row_op) + r0 + r),
                (unsigned long long)__double_as_longlong(mrow));
  }
}

// Scatter-add of NB accumulator values (tile rows row[i], columns col[i],
// all inside the tile) into the result: offsets from the row and column
// tables plus the string-map lookups of mapped result components, issued for
// all NB elements together (one batch of independent loads per component),
// then the updates.
template <int NB, typename Smem, typename T>
__device__ __forceinline__ void scatter(const Smem& S, const int (&row)[NB],
                                        const int (&col)[NB], const T (&v)[NB],
                                        int64_t rows, int64_t cols, double f) {
  const GemmDesc& d = S.d;
  int64_t off[NB];
  float sg[NB];
  bool ok[NB];
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    ok[i] = row[i] < rows && col[i] < cols && v[i] != T(0);
    off[i] = ok[i] ? S.cro[row[i]] + S.cco[col[i]] : 0;
    sg[i] = 1.0f;
  }
  if (d.cmapped) {
    const OpndDesc& od = d.cmap;
    for (int j = 0; j < od.ncomp; ++j) {
      const int32_t* mp = od.map[j];
      if (!mp) continue;
      const bool r1 = od.sp1[j] == d.rowspace, r2 = od.sp2[j] == d.rowspace;
      const int ci1 = od.ci1[j], ci2 = od.ci2[j];
      const int64_t n1 = od.n1[j], ld = od.ldim[j];
      int mv[NB];
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        const int32_t* rc = S.rc[row[i]];
        const int32_t* cc = S.cc[col[i]];
        const int i1 = r1 ? rc[ci1] : cc[ci1], i2 = r2 ? rc[ci2] : cc[ci2];
        mv[i] = ok[i] ? __ldg(mp + (int64_t)i2 * n1 + i1) : 1;
      }
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        int m = mv[i];
        if (m == 0) ok[i] = false;
        if (m < 0) {
          sg[i] = -sg[i];
          m = -m;
        }
        off[i] += (int64_t)(m - 1) * ld;
      }
    }
  }
  double* __restrict__ X = d.c;
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    if (!ok[i]) continue;
    const double val = f * (double)sg[i] * (double)v[i];
    if (d.exclusive)
      X[off[i]] += val;
    else
      atomicAdd(X + off[i], val);
  }
}

// ---- GEMM ------------------------------------------------------------------
__global__ void __launch_bounds__(TNT, 1)
    k_gemm_tc(const GemmDesc* __restrict__ descs, const TileDesc* __restrict__ tiles,
              int64_t ntiles, double alpha, int* err, long wait_limit) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(smem_u32(&S.full[s]), 1);
      mbar_init(smem_u32(&S.empty[s]), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(smem_u32(&S.accf[a]), 1);
      mbar_init(smem_u32(&S.acce[a]), kEpiWarps);
    }
    mbar_init(smem_u32(&S.done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    S.failed = 0;
    S.issued = 0;
    S.consumed = 0;
  }
  if (warp == 0) {  // TMEM: two accumulators of TBN f32 columns x 128 lanes
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(&S.tmem_base)), "r"((uint32_t)(2 * TBN))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  volatile int* failed = &S.failed;
  // tiles of this CTA: blockIdx.x + lt * gridDim.x (the grid is at most ntiles)
  const int64_t nmine = (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
  auto tile_of = [&](int64_t lt) { return tiles[blockIdx.x + lt * gridDim.x]; };
  if (warp == 0) {
    if (lane == 0) {  // producer: panel slices -> stage ring
      int64_t it = 0;
      for (int64_t lt = 0; lt < nmine && !*failed; ++lt) {
        const TileDesc td = tile_of(lt);
        const GemmDesc* dg = descs + td.item;
        const int64_t K = dg->K, nsl = (K + SK - 1) / SK, g0 = td.k0 / BK;
        const int64_t nk = (td.k1 - td.k0 + BK - 1) / BK;
        const int bn = dg->tn;
        const uint32_t stage_bytes = 2u * (uint32_t)(TBM + bn) * BK * sizeof(float);
        const float* pa = (dg->pa_ptr ? dg->pa_ptr : g_tc_ws + dg->pa) +
                          (int64_t)(td.m0 / TBM) * nsl * 2 * TBM * SK;
        const float* pb = (dg->pb_ptr ? dg->pb_ptr : g_tc_ws + dg->pb) +
                          (int64_t)(td.n0 / bn) * nsl * 2 * bn * SK;
        for (int64_t t = 0; t < nk; ++t, ++it) {
          const int s = (int)(it % NST);
          if (it >= NST &&
              !mbar_wait(smem_u32(&S.empty[s]), (uint32_t)((it / NST - 1) & 1), failed,
                         wait_limit)) {
            *failed = 1;
            break;
          }
          const int64_t g = g0 + t, sl = g / 2, half = g % 2;
          const float* sa = pa + sl * 2 * TBM * SK + half * TBM * BK;
          const float* sb = pb + sl * 2 * bn * SK + half * bn * BK;
          const uint32_t bar = smem_u32(&S.full[s]);
          mbar_expect_tx(bar, stage_bytes);
          bulk_g2s(S.a[s][0], sa, TBM * BK * sizeof(float), bar);
          bulk_g2s(S.a[s][1], sa + TBM * SK, TBM * BK * sizeof(float), bar);
          bulk_g2s(S.b[s][0], sb, (uint32_t)bn * BK * sizeof(float), bar);
          bulk_g2s(S.b[s][1], sb + bn * SK, (uint32_t)bn * BK * sizeof(float), bar);
          S.issued = it + 1;
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t kA = TBM * 16;  // next core matrix along K (row operand)
      int64_t it = 0;
      for (int64_t lt = 0; lt < nmine && !*failed; ++lt) {
        const TileDesc td = tile_of(lt);
        const int64_t nk = (td.k1 - td.k0 + BK - 1) / BK;
        const int bn = descs[td.item].tn;
        const uint32_t kIdesc = idesc_tf32(TBM, bn), kB = (uint32_t)bn * 16;
        const int acc = (int)(lt & 1);
        if (lt >= 2 &&  // the epilogue has read this accumulator two tiles ago
            !mbar_wait(smem_u32(&S.acce[acc]), (uint32_t)((lt / 2 - 1) & 1), failed,
                       wait_limit)) {
          *failed = 1;
          break;
        }
        tc_fence_after();
        const uint32_t dacc = tmem + (uint32_t)(acc * TBN);
        for (int64_t t = 0; t < nk; ++t, ++it) {
          const int s = (int)(it % NST);
          if (!mbar_wait(smem_u32(&S.full[s]), (uint32_t)((it / NST) & 1), failed, wait_limit)) {
            *failed = 1;
            break;
          }
          tc_fence_after();
          const uint32_t ah = smem_u32(S.a[s][0]), al = smem_u32(S.a[s][1]);
          const uint32_t bh = smem_u32(S.b[s][0]), bl = smem_u32(S.b[s][1]);
#pragma unroll
          for (int j = 0; j < BK / 8; ++j) {  // K = 8 per MMA = two core matrices
            const uint32_t oa = 2 * j * kA, ob = 2 * j * kB;
            const uint64_t dah = smem_desc(ah + oa, kA, 128), dal = smem_desc(al + oa, kA, 128);
            const uint64_t dbh = smem_desc(bh + ob, kB, 128), dbl = smem_desc(bl + ob, kB, 128);
            mma_tf32(dacc, dah, dbh, kIdesc, (t > 0 || j > 0) ? 1u : 0u);
            mma_tf32(dacc, dah, dbl, kIdesc, 1u);
            mma_tf32(dacc, dal, dbh, kIdesc, 1u);
          }
          mma_commit(smem_u32(&S.empty[s]));
          S.consumed = it + 1;
        }
        if (*failed) break;
        mma_commit(smem_u32(&S.accf[acc]));
      }
      mma_commit(smem_u32(&S.done));  // tracks every MMA this thread issued
    }
    __syncwarp();
  } else if (warp >= kEpiWarp0) {
    const int et = tid - 32 * kEpiWarp0, ew = warp - kEpiWarp0;
    const int quarter = warp & 3, half = ew >> 2;  // TMEM lanes 32*quarter.., column half
    for (int64_t lt = 0; lt < nmine; ++lt) {
      const TileDesc td = tile_of(lt);
      {  // descriptor and tables of the tile (the previous tile's are no longer read)
        const int* src = reinterpret_cast<const int*>(descs + td.item);
        int* dst = reinterpret_cast<int*>(&S.d);
        for (int i = et; i < (int)(sizeof(GemmDesc) / sizeof(int)); i += kEpiThreads)
          dst[i] = src[i];
      }
      epi_sync();
      const GemmDesc& d = S.d;
      const int bn = d.tn;  // tile width
      const int64_t rows = d.M - td.m0 < TBM ? d.M - td.m0 : TBM;
      const int64_t cols = d.N - td.n0 < bn ? d.N - td.n0 : bn;
      const int colspace = d.rowspace == kEx1 ? kEx2 : kEx1;
      for (int i = et; i < TBM; i += kEpiThreads)
        if (i < rows) {
          S.cro[i] = d.cro[td.m0 + i];
          if (d.cmapped) decomp(d.rad[d.rowspace], d.nsp[d.rowspace], td.m0 + i, S.rc[i]);
        }
      for (int i = et; i < TBN; i += kEpiThreads)
        if (i < cols) {
          S.cco[i] = d.cco[td.n0 + i];
          if (d.cmapped) decomp(d.rad[colspace], d.nsp[colspace], td.n0 + i, S.cc[i]);
        }
      const int acc = (int)(lt & 1);
      if (!mbar_wait(smem_u32(&S.accf[acc]), (uint32_t)((lt / 2) & 1), failed, wait_limit))
        *failed = 1;
      epi_sync();
      if (*failed) break;  // the same in every epilogue thread after the barrier
      tc_fence_after();
      const uint32_t tacc = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(acc * TBN);
      const double f = alpha * d.fac;
      // result elements adjacent in memory along the columns: lanes should
      // run along columns, the transpose of TMEM's lane = row order
      const bool colfast = rows > 1 && cols > 1 && S.cco[1] - S.cco[0] == 1 &&
                           S.cro[1] - S.cro[0] != 1;
      if (colfast) {
        // passes of kTcols columns: four warps (one per lane quarter, the two
        // sets taking turns) stage the pass in shared memory, then every
        // epilogue warp scatters rows ew, ew+8, .. with lanes on consecutive
        // columns
        for (int c0 = 0; c0 < cols; c0 += kTcols) {
          if (((c0 / kTcols) & 1) == half) {
            const int row = 32 * quarter + lane;
#pragma unroll
            for (int cb = 0; cb < kTcols; cb += 16) {
              float v[16];
              tmem_ld16(tacc + (uint32_t)(c0 + cb), v);
#pragma unroll
              for (int i = 0; i < 16; ++i) S.t[row][cb + i] = v[i];
            }
          }
          epi_sync();
          constexpr int kRows = TBM / kEpiWarps;
          int rr[kRows], cc[kRows];
          float v[kRows];
#pragma unroll
          for (int i = 0; i < kRows; ++i) {
            rr[i] = ew + kEpiWarps * i;
            cc[i] = c0 + lane;
            v[i] = S.t[rr[i]][lane];
          }
          scatter<kRows>(S, rr, cc, v, rows, cols, f);
          epi_sync();
        }
      } else {
        const int row = 32 * quarter + lane;
        const int c0 = half * (bn / 2);
        for (int cb = 0; cb < bn / 2; cb += 16) {
          if (c0 + cb >= cols) break;  // warp-uniform
          float v[16];
          tmem_ld16(tacc + (uint32_t)(c0 + cb), v);
          int rr[16], cc[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            rr[i] = row;
            cc[i] = c0 + cb + i;
          }
          scatter<16>(S, rr, cc, v, rows, cols, f);
        }
      }
      // accumulator read (tcgen05.ld waited in tmem_ld16): release it
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&S.acce[acc]));
      epi_sync();  // tables and descriptor free for the next tile
    }
  }
  __syncthreads();
  if (!mbar_wait(smem_u32(&S.done), 0u, nullptr)) *failed = 1;  // all MMAs complete
  if (tid == 0) {  // copies issued but never consumed (only after a failure)
    for (int64_t t = S.consumed; t < S.issued; ++t)
      if (!mbar_wait(smem_u32(&S.full[t % NST]), (uint32_t)((t / NST) & 1), nullptr))
        *failed = 1;
  }
  __syncthreads();
  if (*failed && tid == 0) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(tmem), "r"((uint32_t)(2 * TBN))
                 : "memory");
}

// one CTA per SM (the TMEM allocation of all 512 columns never waits)
static_assert(sizeof(TcSmem) <= 227 * 1024, "tensor-core tile exceeds shared memory");
static_assert(TBN <= 256 && TBN % 16 == 0, "UMMA N must be a multiple of 16 up to 256");
static_assert(SK % BK == 0 && SK / BK == 2, "a stage is half a panel slice");
static_assert((TBM * BK * sizeof(float)) % 16 == 0 && (TBN * BK * sizeof(float)) % 16 == 0,
              "bulk copies move multiples of 16 bytes");
static_assert(TBM % kEpiWarps == 0 && kTcols % 16 == 0 && TBN % 32 == 0,
              "epilogue passes (tile widths are multiples of 32)");


// ---- int8-slice GEMM (precision modes 2 and 3) -----------------------------
// The structure of k_gemm_tc (persistent, producer / MMA / epilogue warps,
// bounded waits), with the slices: a stage is one 32-index slice of all IS
// row-operand and column-operand slices (one bulk copy each); the MMA thread
// issues, per stage, the products of slices (s, t) with s + t < IS into
// accumulator s + t (kind::i8, int32, K = 32 per instruction).  The IS
// accumulators of a tile take IS * tn TMEM columns, so there is one set.
// With tiles up to 96 columns (IS = 5) the epilogue reads the set into
// registers (FP64, sum over s + t of 2^(-7(s+t)) times the accumulator, exact
// before the last rounding), releases it to the MMAs of the next tile and
// then scales by the rows' and columns' m / 127 and scatters from the
// registers; with 128-column tiles (IS = 4) a thread's 64 values do not fit
// its registers, so the epilogue combines, scales and scatters column group
// by column group from TMEM and releases the set at the end of the tile.
constexpr int INST = 4;  // pipeline stages

template <int IS, int IBN>
struct __align__(1024) I8Smem {
  static constexpr int kStageA = IS * 2 * TBM * 16;  // bytes of one stage, row operand
  static constexpr int kStageB = IS * 2 * IBN * 16;  // ... column operand, widest tile
  uint8_t a[INST][kStageA];  // [stage][slice s][k/16][row][k%16]
  uint8_t b[INST][kStageB];
  double t[TBM][kTcols + 1];  // column-major epilogue staging
  int64_t cro[TBM], cco[IBN];
  double rs[TBM], cs[IBN];  // row / column scales m / 127
  int32_t rc[TBM][kDevMaxComp];
  int32_t cc[IBN][kDevMaxComp];
  GemmDesc d;
  alignas(8) uint64_t full[INST], empty[INST], accf, acce, done;
  int64_t issued, consumed;
  uint32_t tmem_base;
  int failed;
};

// instruction descriptor: D s32, A/B signed 8-bit, both K-major, M x N
__device__ __forceinline__ uint32_t idesc_i8(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// 8 consecutive 32-bit accumulator columns of this thread's TMEM lane,
// without waiting (tmem_wait_ld before the registers are used)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// the FP64 values of 8 consecutive columns of this thread's TMEM lane:
// sum over the IS accumulators (one per slice order d, d * bn columns on)
// of 2^(-7d) times the int32 sum, smallest orders first
template <int IS>
__device__ __forceinline__ void i8_combine8(uint32_t taddr, int bn, double (&x)[8]) {
  uint32_t q[IS][8];
#pragma unroll
  for (int dd = 0; dd < IS; ++dd) tmem_ld8(taddr + (uint32_t)(dd * bn), q[dd]);
  tmem_wait_ld();
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    double v = 0.0;
#pragma unroll
    for (int dd = IS - 1; dd >= 0; --dd) v += ldexp(1.0, -7 * dd) * (double)(int)q[dd][j];
    x[j] = v;
  }
}

template <int IS, int IBN>
__global__ void __launch_bounds__(TNT, 1)
    k_gemm_i8(const GemmDesc* __restrict__ descs, const TileDesc* __restrict__ tiles,
              int64_t ntiles, double alpha, int* err, long wait_limit) {
  using Sm = I8Smem<IS, IBN>;
  constexpr int kStageA = Sm::kStageA;
  constexpr bool kEarly = IBN <= 96;  // release TMEM before the scatter (values in registers)
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  Sm& S = *reinterpret_cast<Sm*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    for (int s = 0; s < INST; ++s) {
      mbar_init(smem_u32(&S.full[s]), 1);
      mbar_init(smem_u32(&S.empty[s]), 1);
    }
    mbar_init(smem_u32(&S.accf), 1);
    mbar_init(smem_u32(&S.acce), kEpiWarps);
    mbar_init(smem_u32(&S.done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    S.failed = 0;
    S.issued = 0;
    S.consumed = 0;
  }
  if (warp == 0) {  // TMEM: all 512 columns (the IS accumulators of one tile)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(&S.tmem_base)), "r"(512u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  volatile int* failed = &S.failed;
  const int64_t nmine = (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
  auto tile_of = [&](int64_t lt) { return tiles[blockIdx.x + lt * gridDim.x]; };
  if (warp == 0) {
    if (lane == 0) {  // producer: one 32-index slice of all slices per stage
      int64_t it = 0;
      for (int64_t lt = 0; lt < nmine && !*failed; ++lt) {
        const TileDesc td = tile_of(lt);
        const GemmDesc* dg = descs + td.item;
        const int64_t K = dg->K, nsl = (K + SK - 1) / SK, g0 = td.k0 / SK;
        const int64_t nk = (td.k1 - td.k0 + SK - 1) / SK;
        const int bn = dg->tn;
        const uint32_t sb = (uint32_t)(IS * 2 * bn * 16);
        const uint8_t* pa =
            reinterpret_cast<const uint8_t*>(dg->pa_ptr ? dg->pa_ptr : g_tc_ws + dg->pa) +
            (int64_t)(td.m0 / TBM) * nsl * kStageA;
        const uint8_t* pb =
            reinterpret_cast<const uint8_t*>(dg->pb_ptr ? dg->pb_ptr : g_tc_ws + dg->pb) +
            (int64_t)(td.n0 / bn) * nsl * sb;
        for (int64_t t = 0; t < nk; ++t, ++it) {
          const int s = (int)(it % INST);
          if (it >= INST &&
              !mbar_wait(smem_u32(&S.empty[s]), (uint32_t)((it / INST - 1) & 1), failed,
                         wait_limit)) {
            *failed = 1;
            break;
          }
          const uint32_t bar = smem_u32(&S.full[s]);
          mbar_expect_tx(bar, (uint32_t)kStageA + sb);
          bulk_g2s(S.a[s], pa + (g0 + t) * kStageA, (uint32_t)kStageA, bar);
          bulk_g2s(S.b[s], pb + (g0 + t) * sb, sb, bar);
          S.issued = it + 1;
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t kA = TBM * 16;  // next core matrix along K (row operand)
      int64_t it = 0;
      for (int64_t lt = 0; lt < nmine && !*failed; ++lt) {
        const TileDesc td = tile_of(lt);
        const int64_t nk = (td.k1 - td.k0 + SK - 1) / SK;
        const int bn = descs[td.item].tn;
        const uint32_t idesc = idesc_i8(TBM, bn), kB = (uint32_t)bn * 16;
        const uint32_t bslice = 2 * kB / 16;  // next column-operand slice, descriptor units
        if (lt >= 1 &&  // the epilogue has read the previous tile's accumulators
            !mbar_wait(smem_u32(&S.acce), (uint32_t)((lt - 1) & 1), failed, wait_limit)) {
          *failed = 1;
          break;
        }
        tc_fence_after();
        for (int64_t t = 0; t < nk; ++t, ++it) {
          const int s = (int)(it % INST);
          if (!mbar_wait(smem_u32(&S.full[s]), (uint32_t)((it / INST) & 1), failed, wait_limit)) {
            *failed = 1;
            break;
          }
          tc_fence_after();
          // the stage's descriptors once; a slice's descriptor is the base's
          // plus its offset / 16 in the address field (offsets stay inside
          // the 256 KB window the 14-bit field addresses, no carry)
          const uint64_t da0 = smem_desc(smem_u32(S.a[s]), kA, 128);
          const uint64_t db0 = smem_desc(smem_u32(S.b[s]), kB, 128);
          if (t == 0) {
#pragma unroll
            for (int dd = 0; dd < IS; ++dd)
#pragma unroll
              for (int sa = 0; sa <= dd; ++sa)
                mma_i8(tmem + (uint32_t)(dd * bn), da0 + (uint64_t)(sa * 2 * kA / 16),
                       db0 + (uint64_t)((dd - sa) * bslice), idesc, sa > 0 ? 1u : 0u);
          } else {
#pragma unroll
            for (int dd = 0; dd < IS; ++dd)
#pragma unroll
              for (int sa = 0; sa <= dd; ++sa)
                mma_i8(tmem + (uint32_t)(dd * bn), da0 + (uint64_t)(sa * 2 * kA / 16),
                       db0 + (uint64_t)((dd - sa) * bslice), idesc, 1u);
          }
          mma_commit(smem_u32(&S.empty[s]));
          S.consumed = it + 1;
        }
        if (*failed) break;
        mma_commit(smem_u32(&S.accf));
      }
      mma_commit(smem_u32(&S.done));  // tracks every MMA this thread issued
    }
    __syncwarp();
  } else if (warp >= kEpiWarp0) {
    const int et = tid - 32 * kEpiWarp0, ew = warp - kEpiWarp0;
    const int quarter = warp & 3, half = ew >> 2;  // TMEM lanes 32*quarter.., column half
    for (int64_t lt = 0; lt < nmine; ++lt) {
      const TileDesc td = tile_of(lt);
      {
        const int* src = reinterpret_cast<const int*>(descs + td.item);
        int* dst = reinterpret_cast<int*>(&S.d);
        for (int i = et; i < (int)(sizeof(GemmDesc) / sizeof(int)); i += kEpiThreads)
          dst[i] = src[i];
      }
      epi_sync();
      const GemmDesc& d = S.d;
      const int bn = d.tn;
      const int64_t rows = d.M - td.m0 < TBM ? d.M - td.m0 : TBM;
      const int64_t cols = d.N - td.n0 < bn ? d.N - td.n0 : bn;
      const int colspace = d.rowspace == kEx1 ? kEx2 : kEx1;
      const double* mr = panel_max(d, true);
      const double* mc = panel_max(d, false);
      for (int i = et; i < TBM; i += kEpiThreads)
        if (i < rows) {
          S.cro[i] = d.cro[td.m0 + i];
          S.rs[i] = mr[td.m0 + i] * (1.0 / 127.0);
          if (d.cmapped) decomp(d.rad[d.rowspace], d.nsp[d.rowspace], td.m0 + i, S.rc[i]);
        }
      for (int i = et; i < IBN; i += kEpiThreads)
        if (i < cols) {
          S.cco[i] = d.cco[td.n0 + i];
          S.cs[i] = mc[td.n0 + i] * (1.0 / 127.0);
          if (d.cmapped) decomp(d.rad[colspace], d.nsp[colspace], td.n0 + i, S.cc[i]);
        }
      if (!mbar_wait(smem_u32(&S.accf), (uint32_t)(lt & 1), failed, wait_limit)) *failed = 1;
      epi_sync();
      if (*failed) break;  // the same in every epilogue thread after the barrier
      tc_fence_after();
      const int row = 32 * quarter + lane;
      const uint32_t tq = tmem + ((uint32_t)(32 * quarter) << 16);  // this warp's lanes
      const double f = alpha * d.fac;
      const double rsc = row < rows ? S.rs[row] : 0.0;
      const bool colfast = rows > 1 && cols > 1 && S.cco[1] - S.cco[0] == 1 &&
                           S.cro[1] - S.cro[0] != 1;
      constexpr int kRows = TBM / kEpiWarps, kBatch = 8;
      // one staged pass of kTcols columns: every epilogue warp scatters rows
      // ew, ew+8, .. with lanes on consecutive columns
      auto scatter_pass = [&](int p0) {
#pragma unroll
        for (int i0 = 0; i0 < kRows; i0 += kBatch) {
          int rr[kBatch], cc[kBatch];
          double y[kBatch];
#pragma unroll
          for (int i = 0; i < kBatch; ++i) {
            rr[i] = ew + kEpiWarps * (i0 + i);
            cc[i] = p0 + lane;
            y[i] = S.t[rr[i]][lane];
          }
          scatter<kBatch>(S, rr, cc, y, rows, cols, f);
        }
      };
      if constexpr (kEarly) {
        // this thread: columns c0 .. c0 + bn/2 - 1 of its row, into registers
        const int c0 = half * (bn / 2);
        double v[IBN / 2];
#pragma unroll
        for (int cb = 0; cb < IBN / 2; cb += 8) {
          double x[8];
          if (cb < bn / 2) {  // warp-uniform
            i8_combine8<IS>(tq + (uint32_t)(c0 + cb), bn, x);
          } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = 0.0;
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) v[cb + j] = x[j];
        }
        // accumulators read (tcgen05.ld waited): release them to the next tile
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&S.acce));
        if (colfast) {
          for (int p0 = 0; p0 < cols; p0 += kTcols) {
#pragma unroll
            for (int j = 0; j < IBN / 2; ++j) {
              const int col = c0 + j;
              if (j < bn / 2 && col >= p0 && col < p0 + kTcols)
                S.t[row][col - p0] = col < cols ? v[j] * rsc * S.cs[col] : 0.0;
            }
            epi_sync();
            scatter_pass(p0);
            epi_sync();
          }
        } else {
#pragma unroll
          for (int cb = 0; cb < IBN / 2; cb += 8) {
            if (cb >= bn / 2 || c0 + cb >= cols) break;  // warp-uniform
            int rr[8], cc[8];
            double y[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              rr[i] = row;
              cc[i] = c0 + cb + i;
              y[i] = cc[i] < cols ? v[cb + i] * rsc * S.cs[cc[i]] : 0.0;
            }
            scatter<8>(S, rr, cc, y, rows, cols, f);
          }
        }
      } else {
        // combined, scaled and scattered from TMEM column group by column
        // group; the accumulators are released at the end of the tile
        if (colfast) {
          for (int p0 = 0; p0 < cols; p0 += kTcols) {
            if (((p0 / kTcols) & 1) == half) {  // the warps of one half stage the pass
#pragma unroll
              for (int cb = 0; cb < kTcols; cb += 8) {
                double x[8];
                i8_combine8<IS>(tq + (uint32_t)(p0 + cb), bn, x);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                  const int col = p0 + cb + j;
                  S.t[row][cb + j] = col < cols ? x[j] * rsc * S.cs[col] : 0.0;
                }
              }
            }
            epi_sync();
            scatter_pass(p0);
            epi_sync();
          }
        } else {
          const int c0 = half * (bn / 2);
          for (int cb = 0; cb < bn / 2; cb += 8) {
            if (c0 + cb >= cols) break;  // warp-uniform
            double x[8];
            i8_combine8<IS>(tq + (uint32_t)(c0 + cb), bn, x);
            int rr[8], cc[8];
            double y[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              rr[i] = row;
              cc[i] = c0 + cb + i;
              y[i] = cc[i] < cols ? x[i] * rsc * S.cs[cc[i]] : 0.0;
            }
            scatter<8>(S, rr, cc, y, rows, cols, f);
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&S.acce));
      }
      epi_sync();  // tables and descriptor free for the next tile
    }
  }
  __syncthreads();
  if (!mbar_wait(smem_u32(&S.done), 0u, nullptr)) *failed = 1;  // all MMAs complete
  if (tid == 0) {  // copies issued but never consumed (only after a failure)
    for (int64_t t = S.consumed; t < S.issued; ++t)
      if (!mbar_wait(smem_u32(&S.full[t % INST]), (uint32_t)((t / INST) & 1), nullptr))
        *failed = 1;
  }
  __syncthreads();
  if (*failed && tid == 0) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(tmem), "r"(512u)
                 : "memory");
}

static_assert(sizeof(I8Smem<kI8SlicesFine, kI8NFine>) <= 227 * 1024 &&
                  sizeof(I8Smem<kI8SlicesFast, kI8NFast>) <= 227 * 1024,
              "int8 tile exceeds shared memory");
static_assert(kI8NFine % 32 == 0 && kI8NFast % 32 == 0 && kI8NFine / 2 % 8 == 0,
              "int8 tile widths: epilogue column groups");


}  // namespace

cudaError_t set_tc_workspace(float* ws) {
  return cudaMemcpyToSymbol(g_tc_ws, &ws, sizeof(ws));
}

void launch_split_tc(const GemmDesc* descs, const SplitJob* jobs, int64_t njobs, int64_t nchunks,
                     const PackJob* gathers, cudaStream_t s) {
  if (njobs == 0 || nchunks == 0) return;
  k_split_tc<0><<<(unsigned)nchunks, kSplitThreads, 0, s>>>(descs, jobs, njobs, gathers);
}

__global__ void k_zero_tc(float* base, int64_t off, int64_t n) {
  float* p = (base ? base : g_tc_ws) + off;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = 0.0f;
}

void launch_zero_tc(float* base, int64_t off, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  const int64_t blocks = (n + 255) / 256;
  k_zero_tc<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, s>>>(base, off, n);
}

void launch_slice_i8(int phase, int slices, const GemmDesc* descs, const SplitJob* jobs,
                     int64_t njobs, int64_t nchunks, const PackJob* gathers, cudaStream_t s) {
  if (njobs == 0 || nchunks == 0) return;
  if (phase == 0)
    k_split_tc<1><<<(unsigned)nchunks, kSplitThreads, 0, s>>>(descs, jobs, njobs, gathers);
  else if (slices == kI8SlicesFast)
    k_split_tc<2, kI8SlicesFast>
        <<<(unsigned)nchunks, kSplitThreads, 0, s>>>(descs, jobs, njobs, gathers);
  else
    k_split_tc<2, kI8SlicesFine>
        <<<(unsigned)nchunks, kSplitThreads, 0, s>>>(descs, jobs, njobs, gathers);
}

void launch_gemm_tc(const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles, double alpha,
                    int* err, int64_t wait_limit, cudaStream_t s) {
  if (ntiles == 0) return;
  const size_t smem = sizeof(TcSmem);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    configured = true;
  }
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 148;
  }
  const int64_t grid = ntiles < nsm ? ntiles : nsm;
  k_gemm_tc<<<(unsigned)grid, TNT, smem, s>>>(descs, tiles, ntiles, alpha, err,
                                                (long)wait_limit);
}

cudaError_t tc_kernel_attributes(cudaFuncAttributes* attr) {
  return cudaFuncGetAttributes(attr, k_gemm_tc);
}

template <int IS, int IBN>
static void launch_gemm_i8_t(const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles,
                             double alpha, int* err, int64_t wait_limit, cudaStream_t s) {
  const size_t smem = sizeof(I8Smem<IS, IBN>);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_gemm_i8<IS, IBN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    configured = true;
  }
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 148;
  }
  const int64_t grid = ntiles < nsm ? ntiles : nsm;
  k_gemm_i8<IS, IBN><<<(unsigned)grid, TNT, smem, s>>>(descs, tiles, ntiles, alpha, err,
                                                         (long)wait_limit);
}

void launch_gemm_i8(int slices, const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles,
                    double alpha, int* err, int64_t wait_limit, cudaStream_t s) {
  if (ntiles == 0) return;
  if (slices == kI8SlicesFast)
    launch_gemm_i8_t<kI8SlicesFast, kI8NFast>(descs, tiles, ntiles, alpha, err, wait_limit, s);
  else
    launch_gemm_i8_t<kI8SlicesFine, kI8NFine>(descs, tiles, ntiles, alpha, err, wait_limit, s);
}

cudaError_t i8_kernel_attributes(cudaFuncAttributes* attr) {
  return cudaFuncGetAttributes(attr, k_gemm_i8<kI8SlicesFine, kI8NFine>);
}

}  // namespace gccu

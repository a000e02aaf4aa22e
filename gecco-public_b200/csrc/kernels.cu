// Device kernels of the engine (sm_100a).
//
//  k_strmap      signed (str1,str2)->str12 string maps, one thread per pair
//                (set_strmap_kernel, strings/set_strmap_kernel.f:66-119 with
//                iordstr2, strings/iordstr2.f, and idx4sg,
//                strings/idx4sg.f).  Integer work, bit-exact.
//  k_contract    all block contractions of one binary contraction in one
//                launch.  Per 64x64 output tile: the operand panels are
//                gathered through the string maps into shared memory with
//                their signs (collect_block_impr, contract/
//                collect_block_impr.f), multiplied with FP64 tensor-core MMA
//                (the dgemm of contract/contr_blk1blk2_blocked_mm.f:465,523)
//                and scatter-added into the result with sign and factor
//                (scatter_block, contract/scatter_block.f:163).
//  bandwidth     add_opblk, diavc, norms, dot products, scaling, sym_ab.
#include <cstdio>

#include "kernels.hpp"

namespace gccu {
namespace {

constexpr int BM = kTileM, BN = kTileN, BK = kTileK;
constexpr int NT = 128;  // 4 warps, 2x2 warp grid of 32x32 sub-tiles
constexpr int PAD = 8;

// ---------------------------------------------------------------------------
// string maps
// ---------------------------------------------------------------------------
__global__ void k_strmap(const int32_t* __restrict__ t1, int e1, int64_t n1,
                         const int32_t* __restrict__ t2, int e2, int64_t n2,
                         const int64_t* __restrict__ W, const int8_t* __restrict__ irr, int nel,
                         int nsym, int32_t* __restrict__ out) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n1 * n2) return;
  int64_t i1 = idx % n1, i2 = idx / n1;
  int o1[8], s1[8], o2[8], s2[8], o[16], sp[16];
  for (int p = 0; p < e1; ++p) {
    int v = t1[i1 * e1 + p];
    int c = v & 3;
    o1[p] = v >> 2;
    s1[p] = c == 1 ? 1 : (c == 2 ? -1 : 2);
  }
  for (int p = 0; p < e2; ++p) {
    int v = t2[i2 * e2 + p];
    int c = v & 3;
    o2[p] = v >> 2;
    s2[p] = c == 1 ? 1 : (c == 2 ? -1 : 2);
  }
  // merge the two ordered strings; parity of the permutation, 0 if an orbital
  // would be occupied twice with the same spin (iordstr2)
  int p1 = 0, p2 = 0, perm = 0;
  for (int p = 0; p < e1 + e2; ++p) {
    if (p1 < e1 && p2 < e2 && o1[p1] == o2[p2] && s1[p1] * s2[p2] != -1) {
      out[idx] = 0;
      return;
    }
    bool take1 = p2 >= e2 || (p1 < e1 && (o1[p1] < o2[p2] || (o1[p1] == o2[p2] && s1[p1] == 1)));
    if (take1) {
      o[p] = o1[p1];
      sp[p] = s1[p1];
      ++p1;
    } else {
      o[p] = o2[p2];
      sp[p] = s2[p2];
      ++p2;
      perm += e1 - p1;
    }
  }
  for (int p = 0; p + 1 < e1 + e2; ++p)
    if (o[p] == o[p + 1]) sp[p] = sp[p + 1] = 2;
  // lexical address in the merged graph: sum of arc weights
  const int NM = 2 * nel + 1;
  int64_t a = 0;
  int n = 0, m = 0, g = 0;
  for (int p = 0; p < e1 + e2;) {
    int k = o[p];
    int c = sp[p] == 2 ? 3 : (sp[p] > 0 ? 1 : 2);
    a += W[((((int64_t)k * 3 + c - 1) * (nel + 1) + n) * NM + m + nel) * nsym + g];
    if (c == 3) {
      n += 2;
      p += 2;
    } else {
      n += 1;
      m += (c == 1) ? 1 : -1;
      g ^= irr[k];
      p += 1;
    }
  }
  int sign = (perm & 1) ? -1 : 1;
  out[idx] = sign * (int32_t)(a + 1);
}

// ---------------------------------------------------------------------------
// grouped FP64 block contraction
// ---------------------------------------------------------------------------
struct __align__(16) Smem {
  double As[BK][BM + PAD];
  double Bs[BK][BN + PAD];
  int64_t rp1[BM], rp12[BM], cp2[BN], cp12[BN], kp1[BK], kp2[BK];
  int32_t rc[BM][kDevMaxComp];
  int32_t cc[BN][kDevMaxComp];
  int32_t kc[BK][kDevMaxComp];
  ItemDesc it;
};

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// decompose composite index x of a space into its component indices and the
// part of the offsets of the operands that depends on this space only
__device__ __forceinline__ void decomp(const ItemDesc& it, int space, int64_t x, int32_t* comp) {
  for (int q = 0; q < it.nsp[space]; ++q) {
    int32_t r = it.rad[space][q];
    comp[q] = (int32_t)(x % r);
    x /= r;
  }
}
__device__ __forceinline__ int64_t part(const OpndDesc& od, int space, const int32_t* comp) {
  int64_t off = 0;
  for (int j = 0; j < od.ncomp; ++j) {
    if (od.map[j]) continue;
    if (od.sp1[j] == space) off += (int64_t)comp[od.ci1[j]] * od.ldim[j];
    else if (od.sp2[j] == space) off += (int64_t)comp[od.ci2[j]] * od.ldim[j];
  }
  return off;
}
// contributions of the components that merge two spaces (map lookups)
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

__global__ void __launch_bounds__(NT) k_contract(const ItemDesc* __restrict__ items,
                                                 const TileDesc* __restrict__ tiles,
                                                 const double* __restrict__ x1,
                                                 const double* __restrict__ x2,
                                                 double* __restrict__ x12, double alpha) {
  __shared__ Smem S;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const TileDesc td = tiles[blockIdx.x];
  {
    const int* src = reinterpret_cast<const int*>(items + td.item);
    int* dst = reinterpret_cast<int*>(&S.it);
    for (int i = tid; i < (int)(sizeof(ItemDesc) / sizeof(int)); i += NT) dst[i] = src[i];
  }
  __syncthreads();
  const ItemDesc& it = S.it;
  const int64_t M = it.M, N = it.N;
  // rows (ex1) and columns (ex2) of this tile
  if (tid < BM) {
    int64_t r = td.m0 + tid;
    if (r < M) {
      decomp(it, kEx1, r, S.rc[tid]);
      S.rp1[tid] = part(it.op[0], kEx1, S.rc[tid]);
      S.rp12[tid] = part(it.op[2], kEx1, S.rc[tid]);
    }
  } else {
    int j = tid - BM;
    int64_t c = td.n0 + j;
    if (c < N) {
      decomp(it, kEx2, c, S.cc[j]);
      S.cp2[j] = part(it.op[1], kEx2, S.cc[j]);
      S.cp12[j] = part(it.op[2], kEx2, S.cc[j]);
    }
  }
  const int wm = warp >> 1, wn = warp & 1;
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const bool map1 = it.op[0].nmap > 0, map2 = it.op[1].nmap > 0;
  const double* X1 = x1 + it.base1;
  const double* X2 = x2 + it.base2;
  for (int64_t k0 = td.k0; k0 < td.k1; k0 += BK) {
    __syncthreads();  // previous tile consumed, row/col info visible
    if (tid < BK) {
      int64_t k = k0 + tid;
      if (k < td.k1) {
        decomp(it, kCnt, k, S.kc[tid]);
        S.kp1[tid] = part(it.op[0], kCnt, S.kc[tid]);
        S.kp2[tid] = part(it.op[1], kCnt, S.kc[tid]);
      }
    }
    __syncthreads();
    // gather the op1 panel (rows ex1, columns cnt) with signs
#pragma unroll
    for (int e = 0; e < (BM * BK) / NT; ++e) {
      int i, kk;
      if (it.kfast1) {
        kk = tid & (BK - 1);
        i = (tid >> 4) + e * (NT / BK);
      } else {
        i = tid & (BM - 1);
        kk = (tid >> 6) + e * (NT / BM);
      }
      double v = 0.0;
      if (td.m0 + i < M && k0 + kk < td.k1) {
        int64_t off = S.rp1[i] + S.kp1[kk];
        double sg = 1.0;
        bool ok = !map1 || mapped(it.op[0], kEx1, S.rc[i], S.kc[kk], off, sg);
        if (ok) v = sg * __ldg(X1 + off);
      }
      S.As[kk][i] = v;
    }
    // gather the op2 panel (rows cnt, columns ex2)
#pragma unroll
    for (int e = 0; e < (BN * BK) / NT; ++e) {
      int j, kk;
      if (it.kfast2) {
        kk = tid & (BK - 1);
        j = (tid >> 4) + e * (NT / BK);
      } else {
        j = tid & (BN - 1);
        kk = (tid >> 6) + e * (NT / BN);
      }
      double v = 0.0;
      if (td.n0 + j < N && k0 + kk < td.k1) {
        int64_t off = S.cp2[j] + S.kp2[kk];
        double sg = 1.0;
        bool ok = !map2 || mapped(it.op[1], kEx2, S.cc[j], S.kc[kk], off, sg);
        if (ok) v = sg * __ldg(X2 + off);
      }
      S.Bs[kk][j] = v;
    }
    __syncthreads();
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = S.As[k4 + (lane & 3)][wm * 32 + i * 8 + (lane >> 2)];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = S.Bs[k4 + (lane & 3)][wn * 32 + j * 8 + (lane >> 2)];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
  }
  // signed scatter-add into the result (several items and K splits may hit
  // the same elements, hence atomics)
  const double f = alpha * it.fac;
  const bool map12 = it.op[2].nmap > 0;
  double* X12 = x12 + it.base12;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        int row = wm * 32 + i * 8 + (lane >> 2);
        int col = wn * 32 + j * 8 + 2 * (lane & 3) + h;
        double v = acc[i][j][h];
        if (td.m0 + row >= M || td.n0 + col >= N || v == 0.0) continue;
        int64_t off = S.rp12[row] + S.cp12[col];
        double sg = 1.0;
        if (map12 && !mapped(it.op[2], kEx1, S.rc[row], S.cc[col], off, sg)) continue;
        atomicAdd(X12 + off, f * sg * v);
      }
}

// ---------------------------------------------------------------------------
// bandwidth kernels
// ---------------------------------------------------------------------------
__global__ void k_axpy(double* __restrict__ out, const double* __restrict__ in, double fac,
                       int64_t n, int reset) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (reset ? 0.0 : out[i]) + fac * in[i];
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  v = 0.0;
  if (threadIdx.x < (blockDim.x >> 5)) v = red[threadIdx.x];
  if (threadIdx.x < 32)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__global__ void k_dot(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                      double* acc) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    s += a[i] * b[i];
  s = block_sum(s);
  if (threadIdx.x == 0) atomicAdd(acc, s);
}

__global__ void k_scale(double* __restrict__ x, double fac, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= fac;
}

__global__ void k_diavc(double* __restrict__ out, const double* __restrict__ in,
                        const double* __restrict__ diag, double fac, double shift, int64_t n) {
  const double thresh = 1e-10;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double d = diag[i] + shift;
    if (fabs(d) <= thresh) d = thresh;
    out[i] = fac * in[i] / d;
  }
}

__global__ void k_sym_ab(const FlipDesc* __restrict__ ds, double* __restrict__ x, double pre) {
  const FlipDesc& d = ds[blockIdx.y];
  int64_t n = d.lenc * d.lena;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t ia = e / d.lenc, ic = e % d.lenc;
    int64_t o1 = 0, o2 = 0;
    int sg = 1;
    for (int k = 0; k < d.na; ++k) {
      int64_t s = ia % d.la[k];
      ia /= d.la[k];
      int v = d.fa[k][s];
      if (v < 0) sg = -sg, v = -v;
      o1 += s * d.lda[k];
      o2 += (int64_t)(v - 1) * d.lda[k];
    }
    for (int k = 0; k < d.nc; ++k) {
      int64_t s = ic % d.lc[k];
      ic /= d.lc[k];
      int v = d.fc[k][s];
      if (v < 0) sg = -sg, v = -v;
      o1 += s * d.ldc[k];
      o2 += (int64_t)(v - 1) * d.ldc[k];
    }
    int64_t i1 = d.off1 + o1, i2 = d.off2 + o2;
    if (i1 > i2) continue;
    double s = sg * d.sgn;
    double v = pre * (x[i1] + s * x[i2]);
    x[i1] = v;
    x[i2] = s * v;
  }
}

inline int grid_for(int64_t n, int bs) {
  int64_t g = (n + bs - 1) / bs;
  if (g > 148 * 32) g = 148 * 32;
  return (int)(g < 1 ? 1 : g);
}

}  // namespace

void launch_strmap(const int32_t* tab1, int nel1, int64_t n1, const int32_t* tab2, int nel2,
                   int64_t n2, const int64_t* W12, const int8_t* irrep12, int nel12, int nsym,
                   int32_t* out, cudaStream_t s) {
  int64_t n = n1 * n2;
  if (n == 0) return;
  k_strmap<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(tab1, nel1, n1, tab2, nel2, n2, W12,
                                                       irrep12, nel12, nsym, out);
}

void launch_contract(const ItemDesc* items, const TileDesc* tiles, int64_t ntiles,
                     const double* x1, const double* x2, double* x12, double alpha,
                     cudaStream_t s) {
  if (ntiles == 0) return;
  k_contract<<<(unsigned)ntiles, NT, 0, s>>>(items, tiles, x1, x2, x12, alpha);
}

void launch_axpy(double* out, const double* in, double fac, int64_t n, int reset,
                 cudaStream_t s) {
  if (n == 0) return;
  k_axpy<<<grid_for(n, 256), 256, 0, s>>>(out, in, fac, n, reset);
}
void launch_sumsq(const double* x, int64_t n, double* acc, cudaStream_t s) {
  if (n == 0) return;
  k_dot<<<grid_for(n, 256), 256, 0, s>>>(x, x, n, acc);
}
void launch_dot(const double* a, const double* b, int64_t n, double* acc, cudaStream_t s) {
  if (n == 0) return;
  k_dot<<<grid_for(n, 256), 256, 0, s>>>(a, b, n, acc);
}
void launch_scale(double* x, double fac, int64_t n, cudaStream_t s) {
  if (n == 0) return;
  k_scale<<<grid_for(n, 256), 256, 0, s>>>(x, fac, n);
}
void launch_diavc(double* out, const double* in, const double* diag, double fac, double shift,
                  int64_t n, cudaStream_t s) {
  if (n == 0) return;
  k_diavc<<<grid_for(n, 256), 256, 0, s>>>(out, in, diag, fac, shift, n);
}
void launch_sym_ab(const FlipDesc* d, int64_t n, double* x, double prefac, int64_t maxlen,
                   cudaStream_t s) {
  if (n == 0 || maxlen == 0) return;
  dim3 grid((unsigned)std::min<int64_t>((maxlen + 255) / 256, 1024), (unsigned)n);
  k_sym_ab<<<grid, 256, 0, s>>>(d, x, prefac);
}

}  // namespace gccu

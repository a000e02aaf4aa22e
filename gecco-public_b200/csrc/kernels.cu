// Device kernels of the engine (sm_100a).
//
//  k_strmap      signed (str1,str2)->str12 string maps, one thread per pair
//                (set_strmap_kernel, strings/set_strmap_kernel.f:66-119 with
//                iordstr2, strings/iordstr2.f, and idx4sg,
//                strings/idx4sg.f).  Integer work, bit-exact.
//  (the block contractions themselves are in gemm.cu)
//  bandwidth     add_opblk, diavc, norms, dot products, scaling, sym_ab.
#include <algorithm>
#include <cstdio>

#include "kernels.hpp"

namespace gccu {
namespace {


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
// one output distribution per blockIdx.y; consecutive threads on
// consecutive output C indices (the output's fastest creator component)
__global__ void k_add_transp(const TranspDesc* __restrict__ ds, const double* __restrict__ in,
                             double* __restrict__ out, double fac) {
  const TranspDesc& d = ds[blockIdx.y];
  const int64_t n = d.lenc * d.lena;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t ia = e / d.lenc, ic = e % d.lenc;
    int64_t po = 0, pi = 0;
    for (int k = 0; k < d.nc; ++k) {
      const int64_t s = ic % d.lc[k];
      ic /= d.lc[k];
      po += s * d.ldoc[k];
      pi += s * d.ldic[k];
    }
    for (int k = 0; k < d.na; ++k) {
      const int64_t s = ia % d.la[k];
      ia /= d.la[k];
      po += s * d.ldoa[k];
      pi += s * d.ldia[k];
    }
    out[d.off_out + po] += fac * in[d.off_in + pi];
  }
}

void launch_add_transp(const TranspDesc* d, int64_t n, const double* in, double* out, double fac,
                       int64_t maxlen, cudaStream_t s) {
  if (n == 0 || maxlen == 0) return;
  dim3 grid((unsigned)std::min<int64_t>((maxlen + 255) / 256, 4096), (unsigned)n);
  k_add_transp<<<grid, 256, 0, s>>>(d, in, out, fac);
}

void launch_sym_ab(const FlipDesc* d, int64_t n, double* x, double prefac, int64_t maxlen,
                   cudaStream_t s) {
  if (n == 0 || maxlen == 0) return;
  dim3 grid((unsigned)std::min<int64_t>((maxlen + 255) / 256, 1024), (unsigned)n);
  k_sym_ab<<<grid, 256, 0, s>>>(d, x, prefac);
}

}  // namespace gccu

// Learned correction of the diagonal preconditioner step (no counterpart in
// the reference, whose step is diavc, baserout/diavc.f:31-35, inside
// optc_diis_sbsp_add, solve/optc_diis_sbsp_add.f:125-145).
//
// A multilayer perceptron maps three inputs of each amplitude element to a
// factor m = 1 + tanh(o) of the plain step s = fac * in / d, d = diag + shift
// (clamped to 1e-10 in magnitude as diavc does):
//   x0 = d / 4,  x1 = 1 / max(|d|, 0.05),  x2 = clip(u * v, -10, 10),
//   u = s / rms(s) (the current residual's plain step, normalised),
//   v = prev / rms(prev) (the previous step, normalised; 0 when absent),
//   h1 = tanh(W1 x + b1), h2 = tanh(W2 h1 + b2), o = W3 . h2 + b3.
// Weights, FP64, one array of kLpWeights: W1[32][3], b1[32], W2[32][32],
// b2[32], W3[32], b3.  Training rows are (x0, x1, x2, s, target) with the
// loss L = (1/n) sum (s * (1 + tanh(o)) - target)^2; target = converged
// amplitude - amplitude at the sampled iteration ("converged step").
//
// Kernels: k_lp_sums (sum s^2, sum prev^2 over a list), k_lp_apply (inputs,
// forward pass and the corrected step, one element per thread, weights in
// shared memory), k_lp_rows (inputs of sampled elements), k_lp_grad (forward
// and backward of 128 rows per block, per-block gradient sums reduced in
// shared memory), k_lp_reduce (block sums -> gradient and loss), k_lp_adam
// (Adam update).  Training is FP64, so the gradients equal a CPU
// restatement to rounding; the step applied in the solve runs the
// perceptron in FP32 (its factor to about 1e-6 relative; the inputs, the
// plain step and the product stay FP64).
#include <cstdint>

#include "kernels.hpp"

namespace gccu {
namespace {

constexpr int NH = kLpHidden, NI = kLpInputs;
constexpr int OW1 = 0, OB1 = OW1 + NH * NI, OW2 = OB1 + NH, OB2 = OW2 + NH * NH,
              OW3 = OB2 + NH, OB3 = OW3 + NH;
static_assert(OB3 + 1 == kLpWeights, "weight layout");
static_assert(OW2 % 4 == 0 && NH % 4 == 0, "rows of W2 start on 16-byte boundaries");

__device__ __forceinline__ double clampd(double x, double lo, double hi) {
  return x < lo ? lo : (x > hi ? hi : x);
}

// d = diag + shift with the clamp of diavc (|d| <= 1e-10 -> 1e-10)
__device__ __forceinline__ double denom(double diag, double shift) {
  double d = diag + shift;
  return fabs(d) <= 1e-10 ? 1e-10 : d;
}

__device__ __forceinline__ void inputs(double d, double s, double pv, double inv_rs,
                                       double inv_rp, double (&x)[NI]) {
  x[0] = d * 0.25;
  x[1] = 1.0 / fmax(fabs(d), 0.05);
  x[2] = clampd((s * inv_rs) * (pv * inv_rp), -10.0, 10.0);
}

// o = MLP(x) with the weights in w (shared or global memory)
__device__ __forceinline__ double forward(const double* __restrict__ w, const double (&x)[NI],
                                          double (&h1)[NH], double (&h2)[NH]) {
#pragma unroll
  for (int j = 0; j < NH; ++j) {
    double a = w[OB1 + j];
#pragma unroll
    for (int i = 0; i < NI; ++i) a = fma(w[OW1 + j * NI + i], x[i], a);
    h1[j] = tanh(a);
  }
  double o = w[OB3];
#pragma unroll
  for (int j = 0; j < NH; ++j) {
    double a = w[OB2 + j];
#pragma unroll
    for (int k = 0; k < NH; ++k) a = fma(w[OW2 + j * NH + k], h1[k], a);
    h2[j] = tanh(a);
    o = fma(w[OW3 + j], h2[j], o);
  }
  return o;
}

// o = MLP(x) in FP32 for inference of two elements at once (weights in
// shared memory as floats, the first hidden layer of both in registers):
// every weight read from shared memory (four at a time) feeds both
// elements, so the shared-memory pipe is not the bound; the factor
// 1 + tanh(o) to about 1e-6 relative
__device__ __forceinline__ void forward_f32x2(const float* __restrict__ w,
                                              const float (&xa)[NI], const float (&xb)[NI],
                                              float& oa, float& ob) {
  float ha[NH], hb[NH];
#pragma unroll
  for (int j = 0; j < NH; ++j) {
    float a = w[OB1 + j], b = a;
#pragma unroll
    for (int i = 0; i < NI; ++i) {
      const float wi = w[OW1 + j * NI + i];
      a = fmaf(wi, xa[i], a);
      b = fmaf(wi, xb[i], b);
    }
    ha[j] = tanhf(a);
    hb[j] = tanhf(b);
  }
  oa = ob = w[OB3];
#pragma unroll 1
  for (int j = 0; j < NH; ++j) {
    float a = w[OB2 + j], b = a;
    const float4* w4 = reinterpret_cast<const float4*>(w + OW2 + j * NH);
#pragma unroll
    for (int k = 0; k < NH; k += 4) {
      const float4 v = w4[k / 4];
      a = fmaf(v.x, ha[k], a);
      b = fmaf(v.x, hb[k], b);
      a = fmaf(v.y, ha[k + 1], a);
      b = fmaf(v.y, hb[k + 1], b);
      a = fmaf(v.z, ha[k + 2], a);
      b = fmaf(v.z, hb[k + 2], b);
      a = fmaf(v.w, ha[k + 3], a);
      b = fmaf(v.w, hb[k + 3], b);
    }
    const float w3 = w[OW3 + j];
    oa = fmaf(w3, tanhf(a), oa);
    ob = fmaf(w3, tanhf(b), ob);
  }
}

constexpr int kRedThreads = 256;

// acc[0] += sum s^2, acc[1] += sum prev^2
__global__ void __launch_bounds__(kRedThreads)
    k_lp_sums(const double* __restrict__ in, const double* __restrict__ diag,
              const double* __restrict__ prev, double fac, double shift, int64_t n,
              double* __restrict__ acc) {
  double a = 0.0, b = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double s = fac * in[i] / denom(diag[i], shift);
    a = fma(s, s, a);
    if (prev) b = fma(prev[i], prev[i], b);
  }
  __shared__ double ra[kRedThreads / 32], rb[kRedThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) ra[warp] = a, rb[warp] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sa = 0.0, sb = 0.0;
    for (int i = 0; i < kRedThreads / 32; ++i) sa += ra[i], sb += rb[i];
    atomicAdd(acc, sa);
    atomicAdd(acc + 1, sb);
  }
}

// 1/rms of the sums (0 for an all-zero vector)
__device__ __forceinline__ void inv_rms(const double* acc, int64_t n, double& is, double& ip) {
  const double ms = acc[0] / (double)n, mp = acc[1] / (double)n;
  is = ms > 0.0 ? rsqrt(ms) : 0.0;
  ip = mp > 0.0 ? rsqrt(mp) : 0.0;
}

constexpr int kApplyThreads = 256;

// out[i] = s_i * (1 + tanh(o_i)); inputs and the plain step in FP64, the
// perceptron in FP32
__global__ void __launch_bounds__(kApplyThreads, 2)
    k_lp_apply(double* __restrict__ out, const double* __restrict__ in,
               const double* __restrict__ diag, const double* __restrict__ prev, double fac,
               double shift, int64_t n, const double* __restrict__ acc,
               const double* __restrict__ weights) {
  __shared__ __align__(16) float w[kLpWeights + 3];
  for (int i = threadIdx.x; i < kLpWeights; i += blockDim.x) w[i] = (float)weights[i];
  __syncthreads();
  double is, ip;
  inv_rms(acc, n, is, ip);
  // elements i and i + blockDim.x of each pass of 2 * blockDim.x (coalesced)
  const int64_t pass = 2 * (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = 2 * (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += pass) {
    const int64_t i1 = i0 + blockDim.x;
    const bool has1 = i1 < n;
    const double d0 = denom(diag[i0], shift), s0 = fac * in[i0] / d0;
    const double d1 = has1 ? denom(diag[i1], shift) : 1.0;
    const double s1 = has1 ? fac * in[i1] / d1 : 0.0;
    double x0[NI], x1[NI];
    inputs(d0, s0, prev ? prev[i0] : 0.0, is, ip, x0);
    inputs(d1, s1, prev && has1 ? prev[i1] : 0.0, is, ip, x1);
    const float xa[NI] = {(float)x0[0], (float)x0[1], (float)x0[2]};
    const float xb[NI] = {(float)x1[0], (float)x1[1], (float)x1[2]};
    float oa, ob;
    forward_f32x2(w, xa, xb, oa, ob);
    out[i0] = s0 * (double)(1.0f + tanhf(oa));
    if (has1) out[i1] = s1 * (double)(1.0f + tanhf(ob));
  }
}

// rows[r] = (x0, x1, x2, s, amp) of element idx[r]
__global__ void k_lp_rows(const double* __restrict__ in, const double* __restrict__ diag,
                          const double* __restrict__ prev, const double* __restrict__ amp,
                          double fac, double shift, int64_t n, const int64_t* __restrict__ idx,
                          int64_t nrows, const double* __restrict__ acc, double* __restrict__ rows) {
  double is, ip;
  inv_rms(acc, n, is, ip);
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx[r];
    if (i < 0 || i >= n) continue;  // checked on the host; never read out of range
    const double d = denom(diag[i], shift);
    const double s = fac * in[i] / d;
    double x[NI];
    inputs(d, s, prev ? prev[i] : 0.0, is, ip, x);
    double* o = rows + r * kLpRowLen;
    o[0] = x[0];
    o[1] = x[1];
    o[2] = x[2];
    o[3] = s;
    o[4] = amp ? amp[i] : 0.0;
  }
}

// row index of minibatch entry r at training step `step` (hash of seed,
// step, r; every row when batch == 0)
__device__ __forceinline__ int64_t pick(uint64_t seed, uint64_t step, uint64_t r, int64_t n) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + step * 0xD1B54A32D192ED03ull + r + 1;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (int64_t)(z % (uint64_t)n);
}

constexpr int kGradRows = 128;  // rows (threads) per block of k_lp_grad
constexpr int kGradOut = kLpWeights + 1;  // gradient entries and the loss

struct GradSmem {
  double w[kLpWeights];
  double x[kGradRows][NI];
  double h1[kGradRows][NH + 1];  // +1: rows of different threads on different banks
  double d2[kGradRows][NH + 1];  // dL/d(pre-activation of layer 2)
  double d1[kGradRows][NH + 1];  // dL/d(pre-activation of layer 1)
  double h2[kGradRows][NH + 1];
  double dout[kGradRows];        // dL/do
  double loss[kGradRows];
};

// per-block sums of the gradient of (1/n) sum (s (1 + tanh o) - target)^2
// over the block's rows into part[block][kGradOut] (last entry: the loss).
// batch == 0: rows blockIdx.x*128.. of the set in order; else `batch` rows
// drawn with pick() and the loss scaled by 1/batch.
__global__ void __launch_bounds__(kGradRows)
    k_lp_grad(const double* __restrict__ rows, const double* __restrict__ target, int64_t nrows,
              int64_t batch, uint64_t seed, uint64_t step, const double* __restrict__ weights,
              double* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GradSmem& S = *reinterpret_cast<GradSmem*>(smem_raw);
  const int t = threadIdx.x;
  for (int i = t; i < kLpWeights; i += kGradRows) S.w[i] = weights[i];
  __syncthreads();
  const int64_t count = batch ? batch : nrows;
  const int64_t q = (int64_t)blockIdx.x * kGradRows + t;
  const double scale = 1.0 / (double)count;
  double dout = 0.0, loss = 0.0;
  double x[NI], h1[NH], h2[NH];
#pragma unroll
  for (int i = 0; i < NI; ++i) x[i] = 0.0;
#pragma unroll
  for (int j = 0; j < NH; ++j) h1[j] = h2[j] = 0.0;
  if (q < count) {
    const int64_t r = batch ? pick(seed, step, (uint64_t)q, nrows) : q;
    const double* row = rows + r * kLpRowLen;
#pragma unroll
    for (int i = 0; i < NI; ++i) x[i] = row[i];
    const double s = row[3];
    const double o = forward(S.w, x, h1, h2);
    const double c = tanh(o);
    const double res = s * (1.0 + c) - target[r];
    loss = scale * res * res;
    dout = scale * 2.0 * res * s * (1.0 - c * c);
  }
#pragma unroll
  for (int i = 0; i < NI; ++i) S.x[t][i] = x[i];
#pragma unroll
  for (int j = 0; j < NH; ++j) {
    S.h1[t][j] = h1[j];
    S.h2[t][j] = h2[j];
    S.d2[t][j] = dout * S.w[OW3 + j] * (1.0 - h2[j] * h2[j]);
  }
  S.dout[t] = dout;
  S.loss[t] = loss;
#pragma unroll
  for (int k = 0; k < NH; ++k) {
    double a = 0.0;
#pragma unroll 8
    for (int j = 0; j < NH; ++j) a = fma(S.w[OW2 + j * NH + k], S.d2[t][j], a);
    S.d1[t][k] = a * (1.0 - h1[k] * h1[k]);
  }
  __syncthreads();
  // gradient entry e summed over the block's rows, entries spread over threads
  double* out = part + (int64_t)blockIdx.x * kGradOut;
  for (int e = t; e < kGradOut; e += kGradRows) {
    double a = 0.0;
    if (e < OB1) {  // W1[j][i]
      const int j = (e - OW1) / NI, i = (e - OW1) % NI;
      for (int r = 0; r < kGradRows; ++r) a = fma(S.d1[r][j], S.x[r][i], a);
    } else if (e < OW2) {
      const int j = e - OB1;
      for (int r = 0; r < kGradRows; ++r) a += S.d1[r][j];
    } else if (e < OB2) {  // W2[j][k]
      const int j = (e - OW2) / NH, k = (e - OW2) % NH;
      for (int r = 0; r < kGradRows; ++r) a = fma(S.d2[r][j], S.h1[r][k], a);
    } else if (e < OW3) {
      const int j = e - OB2;
      for (int r = 0; r < kGradRows; ++r) a += S.d2[r][j];
    } else if (e < OB3) {
      const int j = e - OW3;
      for (int r = 0; r < kGradRows; ++r) a = fma(S.dout[r], S.h2[r][j], a);
    } else if (e == OB3) {
      for (int r = 0; r < kGradRows; ++r) a += S.dout[r];
    } else {
      for (int r = 0; r < kGradRows; ++r) a += S.loss[r];
    }
    out[e] = a;
  }
}

// grad[e] = sum over blocks of part[b][e] (fixed order: deterministic)
__global__ void k_lp_reduce(const double* __restrict__ part, int64_t nblocks,
                            double* __restrict__ grad) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kGradOut) return;
  double a = 0.0;
  for (int64_t b = 0; b < nblocks; ++b) a += part[b * kGradOut + e];
  grad[e] = a;
}

// Adam (Kingma & Ba, 2015) with bias correction, step t >= 1
__global__ void k_lp_adam(double* __restrict__ w, double* __restrict__ m, double* __restrict__ v,
                          const double* __restrict__ grad, double lr, int64_t t) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kLpWeights) return;
  const double b1 = 0.9, b2 = 0.999, eps = 1e-8;
  const double g = grad[e];
  const double mm = b1 * m[e] + (1.0 - b1) * g, vv = b2 * v[e] + (1.0 - b2) * g * g;
  m[e] = mm;
  v[e] = vv;
  const double mh = mm / (1.0 - pow(b1, (double)t)), vh = vv / (1.0 - pow(b2, (double)t));
  w[e] -= lr * mh / (sqrt(vh) + eps);
}

unsigned grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  return (unsigned)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

}  // namespace

void launch_lp_sums(const double* in, const double* diag, const double* prev, double fac,
                    double shift, int64_t n, double* acc, cudaStream_t s) {
  if (n == 0) return;
  k_lp_sums<<<grid_for(n, kRedThreads), kRedThreads, 0, s>>>(in, diag, prev, fac, shift, n, acc);
}

void launch_lp_apply(double* out, const double* in, const double* diag, const double* prev,
                     double fac, double shift, int64_t n, const double* acc,
                     const double* weights, cudaStream_t s) {
  if (n == 0) return;
  // two elements per thread
  k_lp_apply<<<grid_for((n + 1) / 2, kApplyThreads), kApplyThreads, 0, s>>>(
      out, in, diag, prev, fac, shift, n, acc, weights);
}

void launch_lp_rows(const double* in, const double* diag, const double* prev, const double* amp,
                    double fac, double shift, int64_t n, const int64_t* idx, int64_t nrows,
                    const double* acc, double* rows, cudaStream_t s) {
  if (nrows == 0) return;
  k_lp_rows<<<grid_for(nrows, 128), 128, 0, s>>>(in, diag, prev, amp, fac, shift, n, idx, nrows,
                                                 acc, rows);
}

int64_t lp_grad_blocks(int64_t count) { return (count + kGradRows - 1) / kGradRows; }

void launch_lp_grad(const double* rows, const double* target, int64_t nrows, int64_t batch,
                    uint64_t seed, uint64_t step, const double* weights, double* part,
                    double* grad, cudaStream_t s) {
  const int64_t nb = lp_grad_blocks(batch ? batch : nrows);
  const size_t smem = sizeof(GradSmem);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_lp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    configured = true;
  }
  k_lp_grad<<<(unsigned)nb, kGradRows, smem, s>>>(rows, target, nrows, batch, seed, step, weights,
                                                  part);
  k_lp_reduce<<<(kGradOut + 127) / 128, 128, 0, s>>>(part, nb, grad);
}

void launch_lp_adam(double* w, double* m, double* v, const double* grad, double lr, int64_t t,
                    cudaStream_t s) {
  k_lp_adam<<<(kLpWeights + 127) / 128, 128, 0, s>>>(w, m, v, grad, lr, t);
}

}  // namespace gccu

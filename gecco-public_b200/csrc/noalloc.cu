// Fixed device scratch of the allocation-free contraction entry point
// (gccu_contract_noalloc).  The operand panels that the pack kernel fills and
// the descriptors that point at them live in one file-scope device array,
// sized once at compile time; the entry point copies a contraction's
// descriptors into it with the panel pointers moved into the array, then runs
// the regular pack and GEMM kernels on those copies.
#include "kernels.hpp"

namespace gccu {
namespace {

constexpr size_t round256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kPanelBytes = kStaticPanelDoubles * sizeof(double);
constexpr size_t kDescOff = round256(kPanelBytes);
constexpr size_t kJobOff = kDescOff + round256(sizeof(GemmDesc) * kStaticMaxDescs);
constexpr size_t kScratchBytes = kJobOff + round256(sizeof(PackJob) * kStaticMaxJobs);

// shared by every call in the process on a device: contents persist between calls
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

__device__ __forceinline__ bool inside(const void* p, const double* base, int64_t len) {
  const uintptr_t a = (uintptr_t)p, b = (uintptr_t)base;
  return base && a >= b && a < b + (uintptr_t)len * sizeof(double);
}

__global__ void k_rebase_descs(const GemmDesc* __restrict__ src, GemmDesc* __restrict__ dst,
                               int64_t n, const double* old_base, int64_t old_len,
                               double* new_base) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    GemmDesc d = src[i];
    if (inside(d.a, old_base, old_len)) d.a = new_base + (d.a - old_base);
    if (inside(d.b, old_base, old_len)) d.b = new_base + (d.b - old_base);
    dst[i] = d;
  }
}

__global__ void k_rebase_jobs(const PackJob* __restrict__ src, PackJob* __restrict__ dst,
                              int64_t n, const double* old_base, int64_t old_len,
                              double* new_base) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    PackJob j = src[i];
    if (inside(j.dst, old_base, old_len)) j.dst = new_base + (j.dst - old_base);
    dst[i] = j;
  }
}

unsigned blocks_for(int64_t n) { return (unsigned)std::min<int64_t>((n + 127) / 128, 1024); }

}  // namespace

cudaError_t static_scratch(StaticScratch* out) {
  void* p = nullptr;
  cudaError_t err = cudaGetSymbolAddress(&p, g_scratch);
  if (err != cudaSuccess) return err;
  unsigned char* base = static_cast<unsigned char*>(p);
  out->panels = reinterpret_cast<double*>(base);
  out->descs = reinterpret_cast<GemmDesc*>(base + kDescOff);
  out->jobs = reinterpret_cast<PackJob*>(base + kJobOff);
  return cudaSuccess;
}

void launch_rebase_descs(const GemmDesc* src, GemmDesc* dst, int64_t n, const double* old_base,
                         int64_t old_len, double* new_base, cudaStream_t s) {
  if (n == 0) return;
  k_rebase_descs<<<blocks_for(n), 128, 0, s>>>(src, dst, n, old_base, old_len, new_base);
}

void launch_rebase_jobs(const PackJob* src, PackJob* dst, int64_t n, const double* old_base,
                        int64_t old_len, double* new_base, cudaStream_t s) {
  if (n == 0) return;
  k_rebase_jobs<<<blocks_for(n), 128, 0, s>>>(src, dst, n, old_base, old_len, new_base);
}

}  // namespace gccu

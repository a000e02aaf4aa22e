// Launchers of the device kernels (kernels.cu).  All launches go to the
// given stream; none synchronises.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "device_types.hpp"

namespace gccu {

// signed string map of one (str1 block, str2 block) pair; tables hold the
// strings of each block in address order (orb<<2 | code), W/irrep describe
// the graph of the merged string
void launch_strmap(const int32_t* tab1, int nel1, int64_t n1, const int32_t* tab2, int nel2,
                   int64_t n2, const int64_t* W12, const int8_t* irrep12, int nel12, int nsym,
                   int32_t* out, cudaStream_t s);

// tile shapes of the grouped GEMM: regular items, medium (<= 32 columns) and
// thin (<= 8 columns) items, items with at most 16 result elements
constexpr int kGemmRegular = 0, kGemmSkinny = 1, kGemmSmall = 2, kGemmMedium = 3;
constexpr int kGemmTc = 4;  // tensor-core tiles (precision modes 1-3)
constexpr int kGemmThin = 5;  // thin column side, streaming kernel (k_thin)
constexpr int kGemmKinds = 6;
constexpr int kGemmThinM = 256;       // rows of a thin tile (one thread each)
constexpr int64_t kThinMaxElems = 12288;  // thin-operand elements staged per tile
constexpr int kThinMaxColumns = 32;       // widest thin side (k_thin is compiled up to 32)
constexpr int kGemmTcM = 128, kGemmTcN = 256;
constexpr int64_t kTcChunk = 4096;  // contraction range of one FP32 accumulation
constexpr int64_t kTcMinK = 256;    // shortest contraction sent to the tensor cores
constexpr int64_t kSmallChunk = 1 << 16;  // contraction elements per block of k_small
constexpr int kGemmRegularM = 128, kGemmRegularN = 64;
constexpr int kGemmMediumM = 128, kGemmMediumN = 32;
constexpr int kGemmSkinnyM = 128, kGemmSkinnyN = 8;
constexpr int kGemmK = 16;
// output tile of a kernel kind (the small-item kernel takes a whole item)
inline void gemm_tile(int kind, int& TM, int& TN) {
  TM = kind == kGemmRegular ? kGemmRegularM
       : kind == kGemmMedium ? kGemmMediumM
       : kind == kGemmSkinny ? kGemmSkinnyM
       : kind == kGemmTc     ? kGemmTcM
       : kind == kGemmThin   ? kGemmThinM
                             : 1 << 30;
  TN = kind == kGemmRegular ? kGemmRegularN
       : kind == kGemmMedium ? kGemmMediumN
       : kind == kGemmSkinny ? kGemmSkinnyN
       : kind == kGemmTc     ? kGemmTcN
                             : 1 << 30;
}

// block contractions with at most 32 columns, one thread per row of the
// long operand (read in place, through its gather description when it needs
// map lookups: 1 + index in `gathers`, GemmDesc::ga); nc = thin_columns(the
// launch's widest item), kmax = its longest contraction range per tile
int thin_columns(int64_t N);
void launch_thin(int nc, const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles,
                 const PackJob* gathers, int64_t kmax, double alpha, cudaStream_t s);

// gather map-addressed operands into dense panels (one job per operand/item);
// pack_geometry gives the grid extent one job needs, the launch uses the
// maximum over its jobs
void pack_geometry(const PackJob& j, int64_t& gx, int64_t& gy);
void launch_pack(const PackJob* jobs, int64_t njobs, int64_t gx, int64_t gy, cudaStream_t s);
// split-TF32 tensor-core GEMM (tcgen05) over 128 x kGemmTcN tiles, reading
// the split panels of its items from the workspace; *err is set if a
// pipeline wait (at most wait_limit mbarrier polls) timed out
constexpr int64_t kTcWaitLimitDefault = int64_t(1) << 22;
void launch_gemm_tc(const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles, double alpha,
                    int* err, int64_t wait_limit, cudaStream_t s);
// attributes of the tensor-core GEMM kernel (target architecture of the build)
cudaError_t tc_kernel_attributes(cudaFuncAttributes* attr);
// floats of the split panels of one tensor-core item (both operands)
constexpr int64_t kTcSlice = 32;  // contraction indices per panel slice
inline int64_t tc_panel_floats(int64_t rows, int tile_rows, int64_t K) {
  return (rows + tile_rows - 1) / tile_rows * tile_rows * ((K + kTcSlice - 1) / kTcSlice) *
         kTcSlice * 2;
}
// floats of one 128-row x 32-index chunk kept in FP64 (int8 two-pass staging)
constexpr int64_t kTcGemmChunkFloats = 128 * kTcSlice * 2;
// number of 128-row x 32-index chunks of one operand's panel
inline int64_t tc_split_chunks(int64_t rows, int tile_rows, int64_t K) {
  const int64_t padded = (rows + tile_rows - 1) / tile_rows * tile_rows;
  return (padded + 127) / 128 * ((K + kTcSlice - 1) / kTcSlice);
}
// the split pre-pass's blocks for one operand: 128 rows x kTcSplitGroup
// consecutive 32-index slices each (the rows' tables loaded once)
constexpr int64_t kTcSplitGroup = 4;
inline int64_t tc_split_blocks(int64_t rows, int tile_rows, int64_t K) {
  const int64_t padded = (rows + tile_rows - 1) / tile_rows * tile_rows;
  const int64_t nsl = (K + kTcSlice - 1) / kTcSlice;
  return (padded + 127) / 128 * ((nsl + kTcSplitGroup - 1) / kTcSplitGroup);
}
// tile width of a tensor-core item with N columns: as many tiles as
// widest-wide ones would need, each narrowed to the multiple of 32 that
// covers N
inline int tc_tile_n(int64_t N, int widest = kGemmTcN) {
  const int64_t nt = (N + widest - 1) / widest;
  int64_t w = ((N + nt - 1) / nt + 31) / 32 * 32;
  if (w < 32) w = 32;
  return (int)(w < widest ? w : widest);
}

// FP64 emulation on the int8 tensor cores (precision modes 2 and 3, the
// slicing scheme of Ozaki et al.): an operand row x (row of the row operand,
// column of the column operand) with m = max |x_k| is cut into S signed
// bytes per element, x_k ~ (m / 127) * sum_s a_s,k 2^(-7 s), |a_0| <= 127 and
// |a_s| <= 64 after it (each slice the rounded remainder of the one before);
// the products of slices s and t with s + t < S are summed over the
// contraction in int32 (exactly, for contraction ranges up to kI8Chunk), one
// TMEM accumulator per s + t, and combined in FP64 in the epilogue.  Mode 2
// keeps S = 5 slices (about 35 bits of each element relative to its row
// maximum; 15 products, tiles up to 96 columns), mode 3 S = 4 (28 bits; 10
// products, tiles up to 128 columns).  The panels use the split-TF32 chunk
// geometry (128-row x 32-index chunks); per 32-index slice, a band of TR
// rows holds S x 2 core-matrix planes of TR x 16 bytes:
//   panel[(((band * nslice + slice) * S + s) * 2 + k/16) * TR * 16 + row * 16 + k%16]
// and every panel has an array of its rows' maxima m (FP64, padded rows).
constexpr int kI8SlicesFine = 5, kI8NFine = 96;   // precision mode 2
constexpr int kI8SlicesFast = 4, kI8NFast = 128;  // precision mode 3
constexpr int64_t kI8Chunk = 65536;  // contraction range of one int32 accumulation
inline int i8_slices(int precision) { return precision == 3 ? kI8SlicesFast : kI8SlicesFine; }
inline int i8_widest(int precision) { return precision == 3 ? kI8NFast : kI8NFine; }
// the largest |sum over s + t = d of a_s b_t| per contraction index, d < S
constexpr int64_t i8_term_bound(int S) { return 2 * 127 * 64 + (S - 2) * 64 * 64; }
static_assert(kI8SlicesFine * kI8NFine <= 512 && kI8SlicesFast * kI8NFast <= 512,
              "the accumulators fill at most the 512 TMEM columns");
static_assert(i8_term_bound(kI8SlicesFine) * kI8Chunk < (1ll << 31) &&
                  i8_term_bound(kI8SlicesFast) * kI8Chunk < (1ll << 31) &&
                  127 * 127 * kI8Chunk < (1ll << 31),
              "an int32 accumulator must not overflow over one contraction chunk");
inline int64_t i8_padded_rows(int64_t rows, int tile_rows) {
  return (rows + tile_rows - 1) / tile_rows * tile_rows;
}
// floats of one operand's slice panel (bytes / 4)
inline int64_t i8_panel_floats(int64_t rows, int tile_rows, int64_t K, int slices) {
  return i8_padded_rows(rows, tile_rows) * ((K + kTcSlice - 1) / kTcSlice) * kTcSlice *
         slices / 4;
}
// floats of one operand's row maxima (one double per padded row)
inline int64_t i8_max_floats(int64_t rows, int tile_rows) {
  return i8_padded_rows(rows, tile_rows) * 2;
}
// split the operands of tensor-core items into their panels (jobs sorted by
// cstart, nchunks = total chunks); gathers: descriptions of map-addressed
// operands with at most kTcGatherMaps map components
constexpr int kTcGatherMaps = 4;
void launch_split_tc(const GemmDesc* descs, const SplitJob* jobs, int64_t njobs, int64_t nchunks,
                     const PackJob* gathers, cudaStream_t s);
// precision mode 2: the row maxima of the panels (phase 0; the maxima must be
// zero before it), then the slices (phase 1), same jobs and chunks as the split
void launch_slice_i8(int phase, int slices, const GemmDesc* descs, const SplitJob* jobs,
                     int64_t njobs, int64_t nchunks, const PackJob* gathers, cudaStream_t s);
// zero n floats at base + off (base null: the tensor-core workspace)
void launch_zero_tc(float* base, int64_t off, int64_t n, cudaStream_t s);
// the int8-slice GEMM over 128 x i8_widest tiles with `slices` slices
// (err, wait_limit: as launch_gemm_tc)
void launch_gemm_i8(int slices, const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles,
                    double alpha, int* err, int64_t wait_limit, cudaStream_t s);
cudaError_t i8_kernel_attributes(cudaFuncAttributes* attr);
// device address of the split-TF32 workspace used by the two kernels above
// (a device-side variable, so captured graphs follow a reallocation)
cudaError_t set_tc_workspace(float* ws);
// grouped block-contraction GEMM over the tiles of one tile shape (err,
// wait_limit: see launch_gemm_tc, used by kind kGemmTc)
void launch_gemm(int kind, const GemmDesc* descs, const TileDesc* tiles, int64_t ntiles,
                 double alpha, int* err, int64_t wait_limit, cudaStream_t s);

// reorder of a joined operator class (nitems <= 65535 distribution cases,
// maxlen = largest N0*NK); reo += alpha * signs * ori
void launch_reorder(const ReoItem* items, int64_t nitems, int64_t maxlen, const double* ori,
                    double* reo, double alpha, cudaStream_t s);

// out = (reset ? 0 : out) + fac*in  (add_opblk)
void launch_axpy(double* out, const double* in, double fac, int64_t n, int reset, cudaStream_t s);
// *acc += sum x^2 over n elements (acc must be zeroed by the caller)
void launch_sumsq(const double* x, int64_t n, double* acc, cudaStream_t s);
// *acc += sum a*b
void launch_dot(const double* a, const double* b, int64_t n, double* acc, cudaStream_t s);
void launch_scale(double* x, double fac, int64_t n, cudaStream_t s);
// out = fac*in/(diag+shift) with |diag+shift| <= 1e-10 -> 1e-10 (diavc)
void launch_diavc(double* out, const double* in, const double* diag, double fac, double shift,
                  int64_t n, cudaStream_t s);
// spin-flip symmetrisation of one distribution pair (sym_ab_blk): for every
// element index i < partner p: x[i] = pre*(x[i]+s*x[p]), x[p] = s*x[i]
struct FlipDesc {
  int64_t off1, off2;  // offsets of the distribution and of its flipped partner
  int64_t lenc, lena;
  int32_t nc, na;
  int32_t lc[kDevMaxComp], la[kDevMaxComp];
  int64_t ldc[kDevMaxComp], lda[kDevMaxComp];
  const int32_t* fc[kDevMaxComp];  // flip maps (signed 1-based partner index)
  const int32_t* fa[kDevMaxComp];
  double sgn;  // gsign * relfac2
  int32_t same;  // distribution is its own partner
  int32_t pad;
};
void launch_sym_ab(const FlipDesc* d, int64_t n, double* x, double prefac, int64_t maxlen,
                   cudaStream_t s);
// transposed add of one output distribution (add_opblk_transp): for every
// element (C strings ic, A strings ia) of the output distribution
// out[off_out + pos(ldo)] += fac * in[off_in + pos(ldi)], pos summing the
// component string indices times the leading dimensions
struct TranspDesc {
  int64_t off_out, off_in, lenc, lena;
  int32_t nc, na;
  int32_t lc[kDevMaxComp], la[kDevMaxComp];
  int64_t ldoc[kDevMaxComp], ldoa[kDevMaxComp], ldic[kDevMaxComp], ldia[kDevMaxComp];
};
void launch_add_transp(const TranspDesc* d, int64_t n, const double* in, double* out, double fac,
                       int64_t maxlen, cudaStream_t s);

// Singlet spin projection of one occupation class (spin_prj_blk,
// spinprj.cu).  A class with n creators and n annihilators has C(2n, n)
// spin cases (spins of every particle, equal Ms on both sides); the
// elements of one spatial configuration, one per case, are projected with
// C C^T (C: the genealogical singlet coupling coefficients, [case][path])
// and written back.  One descriptor per skeleton distribution: the
// skeleton's string tuples of each side whose strings are all of the
// reference spin pattern (alternating, alpha last), and for every case the
// partial element offset of each tuple on that side (-1: the case does not
// exist for it; the case's distribution offset is in the loop side's
// values), so that an element's address is the sum of the two sides'.
// Threads run over the side whose strings are contiguous in the list.
constexpr int kSpinPrjMaxPart = 4;     // creators (= annihilators) per class
constexpr int kSpinPrjMaxCases = 70;   // C(8, 4)
constexpr int kSpinPrjMaxCoup = 14;    // singlet coupling paths of eight spins
// coupling paths of the singlet of 2n spins for C(2n, n) cases
constexpr int spin_prj_paths(int ncase) {
  return ncase == 2 ? 1 : ncase == 6 ? 2 : ncase == 20 ? 5 : 14;
}
struct SpinPrjDesc {
  int64_t nt, nl;           // tuples of the thread side and of the loop side
  const int64_t* pt;        // [case][nt] partial offsets of the thread side
  const int64_t* pl;        // [case][nl] of the loop side (distribution offset included)
  const double* coeff;      // [case][path]
};
// thread-side tuples per block and loop-side tuples per thread
constexpr int kSpinPrjThreads = 128, kSpinPrjLoop = 16;
constexpr int64_t spin_prj_blocks(int64_t nt, int64_t nl) {
  return (nt + kSpinPrjThreads - 1) / kSpinPrjThreads * ((nl + kSpinPrjLoop - 1) / kSpinPrjLoop);
}
// descriptors d[0..n), every one with ncase cases (2, 6, 20 or 70);
// maxblocks: the largest spin_prj_blocks among them
void launch_spin_prj(const SpinPrjDesc* d, int64_t n, int ncase, double* x, int64_t maxblocks,
                     cudaStream_t s);

// Learned correction of the diagonal step (learned.cu): a perceptron with
// kLpInputs inputs, two tanh layers of kLpHidden and one output; weights
// W1[hidden][inputs], b1, W2[hidden][hidden], b2, W3[hidden], b3 (FP64)
constexpr int kLpInputs = 3, kLpHidden = 32;
constexpr int kLpWeights = kLpHidden * kLpInputs + kLpHidden + kLpHidden * kLpHidden +
                           kLpHidden + kLpHidden + 1;
constexpr int kLpRowLen = 5;  // sample row: 3 inputs, plain step, amplitude
// acc[0] += sum (fac*in/d)^2, acc[1] += sum prev^2 (acc zeroed by the caller)
void launch_lp_sums(const double* in, const double* diag, const double* prev, double fac,
                    double shift, int64_t n, double* acc, cudaStream_t s);
// out = fac*in/d * (1 + tanh(mlp(inputs))), acc from launch_lp_sums
void launch_lp_apply(double* out, const double* in, const double* diag, const double* prev,
                     double fac, double shift, int64_t n, const double* acc,
                     const double* weights, cudaStream_t s);
// sample rows of the elements idx[0..nrows) (indices checked by the caller)
void launch_lp_rows(const double* in, const double* diag, const double* prev, const double* amp,
                    double fac, double shift, int64_t n, const int64_t* idx, int64_t nrows,
                    const double* acc, double* rows, cudaStream_t s);
// blocks (= partial-sum rows of kLpWeights + 1) of one gradient launch
int64_t lp_grad_blocks(int64_t count);
// grad[0..kLpWeights) = dL/dw, grad[kLpWeights] = L over all rows (batch 0)
// or over `batch` rows drawn from (seed, step); part: lp_grad_blocks rows
void launch_lp_grad(const double* rows, const double* target, int64_t nrows, int64_t batch,
                    uint64_t seed, uint64_t step, const double* weights, double* part,
                    double* grad, cudaStream_t s);
void launch_lp_adam(double* w, double* m, double* v, const double* grad, double lr, int64_t t,
                    cudaStream_t s);

// Fixed scratch of the allocation-free contraction path (noalloc.cu): one
// file-scope device array holding 64 MiB of operand panels and room for the
// descriptors of one contraction.
constexpr int64_t kStaticPanelDoubles = int64_t(8) << 20;
constexpr int64_t kStaticMaxDescs = 16384;
constexpr int64_t kStaticMaxJobs = 16384;
struct StaticScratch {
  double* panels = nullptr;  // kStaticPanelDoubles
  GemmDesc* descs = nullptr;  // kStaticMaxDescs
  PackJob* jobs = nullptr;    // kStaticMaxJobs
};
// device address of the array on the current device (cudaGetSymbolAddress)
cudaError_t static_scratch(StaticScratch* out);
// copy n descriptors, moving operand pointers that lie in the panel range
// [old_base, old_base + old_len) to the same offset from new_base
void launch_rebase_descs(const GemmDesc* src, GemmDesc* dst, int64_t n, const double* old_base,
                         int64_t old_len, double* new_base, cudaStream_t s);
void launch_rebase_jobs(const PackJob* src, PackJob* dst, int64_t n, const double* old_base,
                        int64_t old_len, double* new_base, cudaStream_t s);

}  // namespace gccu

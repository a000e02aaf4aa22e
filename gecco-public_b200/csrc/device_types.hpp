// Plain-old-data descriptors shared by the host planner and the device
// kernels.  One ItemDesc is one block contraction, i.e. one call of the
// reference's inner kernel (contr_blk1blk2_wmaps_c / _blocked_mm) for a fixed
// (Ms, IRREP, distribution) case of ex1, ex2 and the contraction string.
#pragma once
#include <cstdint>

namespace gccu {

constexpr int kDevMaxComp = 8;

// composite string spaces of one item
enum Space : int8_t { kEx1 = 0, kEx2 = 1, kCnt = 2, kNone = -1 };

// How the components of one operand (op1, op2 or the result) are addressed.
// Component j of the operand string is made from a component of space sp1
// (index ci1) and/or of space sp2 (index ci2).  If both are present it is the
// signed string map map[j][i2 * n1 + i1] (strings/set_strmap_kernel.f: str1
// runs fastest); otherwise the component index is used as is (the trivial
// map of strings/get_strmap_blk_c.f:190-198).  Element offset of the operand
// = sum_j (|index_j| - 1) * ldim[j] (contract/set_op_ldim_c.f).
struct OpndDesc {
  int32_t ncomp;
  int32_t nmap;  // number of components that need a map lookup
  int8_t sp1[kDevMaxComp], ci1[kDevMaxComp], sp2[kDevMaxComp], ci2[kDevMaxComp];
  int32_t n1[kDevMaxComp];
  int64_t ldim[kDevMaxComp];
  const int32_t* map[kDevMaxComp];
};

struct ItemDesc {
  int64_t M, N, K;  // |ex1|, |ex2|, |cnt| composite string counts
  double fac;       // xfac * casign * fac_scal
  int64_t base1, base2, base12;
  int32_t nsp[3];              // components per space
  int32_t rad[3][kDevMaxComp];  // string counts per component (first fastest)
  OpndDesc op[3];               // op1, op2, result
  int32_t kfast1, kfast2;       // operand stride is smaller along cnt than along ex
  int32_t pad;
};

struct TileDesc {
  int32_t item;
  int32_t m0, n0;
  int32_t pad;
  int64_t k0, k1;
};

// One block contraction as a GEMM over offset tables:
//   C(r, c) += fac * sum_k A(r, k) B(k, c)
//   A(r, k) = a[aro[r] + ako[k]],  B(k, c) = b[bco[c] + bko[k]]
//   C(r, c) at c[cro[r] + cco[c] + mapped part]
// An operand whose components need string-map lookups is first gathered
// (with signs) into a dense panel by the pack kernel; the tables then address
// the panel.  Rows are ex1 and columns ex2, or the other way round when the
// item is swapped (thin ex1); rowspace tells the epilogue which.
struct GemmDesc {
  int64_t M, N, K;
  double fac;
  const double* a;
  const int64_t *aro, *ako;
  const double* b;
  const int64_t *bco, *bko;
  double* c;
  const int64_t *cro, *cco;
  int32_t afast, bfast;  // 1: contiguous along k (else along rows / columns)
  // k offset tables that are affine, ako[k] = ako[0] + k * akstep (0: not affine)
  int64_t akstep, bkstep;
  // tensor-core items: float offsets of the split operand panels in the
  // split-TF32 workspace (see SplitJob), or, for an operand read from a
  // frozen list, its persistent panel (pa_ptr / pb_ptr, else null)
  int64_t pa, pb;
  float *pa_ptr, *pb_ptr;
  // precision mode 2: float offsets of the panels' row maxima in the
  // workspace (or, for a frozen operand, their persistent arrays)
  int64_t ma, mb;
  double *ma_ptr, *mb_ptr;
  int32_t i8;            // int8 slices per element of a tensor-core item (modes 2, 3), else 0
  int32_t ga;            // thin items: 1 + index of the row operand's gather description, or 0
  int32_t rowspace;      // kEx1 or kEx2 (swapped)
  int32_t cmapped;       // result components that need map lookups
  int32_t exclusive;     // no other tile writes these result elements: plain update
  int32_t tn;            // tensor-core items: tile width (columns, multiple of 32, <= 256)
  int32_t nsp[3];
  int32_t rad[3][kDevMaxComp];
  OpndDesc cmap;  // result operand (map lookups in the epilogue)
};

// One Ms/IRREP distribution case of a reorder (reo_blk_wmaps_c.f:209-840):
// for every string tuple i of the unshifted part I0 (space kEx1: C
// components, then A components) and k of the shifted strings K (space kEx2)
//   reo[base_reo + addr_reo(i, k)] += alpha * signs * ori[base_ori + addr_ori(i, k)]
// where both addresses merge I0 and K components through string maps
// (creators: str1 = I0, str2 = K; annihilators: str1 = K, str2 = I0).
struct ReoItem {
  int64_t N0, NK;
  int64_t base_ori, base_reo;
  int32_t nsp[2];
  int32_t rad[2][kDevMaxComp];
  OpndDesc ori, reo;
};

// Split of one operand of a tensor-core item into its TF32 panel: for the
// row operand (op 0, tile rows TR = 128) and the column operand (op 1, TR =
// the item's tile width tn) of descriptor `desc`, every (TR-row band, 32-index slice) of the
// operand is stored as two planes (hi, lo) of TR x 32 floats in the
// tensor core's K-major core-matrix order, [k/4][row][k%4]:
//   panel[((band * nslice + slice) * 2 + plane) * TR * 32 + (k/4) * TR * 4 + row * 4 + k%4]
// with rows and contraction indices outside the item set to zero.  The job's
// blocks (128 rows x up to four 32-index slices) are numbered from cstart.
// An operand whose
// strings merge an external and a contracted component is read through its
// gather description (PackJob index `gather`, -1: through the descriptor's
// offset tables).
// With int8 slices (two passes over the same chunks) a gathered operand's
// chunks are also kept densely (`stage`: float offset of 128 x 32 FP64 per
// chunk in the workspace, -1 for none), written by the row-maxima pass and
// read by the slicing pass instead of gathering twice.
struct SplitJob {
  int32_t desc, op;
  int64_t cstart;
  int32_t gather, pad;
  int64_t stage;
};

// gather of one operand of one block contraction into a dense panel
// panel[k * R + r] (or panel[r * K + k] when dkfast) = sign * x[address(r, k)],
// address(r, k) = roff[r] + koff[k] + sum_m (|map_m[i2 * n1_m + i1]| - 1) * ldim_m
// where the string indices of map component m come from the tables rmi
// (row side, rmi[m * R + r]) and kmi (contraction side, kmi[m * K + k]);
// row_is_1[m] says which side is str1 (the fast index of the map).
// A thread block covers F consecutive indices of the fast dimension (k when
// the operand is stored contiguously along the contraction index, else r)
// times 256/F indices of the other per pass, so the source reads coalesce.
struct PackJob {
  int64_t R, K;  // rows (ex1 or ex2 composite) and contraction length
  const double* src;
  double* dst;
  const int64_t *roff, *koff;
  const int64_t *rmi, *kmi;
  int32_t kfast;  // threads run fastest along k
  int32_t F;      // power of two <= 256
  int32_t nm;     // map components
  int32_t dkfast; // panel layout: 0 panel[k * R + r], 1 panel[r * K + k] (written along k)
  int32_t row_is_1[kDevMaxComp];
  int32_t n1[kDevMaxComp];
  int64_t ldim[kDevMaxComp];
  const int32_t* map[kDevMaxComp];
};

}  // namespace gccu

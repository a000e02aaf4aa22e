// Contraction planner: flattens the block enumeration of
// contr_op1op2_wmaps_c (contract/contr_op1op2_wmaps_c.f:984-2070) for one
// binary contraction into a static list of block contractions (ItemDesc).
// The list depends only on the operator layouts, never on the numbers, so it
// is built once per formula item and reused in every iteration.
#pragma once

#include <array>
#include <vector>

#include "device_types.hpp"
#include "model.hpp"

namespace gccu {

// (graph1, graph2, idxms1, idxms2, gam1, gam2) of one string-map block
using MapKey = std::array<int, 6>;

struct MapRef {
  int item, opnd, comp;
  MapKey key;
};

struct Plan {
  std::vector<ItemDesc> items;  // fac holds fac_scal only; the call's fact is a launch argument
  std::vector<MapRef> maps;     // map pointers to patch before upload
  bool use_tr = false;          // result class needs sym_ab after the contraction
  double stats[8] = {};         // reference dgemm accounting (str_block = 200)
  double flops = 0;
};

struct ContractionSpec {
  const ListLayout *L1, *L2, *L12;
  int ib1, ib2, ib12;
  Occ ex1, ex2, cnt;
  bool use_tr;
  // operands used transposed (the reference's tra_op1 / tra_op2 / tra_op1op2):
  // the class enters as its adjoint, creators and annihilators swapped
  bool tra1 = false, tra2 = false, tra12 = false;
};

Plan plan_contraction(Model& m, const ContractionSpec& s);

// Reorder of one occupation class of a joined operator into another
// (reo_op_wmaps_c / reo_blk_wmaps_c): the strings K (nshift shifts, each
// moving from vertex from[s] of the original to vertex to[s] of the
// reordered class) change vertex, the rest I0 stays.
constexpr int kMaxShift = 4;
struct ReorderSpec {
  const ListLayout *Lori, *Lreo;
  int ib_ori, ib_reo;
  int nj;
  int nshift;
  Occ shift[kMaxShift];
  int from[kMaxShift], to[kMaxShift];  // 0-based vertices
};

struct ReoPlan {
  std::vector<ReoItem> items;
  std::vector<MapRef> maps;  // opnd 0 = original, 1 = reordered
  int64_t elements = 0;      // sum of N0*NK
};

ReoPlan plan_reorder(Model& m, const ReorderSpec& s);

// Partial trace of one occupation class (trace_op / trace_op_blk):
// res(IC, IA) += f * sum_J op(IC*J, IA*J), the contracted strings J equal on
// the creator and annihilator side.  Planned as a ReoPlan: space kEx1 = the
// result's strings (C, then A components), kEx2 = J (its annihilator
// components; the creator components use the same indices), opnd 0 = op,
// opnd 1 = result.
struct TraceSpec {
  const ListLayout *Lop, *Lres;
  int ib_op, ib_res;
  Occ cnt;
};
ReoPlan plan_trace(Model& m, const TraceSpec& s);

}  // namespace gccu

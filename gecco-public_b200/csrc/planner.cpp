#include "planner.hpp"

#include <algorithm>
#include <cstdlib>

namespace gccu {
namespace {

struct Src {
  int i1 = -1, i2 = -1;
};

// Sources of every component of a merged string side (one vertex): the
// component of the same hpvx type in side 1 and/or side 2
// (set_mapping_info, contract/set_mapping_info.f:88-170).
std::vector<Src> sources(const std::vector<Comp>& tgt, const std::vector<Comp>& s1,
                         const std::vector<Comp>& s2) {
  std::vector<Src> r(tgt.size());
  for (size_t j = 0; j < tgt.size(); ++j) {
    for (size_t i = 0; i < s1.size(); ++i)
      if (s1[i].hpvx == tgt[j].hpvx) r[j].i1 = (int)i;
    for (size_t i = 0; i < s2.size(); ++i)
      if (s2[i].hpvx == tgt[j].hpvx) r[j].i2 = (int)i;
    GCCU_REQUIRE(r[j].i1 >= 0 || r[j].i2 >= 0, "planner: operand component without source");
  }
  return r;
}

// Ms / IRREP of the merged components (contract/merge_msgmdis.f)
void merge_dist(const std::vector<Src>& src, const std::vector<int>& ms1, const std::vector<int>& g1,
                const std::vector<int>& ms2, const std::vector<int>& g2, std::vector<int>& ms,
                std::vector<int>& g) {
  ms.assign(src.size(), 0);
  g.assign(src.size(), 1);
  for (size_t j = 0; j < src.size(); ++j) {
    if (src[j].i1 >= 0) {
      ms[j] += ms1[src[j].i1];
      g[j] = irrep_mult(g[j], g1[src[j].i1]);
    }
    if (src[j].i2 >= 0) {
      ms[j] += ms2[src[j].i2];
      g[j] = irrep_mult(g[j], g2[src[j].i2]);
    }
  }
}

std::vector<int> idxms_of(const std::vector<Comp>& c, const std::vector<int>& ms) {
  std::vector<int> r(c.size());
  for (size_t i = 0; i < c.size(); ++i) r[i] = ms_index(c[i].occ, ms[i]);
  return r;
}

std::vector<int64_t> lengths(Model& m, const std::vector<Comp>& c, const std::vector<int>& ix,
                             const std::vector<int>& g) {
  std::vector<int64_t> r(c.size());
  for (size_t i = 0; i < c.size(); ++i) r[i] = m.G(c[i].graph).nstr(ix[i], g[i]);
  return r;
}

bool has_zero(const std::vector<int64_t>& v) {
  for (auto x : v)
    if (x == 0) return true;
  return false;
}

int sum(const std::vector<Comp>& c) {
  int s = 0;
  for (auto& x : c) s += x.occ;
  return s;
}

// leading dimensions, creator/annihilator sequence, X,P,V,H major
// (contract/set_op_ldim_c.f:38-58); for a class used transposed the
// annihilators of each type come first, in reverse order, then the
// creators (set_op_ldim_c.f:60-76), which is the stored order of the class
void leading_dims(const std::vector<Comp>& c, const std::vector<Comp>& a,
                  const std::vector<int64_t>& lc, const std::vector<int64_t>& la,
                  std::vector<int64_t>& ldc, std::vector<int64_t>& lda, bool transpose = false) {
  ldc.assign(c.size(), 0);
  lda.assign(a.size(), 0);
  int64_t ld = 1;
  for (int ih = 0; ih < 4; ++ih) {
    int t = kHpvxSeq[ih];
    if (!transpose) {
      for (size_t i = 0; i < c.size(); ++i)
        if (c[i].hpvx == t) ldc[i] = ld, ld *= lc[i];
      for (size_t i = 0; i < a.size(); ++i)
        if (a[i].hpvx == t) lda[i] = ld, ld *= la[i];
    } else {
      for (size_t i = a.size(); i-- > 0;)
        if (a[i].hpvx == t) lda[i] = ld, ld *= la[i];
      for (size_t i = c.size(); i-- > 0;)
        if (c[i].hpvx == t) ldc[i] = ld, ld *= lc[i];
    }
  }
}

// One occupation class seen as its adjoint (tra_op flags,
// contract/contr_op1op2_wmaps_c.f:427-429,1127-1145): creators and
// annihilators exchange roles, the total Ms of the list changes sign; every
// stored distribution reappears with its C and A Ms / IRREP exchanged, under
// the (Ms(A), IRREP(A)) key and distribution id of the adjoint, at its stored
// offset.  Returned as a one-class layout (the class at index ib-1).
ListLayout transposed_view(const ListLayout& L, int ib, int nsym) {
  ListLayout T;
  T.op = L.op;
  T.gamt = L.gamt;
  T.mst = -L.mst;
  T.absym = L.absym;
  T.len = L.len;
  T.blk.resize(ib);
  const LayoutBlock& B = L.blk.at(ib - 1);
  LayoutBlock& V = T.blk[ib - 1];
  V.vtx = B.vtx;
  for (auto& o : V.vtx)
    for (int t = 0; t < 4; ++t) std::swap(o[t], o[4 + t]);
  for (int t = 0; t < 4; ++t) V.occ[t] = B.occ[4 + t], V.occ[4 + t] = B.occ[t];
  V.c = B.a;
  V.a = B.c;
  V.off = B.off;
  V.len = B.len;
  const int na = sum(V.a), nc = sum(V.c);
  for (const auto& kv : B.dis) {
    for (const Dist& d : kv.second) {
      Dist e = d;
      e.msc = d.msa;
      e.msa = d.msc;
      e.gc = d.ga;
      e.ga = d.gc;
      int msa = 0, ga = 1;
      for (size_t i = 0; i < e.msa.size(); ++i) msa += e.msa[i], ga = irrep_mult(ga, e.ga[i]);
      std::vector<int> ixc(V.c.size()), ixa(V.a.size());
      for (size_t i = 0; i < V.c.size(); ++i) ixc[i] = ms_index(V.c[i].occ, e.msc[i]);
      for (size_t i = 0; i < V.a.size(); ++i) ixa[i] = ms_index(V.a[i].occ, e.msa[i]);
      e.did = dist_id(V.c, ixc, e.gc, V.a, ixa, e.ga, nsym);
      const auto key = std::make_pair(msa_to_idxms(msa, T.mst, na, nc), ga);
      V.dis[key].push_back(e);
      V.gm_len[key] += e.len;
    }
  }
  return T;
}

const Dist& find_dist(const LayoutBlock& B, int ixms, int gam, int64_t did) {
  const auto& dl = B.dis.at({ixms, gam});
  for (auto& d : dl)
    if (d.did == did) return d;
  throw Error("planner: distribution not found in ME list (idx_msgmdst2)");
}

struct Side {  // one composite side of a component-wise merge
  const std::vector<Comp>* comps;
  int space;    // kEx1 / kEx2 / kCnt
  int offset;   // index of first component of this side within its space
  const std::vector<int>* ixms;
  const std::vector<int>* gam;
  const std::vector<int64_t>* len;
};

// fill part of an operand descriptor for one side (C or A) of the operand
void fill_opnd(OpndDesc& od, int& pos, const std::vector<Src>& src, const Side& s1,
               const Side& s2, const std::vector<int64_t>& ld, int item, int opnd,
               std::vector<MapRef>& refs) {
  for (size_t j = 0; j < src.size(); ++j, ++pos) {
    GCCU_REQUIRE(pos < kDevMaxComp, "planner: too many operand components");
    od.sp1[pos] = od.sp2[pos] = kNone;
    od.ci1[pos] = od.ci2[pos] = -1;
    od.map[pos] = nullptr;
    od.n1[pos] = 0;
    od.ldim[pos] = ld[j];
    if (src[j].i1 >= 0) {
      od.sp1[pos] = (int8_t)s1.space;
      od.ci1[pos] = (int8_t)(s1.offset + src[j].i1);
      od.n1[pos] = (int32_t)(*s1.len)[src[j].i1];
    }
    if (src[j].i2 >= 0) {
      od.sp2[pos] = (int8_t)s2.space;
      od.ci2[pos] = (int8_t)(s2.offset + src[j].i2);
    }
    if (src[j].i1 >= 0 && src[j].i2 >= 0) {
      od.nmap++;
      MapRef r;
      r.item = item;
      r.opnd = opnd;
      r.comp = pos;
      r.key = {(*s1.comps)[src[j].i1].graph, (*s2.comps)[src[j].i2].graph,
               (*s1.ixms)[src[j].i1],       (*s2.ixms)[src[j].i2],
               (*s1.gam)[src[j].i1],        (*s2.gam)[src[j].i2]};
      refs.push_back(r);
    }
  }
  od.ncomp = pos;
}

// stride-1 direction of an operand: does its unit-stride component come
// from the contraction string (then cnt runs fastest in memory)?
int32_t unit_from(const OpndDesc& od, int space) {
  for (int j = 0; j < od.ncomp; ++j)
    if (od.ldim[j] == 1) {
      int sp = od.sp1[j] != kNone ? od.sp1[j] : od.sp2[j];
      return sp == space ? 1 : 0;
    }
  return 0;
}

// reference dgemm accounting for one block contraction: batches of at most
// str_block (200) ex strings, unbatched contraction index
// (contract/contr_blk1blk2_blocked_mm.f:184-239,454-460,512-518)
void account(double* st, int64_t M, int64_t N, int64_t K) {
  const int64_t blk = 200;
  bool op1shorter = M <= N;
  int64_t ns = op1shorter ? M : N, nl = op1shorter ? N : M;
  for (int64_t l0 = 0; l0 < nl; l0 += blk) {
    int64_t bl = std::min(blk, nl - l0);
    for (int64_t s0 = 0; s0 < ns; s0 += blk) {
      int64_t bs = std::min(blk, ns - s0);
      double d1 = (double)(op1shorter ? bs : bl), d2 = (double)(op1shorter ? bl : bs);
      st[0] += 1;
      st[1] += d1;
      st[2] += d1 * d1;
      st[3] += d2;
      st[4] += d2 * d2;
      st[5] += (double)K;
      st[6] += (double)K * K;
      st[7] += 2.0 * d1 * d2 * (double)K;
    }
  }
}

}  // namespace

Plan plan_contraction(Model& m, const ContractionSpec& s) {
  Plan P;
  const int nsym = m.os.nsym;
  ListLayout T1, T2, T12;  // adjoint views of operands used transposed
  if (s.tra1) T1 = transposed_view(*s.L1, s.ib1, nsym);
  if (s.tra2) T2 = transposed_view(*s.L2, s.ib2, nsym);
  if (s.tra12) T12 = transposed_view(*s.L12, s.ib12, nsym);
  const ListLayout &L1 = s.tra1 ? T1 : *s.L1, &L2 = s.tra2 ? T2 : *s.L2,
                   &L12 = s.tra12 ? T12 : *s.L12;
  GCCU_REQUIRE(s.ib1 >= 1 && s.ib1 <= (int)L1.blk.size(), "planner: bad op1 block");
  GCCU_REQUIRE(s.ib2 >= 1 && s.ib2 <= (int)L2.blk.size(), "planner: bad op2 block");
  GCCU_REQUIRE(s.ib12 >= 1 && s.ib12 <= (int)L12.blk.size(), "planner: bad result block");
  const LayoutBlock &B1 = L1.blk[s.ib1 - 1], &B2 = L2.blk[s.ib2 - 1], &B12 = L12.blk[s.ib12 - 1];
  for (int t = 0; t < 4; ++t) {
    GCCU_REQUIRE(B1.occ[t] == s.ex1[t] + s.cnt[t] && B1.occ[4 + t] == s.ex1[4 + t] + s.cnt[4 + t],
                 "contract: op1 occupation != ex1 + cnt");
    GCCU_REQUIRE(B2.occ[t] == s.ex2[t] + s.cnt[4 + t] && B2.occ[4 + t] == s.ex2[4 + t] + s.cnt[t],
                 "contract: op2 occupation != ex2 + cnt^+");
    GCCU_REQUIRE(B12.occ[t] == s.ex1[t] + s.ex2[t] && B12.occ[4 + t] == s.ex1[4 + t] + s.ex2[4 + t],
                 "contract: result occupation != ex1 + ex2");
  }
  GCCU_REQUIRE(irrep_mult(L1.gamt, L2.gamt) == L12.gamt, "contract: inconsistent symmetries");

  // condensed contraction info (contract/condense_bc_info.f)
  std::vector<Comp> ex1c, ex1a, ex2c, ex2a, cntc, cnta;
  m.condense(s.ex1, ex1c, ex1a);
  m.condense(s.ex2, ex2c, ex2a);
  m.condense(s.cnt, cntc, cnta);
  const std::vector<Comp>&op1c = B1.c, &op1a = B1.a, &op2c = B2.c, &op2a = B2.a, &o12c = B12.c,
        &o12a = B12.a;
  // op1 <- (cnt, ex1); op2 <- (cnt^+, ex2); op12: C <- (ex1, ex2), A <- (ex2, ex1)
  auto src1c = sources(op1c, cntc, ex1c), src1a = sources(op1a, cnta, ex1a);
  auto src2c = sources(op2c, cnta, ex2c), src2a = sources(op2a, cntc, ex2a);
  auto src12c = sources(o12c, ex1c, ex2c), src12a = sources(o12a, ex2a, ex1a);

  const int mst1 = L1.mst, mst2 = L2.mst, mst12 = L12.mst;
  const int g1t = L1.gamt, g2t = L2.gamt, g12t = L12.gamt;
  const int na1 = sum(op1a), nc1 = sum(op1c), na2 = sum(op2a), nc2 = sum(op2c), na12 = sum(o12a),
            nc12 = sum(o12c);
  const int ncex1 = sum(ex1c), naex1 = sum(ex1a), ncex2 = sum(ex2c), naex2 = sum(ex2a),
            nccnt = sum(cntc), nacnt = sum(cnta);
  const bool use_tr = s.use_tr && L1.absym != 0 && L2.absym != 0 && L12.absym != 0 &&
                      L1.absym * L2.absym == L12.absym;
  P.use_tr = use_tr;
  const int idx_restr = (na2 > na1) ? 1 : 0;
  const auto oc_ex1c = comp_occs(ex1c), oc_ex1a = comp_occs(ex1a), oc_ex2c = comp_occs(ex2c),
             oc_ex2a = comp_occs(ex2a), oc_cntc = comp_occs(cntc), oc_cnta = comp_occs(cnta);

  // Ms(A) cases of (op1, op2, op12): first index fastest, from max to min
  // (contract/contr_op1op2_wmaps_c.f:984-1019)
  int msa[3] = {na1, na2, na12};
  const int mx[3] = {na1, na2, na12};
  for (bool first = true;; first = false) {
    if (!first) {
      int i = 0;
      for (; i < 3; ++i) {
        if (msa[i] <= -mx[i]) {
          msa[i] = mx[i];
        } else {
          msa[i] -= 2;
          break;
        }
      }
      if (i == 3) break;
    }
    const int msc[3] = {msa[0] + mst1, msa[1] + mst2, msa[2] + mst12};
    if (std::abs(msc[0]) > nc1 || std::abs(msc[1]) > nc2 || std::abs(msc[2]) > nc12) continue;
    const int msc_ac = msa[0] + msa[1] - msa[2];
    if (nacnt + nccnt < std::abs(msc_ac)) continue;
    if (use_tr && (msa[2] < 0 || (msa[2] == 0 && msa[idx_restr] < 0))) continue;
    double fac0 = 1.0;
    if (use_tr && msa[2] > 0) fac0 *= 2.0;
    if (use_tr && msa[2] == 0 && msa[idx_restr] > 0) fac0 *= 2.0;
    // Ms of the contraction string (:1071-1101)
    for (int mcnt_a = nacnt; mcnt_a >= -nacnt; mcnt_a -= 2) {
      const int mcnt_c = msc_ac - mcnt_a;
      if (std::abs(mcnt_c) > nccnt) continue;
      const int mex1c = msc[0] - mcnt_c, mex1a = msa[0] - mcnt_a;
      if (std::abs(mex1c) > ncex1 || std::abs(mex1a) > naex1) continue;
      const int mex2a = msa[1] - mcnt_c, mex2c = msc[1] - mcnt_a;
      if (std::abs(mex2c) > ncex2 || std::abs(mex2a) > naex2) continue;
      if (use_tr && msa[idx_restr] == 0 && msa[2] == 0 && mcnt_c - mcnt_a > 0) continue;
      double fac_scal = fac0;
      if (use_tr && msa[idx_restr] == 0 && msa[2] == 0 && mcnt_c - mcnt_a < 0) fac_scal *= 2.0;
      // IRREP(A) cases of (op1, op2, op12), first index fastest (:1117-1229)
      int graw[3] = {1, 1, 1};
      for (bool f2 = true;; f2 = false) {
        if (!f2) {
          int i = 0;
          for (; i < 3; ++i) {
            if (graw[i] >= nsym) {
              graw[i] = 1;
            } else {
              ++graw[i];
              break;
            }
          }
          if (i == 3) break;
        }
        const int ga[3] = {graw[0], graw[1], graw[2]};
        const int gc[3] = {irrep_mult(ga[0], g1t), irrep_mult(ga[1], g2t), irrep_mult(ga[2], g12t)};
        const int ixm1 = msa_to_idxms(msa[0], mst1, na1, nc1);
        const int ixm2 = msa_to_idxms(msa[1], mst2, na2, nc2);
        const int ixm12 = msa_to_idxms(msa[2], mst12, na12, nc12);
        if (B1.gmlen(ixm1, ga[0]) == 0 || B2.gmlen(ixm2, ga[1]) == 0 ||
            B12.gmlen(ixm12, ga[2]) == 0)
          continue;
        const auto& dl1 = B1.dis.at({ixm1, ga[0]});
        const auto& dl2 = B2.dis.at({ixm2, ga[1]});
        const auto& dl12 = B12.dis.at({ixm12, ga[2]});
        const int gcnt_ac = irrep_mult(irrep_mult(ga[0], ga[1]), ga[2]);
        // IRREP of the contraction string (:1231-1253)
        for (int gcnt_a = 1; gcnt_a <= nsym; ++gcnt_a) {
          const int gcnt_c = irrep_mult(gcnt_a, gcnt_ac);
          if (cntc.empty() && gcnt_c > 1) continue;
          if (cnta.empty() && gcnt_a > 1) continue;
          const int gex1a = irrep_mult(ga[0], gcnt_a), gex1c = irrep_mult(gc[0], gcnt_c);
          const int gex2a = irrep_mult(ga[1], gcnt_c), gex2c = irrep_mult(gc[1], gcnt_a);
          if (ex1c.empty() && gex1c > 1) continue;
          if (ex1a.empty() && gex1a > 1) continue;
          if (ex2c.empty() && gex2c > 1) continue;
          if (ex2a.empty() && gex2a > 1) continue;
          // distributions of ex1 (:1255-1299)
          MsGam d1;
          for (bool f3 = true;
               next_msgam(f3, d1, oc_ex1c, oc_ex1a, mex1c, mex1a, gex1c, gex1a, nsym); f3 = false) {
            auto ix1c = idxms_of(ex1c, d1.msc), ix1a = idxms_of(ex1a, d1.msa);
            auto le1c = lengths(m, ex1c, ix1c, d1.gc), le1a = lengths(m, ex1a, ix1a, d1.ga);
            if (has_zero(le1c) || has_zero(le1a)) continue;
            // distributions of ex2 (:1301-1345)
            MsGam d2;
            for (bool f4 = true;
                 next_msgam(f4, d2, oc_ex2c, oc_ex2a, mex2c, mex2a, gex2c, gex2a, nsym);
                 f4 = false) {
              auto ix2c = idxms_of(ex2c, d2.msc), ix2a = idxms_of(ex2a, d2.msa);
              auto le2c = lengths(m, ex2c, ix2c, d2.gc), le2a = lengths(m, ex2a, ix2a, d2.ga);
              if (has_zero(le2c) || has_zero(le2a)) continue;
              std::vector<int> m12c, g12c, m12a, g12a;
              merge_dist(src12c, d1.msc, d1.gc, d2.msc, d2.gc, m12c, g12c);
              merge_dist(src12a, d2.msa, d2.ga, d1.msa, d1.ga, m12a, g12a);
              auto ix12c = idxms_of(o12c, m12c), ix12a = idxms_of(o12a, m12a);
              auto l12c = lengths(m, o12c, ix12c, g12c), l12a = lengths(m, o12a, ix12a, g12a);
              if (has_zero(l12c) || has_zero(l12a)) continue;
              const Dist& D12 =
                  dl12.size() > 1
                      ? find_dist(B12, ixm12, ga[2],
                                  dist_id(o12c, ix12c, g12c, o12a, ix12a, g12a, nsym))
                      : dl12[0];
              // distributions of the contraction string (:1497-1890)
              MsGam dc;
              for (bool f5 = true; next_msgam(f5, dc, oc_cntc, oc_cnta, mcnt_c, mcnt_a, gcnt_c,
                                              gcnt_a, nsym);
                   f5 = false) {
                auto ixcc = idxms_of(cntc, dc.msc), ixca = idxms_of(cnta, dc.msa);
                auto lcc = lengths(m, cntc, ixcc, dc.gc), lca = lengths(m, cnta, ixca, dc.ga);
                if (has_zero(lcc) || has_zero(lca)) continue;
                std::vector<int> m1c, g1c, m1a, g1a;
                merge_dist(src1c, dc.msc, dc.gc, d1.msc, d1.gc, m1c, g1c);
                merge_dist(src1a, dc.msa, dc.ga, d1.msa, d1.ga, m1a, g1a);
                auto ixo1c = idxms_of(op1c, m1c), ixo1a = idxms_of(op1a, m1a);
                auto lo1c = lengths(m, op1c, ixo1c, g1c), lo1a = lengths(m, op1a, ixo1a, g1a);
                if (has_zero(lo1c) || has_zero(lo1a)) continue;
                const Dist& D1 = dl1.size() > 1 ? find_dist(B1, ixm1, ga[0],
                                                            dist_id(op1c, ixo1c, g1c, op1a, ixo1a,
                                                                    g1a, nsym))
                                                : dl1[0];
                std::vector<int> m2c, g2c, m2a, g2a;
                merge_dist(src2c, dc.msa, dc.ga, d2.msc, d2.gc, m2c, g2c);
                merge_dist(src2a, dc.msc, dc.gc, d2.msa, d2.ga, m2a, g2a);
                auto ixo2c = idxms_of(op2c, m2c), ixo2a = idxms_of(op2a, m2a);
                auto lo2c = lengths(m, op2c, ixo2c, g2c), lo2a = lengths(m, op2a, ixo2a, g2a);
                if (has_zero(lo2c) || has_zero(lo2a)) continue;
                const Dist& D2 = dl2.size() > 1 ? find_dist(B2, ixm2, ga[1],
                                                            dist_id(op2c, ixo2c, g2c, op2a, ixo2a,
                                                                    g2a, nsym))
                                                : dl2[0];
                // one block contraction
                ItemDesc it{};
                const int item = (int)P.items.size();
                it.fac = fac_scal;
                it.base1 = D1.off;
                it.base2 = D2.off;
                it.base12 = D12.off;
                std::vector<int64_t> sp[3];
                sp[kEx1] = le1c;
                sp[kEx1].insert(sp[kEx1].end(), le1a.begin(), le1a.end());
                sp[kEx2] = le2c;
                sp[kEx2].insert(sp[kEx2].end(), le2a.begin(), le2a.end());
                sp[kCnt] = lcc;
                sp[kCnt].insert(sp[kCnt].end(), lca.begin(), lca.end());
                int64_t dims[3];
                for (int q = 0; q < 3; ++q) {
                  GCCU_REQUIRE(sp[q].size() <= (size_t)kDevMaxComp, "planner: too many components");
                  it.nsp[q] = (int32_t)sp[q].size();
                  dims[q] = 1;
                  for (size_t i = 0; i < sp[q].size(); ++i) {
                    it.rad[q][i] = (int32_t)sp[q][i];
                    dims[q] *= sp[q][i];
                  }
                }
                it.M = dims[kEx1];
                it.N = dims[kEx2];
                it.K = dims[kCnt];
                std::vector<int64_t> ld1c, ld1a, ld2c, ld2a, ld12c, ld12a;
                leading_dims(op1c, op1a, lo1c, lo1a, ld1c, ld1a, s.tra1);
                leading_dims(op2c, op2a, lo2c, lo2a, ld2c, ld2a, s.tra2);
                leading_dims(o12c, o12a, l12c, l12a, ld12c, ld12a, s.tra12);
                const int ncx1 = (int)ex1c.size(), ncx2 = (int)ex2c.size(),
                          ncn = (int)cntc.size();
                Side s_cntc{&cntc, kCnt, 0, &ixcc, &dc.gc, &lcc};
                Side s_cnta{&cnta, kCnt, ncn, &ixca, &dc.ga, &lca};
                Side s_ex1c{&ex1c, kEx1, 0, &ix1c, &d1.gc, &le1c};
                Side s_ex1a{&ex1a, kEx1, ncx1, &ix1a, &d1.ga, &le1a};
                Side s_ex2c{&ex2c, kEx2, 0, &ix2c, &d2.gc, &le2c};
                Side s_ex2a{&ex2a, kEx2, ncx2, &ix2a, &d2.ga, &le2a};
                int pos = 0;
                fill_opnd(it.op[0], pos, src1c, s_cntc, s_ex1c, ld1c, item, 0, P.maps);
                fill_opnd(it.op[0], pos, src1a, s_cnta, s_ex1a, ld1a, item, 0, P.maps);
                pos = 0;
                fill_opnd(it.op[1], pos, src2c, s_cnta, s_ex2c, ld2c, item, 1, P.maps);
                fill_opnd(it.op[1], pos, src2a, s_cntc, s_ex2a, ld2a, item, 1, P.maps);
                pos = 0;
                fill_opnd(it.op[2], pos, src12c, s_ex1c, s_ex2c, ld12c, item, 2, P.maps);
                fill_opnd(it.op[2], pos, src12a, s_ex2a, s_ex1a, ld12a, item, 2, P.maps);
                it.kfast1 = unit_from(it.op[0], kCnt);
                it.kfast2 = unit_from(it.op[1], kCnt);
                account(P.stats, it.M, it.N, it.K);
                P.flops += 2.0 * (double)it.M * (double)it.N * (double)it.K;
                P.items.push_back(it);
              }
            }
          }
        }
      }
    }
  }
  return P;
}

namespace {

// Sources of the components of the original (or reordered) class in the
// unshifted part I0 and in the shifts K (get_reo_info2 / set_mapping_info):
// component (type t, vertex v) of one side takes the I0 component of type t
// on vertex v and the K component of type t of the shift that leaves
// (arrives at) vertex v.
std::vector<Src> reo_sources(const std::vector<Comp>& tgt, const std::vector<Comp>& i0,
                             const std::vector<Comp>& k, const int* vtx_of_shift, bool k_first) {
  std::vector<Src> r(tgt.size());
  for (size_t j = 0; j < tgt.size(); ++j) {
    int ii = -1, ik = -1;
    for (size_t i = 0; i < i0.size(); ++i)
      if (i0[i].hpvx == tgt[j].hpvx && i0[i].vtx == tgt[j].vtx) ii = (int)i;
    for (size_t i = 0; i < k.size(); ++i)
      if (k[i].hpvx == tgt[j].hpvx && vtx_of_shift[k[i].vtx] == tgt[j].vtx) {
        GCCU_REQUIRE(ik < 0, "reorder: two shifted strings of one type meet on one vertex");
        ik = (int)i;
      }
    GCCU_REQUIRE(ii >= 0 || ik >= 0, "reorder: component without source");
    r[j].i1 = k_first ? ik : ii;
    r[j].i2 = k_first ? ii : ik;
  }
  return r;
}

// Ms / IRREP of the unshifted part from the original distribution and the
// shifts' distribution (split_msgmdis); false if impossible
bool split_dist(const std::vector<Src>& src, bool k_first, const std::vector<int>& ms,
                const std::vector<int>& g, const std::vector<int>& msk, const std::vector<int>& gk,
                const std::vector<Comp>& i0, std::vector<int>& ms0, std::vector<int>& g0) {
  ms0.assign(i0.size(), 0);
  g0.assign(i0.size(), 1);
  for (size_t j = 0; j < src.size(); ++j) {
    const int ii = k_first ? src[j].i2 : src[j].i1, ik = k_first ? src[j].i1 : src[j].i2;
    const int mk = ik >= 0 ? msk[ik] : 0, gkk = ik >= 0 ? gk[ik] : 1;
    if (ii < 0) {
      if (ms[j] != mk || g[j] != gkk) return false;
      continue;
    }
    ms0[ii] = ms[j] - mk;
    g0[ii] = irrep_mult(g[j], gkk);
  }
  for (size_t i = 0; i < i0.size(); ++i)  // check_ms
    if (std::abs(ms0[i]) > i0[i].occ || ((i0[i].occ - ms0[i]) & 1)) return false;
  return true;
}

}  // namespace

ReoPlan plan_reorder(Model& m, const ReorderSpec& s) {
  ReoPlan P;
  const LayoutBlock& Bo = s.Lori->blk.at(s.ib_ori - 1);
  const LayoutBlock& Br = s.Lreo->blk.at(s.ib_reo - 1);
  const int nsym = m.os.nsym;
  GCCU_REQUIRE((int)Bo.vtx.size() == s.nj && (int)Br.vtx.size() == s.nj,
               "reorder: both classes must have njoined vertices");
  GCCU_REQUIRE(s.Lori->mst == s.Lreo->mst && s.Lori->gamt == s.Lreo->gamt,
               "reorder: lists differ in total Ms or IRREP");
  // I0 per vertex: original minus what leaves, equal to reordered minus what arrives
  std::vector<Occ> i0v(s.nj);
  for (int v = 0; v < s.nj; ++v) {
    for (int q = 0; q < 8; ++q) {
      int a = Bo.vtx[v][q], b = Br.vtx[v][q];
      for (int t = 0; t < s.nshift; ++t) {
        if (s.from[t] == v) a -= s.shift[t][q];
        if (s.to[t] == v) b -= s.shift[t][q];
      }
      GCCU_REQUIRE(a >= 0 && a == b, "reorder: shifts do not connect the two occupation classes");
      i0v[v][q] = a;
    }
  }
  std::vector<Comp> i0c, i0a, kc, ka;
  m.condense(i0v.data(), s.nj, i0c, i0a);
  std::vector<Occ> kv(s.shift, s.shift + s.nshift);
  m.condense(kv.data(), s.nshift, kc, ka);
  // creators merge (I0, K), annihilators (K, I0)
  auto so_c = reo_sources(Bo.c, i0c, kc, s.from, false);
  auto so_a = reo_sources(Bo.a, i0a, ka, s.from, true);
  auto sr_c = reo_sources(Br.c, i0c, kc, s.to, false);
  auto sr_a = reo_sources(Br.a, i0a, ka, s.to, true);
  const int mskc_max = sum(kc), mska_max = sum(ka), ms0c_max = sum(i0c), ms0a_max = sum(i0a);
  std::vector<int> okc = comp_occs(kc), oka = comp_occs(ka);
  for (const auto& kvp : Bo.dis) {
    const auto key = kvp.first;
    for (const Dist& d : kvp.second) {
      int msc = 0, msa = 0, gmc = 1, gma = 1;
      for (size_t j = 0; j < Bo.c.size(); ++j) msc += d.msc[j], gmc = irrep_mult(gmc, d.gc[j]);
      for (size_t j = 0; j < Bo.a.size(); ++j) msa += d.msa[j], gma = irrep_mult(gma, d.ga[j]);
      for (int mska = mska_max; mska >= -mska_max; mska -= 2) {
        if (std::abs(msa - mska) > ms0a_max) continue;
        for (int mskc = mskc_max; mskc >= -mskc_max; mskc -= 2) {
          if (std::abs(msc - mskc) > ms0c_max) continue;
          for (int gka = 1; gka <= nsym; ++gka)
            for (int gkc = 1; gkc <= nsym; ++gkc) {
              MsGam dk;
              bool first = true;
              while (next_msgam(first, dk, okc, oka, mskc, mska, gkc, gka, nsym)) {
                first = false;
                std::vector<int> ms0c, g0c, ms0a, g0a;
                if (!split_dist(so_c, false, d.msc, d.gc, dk.msc, dk.gc, i0c, ms0c, g0c)) continue;
                if (!split_dist(so_a, true, d.msa, d.ga, dk.msa, dk.ga, i0a, ms0a, g0a)) continue;
                // reordered distribution (merge_msgmdis)
                std::vector<int> mrc, grc, mra, gra;
                merge_dist(sr_c, ms0c, g0c, dk.msc, dk.gc, mrc, grc);
                merge_dist(sr_a, dk.msa, dk.ga, ms0a, g0a, mra, gra);
                auto ix0c = idxms_of(i0c, ms0c), ix0a = idxms_of(i0a, ms0a);
                auto ixkc = idxms_of(kc, dk.msc), ixka = idxms_of(ka, dk.msa);
                auto ixoc = idxms_of(Bo.c, d.msc), ixoa = idxms_of(Bo.a, d.msa);
                auto ixrc = idxms_of(Br.c, mrc), ixra = idxms_of(Br.a, mra);
                auto l0c = lengths(m, i0c, ix0c, g0c), l0a = lengths(m, i0a, ix0a, g0a);
                auto lkc = lengths(m, kc, ixkc, dk.gc), lka = lengths(m, ka, ixka, dk.ga);
                auto loc = lengths(m, Bo.c, ixoc, d.gc), loa = lengths(m, Bo.a, ixoa, d.ga);
                auto lrc = lengths(m, Br.c, ixrc, grc), lra = lengths(m, Br.a, ixra, gra);
                if (has_zero(l0c) || has_zero(l0a) || has_zero(lkc) || has_zero(lka) ||
                    has_zero(lrc) || has_zero(lra) || has_zero(loc) || has_zero(loa))
                  continue;
                const Dist& dr =
                    find_dist(Br, key.first, key.second, dist_id(Br.c, ixrc, grc, Br.a, ixra, gra, nsym));
                ReoItem it{};
                it.N0 = it.NK = 1;
                it.nsp[0] = (int)(i0c.size() + i0a.size());
                it.nsp[1] = (int)(kc.size() + ka.size());
                GCCU_REQUIRE(it.nsp[0] <= kDevMaxComp && it.nsp[1] <= kDevMaxComp,
                             "reorder: too many string components");
                int q = 0;
                for (auto x : l0c) it.rad[0][q++] = (int32_t)x, it.N0 *= x;
                for (auto x : l0a) it.rad[0][q++] = (int32_t)x, it.N0 *= x;
                q = 0;
                for (auto x : lkc) it.rad[1][q++] = (int32_t)x, it.NK *= x;
                for (auto x : lka) it.rad[1][q++] = (int32_t)x, it.NK *= x;
                it.base_ori = d.off;
                it.base_reo = dr.off;
                const int item = (int)P.items.size();
                const int nc0 = (int)i0c.size(), nck = (int)kc.size();
                Side s0c{&i0c, kEx1, 0, &ix0c, &g0c, &l0c}, s0a{&i0a, kEx1, nc0, &ix0a, &g0a, &l0a};
                Side skc{&kc, kEx2, 0, &ixkc, &dk.gc, &lkc}, ska{&ka, kEx2, nck, &ixka, &dk.ga, &lka};
                std::vector<int64_t> ldc, lda;
                int pos = 0;
                leading_dims(Bo.c, Bo.a, loc, loa, ldc, lda);
                fill_opnd(it.ori, pos, so_c, s0c, skc, ldc, item, 0, P.maps);
                fill_opnd(it.ori, pos, so_a, ska, s0a, lda, item, 0, P.maps);
                pos = 0;
                leading_dims(Br.c, Br.a, lrc, lra, ldc, lda);
                fill_opnd(it.reo, pos, sr_c, s0c, skc, ldc, item, 1, P.maps);
                fill_opnd(it.reo, pos, sr_a, ska, s0a, lda, item, 1, P.maps);
                P.elements += it.N0 * it.NK;
                P.items.push_back(it);
              }
            }
        }
      }
    }
  }
  return P;
}

ReoPlan plan_trace(Model& m, const TraceSpec& s) {
  ReoPlan P;
  const LayoutBlock& Bo = s.Lop->blk.at(s.ib_op - 1);
  const LayoutBlock& Bt = s.Lres->blk.at(s.ib_res - 1);
  const int nsym = m.os.nsym;
  GCCU_REQUIRE(Bo.vtx.size() == 1 && Bt.vtx.size() == 1, "trace: single-vertex operators only");
  GCCU_REQUIRE(s.Lop->mst == s.Lres->mst && s.Lop->gamt == s.Lres->gamt,
               "trace: operator and result differ in total Ms or IRREP");
  for (int t = 0; t < 4; ++t) {
    GCCU_REQUIRE(s.cnt[t] == s.cnt[4 + t], "trace: contracted creators and annihilators differ");
    GCCU_REQUIRE(Bo.occ[t] == Bt.occ[t] + s.cnt[t] && Bo.occ[4 + t] == Bt.occ[4 + t] + s.cnt[4 + t],
                 "trace: operator != result + contracted strings");
  }
  std::vector<Comp> jc, ja;
  m.condense(s.cnt, jc, ja);  // jc and ja list the same types in the same order
  // sources of the operator's components: J (str1) and the result (str2)
  auto src_of = [](const std::vector<Comp>& tgt, const std::vector<Comp>& j,
                   const std::vector<Comp>& r) {
    std::vector<Src> v(tgt.size());
    for (size_t q = 0; q < tgt.size(); ++q) {
      for (size_t i = 0; i < j.size(); ++i)
        if (j[i].hpvx == tgt[q].hpvx) v[q].i1 = (int)i;
      for (size_t i = 0; i < r.size(); ++i)
        if (r[i].hpvx == tgt[q].hpvx) v[q].i2 = (int)i;
      GCCU_REQUIRE(v[q].i1 >= 0 || v[q].i2 >= 0, "trace: component without source");
    }
    return v;
  };
  auto so_c = src_of(Bo.c, jc, Bt.c), so_a = src_of(Bo.a, ja, Bt.a);
  const int msj_max = sum(ja);
  std::vector<int> oja = comp_occs(ja);
  for (const auto& kvp : Bt.dis) {
    for (const Dist& d : kvp.second) {
      int msta = 0, gta = 1;
      for (size_t q = 0; q < Bt.a.size(); ++q) msta += d.msa[q], gta = irrep_mult(gta, d.ga[q]);
      for (int msj = msj_max; msj >= -msj_max; msj -= 2)
        for (int gj = 1; gj <= nsym; ++gj) {
          MsGam dj;  // next_msgamdist_diag: one distribution for both sides of J
          bool first = true;
          while (next_msgam(first, dj, {}, oja, 0, msj, 1, gj, nsym)) {
            first = false;
            std::vector<int> moc, goc, moa, goa;
            merge_dist(so_c, dj.msa, dj.ga, d.msc, d.gc, moc, goc);
            merge_dist(so_a, dj.msa, dj.ga, d.msa, d.ga, moa, goa);
            auto ixj = idxms_of(ja, dj.msa);
            auto ixtc = idxms_of(Bt.c, d.msc), ixta = idxms_of(Bt.a, d.msa);
            auto ixoc = idxms_of(Bo.c, moc), ixoa = idxms_of(Bo.a, moa);
            auto lj = lengths(m, ja, ixj, dj.ga);
            auto ltc = lengths(m, Bt.c, ixtc, d.gc), lta = lengths(m, Bt.a, ixta, d.ga);
            auto loc = lengths(m, Bo.c, ixoc, goc), loa = lengths(m, Bo.a, ixoa, goa);
            if (has_zero(lj) || has_zero(ltc) || has_zero(lta) || has_zero(loc) || has_zero(loa))
              continue;
            int msoa = msta + msj, goa_tot = irrep_mult(gta, gj);
            const int ixms_op = msa_to_idxms(msoa, s.Lop->mst, sum(Bo.a), sum(Bo.c));
            const Dist& dop = find_dist(Bo, ixms_op, goa_tot,
                                        dist_id(Bo.c, ixoc, goc, Bo.a, ixoa, goa, nsym));
            ReoItem it{};
            it.N0 = it.NK = 1;
            it.nsp[0] = (int)(Bt.c.size() + Bt.a.size());
            it.nsp[1] = (int)ja.size();
            int q = 0;
            for (auto x : ltc) it.rad[0][q++] = (int32_t)x, it.N0 *= x;
            for (auto x : lta) it.rad[0][q++] = (int32_t)x, it.N0 *= x;
            q = 0;
            for (auto x : lj) it.rad[1][q++] = (int32_t)x, it.NK *= x;
            it.base_ori = dop.off;
            it.base_reo = d.off;
            const int item = (int)P.items.size();
            const int ntc = (int)Bt.c.size();
            // J's creator components take the indices of the annihilator ones
            Side sj{&ja, kEx2, 0, &ixj, &dj.ga, &lj};
            Side stc{&Bt.c, kEx1, 0, &ixtc, &d.gc, &ltc}, sta{&Bt.a, kEx1, ntc, &ixta, &d.ga, &lta};
            std::vector<int64_t> ldc, lda;
            int pos = 0;
            leading_dims(Bo.c, Bo.a, loc, loa, ldc, lda);
            std::vector<Src> so_cj(so_c);
            for (auto& x : so_cj)  // creator J component -> index of the same type in ja
              if (x.i1 >= 0) {
                int idx = -1;
                for (size_t i = 0; i < ja.size(); ++i)
                  if (ja[i].hpvx == jc[x.i1].hpvx) idx = (int)i;
                x.i1 = idx;
              }
            fill_opnd(it.ori, pos, so_cj, sj, stc, ldc, item, 0, P.maps);
            fill_opnd(it.ori, pos, so_a, sj, sta, lda, item, 0, P.maps);
            pos = 0;
            leading_dims(Bt.c, Bt.a, ltc, lta, ldc, lda);
            std::vector<Src> dc(Bt.c.size()), da(Bt.a.size());
            for (size_t i = 0; i < dc.size(); ++i) dc[i].i2 = (int)i;
            for (size_t i = 0; i < da.size(); ++i) da[i].i2 = (int)i;
            fill_opnd(it.reo, pos, dc, sj, stc, ldc, item, 1, P.maps);
            fill_opnd(it.reo, pos, da, sj, sta, lda, item, 1, P.maps);
            P.elements += it.N0 * it.NK;
            P.items.push_back(it);
          }
        }
    }
  }
  return P;
}

}  // namespace gccu

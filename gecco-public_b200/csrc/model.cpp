#include "model.hpp"

#include <algorithm>
#include <cstdlib>

namespace gccu {

void OrbSpace::finalize() {
  for (int t = 0; t < kNType; ++t) {
    irrep[t].clear();
    for (int g = 0; g < nsym; ++g)
      for (int i = 0; i < norb[t][g]; ++i) irrep[t].push_back(g + 1);
  }
}

// Arc weights of the lexical addressing graph.  Strings are ordered with the
// highest orbital most significant and, per orbital, empty < alpha < beta <
// doubly occupied (the order generated by lexlstr/nextstr,
// strings/lexlstr.f, strings/nextstr.f).  With N_k(n,m,g) = number of
// strings on the first k orbitals with n electrons, 2Ms = m and irrep g, the
// weight of taking code c at orbital k from prefix state (n,m,g) is the
// number of strings of the same block that agree above k and carry a smaller
// code at k:  W = sum_{c'<c} N_k(state + d(c) - d(c')).  The address is the
// sum of the weights along the string's path (idx4sg_sb, strings/idx4sg_sb.f).
void Graph::build(const OrbSpace& os, int t, int ne) {
  type = t;
  nel = ne;
  nsym = os.nsym;
  norb = os.n(t);
  irrep.resize(norb);
  for (int k = 0; k < norb; ++k) irrep[k] = os.irrep[t][k] - 1;
  GCCU_REQUIRE(nel <= kMaxNel, "graph: too many electrons in one string");
  const int NM = 2 * nel + 1;
  auto nidx = [&](int n, int m, int g) { return ((size_t)n * NM + (m + nel)) * nsym + g; };
  const size_t S = (size_t)(nel + 1) * NM * nsym;
  std::vector<int64_t> N(S, 0), Nn(S, 0);
  N[nidx(0, 0, 0)] = 1;
  W.assign((size_t)norb * 3 * S, 0);
  // code: 0 empty, 1 alpha, 2 beta, 3 pair: electrons, 2Ms, carries irrep
  const int de[4] = {0, 1, 1, 2}, dm[4] = {0, 1, -1, 0};
  for (int k = 0; k < norb; ++k) {
    int gk = irrep[k];
    for (int n = 0; n <= nel; ++n)
      for (int m = -nel; m <= nel; ++m)
        for (int g = 0; g < nsym; ++g)
          for (int c = 1; c <= 3; ++c) {
            int64_t w = 0;
            for (int cp = 0; cp < c; ++cp) {
              int n2 = n + de[c] - de[cp], m2 = m + dm[c] - dm[cp];
              int g2 = g ^ ((c == 1 || c == 2) ? gk : 0) ^ ((cp == 1 || cp == 2) ? gk : 0);
              if (n2 < 0 || n2 > nel || m2 < -nel || m2 > nel) continue;
              w += N[nidx(n2, m2, g2)];
            }
            W[((((size_t)k * 3 + c - 1) * (nel + 1) + n) * NM + m + nel) * nsym + g] = w;
          }
    std::fill(Nn.begin(), Nn.end(), 0);
    for (int n = 0; n <= nel; ++n)
      for (int m = -nel; m <= nel; ++m)
        for (int g = 0; g < nsym; ++g) {
          int64_t v = N[nidx(n, m, g)];
          if (!v) continue;
          for (int c = 0; c < 4; ++c) {
            int n2 = n + de[c], m2 = m + dm[c];
            int g2 = g ^ ((c == 1 || c == 2) ? gk : 0);
            if (n2 > nel || m2 < -nel || m2 > nel) continue;
            Nn[nidx(n2, m2, g2)] += v;
          }
        }
    std::swap(N, Nn);
  }
  len.assign((size_t)(nel + 1) * nsym, 0);
  for (int ix = 1; ix <= nel + 1; ++ix) {
    int ms = nel - 2 * (ix - 1);
    for (int g = 0; g < nsym; ++g) len[(ix - 1) * nsym + g] = N[nidx(nel, ms, g)];
  }
}

int64_t Graph::address(const int* orb, const int* spn) const {
  int64_t a = 0;
  int n = 0, m = 0, g = 0;
  for (int i = 0; i < nel;) {
    int k = orb[i];
    int c = spn[i] == 2 ? 3 : (spn[i] > 0 ? 1 : 2);
    a += weight(k, c, n, m, g);
    if (c == 3) {
      n += 2;
      i += 2;
    } else {
      n += 1;
      m += (c == 1) ? 1 : -1;
      g ^= irrep[k];
      i += 1;
    }
  }
  return a;
}

// Strings of one block in address order, enumerated by recursion over the
// orbitals and placed by their address.
const std::vector<int32_t>& Graph::table(int idxms, int gam) {
  int key = (idxms - 1) * nsym + gam - 1;
  auto it = tables.find(key);
  if (it != tables.end()) return it->second;
  int64_t ns = nstr(idxms, gam);
  std::vector<int32_t> tab((size_t)ns * nel, 0);
  int ms = nel - 2 * (idxms - 1);
  std::vector<int> orb(nel + 1), spn(nel + 1);
  // recursive fill: position p, next orbital k, electrons so far, ms, irrep
  struct Rec {
    Graph* gr;
    std::vector<int32_t>* tab;
    std::vector<int>* orb;
    std::vector<int>* spn;
    int ms, g;
    void go(int p, int k, int m, int gg) {
      if (p == gr->nel) {
        if (m != ms || gg != g) return;
        int64_t a = gr->address(orb->data(), spn->data());
        for (int i = 0; i < gr->nel; ++i) {
          int code = (*spn)[i] == 2 ? 3 : ((*spn)[i] > 0 ? 1 : 2);
          (*tab)[(size_t)a * gr->nel + i] = ((*orb)[i] << 2) | code;
        }
        return;
      }
      int rem = gr->nel - p;
      for (int kk = k; kk < gr->norb; ++kk) {
        if (2 * (gr->norb - kk) < rem) break;
        (*orb)[p] = kk;
        (*spn)[p] = 1;
        go(p + 1, kk + 1, m + 1, gg ^ gr->irrep[kk]);
        (*spn)[p] = -1;
        go(p + 1, kk + 1, m - 1, gg ^ gr->irrep[kk]);
        if (rem >= 2) {
          (*orb)[p + 1] = kk;
          (*spn)[p] = (*spn)[p + 1] = 2;
          go(p + 2, kk + 1, m, gg);
        }
      }
    }
  } rec{this, &tab, &orb, &spn, ms, gam - 1};
  if (nel == 0) {
    // the single empty string
  } else if (ns > 0) {
    rec.go(0, 0, 0, 0);
  }
  return tables[key] = std::move(tab);
}

int Model::graph(int type, int nel) {
  auto k = std::make_pair(type, nel);
  auto it = graph_id.find(k);
  if (it != graph_id.end()) return it->second;
  auto g = std::make_unique<Graph>();
  g->build(os, type, nel);
  graphs.push_back(std::move(g));
  int id = (int)graphs.size();
  graphs.back()->id = id;
  graph_id[k] = id;
  return id;
}

// condense_occ (operators/condense_occ.f:46-62): components in X,P,V,H
// sequence and, within a type, by vertex; creators and annihilators
// separately
void Model::condense(const Occ* vtx, int nj, std::vector<Comp>& c, std::vector<Comp>& a) {
  c.clear();
  a.clear();
  for (int ih = 0; ih < 4; ++ih) {
    int t = kHpvxSeq[ih];
    for (int v = 0; v < nj; ++v) {
      const Occ& o = vtx[v];
      if (o[t] > 0) c.push_back({o[t], graph(t, o[t]), t, v});
      if (o[4 + t] > 0) a.push_back({o[4 + t], graph(t, o[4 + t]), t, v});
    }
  }
}

std::vector<int> comp_occs(const std::vector<Comp>& c) {
  std::vector<int> r;
  for (auto& x : c) r.push_back(x.occ);
  return r;
}

// Ms distributions: first component runs fastest from its maximum downwards,
// the last one is fixed by the total (next_msdistn/first_msdistn)
static bool ms_next(std::vector<int>& ms, int tot, const std::vector<int>& mx) {
  int n = (int)ms.size();
  if (n <= 1) return false;
  for (;;) {
    bool adv = false;
    for (int i = 0; i < n - 1; ++i) {
      if (ms[i] > -mx[i]) {
        ms[i] -= 2;
        adv = true;
        break;
      }
      ms[i] = mx[i];
    }
    if (!adv) return false;
    int s = 0;
    for (int i = 0; i < n - 1; ++i) s += ms[i];
    ms[n - 1] = tot - s;
    if (std::abs(ms[n - 1]) <= mx[n - 1]) return true;
  }
}
static bool ms_first(std::vector<int>& ms, int tot, const std::vector<int>& mx) {
  int n = (int)ms.size();
  if (n == 0) return tot == 0;
  int s = 0;
  for (int i = 0; i < n - 1; ++i) {
    ms[i] = mx[i];
    s += mx[i];
  }
  ms[n - 1] = tot - s;
  if (std::abs(ms[n - 1]) <= mx[n - 1]) return true;
  return ms_next(ms, tot, mx);
}
// IRREP distributions (next_gamdistn/first_gamdistn)
static bool gam_next(std::vector<int>& g, int tot, int nsym) {
  int n = (int)g.size();
  if (n <= 1) return false;
  int last = -1;
  for (int i = 0; i < n - 1; ++i) {
    if (g[i] < nsym) {
      ++g[i];
      last = i;
      break;
    }
    g[i] = 1;
  }
  if (last < 0) return false;
  int acc = tot;
  for (int i = last; i < n - 1; ++i) acc = irrep_mult(acc, g[i]);
  g[n - 1] = acc;
  return true;
}
static bool gam_first(std::vector<int>& g, int tot) {
  int n = (int)g.size();
  if (n == 0) return tot == 1;
  for (int i = 0; i < n - 1; ++i) g[i] = 1;
  g[n - 1] = tot;
  return true;
}

// innermost: IRREP of C, then Ms of C, IRREP of A, Ms of A
bool next_msgam(bool first, MsGam& d, const std::vector<int>& oc, const std::vector<int>& oa,
                int msc, int msa, int gamc, int gama, int nsym) {
  if (first) {
    d.msc.assign(oc.size(), 0);
    d.msa.assign(oa.size(), 0);
    d.gc.assign(oc.size(), 1);
    d.ga.assign(oa.size(), 1);
    return ms_first(d.msc, msc, oc) && ms_first(d.msa, msa, oa) && gam_first(d.gc, gamc) &&
           gam_first(d.ga, gama);
  }
  if (gam_next(d.gc, gamc, nsym)) return true;
  if (ms_next(d.msc, msc, oc)) return gam_first(d.gc, gamc);
  if (gam_next(d.ga, gama, nsym)) return ms_first(d.msc, msc, oc) && gam_first(d.gc, gamc);
  if (ms_next(d.msa, msa, oa))
    return gam_first(d.ga, gama) && ms_first(d.msc, msc, oc) && gam_first(d.gc, gamc);
  return false;
}

// integer id of a distribution (operators/msgmdid2.f)
int64_t dist_id(const std::vector<Comp>& c, const std::vector<int>& ixc, const std::vector<int>& gc,
                const std::vector<Comp>& a, const std::vector<int>& ixa, const std::vector<int>& ga,
                int nsym) {
  int64_t id = 0, base = 1;
  for (size_t i = 0; i < c.size(); ++i) {
    id += ((int64_t)(ixc[i] - 1) * nsym + gc[i] - 1) * base;
    base *= (int64_t)(c[i].occ + 1) * nsym;
  }
  for (size_t i = 0; i < a.size(); ++i) {
    id += ((int64_t)(ixa[i] - 1) * nsym + ga[i] - 1) * base;
    base *= (int64_t)(a[i].occ + 1) * nsym;
  }
  return id;
}

// operators/msa2idxms4op.f
int msa_to_idxms(int msa, int mst, int occ_a, int occ_c) {
  int r = (occ_a - msa) / 2 + 1;
  int off = occ_a - occ_c + mst;
  if (off > 0) r -= off / 2;
  return r;
}

// ME-list layout, the storage sequence of set_op_dim2
// (operators/set_op_dim2.f:176-427): occupation classes, then Ms(A) from
// high to low, IRREP(A), then the Ms/IRREP distributions over components;
// inside a distribution block creators vary fastest (C components, then A
// components, set_op_dim2.f:352-364).
void Model::layout(ListLayout& L) {
  const Operator& op = ops.at(L.op - 1);
  int nsym = os.nsym;
  int64_t pos = 0;
  L.blk.assign(op.nblk(), LayoutBlock());
  for (int64_t ib = 0; ib < op.nblk(); ++ib) {
    LayoutBlock& B = L.blk[ib];
    B.vtx.assign(op.occ.begin() + ib * op.nj, op.occ.begin() + (ib + 1) * op.nj);
    B.occ = Occ{};
    for (auto& o : B.vtx)
      for (int k = 0; k < 8; ++k) B.occ[k] += o[k];
    condense(B.vtx.data(), op.nj, B.c, B.a);
    std::vector<int> oc = comp_occs(B.c), oa = comp_occs(B.a);
    int mscmax = 0, msamax = 0;
    for (int v : oc) mscmax += v;
    for (int v : oa) msamax += v;
    B.off = pos;
    int idxmsa = 0;
    for (int msa = msamax; msa >= -msamax; msa -= 2) {
      int msc = msa + L.mst;
      if (std::abs(msc) > mscmax) continue;
      ++idxmsa;
      for (int gama = 1; gama <= nsym; ++gama) {
        int gamc = irrep_mult(gama, L.gamt);
        auto key = std::make_pair(idxmsa, gama);
        B.gm_off[key] = pos;
        std::vector<Dist>& dl = B.dis[key];
        MsGam d;
        for (bool first = true; next_msgam(first, d, oc, oa, msc, msa, gamc, gama, nsym);
             first = false) {
          std::vector<int> ixc(B.c.size()), ixa(B.a.size());
          std::vector<int64_t> ls;
          for (size_t i = 0; i < B.c.size(); ++i) {
            ixc[i] = ms_index(B.c[i].occ, d.msc[i]);
            ls.push_back(G(B.c[i].graph).nstr(ixc[i], d.gc[i]));
          }
          for (size_t i = 0; i < B.a.size(); ++i) {
            ixa[i] = ms_index(B.a[i].occ, d.msa[i]);
            ls.push_back(G(B.a[i].graph).nstr(ixa[i], d.ga[i]));
          }
          int64_t len = 1;
          for (auto v : ls) len *= v;
          if (len <= 0) continue;
          int64_t ld = 1;
          bool found = false;
          for (int ih = 0; ih < 4 && !found; ++ih) {
            int t = kHpvxSeq[ih];
            for (size_t i = 0; i < B.c.size() && !found; ++i)
              if (B.c[i].hpvx == t) ld = ls[i], found = true;
            for (size_t i = 0; i < B.a.size() && !found; ++i)
              if (B.a[i].hpvx == t) ld = ls[B.c.size() + i], found = true;
          }
          Dist ds;
          ds.off = pos;
          ds.len = len;
          ds.ld = ld;
          ds.did = dist_id(B.c, ixc, d.gc, B.a, ixa, d.ga, nsym);
          ds.msc = d.msc;
          ds.msa = d.msa;
          ds.gc = d.gc;
          ds.ga = d.ga;
          dl.push_back(ds);
          pos += len;
        }
        B.gm_len[key] = pos - B.gm_off[key];
      }
    }
    B.len = pos - B.off;
  }
  L.len = pos;
}

}  // namespace gccu

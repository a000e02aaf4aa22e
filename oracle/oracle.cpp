// ORACLE -- CPU restatement of GeCCo's blocked tensor-contraction path.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h).  Restates, in plain C++, the
// reference routines named at each function.  Scope: single-vertex operators
// (njoined = 1), one GAS per hole/particle/valence/external type (frozen or
// deleted orbitals are simply absent from the orbital counts), no reordering
// step inside a contraction.
//
// Parity pins (tests/golden): string counts and ME-list lengths printed by the
// reference for the HF/cc-pVDZ MOLPRO fixture (test/python-interface.s.ref:
// 176-197 and :459-465) and the converged MP2 energy of that run (:629,:660).
// Block-level values have no reference fixture (the reference's Fortran cannot
// be built here); the restatement is held to those pins plus self-consistency
// of route 2 vs route 3 and invariance tests.
#include "oracle.h"

#include <dlfcn.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

thread_local std::string g_err;

constexpr int NGASTP = 4;
// hpvxseq = (4,2,3,1): X,P,V,H (include/hpvxseq.h:3); 0-based type ids
constexpr int HPVXSEQ[4] = {3, 1, 2, 0};

inline int mult(int a, int b) { return ((a - 1) ^ (b - 1)) + 1; }  // include/multd2h.h

struct Fail : std::runtime_error {
  using std::runtime_error::runtime_error;
};
#define CHECK(c, msg) \
  do {                \
    if (!(c)) throw Fail(msg); \
  } while (0)

// ---------------------------------------------------------------------------
// strings
// ---------------------------------------------------------------------------

// lexically lowest string, single subspace (strings/lexlstr.f:2-145).
// orb: 1-based orbital numbers, spn: +1 alpha, -1 beta, 2 paired.
bool lexlstr(int nel, int itms, int norb, int* orb, int* spn) {
  if (nel == 0) return true;
  int npair = (nel - std::abs(itms)) / 2;
  int nalpht = npair, nbetat = npair;
  if (itms > 0) nalpht += itms;
  if (itms < 0) nbetat -= itms;
  // minimum number of pairs for one subspace of norb orbitals
  if (norb < nel) {
    int need = nel - norb;
    if (need > norb) return false;
  }
  int ipos = 0, inum = 1;
  npair = std::min(nalpht, nbetat);
  if (npair < 0) return false;
  int npair4ss = std::min(npair, nel / 2);
  nalpht -= npair4ss;
  nbetat -= npair4ss;
  for (int ip = 0; ip < npair4ss; ++ip) {
    orb[ipos] = orb[ipos + 1] = inum;
    spn[ipos] = spn[ipos + 1] = 2;
    ipos += 2;
    ++inum;
  }
  int nlone = nel - 2 * npair4ss;
  int nalph4ss = std::min(nalpht, nlone);
  int nbeta4ss = nlone - nalph4ss;
  for (int i = 0; i < nbeta4ss; ++i) {
    orb[ipos] = inum++;
    spn[ipos++] = -1;
  }
  for (int i = 0; i < nalph4ss; ++i) {
    orb[ipos] = inum++;
    spn[ipos++] = +1;
  }
  return inum - 1 <= norb;
}

// lexically next string of same Ms, single subspace (strings/nextstr.f:2-188)
bool nextstr(int nel, int norb, int* orb, int* spn) {
  int ipos = 1, ms_pos = 0, ipairc = 0, ms_sub = 0;
  int idspnn = 0;
  bool lnext = true, lsame = false;
  for (;;) {
    int idorbc = orb[ipos - 1];
    int idspnc = spn[ipos - 1];
    if (!lsame) {
      if (idspnc == 2 && ipairc == 0) {
        ++ipos;
        ipairc = 1;
        continue;
      } else if (idspnc == 2 && ipairc == 1) {
        ipairc = 0;
        idspnc = -1;
      } else {
        ms_pos += idspnc;
      }
    } else {
      lsame = false;
    }
    int nalph = (ipos + ms_pos) / 2;
    int nbeta = (ipos - ms_pos) / 2;
    int iorbmax = norb;
    int idorbn = (ipos < nel) ? orb[ipos] : 1 << 30;
    if (ipos < nel) idspnn = spn[ipos];
    if (idspnc == +1 && nbeta > 0) {
      spn[ipos - 1] = -1;
      ms_sub = ms_pos + 1;
    } else if ((ipos == nel || idorbc < idorbn - 1) && idorbc < iorbmax) {
      orb[ipos - 1] += 1;
      if (idspnc == -1 && nalph > 0) {
        spn[ipos - 1] = +1;
        ms_sub = ms_pos - 1;
      } else {
        ms_sub = ms_pos - idspnc;
      }
    } else if (idorbc < idorbn && idorbc < iorbmax && idspnn == -1 && nalph > 0) {
      orb[ipos - 1] += 1;
      spn[ipos - 1] = 2;
      spn[ipos] = 2;
      ms_sub = ms_pos - 1;
    } else if (ipos == nel) {
      lnext = false;
      break;
    } else {
      ++ipos;
      continue;
    }
    if (ipos == 1) break;
    int nelsb = ipos - 1;
    lnext = lexlstr(nelsb, ms_sub, norb, orb, spn);
    if (lnext && spn[nelsb] == -1 && orb[nelsb - 1] == orb[nelsb]) {
      spn[nelsb - 1] = spn[nelsb] = 2;
    }
    if (lnext) break;
    lsame = true;
  }
  return lnext;
}

struct OrbInfo {
  int nsym = 1;
  int norb[4][8] = {};
  std::vector<int> irrep[4];  // 1-based irrep of each (1-based) orbital in type
  void init() {
    for (int t = 0; t < 4; ++t) {
      irrep[t].assign(1, 0);
      for (int g = 0; g < nsym; ++g)
        for (int i = 0; i < norb[t][g]; ++i) irrep[t].push_back(g + 1);
    }
  }
  int n(int t) const { return (int)irrep[t].size() - 1; }
};

// igamstr2 (strings/igamstr2.f)
int igamstr(const OrbInfo& oi, int t, int nel, const int* orb) {
  int g = 1;
  for (int i = 0; i < nel; ++i) g = mult(g, oi.irrep[t][orb[i]]);
  return g;
}

// all strings of one (type,nel,ms,gam) block in the order of next_string
// (strings/next_string.f:2-205, single subspace, no restriction)
struct StrBlock {
  int nel = 0;
  std::vector<int> orb, spn;  // nstr*nel
  std::unordered_map<std::string, int64_t> index;
  int64_t n() const { return nel ? (int64_t)orb.size() / nel : (int64_t)orb.size(); }
};

std::string key_of(int nel, const int* orb, const int* spn) {
  std::string k(nel * 2, '\0');
  for (int i = 0; i < nel; ++i) {
    k[2 * i] = (char)(orb[i] & 0xff);
    k[2 * i + 1] = (char)(((orb[i] >> 8) & 0x3f) | ((spn[i] + 1) << 6));
  }
  return k;
}

struct Graph {
  int type = 0, nel = 0;
  // blocks[idxms-1][gam-1]
  std::vector<std::vector<StrBlock>> blk;
  int64_t len(int idxms, int gam) const {
    if (idxms < 1 || idxms > nel + 1) return 0;
    return blk[idxms - 1][gam - 1].n();
  }
};

void build_graph(const OrbInfo& oi, Graph& g) {
  int nel = g.nel, t = g.type, norb = oi.n(t);
  g.blk.assign(nel + 1, std::vector<StrBlock>(oi.nsym));
  for (int idxms = 1; idxms <= nel + 1; ++idxms) {
    int ms = nel - (idxms - 1) * 2;
    for (int gm = 1; gm <= oi.nsym; ++gm) {
      StrBlock& b = g.blk[idxms - 1][gm - 1];
      b.nel = nel;
      if (nel == 0) {
        if (gm == 1) {
          b.orb.push_back(0);  // one empty string
          b.index[std::string()] = 0;
        }
        continue;
      }
      std::vector<int> orb(nel), spn(nel);
      bool ok = lexlstr(nel, ms, norb, orb.data(), spn.data());
      while (ok) {
        if (igamstr(oi, t, nel, orb.data()) == gm) {
          b.index[key_of(nel, orb.data(), spn.data())] = b.n();
          b.orb.insert(b.orb.end(), orb.begin(), orb.end());
          b.spn.insert(b.spn.end(), spn.begin(), spn.end());
        }
        ok = nextstr(nel, norb, orb.data(), spn.data());
      }
    }
  }
}

// merge two ordered strings, reorder, return parity sign or 0
// (strings/iordstr2.f:2-119)
int iordstr2(int* o12, int* s12, const int* o1, const int* s1, int n1,
             const int* o2, const int* s2, int n2) {
  if (n1 + n2 == 0) return 1;
  if (n2 == 0) {
    std::copy(o1, o1 + n1, o12);
    std::copy(s1, s1 + n1, s12);
    return 1;
  }
  if (n1 == 0) {
    std::copy(o2, o2 + n2, o12);
    std::copy(s2, s2 + n2, s12);
    return 1;
  }
  int ip1 = 0, ip2 = 0, iperm = 0;
  for (int ip = 0; ip < n1 + n2; ++ip) {
    if (ip1 < n1 && ip2 < n2) {
      int sp = s1[ip1] * s2[ip2];
      if (o1[ip1] == o2[ip2] && sp != -1) return 0;
    }
    if (ip2 >= n2 ||
        (ip1 < n1 && (o1[ip1] < o2[ip2] || (o1[ip1] == o2[ip2] && s1[ip1] == +1)))) {
      o12[ip] = o1[ip1];
      s12[ip] = s1[ip1];
      ++ip1;
    } else {
      o12[ip] = o2[ip2];
      s12[ip] = s2[ip2];
      ++ip2;
      iperm += n1 - ip1;
    }
  }
  for (int i = 0; i + 1 < n1 + n2; ++i)
    if (o12[i] == o12[i + 1]) s12[i] = s12[i + 1] = 2;
  return (iperm % 2) ? -1 : 1;
}

// std_spsign (strings/std_spsign_msdis.f)
int std_spsign(const int* spn, int nel) {
  int trp = 0, nb = 0, idx = 0;
  while (idx < nel) {
    int sig = spn[idx];
    if (sig == 1 || sig == 2) {
      trp += nb;
      ++idx;
    }
    if (sig == -1 || sig == 2) {
      ++nb;
      ++idx;
    }
  }
  return (trp % 2) ? -1 : 1;
}

int std_spsign_msdis(const std::vector<int>& msdis, const std::vector<int>& occ) {
  if (msdis.size() <= 1) return 1;
  std::vector<int> scr;
  for (size_t b = 0; b < msdis.size(); ++b) {
    for (int i = 0; i < (occ[b] + msdis[b]) / 2; ++i) scr.push_back(+1);
    for (int i = 0; i < (occ[b] - msdis[b]) / 2; ++i) scr.push_back(-1);
  }
  return std_spsign(scr.data(), (int)scr.size());
}

// ---------------------------------------------------------------------------
// context: graphs, string maps, operators, lists
// ---------------------------------------------------------------------------

struct Comp {  // one row of a cinfo array (occupation, graph, hpvx)
  int occ, graph, hpvx;
  int vtx = 0;  // vertex of a joined operator (or shift index of a reorder)
};

struct DistRow {
  int64_t off, len, ld;
  int64_t did;
};

struct ListBlock {
  int64_t off_occ = 0, len_occ = 0;
  std::vector<Comp> c, a;  // condensed components
  // per (idxmsa, gama): offset, length, distributions
  std::map<std::pair<int, int>, int64_t> gm_off, gm_len;
  std::map<std::pair<int, int>, std::vector<DistRow>> dis;
};

struct Op {
  int nj = 1;                            // njoined
  std::vector<std::array<int, 8>> occ;  // C[H,P,V,X], A[H,P,V,X]; nblk*nj, vertices consecutive
};

struct List {
  int op = 0, gamt = 1, mst = 0, absym = 0;
  int64_t len = 0;
  std::vector<ListBlock> blk;
};

}  // namespace

struct ora_ctx {
  OrbInfo oi;
  std::map<std::pair<int, int>, int> graph_id;  // (type,nel) -> id
  std::deque<Graph> graphs;  // stable references while graphs are added
  std::vector<Op> ops;
  std::vector<List> lists;
  // string map blocks, keyed by (g1,g2,idxms1,idxms2,gam1,gam2)
  std::map<std::array<int, 6>, std::vector<int>> strmaps;
  std::map<std::array<int, 3>, std::vector<int>> flipmaps;  // (g,idxms,gam)
  std::map<std::array<int, 3>, std::vector<int>> spprjmaps;  // (g,idxms,gam)

  int graph(int type, int nel) {
    auto k = std::make_pair(type, nel);
    auto it = graph_id.find(k);
    if (it != graph_id.end()) return it->second;
    Graph g;
    g.type = type;
    g.nel = nel;
    build_graph(oi, g);
    graphs.push_back(std::move(g));
    int id = (int)graphs.size();
    graph_id[k] = id;
    return id;
  }
  const Graph& G(int id) const { return graphs[id - 1]; }

  // set_strmap_kernel (strings/set_strmap_kernel.f:66-119): loop str2 outer,
  // str1 inner; entry = sign*(idx4sg+1), 0 if Pauli-forbidden
  const std::vector<int>& strmap(int g1, int g2, int idxms1, int idxms2, int gam1,
                                 int gam2) {
    std::array<int, 6> k{g1, g2, idxms1, idxms2, gam1, gam2};
    auto it = strmaps.find(k);
    if (it != strmaps.end()) return it->second;
    const Graph &G1 = G(g1), &G2 = G(g2);
    CHECK(G1.type == G2.type, "set_strmap: incompatible graph types");
    int g12 = graph(G1.type, G1.nel + G2.nel);
    const Graph& G12 = G(g12);
    const StrBlock& b1 = G1.blk[idxms1 - 1][gam1 - 1];
    const StrBlock& b2 = G2.blk[idxms2 - 1][gam2 - 1];
    int n1 = G1.nel, n2 = G2.nel, n12 = n1 + n2;
    int ms12 = (n1 - 2 * (idxms1 - 1)) + (n2 - 2 * (idxms2 - 1));
    int idxms12 = (n12 - ms12) / 2 + 1;
    int gam12 = mult(gam1, gam2);
    const StrBlock& b12 = G12.blk[idxms12 - 1][gam12 - 1];
    std::vector<int> m;
    m.reserve(b1.n() * b2.n());
    std::vector<int> o12(n12 + 1), s12(n12 + 1);
    for (int64_t i2 = 0; i2 < b2.n(); ++i2) {
      for (int64_t i1 = 0; i1 < b1.n(); ++i1) {
        int sg = iordstr2(o12.data(), s12.data(), b1.orb.data() + i1 * n1,
                          b1.spn.data() + i1 * n1, n1, b2.orb.data() + i2 * n2,
                          b2.spn.data() + i2 * n2, n2);
        if (sg == 0) {
          m.push_back(0);
          continue;
        }
        auto f = b12.index.find(key_of(n12, o12.data(), s12.data()));
        CHECK(f != b12.index.end(), "set_strmap_kernel: merged string not addressable");
        m.push_back(sg * (int)(f->second + 1));
      }
    }
    return strmaps[k] = std::move(m);
  }

  // set_flipmap_kernel (strings/set_flipmap_kernel.f): str -> spin-flipped str
  const std::vector<int>& flipmap(int g, int idxms, int gam) {
    std::array<int, 3> k{g, idxms, gam};
    auto it = flipmaps.find(k);
    if (it != flipmaps.end()) return it->second;
    const Graph& Gr = G(g);
    int nel = Gr.nel;
    const StrBlock& b = Gr.blk[idxms - 1][gam - 1];
    const StrBlock& bf = Gr.blk[nel + 1 - idxms][gam - 1];
    std::vector<int> m;
    std::vector<int> sf(nel + 1);
    for (int64_t i = 0; i < b.n(); ++i) {
      const int* o = b.orb.data() + i * nel;
      const int* s = b.spn.data() + i * nel;
      for (int j = 0; j < nel; ++j) sf[j] = (s[j] == 2) ? 2 : -s[j];
      int sg = std_spsign(s, nel) * std_spsign(sf.data(), nel);
      auto f = bf.index.find(key_of(nel, o, sf.data()));
      CHECK(f != bf.index.end(), "flip map: flipped string not addressable");
      m.push_back(sg * (int)(f->second + 1));
    }
    return flipmaps[k] = std::move(m);
  }
};

namespace {

// condense_occ (operators/condense_occ.f:46-62): loop over the hpvx
// sequence X,P,V,H, inside it over the vertices; C and A separately
void condense_n(ora_ctx* cx, const int* occ, int nj, std::vector<Comp>& c,
                std::vector<Comp>& a) {
  c.clear();
  a.clear();
  for (int ih = 0; ih < 4; ++ih) {
    int t = HPVXSEQ[ih];
    for (int v = 0; v < nj; ++v) {
      const int* o = occ + 8 * v;
      if (o[t] > 0) c.push_back({o[t], cx->graph(t, o[t]), t, v});
      if (o[4 + t] > 0) a.push_back({o[4 + t], cx->graph(t, o[4 + t]), t, v});
    }
  }
}
void condense(ora_ctx* cx, const int* occ8, std::vector<Comp>& c, std::vector<Comp>& a) {
  condense_n(cx, occ8, 1, c, a);
}

// ---- Ms / IRREP distributions (operators/next_msgamdist2.f) ----
bool next_msdistn(std::vector<int>& ms, int mst, const std::vector<int>& mx) {
  int n = (int)ms.size();
  if (n <= 1) return false;
  for (;;) {
    bool nxt = false;
    for (int i = 0; i < n - 1; ++i) {
      if (ms[i] > -mx[i]) {
        ms[i] -= 2;
        nxt = true;
        break;
      } else {
        ms[i] = mx[i];
      }
    }
    if (!nxt) return false;
    int s = 0;
    for (int i = 0; i < n - 1; ++i) s += ms[i];
    ms[n - 1] = mst - s;
    if (std::abs(ms[n - 1]) <= mx[n - 1]) return true;
  }
}
bool first_msdistn(std::vector<int>& ms, int mst, const std::vector<int>& mx) {
  int n = (int)ms.size();
  if (n == 0) return mst == 0;
  if (n > 1) {
    int s = 0;
    for (int i = 0; i < n - 1; ++i) {
      ms[i] = mx[i];
      s += mx[i];
    }
    ms[n - 1] = mst - s;
  } else {
    ms[0] = mst;
  }
  if (std::abs(ms[n - 1]) <= mx[n - 1]) return true;
  return next_msdistn(ms, mst, mx);
}
bool next_gamdistn(std::vector<int>& g, int gamt, int nsym) {
  int n = (int)g.size();
  if (n <= 1) return false;
  int ilast = -1;
  for (int i = 0; i < n - 1; ++i) {
    if (g[i] < nsym) {
      g[i] += 1;
      ilast = i;
      break;
    } else {
      g[i] = 1;
    }
  }
  if (ilast < 0) return false;
  int acc = gamt;
  for (int i = ilast; i < n - 1; ++i) acc = mult(acc, g[i]);
  g[n - 1] = acc;
  return true;
}
bool first_gamdistn(std::vector<int>& g, int gamt) {
  int n = (int)g.size();
  if (n == 0) return gamt == 1;
  for (int i = 0; i < n - 1; ++i) g[i] = 1;
  g[n - 1] = gamt;
  return true;
}
struct MsGamDist {
  std::vector<int> msc, msa, gc, ga;
};
bool next_msgamdist2(bool first, MsGamDist& d, const std::vector<int>& occc,
                     const std::vector<int>& occa, int msc, int msa, int gamc, int gama,
                     int nsym) {
  bool ok;
  if (first) {
    d.msc.assign(occc.size(), 0);
    d.msa.assign(occa.size(), 0);
    d.gc.assign(occc.size(), 1);
    d.ga.assign(occa.size(), 1);
    ok = first_msdistn(d.msc, msc, occc);
    ok = ok && first_msdistn(d.msa, msa, occa);
    ok = ok && first_gamdistn(d.gc, gamc);
    ok = ok && first_gamdistn(d.ga, gama);
  } else if (next_gamdistn(d.gc, gamc, nsym)) {
    ok = true;
  } else if (next_msdistn(d.msc, msc, occc)) {
    ok = first_gamdistn(d.gc, gamc);
  } else if (next_gamdistn(d.ga, gama, nsym)) {
    ok = first_msdistn(d.msc, msc, occc);
    ok = ok && first_gamdistn(d.gc, gamc);
  } else if (next_msdistn(d.msa, msa, occa)) {
    ok = first_gamdistn(d.ga, gama);
    ok = ok && first_msdistn(d.msc, msc, occc);
    ok = ok && first_gamdistn(d.gc, gamc);
  } else {
    ok = false;
  }
  return ok;
}

std::vector<int> occs(const std::vector<Comp>& c) {
  std::vector<int> o;
  for (auto& x : c) o.push_back(x.occ);
  return o;
}
inline int idxms_of(int occ, int ms) { return ((occ - ms) >> 1) + 1; }

// msgmdid2 (operators/msgmdid2.f)
int64_t msgmdid2(const std::vector<Comp>& c, const std::vector<int>& idxmsc,
                 const std::vector<int>& gc, const std::vector<Comp>& a,
                 const std::vector<int>& idxmsa, const std::vector<int>& ga, int nsym) {
  int64_t patt = 0, base = 1;
  for (size_t i = 0; i < c.size(); ++i) {
    patt += ((idxmsc[i] - 1) * nsym + gc[i] - 1) * base;
    base *= (c[i].occ + 1) * nsym;
  }
  for (size_t i = 0; i < a.size(); ++i) {
    patt += ((idxmsa[i] - 1) * nsym + ga[i] - 1) * base;
    base *= (a[i].occ + 1) * nsym;
  }
  return patt;
}

// msa2idxms4op (operators/msa2idxms4op.f)
int msa2idxms4op(int msa, int mst, int occ_a, int occ_c) {
  int r = (occ_a - msa) / 2 + 1;
  int off = occ_a - occ_c + mst;
  if (off > 0) r -= off / 2;
  return r;
}

// set_op_dim2 (operators/set_op_dim2.f:1-531), no diag_type, no fixed
// vertex Ms; joined operators through their condensed components
void set_op_dim2(ora_ctx* cx, List& L) {
  const Op& op = cx->ops[L.op - 1];
  int nsym = cx->oi.nsym;
  int64_t idxstr = 0;
  const size_t nblk = op.occ.size() / op.nj;
  L.blk.assign(nblk, ListBlock());
  for (size_t ib = 0; ib < nblk; ++ib) {
    ListBlock& B = L.blk[ib];
    condense_n(cx, op.occ[ib * op.nj].data(), op.nj, B.c, B.a);
    int msc_max = 0, msa_max = 0;
    for (auto& x : B.c) msc_max += x.occ;
    for (auto& x : B.a) msa_max += x.occ;
    B.off_occ = idxstr;
    int idxmsa = 0;
    std::vector<int> oc = occs(B.c), oa = occs(B.a);
    for (int msa = msa_max; msa >= -msa_max; msa -= 2) {
      int msc = msa + L.mst;
      if (std::abs(msc) > msc_max) continue;
      ++idxmsa;
      for (int gama = 1; gama <= nsym; ++gama) {
        int gamc = mult(gama, L.gamt);
        auto key = std::make_pair(idxmsa, gama);
        B.gm_off[key] = idxstr;
        auto& dl = B.dis[key];
        MsGamDist d;
        bool first = true;
        while (next_msgamdist2(first, d, oc, oa, msc, msa, gamc, gama, nsym)) {
          first = false;
          std::vector<int> ixc(B.c.size()), ixa(B.a.size());
          std::vector<int64_t> ls;
          for (size_t i = 0; i < B.c.size(); ++i) {
            ixc[i] = idxms_of(B.c[i].occ, d.msc[i]);
            ls.push_back(cx->G(B.c[i].graph).len(ixc[i], d.gc[i]));
          }
          for (size_t i = 0; i < B.a.size(); ++i) {
            ixa[i] = idxms_of(B.a[i].occ, d.msa[i]);
            ls.push_back(cx->G(B.a[i].graph).len(ixa[i], d.ga[i]));
          }
          int64_t len = 1;
          for (auto v : ls) len *= v;
          // leading dimension: first component in hpvx sequence
          int64_t ld = 1;
          bool found = false;
          for (int ih = 0; ih < 4 && !found; ++ih) {
            int t = HPVXSEQ[ih];
            for (size_t i = 0; i < B.c.size() && !found; ++i)
              if (B.c[i].hpvx == t) {
                ld = ls[i];
                found = true;
              }
            for (size_t i = 0; i < B.a.size() && !found; ++i)
              if (B.a[i].hpvx == t) {
                ld = ls[B.c.size() + i];
                found = true;
              }
          }
          if (len <= 0) continue;
          DistRow r;
          r.off = idxstr;
          r.len = len;
          r.ld = ld;
          r.did = msgmdid2(B.c, ixc, d.gc, B.a, ixa, d.ga, nsym);
          dl.push_back(r);
          idxstr += len;
        }
        B.gm_len[key] = idxstr - B.gm_off[key];
      }
    }
    B.len_occ = idxstr - B.off_occ;
  }
  L.len = idxstr;
}

// set_mapping_info (contract/set_mapping_info.f), njoined = 1: for each
// component of the merged string (condensed order), the component of str1
// and/or str2 of the same hpvx type.  Stored as [n1,(i1),n2,(i2)] per comp.
std::vector<int> mapping_info(const int* occ1, bool dag1, const int* occ2, bool dag2,
                              const int* occ12, int ca) {
  auto seq = [](const int* occ, int ca_, int t) {
    // position of (type t, side ca_) in the condensed list of that side
    int pos = 0;
    for (int ih = 0; ih < 4; ++ih) {
      int tt = HPVXSEQ[ih];
      if (occ[ca_ * 4 + tt] > 0) {
        ++pos;
        if (tt == t) return pos;
      }
    }
    return 0;
  };
  std::vector<int> m;
  int ca1 = dag1 ? 1 - ca : ca, ca2 = dag2 ? 1 - ca : ca;
  for (int ih = 0; ih < 4; ++ih) {
    int t = HPVXSEQ[ih];
    if (occ12[ca * 4 + t] == 0) continue;
    if (occ1[ca1 * 4 + t] > 0) {
      m.push_back(1);
      m.push_back(seq(occ1, ca1, t));
    } else {
      m.push_back(0);
    }
    if (occ2[ca2 * 4 + t] > 0) {
      m.push_back(1);
      m.push_back(seq(occ2, ca2, t));
    } else {
      m.push_back(0);
    }
  }
  return m;
}

// parsed map_info: for merged comp j -> (i1 or -1, i2 or -1) 0-based
struct MapInf {
  std::vector<std::pair<int, int>> src;
};
MapInf parse(const std::vector<int>& m, int n12) {
  MapInf r;
  size_t p = 0;
  for (int j = 0; j < n12; ++j) {
    int i1 = -1, i2 = -1;
    int n = m[p++];
    if (n) i1 = m[p++] - 1;
    n = m[p++];
    if (n) i2 = m[p++] - 1;
    r.src.push_back({i1, i2});
  }
  return r;
}

// merge_msgmdis (contract/merge_msgmdis.f)
void merge_msgm(const MapInf& mi, const std::vector<int>& ms1, const std::vector<int>& g1,
                const std::vector<int>& ms2, const std::vector<int>& g2,
                std::vector<int>& msr, std::vector<int>& gr) {
  msr.assign(mi.src.size(), 0);
  gr.assign(mi.src.size(), 1);
  for (size_t j = 0; j < mi.src.size(); ++j) {
    if (mi.src[j].first >= 0) {
      msr[j] += ms1[mi.src[j].first];
      gr[j] = mult(gr[j], g1[mi.src[j].first]);
    }
    if (mi.src[j].second >= 0) {
      msr[j] += ms2[mi.src[j].second];
      gr[j] = mult(gr[j], g2[mi.src[j].second]);
    }
  }
}

// one string map of a merged side: concatenation of per-component maps
// (strings/get_strmap_blk_c.f:52-203); trivial maps are the identity
struct SideMap {
  std::vector<const int*> ptr;       // null -> identity
  std::vector<int64_t> n1;           // length of str1 component (fast index)
  std::vector<int> s1, s2;           // source component (or -1)
};

SideMap side_map(ora_ctx* cx, const MapInf& mi, const std::vector<Comp>& c1,
                 const std::vector<int>& idxms1, const std::vector<int>& g1,
                 const std::vector<int64_t>& l1, const std::vector<Comp>& c2,
                 const std::vector<int>& idxms2, const std::vector<int>& g2,
                 const std::vector<int64_t>& l2) {
  SideMap s;
  for (auto& p : mi.src) {
    s.s1.push_back(p.first);
    s.s2.push_back(p.second);
    if (p.first >= 0 && p.second >= 0) {
      const auto& m = cx->strmap(c1[p.first].graph, c2[p.second].graph, idxms1[p.first],
                                 idxms2[p.second], g1[p.first], g2[p.second]);
      s.ptr.push_back(m.data());
      s.n1.push_back(l1[p.first]);
    } else {
      s.ptr.push_back(nullptr);
      s.n1.push_back(p.first >= 0 ? l1[p.first] : 0);
    }
  }
  return s;
}

// value (1-based signed index) of merged component j for component strings
// i1 (of side 1), i2 (of side 2), both 0-based
inline int mapval(const SideMap& s, int j, const int64_t* i1, const int64_t* i2) {
  int a = s.s1[j], b = s.s2[j];
  if (!s.ptr[j]) return (int)((a >= 0 ? i1[a] : i2[b]) + 1);
  return s.ptr[j][i2[b] * s.n1[j] + i1[a]];
}

// set_op_ldim_c (contract/set_op_ldim_c.f:27-76): per hpvx type C then A;
// transposed, A (last component first) then C (last first)
void ldims(const std::vector<Comp>& c, const std::vector<Comp>& a,
           const std::vector<int64_t>& ls, std::vector<int64_t>& ldc,
           std::vector<int64_t>& lda, bool transpose = false) {
  ldc.assign(c.size(), 0);
  lda.assign(a.size(), 0);
  int64_t ld = 1;
  for (int ih = 0; ih < 4; ++ih) {
    int t = HPVXSEQ[ih];
    if (!transpose) {
      for (size_t i = 0; i < c.size(); ++i)
        if (c[i].hpvx == t) {
          ldc[i] = ld;
          ld *= ls[i];
        }
      for (size_t i = 0; i < a.size(); ++i)
        if (a[i].hpvx == t) {
          lda[i] = ld;
          ld *= ls[c.size() + i];
        }
    } else {
      for (size_t i = a.size(); i-- > 0;)
        if (a[i].hpvx == t) {
          lda[i] = ld;
          ld *= ls[c.size() + i];
        }
      for (size_t i = c.size(); i-- > 0;)
        if (c[i].hpvx == t) {
          ldc[i] = ld;
          ld *= ls[i];
        }
    }
  }
}

void decompose(int64_t idx, const std::vector<int64_t>& radix, int64_t* out) {
  for (size_t i = 0; i < radix.size(); ++i) {
    out[i] = idx % radix[i];
    idx /= radix[i];
  }
}

int64_t prod(const std::vector<int64_t>& v, size_t b, size_t e) {
  int64_t p = 1;
  for (size_t i = b; i < e; ++i) p *= v[i];
  return p;
}

// everything one block contraction (one call of the inner kernel) needs
struct Blk {
  double xfac;
  double *x12;
  const double *x1, *x2;
  int ncex1, naex1, ncex2, naex2, nccnt, nacnt;
  std::vector<int64_t> lex1, lex2, lcnt;            // component lengths (C then A)
  std::vector<int64_t> ld1c, ld1a, ld2c, ld2a, ld12c, ld12a;
  SideMap m12c, m12a, m1c, m1a, m2c, m2a;
};

// address of op1 element (ex1 comps, cnt comps) -> (offset, sign) ; sign 0 = forbidden
inline int addr1(const Blk& b, const int64_t* e1, const int64_t* cn, int64_t& off) {
  int sg = 1;
  off = 0;
  for (size_t j = 0; j < b.ld1c.size(); ++j) {  // op1 C: (cnt C, ex1 C)
    int v = mapval(b.m1c, (int)j, cn, e1);
    if (!v) return 0;
    if (v < 0) sg = -sg;
    off += (std::abs(v) - 1) * b.ld1c[j];
  }
  for (size_t j = 0; j < b.ld1a.size(); ++j) {  // op1 A: (cnt A, ex1 A)
    int v = mapval(b.m1a, (int)j, cn + b.nccnt, e1 + b.ncex1);
    if (!v) return 0;
    if (v < 0) sg = -sg;
    off += (std::abs(v) - 1) * b.ld1a[j];
  }
  return sg;
}
inline int addr2(const Blk& b, const int64_t* e2, const int64_t* cn, int64_t& off) {
  int sg = 1;
  off = 0;
  for (size_t j = 0; j < b.ld2c.size(); ++j) {  // op2 C: (cnt A, ex2 C)
    int v = mapval(b.m2c, (int)j, cn + b.nccnt, e2);
    if (!v) return 0;
    if (v < 0) sg = -sg;
    off += (std::abs(v) - 1) * b.ld2c[j];
  }
  for (size_t j = 0; j < b.ld2a.size(); ++j) {  // op2 A: (cnt C, ex2 A)
    int v = mapval(b.m2a, (int)j, cn, e2 + b.ncex2);
    if (!v) return 0;
    if (v < 0) sg = -sg;
    off += (std::abs(v) - 1) * b.ld2a[j];
  }
  return sg;
}
inline int addr12(const Blk& b, const int64_t* e1, const int64_t* e2, int64_t& off) {
  int sg = 1;
  off = 0;
  for (size_t j = 0; j < b.ld12c.size(); ++j) {  // C: (ex1 C, ex2 C)
    int v = mapval(b.m12c, (int)j, e1, e2);
    if (!v) return 0;
    if (v < 0) sg = -sg;
    off += (std::abs(v) - 1) * b.ld12c[j];
  }
  for (size_t j = 0; j < b.ld12a.size(); ++j) {  // A: (ex2 A, ex1 A)
    int v = mapval(b.m12a, (int)j, e2 + b.ncex2, e1 + b.ncex1);
    if (!v) return 0;
    if (v < 0) sg = -sg;
    off += (std::abs(v) - 1) * b.ld12a[j];
  }
  return sg;
}

// route 2: contr_blk1blk2_wmaps_c (contract/contr_blk1blk2_wmaps_c.f:186-406)
// loop order ex1a, ex2a, ex1c, ex2c, cnta, cntc; sign = product of map signs
void route2(const Blk& b) {
  std::vector<int64_t> lex1c(b.lex1.begin(), b.lex1.begin() + b.ncex1),
      lex1a(b.lex1.begin() + b.ncex1, b.lex1.end()),
      lex2c(b.lex2.begin(), b.lex2.begin() + b.ncex2),
      lex2a(b.lex2.begin() + b.ncex2, b.lex2.end()),
      lcc(b.lcnt.begin(), b.lcnt.begin() + b.nccnt), lca(b.lcnt.begin() + b.nccnt, b.lcnt.end());
  int64_t n1a = prod(lex1a, 0, lex1a.size()), n2a = prod(lex2a, 0, lex2a.size()),
          n1c = prod(lex1c, 0, lex1c.size()), n2c = prod(lex2c, 0, lex2c.size()),
          nca = prod(lca, 0, lca.size()), ncc = prod(lcc, 0, lcc.size());
  int64_t e1[8], e2[8], cn[8];
  for (int64_t i1a = 0; i1a < n1a; ++i1a) {
    decompose(i1a, lex1a, e1 + b.ncex1);
    for (int64_t i2a = 0; i2a < n2a; ++i2a) {
      decompose(i2a, lex2a, e2 + b.ncex2);
      for (int64_t i1c = 0; i1c < n1c; ++i1c) {
        decompose(i1c, lex1c, e1);
        for (int64_t i2c = 0; i2c < n2c; ++i2c) {
          decompose(i2c, lex2c, e2);
          int64_t o12;
          int s12 = addr12(b, e1, e2, o12);
          if (!s12) continue;
          for (int64_t ica = 0; ica < nca; ++ica) {
            decompose(ica, lca, cn + b.nccnt);
            for (int64_t icc = 0; icc < ncc; ++icc) {
              decompose(icc, lcc, cn);
              int64_t o1, o2;
              int s1 = addr1(b, e1, cn, o1);
              if (!s1) continue;
              int s2 = addr2(b, e2, cn, o2);
              if (!s2) continue;
              double sgn = b.xfac * (double)(s12 * s1 * s2);
              b.x12[o12] += sgn * b.x1[o1] * b.x2[o2];
            }
          }
        }
      }
    }
  }
}

// optional BLAS for the route-3 dgemm (the reference links an ILP64 BLAS,
// configure.ac:107-108); without it a plain loop is used
typedef void (*dgemm_t)(const char*, const char*, const int64_t*, const int64_t*, const int64_t*,
                        const double*, const double*, const int64_t*, const double*,
                        const int64_t*, const double*, double*, const int64_t*);
dgemm_t g_dgemm = nullptr;

// timing sample: only every g_stride-th long-operand batch of route 3 is
// executed (the CPU baseline times a bounded sample of a large workload);
// the short-operand gathers always run
int64_t g_stride = 1, g_batch = 0, g_batches_total = 0, g_batches_done = 0;
int64_t g_short_total = 0, g_short_done = 0;
double g_t_always = 0, g_t_sampled = 0;
// sharding of the block contractions over ranks (ora_set_shard)
int64_t g_shard_rank = 0, g_shard_n = 1, g_shard_item = 0;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// route 3: contr_blk1blk2_blocked_mm (contract/contr_blk1blk2_blocked_mm.f:
// 184-595): batches of str_block ex strings and cnt_block cnt strings,
// collect_block_impr gathers, dgemm('t','n'), scatter_block.
struct Stats {
  double v[8] = {};
};
void route3(const Blk& b, int64_t str_block, int64_t cnt_block, Stats* st) {
  int64_t nex1 = prod(b.lex1, 0, b.lex1.size()), nex2 = prod(b.lex2, 0, b.lex2.size()),
          ncnt = prod(b.lcnt, 0, b.lcnt.size());
  bool op1shorter = nex1 <= nex2;
  int64_t nexs = op1shorter ? nex1 : nex2, nexl = op1shorter ? nex2 : nex1;
  int64_t mexl = std::min(nexl, str_block), mexs = std::min(nexs, str_block);
  int64_t mcnt = ncnt;
  if (cnt_block > 0) mcnt = std::min(mcnt, cnt_block);
  std::vector<double> ps, pl, pr;
  int64_t e1[8], e2[8], cn[8];
  auto gather = [&](bool isop1, int64_t ex0, int64_t nex, int64_t c0, int64_t nc,
                    std::vector<double>& p) {
    p.assign(nex * nc, 0.0);
    for (int64_t l = 0; l < nex; ++l) {
      int64_t* e = isop1 ? e1 : e2;
      decompose(ex0 + l, isop1 ? b.lex1 : b.lex2, e);
      for (int64_t k = 0; k < nc; ++k) {
        decompose(c0 + k, b.lcnt, cn);
        int64_t o;
        int s = isop1 ? addr1(b, e1, cn, o) : addr2(b, e2, cn, o);
        if (s) p[l * nc + k] = s * (isop1 ? b.x1[o] : b.x2[o]);
      }
    }
  };
  for (int64_t c0 = 0; c0 < ncnt; c0 += mcnt) {
    int64_t nc = std::min(mcnt, ncnt - c0);
    // the short operand (all its ex strings) is gathered once per cnt batch,
    // always, also when sampling skips every long-operand batch of it: its
    // cost differs widely between block contractions, so it is measured, not
    // extrapolated
    {
      double t0 = now_s();
      gather(op1shorter, 0, nexs, c0, nc, ps);
      g_t_always += now_s() - t0;
      ++g_short_total;
      ++g_short_done;
    }
    for (int64_t l0 = 0; l0 < nexl; l0 += mexl) {
      ++g_batches_total;
      if ((g_batch++) % g_stride != 0) continue;
      ++g_batches_done;
      double t1 = now_s();
      int64_t nl = std::min(mexl, nexl - l0);
      gather(!op1shorter, l0, nl, c0, nc, pl);
      for (int64_t s0 = 0; s0 < nexs; s0 += mexs) {
        int64_t ns = std::min(mexs, nexs - s0);
        int64_t d1 = op1shorter ? ns : nl, d2 = op1shorter ? nl : ns;
        if (st) {
          st->v[0] += 1;
          st->v[1] += d1;
          st->v[2] += (double)d1 * d1;
          st->v[3] += d2;
          st->v[4] += (double)d2 * d2;
          st->v[5] += nc;
          st->v[6] += (double)nc * nc;
          st->v[7] += 2.0 * d1 * d2 * nc;
        }
        // dgemm('t','n'): R(s,l) = xfac * sum_k S(k,s) L(k,l)
        pr.assign(ns * nl, 0.0);
        if (g_dgemm) {
          const double zero = 0.0;
          g_dgemm("T", "N", &ns, &nl, &nc, &b.xfac, &ps[s0 * nc], &nc, pl.data(), &nc, &zero,
                  pr.data(), &ns);
        } else {
          for (int64_t l = 0; l < nl; ++l)
            for (int64_t s = 0; s < ns; ++s) {
              const double* a = &ps[(s0 + s) * nc];
              const double* c = &pl[l * nc];
              double acc = 0;
              for (int64_t k = 0; k < nc; ++k) acc += a[k] * c[k];
              pr[l * ns + s] = b.xfac * acc;
            }
        }
        // scatter_block: x12(idx) += sign * panel
        for (int64_t l = 0; l < nl; ++l)
          for (int64_t s = 0; s < ns; ++s) {
            int64_t i1 = op1shorter ? s0 + s : l0 + l, i2 = op1shorter ? l0 + l : s0 + s;
            decompose(i1, b.lex1, e1);
            decompose(i2, b.lex2, e2);
            int64_t o;
            int sg = addr12(b, e1, e2, o);
            if (sg) b.x12[o] += sg * pr[l * ns + s];
          }
      }
      g_t_sampled += now_s() - t1;
    }
  }
}

struct CntInfo {
  std::vector<Comp> op1c, op1a, op2c, op2a, ex1c, ex1a, ex2c, ex2a, cntc, cnta, op12c, op12a;
  MapInf m1c, m1a, m2c, m2a, m12c, m12a;
};

int sum_occ(const std::vector<Comp>& c) {
  int s = 0;
  for (auto& x : c) s += x.occ;
  return s;
}

bool next_dist(int* d, int n, const int (*mnmx)[2], int inc) {
  if (inc > 0) {
    for (int i = 0; i < n; ++i) {
      if (d[i] >= mnmx[i][1]) {
        d[i] = mnmx[i][0];
      } else {
        d[i] += inc;
        return true;
      }
    }
  } else {
    for (int i = 0; i < n; ++i) {
      if (d[i] <= mnmx[i][0]) {
        d[i] = mnmx[i][1];
      } else {
        d[i] += inc;
        return true;
      }
    }
  }
  return false;
}

int64_t find_dis(const ListBlock& B, int idxms, int gam, int64_t did) {
  auto it = B.dis.find({idxms, gam});
  CHECK(it != B.dis.end(), "idx_msgmdst2: no distributions");
  for (size_t i = 0; i < it->second.size(); ++i)
    if (it->second[i].did == did) return (int64_t)i;
  throw Fail("idx_msgmdst2: distribution not found");
}

std::vector<int> ixms(const std::vector<Comp>& c, const std::vector<int>& ms) {
  std::vector<int> r;
  for (size_t i = 0; i < c.size(); ++i) r.push_back(idxms_of(c[i].occ, ms[i]));
  return r;
}
std::vector<int64_t> lens(ora_ctx* cx, const std::vector<Comp>& c, const std::vector<int>& ix,
                          const std::vector<int>& g) {
  std::vector<int64_t> r;
  for (size_t i = 0; i < c.size(); ++i) r.push_back(cx->G(c[i].graph).len(ix[i], g[i]));
  return r;
}
bool anyzero(const std::vector<int64_t>& v) {
  for (auto x : v)
    if (x == 0) return true;
  return false;
}
std::vector<int64_t> cat(const std::vector<int64_t>& a, const std::vector<int64_t>& b) {
  std::vector<int64_t> r(a);
  r.insert(r.end(), b.begin(), b.end());
  return r;
}

double ddot_blk(const double* x, int64_t n) {
  double s = 0;
  for (int64_t i = 0; i < n; ++i) s += x[i] * x[i];
  return s;
}

void sym_ab_blk(ora_ctx* cx, List& L, int iblk, double* buf, double prefac, double relfac);

// contr_op1op2_wmaps_c (contract/contr_op1op2_wmaps_c.f:2-2169), buftyp 0.
// tra[0..2]: op1, op2, result used transposed (the vertex's dagger flag,
// contract/get_bc_info3.f:173,191,391): the occupation enters daggered
// (contract/occvtx4contr), the total Ms negated (:427-429), the IRREP loop
// runs over the stored A IRREP which is the C IRREP of the adjoint
// (:1127-1145), distribution ids are taken with C and A exchanged
// (operators/idx_msgmdst2.f:64-66) and leading dimensions in A-C sequence
// (contract/set_op_ldim_c.f:47-76).
void contract(ora_ctx* cx, int route, int l1, int ib1, const double* x1, int l2, int ib2,
              const double* x2, int l12, int ib12, double* x12, const int* oex1,
              const int* oex2, const int* ocnt, double fact, bool update, bool use_tr,
              int64_t str_block, int64_t cnt_block, double* xret, Stats* st,
              const bool* tra = nullptr) {
  static const bool no_tra[3] = {false, false, false};
  if (!tra) tra = no_tra;
  const List &L1 = cx->lists[l1 - 1], &L2 = cx->lists[l2 - 1];
  List& L12 = cx->lists[l12 - 1];
  CHECK(cx->ops[L1.op - 1].nj == 1 && cx->ops[L2.op - 1].nj == 1 &&
            (ib12 == 0 || cx->ops[L12.op - 1].nj == 1),
        "contract: joined operators are not restated");
  const ListBlock &B1 = L1.blk[ib1 - 1], &B2 = L2.blk[ib2 - 1];
  int nsym = cx->oi.nsym;
  // occupations of the operators (daggered when used transposed)
  int o1[8], o2[8];
  auto dag = [](const int* o, bool t, int* out) {
    for (int k = 0; k < 8; ++k) out[k] = t ? o[(k + 4) % 8] : o[k];
  };
  dag(cx->ops[L1.op - 1].occ[ib1 - 1].data(), tra[0], o1);
  dag(cx->ops[L2.op - 1].occ[ib2 - 1].data(), tra[1], o2);
  int o12[8] = {0};
  static const ListBlock scalar_blk = [] {
    ListBlock s;
    return s;
  }();
  bool scalar = ib12 == 0;
  if (!scalar) dag(cx->ops[L12.op - 1].occ[ib12 - 1].data(), tra[2], o12);
  // consistency: op1 = ex1 + cnt, op2 = ex2 + cnt^+, op12 = ex1 + ex2
  for (int t = 0; t < 4; ++t) {
    CHECK(o1[t] == oex1[t] + ocnt[t] && o1[4 + t] == oex1[4 + t] + ocnt[4 + t],
          "contract: op1 != ex1 + cnt");
    CHECK(o2[t] == oex2[t] + ocnt[4 + t] && o2[4 + t] == oex2[4 + t] + ocnt[t],
          "contract: op2 != ex2 + cnt^+");
    CHECK(o12[t] == oex1[t] + oex2[t] && o12[4 + t] == oex1[4 + t] + oex2[4 + t],
          "contract: op12 != ex1 + ex2");
  }
  CHECK(mult(L1.gamt, L2.gamt) == (scalar ? 1 : L12.gamt), "contract: inconsistent symmetries");
  CntInfo ci;
  // condense_bc_info (contract/condense_bc_info.f)
  condense(cx, o1, ci.op1c, ci.op1a);
  condense(cx, o2, ci.op2c, ci.op2a);
  condense(cx, oex1, ci.ex1c, ci.ex1a);
  condense(cx, oex2, ci.ex2c, ci.ex2a);
  condense(cx, ocnt, ci.cntc, ci.cnta);
  condense(cx, o12, ci.op12c, ci.op12a);
  ci.m1c = parse(mapping_info(ocnt, false, oex1, false, o1, 0), (int)ci.op1c.size());
  ci.m1a = parse(mapping_info(ocnt, false, oex1, false, o1, 1), (int)ci.op1a.size());
  ci.m2c = parse(mapping_info(ocnt, true, oex2, false, o2, 0), (int)ci.op2c.size());
  ci.m2a = parse(mapping_info(ocnt, true, oex2, false, o2, 1), (int)ci.op2a.size());
  ci.m12c = parse(mapping_info(oex1, false, oex2, false, o12, 0), (int)ci.op12c.size());
  ci.m12a = parse(mapping_info(oex2, false, oex1, false, o12, 1), (int)ci.op12a.size());

  int mst1 = tra[0] ? -L1.mst : L1.mst, mst2 = tra[1] ? -L2.mst : L2.mst,
      mst12 = scalar ? 0 : (tra[2] ? -L12.mst : L12.mst);
  int g1t = L1.gamt, g2t = L2.gamt, g12t = scalar ? 1 : L12.gamt;
  int na1 = sum_occ(ci.op1a), nc1 = sum_occ(ci.op1c), na2 = sum_occ(ci.op2a),
      nc2 = sum_occ(ci.op2c), na12 = sum_occ(ci.op12a), nc12 = sum_occ(ci.op12c);
  int ncex1 = sum_occ(ci.ex1c), naex1 = sum_occ(ci.ex1a), ncex2 = sum_occ(ci.ex2c),
      naex2 = sum_occ(ci.ex2a), nccnt = sum_occ(ci.cntc), nacnt = sum_occ(ci.cnta);

  bool use_tr_here = use_tr && L1.absym != 0 && L2.absym != 0 && !scalar && L12.absym != 0 &&
                     L1.absym * L2.absym == L12.absym;
  if (scalar) use_tr_here = false;

  const ListBlock& B12 = scalar ? scalar_blk : L12.blk[ib12 - 1];
  int64_t ioff1 = B1.off_occ, ioff2 = B2.off_occ, ioff12 = scalar ? 0 : B12.off_occ;
  const double* xop1 = x1 + ioff1;
  const double* xop2 = x2 + ioff2;
  double* xop12 = scalar ? xret : x12 + ioff12;
  if (!update) {
    if (scalar)
      *xret = 0.0;
    else
      std::fill(xop12, xop12 + B12.len_occ, 0.0);
  }

  int msbnd[3][2] = {{-na1, na1}, {-na2, na2}, {-na12, na12}};
  int idx_restr = (na2 > na1) ? 1 : 0;
  int mscmx_a = nacnt, mscmx_c = nccnt;
  int gbnd[3][2] = {{1, nsym}, {1, nsym}, {1, nsym}};
  int ms_a[3] = {na1, na2, na12};
  bool first1 = true;
  for (;;) {
    if (first1) {
      first1 = false;
    } else if (!next_dist(ms_a, 3, msbnd, -2)) {
      break;
    }
    int ms_c[3] = {ms_a[0] + mst1, ms_a[1] + mst2, ms_a[2] + mst12};
    if (std::abs(ms_c[0]) > nc1 || std::abs(ms_c[1]) > nc2 || std::abs(ms_c[2]) > nc12) continue;
    int msc_ac = ms_a[0] + ms_a[1] - ms_a[2];
    if (mscmx_a + mscmx_c < std::abs(msc_ac)) continue;
    if (use_tr_here && (ms_a[2] < 0 || (ms_a[2] == 0 && ms_a[idx_restr] < 0))) continue;
    double fac0 = 1.0;
    if (use_tr_here && ms_a[2] > 0) fac0 *= 2.0;
    if (use_tr_here && ms_a[2] == 0 && ms_a[idx_restr] > 0) fac0 *= 2.0;
    for (int msc_a = mscmx_a; msc_a >= -mscmx_a; msc_a -= 2) {
      int msc_c = msc_ac - msc_a;
      if (std::abs(msc_c) > mscmx_c) continue;
      int msex1_c = ms_c[0] - msc_c, msex1_a = ms_a[0] - msc_a;
      if (std::abs(msex1_c) > ncex1 || std::abs(msex1_a) > naex1) continue;
      int msex2_a = ms_a[1] - msc_c, msex2_c = ms_c[1] - msc_a;
      if (std::abs(msex2_c) > ncex2 || std::abs(msex2_a) > naex2) continue;
      if (use_tr_here && ms_a[idx_restr] == 0 && ms_a[2] == 0 && msc_c - msc_a > 0) continue;
      double fac_scal = fac0;
      if (use_tr_here && ms_a[idx_restr] == 0 && ms_a[2] == 0 && msc_c - msc_a < 0)
        fac_scal *= 2.0;
      int graw[3] = {1, 1, 1};
      bool first2 = true;
      for (;;) {
        if (first2) {
          first2 = false;
        } else if (!next_dist(graw, 3, gbnd, +1)) {
          break;
        }
        const int gt[3] = {g1t, g2t, g12t};
        int ga[3], gc[3];
        for (int q = 0; q < 3; ++q) {
          ga[q] = tra[q] ? mult(graw[q], gt[q]) : graw[q];
          gc[q] = tra[q] ? graw[q] : mult(graw[q], gt[q]);
        }
        int ixm1 = msa2idxms4op(ms_a[0], mst1, na1, nc1);
        int ixm2 = msa2idxms4op(ms_a[1], mst2, na2, nc2);
        int ixm12 = msa2idxms4op(ms_a[2], mst12, na12, nc12);
        auto glen = [](const ListBlock& B, int ix, int g) -> int64_t {
          auto it = B.gm_len.find({ix, g});
          return it == B.gm_len.end() ? 0 : it->second;
        };
        if (glen(B1, ixm1, graw[0]) == 0 || glen(B2, ixm2, graw[1]) == 0) continue;
        if (!scalar && glen(B12, ixm12, graw[2]) == 0) continue;
        int64_t idxop1 = B1.gm_off.at({ixm1, graw[0]}) - ioff1;
        int64_t idxop2 = B2.gm_off.at({ixm2, graw[1]}) - ioff2;
        int64_t idxop12 = scalar ? 0 : B12.gm_off.at({ixm12, graw[2]}) - ioff12;
        int gc_ac = mult(mult(ga[0], ga[1]), ga[2]);
        for (int gcnt_a = 1; gcnt_a <= nsym; ++gcnt_a) {
          int gcnt_c = mult(gcnt_a, gc_ac);
          if (ci.cntc.empty() && gcnt_c > 1) continue;
          if (ci.cnta.empty() && gcnt_a > 1) continue;
          int gex1_a = mult(ga[0], gcnt_a), gex1_c = mult(gc[0], gcnt_c);
          int gex2_a = mult(ga[1], gcnt_c), gex2_c = mult(gc[1], gcnt_a);
          if (ci.ex1c.empty() && gex1_c > 1) continue;
          if (ci.ex1a.empty() && gex1_a > 1) continue;
          if (ci.ex2c.empty() && gex2_c > 1) continue;
          if (ci.ex2a.empty() && gex2_a > 1) continue;
          MsGamDist d1;
          bool f3 = true;
          while (next_msgamdist2(f3, d1, occs(ci.ex1c), occs(ci.ex1a), msex1_c, msex1_a, gex1_c,
                                 gex1_a, nsym)) {
            f3 = false;
            auto ix1c = ixms(ci.ex1c, d1.msc), ix1a = ixms(ci.ex1a, d1.msa);
            auto le1c = lens(cx, ci.ex1c, ix1c, d1.gc), le1a = lens(cx, ci.ex1a, ix1a, d1.ga);
            if (anyzero(le1c) || anyzero(le1a)) continue;
            MsGamDist d2;
            bool f4 = true;
            while (next_msgamdist2(f4, d2, occs(ci.ex2c), occs(ci.ex2a), msex2_c, msex2_a,
                                   gex2_c, gex2_a, nsym)) {
              f4 = false;
              auto ix2c = ixms(ci.ex2c, d2.msc), ix2a = ixms(ci.ex2a, d2.msa);
              auto le2c = lens(cx, ci.ex2c, ix2c, d2.gc), le2a = lens(cx, ci.ex2a, ix2a, d2.ga);
              if (anyzero(le2c) || anyzero(le2a)) continue;
              std::vector<int> msic, gic, msia, gia;
              merge_msgm(ci.m12c, d1.msc, d1.gc, d2.msc, d2.gc, msic, gic);
              merge_msgm(ci.m12a, d2.msa, d2.ga, d1.msa, d1.ga, msia, gia);
              auto ixic = ixms(ci.op12c, msic), ixia = ixms(ci.op12a, msia);
              auto l12c = lens(cx, ci.op12c, ixic, gic), l12a = lens(cx, ci.op12a, ixia, gia);
              if (anyzero(l12c) || anyzero(l12a)) continue;
              SideMap m12c = side_map(cx, ci.m12c, ci.ex1c, ix1c, d1.gc, le1c, ci.ex2c, ix2c,
                                      d2.gc, le2c);
              SideMap m12a = side_map(cx, ci.m12a, ci.ex2a, ix2a, d2.ga, le2a, ci.ex1a, ix1a,
                                      d1.ga, le1a);
              if (!scalar && B12.dis.at({ixm12, graw[2]}).size() > 1) {
                int64_t did = tra[2] ? msgmdid2(ci.op12a, ixia, gia, ci.op12c, ixic, gic, nsym)
                                     : msgmdid2(ci.op12c, ixic, gic, ci.op12a, ixia, gia, nsym);
                int64_t id = find_dis(B12, ixm12, graw[2], did);
                idxop12 = B12.dis.at({ixm12, graw[2]})[id].off - ioff12;
              }
              MsGamDist dc;
              bool f5 = true;
              while (next_msgamdist2(f5, dc, occs(ci.cntc), occs(ci.cnta), msc_c, msc_a, gcnt_c,
                                     gcnt_a, nsym)) {
                f5 = false;
                auto ixcc = ixms(ci.cntc, dc.msc), ixca = ixms(ci.cnta, dc.msa);
                auto lcc = lens(cx, ci.cntc, ixcc, dc.gc), lca = lens(cx, ci.cnta, ixca, dc.ga);
                if (anyzero(lcc) || anyzero(lca)) continue;
                std::vector<int> ms1c, g1c, ms1a, g1a;
                merge_msgm(ci.m1c, dc.msc, dc.gc, d1.msc, d1.gc, ms1c, g1c);
                merge_msgm(ci.m1a, dc.msa, dc.ga, d1.msa, d1.ga, ms1a, g1a);
                auto ix1oc = ixms(ci.op1c, ms1c), ix1oa = ixms(ci.op1a, ms1a);
                auto lo1c = lens(cx, ci.op1c, ix1oc, g1c), lo1a = lens(cx, ci.op1a, ix1oa, g1a);
                if (anyzero(lo1c) || anyzero(lo1a)) continue;
                if (B1.dis.at({ixm1, graw[0]}).size() > 1) {
                  int64_t did = tra[0] ? msgmdid2(ci.op1a, ix1oa, g1a, ci.op1c, ix1oc, g1c, nsym)
                                       : msgmdid2(ci.op1c, ix1oc, g1c, ci.op1a, ix1oa, g1a, nsym);
                  int64_t id = find_dis(B1, ixm1, graw[0], did);
                  idxop1 = B1.dis.at({ixm1, graw[0]})[id].off - ioff1;
                }
                int64_t len1 = prod(cat(lo1c, lo1a), 0, lo1c.size() + lo1a.size());
                if (ddot_blk(xop1 + idxop1, len1) < 1e-28) continue;
                std::vector<int> ms2c, g2c, ms2a, g2a;
                merge_msgm(ci.m2c, dc.msa, dc.ga, d2.msc, d2.gc, ms2c, g2c);
                merge_msgm(ci.m2a, dc.msc, dc.gc, d2.msa, d2.ga, ms2a, g2a);
                auto ix2oc = ixms(ci.op2c, ms2c), ix2oa = ixms(ci.op2a, ms2a);
                auto lo2c = lens(cx, ci.op2c, ix2oc, g2c), lo2a = lens(cx, ci.op2a, ix2oa, g2a);
                if (anyzero(lo2c) || anyzero(lo2a)) continue;
                if (B2.dis.at({ixm2, graw[1]}).size() > 1) {
                  int64_t did = tra[1] ? msgmdid2(ci.op2a, ix2oa, g2a, ci.op2c, ix2oc, g2c, nsym)
                                       : msgmdid2(ci.op2c, ix2oc, g2c, ci.op2a, ix2oa, g2a, nsym);
                  int64_t id = find_dis(B2, ixm2, graw[1], did);
                  idxop2 = B2.dis.at({ixm2, graw[1]})[id].off - ioff2;
                }
                int64_t len2 = prod(cat(lo2c, lo2a), 0, lo2c.size() + lo2a.size());
                if (ddot_blk(xop2 + idxop2, len2) < 1e-28) continue;
                // sharded evaluation: block contractions dealt round-robin
                // to the ranks, each rank computes its own (the ranks' partial
                // results sum to the whole)
                if ((g_shard_item++) % g_shard_n != g_shard_rank) continue;
                Blk b;
                b.xfac = fact * fac_scal;
                b.x1 = xop1 + idxop1;
                b.x2 = xop2 + idxop2;
                b.x12 = xop12 + idxop12;
                b.ncex1 = (int)ci.ex1c.size();
                b.naex1 = (int)ci.ex1a.size();
                b.ncex2 = (int)ci.ex2c.size();
                b.naex2 = (int)ci.ex2a.size();
                b.nccnt = (int)ci.cntc.size();
                b.nacnt = (int)ci.cnta.size();
                b.lex1 = cat(le1c, le1a);
                b.lex2 = cat(le2c, le2a);
                b.lcnt = cat(lcc, lca);
                ldims(ci.op1c, ci.op1a, cat(lo1c, lo1a), b.ld1c, b.ld1a, tra[0]);
                ldims(ci.op2c, ci.op2a, cat(lo2c, lo2a), b.ld2c, b.ld2a, tra[1]);
                ldims(ci.op12c, ci.op12a, cat(l12c, l12a), b.ld12c, b.ld12a, tra[2]);
                b.m12c = m12c;
                b.m12a = m12a;
                b.m1c = side_map(cx, ci.m1c, ci.cntc, ixcc, dc.gc, lcc, ci.ex1c, ix1c, d1.gc, le1c);
                b.m1a = side_map(cx, ci.m1a, ci.cnta, ixca, dc.ga, lca, ci.ex1a, ix1a, d1.ga, le1a);
                b.m2c = side_map(cx, ci.m2c, ci.cnta, ixca, dc.ga, lca, ci.ex2c, ix2c, d2.gc, le2c);
                b.m2a = side_map(cx, ci.m2a, ci.cntc, ixcc, dc.gc, lcc, ci.ex2a, ix2a, d2.ga, le2a);
                if (route == 2)
                  route2(b);
                else
                  route3(b, str_block, cnt_block, st);
              }
            }
          }
        }
      }
    }
  }
  if (use_tr_here) {
    CHECK(std::abs(L12.absym) == 1, "contract: absym must be +-1 with use_tr");
    sym_ab_blk(cx, L12, ib12, x12, 0.5, (double)L12.absym);
  }
}

// sym_ab_blk (contract/sym_ab_blk.f:2-405): x(idx1) and its spin-flipped
// partner x(idx2) both become prefac*(x1 + s*x2) (resp. times s)
// ---- reorder (contract/reo_op_wmaps_c.f, contract/reo_blk_wmaps_c.f) ----

// map_info_to_ori / map_info_to_reo (get_reo_info2): for each component of
// one side of the operator, the I0 component on the same vertex and the
// shifted component (type t) leaving/arriving at that vertex; -1 if none
struct ReoSrc {
  int i0 = -1, k = -1;
};
std::vector<ReoSrc> reo_map_info(const std::vector<Comp>& tgt, const std::vector<Comp>& i0,
                                 const std::vector<Comp>& k, const int* vtx_of_shift) {
  std::vector<ReoSrc> r(tgt.size());
  for (size_t j = 0; j < tgt.size(); ++j) {
    for (size_t i = 0; i < i0.size(); ++i)
      if (i0[i].hpvx == tgt[j].hpvx && i0[i].vtx == tgt[j].vtx) r[j].i0 = (int)i;
    for (size_t i = 0; i < k.size(); ++i)
      if (k[i].hpvx == tgt[j].hpvx && vtx_of_shift[k[i].vtx] == tgt[j].vtx) {
        CHECK(r[j].k < 0, "reorder: two shifted strings of one type on one vertex");
        r[j].k = (int)i;
      }
    CHECK(r[j].i0 >= 0 || r[j].k >= 0, "reorder: component without source");
  }
  return r;
}

// string map of one component (get_strmap_blk_c): str1/str2 as given, the
// trivial map when one of the two is absent
struct CompMap {
  const std::vector<int>* m = nullptr;  // null: identity
  int64_t n1 = 1;
};

// reo_blk_wmaps_c (contract/reo_blk_wmaps_c.f:2-854) for one distribution of
// the original class, xo = that distribution's elements
void reo_blk(ora_ctx* cx, double fac, double* xreo, const double* xo, int sign_reo,
             int ms_op_c, int ms_op_a, int gm_op_c, int gm_op_a,
             const std::vector<int>& ms_i_c, const std::vector<int>& ms_i_a,
             const std::vector<int>& gm_i_c, const std::vector<int>& gm_i_a,
             const ListBlock& Bo, const ListBlock& Br, const std::vector<Comp>& kc,
             const std::vector<Comp>& ka, const std::vector<Comp>& i0c,
             const std::vector<Comp>& i0a, const std::vector<ReoSrc>& to_ori_c,
             const std::vector<ReoSrc>& to_ori_a, const std::vector<ReoSrc>& to_reo_c,
             const std::vector<ReoSrc>& to_reo_a, int idxms_op_a, int nsym) {
  int ms_k_c_max = 0, ms_k_a_max = 0, ms_i0_c_max = 0, ms_i0_a_max = 0;
  for (auto& x : kc) ms_k_c_max += x.occ;
  for (auto& x : ka) ms_k_a_max += x.occ;
  for (auto& x : i0c) ms_i0_c_max += x.occ;
  for (auto& x : i0a) ms_i0_a_max += x.occ;
  for (int ms_k_a = ms_k_a_max; ms_k_a >= -ms_k_a_max; ms_k_a -= 2) {
    if (std::abs(ms_op_a - ms_k_a) > ms_i0_a_max) continue;
    for (int ms_k_c = ms_k_c_max; ms_k_c >= -ms_k_c_max; ms_k_c -= 2) {
      if (std::abs(ms_op_c - ms_k_c) > ms_i0_c_max) continue;
      for (int gm_k_a = 1; gm_k_a <= nsym; ++gm_k_a) {
        for (int gm_k_c = 1; gm_k_c <= nsym; ++gm_k_c) {
          MsGamDist dk;
          bool first = true;
          while (next_msgamdist2(first, dk, occs(kc), occs(ka), ms_k_c, ms_k_a, gm_k_c, gm_k_a,
                                 nsym)) {
            first = false;
            // split_msgmdis: I0 = I - K, component by component
            std::vector<int> ms0c(i0c.size()), g0c(i0c.size()), ms0a(i0a.size()),
                g0a(i0a.size());
            bool possible = true;
            auto split = [&](const std::vector<ReoSrc>& src, const std::vector<int>& ms,
                             const std::vector<int>& gm, const std::vector<int>& msk,
                             const std::vector<int>& gmk, std::vector<int>& ms0,
                             std::vector<int>& g0) {
              for (size_t j = 0; j < src.size(); ++j) {
                int mk = src[j].k >= 0 ? msk[src[j].k] : 0;
                int gk = src[j].k >= 0 ? gmk[src[j].k] : 1;
                if (src[j].i0 < 0) {
                  if (ms[j] != mk || gm[j] != gk) possible = false;
                  continue;
                }
                ms0[src[j].i0] = ms[j] - mk;
                g0[src[j].i0] = mult(gm[j], gk);
              }
            };
            split(to_ori_c, ms_i_c, gm_i_c, dk.msc, dk.gc, ms0c, g0c);
            split(to_ori_a, ms_i_a, gm_i_a, dk.msa, dk.ga, ms0a, g0a);
            if (!possible) continue;
            bool okms = true;  // check_ms
            for (size_t i = 0; i < i0c.size(); ++i)
              if (std::abs(ms0c[i]) > i0c[i].occ || ((i0c[i].occ - ms0c[i]) & 1)) okms = false;
            for (size_t i = 0; i < i0a.size(); ++i)
              if (std::abs(ms0a[i]) > i0a[i].occ || ((i0a[i].occ - ms0a[i]) & 1)) okms = false;
            if (!okms) continue;
            // merge_msgmdis: distribution of the reordered class
            auto merge = [](const std::vector<ReoSrc>& src, const std::vector<int>& ms0,
                            const std::vector<int>& g0, const std::vector<int>& msk,
                            const std::vector<int>& gk, std::vector<int>& ms,
                            std::vector<int>& gm) {
              ms.assign(src.size(), 0);
              gm.assign(src.size(), 1);
              for (size_t j = 0; j < src.size(); ++j) {
                if (src[j].i0 >= 0) ms[j] += ms0[src[j].i0], gm[j] = mult(gm[j], g0[src[j].i0]);
                if (src[j].k >= 0) ms[j] += msk[src[j].k], gm[j] = mult(gm[j], gk[src[j].k]);
              }
            };
            std::vector<int> msrc, gmrc, msra, gmra;
            merge(to_reo_c, ms0c, g0c, dk.msc, dk.gc, msrc, gmrc);
            merge(to_reo_a, ms0a, g0a, dk.msa, dk.ga, msra, gmra);
            auto ixkc = ixms(kc, dk.msc), ixka = ixms(ka, dk.msa);
            auto ix0c = ixms(i0c, ms0c), ix0a = ixms(i0a, ms0a);
            auto ixrc = ixms(Br.c, msrc), ixra = ixms(Br.a, msra);
            auto ixoc = ixms(Bo.c, ms_i_c), ixoa = ixms(Bo.a, ms_i_a);
            auto lkc = lens(cx, kc, ixkc, dk.gc), lka = lens(cx, ka, ixka, dk.ga);
            auto l0c = lens(cx, i0c, ix0c, g0c), l0a = lens(cx, i0a, ix0a, g0a);
            auto lrc = lens(cx, Br.c, ixrc, gmrc), lra = lens(cx, Br.a, ixra, gmra);
            auto loc = lens(cx, Bo.c, ixoc, gm_i_c), loa = lens(cx, Bo.a, ixoa, gm_i_a);
            if (anyzero(lkc) || anyzero(lka) || anyzero(l0c) || anyzero(l0a) || anyzero(lrc) ||
                anyzero(lra))
              continue;
            // set_op_ldim_c of both classes
            std::vector<int64_t> lso(loc), lsr(lrc), ldoc, ldoa, ldrc, ldra;
            lso.insert(lso.end(), loa.begin(), loa.end());
            lsr.insert(lsr.end(), lra.begin(), lra.end());
            ldims(Bo.c, Bo.a, lso, ldoc, ldoa);
            ldims(Br.c, Br.a, lsr, ldrc, ldra);
            // maps: creators (I0, K), annihilators (K, I0)
            auto maps = [&](const std::vector<ReoSrc>& src, bool cside, std::vector<CompMap>& out) {
              out.assign(src.size(), CompMap());
              for (size_t j = 0; j < src.size(); ++j) {
                const ReoSrc& s = src[j];
                if (s.i0 < 0 || s.k < 0) {
                  out[j].n1 = 1;
                  continue;
                }
                if (cside) {
                  out[j].m = &cx->strmap(i0c[s.i0].graph, kc[s.k].graph, ix0c[s.i0], ixkc[s.k],
                                         g0c[s.i0], dk.gc[s.k]);
                  out[j].n1 = l0c[s.i0];
                } else {
                  out[j].m = &cx->strmap(ka[s.k].graph, i0a[s.i0].graph, ixka[s.k], ix0a[s.i0],
                                         dk.ga[s.k], g0a[s.i0]);
                  out[j].n1 = lka[s.k];
                }
              }
            };
            std::vector<CompMap> m_ori_c, m_ori_a, m_reo_c, m_reo_a;
            maps(to_ori_c, true, m_ori_c);
            maps(to_ori_a, false, m_ori_a);
            maps(to_reo_c, true, m_reo_c);
            maps(to_reo_a, false, m_reo_a);
            // offset of the reordered distribution (idx_msgmdst2 -> d_gam_ms)
            int64_t did = msgmdid2(Br.c, ixrc, gmrc, Br.a, ixra, gmra, nsym);
            const auto& dl = Br.dis.at({idxms_op_a, gm_op_a});
            const int64_t idx00opreo = dl[find_dis(Br, idxms_op_a, gm_op_a, did)].off;
            // element loops: K(A), I0(A), K(C), I0(C)
            const int64_t nka = [&] { int64_t n = 1; for (auto x : lka) n *= x; return n; }();
            const int64_t n0a = [&] { int64_t n = 1; for (auto x : l0a) n *= x; return n; }();
            const int64_t nkc = [&] { int64_t n = 1; for (auto x : lkc) n *= x; return n; }();
            const int64_t n0c = [&] { int64_t n = 1; for (auto x : l0c) n *= x; return n; }();
            std::vector<int64_t> ska(ka.size()), s0a(i0a.size()), skc(kc.size()), s0c(i0c.size());
            // string index of each target component from its sources (1-based map
            // entry index: (str2-1)*n1 + str1)
            auto elem = [](const std::vector<ReoSrc>& src, const std::vector<CompMap>& mp,
                           const std::vector<int64_t>& ldim, bool cside,
                           const std::vector<int64_t>& s0, const std::vector<int64_t>& sk,
                           int64_t& idx, int& sgn) {
              for (size_t j = 0; j < src.size(); ++j) {
                int64_t i0s = src[j].i0 >= 0 ? s0[src[j].i0] : 0;
                int64_t ks = src[j].k >= 0 ? sk[src[j].k] : 0;
                int64_t el;
                if (!mp[j].m) {
                  el = (src[j].i0 >= 0 ? i0s : ks) + 1;
                } else {
                  int64_t i1 = cside ? i0s : ks, i2 = cside ? ks : i0s;
                  el = (*mp[j].m)[i2 * mp[j].n1 + i1];
                  if (el == 0) return false;
                  if (el < 0) sgn = -sgn, el = -el;
                }
                idx += (el - 1) * ldim[j];
              }
              return true;
            };
            for (int64_t ika = 0; ika < nka; ++ika) {
              decompose(ika, lka, ska.data());
              for (int64_t i0a_ = 0; i0a_ < n0a; ++i0a_) {
                decompose(i0a_, l0a, s0a.data());
                int64_t io_a = 0, ir_a = 0;
                int sgna = sign_reo;
                if (!elem(to_ori_a, m_ori_a, ldoa, false, s0a, ska, io_a, sgna)) continue;
                if (!elem(to_reo_a, m_reo_a, ldra, false, s0a, ska, ir_a, sgna)) continue;
                for (int64_t ikc = 0; ikc < nkc; ++ikc) {
                  decompose(ikc, lkc, skc.data());
                  for (int64_t i0c_ = 0; i0c_ < n0c; ++i0c_) {
                    decompose(i0c_, l0c, s0c.data());
                    int64_t io = io_a, ir = ir_a;
                    int sgnt = sgna;
                    if (!elem(to_ori_c, m_ori_c, ldoc, true, s0c, skc, io, sgnt)) continue;
                    if (!elem(to_reo_c, m_reo_c, ldrc, true, s0c, skc, ir, sgnt)) continue;
                    xreo[idx00opreo + ir] += fac * (double)sgnt * xo[io];
                  }
                }
              }
            }
          }
        }
      }
    }
  }
}

// reo_op_wmaps_c (contract/reo_op_wmaps_c.f): loop over Ms(A), IRREP(A) and
// the distributions of the original class, reo_blk_wmaps_c for each
void reorder(ora_ctx* cx, int lori, int ibori, const double* xori, int lreo, int ibreo,
             double* xreo, int nshift, const int* occ_shift, const int* from, const int* to,
             double fac, int sign_reo, bool update) {
  const List& Lo = cx->lists.at(lori - 1);
  const List& Lr = cx->lists.at(lreo - 1);
  const Op& Oo = cx->ops[Lo.op - 1];
  const Op& Or = cx->ops[Lr.op - 1];
  CHECK(Oo.nj == Or.nj, "reorder: njoined differs");
  CHECK(Lo.mst == Lr.mst && Lo.gamt == Lr.gamt, "reorder: inconsistent MS or symmetry");
  const int nj = Oo.nj, nsym = cx->oi.nsym;
  const ListBlock& Bo = Lo.blk.at(ibori - 1);
  const ListBlock& Br = Lr.blk.at(ibreo - 1);
  // I0 (occ_op0) per vertex
  std::vector<int> i0(8 * nj);
  for (int v = 0; v < nj; ++v)
    for (int q = 0; q < 8; ++q) {
      int a = Oo.occ[(ibori - 1) * nj + v][q], b = Or.occ[(ibreo - 1) * nj + v][q];
      for (int s = 0; s < nshift; ++s) {
        if (from[s] == v) a -= occ_shift[8 * s + q];
        if (to[s] == v) b -= occ_shift[8 * s + q];
      }
      CHECK(a >= 0 && a == b, "reorder: shifts do not connect the classes");
      i0[8 * v + q] = a;
    }
  std::vector<Comp> i0c, i0a, kc, ka;
  condense_n(cx, i0.data(), nj, i0c, i0a);
  condense_n(cx, occ_shift, nshift, kc, ka);
  auto to_ori_c = reo_map_info(Bo.c, i0c, kc, from), to_ori_a = reo_map_info(Bo.a, i0a, ka, from);
  auto to_reo_c = reo_map_info(Br.c, i0c, kc, to), to_reo_a = reo_map_info(Br.a, i0a, ka, to);
  if (!update)
    for (int64_t i = 0; i < Br.len_occ; ++i) xreo[Br.off_occ + i] = 0.0;
  int msc_max = 0, msa_max = 0;
  for (auto& x : Bo.c) msc_max += x.occ;
  for (auto& x : Bo.a) msa_max += x.occ;
  for (int msa = msa_max; msa >= -msa_max; msa -= 2) {
    int msc = msa + Lo.mst;
    if (std::abs(msc) > msc_max) continue;
    int idxms = msa2idxms4op(msa, Lo.mst, msa_max, msc_max);
    for (int gama = 1; gama <= nsym; ++gama) {
      int gamc = mult(gama, Lo.gamt);
      MsGamDist d;
      bool first = true;
      while (next_msgamdist2(first, d, occs(Bo.c), occs(Bo.a), msc, msa, gamc, gama, nsym)) {
        first = false;
        auto ixc = ixms(Bo.c, d.msc), ixa = ixms(Bo.a, d.msa);
        auto lc = lens(cx, Bo.c, ixc, d.gc), la = lens(cx, Bo.a, ixa, d.ga);
        if (anyzero(lc) || anyzero(la)) continue;
        int64_t did = msgmdid2(Bo.c, ixc, d.gc, Bo.a, ixa, d.ga, nsym);
        const auto& dl = Bo.dis.at({idxms, gama});
        const int64_t off = dl[find_dis(Bo, idxms, gama, did)].off;
        reo_blk(cx, fac, xreo, xori + off, sign_reo, msc, msa, gamc, gama, d.msc, d.msa, d.gc,
                d.ga, Bo, Br, kc, ka, i0c, i0a, to_ori_c, to_ori_a, to_reo_c, to_reo_a, idxms,
                nsym);
      }
    }
  }
}

// ---- partial trace (contract/trace_op.f, contract/trace_op_blk.f) ----

// trace_op without a reordered result: for every Ms/IRREP case of
// (Op(A), TrOp(A)), every distribution of TrOp and every diagonal
// distribution of the contracted strings J, trace_op_blk adds
// xfac*casign*signs*op(IC*J, IA*J) to trop(IC, IA)
void trace(ora_ctx* cx, int lop, int ibop, const double* xop, int ltr, int ibtr, double* xtr,
           const int* ocnt, double fac, bool update) {
  const List& Lo = cx->lists.at(lop - 1);
  const List& Lt = cx->lists.at(ltr - 1);
  CHECK(cx->ops[Lo.op - 1].nj == 1 && cx->ops[Lt.op - 1].nj == 1,
        "trace: single-vertex operators only");
  CHECK(Lo.gamt == Lt.gamt, "trace_op: inconsistent symmetries");
  const int nsym = cx->oi.nsym;
  const ListBlock& Bo = Lo.blk.at(ibop - 1);
  const ListBlock& Bt = Lt.blk.at(ibtr - 1);
  std::vector<Comp> cntc, cnta;
  condense(cx, ocnt, cntc, cnta);
  // map_info_c / map_info_a: op component <- (J component, TrOp component)
  auto info = [](const std::vector<Comp>& op, const std::vector<Comp>& j,
                 const std::vector<Comp>& t) {
    std::vector<std::pair<int, int>> r(op.size(), {-1, -1});
    for (size_t q = 0; q < op.size(); ++q) {
      for (size_t i = 0; i < j.size(); ++i)
        if (j[i].hpvx == op[q].hpvx) r[q].first = (int)i;
      for (size_t i = 0; i < t.size(); ++i)
        if (t[i].hpvx == op[q].hpvx) r[q].second = (int)i;
    }
    return r;
  };
  auto mi_c = info(Bo.c, cntc, Bt.c), mi_a = info(Bo.a, cnta, Bt.a);
  if (!update)
    for (int64_t i = 0; i < Bt.len_occ; ++i) xtr[Bt.off_occ + i] = 0.0;
  int na_op = 0, nc_op = 0, na_tr = 0, nc_tr = 0, na_cnt = 0;
  for (auto& x : Bo.a) na_op += x.occ;
  for (auto& x : Bo.c) nc_op += x.occ;
  for (auto& x : Bt.a) na_tr += x.occ;
  for (auto& x : Bt.c) nc_tr += x.occ;
  for (auto& x : cnta) na_cnt += x.occ;
  // ms_loop: (Ms(Op(A)), Ms(TrOp(A))) from the maxima down, first fastest
  for (int ms_tr_a = na_tr; ms_tr_a >= -na_tr; ms_tr_a -= 2) {
    for (int ms_op_a = na_op; ms_op_a >= -na_op; ms_op_a -= 2) {
      int ms_op_c = ms_op_a + Lo.mst, ms_tr_c = ms_tr_a + Lt.mst;
      if (std::abs(ms_op_c) > nc_op || std::abs(ms_tr_c) > nc_tr) continue;
      int msc_a = ms_op_a - ms_tr_a;
      CHECK(ms_op_c - ms_tr_c == msc_a, "trace_op: trap 1");
      if (std::abs(msc_a) > na_cnt) continue;
      for (int g_tr_a = 1; g_tr_a <= nsym; ++g_tr_a) {
        for (int g_op_a = 1; g_op_a <= nsym; ++g_op_a) {
          int g_tr_c = mult(g_tr_a, Lt.gamt);
          int g_c_a = mult(g_op_a, g_tr_a);
          int idxms_tr = msa2idxms4op(ms_tr_a, Lt.mst, na_tr, nc_tr);
          int idxms_op = msa2idxms4op(ms_op_a, Lo.mst, na_op, nc_op);
          MsGamDist dt;
          bool first3 = true;
          while (next_msgamdist2(first3, dt, occs(Bt.c), occs(Bt.a), ms_tr_c, ms_tr_a, g_tr_c,
                                 g_tr_a, nsym)) {
            first3 = false;
            auto ixtc = ixms(Bt.c, dt.msc), ixta = ixms(Bt.a, dt.msa);
            auto ltc = lens(cx, Bt.c, ixtc, dt.gc), lta = lens(cx, Bt.a, ixta, dt.ga);
            if (anyzero(ltc) || anyzero(lta)) continue;
            int64_t tdid = msgmdid2(Bt.c, ixtc, dt.gc, Bt.a, ixta, dt.ga, nsym);
            const int64_t idxtrop =
                Bt.dis.at({idxms_tr, g_tr_a})[find_dis(Bt, idxms_tr, g_tr_a, tdid)].off;
            std::vector<int64_t> lst(ltc), ldtc, ldta;
            lst.insert(lst.end(), lta.begin(), lta.end());
            ldims(Bt.c, Bt.a, lst, ldtc, ldta);
            // cac_loop: distributions of J, the same on both sides (next_msgamdist_diag)
            MsGamDist dj;
            bool first5 = true;
            while (next_msgamdist2(first5, dj, {}, occs(cnta), 0, msc_a, 1, g_c_a, nsym)) {
              first5 = false;
              auto ixj = ixms(cnta, dj.msa);
              auto lj = lens(cx, cnta, ixj, dj.ga);
              if (anyzero(lj)) continue;
              // merge_msgmdis: distribution of the operator
              auto merge = [](const std::vector<std::pair<int, int>>& mi,
                              const std::vector<int>& msj, const std::vector<int>& gj,
                              const std::vector<int>& mst, const std::vector<int>& gt,
                              std::vector<int>& ms, std::vector<int>& g) {
                ms.assign(mi.size(), 0);
                g.assign(mi.size(), 1);
                for (size_t q = 0; q < mi.size(); ++q) {
                  if (mi[q].first >= 0) ms[q] += msj[mi[q].first], g[q] = mult(g[q], gj[mi[q].first]);
                  if (mi[q].second >= 0) ms[q] += mst[mi[q].second], g[q] = mult(g[q], gt[mi[q].second]);
                }
              };
              std::vector<int> moc, goc, moa, goa;
              merge(mi_c, dj.msa, dj.ga, dt.msc, dt.gc, moc, goc);
              merge(mi_a, dj.msa, dj.ga, dt.msa, dt.ga, moa, goa);
              auto ixoc = ixms(Bo.c, moc), ixoa = ixms(Bo.a, moa);
              auto loc = lens(cx, Bo.c, ixoc, goc), loa = lens(cx, Bo.a, ixoa, goa);
              if (anyzero(loc) || anyzero(loa)) continue;
              int64_t odid = msgmdid2(Bo.c, ixoc, goc, Bo.a, ixoa, goa, nsym);
              const auto& odl = Bo.dis.at({idxms_op, g_op_a});
              const int64_t idxop = odl[find_dis(Bo, idxms_op, g_op_a, odid)].off;
              int64_t nop = 1;
              for (auto x : loc) nop *= x;
              for (auto x : loa) nop *= x;
              double xnrm = 0;
              for (int64_t i = 0; i < nop; ++i) xnrm += xop[idxop + i] * xop[idxop + i];
              if (xnrm < 1e-28) continue;
              std::vector<int64_t> lso(loc), ldoc, ldoa;
              lso.insert(lso.end(), loa.begin(), loa.end());
              ldims(Bo.c, Bo.a, lso, ldoc, ldoa);
              // maps (str1 = J, str2 = TrOp); trivial where one is absent
              auto maps = [&](const std::vector<std::pair<int, int>>& mi,
                              const std::vector<Comp>& tc, const std::vector<int>& ixt,
                              const std::vector<int>& gt, std::vector<const std::vector<int>*>& m,
                              std::vector<int64_t>& n1) {
                m.assign(mi.size(), nullptr);
                n1.assign(mi.size(), 1);
                for (size_t q = 0; q < mi.size(); ++q) {
                  int ij = mi[q].first, it = mi[q].second;
                  if (ij < 0 || it < 0) continue;
                  m[q] = &cx->strmap(cnta[ij].graph, tc[it].graph, ixj[ij], ixt[it], dj.ga[ij],
                                     gt[it]);
                  n1[q] = lj[ij];
                }
              };
              std::vector<const std::vector<int>*> mc, ma;
              std::vector<int64_t> n1c, n1a;
              maps(mi_c, Bt.c, ixtc, dt.gc, mc, n1c);
              maps(mi_a, Bt.a, ixta, dt.ga, ma, n1a);
              // trace_op_blk
              int64_t ntra = 1, ntrc = 1, nj = 1;
              for (auto x : lta) ntra *= x;
              for (auto x : ltc) ntrc *= x;
              for (auto x : lj) nj *= x;
              std::vector<int64_t> sta(lta.size()), stc(ltc.size()), sj(lj.size());
              auto side = [](const std::vector<std::pair<int, int>>& mi,
                             const std::vector<const std::vector<int>*>& m,
                             const std::vector<int64_t>& n1, const std::vector<int64_t>& ld,
                             const std::vector<int64_t>& str, const std::vector<int64_t>& sj,
                             int64_t& idx, int& sgn) {
                for (size_t q = 0; q < mi.size(); ++q) {
                  int64_t i1 = mi[q].first >= 0 ? sj[mi[q].first] : 0;
                  int64_t i2 = mi[q].second >= 0 ? str[mi[q].second] : 0;
                  int64_t el;
                  if (!m[q]) {
                    el = (mi[q].first >= 0 ? i1 : i2) + 1;
                  } else {
                    el = (*m[q])[i2 * n1[q] + i1];
                    if (el == 0) return false;
                    if (el < 0) sgn = -sgn, el = -el;
                  }
                  idx += (el - 1) * ld[q];
                }
                return true;
              };
              for (int64_t ia = 0; ia < ntra; ++ia) {
                decompose(ia, lta, sta.data());
                int64_t ta_off = 0;
                for (size_t q = 0; q < lta.size(); ++q) ta_off += sta[q] * ldta[q];
                for (int64_t ij = 0; ij < nj; ++ij) {
                  decompose(ij, lj, sj.data());
                  int64_t ida = 0;
                  int sgna = 1;
                  if (!side(mi_a, ma, n1a, ldoa, sta, sj, ida, sgna)) continue;
                  for (int64_t ic = 0; ic < ntrc; ++ic) {
                    decompose(ic, ltc, stc.data());
                    int64_t tc_off = 0;
                    for (size_t q = 0; q < ltc.size(); ++q) tc_off += stc[q] * ldtc[q];
                    int64_t idc = ida;
                    int sgnc = sgna;
                    if (!side(mi_c, mc, n1c, ldoc, stc, sj, idc, sgnc)) continue;
                    xtr[idxtrop + tc_off + ta_off] += fac * (double)sgnc * xop[idxop + idc];
                  }
                }
              }
            }
          }
        }
      }
    }
  }
}

void sym_ab_blk(ora_ctx* cx, List& L, int iblk, double* buf, double prefac, double relfac) {
  CHECK(L.mst == 0, "sym_ab_blk: mst must be 0");
  ListBlock& B = L.blk[iblk - 1];
  int nsym = cx->oi.nsym;
  int msc_max = sum_occ(B.c), msa_max = sum_occ(B.a);
  double relfac2 =
      ((((msc_max + msa_max) / 2 + 1) * (msc_max - msa_max) / 2) % 2 != 0) ? -relfac : relfac;
  std::vector<int> oc = occs(B.c), oa = occs(B.a);
  for (int msa = msa_max; msa >= 0; msa -= 2) {
    int msc = msa + L.mst;
    if (std::abs(msc) > msc_max) continue;
    int msa2 = -msa;
    int idxmsa = msa2idxms4op(msa, L.mst, msa_max, msc_max);
    int idxmsa2 = msa2idxms4op(msa2, L.mst, msa_max, msc_max);
    for (int gama = 1; gama <= nsym; ++gama) {
      int gamc = mult(gama, L.gamt);
      auto itl = B.gm_len.find({idxmsa, gama});
      if (itl == B.gm_len.end() || itl->second <= 0) continue;
      MsGamDist d;
      bool first = true;
      while (next_msgamdist2(first, d, oc, oa, msc, msa, gamc, gama, nsym)) {
        first = false;
        std::vector<int> msc2(d.msc), msa2v(d.msa);
        for (auto& v : msc2) v = -v;
        for (auto& v : msa2v) v = -v;
        int gsign = std_spsign_msdis(d.msc, oc) * std_spsign_msdis(d.msa, oa) *
                    std_spsign_msdis(msc2, oc) * std_spsign_msdis(msa2v, oa);
        auto ixc = ixms(B.c, d.msc), ixc2 = ixms(B.c, msc2);
        auto ixa = ixms(B.a, d.msa), ixa2 = ixms(B.a, msa2v);
        auto lc = lens(cx, B.c, ixc, d.gc), la = lens(cx, B.a, ixa, d.ga);
        int64_t lenc = prod(lc, 0, lc.size()), lena = prod(la, 0, la.size());
        if (lenc == 0 || lena == 0) continue;
        const auto& dl1 = B.dis.at({idxmsa, gama});
        const auto& dl2 = B.dis.at({idxmsa2, gama});
        int64_t id1 = 0, id2 = 0;
        if (dl1.size() > 1)
          id1 = find_dis(B, idxmsa, gama, msgmdid2(B.c, ixc, d.gc, B.a, ixa, d.ga, nsym));
        if (dl2.size() > 1)
          id2 = find_dis(B, idxmsa2, gama, msgmdid2(B.c, ixc2, d.gc, B.a, ixa2, d.ga, nsym));
        int64_t off1 = dl1[id1].off, off2 = dl2[id2].off;
        if (msa == 0 && id1 > id2) continue;
        std::vector<const int*> fc, fa;
        for (size_t i = 0; i < B.c.size(); ++i)
          fc.push_back(cx->flipmap(B.c[i].graph, ixc[i], d.gc[i]).data());
        for (size_t i = 0; i < B.a.size(); ++i)
          fa.push_back(cx->flipmap(B.a[i].graph, ixa[i], d.ga[i]).data());
        std::vector<int64_t> ldc, lda;
        ldims(B.c, B.a, cat(lc, la), ldc, lda);
        for (int64_t ia = 0; ia < lena; ++ia) {
          int64_t istr = ia, o1 = 0, o2 = 0;
          int asign = gsign;
          for (size_t k = 0; k < B.a.size(); ++k) {
            int64_t s = istr % la[k];
            istr /= la[k];
            int v = fa[k][s];
            asign *= (v < 0) ? -1 : 1;
            o1 += s * lda[k];
            o2 += (std::abs(v) - 1) * lda[k];
          }
          for (int64_t ic = 0; ic < lenc; ++ic) {
            int64_t jstr = ic, p1 = o1, p2 = o2;
            int csign = 1;
            for (size_t k = 0; k < B.c.size(); ++k) {
              int64_t s = jstr % lc[k];
              jstr /= lc[k];
              int v = fc[k][s];
              csign *= (v < 0) ? -1 : 1;
              p1 += s * ldc[k];
              p2 += (std::abs(v) - 1) * ldc[k];
            }
            int64_t idx1 = off1 + p1, idx2 = off2 + p2;
            if (idx1 > idx2) continue;
            double s = (double)(csign * asign) * relfac2;
            double value = prefac * (buf[idx1] + s * buf[idx2]);
            buf[idx1] = value;
            buf[idx2] = s * value;
          }
        }
      }
    }
  }
}

// ---- spin projection (contract/spin_prj_list.f, contract/spin_prj_blk.f) ----

// spin patterns of n electrons (set_spprjmap_cases,
// strings/set_spprjmap_cases.f:24-41): position i (0-based) carries bit
// n-1-i, set for beta.  The reference pattern alternates and ends in alpha
// (..., beta, alpha); it is number 0, the others are numbered 1.. in
// increasing bit order.
int spin_ref_bits(int n) {
  int b = 0;
  for (int i = 1; i < n; i += 2) b |= 1 << i;
  return b;
}
int spin_case_number(int n, int bits) {
  int ref = spin_ref_bits(n);
  if (bits == ref) return 0;
  return bits < ref ? bits + 1 : bits;
}
int spin_pattern_bits(const int* spn, int n) {
  int b = 0;
  for (int i = 0; i < n; ++i)
    if (spn[i] == -1) b |= 1 << (n - 1 - i);
  return b;
}

// set_spprjmap_kernel (strings/set_spprjmap_kernel.f:60-130): for every
// string of the block whose spins alternate from the right end (alpha
// last; paired orbitals pass), and every non-reference pattern k = 1..2^n-1,
// sign * (address of the string with the same orbitals and the spins of
// pattern k, + 1); 0 when the string is not of the reference pattern or a
// paired orbital would get two equal spins
const std::vector<int>& spprjmap(ora_ctx* cx, int g, int idxms, int gam) {
  std::array<int, 3> k{g, idxms, gam};
  auto it = cx->spprjmaps.find(k);
  if (it != cx->spprjmaps.end()) return it->second;
  const Graph& Gr = cx->G(g);
  const int nel = Gr.nel;
  CHECK(nel >= 2, "set_spprjmap_kernel: occ=1 uses the trivial map");
  const int ms = nel - (idxms - 1) * 2;
  CHECK(!(nel % 2 == 0 && ms != 0), "set_spprjmap_kernel: only ms=0 for even occ");
  CHECK(!(nel % 2 == 1 && ms != 1), "set_spprjmap_kernel: only ms=1/2 for odd occ");
  const int nmaps = (1 << nel) - 1;
  const StrBlock& b = Gr.blk[idxms - 1][gam - 1];
  std::vector<int> m;
  m.reserve(b.n() * nmaps);
  std::vector<int> pat(nel), sf(nel);
  // patterns in case order
  std::vector<std::vector<int>> cases(nmaps + 1, std::vector<int>(nel));
  for (int bits = 0; bits < (1 << nel); ++bits) {
    int c = spin_case_number(nel, bits);
    for (int i = 0; i < nel; ++i) cases[c][i] = ((bits >> (nel - 1 - i)) & 1) ? -1 : +1;
  }
  for (int64_t s = 0; s < b.n(); ++s) {
    const int* o = b.orb.data() + s * nel;
    const int* sp = b.spn.data() + s * nel;
    bool ref = true;
    for (int i = nel - 1, sg = +1; i >= 0; --i, sg = -sg)
      if (sp[i] != sg && sp[i] != 2) ref = false;
    if (!ref) {
      m.insert(m.end(), nmaps, 0);
      continue;
    }
    for (int c = 1; c <= nmaps; ++c) {
      sf = cases[c];
      bool ok = true;
      for (int i = 0; i < nel && ok; ++i) {
        if (sp[i] == 2 && sf[i] != 2) {
          CHECK(i + 1 < nel && sp[i + 1] == 2, "set_spprjmap_kernel: broken spin pair");
          if (sf[i] * sf[i + 1] != -1) ok = false;
          else sf[i] = sf[i + 1] = 2;
        }
      }
      if (!ok) {
        m.push_back(0);
        continue;
      }
      int msf = 0;
      for (int i = 0; i < nel; ++i) msf += sf[i] == 2 ? 0 : sf[i];
      const StrBlock& bf = Gr.blk[(nel - msf) / 2][gam - 1];
      auto f = bf.index.find(key_of(nel, o, sf.data()));
      CHECK(f != bf.index.end(), "set_spprjmap_kernel: flipped string not addressable");
      int sg = std_spsign(sp, nel) * std_spsign(sf.data(), nel);
      m.push_back(sg * (int)(f->second + 1));
    }
  }
  return cx->spprjmaps[k] = std::move(m);
}

// get_genealogical_coeff (baserout/get_genealogical_coeff.f:32-106) for
// s2 = 0, ms2 = 0: the coefficients of every singlet coupling path (paths of
// the branching diagram that never go below S = 0, in lexical order of the
// up/down sequence) for creators with spins c[0..n-1] followed by the
// annihilators in reverse order a[n-1..0]
std::vector<double> genealogical(const std::vector<int>& c, const std::vector<int>& a) {
  const int nc = (int)c.size(), na = (int)a.size(), nel = nc + na;
  const int nup = nel / 2;
  std::vector<int> br(nel, 1);
  std::fill(br.begin(), br.begin() + nup, 0);
  std::vector<double> out;
  do {
    bool valid = true;
    int down = 0;
    for (int i = 0; i < nel; ++i) {
      down += br[i];
      if (down > (i + 1) / 2) valid = false;
    }
    if (!valid) continue;
    int is2 = 0, ims2 = 0, iel = 0;
    double x = 1.0;
    auto step = [&](int ms_step, double sigma) {
      is2 += 1 - 2 * br[iel];
      ims2 += ms_step;
      if (br[iel] == 0)
        x *= std::sqrt(std::max(0.0, (is2 / 2.0 + sigma * ims2) / is2));
      else
        x = -2.0 * sigma * x * std::sqrt(std::max(0.0, (is2 / 2.0 + 1.0 - sigma * ims2) / (is2 + 2.0)));
      ++iel;
    };
    for (int i = 0; i < nc; ++i) step(c[i], 0.5 * c[i]);
    for (int i = na - 1; i >= 0; --i) {
      step(-a[i], -0.5 * a[i]);
      if (a[i] == -1) x = -x;
    }
    out.push_back(x);
  } while (std::next_permutation(br.begin(), br.end()));
  return out;
}

// get_target_dis (contract/spin_prj_blk.f:440-524): Ms distribution of the
// skeleton strings over the components -- 0 for even occupations; odd ones
// +1 (occupations above 1 first), then +1 from the left and -1 from the
// right in turn
std::vector<int> target_dis(const std::vector<int>& occ) {
  const int n = (int)occ.size();
  std::vector<int> t(n, 0);
  std::vector<bool> as(n, false);
  int nodd = 0, nlarge = 0;
  for (int i = 0; i < n; ++i) {
    if (occ[i] % 2 == 1) {
      ++nodd;
      if (occ[i] > 1) ++nlarge;
    } else {
      as[i] = true;
    }
  }
  const int k = std::min(nlarge, (nodd + 1) / 2);
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < n; ++i)
      if (!as[i] && occ[i] > 1) {
        t[i] = +1;
        as[i] = true;
        break;
      }
  int icnt = k;
  auto done = [&] { return std::all_of(as.begin(), as.end(), [](bool b) { return b; }); };
  while (!done()) {
    if (icnt <= 0) {
      for (int i = 0; i < n; ++i)
        if (!as[i]) {
          t[i] = +1, as[i] = true, ++icnt;
          break;
        }
    } else {
      for (int i = n - 1; i >= 0; --i)
        if (!as[i]) {
          t[i] = -1, as[i] = true, --icnt;
          break;
        }
    }
  }
  return t;
}

// one spin case of a class (set_spinprj_info.f set_case): spins of every
// creator / annihilator, Ms per component, pattern number per component
// relative to the skeleton's reference pattern (0 = the skeleton string
// itself), coupling coefficients
struct SpinCase {
  std::vector<int> sc, sa, msc, msa, mapc, mapa;
  std::vector<double> coeff;
};

// spin_prj_blk (contract/spin_prj_blk.f:97-425) with set_spinprj_info
// (contract/set_spinprj_info.f:55-305), s2 = 0, in place on buf (the whole
// list)
void spin_prj_blk(ora_ctx* cx, List& L, int iblk, double* buf) {
  CHECK(L.mst == 0, "spin_prj_blk: ms.ne.0 not yet considered");
  ListBlock& B = L.blk[iblk - 1];
  const int nsym = cx->oi.nsym;
  const int msc_max = sum_occ(B.c), msa_max = sum_occ(B.a);
  CHECK(msc_max == msa_max, "spin_prj_blk: only particle-conserving operators!");
  if (msc_max == 0) return;  // scalar: the singlet part is the element
  const int npart = msc_max;
  CHECK(npart <= 8, "spin_prj_blk: more than eight creators");
  const std::vector<int> oc = occs(B.c), oa = occs(B.a);
  const std::vector<int> tc = target_dis(oc), ta = target_dis(oa);
  // reference spins per particle: per component alternating, starting with
  // alpha for a +1 target and beta otherwise
  auto ref_spins = [](const std::vector<int>& occ, const std::vector<int>& tgt) {
    std::vector<int> s;
    for (size_t i = 0; i < occ.size(); ++i)
      for (int e = 0, sg = tgt[i] == 1 ? 1 : -1; e < occ[i]; ++e, sg = -sg) s.push_back(sg);
    return s;
  };
  const std::vector<int> setc = ref_spins(oc, tc), seta = ref_spins(oa, ta);
  auto map_type = [](const int* tgt, const int* ref, int n) {
    if (n == 1) return tgt[0] == ref[0] ? 0 : 1;
    CHECK(spin_pattern_bits(ref, n) == spin_ref_bits(n), "set_spinprj_info: error in map_type");
    return spin_case_number(n, spin_pattern_bits(tgt, n));
  };
  // spin cases: annihilator spins outer, creator spins inner, each running
  // from all alpha with the first particle fastest (next_dist2, inc -2);
  // equal Ms on both sides
  std::vector<SpinCase> cases;
  std::vector<int> omni;
  int pm[64][2];
  for (int i = 0; i < npart; ++i) pm[i][0] = -1, pm[i][1] = 1;
  std::vector<int> da(npart, 1), dc(npart, 1);
  for (bool more_a = true; more_a; more_a = next_dist(da.data(), npart, pm, -2)) {
    std::fill(dc.begin(), dc.end(), 1);
    for (bool more_c = true; more_c; more_c = next_dist(dc.data(), npart, pm, -2)) {
      int sc = 0, sa = 0;
      for (int i = 0; i < npart; ++i) sc += dc[i], sa += da[i];
      if (sc != sa) continue;
      SpinCase k;
      k.sc = dc;
      k.sa = da;
      for (int i = 0, o = 0; i < (int)oc.size(); o += oc[i], ++i) {
        int m = 0;
        for (int e = 0; e < oc[i]; ++e) m += dc[o + e];
        k.msc.push_back(m);
        k.mapc.push_back(map_type(dc.data() + o, setc.data() + o, oc[i]));
      }
      for (int i = 0, o = 0; i < (int)oa.size(); o += oa[i], ++i) {
        int m = 0;
        for (int e = 0; e < oa[i]; ++e) m += da[o + e];
        k.msa.push_back(m);
        k.mapa.push_back(map_type(da.data() + o, seta.data() + o, oa[i]));
      }
      k.coeff = genealogical(dc, da);
      // both strings alternate over all particles ("omnipresent" case)
      bool alt = npart > 1;
      for (int i = 0; i + 1 < npart; ++i)
        if (dc[i] * dc[i + 1] != -1 || da[i] * da[i + 1] != -1) alt = false;
      if (alt) omni.push_back((int)cases.size());
      cases.push_back(std::move(k));
    }
  }
  CHECK(omni.size() <= 4, "set_case: increase bound for nomni");
  const int ncase = (int)cases.size(), ncoup = (int)cases[0].coeff.size();

  const int msa = msa_max % 2, msc = msa;
  const int idxmsa = msa2idxms4op(msa, 0, msa_max, msc_max);
  const size_t ncc = B.c.size(), nca = B.a.size();
  for (int gama = 1; gama <= nsym; ++gama) {
    const int gamc = mult(gama, L.gamt);
    auto itl = B.gm_len.find({idxmsa, gama});
    if (itl == B.gm_len.end() || itl->second <= 0) continue;
    MsGamDist d;
    for (bool first = true; next_msgamdist2(first, d, oc, oa, msc, msa, gamc, gama, nsym);
         first = false) {
      if (d.msc != tc || d.msa != ta) continue;
      auto ixc = ixms(B.c, d.msc), ixa = ixms(B.a, d.msa);
      auto lc = lens(cx, B.c, ixc, d.gc), la = lens(cx, B.a, ixa, d.ga);
      const int64_t lenc = prod(lc, 0, lc.size()), lena = prod(la, 0, la.size());
      if (lenc == 0 || lena == 0) continue;
      // per case: offset of its distribution and its leading dimensions
      std::vector<int64_t> off(ncase, -1);
      std::vector<std::vector<int64_t>> ldc(ncase), lda(ncase);
      for (int k = 0; k < ncase; ++k) {
        const SpinCase& K = cases[k];
        auto kxc = ixms(B.c, K.msc), kxa = ixms(B.a, K.msa);
        int msak = 0;
        for (int m : K.msa) msak += m;
        const int kidx = msa2idxms4op(msak, 0, msa_max, msc_max);
        auto kl = cat(lens(cx, B.c, kxc, d.gc), lens(cx, B.a, kxa, d.ga));
        ldims(B.c, B.a, kl, ldc[k], lda[k]);
        auto dit = B.dis.find({kidx, gama});
        if (dit == B.dis.end()) continue;
        const int64_t did = msgmdid2(B.c, kxc, d.gc, B.a, kxa, d.ga, nsym);
        for (const DistRow& r : dit->second)
          if (r.did == did) off[k] = r.off;
      }
      // spin projection maps of the skeleton strings (get_spprjmap_blk,
      // strings/get_spprjmap_blk.f:48-95; one electron: the identity)
      std::vector<const int*> mc(ncc, nullptr), ma(nca, nullptr);
      std::vector<int> nmc(ncc), nma(nca);
      for (size_t i = 0; i < ncc; ++i) {
        nmc[i] = (1 << B.c[i].occ) - 1;
        if (B.c[i].occ > 1) mc[i] = spprjmap(cx, B.c[i].graph, ixc[i], d.gc[i]).data();
      }
      for (size_t i = 0; i < nca; ++i) {
        nma[i] = (1 << B.a[i].occ) - 1;
        if (B.a[i].occ > 1) ma[i] = spprjmap(cx, B.a[i].graph, ixa[i], d.ga[i]).data();
      }
      std::vector<int64_t> sc0(ncc), sa0(nca);
      std::vector<int64_t> idxel(ncase);
      std::vector<int> psign(ncase);
      std::vector<double> value(ncase), overl(ncoup);
      std::vector<char> okc(ncase), oka(ncase);
      std::vector<int64_t> pa(ncase), pc(ncase);
      for (int64_t ia = 0; ia < lena; ++ia) {
        decompose(ia, la, sa0.data());
        for (int k = 0; k < ncase; ++k) {
          oka[k] = 1;
          pa[k] = 0;
          for (size_t i = 0; i < nca; ++i) {
            int64_t s = sa0[i];
            const int mi = cases[k].mapa[i];
            if (mi != 0) {
              const int v = ma[i] ? ma[i][s * nma[i] + mi - 1] : (int)s + 1;
              if (v == 0) oka[k] = 0;
              s = std::abs(v) - 1;
            }
            pa[k] += s * lda[k][i];
          }
        }
        for (int64_t ic = 0; ic < lenc; ++ic) {
          decompose(ic, lc, sc0.data());
          for (int k = 0; k < ncase; ++k) {
            okc[k] = 1;
            pc[k] = 0;
            for (size_t i = 0; i < ncc; ++i) {
              int64_t s = sc0[i];
              const int mi = cases[k].mapc[i];
              if (mi != 0) {
                const int v = mc[i] ? mc[i][s * nmc[i] + mi - 1] : (int)s + 1;
                if (v == 0) okc[k] = 0;
                s = std::abs(v) - 1;
              }
              pc[k] += s * ldc[k][i];
            }
          }
          for (int k = 0; k < ncase; ++k) {
            idxel[k] = -1;
            value[k] = 0.0;
            if (!okc[k] || !oka[k] || off[k] < 0) continue;
            idxel[k] = off[k] + pc[k] + pa[k];
            // the element appears more than once (paired orbitals): the
            // parity of (count - 1) in bits (popcnt_par)
            int cnt = 0;
            for (int j = 0; j <= k; ++j) cnt += idxel[j] == idxel[k];
            psign[k] = (__builtin_popcount(cnt - 1) & 1) ? -1 : 1;
            value[k] = buf[idxel[k]] * psign[k];
          }
          bool skip = false;
          for (int k : omni) skip = skip || idxel[k] < 0;
          if (skip) continue;
          for (int q = 0; q < ncoup; ++q) {
            double s = 0.0;
            for (int k = 0; k < ncase; ++k) s += cases[k].coeff[q] * value[k];
            overl[q] = s;
          }
          for (int k = 0; k < ncase; ++k) {
            double s = 0.0;
            for (int q = 0; q < ncoup; ++q) s += cases[k].coeff[q] * overl[q];
            value[k] = s;
          }
          for (int k = 0; k < ncase; ++k)
            if (idxel[k] >= 0) buf[idxel[k]] = value[k] * psign[k];
        }
      }
    }
  }
}

void spin_prj_list(ora_ctx* cx, List& L, double* x, double* xnorm2) {
  for (size_t ib = 0; ib < L.blk.size(); ++ib) {
    const ListBlock& B = L.blk[ib];
    if (xnorm2) xnorm2[ib] = 0.0;
    if (B.len_occ == 0) continue;
    spin_prj_blk(cx, L, (int)ib + 1, x);
    if (xnorm2) xnorm2[ib] = ddot_blk(x + B.off_occ, B.len_occ);
  }
}

// add_opblk_transp (contract/add_opblk_transp.f:195-321): OUT(IC,IA) +=
// fac * IN(IA,IC) for a class of the output whose adjoint is the input class
// (op_in^tra_in = op_out^tra_out).  Loops over the output's Ms(A), IRREP(A)
// and distributions; the input distribution is the one with C and A strings
// exchanged, looked up at (Ms(C), IRREP(C)) of the output (idx_msgmdst2
// with C and A swapped); the element offsets inside the two distributions
// use set_op_ldim_c over the output's components with tra_in and tra_out.
// Single-vertex operators.
void add_opblk_transp(ora_ctx* cx, List& Li, int iblk_in, const double* xin, List& Lo,
                      int iblk_out, double* xout, double fac, bool tra_in, bool tra_out) {
  CHECK(cx->ops[Li.op - 1].nj == 1 && cx->ops[Lo.op - 1].nj == 1,
        "add_opblk_transp: single-vertex operators only");
  ListBlock& Bo = Lo.blk.at(iblk_out - 1);
  ListBlock& Bi = Li.blk.at(iblk_in - 1);
  auto same = [](const std::vector<Comp>& x, const std::vector<Comp>& y) {
    if (x.size() != y.size()) return false;
    for (size_t i = 0; i < x.size(); ++i)
      if (x[i].occ != y[i].occ || x[i].hpvx != y[i].hpvx) return false;
    return true;
  };
  CHECK(same(Bi.c, Bo.a) && same(Bi.a, Bo.c),
        "add_opblk_transp: input and output list do not have compatible operators");
  int nsym = cx->oi.nsym;
  int msc_max = sum_occ(Bo.c), msa_max = sum_occ(Bo.a);
  std::vector<int> oc = occs(Bo.c), oa = occs(Bo.a);
  int idxmsa = 0;
  for (int msa = msa_max; msa >= -msa_max; msa -= 2) {
    int msc = msa + Lo.mst;
    if (std::abs(msc) > msc_max) continue;
    ++idxmsa;
    int idxmsc = (msc_max - msc) / 2 + 1;
    for (int gama = 1; gama <= nsym; ++gama) {
      int gamc = mult(gama, Lo.gamt);
      auto itl = Bo.gm_len.find({idxmsa, gama});
      if (itl == Bo.gm_len.end() || itl->second <= 0) continue;
      const auto& dlo = Bo.dis.at({idxmsa, gama});
      MsGamDist d;
      bool first = true;
      size_t idxdis = 0;
      while (next_msgamdist2(first, d, oc, oa, msc, msa, gamc, gama, nsym)) {
        first = false;
        auto ixc = ixms(Bo.c, d.msc), ixa = ixms(Bo.a, d.msa);
        auto lc = lens(cx, Bo.c, ixc, d.gc), la = lens(cx, Bo.a, ixa, d.ga);
        int64_t lenc = prod(lc, 0, lc.size()), lena = prod(la, 0, la.size());
        if (lenc == 0 || lena == 0) continue;
        const int64_t off_out = dlo.at(idxdis++).off;
        int64_t id_in = 0;
        const auto& dli = Bi.dis.at({idxmsc, gamc});
        if (dli.size() > 1)
          id_in = find_dis(Bi, idxmsc, gamc, msgmdid2(Bi.c, ixa, d.ga, Bi.a, ixc, d.gc, nsym));
        const int64_t off_in = dli[id_in].off;
        std::vector<int64_t> ldic, ldia, ldoc, ldoa;
        ldims(Bo.c, Bo.a, cat(lc, la), ldic, ldia, tra_in);
        ldims(Bo.c, Bo.a, cat(lc, la), ldoc, ldoa, tra_out);
        for (int64_t ic = 0; ic < lenc; ++ic) {
          int64_t r = ic, pi = 0, po = 0;
          for (size_t k = 0; k < Bo.c.size(); ++k) {
            int64_t sidx = r % lc[k];
            r /= lc[k];
            pi += sidx * ldic[k];
            po += sidx * ldoc[k];
          }
          for (int64_t ia = 0; ia < lena; ++ia) {
            int64_t q = ia, qi = pi, qo = po;
            for (size_t k = 0; k < Bo.a.size(); ++k) {
              int64_t sidx = q % la[k];
              q /= la[k];
              qi += sidx * ldia[k];
              qo += sidx * ldoa[k];
            }
            xout[off_out + qo] += fac * xin[off_in + qi];
          }
        }
      }
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// C API
// ---------------------------------------------------------------------------
#define GUARD_BEGIN try {
#define GUARD_END(ret)            \
  }                               \
  catch (const std::exception& e) { \
    g_err = e.what();             \
    return ret;                   \
  }

extern "C" {

const char* ora_last_error(void) { return g_err.c_str(); }

ora_ctx* ora_create(int64_t nsym, const int64_t* norb) {
  GUARD_BEGIN
  CHECK(nsym == 1 || nsym == 2 || nsym == 4 || nsym == 8, "nsym must be 1,2,4,8");
  auto* c = new ora_ctx();
  c->oi.nsym = (int)nsym;
  for (int t = 0; t < 4; ++t)
    for (int g = 0; g < 8; ++g) c->oi.norb[t][g] = (g < nsym) ? (int)norb[t * 8 + g] : 0;
  c->oi.init();
  return c;
  GUARD_END(nullptr)
}

void ora_destroy(ora_ctx* c) { delete c; }

int64_t ora_graph_nstr(ora_ctx* c, int64_t type, int64_t nel, int64_t idxms, int64_t gam) {
  GUARD_BEGIN
  int g = c->graph((int)type, (int)nel);
  return c->G(g).len((int)idxms, (int)gam);
  GUARD_END(-1)
}

int64_t ora_graph_strings(ora_ctx* c, int64_t type, int64_t nel, int64_t idxms, int64_t gam,
                          int64_t* orb, int64_t* spn) {
  GUARD_BEGIN
  int g = c->graph((int)type, (int)nel);
  const StrBlock& b = c->G(g).blk[idxms - 1][gam - 1];
  for (size_t i = 0; i < b.spn.size(); ++i) {
    orb[i] = b.orb[i];
    spn[i] = b.spn[i];
  }
  return b.n();
  GUARD_END(-1)
}

int64_t ora_strmap_block(ora_ctx* c, int64_t type, int64_t nel1, int64_t nel2, int64_t idxms1,
                         int64_t idxms2, int64_t gam1, int64_t gam2, int64_t* map) {
  GUARD_BEGIN
  int g1 = c->graph((int)type, (int)nel1), g2 = c->graph((int)type, (int)nel2);
  const auto& m = c->strmap(g1, g2, (int)idxms1, (int)idxms2, (int)gam1, (int)gam2);
  for (size_t i = 0; i < m.size(); ++i) map[i] = m[i];
  return (int64_t)m.size();
  GUARD_END(-1)
}

int64_t ora_define_op(ora_ctx* c, const int64_t* occ, int64_t nblk) {
  return ora_define_op_joined(c, occ, 1, nblk);
}

int64_t ora_define_op_joined(ora_ctx* c, const int64_t* occ, int64_t nj, int64_t nblk) {
  GUARD_BEGIN
  CHECK(nj >= 1 && nj <= 8, "njoined must be 1..8");
  Op op;
  op.nj = (int)nj;
  for (int64_t b = 0; b < nblk * nj; ++b) {
    std::array<int, 8> o;
    for (int k = 0; k < 8; ++k) o[k] = (int)occ[b * 8 + k];
    op.occ.push_back(o);
  }
  c->ops.push_back(op);
  return (int64_t)c->ops.size();
  GUARD_END(-1)
}

int64_t ora_define_list(ora_ctx* c, int64_t op, int64_t gamt, int64_t mst, int64_t absym,
                        int64_t* len) {
  GUARD_BEGIN
  CHECK(op >= 1 && op <= (int64_t)c->ops.size(), "bad operator id");
  List L;
  L.op = (int)op;
  L.gamt = (int)gamt;
  L.mst = (int)mst;
  L.absym = (int)absym;
  set_op_dim2(c, L);
  *len = L.len;
  c->lists.push_back(std::move(L));
  return (int64_t)c->lists.size();
  GUARD_END(-1)
}

int ora_list_block(ora_ctx* c, int64_t list, int64_t iblk, int64_t* off, int64_t* len) {
  GUARD_BEGIN
  const ListBlock& B = c->lists.at(list - 1).blk.at(iblk - 1);
  *off = B.off_occ;
  *len = B.len_occ;
  return 0;
  GUARD_END(-1)
}

int64_t ora_list_dists(ora_ctx* c, int64_t list, int64_t* rows, int64_t maxrows) {
  GUARD_BEGIN
  const List& L = c->lists.at(list - 1);
  int64_t n = 0;
  for (size_t ib = 0; ib < L.blk.size(); ++ib)
    for (auto& kv : L.blk[ib].dis)
      for (size_t d = 0; d < kv.second.size(); ++d) {
        if (n < maxrows) {
          int64_t* r = rows + 8 * n;
          r[0] = (int64_t)ib + 1;
          r[1] = kv.first.first;
          r[2] = kv.first.second;
          r[3] = (int64_t)d + 1;
          r[4] = kv.second[d].off;
          r[5] = kv.second[d].len;
          r[6] = kv.second[d].ld;
          r[7] = kv.second[d].did;
        }
        ++n;
      }
  return n;
  GUARD_END(-1)
}

int ora_contract(ora_ctx* c, int64_t route, int64_t list1, int64_t iblk1, const double* x1,
                 int64_t list2, int64_t iblk2, const double* x2, int64_t list12, int64_t iblk12,
                 double* x12, const int64_t* occ_ex1, const int64_t* occ_ex2,
                 const int64_t* occ_cnt, double fact, int64_t update, int64_t use_tr,
                 int64_t str_block, int64_t cnt_block, double* xret, double* stats) {
  GUARD_BEGIN
  CHECK(route == 2 || route == 3, "route must be 2 or 3");
  int e1[8], e2[8], cn[8];
  for (int k = 0; k < 8; ++k) {
    e1[k] = (int)occ_ex1[k];
    e2[k] = (int)occ_ex2[k];
    cn[k] = (int)occ_cnt[k];
  }
  Stats st;
  contract(c, (int)route, (int)list1, (int)iblk1, x1, (int)list2, (int)iblk2, x2, (int)list12,
           (int)iblk12, x12, e1, e2, cn, fact, update != 0, use_tr != 0,
           str_block > 0 ? str_block : 200, cnt_block, xret, &st);
  if (stats)
    for (int k = 0; k < 8; ++k) stats[k] += st.v[k];
  return 0;
  GUARD_END(-1)
}

int ora_contract_t(ora_ctx* c, int64_t route, int64_t list1, int64_t iblk1, const double* x1,
                   int64_t list2, int64_t iblk2, const double* x2, int64_t list12,
                   int64_t iblk12, double* x12, const int64_t* occ_ex1, const int64_t* occ_ex2,
                   const int64_t* occ_cnt, double fact, int64_t update, int64_t use_tr,
                   int64_t tra_op1, int64_t tra_op2, int64_t tra_res, double* xret) {
  GUARD_BEGIN
  CHECK(route == 2 || route == 3, "route must be 2 or 3");
  int e1[8], e2[8], cn[8];
  for (int k = 0; k < 8; ++k) {
    e1[k] = (int)occ_ex1[k];
    e2[k] = (int)occ_ex2[k];
    cn[k] = (int)occ_cnt[k];
  }
  const bool tra[3] = {tra_op1 != 0, tra_op2 != 0, tra_res != 0};
  Stats st;
  contract(c, (int)route, (int)list1, (int)iblk1, x1, (int)list2, (int)iblk2, x2, (int)list12,
           (int)iblk12, x12, e1, e2, cn, fact, update != 0, use_tr != 0, 200, -1, xret, &st,
           tra);
  return 0;
  GUARD_END(-1)
}

int ora_reorder(ora_ctx* c, int64_t list_ori, int64_t iblk_ori, const double* xori,
                int64_t list_reo, int64_t iblk_reo, double* xreo, int64_t nshift,
                const int64_t* occ_shift, const int64_t* from_vtx, const int64_t* to_vtx,
                double fac, int64_t sign_reo, int64_t update) {
  GUARD_BEGIN
  CHECK(nshift >= 0 && nshift <= 4, "reorder: nshift must be 0..4");
  std::vector<int> sh(8 * nshift), fr(nshift), to(nshift);
  for (int64_t s = 0; s < nshift; ++s) {
    for (int q = 0; q < 8; ++q) sh[8 * s + q] = (int)occ_shift[8 * s + q];
    fr[s] = (int)from_vtx[s] - 1;
    to[s] = (int)to_vtx[s] - 1;
  }
  reorder(c, (int)list_ori, (int)iblk_ori, xori, (int)list_reo, (int)iblk_reo, xreo,
          (int)nshift, sh.data(), fr.data(), to.data(), fac, (int)sign_reo, update != 0);
  return 0;
  GUARD_END(-1)
}

int ora_trace(ora_ctx* c, int64_t list_op, int64_t iblk_op, const double* xop, int64_t list_res,
              int64_t iblk_res, double* xres, const int64_t* occ_cnt, double fac,
              int64_t update) {
  GUARD_BEGIN
  int cn[8];
  for (int k = 0; k < 8; ++k) cn[k] = (int)occ_cnt[k];
  trace(c, (int)list_op, (int)iblk_op, xop, (int)list_res, (int)iblk_res, xres, cn, fac,
        update != 0);
  return 0;
  GUARD_END(-1)
}

int ora_sym_ab_blk(ora_ctx* c, int64_t list, int64_t iblk, double* x, double prefac,
                   double relfac) {
  GUARD_BEGIN
  sym_ab_blk(c, c->lists.at(list - 1), (int)iblk, x, prefac, relfac);
  return 0;
  GUARD_END(-1)
}

int ora_spin_prj_list(ora_ctx* c, int64_t list, int64_t s2, double* x, double* xnorm2) {
  GUARD_BEGIN
  CHECK(s2 == 0, "spin_prj_list: not a singlet case");
  spin_prj_list(c, c->lists.at(list - 1), x, xnorm2);
  return 0;
  GUARD_END(-1)
}

int ora_add_opblk(double* xnorm2, int64_t type, double fac, const double* xin, double* xout,
                  int64_t len, int64_t reset) {
  if (reset) std::fill(xout, xout + len, 0.0);
  for (int64_t i = 0; i < len; ++i) xout[i] += fac * xin[i];
  if (type == 1) {
    double s = 0;
    for (int64_t i = 0; i < len; ++i) s += xout[i] * xout[i];
    *xnorm2 = s;
  } else {
    *xnorm2 = len > 0 ? xout[0] : 0.0;
  }
  return 0;
}

int ora_add_opblk_transp(ora_ctx* c, double* xnorm2, int64_t type, double fac, int64_t list_in,
                         int64_t iblk_in, const double* xin, int64_t list_out, int64_t iblk_out,
                         double* xout, int64_t tra_in, int64_t tra_out, int64_t reset) {
  GUARD_BEGIN
  CHECK((tra_in != 0) != (tra_out != 0), "add_opblk_transp: exactly one side is transposed");
  List& Lo = c->lists.at(list_out - 1);
  const ListBlock& Bo = Lo.blk.at(iblk_out - 1);
  if (reset) std::fill(xout + Bo.off_occ, xout + Bo.off_occ + Bo.len_occ, 0.0);
  add_opblk_transp(c, c->lists.at(list_in - 1), (int)iblk_in, xin, Lo, (int)iblk_out, xout, fac,
                   tra_in != 0, tra_out != 0);
  if (type == 1) {
    double sq = 0;
    for (int64_t i = 0; i < Bo.len_occ; ++i) sq += xout[Bo.off_occ + i] * xout[Bo.off_occ + i];
    *xnorm2 = sq;
  } else {
    *xnorm2 = Bo.len_occ > 0 ? xout[Bo.off_occ] : 0.0;
  }
  return 0;
  GUARD_END(-1)
}

int ora_set_blas(const char* path, int64_t nthreads) {
  GUARD_BEGIN
  void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  CHECK(h, std::string("cannot load BLAS: ") + dlerror());
  g_dgemm = (dgemm_t)dlsym(h, "scipy_dgemm_64_");
  if (!g_dgemm) g_dgemm = (dgemm_t)dlsym(h, "dgemm_64_");
  CHECK(g_dgemm, "no ILP64 dgemm in BLAS library");
  typedef void (*nt_t)(int);
  nt_t nt = (nt_t)dlsym(h, "scipy_openblas_set_num_threads64_");
  if (nt && nthreads > 0) nt((int)nthreads);
  return 0;
  GUARD_END(-1)
}

void ora_set_shard(int64_t rank, int64_t nranks) {
  g_shard_n = nranks > 0 ? nranks : 1;
  g_shard_rank = (rank >= 0 && rank < g_shard_n) ? rank : 0;
  g_shard_item = 0;
}

void ora_sampling(int64_t stride) {
  g_stride = stride > 0 ? stride : 1;
  g_batch = g_batches_total = g_batches_done = 0;
  g_short_total = g_short_done = 0;
  g_t_always = g_t_sampled = 0;
}

void ora_sampling_report(double* out4) {
  out4[0] = g_t_always;
  out4[1] = g_t_sampled;
  out4[2] = (double)g_batches_total;
  out4[3] = (double)g_batches_done;
  out4[4] = (double)g_short_total;
  out4[5] = (double)g_short_done;
}

void ora_diavc(double* out, const double* in, double fac, const double* diag, double shift,
               int64_t n) {
  const double thresh = 1e-10;
  for (int64_t i = 0; i < n; ++i) {
    double d = diag[i] + shift;
    if (std::fabs(d) <= thresh) d = thresh;
    out[i] = fac * in[i] / d;
  }
}

}  // extern "C"

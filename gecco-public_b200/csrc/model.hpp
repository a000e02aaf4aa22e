// Host-side model of the reference's string spaces and ME-list layout.
//
//  * Graph: all strings of one (hpvx type, electron count), addressed
//    lexically by arc weights as idx4sg does (strings/idx4sg.f:2-82,
//    strings/idx4sg_sb.f); string order = next_string order
//    (strings/next_string.f), i.e. reverse-lexical over orbitals with the
//    per-orbital code order empty < alpha < beta < pair.
//  * ListLayout: offsets of every (occupation class, Ms(A), IRREP(A),
//    Ms/IRREP distribution) block of an ME list (operators/set_op_dim2.f).
//
// Scope: operators with one or more vertices (njoined >= 1, condensed as
// condense_occ does), one GAS per H/P/V/X type, no diagonal or vertex-Ms
// restrictions; frozen and deleted orbitals are not part of the string
// spaces.
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace gccu {

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};
#define GCCU_REQUIRE(c, msg)                 \
  do {                                       \
    if (!(c)) throw ::gccu::Error(msg);      \
  } while (0)

constexpr int kNType = 4;                  // H, P, V, X
constexpr int kHpvxSeq[4] = {3, 1, 2, 0};  // X,P,V,H (include/hpvxseq.h:3)
constexpr int kMaxComp = 8;                // components per composite string space
constexpr int kMaxNel = 8;                 // electrons per string

inline int irrep_mult(int a, int b) { return ((a - 1) ^ (b - 1)) + 1; }  // include/multd2h.h
inline int ms_index(int nel, int ms) { return ((nel - ms) >> 1) + 1; }     // Ms -> idxms

struct OrbSpace {
  int nsym = 1;
  int norb[kNType][8] = {};
  std::vector<int> irrep[kNType];  // 1-based irrep of orbital k (0-based) of a type
  void finalize();
  int n(int t) const { return (int)irrep[t].size(); }
};

// one string: nel entries, orbital (0-based) and spin code (+1, -1, 2)
struct Graph {
  int id = 0, type = 0, nel = 0, norb = 0, nsym = 1;
  std::vector<int> irrep;  // 0-based irrep per orbital
  // number of strings per block [(idxms-1)*nsym + gam-1]
  std::vector<int64_t> len;
  // arc weights W[((k*3 + c-1)*(nel+1) + n)*(2*nel+1) + m+nel)*nsym + g]
  std::vector<int64_t> W;
  // strings of each block in address order, packed (orb<<2 | code) with
  // code 1 = alpha, 2 = beta, 3 = member of a doubly occupied orbital;
  // filled on demand
  std::map<int, std::vector<int32_t>> tables;

  void build(const OrbSpace& os, int type, int nel);
  int64_t nstr(int idxms, int gam) const {
    if (idxms < 1 || idxms > nel + 1 || gam < 1 || gam > nsym) return 0;
    return len[(idxms - 1) * nsym + gam - 1];
  }
  int64_t weight(int k, int code, int n, int m, int g) const {
    return W[((((size_t)k * 3 + code - 1) * (nel + 1) + n) * (2 * nel + 1) + m + nel) * nsym + g];
  }
  // address of a canonical string (orb 0-based, spn +1/-1/2) within its block
  int64_t address(const int* orb, const int* spn) const;
  const std::vector<int32_t>& table(int idxms, int gam);
};

// condensed component (cinfo row): occupation, graph id, hpvx type
struct Comp {
  int occ = 0, graph = 0, hpvx = 0;
  int vtx = 0;  // vertex of a joined operator the component belongs to
};
using Occ = std::array<int, 8>;  // C[H,P,V,X], A[H,P,V,X]

struct Dist {
  int64_t off = 0, len = 0, ld = 0, did = 0;
  std::vector<int> msc, msa, gc, ga;  // Ms / IRREP per component
};

struct LayoutBlock {
  std::vector<Occ> vtx;  // occupation per vertex
  Occ occ{};             // summed over the vertices
  std::vector<Comp> c, a;
  int64_t off = 0, len = 0;
  // per (idxmsa, gama): offset, length and distributions
  std::map<std::pair<int, int>, int64_t> gm_off, gm_len;
  std::map<std::pair<int, int>, std::vector<Dist>> dis;
  int64_t gmlen(int idxms, int gam) const {
    auto it = gm_len.find({idxms, gam});
    return it == gm_len.end() ? 0 : it->second;
  }
};

struct Operator {
  int nj = 1;             // vertices per occupation class (njoined)
  std::vector<Occ> occ;   // nblk * nj entries, the vertices of a class consecutive
  int64_t nblk() const { return (int64_t)occ.size() / nj; }
};

struct ListLayout {
  int op = 0, gamt = 1, mst = 0, absym = 0;
  int64_t len = 0;
  std::vector<LayoutBlock> blk;
};

class Model {
 public:
  OrbSpace os;
  std::vector<std::unique_ptr<Graph>> graphs;  // id = index+1
  std::map<std::pair<int, int>, int> graph_id;
  std::vector<Operator> ops;

  int graph(int type, int nel);
  Graph& G(int id) { return *graphs.at(id - 1); }
  void condense(const Occ& o, std::vector<Comp>& c, std::vector<Comp>& a) {
    condense(&o, 1, c, a);
  }
  void condense(const Occ* vtx, int nj, std::vector<Comp>& c, std::vector<Comp>& a);
  void layout(ListLayout& L);
};

// --- Ms / IRREP distributions over components (operators/next_msgamdist2.f)
struct MsGam {
  std::vector<int> msc, msa, gc, ga;
};
bool next_msgam(bool first, MsGam& d, const std::vector<int>& occc, const std::vector<int>& occa,
                int msc, int msa, int gamc, int gama, int nsym);
int64_t dist_id(const std::vector<Comp>& c, const std::vector<int>& ixc, const std::vector<int>& gc,
                const std::vector<Comp>& a, const std::vector<int>& ixa, const std::vector<int>& ga,
                int nsym);
int msa_to_idxms(int msa, int mst, int occ_a, int occ_c);
std::vector<int> comp_occs(const std::vector<Comp>& c);

}  // namespace gccu

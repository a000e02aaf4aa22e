// Engine state behind the C ABI (include/gccu.h): the orbital model, ME
// lists resident in device memory, the device string-map store, cached
// contraction plans and their device work lists, CUDA-graph capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <functional>
#include <atomic>
#include <thread>
#include <cstring>
#include <map>
#include <set>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/gccu.h"
#include "kernels.hpp"
#include "model.hpp"
#include "planner.hpp"

namespace gccu {
namespace {

thread_local std::string g_error;

Occ to_occ(const int64_t* o) {
  Occ r{};
  for (int k = 0; k < 8; ++k) {
    GCCU_REQUIRE(o[k] >= 0 && o[k] <= kMaxNel, "occupation out of range");
    r[k] = (int)o[k];
  }
  return r;
}

#define CUDA_OK(x)                                                                   \
  do {                                                                               \
    cudaError_t e_ = (x);                                                            \
    if (e_ != cudaSuccess)                                                           \
      throw ::gccu::Error(std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #x); \
  } while (0)

struct DevList {
  ListLayout L;
  double* d = nullptr;
  // frozen: the host has declared the data constant (gccu_freeze_list);
  // plans may cache panels derived from it; epoch counts unfreezes
  bool frozen = false;
  int64_t epoch = 0;
  // an intermediate of a formula (gccu_register_intermediate): memory is a
  // range of its formula's arena, set when the formula is defined
  bool intermediate = false;
  int64_t formula = 0, arena_off = -1;
};

// a defined formula (gccu_formula_define): its items and the arena holding
// its intermediates
struct FormulaPlan {
  std::vector<gccu_formula_item> items;
  double* arena = nullptr;
  int64_t arena_bytes = 0, sum_bytes = 0, ntargets = 0;
};

struct DevGraph {
  int64_t* W = nullptr;
  int8_t* irrep = nullptr;
  std::map<int, int32_t*> tables;  // (idxms-1)*nsym+gam-1 -> device string table
};

// Tile shapes and routing of a contraction's block contractions: the fixed
// rule (candidate 0) or one of the alternatives the autotuner times
struct TilePolicy {
  int medium_max = kGemmMediumN;  // at most this many columns (rows): the 128 x 32 FP64 tile
  int64_t tc_min_k = kTcMinK;     // shortest contraction sent to the tensor cores
  bool tc_thin = false;           // 9..medium_max columns go to the tensor cores too
  bool ksplit = true;             // split contractions over CTAs when a launch has few tiles
  bool thin = false;              // <= 32 columns (results without map lookups): k_thin
};

// an autotuned alternative must take at most this fraction of the fixed
// rule's time to be chosen
constexpr double kTuneMargin = 0.97;

// candidates per precision mode; candidate 0 is the fixed rule
inline std::vector<TilePolicy> tile_policies(int precision) {
  std::vector<TilePolicy> v(1);
  TilePolicy thin;
  thin.thin = true;
  v.push_back(thin);
  if (precision == 0) {
    TilePolicy a;
    a.medium_max = 64;
    v.push_back(a);
    TilePolicy b;
    b.ksplit = false;
    v.push_back(b);
  } else {
    TilePolicy a;
    a.tc_min_k = 128;
    v.push_back(a);
    TilePolicy b;
    b.tc_min_k = 512;
    v.push_back(b);
    TilePolicy c;
    c.tc_thin = true;
    v.push_back(c);
    TilePolicy d;
    d.tc_thin = true;
    d.tc_min_k = 128;
    v.push_back(d);
  }
  return v;
}

struct DevPlan {
  Plan plan;
  int policy = 0;  // candidate of tile_policies(precision) the plan was built with
  // grouped GEMM launches (regular / thin tiles), pack jobs, tables, scratch
  GemmDesc* d_desc[kGemmKinds] = {};
  TileDesc* d_tiles_g[kGemmKinds] = {};
  int64_t ntiles_g[kGemmKinds] = {};
  int64_t ndesc_g[kGemmKinds] = {};
  int64_t ntiles = 0;
  PackJob* d_jobs = nullptr;
  int64_t njobs = 0, pack_gx = 0, pack_gy = 0;
  // split-TF32 panels of the tensor-core items (workspace floats, jobs)
  SplitJob* d_split = nullptr;
  int64_t nsplit = 0, split_chunks = 0, ws_floats = 0;
  // operands read from lists that were frozen when the plan was made: their
  // packed FP64 panels and split TF32 panels are made once and kept
  PackJob* d_jobs_c = nullptr;
  int64_t njobs_c = 0, pack_gx_c = 0, pack_gy_c = 0;
  SplitJob* d_split_c = nullptr;
  int64_t nsplit_c = 0, split_chunks_c = 0;
  float* const_panels = nullptr;  // persistent split panels (floats)
  // precision mode 2 (int8 slices): the panels' row maxima, zeroed before
  // each slicing (workspace float range; the persistent panels' range)
  int i8 = 0;  // int8 slices per element (precision modes 2, 3), else 0
  // the thin launch: column count it is compiled for, longest contraction range of a tile
  int thin_nc = 1;
  int64_t thin_kmax = 0;
  int64_t max_off = 0, max_floats = 0, max_off_c = 0, max_floats_c = 0;
  std::vector<int> const_lists;   // the frozen lists behind them
  bool const_stale = false;       // a list of const_lists was unfrozen since they were made
  PackJob* d_gather = nullptr;  // gather descriptions of map-addressed tensor-core operands
  int64_t* d_tabs = nullptr;
  double* scratch = nullptr;
  int64_t scratch_len = 0;
  int64_t res_off = 0, res_len = 0;
  int list1 = 0, list2 = 0, list12 = 0;
  // sym_ab descriptors of the result class (use_tr)
  FlipDesc* d_flip = nullptr;
  int64_t nflip = 0, flip_maxlen = 0;
  // kernel timing (gccu_profile): events of launches not yet reported
  std::vector<std::array<cudaEvent_t, 3>> pending;  // start, after pack, end
  int64_t calls = 0;
  double ms = 0, pack_ms = 0;
};

// transposed [ADD] of one class (add_opblk_transp), planned on first use
struct DevTransp {
  TranspDesc* d = nullptr;
  int64_t n = 0, maxlen = 0;
  int list_in = 0, list_out = 0;
  int64_t off_out = 0, len_out = 0;
};

struct DevReo {
  ReoPlan plan;
  ReoItem* d_items = nullptr;
  int64_t maxlen = 0;
  int list_ori = 0, list_reo = 0;
  int64_t reo_off = 0, reo_len = 0;
};

// singlet spin projection of one list (spin_prj_list), planned on first
// use: per case-count bucket (2, 6, 20, 70 cases) the skeleton descriptors
struct DevSpinPrj {
  SpinPrjDesc* d[4] = {};
  int64_t n[4] = {}, maxblocks[4] = {};
};
constexpr int kSpinPrjBucket[4] = {2, 6, 20, kSpinPrjMaxCases};
// pattern map of one string block (set_spprjmap_kernel): per string
// [pattern-1] entries, and whether the string is a skeleton string
struct PatternMap {
  std::vector<int32_t> m;
  std::vector<char> skel;
};

// spin patterns of n electrons (set_spprjmap_cases,
// strings/set_spprjmap_cases.f:24-41): bit n-1-i set for a beta spin at
// position i; the pattern that alternates and ends in alpha is number 0, the
// others are numbered from 1 in increasing bit order
int spin_ref_bits(int n) {
  int b = 0;
  for (int i = 1; i < n; i += 2) b |= 1 << i;
  return b;
}
int spin_pattern_number(int n, int bits) {
  const int ref = spin_ref_bits(n);
  return bits == ref ? 0 : (bits < ref ? bits + 1 : bits);
}
int spin_bits(const int* s, int n) {
  int b = 0;
  for (int i = 0; i < n; ++i)
    if (s[i] == -1) b |= 1 << (n - 1 - i);
  return b;
}
// std_spsign (strings/std_spsign_msdis.f): parity of moving every alpha in
// front of the betas
int spin_sign(const int* s, int ne) {
  int trp = 0, nb = 0;
  for (int i = 0; i < ne;) {
    const int sg = s[i];
    if (sg == 1 || sg == 2) trp += nb, ++i;
    if (sg == -1 || sg == 2) ++nb, ++i;
  }
  return (trp & 1) ? -1 : 1;
}

// singlet genealogical coupling coefficients (get_genealogical_coeff,
// baserout/get_genealogical_coeff.f:32-106, S = Ms = 0) of the creator spins
// c followed by the annihilator spins a in reverse order: one value per path
// of the branching diagram that stays at S >= 0, paths in lexical order of
// their up (0) / down (1) steps
std::vector<double> singlet_coupling(const std::vector<int>& c, const std::vector<int>& a) {
  const int nc = (int)c.size(), na = (int)a.size(), nel = nc + na;
  std::vector<int> step(nel, 1);
  std::fill(step.begin(), step.begin() + nel / 2, 0);
  std::vector<double> out;
  do {
    int down = 0;
    bool ok = true;
    for (int i = 0; i < nel; ++i) {
      down += step[i];
      ok = ok && down <= (i + 1) / 2;
    }
    if (!ok) continue;
    int s2 = 0, m2 = 0, k = 0;
    double x = 1.0;
    auto couple = [&](int dm, double sigma) {
      s2 += 1 - 2 * step[k];
      m2 += dm;
      if (step[k] == 0)
        x *= std::sqrt(std::max(0.0, (0.5 * s2 + sigma * m2) / s2));
      else
        x = -2.0 * sigma * x * std::sqrt(std::max(0.0, (0.5 * s2 + 1.0 - sigma * m2) / (s2 + 2.0)));
      ++k;
    };
    for (int i = 0; i < nc; ++i) couple(c[i], 0.5 * c[i]);
    for (int i = na - 1; i >= 0; --i) {
      couple(-a[i], -0.5 * a[i]);
      if (a[i] == -1) x = -x;
    }
    out.push_back(x);
  } while (std::next_permutation(step.begin(), step.end()));
  return out;
}

// Ms per component of the skeleton distribution (get_target_dis,
// contract/spin_prj_blk.f:440-524): 0 for even occupations; odd ones +1
// (occupations above 1 first), the rest +1 from the left and -1 from the
// right in turn
std::vector<int> skeleton_ms(const std::vector<int>& occ) {
  const int n = (int)occ.size();
  std::vector<int> t(n, 0);
  std::vector<char> set(n, 0);
  int nodd = 0, nlarge = 0;
  for (int i = 0; i < n; ++i) {
    if (occ[i] % 2) {
      ++nodd;
      nlarge += occ[i] > 1;
    } else {
      set[i] = 1;
    }
  }
  const int k = std::min(nlarge, (nodd + 1) / 2);
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < n; ++i)
      if (!set[i] && occ[i] > 1) {
        t[i] = 1, set[i] = 1;
        break;
      }
  int bal = k;
  for (int left = nodd - k; left > 0; --left) {
    if (bal <= 0) {
      for (int i = 0; i < n; ++i)
        if (!set[i]) {
          t[i] = 1, set[i] = 1, ++bal;
          break;
        }
    } else {
      for (int i = n - 1; i >= 0; --i)
        if (!set[i]) {
          t[i] = -1, set[i] = 1, --bal;
          break;
        }
    }
  }
  return t;
}

class Engine {
 public:
  Model model;
  bool have_orbs = false;
  int device = 0;
  int64_t memmax = 0, mem_used = 0;
  cudaStream_t stream = nullptr;
  // host-to-device copies of plan tables and descriptors: a stream of their
  // own, so that planning the next contraction does not wait for the
  // kernels already queued on `stream` (the host waits for the copy only)
  cudaStream_t ustream = nullptr;
  std::vector<DevList> lists;
  std::map<int, DevGraph> dgraphs;
  std::map<MapKey, int32_t*> maps;
  std::map<std::array<int, 3>, int32_t*> flips;
  std::map<std::array<int, 3>, PatternMap> spprjs;  // spin-projection pattern maps (host)
  std::map<int64_t, std::unique_ptr<DevSpinPrj>> spinprjs;  // singlet projection per list
  std::vector<FormulaPlan> formulas;  // gccu_formula_define
  std::map<std::string, std::unique_ptr<DevPlan>> plans;
  std::vector<void*> allocs;  // cudaMalloc'd one per request, freed by release()
  std::vector<void*> slabs;   // bases of the slabs small requests are cut from
  double* d_red = nullptr;  // reduction scalars
  double stats[8] = {};
  int64_t launches = 0;
  bool capturing = false;
  std::vector<cudaGraphExec_t> graphs;
  std::vector<int64_t> graph_kernels;  // kernel launches recorded in each graph
  // (list, epoch) pairs whose cached panels a graph reads without re-making
  // them: the graph is valid while each list stays frozen in that epoch
  std::vector<std::vector<std::pair<int, int64_t>>> graph_deps;
  std::vector<std::pair<int, int64_t>> capture_deps;
  int64_t capture_start = 0;
  cudaEvent_t slots[64] = {};
  bool profiling = false;
  int precision = 0;     // 0: FP64 DMMA, 1: split TF32 on tcgen05 for regular/medium items,
                         // 2, 3: FP64 emulated with 5 / 4 int8 slices on tcgen05 for the
                         // same items
  // split-TF32 operand panels, shared by all plans (one stream orders them);
  // grown to the largest plan's need, never while a graph is being captured
  float* tc_ws = nullptr;
  int64_t tc_ws_floats = 0;
  int* d_err = nullptr;  // set by kernels whose bounded pipeline waits ran out
  int64_t wait_limit = kTcWaitLimitDefault;  // mbarrier polls per pipeline wait
  // contractions run the tiles [ntiles*rank/nranks, ntiles*(rank+1)/nranks)
  // of every tile list (gccu_set_shard); 0 of 1: all
  int64_t shard_rank = 0, shard_n = 1;
  void shard_range(int64_t ntiles, int64_t& lo, int64_t& hi) const {
    lo = ntiles * shard_rank / shard_n;
    hi = ntiles * (shard_rank + 1) / shard_n;
  }
  // fixed scratch of gccu_contract_noalloc, looked up on its first call
  bool have_static = false;
  StaticScratch static_ss;
  std::vector<cudaEvent_t> event_pool;
  std::vector<DevPlan*> plan_order;  // plans in first-use order (profile report)
  std::map<std::string, std::unique_ptr<DevReo>> reos;  // reorder plans per descriptor
  std::map<std::string, std::unique_ptr<DevTransp>> transps;  // transposed [ADD] plans
  // learned correction of the diagonal step: weights, Adam moments, sample
  // set (rows and targets), gradient buffers
  double *lp_w = nullptr, *lp_m = nullptr, *lp_v = nullptr;
  int64_t lp_t = 0;
  bool lp_have_w = false;
  double *lp_rows = nullptr, *lp_tgt = nullptr;
  int64_t lp_nrows = 0, lp_cap = 0;
  double *lp_part = nullptr, *lp_grad = nullptr;
  int64_t lp_part_rows = 0;
  int64_t* lp_idx = nullptr;  // sampled element indices
  double* lp_out = nullptr;   // sampled rows
  int64_t lp_idx_cap = 0;

  void lp_alloc_weights() {
    if (lp_w) return;
    lp_w = (double*)alloc(kLpWeights * sizeof(double));
    lp_m = (double*)alloc(kLpWeights * sizeof(double));
    lp_v = (double*)alloc(kLpWeights * sizeof(double));
    lp_grad = (double*)alloc((kLpWeights + 1) * sizeof(double));
  }
  double* lp_partials(int64_t blocks) {
    if (blocks > lp_part_rows) {
      if (lp_part) release(lp_part, (size_t)lp_part_rows * (kLpWeights + 1) * sizeof(double));
      lp_part = (double*)alloc((size_t)blocks * (kLpWeights + 1) * sizeof(double));
      lp_part_rows = blocks;
    }
    return lp_part;
  }

  cudaEvent_t get_event() {
    if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    CUDA_OK(cudaEventCreate(&e));
    return e;
  }

  bool host_only = false;  // no device: model, layout and planning queries only

  // autotuner: 0 fixed rule, 1 time the candidates at a contraction's first
  // call (cached by block-shape histogram), 2 force candidate tune_forced
  int tune = 0, tune_forced = 0;
  std::map<std::string, int> tuned;  // (precision, histogram) -> chosen candidate
  // seconds spent making contraction plans: host planner, string maps,
  // autotuner trials, plan build (tables, packs and splits of cached panels)
  struct PlanStats {
    double host_s = 0, maps_s = 0, tune_s = 0, build_s = 0;
    // parts of build_s: host tables, their upload, descriptors / tiles /
    // allocations, cached operand panels; alloc_s: cudaMalloc and cudaFree
    // calls of plans (inside the stages above)
    double tables_s = 0, upload_s = 0, desc_s = 0, const_s = 0, alloc_s = 0;
    int64_t plans = 0;
  } pstats;
  std::chrono::steady_clock::time_point bt;  // stage clock inside build_gemm
  void blap(double& acc) {
    const auto now = std::chrono::steady_clock::now();
    acc += std::chrono::duration<double>(now - bt).count();
    bt = now;
  }
  struct TuneRecord {
    int64_t items;
    int chosen;
    std::vector<double> ms;  // per candidate
  };
  std::vector<TuneRecord> tune_log;

  explicit Engine(int dev, int64_t mm) : device(dev), memmax(mm), host_only(dev < 0) {
    if (host_only) return;
    CUDA_OK(cudaSetDevice(dev));
    CUDA_OK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CUDA_OK(cudaStreamCreateWithFlags(&ustream, cudaStreamNonBlocking));
    d_red = (double*)alloc(64 * sizeof(double));
    d_err = (int*)alloc(sizeof(int));
    CUDA_OK(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
  }
  ~Engine() {
    for (auto g : graphs) cudaGraphExecDestroy(g);
    for (auto ev : slots)
      if (ev) cudaEventDestroy(ev);
    for (auto ev : event_pool) cudaEventDestroy(ev);
    for (auto& kv : plans)
      for (auto& pr : kv.second->pending)
        for (auto ev : pr) cudaEventDestroy(ev);
    if (stream) cudaStreamSynchronize(stream);
    for (void* p : allocs) cudaFree(p);
    for (void* p : slabs) cudaFree(p);
    if (tabs_host) cudaFreeHost(tabs_host);
    if (ustream) cudaStreamDestroy(ustream);
    if (stream) cudaStreamDestroy(stream);
  }

  // page-locked host buffer the offset tables of a plan are built in (grown
  // to the largest plan so far, reused): filled by the host threads, then
  // copied at the link's rate instead of through a pageable staging copy
  int64_t* tabs_host = nullptr;
  int64_t tabs_cap = 0;
  int64_t* host_tables(int64_t n) {
    if (n > tabs_cap) {
      CUDA_OK(cudaStreamSynchronize(ustream));
      if (tabs_host) CUDA_OK(cudaFreeHost(tabs_host));
      tabs_host = nullptr;
      const int64_t cap = std::max<int64_t>(n, tabs_cap + tabs_cap / 2);
      CUDA_OK(cudaMallocHost(&tabs_host, (size_t)cap * sizeof(int64_t)));
      tabs_cap = cap;
    }
    return tabs_host;
  }

  // allocations made while set are also recorded here (plans built on trial
  // by the autotuner, released afterwards)
  std::vector<std::pair<void*, size_t>>* track = nullptr;

  // Device memory.  Requests up to kSlabSmall bytes (plan tables and
  // descriptors, hundreds per formula) are cut from kSlabBytes slabs, 256-byte
  // aligned, and never handed out again; larger ones get their own
  // cudaMalloc.  One cudaMalloc per plan table would cost 0.2-0.7 ms each.
  static constexpr size_t kSlabBytes = size_t(16) << 20, kSlabSmall = size_t(1) << 20;
  char* slab = nullptr;
  size_t slab_used = kSlabBytes;
  void* alloc(size_t bytes) {
    GCCU_REQUIRE(!host_only, "engine was initialised without a device (host-only mode)");
    GCCU_REQUIRE(!capturing, "device allocation requested while capturing a CUDA graph");
    if (memmax > 0 && mem_used + (int64_t)bytes > memmax)
      throw Error("device memory cap (memmax) exceeded");
    const size_t rounded = (std::max<size_t>(bytes, 16) + 255) / 256 * 256;
    void* p = nullptr;
    if (rounded <= kSlabSmall) {
      if (slab_used + rounded > kSlabBytes) {
        // slab bases are kept apart from allocs: the first piece of a slab has
        // the slab's address, and release() must not free the slab with it
        slab = (char*)device_malloc(kSlabBytes, slabs);
        slab_used = 0;
      }
      p = slab + slab_used;
      slab_used += rounded;
    } else {
      p = device_malloc(rounded, allocs);
    }
    if (track) track->push_back({p, bytes});
    mem_used += (int64_t)bytes;
    return p;
  }
  void* device_malloc(size_t bytes, std::vector<void*>& owner) {
    void* p = nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    CUDA_OK(cudaMalloc(&p, bytes));
    pstats.alloc_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    owner.push_back(p);
    return p;
  }
  // frees an allocation of its own (found in allocs); a slab piece is never
  // in allocs and is only taken off the count
  void release(void* p, size_t bytes) {
    mem_used -= (int64_t)bytes;
    for (size_t i = 0; i < allocs.size(); ++i)
      if (allocs[i] == p) {
        allocs.erase(allocs.begin() + (long)i);
        const auto t0 = std::chrono::steady_clock::now();
        CUDA_OK(cudaFree(p));
        pstats.alloc_s +=
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return;
      }
  }

  void ensure_tc_ws(int64_t floats) {
    if (floats <= tc_ws_floats) return;
    GCCU_REQUIRE(!capturing, "split-TF32 workspace must grow outside a graph capture");
    CUDA_OK(cudaStreamSynchronize(stream));  // earlier launches may still read it
    // the workspace belongs to the engine, not to the plan being built: it is
    // never recorded for release with a trial plan of the autotuner
    auto* saved = track;
    track = nullptr;
    if (tc_ws) release(tc_ws, (size_t)tc_ws_floats * sizeof(float));
    tc_ws = nullptr;
    tc_ws_floats = 0;
    tc_ws = (float*)alloc((size_t)floats * sizeof(float));
    track = saved;
    tc_ws_floats = floats;
    CUDA_OK(set_tc_workspace(tc_ws));
  }

  template <class T>
  T* upload(const std::vector<T>& v) {
    T* p = (T*)alloc(v.size() * sizeof(T));
    if (!v.empty())
      CUDA_OK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice,
                              ustream));
    CUDA_OK(cudaStreamSynchronize(ustream));
    return p;
  }

  DevList& list(int64_t id) {
    DevList& l = layout_list(id);
    GCCU_REQUIRE(host_only || l.d,
                 "intermediate list without memory: define the formula that creates it first");
    return l;
  }
  // a list whose layout (not its memory) is needed
  DevList& layout_list(int64_t id) {
    GCCU_REQUIRE(id >= 1 && id <= (int64_t)lists.size(), "invalid ME-list handle");
    return lists[id - 1];
  }
  // a list the call is about to write
  DevList& wlist(int64_t id) {
    DevList& l = list(id);
    GCCU_REQUIRE(!l.frozen, "the ME list is frozen (gccu_freeze_list): unfreeze it before "
                            "writing it");
    return l;
  }

  // do the cached panels of a plan have to be (re)made by this call?
  bool need_const(const DevPlan& dp) {
    if (dp.const_stale) return true;
    for (int l : dp.const_lists)
      if (!list(l).frozen) return true;
    return false;
  }
  // operand panels of a plan's tensor-core items over a split job list:
  // split TF32 (mode 1), or row maxima then int8 slices (mode 2), in the
  // workspace or (cached) in the plan's persistent panels
  void run_split(const DevPlan& dp, const GemmDesc* descs, const SplitJob* jobs, int64_t njobs,
                 int64_t nchunks, bool cached) {
    if (!dp.i8) {
      launch_split_tc(descs, jobs, njobs, nchunks, dp.d_gather, stream);
      ++launches;
      return;
    }
    if (cached)
      launch_zero_tc(dp.const_panels, dp.max_off_c, dp.max_floats_c, stream);
    else
      launch_zero_tc(nullptr, dp.max_off, dp.max_floats, stream);
    launch_slice_i8(0, dp.i8, descs, jobs, njobs, nchunks, dp.d_gather, stream);
    launch_slice_i8(1, dp.i8, descs, jobs, njobs, nchunks, dp.d_gather, stream);
    launches += 3;
  }
  // the GEMM launch of one tile kind (the int8-slice kernel for the
  // tensor-core tiles of a mode-2 plan)
  void run_gemm(const DevPlan& dp, int kind, const GemmDesc* descs, const TileDesc* tiles,
                int64_t ntiles, double fact) {
    if (kind == kGemmTc && dp.i8)
      launch_gemm_i8(dp.i8, descs, tiles, ntiles, fact, d_err, wait_limit, stream);
    else if (kind == kGemmThin)
      launch_thin(dp.thin_nc, descs, tiles, ntiles, dp.d_gather, dp.thin_kmax, fact, stream);
    else
      launch_gemm(kind, descs, tiles, ntiles, fact, d_err, wait_limit, stream);
    ++launches;
  }
  // make the cached panels of a plan (packs before splits: a split may read
  // a packed panel); during a capture, or else note what the graph relies on
  void run_const(DevPlan& dp, bool force = false) {
    if (dp.const_lists.empty()) return;
    if (force || need_const(dp)) {
      if (dp.njobs_c) {
        launch_pack(dp.d_jobs_c, dp.njobs_c, dp.pack_gx_c, dp.pack_gy_c, stream);
        ++launches;
      }
      if (dp.nsplit_c)
        run_split(dp, dp.d_desc[kGemmTc], dp.d_split_c, dp.nsplit_c, dp.split_chunks_c, true);
      bool all_frozen = true;
      for (int l : dp.const_lists) all_frozen = all_frozen && list(l).frozen;
      if (all_frozen) dp.const_stale = false;
    } else if (capturing) {
      for (int l : dp.const_lists) capture_deps.push_back({l, list(l).epoch});
    }
  }

  DevGraph& dgraph(int gid) {
    auto it = dgraphs.find(gid);
    if (it != dgraphs.end()) return it->second;
    Graph& g = model.G(gid);
    DevGraph dg;
    dg.W = upload(g.W);
    std::vector<int8_t> ir(g.irrep.begin(), g.irrep.end());
    if (ir.empty()) ir.push_back(0);
    dg.irrep = upload(ir);
    return dgraphs[gid] = dg;
  }
  int32_t* dtable(int gid, int idxms, int gam) {
    DevGraph& dg = dgraph(gid);
    int key = (idxms - 1) * model.os.nsym + gam - 1;
    auto it = dg.tables.find(key);
    if (it != dg.tables.end()) return it->second;
    const auto& t = model.G(gid).table(idxms, gam);
    std::vector<int32_t> v(t);
    if (v.empty()) v.push_back(0);
    return dg.tables[key] = upload(v);
  }

  // device string map of one block pair, built on first use
  int32_t* strmap(const MapKey& k) {
    auto it = maps.find(k);
    if (it != maps.end()) return it->second;
    Graph &g1 = model.G(k[0]), &g2 = model.G(k[1]);
    GCCU_REQUIRE(g1.type == g2.type, "string map between different hpvx types");
    int g12 = model.graph(g1.type, g1.nel + g2.nel);
    int64_t n1 = g1.nstr(k[2], k[4]), n2 = g2.nstr(k[3], k[5]);
    int32_t* t1 = dtable(k[0], k[2], k[4]);
    int32_t* t2 = dtable(k[1], k[3], k[5]);
    DevGraph& d12 = dgraph(g12);
    int32_t* out = (int32_t*)alloc(std::max<int64_t>(n1 * n2, 1) * sizeof(int32_t));
    launch_strmap(t1, g1.nel, n1, t2, g2.nel, n2, d12.W, d12.irrep, g1.nel + g2.nel,
                  model.os.nsym, out, stream);
    ++launches;
    CUDA_OK(cudaGetLastError());
    return maps[k] = out;
  }

  // spin-flip map of one graph block (set_flipmap_kernel,
  // strings/set_flipmap_kernel.f:47-88): str -> sign * (address of the
  // flipped string + 1), sign = std_spsign(str)*std_spsign(flipped)
  int32_t* flipmap(int gid, int idxms, int gam) {
    std::array<int, 3> key{gid, idxms, gam};
    auto it = flips.find(key);
    if (it != flips.end()) return it->second;
    Graph& g = model.G(gid);
    const auto& t = g.table(idxms, gam);
    int nel = g.nel;
    int64_t n = g.nstr(idxms, gam);
    std::vector<int32_t> m(std::max<int64_t>(n, 1), 0);
    std::vector<int> orb(nel), spn(nel), spf(nel);
    auto spsign = [](const int* s, int ne) {
      int trp = 0, nb = 0, i = 0;
      while (i < ne) {
        int sg = s[i];
        if (sg == 1 || sg == 2) trp += nb, ++i;
        if (sg == -1 || sg == 2) ++nb, ++i;
      }
      return (trp & 1) ? -1 : 1;
    };
    for (int64_t s = 0; s < n; ++s) {
      for (int p = 0; p < nel; ++p) {
        int v = t[s * nel + p], c = v & 3;
        orb[p] = v >> 2;
        spn[p] = c == 1 ? 1 : (c == 2 ? -1 : 2);
        spf[p] = spn[p] == 2 ? 2 : -spn[p];
      }
      int sg = spsign(spn.data(), nel) * spsign(spf.data(), nel);
      m[s] = sg * (int32_t)(g.address(orb.data(), spf.data()) + 1);
    }
    return flips[key] = upload(m);
  }

  // reorder plan of a descriptor, built on first use
  DevReo& reo_for(const gccu_reo_desc* r) {
    GCCU_REQUIRE(r->nshift >= 0 && r->nshift <= kMaxShift, "reorder: nshift must be 0..4");
    std::ostringstream os;
    os << r->list_ori << ',' << r->iblk_ori << ',' << r->list_reo << ',' << r->iblk_reo << ','
       << r->nshift;
    for (int s = 0; s < r->nshift; ++s) {
      os << ';' << r->from_vtx[s] << ',' << r->to_vtx[s];
      for (int k = 0; k < 8; ++k) os << ',' << r->occ_shift[s][k];
    }
    auto it = reos.find(os.str());
    if (it != reos.end()) return *it->second;
    GCCU_REQUIRE(!capturing, "reorder must be run once before it is captured in a graph");
    const ListLayout& Lo = list(r->list_ori).L;
    const ListLayout& Lr = list(r->list_reo).L;
    const int nj = model.ops.at(Lo.op - 1).nj;
    GCCU_REQUIRE(model.ops.at(Lr.op - 1).nj == nj, "reorder: operators differ in njoined");
    GCCU_REQUIRE(r->iblk_ori >= 1 && r->iblk_ori <= (int64_t)Lo.blk.size() && r->iblk_reo >= 1 &&
                     r->iblk_reo <= (int64_t)Lr.blk.size(),
                 "reorder: occupation class out of range");
    ReorderSpec s;
    s.Lori = &Lo;
    s.Lreo = &Lr;
    s.ib_ori = (int)r->iblk_ori;
    s.ib_reo = (int)r->iblk_reo;
    s.nj = nj;
    s.nshift = (int)r->nshift;
    for (int t = 0; t < s.nshift; ++t) {
      s.shift[t] = to_occ(r->occ_shift[t]);
      GCCU_REQUIRE(r->from_vtx[t] >= 1 && r->from_vtx[t] <= nj && r->to_vtx[t] >= 1 &&
                       r->to_vtx[t] <= nj,
                   "reorder: vertex out of range");
      s.from[t] = (int)r->from_vtx[t] - 1;
      s.to[t] = (int)r->to_vtx[t] - 1;
    }
    auto dr = std::make_unique<DevReo>();
    dr->plan = plan_reorder(model, s);
    dr->list_ori = (int)r->list_ori;
    dr->list_reo = (int)r->list_reo;
    dr->reo_off = Lr.blk[r->iblk_reo - 1].off;
    dr->reo_len = Lr.blk[r->iblk_reo - 1].len;
    ReoPlan& P = dr->plan;
    GCCU_REQUIRE(P.items.size() <= 65535, "reorder: too many distribution cases");
    for (auto& it2 : P.items) dr->maxlen = std::max(dr->maxlen, it2.N0 * it2.NK);
    if (!host_only) {
      for (auto& m : P.maps) {
        ReoItem& ri = P.items[m.item];
        (m.opnd == 0 ? ri.ori : ri.reo).map[m.comp] = strmap(m.key);
      }
      if (!P.items.empty()) dr->d_items = upload(P.items);
    }
    return *(reos[os.str()] = std::move(dr));
  }

  // leading dimensions of set_op_ldim_c (contract/set_op_ldim_c.f) over the
  // components c, a with string counts lc, la: C before A per hpvx type, or
  // with transpose A before C, the components of a type in reverse order
  static void op_ldims(const std::vector<Comp>& c, const std::vector<Comp>& a,
                       const std::vector<int64_t>& lc, const std::vector<int64_t>& la,
                       bool transpose, int64_t* ldc, int64_t* lda) {
    int64_t ld = 1;
    for (int ih = 0; ih < 4; ++ih) {
      const int t = kHpvxSeq[ih];
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

  // plan of a transposed [ADD] (add_opblk_transp, contract/add_opblk_transp.f:
  // 195-321): per distribution of the output class, the input distribution
  // with C and A strings exchanged (at Ms(C), IRREP(C) of the output) and the
  // leading dimensions of both over the output's components
  DevTransp& transp_for(int64_t lin, int64_t ibin, int64_t lout, int64_t ibout, bool tra_in,
                        bool tra_out) {
    std::ostringstream os;
    os << lin << ',' << ibin << ',' << lout << ',' << ibout << ',' << tra_in << tra_out;
    auto it = transps.find(os.str());
    if (it != transps.end()) return *it->second;
    GCCU_REQUIRE(!capturing, "transposed add must be run once before it is captured in a graph");
    GCCU_REQUIRE(tra_in != tra_out, "add_opblk_transp: exactly one side is transposed");
    const ListLayout& Li = list(lin).L;
    const ListLayout& Lo = list(lout).L;
    GCCU_REQUIRE(model.ops.at(Li.op - 1).nj == 1 && model.ops.at(Lo.op - 1).nj == 1,
                 "add_opblk_transp: operators of one vertex only in this engine version");
    GCCU_REQUIRE(ibin >= 1 && ibin <= (int64_t)Li.blk.size() && ibout >= 1 &&
                     ibout <= (int64_t)Lo.blk.size(),
                 "add_opblk_transp: occupation class out of range");
    const LayoutBlock& Bi = Li.blk[ibin - 1];
    const LayoutBlock& Bo = Lo.blk[ibout - 1];
    auto same = [](const std::vector<Comp>& x, const std::vector<Comp>& y) {
      if (x.size() != y.size()) return false;
      for (size_t i = 0; i < x.size(); ++i)
        if (x[i].occ != y[i].occ || x[i].hpvx != y[i].hpvx) return false;
      return true;
    };
    GCCU_REQUIRE(same(Bi.c, Bo.a) && same(Bi.a, Bo.c),
                 "add_opblk_transp: input and output list do not have compatible operators");
    GCCU_REQUIRE(Bo.c.size() <= (size_t)kDevMaxComp && Bo.a.size() <= (size_t)kDevMaxComp,
                 "add_opblk_transp: too many components");
    int msc_max = 0, msa_max = 0;
    for (auto& x : Bo.c) msc_max += x.occ;
    for (auto& x : Bo.a) msa_max += x.occ;
    const int nsym = model.os.nsym;
    auto dt = std::make_unique<DevTransp>();
    std::vector<TranspDesc> v;
    for (auto& kv : Bo.dis) {
      const int gama = kv.first.second;
      for (const Dist& d : kv.second) {
        if (d.len <= 0) continue;
        int msc = 0;
        for (int m : d.msc) msc += m;
        std::vector<int> ixc(Bo.c.size()), ixa(Bo.a.size());
        std::vector<int64_t> lc(Bo.c.size()), la(Bo.a.size());
        TranspDesc t{};
        t.nc = (int32_t)Bo.c.size();
        t.na = (int32_t)Bo.a.size();
        t.lenc = t.lena = 1;
        for (size_t i = 0; i < Bo.c.size(); ++i) {
          ixc[i] = ms_index(Bo.c[i].occ, d.msc[i]);
          lc[i] = model.G(Bo.c[i].graph).nstr(ixc[i], d.gc[i]);
          t.lc[i] = (int32_t)lc[i];
          t.lenc *= lc[i];
        }
        for (size_t i = 0; i < Bo.a.size(); ++i) {
          ixa[i] = ms_index(Bo.a[i].occ, d.msa[i]);
          la[i] = model.G(Bo.a[i].graph).nstr(ixa[i], d.ga[i]);
          t.la[i] = (int32_t)la[i];
          t.lena *= la[i];
        }
        if (t.lenc == 0 || t.lena == 0) continue;
        const int ix_in = msa_to_idxms(msc, Li.mst, msc_max, msa_max);
        const int gam_in = irrep_mult(gama, Lo.gamt);
        auto f = Bi.dis.find({ix_in, gam_in});
        GCCU_REQUIRE(f != Bi.dis.end(),
                     "add_opblk_transp: the input list has no distribution for this case "
                     "(total Ms or IRREP differ from the output's adjoint)");
        const int64_t did = dist_id(Bi.c, ixa, d.ga, Bi.a, ixc, d.gc, nsym);
        const Dist* src = nullptr;
        for (const Dist& di : f->second)
          if (di.did == did) src = &di;
        GCCU_REQUIRE(src && src->len == d.len, "add_opblk_transp: distribution not found");
        t.off_out = d.off;
        t.off_in = src->off;
        op_ldims(Bo.c, Bo.a, lc, la, tra_out, t.ldoc, t.ldoa);
        op_ldims(Bo.c, Bo.a, lc, la, tra_in, t.ldic, t.ldia);
        v.push_back(t);
        dt->maxlen = std::max(dt->maxlen, t.lenc * t.lena);
      }
    }
    GCCU_REQUIRE(v.size() <= 65535, "add_opblk_transp: too many distributions");
    dt->n = (int64_t)v.size();
    if (!v.empty() && !host_only) dt->d = upload(v);
    dt->list_in = (int)lin;
    dt->list_out = (int)lout;
    dt->off_out = Bo.off;
    dt->len_out = Bo.len;
    return *(transps[os.str()] = std::move(dt));
  }

  // trace plan (same device form as a reorder), built on first use
  DevReo& trace_for(int64_t lop, int64_t ibop, int64_t lres, int64_t ibres, const int64_t* cnt) {
    std::ostringstream os;
    os << "T" << lop << ',' << ibop << ',' << lres << ',' << ibres;
    for (int k = 0; k < 8; ++k) os << ',' << cnt[k];
    auto it = reos.find(os.str());
    if (it != reos.end()) return *it->second;
    GCCU_REQUIRE(!capturing, "trace must be run once before it is captured in a graph");
    const ListLayout& Lo = list(lop).L;
    const ListLayout& Lr = list(lres).L;
    GCCU_REQUIRE(ibop >= 1 && ibop <= (int64_t)Lo.blk.size() && ibres >= 1 &&
                     ibres <= (int64_t)Lr.blk.size(),
                 "trace: occupation class out of range");
    TraceSpec s;
    s.Lop = &Lo;
    s.Lres = &Lr;
    s.ib_op = (int)ibop;
    s.ib_res = (int)ibres;
    s.cnt = to_occ(cnt);
    auto dr = std::make_unique<DevReo>();
    dr->plan = plan_trace(model, s);
    dr->list_ori = (int)lop;
    dr->list_reo = (int)lres;
    dr->reo_off = Lr.blk[ibres - 1].off;
    dr->reo_len = Lr.blk[ibres - 1].len;
    ReoPlan& P = dr->plan;
    GCCU_REQUIRE(P.items.size() <= 65535, "trace: too many distribution cases");
    for (auto& it2 : P.items) dr->maxlen = std::max(dr->maxlen, it2.N0 * it2.NK);
    if (!host_only) {
      for (auto& m : P.maps) {
        ReoItem& ri = P.items[m.item];
        (m.opnd == 0 ? ri.ori : ri.reo).map[m.comp] = strmap(m.key);
      }
      if (!P.items.empty()) dr->d_items = upload(P.items);
    }
    return *(reos[os.str()] = std::move(dr));
  }

  std::string plan_key(const gccu_bc_desc* bc, bool use_tr) const {
    std::ostringstream os;
    os << bc->list_op1 << ',' << bc->iblk_op1 << ',' << bc->list_op2 << ',' << bc->iblk_op2 << ','
       << bc->list_res << ',' << bc->iblk_res << ',' << use_tr << ",p" << precision
       << ",u" << tune << (tune == 2 ? "." + std::to_string(tune_forced) : std::string()) << ",t"
       << (bc->tra_op1 != 0) << (bc->tra_op2 != 0) << (bc->tra_res != 0);
    for (int k = 0; k < 8; ++k) os << ',' << bc->occ_ex1[k] << ',' << bc->occ_ex2[k] << ','
                                   << bc->occ_cnt[k];
    return os.str();
  }

  // cached plan of a descriptor, or null; never plans (gccu_contract_noalloc)
  DevPlan* find_plan(const gccu_bc_desc* bc, bool use_tr) {
    auto it = plans.find(plan_key(bc, use_tr));
    return it == plans.end() ? nullptr : it->second.get();
  }

  DevPlan& plan_for(const gccu_bc_desc* bc, bool use_tr) {
    std::string key = plan_key(bc, use_tr);
    auto it = plans.find(key);
    if (it != plans.end()) return *it->second;
    GCCU_REQUIRE(!capturing, "contraction must be run once before it is captured in a graph");
    ContractionSpec s;
    for (int64_t l : {bc->list_op1, bc->list_op2, bc->list_res})
      GCCU_REQUIRE(model.ops.at(list(l).L.op - 1).nj == 1,
                   "contractions of joined (multi-vertex) operators are not supported by this "
                   "engine version");
    s.L1 = &list(bc->list_op1).L;
    s.L2 = &list(bc->list_op2).L;
    s.L12 = &list(bc->list_res).L;
    s.ib1 = (int)bc->iblk_op1;
    s.ib2 = (int)bc->iblk_op2;
    s.ib12 = (int)bc->iblk_res;
    for (int k = 0; k < 8; ++k) {
      s.ex1[k] = (int)bc->occ_ex1[k];
      s.ex2[k] = (int)bc->occ_ex2[k];
      s.cnt[k] = (int)bc->occ_cnt[k];
    }
    s.use_tr = use_tr;
    s.tra1 = bc->tra_op1 != 0;
    s.tra2 = bc->tra_op2 != 0;
    s.tra12 = bc->tra_res != 0;
    auto dp = std::make_unique<DevPlan>();
    const auto t0 = std::chrono::steady_clock::now();
    dp->plan = plan_contraction(model, s);
    dp->list1 = (int)bc->list_op1;
    dp->list2 = (int)bc->list_op2;
    dp->list12 = (int)bc->list_res;
    const LayoutBlock& B12 = s.L12->blk[s.ib12 - 1];
    dp->res_off = B12.off;
    dp->res_len = B12.len;
    Plan& P = dp->plan;
    if (host_only) return *(plans[key] = std::move(dp));
    // host time of each planning stage (the device work a stage queues, for
    // instance cached panels, is not waited for)
    auto lap = [&](double& acc, std::chrono::steady_clock::time_point& t) {
      const auto now = std::chrono::steady_clock::now();
      acc += std::chrono::duration<double>(now - t).count();
      t = now;
    };
    auto t = t0;
    lap(pstats.host_s, t);
    for (auto& r : P.maps) P.items[r.item].op[r.opnd].map[r.comp] = strmap(r.key);
    lap(pstats.maps_s, t);
    // a sharded engine keeps the fixed rule: the ranks' shares partition the
    // tile lists only if every rank builds the same ones, which independent
    // timings do not guarantee
    dp->policy = tune == 2 ? tune_forced : (tune == 1 && shard_n == 1) ? autotune(*dp) : 0;
    lap(pstats.tune_s, t);
    build_gemm(*dp, tile_policies(precision).at(dp->policy));
    if (P.use_tr) build_flip(*dp, list(bc->list_res), (int)bc->iblk_res);
    lap(pstats.build_s, t);
    ++pstats.plans;
    plan_order.push_back(dp.get());
    return *(plans[key] = std::move(dp));
  }

  // the kernels of one contraction after the result's reset: cached panels
  // (when out of date), packs, splits, the GEMMs of every tile shape (this
  // rank's share), the spin-flip symmetrisation; evp (optional) is recorded
  // after the packs and splits
  void launch_plan(DevPlan& dp, double fact, cudaEvent_t evp = nullptr, bool flip = true) {
    run_const(dp);
    if (dp.njobs) {
      launch_pack(dp.d_jobs, dp.njobs, dp.pack_gx, dp.pack_gy, stream);
      ++launches;
    }
    if (dp.nsplit)  // operand split of the tensor-core items (after the pack it may read)
      run_split(dp, dp.d_desc[kGemmTc], dp.d_split, dp.nsplit, dp.split_chunks, false);
    if (evp) CUDA_OK(cudaEventRecord(evp, stream));
    for (int kind = 0; kind < kGemmKinds; ++kind) {
      if (!dp.ntiles_g[kind]) continue;
      int64_t lo, hi;
      shard_range(dp.ntiles_g[kind], lo, hi);
      if (hi <= lo) continue;
      run_gemm(dp, kind, dp.d_desc[kind], dp.d_tiles_g[kind] + lo, hi - lo, fact);
    }
    if (flip && dp.plan.use_tr && dp.nflip) {
      launch_sym_ab(dp.d_flip, dp.nflip, list(dp.list12).d, 0.5, dp.flip_maxlen, stream);
      ++launches;
    }
  }

  // block-shape histogram of a plan: per item the binary orders of M, N, K
  // and which operands need map lookups, counted
  // kernel kind per item of a plan under a tile policy (and whether its
  // operands are swapped)
  static void route_items(const Plan& P, const TilePolicy& pol, int precision,
                          std::vector<int>& kind_of, std::vector<char>& swapped) {
    // kernel kind per item: small result, skinny or medium (thin ex2, or thin
    // ex1 with the operands swapped), else regular
    kind_of.assign(P.items.size(), kGemmRegular);
    swapped.assign(P.items.size(), 0);
    for (size_t i = 0; i < P.items.size(); ++i) {
      const ItemDesc& it = P.items[i];
      kind_of[i] = kGemmRegular;
      if (it.M * it.N <= 16) {
        kind_of[i] = kGemmSmall;
      } else if (it.N <= kGemmSkinnyN) {
        kind_of[i] = kGemmSkinny;
      } else if (it.M <= kGemmSkinnyN) {
        kind_of[i] = kGemmSkinny;
        swapped[i] = 1;
      } else if (it.N <= pol.medium_max) {
        kind_of[i] = kGemmMedium;
      } else if (it.M <= pol.medium_max) {
        kind_of[i] = kGemmMedium;
        swapped[i] = 1;
      }
      // split-TF32 mode: the GEMM-sized items go to the tensor-core kernel
      // (items with at most 32 columns keep the FP64 128 x 32 tile, which
      // wastes less than a 256-wide tensor-core tile; items with fewer than
      // kTcMinK contraction indices keep FP64, their tiles would be set-up
      // and epilogue only)
      if (precision >= 1 && it.K >= pol.tc_min_k &&
          (kind_of[i] == kGemmRegular ||
           (pol.tc_thin && kind_of[i] == kGemmMedium && !swapped[i] && it.M > kGemmMediumN))) {
        kind_of[i] = kGemmTc;
        swapped[i] = 0;
      }
      // thin column side (after the swap), result without map lookups, long
      // operand read in place: the streaming kernel
      if (pol.thin && (kind_of[i] == kGemmMedium || kind_of[i] == kGemmSkinny) &&
          (swapped[i] ? it.M : it.N) <= kThinMaxColumns && it.op[2].nmap == 0 &&
          it.op[swapped[i] ? 1 : 0].nmap <= kTcGatherMaps)
        kind_of[i] = kGemmThin;
    }
  }

  // what a tile policy changes in a plan: the kind and operand order of
  // every item, and for FP64 launches whether contractions may be split
  static std::string routing_signature(const Plan& P, const TilePolicy& pol, int precision) {
    std::vector<int> kind_of;
    std::vector<char> swapped;
    route_items(P, pol, precision, kind_of, swapped);
    std::string sig(kind_of.size() * 2 + 1, ' ');
    for (size_t i = 0; i < kind_of.size(); ++i) {
      sig[2 * i] = (char)('0' + kind_of[i]);
      sig[2 * i + 1] = swapped[i] ? 's' : '-';
    }
    sig.back() = pol.ksplit ? 'k' : '-';
    return sig;
  }

  static std::string histogram_key(int precision, const Plan& P, bool frozen1, bool frozen2) {
    std::map<std::array<int, 6>, int> h;
    auto lg = [](int64_t x) {
      int b = 0;
      while ((int64_t(1) << b) < x) ++b;
      return b;
    };
    for (const auto& it : P.items)
      h[{lg(it.M), lg(it.N), lg(it.K), it.op[0].nmap > 0, it.op[1].nmap > 0,
         it.op[2].nmap > 0}]++;
    std::ostringstream os;
    os << "p" << precision << "f" << frozen1 << frozen2;  // cached operand panels
    for (auto& kv : h) {
      os << ';';
      for (int v : kv.first) os << v << ',';
      os << kv.second;
    }
    return os.str();
  }

  // the candidate tile policy for a new plan: the cached choice of its
  // histogram, else each candidate built on trial and timed on the actual
  // lists (best of two launches, the result block restored around them)
  int autotune(DevPlan& dp) {
    const std::string key =
        histogram_key(precision, dp.plan, list(dp.list1).frozen, list(dp.list2).frozen);
    auto f = tuned.find(key);
    if (f != tuned.end()) return f->second;
    const auto cands = tile_policies(precision);
    if (cands.size() == 1) return tuned[key] = 0;
    DevList& r = list(dp.list12);
    double* snap = (double*)alloc(std::max<int64_t>(dp.res_len, 1) * sizeof(double));
    CUDA_OK(cudaMemcpyAsync(snap, r.d + dp.res_off, dp.res_len * sizeof(double),
                            cudaMemcpyDeviceToDevice, stream));
    cudaEvent_t e0 = get_event(), e1 = get_event();
    TuneRecord rec{(int64_t)dp.plan.items.size(), 0, {}};
    std::vector<std::string> sigs;
    for (size_t c = 0; c < cands.size(); ++c) {
      // a candidate that routes every item as an earlier one would build the
      // same plan: it takes that candidate's time without a trial
      sigs.push_back(routing_signature(dp.plan, cands[c], precision));
      const size_t same = std::find(sigs.begin(), sigs.end(), sigs.back()) - sigs.begin();
      if (same < c) {
        rec.ms.push_back(rec.ms[same]);
        continue;
      }
      std::vector<std::pair<void*, size_t>> owned;
      auto trial = std::make_unique<DevPlan>();
      trial->plan = dp.plan;
      trial->list1 = dp.list1;
      trial->list2 = dp.list2;
      trial->list12 = dp.list12;
      trial->res_off = dp.res_off;
      trial->res_len = dp.res_len;
      track = &owned;
      double best = 1e30;
      try {
        build_gemm(*trial, cands[c]);
        for (int rep = 0; rep < 2; ++rep) {
          CUDA_OK(cudaEventRecord(e0, stream));
          launch_plan(*trial, 1.0, nullptr, false);
          CUDA_OK(cudaEventRecord(e1, stream));
          CUDA_OK(cudaEventSynchronize(e1));
          float ms = 0;
          CUDA_OK(cudaEventElapsedTime(&ms, e0, e1));
          best = std::min(best, (double)ms);
        }
      } catch (...) {
        track = nullptr;
        throw;
      }
      track = nullptr;
      CUDA_OK(cudaStreamSynchronize(stream));
      for (auto& pr : owned) release(pr.first, pr.second);
      rec.ms.push_back(best);
      if (best < rec.ms[rec.chosen]) rec.chosen = (int)c;
      CUDA_OK(cudaMemcpyAsync(r.d + dp.res_off, snap, dp.res_len * sizeof(double),
                              cudaMemcpyDeviceToDevice, stream));
    }
    // an alternative replaces the fixed rule only when it is clearly faster
    // (differences of a few percent are within the timing noise of two runs)
    if (rec.chosen != 0 && rec.ms[rec.chosen] > kTuneMargin * rec.ms[0]) rec.chosen = 0;
    event_pool.push_back(e0);
    event_pool.push_back(e1);
    CUDA_OK(cudaStreamSynchronize(stream));
    release(snap, std::max<int64_t>(dp.res_len, 1) * sizeof(double));
    check_err();
    tune_log.push_back(rec);
    return tuned[key] = rec.chosen;
  }

  // offsets of the single-source components of operand od that belong to
  // space sp, for every composite index of that space
  static void part_table(const ItemDesc& it, const OpndDesc& od, int sp, int64_t n,
                         int64_t* out) {
    // offset = sum over the space's components q of comp_q * coef_q; the
    // composite index advances like an odometer (first component fastest),
    // so each entry costs one addition instead of a mixed-radix division
    const int nq = it.nsp[sp];
    int64_t coef[kDevMaxComp] = {};
    for (int j = 0; j < od.ncomp; ++j) {
      if (od.map[j] || (od.sp1[j] != kNone && od.sp2[j] != kNone)) continue;
      if (od.sp1[j] == sp) coef[od.ci1[j]] += od.ldim[j];
      else if (od.sp2[j] == sp) coef[od.ci2[j]] += od.ldim[j];
    }
    int64_t comp[kDevMaxComp] = {};
    int64_t off = 0;
    for (int64_t x = 0; x < n; ++x) {
      out[x] = off;
      for (int q = 0; q < nq; ++q) {
        if (++comp[q] < it.rad[sp][q]) {
          off += coef[q];
          break;
        }
        off -= (comp[q] - 1) * coef[q];  // the component wraps to 0, carry
        comp[q] = 0;
      }
    }
  }

  // for each map component of operand od (in component order) and every
  // composite index of space sp: the string index that space contributes to
  // the map lookup (layout [map component][index]), nmap * n entries
  static void map_index_table(const ItemDesc& it, const OpndDesc& od, int sp, int64_t n,
                              int64_t* out) {
    const int nq = it.nsp[sp];
    for (int j = 0; j < od.ncomp; ++j) {
      if (!od.map[j]) continue;
      const int c = od.sp1[j] == sp ? od.ci1[j] : od.ci2[j];
      int64_t comp[kDevMaxComp] = {};
      for (int64_t x = 0; x < n; ++x) {
        *out++ = comp[c];
        for (int q = 0; q < nq; ++q) {
          if (++comp[q] < it.rad[sp][q]) break;
          comp[q] = 0;
        }
      }
    }
  }

  // step of an offset table that is affine in its index (tab[k] = tab[0] +
  // k * step, step != 0), else 0
  static int64_t affine_step(const int64_t* tabs, int64_t at, int64_t n) {
    if (n < 2) return 0;
    const int64_t step = tabs[at + 1] - tabs[at];
    if (step == 0) return 0;
    for (int64_t k = 2; k < n; ++k)
      if (tabs[at + k] - tabs[at] != k * step) return 0;
    return step;
  }

  // run njobs table fills on up to 16 host threads, the largest first, each
  // thread taking the next unclaimed job
  template <typename Run, typename Size>
  static void fill_tables(size_t njobs, Run run, Size size) {
    std::vector<size_t> order(njobs);
    for (size_t j = 0; j < njobs; ++j) order[j] = j;
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return size(a) > size(b); });
    int64_t total = 0;
    for (size_t j = 0; j < njobs; ++j) total += size(j);
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = total < (1 << 20) ? 1u : std::min<unsigned>(16u, hw);
    std::atomic<size_t> next{0};
    auto worker = [&]() {
      for (size_t q; (q = next.fetch_add(1)) < njobs;) run(order[q]);
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
  }

  // GEMM descriptors, offset tables, pack jobs and tiles of one plan
  void build_gemm(DevPlan& dp, const TilePolicy& pol) {
    bt = std::chrono::steady_clock::now();
    Plan& P = dp.plan;
    const double* x1 = list(dp.list1).d;
    const double* x2 = list(dp.list2).d;
    double* x12 = list(dp.list12).d;
    struct Tab { int64_t aro, ako, bco, bko, cro, cco; };
    std::vector<Tab> toff(P.items.size());
    std::vector<PackJob> jobs, jobs_c;
    std::vector<int64_t> pack_off1(P.items.size(), -1), pack_off2(P.items.size(), -1);
    // operands of frozen lists: made once (plan time), kept with the plan
    const bool frozen_op[2] = {list(dp.list1).frozen, list(dp.list2).frozen};
    bool const_used[2] = {false, false};
    int64_t scratch = 0;
    dp.pack_gx = dp.pack_gy = 0;
    // the tables are laid out first (offsets in `tabs`) and filled
    // afterwards, several at a time on the host's cores
    struct TabJob {
      int64_t off, n;
      std::function<void(int64_t*)> fill;
    };
    std::vector<TabJob> tjobs;
    int64_t ntab = 0;
    auto put = [&](int64_t n, std::function<void(int64_t*)> fill) {
      const int64_t o = ntab;
      tjobs.push_back({o, n, std::move(fill)});
      ntab += n;
      return o;
    };
    std::vector<int> kind_of;
    std::vector<char> swapped;
    route_items(P, pol, precision, kind_of, swapped);
    // an operand whose strings need map lookups is packed into a dense panel,
    // except for tensor-core items, whose split pre-pass reads it in place
    // through the same gather description
    auto maps_of = [&](size_t i, int op) { return P.items[i].op[op].nmap > 0; };
    auto tcgather = [&](size_t i, int op) {
      return maps_of(i, op) && kind_of[i] == kGemmTc && P.items[i].op[op].nmap <= kTcGatherMaps;
    };
    // the long operand of a thin item (the row side after the swap), read in
    // place by k_thin through its gather description
    auto thingather = [&](size_t i, int op) {
      return maps_of(i, op) && kind_of[i] == kGemmThin && op == (swapped[i] ? 1 : 0);
    };
    auto packed = [&](size_t i, int op) {
      return maps_of(i, op) && !tcgather(i, op) && !thingather(i, op);
    };
    struct PackTab { int64_t roff, koff, rmi, kmi; };
    std::vector<PackTab> ptab1(P.items.size()), ptab2(P.items.size());
    auto pack_tabs = [&](const ItemDesc& it, int op, PackTab& pt) {
      const OpndDesc* od = &it.op[op];
      const ItemDesc* ip = &it;
      const int rsp = op == 0 ? kEx1 : kEx2;
      const int64_t R = op == 0 ? it.M : it.N, K = it.K;
      int64_t nm = 0;  // the components map_index_table writes a block for
      for (int j = 0; j < od->ncomp; ++j) nm += od->map[j] != nullptr;
      pt.roff = put(R, [=](int64_t* v) { part_table(*ip, *od, rsp, R, v); });
      pt.koff = put(K, [=](int64_t* v) { part_table(*ip, *od, kCnt, K, v); });
      pt.rmi = put(nm * R, [=](int64_t* v) { map_index_table(*ip, *od, rsp, R, v); });
      pt.kmi = put(nm * K, [=](int64_t* v) { map_index_table(*ip, *od, kCnt, K, v); });
    };
    // identity tables of a packed panel: rows r, indices k * rows
    auto iota = [&](int64_t n, int64_t step) {
      return put(n, [=](int64_t* v) {
        for (int64_t x = 0; x < n; ++x) v[x] = x * step;
      });
    };
    auto part = [&](const ItemDesc& it, int op, int sp, int64_t n) {
      const ItemDesc* ip = &it;
      const OpndDesc* od = &it.op[op];
      return put(n, [=](int64_t* v) { part_table(*ip, *od, sp, n, v); });
    };
    for (size_t i = 0; i < P.items.size(); ++i) {
      const ItemDesc& it = P.items[i];
      Tab& t = toff[i];
      if (maps_of(i, 0)) pack_tabs(it, 0, ptab1[i]);
      if (maps_of(i, 1)) pack_tabs(it, 1, ptab2[i]);
      if (tcgather(i, 0) || thingather(i, 0)) {  // read in place by the split pre-pass / k_thin
        t.aro = ptab1[i].roff;
        t.ako = ptab1[i].koff;
      } else if (packed(i, 0)) {  // panel[k*M + r], or panel[r*K + k] when read along k
        pack_off1[i] = scratch;
        scratch += it.M * it.K;
        t.aro = it.kfast1 ? iota(it.M, it.K) : iota(it.M, 1);
        t.ako = it.kfast1 ? iota(it.K, 1) : iota(it.K, it.M);
      } else {
        t.aro = part(it, 0, kEx1, it.M);
        t.ako = part(it, 0, kCnt, it.K);
      }
      if (tcgather(i, 1) || thingather(i, 1)) {
        t.bco = ptab2[i].roff;
        t.bko = ptab2[i].koff;
      } else if (packed(i, 1)) {  // panel[k*N + c], or panel[c*K + k] when read along k
        pack_off2[i] = scratch;
        scratch += it.N * it.K;
        t.bco = it.kfast2 ? iota(it.N, it.K) : iota(it.N, 1);
        t.bko = it.kfast2 ? iota(it.K, 1) : iota(it.K, it.N);
      } else {
        t.bco = part(it, 1, kEx2, it.N);
        t.bko = part(it, 1, kCnt, it.K);
      }
      t.cro = part(it, 2, kEx1, it.M);
      t.cco = part(it, 2, kEx2, it.N);
    }
    int64_t* tabs = host_tables(std::max<int64_t>(ntab, 1));
    if (!ntab) tabs[0] = 0;
    fill_tables(tjobs.size(), [&](size_t j) { tjobs[j].fill(tabs + tjobs[j].off); },
                [&](size_t j) { return tjobs[j].n; });
    blap(pstats.tables_s);
    dp.d_tabs = (int64_t*)alloc((size_t)std::max<int64_t>(ntab, 1) * sizeof(int64_t));
    CUDA_OK(cudaMemcpyAsync(dp.d_tabs, tabs, (size_t)std::max<int64_t>(ntab, 1) * sizeof(int64_t),
                            cudaMemcpyHostToDevice, ustream));
    CUDA_OK(cudaStreamSynchronize(ustream));
    blap(pstats.upload_s);
    dp.scratch = scratch ? (double*)alloc(scratch * sizeof(double)) : nullptr;
    dp.scratch_len = scratch;
    std::vector<GemmDesc> g[kGemmKinds];
    std::vector<int32_t> group_of(P.items.size());
    // gather description of operand op of item i (a k_pack job into dst, or
    // read in place by the split pre-pass when dst is null)
    auto job_of = [&](size_t i, int op, double* dst) {
      const ItemDesc& it = P.items[i];
      PackJob j{};
      j.R = op == 0 ? it.M : it.N;
      j.K = it.K;
      j.src = op == 0 ? x1 + it.base1 : x2 + it.base2;
      j.dst = dst;
      const PackTab& pt = op == 0 ? ptab1[i] : ptab2[i];
      j.roff = dp.d_tabs + pt.roff;
      j.koff = dp.d_tabs + pt.koff;
      j.rmi = dp.d_tabs + pt.rmi;
      j.kmi = dp.d_tabs + pt.kmi;
      const OpndDesc& od = it.op[op];
      const int rsp = op == 0 ? kEx1 : kEx2;
      j.nm = 0;
      for (int c = 0; c < od.ncomp; ++c) {
        if (!od.map[c]) continue;
        GCCU_REQUIRE((od.sp1[c] == rsp && od.sp2[c] == kCnt) ||
                         (od.sp1[c] == kCnt && od.sp2[c] == rsp),
                     "string map of an operand must merge an external and a contracted string");
        j.row_is_1[j.nm] = od.sp1[c] == rsp;
        j.n1[j.nm] = od.n1[c];
        j.ldim[j.nm] = od.ldim[c];
        j.map[j.nm] = od.map[c];
        ++j.nm;
      }
      GCCU_REQUIRE(j.R < INT32_MAX && j.K < INT32_MAX, "block too large for the pack kernel");
      j.kfast = op == 0 ? it.kfast1 : it.kfast2;
      j.dkfast = j.kfast;  // the panel is written along the direction it is read
      const int64_t nf = j.kfast ? j.K : j.R;
      j.F = 1;
      while (j.F < 256 && j.F < nf) j.F *= 2;
      return j;
    };
    std::vector<PackJob> gathers;
    std::map<std::pair<size_t, int>, int32_t> gather_of;  // (index in g[kGemmTc], op) -> gather
    for (size_t i = 0; i < P.items.size(); ++i) {
      const ItemDesc& it = P.items[i];
      const Tab& t = toff[i];
      GemmDesc d{};
      d.M = it.M;
      d.N = it.N;
      d.K = it.K;
      d.fac = it.fac;
      d.a = pack_off1[i] >= 0 ? dp.scratch + pack_off1[i] : x1 + it.base1;
      d.aro = dp.d_tabs + t.aro;
      d.ako = dp.d_tabs + t.ako;
      d.akstep = affine_step(tabs, t.ako, it.K);
      d.afast = it.kfast1;  // a packed panel keeps the operand's fast direction
      d.b = pack_off2[i] >= 0 ? dp.scratch + pack_off2[i] : x2 + it.base2;
      d.bco = dp.d_tabs + t.bco;
      d.bko = dp.d_tabs + t.bko;
      d.bkstep = affine_step(tabs, t.bko, it.K);
      d.bfast = it.kfast2;
      d.c = x12 + it.base12;
      d.cro = dp.d_tabs + t.cro;
      d.cco = dp.d_tabs + t.cco;
      d.rowspace = kEx1;
      d.cmapped = it.op[2].nmap > 0;
      for (int q = 0; q < 3; ++q) {
        d.nsp[q] = it.nsp[q];
        for (int c = 0; c < kDevMaxComp; ++c) d.rad[q][c] = it.rad[q][c];
      }
      d.cmap = it.op[2];
      const int kind = kind_of[i];
      if (swapped[i]) {  // thin ex1: ex2 becomes the row space
        std::swap(d.M, d.N);
        std::swap(d.a, d.b);
        std::swap(d.aro, d.bco);
        std::swap(d.ako, d.bko);
        std::swap(d.akstep, d.bkstep);
        std::swap(d.afast, d.bfast);
        std::swap(d.cro, d.cco);
        d.rowspace = kEx2;
      }
      group_of[i] = kind;
      g[kind].push_back(d);
      for (int op = 0; op < 2; ++op)
        if (thingather(i, op)) {
          g[kind].back().ga = (int32_t)gathers.size() + 1;
          gathers.push_back(job_of(i, op, nullptr));
        }
      for (int op = 0; op < 2; ++op) {
        if (!tcgather(i, op)) continue;
        GCCU_REQUIRE(!swapped[i], "tensor-core items keep their operand roles");
        gather_of[{g[kind].size() - 1, op}] = (int32_t)gathers.size();
        gathers.push_back(job_of(i, op, nullptr));
      }
      for (int op = 0; op < 2; ++op) {
        int64_t po = op == 0 ? pack_off1[i] : pack_off2[i];
        if (po < 0) continue;
        PackJob j = job_of(i, op, dp.scratch + po);
        int64_t gx, gy;
        pack_geometry(j, gx, gy);
        if (frozen_op[op]) {
          dp.pack_gx_c = std::max(dp.pack_gx_c, gx);
          dp.pack_gy_c = std::max(dp.pack_gy_c, gy);
          jobs_c.push_back(j);
          const_used[op] = true;
        } else {
          dp.pack_gx = std::max(dp.pack_gx, gx);
          dp.pack_gy = std::max(dp.pack_gy, gy);
          jobs.push_back(j);
        }
      }
    }
    dp.njobs = (int64_t)jobs.size();
    dp.njobs_c = (int64_t)jobs_c.size();
    GCCU_REQUIRE(dp.njobs <= 65535 && dp.pack_gy <= 65535 && dp.pack_gx < INT32_MAX &&
                     dp.njobs_c <= 65535 && dp.pack_gy_c <= 65535 && dp.pack_gx_c < INT32_MAX,
                 "contraction has too many or too large map-addressed operand blocks");
    if (!jobs.empty()) dp.d_jobs = upload(jobs);
    if (!jobs_c.empty()) dp.d_jobs_c = upload(jobs_c);
    if (!gathers.empty()) dp.d_gather = upload(gathers);
    // result blocks written by more than one item need atomic updates
    std::map<const double*, int> writers;
    for (int kind = 0; kind < kGemmKinds; ++kind)
      for (auto& d : g[kind]) writers[d.c]++;
    for (int kind = 0; kind < kGemmKinds; ++kind) {
      int TM, TN0;
      gemm_tile(kind, TM, TN0);
      if (kind == kGemmTc) {
        dp.i8 = precision >= 2 ? i8_slices(precision) : 0;
        for (auto& d : g[kind]) {
          d.tn = dp.i8 ? tc_tile_n(d.N, i8_widest(precision)) : tc_tile_n(d.N);
          d.i8 = dp.i8;
        }
      }
      auto width = [&](const GemmDesc& d) { return kind == kGemmTc ? d.tn : TN0; };
      if (kind == kGemmThin) {  // one launch: the widest item's column count
        dp.thin_nc = 1;
        dp.thin_kmax = 0;
        for (auto& d : g[kind]) dp.thin_nc = std::max(dp.thin_nc, thin_columns(d.N));
        GCCU_REQUIRE(dp.thin_nc <= kThinMaxColumns, "thin tiles take at most 32 columns");
      }
      std::vector<TileDesc> tiles;
      int64_t total = 0;
      for (auto& d : g[kind]) total += ((d.M + TM - 1) / TM) * ((d.N + width(d) - 1) / width(d));
      const int64_t want = 2 * 148;
      for (size_t i = 0; i < g[kind].size(); ++i) {
        GemmDesc& d = g[kind][i];
        const int TN = width(d);
        int64_t mt = (d.M + TM - 1) / TM, nt = (d.N + TN - 1) / TN;
        int64_t ks = 1;
        if (kind == kGemmSmall) {
          ks = std::max<int64_t>(1, (d.K + kSmallChunk - 1) / kSmallChunk);
        } else if (kind == kGemmTc) {  // FP32 (int32) accumulation over at most kTcChunk
          const int64_t ch = dp.i8 ? kI8Chunk : kTcChunk;  // (kI8Chunk) indices
          ks = std::max<int64_t>(1, (d.K + ch - 1) / ch);
        } else if (kind == kGemmThin) {
          // a tile's range of the thin operand fits the staged panel; with
          // few tiles the contraction is split over CTAs as well
          const int64_t lim = dp.thin_nc > 1 ? kThinMaxElems / dp.thin_nc : d.K;
          ks = std::max<int64_t>(1, (d.K + lim - 1) / lim);
          if (total < want && d.K > 64)
            ks = std::max(ks, std::min<int64_t>((d.K + 63) / 64,
                                                (want + total - 1) / std::max<int64_t>(total, 1)));
        } else if (pol.ksplit && total < want && d.K > 4 * kGemmK) {
          ks = std::min<int64_t>((d.K + 255) / 256, (want + total - 1) / std::max<int64_t>(total, 1));
          ks = std::max<int64_t>(ks, 1);
        }
        int64_t kchunk = ((d.K + ks - 1) / ks + kGemmK - 1) / kGemmK * kGemmK;
        d.exclusive = kind != kGemmSmall && !d.cmapped && writers[d.c] == 1 && kchunk >= d.K;
        if (kind == kGemmThin) dp.thin_kmax = std::max(dp.thin_kmax, std::min(kchunk, d.K));
        auto add = [&](int64_t m, int64_t n, int64_t k0) {
          TileDesc tl{};
          tl.item = (int32_t)i;
          tl.m0 = (int32_t)(m * TM);
          tl.n0 = (int32_t)(n * TN);
          tl.k0 = k0;
          tl.k1 = std::min(d.K, k0 + kchunk);
          tiles.push_back(tl);
        };
        if (kind == kGemmTc) {
          // contraction chunk outermost, then groups of column tiles whose
          // split panels of the chunk (8 bytes per element) fit in about 32 MB
          // of L2, then row bands, then the columns of the group: the tiles in
          // flight share one group of column panels while each row band's
          // chunk is reused by the group's tiles one after the other
          const int64_t band = (int64_t)TN * kchunk * 8;
          const int64_t grp = std::max<int64_t>(1, std::min<int64_t>(nt, (32ll << 20) / band));
          for (int64_t k0 = 0; k0 < d.K; k0 += kchunk)
            for (int64_t n0 = 0; n0 < nt; n0 += grp)
              for (int64_t m = 0; m < mt; ++m)
                for (int64_t n = n0; n < std::min(nt, n0 + grp); ++n) add(m, n, k0);
        } else {
          for (int64_t m = 0; m < mt; ++m)
            for (int64_t n = 0; n < nt; ++n)
              for (int64_t k0 = 0; k0 < d.K; k0 += kchunk) add(m, n, k0);
        }
      }
      if (kind == kGemmTc && !g[kind].empty()) {
        // operand panels of every item, row operand then column operand: in
        // the shared workspace, or, for an operand of a frozen list, in the
        // plan's persistent panels (split once, at plan time)
        std::vector<SplitJob> sj, sj_c;
        int64_t off = 0, cs = 0, off_c = 0, cs_c = 0;
        for (size_t i = 0; i < g[kind].size(); ++i) {
          GemmDesc& d = g[kind][i];
          auto gat = [&](int op) {
            auto f = gather_of.find({i, op});
            return f == gather_of.end() ? -1 : f->second;
          };
          for (int op = 0; op < 2; ++op) {
            const int64_t rows = op == 0 ? d.M : d.N;
            const int tr = op == 0 ? kGemmTcM : d.tn;
            const int64_t fl =
                dp.i8 ? i8_panel_floats(rows, tr, d.K, dp.i8) : tc_panel_floats(rows, tr, d.K);
            const int64_t ch = tc_split_chunks(rows, tr, d.K);   // 128 x 32 chunks
            const int64_t nb = tc_split_blocks(rows, tr, d.K);   // pre-pass blocks
            int64_t& po = op == 0 ? d.pa : d.pb;
            if (frozen_op[op]) {
              po = off_c;  // made absolute below
              off_c += fl;
              sj_c.push_back(SplitJob{(int32_t)i, op, cs_c, gat(op), 0, -1});
              cs_c += nb;
              const_used[op] = true;
            } else {
              po = off;
              off += fl;
              // int8 slices of a gathered operand: its chunks kept densely
              // between the two passes
              int64_t stage = -1;
              if (dp.i8 && gat(op) >= 0) {
                stage = off;
                off += ch * kTcGemmChunkFloats;
              }
              sj.push_back(SplitJob{(int32_t)i, op, cs, gat(op), 0, stage});
              cs += nb;
            }
          }
        }
        GCCU_REQUIRE(cs < INT32_MAX && cs_c < INT32_MAX,
                     "tensor-core operands too large for one split launch");
        if (dp.i8) {  // row maxima of every panel, after the panels (one range each)
          dp.max_off = off;
          dp.max_off_c = off_c;
          for (auto& d : g[kind])
            for (int op = 0; op < 2; ++op) {
              const int64_t fl = i8_max_floats(op == 0 ? d.M : d.N, op == 0 ? kGemmTcM : d.tn);
              int64_t& mo = op == 0 ? d.ma : d.mb;
              int64_t& end = frozen_op[op] ? off_c : off;
              mo = end;
              end += fl;
            }
          dp.max_floats = off - dp.max_off;
          dp.max_floats_c = off_c - dp.max_off_c;
        }
        if (off_c) {
          dp.const_panels = (float*)alloc((size_t)off_c * sizeof(float));
          for (auto& d : g[kind]) {
            if (frozen_op[0]) d.pa_ptr = dp.const_panels + d.pa;
            if (frozen_op[1]) d.pb_ptr = dp.const_panels + d.pb;
            if (dp.i8 && frozen_op[0]) d.ma_ptr = reinterpret_cast<double*>(dp.const_panels + d.ma);
            if (dp.i8 && frozen_op[1]) d.mb_ptr = reinterpret_cast<double*>(dp.const_panels + d.mb);
          }
        }
        dp.ws_floats = off;
        dp.nsplit = (int64_t)sj.size();
        dp.split_chunks = cs;
        if (!sj.empty()) dp.d_split = upload(sj);
        dp.nsplit_c = (int64_t)sj_c.size();
        dp.split_chunks_c = cs_c;
        if (!sj_c.empty()) dp.d_split_c = upload(sj_c);
        ensure_tc_ws(off);
      }
      dp.ntiles_g[kind] = (int64_t)tiles.size();
      dp.ndesc_g[kind] = (int64_t)g[kind].size();
      if (!tiles.empty()) {
        dp.d_desc[kind] = upload(g[kind]);
        dp.d_tiles_g[kind] = upload(tiles);
      }
    }
    dp.ntiles = 0;
    for (int kind = 0; kind < kGemmKinds; ++kind) dp.ntiles += dp.ntiles_g[kind];
    if (const_used[0]) dp.const_lists.push_back(dp.list1);
    if (const_used[1] && dp.list2 != dp.list1) dp.const_lists.push_back(dp.list2);
    blap(pstats.desc_s);
    run_const(dp, true);  // the cached panels, made once here
    blap(pstats.const_s);
  }

  // pattern map of one string block for the spin projection
  // (set_spprjmap_kernel, strings/set_spprjmap_kernel.f:60-130): a string is
  // a skeleton string if its spins alternate from the right end (alpha
  // last; the two members of a paired orbital pass); for those and every
  // pattern k = 1..2^n-1, sign * (address of the string with the same
  // orbitals and the spins of pattern k, + 1), sign = std_spsign(string) *
  // std_spsign(result); 0 where a paired orbital would get two equal spins
  const PatternMap& spprjmap(int gid, int idxms, int gam) {
    std::array<int, 3> key{gid, idxms, gam};
    auto it = spprjs.find(key);
    if (it != spprjs.end()) return it->second;
    Graph& g = model.G(gid);
    const int nel = g.nel, nmaps = (1 << nel) - 1;
    const int ms = nel - 2 * (idxms - 1);
    GCCU_REQUIRE(nel % 2 == 0 ? ms == 0 : ms == 1,
                 "spin projection: skeleton strings need Ms 0 (even occupation) or 1/2 (odd)");
    const auto& t = g.table(idxms, gam);
    const int64_t n = g.nstr(idxms, gam);
    std::vector<std::vector<int>> pat(nmaps + 1, std::vector<int>(nel));
    for (int bits = 0; bits <= nmaps; ++bits) {
      const int c = spin_pattern_number(nel, bits);
      for (int i = 0; i < nel; ++i) pat[c][i] = ((bits >> (nel - 1 - i)) & 1) ? -1 : 1;
    }
    PatternMap pm;
    pm.m.assign(n * nmaps, 0);
    pm.skel.assign(n, 0);
    std::vector<int> orb(nel), spn(nel), sf(nel);
    for (int64_t s = 0; s < n; ++s) {
      for (int p = 0; p < nel; ++p) {
        const int v = t[s * nel + p], c = v & 3;
        orb[p] = v >> 2;
        spn[p] = c == 1 ? 1 : (c == 2 ? -1 : 2);
      }
      bool ref = true;
      for (int i = nel - 1, sg = 1; i >= 0; --i, sg = -sg) ref = ref && (spn[i] == sg || spn[i] == 2);
      if (!ref) continue;
      pm.skel[s] = 1;
      for (int c = 1; c <= nmaps; ++c) {
        sf = pat[c];
        bool ok = true;
        for (int i = 0; i < nel && ok; ++i) {
          if (spn[i] != 2 || sf[i] == 2) continue;
          GCCU_REQUIRE(i + 1 < nel && spn[i + 1] == 2, "spin projection: broken spin pair");
          if (sf[i] * sf[i + 1] != -1) ok = false;
          else sf[i] = sf[i + 1] = 2;
        }
        if (!ok) continue;
        pm.m[s * nmaps + c - 1] = spin_sign(spn.data(), nel) * spin_sign(sf.data(), nel) *
                                  (int32_t)(g.address(orb.data(), sf.data()) + 1);
      }
    }
    return spprjs[key] = std::move(pm);
  }

  // partial element offsets of one side of a skeleton distribution: the
  // tuples of component strings (first component fastest) whose strings of
  // two or more electrons are skeleton strings, and per spin case k the sum
  // over the components of (the string of pattern pat[k][i]) * ld[k][i],
  // -1 where a pattern map entry is 0; out is [case][tuple]
  int64_t side_offsets(const std::vector<Comp>& comps, const std::vector<int>& ix,
                       const std::vector<int>& gm, const std::vector<std::vector<int>>& pat,
                       const std::vector<std::vector<int64_t>>& ld, std::vector<int64_t>& out) {
    const size_t nc = comps.size(), ncase = pat.size();
    std::vector<int64_t> len(nc);
    std::vector<const PatternMap*> pm(nc, nullptr);
    int64_t total = 1;
    for (size_t i = 0; i < nc; ++i) {
      len[i] = model.G(comps[i].graph).nstr(ix[i], gm[i]);
      total *= len[i];
      if (comps[i].occ > 1) pm[i] = &spprjmap(comps[i].graph, ix[i], gm[i]);
    }
    std::vector<std::vector<int64_t>> cols(ncase);
    std::vector<int64_t> s(nc, 0);
    for (int64_t t = 0; t < total; ++t) {
      bool skel = true;
      for (size_t i = 0; i < nc; ++i) skel = skel && (!pm[i] || pm[i]->skel[s[i]]);
      if (skel) {
        for (size_t k = 0; k < ncase; ++k) {
          int64_t p = 0;
          for (size_t i = 0; i < nc && p >= 0; ++i) {
            int64_t si = s[i];
            const int m = pat[k][i];
            if (m != 0 && pm[i]) {
              const int nm = (1 << comps[i].occ) - 1;
              const int v = pm[i]->m[si * nm + m - 1];
              if (v == 0) p = -1;
              si = std::abs(v) - 1;
            }
            if (p >= 0) p += si * ld[k][i];
          }
          cols[k].push_back(p);
        }
      }
      for (size_t i = 0; i < nc && ++s[i] == len[i]; ++i) s[i] = 0;
    }
    const int64_t nt = ncase ? (int64_t)cols[0].size() : 0;
    for (auto& c : cols) out.insert(out.end(), c.begin(), c.end());
    return nt;
  }

  // singlet projection plan of a list (spin_prj_list, contract/spin_prj_list.f:
  // 166-199, with spin_prj_blk, contract/spin_prj_blk.f:97-400, and
  // set_spinprj_info, contract/set_spinprj_info.f:55-305, per class)
  DevSpinPrj& spinprj_for(int64_t list_id) {
    auto it = spinprjs.find(list_id);
    if (it != spinprjs.end()) return *it->second;
    GCCU_REQUIRE(!capturing, "spin projection must be run once before it is captured in a graph");
    const ListLayout& L = list(list_id).L;
    GCCU_REQUIRE(L.mst == 0, "spin projection: ms.ne.0 not yet considered (lists of Ms 0 only)");
    const int nsym = model.os.nsym;
    std::vector<SpinPrjDesc> descs[4];
    std::vector<int64_t> tab_t[4], tab_l[4], coef_at[4];
    std::vector<int64_t> tables;
    std::vector<double> coef;
    for (const LayoutBlock& B : L.blk) {
      if (B.len <= 0) continue;
      const std::vector<int> oc = comp_occs(B.c), oa = comp_occs(B.a);
      int np = 0, na_el = 0;
      for (int v : oc) np += v;
      for (int v : oa) na_el += v;
      GCCU_REQUIRE(np == na_el, "spin projection: only particle-conserving operators");
      if (np == 0) continue;  // scalar: its own singlet part
      GCCU_REQUIRE(np <= kSpinPrjMaxPart,
                   "spin projection: at most four creators and annihilators per class");
      const std::vector<int> tc = skeleton_ms(oc), ta = skeleton_ms(oa);
      // reference spins of the skeleton strings per particle: alternating in
      // each component, starting with alpha for Ms +1, beta otherwise
      auto ref_spins = [](const std::vector<int>& occ, const std::vector<int>& ms) {
        std::vector<int> s;
        for (size_t i = 0; i < occ.size(); ++i)
          for (int e = 0, sg = ms[i] == 1 ? 1 : -1; e < occ[i]; ++e, sg = -sg) s.push_back(sg);
        return s;
      };
      const std::vector<int> rc = ref_spins(oc, tc), ra = ref_spins(oa, ta);
      auto pattern = [](const int* spins, const int* ref, int n) {
        if (n == 1) return spins[0] == ref[0] ? 0 : 1;
        GCCU_REQUIRE(spin_bits(ref, n) == spin_ref_bits(n),
                     "spin projection: odd component with skeleton Ms -1/2 (map_type)");
        return spin_pattern_number(n, spin_bits(spins, n));
      };
      // the spin cases: annihilator spins outer, creator spins inner, each
      // from all alpha with the first particle changing fastest; Ms equal on
      // both sides (set_spinprj_info.f set_case)
      std::vector<std::vector<int>> msc, msa, patc, pata;
      const size_t coef0 = coef.size();
      std::vector<int> sa(np, 1), sc(np, 1);
      auto next = [np](std::vector<int>& s) {
        for (int i = 0; i < np; ++i) {
          if (s[i] == 1) {
            s[i] = -1;
            return true;
          }
          s[i] = 1;
        }
        return false;
      };
      for (bool ma = true; ma; ma = next(sa)) {
        std::fill(sc.begin(), sc.end(), 1);
        for (bool mc = true; mc; mc = next(sc)) {
          int tsc = 0, tsa = 0;
          for (int i = 0; i < np; ++i) tsc += sc[i], tsa += sa[i];
          if (tsc != tsa) continue;
          std::vector<int> m1, m2, p1, p2;
          for (size_t i = 0, o = 0; i < oc.size(); o += oc[i], ++i) {
            int m = 0;
            for (int e = 0; e < oc[i]; ++e) m += sc[o + e];
            m1.push_back(m);
            p1.push_back(pattern(sc.data() + o, rc.data() + o, oc[i]));
          }
          for (size_t i = 0, o = 0; i < oa.size(); o += oa[i], ++i) {
            int m = 0;
            for (int e = 0; e < oa[i]; ++e) m += sa[o + e];
            m2.push_back(m);
            p2.push_back(pattern(sa.data() + o, ra.data() + o, oa[i]));
          }
          msc.push_back(m1);
          msa.push_back(m2);
          patc.push_back(p1);
          pata.push_back(p2);
          const std::vector<double> cf = singlet_coupling(sc, sa);
          coef.insert(coef.end(), cf.begin(), cf.end());
        }
      }
      const int ncase = (int)msc.size();
      const int ncoup = (int)((coef.size() - coef0) / ncase);
      int bucket = 0;
      while (kSpinPrjBucket[bucket] < ncase) ++bucket;
      GCCU_REQUIRE(kSpinPrjBucket[bucket] == ncase && ncoup == spin_prj_paths(ncase),
                   "spin projection: unexpected number of spin cases");
      // the side whose first component has leading dimension 1 (the first
      // hpvx type of X,P,V,H with a component; creators before annihilators)
      bool thread_c = false;
      for (int ih = 0; ih < 4; ++ih) {
        const int t = kHpvxSeq[ih];
        bool hc = false, ha = false;
        for (auto& c : B.c) hc = hc || c.hpvx == t;
        for (auto& a : B.a) ha = ha || a.hpvx == t;
        if (hc || ha) {
          thread_c = hc;
          break;
        }
      }
      // skeleton distributions: Ms(A) = Ms(C) = np mod 2 and the skeleton Ms
      // per component, every IRREP distribution
      const int msk = np % 2;
      const int ix_skel = msa_to_idxms(msk, 0, np, np);
      for (int gama = 1; gama <= nsym; ++gama) {
        const int gamc = irrep_mult(gama, L.gamt);
        if (B.gmlen(ix_skel, gama) <= 0) continue;
        MsGam d;
        for (bool first = true; next_msgam(first, d, oc, oa, msk, msk, gamc, gama, nsym);
             first = false) {
          if (d.msc != tc || d.msa != ta) continue;
          std::vector<int> ixc(B.c.size()), ixa(B.a.size());
          int64_t lenc = 1, lena = 1;
          for (size_t i = 0; i < B.c.size(); ++i) {
            ixc[i] = ms_index(B.c[i].occ, d.msc[i]);
            lenc *= model.G(B.c[i].graph).nstr(ixc[i], d.gc[i]);
          }
          for (size_t i = 0; i < B.a.size(); ++i) {
            ixa[i] = ms_index(B.a[i].occ, d.msa[i]);
            lena *= model.G(B.a[i].graph).nstr(ixa[i], d.ga[i]);
          }
          if (lenc == 0 || lena == 0) continue;
          // per case: distribution offset and leading dimensions
          std::vector<int64_t> off(ncase, -1);
          std::vector<std::vector<int64_t>> ldc(ncase), lda(ncase);
          for (int k = 0; k < ncase; ++k) {
            std::vector<int> kxc(B.c.size()), kxa(B.a.size());
            std::vector<int64_t> klc(B.c.size()), kla(B.a.size());
            int kmsa = 0;
            int64_t klen = 1;
            for (size_t i = 0; i < B.c.size(); ++i) {
              kxc[i] = ms_index(B.c[i].occ, msc[k][i]);
              klc[i] = model.G(B.c[i].graph).nstr(kxc[i], d.gc[i]);
              klen *= klc[i];
            }
            for (size_t i = 0; i < B.a.size(); ++i) {
              kxa[i] = ms_index(B.a[i].occ, msa[k][i]);
              kla[i] = model.G(B.a[i].graph).nstr(kxa[i], d.ga[i]);
              klen *= kla[i];
              kmsa += msa[k][i];
            }
            ldc[k].assign(B.c.size(), 0);
            lda[k].assign(B.a.size(), 0);
            op_ldims(B.c, B.a, klc, kla, false, ldc[k].data(), lda[k].data());
            auto f = B.dis.find({msa_to_idxms(kmsa, 0, np, np), gama});
            if (f == B.dis.end()) continue;
            const int64_t did = dist_id(B.c, kxc, d.gc, B.a, kxa, d.ga, nsym);
            for (const Dist& x : f->second)
              if (x.did == did) {
                GCCU_REQUIRE(x.len == klen, "spin projection: distribution length mismatch");
                off[k] = x.off;
              }
          }
          std::vector<int64_t> tcv, tav;
          const int64_t nrc = side_offsets(B.c, ixc, d.gc, patc, ldc, tcv);
          const int64_t nra = side_offsets(B.a, ixa, d.ga, pata, lda, tav);
          if (nrc == 0 || nra == 0) continue;
          // the case's distribution offset goes into the loop side
          std::vector<int64_t>& lv = thread_c ? tav : tcv;
          const int64_t nl = thread_c ? nra : nrc;
          for (int k = 0; k < ncase; ++k)
            for (int64_t j = 0; j < nl; ++j) {
              int64_t& v = lv[k * nl + j];
              v = (v < 0 || off[k] < 0) ? -1 : v + off[k];
            }
          SpinPrjDesc D{};
          D.nt = thread_c ? nrc : nra;
          D.nl = nl;
          tab_t[bucket].push_back((int64_t)tables.size());
          tables.insert(tables.end(), (thread_c ? tcv : tav).begin(), (thread_c ? tcv : tav).end());
          tab_l[bucket].push_back((int64_t)tables.size());
          tables.insert(tables.end(), lv.begin(), lv.end());
          coef_at[bucket].push_back((int64_t)coef0);
          descs[bucket].push_back(D);
        }
      }
    }
    auto sp = std::make_unique<DevSpinPrj>();
    int64_t* d_tab = tables.empty() ? nullptr : upload(tables);
    double* d_coef = coef.empty() ? nullptr : upload(coef);
    for (int b = 0; b < 4; ++b) {
      for (size_t j = 0; j < descs[b].size(); ++j) {
        SpinPrjDesc& D = descs[b][j];
        D.pt = d_tab + tab_t[b][j];
        D.pl = d_tab + tab_l[b][j];
        D.coeff = d_coef + coef_at[b][j];
        sp->maxblocks[b] = std::max(sp->maxblocks[b], spin_prj_blocks(D.nt, D.nl));
      }
      sp->n[b] = (int64_t)descs[b].size();
      if (sp->n[b]) sp->d[b] = upload(descs[b]);
    }
    return *(spinprjs[list_id] = std::move(sp));
  }

  // sym_ab descriptors of one result class (contract/sym_ab_blk.f:170-330)
  void build_flip(DevPlan& dp, DevList& dl, int iblk) {
    ListLayout& L = dl.L;
    GCCU_REQUIRE(L.mst == 0, "sym_ab: open-shell lists are not supported");
    GCCU_REQUIRE(std::abs(L.absym) == 1, "sym_ab: absym must be +-1");
    dp.nflip = 0;
    std::vector<FlipDesc> v = flip_descs(L, iblk, (double)L.absym, dp.flip_maxlen);
    if (!v.empty()) dp.d_flip = upload(v);
    dp.nflip = (int64_t)v.size();
  }

  std::vector<FlipDesc> flip_descs(ListLayout& L, int iblk, double relfac, int64_t& maxlen) {
    LayoutBlock& B = L.blk.at(iblk - 1);
    int nsym = model.os.nsym;
    std::vector<int> oc = comp_occs(B.c), oa = comp_occs(B.a);
    int mscmax = 0, msamax = 0;
    for (int v : oc) mscmax += v;
    for (int v : oa) msamax += v;
    double relfac2 =
        ((((mscmax + msamax) / 2 + 1) * (mscmax - msamax) / 2) % 2 != 0) ? -relfac : relfac;
    auto spsign_dist = [](const std::vector<int>& ms, const std::vector<int>& occ) {
      if (ms.size() <= 1) return 1;
      int trp = 0, nb = 0;
      for (size_t b = 0; b < ms.size(); ++b) {
        int na = (occ[b] + ms[b]) / 2, nbeta = (occ[b] - ms[b]) / 2;
        trp += na * nb;
        nb += nbeta;
      }
      return (trp & 1) ? -1 : 1;
    };
    std::vector<FlipDesc> out;
    maxlen = 0;
    for (int msa = msamax; msa >= 0; msa -= 2) {
      int msc = msa + L.mst;
      if (std::abs(msc) > mscmax) continue;
      int ix1 = msa_to_idxms(msa, L.mst, msamax, mscmax);
      int ix2 = msa_to_idxms(-msa, L.mst, msamax, mscmax);
      for (int gama = 1; gama <= nsym; ++gama) {
        int gamc = irrep_mult(gama, L.gamt);
        if (B.gmlen(ix1, gama) <= 0) continue;
        MsGam d;
        for (bool first = true; next_msgam(first, d, oc, oa, msc, msa, gamc, gama, nsym);
             first = false) {
          std::vector<int> mc2(d.msc), ma2(d.msa);
          for (auto& x : mc2) x = -x;
          for (auto& x : ma2) x = -x;
          int gsign = spsign_dist(d.msc, oc) * spsign_dist(d.msa, oa) * spsign_dist(mc2, oc) *
                      spsign_dist(ma2, oa);
          std::vector<int> ixc(B.c.size()), ixa(B.a.size()), ixc2(B.c.size()), ixa2(B.a.size());
          std::vector<int64_t> lc, la;
          int64_t lenc = 1, lena = 1;
          for (size_t i = 0; i < B.c.size(); ++i) {
            ixc[i] = ms_index(B.c[i].occ, d.msc[i]);
            ixc2[i] = ms_index(B.c[i].occ, mc2[i]);
            lc.push_back(model.G(B.c[i].graph).nstr(ixc[i], d.gc[i]));
            lenc *= lc.back();
          }
          for (size_t i = 0; i < B.a.size(); ++i) {
            ixa[i] = ms_index(B.a[i].occ, d.msa[i]);
            ixa2[i] = ms_index(B.a[i].occ, ma2[i]);
            la.push_back(model.G(B.a[i].graph).nstr(ixa[i], d.ga[i]));
            lena *= la.back();
          }
          if (lenc == 0 || lena == 0) continue;
          const auto& dl1 = B.dis.at({ix1, gama});
          const auto& dl2 = B.dis.at({ix2, gama});
          size_t id1 = 0, id2 = 0;
          int64_t did1 = dist_id(B.c, ixc, d.gc, B.a, ixa, d.ga, nsym);
          int64_t did2 = dist_id(B.c, ixc2, d.gc, B.a, ixa2, d.ga, nsym);
          for (size_t q = 0; q < dl1.size(); ++q)
            if (dl1[q].did == did1) id1 = q;
          for (size_t q = 0; q < dl2.size(); ++q)
            if (dl2[q].did == did2) id2 = q;
          if (msa == 0 && id1 > id2) continue;
          FlipDesc f{};
          f.off1 = dl1[id1].off;
          f.off2 = dl2[id2].off;
          f.lenc = lenc;
          f.lena = lena;
          f.nc = (int32_t)B.c.size();
          f.na = (int32_t)B.a.size();
          std::vector<int64_t> ldc(B.c.size()), lda(B.a.size());
          int64_t ld = 1;
          for (int ih = 0; ih < 4; ++ih) {
            int t = kHpvxSeq[ih];
            for (size_t i = 0; i < B.c.size(); ++i)
              if (B.c[i].hpvx == t) ldc[i] = ld, ld *= lc[i];
            for (size_t i = 0; i < B.a.size(); ++i)
              if (B.a[i].hpvx == t) lda[i] = ld, ld *= la[i];
          }
          for (size_t i = 0; i < B.c.size(); ++i) {
            f.lc[i] = (int32_t)lc[i];
            f.ldc[i] = ldc[i];
            f.fc[i] = flipmap(B.c[i].graph, ixc[i], d.gc[i]);
          }
          for (size_t i = 0; i < B.a.size(); ++i) {
            f.la[i] = (int32_t)la[i];
            f.lda[i] = lda[i];
            f.fa[i] = flipmap(B.a[i].graph, ixa[i], d.ga[i]);
          }
          f.sgn = gsign * relfac2;
          f.same = (f.off1 == f.off2);
          out.push_back(f);
          maxlen = std::max(maxlen, lenc * lena);
        }
      }
    }
    return out;
  }

  double read_red(int slot) {
    double v = 0;
    CUDA_OK(cudaMemcpyAsync(&v, d_red + slot, sizeof(double), cudaMemcpyDeviceToHost, stream));
    CUDA_OK(cudaStreamSynchronize(stream));
    check_err();
    return v;
  }
  // after a synchronisation: did a tensor-core pipeline wait time out?
  void check_err() {
    int h = 0;
    CUDA_OK(cudaMemcpy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
      CUDA_OK(cudaMemset(d_err, 0, sizeof(int)));
      throw Error("a tensor-core pipeline wait timed out in a contraction kernel");
    }
  }
};

std::unique_ptr<Engine> g_eng;

Engine& eng() {
  if (!g_eng) throw Error("gccu_init has not been called");
  return *g_eng;
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

// lists a formula item names
std::vector<int64_t> item_lists(const gccu_formula_item& it) {
  switch (it.command) {
    case GCCU_CMD_TARGET:
    case GCCU_CMD_NEW:
    case GCCU_CMD_DEL:
      return {it.list};
    case GCCU_CMD_ADD:
      return {it.list, it.list_in};
    case GCCU_CMD_CONTR:
      return {it.bc.list_op1, it.bc.list_op2, it.bc.list_res};
    case GCCU_CMD_REORDER:
      return {it.reo.list_ori, it.reo.list_reo};
    default:
      throw Error("formula: unknown command");
  }
}

// a nested entry point's status as an exception (its message kept)
void check_rc(int rc) {
  if (rc != 0) throw Error(g_error);
}

}  // namespace
}  // namespace gccu

using namespace gccu;

extern "C" {

int gccu_init(int64_t device, int64_t memmax_bytes) {
  return guarded([&] {
    GCCU_REQUIRE(!g_eng, "gccu_init called twice");
    if (device >= 0) {
      int n = 0;
      CUDA_OK(cudaGetDeviceCount(&n));
      GCCU_REQUIRE(device < n, "no such CUDA device");
    }
    g_eng = std::make_unique<Engine>((int)device, memmax_bytes);
  });
}

int gccu_finalize(void) {
  return guarded([&] { g_eng.reset(); });
}

int gccu_last_error(char* buf, int64_t len) {
  if (!buf || len <= 0) return 1;
  std::strncpy(buf, g_error.c_str(), (size_t)len - 1);
  buf[len - 1] = '\0';
  return 0;
}

int gccu_register_orbinfo(int64_t nsym, const int64_t* norb) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.have_orbs, "orbital space already registered");
    GCCU_REQUIRE(nsym == 1 || nsym == 2 || nsym == 4 || nsym == 8, "nsym must be 1, 2, 4 or 8");
    e.model.os.nsym = (int)nsym;
    for (int t = 0; t < 4; ++t)
      for (int g = 0; g < 8; ++g) {
        int64_t v = g < nsym ? norb[t * 8 + g] : 0;
        GCCU_REQUIRE(v >= 0 && v < (1 << 20), "orbital count out of range");
        e.model.os.norb[t][g] = (int)v;
      }
    e.model.os.finalize();
    e.have_orbs = true;
  });
}

int gccu_graph_nstr(int64_t type, int64_t nel, int64_t idxms, int64_t gam, int64_t* nstr) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(e.have_orbs, "orbital space not registered");
    GCCU_REQUIRE(type >= 0 && type < 4 && nel >= 0 && nel <= kMaxNel, "bad graph");
    *nstr = e.model.G(e.model.graph((int)type, (int)nel)).nstr((int)idxms, (int)gam);
  });
}

int gccu_graph_index(int64_t type, int64_t nel, const int64_t* orb, const int64_t* spn,
                     int64_t* index) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(e.have_orbs, "orbital space not registered");
    Graph& g = e.model.G(e.model.graph((int)type, (int)nel));
    std::vector<int> o(nel), s(nel);
    for (int i = 0; i < nel; ++i) {
      GCCU_REQUIRE(orb[i] >= 1 && orb[i] <= g.norb, "orbital out of range");
      o[i] = (int)orb[i] - 1;
      s[i] = (int)spn[i];
    }
    *index = g.address(o.data(), s.data());
  });
}

int gccu_graph_strings(int64_t type, int64_t nel, int64_t idxms, int64_t gam, int64_t* orb,
                       int64_t* spn, int64_t maxn, int64_t* n) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(e.have_orbs, "orbital space not registered");
    GCCU_REQUIRE(type >= 0 && type < 4 && nel >= 1 && nel <= kMaxNel, "bad graph");
    Graph& g = e.model.G(e.model.graph((int)type, (int)nel));
    GCCU_REQUIRE(idxms >= 1 && idxms <= nel + 1 && gam >= 1 && gam <= g.nsym, "bad block");
    int64_t ns = g.nstr((int)idxms, (int)gam);
    *n = ns;
    if (ns > maxn) return;
    const auto& t = g.table((int)idxms, (int)gam);
    for (int64_t i = 0; i < ns * nel; ++i) {
      int c = t[i] & 3;
      orb[i] = (t[i] >> 2) + 1;
      spn[i] = c == 1 ? 1 : (c == 2 ? -1 : 2);
    }
  });
}

int gccu_strmap_block(int64_t type, int64_t nel1, int64_t nel2, int64_t idxms1, int64_t idxms2,
                      int64_t gam1, int64_t gam2, int64_t* map, int64_t n) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(e.have_orbs, "orbital space not registered");
    int g1 = e.model.graph((int)type, (int)nel1), g2 = e.model.graph((int)type, (int)nel2);
    MapKey k{g1, g2, (int)idxms1, (int)idxms2, (int)gam1, (int)gam2};
    int64_t n1 = e.model.G(g1).nstr((int)idxms1, (int)gam1),
            n2 = e.model.G(g2).nstr((int)idxms2, (int)gam2);
    GCCU_REQUIRE(n >= n1 * n2, "map buffer too small");
    int32_t* d = e.strmap(k);
    std::vector<int32_t> h(std::max<int64_t>(n1 * n2, 1));
    CUDA_OK(cudaMemcpyAsync(h.data(), d, n1 * n2 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            e.stream));
    CUDA_OK(cudaStreamSynchronize(e.stream));
    for (int64_t i = 0; i < n1 * n2; ++i) map[i] = h[i];
  });
}

int gccu_define_operator(const int64_t* occ, int64_t nblk, int64_t* op_id) {
  return gccu_define_operator_joined(occ, 1, nblk, op_id);
}

int gccu_define_operator_joined(const int64_t* occ, int64_t njoined, int64_t nblk,
                                int64_t* op_id) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(nblk >= 1, "operator without occupation classes");
    GCCU_REQUIRE(njoined >= 1 && njoined <= 8, "njoined must be 1..8");
    Operator op;
    op.nj = (int)njoined;
    for (int64_t b = 0; b < nblk * njoined; ++b) op.occ.push_back(to_occ(occ + 8 * b));
    e.model.ops.push_back(op);
    *op_id = (int64_t)e.model.ops.size();
  });
}

int gccu_register_list(int64_t op_id, int64_t gamt, int64_t mst, int64_t absym, int64_t* list_id,
                       int64_t* len_op) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(e.have_orbs, "orbital space not registered");
    GCCU_REQUIRE(op_id >= 1 && op_id <= (int64_t)e.model.ops.size(), "invalid operator id");
    GCCU_REQUIRE(gamt >= 1 && gamt <= e.model.os.nsym, "invalid total irrep");
    DevList dl;
    dl.L.op = (int)op_id;
    dl.L.gamt = (int)gamt;
    dl.L.mst = (int)mst;
    dl.L.absym = (int)absym;
    e.model.layout(dl.L);
    if (!e.host_only) {
      dl.d = (double*)e.alloc(std::max<int64_t>(dl.L.len, 1) * sizeof(double));
      CUDA_OK(cudaMemsetAsync(dl.d, 0, std::max<int64_t>(dl.L.len, 1) * sizeof(double),
                              e.stream));
    }
    e.lists.push_back(std::move(dl));
    *list_id = (int64_t)e.lists.size();
    *len_op = e.lists.back().L.len;
  });
}

int gccu_register_intermediate(int64_t op_id, int64_t gamt, int64_t mst, int64_t absym,
                               int64_t* list_id, int64_t* len_op) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(e.have_orbs, "orbital space not registered");
    GCCU_REQUIRE(op_id >= 1 && op_id <= (int64_t)e.model.ops.size(), "invalid operator id");
    GCCU_REQUIRE(gamt >= 1 && gamt <= e.model.os.nsym, "invalid total irrep");
    DevList dl;
    dl.L.op = (int)op_id;
    dl.L.gamt = (int)gamt;
    dl.L.mst = (int)mst;
    dl.L.absym = (int)absym;
    e.model.layout(dl.L);
    dl.intermediate = true;
    e.lists.push_back(std::move(dl));
    *list_id = (int64_t)e.lists.size();
    *len_op = e.lists.back().L.len;
  });
}

int gccu_list_block(int64_t list_id, int64_t iblk, int64_t* off, int64_t* len) {
  return guarded([&] {
    DevList& dl = eng().layout_list(list_id);
    GCCU_REQUIRE(iblk >= 1 && iblk <= (int64_t)dl.L.blk.size(), "invalid occupation class");
    *off = dl.L.blk[iblk - 1].off;
    *len = dl.L.blk[iblk - 1].len;
  });
}

int gccu_list_dists(int64_t list_id, int64_t* rows, int64_t maxrows, int64_t* nrows) {
  return guarded([&] {
    DevList& dl = eng().layout_list(list_id);
    int64_t n = 0;
    for (size_t ib = 0; ib < dl.L.blk.size(); ++ib)
      for (auto& kv : dl.L.blk[ib].dis)
        for (size_t d = 0; d < kv.second.size(); ++d, ++n) {
          if (n >= maxrows) continue;
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
    *nrows = n;
  });
}

int gccu_upload_list(int64_t list_id, const double* host, int64_t n) {
  return guarded([&] {
    Engine& e = eng();
    DevList& dl = e.wlist(list_id);
    GCCU_REQUIRE(n == dl.L.len, "upload length differs from the list length");
    CUDA_OK(cudaMemcpyAsync(dl.d, host, n * sizeof(double), cudaMemcpyHostToDevice, e.stream));
    CUDA_OK(cudaStreamSynchronize(e.stream));
  });
}

int gccu_download_list(int64_t list_id, double* host, int64_t n) {
  return guarded([&] {
    Engine& e = eng();
    DevList& dl = e.list(list_id);
    GCCU_REQUIRE(n == dl.L.len, "download length differs from the list length");
    CUDA_OK(cudaMemcpyAsync(host, dl.d, n * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
    CUDA_OK(cudaStreamSynchronize(e.stream));
  });
}

int gccu_zero_list(int64_t list_id) {
  return guarded([&] {
    Engine& e = eng();
    DevList& dl = e.wlist(list_id);
    CUDA_OK(cudaMemsetAsync(dl.d, 0, dl.L.len * sizeof(double), e.stream));
  });
}

int gccu_list_device_ptr(int64_t list_id, void** dptr) {
  return guarded([&] { *dptr = eng().list(list_id).d; });
}

int gccu_reorder(const gccu_reo_desc* reo, double fac, int64_t sign_reo, int64_t update,
                 int64_t type_xret, double* xret) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.host_only, "gccu_reorder needs a device");
    GCCU_REQUIRE(reo, "null reorder descriptor");
    GCCU_REQUIRE(sign_reo == 1 || sign_reo == -1, "sign_reo must be +1 or -1");
    GCCU_REQUIRE(!(e.capturing && type_xret != 0), "type_xret must be 0 inside a graph capture");
    DevReo& dr = e.reo_for(reo);
    DevList& lo = e.list(dr.list_ori);
    DevList& lr = e.wlist(dr.list_reo);
    GCCU_REQUIRE(lo.d != lr.d, "reorder: original and reordered list must differ");
    if (!update)
      CUDA_OK(cudaMemsetAsync(lr.d + dr.reo_off, 0, dr.reo_len * sizeof(double), e.stream));
    if (!dr.plan.items.empty()) {
      launch_reorder(dr.d_items, (int64_t)dr.plan.items.size(), dr.maxlen, lo.d, lr.d,
                     fac * (double)sign_reo, e.stream);
      ++e.launches;
    }
    CUDA_OK(cudaGetLastError());
    if (type_xret == 1) {
      CUDA_OK(cudaMemsetAsync(e.d_red, 0, sizeof(double), e.stream));
      launch_sumsq(lr.d + dr.reo_off, dr.reo_len, e.d_red, e.stream);
      ++e.launches;
      *xret = e.read_red(0);
    } else if (type_xret == 2) {
      CUDA_OK(cudaMemcpyAsync(xret, lr.d + dr.reo_off, sizeof(double), cudaMemcpyDeviceToHost,
                              e.stream));
      CUDA_OK(cudaStreamSynchronize(e.stream));
    }
  });
}

int gccu_trace(int64_t list_op, int64_t iblk_op, int64_t list_res, int64_t iblk_res,
               const int64_t* occ_cnt, double fact, int64_t update, int64_t type_xret,
               double* xret) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.host_only, "gccu_trace needs a device");
    GCCU_REQUIRE(occ_cnt, "null contraction occupation");
    GCCU_REQUIRE(!(e.capturing && type_xret != 0), "type_xret must be 0 inside a graph capture");
    DevReo& dr = e.trace_for(list_op, iblk_op, list_res, iblk_res, occ_cnt);
    DevList& lo = e.list(dr.list_ori);
    DevList& lr = e.wlist(dr.list_reo);
    GCCU_REQUIRE(lo.d != lr.d, "trace: operator and result list must differ");
    if (!update)
      CUDA_OK(cudaMemsetAsync(lr.d + dr.reo_off, 0, dr.reo_len * sizeof(double), e.stream));
    if (!dr.plan.items.empty()) {
      launch_reorder(dr.d_items, (int64_t)dr.plan.items.size(), dr.maxlen, lo.d, lr.d, fact,
                     e.stream);
      ++e.launches;
    }
    CUDA_OK(cudaGetLastError());
    if (type_xret == 1) {
      CUDA_OK(cudaMemsetAsync(e.d_red, 0, sizeof(double), e.stream));
      launch_sumsq(lr.d + dr.reo_off, dr.reo_len, e.d_red, e.stream);
      ++e.launches;
      *xret = e.read_red(0);
    } else if (type_xret == 2) {
      CUDA_OK(cudaMemcpyAsync(xret, lr.d + dr.reo_off, sizeof(double), cudaMemcpyDeviceToHost,
                              e.stream));
      CUDA_OK(cudaStreamSynchronize(e.stream));
    }
  });
}

int gccu_trace_info(int64_t list_op, int64_t iblk_op, int64_t list_res, int64_t iblk_res,
                    const int64_t* occ_cnt, int64_t* ncases, int64_t* nelements) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(occ_cnt, "null contraction occupation");
    DevReo& dr = e.trace_for(list_op, iblk_op, list_res, iblk_res, occ_cnt);
    *ncases = (int64_t)dr.plan.items.size();
    *nelements = dr.plan.elements;
  });
}

int gccu_reorder_info(const gccu_reo_desc* reo, int64_t* ncases, int64_t* nelements) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(reo, "null reorder descriptor");
    DevReo& dr = e.reo_for(reo);
    *ncases = (int64_t)dr.plan.items.size();
    *nelements = dr.plan.elements;
  });
}

int gccu_contract_noalloc(const gccu_bc_desc* bc, double fact, int64_t update, int64_t use_tr) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.host_only, "gccu_contract_noalloc needs a device");
    GCCU_REQUIRE(bc, "null contraction descriptor");
    DevPlan* pp = e.find_plan(bc, use_tr != 0);
    GCCU_REQUIRE(pp, "gccu_contract_noalloc: this contraction has not been planned; planning "
                     "allocates device memory, so run it once through gccu_contract first");
    DevPlan& dp = *pp;
    int64_t ndesc = 0;
    for (int kind = 0; kind < kGemmKinds; ++kind) ndesc += dp.ndesc_g[kind];
    GCCU_REQUIRE(!dp.i8, "gccu_contract_noalloc: precision modes 2 and 3 (int8 slices) are "
                         "not supported by the allocation-free entry point");
    if (dp.scratch_len > kStaticPanelDoubles) {
      std::ostringstream os;
      os << "gccu_contract_noalloc: the operand panels of this contraction need "
         << (double)dp.scratch_len * sizeof(double) / (1 << 20) << " MiB, the fixed scratch holds "
         << kStaticPanelDoubles * sizeof(double) / (1 << 20) << " MiB";
      throw Error(os.str());
    }
    GCCU_REQUIRE(ndesc <= kStaticMaxDescs && dp.njobs + dp.njobs_c <= kStaticMaxJobs,
                 "gccu_contract_noalloc: the contraction has more block contractions than the "
                 "fixed scratch holds descriptors for (16384)");
    // the symbol look-up may load the module lazily, which a stream capture
    // does not allow
    GCCU_REQUIRE(!e.capturing || e.have_static,
                 "gccu_contract_noalloc: the first call of an engine looks up the fixed "
                 "scratch array and must come before any graph capture");
    if (!e.have_static) {  // once per engine (and so per device), with its device current
      CUDA_OK(cudaSetDevice(e.device));
      CUDA_OK(static_scratch(&e.static_ss));
      e.have_static = true;
    }
    const StaticScratch& ss = e.static_ss;
    DevList& r = e.wlist(dp.list12);
    if (!update) {
      CUDA_OK(cudaMemsetAsync(r.d + dp.res_off, 0, dp.res_len * sizeof(double), e.stream));
    }
    // every packed panel, those of frozen operands included, is made in the
    // fixed array (the descriptors are moved there); the split panels of
    // frozen operands stay in the plan
    if (dp.njobs) {
      launch_rebase_jobs(dp.d_jobs, ss.jobs, dp.njobs, dp.scratch, dp.scratch_len, ss.panels,
                         e.stream);
      launch_pack(ss.jobs, dp.njobs, dp.pack_gx, dp.pack_gy, e.stream);
      e.launches += 2;
    }
    if (dp.njobs_c) {
      launch_rebase_jobs(dp.d_jobs_c, ss.jobs + dp.njobs, dp.njobs_c, dp.scratch,
                         dp.scratch_len, ss.panels, e.stream);
      launch_pack(ss.jobs + dp.njobs, dp.njobs_c, dp.pack_gx_c, dp.pack_gy_c, e.stream);
      e.launches += 2;
    }
    const bool remake = e.need_const(dp);
    int64_t first = 0;
    for (int kind = 0; kind < kGemmKinds; ++kind) {
      if (!dp.ntiles_g[kind]) continue;
      GemmDesc* descs = ss.descs + first;
      first += dp.ndesc_g[kind];
      launch_rebase_descs(dp.d_desc[kind], descs, dp.ndesc_g[kind], dp.scratch, dp.scratch_len,
                          ss.panels, e.stream);
      if (kind == kGemmTc && remake && dp.nsplit_c) {  // persistent panels, out of date
        launch_split_tc(descs, dp.d_split_c, dp.nsplit_c, dp.split_chunks_c, dp.d_gather,
                        e.stream);
        ++e.launches;
      }
      if (kind == kGemmTc && dp.nsplit) {  // panels in the engine's existing workspace
        launch_split_tc(descs, dp.d_split, dp.nsplit, dp.split_chunks, dp.d_gather, e.stream);
        ++e.launches;
      }
      int64_t lo, hi;
      e.shard_range(dp.ntiles_g[kind], lo, hi);
      if (hi > lo) e.run_gemm(dp, kind, descs, dp.d_tiles_g[kind] + lo, hi - lo, fact);
      ++e.launches;
    }
    if (dp.plan.use_tr && dp.nflip) {
      launch_sym_ab(dp.d_flip, dp.nflip, r.d, 0.5, dp.flip_maxlen, e.stream);
      ++e.launches;
    }
    CUDA_OK(cudaGetLastError());
    if (remake) {
      bool all_frozen = true;
      for (int l : dp.const_lists) all_frozen = all_frozen && e.list(l).frozen;
      if (all_frozen) dp.const_stale = false;
    } else if (e.capturing) {
      for (int l : dp.const_lists) e.capture_deps.push_back({l, e.list(l).epoch});
    }
    for (int k = 0; k < 8; ++k) e.stats[k] += dp.plan.stats[k];
  });
}

int gccu_plan_items(const gccu_bc_desc* bc, int64_t use_tr, int64_t* rows8, int64_t maxrows,
                    int64_t* nrows) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(bc && nrows, "null argument");
    DevPlan& dp = e.plan_for(bc, use_tr != 0);
    const auto& items = dp.plan.items;
    *nrows = (int64_t)items.size();
    for (int64_t i = 0; i < std::min<int64_t>(maxrows, *nrows); ++i) {
      const ItemDesc& it = items[i];
      int64_t* r = rows8 + 8 * i;
      r[0] = it.M;
      r[1] = it.N;
      r[2] = it.K;
      r[3] = it.op[0].nmap;
      r[4] = it.op[1].nmap;
      r[5] = it.op[2].nmap;
      r[6] = it.kfast1;
      r[7] = it.kfast2;
    }
  });
}

int gccu_plan_info(const gccu_bc_desc* bc, int64_t use_tr, int64_t* nitems, double* stats8) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(bc, "null contraction descriptor");
    DevPlan& dp = e.plan_for(bc, use_tr != 0);
    *nitems = (int64_t)dp.plan.items.size();
    for (int k = 0; k < 8; ++k) stats8[k] = dp.plan.stats[k];
  });
}

int gccu_contract(const gccu_bc_desc* bc, double fact, int64_t update, int64_t use_tr,
                  int64_t type_xret, double* xret) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.host_only, "gccu_contract needs a device");
    GCCU_REQUIRE(bc, "null contraction descriptor");
    GCCU_REQUIRE(!(e.capturing && type_xret != 0), "type_xret must be 0 inside a graph capture");
    DevList& r = e.wlist(bc->list_res);
    DevPlan& dp = e.plan_for(bc, use_tr != 0);
    if (!update) {
      CUDA_OK(cudaMemsetAsync(r.d + dp.res_off, 0, dp.res_len * sizeof(double), e.stream));
    }
    const bool timed = e.profiling && !e.capturing;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (timed) {
      ev0 = e.get_event();
      ev1 = e.get_event();
      CUDA_OK(cudaEventRecord(ev0, e.stream));
    }
    cudaEvent_t evp = timed ? e.get_event() : nullptr;
    e.launch_plan(dp, fact, evp, false);
    if (timed) {
      CUDA_OK(cudaEventRecord(ev1, e.stream));
      dp.pending.push_back({ev0, evp, ev1});
      ++dp.calls;
    }
    if (dp.plan.use_tr && dp.nflip) {
      launch_sym_ab(dp.d_flip, dp.nflip, r.d, 0.5, dp.flip_maxlen, e.stream);
      ++e.launches;
    }
    CUDA_OK(cudaGetLastError());
    for (int k = 0; k < 8; ++k) e.stats[k] += dp.plan.stats[k];
    if (type_xret == 1) {
      CUDA_OK(cudaMemsetAsync(e.d_red, 0, sizeof(double), e.stream));
      launch_sumsq(r.d + dp.res_off, dp.res_len, e.d_red, e.stream);
      ++e.launches;
      *xret = e.read_red(0);
    } else if (type_xret == 2) {
      CUDA_OK(cudaMemcpyAsync(xret, r.d + dp.res_off, sizeof(double), cudaMemcpyDeviceToHost,
                              e.stream));
      CUDA_OK(cudaStreamSynchronize(e.stream));
    }
  });
}

int gccu_put_vec(int64_t list_id, int64_t offset, const void* src, int64_t n) {
  return guarded([&] {
    Engine& e = eng();
    DevList& dl = e.wlist(list_id);
    GCCU_REQUIRE(offset >= 0 && n >= 0 && offset + n <= dl.L.len, "put_vec out of range");
    CUDA_OK(cudaMemcpyAsync(dl.d + offset, src, n * sizeof(double), cudaMemcpyDefault, e.stream));
    CUDA_OK(cudaStreamSynchronize(e.stream));
  });
}

int gccu_get_vec(int64_t list_id, int64_t offset, void* dst, int64_t n) {
  return guarded([&] {
    Engine& e = eng();
    DevList& dl = e.list(list_id);
    GCCU_REQUIRE(offset >= 0 && n >= 0 && offset + n <= dl.L.len, "get_vec out of range");
    CUDA_OK(cudaMemcpyAsync(dst, dl.d + offset, n * sizeof(double), cudaMemcpyDefault, e.stream));
    CUDA_OK(cudaStreamSynchronize(e.stream));
  });
}

int gccu_add_block(double fac, int64_t list_in, int64_t iblk_in, int64_t list_out,
                   int64_t iblk_out, int64_t reset, int64_t type, double* xnorm2) {
  return guarded([&] {
    Engine& e = eng();
    DevList &a = e.list(list_in), &b = e.wlist(list_out);
    GCCU_REQUIRE(iblk_in >= 1 && iblk_in <= (int64_t)a.L.blk.size(), "invalid input class");
    GCCU_REQUIRE(iblk_out >= 1 && iblk_out <= (int64_t)b.L.blk.size(), "invalid output class");
    const LayoutBlock &Bi = a.L.blk[iblk_in - 1], &Bo = b.L.blk[iblk_out - 1];
    GCCU_REQUIRE(Bi.vtx == Bo.vtx && Bi.len == Bo.len, "add_opblk: blocks differ in occupation");
    launch_axpy(b.d + Bo.off, a.d + Bi.off, fac, Bo.len, (int)reset, e.stream);
    ++e.launches;
    if (type == 1) {
      GCCU_REQUIRE(!e.capturing, "type must be 0 inside a graph capture");
      CUDA_OK(cudaMemsetAsync(e.d_red, 0, sizeof(double), e.stream));
      launch_sumsq(b.d + Bo.off, Bo.len, e.d_red, e.stream);
      ++e.launches;
      *xnorm2 = e.read_red(0);
    } else if (type == 2) {
      GCCU_REQUIRE(!e.capturing, "type must be 0 inside a graph capture");
      CUDA_OK(cudaMemcpyAsync(xnorm2, b.d + Bo.off, sizeof(double), cudaMemcpyDeviceToHost,
                              e.stream));
      CUDA_OK(cudaStreamSynchronize(e.stream));
    }
    CUDA_OK(cudaGetLastError());
  });
}

int gccu_add_block_transp(double fac, int64_t list_in, int64_t iblk_in, int64_t list_out,
                          int64_t iblk_out, int64_t tra_in, int64_t tra_out, int64_t reset,
                          int64_t type, double* xnorm2) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.host_only, "gccu_add_block_transp needs a device");
    DevList& b = e.wlist(list_out);
    DevList& a = e.list(list_in);
    GCCU_REQUIRE(a.d != b.d, "add_opblk_transp: input and output list must differ");
    DevTransp& dt = e.transp_for(list_in, iblk_in, list_out, iblk_out, tra_in != 0, tra_out != 0);
    if (reset)
      CUDA_OK(cudaMemsetAsync(b.d + dt.off_out, 0, dt.len_out * sizeof(double), e.stream));
    if (dt.n) {
      launch_add_transp(dt.d, dt.n, a.d, b.d, fac, dt.maxlen, e.stream);
      ++e.launches;
    }
    CUDA_OK(cudaGetLastError());
    if (type == 1) {
      GCCU_REQUIRE(!e.capturing, "type must be 0 inside a graph capture");
      CUDA_OK(cudaMemsetAsync(e.d_red, 0, sizeof(double), e.stream));
      launch_sumsq(b.d + dt.off_out, dt.len_out, e.d_red, e.stream);
      ++e.launches;
      *xnorm2 = e.read_red(0);
    } else if (type == 2) {
      GCCU_REQUIRE(!e.capturing, "type must be 0 inside a graph capture");
      CUDA_OK(cudaMemcpyAsync(xnorm2, b.d + dt.off_out, sizeof(double), cudaMemcpyDeviceToHost,
                              e.stream));
      CUDA_OK(cudaStreamSynchronize(e.stream));
    }
  });
}

int gccu_scale_list(int64_t list_id, double fac) {
  return guarded([&] {
    Engine& e = eng();
    DevList& l = e.wlist(list_id);
    launch_scale(l.d, fac, l.L.len, e.stream);
    ++e.launches;
    CUDA_OK(cudaGetLastError());
  });
}

int gccu_dot_lists(int64_t list_a, int64_t list_b, double* dot) {
  return guarded([&] {
    Engine& e = eng();
    DevList &a = e.list(list_a), &b = e.list(list_b);
    GCCU_REQUIRE(a.L.len == b.L.len, "dot: lists differ in length");
    CUDA_OK(cudaMemsetAsync(e.d_red, 0, sizeof(double), e.stream));
    launch_dot(a.d, b.d, a.L.len, e.d_red, e.stream);
    ++e.launches;
    *dot = e.read_red(0);
  });
}

int gccu_sym_ab(int64_t list_id, int64_t iblk, double prefac, double relfac) {
  return guarded([&] {
    Engine& e = eng();
    DevList& l = e.wlist(list_id);
    GCCU_REQUIRE(iblk >= 1 && iblk <= (int64_t)l.L.blk.size(), "invalid occupation class");
    int64_t maxlen = 0;
    std::vector<FlipDesc> v = e.flip_descs(l.L, (int)iblk, relfac, maxlen);
    if (v.empty()) return;
    FlipDesc* d = e.upload(v);
    launch_sym_ab(d, (int64_t)v.size(), l.d, prefac, maxlen, e.stream);
    ++e.launches;
    CUDA_OK(cudaGetLastError());
  });
}

int gccu_spin_prj_list(int64_t list_id, int64_t s2, double* xnorm2_blk) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.host_only, "gccu_spin_prj_list needs a device");
    GCCU_REQUIRE(s2 == 0, "spin projection: not a singlet case (s2 = 0 only)");
    DevList& l = e.wlist(list_id);
    DevSpinPrj& sp = e.spinprj_for(list_id);
    for (int b = 0; b < 4; ++b) {
      if (sp.n[b] == 0) continue;
      launch_spin_prj(sp.d[b], sp.n[b], kSpinPrjBucket[b], l.d, sp.maxblocks[b], e.stream);
      e.launches += (sp.n[b] + 65534) / 65535;
    }
    CUDA_OK(cudaGetLastError());
    if (!xnorm2_blk) return;
    GCCU_REQUIRE(!e.capturing, "xnorm2_blk must be NULL inside a graph capture");
    const int64_t nb = (int64_t)l.L.blk.size();
    for (int64_t b0 = 0; b0 < nb; b0 += 64) {
      const int64_t m = std::min<int64_t>(64, nb - b0);
      CUDA_OK(cudaMemsetAsync(e.d_red, 0, m * sizeof(double), e.stream));
      for (int64_t i = 0; i < m; ++i) {
        const LayoutBlock& B = l.L.blk[b0 + i];
        if (B.len <= 0) continue;
        launch_sumsq(l.d + B.off, B.len, e.d_red + i, e.stream);
        ++e.launches;
      }
      CUDA_OK(cudaMemcpyAsync(xnorm2_blk + b0, e.d_red, m * sizeof(double),
                              cudaMemcpyDeviceToHost, e.stream));
      CUDA_OK(cudaStreamSynchronize(e.stream));
    }
    e.check_err();
  });
}

int gccu_formula_define(const gccu_formula_item* items, int64_t n, int64_t* formula_id) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(n >= 0 && (items || n == 0), "formula: no items");
    GCCU_REQUIRE(!e.capturing, "formula: define it outside a graph capture");
    FormulaPlan F;
    F.items.assign(items, items + n);
    const int64_t fid = (int64_t)e.formulas.size() + 1;
    std::map<int64_t, int64_t> open;           // intermediate -> item of its [NEW]
    std::vector<std::array<int64_t, 3>> life;  // ([NEW] item, [DEL] item, list)
    std::set<int64_t> made;
    for (int64_t i = 0; i < n; ++i) {
      const gccu_formula_item& it = F.items[i];
      for (int64_t l : item_lists(it)) {
        DevList& dl = e.layout_list(l);
        if (!dl.intermediate) continue;
        GCCU_REQUIRE(dl.formula == 0, "formula: an intermediate belongs to one formula");
        GCCU_REQUIRE(it.command == GCCU_CMD_NEW || open.count(l),
                     "formula: intermediate named outside its [NEW] .. [DEL]");
      }
      switch (it.command) {
        case GCCU_CMD_TARGET:
          GCCU_REQUIRE(it.mult == 0 || it.mult == 1,
                       "formula: a target is projected onto the singlet (mult 1) or not (0)");
          ++F.ntargets;
          break;
        case GCCU_CMD_NEW:
          GCCU_REQUIRE(e.layout_list(it.list).intermediate,
                       "formula: [NEW] of a list that is not an intermediate");
          GCCU_REQUIRE(!made.count(it.list), "formula: an intermediate is created once");
          made.insert(it.list);
          open[it.list] = i;
          break;
        case GCCU_CMD_DEL:
          GCCU_REQUIRE(e.layout_list(it.list).intermediate,
                       "formula: [DEL] of a list that is not an intermediate");
          life.push_back({open[it.list], i, it.list});
          open.erase(it.list);
          break;
        case GCCU_CMD_ADD:
        case GCCU_CMD_CONTR:
        case GCCU_CMD_REORDER:
          break;
        default:
          GCCU_REQUIRE(false, "formula: unknown command");
      }
    }
    for (auto& kv : open) life.push_back({kv.second, n, kv.first});
    std::sort(life.begin(), life.end());
    // first fit in the order of the [NEW]s among the ranges still alive
    struct Range {
      int64_t off, bytes, until;
    };
    std::vector<Range> live;
    std::map<int64_t, int64_t> offset_of;
    for (const auto& lf : life) {
      live.erase(std::remove_if(live.begin(), live.end(),
                                [&](const Range& r) { return r.until < lf[0]; }),
                 live.end());
      std::sort(live.begin(), live.end(),
                [](const Range& a, const Range& b) { return a.off < b.off; });
      const int64_t len = std::max<int64_t>(e.layout_list(lf[2]).L.len, 1);
      const int64_t bytes = (len * (int64_t)sizeof(double) + 255) / 256 * 256;
      int64_t off = 0;
      for (const Range& r : live) {
        if (off + bytes <= r.off) break;
        off = std::max(off, r.off + r.bytes);
      }
      live.push_back({off, bytes, lf[1]});
      offset_of[lf[2]] = off;
      F.arena_bytes = std::max(F.arena_bytes, off + bytes);
      F.sum_bytes += bytes;
    }
    if (!e.host_only && F.arena_bytes > 0) {
      F.arena = (double*)e.alloc(F.arena_bytes);
      CUDA_OK(cudaMemsetAsync(F.arena, 0, F.arena_bytes, e.stream));
    }
    for (const auto& kv : offset_of) {
      DevList& dl = e.layout_list(kv.first);
      dl.formula = fid;
      dl.arena_off = kv.second;
      if (F.arena) dl.d = F.arena + kv.second / (int64_t)sizeof(double);
    }
    e.formulas.push_back(std::move(F));
    *formula_id = fid;
  });
}

int gccu_formula_run(int64_t formula_id, double* xret, int64_t nxret) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.host_only, "gccu_formula_run needs a device");
    GCCU_REQUIRE(formula_id >= 1 && formula_id <= (int64_t)e.formulas.size(),
                 "invalid formula id");
    const FormulaPlan& F = e.formulas[formula_id - 1];
    GCCU_REQUIRE(!xret || nxret >= F.ntargets,
                 "formula: xret is shorter than the number of targets");
    GCCU_REQUIRE(!xret || !e.capturing, "formula: xret must be NULL inside a graph capture");
    int64_t target = 0, mult = 0, ti = -1;
    auto end_target = [&] {
      if (!target) return;
      if (mult > 0) check_rc(gccu_spin_prj_list(target, mult - 1, nullptr));
      if (!xret) return;
      DevList& l = e.list(target);
      if (l.L.len == 1) {
        CUDA_OK(cudaMemcpyAsync(&xret[ti], l.d, sizeof(double), cudaMemcpyDeviceToHost,
                                e.stream));
        CUDA_OK(cudaStreamSynchronize(e.stream));
      } else {
        double d2 = 0;
        check_rc(gccu_dot_lists(target, target, &d2));
        xret[ti] = std::sqrt(d2);
      }
    };
    for (const gccu_formula_item& it : F.items) {
      switch (it.command) {
        case GCCU_CMD_TARGET:
          end_target();
          target = it.list;
          mult = it.mult;
          ++ti;
          if (it.init) check_rc(gccu_zero_list(it.list));
          break;
        case GCCU_CMD_ADD:
          if (it.tra_in || it.tra_out)
            check_rc(gccu_add_block_transp(it.fac, it.list_in, it.iblk_in, it.list, it.iblk_out,
                                           it.tra_in, it.tra_out, it.reset, 0, nullptr));
          else
            check_rc(gccu_add_block(it.fac, it.list_in, it.iblk_in, it.list, it.iblk_out,
                                    it.reset, 0, nullptr));
          break;
        case GCCU_CMD_CONTR:
          check_rc(gccu_contract(&it.bc, it.fac, it.update, it.use_tr, 0, nullptr));
          break;
        case GCCU_CMD_REORDER:
          check_rc(gccu_reorder(&it.reo, it.fac, it.sign_reo, it.update, 0, nullptr));
          break;
        default:  // [NEW] / [DEL]: the arena was laid out when the formula was defined
          break;
      }
    }
    end_target();
  });
}

int gccu_formula_info(int64_t formula_id, int64_t* info4) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(formula_id >= 1 && formula_id <= (int64_t)e.formulas.size(),
                 "invalid formula id");
    const FormulaPlan& F = e.formulas[formula_id - 1];
    info4[0] = F.arena_bytes;
    info4[1] = F.sum_bytes;
    info4[2] = F.ntargets;
    info4[3] = (int64_t)F.items.size();
  });
}

int gccu_intermediate_offset(int64_t list_id, int64_t* offset) {
  return guarded([&] {
    DevList& dl = eng().layout_list(list_id);
    GCCU_REQUIRE(dl.intermediate, "not an intermediate list");
    *offset = dl.arena_off;
  });
}

int gccu_precondition(int64_t list_out, int64_t list_in, int64_t list_diag, double fac,
                      double shift) {
  return guarded([&] {
    Engine& e = eng();
    DevList &o = e.wlist(list_out), &i = e.list(list_in), &d = e.list(list_diag);
    GCCU_REQUIRE(o.L.len == i.L.len && i.L.len == d.L.len, "diavc: lists differ in length");
    launch_diavc(o.d, i.d, d.d, fac, shift, o.L.len, e.stream);
    ++e.launches;
    CUDA_OK(cudaGetLastError());
  });
}

int gccu_graph_begin(void) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.capturing, "graph capture already active");
    CUDA_OK(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
    e.capturing = true;
    e.capture_start = e.launches;
    e.capture_deps.clear();
  });
}

int gccu_graph_end(int64_t* graph_id) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(e.capturing, "no graph capture active");
    cudaGraph_t g = nullptr;
    e.capturing = false;
    CUDA_OK(cudaStreamEndCapture(e.stream, &g));
    cudaGraphExec_t ex = nullptr;
    CUDA_OK(cudaGraphInstantiate(&ex, g, 0));
    cudaGraphDestroy(g);
    e.graphs.push_back(ex);
    e.graph_kernels.push_back(e.launches - e.capture_start);
    e.graph_deps.push_back(e.capture_deps);
    e.launches = e.capture_start;
    *graph_id = (int64_t)e.graphs.size();
  });
}

int gccu_graph_launch(int64_t graph_id) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(graph_id >= 1 && graph_id <= (int64_t)e.graphs.size(), "invalid graph id");
    for (auto& dep : e.graph_deps[graph_id - 1])
      GCCU_REQUIRE(e.list(dep.first).frozen && e.list(dep.first).epoch == dep.second,
                   "the graph reads panels cached from a list that has been unfrozen since it "
                   "was captured: capture it again");
    CUDA_OK(cudaGraphLaunch(e.graphs[graph_id - 1], e.stream));
    e.launches += e.graph_kernels[graph_id - 1];
  });
}

int gccu_sync(void) {
  return guarded([&] {
    Engine& e = eng();
    CUDA_OK(cudaStreamSynchronize(e.stream));
    if (!e.host_only) e.check_err();
  });
}

int gccu_freeze_list(int64_t list_id, int64_t frozen) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.capturing, "a list cannot be frozen or unfrozen during a graph capture");
    DevList& l = e.list(list_id);
    if (frozen) {
      l.frozen = true;
    } else if (l.frozen) {
      l.frozen = false;
      ++l.epoch;
      for (auto& kv : e.plans)
        for (int c : kv.second->const_lists)
          if (c == (int)list_id) kv.second->const_stale = true;
    }
  });
}

int gccu_lp_set_weights(const double* w, int64_t n) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.host_only, "the learned preconditioner needs a device");
    GCCU_REQUIRE(w && n == kLpWeights, "learned preconditioner: wrong number of weights");
    e.lp_alloc_weights();
    CUDA_OK(cudaMemcpyAsync(e.lp_w, w, n * sizeof(double), cudaMemcpyHostToDevice, e.stream));
    CUDA_OK(cudaMemsetAsync(e.lp_m, 0, n * sizeof(double), e.stream));
    CUDA_OK(cudaMemsetAsync(e.lp_v, 0, n * sizeof(double), e.stream));
    CUDA_OK(cudaStreamSynchronize(e.stream));
    e.lp_t = 0;
    e.lp_have_w = true;
  });
}

int gccu_lp_get_weights(double* w, int64_t n) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(e.lp_have_w, "learned preconditioner: no weights loaded");
    GCCU_REQUIRE(w && n == kLpWeights, "learned preconditioner: wrong number of weights");
    CUDA_OK(cudaMemcpyAsync(w, e.lp_w, n * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
    CUDA_OK(cudaStreamSynchronize(e.stream));
  });
}

int gccu_lp_precondition(int64_t list_out, int64_t list_in, int64_t list_diag,
                         int64_t list_prev, double fac, double shift) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(e.lp_have_w, "learned preconditioner: no weights loaded");
    DevList &o = e.wlist(list_out), &i = e.list(list_in), &d = e.list(list_diag);
    const double* prev = nullptr;
    if (list_prev) {
      DevList& p = e.list(list_prev);
      GCCU_REQUIRE(p.L.len == o.L.len, "learned preconditioner: lists differ in length");
      GCCU_REQUIRE(p.d != o.d, "learned preconditioner: previous step and output must differ");
      prev = p.d;
    }
    GCCU_REQUIRE(o.L.len == i.L.len && i.L.len == d.L.len,
                 "learned preconditioner: lists differ in length");
    CUDA_OK(cudaMemsetAsync(e.d_red + 2, 0, 2 * sizeof(double), e.stream));
    launch_lp_sums(i.d, d.d, prev, fac, shift, o.L.len, e.d_red + 2, e.stream);
    launch_lp_apply(o.d, i.d, d.d, prev, fac, shift, o.L.len, e.d_red + 2, e.lp_w, e.stream);
    e.launches += 2;
    CUDA_OK(cudaGetLastError());
  });
}

int gccu_lp_rows(int64_t list_in, int64_t list_diag, int64_t list_prev, int64_t list_amp,
                 double fac, double shift, const int64_t* idx, int64_t n, double* rows) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.host_only, "the learned preconditioner needs a device");
    GCCU_REQUIRE(!e.capturing, "learned preconditioner: sampling reads back to the host");
    DevList &i = e.list(list_in), &d = e.list(list_diag);
    GCCU_REQUIRE(i.L.len == d.L.len, "learned preconditioner: lists differ in length");
    const double* prev = list_prev ? e.list(list_prev).d : nullptr;
    const double* amp = list_amp ? e.list(list_amp).d : nullptr;
    if (list_prev) GCCU_REQUIRE(e.list(list_prev).L.len == i.L.len, "lists differ in length");
    if (list_amp) GCCU_REQUIRE(e.list(list_amp).L.len == i.L.len, "lists differ in length");
    GCCU_REQUIRE(n >= 0 && (n == 0 || (idx && rows)), "null argument");
    for (int64_t r = 0; r < n; ++r)
      GCCU_REQUIRE(idx[r] >= 0 && idx[r] < i.L.len, "learned preconditioner: index out of range");
    if (n == 0) return;
    if (n > e.lp_idx_cap) {
      if (e.lp_idx) e.release(e.lp_idx, (size_t)e.lp_idx_cap * sizeof(int64_t));
      if (e.lp_out) e.release(e.lp_out, (size_t)e.lp_idx_cap * kLpRowLen * sizeof(double));
      e.lp_idx = nullptr;
      e.lp_out = nullptr;
      e.lp_idx = (int64_t*)e.alloc((size_t)n * sizeof(int64_t));
      e.lp_out = (double*)e.alloc((size_t)n * kLpRowLen * sizeof(double));
      e.lp_idx_cap = n;
    }
    CUDA_OK(cudaMemcpyAsync(e.lp_idx, idx, n * sizeof(int64_t), cudaMemcpyHostToDevice, e.stream));
    CUDA_OK(cudaMemsetAsync(e.d_red + 2, 0, 2 * sizeof(double), e.stream));
    launch_lp_sums(i.d, d.d, prev, fac, shift, i.L.len, e.d_red + 2, e.stream);
    launch_lp_rows(i.d, d.d, prev, amp, fac, shift, i.L.len, e.lp_idx, n, e.d_red + 2, e.lp_out,
                   e.stream);
    e.launches += 2;
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaMemcpyAsync(rows, e.lp_out, n * kLpRowLen * sizeof(double),
                            cudaMemcpyDeviceToHost, e.stream));
    CUDA_OK(cudaStreamSynchronize(e.stream));
  });
}

int gccu_lp_load_samples(const double* rows, const double* target, int64_t n) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.host_only, "the learned preconditioner needs a device");
    GCCU_REQUIRE(n >= 1 && rows && target, "learned preconditioner: empty sample set");
    if (n > e.lp_cap) {
      if (e.lp_rows) e.release(e.lp_rows, (size_t)e.lp_cap * kLpRowLen * sizeof(double));
      if (e.lp_tgt) e.release(e.lp_tgt, (size_t)e.lp_cap * sizeof(double));
      e.lp_rows = nullptr;
      e.lp_tgt = nullptr;
      e.lp_rows = (double*)e.alloc((size_t)n * kLpRowLen * sizeof(double));
      e.lp_tgt = (double*)e.alloc((size_t)n * sizeof(double));
      e.lp_cap = n;
    }
    CUDA_OK(cudaMemcpyAsync(e.lp_rows, rows, n * kLpRowLen * sizeof(double),
                            cudaMemcpyHostToDevice, e.stream));
    CUDA_OK(cudaMemcpyAsync(e.lp_tgt, target, n * sizeof(double), cudaMemcpyHostToDevice,
                            e.stream));
    CUDA_OK(cudaStreamSynchronize(e.stream));
    e.lp_nrows = n;
  });
}

int gccu_lp_gradient(double* grad, double* loss) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(e.lp_have_w && e.lp_nrows > 0, "learned preconditioner: weights or samples missing");
    GCCU_REQUIRE(grad && loss, "null argument");
    double* part = e.lp_partials(lp_grad_blocks(e.lp_nrows));
    launch_lp_grad(e.lp_rows, e.lp_tgt, e.lp_nrows, 0, 0, 0, e.lp_w, part, e.lp_grad, e.stream);
    e.launches += 2;
    CUDA_OK(cudaGetLastError());
    std::vector<double> h(kLpWeights + 1);
    CUDA_OK(cudaMemcpyAsync(h.data(), e.lp_grad, h.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, e.stream));
    CUDA_OK(cudaStreamSynchronize(e.stream));
    std::copy(h.begin(), h.begin() + kLpWeights, grad);
    *loss = h[kLpWeights];
  });
}

int gccu_lp_train(int64_t steps, int64_t batch, double lr, int64_t seed, double* loss) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(e.lp_have_w && e.lp_nrows > 0, "learned preconditioner: weights or samples missing");
    GCCU_REQUIRE(steps >= 1 && batch >= 1 && lr > 0, "learned preconditioner: bad training parameters");
    GCCU_REQUIRE(!e.capturing, "learned preconditioner: training is not captured");
    double* part = e.lp_partials(lp_grad_blocks(batch));
    for (int64_t k = 0; k < steps; ++k) {
      launch_lp_grad(e.lp_rows, e.lp_tgt, e.lp_nrows, batch, (uint64_t)seed, (uint64_t)k, e.lp_w,
                     part, e.lp_grad, e.stream);
      launch_lp_adam(e.lp_w, e.lp_m, e.lp_v, e.lp_grad, lr, ++e.lp_t, e.stream);
      e.launches += 3;
    }
    CUDA_OK(cudaGetLastError());
    double l = 0;
    CUDA_OK(cudaMemcpyAsync(&l, e.lp_grad + kLpWeights, sizeof(double), cudaMemcpyDeviceToHost,
                            e.stream));
    CUDA_OK(cudaStreamSynchronize(e.stream));
    if (loss) *loss = l;
  });
}

int gccu_set_shard(int64_t rank, int64_t nranks) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(nranks >= 1 && rank >= 0 && rank < nranks, "shard: need 0 <= rank < nranks");
    e.shard_rank = rank;
    e.shard_n = nranks;
  });
}

int gccu_set_tuning(int64_t mode, int64_t candidate) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(mode >= 0 && mode <= 2, "tuning mode must be 0, 1 or 2");
    if (mode == 2)
      GCCU_REQUIRE(candidate >= 0 && candidate < (int64_t)tile_policies(e.precision).size(),
                   "no such tile-policy candidate for the current precision mode");
    e.tune = (int)mode;
    e.tune_forced = (int)candidate;
  });
}

int gccu_tuning_report(double* rows, int64_t maxrows, int64_t* nrows) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(nrows, "null argument");
    *nrows = (int64_t)e.tune_log.size();
    for (int64_t i = 0; i < std::min<int64_t>(maxrows, *nrows); ++i) {
      const auto& t = e.tune_log[i];
      double* r = rows + 8 * i;
      for (int k = 0; k < 8; ++k) r[k] = -1.0;
      r[0] = (double)t.items;
      r[1] = (double)t.chosen;
      for (size_t c = 0; c < t.ms.size() && c < 6; ++c) r[2 + c] = t.ms[c];
    }
  });
}

int gccu_plan_stats(double* out) {
  return guarded([&] {
    GCCU_REQUIRE(out, "null argument");
    const Engine& e = eng();
    out[0] = (double)e.pstats.plans;
    out[1] = e.pstats.host_s;
    out[2] = e.pstats.maps_s;
    out[3] = e.pstats.tune_s;
    out[4] = e.pstats.build_s;
    out[5] = e.pstats.tables_s;
    out[6] = e.pstats.upload_s;
    out[7] = e.pstats.const_s;
    out[8] = e.pstats.desc_s;
    out[9] = e.pstats.alloc_s;
  });
}

int gccu_set_wait_limit(int64_t polls) {
  return guarded([&] {
    eng().wait_limit = polls < 0 ? kTcWaitLimitDefault : polls;
  });
}

int gccu_mem_info(int64_t* used_bytes, int64_t* cap_bytes) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(used_bytes && cap_bytes, "null argument");
    *used_bytes = e.mem_used;
    *cap_bytes = e.memmax;
  });
}

int gccu_device_info(int64_t* info4) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(!e.host_only, "gccu_device_info needs a device");
    GCCU_REQUIRE(info4, "null argument");
    cudaDeviceProp prop;
    CUDA_OK(cudaGetDeviceProperties(&prop, e.device));
    cudaFuncAttributes attr;
    CUDA_OK(tc_kernel_attributes(&attr));
    info4[0] = 10 * prop.major + prop.minor;
    info4[1] = prop.multiProcessorCount;
    info4[2] = attr.binaryVersion;
    info4[3] = attr.ptxVersion;
  });
}

int gccu_set_precision(int64_t mode) {
  return guarded([&] {
    GCCU_REQUIRE(mode >= 0 && mode <= 3,
                 "precision mode must be 0 (FP64), 1 (split TF32), 2 (five int8 slices) or 3 "
                 "(four int8 slices)");
    eng().precision = (int)mode;
  });
}

int gccu_stats(double* stats8, int64_t* launches) {
  return guarded([&] {
    Engine& e = eng();
    for (int k = 0; k < 8; ++k) stats8[k] = e.stats[k];
    *launches = e.launches;
  });
}

int gccu_event_record(int64_t slot) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(slot >= 0 && slot < 64, "event slot out of range");
    if (!e.slots[slot]) CUDA_OK(cudaEventCreate(&e.slots[slot]));
    CUDA_OK(cudaEventRecord(e.slots[slot], e.stream));
  });
}

int gccu_event_elapsed(int64_t a, int64_t b, double* ms) {
  return guarded([&] {
    Engine& e = eng();
    GCCU_REQUIRE(a >= 0 && a < 64 && b >= 0 && b < 64 && e.slots[a] && e.slots[b],
                 "event slot not recorded");
    CUDA_OK(cudaEventSynchronize(e.slots[b]));
    float f = 0;
    CUDA_OK(cudaEventElapsedTime(&f, e.slots[a], e.slots[b]));
    *ms = f;
  });
}

int gccu_profile(int64_t enable) {
  return guarded([&] { eng().profiling = enable != 0; });
}

int gccu_profile_report(double* rows, int64_t maxrows, int64_t* nrows) {
  return guarded([&] {
    Engine& e = eng();
    CUDA_OK(cudaStreamSynchronize(e.stream));
    int64_t n = 0;
    for (DevPlan* dp : e.plan_order) {
      for (auto& pr : dp->pending) {
        float f = 0, fp = 0;
        CUDA_OK(cudaEventElapsedTime(&f, pr[0], pr[2]));
        CUDA_OK(cudaEventElapsedTime(&fp, pr[0], pr[1]));
        dp->ms += f;
        dp->pack_ms += fp;
        for (auto ev : pr) e.event_pool.push_back(ev);
      }
      dp->pending.clear();
      if (dp->calls == 0) continue;
      if (n < maxrows) {
        double* r = rows + 6 * n;
        r[0] = dp->plan.flops;
        r[1] = (double)dp->calls;
        r[2] = dp->ms;
        r[3] = (double)dp->plan.items.size();
        r[4] = (double)dp->ntiles;
        r[5] = dp->pack_ms;
      }
      ++n;
      dp->calls = 0;
      dp->ms = 0;
      dp->pack_ms = 0;
    }
    *nrows = n;
  });
}

int gccu_reset_stats(void) {
  return guarded([&] {
    Engine& e = eng();
    for (double& s : e.stats) s = 0;
    e.launches = 0;
  });
}

}  // extern "C"

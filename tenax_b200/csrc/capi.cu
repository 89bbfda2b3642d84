// C ABI of the library (declared in include/tenax_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "../../include/tenax_b200.h"
#include "common.cuh"
#include "kernels.cuh"
#include "planner.hpp"
#include "planner_dev.hpp"
#include "svd.hpp"

using namespace tnx;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

static int set_err(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define TNX_TRY(...)                                                         \
  try {                                                                      \
    __VA_ARGS__                                                              \
  } catch (const PlanError& e) {                                             \
    return set_err(e.code, e.msg);                                           \
  } catch (const std::bad_alloc&) {                                          \
    return set_err(TNX_ERR_RUNTIME, "host allocation failed");               \
  } catch (const std::exception& e) {                                        \
    return set_err(TNX_ERR_RUNTIME, e.what());                               \
  }

#define CUDA_OK(x)                                                                                  \
  do {                                                                                              \
    cudaError_t _e = (x);                                                                           \
    if (_e != cudaSuccess) throw PlanError{TNX_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)}; \
  } while (0)

// ---------------------------------------------------------------------------
// device memory
// ---------------------------------------------------------------------------
namespace {
// Plans, operators and batches are created per DMRG site, so their buffers
// come from the device's stream-ordered memory pool (cudaMallocAsync on the
// legacy default stream, which orders against all blocking streams) with the
// pool told to keep freed memory: no device-wide synchronisation per buffer.
void retain_pool_memory() {
  static std::once_flag once;
  std::call_once(once, [] {
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  });
}

struct DevMem {
  void* p = nullptr;
  size_t n = 0;
  DevMem() = default;
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
  ~DevMem() {
    if (p) cudaFreeAsync(p, cudaStreamLegacy);
  }
  void alloc(size_t bytes) {
    if (p) cudaFreeAsync(p, cudaStreamLegacy);
    p = nullptr;
    n = bytes;
    retain_pool_memory();
    if (bytes) CUDA_OK(cudaMallocAsync(&p, bytes, cudaStreamLegacy));
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

template <class T>
void upload(DevMem& m, const std::vector<T>& v, cudaStream_t st = nullptr) {
  m.alloc(v.size() * sizeof(T));
  if (!v.empty()) CUDA_OK(cudaMemcpyAsync(m.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

constexpr int kMaxSlots = 256;
struct PtrTab {
  uint64_t p[kMaxSlots];
};

TensorStruct parse_desc(const tnx_tensor_desc* d, const char* default_subs) {
  if (!d) throw PlanError{TNX_ERR_VALUE, "null tensor descriptor"};
  if (d->n_legs < 0 || d->n_legs > kMaxLegs) throw PlanError{TNX_ERR_UNSUPPORTED, "at most " + std::to_string(kMaxLegs) + " legs per tensor"};
  TensorStruct t;
  t.nl = d->n_legs;
  if (d->subs)
    t.subs = std::string(d->subs);
  else if (default_subs)
    t.subs = default_subs;
  if (static_cast<int>(t.subs.size()) != t.nl) throw PlanError{TNX_ERR_VALUE, "subscripts do not match leg count"};
  t.flows.assign(d->flows, d->flows + t.nl);
  int64_t off = 0;
  t.charges.resize(t.nl);
  for (int l = 0; l < t.nl; ++l) {
    t.charges[l].assign(d->charges + off, d->charges + off + d->leg_dims[l]);
    off += d->leg_dims[l];
  }
  t.finalize_leg_maps();
  t.keys.resize(d->n_blocks);
  for (int64_t b = 0; b < d->n_blocks; ++b) t.keys[b].assign(d->keys + b * t.nl, d->keys + (b + 1) * t.nl);
  t.layout_blocks();
  return t;
}

int img_mode_of(int precision) {
  if (precision == TNX_PREC_FP64) return IMG_F64;
  if (precision == TNX_PREC_BF16X3) return IMG_BF16;
  if (precision == TNX_PREC_TF32) return IMG_TF32;
  throw PlanError{TNX_ERR_VALUE, "unknown precision"};
}

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// tcgen05 groups: MMA K steps (a quarter slab each) that the last K slab of a
// group of extent K needs; the image past K is zero, so skipping the rest is exact
int32_t kk_last_of(int64_t K, int mode) {
  if (mode == IMG_F64 || K <= 0) return 0;
  const int tk = img_geom(mode).tk, step = tk / 4;
  const int64_t last = K - (cdiv(K, tk) - 1) * tk;
  return static_cast<int32_t>(cdiv(last, step));
}

// row length of an H_eff stage-1 result matrix: N rounded up to 4 elements so
// every row starts 16-byte aligned (FP32) and the epilogue stores float4s
int64_t x1_ld(int64_t n) { return (n + 3) / 4 * 4; }

// image geometry of one pair plan for one mode
struct PairGeom {
  std::vector<int64_t> a_tile0, b_tile0;  // per group, in tiles
  std::vector<int32_t> nMt, nNt, nKt;
  int64_t a_tiles = 0, b_tiles = 0;
};

PairGeom pair_geom(const PairPlan& P, int mode) {
  ImgGeom g = img_geom(mode);
  PairGeom G;
  for (auto& gs : P.groups) {
    int32_t mt = static_cast<int32_t>(cdiv(gs.M, g.tm)), nt = static_cast<int32_t>(cdiv(gs.N, g.tm)),
            kt = static_cast<int32_t>(cdiv(gs.K, g.tk));
    G.nMt.push_back(mt);
    G.nNt.push_back(nt);
    G.nKt.push_back(kt);
    G.a_tile0.push_back(G.a_tiles);
    G.b_tile0.push_back(G.b_tiles);
    G.a_tiles += static_cast<int64_t>(mt) * kt;
    G.b_tiles += static_cast<int64_t>(nt) * kt;
  }
  return G;
}

void build_pack(const std::vector<PackSeg>& segs, const PairGeom& G, bool a_side, uint64_t img_base,
                int64_t lo_off, int tile_bytes, int src_slot, std::vector<DevPackSeg>& out,
                std::vector<DevChunk>& chunks, double scale = 1.0) {
  for (auto& s : segs) {
    DevPackSeg d{};
    d.src_off = s.src_off;
    int64_t t0 = a_side ? G.a_tile0[s.group] : G.b_tile0[s.group];
    d.img_addr = img_base + static_cast<uint64_t>(t0) * tile_bytes;
    d.lo_off = lo_off;
    d.row0 = s.row0;
    d.k0 = s.k0;
    d.nKt = G.nKt[s.group];
    d.nlegs = s.nlegs;
    d.src_slot = src_slot;
    d.kcount = 1;
    d.scale = s.neg ? -scale : scale;
    for (int l = 0; l < s.nlegs; ++l) {
      d.dims[l] = s.dims[l];
      d.rstr[l] = s.rstr[l];
      d.kstr[l] = s.kstr[l];
      d.kdstr[l] = s.kdstr[l];
      if (s.kstr[l]) d.kcount *= s.dims[l];
    }
    int seg_id = static_cast<int>(out.size());
    out.push_back(d);
    for (int64_t st = 0; st < s.count; st += 2048) chunks.push_back({seg_id, 0, st, std::min<int64_t>(2048, s.count - st)});
  }
}

void build_tiles(const PairPlan& P, const PairGeom& G, int group_base, std::vector<std::pair<int64_t, DevTile>>& tl) {
  for (size_t g = 0; g < P.groups.size(); ++g)
    for (int mt = 0; mt < G.nMt[g]; ++mt)
      for (int nt = 0; nt < G.nNt[g]; ++nt) tl.push_back({G.nKt[g], DevTile{group_base + static_cast<int>(g), mt, nt, 0}});
}

std::vector<DevTile> sorted_tiles(std::vector<std::pair<int64_t, DevTile>>& tl) {
  std::stable_sort(tl.begin(), tl.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  std::vector<DevTile> out;
  out.reserve(tl.size());
  for (auto& x : tl) out.push_back(x.second);
  return out;
}

void gemm_launch(int mode, const DevMem& groups, const DevMem& tiles, int n_tiles, const DevMem& rowoff,
                 const PtrTab& out_tab, bool out_f64, int32_t* err, const int32_t* skip, cudaStream_t st,
                 DevMem& out_tab_dev) {
  // out_tab travels through a small device array (kernels index it per group)
  CUDA_OK(cudaMemcpyAsync(out_tab_dev.p, out_tab.p, sizeof(PtrTab), cudaMemcpyHostToDevice, st));
  if (mode == IMG_F64)
    launch_gemm_f64(groups.as<DevGroup>(), tiles.as<DevTile>(), n_tiles, rowoff.as<int64_t>(),
                    out_tab_dev.as<uint64_t>(), skip, st);
  else
    launch_gemm_tc(mode, groups.as<DevGroup>(), tiles.as<DevTile>(), n_tiles, rowoff.as<int64_t>(),
                   out_tab_dev.as<uint64_t>(), out_f64, err, skip, st);
}
}  // namespace

// ---------------------------------------------------------------------------
// generic plans
// ---------------------------------------------------------------------------
struct StepDev {
  int mode = -1;
  PairGeom G;
  DevMem a_img, b_img, c_res;  // images and result matrices
  int64_t a_lo = 0, b_lo = 0;
  DevMem packA, chunksA, packB, chunksB, groups, tiles, rowoff, scat, chunksS, out_tab;
  int nA = 0, nB = 0, nT = 0, nS = 0;
  bool res_f32 = false;
};

struct tnx_plan {
  int mode_sem = 0;
  std::vector<TensorStruct> ins;
  std::vector<PairPlan> steps;
  std::vector<int> a_src;  // operand index for step 0, -1 = previous intermediate
  std::vector<int> b_src;
  bool empty_result = false;  // filtered >=3 operands with no common signature
  bool has_scalar = false;    // single-operand plan: B is an internal scalar 1.0
  TensorStruct out;
  bool has_target = false;
  int64_t target = 0;
  double flops = 0.0;
  // device state
  int dev_prec = -1;
  std::vector<std::unique_ptr<StepDev>> dev;
  std::vector<std::unique_ptr<DevMem>> inter;  // intermediate block buffers (fp64)
  DevMem scalar_one;                           // operand for single-tensor plans
  DevMem err_flag, src_tab;
};

static void finalize_plan_out(tnx_plan* p) {
  if (p->empty_result) return;
  p->out = p->steps.back().out;
}

extern "C" {

const char* tnx_last_error(void) { return g_last_error.c_str(); }
int tnx_version(void) { return 1; }

int tnx_valid_blocks(int32_t n_legs, const int32_t* charges, const int64_t* leg_dims, const int32_t* flows,
                     int32_t modulus, int32_t has_target, int64_t target, int64_t* n_keys, int32_t* keys_out,
                     int64_t keys_cap) {
  TNX_TRY({
    std::vector<std::vector<int32_t>> ch(n_legs);
    int64_t off = 0;
    for (int l = 0; l < n_legs; ++l) {
      ch[l].assign(charges + off, charges + off + leg_dims[l]);
      off += leg_dims[l];
    }
    std::vector<int32_t> fl(flows, flows + n_legs);
    auto keys = valid_blocks(ch, fl, modulus, has_target != 0, target);
    *n_keys = static_cast<int64_t>(keys.size());
    if (keys_out) {
      if (keys_cap < static_cast<int64_t>(keys.size()) * n_legs)
        return set_err(TNX_ERR_VALUE, "keys_out capacity too small");
      for (size_t i = 0; i < keys.size(); ++i)
        for (int l = 0; l < n_legs; ++l) keys_out[i * n_legs + l] = keys[i][l];
    }
    return TNX_OK;
  })
}

int tnx_plan_create(const tnx_tensor_desc* ops, int32_t n_ops, const char* out_subs, int32_t mode,
                    int32_t modulus, const int32_t* out_charges, const int64_t* out_leg_dims,
                    const int32_t* out_flows, tnx_plan** plan) {
  return tnx_plan_create_graded(ops, n_ops, out_subs, mode, modulus, out_charges, out_leg_dims, out_flows, 0, plan);
}

}  // extern "C"

namespace {
// Character pairs whose exchange can flip a fermionic contraction's sign
// (contraction/contractor.py:206-285): the input characters in order, each
// mapped to its target slot -- the output characters, then the contracted
// characters by first appearance, a contracted character's two occurrences
// taking consecutive half-slots -- and every inverted pair kept.
std::vector<std::pair<char, char>> inversion_pairs(const std::vector<std::string>& in_subs, const std::string& out) {
  std::string all;
  for (auto& s : in_subs) all += s;
  std::map<char, int> cnt;
  for (char c : all) cnt[c]++;
  std::string target = out;
  for (char c : all)
    if (cnt[c] >= 2 && target.find(c) == std::string::npos) target.push_back(c);
  std::map<char, int> used;
  std::vector<int> perm;
  for (char c : all) {
    const size_t pos = target.find(c);
    if (pos == std::string::npos) throw PlanError{TNX_ERR_VALUE, std::string("free subscript '") + c +
                                                                     "' missing from the output"};
    perm.push_back(static_cast<int>(pos) * 2 + (cnt[c] >= 2 ? used[c] : 0));
    used[c]++;
  }
  std::vector<std::pair<char, char>> pairs;
  for (size_t i = 0; i < all.size(); ++i)
    for (size_t j = i + 1; j < all.size(); ++j)
      if (perm[i] > perm[j]) pairs.push_back({all[i], all[j]});
  return pairs;
}

int parity_of(int64_t q) { return static_cast<int>(((q % 2) + 2) % 2); }

// Fermionic exchange signs of a one- or two-operand plan (contractor.py:
// 460-470), split so that every factor is exact and local: pairs of A's
// characters (free or contracted) depend on the A block alone and negate its
// packed copy, pairs of B's characters likewise, and pairs of one A-free and
// one B-free character depend on the output block and negate its scatter.
void assign_fermionic_signs(tnx_plan* p, const std::string& osubs) {
  PairPlan& P = p->steps[0];
  const TensorStruct& A = p->ins[0];
  const TensorStruct& B = p->ins[1];
  std::vector<std::string> in_subs{A.subs};
  if (!p->has_scalar) in_subs.push_back(B.subs);
  const auto pairs = inversion_pairs(in_subs, osubs);
  auto in = [](const std::string& s, char c) { return s.find(c) != std::string::npos; };
  std::vector<std::pair<char, char>> pa, pb, po;
  for (auto& pr : pairs) {
    if (in(A.subs, pr.first) && in(A.subs, pr.second))
      pa.push_back(pr);
    else if (in(B.subs, pr.first) && in(B.subs, pr.second))
      pb.push_back(pr);
    else
      po.push_back(pr);
  }
  auto neg_of = [&](const std::vector<std::pair<char, char>>& prs, const std::string& subs, const Key& key) {
    int odd = 0;
    for (auto& pr : prs)
      odd ^= parity_of(key[subs.find(pr.first)]) & parity_of(key[subs.find(pr.second)]);
    return odd;
  };
  auto seg_neg = [&](std::vector<PackSeg>& segs, const TensorStruct& T, const std::vector<std::pair<char, char>>& prs) {
    std::map<int64_t, size_t> by_off;
    for (size_t b = 0; b < T.keys.size(); ++b) by_off[T.offs[b]] = b;
    for (auto& sg : segs) {
      auto it = by_off.find(sg.src_off);
      if (it == by_off.end()) throw PlanError{TNX_ERR_RUNTIME, "internal: pack segment without its block"};
      sg.neg = neg_of(prs, T.subs, T.keys[it->second]);
    }
  };
  seg_neg(P.packA, A, pa);
  seg_neg(P.packB, B, pb);
  std::map<int64_t, size_t> out_by_off;
  for (size_t b = 0; b < P.out.keys.size(); ++b) out_by_off[P.out.offs[b]] = b;
  for (auto& sc : P.scatter) {
    auto it = out_by_off.find(sc.dst_off);
    if (it == out_by_off.end()) throw PlanError{TNX_ERR_RUNTIME, "internal: scatter segment without its block"};
    sc.neg = neg_of(po, osubs, P.out.keys[it->second]);
  }
}
}  // namespace

extern "C" {

int tnx_plan_create_graded(const tnx_tensor_desc* ops, int32_t n_ops, const char* out_subs, int32_t mode,
                           int32_t modulus, const int32_t* out_charges, const int64_t* out_leg_dims,
                           const int32_t* out_flows, int32_t fermionic, tnx_plan** plan) {
  TNX_TRY({
    if (n_ops < 1) return set_err(TNX_ERR_VALUE, "contract() requires at least one tensor");
    if (!out_subs) return set_err(TNX_ERR_VALUE, "null output subscripts");
    auto p = std::make_unique<tnx_plan>();
    p->mode_sem = mode;
    for (int i = 0; i < n_ops; ++i) p->ins.push_back(parse_desc(&ops[i], nullptr));
    const std::string osubs(out_subs);
    std::vector<std::vector<int32_t>> och;
    std::vector<int32_t> ofl;
    if (out_charges && out_leg_dims && out_flows) {
      int64_t off = 0;
      for (size_t l = 0; l < osubs.size(); ++l) {
        och.emplace_back(out_charges + off, out_charges + off + out_leg_dims[l]);
        off += out_leg_dims[l];
      }
      ofl.assign(out_flows, out_flows + osubs.size());
    }
    // character counts
    std::map<char, int> cnt;
    for (auto& t : p->ins)
      for (char c : t.subs) cnt[c]++;
    for (auto& kv : cnt)
      if (kv.second > 2) return set_err(TNX_ERR_VALUE, std::string("subscript '") + kv.first + "' used more than twice");
    KeyFilter filt;
    if (mode == TNX_MATCH_FILTERED) {
      if (och.empty() && !osubs.empty())
        return set_err(TNX_ERR_VALUE, "filtered plans need the output leg charges");
      // output target inference (contractor.py:344-355): plain integer sum
      int64_t total = 0;
      for (auto& t : p->ins) {
        if (t.keys.empty()) continue;
        std::set<int64_t> tg;
        for (auto& k : t.keys) {
          int64_t s = 0;
          for (int l = 0; l < t.nl; ++l) s += static_cast<int64_t>(t.flows[l]) * k[l];
          tg.insert(s);
        }
        if (tg.size() == 1) total += *tg.begin();
      }
      p->has_target = total != 0;
      p->target = total;
      auto vk = valid_blocks(och, ofl, modulus, p->has_target, total);
      filt.active = true;
      for (auto& k : vk) filt.allowed[k] = 1;
      if (n_ops >= 3) {
        // signature intersection (contractor.py:373-403)
        std::set<char> contracted;
        for (auto& kv : cnt)
          if (kv.second >= 2) contracted.insert(kv.first);
        std::vector<std::set<Key>> sigs;
        std::vector<size_t> siglen;
        for (auto& t : p->ins) {
          std::vector<std::pair<char, int>> pos;
          for (int l = 0; l < t.nl; ++l)
            if (contracted.count(t.subs[l])) pos.push_back({t.subs[l], l});
          std::sort(pos.begin(), pos.end());
          std::set<Key> s;
          for (auto& k : t.keys) {
            Key sg;
            for (auto& pp : pos) sg.push_back(k[pp.second]);
            s.insert(sg);
          }
          sigs.push_back(s);
          siglen.push_back(pos.size());
        }
        std::set<Key> common = sigs[0];
        for (size_t i = 1; i < sigs.size(); ++i) {
          std::set<Key> nx;
          for (auto& k : common)
            if (sigs[i].count(k)) nx.insert(k);
          common.swap(nx);
        }
        if (common.empty()) {
          p->empty_result = true;
          p->out.nl = static_cast<int>(osubs.size());
          p->out.subs = osubs;
          p->out.charges = och;
          p->out.flows = ofl;
          p->out.finalize_leg_maps();
          *plan = p.release();
          return TNX_OK;
        }
        return set_err(TNX_ERR_UNSUPPORTED,
                       "filtered contraction of >=3 operands with a common contracted signature is not supported; "
                       "contract pairwise");
      }
    }
    if (n_ops == 1) {
      // a single operand: contract with a scalar (no contracted legs)
      TensorStruct one;
      one.nl = 0;
      one.keys.push_back({});
      one.dims.push_back({});
      one.offs.push_back(0);
      one.total = 1;
      p->ins.push_back(one);
      p->has_scalar = true;
      p->steps.push_back(plan_pair(p->ins[0], p->ins[1], osubs, filt, och.empty() ? nullptr : &och,
                                   ofl.empty() ? nullptr : &ofl));
      p->a_src.push_back(0);
      p->b_src.push_back(1);
    } else {
      TensorStruct cur = p->ins[0];
      for (int i = 1; i < n_ops; ++i) {
        const TensorStruct& B = p->ins[i];
        std::string step_out;
        if (i == n_ops - 1) {
          step_out = osubs;
        } else {
          for (char c : cur.subs)
            if (B.subs.find(c) == std::string::npos) step_out.push_back(c);
          for (char c : B.subs)
            if (cur.subs.find(c) == std::string::npos) step_out.push_back(c);
        }
        const bool last = i == n_ops - 1;
        PairPlan pp = plan_pair(cur, B, step_out, last ? filt : KeyFilter{}, last && !och.empty() ? &och : nullptr,
                                last && !ofl.empty() ? &ofl : nullptr);
        p->a_src.push_back(i == 1 ? 0 : -1);
        p->b_src.push_back(i);
        cur = pp.out;
        // the intermediate's per-leg charge maps come from its blocks
        cur.cdim.assign(cur.nl, {});
        for (size_t b = 0; b < cur.keys.size(); ++b)
          for (int l = 0; l < cur.nl; ++l) cur.cdim[l][cur.keys[b][l]] = cur.dims[b][l];
        p->steps.push_back(std::move(pp));
      }
    }
    for (auto& s : p->steps) p->flops += s.flops;
    if (fermionic) {
      if (p->steps.size() != 1)
        return set_err(TNX_ERR_UNSUPPORTED, "fermionic contraction of three or more operands: contract pairwise");
      assign_fermionic_signs(p.get(), osubs);
    }
    finalize_plan_out(p.get());
    *plan = p.release();
    return TNX_OK;
  })
}

int tnx_plan_output(const tnx_plan* plan, int64_t* n_blocks, int32_t* keys, int64_t* total_elems,
                    int32_t* has_target, int64_t* target) {
  TNX_TRY({
    const TensorStruct& o = plan->out;
    if (n_blocks) *n_blocks = static_cast<int64_t>(o.keys.size());
    if (total_elems) *total_elems = o.total;
    if (has_target) *has_target = plan->has_target ? 1 : 0;
    if (target) *target = plan->target;
    if (keys)
      for (size_t b = 0; b < o.keys.size(); ++b)
        for (int l = 0; l < o.nl; ++l) keys[b * o.nl + l] = o.keys[b][l];
    return TNX_OK;
  })
}

double tnx_plan_flops(const tnx_plan* plan) { return plan ? plan->flops : 0.0; }

int tnx_plan_workspace(const tnx_plan* plan, int32_t precision, size_t* bytes) {
  TNX_TRY({
    (void)plan;
    (void)precision;
    *bytes = 0;  // plans own their scratch
    return TNX_OK;
  })
}

static void plan_build_device(tnx_plan* p, int precision) {
  const int mode = img_mode_of(precision);
  const ImgGeom ig = img_geom(mode);
  p->dev.clear();
  p->inter.clear();
  p->err_flag.alloc(sizeof(int32_t));
  CUDA_OK(cudaMemset(p->err_flag.p, 0, sizeof(int32_t)));
  if (p->has_scalar) upload(p->scalar_one, std::vector<double>{1.0});
  for (size_t s = 0; s + 1 < p->steps.size(); ++s) {
    auto m = std::make_unique<DevMem>();
    m->alloc(std::max<int64_t>(1, p->steps[s].out.total) * sizeof(double));
    p->inter.push_back(std::move(m));
  }
  for (size_t s = 0; s < p->steps.size(); ++s) {
    const PairPlan& P = p->steps[s];
    auto d = std::make_unique<StepDev>();
    d->mode = mode;
    d->G = pair_geom(P, mode);
    const int split = mode == IMG_BF16 ? 2 : 1;
    d->a_img.alloc(std::max<int64_t>(1, d->G.a_tiles) * ig.tile_bytes * split);
    d->b_img.alloc(std::max<int64_t>(1, d->G.b_tiles) * ig.tile_bytes * split);
    d->a_lo = d->G.a_tiles * ig.tile_bytes;
    d->b_lo = d->G.b_tiles * ig.tile_bytes;
    d->res_f32 = mode != IMG_F64;
    // result matrices
    std::vector<int64_t> res_off;
    int64_t roff = 0;
    for (auto& g : P.groups) {
      res_off.push_back(roff);
      roff += g.M * g.N;
    }
    d->c_res.alloc(std::max<int64_t>(1, roff) * (d->res_f32 ? 4 : 8));
    std::vector<DevPackSeg> pa, pb;
    std::vector<DevChunk> ca, cb;
    build_pack(P.packA, d->G, true, reinterpret_cast<uint64_t>(d->a_img.p), d->a_lo, ig.tile_bytes, 0, pa, ca);
    build_pack(P.packB, d->G, false, reinterpret_cast<uint64_t>(d->b_img.p), d->b_lo, ig.tile_bytes, 1, pb, cb);
    upload(d->packA, pa);
    upload(d->chunksA, ca);
    upload(d->packB, pb);
    upload(d->chunksB, cb);
    d->nA = static_cast<int>(ca.size());
    d->nB = static_cast<int>(cb.size());
    std::vector<DevGroup> gr;
    std::vector<int64_t> ro;
    for (size_t g = 0; g < P.groups.size(); ++g) {
      DevGroup x{};
      x.a_addr = reinterpret_cast<uint64_t>(d->a_img.p) + static_cast<uint64_t>(d->G.a_tile0[g]) * ig.tile_bytes;
      x.b_addr = reinterpret_cast<uint64_t>(d->b_img.p) + static_cast<uint64_t>(d->G.b_tile0[g]) * ig.tile_bytes;
      x.a_lo = d->a_lo;
      x.b_lo = d->b_lo;
      x.rowoff0 = static_cast<int64_t>(ro.size());
      x.M = static_cast<int32_t>(P.groups[g].M);
      x.N = static_cast<int32_t>(P.groups[g].N);
      x.nKt = d->G.nKt[g];
      x.kk_last = kk_last_of(P.groups[g].K, d->mode);
      x.out_slot = 0;
      x.scale = 1.0;
      gr.push_back(x);
      for (int64_t r = 0; r < P.groups[g].M; ++r) ro.push_back(res_off[g] + r * P.groups[g].N);
    }
    upload(d->groups, gr);
    upload(d->rowoff, ro);
    std::vector<std::pair<int64_t, DevTile>> tl;
    build_tiles(P, d->G, 0, tl);
    auto tiles = sorted_tiles(tl);
    upload(d->tiles, tiles);
    d->nT = static_cast<int>(tiles.size());
    std::vector<DevScatSeg> ss;
    std::vector<DevChunk> cs;
    for (auto& sc : P.scatter) {
      DevScatSeg x{};
      x.dst_off = sc.dst_off;
      x.ld = P.groups[sc.group].N;
      x.src_base = res_off[sc.group] + static_cast<int64_t>(sc.row0) * x.ld + sc.col0;
      x.nlegs = sc.nlegs;
      x.neg = sc.neg;
      for (int l = 0; l < sc.nlegs; ++l) {
        x.dims[l] = sc.dims[l];
        x.rstr[l] = sc.rstr[l];
        x.cstr[l] = sc.cstr[l];
      }
      int id = static_cast<int>(ss.size());
      ss.push_back(x);
      for (int64_t st = 0; st < sc.count; st += 2048) cs.push_back({id, 0, st, std::min<int64_t>(2048, sc.count - st)});
    }
    upload(d->scat, ss);
    upload(d->chunksS, cs);
    d->nS = static_cast<int>(cs.size());
    d->out_tab.alloc(sizeof(PtrTab));
    p->dev.push_back(std::move(d));
  }
  CUDA_OK(cudaDeviceSynchronize());
  p->dev_prec = precision;
}

int tnx_plan_execute(tnx_plan* plan, const double* const* inputs, double* out, int32_t precision, void* workspace,
                     size_t workspace_bytes, void* stream) {
  TNX_TRY({
    (void)workspace;
    (void)workspace_bytes;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (plan->empty_result) return TNX_OK;
    if (plan->dev_prec != precision) plan_build_device(plan, precision);
    const ImgGeom ig = img_geom(img_mode_of(precision));
    const int split = precision == TNX_PREC_BF16X3 ? 2 : 1;
    for (size_t s = 0; s < plan->steps.size(); ++s) {
      StepDev& d = *plan->dev[s];
      const PairPlan& P = plan->steps[s];
      const double* a_ptr = plan->a_src[s] >= 0 ? inputs[plan->a_src[s]] : plan->inter[s - 1]->as<double>();
      const double* b_ptr = plan->has_scalar ? plan->scalar_one.as<double>() : inputs[plan->b_src[s]];
      double* o_ptr = (s + 1 == plan->steps.size()) ? out : plan->inter[s]->as<double>();
      PtrTab src{};
      src.p[0] = reinterpret_cast<uint64_t>(a_ptr);
      src.p[1] = reinterpret_cast<uint64_t>(b_ptr);
      // the pack kernels read operand pointers from a device table
      DevMem& srcdev = plan->src_tab;
      if (!srcdev.p) srcdev.alloc(sizeof(PtrTab));
      CUDA_OK(cudaMemcpyAsync(srcdev.p, &src, 2 * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
      CUDA_OK(cudaMemsetAsync(d.a_img.p, 0, std::max<int64_t>(1, d.G.a_tiles) * ig.tile_bytes * split, st));
      CUDA_OK(cudaMemsetAsync(d.b_img.p, 0, std::max<int64_t>(1, d.G.b_tiles) * ig.tile_bytes * split, st));
      launch_pack(srcdev.as<uint64_t>(), d.packA.as<DevPackSeg>(), d.chunksA.as<DevChunk>(), d.nA, d.mode, nullptr,
                  st);
      launch_pack(srcdev.as<uint64_t>(), d.packB.as<DevPackSeg>(), d.chunksB.as<DevChunk>(), d.nB, d.mode, nullptr,
                  st);
      PtrTab ot{};
      ot.p[0] = reinterpret_cast<uint64_t>(d.c_res.p);
      gemm_launch(d.mode, d.groups, d.tiles, d.nT, d.rowoff, ot, false, plan->err_flag.as<int32_t>(), nullptr, st,
                  d.out_tab);
      if (P.out.total > 0)
        CUDA_OK(cudaMemsetAsync(o_ptr, 0, P.out.total * sizeof(double), st));
      launch_scatter(d.c_res.p, d.res_f32, o_ptr, d.scat.as<DevScatSeg>(), d.chunksS.as<DevChunk>(), d.nS, st);
      CUDA_OK(cudaGetLastError());
    }
    return TNX_OK;
  })
}

void tnx_plan_destroy(tnx_plan* plan) { delete plan; }

// ---------------------------------------------------------------------------
// leg fusion
// ---------------------------------------------------------------------------
struct tnx_fuse_plan {
  FusePlan F;
  DevMem segs, chunks;
  int n_chunks = 0;
  bool on_device = false;
};

int tnx_fuse_plan_create(const tnx_tensor_desc* in, int32_t modulus, int32_t axis_a, int32_t axis_b,
                         int32_t fused_flow, tnx_fuse_plan** out) {
  TNX_TRY({
    if (!out) return set_err(TNX_ERR_VALUE, "null output pointer");
    *out = nullptr;
    if (!in) return set_err(TNX_ERR_VALUE, "null tensor descriptor");
    std::string subs(static_cast<size_t>(std::max(0, in->n_legs)), 'a');
    for (int l = 0; l < in->n_legs; ++l) subs[l] = static_cast<char>('a' + l);
    TensorStruct T = parse_desc(in, in->subs ? nullptr : subs.c_str());
    auto p = std::make_unique<tnx_fuse_plan>();
    p->F = plan_fuse(T, axis_a, axis_b, fused_flow, modulus);
    *out = p.release();
    return TNX_OK;
  })
}

int tnx_fuse_plan_output(const tnx_fuse_plan* p, int32_t* fused_charges, int64_t* n_fused, int64_t* n_blocks,
                         int32_t* keys, int64_t* total) {
  TNX_TRY({
    if (!p) return set_err(TNX_ERR_VALUE, "null fuse plan");
    const FusePlan& F = p->F;
    if (n_fused) *n_fused = static_cast<int64_t>(F.fused_charges.size());
    if (fused_charges) std::memcpy(fused_charges, F.fused_charges.data(), F.fused_charges.size() * sizeof(int32_t));
    if (n_blocks) *n_blocks = static_cast<int64_t>(F.out.keys.size());
    if (keys)
      for (size_t b = 0; b < F.out.keys.size(); ++b)
        std::memcpy(keys + b * F.out.nl, F.out.keys[b].data(), F.out.nl * sizeof(int32_t));
    if (total) *total = F.out.total;
    return TNX_OK;
  })
}

int tnx_fuse_execute(tnx_fuse_plan* p, const double* in, double* out, void* stream) {
  TNX_TRY({
    if (!p) return set_err(TNX_ERR_VALUE, "null fuse plan");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!p->on_device) {
      std::vector<DevCopySeg> segs;
      std::vector<DevChunk> chunks;
      for (const CopySeg& c : p->F.segs) {
        DevCopySeg d{};
        d.src_off = c.src_off;
        d.dst_off = c.dst_off;
        d.nlegs = c.nlegs;
        for (int l = 0; l < c.nlegs; ++l) {
          d.dims[l] = c.dims[l];
          d.dstr[l] = c.dstr[l];
        }
        const int id = static_cast<int>(segs.size());
        segs.push_back(d);
        for (int64_t s = 0; s < c.count; s += 2048) chunks.push_back({id, 0, s, std::min<int64_t>(2048, c.count - s)});
      }
      upload(p->segs, segs);
      upload(p->chunks, chunks);
      p->n_chunks = static_cast<int>(chunks.size());
      CUDA_OK(cudaDeviceSynchronize());
      p->on_device = true;
    }
    if (p->F.out.total > 0) CUDA_OK(cudaMemsetAsync(out, 0, p->F.out.total * sizeof(double), st));
    launch_strided_copy(in, out, p->segs.as<DevCopySeg>(), p->chunks.as<DevChunk>(), p->n_chunks, st);
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

void tnx_fuse_plan_destroy(tnx_fuse_plan* p) { delete p; }

int tnx_fuse_row_map(const int32_t* charges_a, int64_t d_a, int32_t flow_a, const int32_t* charges_b, int64_t d_b,
                     int32_t flow_b, int32_t fused_flow, int32_t modulus, int64_t* map) {
  TNX_TRY({
    if (d_a < 0 || d_b < 0 || (!map && d_a * d_b > 0)) return set_err(TNX_ERR_VALUE, "fuse_row_map: bad arguments");
    std::vector<int32_t> qa(charges_a, charges_a + d_a), qb(charges_b, charges_b + d_b);
    auto m = fuse_row_map(qa, flow_a, qb, flow_b, fused_flow, modulus);
    if (!m.empty()) std::memcpy(map, m.data(), m.size() * sizeof(int64_t));
    return TNX_OK;
  })
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Contraction without device allocation.
//
// Some callers cannot call cudaMalloc: an XLA custom call runs inside a
// process where JAX has already reserved most of the GPU's memory for its own
// pool, and code that must not allocate behind its host framework's allocator
// cannot create the per-plan buffers tnx_plan_execute owns.  For them,
// tnx_plan_execute_static carves every buffer it needs (operand images,
// sector result matrices, intermediates of multi-operand plans and the
// device-side index tables) out of one file-scope device array of
// kStaticArenaBytes.  Every GPU that loads this library holds that array
// until the process exits.  The array is shared by all calls and keeps the
// previous call's contents, so each call zeroes what must start at zero (the
// operand images and the output); calls that overlap on the GPU race on it.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kStaticArenaBytes = static_cast<size_t>(16) << 20;  // 16 MiB
__device__ __align__(256) unsigned char g_static_arena[kStaticArenaBytes];

std::mutex g_static_mu;
std::map<int, uint8_t*> g_static_ptr;  // device ordinal -> device address of g_static_arena

// Device address of the arena for the current device (host code must not use
// the symbol itself: on the host it is only a stand-in).  Looked up once per
// device, with that device current.
uint8_t* static_arena_for_current_device() {
  int dev = 0;
  CUDA_OK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_static_mu);
  auto it = g_static_ptr.find(dev);
  if (it != g_static_ptr.end()) return it->second;
  void* ptr = nullptr;
  CUDA_OK(cudaGetSymbolAddress(&ptr, g_static_arena));
  g_static_ptr[dev] = static_cast<uint8_t*>(ptr);
  return static_cast<uint8_t*>(ptr);
}

struct ArenaCursor {
  uint8_t* base;
  size_t used = 0;
  uint8_t* take(size_t bytes) {
    used = (used + 255) & ~static_cast<size_t>(255);
    uint8_t* p = base + used;
    used += bytes;
    return p;
  }
};
}  // namespace

extern "C" int tnx_plan_execute_static(const tnx_plan* plan, const double* const* inputs, double* out,
                                       void* stream) {
  TNX_TRY({
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (plan->empty_result) return TNX_OK;
    const int mode = IMG_F64;
    const ImgGeom ig = img_geom(mode);
    // layout pass (sizes only), then the real pass against the arena
    struct Tables {
      std::vector<DevPackSeg> pa, pb;
      std::vector<DevChunk> ca, cb, cs;
      std::vector<DevGroup> gr;
      std::vector<int64_t> ro;
      std::vector<DevTile> tiles;
      std::vector<DevScatSeg> ss;
    };
    uint8_t* arena = static_arena_for_current_device();
    for (int pass = 0; pass < 2; ++pass) {
      ArenaCursor cur{pass == 0 ? nullptr : arena};
      uint64_t* src_tab = reinterpret_cast<uint64_t*>(cur.take(2 * sizeof(uint64_t)));
      uint64_t* out_tab = reinterpret_cast<uint64_t*>(cur.take(sizeof(uint64_t)));
      double* one = reinterpret_cast<double*>(cur.take(sizeof(double)));
      std::vector<double*> inter(plan->steps.size(), nullptr);
      for (size_t s = 0; s + 1 < plan->steps.size(); ++s)
        inter[s] = reinterpret_cast<double*>(cur.take(std::max<int64_t>(1, plan->steps[s].out.total) * 8));
      for (size_t s = 0; s < plan->steps.size(); ++s) {
        const PairPlan& P = plan->steps[s];
        PairGeom G = pair_geom(P, mode);
        const size_t a_bytes = std::max<int64_t>(1, G.a_tiles) * ig.tile_bytes;
        const size_t b_bytes = std::max<int64_t>(1, G.b_tiles) * ig.tile_bytes;
        uint8_t* a_img = cur.take(a_bytes);
        uint8_t* b_img = cur.take(b_bytes);
        int64_t roff = 0;
        std::vector<int64_t> res_off;
        for (auto& g : P.groups) {
          res_off.push_back(roff);
          roff += g.M * g.N;
        }
        double* res = reinterpret_cast<double*>(cur.take(std::max<int64_t>(1, roff) * 8));
        Tables T;
        build_pack(P.packA, G, true, reinterpret_cast<uint64_t>(a_img), 0, ig.tile_bytes, 0, T.pa, T.ca);
        build_pack(P.packB, G, false, reinterpret_cast<uint64_t>(b_img), 0, ig.tile_bytes, 1, T.pb, T.cb);
        for (size_t g = 0; g < P.groups.size(); ++g) {
          DevGroup x{};
          x.a_addr = reinterpret_cast<uint64_t>(a_img) + static_cast<uint64_t>(G.a_tile0[g]) * ig.tile_bytes;
          x.b_addr = reinterpret_cast<uint64_t>(b_img) + static_cast<uint64_t>(G.b_tile0[g]) * ig.tile_bytes;
          x.rowoff0 = static_cast<int64_t>(T.ro.size());
          x.M = static_cast<int32_t>(P.groups[g].M);
          x.N = static_cast<int32_t>(P.groups[g].N);
          x.nKt = G.nKt[g];
          x.out_slot = 0;
          x.scale = 1.0;
          T.gr.push_back(x);
          for (int64_t r = 0; r < P.groups[g].M; ++r) T.ro.push_back(res_off[g] + r * P.groups[g].N);
        }
        std::vector<std::pair<int64_t, DevTile>> tl;
        build_tiles(P, G, 0, tl);
        T.tiles = sorted_tiles(tl);
        for (auto& sc : P.scatter) {
          DevScatSeg x{};
          x.dst_off = sc.dst_off;
          x.ld = P.groups[sc.group].N;
          x.src_base = res_off[sc.group] + static_cast<int64_t>(sc.row0) * x.ld + sc.col0;
          x.nlegs = sc.nlegs;
          x.neg = sc.neg;
          for (int l = 0; l < sc.nlegs; ++l) {
            x.dims[l] = sc.dims[l];
            x.rstr[l] = sc.rstr[l];
            x.cstr[l] = sc.cstr[l];
          }
          const int id = static_cast<int>(T.ss.size());
          T.ss.push_back(x);
          for (int64_t k = 0; k < sc.count; k += 2048)
            T.cs.push_back({id, 0, k, std::min<int64_t>(2048, sc.count - k)});
        }
        auto put = [&](const auto& v) {
          using E = typename std::decay_t<decltype(v)>::value_type;
          E* d = reinterpret_cast<E*>(cur.take(std::max<size_t>(1, v.size()) * sizeof(E)));
          if (pass == 1 && !v.empty())
            CUDA_OK(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(E), cudaMemcpyHostToDevice, st));
          return d;
        };
        DevPackSeg* dpa = put(T.pa);
        DevChunk* dca = put(T.ca);
        DevPackSeg* dpb = put(T.pb);
        DevChunk* dcb = put(T.cb);
        DevGroup* dgr = put(T.gr);
        int64_t* dro = put(T.ro);
        DevTile* dtl = put(T.tiles);
        DevScatSeg* dss = put(T.ss);
        DevChunk* dcs = put(T.cs);
        if (cur.used > kStaticArenaBytes)
          return set_err(TNX_ERR_VALUE, "contraction needs " + std::to_string(cur.used) +
                                            " bytes of device scratch; the static arena of tnx_plan_execute_static "
                                            "holds " + std::to_string(kStaticArenaBytes) + " bytes");
        if (pass == 0) continue;
        const double* a_ptr = plan->a_src[s] >= 0 ? inputs[plan->a_src[s]] : inter[s - 1];
        // a single-operand plan pairs its operand with the scalar 1.0: its
        // caller passes one input pointer, so inputs[b_src] is never read
        const double* b_ptr = plan->has_scalar ? nullptr : inputs[plan->b_src[s]];
        if (plan->has_scalar) {
          const double v1 = 1.0;
          CUDA_OK(cudaMemcpyAsync(one, &v1, sizeof(double), cudaMemcpyHostToDevice, st));
          b_ptr = one;
        }
        double* o_ptr = (s + 1 == plan->steps.size()) ? out : inter[s];
        const uint64_t src2[2] = {reinterpret_cast<uint64_t>(a_ptr), reinterpret_cast<uint64_t>(b_ptr)};
        const uint64_t res1 = reinterpret_cast<uint64_t>(res);
        CUDA_OK(cudaMemcpyAsync(src_tab, src2, sizeof(src2), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemcpyAsync(out_tab, &res1, sizeof(res1), cudaMemcpyHostToDevice, st));
        CUDA_OK(cudaMemsetAsync(a_img, 0, a_bytes, st));
        CUDA_OK(cudaMemsetAsync(b_img, 0, b_bytes, st));
        launch_pack(src_tab, dpa, dca, static_cast<int>(T.ca.size()), mode, nullptr, st);
        launch_pack(src_tab, dpb, dcb, static_cast<int>(T.cb.size()), mode, nullptr, st);
        launch_gemm_f64(dgr, dtl, static_cast<int>(T.tiles.size()), dro, out_tab, nullptr, st);
        if (P.out.total > 0) CUDA_OK(cudaMemsetAsync(o_ptr, 0, P.out.total * sizeof(double), st));
        launch_scatter(res, false, o_ptr, dss, dcs, static_cast<int>(T.cs.size()), st);
        CUDA_OK(cudaGetLastError());
      }
    }
    return TNX_OK;
  })
}

namespace {
// ---------------------------------------------------------------------------
// Fused H_eff stages 1-3 (heff_fused.cu): the per-operator layout.  A tile is
// (MPO pair (q_c, q_d), c-tile of cc values, d-tile of 128); every input
// block (q_b, q_p, q_q) and physical element pair (p, q) of the pair is one
// MMA chain: A = the theta block's (p, q) slice as rows d, B = the L block's
// rows (c, b) of the tile's c values, both K = a.
// ---------------------------------------------------------------------------
struct FusedBlk {
  int32_t th_blk, pp, qq, l_blk, mb, ma, n_mma, col, slot0, slot_stride;
};
struct FusedLayout {
  int32_t cc = 0;
  std::vector<std::vector<FusedBlk>> blocks;  // per MPO pair
  std::vector<int64_t> lp_off;                // per L block: byte offset of its panels in one plane (-1: unused)
  std::vector<int32_t> lp_nmma, lp_nKt;
  int64_t lp_bytes = 0;                       // bytes of one plane (hi; lo follows for BF16x3)
  std::map<std::array<int32_t, 3>, int64_t> thp_tile0;  // (theta block, p, q) -> first 16 KB tile
  int64_t thp_tiles = 0;
  std::string why_not;  // non-empty: the structure does not fit the fused kernel
};

int32_t round16(int64_t x) { return static_cast<int32_t>((x + 15) / 16 * 16); }

// Every X1 block of every MPO pair as (L block, theta block, p, q): the
// stage-1 product L[a, b, c] theta[a, p, q, d] over a that fills the input
// slots (b, p, q) of the pair (q_c, q_d).  Returns why the structure has no
// such decomposition (empty: it has).
std::string pair_blocks(const HeffPlan& H, std::vector<std::vector<FusedBlk>>& blocks) {
  std::map<std::pair<int32_t, int32_t>, int> l_by_bc;  // (q_b, q_c) -> L block
  for (size_t i = 0; i < H.L.keys.size(); ++i) {
    auto key = std::make_pair(H.L.keys[i][1], H.L.keys[i][2]);
    if (l_by_bc.count(key)) return "an L block is not determined by its (q_b, q_c)";
    l_by_bc[key] = static_cast<int>(i);
  }
  std::map<Key, int> th_by_key;
  for (size_t i = 0; i < H.th.keys.size(); ++i) th_by_key[H.th.keys[i]] = static_cast<int>(i);
  blocks.assign(H.pairs.size(), {});
  for (size_t p = 0; p < H.pairs.size(); ++p) {
    const MpoPair& mp = H.pairs[p];
    for (size_t ii = 0; ii < mp.ins.size(); ++ii) {
      const MpoIn& in = mp.ins[ii];
      const Key& ik = H.mpo_in_keys[p][ii];  // (q_b, q_p, q_q)
      auto lit = l_by_bc.find({ik[0], mp.qc});
      if (lit == l_by_bc.end()) return "internal: no L block for an X1 block";
      const int lb = lit->second;
      const int32_t qa = H.L.keys[lb][0];
      auto tit = th_by_key.find(Key{qa, ik[1], ik[2], mp.qd});
      if (tit == th_by_key.end()) return "internal: no theta block for an X1 block";
      const int tb = tit->second;
      const auto& ld = H.L.dims[lb];
      const auto& td = H.th.dims[tb];
      if (ld[0] != td[0] || ld[1] != in.mb || ld[2] != mp.mc || td[1] != in.mp || td[2] != in.mq || td[3] != mp.md)
        return "internal: inconsistent block dims";
      for (int pp = 0; pp < in.mp; ++pp)
        for (int qq = 0; qq < in.mq; ++qq)
          blocks[p].push_back(FusedBlk{tb, pp, qq, lb, in.mb, static_cast<int32_t>(ld[0]), 0, 0,
                                       mp.in_slot0[ii] + pp * in.mq + qq, in.mp * in.mq});
    }
  }
  return "";
}

FusedLayout fused_layout(const HeffPlan& H, int mode, int32_t cc_req) {
  FusedLayout F;
  const int tk = img_geom(mode).tk;
  for (const MpoPair& mp : H.pairs)
    if (mp.n_in_slots > kFusedMaxSlots || mp.n_out_slots > kFusedMaxOut) {
      F.why_not = "an MPO pair has more than " + std::to_string(kFusedMaxSlots) + " input or " +
                  std::to_string(kFusedMaxOut) + " output slots";
      return F;
    }
  F.why_not = pair_blocks(H, F.blocks);
  if (!F.why_not.empty()) return F;
  // c values per tile: the largest that fits every pair's blocks side by side
  // in one accumulator, each block's panel within the kernel's operand stage
  int64_t max_mc = 1;
  for (auto& mp : H.pairs) max_mc = std::max<int64_t>(max_mc, mp.mc);
  auto fits = [&](int32_t cc) {
    for (auto& bl : F.blocks) {
      int64_t cols = 0;
      for (auto& b : bl) {
        const int32_t n = round16(static_cast<int64_t>(b.mb) * cc);
        if (n > kFusedMaxN) return false;
        cols += n;
      }
      if (cols > kFusedAccCols) return false;
    }
    return true;
  };
  int32_t cc = 0;
  if (cc_req > 0) {
    if (fits(cc_req)) cc = cc_req;
  } else {
    for (int32_t c = 1; c <= std::min<int64_t>(32, max_mc); ++c)
      if (fits(c)) cc = c;
  }
  if (cc == 0) {
    F.why_not = "no c-tile fits the tensor-memory accumulator";
    return F;
  }
  F.cc = cc;
  // TMEM columns, the L panel layout and the theta panel tiles
  F.lp_off.assign(H.L.keys.size(), -1);
  F.lp_nmma.assign(H.L.keys.size(), 0);
  F.lp_nKt.assign(H.L.keys.size(), 0);
  for (auto& bl : F.blocks) {
    int32_t col = 0;
    for (auto& b : bl) {
      b.n_mma = round16(static_cast<int64_t>(b.mb) * cc);
      b.col = col;
      col += b.n_mma;
      if (F.lp_off[b.l_blk] < 0) {
        const auto& ld = H.L.dims[b.l_blk];
        F.lp_nmma[b.l_blk] = b.n_mma;
        F.lp_nKt[b.l_blk] = static_cast<int32_t>(cdiv(ld[0], tk));
        F.lp_off[b.l_blk] = F.lp_bytes;
        F.lp_bytes += cdiv(ld[2], cc) * F.lp_nKt[b.l_blk] * static_cast<int64_t>(b.n_mma) * 128;
      }
      const std::array<int32_t, 3> tkey{b.th_blk, b.pp, b.qq};
      if (!F.thp_tile0.count(tkey)) {
        const auto& td = H.th.dims[b.th_blk];
        F.thp_tile0[tkey] = F.thp_tiles;
        F.thp_tiles += cdiv(td[3], 128) * cdiv(td[0], tk);
      }
    }
  }
  return F;
}

// Routed stages 1-3 (mixed precisions): the stage-1 GEMM groups and operand
// images of the unfused path, with an epilogue that writes every output slot
// with a single W_l W_r term straight into the stage-4 image and keeps X1
// (FP32) only for the input slots that multi-term output slots read; the MPO
// kernel then forms just those outputs.
struct RoutedLayout {
  std::vector<std::vector<int32_t>> out_terms;  // per pair and output slot: number of terms
  std::vector<std::vector<char>> in_kept;       // per pair and input slot: read by a multi-term output
};

// The destinations of one X1 row class (an L block's b: rows rkey .. rkey +
// mc - 1 of a stage-1 group) in one column class (a theta block's (p, q): the
// d range starting at column ckey).
struct RoutedEntry {
  int32_t g = 0, rkey = 0, ckey = 0, mc = 0, md_pad = 0;
  std::vector<DevRoute> routes;
};

RoutedLayout routed_layout(const HeffPlan& H) {
  RoutedLayout F;
  F.out_terms.resize(H.pairs.size());
  F.in_kept.resize(H.pairs.size());
  for (size_t p = 0; p < H.pairs.size(); ++p) {
    const MpoPair& mp = H.pairs[p];
    F.out_terms[p].assign(mp.n_out_slots, 0);
    F.in_kept[p].assign(mp.n_in_slots, 0);
    for (const MpoTerm& t : mp.terms) ++F.out_terms[p][t.out_slot];
    for (const MpoTerm& t : mp.terms)
      if (F.out_terms[p][t.out_slot] > 1) F.in_kept[p][t.in_slot] = 1;
  }
  return F;
}
}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// H_eff
// ---------------------------------------------------------------------------
// Schedule of an operator that was given none: routed stages 1-3 for the
// mixed precisions at or above kRoutedMinFlops (on the cylinder MPO the routed
// epilogue gains from chi ~ 1024 on, where sectors are wide enough that a
// warp's rows share one destination list), the three kernels below it.
constexpr int32_t kAutoFuse = -1;
constexpr double kRoutedMinFlops = 5e9;
static int32_t resolved_fuse(int32_t fuse, double flops) {
  return fuse != kAutoFuse ? fuse : (flops >= kRoutedMinFlops ? 2 : 0);
}

struct tnx_heff {
  HeffPlan H;
  int prec = -1;
  DevMem l_img, r_img;  // stage-1 A image (L), stage-4 B image (R)
  int64_t l_lo = 0, r_lo = 0;
  PairGeom g1, g4;
  bool terms_ready = false;
  double out_scale = 1.0;  // 2^(eL + eR): undoes the operator range scaling
  // schedule requested by tnx_heff_set_schedule, applied by tnx_heff_set_operators
  int32_t sched_fuse = kAutoFuse, sched_cc = 0;
  int32_t plan_prec = TNX_PREC_FP64;  // precision given to tnx_heff_create_for
  // fused stages 1-3 (mixed precisions): layout and L panels (hi plane, then lo)
  bool fused = false;
  FusedLayout fl;
  DevMem lp_img;
  // routed stages 1-3 (mixed precisions): which output slots the epilogue writes
  bool routed = false;
  RoutedLayout rl;
};

int tnx_heff_create(const tnx_tensor_desc* L, const tnx_tensor_desc* theta, const tnx_tensor_desc* Wl,
                    const tnx_tensor_desc* Wr, const tnx_tensor_desc* R, tnx_heff** h) {
  return tnx_heff_create_for(L, theta, Wl, Wr, R, TNX_PREC_FP64, h);
}

int tnx_heff_create_for(const tnx_tensor_desc* L, const tnx_tensor_desc* theta, const tnx_tensor_desc* Wl,
                        const tnx_tensor_desc* Wr, const tnx_tensor_desc* R, int32_t precision, tnx_heff** h) {
  TNX_TRY({
    auto x = std::make_unique<tnx_heff>();
    TensorStruct tL = parse_desc(L, "abc"), tT = parse_desc(theta, "apqd"), tWl = parse_desc(Wl, "bpse"),
                 tWr = parse_desc(Wr, "eqtf"), tR = parse_desc(R, "dfg");
    tL.subs = "abc";
    tT.subs = "apqd";
    tWl.subs = "bpse";
    tWr.subs = "eqtf";
    tR.subs = "dfg";
    // the mixed precisions read X1 with aligned 32-byte loads (see tnx_heff_set_operators)
    x->H = plan_heff(tL, tT, tWl, tWr, tR, img_mode_of(precision) == IMG_F64 ? 1 : kMpoKAlign);
    x->plan_prec = precision;
    *h = x.release();
    return TNX_OK;
  })
}

int tnx_heff_set_schedule(tnx_heff* h, const tnx_heff_schedule* sched) {
  if (!h || !sched) return set_err(TNX_ERR_VALUE, "null argument");
  if (sched->c_per_tile < 0 || sched->c_per_tile > 32) return set_err(TNX_ERR_VALUE, "c_per_tile must be in [0, 32]");
  if (sched->fuse_mpo < -1 || sched->fuse_mpo > 2) return set_err(TNX_ERR_VALUE, "fuse_mpo must be -1, 0, 1 or 2");
  h->sched_fuse = sched->fuse_mpo;
  h->sched_cc = sched->c_per_tile;
  return TNX_OK;
}

int tnx_heff_get_schedule(const tnx_heff* h, tnx_heff_schedule* sched) {
  if (!h || !sched) return set_err(TNX_ERR_VALUE, "null argument");
  TNX_TRY({
    if (h->prec < 0) {
      // before tnx_heff_set_operators: the schedule the planned precision would get
      const int mode = img_mode_of(h->plan_prec);
      bool fz = false, rt = false;
      int32_t cc = 0;
      const int32_t fz_req = resolved_fuse(h->sched_fuse, h->H.flops);
      if (mode != IMG_F64 && fz_req == 1 && h->H.closed && h->H.s4_separable) {
        const FusedLayout fl = fused_layout(h->H, mode, h->sched_cc);
        fz = fl.why_not.empty();
        cc = fl.cc;
      }
      if (mode != IMG_F64 && fz_req == 2 && h->H.closed && h->H.s4_separable) rt = true;
      sched->fuse_mpo = fz ? 1 : (rt ? 2 : 0);
      sched->c_per_tile = fz ? cc : 0;
      return TNX_OK;
    }
    sched->fuse_mpo = h->fused ? 1 : (h->routed ? 2 : 0);
    sched->c_per_tile = h->fused ? h->fl.cc : 0;
    return TNX_OK;
  })
}

int tnx_heff_closed(const tnx_heff* h, int32_t* closed) {
  *closed = (h->H.closed && h->H.s4_separable) ? 1 : 0;
  return TNX_OK;
}

int tnx_heff_out_keys(const tnx_heff* h, int64_t* n_keys, int32_t* keys) {
  *n_keys = static_cast<int64_t>(h->H.out_keys.size());
  if (keys)
    for (size_t i = 0; i < h->H.out_keys.size(); ++i)
      for (int l = 0; l < 4; ++l) keys[i * 4 + l] = h->H.out_keys[i][l];
  return TNX_OK;
}

double tnx_heff_flops(const tnx_heff* h) { return h ? h->H.flops : 0.0; }

int tnx_heff_set_operators(tnx_heff* h, const double* L, const double* Wl, const double* Wr, const double* R,
                           int32_t precision, void* stream) {
  TNX_TRY({
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    HeffPlan& H = h->H;
    if (!H.closed || !H.s4_separable)
      return set_err(TNX_ERR_VALUE, "H_eff output keys are not a subset of theta's keys; extend theta first");
    const int mode = img_mode_of(precision);
    const ImgGeom ig = img_geom(mode);
    const int split = mode == IMG_BF16 ? 2 : 1;
    // the mixed paths read X1 in FP32 with 32-byte vector loads: every d range
    // of the stage-1 result starts on a multiple of 8 columns
    const int want_align = mode == IMG_F64 ? 1 : kMpoKAlign;
    if (H.x1_align != want_align) {
      const TensorStruct tL = H.L, tT = H.th, tWl = H.Wl, tWr = H.Wr, tR = H.R;
      H = plan_heff(tL, tT, tWl, tWr, tR, want_align);
    }
    // W data to host for the fused MPO terms
    std::vector<double> wl(H.Wl.total), wr(H.Wr.total);
    if (H.Wl.total) CUDA_OK(cudaMemcpyAsync(wl.data(), Wl, H.Wl.total * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (H.Wr.total) CUDA_OK(cudaMemcpyAsync(wr.data(), Wr, H.Wr.total * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    heff_mpo_terms(H, wl, wr);
    h->terms_ready = true;
    h->g1 = pair_geom(H.s1, mode);
    h->g4 = pair_geom(H.s4, mode);
    // fused stages 1-3 where the schedule asks for it and the structure fits
    h->fused = false;
    h->fl = FusedLayout{};
    const int32_t fz_req = resolved_fuse(h->sched_fuse, H.flops);
    if (mode != IMG_F64 && fz_req == 1) {
      h->fl = fused_layout(H, mode, h->sched_cc);
      for (auto& mp : H.pairs)
        if (mp.terms.size() > static_cast<size_t>(kFusedMaxTerms))
          h->fl.why_not = "an MPO pair has more than " + std::to_string(kFusedMaxTerms) + " W_l W_r terms";
      h->fused = h->fl.why_not.empty();
    }
    h->routed = false;
    h->rl = RoutedLayout{};
    if (mode != IMG_F64 && fz_req == 2) {
      h->rl = routed_layout(H);
      h->routed = true;
    }
    // the stage-1 A image (L) serves the unfused and routed paths
    const bool plain = !h->fused;
    h->l_img.alloc(plain ? std::max<int64_t>(1, h->g1.a_tiles) * ig.tile_bytes * split : 0);
    h->r_img.alloc(std::max<int64_t>(1, h->g4.b_tiles) * ig.tile_bytes * split);
    h->l_lo = h->g1.a_tiles * ig.tile_bytes;
    h->r_lo = h->g4.b_tiles * ig.tile_bytes;
    if (h->l_img.n) CUDA_OK(cudaMemsetAsync(h->l_img.p, 0, h->l_img.n, st));
    CUDA_OK(cudaMemsetAsync(h->r_img.p, 0, h->r_img.n, st));
    // Environments can sit far outside the FP32/BF16 range (a random MPS's
    // environments shrink geometrically with length): pack L and R divided by
    // powers of two near their max-abs and multiply 2^(eL+eR) back in the
    // stage-4 epilogue.  Powers of two keep the FP64 path bit-exact.
    DevMem red;
    const int np = reduce_partials_count();
    red.alloc((np + 2) * sizeof(double));
    double mx[2] = {0.0, 0.0};
    if (H.L.total) launch_maxabs(L, H.L.total, red.as<double>() + np, red.as<double>(), st);
    if (H.R.total) launch_maxabs(R, H.R.total, red.as<double>() + np + 1, red.as<double>(), st);
    CUDA_OK(cudaMemcpyAsync(mx, red.as<double>() + np, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    auto pow2_of = [](double m) { return (m > 0.0 && std::isfinite(m)) ? std::ldexp(1.0, std::ilogb(m)) : 1.0; };
    const double sL = pow2_of(mx[0]), sR = pow2_of(mx[1]);
    h->out_scale = sL * sR;
    if (h->fused) {
      h->lp_img.alloc(std::max<int64_t>(1, h->fl.lp_bytes) * split);
      CUDA_OK(cudaMemsetAsync(h->lp_img.p, 0, h->lp_img.n, st));
      std::vector<DevLPanelSeg> segs;
      std::vector<int4> chunks;
      for (size_t lb = 0; lb < H.L.keys.size(); ++lb) {
        if (h->fl.lp_off[lb] < 0) continue;
        const auto& ld = H.L.dims[lb];
        DevLPanelSeg g{};
        g.src_off = H.L.offs[lb];
        g.img_addr = reinterpret_cast<uint64_t>(h->lp_img.p) + static_cast<uint64_t>(h->fl.lp_off[lb]);
        g.lo_off = h->fl.lp_bytes;
        g.ma = static_cast<int32_t>(ld[0]);
        g.mb = static_cast<int32_t>(ld[1]);
        g.mc = static_cast<int32_t>(ld[2]);
        g.cc = h->fl.cc;
        g.n_mma = h->fl.lp_nmma[lb];
        g.nKt = h->fl.lp_nKt[lb];
        g.scale = 1.0 / sL;
        const int id = static_cast<int>(segs.size());
        segs.push_back(g);
        const int64_t n = ld[0] * ld[1] * ld[2];
        for (int64_t e0 = 0; e0 < n; e0 += 256) chunks.push_back(make_int4(id, static_cast<int>(e0 / 256), 0, 0));
      }
      DevMem dseg, dch;
      upload(dseg, segs, st);
      upload(dch, chunks, st);
      launch_pack_lpanels(mode, L, dseg.as<DevLPanelSeg>(), dch.as<int4>(), static_cast<int>(chunks.size()), st);
      CUDA_OK(cudaGetLastError());
      CUDA_OK(cudaStreamSynchronize(st));
    } else {
      h->lp_img.alloc(0);
    }
    std::vector<DevPackSeg> pl, pr;
    std::vector<DevChunk> cl, cr;
    if (plain)
      build_pack(H.s1.packA, h->g1, true, reinterpret_cast<uint64_t>(h->l_img.p), h->l_lo, ig.tile_bytes, 0, pl, cl,
                 1.0 / sL);
    build_pack(H.s4.packB, h->g4, false, reinterpret_cast<uint64_t>(h->r_img.p), h->r_lo, ig.tile_bytes, 1, pr, cr,
               1.0 / sR);
    DevMem dpl, dcl, dpr, dcr, tab;
    upload(dpl, pl, st);
    upload(dcl, cl, st);
    upload(dpr, pr, st);
    upload(dcr, cr, st);
    uint64_t ptrs[2] = {reinterpret_cast<uint64_t>(L), reinterpret_cast<uint64_t>(R)};
    tab.alloc(sizeof(ptrs));
    CUDA_OK(cudaMemcpyAsync(tab.p, ptrs, sizeof(ptrs), cudaMemcpyHostToDevice, st));
    launch_pack(tab.as<uint64_t>(), dpl.as<DevPackSeg>(), dcl.as<DevChunk>(), static_cast<int>(cl.size()), mode,
                nullptr, st);
    launch_pack(tab.as<uint64_t>(), dpr.as<DevPackSeg>(), dcr.as<DevChunk>(), static_cast<int>(cr.size()), mode,
                nullptr, st);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaStreamSynchronize(st));
    h->prec = precision;
    return TNX_OK;
  })
}

void tnx_heff_destroy(tnx_heff* h) { delete h; }

// ---------------------------------------------------------------------------
// batched H_eff
// ---------------------------------------------------------------------------
struct tnx_heff_batch {
  std::vector<tnx_heff*> hs;
  int prec = 0, mode = 0;
  DevMem th_img, x1, x3_img;
  int64_t th_lo = 0, x3_lo = 0;
  DevMem th_pack, th_chunks;
  int n_th_chunks = 0;
  // theta by rows (k-major blocks, 8 consecutive k per thread) when every segment qualifies
  DevMem th_rows, th_row_chunks;
  int n_th_row_chunks = 0;
  bool th_by_rows = false;
  DevMem g1, t1, ro1, g4, t4, ro4;
  int n_t1 = 0, n_t4 = 0;
  DevMem mpo_pairs, mpo_slots, mpo_oslots, mpo_terms, mpo_chunks;
  int n_mpo_chunks = 0;
  size_t mpo_smem = 16;
  DevMem zero_chunks;  // theta-layout blocks H_eff never writes (slot = problem + 1)
  int n_zero_chunks = 0;
  DevMem err, src_tab, out_tab1, out_tab4;
  // fused stages 1-3: theta panels (hi plane, then lo) and the kernel's tables
  bool fused = false;
  DevMem thp_img, thp_rows, thp_row_chunks;
  int n_thp_row_chunks = 0;
  DevMem f_pairs, f_blocks, f_tb, f_terms, f_tiles;
  int n_f_tiles = 0;
  // routed stages 1-3: the stage-1 epilogue's destinations (per row class b:
  // a range of routes) and X1 of the input slots multi-term outputs read
  bool routed = false;
  DevMem routes, route_win, route_rows, route_cols;
  int64_t n_routes = 0;
  int32_t route_win_max = 0;  // records in the largest (tile, lane quarter, chunk) window
  const int32_t* skip = nullptr;
  int n_launches = 0;
  std::vector<uint64_t> last_src, last_out;
  // host-resident streaming (tnx_heff_batch_apply_host): each problem's theta
  // at th_off[i] of one concatenated buffer; two device copies of the inputs
  // and outputs with their pointer tables, two copy streams and the events
  // that order them against the compute stream
  std::vector<int64_t> th_off;
  int64_t th_total = 0;
  DevMem pipe_in[2], pipe_out[2], pipe_src_tab[2], pipe_out_tab[2];
  cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
  cudaEvent_t ev_start = nullptr, ev_in_ready[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr},
              ev_out_free[2] = {nullptr, nullptr};
  tnx_heff_batch() = default;
  tnx_heff_batch(const tnx_heff_batch&) = delete;
  tnx_heff_batch& operator=(const tnx_heff_batch&) = delete;
  ~tnx_heff_batch() {
    // copies still in flight must land before the buffers are released
    if (s_h2d) cudaStreamSynchronize(s_h2d);
    if (s_d2h) cudaStreamSynchronize(s_d2h);
    if (s_h2d) cudaStreamDestroy(s_h2d);
    if (s_d2h) cudaStreamDestroy(s_d2h);
    for (cudaEvent_t e : {ev_start, ev_in_ready[0], ev_in_ready[1], ev_done[0], ev_done[1], ev_out_free[0],
                          ev_out_free[1]})
      if (e) cudaEventDestroy(e);
  }
};

int tnx_heff_batch_create(tnx_heff* const* hs, int32_t n, int32_t precision, tnx_heff_batch** out) {
  TNX_TRY({
    if (n < 1 || n > kMaxSlots - 1) return set_err(TNX_ERR_VALUE, "batch size must be in [1, 255]");
    auto b = std::make_unique<tnx_heff_batch>();
    b->prec = precision;
    b->mode = img_mode_of(precision);
    const int mode = b->mode;
    const ImgGeom ig = img_geom(mode);
    const int split = mode == IMG_BF16 ? 2 : 1;
    const bool f32 = mode != IMG_F64;
    for (int i = 0; i < n; ++i) {
      if (hs[i]->prec != precision) return set_err(TNX_ERR_VALUE, "operators were packed for another precision");
      if (hs[i]->fused != hs[0]->fused)
        return set_err(TNX_ERR_VALUE, "operators of one batch must all run fused stages 1-3 or none");
      b->hs.push_back(hs[i]);
    }
    // routed and unfused operators share a batch: one stage-1 launch holds
    // both kinds of groups, the MPO tables are per problem
    b->fused = hs[0]->fused;
    b->routed = false;
    for (int i = 0; i < n; ++i) b->routed = b->routed || hs[i]->routed;
    for (int i = 0; i < n; ++i) {
      b->th_off.push_back(b->th_total);
      b->th_total += hs[i]->H.th.total;
    }
    // sizes: theta images (stage-1 B), X1 results, X3 images (stage-4 A)
    const bool fz = b->fused, rt = b->routed;
    int64_t th_tiles = 0, x3_tiles = 0, x1_elems = 0;
    std::vector<int64_t> th_t0(n), x3_t0(n), x1_0(n);
    for (int i = 0; i < n; ++i) {
      const HeffPlan& H = hs[i]->H;
      th_t0[i] = th_tiles;
      x3_t0[i] = x3_tiles;
      x1_0[i] = x1_elems;
      th_tiles += hs[i]->g1.b_tiles;
      x3_tiles += hs[i]->g4.a_tiles;
      if (hs[i]->routed) {
        // X1 of the kept input slots only: (c, d) with d padded to kMpoKAlign
        for (size_t pi = 0; pi < H.pairs.size(); ++pi) {
          const int64_t md_pad = (H.pairs[pi].md + kMpoKAlign - 1) / kMpoKAlign * kMpoKAlign;
          for (char k : hs[i]->rl.in_kept[pi])
            if (k) x1_elems += H.pairs[pi].mc * md_pad;
        }
      } else {
        for (auto& g : H.s1.groups) x1_elems += g.M * x1_ld(g.N);
      }
    }
    // the unfused and routed paths' stage-1 B image and X1 result (routed:
    // the kept X1 slots only); the fused path's theta panels
    b->th_img.alloc(fz ? 16 : std::max<int64_t>(1, th_tiles) * ig.tile_bytes * split);
    b->x3_img.alloc(std::max<int64_t>(1, x3_tiles) * ig.tile_bytes * split);
    b->th_lo = th_tiles * ig.tile_bytes;
    b->x3_lo = x3_tiles * ig.tile_bytes;
    b->x1.alloc(fz ? 16 : std::max<int64_t>(1, x1_elems) * (f32 ? 4 : 8));
    CUDA_OK(cudaMemset(b->th_img.p, 0, b->th_img.n));
    CUDA_OK(cudaMemset(b->x3_img.p, 0, b->x3_img.n));
    std::vector<int64_t> thp_t0(n, 0);
    int64_t thp_tiles = 0;
    if (fz) {
      for (int i = 0; i < n; ++i) {
        thp_t0[i] = thp_tiles;
        thp_tiles += hs[i]->fl.thp_tiles;
      }
      b->thp_img.alloc(std::max<int64_t>(1, thp_tiles) * ig.tile_bytes * split);
      CUDA_OK(cudaMemset(b->thp_img.p, 0, b->thp_img.n));
    }
    const uint64_t thp_base = reinterpret_cast<uint64_t>(b->thp_img.p);
    const int64_t thp_lo = thp_tiles * ig.tile_bytes;
    std::vector<DevRowPackSeg> fth;
    std::vector<int4> fthc;
    std::vector<DevFPair> FP;
    std::vector<DevFBlock> FB;
    std::vector<int32_t> FTB;
    std::vector<DevFTerm> FT;
    std::vector<std::pair<int64_t, DevFTile>> FTL;
    const uint64_t th_base = reinterpret_cast<uint64_t>(b->th_img.p);
    const uint64_t x3_base = reinterpret_cast<uint64_t>(b->x3_img.p);
    const uint64_t x1_base = reinterpret_cast<uint64_t>(b->x1.p);
    const int esz = f32 ? 4 : 8;
    std::vector<DevPackSeg> tp;
    std::vector<DevChunk> tc;
    std::vector<DevRowPackSeg> trs;
    std::vector<int4> trc;
    bool rows_ok = true;
    std::vector<DevGroup> G1, G4;
    std::vector<int64_t> R1, R4;
    std::vector<std::pair<int64_t, DevTile>> T1, T4;
    std::vector<DevMpoPair> MP;
    std::vector<DevMpoSlot> MI;
    std::vector<DevMpoOutSlot> MO;
    std::vector<DevMpoTerm> MT;
    std::vector<int2> MC;
    std::vector<DevChunk> ZC;
    std::vector<DevRoute> RT;
    std::vector<int2> RB, RI, CI;
    std::vector<int2> RG;  // routed groups: (first RB entry, column classes)
    for (int i = 0; i < n; ++i) {
      tnx_heff* h = hs[i];
      const bool rti = h->routed;
      std::vector<RoutedEntry> rents;
      const HeffPlan& H = h->H;
      // theta pack: source slot i, images into the batch theta buffer
      PairGeom gth = h->g1;  // b_tile0 relative to this problem
      for (auto& t : gth.b_tile0) t += th_t0[i];
      build_pack(H.s1.packB, gth, false, th_base, b->th_lo, ig.tile_bytes, i, tp, tc);
      for (const PackSeg& ps : H.s1.packB) {
        // eligible: leg 0 is the only contracted leg and the free legs (1..)
        // map to consecutive image rows (legs of extent 1 carry no stride)
        bool ok = ps.nlegs >= 2 && ps.kstr[0] == 1 && ps.k0 % kMpoKAlign == 0;
        int64_t expect = 1;
        for (int l = ps.nlegs - 1; l >= 1 && ok; --l) {
          ok = ps.kstr[l] == 0 && (ps.dims[l] == 1 || ps.rstr[l] == expect);
          expect *= ps.dims[l];
        }
        if (!ok) {
          rows_ok = false;
          continue;
        }
        DevRowPackSeg rs{};
        rs.src_off = ps.src_off;
        rs.img_addr = th_base + static_cast<uint64_t>(gth.b_tile0[ps.group]) * ig.tile_bytes;
        rs.lo_off = b->th_lo;
        rs.row0 = ps.row0;
        rs.k0 = ps.k0;
        rs.nKt = gth.nKt[ps.group];
        rs.kval = ps.dims[0];
        rs.rows = static_cast<int32_t>(ps.count / ps.dims[0]);
        rs.src_slot = i;
        rs.scale = 1.0;
        rs.kstride = rs.rows;
        const int id = static_cast<int>(trs.size());
        trs.push_back(rs);
        const int nkc = (rs.kval + kMpoKAlign - 1) / kMpoKAlign, cpt = pack_rows_chunks_per_thread();
        for (int r0 = 0; r0 < rs.rows; r0 += pack_rows_per_cta())
          for (int kc = 0; kc < nkc; kc += cpt) trc.push_back(make_int4(id, r0, kc, 0));
      }
      if (fz) {
        // theta panels: each referenced (theta block, p, q) slice as rows d, K = a
        const int tk = ig.tk;
        for (const auto& kv : h->fl.thp_tile0) {
          const int tb = kv.first[0], pp = kv.first[1], qq = kv.first[2];
          const auto& td = H.th.dims[tb];
          DevRowPackSeg rs{};
          rs.src_off = H.th.offs[tb] + (static_cast<int64_t>(pp) * td[2] + qq) * td[3];
          rs.img_addr = thp_base + static_cast<uint64_t>(thp_t0[i] + kv.second) * ig.tile_bytes;
          rs.lo_off = thp_lo;
          rs.row0 = 0;
          rs.k0 = 0;
          rs.nKt = static_cast<int32_t>(cdiv(td[0], tk));
          rs.rows = static_cast<int32_t>(td[3]);
          rs.kval = static_cast<int32_t>(td[0]);
          rs.src_slot = i;
          rs.scale = 1.0;
          rs.kstride = td[1] * td[2] * td[3];
          const int id = static_cast<int>(fth.size());
          fth.push_back(rs);
          const int nkc = (rs.kval + kMpoKAlign - 1) / kMpoKAlign, cpt = pack_rows_chunks_per_thread();
          for (int r0 = 0; r0 < rs.rows; r0 += pack_rows_per_cta())
            for (int kc = 0; kc < nkc; kc += cpt) fthc.push_back(make_int4(id, r0, kc, 0));
        }
      }
      // stage-1 groups (routed: their rows and 8-column units get classes and
      // destinations with the MPO tables below)
      std::vector<int64_t> x1_goff;
      int64_t xo = x1_0[i];
      const int g1base = static_cast<int>(G1.size());
      for (size_t g = 0; g < H.s1.groups.size(); ++g) {
        x1_goff.push_back(xo);
        DevGroup x{};
        x.a_addr = reinterpret_cast<uint64_t>(h->l_img.p) + static_cast<uint64_t>(h->g1.a_tile0[g]) * ig.tile_bytes;
        x.b_addr = th_base + static_cast<uint64_t>(gth.b_tile0[g]) * ig.tile_bytes;
        x.a_lo = h->l_lo;
        x.b_lo = b->th_lo;
        x.rowoff0 = static_cast<int64_t>(R1.size());
        x.M = static_cast<int32_t>(H.s1.groups[g].M);
        x.N = static_cast<int32_t>(H.s1.groups[g].N);
        x.nKt = h->g1.nKt[g];
        x.kk_last = kk_last_of(H.s1.groups[g].K, b->mode);
        x.out_slot = 0;
        x.scale = 1.0;
        if (rti) {
          // row and 8-column-unit classes, filled with the MPO tables below
          x.routed = 1;
          x.rowoff0 = static_cast<int64_t>(RI.size());
          x.cinfo0 = static_cast<int32_t>(CI.size());
          RI.resize(RI.size() + H.s1.groups[g].M, make_int2(-1, 0));
          CI.resize(CI.size() + cdiv(H.s1.groups[g].N, 8), make_int2(-1, 0));
          G1.push_back(x);
          RG.resize(G1.size(), make_int2(0, 1));
          continue;
        }
        const int64_t ld = x1_ld(H.s1.groups[g].N);
        x.vec_ld = static_cast<int32_t>(ld);
        for (int64_t r = 0; r < H.s1.groups[g].M; ++r) R1.push_back(xo + r * ld);
        xo += H.s1.groups[g].M * ld;
        G1.push_back(x);
      }
      RG.resize(G1.size(), make_int2(0, 1));
      std::vector<std::pair<int64_t, DevTile>> tl;
      build_tiles(H.s1, h->g1, g1base, tl);
      T1.insert(T1.end(), tl.begin(), tl.end());
      // stage-4 groups
      PairGeom gx3 = h->g4;
      for (auto& t : gx3.a_tile0) t += x3_t0[i];
      const int g4base = static_cast<int>(G4.size());
      for (size_t g = 0; g < H.s4.groups.size(); ++g) {
        DevGroup x{};
        x.a_addr = x3_base + static_cast<uint64_t>(gx3.a_tile0[g]) * ig.tile_bytes;
        x.b_addr = reinterpret_cast<uint64_t>(h->r_img.p) + static_cast<uint64_t>(h->g4.b_tile0[g]) * ig.tile_bytes;
        x.a_lo = b->x3_lo;
        x.b_lo = h->r_lo;
        x.rowoff0 = static_cast<int64_t>(R4.size());
        x.M = static_cast<int32_t>(H.s4.groups[g].M);
        x.N = static_cast<int32_t>(H.s4.groups[g].N);
        x.nKt = h->g4.nKt[g];
        x.kk_last = kk_last_of(H.s4.groups[g].K, b->mode);
        x.out_slot = 1 + i;
        x.scale = h->out_scale;  // undoes the power-of-two scaling of L and R
        for (auto v : H.s4_rowoff[g]) R4.push_back(v);
        G4.push_back(x);
      }
      tl.clear();
      build_tiles(H.s4, h->g4, g4base, tl);
      T4.insert(T4.end(), tl.begin(), tl.end());
      for (auto& zr : H.zero_ranges)
        for (int64_t st = 0; st < zr.second; st += 4096)
          ZC.push_back({1 + i, 0, zr.first + st, std::min<int64_t>(4096, zr.second - st)});
      // MPO tables (routed: the multi-term output slots only, reading the kept X1 slots)
      int64_t x1k = x1_0[i];
      for (size_t pi = 0; pi < H.pairs.size(); ++pi) {
        const MpoPair& mp = H.pairs[pi];
        const int32_t md_pad = (mp.md + kMpoKAlign - 1) / kMpoKAlign * kMpoKAlign;
        std::vector<MpoTerm> terms;
        for (const MpoTerm& t : mp.terms)
          if (!rti || h->rl.out_terms[pi][t.out_slot] > 1) terms.push_back(t);
        DevMpoPair dp{};
        dp.mc = mp.mc;
        dp.md = mp.md;
        dp.in0 = static_cast<int32_t>(MI.size());
        dp.n_in = static_cast<int32_t>(mp.ins.size());
        dp.out0 = static_cast<int32_t>(MO.size());
        dp.n_out = mp.n_out_slots;
        dp.term0 = static_cast<int32_t>(MT.size());
        dp.n_terms = static_cast<int32_t>(terms.size());
        dp.n_in_slots = mp.n_in_slots;
        dp.n_out_slots = mp.n_out_slots;
        b->mpo_smem = std::max<size_t>(b->mpo_smem, terms.size() * sizeof(DevMpoTerm) +
                                                       mp.n_in_slots * sizeof(DevMpoSlot) +
                                                       mp.n_out_slots * sizeof(DevMpoOutSlot));
        // X1 columns of one (p,q) slot: its d range padded to H.x1_align
        const int64_t md_x1 = (mp.md + H.x1_align - 1) / H.x1_align * H.x1_align;
        for (int32_t sl = 0; sl < mp.n_in_slots && rti; ++sl) {
          // kept slots: X1 rows (c, d), d padded to kMpoKAlign; the others are never read
          DevMpoSlot r{};
          r.base = x1_base;
          r.ld = md_pad;
          if (h->rl.in_kept[pi][sl]) {
            r.base = x1_base + static_cast<uint64_t>(x1k) * 4;
            x1k += static_cast<int64_t>(mp.mc) * md_pad;
            if (x1k * 4 > static_cast<int64_t>(b->x1.n))
              return set_err(TNX_ERR_RUNTIME, "internal: kept X1 slots outside their buffer");
          }
          MI.push_back(r);
        }
        for (size_t k = 0; k < mp.ins.size() && !rti; ++k) {
          // one record per input slot (b,p,q): address of its point (c=0, d=0)
          const MpoIn& in = mp.ins[k];
          const int64_t ld = x1_ld(H.s1.groups[in.g1].N);
          const int64_t blk = x1_goff[in.g1] + static_cast<int64_t>(in.row0) * ld + in.col0;
          for (int bb = 0; bb < in.mb; ++bb)
            for (int pp = 0; pp < in.mp; ++pp)
              for (int qq = 0; qq < in.mq; ++qq) {
                DevMpoSlot sl{};
                sl.base = x1_base + static_cast<uint64_t>(blk + static_cast<int64_t>(bb) * mp.mc * ld +
                                                          static_cast<int64_t>(pp * in.mq + qq) * md_x1) *
                                        esz;
                sl.ld = ld;
                // the FP32 MPO kernel loads 8 consecutive d (padding included) with 16-byte loads
                if (f32 && !fz && (H.x1_align != kMpoKAlign || sl.base % 32 != 0 || ld % 8 != 0))
                  return set_err(TNX_ERR_RUNTIME, "internal: X1 slot not aligned for the vector MPO loads");
                MI.push_back(sl);
              }
        }
        // stage-4 K places each f block's d range at a multiple of kMpoKAlign
        for (size_t k = 0; k < mp.outs.size(); ++k) {
          const MpoOut& o = mp.outs[k];
          const int64_t img_rows = cdiv(H.s4.groups[o.g4].M, 128) * 128;
          for (int s = 0; s < o.ms; ++s)
            for (int t = 0; t < o.mt; ++t)
              for (int f = 0; f < o.mf; ++f) {
                DevMpoOutSlot os{};
                os.img_addr = x3_base + static_cast<uint64_t>(gx3.a_tile0[o.g4]) * ig.tile_bytes;
                os.lo_off = b->x3_lo;
                os.nKt = h->g4.nKt[o.g4];
                os.row0 = o.row0;
                os.k0 = o.k0;
                os.rows_per_c = o.ms * o.mt;
                os.row_add = s * o.mt + t;
                os.k_add = f * md_pad;
                // every (c, d) of the slot lands inside its group's image
                if (os.row0 + os.row_add + static_cast<int64_t>(mp.mc - 1) * os.rows_per_c >= img_rows ||
                    os.k0 + os.k_add + md_pad > static_cast<int64_t>(os.nKt) * ig.tk)
                  return set_err(TNX_ERR_RUNTIME, "internal: an X3 slot lies outside its stage-4 image");
                MO.push_back(os);
              }
        }
        for (auto& t : terms) MT.push_back({t.out_slot, t.in_slot, t.w});
        const int pair_id = static_cast<int>(MP.size());
        MP.push_back(dp);
        if (rti) {
          // the destinations of every X1 row (b, c) and (p, q) column range of
          // this pair: the single-term output slots its input slot feeds and,
          // when a multi-term output reads that slot, its kept X1 rows
          std::vector<std::vector<std::pair<int32_t, double>>> singles(mp.n_in_slots);
          for (const MpoTerm& t : mp.terms)
            if (h->rl.out_terms[pi][t.out_slot] == 1) singles[t.in_slot].push_back({t.out_slot, t.w});
          for (size_t k = 0; k < mp.ins.size(); ++k) {
            const MpoIn& in = mp.ins[k];
            for (int32_t bb = 0; bb < in.mb; ++bb)
              for (int32_t pp = 0; pp < in.mp; ++pp)
                for (int32_t qq = 0; qq < in.mq; ++qq) {
                  const int32_t sl = mp.in_slot0[k] + (bb * in.mp + pp) * in.mq + qq;
                  RoutedEntry e;
                  e.g = in.g1;
                  e.rkey = in.row0 + bb * mp.mc;
                  e.ckey = static_cast<int32_t>(in.col0 + (pp * in.mq + qq) * md_x1);
                  e.mc = mp.mc;
                  for (const auto& ow : singles.at(sl)) {
                    const DevMpoOutSlot& os = MO[dp.out0 + ow.first];
                    DevRoute r{};
                    r.addr = os.img_addr;
                    if (os.nKt > 65535) return set_err(TNX_ERR_UNSUPPORTED, "a stage-4 group has more than 65535 K tiles");
                    r.nKt = static_cast<uint16_t>(os.nKt);
                    r.row0 = os.row0 + os.row_add;
                    r.rstride = os.rows_per_c;
                    r.k0 = os.k0 + os.k_add;
                    r.w = static_cast<float>(ow.second);
                    r.kind = 0;
                    e.routes.push_back(r);
                  }
                  if (h->rl.in_kept[pi][sl]) {
                    DevRoute r{};
                    r.addr = MI[dp.in0 + sl].base;
                    r.rstride = md_pad;
                    r.w = 1.0f;
                    r.kind = 1;
                    e.routes.push_back(r);
                  }
                  e.md_pad = md_pad;
                  rents.push_back(std::move(e));
                }
          }
        }
        if (fz) {
          // fused tables of this pair: its MMA blocks, its terms by output slot, its tiles
          const FusedLayout& fl = h->fl;
          const int tk = ig.tk;
          DevFPair fp{};
          fp.blk0 = static_cast<int32_t>(FB.size());
          fp.n_blk = static_cast<int32_t>(fl.blocks[pi].size());
          fp.tb0 = static_cast<int32_t>(FTB.size());
          fp.n_out = mp.n_out_slots;
          fp.out0 = dp.out0;
          fp.n_in = mp.n_in_slots;
          fp.mc = mp.mc;
          fp.md = mp.md;
          fp.cc = fl.cc;
          int64_t work = 0;
          for (const FusedBlk& fb : fl.blocks[pi]) {
            DevFBlock d{};
            d.a_addr = thp_base + static_cast<uint64_t>(thp_t0[i] + fl.thp_tile0.at({fb.th_blk, fb.pp, fb.qq})) *
                                      ig.tile_bytes;
            d.b_addr = reinterpret_cast<uint64_t>(h->lp_img.p) + static_cast<uint64_t>(fl.lp_off[fb.l_blk]);
            d.a_lo = thp_lo;
            d.b_lo = fl.lp_bytes;
            d.nKt = static_cast<int32_t>(cdiv(fb.ma, tk));
            d.kk_last = kk_last_of(fb.ma, b->mode);
            d.n_mma = fb.n_mma;
            d.col = fb.col;
            d.mb = fb.mb;
            d.slot0 = fb.slot0;
            d.slot_stride = fb.slot_stride;
            FB.push_back(d);
            work += static_cast<int64_t>(fb.n_mma) * d.nKt;
          }
          // an input slot's TMEM column (for c = 0) and its stride per c
          std::vector<std::pair<int32_t, int32_t>> slot_col(mp.n_in_slots, {-1, 0});
          for (const FusedBlk& fb : fl.blocks[pi])
            for (int32_t bb = 0; bb < fb.mb; ++bb) slot_col[fb.slot0 + bb * fb.slot_stride] = {fb.col + bb, fb.mb};
          size_t u = 0;
          for (int32_t o = 0; o < mp.n_out_slots; ++o) {
            FTB.push_back(static_cast<int32_t>(FT.size()));
            for (; u < mp.terms.size() && mp.terms[u].out_slot == o; ++u) {
              const auto sc = slot_col.at(mp.terms[u].in_slot);
              if (sc.first < 0) return set_err(TNX_ERR_RUNTIME, "internal: MPO term reads an unmapped input slot");
              FT.push_back(DevFTerm{static_cast<int16_t>(sc.first), static_cast<int16_t>(sc.second),
                                    static_cast<float>(mp.terms[u].w)});
            }
          }
          FTB.push_back(static_cast<int32_t>(FT.size()));
          if (u != mp.terms.size()) return set_err(TNX_ERR_RUNTIME, "internal: MPO terms not sorted by output slot");
          const int fpair = static_cast<int>(FP.size());
          FP.push_back(fp);
          for (int64_t dt = 0; dt < cdiv(mp.md, 128); ++dt)
            for (int64_t ct = 0; ct < cdiv(mp.mc, fl.cc); ++ct)
              FTL.push_back({work, DevFTile{fpair, static_cast<int32_t>(ct), static_cast<int32_t>(dt), 0}});
        }
        const int ppc = mpo_points_per_cta();
        const int dpt = mpo_d_per_thread(b->mode);
        const int npts = mp.mc * ((mp.md + dpt - 1) / dpt);
        for (int p0 = 0; p0 < npts && dp.n_terms > 0; p0 += ppc) MC.push_back(make_int2(pair_id, p0));
      }
      if (rti) {
        // classes of each group in row and column order, the rows' and
        // units' classes, and the routes in (row class, column class) order,
        // so that the rows of one warp read one contiguous range of routes
        const size_t ng = H.s1.groups.size();
        std::vector<std::map<int32_t, int32_t>> rcl(ng), ccl(ng);
        std::vector<int64_t> rb0;
        std::vector<int32_t> ncc;
        for (const RoutedEntry& e : rents) {
          if (e.ckey % 8 || e.g < 0 || static_cast<size_t>(e.g) >= ng)
            return set_err(TNX_ERR_RUNTIME, "internal: a routed column range is not 8-aligned");
          rcl[e.g][e.rkey] = 0;
          ccl[e.g][e.ckey] = 0;
        }
        for (size_t g = 0; g < ng; ++g) {
          int32_t id = 0;
          for (auto& kv : rcl[g]) kv.second = id++;
          id = 0;
          for (auto& kv : ccl[g]) kv.second = id++;
          if (ccl[g].size() > 255) return set_err(TNX_ERR_UNSUPPORTED, "a stage-1 group has more than 255 column classes");
          rb0.push_back(static_cast<int64_t>(RB.size()));
          ncc.push_back(std::max<int32_t>(1, static_cast<int32_t>(ccl[g].size())));
          RB.resize(RB.size() + rcl[g].size() * static_cast<size_t>(ncc.back()), make_int2(0, 0));
        }
        std::vector<std::array<int64_t, 4>> order;  // (group, RB index, entry, classes)
        for (size_t k = 0; k < rents.size(); ++k) {
          const RoutedEntry& e = rents[k];
          const DevGroup& x = G1[g1base + e.g];
          const int32_t rc = rcl[e.g][e.rkey], cc = ccl[e.g][e.ckey];
          const GroupShape& gs = H.s1.groups[e.g];
          if (e.rkey < 0 || e.rkey + e.mc > gs.M || e.ckey + e.md_pad > cdiv(gs.N, 8) * 8)
            return set_err(TNX_ERR_RUNTIME, "internal: a routed X1 block lies outside its group");
          for (int32_t c = 0; c < e.mc; ++c) RI[x.rowoff0 + e.rkey + c] = make_int2(rc, c);
          for (int32_t j = 0; j < e.md_pad / 8; ++j) CI[x.cinfo0 + e.ckey / 8 + j] = make_int2(cc, 8 * j);
          order.push_back({e.g, rb0[e.g] + static_cast<int64_t>(rc) * ncc[e.g] + cc, static_cast<int64_t>(k),
                           (static_cast<int64_t>(rc) << 8) | cc});
        }
        std::sort(order.begin(), order.end());
        for (size_t g = 0; g < ng; ++g) {
          RG[g1base + g] = make_int2(static_cast<int32_t>(rb0[g]), ncc[g]);
        }
        const uint64_t x1_end = x1_base + static_cast<uint64_t>(b->x1.n);
        for (const auto& o : order) {
          const RoutedEntry& e = rents[o[2]];
          if (RB[o[1]].y != 0) return set_err(TNX_ERR_RUNTIME, "internal: two X1 blocks share a routed class pair");
          RB[o[1]] = make_int2(static_cast<int32_t>(RT.size()), static_cast<int32_t>(e.routes.size()));
          for (DevRoute r : e.routes) {
            r.rc = static_cast<int32_t>(o[3] >> 8);
            r.cc = static_cast<uint8_t>(o[3] & 255);
            // every (c, d) of the entry lands inside the X3 image or the kept X1 slots
            const int64_t last = static_cast<int64_t>(e.mc - 1) * r.rstride;
            // the epilogue forms row indices and tile indices in 32 bits
            if (r.row0 + last + e.md_pad >= (int64_t{1} << 31) ||
                cdiv(r.row0 + last + 1, 128) * static_cast<int64_t>(r.nKt) >= (int64_t{1} << 32))
              return set_err(TNX_ERR_UNSUPPORTED, "a routed destination exceeds 32-bit row indexing");
            if (r.kind != 1) {
              const uint64_t end = r.addr + static_cast<uint64_t>(cdiv(r.row0 + last + 1, 128) * r.nKt) * ig.tile_bytes;
              if (r.addr < x3_base || end > x3_base + static_cast<uint64_t>(x3_tiles) * ig.tile_bytes ||
                  r.k0 + e.md_pad > static_cast<int64_t>(r.nKt) * ig.tk)
                return set_err(TNX_ERR_RUNTIME, "internal: a route writes outside the X3 image");
            } else {
              const uint64_t end = r.addr + static_cast<uint64_t>(last + e.md_pad) * 4;
              if (r.addr < x1_base || end > x1_end || r.addr % 32 || r.rstride % kMpoKAlign)
                return set_err(TNX_ERR_RUNTIME, "internal: a route writes outside the kept X1 slots");
            }
            RT.push_back(r);
          }
        }
      }
    }
    if (b->mpo_smem > 200 * 1024)
      return set_err(TNX_ERR_UNSUPPORTED, "MPO term tables too large for the fused MPO kernel");
    upload(b->th_pack, tp);
    upload(b->th_chunks, tc);
    b->n_th_chunks = static_cast<int>(tc.size());
    b->th_by_rows = rows_ok;
    if (rows_ok) {
      upload(b->th_rows, trs);
      upload(b->th_row_chunks, trc);
      b->n_th_row_chunks = static_cast<int>(trc.size());
    }
    upload(b->g1, G1);
    upload(b->ro1, R1);
    auto t1 = sorted_tiles(T1);
    upload(b->t1, t1);
    if (rt) {
      // per (tile, lane quarter, 32-column chunk): the one range of routes
      // holding every (row class, column class) pair of its 32 rows and 4 units
      std::vector<int2> TW(t1.size() * 16, make_int2(0, 0));
      for (size_t t = 0; t < t1.size(); ++t) {
        const DevGroup& g = G1[t1[t].g];
        if (!g.routed) continue;
        const int2 rg = RG[t1[t].g];
        for (int q = 0; q < 4; ++q)
          for (int ch = 0; ch < 4; ++ch) {
            const int col0 = t1[t].nt * 128 + 32 * ch;
            int lo = 0x7fffffff, hi = 0;
            for (int lane = 0; lane < 32; ++lane) {
              const int row = t1[t].mt * 128 + 32 * q + lane;
              if (row >= g.M || RI[g.rowoff0 + row].x < 0) continue;
              for (int u = 0; u < 4; ++u) {
                const int col = col0 + 8 * u;
                if (col >= g.N || CI[g.cinfo0 + col / 8].x < 0) continue;
                const int2 r = RB[rg.x + static_cast<int64_t>(RI[g.rowoff0 + row].x) * rg.y + CI[g.cinfo0 + col / 8].x];
                if (r.y > 0) {
                  lo = std::min(lo, r.x);
                  hi = std::max(hi, r.x + r.y);
                }
              }
            }
            if (hi > lo) {
              TW[t * 16 + q * 4 + ch] = make_int2(lo, hi - lo);
              b->route_win_max = std::max(b->route_win_max, hi - lo);
            }
          }
      }
      upload(b->route_win, TW);
    }
    b->n_t1 = static_cast<int>(t1.size());
    upload(b->g4, G4);
    upload(b->ro4, R4);
    auto t4 = sorted_tiles(T4);
    upload(b->t4, t4);
    b->n_t4 = static_cast<int>(t4.size());
    upload(b->mpo_pairs, MP);
    upload(b->mpo_slots, MI);
    upload(b->mpo_oslots, MO);
    upload(b->mpo_terms, MT);
    upload(b->mpo_chunks, MC);
    upload(b->zero_chunks, ZC);
    b->n_zero_chunks = static_cast<int>(ZC.size());
    if (fz) {
      // every access of the fused kernel stays inside its buffers: theta panel
      // tiles, L panels, TMEM columns, staging rows, terms and output slots
      const uint64_t thp_end = thp_base + static_cast<uint64_t>(thp_tiles) * ig.tile_bytes;
      for (const DevFPair& fp : FP) {
        if (fp.n_blk < 1 || fp.n_in > kFusedMaxSlots || fp.out0 < 0 ||
            fp.out0 + fp.n_out > static_cast<int64_t>(MO.size()) ||
            fp.tb0 + fp.n_out + 1 > static_cast<int64_t>(FTB.size()) || fp.cc < 1)
          return set_err(TNX_ERR_RUNTIME, "internal: fused pair table out of range");
        if (fp.n_out > kFusedMaxOut || FTB[fp.tb0 + fp.n_out] - FTB[fp.tb0] > kFusedMaxTerms)
          return set_err(TNX_ERR_RUNTIME, "internal: fused pair tables exceed the kernel's per-warp tables");
        for (int o = 0; o < fp.n_out; ++o)
          for (int u = FTB[fp.tb0 + o]; u < FTB[fp.tb0 + o + 1]; ++u)
            if (FT[u].col0 < 0 || FT[u].cstride < 1 || FT[u].col0 + (fp.cc - 1) * FT[u].cstride >= kFusedAccCols)
              return set_err(TNX_ERR_RUNTIME, "internal: fused term reads outside its tile's accumulator");
        const int64_t n_dt = cdiv(fp.md, 128);
        for (int j = 0; j < fp.n_blk; ++j) {
          const DevFBlock& d = FB[fp.blk0 + j];
          if (d.n_mma < 16 || d.n_mma % 16 || d.n_mma > kFusedMaxN || d.col < 0 || d.col + d.n_mma > kFusedAccCols ||
              d.mb * fp.cc > d.n_mma || d.nKt < 1 || d.slot0 < 0 || d.slot0 + (d.mb - 1) * d.slot_stride >= fp.n_in)
            return set_err(TNX_ERR_RUNTIME, "internal: fused block geometry out of range");
          const uint64_t a_last = d.a_addr + static_cast<uint64_t>(n_dt * d.nKt) * ig.tile_bytes;
          if (d.a_addr < thp_base || a_last > thp_end)
            return set_err(TNX_ERR_RUNTIME, "internal: fused theta panel outside its image");
        }
      }
      for (int i = 0; i < n; ++i) {
        const tnx_heff* h = hs[i];
        const uint64_t lp0 = reinterpret_cast<uint64_t>(h->lp_img.p);
        for (size_t lb = 0; lb < h->H.L.keys.size(); ++lb) {
          if (h->fl.lp_off[lb] < 0) continue;
          const int64_t bytes = cdiv(h->H.L.dims[lb][2], h->fl.cc) * h->fl.lp_nKt[lb] *
                                static_cast<int64_t>(h->fl.lp_nmma[lb]) * 128;
          if (h->fl.lp_off[lb] + bytes > h->fl.lp_bytes || lp0 == 0)
            return set_err(TNX_ERR_RUNTIME, "internal: L panels outside their image");
        }
      }
      upload(b->f_pairs, FP);
      upload(b->f_blocks, FB);
      upload(b->f_tb, FTB);
      upload(b->f_terms, FT);
      std::stable_sort(FTL.begin(), FTL.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
      std::vector<DevFTile> ftl;
      ftl.reserve(FTL.size());
      for (auto& x : FTL) ftl.push_back(x.second);
      upload(b->f_tiles, ftl);
      b->n_f_tiles = static_cast<int>(ftl.size());
    }
    if (fz) {
      upload(b->thp_rows, fth);
      upload(b->thp_row_chunks, fthc);
      b->n_thp_row_chunks = static_cast<int>(fthc.size());
    }
    if (rt) {
      b->n_routes = static_cast<int64_t>(RT.size());
      upload(b->routes, RT);
      upload(b->route_rows, RI);
      upload(b->route_cols, CI);
    }
    b->n_mpo_chunks = static_cast<int>(MC.size());
    b->err.alloc(sizeof(int32_t));
    CUDA_OK(cudaMemset(b->err.p, 0, sizeof(int32_t)));
    b->src_tab.alloc(sizeof(PtrTab));
    b->out_tab1.alloc(sizeof(PtrTab));
    b->out_tab4.alloc(sizeof(PtrTab));
    // stage-1 output table is fixed (slot 0 = X1 buffer)
    PtrTab t1tab{};
    t1tab.p[0] = x1_base;
    CUDA_OK(cudaMemcpy(b->out_tab1.p, &t1tab, sizeof(PtrTab), cudaMemcpyHostToDevice));
    CUDA_OK(cudaDeviceSynchronize());
    b->n_launches = (b->fused ? 3 : 4) + (b->n_zero_chunks > 0 ? 1 : 0);
    *out = b.release();
    return TNX_OK;
  })
}

int tnx_heff_batch_set_skip_flag(tnx_heff_batch* b, const int32_t* flag) {
  b->skip = flag;
  return TNX_OK;
}

int tnx_heff_batch_launches(const tnx_heff_batch* b, int32_t* n_launches) {
  *n_launches = b->n_launches;
  return TNX_OK;
}

int tnx_heff_batch_route_stats(const tnx_heff_batch* b, int64_t* n_routes, int32_t* max_window) {
  if (!b || !n_routes || !max_window) return set_err(TNX_ERR_VALUE, "null argument");
  *n_routes = b->n_routes;
  *max_window = b->route_win_max;
  return TNX_OK;
}

// stage 0: pack theta; 1: stage-1 GEMM; 2: fused MPO; 3: stage-4 GEMM into theta layout.
// src_tab / out_tab4: device pointer tables of the inputs (problem i) and outputs (slot 1 + i)
static void heff_batch_stage(tnx_heff_batch* b, int stage, cudaStream_t st, const uint64_t* src_tab,
                             const uint64_t* out_tab4) {
  const bool f32 = b->mode != IMG_F64;
  if (b->fused && stage < 3) {
    // 0: theta panels; 1: fused stages 1-3 (X3 image); 2: nothing (the MPO ran inside stage 1)
    if (stage == 0)
      launch_pack_rows(src_tab, b->thp_rows.as<DevRowPackSeg>(), b->thp_row_chunks.as<int4>(), b->n_thp_row_chunks,
                       b->mode, b->skip, st);
    else if (stage == 1)
      launch_heff_fused(b->mode, b->f_pairs.as<DevFPair>(), b->f_blocks.as<DevFBlock>(), b->f_tb.as<int32_t>(),
                        b->f_terms.as<DevFTerm>(), b->mpo_oslots.as<DevMpoOutSlot>(), b->f_tiles.as<DevFTile>(),
                        b->n_f_tiles, b->err.as<int32_t>(), b->skip, st);
    return;
  }
  switch (stage) {
    case 0:
      if (b->th_by_rows)
        launch_pack_rows(src_tab, b->th_rows.as<DevRowPackSeg>(), b->th_row_chunks.as<int4>(),
                         b->n_th_row_chunks, b->mode, b->skip, st);
      else
        launch_pack(src_tab, b->th_pack.as<DevPackSeg>(), b->th_chunks.as<DevChunk>(),
                    b->n_th_chunks, b->mode, b->skip, st);
      break;
    case 1:
      if (b->mode == IMG_F64)
        launch_gemm_f64(b->g1.as<DevGroup>(), b->t1.as<DevTile>(), b->n_t1, b->ro1.as<int64_t>(),
                        b->out_tab1.as<uint64_t>(), b->skip, st);
      else
        launch_gemm_tc(b->mode, b->g1.as<DevGroup>(), b->t1.as<DevTile>(), b->n_t1, b->ro1.as<int64_t>(),
                       b->out_tab1.as<uint64_t>(), false, b->err.as<int32_t>(), b->skip, st,
                       b->routed ? DevRouteTabs{b->x3_lo, b->routes.as<DevRoute>(), b->route_win.as<int2>(),
                                                b->route_rows.as<int2>(), b->route_cols.as<int2>()}
                                 : DevRouteTabs{});
      break;
    case 2:
      launch_mpo_apply(f32, b->mode, b->mpo_pairs.as<DevMpoPair>(), b->mpo_slots.as<DevMpoSlot>(),
                       b->mpo_oslots.as<DevMpoOutSlot>(), b->mpo_terms.as<DevMpoTerm>(), b->mpo_chunks.as<int2>(),
                       b->n_mpo_chunks, b->mpo_smem, b->skip, st);
      break;
    default:
      launch_zero_ranges(out_tab4, b->zero_chunks.as<DevChunk>(), b->n_zero_chunks, b->skip, st);
      if (b->mode == IMG_F64)
        launch_gemm_f64(b->g4.as<DevGroup>(), b->t4.as<DevTile>(), b->n_t4, b->ro4.as<int64_t>(),
                        out_tab4, b->skip, st);
      else
        launch_gemm_tc(b->mode, b->g4.as<DevGroup>(), b->t4.as<DevTile>(), b->n_t4, b->ro4.as<int64_t>(),
                       out_tab4, true, b->err.as<int32_t>(), b->skip, st);
  }
}

int tnx_heff_batch_apply(tnx_heff_batch* b, const double* const* thetas, double* const* outs, void* stream) {
  TNX_TRY({
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n = static_cast<int>(b->hs.size());
    std::vector<uint64_t> src(n), o4(n + 1, 0);
    for (int i = 0; i < n; ++i) {
      src[i] = reinterpret_cast<uint64_t>(thetas[i]);
      o4[1 + i] = reinterpret_cast<uint64_t>(outs[i]);
    }
    // pointer tables are re-uploaded only when they change, so an apply with
    // the same buffers issues kernels only (and can be captured in a graph)
    if (src != b->last_src) {
      CUDA_OK(cudaMemcpyAsync(b->src_tab.p, src.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
      b->last_src = src;
    }
    if (o4 != b->last_out) {
      CUDA_OK(cudaMemcpyAsync(b->out_tab4.p, o4.data(), (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
      b->last_out = o4;
    }
    for (int stage = 0; stage < 4; ++stage)
      heff_batch_stage(b, stage, st, b->src_tab.as<uint64_t>(), b->out_tab4.as<uint64_t>());
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

int tnx_heff_batch_apply_host(tnx_heff_batch* b, const double* const* host_in, double* const* host_out,
                              int32_t n_steps, void* stream) {
  TNX_TRY({
    if (n_steps < 0) return set_err(TNX_ERR_VALUE, "n_steps must be >= 0");
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    const int n = static_cast<int>(b->hs.size());
    const size_t bytes = static_cast<size_t>(b->th_total) * sizeof(double);
    if (!b->s_h2d) {
      CUDA_OK(cudaStreamCreateWithFlags(&b->s_h2d, cudaStreamNonBlocking));
      CUDA_OK(cudaStreamCreateWithFlags(&b->s_d2h, cudaStreamNonBlocking));
      CUDA_OK(cudaEventCreateWithFlags(&b->ev_start, cudaEventDisableTiming));
      for (int k = 0; k < 2; ++k) {
        CUDA_OK(cudaEventCreateWithFlags(&b->ev_in_ready[k], cudaEventDisableTiming));
        CUDA_OK(cudaEventCreateWithFlags(&b->ev_done[k], cudaEventDisableTiming));
        CUDA_OK(cudaEventCreateWithFlags(&b->ev_out_free[k], cudaEventDisableTiming));
        b->pipe_in[k].alloc(std::max<size_t>(8, bytes));
        b->pipe_out[k].alloc(std::max<size_t>(8, bytes));
        std::vector<uint64_t> src(n), o4(n + 1, 0);
        for (int i = 0; i < n; ++i) {
          src[i] = reinterpret_cast<uint64_t>(b->pipe_in[k].as<double>() + b->th_off[i]);
          o4[1 + i] = reinterpret_cast<uint64_t>(b->pipe_out[k].as<double>() + b->th_off[i]);
        }
        upload(b->pipe_src_tab[k], src);
        upload(b->pipe_out_tab[k], o4);
      }
      CUDA_OK(cudaDeviceSynchronize());
    }
    if (n_steps == 0) return TNX_OK;
    // the copy streams start after the work already queued on the caller's stream
    CUDA_OK(cudaEventRecord(b->ev_start, cs));
    CUDA_OK(cudaStreamWaitEvent(b->s_h2d, b->ev_start, 0));
    CUDA_OK(cudaStreamWaitEvent(b->s_d2h, b->ev_start, 0));
    for (int i = 0; i < n_steps; ++i) {
      const int k = i & 1;
      // in[k] is free once step i-2 has computed; out[k] once its copy-out ended
      if (i >= 2) CUDA_OK(cudaStreamWaitEvent(b->s_h2d, b->ev_done[k], 0));
      if (bytes) CUDA_OK(cudaMemcpyAsync(b->pipe_in[k].p, host_in[i], bytes, cudaMemcpyHostToDevice, b->s_h2d));
      CUDA_OK(cudaEventRecord(b->ev_in_ready[k], b->s_h2d));
      CUDA_OK(cudaStreamWaitEvent(cs, b->ev_in_ready[k], 0));
      if (i >= 2) CUDA_OK(cudaStreamWaitEvent(cs, b->ev_out_free[k], 0));
      for (int stage = 0; stage < 4; ++stage)
        heff_batch_stage(b, stage, cs, b->pipe_src_tab[k].as<uint64_t>(), b->pipe_out_tab[k].as<uint64_t>());
      CUDA_OK(cudaEventRecord(b->ev_done[k], cs));
      CUDA_OK(cudaStreamWaitEvent(b->s_d2h, b->ev_done[k], 0));
      if (bytes) CUDA_OK(cudaMemcpyAsync(host_out[i], b->pipe_out[k].p, bytes, cudaMemcpyDeviceToHost, b->s_d2h));
      CUDA_OK(cudaEventRecord(b->ev_out_free[k], b->s_d2h));
    }
    // the caller's stream completes after the last copy-out
    CUDA_OK(cudaStreamWaitEvent(cs, b->ev_out_free[(n_steps - 1) & 1], 0));
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

int tnx_heff_batch_size(const tnx_heff_batch* b, int64_t* total, int64_t* offsets) {
  *total = b->th_total;
  if (offsets)
    for (size_t i = 0; i < b->th_off.size(); ++i) offsets[i] = b->th_off[i];
  return TNX_OK;
}

int tnx_heff_batch_apply_stage(tnx_heff_batch* b, int32_t stage, void* stream) {
  TNX_TRY({
    if (stage < 0 || stage > 3) return set_err(TNX_ERR_VALUE, "stage must be 0..3");
    if (b->last_src.empty()) return set_err(TNX_ERR_VALUE, "call tnx_heff_batch_apply once first");
    heff_batch_stage(b, stage, static_cast<cudaStream_t>(stream), b->src_tab.as<uint64_t>(),
                     b->out_tab4.as<uint64_t>());
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

int tnx_heff_stage_flops(const tnx_heff* h, double* flops3) {
  flops3[0] = h->H.flops_s1;
  flops3[1] = h->H.flops_mpo;
  flops3[2] = h->H.flops_s4;
  return TNX_OK;
}

void tnx_heff_batch_destroy(tnx_heff_batch* b) { delete b; }

int tnx_heff_batch_error(tnx_heff_batch* b, int32_t* err) {
  TNX_TRY({
    CUDA_OK(cudaMemcpy(err, b->err.p, sizeof(int32_t), cudaMemcpyDeviceToHost));
    return TNX_OK;
  })
}

// ---------------------------------------------------------------------------
// vectors
// ---------------------------------------------------------------------------
int64_t tnx_reduce_scratch_len(void) { return reduce_partials_count(); }

}  // extern "C"

// ---------------------------------------------------------------------------
// device-side sector planning
// ---------------------------------------------------------------------------
namespace {
// Distinct charges of every leg on the device, with their counts read back.
struct DevLegs {
  DevMem charges, leg_off, uniq, mult, n_uniq, status;
  std::vector<int64_t> off;
  std::vector<int32_t> nu;
};

// Gather legs' device charge arrays into one buffer and find their distinct
// charges; throws on a range the kernel cannot histogram.
void dev_legs(DevLegs& D, const std::vector<const int32_t*>& ch, const std::vector<int64_t>& dims, cudaStream_t st) {
  const int n = static_cast<int>(ch.size());
  D.off.assign(n + 1, 0);
  for (int l = 0; l < n; ++l) D.off[l + 1] = D.off[l] + dims[l];
  D.charges.alloc(std::max<int64_t>(1, D.off[n]) * 4);
  for (int l = 0; l < n; ++l)
    if (dims[l])
      CUDA_OK(cudaMemcpyAsync(D.charges.as<int32_t>() + D.off[l], ch[l], dims[l] * 4, cudaMemcpyDeviceToDevice, st));
  upload(D.leg_off, D.off, st);
  D.uniq.alloc(std::max<int64_t>(1, D.off[n]) * 4);
  D.mult.alloc(std::max<int64_t>(1, D.off[n]) * 4);
  D.n_uniq.alloc(std::max(1, n) * 4);
  D.status.alloc(std::max(1, n) * 4);
  launch_unique_charges(n, D.charges.as<int32_t>(), D.leg_off.as<int64_t>(), D.uniq.as<int32_t>(),
                        D.mult.as<int32_t>(), D.n_uniq.as<int32_t>(), D.status.as<int32_t>(), st);
  CUDA_OK(cudaGetLastError());
  D.nu.assign(n, 0);
  std::vector<int32_t> stat(n, 0);
  if (n) {
    CUDA_OK(cudaMemcpyAsync(D.nu.data(), D.n_uniq.p, n * 4, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(stat.data(), D.status.p, n * 4, cudaMemcpyDeviceToHost, st));
  }
  CUDA_OK(cudaStreamSynchronize(st));
  for (int l = 0; l < n; ++l)
    if (stat[l]) throw PlanError{TNX_ERR_UNSUPPORTED, "a leg's charge range exceeds 65536 (device planner)"};
}

// The reference-order valid keys of the legs in D into an owned device
// buffer; returns the count.
int64_t dev_valid_blocks(const DevLegs& D, const std::vector<int32_t>& flows, int32_t modulus, int64_t eff,
                         DevMem& keys_out, cudaStream_t st) {
  const int n = static_cast<int>(flows.size());
  if (n == 0) {
    keys_out.alloc(4);
    return 1;  // the empty key
  }
  const int64_t kCap = int64_t(1) << 24;
  int64_t entries = 1, max_nq = 1;
  for (int l = 0; l < n; ++l) max_nq = std::max<int64_t>(max_nq, D.nu[l]);
  for (int l = 0; l + 1 < n; ++l) {
    entries *= std::max<int64_t>(1, D.nu[l]);
    if (entries > kCap) throw PlanError{TNX_ERR_UNSUPPORTED, "too many partial keys for the device planner"};
  }
  entries = std::max(entries, max_nq);
  const int64_t cap_grid = std::min<int64_t>(kCap, entries * max_nq);
  const int64_t out_cap = std::min<int64_t>(kCap, entries * max_nq);
  DevMem kb[2], ob[2], sb[2], cb[2], gnf, grank, goff, gfirst, cnt;
  int32_t* kp[2];
  int64_t* op[2];
  int32_t* sp[2];
  int32_t* cp[2];
  for (int i = 0; i < 2; ++i) {
    kb[i].alloc(entries * kMaxLegsDev * 4);
    ob[i].alloc(entries * 8);
    sb[i].alloc(entries * 4);
    cb[i].alloc(entries * 4);
    kp[i] = kb[i].as<int32_t>();
    op[i] = ob[i].as<int64_t>();
    sp[i] = sb[i].as<int32_t>();
    cp[i] = cb[i].as<int32_t>();
  }
  gnf.alloc(cap_grid * 8);
  grank.alloc(cap_grid * 4);
  goff.alloc(cap_grid * 4);
  gfirst.alloc(cap_grid * 4);
  cnt.alloc(8);
  keys_out.alloc(std::max<int64_t>(1, out_cap) * n * 4);
  DevMem dfl;
  upload(dfl, flows, st);
  launch_valid_blocks(n, D.uniq.as<int32_t>(), D.leg_off.as<int64_t>(), D.n_uniq.as<int32_t>(), dfl.as<int32_t>(),
                      modulus, eff, kp, op, sp, cp, gnf.as<int64_t>(), grank.as<int32_t>(), goff.as<int32_t>(),
                      gfirst.as<int32_t>(), entries, entries, cap_grid, keys_out.as<int32_t>(), out_cap,
                      cnt.as<int64_t>(), st);
  CUDA_OK(cudaGetLastError());
  int64_t count = 0;
  CUDA_OK(cudaMemcpyAsync(&count, cnt.p, 8, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  if (count < 0) throw PlanError{TNX_ERR_UNSUPPORTED, "device planner capacity exceeded"};
  return count;
}
}  // namespace

extern "C" {

int tnx_valid_blocks_dev(int32_t n_legs, const int32_t* charges_dev, const int64_t* leg_dims, const int32_t* flows,
                         int32_t modulus, int32_t has_target, int64_t target, int64_t* n_keys, int32_t* keys_dev,
                         int64_t keys_cap, void* stream) {
  TNX_TRY({
    if (n_legs < 0 || n_legs > kMaxLegs) return set_err(TNX_ERR_UNSUPPORTED, "at most 12 legs");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<const int32_t*> ch(n_legs);
    std::vector<int64_t> dims(leg_dims, leg_dims + n_legs);
    int64_t off = 0;
    for (int l = 0; l < n_legs; ++l) {
      ch[l] = charges_dev + off;
      off += dims[l];
    }
    DevLegs D;
    dev_legs(D, ch, dims, st);
    DevMem keys;
    const int64_t n = dev_valid_blocks(D, std::vector<int32_t>(flows, flows + n_legs), modulus,
                                       has_target ? target : 0, keys, st);
    *n_keys = n;
    if (keys_dev) {
      if (keys_cap < n * n_legs) return set_err(TNX_ERR_VALUE, "keys_out capacity too small");
      if (n * n_legs) CUDA_OK(cudaMemcpyAsync(keys_dev, keys.p, n * n_legs * 4, cudaMemcpyDeviceToDevice, st));
    }
    CUDA_OK(cudaStreamSynchronize(st));
    return TNX_OK;
  })
}

int tnx_contract_structure_dev(const tnx_tensor_desc* a, const tnx_tensor_desc* b, const char* out_subs,
                               int32_t modulus, int64_t* n_out_blocks, int32_t* out_keys_dev, int64_t* out_offsets_dev,
                               int64_t out_cap, int64_t* n_pairs, int32_t* pairs_dev, int64_t pairs_cap,
                               void* stream) {
  TNX_TRY({
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!a || !b || !out_subs || !a->subs || !b->subs) return set_err(TNX_ERR_VALUE, "null argument");
    const std::string sa(a->subs), sb(b->subs), so(out_subs);
    if (static_cast<int>(sa.size()) != a->n_legs || static_cast<int>(sb.size()) != b->n_legs)
      return set_err(TNX_ERR_VALUE, "subscripts do not match leg counts");
    if (static_cast<int>(so.size()) > kMaxLegs || a->n_legs > kMaxLegs || b->n_legs > kMaxLegs)
      return set_err(TNX_ERR_UNSUPPORTED, "at most 12 legs");
    MatchArgs m{};
    m.la = a->n_legs;
    m.lb = b->n_legs;
    m.lo = static_cast<int32_t>(so.size());
    std::string con;
    for (char c : sa)
      if (sb.find(c) != std::string::npos) con.push_back(c);
    std::sort(con.begin(), con.end());
    m.n_con = static_cast<int32_t>(con.size());
    for (int i = 0; i < m.n_con; ++i) {
      m.a_con[i] = static_cast<int32_t>(sa.find(con[i]));
      m.b_con[i] = static_cast<int32_t>(sb.find(con[i]));
    }
    std::vector<int64_t> a_off(m.la + 1, 0), b_off(m.lb + 1, 0);
    for (int l = 0; l < m.la; ++l) a_off[l + 1] = a_off[l] + a->leg_dims[l];
    for (int l = 0; l < m.lb; ++l) b_off[l + 1] = b_off[l] + b->leg_dims[l];
    std::vector<const int32_t*> och;
    std::vector<int64_t> odims;
    std::vector<int32_t> oflows;
    for (int l = 0; l < m.lo; ++l) {
      const char c = so[l];
      const size_t pa = sa.find(c), pb = sb.find(c);
      if (con.find(c) != std::string::npos) return set_err(TNX_ERR_VALUE, "an output subscript is contracted");
      if (pa != std::string::npos) {
        m.o_src[l] = static_cast<int32_t>(pa);
        och.push_back(a->charges + a_off[pa]);
        odims.push_back(a->leg_dims[pa]);
        oflows.push_back(a->flows[pa]);
      } else if (pb != std::string::npos) {
        m.o_src[l] = m.la + static_cast<int32_t>(pb);
        och.push_back(b->charges + b_off[pb]);
        odims.push_back(b->leg_dims[pb]);
        oflows.push_back(b->flows[pb]);
      } else {
        return set_err(TNX_ERR_VALUE, std::string("output subscript '") + c + "' is not a free index");
      }
    }
    // the output target: operands whose blocks all carry one total charge
    DevMem fa, fb, tg;
    upload(fa, std::vector<int32_t>(a->flows, a->flows + m.la), st);
    upload(fb, std::vector<int32_t>(b->flows, b->flows + m.lb), st);
    tg.alloc(4 * 8);
    launch_operand_target(a->keys, m.la, a->n_blocks, fa.as<int32_t>(), tg.as<int64_t>(), st);
    launch_operand_target(b->keys, m.lb, b->n_blocks, fb.as<int32_t>(), tg.as<int64_t>() + 2, st);
    CUDA_OK(cudaGetLastError());
    int64_t t[4];
    CUDA_OK(cudaMemcpyAsync(t, tg.p, sizeof(t), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    const int64_t total = (t[1] ? t[0] : 0) + (t[3] ? t[2] : 0);
    // valid output keys (reference order), sorted for lookup
    DevLegs D;
    dev_legs(D, och, odims, st);
    DevMem valid;
    const int64_t nv = dev_valid_blocks(D, oflows, modulus, total, valid, st);
    int64_t pow2 = 1;
    while (pow2 < nv) pow2 <<= 1;
    if (pow2 > (int64_t(1) << 16)) return set_err(TNX_ERR_UNSUPPORTED, "too many valid output keys (device planner)");
    DevMem perm, vsorted;
    perm.alloc(pow2 * 4);
    vsorted.alloc(std::max<int64_t>(1, nv * m.lo) * 4);
    if (m.lo > 0 && nv > 0) launch_sort_keys(valid.as<int32_t>(), m.lo, perm.as<int32_t>(), nv, pow2,
                                             vsorted.as<int32_t>(), st);
    // matching: counts per A block, their offsets, then the pairs
    const int64_t na = a->n_blocks, nb = b->n_blocks;
    DevMem rc, rb, pr, present;
    rc.alloc(std::max<int64_t>(1, na) * 4);
    launch_match(m, a->keys, na, b->keys, nb, vsorted.as<int32_t>(), nv, 0, rc.as<int32_t>(), nullptr, nullptr,
                 nullptr, st);
    CUDA_OK(cudaGetLastError());
    std::vector<int32_t> counts(na);
    if (na) CUDA_OK(cudaMemcpyAsync(counts.data(), rc.p, na * 4, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    std::vector<int64_t> base(na + 1, 0);
    for (int64_t i = 0; i < na; ++i) base[i + 1] = base[i] + counts[i];
    const int64_t np = base[na];
    upload(rb, base, st);
    pr.alloc(std::max<int64_t>(1, np) * sizeof(int4));
    present.alloc(std::max<int64_t>(1, nv) * 4);
    CUDA_OK(cudaMemsetAsync(present.p, 0, present.n, st));
    launch_match(m, a->keys, na, b->keys, nb, vsorted.as<int32_t>(), nv, 1, nullptr, rb.as<int64_t>(),
                 pr.as<int4>(), present.as<int32_t>(), st);
    DevMem vmap, okeys, ooffs, nout;
    vmap.alloc(std::max<int64_t>(1, nv) * 4);
    okeys.alloc(std::max<int64_t>(1, nv * std::max(1, static_cast<int>(m.lo))) * 4);
    ooffs.alloc((nv + 1) * 8);
    nout.alloc(8);
    launch_compact_out(vsorted.as<int32_t>(), nv, m.lo, present.as<int32_t>(), D.uniq.as<int32_t>(),
                       D.mult.as<int32_t>(), D.leg_off.as<int64_t>(), D.n_uniq.as<int32_t>(), vmap.as<int32_t>(),
                       okeys.as<int32_t>(), ooffs.as<int64_t>(), nout.as<int64_t>(), pr.as<int4>(), np, st);
    CUDA_OK(cudaGetLastError());
    int64_t no = 0;
    CUDA_OK(cudaMemcpyAsync(&no, nout.p, 8, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    *n_out_blocks = no;
    *n_pairs = np;
    if (out_keys_dev || out_offsets_dev) {
      if (out_cap < no) return set_err(TNX_ERR_VALUE, "output capacity too small");
      if (out_keys_dev && no * m.lo)
        CUDA_OK(cudaMemcpyAsync(out_keys_dev, okeys.p, no * m.lo * 4, cudaMemcpyDeviceToDevice, st));
      if (out_offsets_dev)
        CUDA_OK(cudaMemcpyAsync(out_offsets_dev, ooffs.p, (no + 1) * 8, cudaMemcpyDeviceToDevice, st));
    }
    if (pairs_dev) {
      if (pairs_cap < np) return set_err(TNX_ERR_VALUE, "pairs capacity too small");
      // (A block, B block, output block) per pair
      if (np)
        CUDA_OK(cudaMemcpy2DAsync(pairs_dev, 3 * 4, pr.p, sizeof(int4), 3 * 4, np, cudaMemcpyDeviceToDevice, st));
    }
    CUDA_OK(cudaStreamSynchronize(st));
    return TNX_OK;
  })
}

int tnx_fused_charges_dev(const int32_t* qa_dev, int64_t da, int32_t fa, const int32_t* qb_dev, int64_t db,
                          int32_t fb, int32_t fused_flow, int32_t modulus, int32_t* out_dev, void* stream) {
  TNX_TRY({
    launch_fused_charges(qa_dev, da, fa, qb_dev, db, fb, fused_flow, modulus, out_dev,
                         static_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

int tnx_dot(const double* x, const double* y, int64_t n, double* result, double* scratch, void* stream) {
  TNX_TRY({
    launch_dot(x, y, n, 0, result, scratch, nullptr, static_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

int64_t tnx_renorm_scratch_len(void) { return 2 * kRenormMax * kRenormBlocks; }

static int renorm_args(int n_tensors, const double* const* x, const double* const* g, double* const* y,
                       const int64_t* n, RenormArgs& a) {
  if (n_tensors < 1 || n_tensors > kRenormMax) {
    return set_err(TNX_ERR_VALUE, "renormalisation takes between 1 and " + std::to_string(kRenormMax) +
                                      " tensors per call, got " + std::to_string(n_tensors));
  }
  a = RenormArgs{};
  for (int t = 0; t < n_tensors; ++t) {
    if (n[t] < 0) return set_err(TNX_ERR_VALUE, "renormalisation: negative tensor size");
    a.x[t] = x[t];
    a.g[t] = g ? g[t] : nullptr;
    a.y[t] = y[t];
    a.n[t] = n[t];
  }
  return TNX_OK;
}

int tnx_renorm_maxabs(int n_tensors, const double* const* x, double* const* y, const int64_t* n, double eps,
                      double* stat, double* scratch, void* stream) {
  TNX_TRY({
    RenormArgs a;
    int rc = renorm_args(n_tensors, x, nullptr, y, n, a);
    if (rc != TNX_OK) return rc;
    launch_renorm(a, n_tensors, eps, stat, scratch, static_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

int tnx_renorm_maxabs_adjoint(int n_tensors, const double* const* x, const double* const* gy, double* const* gx,
                              const int64_t* n, double eps, const double* stat, double* scratch, void* stream) {
  TNX_TRY({
    RenormArgs a;
    int rc = renorm_args(n_tensors, x, gy, gx, n, a);
    if (rc != TNX_OK) return rc;
    launch_renorm_adjoint(a, n_tensors, eps, stat, scratch, static_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

int tnx_wait_flag(const int32_t* flag, int32_t expected, int64_t timeout_ns, int32_t* status, void* stream) {
  TNX_TRY({
    if (!flag || !status) return set_err(TNX_ERR_VALUE, "tnx_wait_flag: null flag or status");
    if (timeout_ns <= 0 || timeout_ns > 10000000000ll)
      return set_err(TNX_ERR_VALUE, "tnx_wait_flag: timeout must be in (0, 10 s]");
    launch_wait_flag(flag, expected, static_cast<uint64_t>(timeout_ns), status, static_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

int tnx_svd_batch(int32_t n, const int64_t* m, const int64_t* k, const double* const* a, double* const* u,
                  double* const* s, double* const* vh, int64_t polar_min, int32_t n_workers, double* err_sigma,
                  void* stream) {
  TNX_TRY({
    if (n < 0) return set_err(TNX_ERR_VALUE, "tnx_svd_batch: negative sector count");
    if (n > 0 && (!m || !k || !a || !u || !s || !vh)) return set_err(TNX_ERR_VALUE, "tnx_svd_batch: null array");
    std::vector<SvdJob> jobs(static_cast<size_t>(n));
    for (int32_t i = 0; i < n; ++i) jobs[i] = SvdJob{m[i], k[i], a[i], u[i], s[i], vh[i]};
    const double e = svd_batch(jobs, polar_min, n_workers, static_cast<cudaStream_t>(stream));
    if (err_sigma) *err_sigma = e;
    return TNX_OK;
  })
}

int tnx_nrm2(const double* x, int64_t n, double* result, double* scratch, void* stream) {
  TNX_TRY({
    launch_dot(x, x, n, 1, result, scratch, nullptr, static_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

int tnx_lanczos_step(double* w, const double* v, const double* v_prev, double* v_next, int64_t n, double* alpha,
                     double* beta, int32_t k, double tol, double tol_rel, int32_t* done, double* scratch,
                     void* stream) {
  TNX_TRY({
    launch_lanczos_step(w, v, k > 0 ? v_prev : nullptr, v_next, n, alpha + k, beta + k + 1, beta + k, tol, tol_rel,
                        done, scratch, static_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

int tnx_combine(const double* const* basis_dev_table, const double* coefs_dev, int32_t n_vec, int64_t n, double* out,
                void* stream) {
  TNX_TRY({
    launch_combine(basis_dev_table, coefs_dev, n_vec, n, out, static_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

int tnx_scale(const double* x, double* out, int64_t n, const double* scale_dev, int32_t mode, void* stream) {
  TNX_TRY({
    launch_scale(x, out, n, scale_dev, mode, nullptr, static_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TNX_OK;
  })
}

}  // extern "C"

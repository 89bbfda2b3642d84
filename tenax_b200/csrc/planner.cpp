// Exact integer planning for block-sparse symmetric contractions (host side).
#include "planner.hpp"

#include <algorithm>
#include <numeric>
#include <set>
#include <utility>

namespace tnx {

static int64_t fuse_q(int64_t a, int64_t b, int32_t modulus) {
  // U(1): a + b; Z_n: (a + b) mod n with a Python-style non-negative result
  // (core/symmetry.py:194-195, 236-237)
  if (modulus == 0) return a + b;
  int64_t r = (a + b) % modulus;
  return r < 0 ? r + modulus : r;
}

void TensorStruct::finalize_leg_maps() {
  cdim.assign(nl, {});
  for (int l = 0; l < nl; ++l)
    for (int32_t q : charges[l]) cdim[l][q] += 1;
}

void TensorStruct::layout_blocks() {
  dims.assign(keys.size(), std::vector<int64_t>(nl, 0));
  offs.assign(keys.size(), 0);
  int64_t off = 0;
  for (size_t b = 0; b < keys.size(); ++b) {
    int64_t n = 1;
    for (int l = 0; l < nl; ++l) {
      dims[b][l] = leg_dim(l, keys[b][l]);
      n *= dims[b][l];
    }
    offs[b] = off;
    off += n;
  }
  total = off;
}

// _compute_valid_blocks (core/tensor.py:53-165): unique charges sorted per leg,
// partial sums kept in first-insertion order, last leg solved (U1) or
// enumerated (Z_n).
std::vector<Key> valid_blocks(const std::vector<std::vector<int32_t>>& charges, const std::vector<int32_t>& flows,
                              int32_t modulus, bool has_target, int64_t target) {
  const int n = static_cast<int>(charges.size());
  std::vector<Key> out;
  if (n == 0) {
    out.push_back({});
    return out;
  }
  const int64_t eff = has_target ? target : 0;
  std::vector<std::vector<int32_t>> uniq(n);
  for (int l = 0; l < n; ++l) {
    std::set<int32_t> s(charges[l].begin(), charges[l].end());
    uniq[l].assign(s.begin(), s.end());
  }
  if (n == 1) {
    for (int32_t q : uniq[0])
      if (static_cast<int64_t>(flows[0]) * q == eff) out.push_back({q});
    return out;
  }
  // ordered dict: fused value -> list of partial keys
  std::vector<int64_t> order;
  std::unordered_map<int64_t, std::vector<Key>> part;
  for (int32_t q : uniq[0]) {
    int64_t f = static_cast<int64_t>(flows[0]) * q;
    if (!part.count(f)) order.push_back(f);
    part[f].push_back({q});
  }
  const int last = n - 1;
  for (int li = 1; li < last; ++li) {
    std::vector<int64_t> norder;
    std::unordered_map<int64_t, std::vector<Key>> npart;
    for (int32_t q : uniq[li]) {
      int64_t eq = static_cast<int64_t>(flows[li]) * q;
      for (int64_t prev : order) {
        // the reference fuses through int32 numpy arrays; charges stay small
        int64_t nf = fuse_q(prev, eq, modulus);
        auto& dst = npart[nf];
        if (dst.empty() && std::find(norder.begin(), norder.end(), nf) == norder.end()) norder.push_back(nf);
        for (const Key& c : part[prev]) {
          Key k = c;
          k.push_back(q);
          dst.push_back(std::move(k));
        }
      }
    }
    order.swap(norder);
    part.swap(npart);
  }
  const int64_t fl = flows[last];
  if (modulus == 0) {
    std::set<int32_t> lastset(uniq[last].begin(), uniq[last].end());
    for (int64_t prev : order) {
      if (fl == 0) continue;
      int64_t ql = (eff - prev) * fl;
      if (ql >= INT32_MIN && ql <= INT32_MAX && lastset.count(static_cast<int32_t>(ql))) {
        for (const Key& c : part[prev]) {
          Key k = c;
          k.push_back(static_cast<int32_t>(ql));
          out.push_back(std::move(k));
        }
      }
    }
  } else {
    for (int32_t q : uniq[last]) {
      int64_t eq = fl * q;
      for (int64_t prev : order) {
        if (fuse_q(prev, eq, modulus) == eff) {
          for (const Key& c : part[prev]) {
            Key k = c;
            k.push_back(q);
            out.push_back(std::move(k));
          }
        }
      }
    }
  }
  return out;
}

// --------------------------------------------------------------------------
// union-find
// --------------------------------------------------------------------------
namespace {
struct DSU {
  std::vector<int> p;
  int add() {
    p.push_back(static_cast<int>(p.size()));
    return static_cast<int>(p.size()) - 1;
  }
  int find(int x) {
    while (p[x] != x) {
      p[x] = p[p[x]];
      x = p[x];
    }
    return x;
  }
  void unite(int a, int b) {
    a = find(a);
    b = find(b);
    if (a != b) p[std::max(a, b)] = std::min(a, b);
  }
};

struct NodeTable {
  std::map<Key, int> idx;  // ordered for determinism
  std::vector<Key> keys;
  std::vector<int64_t> size;
  std::vector<int> dsu_id;
  int get(const Key& k, int64_t sz, DSU& d) {
    auto it = idx.find(k);
    if (it != idx.end()) return it->second;
    int id = static_cast<int>(keys.size());
    idx.emplace(k, id);
    keys.push_back(k);
    size.push_back(sz);
    dsu_id.push_back(d.add());
    return id;
  }
};
}  // namespace

PairPlan plan_pair(const TensorStruct& A, const TensorStruct& B, const std::string& out_subs,
                   const KeyFilter& filter, const std::vector<std::vector<int32_t>>* out_charges,
                   const std::vector<int32_t>* out_flows, int k_align, int n_align) {
  if (k_align < 1) k_align = 1;
  if (n_align < 1) n_align = 1;
  PairPlan P;
  P.a_subs = A.subs;
  P.b_subs = B.subs;
  P.out_subs = out_subs;
  // classify chars
  for (int i = 0; i < A.nl; ++i)
    for (int j = i + 1; j < A.nl; ++j)
      if (A.subs[i] == A.subs[j]) throw PlanError{6, "repeated subscript within one operand (trace) is not supported"};
  for (int i = 0; i < B.nl; ++i)
    for (int j = i + 1; j < B.nl; ++j)
      if (B.subs[i] == B.subs[j]) throw PlanError{6, "repeated subscript within one operand (trace) is not supported"};
  std::vector<int> a_con, a_free, b_con, b_free;  // leg positions
  std::vector<char> con_chars;                     // canonical order: as in A
  for (int i = 0; i < A.nl; ++i) {
    if (B.subs.find(A.subs[i]) != std::string::npos) {
      a_con.push_back(i);
      con_chars.push_back(A.subs[i]);
    } else {
      a_free.push_back(i);
    }
  }
  for (char c : con_chars) b_con.push_back(static_cast<int>(B.subs.find(c)));
  for (int j = 0; j < B.nl; ++j)
    if (A.subs.find(B.subs[j]) == std::string::npos) b_free.push_back(j);
  // output legs map to A-free or B-free
  if (out_subs.size() != a_free.size() + b_free.size())
    throw PlanError{1, "output subscripts must list every free index exactly once"};
  if (static_cast<int>(out_subs.size()) > kMaxLegs)
    throw PlanError{6, "contraction result has " + std::to_string(out_subs.size()) + " legs; at most " +
                           std::to_string(kMaxLegs) + " are supported"};
  struct OutLeg {
    bool from_a;
    int pos;  // leg position in A or B
    int fidx; // index into a_free / b_free
  };
  std::vector<OutLeg> olegs;
  for (char c : out_subs) {
    size_t pa = A.subs.find(c), pb = B.subs.find(c);
    if (pa != std::string::npos && std::find(a_free.begin(), a_free.end(), static_cast<int>(pa)) != a_free.end()) {
      olegs.push_back({true, static_cast<int>(pa),
                       static_cast<int>(std::find(a_free.begin(), a_free.end(), static_cast<int>(pa)) - a_free.begin())});
    } else if (pb != std::string::npos &&
               std::find(b_free.begin(), b_free.end(), static_cast<int>(pb)) != b_free.end()) {
      olegs.push_back({false, static_cast<int>(pb),
                       static_cast<int>(std::find(b_free.begin(), b_free.end(), static_cast<int>(pb)) - b_free.begin())});
    } else {
      throw PlanError{1, std::string("output subscript '") + c + "' is not a free index"};
    }
  }

  DSU dsu;
  NodeTable rn, kn, cn;
  std::vector<int64_t> k_real, c_real;  // unpadded K / column extents of each node (FLOP count)
  struct Edge {
    int block, r_or_c, k;
  };
  std::vector<Edge> ea, eb;
  for (size_t b = 0; b < A.keys.size(); ++b) {
    Key rk, kk;
    int64_t rs = 1, ks = 1;
    bool empty = false;
    for (int p : a_free) {
      rk.push_back(A.keys[b][p]);
      rs *= A.dims[b][p];
    }
    int64_t ks_img = 1;  // K extent in the image (innermost contracted leg padded)
    for (size_t i = 0; i < a_con.size(); ++i) {
      const int p = a_con[i];
      kk.push_back(A.keys[b][p]);
      ks *= A.dims[b][p];
      const int64_t d = A.dims[b][p];
      ks_img *= (i + 1 == a_con.size()) ? (d + k_align - 1) / k_align * k_align : d;
    }
    // kappa identity includes the contracted dims (mismatched dims never pair)
    for (int p : a_con) kk.push_back(static_cast<int32_t>(A.dims[b][p]));
    if (rs == 0 || ks == 0) empty = true;
    if (empty) continue;
    int r = rn.get(rk, rs, dsu), k = kn.get(kk, ks_img, dsu);
    if (static_cast<size_t>(k) >= k_real.size()) k_real.resize(k + 1, 0);
    k_real[k] = ks;
    dsu.unite(rn.dsu_id[r], kn.dsu_id[k]);
    ea.push_back({static_cast<int>(b), r, k});
  }
  for (size_t b = 0; b < B.keys.size(); ++b) {
    Key ck, kk;
    int64_t cs = 1, ks = 1, cs_img = 1;  // cs_img: column extent with the innermost free leg padded
    for (size_t i = 0; i < b_free.size(); ++i) {
      const int p = b_free[i];
      ck.push_back(B.keys[b][p]);
      cs *= B.dims[b][p];
      const int64_t d = B.dims[b][p];
      cs_img *= (i + 1 == b_free.size()) ? (d + n_align - 1) / n_align * n_align : d;
    }
    for (int p : b_con) {
      kk.push_back(B.keys[b][p]);
      ks *= B.dims[b][p];
    }
    for (int p : b_con) kk.push_back(static_cast<int32_t>(B.dims[b][p]));
    if (cs == 0 || ks == 0) continue;
    auto it = kn.idx.find(kk);
    if (it == kn.idx.end()) continue;  // no A block shares this contracted tuple
    int c = cn.get(ck, cs_img, dsu);
    if (static_cast<size_t>(c) >= c_real.size()) c_real.resize(c + 1, 0);
    c_real[c] = cs;
    dsu.unite(cn.dsu_id[c], kn.dsu_id[it->second]);
    eb.push_back({static_cast<int>(b), c, it->second});
  }
  // contributing pairs: A(r,k) and B(k,c)
  std::vector<std::vector<int>> a_by_k(kn.keys.size()), b_by_k(kn.keys.size());
  for (size_t i = 0; i < ea.size(); ++i) a_by_k[ea[i].k].push_back(static_cast<int>(i));
  for (size_t i = 0; i < eb.size(); ++i) b_by_k[eb[i].k].push_back(static_cast<int>(i));
  // components that hold at least one contributing pair
  std::map<int, int> comp_gid;  // dsu root -> group id
  std::vector<int> k_root(kn.keys.size());
  for (size_t k = 0; k < kn.keys.size(); ++k) k_root[k] = dsu.find(kn.dsu_id[k]);
  // groups ordered by their smallest kappa key (NodeTable keys are map-ordered
  // by id of first appearance; use sorted kappa keys for determinism)
  std::vector<int> k_sorted(kn.keys.size());
  std::iota(k_sorted.begin(), k_sorted.end(), 0);
  std::sort(k_sorted.begin(), k_sorted.end(), [&](int x, int y) { return kn.keys[x] < kn.keys[y]; });
  for (int k : k_sorted) {
    if (a_by_k[k].empty() || b_by_k[k].empty()) continue;
    int root = k_root[k];
    if (!comp_gid.count(root)) {
      int gid = static_cast<int>(comp_gid.size());
      comp_gid[root] = gid;
    }
  }
  const int G = static_cast<int>(comp_gid.size());
  P.groups.assign(G, {});
  P.g_rows.assign(G, {});
  P.g_cols.assign(G, {});
  P.g_ks.assign(G, {});
  std::vector<int64_t> r_start(rn.keys.size(), -1), c_start(cn.keys.size(), -1), k_start(kn.keys.size(), -1);
  std::vector<int> r_group(rn.keys.size(), -1), c_group(cn.keys.size(), -1), k_group(kn.keys.size(), -1);
  // assign kappa ranges (sorted kappa order)
  for (int k : k_sorted) {
    if (a_by_k[k].empty() || b_by_k[k].empty()) continue;
    int g = comp_gid[k_root[k]];
    k_group[k] = g;
    k_start[k] = P.groups[g].K;
    P.g_ks[g].push_back({kn.keys[k], P.groups[g].K, kn.size[k]});
    P.groups[g].K += kn.size[k];
  }
  // rows: r nodes that have an edge to a used kappa, sorted by key
  {
    std::vector<int> rs(rn.keys.size());
    std::iota(rs.begin(), rs.end(), 0);
    std::sort(rs.begin(), rs.end(), [&](int x, int y) { return rn.keys[x] < rn.keys[y]; });
    std::vector<char> used(rn.keys.size(), 0);
    for (auto& e : ea)
      if (k_group[e.k] >= 0) used[e.r_or_c] = 1;
    for (int r : rs) {
      if (!used[r]) continue;
      int g = comp_gid[dsu.find(rn.dsu_id[r])];
      r_group[r] = g;
      r_start[r] = P.groups[g].M;
      P.g_rows[g].push_back({rn.keys[r], P.groups[g].M, rn.size[r]});
      P.groups[g].M += rn.size[r];
    }
    std::vector<int> cs(cn.keys.size());
    std::iota(cs.begin(), cs.end(), 0);
    std::sort(cs.begin(), cs.end(), [&](int x, int y) { return cn.keys[x] < cn.keys[y]; });
    std::vector<char> cused(cn.keys.size(), 0);
    for (auto& e : eb)
      if (k_group[e.k] >= 0) cused[e.r_or_c] = 1;
    for (int c : cs) {
      if (!cused[c]) continue;
      int g = comp_gid[dsu.find(cn.dsu_id[c])];
      c_group[c] = g;
      c_start[c] = P.groups[g].N;
      P.g_cols[g].push_back({cn.keys[c], P.groups[g].N, cn.size[c]});
      P.groups[g].N += cn.size[c];
    }
  }
  // pack segments
  auto fill_strides = [](const std::vector<int64_t>& dims, const std::vector<int>& legs_in_order,
                         int32_t* out_str, int nl, int align = 1) {
    // stride of each leg in the row-major flattening over legs_in_order
    // (the innermost extent rounded up to a multiple of align)
    for (int l = 0; l < nl; ++l) out_str[l] = 0;
    int64_t s = 1;
    for (int i = static_cast<int>(legs_in_order.size()) - 1; i >= 0; --i) {
      out_str[legs_in_order[i]] = static_cast<int32_t>(s);
      const int64_t d = dims[legs_in_order[i]];
      s *= (i + 1 == static_cast<int>(legs_in_order.size())) ? (d + align - 1) / align * align : d;
    }
  };
  for (auto& e : ea) {
    if (k_group[e.k] < 0) continue;
    int b = e.block;
    PackSeg s{};
    s.src_off = A.offs[b];
    s.count = 1;
    for (int l = 0; l < A.nl; ++l) s.count *= A.dims[b][l];
    s.group = k_group[e.k];
    s.row0 = static_cast<int32_t>(r_start[e.r_or_c]);
    s.k0 = static_cast<int32_t>(k_start[e.k]);
    s.nlegs = A.nl;
    for (int l = 0; l < A.nl; ++l) s.dims[l] = static_cast<int32_t>(A.dims[b][l]);
    fill_strides(A.dims[b], a_free, s.rstr, A.nl);
    fill_strides(A.dims[b], a_con, s.kstr, A.nl);
    fill_strides(A.dims[b], a_con, s.kdstr, A.nl, k_align);
    P.packA.push_back(s);
  }
  for (auto& e : eb) {
    if (k_group[e.k] < 0) continue;
    int b = e.block;
    PackSeg s{};
    s.src_off = B.offs[b];
    s.count = 1;
    for (int l = 0; l < B.nl; ++l) s.count *= B.dims[b][l];
    s.group = k_group[e.k];
    s.row0 = static_cast<int32_t>(c_start[e.r_or_c]);
    s.k0 = static_cast<int32_t>(k_start[e.k]);
    s.nlegs = B.nl;
    for (int l = 0; l < B.nl; ++l) s.dims[l] = static_cast<int32_t>(B.dims[b][l]);
    fill_strides(B.dims[b], b_free, s.rstr, B.nl, n_align);
    fill_strides(B.dims[b], b_con, s.kstr, B.nl);
    fill_strides(B.dims[b], b_con, s.kdstr, B.nl, k_align);
    P.packB.push_back(s);
  }
  // contributing (r, c) pairs and flops
  std::map<std::pair<int, int>, int> present;  // (r,c) -> group
  for (size_t k = 0; k < kn.keys.size(); ++k) {
    if (k_group[k] < 0) continue;
    for (int ia : a_by_k[k])
      for (int ib : b_by_k[k]) {
        int r = ea[ia].r_or_c, c = eb[ib].r_or_c;
        present[{r, c}] = static_cast<int>(k_group[k]);
        P.flops += 2.0 * static_cast<double>(rn.size[r]) * static_cast<double>(c_real[c]) *
                   static_cast<double>(k_real[k]);
      }
  }
  // output blocks
  struct OutRec {
    Key key;
    int r, c, g;
  };
  std::vector<OutRec> outs;
  for (auto& kv : present) {
    int r = kv.first.first, c = kv.first.second;
    Key ok;
    for (auto& ol : olegs) ok.push_back(ol.from_a ? rn.keys[r][ol.fidx] : cn.keys[c][ol.fidx]);
    if (filter.active && !filter.allowed.count(ok)) continue;
    outs.push_back({ok, r, c, kv.second});
  }
  std::sort(outs.begin(), outs.end(), [](const OutRec& x, const OutRec& y) { return x.key < y.key; });
  for (size_t i = 1; i < outs.size(); ++i)
    if (outs[i].key == outs[i - 1].key) throw PlanError{3, "internal: duplicate output key"};
  TensorStruct& O = P.out;
  O.nl = static_cast<int>(out_subs.size());
  O.subs = out_subs;
  if (out_charges) O.charges = *out_charges;
  if (out_flows) O.flows = *out_flows;
  O.keys.clear();
  O.dims.clear();
  O.offs.clear();
  int64_t off = 0;
  for (auto& o : outs) {
    std::vector<int64_t> d(O.nl);
    // dims from the operand legs
    int b_a = -1, b_b = -1;
    (void)b_a;
    (void)b_b;
    std::vector<int64_t> rdims, cdims;  // dims of A-free / B-free legs
    for (size_t i = 0; i < olegs.size(); ++i) {
      const auto& ol = olegs[i];
      if (ol.from_a)
        d[i] = A.leg_dim(ol.pos, o.key[i]);
      else
        d[i] = B.leg_dim(ol.pos, o.key[i]);
    }
    int64_t n = 1;
    for (auto x : d) n *= x;
    O.keys.push_back(o.key);
    O.dims.push_back(d);
    O.offs.push_back(off);
    // scatter segment: out leg i contributes idx * stride to the group row or col
    ScatSeg s{};
    s.dst_off = off;
    s.count = n;
    s.group = o.g;
    s.row0 = static_cast<int32_t>(r_start[o.r]);
    s.col0 = static_cast<int32_t>(c_start[o.c]);
    s.nlegs = O.nl;
    // row flattening over A-free legs in A order; col over B-free in B order
    std::vector<int64_t> fa(a_free.size()), fb(b_free.size());
    for (size_t i = 0; i < olegs.size(); ++i) {
      if (olegs[i].from_a)
        fa[olegs[i].fidx] = d[i];
      else
        fb[olegs[i].fidx] = d[i];
    }
    std::vector<int64_t> sa(a_free.size()), sb(b_free.size());
    int64_t acc = 1;
    for (int i = static_cast<int>(fa.size()) - 1; i >= 0; --i) {
      sa[i] = acc;
      acc *= fa[i];
    }
    acc = 1;
    for (int i = static_cast<int>(fb.size()) - 1; i >= 0; --i) {
      sb[i] = acc;
      acc *= (i + 1 == static_cast<int>(fb.size())) ? (fb[i] + n_align - 1) / n_align * n_align : fb[i];
    }
    for (size_t i = 0; i < olegs.size(); ++i) {
      s.dims[i] = static_cast<int32_t>(d[i]);
      s.rstr[i] = olegs[i].from_a ? static_cast<int32_t>(sa[olegs[i].fidx]) : 0;
      s.cstr[i] = olegs[i].from_a ? 0 : static_cast<int32_t>(sb[olegs[i].fidx]);
    }
    P.scatter.push_back(s);
    off += n;
  }
  O.total = off;
  if (out_charges) O.finalize_leg_maps();
  return P;
}

// --------------------------------------------------------------------------
// H_eff plan
// --------------------------------------------------------------------------

static TensorStruct sub_struct(const std::string& subs, int nl) {
  TensorStruct t;
  t.nl = nl;
  t.subs = subs;
  return t;
}

HeffPlan plan_heff(const TensorStruct& L, const TensorStruct& th, const TensorStruct& Wl, const TensorStruct& Wr,
                   const TensorStruct& R, int x1_align) {
  HeffPlan H;
  H.x1_align = x1_align < 1 ? 1 : x1_align;
  H.L = L;
  H.th = th;
  H.Wl = Wl;
  H.Wr = Wr;
  H.R = R;
  H.L.subs = "abc";
  H.th.subs = "apqd";
  H.Wl.subs = "bpse";
  H.Wr.subs = "eqtf";
  H.R.subs = "dfg";
  if (L.nl != 3 || th.nl != 4 || Wl.nl != 4 || Wr.nl != 4 || R.nl != 3)
    throw PlanError{1, "H_eff operands must have 3,4,4,4,3 legs"};
  KeyFilter none;
  // stage 1: X1[b,c,p,q,d] = L[a,b,c] th[a,p,q,d]
  // K = a padded to a multiple of 8 per sector: theta is packed by whole
  // 8-wide K chunks (pack_rows_kernel)
  // N = (p,q,d) with d padded to a multiple of x1_align: every MPO input
  // slot of X1 starts on an aligned column (vector loads in the MPO kernel)
  H.s1 = plan_pair(H.L, H.th, "bcpqd", none, nullptr, nullptr, kMpoKAlign, H.x1_align);
  H.flops_s1 = H.s1.flops;
  // X1 blocks (present (r,c) pairs): r = (qb,qc), c = (qp,qq,qd)
  // stage 2 structure/flops: X2[c,s,e,q,d] = X1[b,c,p,q,d] Wl[b,p,s,e]
  // stage 3: X3[c,s,t,f,d] = X2[c,s,e,q,d] Wr[e,q,t,f]
  // Build X1 key list with dims
  struct Blk {
    Key k;
    std::vector<int64_t> d;
  };
  std::vector<Blk> x1;
  for (size_t i = 0; i < H.s1.out.keys.size(); ++i) x1.push_back({H.s1.out.keys[i], H.s1.out.dims[i]});
  // Wl by (qb,qp)
  std::map<std::pair<int32_t, int32_t>, std::vector<int>> wl_by_bp;
  for (size_t i = 0; i < Wl.keys.size(); ++i) {
    bool nz = true;
    for (int l = 0; l < 4; ++l) nz &= Wl.dims[i][l] > 0;
    if (nz) wl_by_bp[{Wl.keys[i][0], Wl.keys[i][1]}].push_back(static_cast<int>(i));
  }
  std::map<std::pair<int32_t, int32_t>, std::vector<int>> wr_by_eq;
  for (size_t i = 0; i < Wr.keys.size(); ++i) {
    bool nz = true;
    for (int l = 0; l < 4; ++l) nz &= Wr.dims[i][l] > 0;
    if (nz) wr_by_eq[{Wr.keys[i][0], Wr.keys[i][1]}].push_back(static_cast<int>(i));
  }
  // X2 keys (c,s,e,q,d) with dims, and flops of stage 2
  std::map<Key, std::vector<int64_t>> x2;
  H.flops_mpo = 0.0;
  for (auto& b : x1) {
    // X1 key order "bcpqd"
    int32_t qb = b.k[0], qc = b.k[1], qp = b.k[2], qq = b.k[3], qd = b.k[4];
    auto it = wl_by_bp.find({qb, qp});
    if (it == wl_by_bp.end()) continue;
    for (int wi : it->second) {
      int32_t qs = Wl.keys[wi][2], qe = Wl.keys[wi][3];
      int64_t ms = Wl.dims[wi][2], me = Wl.dims[wi][3];
      if (b.d[0] != Wl.dims[wi][0] || b.d[2] != Wl.dims[wi][1])
        throw PlanError{1, "H_eff: inconsistent block dims between theta/L and W_l"};
      Key k2 = {qc, qs, qe, qq, qd};
      x2[k2] = {b.d[1], ms, me, b.d[3], b.d[4]};
      H.flops_mpo += 2.0 * (double)(b.d[1] * b.d[3] * b.d[4]) * (double)(ms * me) * (double)(b.d[0] * b.d[2]);
    }
  }
  std::map<Key, std::vector<int64_t>> x3;  // key (c,s,t,f,d)
  for (auto& kv : x2) {
    const Key& k = kv.first;
    const auto& d = kv.second;
    auto it = wr_by_eq.find({k[2], k[3]});
    if (it == wr_by_eq.end()) continue;
    for (int wi : it->second) {
      int32_t qt = Wr.keys[wi][2], qf = Wr.keys[wi][3];
      int64_t mt = Wr.dims[wi][2], mf = Wr.dims[wi][3];
      if (d[2] != Wr.dims[wi][0] || d[3] != Wr.dims[wi][1])
        throw PlanError{1, "H_eff: inconsistent block dims between W_l and W_r"};
      Key k3 = {k[0], k[1], qt, qf, k[4]};
      x3[k3] = {d[0], d[1], mt, mf, d[4]};
      H.flops_mpo += 2.0 * (double)(d[0] * d[1] * d[4]) * (double)(mt * mf) * (double)(d[2] * d[3]);
    }
  }
  // X3 as a TensorStruct with explicit per-block dims (legs c,s,t,f,d)
  TensorStruct X3 = sub_struct("cstfd", 5);
  for (auto& kv : x3) {
    X3.keys.push_back(kv.first);
    X3.dims.push_back(kv.second);
  }
  {
    int64_t off = 0;
    X3.offs.resize(X3.keys.size());
    for (size_t i = 0; i < X3.keys.size(); ++i) {
      X3.offs[i] = off;
      int64_t n = 1;
      for (auto x : X3.dims[i]) n *= x;
      off += n;
    }
    X3.total = off;
  }
  // leg charge maps for X3 are not needed by plan_pair (it reads dims per block)
  // but leg_dim() is used for output dims -> provide maps from the operand legs
  X3.cdim.assign(5, {});
  for (size_t i = 0; i < X3.keys.size(); ++i)
    for (int l = 0; l < 5; ++l) X3.cdim[l][X3.keys[i][l]] = X3.dims[i][l];
  H.x3 = X3;
  // stage 4: Y[c,s,t,g] = X3[c,s,t,f,d] R[d,f,g]
  // K = (f, d) with the d extent padded to a multiple of 8: the fused MPO
  // kernel writes X3 in whole 8-wide K chunks (one 16-byte swizzle unit of a
  // BF16 image row)
  H.s4 = plan_pair(X3, H.R, "cstg", none, nullptr, nullptr, kMpoKAlign);
  H.flops_s4 = H.s4.flops;
  H.flops = H.flops_s1 + H.flops_mpo + H.flops_s4;
  // output keys vs theta keys
  std::unordered_map<Key, int, KeyHash> th_idx;
  for (size_t i = 0; i < th.keys.size(); ++i) th_idx[th.keys[i]] = static_cast<int>(i);
  H.out_keys = H.s4.out.keys;
  H.closed = true;
  for (auto& k : H.out_keys)
    if (!th_idx.count(k)) H.closed = false;
  {
    std::unordered_map<Key, int, KeyHash> written;
    for (auto& k : H.out_keys) written[k] = 1;
    for (size_t i = 0; i < th.keys.size(); ++i) {
      if (written.count(th.keys[i])) continue;
      int64_t n = 1;
      for (auto x : th.dims[i]) n *= x;
      if (n > 0) H.zero_ranges.push_back({th.offs[i], n});
    }
  }
  // stage-4 epilogue row offsets into theta's layout: each group must hold a
  // single col block (one qg) for the direct store
  H.s4_separable = true;
  for (size_t g = 0; g < H.s4.groups.size(); ++g)
    if (H.s4.g_cols[g].size() != 1) H.s4_separable = false;
  if (H.closed && H.s4_separable) {
    H.s4_rowoff.assign(H.s4.groups.size(), {});
    for (size_t g = 0; g < H.s4.groups.size(); ++g) {
      auto& rows = H.s4.g_rows[g];
      const Key& ckey = H.s4.g_cols[g][0].key;  // (qg)
      std::vector<int64_t> ro(H.s4.groups[g].M, -1);
      for (auto& r : rows) {
        Key ok = {r.key[0], r.key[1], r.key[2], ckey[0]};
        auto it = th_idx.find(ok);
        int64_t mg = H.s4.g_cols[g][0].size;
        if (it == th_idx.end()) continue;  // (r, c) not an output block: rows stay unwritten
        int64_t base = th.offs[it->second];
        for (int64_t i = 0; i < r.size; ++i) ro[r.start + i] = base + i * mg;
      }
      H.s4_rowoff[g] = std::move(ro);
    }
  }
  // MPO pair tables: for each (qc, qd): inputs = present X1 blocks
  // (qb,qc,qp,qq,qd), outputs = X3 blocks (qc,qs,qt,qf,qd) used by stage 4.
  std::map<Key, std::pair<int, int64_t>> s1_row, s1_col;  // r=(qb,qc) / c=(qp,qq,qd) -> (g1, start)
  for (size_t g = 0; g < H.s1.groups.size(); ++g) {
    for (auto& r : H.s1.g_rows[g]) s1_row[r.key] = {static_cast<int>(g), r.start};
    for (auto& c : H.s1.g_cols[g]) s1_col[c.key] = {static_cast<int>(g), c.start};
  }
  std::map<std::pair<int32_t, int32_t>, int> pair_idx;
  for (size_t i = 0; i < H.s1.out.keys.size(); ++i) {
    const Key& k = H.s1.out.keys[i];  // (qb,qc,qp,qq,qd)
    const auto& d = H.s1.out.dims[i];
    auto rit = s1_row.find({k[0], k[1]});
    auto cit = s1_col.find({k[2], k[3], k[4]});
    if (rit == s1_row.end() || cit == s1_col.end() || rit->second.first != cit->second.first)
      throw PlanError{3, "internal: X1 block outside its stage-1 group"};
    auto pk = std::make_pair(k[1], k[4]);
    if (!pair_idx.count(pk)) {
      pair_idx[pk] = static_cast<int>(H.pairs.size());
      H.pairs.push_back({});
      H.mpo_in_keys.push_back({});
      H.mpo_out_keys.push_back({});
      H.pairs.back().qc = k[1];
      H.pairs.back().qd = k[4];
      H.pairs.back().mc = static_cast<int32_t>(d[1]);
      H.pairs.back().md = static_cast<int32_t>(d[4]);
    }
    int p = pair_idx[pk];
    MpoIn in{};
    in.g1 = rit->second.first;
    in.row0 = static_cast<int32_t>(rit->second.second);
    in.col0 = static_cast<int32_t>(cit->second.second);
    in.mb = static_cast<int32_t>(d[0]);
    in.mp = static_cast<int32_t>(d[2]);
    in.mq = static_cast<int32_t>(d[3]);
    H.pairs[p].ins.push_back(in);
    H.mpo_in_keys[p].push_back({k[0], k[2], k[3]});
  }
  std::map<Key, std::pair<int, int64_t>> x3_row;  // (qc,qs,qt) -> (g4, row start)
  std::map<Key, std::pair<int, int64_t>> x3_k;    // (qf,qd,mf,md) -> (g4, k start)
  for (size_t g = 0; g < H.s4.groups.size(); ++g) {
    for (auto& r : H.s4.g_rows[g]) x3_row[r.key] = {static_cast<int>(g), r.start};
    for (auto& k : H.s4.g_ks[g]) x3_k[k.key] = {static_cast<int>(g), k.start};
  }
  for (size_t i = 0; i < X3.keys.size(); ++i) {
    const Key& k = X3.keys[i];  // (qc,qs,qt,qf,qd)
    auto pit = pair_idx.find({k[0], k[4]});
    if (pit == pair_idx.end()) continue;
    auto rit = x3_row.find({k[0], k[1], k[2]});
    Key kk = {k[3], k[4], static_cast<int32_t>(X3.dims[i][3]), static_cast<int32_t>(X3.dims[i][4])};
    auto kit = x3_k.find(kk);
    if (rit == x3_row.end() || kit == x3_k.end()) continue;  // X3 block never read by stage 4
    if (rit->second.first != kit->second.first) throw PlanError{3, "internal: X3 row/k in different groups"};
    MpoPair& mp = H.pairs[pit->second];
    MpoOut o{};
    o.g4 = rit->second.first;
    o.row0 = static_cast<int32_t>(rit->second.second);
    o.k0 = static_cast<int32_t>(kit->second.second);
    o.ms = static_cast<int32_t>(X3.dims[i][1]);
    o.mt = static_cast<int32_t>(X3.dims[i][2]);
    o.mf = static_cast<int32_t>(X3.dims[i][3]);
    mp.outs.push_back(o);
    H.mpo_out_keys[pit->second].push_back({k[1], k[2], k[3]});
  }
  for (auto& mp : H.pairs) {
    int32_t s = 0;
    for (auto& in : mp.ins) {
      mp.in_slot0.push_back(s);
      s += in.mb * in.mp * in.mq;
    }
    mp.n_in_slots = s;
    s = 0;
    for (auto& o : mp.outs) {
      mp.out_slot0.push_back(s);
      s += o.ms * o.mt * o.mf;
    }
    mp.n_out_slots = s;
  }
  return H;
}

void heff_mpo_terms(HeffPlan& H, const std::vector<double>& wl, const std::vector<double>& wr) {
  // W_lr[(qb,qp,qq),(qs,qt,qf)][b,p,q,s,t,f] = sum_{qe,e} Wl[qb,qp,qs,qe][b,p,s,e] Wr[qe,qq,qt,qf][e,q,t,f]
  std::map<Key, int> wl_idx, wr_idx;
  for (size_t i = 0; i < H.Wl.keys.size(); ++i) wl_idx[H.Wl.keys[i]] = static_cast<int>(i);
  for (size_t i = 0; i < H.Wr.keys.size(); ++i) wr_idx[H.Wr.keys[i]] = static_cast<int>(i);
  // qe values present on the W_l right leg
  std::set<int32_t> qes;
  for (auto& k : H.Wl.keys) qes.insert(k[3]);
  for (size_t p = 0; p < H.pairs.size(); ++p) {
    MpoPair& mp = H.pairs[p];
    mp.terms.clear();
    for (size_t oi = 0; oi < mp.outs.size(); ++oi) {
      const Key& ok = H.mpo_out_keys[p][oi];  // (qs,qt,qf)
      const MpoOut& o = mp.outs[oi];
      for (size_t ii = 0; ii < mp.ins.size(); ++ii) {
        const Key& ik = H.mpo_in_keys[p][ii];  // (qb,qp,qq)
        const MpoIn& in = mp.ins[ii];
        // dense sub-block w[b,p,q,s,t,f]
        std::vector<double> w(static_cast<size_t>(in.mb) * in.mp * in.mq * o.ms * o.mt * o.mf, 0.0);
        bool any = false;
        for (int32_t qe : qes) {
          auto a = wl_idx.find({ik[0], ik[1], ok[0], qe});
          auto b = wr_idx.find({qe, ik[2], ok[1], ok[2]});
          if (a == wl_idx.end() || b == wr_idx.end()) continue;
          const auto& da = H.Wl.dims[a->second];  // b,p,s,e
          const auto& db = H.Wr.dims[b->second];  // e,q,t,f
          const double* A = wl.data() + H.Wl.offs[a->second];
          const double* B = wr.data() + H.Wr.offs[b->second];
          int64_t me = da[3];
          for (int bb = 0; bb < in.mb; ++bb)
            for (int pp = 0; pp < in.mp; ++pp)
              for (int ss = 0; ss < o.ms; ++ss)
                for (int64_t e = 0; e < me; ++e) {
                  double va = A[((bb * da[1] + pp) * da[2] + ss) * da[3] + e];
                  if (va == 0.0) continue;
                  for (int qq = 0; qq < in.mq; ++qq)
                    for (int tt = 0; tt < o.mt; ++tt)
                      for (int ff = 0; ff < o.mf; ++ff) {
                        double vb = B[((e * db[1] + qq) * db[2] + tt) * db[3] + ff];
                        if (vb == 0.0) continue;
                        size_t idx = ((((static_cast<size_t>(bb) * in.mp + pp) * in.mq + qq) * o.ms + ss) * o.mt + tt) *
                                         o.mf + ff;
                        w[idx] += va * vb;
                        any = true;
                      }
                }
        }
        if (!any) continue;
        for (int bb = 0; bb < in.mb; ++bb)
          for (int pp = 0; pp < in.mp; ++pp)
            for (int qq = 0; qq < in.mq; ++qq)
              for (int ss = 0; ss < o.ms; ++ss)
                for (int tt = 0; tt < o.mt; ++tt)
                  for (int ff = 0; ff < o.mf; ++ff) {
                    size_t idx = ((((static_cast<size_t>(bb) * in.mp + pp) * in.mq + qq) * o.ms + ss) * o.mt + tt) *
                                     o.mf + ff;
                    if (w[idx] == 0.0) continue;
                    MpoTerm t;
                    t.in_slot = mp.in_slot0[ii] + (bb * in.mp + pp) * in.mq + qq;
                    t.out_slot = mp.out_slot0[oi] + (ss * o.mt + tt) * o.mf + ff;
                    t.w = w[idx];
                    mp.terms.push_back(t);
                  }
      }
    }
    std::stable_sort(mp.terms.begin(), mp.terms.end(),
                     [](const MpoTerm& a, const MpoTerm& b) { return a.out_slot < b.out_slot; });
  }
}

}  // namespace tnx

namespace tnx {

// ---------------------------------------------------------------------------
// Leg fusion (algorithms/_tensor_utils.py:106-325).
//  * fused charge of position i*d_b + j: fused_flow*(flow_a q_a[i] + flow_b q_b[j]), mod n (:168-203);
//  * pairs (q_a, q_b) over the sorted unique charges of each leg, q_a outer;
//    a fused sector stacks its pairs in that order, d(q_a)*d(q_b) rows each (:255-270);
//  * each block is permuted so the legs are adjacent at axis_a, merged, and
//    placed at its pair's offset in a zero-initialised fused block (:282-320).
// ---------------------------------------------------------------------------
static int32_t fuse_mod(int64_t q, int32_t modulus) {
  if (modulus <= 0) return static_cast<int32_t>(q);
  int64_t r = q % modulus;
  return static_cast<int32_t>(r < 0 ? r + modulus : r);
}

FusePlan plan_fuse(const TensorStruct& T, int axis_a, int axis_b, int32_t fused_flow, int32_t modulus) {
  if (T.nl < 2) throw PlanError{1, "fuse_indices needs a tensor with at least two legs"};
  if (axis_a < 0 || axis_a >= T.nl || axis_b < 0 || axis_b >= T.nl || axis_a == axis_b)
    throw PlanError{1, "fuse_indices: axes must be two distinct legs of the tensor"};
  if (fused_flow != 1 && fused_flow != -1) throw PlanError{1, "fuse_indices: fused flow must be +1 or -1"};
  FusePlan F;
  const int a = std::min(axis_a, axis_b), b = std::max(axis_a, axis_b);
  F.axis_a = a;
  F.axis_b = b;
  const auto& qa = T.charges[a];
  const auto& qb = T.charges[b];
  const int64_t fa = T.flows[a], fb = T.flows[b];
  F.fused_charges.resize(qa.size() * qb.size());
  for (size_t i = 0; i < qa.size(); ++i)
    for (size_t j = 0; j < qb.size(); ++j)
      F.fused_charges[i * qb.size() + j] = fuse_mod(fused_flow * (fa * qa[i] + fb * qb[j]), modulus);
  std::vector<int32_t> ua(qa.begin(), qa.end()), ub(qb.begin(), qb.end());
  std::sort(ua.begin(), ua.end());
  ua.erase(std::unique(ua.begin(), ua.end()), ua.end());
  std::sort(ub.begin(), ub.end());
  ub.erase(std::unique(ub.begin(), ub.end()), ub.end());
  // offset of each pair inside its fused sector
  std::map<int32_t, int64_t> sector_fill;
  std::map<std::pair<int32_t, int32_t>, std::pair<int32_t, int64_t>> where;
  for (int32_t x : ua)
    for (int32_t y : ub) {
      const int32_t qf = fuse_mod(fused_flow * (fa * x + fb * y), modulus);
      int64_t& fill = sector_fill[qf];
      where[{x, y}] = {qf, fill};
      fill += T.leg_dim(a, x) * T.leg_dim(b, y);
    }
  // output structure
  std::vector<int> others;
  for (int i = 0; i < T.nl; ++i)
    if (i != a && i != b) others.push_back(i);
  TensorStruct& O = F.out;
  O.nl = T.nl - 1;
  O.subs.clear();
  for (int j = 0; j < static_cast<int>(others.size()); ++j) {
    if (j == a) {
      O.flows.push_back(fused_flow);
      O.charges.push_back(F.fused_charges);
    }
    O.flows.push_back(T.flows[others[j]]);
    O.charges.push_back(T.charges[others[j]]);
  }
  if (a == static_cast<int>(others.size())) {
    O.flows.push_back(fused_flow);
    O.charges.push_back(F.fused_charges);
  }
  O.finalize_leg_maps();
  auto new_key = [&](const Key& k) {
    Key nk;
    for (int j = 0; j < static_cast<int>(others.size()); ++j) {
      if (j == a) nk.push_back(where.at({k[a], k[b]}).first);
      nk.push_back(k[others[j]]);
    }
    if (a == static_cast<int>(others.size())) nk.push_back(where.at({k[a], k[b]}).first);
    return nk;
  };
  std::set<Key> keyset;
  for (const auto& k : T.keys) keyset.insert(new_key(k));
  O.keys.assign(keyset.begin(), keyset.end());
  O.layout_blocks();
  std::map<Key, size_t> kidx;
  for (size_t i = 0; i < O.keys.size(); ++i) kidx[O.keys[i]] = i;
  // copy segments: source legs -> destination strides
  for (size_t bi = 0; bi < T.keys.size(); ++bi) {
    int64_t n = 1;
    for (int l = 0; l < T.nl; ++l) n *= T.dims[bi][l];
    if (n == 0) continue;
    const Key& k = T.keys[bi];
    const size_t ob = kidx.at(new_key(k));
    const auto& od = O.dims[ob];
    std::vector<int64_t> ostr(O.nl);
    int64_t s = 1;
    for (int l = O.nl - 1; l >= 0; --l) {
      ostr[l] = s;
      s *= od[l];
    }
    CopySeg c{};
    c.src_off = T.offs[bi];
    c.count = n;
    c.nlegs = T.nl;
    c.dst_off = O.offs[ob] + where.at({k[a], k[b]}).second * ostr[a];
    for (int l = 0; l < T.nl; ++l) c.dims[l] = static_cast<int32_t>(T.dims[bi][l]);
    c.dstr[a] = ostr[a] * T.dims[bi][b];
    c.dstr[b] = ostr[a];
    for (int j = 0; j < static_cast<int>(others.size()); ++j) c.dstr[others[j]] = ostr[j < a ? j : j + 1];
    F.segs.push_back(c);
  }
  return F;
}

}  // namespace tnx

namespace tnx {

// Where todense() of a fused tensor puts natural row n = i*d_b + j: row
// off(q_a, q_b) + rank_a(i)*d(q_b) + rank_b(j) of its fused sector (see
// plan_fuse), which todense() (core/tensor.py:760-781) places at the k-th
// position of the fused leg carrying that charge.
std::vector<int64_t> fuse_row_map(const std::vector<int32_t>& qa, int32_t fa, const std::vector<int32_t>& qb,
                                  int32_t fb, int32_t fused_flow, int32_t modulus) {
  if (fused_flow != 1 && fused_flow != -1) throw PlanError{1, "fused flow must be +1 or -1"};
  const size_t na = qa.size(), nb = qb.size();
  std::map<int32_t, int64_t> da, db;
  for (int32_t q : qa) da[q] += 1;
  for (int32_t q : qb) db[q] += 1;
  auto fq = [&](int32_t x, int32_t y) { return fuse_mod(fused_flow * (int64_t(fa) * x + int64_t(fb) * y), modulus); };
  std::map<int32_t, int64_t> fill;
  std::map<std::pair<int32_t, int32_t>, int64_t> off;
  for (auto& x : da)
    for (auto& y : db) {
      const int32_t q = fq(x.first, y.first);
      off[{x.first, y.first}] = fill[q];
      fill[q] += x.second * y.second;
    }
  std::map<int32_t, std::vector<int64_t>> pos;
  for (size_t i = 0; i < na; ++i)
    for (size_t j = 0; j < nb; ++j) pos[fq(qa[i], qb[j])].push_back(static_cast<int64_t>(i * nb + j));
  std::vector<int64_t> rank_a(na), rank_b(nb);
  {
    std::map<int32_t, int64_t> c;
    for (size_t i = 0; i < na; ++i) rank_a[i] = c[qa[i]]++;
    c.clear();
    for (size_t j = 0; j < nb; ++j) rank_b[j] = c[qb[j]]++;
  }
  std::vector<int64_t> out(na * nb);
  for (size_t i = 0; i < na; ++i)
    for (size_t j = 0; j < nb; ++j) {
      const int64_t k = off[{qa[i], qb[j]}] + rank_a[i] * db[qb[j]] + rank_b[j];
      out[i * nb + j] = pos[fq(qa[i], qb[j])][static_cast<size_t>(k)];
    }
  return out;
}

}  // namespace tnx

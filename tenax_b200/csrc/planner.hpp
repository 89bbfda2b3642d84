// Exact integer planning for block-sparse symmetric contractions.
//
// Everything here is host-side integer work: block key sets, block shapes,
// matching of blocks over contracted legs, grouping of matching blocks into
// sector GEMMs, and the gather/scatter tables the device kernels consume.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

namespace tnx {

constexpr int kMaxLegs = 12;  // legs per tensor (operands, intermediates and outputs)
constexpr int kMpoKAlign = 8;  // d-extent padding of the H_eff stage-4 K blocks

using Key = std::vector<int32_t>;

struct KeyHash {
  size_t operator()(const Key& k) const noexcept {
    uint64_t h = 1469598103934665603ull;
    for (int32_t v : k) {
      h ^= static_cast<uint32_t>(v);
      h *= 1099511628211ull;
    }
    return static_cast<size_t>(h ^ (h >> 29));
  }
};

struct PlanError {
  int code;
  std::string msg;
};

// One operand: leg metadata + block keys (data lives elsewhere).
struct TensorStruct {
  int nl = 0;
  std::string subs;
  std::vector<int32_t> flows;
  std::vector<std::vector<int32_t>> charges;              // per leg
  std::vector<std::unordered_map<int32_t, int64_t>> cdim; // per leg: charge -> multiplicity
  std::vector<Key> keys;                                  // per block
  std::vector<std::vector<int64_t>> dims;                 // per block, per leg
  std::vector<int64_t> offs;                              // element offset per block
  int64_t total = 0;

  void finalize_leg_maps();
  // fill dims/offs from keys (blocks stored in key-list order)
  void layout_blocks();
  int64_t leg_dim(int leg, int32_t q) const {
    auto it = cdim[leg].find(q);
    return it == cdim[leg].end() ? 0 : it->second;
  }
};

std::vector<Key> valid_blocks(const std::vector<std::vector<int32_t>>& charges, const std::vector<int32_t>& flows,
                              int32_t modulus, bool has_target, int64_t target);

// ---------------------------------------------------------------------------
// Pairwise contraction plan: C = A (x) B over shared chars.
// ---------------------------------------------------------------------------

// Copy one source block into a GEMM operand matrix (row-major M x K view of
// a group); the row/k coordinates of an element are affine in its leg indices.
struct PackSeg {
  int64_t src_off;  // element offset of the block in the operand buffer
  int64_t count;    // elements in the block
  int32_t group;    // GEMM group
  int32_t row0, k0; // origin inside the group's operand matrix
  int32_t nlegs;
  int32_t dims[kMaxLegs];
  int32_t rstr[kMaxLegs];
  int32_t kstr[kMaxLegs];   // K strides of the contracted legs (unpadded: element order)
  int32_t kdstr[kMaxLegs];  // K strides in the operand image (the innermost may be padded)
  int32_t neg = 0;          // fermionic exchange sign of this block: 1 packs the negated block
};

// Copy one output block out of a group's result matrix (M x N, row-major).
struct ScatSeg {
  int64_t dst_off;  // element offset of the output block
  int64_t count;
  int32_t group;
  int32_t row0, col0;
  int32_t nlegs;
  int32_t dims[kMaxLegs];
  int32_t rstr[kMaxLegs];
  int32_t cstr[kMaxLegs];
  int32_t neg = 0;  // fermionic exchange sign of this output block: 1 negates it
};

struct GroupShape {
  int64_t M = 0, N = 0, K = 0;
};

struct PairPlan {
  std::string a_subs, b_subs, out_subs;
  std::vector<GroupShape> groups;
  std::vector<PackSeg> packA, packB;
  std::vector<ScatSeg> scatter;
  // output structure (sorted keys)
  TensorStruct out;
  double flops = 0.0;
  // per group: row blocks (A-free charge tuple) and col blocks
  struct Span {
    Key key;
    int64_t start, size;
  };
  std::vector<std::vector<Span>> g_rows, g_cols, g_ks;
};

// keep_key(out_key) decides whether a present output block is kept
// (filtered semantics); nullptr keeps all.
struct KeyFilter {
  bool active = false;
  std::unordered_map<Key, int, KeyHash> allowed;
};

// k_align > 1 pads the innermost contracted leg of every K block to a
// multiple of k_align in the GEMM's K coordinate (zero rows of K), so that a
// producer can write whole aligned K chunks.  n_align > 1 pads the innermost
// free leg of B in the GEMM's N coordinate the same way (zero rows of the B
// image, zero result columns), so that every result slot starts on an
// aligned column.  FLOP counts stay unpadded.
PairPlan plan_pair(const TensorStruct& A, const TensorStruct& B, const std::string& out_subs,
                   const KeyFilter& filter, const std::vector<std::vector<int32_t>>* out_charges,
                   const std::vector<int32_t>* out_flows, int k_align = 1, int n_align = 1);

// ---------------------------------------------------------------------------
// Two-site H_eff plan: Y[c,s,t,g] = L[a,b,c] th[a,p,q,d] Wl[b,p,s,e] Wr[e,q,t,f] R[d,f,g]
// ---------------------------------------------------------------------------

struct MpoIn {   // one X1 block feeding a (qc,qd) point grid
  int32_t g1;    // stage-1 group
  int32_t row0;  // row of (b=0,c=0) inside the group matrix
  int32_t col0;  // col of (p=0,q=0,d=0)
  int32_t mb, mp, mq;
};
struct MpoOut {  // one X3 block written by the (qc,qd) point grid
  int32_t g4;
  int32_t row0;  // image row of (c=0,s=0,t=0)
  int32_t k0;    // image k of (f=0,d=0)
  int32_t ms, mt, mf;
};
struct MpoTerm { // y[out_slot] += w * x[in_slot]
  int32_t out_slot, in_slot;
  double w;
};
struct MpoPair {
  int32_t qc = 0, qd = 0;  // charges of the pair's c and d sectors
  int32_t mc, md;
  std::vector<MpoIn> ins;
  std::vector<MpoOut> outs;
  std::vector<int32_t> in_slot0, out_slot0;  // first slot of each in/out block
  int32_t n_in_slots = 0, n_out_slots = 0;
  std::vector<MpoTerm> terms;  // sorted by out_slot
};

struct HeffPlan {
  TensorStruct L, th, Wl, Wr, R;
  int x1_align = 1;             // stage-1 result columns: each d range padded to a multiple of this
  PairPlan s1;                  // L (x) theta over a -> X1 group matrices
  PairPlan s4;                  // X3 (x) R over (f,d) -> Y
  TensorStruct x3;              // structure of X3[c,s,t,f,d]
  std::vector<MpoPair> pairs;
  std::vector<Key> out_keys;    // keys H_eff writes (sorted)
  bool closed = true;           // out_keys subset of theta keys
  bool s4_separable = true;     // every stage-4 group has one col block
  double flops = 0.0;           // 4-stage algorithmic count
  double flops_s1 = 0.0, flops_s4 = 0.0, flops_mpo = 0.0;
  // rowoff table for the stage-4 epilogue (per group, per row): output element offset of col 0
  std::vector<std::vector<int64_t>> s4_rowoff;
  // charge tuples of each MPO pair's inputs (qb,qp,qq) and outputs (qs,qt,qf)
  std::vector<std::vector<Key>> mpo_in_keys, mpo_out_keys;
  // theta-layout (offset, length) of blocks H_eff never writes: zeroed per apply
  std::vector<std::pair<int64_t, int64_t>> zero_ranges;
};

HeffPlan plan_heff(const TensorStruct& L, const TensorStruct& th, const TensorStruct& Wl, const TensorStruct& Wr,
                   const TensorStruct& R, int x1_align = 1);
// Fill the MPO terms (W_l W_r contracted over e) from host copies of the
// W_l / W_r block buffers.
void heff_mpo_terms(HeffPlan& p, const std::vector<double>& wl, const std::vector<double>& wr);

// ---------------------------------------------------------------------------
// Leg fusion (fuse_indices, algorithms/_tensor_utils.py:106-325).
// ---------------------------------------------------------------------------
struct CopySeg {
  int64_t src_off, dst_off, count;
  int32_t nlegs;
  int32_t dims[kMaxLegs];
  int64_t dstr[kMaxLegs];
};

struct FusePlan {
  int axis_a = 0, axis_b = 0;         // sorted: axis_a < axis_b
  std::vector<int32_t> fused_charges; // position i*d_b + j
  TensorStruct out;                   // fused leg at axis_a; keys sorted
  std::vector<CopySeg> segs;          // one per input block with a nonzero size
};

FusePlan plan_fuse(const TensorStruct& T, int axis_a, int axis_b, int32_t fused_flow, int32_t modulus);
// todense() position of each natural row i*d_b + j of a fused pair of legs
std::vector<int64_t> fuse_row_map(const std::vector<int32_t>& qa, int32_t fa, const std::vector<int32_t>& qb,
                                  int32_t fb, int32_t fused_flow, int32_t modulus);

}  // namespace tnx

// Device-side sector planning: the integer core of a block-sparse
// contraction's structure computed by kernels, bit-exact against the host
// planner (planner.cpp) and the reference it restates.
//
//   * unique_charges_kernel: per leg, the sorted distinct charges and their
//     multiplicities (a presence bitmap over the leg's charge range).
//   * valid_blocks_kernel: _compute_valid_blocks (tenax core/tensor.py:53-165)
//     in the reference's output order.  Leg by leg, the distinct partial sums
//     keep dict-insertion order: the new order is the order in which the
//     (new charge, old partial sum) grid -- new charge outer -- first reaches
//     each value, and each value's prefixes are appended in that grid order.
//     U(1) solves the last leg directly; Z_n enumerates it.
//   * target / matching kernels: _contract_symmetric's output structure for
//     two operands (contraction/contractor.py:344-441): the output target
//     inferred from operands whose blocks all carry one total charge, the
//     valid output keys, blocks matched on their contracted charges (the
//     reference's signature index), kept when their output key is valid; the
//     output keys in sorted order with their block offsets.
//   * fused_charges_kernel: _compute_fused_charges (algorithms/
//     _tensor_utils.py:191-203), position i * d_b + j of a fused leg.
//
// Everything runs on `stream`; the entry points read back only the counts
// they return.  Sizes: at most kMaxLegsDev legs, charge ranges up to 2^16
// per leg, at most 2^16 valid keys per call.
#include <cuda_runtime.h>

#include "common.cuh"
#include "planner_dev.hpp"

namespace tnx {

namespace {
constexpr int kRangeMax = 1 << 16;  // charge range (max - min + 1) of one leg
constexpr int kPlanThreads = 1024;

__device__ __forceinline__ int64_t fuse_dev(int64_t a, int64_t b, int32_t modulus) {
  if (modulus == 0) return a + b;
  int64_t r = (a + b) % modulus;
  return r < 0 ? r + modulus : r;
}

// one CTA per leg: sorted distinct charges, their multiplicities and count;
// status[leg] = 0, or 1 when the leg's charge range exceeds kRangeMax
__global__ void __launch_bounds__(kPlanThreads) unique_charges_kernel(const int32_t* __restrict__ charges,
                                                                      const int64_t* __restrict__ leg_off,
                                                                      int32_t* __restrict__ uniq,
                                                                      int32_t* __restrict__ mult,
                                                                      int32_t* __restrict__ n_uniq,
                                                                      int32_t* __restrict__ status) {
  constexpr int kWords = kRangeMax / 32;
  constexpr int kPer = (kWords + kPlanThreads - 1) / kPlanThreads;
  __shared__ int32_t s_min[32], s_max[32];
  __shared__ uint32_t hist_words[kWords];  // presence bitmap (8 KB)
  __shared__ int32_t s_tot[kPlanThreads];
  const int leg = blockIdx.x;
  const int64_t b0 = leg_off[leg], n = leg_off[leg + 1] - b0;
  const int32_t* c = charges + b0;
  int32_t mn = INT32_MAX, mx = INT32_MIN;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    mn = min(mn, c[i]);
    mx = max(mx, c[i]);
  }
  for (int o = 16; o; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    s_min[threadIdx.x >> 5] = mn;
    s_max[threadIdx.x >> 5] = mx;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    mn = threadIdx.x < blockDim.x / 32 ? s_min[threadIdx.x] : INT32_MAX;
    mx = threadIdx.x < blockDim.x / 32 ? s_max[threadIdx.x] : INT32_MIN;
    for (int o = 16; o; o >>= 1) {
      mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (threadIdx.x == 0) {
      s_min[0] = mn;
      s_max[0] = mx;
    }
  }
  __syncthreads();
  mn = s_min[0];
  mx = s_max[0];
  if (n == 0) {
    if (threadIdx.x == 0) {
      n_uniq[leg] = 0;
      status[leg] = 0;
    }
    return;
  }
  const int64_t range = static_cast<int64_t>(mx) - mn + 1;
  if (range > kRangeMax) {
    if (threadIdx.x == 0) {
      status[leg] = 1;
      n_uniq[leg] = 0;
    }
    return;
  }
  for (int w = threadIdx.x; w < kWords; w += blockDim.x) hist_words[w] = 0u;
  __syncthreads();
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const int v = c[i] - mn;
    atomicOr(&hist_words[v >> 5], 1u << (v & 31));
  }
  __syncthreads();
  // sorted distinct charges: words in order, each word's set bits in order;
  // word w = t + j*T is handled in round j by thread t after a block-wide
  // (Hillis-Steele) scan of the round's popcounts
  int base_j = 0;
  for (int j = 0; j < kPer; ++j) {
    const int w = threadIdx.x + j * kPlanThreads;
    const int pc = w < kWords ? __popc(hist_words[w]) : 0;
    s_tot[threadIdx.x] = pc;
    __syncthreads();
    for (int o = 1; o < kPlanThreads; o <<= 1) {
      const int add = threadIdx.x >= o ? s_tot[threadIdx.x - o] : 0;
      __syncthreads();
      s_tot[threadIdx.x] += add;
      __syncthreads();
    }
    const int incl = s_tot[threadIdx.x];
    const int total = s_tot[kPlanThreads - 1];
    __syncthreads();
    if (w < kWords) {
      uint32_t bits = hist_words[w];
      int pos = base_j + incl - pc;
      while (bits) {
        const int b = __ffs(bits) - 1;
        bits &= bits - 1;
        uniq[b0 + pos] = mn + w * 32 + b;
        mult[b0 + pos] = 0;
        ++pos;
      }
    }
    base_j += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    n_uniq[leg] = base_j;
    status[leg] = 0;
  }
  __syncthreads();
  // multiplicities: each charge's count, by binary search in the sorted list
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const int32_t v = c[i];
    int lo = 0, hi = base_j - 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (uniq[b0 + mid] < v)
        lo = mid + 1;
      else
        hi = mid;
    }
    atomicAdd(&mult[b0 + lo], 1);
  }
}

// Scratch of the enumeration (global): two prefix-key buffers of
// cap_entries x kMaxLegsDev, two order buffers (int64 partial sums) with
// per-rank start/count, and per-grid arrays of cap_grid entries.
struct EnumScratch {
  int32_t* keys[2];
  int64_t* ord[2];
  int32_t* start[2];
  int32_t* cnt[2];
  int64_t* g_nf;
  int32_t* g_rank;
  int32_t* g_off;
  int32_t* g_first;
  int64_t cap_entries, cap_ord, cap_grid;
};

// Single CTA: the reference's leg-by-leg enumeration (see the file comment).
// out_count[0] = number of keys, or -1 when a capacity would overflow.
__global__ void __launch_bounds__(kPlanThreads) valid_blocks_kernel(int n_legs, const int32_t* __restrict__ uniq,
                                                                    const int64_t* __restrict__ leg_off,
                                                                    const int32_t* __restrict__ n_uniq,
                                                                    const int32_t* __restrict__ flows,
                                                                    int32_t modulus, int64_t eff, EnumScratch S,
                                                                    int32_t* __restrict__ keys_out, int64_t out_cap,
                                                                    int64_t* __restrict__ out_count) {
  __shared__ int64_t s_n_ord, s_total;
  __shared__ int s_overflow;
  const int T = blockDim.x;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31, nwarps = T >> 5;
  if (tid == 0) s_overflow = 0;
  __syncthreads();
  const int last = n_legs - 1;
  // leg 0: every distinct charge is its own partial sum (flows are +-1)
  int cur = 0;
  {
    const int nq = n_uniq[0];
    const int32_t* q0 = uniq + leg_off[0];
    if (nq > S.cap_ord || nq > S.cap_entries) {
      if (tid == 0) out_count[0] = -1;
      return;
    }
    for (int i = tid; i < nq; i += T) {
      S.ord[0][i] = static_cast<int64_t>(flows[0]) * q0[i];
      S.start[0][i] = i;
      S.cnt[0][i] = 1;
      S.keys[0][static_cast<int64_t>(i) * kMaxLegsDev] = q0[i];
    }
    if (tid == 0) s_n_ord = nq;
    __syncthreads();
  }
  if (n_legs == 1) {
    // keys (q) with flow * q == eff, in charge order
    if (tid == 0) {
      int64_t k = 0;
      for (int64_t r = 0; r < s_n_ord; ++r)
        if (S.ord[0][r] == eff) {
          if (k < out_cap) keys_out[k] = S.keys[0][r * kMaxLegsDev];
          ++k;
        }
      out_count[0] = k <= out_cap ? k : -1;
    }
    return;
  }
  for (int li = 1; li < last; ++li) {
    const int nq = n_uniq[li];
    const int32_t* ql = uniq + leg_off[li];
    const int64_t n_ord = s_n_ord;
    const int64_t G = static_cast<int64_t>(nq) * n_ord;
    if (G > S.cap_grid) {
      if (tid == 0) out_count[0] = -1;
      return;
    }
    const int nx = cur ^ 1;
    // grid point g = (charge index qi, old rank r), qi outer
    for (int64_t g = tid; g < G; g += T) {
      const int qi = static_cast<int>(g / n_ord);
      const int64_t r = g - static_cast<int64_t>(qi) * n_ord;
      S.g_nf[g] = fuse_dev(S.ord[cur][r], static_cast<int64_t>(flows[li]) * ql[qi], modulus);
    }
    __syncthreads();
    // first occurrence of each value in grid order
    for (int64_t g = tid; g < G; g += T) {
      const int64_t v = S.g_nf[g];
      int first = 1;
      for (int64_t h = 0; h < g; ++h)
        if (S.g_nf[h] == v) {
          first = 0;
          break;
        }
      S.g_first[g] = first;
    }
    __syncthreads();
    // ranks of first occurrences (serial: grids hold a few thousand points)
    if (tid == 0) {
      int32_t rk = 0;
      for (int64_t g = 0; g < G; ++g)
        if (S.g_first[g]) {
          if (rk >= S.cap_ord) {
            s_overflow = 1;
            break;
          }
          S.g_rank[g] = rk;
          S.ord[nx][rk] = S.g_nf[g];
          ++rk;
        }
      s_n_ord = rk;
    }
    __syncthreads();
    if (s_overflow) {
      if (tid == 0) out_count[0] = -1;
      return;
    }
    // every grid point takes its value's rank and its offset inside the
    // value's prefix list (the prefixes of earlier grid points with that value)
    for (int64_t g = tid; g < G; g += T) {
      const int64_t v = S.g_nf[g];
      int32_t rk = -1, off = 0;
      for (int64_t h = 0; h < g; ++h)
        if (S.g_nf[h] == v) {
          if (rk < 0) rk = S.g_rank[h];
          off += S.cnt[cur][h - (h / n_ord) * n_ord];
        }
      // the first match is the value's first occurrence, whose rank thread 0
      // set (and which rewrites that same rank): no conflicting accesses
      if (rk < 0) rk = S.g_rank[g];
      S.g_rank[g] = rk;
      S.g_off[g] = off;
    }
    __syncthreads();
    // per new rank: prefix count and start (serial over ranks)
    if (tid == 0) {
      for (int64_t r = 0; r < s_n_ord; ++r) S.cnt[nx][r] = 0;
      for (int64_t g = 0; g < G; ++g) S.cnt[nx][S.g_rank[g]] += S.cnt[cur][g - (g / n_ord) * n_ord];
      int64_t acc = 0;
      for (int64_t r = 0; r < s_n_ord; ++r) {
        S.start[nx][r] = static_cast<int32_t>(acc);
        acc += S.cnt[nx][r];
      }
      if (acc > S.cap_entries) s_overflow = 1;
    }
    __syncthreads();
    if (s_overflow) {
      if (tid == 0) out_count[0] = -1;
      return;
    }
    // copy prefixes + the new charge: one warp per grid point
    for (int64_t g = warp; g < G; g += nwarps) {
      const int qi = static_cast<int>(g / n_ord);
      const int64_t r = g - static_cast<int64_t>(qi) * n_ord;
      const int64_t src0 = S.start[cur][r], n = S.cnt[cur][r];
      const int64_t dst0 = static_cast<int64_t>(S.start[nx][S.g_rank[g]]) + S.g_off[g];
      for (int64_t e = lane; e < n; e += 32) {
        const int32_t* src = S.keys[cur] + (src0 + e) * kMaxLegsDev;
        int32_t* dst = S.keys[nx] + (dst0 + e) * kMaxLegsDev;
        for (int l = 0; l < li; ++l) dst[l] = src[l];
        dst[li] = ql[qi];
      }
    }
    __syncthreads();
    cur = nx;
  }
  // last leg
  const int nq = n_uniq[last];
  const int32_t* qlast = uniq + leg_off[last];
  const int64_t n_ord = s_n_ord;
  const int64_t fl = flows[last];
  const int64_t G = modulus == 0 ? n_ord : static_cast<int64_t>(nq) * n_ord;
  if (G > S.cap_grid) {
    if (tid == 0) out_count[0] = -1;
    return;
  }
  // grid point: U(1) one per rank (the last charge solved directly), Z_n
  // (charge index outer, rank inner); g_rank holds the last charge, or
  // INT32_MIN when the point yields no key
  for (int64_t g = tid; g < G; g += T) {
    int32_t qv = INT32_MIN;
    if (modulus == 0) {
      if (fl != 0) {
        const int64_t want = (eff - S.ord[cur][g]) * fl;
        if (nq > 0 && want >= INT32_MIN && want <= INT32_MAX) {
          int lo = 0, hi = nq - 1;
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (qlast[mid] < want)
              lo = mid + 1;
            else
              hi = mid;
          }
          if (qlast[lo] == want) qv = static_cast<int32_t>(want);
        }
      }
    } else {
      const int qi = static_cast<int>(g / n_ord);
      const int64_t r = g - static_cast<int64_t>(qi) * n_ord;
      if (fuse_dev(S.ord[cur][r], fl * qlast[qi], modulus) == eff) qv = qlast[qi];
    }
    S.g_rank[g] = qv;
  }
  __syncthreads();
  if (tid == 0) {
    int64_t acc = 0;
    for (int64_t g = 0; g < G; ++g) {
      S.g_off[g] = static_cast<int32_t>(acc);
      if (S.g_rank[g] != INT32_MIN) acc += S.cnt[cur][modulus == 0 ? g : g - (g / n_ord) * n_ord];
    }
    s_total = acc;
    out_count[0] = acc <= out_cap ? acc : -1;
  }
  __syncthreads();
  if (s_total > out_cap) return;
  for (int64_t g = warp; g < G; g += nwarps) {
    if (S.g_rank[g] == INT32_MIN) continue;
    const int64_t r = modulus == 0 ? g : g - (g / n_ord) * n_ord;
    const int64_t src0 = S.start[cur][r], n = S.cnt[cur][r];
    for (int64_t e = lane; e < n; e += 32) {
      const int32_t* src = S.keys[cur] + (src0 + e) * kMaxLegsDev;
      int32_t* dst = keys_out + (S.g_off[g] + e) * n_legs;
      for (int l = 0; l < last; ++l) dst[l] = src[l];
      dst[last] = S.g_rank[g];
    }
  }
}

// lexicographic comparison of two keys of n int32
__device__ __forceinline__ int key_cmp(const int32_t* a, const int32_t* b, int n) {
  for (int l = 0; l < n; ++l) {
    if (a[l] < b[l]) return -1;
    if (a[l] > b[l]) return 1;
  }
  return 0;
}

// Single CTA: sort n keys by a bitonic network over an index permutation of
// pow2 >= n entries (entries >= n sort last); keys are copied out in order.
__global__ void __launch_bounds__(kPlanThreads) sort_keys_kernel(const int32_t* __restrict__ keys, int n_legs,
                                                                 int32_t* __restrict__ perm, int64_t n, int64_t pow2,
                                                                 int32_t* __restrict__ sorted_out) {
  for (int64_t i = threadIdx.x; i < pow2; i += blockDim.x) perm[i] = static_cast<int32_t>(i);
  __syncthreads();
  for (int64_t k = 2; k <= pow2; k <<= 1) {
    for (int64_t j = k >> 1; j > 0; j >>= 1) {
      for (int64_t i = threadIdx.x; i < pow2; i += blockDim.x) {
        const int64_t ixj = i ^ j;
        if (ixj > i) {
          const int32_t a = perm[i], b = perm[ixj];
          int c;
          if (a >= n && b >= n)
            c = 0;
          else if (a >= n)
            c = 1;
          else if (b >= n)
            c = -1;
          else
            c = key_cmp(keys + static_cast<int64_t>(a) * n_legs, keys + static_cast<int64_t>(b) * n_legs, n_legs);
          const bool up = (i & k) == 0;
          if ((up && c > 0) || (!up && c < 0)) {
            perm[i] = b;
            perm[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
    for (int l = 0; l < n_legs; ++l)
      sorted_out[i * n_legs + l] = keys[static_cast<int64_t>(perm[i]) * n_legs + l];
}

// Per operand: target[0] = the common total charge sum(flow * q) of its
// blocks when they all agree (and there is at least one), target[1] = 1 then.
__global__ void __launch_bounds__(kPlanThreads) operand_target_kernel(const int32_t* __restrict__ keys, int n_legs,
                                                                      int64_t n_blocks,
                                                                      const int32_t* __restrict__ flows,
                                                                      int64_t* __restrict__ target) {
  __shared__ int s_mixed;
  __shared__ int64_t s_first;
  if (threadIdx.x == 0) {
    s_mixed = 0;
    s_first = 0;
    if (n_blocks > 0)
      for (int l = 0; l < n_legs; ++l) s_first += static_cast<int64_t>(flows[l]) * keys[l];
  }
  __syncthreads();
  for (int64_t b = threadIdx.x; b < n_blocks; b += blockDim.x) {
    int64_t t = 0;
    for (int l = 0; l < n_legs; ++l) t += static_cast<int64_t>(flows[l]) * keys[b * n_legs + l];
    if (t != s_first) s_mixed = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    target[0] = (n_blocks > 0 && !s_mixed) ? s_first : 0;
    target[1] = (n_blocks > 0 && !s_mixed) ? 1 : 0;
  }
}

// Thread per A block, B blocks in order: the matching pairs whose output key
// is one of the (sorted) valid output keys.  Pass 0 counts per A block; pass
// 1 writes (ia, ib, valid-key index) at the A block's offset and marks the
// valid key present.
__global__ void match_kernel(MatchArgs m, const int32_t* __restrict__ akeys, int64_t na,
                             const int32_t* __restrict__ bkeys, int64_t nb, const int32_t* __restrict__ valid_sorted,
                             int64_t n_valid, int pass, int32_t* __restrict__ row_count,
                             const int64_t* __restrict__ row_base, int4* __restrict__ pairs,
                             int32_t* __restrict__ present) {
  const int64_t ia = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (ia >= na) return;
  const int32_t* ka = akeys + ia * m.la;
  int32_t ok[kMaxLegsDev];
  int32_t cnt = 0;
  for (int64_t ib = 0; ib < nb; ++ib) {
    const int32_t* kb = bkeys + ib * m.lb;
    bool match = true;
    for (int c = 0; c < m.n_con && match; ++c) match = ka[m.a_con[c]] == kb[m.b_con[c]];
    if (!match) continue;
    for (int l = 0; l < m.lo; ++l) ok[l] = m.o_src[l] < m.la ? ka[m.o_src[l]] : kb[m.o_src[l] - m.la];
    int64_t lo = 0, hi = n_valid;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (key_cmp(valid_sorted + mid * m.lo, ok, m.lo) < 0)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo >= n_valid || key_cmp(valid_sorted + lo * m.lo, ok, m.lo) != 0) continue;
    if (pass == 1) {
      pairs[row_base[ia] + cnt] = make_int4(static_cast<int32_t>(ia), static_cast<int32_t>(ib),
                                            static_cast<int32_t>(lo), 0);
      present[lo] = 1;
    }
    ++cnt;
  }
  if (pass == 0) row_count[ia] = cnt;
}

// Single CTA: present valid keys -> the output key list (sorted order), each
// block's size from the output legs' multiplicities, and its offset; the
// pairs' valid-key index becomes the output block index.
__global__ void __launch_bounds__(kPlanThreads) compact_out_kernel(
    const int32_t* __restrict__ valid_sorted, int64_t n_valid, int lo_legs, const int32_t* __restrict__ present,
    const int32_t* __restrict__ o_uniq, const int32_t* __restrict__ o_mult, const int64_t* __restrict__ o_leg_off,
    const int32_t* __restrict__ o_n_uniq, int32_t* __restrict__ vmap, int32_t* __restrict__ keys_out,
    int64_t* __restrict__ offs_out, int64_t* __restrict__ n_out, int4* __restrict__ pairs, int64_t n_pairs) {
  if (threadIdx.x == 0) {
    int64_t k = 0, off = 0;
    for (int64_t v = 0; v < n_valid; ++v) {
      if (!present[v]) {
        vmap[v] = -1;
        continue;
      }
      vmap[v] = static_cast<int32_t>(k);
      int64_t size = 1;
      for (int l = 0; l < lo_legs; ++l) {
        const int32_t q = valid_sorted[v * lo_legs + l];
        const int32_t* u = o_uniq + o_leg_off[l];
        const int nu = o_n_uniq[l];
        int a = 0, b = nu - 1;
        while (a < b) {
          const int mid = (a + b) >> 1;
          if (u[mid] < q)
            a = mid + 1;
          else
            b = mid;
        }
        size *= (nu > 0 && u[a] == q) ? o_mult[o_leg_off[l] + a] : 0;
      }
      for (int l = 0; l < lo_legs; ++l) keys_out[k * lo_legs + l] = valid_sorted[v * lo_legs + l];
      offs_out[k] = off;
      off += size;
      ++k;
    }
    offs_out[k] = off;
    n_out[0] = k;
  }
  __syncthreads();
  for (int64_t p = threadIdx.x; p < n_pairs; p += blockDim.x) pairs[p].z = vmap[pairs[p].z];
}

__global__ void fused_charges_kernel(const int32_t* __restrict__ qa, int64_t da, int32_t fa,
                                     const int32_t* __restrict__ qb, int64_t db, int32_t fb, int32_t fused_flow,
                                     int32_t modulus, int32_t* __restrict__ out) {
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= da * db) return;
  const int64_t i = p / db, j = p - i * db;
  const int64_t v = static_cast<int64_t>(fused_flow) *
                    fuse_dev(static_cast<int64_t>(fa) * qa[i], static_cast<int64_t>(fb) * qb[j], modulus);
  out[p] = static_cast<int32_t>(modulus == 0 ? v : fuse_dev(v, 0, modulus));
}
}  // namespace

// ---------------------------------------------------------------------------
// launchers (planner_dev.hpp)
// ---------------------------------------------------------------------------
void launch_unique_charges(int n_legs, const int32_t* charges, const int64_t* leg_off, int32_t* uniq, int32_t* mult,
                           int32_t* n_uniq, int32_t* status, cudaStream_t st) {
  if (n_legs > 0) unique_charges_kernel<<<n_legs, kPlanThreads, 0, st>>>(charges, leg_off, uniq, mult, n_uniq, status);
}

void launch_valid_blocks(int n_legs, const int32_t* uniq, const int64_t* leg_off, const int32_t* n_uniq,
                         const int32_t* flows, int32_t modulus, int64_t eff, int32_t* const keys[2],
                         int64_t* const ord[2], int32_t* const start[2], int32_t* const cnt[2], int64_t* g_nf,
                         int32_t* g_rank, int32_t* g_off, int32_t* g_first, int64_t cap_entries, int64_t cap_ord,
                         int64_t cap_grid, int32_t* keys_out, int64_t out_cap, int64_t* out_count, cudaStream_t st) {
  EnumScratch S;
  for (int i = 0; i < 2; ++i) {
    S.keys[i] = keys[i];
    S.ord[i] = ord[i];
    S.start[i] = start[i];
    S.cnt[i] = cnt[i];
  }
  S.g_nf = g_nf;
  S.g_rank = g_rank;
  S.g_off = g_off;
  S.g_first = g_first;
  S.cap_entries = cap_entries;
  S.cap_ord = cap_ord;
  S.cap_grid = cap_grid;
  valid_blocks_kernel<<<1, kPlanThreads, 0, st>>>(n_legs, uniq, leg_off, n_uniq, flows, modulus, eff, S, keys_out,
                                                  out_cap, out_count);
}

void launch_sort_keys(int32_t* keys, int n_legs, int32_t* perm, int64_t n, int64_t pow2, int32_t* sorted_out,
                      cudaStream_t st) {
  sort_keys_kernel<<<1, kPlanThreads, 0, st>>>(keys, n_legs, perm, n, pow2, sorted_out);
}

void launch_operand_target(const int32_t* keys, int n_legs, int64_t n_blocks, const int32_t* flows, int64_t* target,
                           cudaStream_t st) {
  operand_target_kernel<<<1, kPlanThreads, 0, st>>>(keys, n_legs, n_blocks, flows, target);
}

void launch_match(const MatchArgs& m, const int32_t* akeys, int64_t na, const int32_t* bkeys, int64_t nb,
                  const int32_t* valid_sorted, int64_t n_valid, int pass, int32_t* row_count, const int64_t* row_base,
                  int4* pairs, int32_t* present, cudaStream_t st) {
  if (na <= 0) return;
  const int threads = 128;
  const int grid = static_cast<int>((na + threads - 1) / threads);
  match_kernel<<<grid, threads, 0, st>>>(m, akeys, na, bkeys, nb, valid_sorted, n_valid, pass, row_count, row_base,
                                         pairs, present);
}

void launch_compact_out(const int32_t* valid_sorted, int64_t n_valid, int lo_legs, const int32_t* present,
                        const int32_t* o_uniq, const int32_t* o_mult, const int64_t* o_leg_off,
                        const int32_t* o_n_uniq, int32_t* vmap, int32_t* keys_out, int64_t* offs_out, int64_t* n_out,
                        int4* pairs, int64_t n_pairs, cudaStream_t st) {
  compact_out_kernel<<<1, kPlanThreads, 0, st>>>(valid_sorted, n_valid, lo_legs, present, o_uniq, o_mult, o_leg_off,
                                                 o_n_uniq, vmap, keys_out, offs_out, n_out, pairs, n_pairs);
}

void launch_fused_charges(const int32_t* qa, int64_t da, int32_t fa, const int32_t* qb, int64_t db, int32_t fb,
                          int32_t fused_flow, int32_t modulus, int32_t* out, cudaStream_t st) {
  const int64_t n = da * db;
  if (n <= 0) return;
  fused_charges_kernel<<<static_cast<int>((n + 255) / 256), 256, 0, st>>>(qa, da, fa, qb, db, fb, fused_flow, modulus,
                                                                         out);
}

}  // namespace tnx

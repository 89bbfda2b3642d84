// Launchers of the device-side sector planning kernels (planner_dev.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace tnx {

// One pairwise contraction's matching geometry.
struct MatchArgs {
  int32_t la, lb, lo;          // legs of A, B and the output
  int32_t n_con;               // contracted legs
  int32_t a_con[kMaxLegsDev];  // contracted positions in A (sorted contracted chars)
  int32_t b_con[kMaxLegsDev];  // the same chars' positions in B
  int32_t o_src[kMaxLegsDev];  // output leg l: A position (< la) or la + B position
};

// per leg (CTA): sorted distinct charges uniq[leg_off[l] + i], multiplicities
// mult[...], counts n_uniq[l]; status[l] = 1 when the charge range exceeds 2^16
void launch_unique_charges(int n_legs, const int32_t* charges, const int64_t* leg_off, int32_t* uniq, int32_t* mult,
                           int32_t* n_uniq, int32_t* status, cudaStream_t st);
// the reference-order valid keys (single CTA); *out_count = keys or -1 on a capacity overflow
void launch_valid_blocks(int n_legs, const int32_t* uniq, const int64_t* leg_off, const int32_t* n_uniq,
                         const int32_t* flows, int32_t modulus, int64_t eff, int32_t* const keys[2],
                         int64_t* const ord[2], int32_t* const start[2], int32_t* const cnt[2], int64_t* g_nf,
                         int32_t* g_rank, int32_t* g_off, int32_t* g_first, int64_t cap_entries, int64_t cap_ord,
                         int64_t cap_grid, int32_t* keys_out, int64_t out_cap, int64_t* out_count, cudaStream_t st);
// n keys of n_legs sorted lexicographically into sorted_out (pow2 >= n, perm holds pow2 entries)
void launch_sort_keys(int32_t* keys, int n_legs, int32_t* perm, int64_t n, int64_t pow2, int32_t* sorted_out,
                      cudaStream_t st);
// target[0] = the common sum(flow * q) of an operand's blocks, target[1] = 1 when all agree
void launch_operand_target(const int32_t* keys, int n_legs, int64_t n_blocks, const int32_t* flows, int64_t* target,
                           cudaStream_t st);
void launch_match(const MatchArgs& m, const int32_t* akeys, int64_t na, const int32_t* bkeys, int64_t nb,
                  const int32_t* valid_sorted, int64_t n_valid, int pass, int32_t* row_count, const int64_t* row_base,
                  int4* pairs, int32_t* present, cudaStream_t st);
void launch_compact_out(const int32_t* valid_sorted, int64_t n_valid, int lo_legs, const int32_t* present,
                        const int32_t* o_uniq, const int32_t* o_mult, const int64_t* o_leg_off,
                        const int32_t* o_n_uniq, int32_t* vmap, int32_t* keys_out, int64_t* offs_out, int64_t* n_out,
                        int4* pairs, int64_t n_pairs, cudaStream_t st);
void launch_fused_charges(const int32_t* qa, int64_t da, int32_t fa, const int32_t* qb, int64_t db, int32_t fb,
                          int32_t fused_flow, int32_t modulus, int32_t* out, cudaStream_t st);

}  // namespace tnx

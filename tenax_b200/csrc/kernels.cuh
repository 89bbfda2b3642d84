// Host-side launch wrappers of the device kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace tnx {

void launch_pack(const uint64_t* src_tab, const DevPackSeg* segs, const DevChunk* chunks, int n_chunks, int mode,
                 const int32_t* skip, cudaStream_t st);
// chunks: (segment, first row, first 8-wide K chunk, -): pack_rows_per_cta() rows x pack_rows_chunks_per_thread()
// K chunks each; K blocks of the image start at multiples of 8
void launch_pack_rows(const uint64_t* src_tab, const DevRowPackSeg* segs, const int4* chunks, int n_chunks, int mode,
                      const int32_t* skip, cudaStream_t st);
int pack_rows_chunks_per_thread();
int pack_rows_per_cta();  // rows of one chunk
// chunks: seg = pointer-table slot, [start, start+count) elements set to 0
void launch_zero_ranges(const uint64_t* out_tab, const DevChunk* chunks, int n_chunks, const int32_t* skip,
                        cudaStream_t st);
void launch_scatter(const void* res, bool res_f32, double* out, const DevScatSeg* segs, const DevChunk* chunks,
                    int n_chunks, cudaStream_t st);
void launch_mpo_apply(bool x1_f32, int mode, const DevMpoPair* pairs, const DevMpoSlot* islots,
                      const DevMpoOutSlot* oslots, const DevMpoTerm* terms, const int2* chunks, int n_chunks,
                      size_t smem_bytes, const int32_t* skip, cudaStream_t st);
int mpo_points_per_cta();
// consecutive d one MPO thread produces: the stage-4 d padding for the mixed images, 1 for FP64
int mpo_d_per_thread(int mode);
// dst[seg.dst_off + sum idx_l dstr_l] = src[seg.src_off + e] for each chunk's range of elements e
void launch_strided_copy(const double* src, double* dst, const DevCopySeg* segs, const DevChunk* chunks, int n_chunks,
                         cudaStream_t st);
void launch_dot(const double* x, const double* y, int64_t n, int kind, double* result, double* partials,
                const int32_t* skip, cudaStream_t st);
void launch_lanczos_step(double* w, const double* v, const double* vp, double* vnext, int64_t n, double* alpha,
                         double* beta_next, const double* beta_prev, double tol, double tol_rel, int32_t* done,
                         double* partials, cudaStream_t st);
void launch_scale(const double* w, double* out, int64_t n, const double* s, int mode, const int32_t* skip,
                  cudaStream_t st);
void launch_combine(const double* const* basis, const double* coefs, int nv, int64_t n, double* out,
                    cudaStream_t st);
// *status = 0 once *flag == expected, TNX_ERR_TIMEOUT after timeout_ns (one thread)
void launch_wait_flag(const int32_t* flag, int32_t expected, uint64_t timeout_ns, int32_t* status, cudaStream_t st);
int reduce_partials_count();
// *result = max |x_i| (partials: reduce_partials_count() doubles)
void launch_maxabs(const double* x, int64_t n, double* result, double* partials, cudaStream_t st);

// batched max-abs renormalisation (forward: x -> y; adjoint: g = dL/dy, y <- dL/dx)
constexpr int kRenormMax = 8;
constexpr int kRenormBlocks = 64;  // per tensor; the per-tensor totals assume exactly 64
struct RenormArgs {
  const double* x[kRenormMax];
  const double* g[kRenormMax];
  double* y[kRenormMax];
  int64_t n[kRenormMax];
};
// partials: 2 * kRenormMax * kRenormBlocks doubles
void launch_renorm(const RenormArgs& a, int nt, double eps, double* stat, double* partials, cudaStream_t st);
void launch_renorm_adjoint(const RenormArgs& a, int nt, double eps, const double* stat, double* partials,
                           cudaStream_t st);

// grouped GEMMs: out_tab[g.out_slot][rowoff[g.rowoff0 + row] + col] = sum_k A_g[row,k] B_g[col,k]
void launch_gemm_f64(const DevGroup* groups, const DevTile* tiles, int n_tiles, const int64_t* rowoff,
                     const uint64_t* out_tab, const int32_t* skip, cudaStream_t st);
// tcgen05 grouped GEMM; mode IMG_BF16 (3 products over hi/lo images) or IMG_TF32.
// rt: the routed groups' tables (FP32 results only; empty when no group is routed)
void launch_gemm_tc(int mode, const DevGroup* groups, const DevTile* tiles, int n_tiles, const int64_t* rowoff,
                    const uint64_t* out_tab, bool out_f64, int32_t* err_flag, const int32_t* skip, cudaStream_t st,
                    const DevRouteTabs& rt = DevRouteTabs{});
int device_sm_count();
// fused H_eff stages 1-3 (tcgen05, mode IMG_BF16 or IMG_TF32): X3 image from theta and L panels
void launch_heff_fused(int mode, const DevFPair* pairs, const DevFBlock* blocks, const int32_t* term_begin,
                       const DevFTerm* terms, const DevMpoOutSlot* oslots, const DevFTile* tiles, int n_tiles,
                       int32_t* err_flag, const int32_t* skip, cudaStream_t st);
// L block -> panel image (chunks: (segment, 256-element block, -, -))
void launch_pack_lpanels(int mode, const double* L, const DevLPanelSeg* segs, const int4* chunks, int n_chunks,
                         cudaStream_t st);

}  // namespace tnx

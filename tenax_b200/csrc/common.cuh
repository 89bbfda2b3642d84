// Device-side shared definitions: operand-image layouts, table structs,
// and thin PTX wrappers (mbarrier, bulk copy, tcgen05) with bounded waits.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tnx {

// ---------------------------------------------------------------------------
// GEMM operand images.  A group's operand matrix (rows x K, K contiguous) is
// stored as consecutive tiles, tile (rt, kt) at index rt * nKt + kt; a tile is
// the exact shared-memory image the MMA consumes, so it moves with one bulk
// copy.  Padding rows/cols are zero.
//   FP64   : 64 x 16 doubles, element (r,k) at r*16 + (k ^ ((r & 3) << 2))
//            (XOR spreads the DMMA fragment loads over all banks)
//   BF16   : 128 x 64 bf16, byte r*128 + (((2k)>>4) ^ (r&7))*16 + (2k & 15)
//            (the SWIZZLE_128B K-major canonical layout of tcgen05)
//   TF32   : 128 x 32 fp32, byte r*128 + (((4k)>>4) ^ (r&7))*16 + (4k & 15)
// ---------------------------------------------------------------------------
enum ImgMode { IMG_F64 = 0, IMG_BF16 = 1, IMG_TF32 = 2 };

struct ImgGeom {
  int tm, tk, tile_bytes, elem_bytes;
};

__host__ __device__ inline ImgGeom img_geom(int mode) {
  if (mode == IMG_F64) return {64, 16, 8192, 8};
  if (mode == IMG_BF16) return {128, 64, 16384, 2};
  return {128, 32, 16384, 4};
}

// byte offset of element (row, k) inside a group image starting at tile0
__host__ __device__ inline int64_t img_byte_offset(int mode, int64_t tile0, int nKt, int64_t row, int64_t k) {
  if (mode == IMG_F64) {
    int64_t rt = row >> 6, kt = k >> 4;
    int r = static_cast<int>(row & 63), kk = static_cast<int>(k & 15);
    int64_t tile = tile0 + rt * nKt + kt;
    return tile * 8192 + static_cast<int64_t>(r * 16 + (kk ^ ((r & 3) << 2))) * 8;
  }
  if (mode == IMG_BF16) {
    int64_t rt = row >> 7, kt = k >> 6;
    int r = static_cast<int>(row & 127), kb = static_cast<int>(k & 63) * 2;
    int64_t tile = tile0 + rt * nKt + kt;
    return tile * 16384 + r * 128 + (((kb >> 4) ^ (r & 7)) << 4) + (kb & 15);
  }
  int64_t rt = row >> 7, kt = k >> 5;
  int r = static_cast<int>(row & 127), kb = static_cast<int>(k & 31) * 4;
  int64_t tile = tile0 + rt * nKt + kt;
  return tile * 16384 + r * 128 + (((kb >> 4) ^ (r & 7)) << 4) + (kb & 15);
}

// ---------------------------------------------------------------------------
// device tables
// ---------------------------------------------------------------------------
constexpr int kMaxLegsDev = 12;  // equals kMaxLegs of the planner
constexpr int kMpoKAlignDev = 8;  // equals kMpoKAlign of the planner (stage-4 d padding)
constexpr int kFusedMaxN = 96;     // fused H_eff: largest L panel (MMA N) of one input block
constexpr int kFusedMaxSlots = 48; // fused H_eff: input slots of one MPO pair
constexpr int kFusedMaxOut = 64;   // fused H_eff: output slots of one MPO pair (per-warp table rows)
constexpr int kFusedMaxTerms = 160; // fused H_eff: W_l W_r terms of one MPO pair
constexpr int kFusedAccCols = 256; // fused H_eff: TMEM columns of one tile's accumulator

struct DevPackSeg {
  int64_t src_off;    // element offset of the block in operand buffer src_tab[src_slot]
  uint64_t img_addr;  // absolute address of the destination group image (tile 0)
  int64_t lo_off;     // byte offset of the low-part image (BF16 split) from img_addr
  int32_t row0, k0, nKt, nlegs;
  int32_t src_slot, kcount;  // kcount: k extent of the block (product of contracted dims)
  double scale;              // multiplies every packed value (an exact power of two)
  int32_t dims[kMaxLegsDev];
  int32_t rstr[kMaxLegsDev];
  int32_t kstr[kMaxLegsDev];   // contracted-leg strides of the element order (k fastest)
  int32_t kdstr[kMaxLegsDev];  // contracted-leg strides in the image's K coordinate
};

// A block stored k-major with contiguous rows (source offset = k * rows + r,
// one contracted leg first, free legs after it in row-major order), packed
// into an image whose K blocks start at multiples of 8: one thread per row
// writes 8 consecutive k at a time.
struct DevRowPackSeg {
  int64_t src_off;    // element offset of the block in src_tab[src_slot]
  uint64_t img_addr;  // destination group image (tile 0)
  int64_t lo_off;     // byte offset of the low-part image (BF16 split)
  int32_t row0, k0, nKt, rows, kval, src_slot;
  double scale;
  int64_t kstride;    // source elements between consecutive k (>= rows)
};

struct DevScatSeg {
  int64_t dst_off;
  int64_t src_base;  // element offset of (row0, col0) in the result scratch
  int64_t ld;
  int32_t nlegs, neg;  // neg = 1: the block is written negated (a fermionic exchange sign)
  int32_t dims[kMaxLegsDev];
  int32_t rstr[kMaxLegsDev];
  int32_t cstr[kMaxLegsDev];
};

// Copy one block element-for-element: source element e (row-major over
// dims) lands at dst_off + sum_l idx_l * dstr[l].
struct DevCopySeg {
  int64_t src_off;
  int64_t dst_off;
  int32_t nlegs, pad;
  int32_t dims[kMaxLegsDev];
  int64_t dstr[kMaxLegsDev];
};

struct DevChunk {  // one CTA's share of a segment list
  int32_t seg;
  int32_t pad;
  int64_t start;
  int64_t count;
};

struct DevGroup {
  uint64_t a_addr, b_addr;  // absolute addresses of the group's A / B images
  int64_t a_lo, b_lo;       // byte offsets of the low-part images (BF16 split)
  int64_t rowoff0;          // index of row 0 in the row-offset table
  int32_t M, N, nKt, out_slot;  // result rows go to out_tab[out_slot] + rowoff[.] + col
  double scale;             // result = scale * sum_k A B (undoes operand range scaling)
  int32_t vec_ld;           // > 0: every row offset is a multiple of 4 elements and the first
                            // vec_ld (a multiple of 4, >= N) columns may be written: 16-byte stores
  int32_t kk_last;          // tcgen05: MMA K steps (of the 4 per slab) the last K slab needs; 0 = all 4
  // routed epilogue (tcgen05 H_eff stage 1), instead of the row-offset table:
  // row r has (row class, c) = rows[rowoff0 + r], the 8-column unit u has
  // (column class, d of its first column) = cols[cinfo0 + u]; the routes a
  // warp's rows and chunk may need are one window of the route list, named
  // per tile.  routed = 0: plain rows.
  int32_t routed, cinfo0, pad0, pad1;
};

// One destination of the routed stage-1 rows of one (row class, column class)
// pair: kind 0 writes w * row (rounded to FP32, as the MPO kernel computes a
// single-term output) into the stage-4 operand image at image row
// row0 + c * rstride, K k0 + d (8 d per aligned unit, the image's own
// precision split); kind 1 writes w * row in FP32 at
// addr + (c * rstride + d) * 4.  32 bytes: two 16-byte asynchronous copies.
struct DevRoute {
  uint64_t addr;     // kind 0: image tile 0; kind 1: element (c = 0, d = 0)
  int32_t row0, rstride, k0;
  float w;
  uint16_t nKt;
  uint8_t kind, cc;  // cc: the column class the route serves
  int32_t rc;        // the row class the route serves
};
static_assert(sizeof(DevRoute) == 32, "route records are two 16-byte units");

// The routed epilogue's tables (see DevGroup and DevRoute).
struct DevRouteTabs {
  int64_t lo_off;    // byte offset of the low-part stage-4 image (kind 0)
  const DevRoute* routes;
  const int2* win;   // per (tile, lane quarter, 32-column chunk): (first route, count)
  const int2* rows;  // (row class, c) per group row; class -1: no destinations
  const int2* cols;  // (column class, d) per 8-column unit; class -1: padding
};

struct DevTile {
  int32_t g, mt, nt, pad;
};

struct DevMpoPair {
  int32_t mc, md;
  int32_t in0, n_in;
  int32_t out0, n_out;
  int32_t term0, n_terms;
  int32_t n_in_slots, n_out_slots;
};
struct DevMpoSlot {  // one input slot (b,p,q) of one X1 block
  uint64_t base;      // absolute address of the slot's point (c=0, d=0) in the stage-1 result
  int64_t ld;         // element stride between consecutive c (the result matrix's row length)
};
struct DevMpoOutSlot {  // one output slot (s,t,f) of one X3 block
  uint64_t img_addr;    // stage-4 A image of the group (tile 0)
  int64_t lo_off;
  int32_t nKt, row0, k0, rows_per_c, row_add, k_add;
};
struct DevMpoTerm {
  int32_t out_slot, in_slot;
  double w;
};

// Fused H_eff stages 1-3 (heff_fused.cu).  A tile is (MPO pair (q_c, q_d),
// c-tile, d-tile): its TMEM accumulator holds X1[d, (c, b)] of every input
// block of the pair side by side, and its epilogue applies W_l W_r to write
// X3 straight into the stage-4 operand image.
struct DevFPair {
  int32_t blk0, n_blk;  // DevFBlock range (one per input block and physical element pair (p, q))
  int32_t tb0, n_out;   // term_begin[tb0 + o] .. [tb0 + o + 1]: the terms of output slot o
  int32_t out0, n_in;   // DevMpoOutSlot range start; input slots (per-warp staging rows)
  int32_t mc, md, cc;   // c extent, d extent, c values per tile
  int32_t pad;
};
struct DevFBlock {
  uint64_t a_addr;  // theta panel image (128-row tiles; tile (dt, kt) at index dt * nKt + kt)
  uint64_t b_addr;  // L panel image (panel (ct, kt) at index ct * nKt + kt, n_mma rows each)
  int64_t a_lo, b_lo;
  int32_t nKt, kk_last, n_mma, col;  // K slabs, MMA K steps of the last slab, MMA N, TMEM column
  int32_t mb, slot0, slot_stride;    // b extent; staging slot of (b = 0) and its stride per b
  int32_t pad;
};
struct DevFTerm {  // y[o] += w * X1[d, col0 + c_local * cstride] (TMEM column of the input slot)
  int16_t col0, cstride;
  float w;
};
struct DevFTile {
  int32_t pair, ct, dt, pad;
};
// An L block (a, b, c) -> panel image: row (c % cc) * mb + b of panel c / cc, K = a.
struct DevLPanelSeg {
  int64_t src_off;    // element offset of the block in the L buffer
  uint64_t img_addr;  // panel 0 of this block
  int64_t lo_off;
  int32_t ma, mb, mc, cc, n_mma, nKt;
  double scale;
};

// One aligned chunk of kMpoVec consecutive K of one image row (k a multiple
// of kMpoVec): a single 16-byte swizzle unit of a BF16 row (hi and lo
// images), two for TF32, four double pairs for FP64.
constexpr int kMpoVec = kMpoKAlignDev;

template <int MODE, typename AccT>
static __device__ __forceinline__ void img_store_chunk(uint8_t* img, int64_t lo_offset, int nKt, int64_t row, int64_t k,
                                                const AccT (&v)[kMpoVec]) {
  // k is a multiple of kMpoVec
  if constexpr (MODE == IMG_BF16) {
    const int64_t off = img_byte_offset(MODE, 0, nKt, row, k);
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const float a = static_cast<float>(v[2 * u]), b = static_cast<float>(v[2 * u + 1]);
      const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
      const __nv_bfloat162 l = __floats2bfloat162_rn(a - __low2float(h), b - __high2float(h));
      hi[u] = *reinterpret_cast<const uint32_t*>(&h);
      lo[u] = *reinterpret_cast<const uint32_t*>(&l);
    }
    *reinterpret_cast<uint4*>(img + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(img + lo_offset + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  } else if constexpr (MODE == IMG_TF32) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint32_t t[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t[u]) : "f"(static_cast<float>(v[4 * h + u])));
      *reinterpret_cast<uint4*>(img + img_byte_offset(MODE, 0, nKt, row, k + 4 * h)) = make_uint4(t[0], t[1], t[2],
                                                                                                   t[3]);
    }
  } else {
    // FP64 tiles XOR bits 2-3 of the in-row index: element pairs (2u, 2u+1) stay adjacent
#pragma unroll
    for (int u = 0; u < kMpoVec; u += 2)
      *reinterpret_cast<double2*>(img + img_byte_offset(MODE, 0, nKt, row, k + u)) =
          make_double2(static_cast<double>(v[u]), static_cast<double>(v[u + 1]));
  }
}

// ---------------------------------------------------------------------------
// PTX wrappers (sm_100a)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: returns false (and never blocks forever) after max_polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t max_polls) {
  for (uint32_t i = 0; i < max_polls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 1-D bulk async copy global -> shared, completion counted on an mbarrier.
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}


}  // namespace tnx

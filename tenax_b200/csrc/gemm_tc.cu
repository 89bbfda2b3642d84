// Persistent grouped GEMM on the 5th-generation tensor cores (tcgen05 + TMEM).
//
// C_g[row, col] = sum_k A_g[row, k] * B_g[col, k] over every sector group g,
// one work-list entry per 128x128 output tile.  Operands are pre-swizzled
// SWIZZLE_128B K-major image tiles (16 KB each) moved by 1-D bulk async copies
// (cp.async.bulk, no tensor map; every CTA fetches its own tiles) into a
// STAGES-deep ring.
//   BF16X3: A = A_hi + A_lo, B = B_hi + B_lo (bf16 splits of FP64 data);
//           acc += A_hi B_hi + A_hi B_lo + A_lo B_hi, FP32 accumulation in TMEM.
//   TF32:   acc += A B with kind::tf32.
// Warp roles: warp 0 = copy producer, warp 1 = TMEM owner + single-thread MMA
// issuer, warps 2.. = epilogue warps (TMEM -> registers -> global through a
// per-row offset table).  Two TMEM accumulators let the epilogue of tile i
// overlap the MMAs of tile i+1.  Every wait is bounded by a globaltimer
// deadline; on expiry the kernel raises *err_flag, drains its own copies and
// MMAs, frees TMEM and returns.
#include "common.cuh"
#include "kernels.cuh"
#include "tcgen05.cuh"

namespace tnx {

namespace {
constexpr int TBM = 128, TBN = 128;
constexpr int TILE_BYTES = 16384;
// epilogue warps: 4 (one per TMEM lane quarter) or 8 (two per quarter,
// splitting the columns).  Short-K sector GEMMs are epilogue-bound: on the
// 64-problem H_eff batch stage 1 takes 2.21 ms with 8 warps, 2.96 ms with 4.
#ifndef TNX_EPI_WARPS
#define TNX_EPI_WARPS 8
#endif
constexpr int EPI_WARPS = TNX_EPI_WARPS;
static_assert(EPI_WARPS == 4 || EPI_WARPS == 8, "epilogue warps: 4 or 8");
constexpr int THREADS = 64 + 32 * EPI_WARPS;
// TMEM accumulators: the MMAs may run NACC - 1 tiles ahead of the epilogue.
// Four (all 512 columns) measured the same as two on the 64-problem H_eff
// batch (stage 1: 1.84-1.88 vs 1.84-1.86 ms).
#ifndef TNX_TMEM_ACC
#define TNX_TMEM_ACC 2
#endif
constexpr int NACC = TNX_TMEM_ACC;
static_assert(NACC == 2 || NACC == 4, "TMEM accumulators: 2 or 4 (512 columns)");
// The persistent loop over a CTA's tiles with the descriptors of the next
// tiles in flight: the group record of tile t+1 and the tile record of t+2
// are requested while tile t is processed, so no role waits on the
// tile -> group chain of global loads between tiles.
struct TileIter {
  const DevTile* tiles;
  const DevGroup* groups;
  int n, step, t;
  DevTile tl, tl1, tl2;
  DevGroup g, g1;
  __device__ __forceinline__ TileIter(const DevTile* tiles_, const DevGroup* groups_, int n_, int t0)
      : tiles(tiles_), groups(groups_), n(n_), step(static_cast<int>(gridDim.x)), t(t0) {
    if (t < n) {
      tl = tiles[t];
      g = groups[tl.g];
    }
    if (t + step < n) tl1 = tiles[t + step];
  }
  __device__ __forceinline__ void prefetch() {
    if (t + step < n) g1 = groups[tl1.g];
    if (t + 2 * step < n) tl2 = tiles[t + 2 * step];
  }
  __device__ __forceinline__ void advance() {
    t += step;
    tl = tl1;
    g = g1;
    tl1 = tl2;
  }
};

constexpr int kStagePitch = 33;  // fp32 words per staged row (+1 breaks bank conflicts)
constexpr int kEpiStageBytes = EPI_WARPS * 32 * kStagePitch * 4;

// route records of one 32-column chunk's window a warp's staging buffer holds
// (two buffers of NCH windows); larger windows are read from global memory
constexpr int kWin = 64;

template <bool TF32, bool ROUTED>
__host__ __device__ constexpr int gemm_tc_stages() {
  return ROUTED ? (TF32 ? 4 : 2) : (TF32 ? 6 : 3);
}
// dynamic shared memory: operand ring, alignment slack, barriers, per
// epilogue warp a 32 x 33 FP32 staging buffer and (routed) two route windows
template <bool TF32, bool ROUTED>
constexpr int gemm_tc_smem() {
  return gemm_tc_stages<TF32, ROUTED>() * (TF32 ? 2 : 4) * TILE_BYTES + 1024 + 256 + kEpiStageBytes +
         (ROUTED ? EPI_WARPS * 2 * (TBN / 32 / (EPI_WARPS / 4)) * kWin * static_cast<int>(sizeof(DevRoute)) : 0);
}
static_assert(gemm_tc_smem<false, false>() <= 232448 && gemm_tc_smem<false, true>() <= 232448 &&
                  gemm_tc_smem<true, true>() <= 232448, "fits 227 KB of shared memory");

// 16-byte asynchronous copy global -> shared (L2 only), its group commit and
// the wait for every group but the most recent one
static __device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
static __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
static __device__ __forceinline__ void cp_async_wait_prior() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}

// Packed FP32 pairs (sm_100a f32x2): one instruction rounds both lanes of the
// pair exactly as the scalar .rn operation rounds each of them.
static __device__ __forceinline__ uint64_t f2_pack(uint32_t lo, uint32_t hi) {
  uint64_t d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "r"(lo), "r"(hi));
  return d;
}
static __device__ __forceinline__ void f2_unpack(uint64_t a, uint32_t& lo, uint32_t& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=r"(lo), "=r"(hi) : "l"(a));
}
static __device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
static __device__ __forceinline__ uint64_t f2_sub(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// The routed epilogue's store of 8 consecutive K (k a multiple of 8) of image
// row `irow` of the stage-4 image at `img` (16 KB tiles of 128 rows x 128
// bytes, nKt K tiles per 128-row band, SWIZZLE_128B: the 16-byte unit j of a
// row sits at unit j ^ (row & 7)), from 4 packed FP32 pairs: split BF16 hi and lo units (split as the
// packing kernels split), or two TF32 units.  Tile index and in-tile offset
// are formed in 32 bits (the host checks that the route's rows and tiles fit).
template <bool TF32>
static __device__ __forceinline__ void route_store(uint8_t* img, int64_t lo_off, int irow, int nKt, int k,
                                                   const uint64_t (&x)[4]) {
  static_assert(TILE_BYTES == (1 << 14) && TBM == 128, "tile offsets are formed by shifts");
  if constexpr (TF32) {
    const uint32_t tile = static_cast<uint32_t>(irow >> 7) * static_cast<uint32_t>(nKt) + static_cast<uint32_t>(k >> 5);
    uint8_t* row = img + ((static_cast<uint64_t>(tile) << 14) | (static_cast<uint32_t>(irow & 127) << 7));
    const int j = (k >> 2) & 7;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint32_t f[4], w[4];
      f2_unpack(x[2 * h], f[0], f[1]);
      f2_unpack(x[2 * h + 1], f[2], f[3]);
#pragma unroll
      for (int u = 0; u < 4; ++u) asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(w[u]) : "f"(__uint_as_float(f[u])));
      *reinterpret_cast<uint4*>(row + ((static_cast<uint32_t>((j + h) ^ irow) & 7u) << 4)) =
          make_uint4(w[0], w[1], w[2], w[3]);
    }
  } else {
    const uint32_t tile = static_cast<uint32_t>(irow >> 7) * static_cast<uint32_t>(nKt) + static_cast<uint32_t>(k >> 6);
    const uint32_t low = (static_cast<uint32_t>(irow & 127) << 7) | ((static_cast<uint32_t>((k >> 3) ^ irow) & 7u) << 4);
    uint8_t* t = img + ((static_cast<uint64_t>(tile) << 14) | low);
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      uint32_t a, b;
      f2_unpack(x[u], a, b);
      const __nv_bfloat162 h = __floats2bfloat162_rn(__uint_as_float(a), __uint_as_float(b));
      hi[u] = *reinterpret_cast<const uint32_t*>(&h);
      // x - hi, both lanes in one instruction (hi's BF16 halves widened exactly)
      f2_unpack(f2_sub(x[u], f2_pack(hi[u] << 16, hi[u] & 0xffff0000u)), a, b);
      const __nv_bfloat162 l = __floats2bfloat162_rn(__uint_as_float(a), __uint_as_float(b));
      lo[u] = *reinterpret_cast<const uint32_t*>(&l);
    }
    *reinterpret_cast<uint4*>(t) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(t + lo_off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  }
}

// ROUTED: the H_eff stage-1 instance whose groups all carry destinations per
// row class (DevRouteTabs); it runs a 2-stage operand ring (stage 1 is
// short-K) so that each epilogue warp also holds a transpose buffer and two
// route windows in shared memory.
template <bool TF32, typename OutT, bool ROUTED>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_tc_kernel(const DevGroup* __restrict__ groups, const DevTile* __restrict__ tiles, int n_tiles,
                   const int64_t* __restrict__ rowoff, const uint64_t* __restrict__ out_tab, int32_t* err_flag,
                   const int32_t* __restrict__ skip, const DevRouteTabs rt) {
  constexpr int NT = TF32 ? 2 : 4;          // operand tiles per stage
  constexpr int STAGES = gemm_tc_stages<TF32, ROUTED>();  // 192 KB of operand ring (128 KB routed)
  constexpr int KSUB = 4;                   // MMAs per 128-byte K slab (32 B each)
  // TMEM accumulators: the routed instance runs 4 (all 512 columns), so the
  // MMAs run up to three tiles ahead of its longer epilogue
  constexpr int NACC = ROUTED ? 4 : ::tnx::NACC;
  constexpr int TMEM_COLS = NACC * TBN;
  if (skip && *skip) return;

  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_addr = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + ((1024u - (raw_addr & 1023u)) & 1023u);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * NT * TILE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;
  uint64_t* tempty = tfull + NACC;
  uint64_t* drain = tempty + NACC;
  // split BF16: each stage lands in two halves, the hi planes of A and B on
  // full[s] and the lo planes on full2[s], so the hi x hi products start
  // while the lo planes are still in flight
  uint64_t* full2 = drain + 1;
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(full2 + (TF32 ? 0 : STAGES));
  static_assert((2 * STAGES + 2 * NACC + 1 + (TF32 ? 0 : STAGES)) * 8 + 8 <= 256,
                "barriers, TMEM address and abort flag fit the 256 bytes before the epilogue staging");
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);
  // epilogue staging: one 32 x 33 fp32 buffer per epilogue warp, after 256 B of barriers
  float* epi_stage = reinterpret_cast<float*>(smem + STAGES * NT * TILE_BYTES + 256);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      if (!TF32) mbar_init(&full2[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < NACC; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], 32 * EPI_WARPS);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      int last_par[STAGES];
      for (int i = 0; i < STAGES; ++i) last_par[i] = -1;
      bool ok = true;
      for (TileIter it(tiles, groups, n_tiles, blockIdx.x); it.t < n_tiles && ok; it.advance()) {
        it.prefetch();
        const DevTile tl = it.tl;
        const DevGroup g = it.g;
        const uint8_t* ga = reinterpret_cast<const uint8_t*>(g.a_addr) + static_cast<int64_t>(tl.mt) * g.nKt * TILE_BYTES;
        const uint8_t* gb = reinterpret_cast<const uint8_t*>(g.b_addr) + static_cast<int64_t>(tl.nt) * g.nKt * TILE_BYTES;
        for (int kt = 0; kt < g.nKt; ++kt) {
          if (!wait_or_abort(&empty[s], ph ^ 1u, abort_flag, err_flag)) {
            ok = false;
            break;
          }
          uint8_t* st = smem + s * NT * TILE_BYTES;
          const int64_t ko = static_cast<int64_t>(kt) * TILE_BYTES;
          if (TF32) {
            mbar_expect_tx(&full[s], NT * TILE_BYTES);
            bulk_g2s(st, ga + ko, TILE_BYTES, &full[s]);
            bulk_g2s(st + TILE_BYTES, gb + ko, TILE_BYTES, &full[s]);
          } else {
            // stage layout [A hi][A lo][B hi][B lo]; hi planes first
            mbar_expect_tx(&full[s], 2 * TILE_BYTES);
            bulk_g2s(st, ga + ko, TILE_BYTES, &full[s]);
            bulk_g2s(st + 2 * TILE_BYTES, gb + ko, TILE_BYTES, &full[s]);
            mbar_expect_tx(&full2[s], 2 * TILE_BYTES);
            bulk_g2s(st + TILE_BYTES, ga + g.a_lo + ko, TILE_BYTES, &full2[s]);
            bulk_g2s(st + 3 * TILE_BYTES, gb + g.b_lo + ko, TILE_BYTES, &full2[s]);
          }
          last_par[s] = static_cast<int>(ph);
          if (++s == STAGES) {
            s = 0;
            ph ^= 1u;
          }
        }
      }
      if (!ok) {
        // let every copy this thread issued land before the CTA exits
        for (int i = 0; i < STAGES; ++i) {
          if (last_par[i] < 0) continue;
          uint64_t t0 = gtimer();
          while (!mbar_try_wait(&full[i], static_cast<uint32_t>(last_par[i])) && gtimer() - t0 < kTimeoutNs) {
          }
          if (TF32) continue;
          t0 = gtimer();
          while (!mbar_try_wait(&full2[i], static_cast<uint32_t>(last_par[i])) && gtimer() - t0 < kTimeoutNs) {
          }
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      // instruction descriptor without N: FP32 accumulate, operand kinds, M = 128
      const uint32_t idesc0 = (1u << 4) | ((TF32 ? 2u : 1u) << 7) | ((TF32 ? 2u : 1u) << 10) |
                              (static_cast<uint32_t>(TBM >> 4) << 24);
      int s = 0;
      uint32_t ph = 0;
      int acc = 0;
      uint32_t aph = 0;
      bool ok = true;
      bool issued = false;
      for (TileIter it(tiles, groups, n_tiles, blockIdx.x); it.t < n_tiles && ok; it.advance()) {
        it.prefetch();
        const DevTile tl = it.tl;
        const DevGroup g = it.g;
        // MMA extent trimmed to the tile's valid columns (rounded to 16) and
        // the last slab's valid K steps: the operand images are zero beyond
        // both, so the skipped products are exact zeros
        int ncols = g.N - tl.nt * TBN;
        ncols = ncols > TBN ? TBN : ncols;
        const uint32_t n_mma = static_cast<uint32_t>((ncols + 15) / 16 * 16);
        const uint32_t idesc = idesc0 | ((n_mma >> 3) << 17);
        const int ksub_last = g.kk_last > 0 ? g.kk_last : KSUB;
        if (!wait_or_abort(&tempty[acc], aph ^ 1u, abort_flag, err_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + static_cast<uint32_t>(acc * TBN);
        for (int kt = 0; kt < g.nKt; ++kt) {
          if (!wait_or_abort(&full[s], ph, abort_flag, err_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + s * NT * TILE_BYTES);
          const uint64_t da = sw128_desc(sa);
          const int nk = kt + 1 == g.nKt ? ksub_last : KSUB;
          if (TF32) {
            const uint64_t db = sw128_desc(sa + TILE_BYTES);
#pragma unroll
            for (int kk = 0; kk < KSUB; ++kk)
              if (kk < nk) mma_issue<TF32>(d_tmem, da + 2 * kk, db + 2 * kk, idesc, (kt | kk) ? 1u : 0u);
          } else {
            const uint64_t dal = sw128_desc(sa + TILE_BYTES);
            const uint64_t db = sw128_desc(sa + 2 * TILE_BYTES);
            const uint64_t dbl = sw128_desc(sa + 3 * TILE_BYTES);
            // hi x hi on the hi planes, then hi x lo and lo x hi once the lo planes land
#pragma unroll
            for (int kk = 0; kk < KSUB; ++kk) {
              if (kk >= nk) break;
              mma_issue<TF32>(d_tmem, da + 2 * kk, db + 2 * kk, idesc, (kt | kk) ? 1u : 0u);
            }
            issued = true;  // an abort below still waits for these MMAs before TMEM is freed
            if (!wait_or_abort(&full2[s], ph, abort_flag, err_flag)) {
              ok = false;
              break;
            }
            tc_fence_after();
#pragma unroll
            for (int kk = 0; kk < KSUB; ++kk) {
              if (kk >= nk) break;
              mma_issue<TF32>(d_tmem, da + 2 * kk, dbl + 2 * kk, idesc, 1u);
              mma_issue<TF32>(d_tmem, dal + 2 * kk, db + 2 * kk, idesc, 1u);
            }
          }
          issued = true;
          mma_commit(&empty[s]);
          if (++s == STAGES) {
            s = 0;
            ph ^= 1u;
          }
        }
        if (!ok) break;
        mma_commit(&tfull[acc]);
        if (++acc == NACC) {
          acc = 0;
          aph ^= 1u;
        }
      }
      if (!ok && issued) {
        // wait for every MMA this thread issued before TMEM is freed
        mma_commit(drain);
        uint64_t t0 = gtimer();
        while (!mbar_try_wait(drain, 0) && gtimer() - t0 < kTimeoutNs) {
        }
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int r_in_tile = q * 32 + lane;
    const int e = warp - 2;  // epilogue warp 0..EPI_WARPS-1
    constexpr int kColsPerWarp = TBN / (EPI_WARPS / 4);
    const int c_begin = (e / 4) * kColsPerWarp;
    float* stg = epi_stage + e * 32 * kStagePitch;
    int acc = 0;
    uint32_t aph = 0;
    // Routed launches: each warp's route windows of a tile (one per 32-column
    // chunk it writes) are copied into its staging buffer asynchronously one
    // tile ahead (two buffers), the window bounds two tiles ahead, and the
    // next tile's row and column classes one tile ahead, so no table load
    // sits between a tile's accumulator and its stores.
    constexpr int NCH = TBN / 32 / (EPI_WARPS / 4);  // 32-column chunks per warp
    constexpr bool routed_launch = ROUTED;
    // [2 buffers][NCH chunks][kWin records], after every warp's transpose buffer
    DevRoute* wbuf = reinterpret_cast<DevRoute*>(epi_stage + EPI_WARPS * 32 * kStagePitch) + e * 2 * NCH * kWin;
    const int step = static_cast<int>(gridDim.x);
    int par = 0;
    int2 tw0[NCH], tw1[NCH], tw2[NCH];
    int2 ri_n = make_int2(-1, 0), cu_n[NCH];
    auto win_of = [&](int t, int j) -> int2 {
      return t < n_tiles ? rt.win[static_cast<int64_t>(t) * 16 + q * 4 + (e / 4) + (EPI_WARPS / 4) * j] : make_int2(0, 0);
    };
    auto copy_windows = [&](const int2 (&w)[NCH], int buf) {
#pragma unroll
      for (int j = 0; j < NCH; ++j)
        if (w[j].y <= kWin)
          for (int k = lane; k < w[j].y; k += 32) {
            const DevRoute* src = rt.routes + w[j].x + k;
            DevRoute* dst = wbuf + (buf * NCH + j) * kWin + k;
            cp_async16(dst, src);
            cp_async16(reinterpret_cast<uint8_t*>(dst) + 16, reinterpret_cast<const uint8_t*>(src) + 16);
          }
      cp_async_commit();
    };
    auto classes_of = [&](int t, const DevGroup& gg, const DevTile& tt) {
      // this lane's row class and the chunk units' column classes (lane u < 4: unit u)
      const int row = tt.mt * TBM + r_in_tile;
      ri_n = (t < n_tiles && gg.routed && row < gg.M) ? rt.rows[gg.rowoff0 + row] : make_int2(-1, 0);
#pragma unroll
      for (int j = 0; j < NCH; ++j) {
        const int col = tt.nt * TBN + 32 * (e / 4) + 32 * (EPI_WARPS / 4) * j + 8 * (lane & 3);
        cu_n[j] = (t < n_tiles && gg.routed && col < gg.N) ? rt.cols[gg.cinfo0 + col / 8] : make_int2(-1, 0);
      }
    };
    if (routed_launch && static_cast<int>(blockIdx.x) < n_tiles) {
#pragma unroll
      for (int j = 0; j < NCH; ++j) {
        tw0[j] = win_of(blockIdx.x, j);
        tw1[j] = win_of(blockIdx.x + step, j);
        tw2[j] = win_of(blockIdx.x + 2 * step, j);
      }
      copy_windows(tw0, 0);
      const DevTile t0 = tiles[blockIdx.x];
      classes_of(blockIdx.x, groups[t0.g], t0);
    }
    for (TileIter it(tiles, groups, n_tiles, blockIdx.x); it.t < n_tiles; it.advance()) {
      it.prefetch();
      const DevTile tl = it.tl;
      const DevGroup g = it.g;
      // Routed launches advance the window and class pipeline on every tile,
      // whichever kind of group it belongs to: this tile's classes and
      // windows were requested a tile ago; request the next tile's.
      int2 ri = make_int2(-1, 0), cu[NCH], tw[NCH];
      const int cur_par = par;
      if constexpr (routed_launch) {
        ri = ri_n;
#pragma unroll
        for (int j = 0; j < NCH; ++j) {
          cu[j] = cu_n[j];
          tw[j] = tw0[j];
        }
        copy_windows(tw1, par ^ 1);
        if (it.t + step < n_tiles) classes_of(it.t + step, it.g1, it.tl1);
#pragma unroll
        for (int j = 0; j < NCH; ++j) {
          tw0[j] = tw1[j];
          tw1[j] = tw2[j];
          tw2[j] = win_of(it.t + 3 * step, j);
        }
        par ^= 1;
      }
      if constexpr (sizeof(OutT) == 4) {
        if (g.routed && routed_launch) {
          // Routed rows (b, c): the lane quarter's 32 rows, 32-column chunks.
          // A chunk is staged through shared memory so that each lane then
          // holds its 8-column unit (lane % 4) of four rows (lane / 4 + 8 i)
          // and the four lanes of a quad write one row's 32 columns: every
          // store instruction fills whole 32-byte sectors of 8 rows.  A row's
          // row class and a unit's column class select the routes of the
          // tile's window that apply.
          int rcl[4], crow[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            rcl[i] = __shfl_sync(0xffffffffu, ri.x, (lane >> 2) + 8 * i);
            crow[i] = __shfl_sync(0xffffffffu, ri.y, (lane >> 2) + 8 * i);
          }
          cp_async_wait_prior();  // this tile's windows have landed
          __syncwarp();
          if (!wait_or_abort(&tfull[acc], aph, abort_flag, err_flag)) break;
          tc_fence_after();
          const uint32_t tbase = tmem_base + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(acc * TBN);
#pragma unroll
          for (int j = 0; j < NCH; ++j) {
            const int c0 = 32 * (e / 4) + 32 * (EPI_WARPS / 4) * j;
            if (tl.nt * TBN + c0 >= g.N || tw[j].y == 0) continue;  // warp-uniform: nothing to write
            // the chunk in shared memory as 32 rows of 8 16-byte units, unit c
            // of row r at r * 8 + (c ^ (r & 7)): the row-per-lane writes and
            // the quad-per-row reads are both free of bank conflicts
            uint4* s4 = reinterpret_cast<uint4*>(stg);
            {
              uint32_t v[32];
              tmem_ld32(tbase + c0, v);
#pragma unroll
              for (int c = 0; c < 8; ++c)
                s4[lane * 8 + (c ^ (lane & 7))] = make_uint4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
            }
            __syncwarp();
            uint64_t xv[4][kMpoVec / 2];  // rows lane / 4 + 8 i: the unit's 8 columns as packed pairs
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                const uint4 u = s4[((lane >> 2) + 8 * i) * 8 + ((2 * (lane & 3) + h) ^ ((lane >> 2) & 7))];
                xv[i][2 * h] = f2_pack(u.x, u.y);
                xv[i][2 * h + 1] = f2_pack(u.z, u.w);
              }
            __syncwarp();  // the staging buffer is free for the next chunk
            const int ccl = cu[j].x, dl = cu[j].y;  // this lane's unit: column class, d
            DevRoute* wr = wbuf + (cur_par * NCH + j) * kWin;
            const bool in_smem = tw[j].y <= kWin;  // warp-uniform
#pragma unroll 1
            for (int r = 0; r < tw[j].y; ++r) {
              if (!in_smem && r % kWin == 0) {
                // a window larger than the buffer: the next kWin records, copied in by the warp
                __syncwarp();
                for (int k = lane; k < kWin && r + k < tw[j].y; k += 32) wr[k] = rt.routes[tw[j].x + r + k];
                __syncwarp();
              }
              const DevRoute R = wr[r % kWin];
              if (R.cc != ccl) continue;
              const uint32_t wb = __float_as_uint(R.w);
              const uint64_t w2 = f2_pack(wb, wb);
#pragma unroll
              for (int i = 0; i < 4; ++i) {
                if (R.rc != rcl[i]) continue;
                uint64_t x[kMpoVec / 2];
#pragma unroll
                for (int u = 0; u < kMpoVec / 2; ++u) x[u] = f2_mul(xv[i][u], w2);
                // rows and offsets fit 32 bits (checked when the routes are built)
                const int rrel = crow[i] * R.rstride;
                if (R.kind == 1) {
                  uint32_t f[8];
#pragma unroll
                  for (int u = 0; u < 4; ++u) f2_unpack(x[u], f[2 * u], f[2 * u + 1]);
                  uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<float*>(R.addr) + (rrel + dl));
                  dst[0] = make_uint4(f[0], f[1], f[2], f[3]);
                  dst[1] = make_uint4(f[4], f[5], f[6], f[7]);
                } else {
                  route_store<TF32>(reinterpret_cast<uint8_t*>(R.addr), rt.lo_off, R.row0 + rrel, R.nKt, R.k0 + dl, x);
                }
              }
            }
          }
          __syncwarp();  // this window buffer is rewritten by the next tile
          tc_fence_before();
          mbar_arrive(&tempty[acc]);
          if (++acc == NACC) {
            acc = 0;
            aph ^= 1u;
          }
          continue;
        }
      }
      // the row offset does not depend on the accumulator: request it before waiting
      const int row = tl.mt * TBM + r_in_tile;
      const int64_t ro = row < g.M ? rowoff[g.rowoff0 + row] : -1;
      // all lanes wait (the tcgen05.ld below is warp-collective)
      if (!wait_or_abort(&tfull[acc], aph, abort_flag, err_flag)) break;
      tc_fence_after();
      OutT* out = reinterpret_cast<OutT*>(out_tab[g.out_slot]);
      const uint32_t tbase = tmem_base + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(acc * TBN);
      // group scales are powers of two, so the multiply is exact in the
      // output's own precision (FP32 outputs only ever carry scale 1; a
      // per-element FP64 round trip there doubled the epilogue's cost)
      const OutT scale = static_cast<OutT>(g.scale);
      // FP32 results with aligned rows store straight from the 16x256b
      // fragments; otherwise each lane holds one row (32x32b) and 32x32
      // chunks are staged through shared memory so that every store
      // instruction writes 32 consecutive columns of one row.
#pragma unroll 1
      for (int c0 = c_begin; c0 < c_begin + kColsPerWarp; c0 += 32) {
        bool done = false;
        if constexpr (sizeof(OutT) == 4) {
          if (g.vec_ld > 0) {
            // register-direct path (no staging): two 16-row slabs in the
            // 16x256b fragment layout; four lanes hold 8 consecutive columns
            // of one row, so every 8-byte store instruction fills whole
            // 32-byte sectors of 8 rows
            uint32_t v0[16], v1[16];
            tmem_ld16x256b_x4(tbase + c0, v0);
            tmem_ld16x256b_x4(tbase + (16u << 16) + c0, v1);
            tmem_wait_ld();
            const float fs = static_cast<float>(scale);
            const int cl = tl.nt * TBN + c0 + 2 * (lane & 3);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const uint32_t(&v)[16] = h ? v1 : v0;
              const int r = 16 * h + (lane >> 2);
              const int64_t ro_a = __shfl_sync(0xffffffffu, ro, r);
              const int64_t ro_b = __shfl_sync(0xffffffffu, ro, r + 8);
#pragma unroll
              for (int j = 0; j < 4; ++j) {
                const int col = cl + 8 * j;  // even; vec_ld is a multiple of 4
                if (col < g.vec_ld) {
                  if (ro_a >= 0)
                    *reinterpret_cast<float2*>(reinterpret_cast<float*>(out) + ro_a + col) =
                        make_float2(__uint_as_float(v[4 * j]) * fs, __uint_as_float(v[4 * j + 1]) * fs);
                  if (ro_b >= 0)
                    *reinterpret_cast<float2*>(reinterpret_cast<float*>(out) + ro_b + col) =
                        make_float2(__uint_as_float(v[4 * j + 2]) * fs, __uint_as_float(v[4 * j + 3]) * fs);
                }
              }
            }
            done = true;
          }
        }
        if (!done) {
          uint32_t v[32];
          tmem_ld32(tbase + c0, v);
#pragma unroll
          for (int j = 0; j < 32; ++j) stg[lane * kStagePitch + j] = __uint_as_float(v[j]);
          __syncwarp();
          const int col = tl.nt * TBN + c0 + lane;
          const bool col_ok = col < g.N;
#pragma unroll 4
          for (int r = 0; r < 32; ++r) {
            const int64_t ro_r = __shfl_sync(0xffffffffu, ro, r);
            if (ro_r >= 0 && col_ok)
              out[ro_r + col] = static_cast<OutT>(stg[r * kStagePitch + lane]) * scale;
          }
          __syncwarp();
        }
      }
      tc_fence_before();
      mbar_arrive(&tempty[acc]);
      if (++acc == NACC) {
        acc = 0;
        aph ^= 1u;
      }
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");  // no route copy outlives the CTA
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS)
                 : "memory");
  }
}

template <bool TF32, typename OutT, bool ROUTED>
void launch_tc_impl(const DevGroup* groups, const DevTile* tiles, int n_tiles, const int64_t* rowoff,
                    const uint64_t* out_tab, int32_t* err_flag, const int32_t* skip, cudaStream_t st,
                    const DevRouteTabs& rt) {
  constexpr int smem = gemm_tc_smem<TF32, ROUTED>();
  if (cudaFuncSetAttribute(gemm_tc_kernel<TF32, OutT, ROUTED>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
      cudaSuccess)
    return;  // the thread's last CUDA error, checked by every caller
  int grid = device_sm_count();
  if (grid > n_tiles) grid = n_tiles;
  gemm_tc_kernel<TF32, OutT, ROUTED>
      <<<grid, THREADS, smem, st>>>(groups, tiles, n_tiles, rowoff, out_tab, err_flag, skip, rt);
}
}  // namespace

void launch_gemm_tc(int mode, const DevGroup* groups, const DevTile* tiles, int n_tiles, const int64_t* rowoff,
                    const uint64_t* out_tab, bool out_f64, int32_t* err_flag, const int32_t* skip, cudaStream_t st,
                    const DevRouteTabs& rt) {
  if (n_tiles <= 0) return;
  const bool routed = rt.win != nullptr;  // every group routed, FP32 results
  if (mode == IMG_TF32) {
    if (out_f64)
      launch_tc_impl<true, double, false>(groups, tiles, n_tiles, rowoff, out_tab, err_flag, skip, st, rt);
    else if (routed)
      launch_tc_impl<true, float, true>(groups, tiles, n_tiles, rowoff, out_tab, err_flag, skip, st, rt);
    else
      launch_tc_impl<true, float, false>(groups, tiles, n_tiles, rowoff, out_tab, err_flag, skip, st, rt);
  } else {
    if (out_f64)
      launch_tc_impl<false, double, false>(groups, tiles, n_tiles, rowoff, out_tab, err_flag, skip, st, rt);
    else if (routed)
      launch_tc_impl<false, float, true>(groups, tiles, n_tiles, rowoff, out_tab, err_flag, skip, st, rt);
    else
      launch_tc_impl<false, float, false>(groups, tiles, n_tiles, rowoff, out_tab, err_flag, skip, st, rt);
  }
}

}  // namespace tnx

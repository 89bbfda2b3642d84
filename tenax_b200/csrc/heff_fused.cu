// Fused stages 1-3 of the two-site H_eff on the tcgen05 tensor cores:
//
//   X3[c,s,t,f,d] = sum_{b,p,q} Wlr[b,p,q,s,t,f] * sum_a L[a,b,c] theta[a,p,q,d]
//
// written straight into the stage-4 operand image, with no X1 in HBM.
//
// Work unit: one MPO pair (q_c, q_d) of one problem, a tile of cc values of c
// and 128 values of d.  Every input block of the pair -- one per (q_b, q_p,
// q_q) and physical element (p, q) -- is one MMA chain with
//   A = theta panel: 128 rows d (of the pair's q_d sector), K = a;
//   B = L panel:     n_mma rows (c, b) of the tile's c values, K = a;
// accumulating D[d, (c, b)] into its own TMEM column range.  TMEM lane = d for
// every block, so after the MMAs one thread holds, for its d, every input
// slot (b, p, q) of every c of the tile: the W_l W_r application is
// thread-local.  Each epilogue warp keeps the current pair's output slots
// and terms in its own shared-memory table, sums each output slot's terms
// straight from TMEM (one column load per term), and transposes groups of 8
// outputs across 8 lanes with XOR shuffles so that
// every lane ends with 8 consecutive d of one output: one aligned 16-byte
// chunk of a stage-4 image row (hi and lo images for BF16x3).
//
// Roles as in gemm_tc.cu: warp 0 issues the bulk copies into a ring of
// operand stages, warp 1 owns TMEM (two 256-column accumulators, so a
// tile's epilogue overlaps the next tile's MMAs) and one thread issues the
// MMAs, warps 2-9 are the epilogue (two per TMEM lane quarter, alternating
// c values).  Every wait is bounded by a GPU-timer deadline; on expiry the
// kernel raises *err_flag, drains its own copies and MMAs, frees TMEM and
// returns.  No TMA tensor maps and no multicast: each CTA copies its own
// tiles from this GPU's memory.
#include "common.cuh"
#include "kernels.cuh"
#include "tcgen05.cuh"

namespace tnx {

namespace {
constexpr int F_A_BYTES = 16384;             // one theta image tile: 128 rows x 128 bytes
constexpr int F_B_BYTES = kFusedMaxN * 128;  // one L panel at its largest
constexpr int F_EPI_WARPS = 8;
constexpr int F_THREADS = 64 + 32 * F_EPI_WARPS;
constexpr int F_ACC_COLS = kFusedAccCols;  // per accumulator; two accumulators = all 512 TMEM columns
constexpr int F_STAGE_BYTES_BF16 = 2 * F_A_BYTES + 2 * F_B_BYTES;
constexpr int F_STAGE_BYTES_TF32 = F_A_BYTES + F_B_BYTES;
constexpr int F_STAGES_BF16 = 3;
constexpr int F_STAGES_TF32 = 6;
// per-warp copy of the current MPO pair's output slots, term offsets and terms
constexpr int F_TAB_SO = kFusedMaxOut * static_cast<int>(sizeof(DevMpoOutSlot));
constexpr int F_TAB_TB = (kFusedMaxOut + 1) * 4;
constexpr int F_TAB_TM = kFusedMaxTerms * static_cast<int>(sizeof(DevFTerm));
constexpr int F_TAB_BYTES = (F_TAB_SO + F_TAB_TB + F_TAB_TM + 15) / 16 * 16;
constexpr int F_XS_BYTES = F_EPI_WARPS * F_TAB_BYTES;
static_assert(F_A_BYTES % 1024 == 0 && F_B_BYTES % 1024 == 0, "SW128 operand tiles must start on 1024 bytes");

// 8x8 transpose among the 8 lanes of each aligned lane group: on entry lane
// i holds v[j] = M[j][i], on exit v[j] = M[i][j].
__device__ __forceinline__ void transpose8(float (&v)[8], int lane) {
#pragma unroll
  for (int s = 4; s >= 1; s >>= 1) {
    const bool upper = (lane & s) != 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (j & s) continue;
      const float send = upper ? v[j] : v[j | s];
      const float recv = __shfl_xor_sync(0xffffffffu, send, s);
      if (upper)
        v[j] = recv;
      else
        v[j | s] = recv;
    }
  }
}

template <bool TF32>
struct FGeom {
  static constexpr int kStageBytes = TF32 ? F_STAGE_BYTES_TF32 : F_STAGE_BYTES_BF16;
  static constexpr int kStages = TF32 ? F_STAGES_TF32 : F_STAGES_BF16;
};

template <bool TF32>
__global__ void __launch_bounds__(F_THREADS, 1)
    heff_fused_kernel(const DevFPair* __restrict__ pairs, const DevFBlock* __restrict__ blocks,
                      const int32_t* __restrict__ term_begin, const DevFTerm* __restrict__ terms,
                      const DevMpoOutSlot* __restrict__ oslots, const DevFTile* __restrict__ tiles, int n_tiles,
                      int32_t* err_flag, const int32_t* __restrict__ skip) {
  constexpr int STAGE_BYTES = FGeom<TF32>::kStageBytes;
  constexpr int STAGES = FGeom<TF32>::kStages;
  constexpr int KSUB = 4;  // MMA K steps per 128-byte slab
  constexpr int MODE = TF32 ? IMG_TF32 : IMG_BF16;
  if (skip && *skip) return;

  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_addr = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + ((1024u - (raw_addr & 1023u)) & 1023u);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);
  uint8_t* tab_all = smem + STAGES * STAGE_BYTES + 256;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], 32 * F_EPI_WARPS);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(2 * F_ACC_COLS)
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
      for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        const DevFTile tl = tiles[t];
        const DevFPair pr = pairs[tl.pair];
        for (int j = 0; j < pr.n_blk && ok; ++j) {
          const DevFBlock bk = blocks[pr.blk0 + j];
          const int b_bytes = bk.n_mma * 128;
          const uint8_t* ga = reinterpret_cast<const uint8_t*>(bk.a_addr) +
                              static_cast<int64_t>(tl.dt) * bk.nKt * F_A_BYTES;
          const uint8_t* gb = reinterpret_cast<const uint8_t*>(bk.b_addr) +
                              static_cast<int64_t>(tl.ct) * bk.nKt * b_bytes;
          for (int kt = 0; kt < bk.nKt; ++kt) {
            if (!wait_or_abort(&empty[s], ph ^ 1u, abort_flag, err_flag)) {
              ok = false;
              break;
            }
            uint8_t* st = smem + s * STAGE_BYTES;
            const int64_t ka = static_cast<int64_t>(kt) * F_A_BYTES, kb = static_cast<int64_t>(kt) * b_bytes;
            if (TF32) {
              mbar_expect_tx(&full[s], F_A_BYTES + b_bytes);
              bulk_g2s(st, ga + ka, F_A_BYTES, &full[s]);
              bulk_g2s(st + F_A_BYTES, gb + kb, b_bytes, &full[s]);
            } else {
              mbar_expect_tx(&full[s], 2 * F_A_BYTES + 2 * b_bytes);
              bulk_g2s(st, ga + ka, F_A_BYTES, &full[s]);
              bulk_g2s(st + F_A_BYTES, ga + bk.a_lo + ka, F_A_BYTES, &full[s]);
              bulk_g2s(st + 2 * F_A_BYTES, gb + kb, b_bytes, &full[s]);
              bulk_g2s(st + 2 * F_A_BYTES + F_B_BYTES, gb + bk.b_lo + kb, b_bytes, &full[s]);
            }
            last_par[s] = static_cast<int>(ph);
            if (++s == STAGES) {
              s = 0;
              ph ^= 1u;
            }
          }
        }
      }
      if (!ok) {
        // let every copy this thread issued land before the CTA exits
        for (int i = 0; i < STAGES; ++i) {
          if (last_par[i] < 0) continue;
          const uint64_t t0 = gtimer();
          while (!mbar_try_wait(&full[i], static_cast<uint32_t>(last_par[i])) && gtimer() - t0 < kTimeoutNs) {
          }
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      // instruction descriptor without N: FP32 accumulate, operand kinds, M = 128
      const uint32_t idesc0 = (1u << 4) | ((TF32 ? 2u : 1u) << 7) | ((TF32 ? 2u : 1u) << 10) | (8u << 24);
      int s = 0;
      uint32_t ph = 0;
      int acc = 0;
      uint32_t aph = 0;
      bool ok = true, issued = false;
      for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        const DevFTile tl = tiles[t];
        const DevFPair pr = pairs[tl.pair];
        if (!wait_or_abort(&tempty[acc], aph ^ 1u, abort_flag, err_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        for (int j = 0; j < pr.n_blk && ok; ++j) {
          const DevFBlock bk = blocks[pr.blk0 + j];
          const uint32_t idesc = idesc0 | ((static_cast<uint32_t>(bk.n_mma) >> 3) << 17);
          const uint32_t d_tmem = tmem_base + static_cast<uint32_t>(acc * F_ACC_COLS + bk.col);
          const int ksub_last = bk.kk_last > 0 ? bk.kk_last : KSUB;
          for (int kt = 0; kt < bk.nKt; ++kt) {
            if (!wait_or_abort(&full[s], ph, abort_flag, err_flag)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
            const int nk = kt + 1 == bk.nKt ? ksub_last : KSUB;
            if (TF32) {
              const uint64_t da = sw128_desc(sa), db = sw128_desc(sa + F_A_BYTES);
#pragma unroll
              for (int kk = 0; kk < KSUB; ++kk)
                if (kk < nk) mma_issue<true>(d_tmem, da + 2 * kk, db + 2 * kk, idesc, (kt | kk) ? 1u : 0u);
            } else {
              const uint64_t da = sw128_desc(sa), dal = sw128_desc(sa + F_A_BYTES);
              const uint64_t db = sw128_desc(sa + 2 * F_A_BYTES), dbl = sw128_desc(sa + 2 * F_A_BYTES + F_B_BYTES);
#pragma unroll
              for (int kk = 0; kk < KSUB; ++kk) {
                if (kk >= nk) break;
                mma_issue<false>(d_tmem, da + 2 * kk, db + 2 * kk, idesc, (kt | kk) ? 1u : 0u);
                mma_issue<false>(d_tmem, da + 2 * kk, dbl + 2 * kk, idesc, 1u);
                mma_issue<false>(d_tmem, dal + 2 * kk, db + 2 * kk, idesc, 1u);
              }
            }
            issued = true;
            mma_commit(&empty[s]);
            if (++s == STAGES) {
              s = 0;
              ph ^= 1u;
            }
          }
        }
        if (!ok) break;
        mma_commit(&tfull[acc]);
        acc ^= 1;
        if (acc == 0) aph ^= 1u;
      }
      if (!ok && issued) {
        // wait for every MMA this thread issued before TMEM is freed
        mma_commit(drain);
        const uint64_t t0 = gtimer();
        while (!mbar_try_wait(drain, 0) && gtimer() - t0 < kTimeoutNs) {
        }
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;   // TMEM lane quarter this warp may access
    const int e = warp - 2;   // epilogue warp 0..7
    const int half = e >> 2;  // c values of this parity
    // this warp's copy of the current pair's tables (reloaded when the pair changes)
    uint8_t* tab = tab_all + e * F_TAB_BYTES;
    DevMpoOutSlot* wso = reinterpret_cast<DevMpoOutSlot*>(tab);
    int32_t* wtb = reinterpret_cast<int32_t*>(tab + F_TAB_SO);
    DevFTerm* wtm = reinterpret_cast<DevFTerm*>(tab + F_TAB_SO + F_TAB_TB);
    int cached_pair = -1;
    int acc = 0;
    uint32_t aph = 0;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
      const DevFTile tl = tiles[t];
      const DevFPair pr = pairs[tl.pair];
      if (tl.pair != cached_pair) {
        __syncwarp();
        const uint32_t* so_src = reinterpret_cast<const uint32_t*>(oslots + pr.out0);
        uint32_t* so_dst = reinterpret_cast<uint32_t*>(wso);
        constexpr int kSoWords = static_cast<int>(sizeof(DevMpoOutSlot) / 4);
        for (int i = lane; i < pr.n_out * kSoWords; i += 32) so_dst[i] = so_src[i];
        const int t0 = term_begin[pr.tb0];
        for (int i = lane; i <= pr.n_out; i += 32) wtb[i] = term_begin[pr.tb0 + i] - t0;
        const int nterm = term_begin[pr.tb0 + pr.n_out] - t0;
        for (int i = lane; i < nterm; i += 32) wtm[i] = terms[t0 + i];
        __syncwarp();
        cached_pair = tl.pair;
      }
      // all lanes wait (the tcgen05.ld below is warp-collective)
      if (!wait_or_abort(&tfull[acc], aph, abort_flag, err_flag)) break;
      tc_fence_after();
      const uint32_t tbase =
          tmem_base + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(acc * F_ACC_COLS);
      const int d_chunk = tl.dt * 128 + q * 32 + (lane >> 3) * 8;  // first d of this lane's output chunk
      // a lane quarter whose d rows all lie past the sector has nothing to write
      const bool live = tl.dt * 128 + q * 32 < pr.md;
      for (int og = 0; live && og < pr.n_out; og += 8) {
        // this group's table entries (every output's first two terms), read
        // once and applied to each of this warp's c values
        int nt[8], tb[8], col[8][2], cs[8][2];
        float w[8][2];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int o = og + i;
          tb[i] = o < pr.n_out ? wtb[o] : 0;
          nt[i] = o < pr.n_out ? wtb[o + 1] - tb[i] : 0;
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            const DevFTerm tm = k < nt[i] ? wtm[tb[i] + k] : DevFTerm{0, 0, 0.0f};
            col[i][k] = tm.col0;
            cs[i][k] = tm.cstride;
            w[i][k] = tm.w;
          }
        }
        const int o_mine = og + (lane & 7);
        const bool store = o_mine < pr.n_out && d_chunk < pr.md;
        DevMpoOutSlot so{};
        if (store) so = wso[o_mine];
        for (int cl = half; cl < pr.cc; cl += 2) {
          const int64_t c = static_cast<int64_t>(tl.ct) * pr.cc + cl;
          if (c >= pr.mc) break;
          float y[8];
          uint32_t v[8][2];
#pragma unroll
          for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int k = 0; k < 2; ++k)
              if (k < nt[i]) v[i][k] = tmem_ld1(tbase + static_cast<uint32_t>(col[i][k] + cl * cs[i][k]));
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            y[i] = 0.0f;
#pragma unroll
            for (int k = 0; k < 2; ++k)
              if (k < nt[i]) y[i] = fmaf(w[i][k], __uint_as_float(v[i][k]), y[i]);
            for (int k = 2; k < nt[i]; ++k) {
              const DevFTerm tm = wtm[tb[i] + k];
              const uint32_t x = tmem_ld1(tbase + static_cast<uint32_t>(tm.col0 + cl * tm.cstride));
              tmem_wait_ld();
              y[i] = fmaf(tm.w, __uint_as_float(x), y[i]);
            }
          }
          transpose8(y, lane);
          if (store)
            img_store_chunk<MODE>(reinterpret_cast<uint8_t*>(so.img_addr), so.lo_off, so.nKt,
                                  so.row0 + c * so.rows_per_c + so.row_add, so.k0 + so.k_add + d_chunk, y);
        }
      }
      tc_fence_before();
      mbar_arrive(&tempty[acc]);
      acc ^= 1;
      if (acc == 0) aph ^= 1u;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(2 * F_ACC_COLS)
                 : "memory");
  }
}

template <bool TF32>
void launch_fused_impl(const DevFPair* pairs, const DevFBlock* blocks, const int32_t* term_begin,
                       const DevFTerm* terms, const DevMpoOutSlot* oslots, const DevFTile* tiles, int n_tiles,
                       int32_t* err_flag, const int32_t* skip, cudaStream_t st) {
  const int smem = FGeom<TF32>::kStages * FGeom<TF32>::kStageBytes + 1024 /*align*/ + 256 /*barriers*/ + F_XS_BYTES;
  if (cudaFuncSetAttribute(heff_fused_kernel<TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
      cudaSuccess)
    return;  // the thread's last CUDA error, checked by every caller
  int grid = device_sm_count();
  if (grid > n_tiles) grid = n_tiles;
  heff_fused_kernel<TF32>
      <<<grid, F_THREADS, smem, st>>>(pairs, blocks, term_begin, terms, oslots, tiles, n_tiles, err_flag, skip);
}

// ---------------------------------------------------------------------------
// L panels: one thread per element of an L block (a, b, c), c fastest, so the
// reads are coalesced; the image is written once per operator.
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(256) pack_lpanel_kernel(const double* __restrict__ L,
                                                          const DevLPanelSeg* __restrict__ segs,
                                                          const int4* __restrict__ chunks) {
  const int4 ch = chunks[blockIdx.x];  // (segment, first element / 256, -, -)
  const DevLPanelSeg s = segs[ch.x];
  const int64_t e = static_cast<int64_t>(ch.y) * 256 + threadIdx.x;
  const int64_t n = static_cast<int64_t>(s.ma) * s.mb * s.mc;
  if (e >= n) return;
  const int c = static_cast<int>(e % s.mc);
  const int b = static_cast<int>((e / s.mc) % s.mb);
  const int a = static_cast<int>(e / (static_cast<int64_t>(s.mc) * s.mb));
  const double v = L[s.src_off + e] * s.scale;
  constexpr int TK = MODE == IMG_TF32 ? 32 : 64;
  const int ct = c / s.cc, r = (c - ct * s.cc) * s.mb + b, kt = a / TK;
  const int kb = (a - kt * TK) * (MODE == IMG_TF32 ? 4 : 2);
  const int64_t off = (static_cast<int64_t>(ct) * s.nKt + kt) * (s.n_mma * 128) + r * 128 +
                      (((kb >> 4) ^ (r & 7)) << 4) + (kb & 15);
  uint8_t* img = reinterpret_cast<uint8_t*>(s.img_addr);
  if constexpr (MODE == IMG_BF16) {
    const __nv_bfloat16 hi = __double2bfloat16(v);
    const __nv_bfloat16 lo = __double2bfloat16(v - static_cast<double>(__bfloat162float(hi)));
    *reinterpret_cast<__nv_bfloat16*>(img + off) = hi;
    *reinterpret_cast<__nv_bfloat16*>(img + s.lo_off + off) = lo;
  } else {
    uint32_t t;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(static_cast<float>(v)));
    *reinterpret_cast<uint32_t*>(img + off) = t;
  }
}
}  // namespace

void launch_heff_fused(int mode, const DevFPair* pairs, const DevFBlock* blocks, const int32_t* term_begin,
                       const DevFTerm* terms, const DevMpoOutSlot* oslots, const DevFTile* tiles, int n_tiles,
                       int32_t* err_flag, const int32_t* skip, cudaStream_t st) {
  if (n_tiles <= 0) return;
  if (mode == IMG_TF32)
    launch_fused_impl<true>(pairs, blocks, term_begin, terms, oslots, tiles, n_tiles, err_flag, skip, st);
  else
    launch_fused_impl<false>(pairs, blocks, term_begin, terms, oslots, tiles, n_tiles, err_flag, skip, st);
}

void launch_pack_lpanels(int mode, const double* L, const DevLPanelSeg* segs, const int4* chunks, int n_chunks,
                         cudaStream_t st) {
  if (n_chunks <= 0) return;
  if (mode == IMG_TF32)
    pack_lpanel_kernel<IMG_TF32><<<n_chunks, 256, 0, st>>>(L, segs, chunks);
  else
    pack_lpanel_kernel<IMG_BF16><<<n_chunks, 256, 0, st>>>(L, segs, chunks);
}

}  // namespace tnx

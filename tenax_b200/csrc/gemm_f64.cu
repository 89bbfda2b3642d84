// Persistent grouped FP64 GEMM on the DMMA tensor-core path (mma.sync m8n8k4 f64).
//
// C_g[row, col] = sum_k A_g[row, k] * B_g[col, k] for every sector group g;
// the work list holds one entry per 64x64 output tile of every group, sorted
// by cost.  Operands come from pre-swizzled 64x16 FP64 image tiles (8 KB,
// conflict-free fragment loads); a 4-stage cp.async pipeline feeds the MMAs.
#include "common.cuh"
#include "kernels.cuh"

namespace tnx {

namespace {
constexpr int BM = 64, BN = 64, BK = 16;
constexpr int STAGES = 4;
constexpr int THREADS = 128;
constexpr int TILE_DBL = BM * BK;  // 1024 doubles = 8 KB

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(THREADS) gemm_f64_kernel(const DevGroup* __restrict__ groups,
                                                           const DevTile* __restrict__ tiles, int n_tiles,
                                                           const int64_t* __restrict__ rowoff,
                                                           const uint64_t* __restrict__ out_tab,
                                                           const int32_t* __restrict__ skip) {
  if (skip && *skip) return;
  extern __shared__ __align__(128) double smem[];
  double* As = smem;                      // [STAGES][1024]
  double* Bs = smem + STAGES * TILE_DBL;  // [STAGES][1024]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;

  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const DevTile tl = tiles[t];
    const DevGroup g = groups[tl.g];
    const int nKt = g.nKt;
    const double* a_base = reinterpret_cast<const double*>(g.a_addr) + static_cast<int64_t>(tl.mt) * nKt * TILE_DBL;
    const double* b_base = reinterpret_cast<const double*>(g.b_addr) + static_cast<int64_t>(tl.nt) * nKt * TILE_DBL;
    double* out = reinterpret_cast<double*>(out_tab[g.out_slot]);

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    auto load_stage = [&](int kt, int s) {
      // 8 KB per operand tile = 512 x 16 B; 128 threads x 4 each
      const double* ga = a_base + static_cast<int64_t>(kt) * TILE_DBL;
      const double* gb = b_base + static_cast<int64_t>(kt) * TILE_DBL;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        int c = tid + i * THREADS;  // 16-byte chunk index
        cp_async16(As + s * TILE_DBL + c * 2, ga + c * 2);
        cp_async16(Bs + s * TILE_DBL + c * 2, gb + c * 2);
      }
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < nKt) load_stage(s, s);
      cp_commit();
    }
    for (int kt = 0; kt < nKt; ++kt) {
      cp_wait<STAGES - 2>();
      __syncthreads();
      {
        int nk = kt + STAGES - 1;
        if (nk < nKt) load_stage(nk, nk % STAGES);
        cp_commit();
      }
      const double* A = As + (kt % STAGES) * TILE_DBL;
      const double* B = Bs + (kt % STAGES) * TILE_DBL;
#pragma unroll
      for (int k4 = 0; k4 < 4; ++k4) {
        const int kk = k4 * 4 + (lane & 3);
        double af[4], bf[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r = wm * 32 + i * 8 + (lane >> 2);
          af[i] = A[r * 16 + (kk ^ ((r & 3) << 2))];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int r = wn * 32 + j * 8 + (lane >> 2);
          bf[j] = B[r * 16 + (kk ^ ((r & 3) << 2))];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
      }
    }
    cp_wait<0>();
    // epilogue
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = tl.mt * BM + wm * 32 + i * 8 + (lane >> 2);
      if (row >= g.M) continue;
      const int64_t ro = rowoff[g.rowoff0 + row];
      if (ro < 0) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int col = tl.nt * BN + wn * 32 + j * 8 + (lane & 3) * 2;
        if (col < g.N) out[ro + col] = acc[i][j][0] * g.scale;
        if (col + 1 < g.N) out[ro + col + 1] = acc[i][j][1] * g.scale;
      }
    }
    __syncthreads();
  }
}
}  // namespace

int device_sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 1;
}

void launch_gemm_f64(const DevGroup* groups, const DevTile* tiles, int n_tiles, const int64_t* rowoff,
                     const uint64_t* out_tab, const int32_t* skip, cudaStream_t st) {
  if (n_tiles <= 0) return;
  const int smem = 2 * STAGES * TILE_DBL * static_cast<int>(sizeof(double));
  // set on every launch: the attribute belongs to the current device, and one
  // process may drive several.  A failure is the thread's last CUDA error,
  // which every caller checks after its launches.
  if (cudaFuncSetAttribute(gemm_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
    return;
  int grid = device_sm_count() * 3;
  if (grid > n_tiles) grid = n_tiles;
  gemm_f64_kernel<<<grid, THREADS, smem, st>>>(groups, tiles, n_tiles, rowoff, out_tab, skip);
}

}  // namespace tnx

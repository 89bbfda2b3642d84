// HBM-bound kernels: operand-image packing, result scatter, the fused MPO
// application of the two-site H_eff, and FP64 vector primitives.
#include <type_traits>

#include "common.cuh"
#include "kernels.cuh"

namespace tnx {

// ---------------------------------------------------------------------------
// image stores
// ---------------------------------------------------------------------------
__device__ __forceinline__ void img_store(int mode, uint8_t* img, int64_t lo_offset, int64_t tile0, int nKt,
                                          int64_t row, int64_t k, double v) {
  int64_t off = img_byte_offset(mode, tile0, nKt, row, k);
  if (mode == IMG_F64) {
    *reinterpret_cast<double*>(img + off) = v;
  } else if (mode == IMG_BF16) {
    __nv_bfloat16 hi = __double2bfloat16(v);
    __nv_bfloat16 lo = __double2bfloat16(v - static_cast<double>(__bfloat162float(hi)));
    *reinterpret_cast<__nv_bfloat16*>(img + off) = hi;
    *reinterpret_cast<__nv_bfloat16*>(img + lo_offset + off) = lo;
  } else {
    float f = static_cast<float>(v);
    uint32_t t;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(f));
    *reinterpret_cast<uint32_t*>(img + off) = t;
  }
}

// ---------------------------------------------------------------------------
// pack: operand blocks -> group operand images
// ---------------------------------------------------------------------------
__global__ void pack_image_kernel(const uint64_t* __restrict__ src_tab, const DevPackSeg* __restrict__ segs,
                                  const DevChunk* __restrict__ chunks, int mode, const int32_t* __restrict__ skip) {
  if (skip && *skip) return;
  const DevChunk ch = chunks[blockIdx.x];
  const DevPackSeg& s = segs[ch.seg];
  const double* src = reinterpret_cast<const double*>(src_tab[s.src_slot]) + s.src_off;
  uint8_t* img = reinterpret_cast<uint8_t*>(s.img_addr);
  // walk the block in destination order (k fastest) so consecutive threads
  // write consecutive k of one image row; the strided source reads hit cache
  for (int64_t e = ch.start + threadIdx.x; e < ch.start + ch.count; e += blockDim.x) {
    const int64_t kl = e % s.kcount, rl = e / s.kcount;
    int64_t src_off = 0, stride = 1, kd = 0;
    for (int l = s.nlegs - 1; l >= 0; --l) {
      const int64_t d = s.dims[l];
      int64_t idx = 0;
      if (s.rstr[l]) {
        idx = (rl / s.rstr[l]) % d;
      } else if (s.kstr[l]) {
        idx = (kl / s.kstr[l]) % d;
        kd += idx * s.kdstr[l];  // image K coordinate (padded strides)
      }
      src_off += idx * stride;
      stride *= d;
    }
    img_store(mode, img, s.lo_off, 0, s.nKt, s.row0 + rl, s.k0 + kd, src[src_off] * s.scale);
  }
}

void launch_pack(const uint64_t* src_tab, const DevPackSeg* segs, const DevChunk* chunks, int n_chunks, int mode,
                 const int32_t* skip, cudaStream_t st) {
  if (n_chunks <= 0) return;
  pack_image_kernel<<<n_chunks, 256, 0, st>>>(src_tab, segs, chunks, mode, skip);
}

// ---------------------------------------------------------------------------
// scatter: group result matrices -> output blocks (any leg permutation)
// ---------------------------------------------------------------------------
template <typename TS>
__global__ void scatter_kernel(const TS* __restrict__ res, double* __restrict__ out,
                               const DevScatSeg* __restrict__ segs, const DevChunk* __restrict__ chunks) {
  const DevChunk ch = chunks[blockIdx.x];
  const DevScatSeg& s = segs[ch.seg];
  for (int64_t e = ch.start + threadIdx.x; e < ch.start + ch.count; e += blockDim.x) {
    int64_t rem = e, row = 0, col = 0;
    for (int l = s.nlegs - 1; l >= 0; --l) {
      int64_t d = s.dims[l];
      int64_t idx = rem % d;
      rem /= d;
      row += idx * s.rstr[l];
      col += idx * s.cstr[l];
    }
    const double v = static_cast<double>(res[s.src_base + row * s.ld + col]);
    out[s.dst_off + e] = s.neg ? -v : v;
  }
}

void launch_scatter(const void* res, bool res_f32, double* out, const DevScatSeg* segs, const DevChunk* chunks,
                    int n_chunks, cudaStream_t st) {
  if (n_chunks <= 0) return;
  if (res_f32)
    scatter_kernel<float><<<n_chunks, 256, 0, st>>>(static_cast<const float*>(res), out, segs, chunks);
  else
    scatter_kernel<double><<<n_chunks, 256, 0, st>>>(static_cast<const double*>(res), out, segs, chunks);
}

// ---------------------------------------------------------------------------
// strided block copy (leg fusion): reads in source order, writes permuted
// ---------------------------------------------------------------------------
__global__ void strided_copy_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                    const DevCopySeg* __restrict__ segs, const DevChunk* __restrict__ chunks) {
  const DevChunk ch = chunks[blockIdx.x];
  const DevCopySeg& s = segs[ch.seg];
  for (int64_t e = ch.start + threadIdx.x; e < ch.start + ch.count; e += blockDim.x) {
    int64_t rem = e, off = 0;
    for (int l = s.nlegs - 1; l >= 0; --l) {
      const int64_t d = s.dims[l];
      off += (rem % d) * s.dstr[l];
      rem /= d;
    }
    dst[s.dst_off + off] = src[s.src_off + e];
  }
}

void launch_strided_copy(const double* src, double* dst, const DevCopySeg* segs, const DevChunk* chunks, int n_chunks,
                         cudaStream_t st) {
  if (n_chunks <= 0) return;
  strided_copy_kernel<<<n_chunks, 256, 0, st>>>(src, dst, segs, chunks);
}

// ---------------------------------------------------------------------------
// zero fill of output ranges addressed through a pointer table
// ---------------------------------------------------------------------------
__global__ void zero_ranges_kernel(const uint64_t* __restrict__ out_tab, const DevChunk* __restrict__ chunks,
                                   const int32_t* __restrict__ skip) {
  if (skip && *skip) return;
  const DevChunk ch = chunks[blockIdx.x];  // seg = pointer slot, start = element offset
  double* out = reinterpret_cast<double*>(out_tab[ch.seg]) + ch.start;
  for (int64_t e = threadIdx.x; e < ch.count; e += blockDim.x) out[e] = 0.0;
}

void launch_zero_ranges(const uint64_t* out_tab, const DevChunk* chunks, int n_chunks, const int32_t* skip,
                        cudaStream_t st) {
  if (n_chunks <= 0) return;
  zero_ranges_kernel<<<n_chunks, 256, 0, st>>>(out_tab, chunks, skip);
}

// ---------------------------------------------------------------------------
// fused MPO application (stages 2+3 of the two-site H_eff):
//   X3[c,s,t,f,d] = sum_{b,p,q} Wlr[b,p,q,s,t,f] X1[b,c,p,q,d],  Wlr = W_l W_r over e
// Wlr is very sparse (an MPO is mostly pass-through states), so each output
// slot (s,t,f) is a short sum of scaled input slots (b,p,q): the kernel walks
// the pair's terms, sorted by output slot and staged in shared memory with the
// input- and output-slot tables.  Mixed paths (FP32 stage-1 results): one
// thread owns kMpoVec consecutive d of one point row c; the stage-1 N layout
// and the stage-4 K layout both pad every d range to a multiple of kMpoVec, so
// the thread reads each term's 8 values with two aligned 16-byte loads and its
// outputs of one slot form one aligned K chunk -- a single 16-byte swizzle
// unit of a BF16 image row (two for TF32) -- and the table reads and image
// addressing are paid once per chunk instead of once per element.  kMpoTerms
// terms' loads are kept in flight per thread.  FP64 uses the per-point kernel.
// ---------------------------------------------------------------------------
constexpr int kMpoThreads = 256;
constexpr int kMpoTerms = 4;

template <int MODE>
__global__ void __launch_bounds__(kMpoThreads) mpo_apply_kernel(
    const DevMpoPair* __restrict__ pairs, const DevMpoSlot* __restrict__ islots,
    const DevMpoOutSlot* __restrict__ oslots, const DevMpoTerm* __restrict__ terms,
    const int2* __restrict__ chunks, const int32_t* __restrict__ skip) {
  // FP32 stage-1 results: every input slot's d range starts on a 32-byte
  // boundary and is padded to a multiple of kMpoVec with zero columns (the
  // planner's N padding), so a thread's 8 d of one term are two aligned
  // 16-byte loads and need no bounds mask
  if (skip && *skip) return;
  extern __shared__ __align__(16) unsigned char mpo_smem[];
  const int2 ch = chunks[blockIdx.x];
  const DevMpoPair pr = pairs[ch.x];
  DevMpoTerm* st = reinterpret_cast<DevMpoTerm*>(mpo_smem);
  DevMpoSlot* si = reinterpret_cast<DevMpoSlot*>(st + pr.n_terms);
  DevMpoOutSlot* so = reinterpret_cast<DevMpoOutSlot*>(si + pr.n_in_slots);
  for (int i = threadIdx.x; i < pr.n_terms; i += blockDim.x) st[i] = terms[pr.term0 + i];
  for (int i = threadIdx.x; i < pr.n_in_slots; i += blockDim.x) si[i] = islots[pr.in0 + i];
  for (int i = threadIdx.x; i < pr.n_out_slots; i += blockDim.x) so[i] = oslots[pr.out0 + i];
  __syncthreads();
  const int nchunk = (pr.md + kMpoVec - 1) / kMpoVec;
  const int p = ch.y + threadIdx.x;
  if (p >= pr.mc * nchunk || pr.n_terms == 0) return;
  const int64_t c = p / nchunk;
  const int d0 = (p - static_cast<int>(c) * nchunk) * kMpoVec;
  float acc[kMpoVec];
#pragma unroll
  for (int u = 0; u < kMpoVec; ++u) acc[u] = 0.0f;
  int cur = st[0].out_slot;
  for (int t0 = 0; t0 < pr.n_terms; t0 += kMpoTerms) {
    float4 xv[kMpoTerms][2];
#pragma unroll
    for (int j = 0; j < kMpoTerms; ++j) {
      if (t0 + j < pr.n_terms) {
        const DevMpoSlot sl = si[st[t0 + j].in_slot];
        const float4* src = reinterpret_cast<const float4*>(reinterpret_cast<const float*>(sl.base) + c * sl.ld + d0);
        xv[j][0] = __ldg(src);
        xv[j][1] = __ldg(src + 1);
      } else {
        xv[j][0] = xv[j][1] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
#pragma unroll
    for (int j = 0; j < kMpoTerms; ++j) {
      if (t0 + j >= pr.n_terms) break;
      const DevMpoTerm tm = st[t0 + j];
      if (tm.out_slot != cur) {
        const DevMpoOutSlot o = so[cur];
        img_store_chunk<MODE>(reinterpret_cast<uint8_t*>(o.img_addr), o.lo_off, o.nKt,
                              o.row0 + c * o.rows_per_c + o.row_add, o.k0 + o.k_add + d0, acc);
        cur = tm.out_slot;
#pragma unroll
        for (int u = 0; u < kMpoVec; ++u) acc[u] = 0.0f;
      }
      const float w = static_cast<float>(tm.w);
      acc[0] += w * xv[j][0].x;
      acc[1] += w * xv[j][0].y;
      acc[2] += w * xv[j][0].z;
      acc[3] += w * xv[j][0].w;
      acc[4] += w * xv[j][1].x;
      acc[5] += w * xv[j][1].y;
      acc[6] += w * xv[j][1].z;
      acc[7] += w * xv[j][1].w;
    }
  }
  const DevMpoOutSlot o = so[cur];
  img_store_chunk<MODE>(reinterpret_cast<uint8_t*>(o.img_addr), o.lo_off, o.nKt,
                        o.row0 + c * o.rows_per_c + o.row_add, o.k0 + o.k_add + d0, acc);
}

// FP64 images: one thread per point (c, d) writes single doubles.  An
// 8-wide chunk of doubles per thread holds too many registers to beat this
// (3.78 vs 3.17 ms on the 64-problem batch); the padded K layout is the same.
__global__ void __launch_bounds__(kMpoThreads) mpo_apply_point_kernel(
    const DevMpoPair* __restrict__ pairs, const DevMpoSlot* __restrict__ islots,
    const DevMpoOutSlot* __restrict__ oslots, const DevMpoTerm* __restrict__ terms,
    const int2* __restrict__ chunks, const int32_t* __restrict__ skip) {
  constexpr int kLoads = 8;
  if (skip && *skip) return;
  extern __shared__ __align__(16) unsigned char mpo_smem[];
  const int2 ch = chunks[blockIdx.x];
  const DevMpoPair pr = pairs[ch.x];
  DevMpoTerm* st = reinterpret_cast<DevMpoTerm*>(mpo_smem);
  DevMpoSlot* si = reinterpret_cast<DevMpoSlot*>(st + pr.n_terms);
  DevMpoOutSlot* so = reinterpret_cast<DevMpoOutSlot*>(si + pr.n_in_slots);
  for (int i = threadIdx.x; i < pr.n_terms; i += blockDim.x) st[i] = terms[pr.term0 + i];
  for (int i = threadIdx.x; i < pr.n_in_slots; i += blockDim.x) si[i] = islots[pr.in0 + i];
  for (int i = threadIdx.x; i < pr.n_out_slots; i += blockDim.x) so[i] = oslots[pr.out0 + i];
  __syncthreads();
  const int p = ch.y + threadIdx.x;
  if (p >= pr.mc * pr.md || pr.n_terms == 0) return;
  const int64_t c = p / pr.md;
  const int d = p - static_cast<int>(c) * pr.md;
  double acc = 0.0;
  int cur = st[0].out_slot;
  for (int t0 = 0; t0 < pr.n_terms; t0 += kLoads) {
    double xv[kLoads];
#pragma unroll
    for (int u = 0; u < kLoads; ++u) {
      xv[u] = 0.0;
      if (t0 + u < pr.n_terms) {
        const DevMpoSlot sl = si[st[t0 + u].in_slot];
        xv[u] = reinterpret_cast<const double*>(sl.base)[c * sl.ld + d];
      }
    }
#pragma unroll
    for (int u = 0; u < kLoads; ++u) {
      if (t0 + u >= pr.n_terms) break;
      const DevMpoTerm tm = st[t0 + u];
      if (tm.out_slot != cur) {
        const DevMpoOutSlot o = so[cur];
        *reinterpret_cast<double*>(reinterpret_cast<uint8_t*>(o.img_addr) +
                                   img_byte_offset(IMG_F64, 0, o.nKt, o.row0 + c * o.rows_per_c + o.row_add,
                                                   o.k0 + o.k_add + d)) = acc;
        cur = tm.out_slot;
        acc = 0.0;
      }
      acc += tm.w * xv[u];
    }
  }
  const DevMpoOutSlot o = so[cur];
  *reinterpret_cast<double*>(reinterpret_cast<uint8_t*>(o.img_addr) +
                             img_byte_offset(IMG_F64, 0, o.nKt, o.row0 + c * o.rows_per_c + o.row_add,
                                             o.k0 + o.k_add + d)) = acc;
}

// ---------------------------------------------------------------------------
// row pack: k-major blocks with contiguous rows (theta of the H_eff stage 1)
// -> operand image, 8 consecutive k per thread and store (see DevRowPackSeg)
// ---------------------------------------------------------------------------
// rows per CTA: small theta slices (a few rows of d) leave fewer threads idle than 256
constexpr int kPackRows = 128;

template <int MODE>
__global__ void __launch_bounds__(kPackRows) pack_rows_kernel(const uint64_t* __restrict__ src_tab,
                                                        const DevRowPackSeg* __restrict__ segs,
                                                        const int4* __restrict__ chunks,
                                                        const int32_t* __restrict__ skip) {
  using ValT = typename std::conditional<MODE == IMG_F64, double, float>::type;
  constexpr int kChunks = 4;  // K chunks of 8 per thread, all loads issued before the stores
  if (skip && *skip) return;
  const int4 ch = chunks[blockIdx.x];  // (segment, first row, first K chunk, -)
  const DevRowPackSeg s = segs[ch.x];
  const int r = ch.y + static_cast<int>(threadIdx.x);
  // BF16 / TF32 CTAs all reach the shared-memory exchange below: a row past
  // the segment loads zeros and is not stored
  if (MODE == IMG_F64 && r >= s.rows) return;
  const int rr = r < s.rows ? r : s.rows - 1;
  const double* src = reinterpret_cast<const double*>(src_tab[s.src_slot]) + s.src_off + rr;
  uint8_t* img = reinterpret_cast<uint8_t*>(s.img_addr);
  const int nkc = (s.kval + kMpoVec - 1) / kMpoVec;
  ValT v[kChunks][kMpoVec];
#pragma unroll
  for (int j = 0; j < kChunks; ++j)
#pragma unroll
    for (int u = 0; u < kMpoVec; ++u) {
      const int a = (ch.z + j) * kMpoVec + u;
      v[j][u] = (a < s.kval && r < s.rows) ? static_cast<ValT>(src[static_cast<int64_t>(a) * s.kstride] * s.scale)
                                           : ValT(0);
    }
  if constexpr (MODE == IMG_F64) {
#pragma unroll
    for (int j = 0; j < kChunks; ++j)
      if (ch.z + j < nkc) img_store_chunk<MODE>(img, s.lo_off, s.nKt, s.row0 + r, s.k0 + (ch.z + j) * kMpoVec, v[j]);
  } else {
    // BF16 / TF32: each row's 4 chunks in their image form go through shared
    // memory, so that the four lanes of a quad then write one row's 64 bytes
    // (of each plane) and a store instruction fills whole sectors of 8 rows
    __shared__ uint4 sh[kPackRows * 9];  // per row: 4 chunks x (hi or first unit, lo or second unit), pitch 9
#pragma unroll
    for (int j = 0; j < kChunks; ++j) {
      uint32_t a[4], b[4];
      if constexpr (MODE == IMG_BF16) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const __nv_bfloat162 h = __floats2bfloat162_rn(v[j][2 * u], v[j][2 * u + 1]);
          const __nv_bfloat162 l =
              __floats2bfloat162_rn(v[j][2 * u] - __low2float(h), v[j][2 * u + 1] - __high2float(h));
          a[u] = *reinterpret_cast<const uint32_t*>(&h);
          b[u] = *reinterpret_cast<const uint32_t*>(&l);
        }
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(a[u]) : "f"(v[j][u]));
          asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b[u]) : "f"(v[j][4 + u]));
        }
      }
      sh[threadIdx.x * 9 + 2 * j] = make_uint4(a[0], a[1], a[2], a[3]);
      sh[threadIdx.x * 9 + 2 * j + 1] = make_uint4(b[0], b[1], b[2], b[3]);
    }
    __syncthreads();
    const int j = threadIdx.x & 3;  // this thread's chunk
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int rl = (threadIdx.x >> 2) + (kPackRows / 4) * i;  // row within the CTA's kPackRows
      if (ch.y + rl >= s.rows || ch.z + j >= nkc) continue;
      const int64_t row = s.row0 + ch.y + rl;
      const int64_t k = s.k0 + (ch.z + j) * kMpoVec;
      const uint4 x0 = sh[rl * 9 + 2 * j], x1 = sh[rl * 9 + 2 * j + 1];
      if constexpr (MODE == IMG_BF16) {
        const int64_t off = img_byte_offset(MODE, 0, s.nKt, row, k);
        *reinterpret_cast<uint4*>(img + off) = x0;
        *reinterpret_cast<uint4*>(img + s.lo_off + off) = x1;
      } else {
        *reinterpret_cast<uint4*>(img + img_byte_offset(MODE, 0, s.nKt, row, k)) = x0;
        *reinterpret_cast<uint4*>(img + img_byte_offset(MODE, 0, s.nKt, row, k + 4)) = x1;
      }
    }
  }
}

void launch_pack_rows(const uint64_t* src_tab, const DevRowPackSeg* segs, const int4* chunks, int n_chunks, int mode,
                      const int32_t* skip, cudaStream_t st) {
  if (n_chunks <= 0) return;
  if (mode == IMG_F64)
    pack_rows_kernel<IMG_F64><<<n_chunks, kPackRows, 0, st>>>(src_tab, segs, chunks, skip);
  else if (mode == IMG_BF16)
    pack_rows_kernel<IMG_BF16><<<n_chunks, kPackRows, 0, st>>>(src_tab, segs, chunks, skip);
  else
    pack_rows_kernel<IMG_TF32><<<n_chunks, kPackRows, 0, st>>>(src_tab, segs, chunks, skip);
}

void launch_mpo_apply(bool x1_f32, int mode, const DevMpoPair* pairs, const DevMpoSlot* islots,
                      const DevMpoOutSlot* oslots, const DevMpoTerm* terms, const int2* chunks, int n_chunks,
                      size_t smem_bytes, const int32_t* skip, cudaStream_t st) {
  if (n_chunks <= 0) return;
  const int smem = static_cast<int>(smem_bytes);
  auto go = [&](auto kernel) {
    // a failure here is the thread's last CUDA error, checked by every caller
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return;
    kernel<<<n_chunks, kMpoThreads, smem, st>>>(pairs, islots, oslots, terms, chunks, skip);
  };
  if (!x1_f32)
    go(mpo_apply_point_kernel);
  else if (mode == IMG_BF16)
    go(mpo_apply_kernel<IMG_BF16>);
  else
    go(mpo_apply_kernel<IMG_TF32>);
}

int mpo_points_per_cta() { return kMpoThreads; }
int pack_rows_per_cta() { return kPackRows; }

int pack_rows_chunks_per_thread() { return 4; }
int mpo_d_per_thread(int mode) { return mode == IMG_F64 ? 1 : kMpoVec; }

// ---------------------------------------------------------------------------
// FP64 vector primitives: deterministic two-pass reductions
// ---------------------------------------------------------------------------
constexpr int kRedBlocks = 592;  // 4 x 148 SMs
constexpr int kRedThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[32];
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) ws[w] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? ws[threadIdx.x] : 0.0;
  if (w == 0) v = warp_sum(v);
  return v;
}

// kind 0: sum x*y; kind 1: sum x*x
__global__ void partial_dot_kernel(const double* __restrict__ x, const double* __restrict__ y, int64_t n, int kind,
                                   double* __restrict__ partials, const int32_t* __restrict__ skip) {
  if (skip && *skip) return;
  double acc = 0.0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t n2 = n / 2;
  const double2* x2 = reinterpret_cast<const double2*>(x);
  const double2* y2 = reinterpret_cast<const double2*>(y);
  bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
  if (aligned) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n2; i += stride) {
      double2 a = x2[i];
      double2 b = kind ? a : y2[i];
      acc += a.x * b.x + a.y * b.y;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (n & 1)) acc += x[n - 1] * (kind ? x[n - 1] : y[n - 1]);
  } else {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
      acc += x[i] * (kind ? x[i] : y[i]);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double block_max(double v) {
  __shared__ double wm[32];
  v = warp_max(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) wm[w] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? wm[threadIdx.x] : 0.0;
  if (w == 0) v = warp_max(v);
  return v;
}

// max |x| in two passes (partials, then one block)
__global__ void partial_maxabs_kernel(const double* __restrict__ x, int64_t n, double* __restrict__ partials) {
  double m = 0.0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
    m = fmax(m, fabs(x[i]));
  m = block_max(m);
  if (threadIdx.x == 0) partials[blockIdx.x] = m;
}

__global__ void finish_max_kernel(const double* __restrict__ partials, int np, double* __restrict__ result) {
  double m = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) m = fmax(m, partials[i]);
  m = block_max(m);
  if (threadIdx.x == 0) *result = m;
}

// ---------------------------------------------------------------------------
// bounded wait on a device flag: the same deadline discipline as the GEMMs'
// mbarrier waits (%globaltimer, plus an iteration cap), reporting through a
// status word instead of hanging
// ---------------------------------------------------------------------------
__global__ void wait_flag_kernel(const volatile int32_t* flag, int32_t expected, uint64_t timeout_ns,
                                 int32_t* status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint64_t t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (uint32_t it = 0; it < (1u << 26); ++it) {
    if (*flag == expected) {
      *status = 0;
      return;
    }
    if ((it & 63u) == 63u) {
      uint64_t now;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
      if (now - t0 > timeout_ns) break;
    }
  }
  *status = 5;  // TNX_ERR_TIMEOUT
}

void launch_wait_flag(const int32_t* flag, int32_t expected, uint64_t timeout_ns, int32_t* status, cudaStream_t st) {
  wait_flag_kernel<<<1, 32, 0, st>>>(flag, expected, timeout_ns, status);
}

void launch_maxabs(const double* x, int64_t n, double* result, double* partials, cudaStream_t st) {
  partial_maxabs_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(x, n, partials);
  finish_max_kernel<<<1, 1024, 0, st>>>(partials, kRedBlocks, result);
}

// final: result = sum partials (op 0), sqrt(sum) (op 1)
__global__ void finish_sum_kernel(const double* __restrict__ partials, int np, double* __restrict__ result, int op,
                                  const int32_t* __restrict__ skip) {
  if (skip && *skip) return;
  double acc = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partials[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) *result = op == 1 ? sqrt(acc) : acc;
}

void launch_dot(const double* x, const double* y, int64_t n, int kind, double* result, double* partials,
                const int32_t* skip, cudaStream_t st) {
  partial_dot_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(x, y, n, kind, partials, skip);
  finish_sum_kernel<<<1, 1024, 0, st>>>(partials, kRedBlocks, result, kind, skip);
}

// w -= alpha v (+ beta v_prev); partial sums of w*w
__global__ void lanczos_axpy_kernel(double* __restrict__ w, const double* __restrict__ v,
                                    const double* __restrict__ vp, int64_t n, const double* __restrict__ alpha,
                                    const double* __restrict__ beta, double* __restrict__ partials,
                                    const int32_t* __restrict__ skip) {
  if (skip && *skip) return;
  const double a = *alpha;
  const double b = vp ? *beta : 0.0;
  double acc = 0.0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    double x = w[i] - v[i] * a;
    if (vp) x = x - vp[i] * b;
    w[i] = x;
    acc += x * x;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// beta = ||w||; stop when beta < tol (the reference's absolute test) or, with
// an inexact matvec, when beta < tol_rel * |alpha| (below the matvec's noise)
__global__ void lanczos_beta_kernel(const double* __restrict__ partials, int np, double* __restrict__ beta_out,
                                    const double* __restrict__ alpha, double tol, double tol_rel,
                                    int32_t* __restrict__ done) {
  if (*done) return;
  double acc = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partials[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) {
    double b = sqrt(acc);
    *beta_out = b;
    if (b < tol || b < tol_rel * fabs(*alpha)) *done = 1;
  }
}

__global__ void scale_into_kernel(const double* __restrict__ w, double* __restrict__ out, int64_t n,
                                  const double* __restrict__ s, int mode, const int32_t* __restrict__ skip) {
  if (skip && *skip) return;
  // mode 0: out = w * s; mode 1: out = w / s; mode 2: out = w * (1 / (s + 1e-15))
  double f = *s;
  if (mode == 2) f = 1.0 / (f + 1e-15);
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
    out[i] = mode == 1 ? w[i] * (1.0 / f) : w[i] * f;
}

void launch_lanczos_step(double* w, const double* v, const double* vp, double* vnext, int64_t n, double* alpha,
                         double* beta_next, const double* beta_prev, double tol, double tol_rel, int32_t* done,
                         double* partials, cudaStream_t st) {
  // alpha = <v, w>
  partial_dot_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(v, w, n, 0, partials, done);
  finish_sum_kernel<<<1, 1024, 0, st>>>(partials, kRedBlocks, alpha, 0, done);
  lanczos_axpy_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(w, v, vp, n, alpha, beta_prev, partials, done);
  lanczos_beta_kernel<<<1, 1024, 0, st>>>(partials, kRedBlocks, beta_next, alpha, tol, tol_rel, done);
  if (vnext) scale_into_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(w, vnext, n, beta_next, 1, done);
}

void launch_scale(const double* w, double* out, int64_t n, const double* s, int mode, const int32_t* skip,
                  cudaStream_t st) {
  scale_into_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(w, out, n, s, mode, skip);
}

__global__ void combine_kernel(const double* const* __restrict__ basis, const double* __restrict__ coefs, int nv,
                               int64_t n, double* __restrict__ out) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    // same association as the reference: ((b0 c0 + b1 c1) + b2 c2) + ...
    double acc = basis[0][i] * coefs[0];
    for (int k = 1; k < nv; ++k) acc = acc + basis[k][i] * coefs[k];
    out[i] = acc;
  }
}

void launch_combine(const double* const* basis, const double* coefs, int nv, int64_t n, double* out,
                    cudaStream_t st) {
  combine_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(basis, coefs, nv, n, out);
}

int reduce_partials_count() { return kRedBlocks; }

// ---------------------------------------------------------------------------
// Max-abs renormalisation of a batch of tensors and its adjoint.
// Forward: y_t = x_t / (m_t + eps), m_t = max |x_t|.
// Adjoint: gx_t = gy_t / (m_t + eps) - <gy_t, x_t> / (m_t + eps)^2 * dm_t/dx_t,
// where dm/dx puts sign(x_i) / c on each of the c entries with |x_i| == m.
// Grid (kRenormBlocks, n_tensors); each tensor's reduction is a fixed-order
// two-pass sum, so results do not depend on scheduling.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t renorm_stride() { return static_cast<int64_t>(kRenormBlocks) * blockDim.x; }

__global__ void renorm_max_partial_kernel(RenormArgs a, double* __restrict__ partials) {
  const int t = blockIdx.y;
  const double* __restrict__ x = a.x[t];
  const int64_t n = a.n[t];
  double m = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += renorm_stride())
    m = fmax(m, fabs(x[i]));
  m = block_max(m);
  if (threadIdx.x == 0) partials[t * kRenormBlocks + blockIdx.x] = m;
}

// per-tensor total of kRenormBlocks partials in a fixed order (warp 0), broadcast via smem
__device__ __forceinline__ double renorm_total(const double* __restrict__ p, bool is_max) {
  __shared__ double tot;
  if (threadIdx.x < 32) {
    double v0 = p[threadIdx.x], v1 = p[threadIdx.x + 32];
    double v = is_max ? fmax(v0, v1) : v0 + v1;
    v = is_max ? warp_max(v) : warp_sum(v);
    if (threadIdx.x == 0) tot = v;
  }
  __syncthreads();
  const double r = tot;
  __syncthreads();
  return r;
}

__global__ void renorm_apply_kernel(RenormArgs a, const double* __restrict__ partials, double eps,
                                    double* __restrict__ stat) {
  const int t = blockIdx.y;
  const double m = renorm_total(partials + t * kRenormBlocks, true);
  if (blockIdx.x == 0 && threadIdx.x == 0) stat[t] = m;
  const double den = m + eps;  // a true division per element, as x / (max|x| + eps) is written
  const double* __restrict__ x = a.x[t];
  double* __restrict__ y = a.y[t];
  const int64_t n = a.n[t];
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += renorm_stride())
    y[i] = x[i] / den;
}

__global__ void renorm_adj_partial_kernel(RenormArgs a, const double* __restrict__ stat,
                                          double* __restrict__ partials) {
  const int t = blockIdx.y;
  const double* __restrict__ x = a.x[t];
  const double* __restrict__ g = a.g[t];
  const int64_t n = a.n[t];
  const double m = stat[t];
  double dot = 0.0, cnt = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += renorm_stride()) {
    const double xi = x[i];
    dot += g[i] * xi;
    cnt += fabs(xi) == m ? 1.0 : 0.0;
  }
  dot = block_sum(dot);
  __syncthreads();
  cnt = block_sum(cnt);
  if (threadIdx.x == 0) {
    partials[(2 * t) * kRenormBlocks + blockIdx.x] = dot;
    partials[(2 * t + 1) * kRenormBlocks + blockIdx.x] = cnt;
  }
}

__global__ void renorm_adj_apply_kernel(RenormArgs a, const double* __restrict__ stat,
                                        const double* __restrict__ partials, double eps) {
  const int t = blockIdx.y;
  const double dot = renorm_total(partials + (2 * t) * kRenormBlocks, false);
  const double cnt = renorm_total(partials + (2 * t + 1) * kRenormBlocks, false);
  const double m = stat[t];
  const double den = m + eps;
  const double w = cnt > 0.0 ? dot / (den * den) / cnt : 0.0;
  const double* __restrict__ x = a.x[t];
  const double* __restrict__ g = a.g[t];
  double* __restrict__ gx = a.y[t];
  const int64_t n = a.n[t];
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += renorm_stride()) {
    const double xi = x[i];
    double v = g[i] / den;
    if (fabs(xi) == m && xi != 0.0) v -= xi > 0.0 ? w : -w;
    gx[i] = v;
  }
}

void launch_renorm(const RenormArgs& a, int nt, double eps, double* stat, double* partials, cudaStream_t st) {
  const dim3 grid(kRenormBlocks, nt);
  renorm_max_partial_kernel<<<grid, kRedThreads, 0, st>>>(a, partials);
  renorm_apply_kernel<<<grid, kRedThreads, 0, st>>>(a, partials, eps, stat);
}

void launch_renorm_adjoint(const RenormArgs& a, int nt, double eps, const double* stat, double* partials,
                           cudaStream_t st) {
  const dim3 grid(kRenormBlocks, nt);
  renorm_adj_partial_kernel<<<grid, kRedThreads, 0, st>>>(a, stat, partials);
  renorm_adj_apply_kernel<<<grid, kRedThreads, 0, st>>>(a, stat, partials, eps);
}

}  // namespace tnx

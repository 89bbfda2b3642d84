// Sector SVDs of the block-diagonal truncated SVD (tenax linalg.py:186-192:
// one jnp.linalg.svd(matrix, full_matrices=False) per charge sector).
//
// Large sectors run cuSOLVER's polar-decomposition SVD (Xgesvdp: QDWH polar
// factor, then a symmetric eigensolver), small ones the one-sided Jacobi SVD
// (gesvdj).  On the sector matrices of chi = 2048 DMRG two-site tensors the
// polar driver took 45 / 38 / 20 / 7.9 ms for 924 / 792 / 495 / 220 square
// sectors against 147 / 114 / 50 / 14 ms for Jacobi, but 4.0 against 2.8 ms
// at 66: its fixed cost dominates small sectors.  Both are at least as
// accurate as LAPACK's in the singular values.  Xgesvdp returns a host-side
// error estimate, so every call blocks its host thread until the
// decomposition has finished: sectors are therefore spread over worker
// threads, each with its own stream and cuSOLVER handle, so that the
// decompositions overlap.
//
// cuSOLVER is column-major and the sector matrices are row-major.  A
// row-major m x k buffer read column-major is the k x m transpose, so for
// k > m the buffer is decomposed as the tall matrix B = A^T = U_B S V_B^T:
// U_B (k x m, column-major) is already Vh in row-major order, and U = V_B is
// transposed.  For k <= m the input is first transposed into a column-major
// m x k copy C = A = U_C S V_C^T: V_C (k x k, column-major) is Vh in row-major
// order, and U = U_C is transposed.
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tenax_b200.h"
#include "planner.hpp"
#include "svd.hpp"

namespace tnx {
namespace {

// out (rows x cols, row-major) = in (rows x cols, column-major, leading dimension rows)
__global__ void transpose_cm_to_rm(const double* __restrict__ in, double* __restrict__ out, int64_t rows, int64_t cols) {
  __shared__ double tile[32][33];
  const int64_t r0 = static_cast<int64_t>(blockIdx.y) * 32, c0 = static_cast<int64_t>(blockIdx.x) * 32;
  for (int j = threadIdx.y; j < 32; j += 8) {
    const int64_t r = r0 + threadIdx.x, c = c0 + j;
    if (r < rows && c < cols) tile[j][threadIdx.x] = in[r + c * rows];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += 8) {
    const int64_t r = r0 + j, c = c0 + threadIdx.x;
    if (r < rows && c < cols) out[r * cols + c] = tile[threadIdx.x][j];
  }
}

void transpose(const double* in, double* out, int64_t rows, int64_t cols, cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return;
  const dim3 grid(static_cast<unsigned>((cols + 31) / 32), static_cast<unsigned>((rows + 31) / 32));
  if (grid.y > 65535u) throw PlanError{TNX_ERR_UNSUPPORTED, "sector matrix too tall for the transpose grid"};
  transpose_cm_to_rm<<<grid, dim3(32, 8), 0, st>>>(in, out, rows, cols);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw PlanError{TNX_ERR_CUDA, std::string("transpose launch: ") + cudaGetErrorString(e)};
}

#define SVD_CUDA(x)                                                                                   \
  do {                                                                                                \
    cudaError_t _e = (x);                                                                             \
    if (_e != cudaSuccess) throw PlanError{TNX_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)}; \
  } while (0)
#define SVD_SOLVER(x)                                                                                  \
  do {                                                                                                 \
    cusolverStatus_t _s = (x);                                                                         \
    if (_s != CUSOLVER_STATUS_SUCCESS)                                                                 \
      throw PlanError{TNX_ERR_RUNTIME, std::string(#x) + ": cuSOLVER status " + std::to_string(static_cast<int>(_s))}; \
  } while (0)

// Grow-only device buffer owned by one worker.
struct Scratch {
  void* p = nullptr;
  size_t n = 0;
  void* need(size_t bytes) {
    if (bytes > n) {
      if (p) SVD_CUDA(cudaFree(p));
      p = nullptr;
      n = 0;
      SVD_CUDA(cudaMalloc(&p, bytes));
      n = bytes;
    }
    return p;
  }
};

struct Worker {
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  cusolverDnHandle_t h = nullptr;
  cusolverDnParams_t prm = nullptr;
  gesvdjInfo_t jac = nullptr;
  Scratch ws, tall, utmp, info;
  std::vector<char> host_ws;

  // the first worker receives the largest sector (longest-first assignment)
  // and gets the highest stream priority: its decomposition is the batch's
  // critical path (8-worker batch of chi = 2048 sector shapes: 64-65 ms
  // against 66-68 ms at equal priorities; the largest sector alone 42 ms)
  void init(bool high) {
    int least = 0, greatest = 0;
    SVD_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    SVD_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, high ? greatest : least));
    SVD_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    SVD_SOLVER(cusolverDnCreate(&h));
    SVD_SOLVER(cusolverDnSetStream(h, st));
    SVD_SOLVER(cusolverDnCreateParams(&prm));
    SVD_SOLVER(cusolverDnCreateGesvdjInfo(&jac));  // default: tolerance = machine epsilon, sorted output
  }

  // one sector: a (m x k row-major) -> u (m x r), s (r), vh (r x k), r = min(m, k)
  double run(const SvdJob& j, bool polar, int* d_info) {
    // the row-major buffer read column-major is A^T: tall when k > m; square
    // matrices take the transposed copy, so the solver sees A itself
    const bool wide = j.k > j.m;
    const int64_t rows = wide ? j.k : j.m, cols = wide ? j.m : j.k;  // the tall column-major matrix
    double* t = static_cast<double*>(tall.need(sizeof(double) * static_cast<size_t>(rows * cols)));
    if (wide)
      SVD_CUDA(cudaMemcpyAsync(t, j.a, sizeof(double) * static_cast<size_t>(rows * cols), cudaMemcpyDeviceToDevice, st));
    else
      transpose(j.a, t, j.k, j.m, st);  // row-major k x m view of the column-major m x k copy
    // tall = Ut S Vt^T with Ut rows x cols and Vt cols x cols (column-major)
    double* Ut = wide ? j.vh : static_cast<double*>(utmp.need(sizeof(double) * static_cast<size_t>(rows * cols)));
    double* Vt = wide ? static_cast<double*>(utmp.need(sizeof(double) * static_cast<size_t>(cols * cols))) : j.vh;
    if (!polar) {
      int lwork = 0;
      SVD_SOLVER(cusolverDnDgesvdj_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, 1, static_cast<int>(rows), static_cast<int>(cols),
                                              t, static_cast<int>(rows), j.s, Ut, static_cast<int>(rows), Vt,
                                              static_cast<int>(cols), &lwork, jac));
      double* w = static_cast<double*>(ws.need(sizeof(double) * std::max<size_t>(static_cast<size_t>(lwork), 2)));
      SVD_SOLVER(cusolverDnDgesvdj(h, CUSOLVER_EIG_MODE_VECTOR, 1, static_cast<int>(rows), static_cast<int>(cols), t,
                                   static_cast<int>(rows), j.s, Ut, static_cast<int>(rows), Vt, static_cast<int>(cols), w,
                                   lwork, d_info, jac));
      transpose(static_cast<const double*>(utmp.p), j.u, j.m, wide ? j.m : j.k, st);
      return 0.0;
    }
    size_t dbytes = 0, hbytes = 0;
    SVD_SOLVER(cusolverDnXgesvdp_bufferSize(h, prm, CUSOLVER_EIG_MODE_VECTOR, 1, rows, cols, CUDA_R_64F, t, rows,
                                            CUDA_R_64F, j.s, CUDA_R_64F, Ut, rows, CUDA_R_64F, Vt, cols, CUDA_R_64F,
                                            &dbytes, &hbytes));
    void* dws = ws.need(std::max<size_t>(dbytes, 16));
    if (host_ws.size() < hbytes) host_ws.resize(hbytes);
    double err_sigma = 0.0;
    SVD_SOLVER(cusolverDnXgesvdp(h, prm, CUSOLVER_EIG_MODE_VECTOR, 1, rows, cols, CUDA_R_64F, t, rows, CUDA_R_64F, j.s,
                                 CUDA_R_64F, Ut, rows, CUDA_R_64F, Vt, cols, CUDA_R_64F, dws, dbytes,
                                 hbytes ? host_ws.data() : nullptr, hbytes, d_info, &err_sigma));
    // U: wide -> V_B (m x m column-major in utmp); tall -> U_C (m x k column-major in utmp)
    transpose(static_cast<const double*>(utmp.p), j.u, j.m, wide ? j.m : j.k, st);
    return err_sigma;
  }
};

struct Pool {
  std::mutex mu;  // one batch at a time per device
  std::vector<Worker> workers;
};

std::mutex g_pools_mu;
std::map<int, Pool*> g_pools;  // per device; intentionally never destroyed (handles outlive static teardown order)

Pool& pool_for(int dev) {
  std::lock_guard<std::mutex> lk(g_pools_mu);
  Pool*& p = g_pools[dev];
  if (!p) p = new Pool();
  return *p;
}

}  // namespace

double svd_batch(const std::vector<SvdJob>& jobs, int64_t polar_min, int n_workers, cudaStream_t stream) {
  for (const SvdJob& j : jobs) {
    if (j.m < 0 || j.k < 0) throw PlanError{TNX_ERR_VALUE, "negative sector matrix extent"};
    if (j.m > INT32_MAX || j.k > INT32_MAX) throw PlanError{TNX_ERR_UNSUPPORTED, "sector matrix extent above 2^31 - 1"};
    if (j.m > 0 && j.k > 0 && (!j.a || !j.u || !j.s || !j.vh)) throw PlanError{TNX_ERR_VALUE, "null sector pointer"};
  }
  n_workers = std::max(1, std::min(n_workers, 32));
  int dev = 0;
  SVD_CUDA(cudaGetDevice(&dev));
  Pool& pool = pool_for(dev);
  std::lock_guard<std::mutex> lk(pool.mu);
  while (static_cast<int>(pool.workers.size()) < n_workers) {
    pool.workers.emplace_back();
    pool.workers.back().init(pool.workers.size() == 1);
  }
  // longest first, greedy by m*k*min(m,k)
  std::vector<int> order;
  for (int i = 0; i < static_cast<int>(jobs.size()); ++i)
    if (jobs[i].m > 0 && jobs[i].k > 0) order.push_back(i);
  auto cost = [&](int i) { return static_cast<double>(jobs[i].m) * jobs[i].k * std::min(jobs[i].m, jobs[i].k); };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
  std::vector<std::vector<int>> parts(n_workers);
  std::vector<double> load(n_workers, 0.0);
  for (int i : order) {
    const int w = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
    parts[w].push_back(i);
    load[w] += cost(i);
  }
  cudaEvent_t ready = nullptr;
  SVD_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  struct EventGuard {
    cudaEvent_t e;
    ~EventGuard() { cudaEventDestroy(e); }
  } guard{ready};
  SVD_CUDA(cudaEventRecord(ready, stream));

  std::vector<std::string> errors(n_workers);
  std::vector<int> codes(n_workers, 0);
  std::vector<double> err_sigma(n_workers, 0.0);
  auto work = [&](int w) {
    try {
      SVD_CUDA(cudaSetDevice(dev));
      Worker& wk = pool.workers[w];
      SVD_CUDA(cudaStreamWaitEvent(wk.st, ready, 0));
      const size_t nj = parts[w].size();
      int* d_info = static_cast<int*>(wk.info.need(sizeof(int) * std::max<size_t>(nj, 1)));
      SVD_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int) * std::max<size_t>(nj, 1), wk.st));
      for (size_t q = 0; q < nj; ++q) {
        const SvdJob& j = jobs[parts[w][q]];
        err_sigma[w] = std::max(err_sigma[w], wk.run(j, std::min(j.m, j.k) >= polar_min, d_info + q));
      }
      std::vector<int> info(nj);
      if (nj) SVD_CUDA(cudaMemcpyAsync(info.data(), d_info, sizeof(int) * nj, cudaMemcpyDeviceToHost, wk.st));
      SVD_CUDA(cudaEventRecord(wk.done, wk.st));
      SVD_CUDA(cudaStreamSynchronize(wk.st));
      for (size_t q = 0; q < nj; ++q)
        if (info[q] != 0)
          throw PlanError{TNX_ERR_RUNTIME, "cuSOLVER SVD reported info " + std::to_string(info[q]) + " for sector " +
                                               std::to_string(parts[w][q])};
    } catch (const PlanError& e) {
      codes[w] = e.code;
      errors[w] = e.msg;
    } catch (const std::exception& e) {
      codes[w] = TNX_ERR_RUNTIME;
      errors[w] = e.what();
    }
  };
  int used = 0;
  for (int w = 0; w < n_workers; ++w) used += parts[w].empty() ? 0 : 1;
  if (used <= 1) {
    for (int w = 0; w < n_workers; ++w)
      if (!parts[w].empty()) work(w);
  } else {
    std::vector<std::thread> threads;
    for (int w = 0; w < n_workers; ++w)
      if (!parts[w].empty()) threads.emplace_back(work, w);
    for (auto& t : threads) t.join();
  }
  for (int w = 0; w < n_workers; ++w)
    if (codes[w]) throw PlanError{codes[w], errors[w]};
  for (int w = 0; w < n_workers; ++w)
    if (!parts[w].empty()) SVD_CUDA(cudaStreamWaitEvent(stream, pool.workers[w].done, 0));
  double e = 0.0;
  for (double x : err_sigma) e = std::max(e, x);
  return e;
}

}  // namespace tnx

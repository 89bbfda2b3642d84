// Sector SVDs on the device (svd.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace tnx {

// a (m x k, row-major, preserved) = u (m x r) diag(s) vh (r x k), r = min(m, k),
// singular values descending; all device pointers.
struct SvdJob {
  int64_t m, k;
  const double* a;
  double* u;
  double* s;
  double* vh;
};

// Decomposes every job on up to n_workers worker streams ordered after
// `stream`; `stream` waits for all of them.  Jobs with min(m, k) >= polar_min
// use the polar-decomposition driver, the others Jacobi.  Blocks the calling
// host thread until the decompositions have finished.  Returns the largest
// error estimate the polar driver reported.  Throws PlanError.
double svd_batch(const std::vector<SvdJob>& jobs, int64_t polar_min, int n_workers, cudaStream_t stream);

}  // namespace tnx

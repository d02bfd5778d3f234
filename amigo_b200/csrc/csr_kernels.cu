// KKT CSR utilities on the device: diagonal add (CSRMat::add_diagonal,
// include/csr_matrix.h:508-528) and the symmetric matrix-vector product used
// by iterative refinement (amigo/algorithm/solvers/linear_solver.py:196).
#include <cuda_runtime.h>

#include "ipm_internal.h"
#include "launch_count.h"

namespace ab {
namespace {

__global__ void k_add_diagonal(int n, const int* diag_pos, const double* d,
                               double* vals) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    vals[diag_pos[i]] += d[i];
}

// One warp per row; lanes stride the row, warp-shuffle sum in a fixed order.
__global__ void k_matvec(int n, const int* __restrict__ rowp,
                         const int* __restrict__ cols,
                         const double* __restrict__ vals,
                         const double* __restrict__ x, double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n;
       r += warps) {
    double acc = 0.0;
    for (int p = rowp[r] + lane; p < rowp[r + 1]; p += 32)
      acc += vals[p] * x[cols[p]];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) y[r] = acc;
  }
}

}  // namespace

int csr_add_diagonal(int n, const int* diag_pos, const double* d,
                     double* vals, cudaStream_t st) {
  if (n <= 0) return 0;
  int g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  { k_add_diagonal<<<g, 256, 0, st>>>(n, diag_pos, d, vals); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int csr_matvec(int n, const int* rowp, const int* cols, const double* vals,
               const double* x, double* y, cudaStream_t st) {
  if (n <= 0) return 0;
  long long g = ((long long)n + 7) / 8;
  if (g > 148 * 32) g = 148 * 32;
  { k_matvec<<<(int)g, 256, 0, st>>>(n, rowp, cols, vals, x, y); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

}  // namespace ab

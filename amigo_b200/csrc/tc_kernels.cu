// Stand-alone entry to the tensor-core Schur update (tc_update.cuh) on
// plain column-major arrays, used to check the tcgen05 path against an
// FP64 product.
#include <cuda_runtime.h>

#include "../../include/amigo_b200.h"
#include "launch_count.h"
#include "tc_update.cuh"

namespace ab {
namespace {

__device__ __forceinline__ void tri_coords(int t, int& ti, int& tj) {
  int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) i++;
  while (i * (i + 1) / 2 > t) i--;
  ti = i;
  tj = t - i * (i + 1) / 2;
}

__global__ void __launch_bounds__(tc::kThreads)
k_tc_syrk(int n, int kw, const float* A, int lda, const float* B, int ldb,
          float* C, int ldc, int* status) {
  extern __shared__ __align__(1024) char smem[];
  const int nt = (n + tc::TM - 1) / tc::TM;
  const int ntiles = nt * (nt + 1) / 2;
  if ((int)blockIdx.x >= ntiles) return;
  tc::TcCta c = tc::tc_begin(smem);
  for (int t = blockIdx.x; t < ntiles && c.ok; t += gridDim.x) {
    int ti, tj;
    tri_coords(t, ti, tj);
    tc::tc_tile(c, C, ldc, A, lda, B, ldb, n, kw, ti * tc::TM, tj * tc::TN,
                status);
  }
  tc::tc_end(c);
}

}  // namespace
}  // namespace ab

extern "C" int ab_tc_syrk_tf32x3(int n, int kw, const float* A, int lda,
                                 const float* B, int ldb, float* C, int ldc,
                                 int* d_status, void* stream) {
  if (n < 0 || kw < 0 || kw > 31 || (n > 0 && (!A || !B || !C || !d_status)) ||
      lda < n || ldb < n || ldc < n)
    return AB_ERR_ARG;
  if (n == 0 || kw == 0) return AB_OK;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(ab::k_tc_syrk,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             ab::tc::kSmemBytes) != cudaSuccess)
      return AB_ERR_CUDA;
    attr = true;
  }
  const long long nt = (n + ab::tc::TM - 1) / ab::tc::TM;
  const long long ntiles = nt * (nt + 1) / 2;
  const int grid = (int)(ntiles < 3 * 148 ? ntiles : 3 * 148);
  ab::k_tc_syrk<<<grid, ab::tc::kThreads, ab::tc::kSmemBytes,
                  (cudaStream_t)stream>>>(n, kw, A, lda, B, ldb, C, ldc,
                                          d_status);
  ab::count_launch();
  return cudaGetLastError() == cudaSuccess ? AB_OK : AB_ERR_CUDA;
}

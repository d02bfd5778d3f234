// The InteriorPointOptimizer operations around the IPM vector kernels: NLP
// scaling (include/interior_point_optimizer.h:502-598), slack
// initialisation from the constraint residuals (:476-489), the dual
// residual vector (include/interior_point_backend.h:579-586) and the
// primal / multiplier gathers (interior_point_backend.h:99-121).
//
// Compiled with --fmad=false like the other IPM kernels: every product is
// evaluated in the reference's order, so the scaled values equal the
// reference's bit for bit.
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/amigo_b200.h"
#include "launch_count.h"

namespace ab {
namespace {

constexpr int ST = 256;

int grid_for(long long n) {
  long long g = (n + ST - 1) / ST;
  if (g > 148 * 8) g = 148 * 8;
  return g < 1 ? 1 : (int)g;
}

int done() { return cudaGetLastError() == cudaSuccess ? AB_OK : AB_ERR_CUDA; }

// Non-negative doubles order like their bit patterns, so an atomic max on
// the 64-bit pattern is an exact (and order-independent) maximum.
__device__ __forceinline__ void atomic_max_nonneg(double* out, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(out),
            (unsigned long long)__double_as_longlong(v));
}

__global__ void k_absmax_gather(int m, const int* __restrict__ idx,
                                const double* __restrict__ x, double* out) {
  double v = 0.0;
  for (int j = blockIdx.x * ST + threadIdx.x; j < m; j += gridDim.x * ST) {
    const double a = fabs(x[idx[j]]);
    if (a > v) v = a;
  }
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0 && v > 0.0) atomic_max_nonneg(out, v);
}

// One warp per selected row: the largest |value| of the row.
__global__ void k_rows_absmax(int m, const int* __restrict__ rows,
                              const int* __restrict__ rowp,
                              const double* __restrict__ vals, double* out) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (ST / 32);
  for (int j = blockIdx.x * (ST / 32) + (threadIdx.x >> 5); j < m; j += warps) {
    const int r = rows[j];
    double v = 0.0;
    for (int p = rowp[r] + lane; p < rowp[r + 1]; p += 32) {
      const double a = fabs(vals[p]);
      if (a > v) v = a;
    }
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) out[j] = v;
  }
}

// dc = min(1, max_gradient / rowmax) floored at min_value; lbh *= dc where
// dc != 1; scale[cidx[j]] = dc (1 elsewhere, set by the caller).
__global__ void k_constraint_scale(int m, const int* __restrict__ cidx,
                                   double max_gradient, double min_value,
                                   double* rowmax_dc, double* lbh,
                                   double* scale) {
  for (int j = blockIdx.x * ST + threadIdx.x; j < m; j += gridDim.x * ST) {
    const double rm = rowmax_dc[j];
    double dc = (rm > max_gradient) ? max_gradient / rm : 1.0;
    if (dc < min_value) dc = min_value;
    rowmax_dc[j] = dc;
    if (dc != 1.0) lbh[j] *= dc;
    scale[cidx[j]] = dc;
  }
}

__global__ void k_fill(long long n, double v, double* x) {
  for (long long i = (long long)blockIdx.x * ST + threadIdx.x; i < n;
       i += (long long)gridDim.x * ST)
    x[i] = v;
}

// vals[k] *= s[i] * s[cols[k]] over the rows of a CSR matrix: D H D.
__global__ void k_scale_symmetric(int n, const int* __restrict__ rowp,
                                  const int* __restrict__ cols,
                                  const double* __restrict__ s, double* vals) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (ST / 32);
  for (int r = blockIdx.x * (ST / 32) + (threadIdx.x >> 5); r < n; r += warps) {
    const double di = s[r];
    for (int p = rowp[r] + lane; p < rowp[r + 1]; p += 32)
      vals[p] *= di * s[cols[p]];
  }
}

// x[idx[j]] *= s[j] (divide: x[idx[j]] /= s[j]).
__global__ void k_scale_gather(int m, const int* __restrict__ idx,
                               const double* __restrict__ s, double* x,
                               int divide) {
  for (int j = blockIdx.x * ST + threadIdx.x; j < m; j += gridDim.x * ST) {
    if (divide) x[idx[j]] /= s[j];
    else x[idx[j]] *= s[j];
  }
}

// xlam[slack_k] = grad[constr_k] + xlam[slack_k]: the constraint body
// d_k(x) recovered from the residual c_k(x) - s_k.
__global__ void k_init_slacks(int m, const int* __restrict__ sidx,
                              const int* __restrict__ cidx,
                              const double* __restrict__ grad, double* xlam) {
  for (int k = blockIdx.x * ST + threadIdx.x; k < m; k += gridDim.x * ST) {
    const int si = sidx[k];
    const double residual = grad[cidx[k]];
    const double s_old = xlam[si];
    xlam[si] = residual + s_old;
  }
}

__global__ void k_dual_residual(int np, const int* __restrict__ pidx,
                                const double* __restrict__ grad,
                                const double* __restrict__ zl,
                                const double* __restrict__ zu, double* out) {
  for (int i = blockIdx.x * ST + threadIdx.x; i < np; i += gridDim.x * ST) {
    const int idx = pidx[i];
    out[idx] = grad[idx] - zl[i] + zu[i];
  }
}

__global__ void k_copy_gather(int m, const int* __restrict__ idx,
                              const double* __restrict__ src, double* dst) {
  for (int j = blockIdx.x * ST + threadIdx.x; j < m; j += gridDim.x * ST)
    dst[idx[j]] = src[idx[j]];
}

}  // namespace
}  // namespace ab

extern "C" {

int ab_vec_absmax_gather(int m, const int* idx, const double* x,
                         double* d_out, void* stream) {
  if (m < 0 || !d_out || (m > 0 && (!idx || !x))) return AB_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(d_out, 0, sizeof(double), st) != cudaSuccess) return AB_ERR_CUDA;
  if (m > 0) {
    ab::k_absmax_gather<<<ab::grid_for(m), ab::ST, 0, st>>>(m, idx, x, d_out);
    ab::count_launch();
  }
  return ab::done();
}

int ab_ipm_constraint_scale(int n, int nc, const int* cidx, const int* rowp,
                            const double* hess_vals, double max_gradient,
                            double min_value, double* dc, double* lbh,
                            double* scale, void* stream) {
  if (n < 0 || nc < 0 || !scale || (nc > 0 && (!cidx || !rowp || !hess_vals ||
                                               !dc || !lbh)))
    return AB_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (n > 0) {
    ab::k_fill<<<ab::grid_for(n), ab::ST, 0, st>>>(n, 1.0, scale);
    ab::count_launch();
  }
  if (nc > 0) {
    ab::k_rows_absmax<<<ab::grid_for(32LL * nc), ab::ST, 0, st>>>(nc, cidx, rowp,
                                                                hess_vals, dc);
    ab::count_launch();
    ab::k_constraint_scale<<<ab::grid_for(nc), ab::ST, 0, st>>>(
        nc, cidx, max_gradient, min_value, dc, lbh, scale);
    ab::count_launch();
  }
  return ab::done();
}

int ab_csr_scale_symmetric(int n, const int* rowp, const int* cols,
                           const double* scale, double* vals, void* stream) {
  if (n < 0 || (n > 0 && (!rowp || !cols || !scale || !vals))) return AB_ERR_ARG;
  if (n == 0) return AB_OK;
  ab::k_scale_symmetric<<<ab::grid_for(32LL * n), ab::ST, 0, (cudaStream_t)stream>>>(
      n, rowp, cols, scale, vals);
  ab::count_launch();
  return ab::done();
}

int ab_vec_scale_gather(int m, const int* idx, const double* s, double* x,
                        int divide, void* stream) {
  if (m < 0 || (m > 0 && (!idx || !s || !x))) return AB_ERR_ARG;
  if (m == 0) return AB_OK;
  ab::k_scale_gather<<<ab::grid_for(m), ab::ST, 0, (cudaStream_t)stream>>>(
      m, idx, s, x, divide);
  ab::count_launch();
  return ab::done();
}

int ab_ipm_initialize_slacks(int nslack, const int* slack_idx,
                             const int* constr_idx, const double* grad,
                             double* xlam, void* stream) {
  if (nslack < 0 || (nslack > 0 && (!slack_idx || !constr_idx || !grad || !xlam)))
    return AB_ERR_ARG;
  if (nslack == 0) return AB_OK;
  ab::k_init_slacks<<<ab::grid_for(nslack), ab::ST, 0, (cudaStream_t)stream>>>(
      nslack, slack_idx, constr_idx, grad, xlam);
  ab::count_launch();
  return ab::done();
}

int ab_ipm_dual_residual_vector(int n, int np, const int* pidx,
                                const double* grad, const double* zl,
                                const double* zu, double* out, void* stream) {
  if (n < 0 || np < 0 || !out || (np > 0 && (!pidx || !grad || !zl || !zu)))
    return AB_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (n > 0 && cudaMemsetAsync(out, 0, sizeof(double) * (size_t)n, st) != cudaSuccess)
    return AB_ERR_CUDA;
  if (np > 0) {
    ab::k_dual_residual<<<ab::grid_for(np), ab::ST, 0, st>>>(np, pidx, grad, zl, zu, out);
    ab::count_launch();
  }
  return ab::done();
}

int ab_vec_copy_gather(int m, const int* idx, const double* src, double* dst,
                       void* stream) {
  if (m < 0 || (m > 0 && (!idx || !src || !dst))) return AB_ERR_ARG;
  if (m == 0) return AB_OK;
  ab::k_copy_gather<<<ab::grid_for(m), ab::ST, 0, (cudaStream_t)stream>>>(m, idx, src, dst);
  ab::count_launch();
  return ab::done();
}

}  // extern "C"

// Component kernels of the cart-pole trapezoidal-collocation model: the
// gradient of the Lagrangian and its Hessian scattered into the CSR KKT
// values, with exact derivatives from hyper-dual numbers (hyperdual.h).
//
// One thread per interval instance; even and odd intervals are launched
// separately because consecutive intervals share a node (no atomics, a
// deterministic scatter).  Replaces, for this model, the generated
// component code behind OptimizationProblem::gradient / hessian
// (include/optimization_problem.h:742-818).
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/amigo_b200.h"
#include "launch_count.h"
#include "hyperdual.h"

namespace ab {
namespace {

// Per-interval constants: step h and pole mass (a batch of instances has
// one value per interval; a single model uses its scalars).
struct IvParams {
  double h, mp;
};
__device__ __forceinline__ IvParams iv_params(const ab_cartpole& m, int k) {
  return IvParams{m.h_iv ? m.h_iv[k] : m.h, m.m_iv ? m.m_iv[k] : m.m};
}

// Cart-pole dynamics f(q, u) for q = (x, theta, xdot, thetadot).
template <typename T>
__device__ __forceinline__ void dynamics(const ab_cartpole& m, double mp,
                                         const T* q, const T& u, T* f) {
  const T s = sin(q[1]), c = cos(q[1]);
  const T td2 = q[3] * q[3];
  const T den = m.M + mp * (1.0 - c * c);
  f[0] = q[2];
  f[1] = q[3];
  f[2] = (m.l * mp * s * td2 + u + mp * m.g * c * s) / den;
  f[3] = -(m.l * mp * c * s * td2 + u * c + (m.M + mp) * m.g * s) / (m.l * den);
}

// phi(z) = alpha h/2 u^2 - h/2 lam^T f(z) for one node z = (q, u):
// value, gradient (5) and Hessian (5x5, symmetric) and the Jacobian of f
// (4x5) at z.
__device__ void node_derivs(const ab_cartpole& m, IvParams ip, const double* z,
                            const double* lam, double alpha, double* grad,
                            double* hess, double* jac) {
  const double hh = 0.5 * ip.h;
  for (int i = 0; i < 5; i++) {
    for (int j = i; j < 5; j++) {
      HD zz[5];
      for (int t = 0; t < 5; t++) zz[t] = HD(z[t]);
      zz[i].b = 1.0;
      zz[j].c += 1.0;
      HD f[4];
      dynamics(m, ip.mp, zz, zz[4], f);
      HD phi = alpha * hh * zz[4] * zz[4];
      for (int t = 0; t < 4; t++) phi = phi - hh * lam[t] * f[t];
      hess[i * 5 + j] = phi.d;
      hess[j * 5 + i] = phi.d;
      if (i == j) {
        grad[i] = phi.b;
        for (int t = 0; t < 4; t++) jac[t * 5 + i] = f[t].b;
      }
    }
  }
}

__device__ void interval_values(const ab_cartpole& m, const double* x, int k,
                                double alpha, double* g20, double* blk,
                                double* defect) {
  const int* iv = m.iv + 14 * k;
  double z0[5], z1[5], lam[4];
  for (int t = 0; t < 5; t++) z0[t] = x[iv[t]];
  for (int t = 0; t < 5; t++) z1[t] = x[iv[5 + t]];
  for (int t = 0; t < 4; t++) lam[t] = x[iv[10 + t]];
  const IvParams ip = iv_params(m, k);
  double g0[5], g1[5], h0[25], h1[25], j0[20], j1[20];
  node_derivs(m, ip, z0, lam, alpha, g0, h0, j0);
  node_derivs(m, ip, z1, lam, alpha, g1, h1, j1);
  // defect d = q1 - q0 - h/2 (f(z0) + f(z1))
  double f0[4], f1[4];
  dynamics(m, ip.mp, z0, z0[4], f0);
  dynamics(m, ip.mp, z1, z1[4], f1);
  for (int t = 0; t < 4; t++)
    defect[t] = z1[t] - z0[t] - 0.5 * ip.h * (f0[t] + f1[t]);
  // gradient w.r.t. [z0 | z1]: phi terms plus the linear -lam / +lam parts
  for (int t = 0; t < 5; t++) {
    g20[t] = g0[t] - (t < 4 ? lam[t] : 0.0);
    g20[5 + t] = g1[t] + (t < 4 ? lam[t] : 0.0);
  }
  if (!blk) return;
  for (int t = 0; t < 196; t++) blk[t] = 0.0;
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++) {
      blk[i * 14 + j] = h0[i * 5 + j];
      blk[(5 + i) * 14 + 5 + j] = h1[i * 5 + j];
    }
  // Jacobian rows (lam) x cols (z0, z1) and the transposed block
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 5; c++) {
      const double a = (c == r ? -1.0 : 0.0) - 0.5 * ip.h * j0[r * 5 + c];
      const double b = (c == r ? 1.0 : 0.0) - 0.5 * ip.h * j1[r * 5 + c];
      blk[(10 + r) * 14 + c] = a;
      blk[c * 14 + 10 + r] = a;
      blk[(10 + r) * 14 + 5 + c] = b;
      blk[(5 + c) * 14 + 10 + r] = b;
    }
}

__global__ void k_cartpole_hessian(ab_cartpole m, int parity,
                                   const double* __restrict__ x, double alpha,
                                   double* __restrict__ vals) {
  const int k = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + parity;
  if (k >= m.N) return;
  double g[10], d[4], blk[196];
  interval_values(m, x, k, alpha, g, blk, d);
  const int* pos = m.ipos + 196 * k;
  for (int t = 0; t < 196; t++)
    if (blk[t] != 0.0) vals[pos[t]] += blk[t];
}

__global__ void k_cartpole_gradient(ab_cartpole m, int parity,
                                    const double* __restrict__ x, double alpha,
                                    double* __restrict__ grad) {
  const int k = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + parity;
  if (k >= m.N) return;
  double g[10], d[4];
  interval_values(m, x, k, alpha, g, nullptr, d);
  const int* iv = m.iv + 14 * k;
  for (int t = 0; t < 10; t++) grad[iv[t]] += g[t];
  for (int t = 0; t < 4; t++) grad[iv[10 + t]] += d[t];
}

// Boundary components: mu^T q (targets in lbh): gradient mu / q, Hessian
// (mu_j, q_j) = 1.
__global__ void k_cartpole_bc(ab_cartpole m, const double* __restrict__ x,
                              double* grad, double* vals) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= (m.nbc > 0 ? m.nbc : 2)) return;
  const int* bv = m.bv + 8 * b;
  if (grad) {
    for (int t = 0; t < 4; t++) {
      grad[bv[t]] += x[bv[4 + t]];
      grad[bv[4 + t]] += x[bv[t]];
    }
  }
  if (vals) {
    const int* pos = m.bpos + 64 * b;
    for (int t = 0; t < 4; t++) {
      vals[pos[(4 + t) * 8 + t]] += 1.0;
      vals[pos[t * 8 + 4 + t]] += 1.0;
    }
  }
}

// Objective sum_k h/2 (u_k^2 + u_k+1^2); one block per instance (its
// intervals [inst_iv[b], inst_iv[b+1]); a single model is one instance),
// fixed summation order.
__global__ void k_cartpole_objective(ab_cartpole m, const double* x,
                                     double* out) {
  __shared__ double part[256];
  const int b = blockIdx.x;
  const int k0 = m.inst_iv ? m.inst_iv[b] : 0;
  const int k1 = m.inst_iv ? m.inst_iv[b + 1] : m.N;
  double acc = 0.0;
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    const int* iv = m.iv + 14 * k;
    const double u0 = x[iv[4]], u1 = x[iv[9]];
    acc += 0.5 * iv_params(m, k).h * (u0 * u0 + u1 * u1);
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[b] = part[0];
}

}  // namespace
}  // namespace ab

extern "C" {

int ab_cartpole_objective(const ab_cartpole* m, const double* x, double* out,
                          void* stream) {
  if (!m || !x || !out) return AB_ERR_ARG;
  const int nb = m->inst_iv ? (m->ninst > 0 ? m->ninst : 1) : 1;
  { ab::k_cartpole_objective<<<nb, 256, 0, (cudaStream_t)stream>>>(*m, x, out); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? AB_OK : AB_ERR_CUDA;
}

int ab_cartpole_gradient(const ab_cartpole* m, const double* x, double alpha,
                         double* grad, void* stream) {
  if (!m || !x || !grad || m->N < 1) return AB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaMemsetAsync(grad, 0, (size_t)m->n * sizeof(double), s);
  const int half = (m->N + 1) / 2;
  for (int parity = 0; parity < 2; parity++)
    { ab::k_cartpole_gradient<<<(half + 127) / 128, 128, 0, s>>>(*m, parity, x,
                                                               alpha, grad); ab::count_launch(); }
  { ab::k_cartpole_bc<<<(std::max(m->nbc, 2) + 127) / 128, 128, 0, s>>>(
      *m, x, grad, nullptr); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? AB_OK : AB_ERR_CUDA;
}

int ab_cartpole_hessian(const ab_cartpole* m, const double* x, double alpha,
                        double* vals, void* stream) {
  if (!m || !x || !vals || m->N < 1) return AB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaMemsetAsync(vals, 0, (size_t)m->nnz * sizeof(double), s);
  const int half = (m->N + 1) / 2;
  for (int parity = 0; parity < 2; parity++)
    { ab::k_cartpole_hessian<<<(half + 127) / 128, 128, 0, s>>>(*m, parity, x,
                                                              alpha, vals); ab::count_launch(); }
  { ab::k_cartpole_bc<<<(std::max(m->nbc, 2) + 127) / 128, 128, 0, s>>>(
      *m, x, nullptr, vals); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? AB_OK : AB_ERR_CUDA;
}

}  // extern "C"

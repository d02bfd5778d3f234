// Element kernels of the 2D SIMP full-space model: gradient of the
// Lagrangian and its Hessian scattered into the CSR KKT pattern.
//
// These replace, for this model, the reference's generated component code
// driven by OptimizationProblem::gradient / hessian
// (include/optimization_problem.h:742-818) and the CUDA atomic scatter
// kernels (include/cuda/component_group_backend.cuh:37-120).  One warp per
// element instance: the lanes gather the element's variables (coalesced
// from the element's index rows), each computes the per-element scalars
// redundantly, then the lanes stride over the element's KKT block entries
// and add them at precomputed CSR positions.  Elements are processed one
// colour at a time (no two elements of a colour share a node), so the
// scatter needs no atomics and the result is deterministic.
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/amigo_b200.h"

namespace ab {
namespace {

struct ElemScalars {
  double E, dE, d2E;  // stiffness and its first/second derivative in rt_e
  double Ku[8], Kl[8], lKu;
};

__device__ __forceinline__ void stiffness(const ab_simp2d* m, double r,
                                          double& E, double& dE,
                                          double& d2E) {
  const double p = m->penalty, dEr = m->E0 - m->Emin;
  const double rp2 = pow(r, p - 2.0);
  E = m->Emin + rp2 * r * r * dEr;
  dE = p * rp2 * r * dEr;
  d2E = p * (p - 1.0) * rp2 * dEr;
}

// Gathers the element's variables and forms K0 u, K0 lam, lam^T K0 u.
__device__ void element_scalars(const ab_simp2d* m, const double* K0,
                                const double* x, int e, ElemScalars& s,
                                double* u, double* rt, double* lam) {
  const int* ev = m->ev + (size_t)e * 20;
  for (int a = 0; a < 8; a++) u[a] = x[ev[a]];
  for (int a = 0; a < 4; a++) rt[a] = x[ev[8 + a]];
  for (int a = 0; a < 8; a++) lam[a] = x[ev[12 + a]];
  const double r = 0.25 * (rt[0] + rt[1] + rt[2] + rt[3]);
  stiffness(m, r, s.E, s.dE, s.d2E);
  s.lKu = 0.0;
  for (int a = 0; a < 8; a++) {
    double ku = 0.0, kl = 0.0;
    for (int b = 0; b < 8; b++) {
      ku += K0[a * 8 + b] * u[b];
      kl += K0[a * 8 + b] * lam[b];
    }
    s.Ku[a] = ku;
    s.Kl[a] = kl;
    s.lKu += lam[a] * ku;
  }
}

__global__ void k_simp2d_hessian(ab_simp2d m, const int* __restrict__ elems,
                                 int count, const double* __restrict__ x,
                                 double* __restrict__ vals) {
  __shared__ double K0[64], A[16];
  for (int t = threadIdx.x; t < 64; t += blockDim.x) K0[t] = m.K0[t];
  for (int t = threadIdx.x; t < 16; t += blockDim.x) A[t] = m.A[t];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= count) return;
  const int e = elems[w];
  ElemScalars s;
  double u[8], rt[4], lam[8];
  element_scalars(&m, K0, x, e, s, u, rt, lam);
  const double q1 = 0.25 * s.dE, q2 = 0.0625 * s.d2E * s.lKu;
  const int* ep = m.epos + (size_t)e * 400;
  for (int t = lane; t < 400; t += 32) {
    const int r = t / 20, c = t % 20;
    double v = 0.0;
    const bool ru = r < 8, rr = r >= 8 && r < 12, rl = r >= 12;
    const bool cu = c < 8, cr = c >= 8 && c < 12, cl = c >= 12;
    if (ru && cr) v = q1 * s.Kl[r];
    else if (ru && cl) v = s.E * K0[r * 8 + (c - 12)];
    else if (rr && cu) v = q1 * s.Kl[c];
    else if (rr && cr) v = q2;
    else if (rr && cl) v = q1 * s.Ku[c - 12];
    else if (rl && cu) v = s.E * K0[(r - 12) * 8 + c];
    else if (rl && cr) v = q1 * s.Ku[r - 12];
    else continue;
    vals[ep[t]] += v;
  }
  // Helmholtz filter block [rt(4) | re | mu(4)] (linear: Jacobian only)
  const int* fp = m.fpos + (size_t)e * 81;
  for (int t = lane; t < 81; t += 32) {
    const int r = t / 9, c = t % 9;
    double v;
    if (r >= 5 && c < 4) v = A[(r - 5) * 4 + c];
    else if (c >= 5 && r < 4) v = A[(c - 5) * 4 + r];
    else if ((r >= 5 && c == 4) || (r == 4 && c >= 5)) v = -m.Bq;
    else continue;
    vals[fp[t]] += v;
  }
  if (lane < 2) vals[m.vpos[2 * e + lane]] += m.vcoef;
}

__global__ void k_simp2d_gradient(ab_simp2d m, const int* __restrict__ elems,
                                  int count, const double* __restrict__ x,
                                  double* __restrict__ g) {
  __shared__ double K0[64], A[16];
  for (int t = threadIdx.x; t < 64; t += blockDim.x) K0[t] = m.K0[t];
  for (int t = threadIdx.x; t < 16; t += blockDim.x) A[t] = m.A[t];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= count) return;
  const int e = elems[w];
  ElemScalars s;
  double u[8], rt[4], lam[8];
  element_scalars(&m, K0, x, e, s, u, rt, lam);
  const int* ev = m.ev + (size_t)e * 20;
  const int* fv = m.fv + (size_t)e * 9;
  const double re = x[fv[4]];
  double mu[4];
  for (int a = 0; a < 4; a++) mu[a] = x[fv[5 + a]];
  // lanes 0-7: u rows, 8-11: rt rows, 12-19: lam rows, 20: re, 21-24: mu
  if (lane < 8) {
    g[ev[lane]] += s.E * s.Kl[lane];
  } else if (lane < 12) {
    const int i = lane - 8;
    double v = 0.25 * s.dE * s.lKu;
    for (int k = 0; k < 4; k++) v += mu[k] * A[k * 4 + i];
    g[ev[lane]] += v;
  } else if (lane < 20) {
    g[ev[lane]] += s.E * s.Ku[lane - 12];
  } else if (lane == 20) {
    g[fv[4]] += -m.Bq * (mu[0] + mu[1] + mu[2] + mu[3]) + m.vcoef * x[m.nu_index];
  } else if (lane < 25) {
    const int k = lane - 21;
    double v = -m.Bq * re;
    for (int l = 0; l < 4; l++) v += A[k * 4 + l] * rt[l];
    g[fv[5 + k]] += v;
  }
}

// Terms outside the element loop: alpha f^T u, -f in the equilibrium
// residual, the volume row v^T re - volfrac - s, the slack column -nu.
__global__ void k_simp2d_global_grad(ab_simp2d m, const double* x,
                                     double alpha, double* g) {
  __shared__ double part[256];
  double acc = 0.0;
  for (int e = threadIdx.x; e < m.nelems; e += blockDim.x)
    acc += x[m.re0 + e];
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  for (int t = threadIdx.x; t < m.nload; t += blockDim.x) {
    const int i = m.load_idx[t];
    g[m.u0 + i] += alpha * m.load_val[t];
    g[m.lam0 + i] -= m.load_val[t];
  }
  if (threadIdx.x == 0) {
    g[m.nu_index] += m.vcoef * part[0] - m.volfrac - x[m.s_index];
    g[m.s_index] += -x[m.nu_index];
  }
}

__global__ void k_simp2d_global_hess(ab_simp2d m, double* vals) {
  if (threadIdx.x < 2) vals[m.spos[threadIdx.x]] += -1.0;
}

__global__ void k_set_values(int n, const int* pos, double v, double* vals) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    vals[pos[i]] = v;
}

}  // namespace
}  // namespace ab

extern "C" {

int ab_simp2d_gradient(const ab_simp2d* m, const double* x, double alpha,
                       double* grad, void* stream) {
  if (!m || !x || !grad) return AB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaMemsetAsync(grad, 0, (size_t)m->n * sizeof(double), s);
  for (int c = 0; c < 4; c++) {
    const int cnt = m->color_ptr[c + 1] - m->color_ptr[c];
    if (!cnt) continue;
    ab::k_simp2d_gradient<<<(cnt + 7) / 8, 256, 0, s>>>(
        *m, m->color_elems + m->color_ptr[c], cnt, x, grad);
  }
  ab::k_simp2d_global_grad<<<1, 256, 0, s>>>(*m, x, alpha, grad);
  // fixed variables: zero their gradient rows
  if (m->nfixed)
    ab::k_set_values<<<(m->nfixed + 255) / 256, 256, 0, s>>>(m->nfixed, m->fixed,
                                                             0.0, grad);
  return cudaGetLastError() == cudaSuccess ? AB_OK : AB_ERR_CUDA;
}

int ab_simp2d_hessian(const ab_simp2d* m, const double* x, double alpha,
                      double* vals, void* stream) {
  (void)alpha;  // the objective f^T u is linear: no Hessian term
  if (!m || !x || !vals) return AB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaMemsetAsync(vals, 0, (size_t)m->nnz * sizeof(double), s);
  for (int c = 0; c < 4; c++) {
    const int cnt = m->color_ptr[c + 1] - m->color_ptr[c];
    if (!cnt) continue;
    ab::k_simp2d_hessian<<<(cnt + 7) / 8, 256, 0, s>>>(
        *m, m->color_elems + m->color_ptr[c], cnt, x, vals);
  }
  ab::k_simp2d_global_hess<<<1, 32, 0, s>>>(*m, vals);
  if (m->nfixed_zero)
    ab::k_set_values<<<(m->nfixed_zero + 255) / 256, 256, 0, s>>>(
        m->nfixed_zero, m->fixed_zero_pos, 0.0, vals);
  if (m->nfixed)
    ab::k_set_values<<<(m->nfixed + 255) / 256, 256, 0, s>>>(
        m->nfixed, m->fixed_diag_pos, 1.0, vals);
  return cudaGetLastError() == cudaSuccess ? AB_OK : AB_ERR_CUDA;
}

}  // extern "C"

// Element kernels of the SIMP full-space compliance models (2D bilinear
// quads and 3D trilinear hexahedra): gradient of the Lagrangian and its
// Hessian scattered into the CSR KKT pattern.
//
// These replace, for these models, the reference's generated component code
// driven by OptimizationProblem::gradient / hessian
// (include/optimization_problem.h:742-818) and the CUDA atomic scatter
// kernels (include/cuda/component_group_backend.cuh:37-120).  One warp per
// element instance: the lanes gather the element's variables (coalesced
// from the element's index row) into the warp's shared-memory slot, lanes
// a < ND form row a of K0 u and K0 lam, lane 0 the element scalars, then
// the lanes stride over the element's KKT block entries and add them at
// precomputed CSR positions.  Elements are processed one colour at a time
// (no two elements of a colour share a node), so the scatter needs no
// atomics and the result is deterministic.
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/amigo_b200.h"
#include "launch_count.h"

namespace ab {
namespace {

// Fields shared by ab_simp2d and ab_simp3d.
struct SimpView {
  int n, nnz, nelems, nnodes;
  int u0, rt0, re0, s_index, lam0, mu0, nu_index;
  int ncolors;
  int color_ptr[9];
  const int* color_elems;
  const int* ev;
  const int* fv;
  const int* epos;
  const int* fpos;
  const int* vpos;
  const int* spos;
  const int* fixed;
  const int* fixed_zero_pos;
  const int* fixed_diag_pos;
  const int* load_idx;
  const double* load_val;
  const double* K0;
  const double* A;
  int nfixed, nfixed_zero, nload;
  double Bq, vcoef, volfrac, E0, Emin, penalty;
};

template <class M>
SimpView view(const M* m, int ncolors) {
  SimpView v;
  v.n = m->n; v.nnz = m->nnz; v.nelems = m->nelems; v.nnodes = m->nnodes;
  v.u0 = m->u0; v.rt0 = m->rt0; v.re0 = m->re0; v.s_index = m->s_index;
  v.lam0 = m->lam0; v.mu0 = m->mu0; v.nu_index = m->nu_index;
  v.ncolors = ncolors;
  for (int c = 0; c < 9; c++) v.color_ptr[c] = c <= ncolors ? m->color_ptr[c] : 0;
  v.color_elems = m->color_elems; v.ev = m->ev; v.fv = m->fv;
  v.epos = m->epos; v.fpos = m->fpos; v.vpos = m->vpos; v.spos = m->spos;
  v.fixed = m->fixed; v.fixed_zero_pos = m->fixed_zero_pos;
  v.fixed_diag_pos = m->fixed_diag_pos; v.load_idx = m->load_idx;
  v.load_val = m->load_val; v.K0 = m->K0; v.A = m->A;
  v.nfixed = m->nfixed; v.nfixed_zero = m->nfixed_zero; v.nload = m->nload;
  v.Bq = m->Bq; v.vcoef = m->vcoef; v.volfrac = m->volfrac; v.E0 = m->E0;
  v.Emin = m->Emin; v.penalty = m->penalty;
  return v;
}

// Element sizes: NV nodes, ND displacement dofs, NE = |ev row|, NF = |fv row|.
template <int DIM>
struct Dims {
  static constexpr int NV = 1 << DIM;
  static constexpr int ND = DIM * NV;
  static constexpr int NE = 2 * ND + NV;
  static constexpr int NF = 2 * NV + 1;
  // per-warp shared slot: v[NE] (u | rt | lam), Ku[ND], Kl[ND], scalars[4]
  static constexpr int SLOT = NE + 2 * ND + 4;
  static constexpr int WARPS = 8;
  static constexpr size_t smem() {
    return sizeof(double) * (ND * ND + NV * NV + WARPS * SLOT);
  }
};

__device__ __forceinline__ void stiffness(const SimpView& m, double r,
                                          double& E, double& dE,
                                          double& d2E) {
  const double p = m.penalty, dEr = m.E0 - m.Emin;
  const double rp2 = pow(r, p - 2.0);
  E = m.Emin + rp2 * r * r * dEr;
  dE = p * rp2 * r * dEr;
  d2E = p * (p - 1.0) * rp2 * dEr;
}

// Stages K0 and A, then fills the warp's slot for element e:
// v = x[ev], Ku = K0 u, Kl = K0 lam, sc = {E, dE, d2E, lam^T K0 u}.
template <int DIM>
__device__ void element_slot(const SimpView& m, const double* x, int e,
                             const double* K0, double* v, double* Ku,
                             double* Kl, double* sc, int lane) {
  using D = Dims<DIM>;
  const int* ev = m.ev + (size_t)e * D::NE;
  for (int t = lane; t < D::NE; t += 32) v[t] = x[ev[t]];
  __syncwarp();
  const double* u = v;
  const double* lam = v + D::ND + D::NV;
  if (lane < D::ND) {
    double ku = 0.0, kl = 0.0;
    for (int b = 0; b < D::ND; b++) {
      ku += K0[lane * D::ND + b] * u[b];
      kl += K0[lane * D::ND + b] * lam[b];
    }
    Ku[lane] = ku;
    Kl[lane] = kl;
  }
  __syncwarp();
  if (lane == 0) {
    const double* rt = v + D::ND;
    double r = 0.0;
    for (int a = 0; a < D::NV; a++) r += rt[a];
    r *= 1.0 / D::NV;
    stiffness(m, r, sc[0], sc[1], sc[2]);
    double lku = 0.0;
    for (int a = 0; a < D::ND; a++) lku += lam[a] * Ku[a];
    sc[3] = lku;
  }
  __syncwarp();
}

template <int DIM>
__global__ void k_simp_hessian(SimpView m, const int* __restrict__ elems,
                               int count, const double* __restrict__ x,
                               double* __restrict__ vals) {
  using D = Dims<DIM>;
  extern __shared__ double sm[];
  double* K0 = sm;
  double* A = K0 + D::ND * D::ND;
  for (int t = threadIdx.x; t < D::ND * D::ND; t += blockDim.x) K0[t] = m.K0[t];
  for (int t = threadIdx.x; t < D::NV * D::NV; t += blockDim.x) A[t] = m.A[t];
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int w = blockIdx.x * D::WARPS + wid;
  if (w >= count) return;
  const int e = elems[w];
  double* v = A + D::NV * D::NV + wid * D::SLOT;
  double* Ku = v + D::NE;
  double* Kl = Ku + D::ND;
  double* sc = Kl + D::ND;
  element_slot<DIM>(m, x, e, K0, v, Ku, Kl, sc, lane);
  const double E = sc[0];
  const double q1 = sc[1] * (1.0 / D::NV);
  const double q2 = sc[2] * sc[3] * (1.0 / (D::NV * D::NV));
  constexpr int R0 = D::ND, L0 = D::ND + D::NV;  // first rt / lam slot
  const int* ep = m.epos + (size_t)e * D::NE * D::NE;
  for (int t = lane; t < D::NE * D::NE; t += 32) {
    const int r = t / D::NE, c = t % D::NE;
    const bool ru = r < R0, rr = r >= R0 && r < L0, rl = r >= L0;
    const bool cu = c < R0, cr = c >= R0 && c < L0, cl = c >= L0;
    double val;
    if (ru && cr) val = q1 * Kl[r];
    else if (ru && cl) val = E * K0[r * D::ND + (c - L0)];
    else if (rr && cu) val = q1 * Kl[c];
    else if (rr && cr) val = q2;
    else if (rr && cl) val = q1 * Ku[c - L0];
    else if (rl && cu) val = E * K0[(r - L0) * D::ND + c];
    else if (rl && cr) val = q1 * Ku[r - L0];
    else continue;
    vals[ep[t]] += val;
  }
  // Helmholtz filter block [rt(NV) | re | mu(NV)] (linear: Jacobian only)
  const int* fp = m.fpos + (size_t)e * D::NF * D::NF;
  for (int t = lane; t < D::NF * D::NF; t += 32) {
    const int r = t / D::NF, c = t % D::NF;
    constexpr int V = D::NV;
    double val;
    if (r > V && c < V) val = A[(r - V - 1) * V + c];
    else if (c > V && r < V) val = A[(c - V - 1) * V + r];
    else if ((r > V && c == V) || (r == V && c > V)) val = -m.Bq;
    else continue;
    vals[fp[t]] += val;
  }
  if (lane < 2) vals[m.vpos[2 * e + lane]] += m.vcoef;
}

template <int DIM>
__global__ void k_simp_gradient(SimpView m, const int* __restrict__ elems,
                                int count, const double* __restrict__ x,
                                double* __restrict__ g) {
  using D = Dims<DIM>;
  extern __shared__ double sm[];
  double* K0 = sm;
  double* A = K0 + D::ND * D::ND;
  for (int t = threadIdx.x; t < D::ND * D::ND; t += blockDim.x) K0[t] = m.K0[t];
  for (int t = threadIdx.x; t < D::NV * D::NV; t += blockDim.x) A[t] = m.A[t];
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int w = blockIdx.x * D::WARPS + wid;
  if (w >= count) return;
  const int e = elems[w];
  double* v = A + D::NV * D::NV + wid * D::SLOT;
  double* Ku = v + D::NE;
  double* Kl = Ku + D::ND;
  double* sc = Kl + D::ND;
  element_slot<DIM>(m, x, e, K0, v, Ku, Kl, sc, lane);
  constexpr int V = D::NV, R0 = D::ND, L0 = D::ND + D::NV;
  const int* ev = m.ev + (size_t)e * D::NE;
  const int* fv = m.fv + (size_t)e * D::NF;
  const double* rt = v + R0;
  const double re = x[fv[V]];
  // rows: ev slots (u | rt | lam), then re, then the NV filter multipliers
  for (int t = lane; t < D::NE + 1 + V; t += 32) {
    if (t < R0) {
      g[ev[t]] += sc[0] * Kl[t];
    } else if (t < L0) {
      const int i = t - R0;
      double val = (1.0 / V) * sc[1] * sc[3];
      for (int k = 0; k < V; k++) val += x[fv[V + 1 + k]] * A[k * V + i];
      g[ev[t]] += val;
    } else if (t < D::NE) {
      g[ev[t]] += sc[0] * Ku[t - L0];
    } else if (t == D::NE) {
      double smu = 0.0;
      for (int k = 0; k < V; k++) smu += x[fv[V + 1 + k]];
      g[fv[V]] += -m.Bq * smu + m.vcoef * x[m.nu_index];
    } else {
      const int k = t - D::NE - 1;
      double val = -m.Bq * re;
      for (int l = 0; l < V; l++) val += A[k * V + l] * rt[l];
      g[fv[V + 1 + k]] += val;
    }
  }
}

// Terms outside the element loop: alpha f^T u, -f in the equilibrium
// residual, the volume row v^T re - volfrac - s, the slack column -nu.
__global__ void k_simp_global_grad(SimpView m, const double* x, double alpha,
                                   double* g) {
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

__global__ void k_simp_global_hess(SimpView m, double* vals) {
  if (threadIdx.x < 2) vals[m.spos[threadIdx.x]] += -1.0;
}

__global__ void k_set_values(int n, const int* pos, double v, double* vals) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    vals[pos[i]] = v;
}

template <int DIM>
int gradient(const SimpView& m, const double* x, double alpha, double* grad,
             cudaStream_t s) {
  using D = Dims<DIM>;
  cudaMemsetAsync(grad, 0, (size_t)m.n * sizeof(double), s);
  for (int c = 0; c < m.ncolors; c++) {
    const int cnt = m.color_ptr[c + 1] - m.color_ptr[c];
    if (!cnt) continue;
    { k_simp_gradient<DIM><<<(cnt + D::WARPS - 1) / D::WARPS, 32 * D::WARPS,
                           D::smem(), s>>>(m, m.color_elems + m.color_ptr[c],
                                           cnt, x, grad); ab::count_launch(); }
  }
  { k_simp_global_grad<<<1, 256, 0, s>>>(m, x, alpha, grad); ab::count_launch(); }
  // fixed variables: zero their gradient rows
  if (m.nfixed)
    { k_set_values<<<(m.nfixed + 255) / 256, 256, 0, s>>>(m.nfixed, m.fixed, 0.0,
                                                        grad); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? AB_OK : AB_ERR_CUDA;
}

template <int DIM>
int hessian(const SimpView& m, const double* x, double* vals, cudaStream_t s) {
  using D = Dims<DIM>;
  cudaMemsetAsync(vals, 0, (size_t)m.nnz * sizeof(double), s);
  for (int c = 0; c < m.ncolors; c++) {
    const int cnt = m.color_ptr[c + 1] - m.color_ptr[c];
    if (!cnt) continue;
    { k_simp_hessian<DIM><<<(cnt + D::WARPS - 1) / D::WARPS, 32 * D::WARPS,
                          D::smem(), s>>>(m, m.color_elems + m.color_ptr[c],
                                          cnt, x, vals); ab::count_launch(); }
  }
  { k_simp_global_hess<<<1, 32, 0, s>>>(m, vals); ab::count_launch(); }
  if (m.nfixed_zero)
    { k_set_values<<<(m.nfixed_zero + 255) / 256, 256, 0, s>>>(
        m.nfixed_zero, m.fixed_zero_pos, 0.0, vals); ab::count_launch(); }
  if (m.nfixed)
    { k_set_values<<<(m.nfixed + 255) / 256, 256, 0, s>>>(
        m.nfixed, m.fixed_diag_pos, 1.0, vals); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? AB_OK : AB_ERR_CUDA;
}

}  // namespace
}  // namespace ab

extern "C" {

int ab_simp2d_gradient(const ab_simp2d* m, const double* x, double alpha,
                       double* grad, void* stream) {
  if (!m || !x || !grad) return AB_ERR_ARG;
  return ab::gradient<2>(ab::view(m, 4), x, alpha, grad, (cudaStream_t)stream);
}

int ab_simp2d_hessian(const ab_simp2d* m, const double* x, double alpha,
                      double* vals, void* stream) {
  (void)alpha;  // the objective f^T u is linear: no Hessian term
  if (!m || !x || !vals) return AB_ERR_ARG;
  return ab::hessian<2>(ab::view(m, 4), x, vals, (cudaStream_t)stream);
}

int ab_simp3d_gradient(const ab_simp3d* m, const double* x, double alpha,
                       double* grad, void* stream) {
  if (!m || !x || !grad) return AB_ERR_ARG;
  return ab::gradient<3>(ab::view(m, 8), x, alpha, grad, (cudaStream_t)stream);
}

int ab_simp3d_hessian(const ab_simp3d* m, const double* x, double alpha,
                      double* vals, void* stream) {
  (void)alpha;
  if (!m || !x || !vals) return AB_ERR_ARG;
  return ab::hessian<3>(ab::view(m, 8), x, vals, (cudaStream_t)stream);
}

}  // extern "C"

// IPM vector kernels (include/interior_point_backend.h on the device).
//
// Elementwise kernels evaluate exactly the reference's expressions in the
// same order; this file is compiled with --fmad=false so no multiply-add is
// contracted and the results equal the reference's CPU results bit for bit.
// Reductions are deterministic: a fixed grid writes per-block partials in a
// fixed order to a scratch array and one block combines them in order.
// Argmin reductions keep the first index among equal minima, which is what
// the reference's sequential strict-less-than loop returns.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/amigo_b200.h"
#include "ipm_internal.h"
#include "launch_count.h"

namespace ab {
namespace {

constexpr int RT = 256;          // threads per block
constexpr int kRedBlocks = 296;  // 2 x 148 SMs: fixed grid for reductions

__device__ __forceinline__ bool finite_bound(double b) { return !isinf(b); }

struct P {
  int n, np, nc;
  const int* pidx;
  const int* cidx;
  const double* lbx;
  const double* ubx;
  const double* lbh;
  // batched problems: barrier parameter per instance and the instance of
  // every primal entry / n-vector entry (null for a single problem)
  const double* mu_inst;
  const int* pinst;
  const int* vinst;
  int ninst;
  const int* poff;
  const int* coff;
};

// Barrier parameter of primal entry i: the call's scalar, or the entry's
// instance value in a batched problem.
__device__ __forceinline__ double mu_at(const P& p, double mu, int i) {
  return p.mu_inst ? p.mu_inst[p.pinst[i]] : mu;
}
// Per-instance maximum of non-negative values: seg[k] = max(seg[k], v).
// Non-negative doubles order like their bit patterns, so an integer atomic
// max is exact; the plain read first skips most atomics (the stored value
// only grows, so a stale read can only let an unneeded atomic through).
// NaN is skipped, as fmax skips it.
__device__ __forceinline__ void seg_max(double* seg, int k, double v) {
  if (v > 0.0 && v > seg[k])
    atomicMax(reinterpret_cast<unsigned long long*>(seg + k),
              static_cast<unsigned long long>(__double_as_longlong(v)));
}
struct S {
  const double* xlam;
  const double* zl;
  const double* zu;
  const double* sl;
  const double* su;
};
P mkP(const ab_ipm_problem* p) {
  return P{p->n,      p->np,    p->nc,    p->pidx,  p->cidx,
           p->lbx,    p->ubx,   p->lbh,   p->mu_inst, p->pinst,
           p->vinst,  p->ninst, p->poff,  p->coff};
}
S mkS(const ab_ipm_state* s) { return S{s->xlam, s->zl, s->zu, s->sl, s->su}; }

int grid_for(long long m) {
  long long g = (m + RT - 1) / RT;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (int)g;
}

// ---------------------------------------------------------------- residual
// interior_point_backend.h:203-266
__global__ void k_residual(P p, S s, double mu, const double* grad,
                           double* res, double* partial) {
  double dsq = 0.0, psq = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    const int idx = p.pidx[i];
    const double mu_i = mu_at(p, mu, i);
    const double rhs_stat = grad[idx] - s.zl[i] + s.zu[i];
    dsq += rhs_stat * rhs_stat;
    double aug = rhs_stat;
    if (finite_bound(p.lbx[i])) {
      const double gap = s.sl[i];
      aug += (gap * s.zl[i] - mu_i) / gap;
    }
    if (finite_bound(p.ubx[i])) {
      const double gap = s.su[i];
      aug -= (gap * s.zu[i] - mu_i) / gap;
    }
    res[idx] = -aug;
  }
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p.nc; j += stride) {
    const int idx = p.cidx[j];
    const double rp = grad[idx] - p.lbh[j];
    psq += rp * rp;
    res[idx] = -rp;
  }
  if (partial) block_sum2(dsq, psq, partial);
}

// ---------------------------------------------------------------- diagonal
// interior_point_backend.h:277-288
__global__ void k_diagonal(P p, S s, double* diag) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    double sigma = 0.0;
    if (finite_bound(p.lbx[i])) sigma += s.zl[i] / s.sl[i];
    if (finite_bound(p.ubx[i])) sigma += s.zu[i] / s.su[i];
    diag[p.pidx[i]] = sigma;
  }
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p.nc; j += stride)
    diag[p.cidx[j]] = 0.0;
}

// ------------------------------------------------------- bound dual step
// interior_point_backend.h:303-321
__global__ void k_bound_dual_step(P p, S s, double mu, const double* px,
                                  double* dzl, double* dzu) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    const double dx = px[p.pidx[i]];
    const double mu_i = mu_at(p, mu, i);
    double a = 0.0, b = 0.0;
    if (finite_bound(p.lbx[i])) {
      const double gap = s.sl[i];
      const double rc = gap * s.zl[i] - mu_i;
      a = -(rc + s.zl[i] * dx) / gap;
    }
    if (finite_bound(p.ubx[i])) {
      const double gap = s.su[i];
      const double rc = gap * s.zu[i] - mu_i;
      b = -(rc - s.zu[i] * dx) / gap;
    }
    dzl[i] = a;
    dzu[i] = b;
  }
}

// ------------------------------------------------------------- max step
// interior_point_backend.h:329-369.  Candidates are only considered when
// strictly below the running minimum, starting from 1.0 (the binding's
// seed), so the result is (min over candidates < 1, first index) or
// (1, -1).
__device__ __forceinline__ void amin(double& v, int& i, double v2, int i2) {
  if (v2 < v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

// Final combination of per-block partials by one warp: lane l folds blocks
// l, l + 32, ... in order, then a fixed shuffle tree; the result (in lane
// 0) does not depend on timing.  partial[b * stride + q] is block b's value.
enum class Fold { Sum, Max, Min };
__device__ __forceinline__ double fold_op(Fold op, double a, double b) {
  return op == Fold::Sum ? a + b : (op == Fold::Max ? fmax(a, b) : fmin(a, b));
}
__device__ double warp_fold(const double* partial, int nblocks, int stride,
                            int q, Fold op, double init) {
  const int lane = threadIdx.x & 31;
  double v = init;
  for (int b = lane; b < nblocks; b += 32) v = fold_op(op, v, partial[b * stride + q]);
  for (int o = 16; o > 0; o >>= 1)
    v = fold_op(op, v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

__global__ void k_max_step(P p, S s, double tau, const double* px,
                           const double* dzl, const double* dzu,
                           double* pv, int* pi) {
  double ax = 1.0, az = 1.0;
  int xo = 0x7fffffff, zo = 0x7fffffff;  // order key: primal position
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    const double dx = px[p.pidx[i]];
    if (finite_bound(p.lbx[i])) {
      if (dx < 0.0) {
        double a = -tau * s.sl[i] / dx;
        if (a < ax) { ax = a; xo = i; }
      }
      if (dzl[i] < 0.0) {
        double a = -tau * s.zl[i] / dzl[i];
        if (a < az) { az = a; zo = i; }
      }
    }
    if (finite_bound(p.ubx[i])) {
      if (dx > 0.0) {
        double a = tau * s.su[i] / dx;
        if (a < ax) { ax = a; xo = i; }
      }
      if (dzu[i] < 0.0) {
        double a = -tau * s.zu[i] / dzu[i];
        if (a < az) { az = a; zo = i; }
      }
    }
  }
  // Within a thread the loop visits increasing i, so (value, first i) is
  // kept; across threads merge lexicographically.
  __shared__ double sv[2][RT / 32];
  __shared__ int si[2][RT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    double v2 = __shfl_down_sync(0xffffffffu, ax, o);
    int i2 = __shfl_down_sync(0xffffffffu, xo, o);
    amin(ax, xo, v2, i2);
    v2 = __shfl_down_sync(0xffffffffu, az, o);
    i2 = __shfl_down_sync(0xffffffffu, zo, o);
    amin(az, zo, v2, i2);
  }
  if (lane == 0) {
    sv[0][warp] = ax; si[0][warp] = xo;
    sv[1][warp] = az; si[1][warp] = zo;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < RT / 32; w++) {
      amin(sv[0][0], si[0][0], sv[0][w], si[0][w]);
      amin(sv[1][0], si[1][0], sv[1][w], si[1][w]);
    }
    pv[2 * blockIdx.x] = sv[0][0];
    pv[2 * blockIdx.x + 1] = sv[1][0];
    pi[2 * blockIdx.x] = si[0][0];
    pi[2 * blockIdx.x + 1] = si[1][0];
  }
}

__global__ void k_max_step_final(int nblocks, const int* pidx,
                                 const double* pv, const int* pi,
                                 double* out, int* iout) {
  // warp 0: primal step, warp 1: dual step; (value, first index) minimum
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w > 1) return;
  double v = 1.0;
  int o = 0x7fffffff;
  for (int b = lane; b < nblocks; b += 32) amin(v, o, pv[2 * b + w], pi[2 * b + w]);
  for (int sh = 16; sh > 0; sh >>= 1) {
    const double v2 = __shfl_down_sync(0xffffffffu, v, sh);
    const int o2 = __shfl_down_sync(0xffffffffu, o, sh);
    amin(v, o, v2, o2);
  }
  if (lane == 0) {
    out[w] = v;
    iout[w] = o == 0x7fffffff ? -1 : pidx[o];
  }
}

// ------------------------------------------------------------ apply step
// interior_point_backend.h:376-392
__global__ void k_apply_step(P p, S s, double ax, double az,
                             const double* dxlam, const double* dzl,
                             const double* dzu, double* xlam_new,
                             double* zl_new, double* zu_new, double* sl_new,
                             double* su_new) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride)
    xlam_new[i] = s.xlam[i] + ax * dxlam[i];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    const bool hl = finite_bound(p.lbx[i]), hu = finite_bound(p.ubx[i]);
    if (hl) zl_new[i] = s.zl[i] + az * dzl[i];
    if (hu) zu_new[i] = s.zu[i] + az * dzu[i];
    const double dx = ax * dxlam[p.pidx[i]];
    if (hl) sl_new[i] = s.sl[i] + dx;
    if (hu) su_new[i] = s.su[i] - dx;
  }
}

// ------------------------------------------------------------ reductions
// Ten quantities per block (see ab_ipm_reductions in amigo_b200.h).
constexpr int NQ = 13;
__global__ void k_reductions(P p, S s, double mu, const double* grad,
                             double* partial) {
  double q[NQ];
  q[0] = 0.0;                 // sum of complementarity products
  q[1] = 0.0;                 // count
  q[2] = INFINITY;            // min product
  q[3] = 0.0;                 // dual inf-norm
  q[4] = 0.0;                 // primal inf-norm
  q[5] = 0.0;                 // comp inf-norm (|gap z - mu|)
  q[6] = 0.0;                 // barrier log-sum
  q[7] = 0.0;                 // constraint violation 1-norm
  q[8] = 0.0;                 // max comp deviation
  q[9] = 0.0;                 // sum of squared (gap z - mu)
  q[10] = 0.0;                // dual residual sum of squares
  q[11] = 0.0;                // primal residual sum of squares
  q[12] = 0.0;                // sum of squared products gap z
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    if (grad) {
      const int idx = p.pidx[i];
      const double rd = grad[idx] - s.zl[i] + s.zu[i];
      q[3] = fmax(q[3], fabs(rd));
      q[10] += rd * rd;
    }
    if (finite_bound(p.lbx[i])) {
      const double c = s.sl[i] * s.zl[i];
      q[0] += c;
      q[1] += 1.0;
      q[2] = fmin(q[2], c);
      const double dev = fabs(c - mu);
      q[5] = fmax(q[5], dev);
      q[8] = fmax(q[8], dev);
      q[9] += (c - mu) * (c - mu);
      q[12] += c * c;
      const double g = s.sl[i];
      if (g > 0) q[6] -= mu * log(g);
    }
    if (finite_bound(p.ubx[i])) {
      const double c = s.su[i] * s.zu[i];
      q[0] += c;
      q[1] += 1.0;
      q[2] = fmin(q[2], c);
      const double dev = fabs(c - mu);
      q[5] = fmax(q[5], dev);
      q[8] = fmax(q[8], dev);
      q[9] += (c - mu) * (c - mu);
      q[12] += c * c;
      const double g = s.su[i];
      if (g > 0) q[6] -= mu * log(g);
    }
  }
  if (grad) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p.nc; j += stride) {
      const double rp = grad[p.cidx[j]] - p.lbh[j];
      const double r = fabs(rp);
      q[4] = fmax(q[4], r);
      q[7] += r;
      q[11] += rp * rp;
    }
  }
  __shared__ double sh[NQ][RT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < NQ; t++) {
    double v = q[t];
    for (int o = 16; o > 0; o >>= 1) {
      double w = __shfl_down_sync(0xffffffffu, v, o);
      if (t == 2) v = fmin(v, w);
      else if (t == 3 || t == 4 || t == 5 || t == 8) v = fmax(v, w);
      else v += w;
    }
    if (lane == 0) sh[t][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < NQ) {
    const int t = threadIdx.x;
    double v = sh[t][0];
    for (int w = 1; w < RT / 32; w++) {
      double x = sh[t][w];
      if (t == 2) v = fmin(v, x);
      else if (t == 3 || t == 4 || t == 5 || t == 8) v = fmax(v, x);
      else v += x;
    }
    partial[blockIdx.x * NQ + t] = v;
  }
}

__global__ void k_reductions_final(int nblocks, const double* partial,
                                   double* out) {
  const int t = threadIdx.x >> 5;  // one warp per quantity
  if (t >= NQ) return;
  const Fold op = t == 2 ? Fold::Min
                         : (t == 3 || t == 4 || t == 5 || t == 8) ? Fold::Max
                                                                  : Fold::Sum;
  const double init = t == 2 ? INFINITY : 0.0;
  const double v = warp_fold(partial, nblocks, NQ, t, op, init);
  if ((threadIdx.x & 31) == 0) out[t] = v;
}

// ------------------------------------------------------------ barrier dphi
// interior_point_backend.h:491-502
__global__ void k_barrier_dphi(P p, S s, double mu, const double* grad,
                               const double* px, double* partial) {
  double acc = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    const int idx = p.pidx[i];
    const double dx = px[idx];
    acc += grad[idx] * dx;
    if (finite_bound(p.lbx[i])) acc -= mu * dx / s.sl[i];
    if (finite_bound(p.ubx[i])) acc += mu * dx / s.su[i];
  }
  block_sum2(acc, 0.0, partial);
}

// ----------------------------------------------- multiplier reset / start
// interior_point_backend.h:508-535
__global__ void k_reset_bound_multipliers(P p, S s, double mu, double kappa,
                                          double* zl_out, double* zu_out) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    const double mu_i = mu_at(p, mu, i);
    if (finite_bound(p.lbx[i])) {
      const double g = s.sl[i];
      zl_out[i] = fmax(fmin(s.zl[i], kappa * mu_i / g), mu_i / (kappa * g));
    }
    if (finite_bound(p.ubx[i])) {
      const double g = s.su[i];
      zu_out[i] = fmax(fmin(s.zu[i], kappa * mu_i / g), mu_i / (kappa * g));
    }
  }
}

__global__ void k_affine_start_point(P p, S s, double beta_min,
                                     const double* dzl, const double* dzu,
                                     double* zl_out, double* zu_out) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    if (finite_bound(p.lbx[i])) zl_out[i] = fmax(s.zl[i] + dzl[i], beta_min);
    if (finite_bound(p.ubx[i])) zu_out[i] = fmax(s.zu[i] + dzu[i], beta_min);
  }
}

// compute_barrier_dphi_from_kkt (interior_point_backend.h:597-611)
__global__ void k_barrier_dphi_kkt(P p, S s, const double* res,
                                   const double* px, const double* diag,
                                   double* partial) {
  double acc = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    const int idx = p.pidx[i];
    acc -= res[idx] * px[idx];
  }
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p.nc; j += stride) {
    const int idx = p.cidx[j];
    const double lam = s.xlam[idx];
    const double jdx = res[idx] - diag[idx] * px[idx];
    acc -= lam * jdx;
  }
  block_sum2(acc, 0.0, partial);
}

// relax_bounds (interior_point_backend.h:126-146)
__global__ void k_relax_bounds(int np, const double* lbx, const double* ubx,
                               double* lo, double* hi, double factor,
                               double tol) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += gridDim.x * blockDim.x) {
    const double l = lbx[i], u = ubx[i];
    lo[i] = isinf(l) ? l : l - fmin(tol, factor * fmax(1.0, fabs(l)));
    hi[i] = isinf(u) ? u : u + fmin(tol, factor * fmax(1.0, fabs(u)));
  }
}

// project_primals_into_interior + initialize_bound_duals +
// initialize_slacks (interior_point_backend.h:82-88, 156-188)
__global__ void k_initialize(P p, double* xlam, double* zl, double* zu,
                             double* sl, double* su, double kappa1,
                             double kappa2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np;
       i += gridDim.x * blockDim.x) {
    const int idx = p.pidx[i];
    double x = xlam[idx];
    const double lb = p.lbx[i], ub = p.ubx[i];
    const bool hl = !isinf(lb), hu = !isinf(ub);
    if (hl && hu) {
      const double range = ub - lb;
      const double pl = fmin(kappa1 * fmax(1.0, fabs(lb)), kappa2 * range);
      const double pu = fmin(kappa1 * fmax(1.0, fabs(ub)), kappa2 * range);
      x = fmax(fmin(x, ub - pu), lb + pl);
    } else if (hl) {
      x = fmax(x, lb + kappa1 * fmax(1.0, fabs(lb)));
    } else if (hu) {
      x = fmin(x, ub - kappa1 * fmax(1.0, fabs(ub)));
    }
    xlam[idx] = x;
    zl[i] = hl ? 1.0 : 0.0;
    zu[i] = hu ? 1.0 : 0.0;
    sl[i] = hl ? (x - lb) : 1.0;
    su[i] = hu ? (ub - x) : 1.0;
  }
}

// ---------------------------------------------------- iterative refinement
// Refinement on the unreduced 8-block Newton system, restating
// DirectSparseSolver.iterative_refinement
// (amigo/algorithm/solvers/linear_solver.py:109-264) on the device.
// gl = sl where the lower bound is finite, else 1 (gu likewise).
__device__ __forceinline__ void ir_bounds(const P& p, const S& s, int i,
                                          bool& fl, bool& fu, double& gl,
                                          double& gu) {
  fl = finite_bound(p.lbx[i]);
  fu = finite_bound(p.ubx[i]);
  gl = fl ? s.sl[i] : 1.0;
  gu = fu ? s.su[i] : 1.0;
}

// Initial bound-dual steps from back-substitution and ||rhs||_inf over the
// four blocks (linear_solver.py:168-191).
__global__ void k_ir_init(P p, S s, double mu, const double* grad,
                          const double* rhs_saved, const double* px,
                          double* dzl, double* dzu, double* partial,
                          double* seg) {
  double nrm = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    bool fl, fu;
    double gl, gu;
    ir_bounds(p, s, i, fl, fu, gl, gu);
    const int idx = p.pidx[i];
    const double mu_i = mu_at(p, mu, i);
    const double zl = s.zl[i], zu = s.zu[i], dx = px[idx];
    dzl[i] = fl ? (mu_i - gl * zl - zl * dx) / gl : 0.0;
    dzu[i] = fu ? (mu_i - gu * zu + zu * dx) / gu : 0.0;
    const double rx = -(grad[idx] - zl + zu);
    double e = fabs(rx);
    if (fl) e = fmax(e, fabs(mu_i - gl * zl));
    if (fu) e = fmax(e, fabs(mu_i - gu * zu));
    nrm = fmax(nrm, e);
    if (seg) seg_max(seg, p.pinst[i], e);
  }
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p.nc; j += stride) {
    const int idx = p.cidx[j];
    const double e = fabs(rhs_saved[idx]);
    nrm = fmax(nrm, e);
    if (seg) seg_max(seg, p.vinst[idx], e);
  }
  block_max2(nrm, 0.0, partial);
}

// Residuals of the 8-block system at (px, dzl, dzu), the condensed
// correction right-hand side, and the two norms of the stopping test
// (linear_solver.py:202-244).
__global__ void k_ir_residual(P p, S s, double mu, const double* grad,
                              const double* rhs_saved, const double* kpx,
                              const double* px, const double* dzl,
                              const double* dzu, double* e_cond,
                              double* e_zl, double* e_zu, double* partial,
                              double* seg) {
  double nres = 0.0, nsol = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    bool fl, fu;
    double gl, gu;
    ir_bounds(p, s, i, fl, fu, gl, gu);
    const int idx = p.pidx[i];
    const double zl = s.zl[i], zu = s.zu[i], dx = px[idx];
    const double sigma = (fl ? zl / gl : 0.0) + (fu ? zu / gu : 0.0);
    const double rx = -(grad[idx] - zl + zu);
    const double ex = rx - kpx[idx] + sigma * dx + dzl[i] - dzu[i];
    const double mu_i = mu_at(p, mu, i);
    const double ezl = fl ? (mu_i - gl * zl) - zl * dx - gl * dzl[i] : 0.0;
    const double ezu = fu ? (mu_i - gu * zu) + zu * dx - gu * dzu[i] : 0.0;
    e_zl[i] = ezl;
    e_zu[i] = ezu;
    e_cond[idx] = ex + (fl ? ezl / gl : 0.0) - (fu ? ezu / gu : 0.0);
    const double r = fmax(fabs(ex), fmax(fabs(ezl), fabs(ezu)));
    const double x = fmax(fabs(dx), fmax(fabs(dzl[i]), fabs(dzu[i])));
    nres = fmax(nres, r);
    nsol = fmax(nsol, x);
    if (seg) {
      seg_max(seg, 2 * p.pinst[i], r);
      seg_max(seg, 2 * p.pinst[i] + 1, x);
    }
  }
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p.nc; j += stride) {
    const int idx = p.cidx[j];
    const double ec = rhs_saved[idx] - kpx[idx];
    e_cond[idx] = ec;
    nres = fmax(nres, fabs(ec));
    nsol = fmax(nsol, fabs(px[idx]));
    if (seg) {
      seg_max(seg, 2 * p.vinst[idx], fabs(ec));
      seg_max(seg, 2 * p.vinst[idx] + 1, fabs(px[idx]));
    }
  }
  block_max2(nres, nsol, partial);
}

// Back-substitute the bound-dual corrections and accumulate the solution
// (linear_solver.py:255-262).
__global__ void k_ir_update(P p, S s, const double* corr, const double* e_zl,
                            const double* e_zu, double* px, double* dzl,
                            double* dzu, const int* active) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    if (active && !active[p.pinst[i]]) continue;
    bool fl, fu;
    double gl, gu;
    ir_bounds(p, s, i, fl, fu, gl, gu);
    const double dc = corr[p.pidx[i]];
    if (fl) dzl[i] += (e_zl[i] - s.zl[i] * dc) / gl;
    if (fu) dzu[i] += (e_zu[i] + s.zu[i] * dc) / gu;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride)
    if (!active || active[p.vinst[i]]) px[i] += corr[i];
}

__global__ void k_max2_final(int nblocks, const double* partial, double* out) {
  const int t = threadIdx.x >> 5;
  if (t > 1) return;
  const double v = warp_fold(partial, nblocks, 2, t, Fold::Max, 0.0);
  if ((threadIdx.x & 31) == 0) out[t] = v;
}

// ------------------------------------------------- batched (per instance)
// One block per instance over its contiguous primal / constraint ranges;
// every quantity is reduced in a fixed order (deterministic).  Outputs per
// instance k at out[k * kSegQ + q]:
//   0 dual inf-norm, 1 primal inf-norm, 2 complementarity inf-norm
//   (|gap z - mu_k|), 3 constraint violation 1-norm, 4 barrier log-sum,
//   5 max primal step, 6 max dual step (fraction to the boundary, seeded
//   at 1), 7 barrier directional derivative, 8 max |lam + dlam|, 9 / 10 the
//   largest / smallest gap product s z over the bounded entries (-/+inf
//   when there are none): the complementarity inf-norm for any barrier
//   parameter m is then max(0, q9 - m, m - q10), the same value the
//   element-wise max of |s z - m| gives, because rounding is monotone.
constexpr int kSegQ = 12;
__global__ void k_seg_reduce(P p, S s, double tau, const double* grad,
                             const double* px, const double* dzl,
                             const double* dzu, const double* gf,
                             double* out) {
  const int k = blockIdx.x;
  const double mu = p.mu_inst[k];
  // tau < 0 selects the per-instance fraction max(-tau, 1 - mu_k)
  const double tk = tau < 0.0 ? fmax(-tau, 1.0 - mu) : tau;
  const int p0 = p.poff[k], p1 = p.poff[k + 1];
  const int c0 = p.coff[k], c1 = p.coff[k + 1];
  double q[11] = {0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0, -INFINITY, INFINITY};
  for (int i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
    const int idx = p.pidx[i];
    const bool hl = finite_bound(p.lbx[i]), hu = finite_bound(p.ubx[i]);
    if (grad) q[0] = fmax(q[0], fabs(grad[idx] - s.zl[i] + s.zu[i]));
    if (hl) {
      const double g = s.sl[i] * s.zl[i];
      q[2] = fmax(q[2], fabs(g - mu));
      q[9] = fmax(q[9], g);
      q[10] = fmin(q[10], g);
      if (s.sl[i] > 0) q[4] -= mu * log(s.sl[i]);
    }
    if (hu) {
      const double g = s.su[i] * s.zu[i];
      q[2] = fmax(q[2], fabs(g - mu));
      q[9] = fmax(q[9], g);
      q[10] = fmin(q[10], g);
      if (s.su[i] > 0) q[4] -= mu * log(s.su[i]);
    }
    if (px && dzl) {
      const double dx = px[idx];
      if (hl) {
        if (dx < 0.0) q[5] = fmin(q[5], -tk * s.sl[i] / dx);
        if (dzl[i] < 0.0) q[6] = fmin(q[6], -tk * s.zl[i] / dzl[i]);
      }
      if (hu) {
        if (dx > 0.0) q[5] = fmin(q[5], tk * s.su[i] / dx);
        if (dzu[i] < 0.0) q[6] = fmin(q[6], -tk * s.zu[i] / dzu[i]);
      }
    }
    if (gf && px) {
      const double dx = px[idx];
      q[7] += gf[idx] * dx;
      if (hl) q[7] -= mu * dx / s.sl[i];
      if (hu) q[7] += mu * dx / s.su[i];
    }
  }
  for (int j = c0 + threadIdx.x; j < c1; j += blockDim.x) {
    const int idx = p.cidx[j];
    if (grad) {
      const double r = fabs(grad[idx] - p.lbh[j]);
      q[1] = fmax(q[1], r);
      q[3] += r;
    }
    if (px && s.xlam) q[8] = fmax(q[8], fabs(s.xlam[idx] + px[idx]));
  }
  __shared__ double sh[11][RT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < 11; t++) {
    double v = q[t];
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_down_sync(0xffffffffu, v, o);
      if (t == 5 || t == 6 || t == 10) v = fmin(v, w);
      else if (t == 3 || t == 4 || t == 7) v += w;
      else v = fmax(v, w);
    }
    if (lane == 0) sh[t][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 11) {
    const int t = threadIdx.x;
    double v = sh[t][0];
    for (int w = 1; w < RT / 32; w++) {
      const double x = sh[t][w];
      if (t == 5 || t == 6 || t == 10) v = fmin(v, x);
      else if (t == 3 || t == 4 || t == 7) v += x;
      else v = fmax(v, x);
    }
    out[k * kSegQ + t] = v;
  }
}

// apply_step with per-instance step lengths (interior_point_backend.h:
// 376-392): xlam += ax_k dxlam, z += az_k dz, s +- ax_k dx.
__global__ void k_apply_step_seg(P p, S s, const double* ax, const double* az,
                                 const double* dxlam, const double* dzl,
                                 const double* dzu, double* xlam_new,
                                 double* zl_new, double* zu_new,
                                 double* sl_new, double* su_new) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride)
    xlam_new[i] = s.xlam[i] + ax[p.vinst[i]] * dxlam[i];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.np; i += stride) {
    const int k = p.pinst[i];
    const bool hl = finite_bound(p.lbx[i]), hu = finite_bound(p.ubx[i]);
    if (hl) zl_new[i] = s.zl[i] + az[k] * dzl[i];
    if (hu) zu_new[i] = s.zu[i] + az[k] * dzu[i];
    const double dx = ax[k] * dxlam[p.pidx[i]];
    if (hl) sl_new[i] = s.sl[i] + dx;
    if (hu) su_new[i] = s.su[i] - dx;
  }
}

__global__ void k_sum2_final(int nblocks, const double* partial, double* out) {
  const int t = threadIdx.x >> 5;
  if (t > 1) return;
  const double v = warp_fold(partial, nblocks, 2, t, Fold::Sum, 0.0);
  if ((threadIdx.x & 31) == 0) out[t] = v;
}

__global__ void k_sum1_final(int nblocks, const double* partial, double* out) {
  const double v = warp_fold(partial, nblocks, 2, 0, Fold::Sum, 0.0);
  if (threadIdx.x == 0) out[0] = v;
}

}  // namespace

// Two-value block maximum written to partial[2 * blockIdx.x + {0, 1}].
__device__ void block_max2(double a, double b, double* partial) {
  __shared__ double sa[RT / 32], sb[RT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    a = fmax(a, __shfl_down_sync(0xffffffffu, a, o));
    b = fmax(b, __shfl_down_sync(0xffffffffu, b, o));
  }
  if (lane == 0) {
    sa[warp] = a;
    sb[warp] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0, y = 0.0;
    for (int w = 0; w < RT / 32; w++) {
      x = fmax(x, sa[w]);
      y = fmax(y, sb[w]);
    }
    partial[2 * blockIdx.x] = x;
    partial[2 * blockIdx.x + 1] = y;
  }
}

// Two-value block sum written to partial[2 * blockIdx.x + {0, 1}].
__device__ void block_sum2(double a, double b, double* partial) {
  __shared__ double sa[RT / 32], sb[RT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    sa[warp] = a;
    sb[warp] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0, y = 0.0;
    for (int w = 0; w < RT / 32; w++) {
      x += sa[w];
      y += sb[w];
    }
    partial[2 * blockIdx.x] = x;
    partial[2 * blockIdx.x + 1] = y;
  }
}

int ipm_residual(const ab_ipm_problem* p, const ab_ipm_state* s, double mu,
                 const double* grad, double* res, double* out2,
                 cudaStream_t st, double* scratch) {
  P pp = mkP(p);
  S ss = mkS(s);
  if (out2) {
    { k_residual<<<kRedBlocks, RT, 0, st>>>(pp, ss, mu, grad, res, scratch); ab::count_launch(); }
    { k_sum2_final<<<1, 64, 0, st>>>(kRedBlocks, scratch, out2); ab::count_launch(); }
  } else {
    long long m = p->np > p->nc ? p->np : p->nc;
    { k_residual<<<grid_for(m), RT, 0, st>>>(pp, ss, mu, grad, res, nullptr); ab::count_launch(); }
  }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_diagonal(const ab_ipm_problem* p, const ab_ipm_state* s, double* diag,
                 cudaStream_t st) {
  long long m = p->np > p->nc ? p->np : p->nc;
  { k_diagonal<<<grid_for(m), RT, 0, st>>>(mkP(p), mkS(s), diag); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_bound_dual_step(const ab_ipm_problem* p, const ab_ipm_state* s,
                        double mu, const double* px, double* dzl, double* dzu,
                        cudaStream_t st) {
  { k_bound_dual_step<<<grid_for(p->np), RT, 0, st>>>(mkP(p), mkS(s), mu, px,
                                                     dzl, dzu); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_max_step(const ab_ipm_problem* p, const ab_ipm_state* s, double tau,
                 const double* px, const double* dzl, const double* dzu,
                 double* out, int* iout, cudaStream_t st, double* scratch) {
  double* pv = scratch;
  int* pi = reinterpret_cast<int*>(scratch + 2 * kRedBlocks);
  { k_max_step<<<kRedBlocks, RT, 0, st>>>(mkP(p), mkS(s), tau, px, dzl, dzu, pv,
                                        pi); ab::count_launch(); }
  { k_max_step_final<<<1, 64, 0, st>>>(kRedBlocks, p->pidx, pv, pi, out, iout); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_apply_step(const ab_ipm_problem* p, const ab_ipm_state* s, double ax,
                   double az, const double* dxlam, const double* dzl,
                   const double* dzu, double* xlam_new, double* zl_new,
                   double* zu_new, double* sl_new, double* su_new,
                   cudaStream_t st) {
  long long m = p->n > p->np ? p->n : p->np;
  { k_apply_step<<<grid_for(m), RT, 0, st>>>(mkP(p), mkS(s), ax, az, dxlam, dzl,
                                           dzu, xlam_new, zl_new, zu_new,
                                           sl_new, su_new); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_reductions(const ab_ipm_problem* p, const ab_ipm_state* s, double mu,
                   const double* grad, double* out, cudaStream_t st,
                   double* scratch) {
  { k_reductions<<<kRedBlocks, RT, 0, st>>>(mkP(p), mkS(s), mu, grad, scratch); ab::count_launch(); }
  { k_reductions_final<<<1, 32 * NQ, 0, st>>>(kRedBlocks, scratch, out); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_barrier_dphi(const ab_ipm_problem* p, const ab_ipm_state* s,
                     double mu, const double* grad, const double* px,
                     double* out, cudaStream_t st, double* scratch) {
  { k_barrier_dphi<<<kRedBlocks, RT, 0, st>>>(mkP(p), mkS(s), mu, grad, px,
                                            scratch); ab::count_launch(); }
  { k_sum1_final<<<1, 32, 0, st>>>(kRedBlocks, scratch, out); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_reset_bound_multipliers(const ab_ipm_problem* p,
                                const ab_ipm_state* s, double mu,
                                double kappa, double* zl_out, double* zu_out,
                                cudaStream_t st) {
  { k_reset_bound_multipliers<<<grid_for(p->np), RT, 0, st>>>(
      mkP(p), mkS(s), mu, kappa, zl_out, zu_out); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_affine_start_point(const ab_ipm_problem* p, const ab_ipm_state* s,
                           double beta_min, const double* dzl,
                           const double* dzu, double* zl_out, double* zu_out,
                           cudaStream_t st) {
  { k_affine_start_point<<<grid_for(p->np), RT, 0, st>>>(
      mkP(p), mkS(s), beta_min, dzl, dzu, zl_out, zu_out); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_barrier_dphi_kkt(const ab_ipm_problem* p, const ab_ipm_state* s,
                         const double* res, const double* px,
                         const double* diag, double* out, cudaStream_t st,
                         double* scratch) {
  { k_barrier_dphi_kkt<<<kRedBlocks, RT, 0, st>>>(mkP(p), mkS(s), res, px, diag,
                                                scratch); ab::count_launch(); }
  { k_sum1_final<<<1, 32, 0, st>>>(kRedBlocks, scratch, out); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_relax_bounds(int np, const double* lbx, const double* ubx,
                     double* lo, double* hi, double factor, double tol,
                     cudaStream_t st) {
  if (np <= 0) return 0;
  { k_relax_bounds<<<grid_for(np), RT, 0, st>>>(np, lbx, ubx, lo, hi, factor,
                                               tol); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_initialize(const ab_ipm_problem* p, double* xlam, double* zl,
                   double* zu, double* sl, double* su, double kappa1,
                   double kappa2, cudaStream_t st) {
  if (p->np <= 0) return 0;
  { k_initialize<<<grid_for(p->np), RT, 0, st>>>(mkP(p), xlam, zl, zu, sl, su,
                                                kappa1, kappa2); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_seg_reduce(const ab_ipm_problem* p, const ab_ipm_state* s,
                   double tau, const double* grad, const double* px,
                   const double* dzl, const double* dzu, const double* gf,
                   double* out, cudaStream_t st) {
  if (p->ninst <= 0) return 0;
  { k_seg_reduce<<<p->ninst, RT, 0, st>>>(mkP(p), mkS(s), tau, grad, px, dzl,
                                        dzu, gf, out); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_apply_step_seg(const ab_ipm_problem* p, const ab_ipm_state* s,
                       const double* ax, const double* az, const double* dxlam,
                       const double* dzl, const double* dzu, double* xlam_new,
                       double* zl_new, double* zu_new, double* sl_new,
                       double* su_new, cudaStream_t st) {
  long long m = p->n > p->np ? p->n : p->np;
  { k_apply_step_seg<<<grid_for(m), RT, 0, st>>>(mkP(p), mkS(s), ax, az, dxlam,
                                               dzl, dzu, xlam_new, zl_new,
                                               zu_new, sl_new, su_new); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_refine_init(const ab_ipm_problem* p, const ab_ipm_state* s,
                    double mu, const double* grad, const double* rhs_saved,
                    const double* px, double* dzl, double* dzu, double* out,
                    cudaStream_t st, double* scratch, double* seg) {
  if (seg && cudaMemsetAsync(seg, 0, sizeof(double) * p->ninst, st) !=
                 cudaSuccess)
    return AB_ERR_CUDA;
  { k_ir_init<<<kRedBlocks, RT, 0, st>>>(mkP(p), mkS(s), mu, grad, rhs_saved,
                                       px, dzl, dzu, scratch, seg); ab::count_launch(); }
  { k_max2_final<<<1, 64, 0, st>>>(kRedBlocks, scratch, out); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_refine_residual(const ab_ipm_problem* p, const ab_ipm_state* s,
                        double mu, const double* grad, const double* rhs_saved,
                        const double* kpx, const double* px, const double* dzl,
                        const double* dzu, double* e_cond, double* e_zl,
                        double* e_zu, double* out, cudaStream_t st,
                        double* scratch, double* seg) {
  if (seg && cudaMemsetAsync(seg, 0, sizeof(double) * 2 * p->ninst, st) !=
                 cudaSuccess)
    return AB_ERR_CUDA;
  { k_ir_residual<<<kRedBlocks, RT, 0, st>>>(mkP(p), mkS(s), mu, grad, rhs_saved,
                                           kpx, px, dzl, dzu, e_cond, e_zl,
                                           e_zu, scratch, seg); ab::count_launch(); }
  { k_max2_final<<<1, 64, 0, st>>>(kRedBlocks, scratch, out); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

int ipm_refine_update(const ab_ipm_problem* p, const ab_ipm_state* s,
                      const double* corr, const double* e_zl,
                      const double* e_zu, double* px, double* dzl,
                      double* dzu, cudaStream_t st, const int* active) {
  long long m = p->n > p->np ? p->n : p->np;
  { k_ir_update<<<grid_for(m), RT, 0, st>>>(mkP(p), mkS(s), corr, e_zl, e_zu,
                                          px, dzl, dzu, active); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? 0 : AB_ERR_CUDA;
}

long long ipm_scratch_doubles() { return (long long)kRedBlocks * 16 + 64; }

}  // namespace ab

// ---------------------------------------------------------------------------
// Fraction-to-boundary step length without any device allocation.
//
// ab_ipm_max_step needs a scratch array for its per-block partial minima and
// takes it from a buffer the library cudaMalloc's on first use.  Some callers
// cannot let a library allocate device memory: a host that hands the whole
// device to its own caching allocator (PyTorch, a serving runtime with a
// fixed memory plan), code that must not allocate once its iteration loop
// is running, or an embedding where every device buffer is owned by the
// caller.  This variant runs the same two kernels with their scratch taken
// from a fixed array compiled into the library instead.
//
// The array holds one partial per 256 primal entries (the variant launches
// one block per 256 entries, not the fixed grid), at most kNoAllocBlocks
// blocks, so np is limited to kNoAllocBlocks * 256 = 2,097,152 primal
// entries; larger problems are rejected with AB_ERR_CAPACITY.  Every GPU
// that loads the library holds the array (8192 x (2 doubles + 2 ints) =
// 192 KiB) until the process exits.
namespace ab {
namespace {
constexpr int kNoAllocBlocks = 8192;
constexpr int kNoAllocPartials = 2 * kNoAllocBlocks;  // (ax, az) per block

// Doubles [0, 2*kNoAllocBlocks) hold the value partials; the int partials
// follow them (two ints per block, 4 bytes each: kNoAllocBlocks doubles).
static __device__ __align__(256) double g_noalloc_max_step[kNoAllocPartials +
                                                           kNoAllocBlocks];

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[64] = {nullptr};

// Device address of the array on the current device (host code cannot use
// the symbol itself: its host-side name is only a stand-in).  Looked up once
// per device; the first call on a device therefore performs a runtime query
// and should come before any stream capture.
double* noalloc_scratch(int* rc) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    *rc = AB_ERR_CUDA;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_max_step);
    if (e != cudaSuccess || p == nullptr) {
      *rc = AB_ERR_CUDA;
      return nullptr;
    }
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *rc = AB_OK;
  return g_noalloc_ptr[dev];
}
}  // namespace
}  // namespace ab

extern "C" int ab_ipm_max_step_noalloc(const ab_ipm_problem* p,
                                       const ab_ipm_state* s, double tau,
                                       const double* px, const double* dzl,
                                       const double* dzu, double* out,
                                       int* iout, void* stream) {
  // the same argument check as ab_ipm_max_step
  if (ab::ipm_args_bad(p, s) || !out || !iout ||
      (p->np > 0 && (!px || !dzl || !dzu)))
    return AB_ERR_ARG;
  const long long nblocks = ((long long)p->np + ab::RT - 1) / ab::RT;
  if (nblocks > ab::kNoAllocBlocks) {
    std::fprintf(stderr,
                 "ab_ipm_max_step_noalloc: %d primal entries exceed the "
                 "static scratch limit of %d\n",
                 p->np, ab::kNoAllocBlocks * ab::RT);
    return AB_ERR_CAPACITY;
  }
  int rc = AB_OK;
  double* scratch = ab::noalloc_scratch(&rc);
  if (!scratch) return rc;
  const int grid = nblocks > 0 ? (int)nblocks : 1;
  double* pv = scratch;
  int* pi = reinterpret_cast<int*>(scratch + ab::kNoAllocPartials);
  cudaStream_t st = (cudaStream_t)stream;
  // Every block writes its two partials before the final pass reads them,
  // so nothing in the array has to start at zero.
  { ab::k_max_step<<<grid, ab::RT, 0, st>>>(ab::mkP(p), ab::mkS(s), tau, px, dzl,
                                          dzu, pv, pi); ab::count_launch(); }
  { ab::k_max_step_final<<<1, 64, 0, st>>>(grid, p->pidx, pv, pi, out, iout); ab::count_launch(); }
  return cudaGetLastError() == cudaSuccess ? AB_OK : AB_ERR_CUDA;
}

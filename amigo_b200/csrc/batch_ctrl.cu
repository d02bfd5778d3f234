// Device-side decisions of the batched interior-point loop.
//
// The batched engine (amigo_b200/batch_engine.py) runs the interior-point
// iteration of amigo_b200/ipm_driver.py on many independent instances at
// once.  Every decision of an iteration is taken per instance: the
// convergence test and the monotone barrier update (the reference's
// "monotone" strategy, amigo/algorithm/barrier_strategy: reduce mu while
// E_mu <= kappa_eps mu), inertia correction (Algorithm IC,
// amigo/algorithm/inertia_correction.py:261-402), the refinement stopping
// rule, fraction to the boundary and the l1-merit backtracking line search.
// These kernels take those decisions on the device, one thread per
// instance, from the per-instance reductions of ab_ipm_seg_reduce, the
// factorization's per-instance inertia and the per-instance objective, so
// that no per-instance array crosses to the host inside an iteration: the
// host reads only the flags word (is any instance still pending, searching,
// refining; did any retire).
//
// Compiled with --fmad=false: every expression rounds like the same
// expression evaluated in Python floats (mu^1.5 is mu * sqrt(mu) and
// mu^0.25 is sqrt(sqrt(mu)) on both sides; sqrt is correctly rounded).
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/amigo_b200.h"
#include "launch_count.h"

namespace {

constexpr int kT = 128;

__device__ __forceinline__ double pw(double m, double e) {
  if (e == 1.5) return m * sqrt(m);
  if (e == 0.25) return sqrt(sqrt(m));
  if (e == 1.0) return m;
  return pow(m, e);
}

// Complementarity inf-norm for barrier parameter m from the gap-product
// extremes of ab_ipm_seg_reduce (slots 9, 10).
__device__ __forceinline__ double comp_norm(const double* q, double m) {
  return fmax(0.0, fmax(q[9] - m, m - q[10]));
}

__device__ __forceinline__ void flag(int* flags, int i) { atomicOr(flags + i, 1); }

constexpr int kQ = 12;  // per-instance stride of ab_ipm_seg_reduce's output

__global__ void k_converge_barrier(ab_bctl c, ab_bctl_opts o, const double* q) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.ninst) return;
  c.retire[k] = 0;
  if (!c.live[k]) return;
  const double* qk = q + (size_t)k * kQ;
  const double e0 = fmax(fmax(qk[0], qk[1]), comp_norm(qk, 0.0));
  c.e0[k] = e0;
  if (e0 <= o.tol || c.its[k] >= o.max_iter) {
    c.retire[k] = e0 <= o.tol ? 1 : 2;
    c.live[k] = 0;
    flag(c.flags, AB_BCTL_RETIRED);
    return;
  }
  flag(c.flags, AB_BCTL_LIVE);
  double mu = c.mu[k];
  for (int pass = 0; pass < 1000; pass++) {
    const double emu = fmax(fmax(qk[0], qk[1]), comp_norm(qk, mu));
    if (!(emu <= o.kappa_eps * mu && mu > o.mu_min)) break;
    mu = fmax(o.mu_min, fmin(o.kappa_mu * mu, pw(mu, o.theta_mu)));
  }
  c.mu[k] = mu;
}

__global__ void k_ic_begin(ab_bctl c) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.ninst) return;
  c.dw[k] = c.dc[k] = c.dwf[k] = c.dcf[k] = 0.0;
  c.pending[k] = c.live[k];
}

__global__ void k_shift_diag(ab_bctl c, int n, const int* vinst, const double* primal,
                             const double* diag, double* dtot) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = vinst[i];
    const double pr = primal[i];
    const double a = c.dwf[k] * pr;
    const double b = c.dcf[k] * (1.0 - pr);
    dtot[i] = (diag[i] + a) - b;
  }
}

__global__ void k_ic_step(ab_bctl c, ab_bctl_opts o, const int* inertia) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.ninst || !c.pending[k]) return;
  const int npos = inertia[2 * k], nneg = inertia[2 * k + 1];
  if (npos == c.np_each[k] && nneg == c.nc_each[k]) {
    c.pending[k] = 0;
    return;
  }
  c.n_ic[k] += 1;
  if (npos + nneg < c.n_each[k] && c.dc[k] == 0.0) c.dc[k] = o.dc * pw(c.mu[k], o.kappa_c);
  const double dwl = c.dw_last[k];
  double dw = c.dw[k];
  if (dw == 0.0)
    dw = dwl == 0.0 ? o.dw_first : fmax(o.dw_min, o.kw_minus * dwl);
  else
    dw *= dwl == 0.0 ? o.kw_plus_first : o.kw_plus;
  c.dw[k] = dw;
  if (dw <= o.dw_max) {
    c.dwf[k] = dw;
    c.dcf[k] = c.dc[k];
    flag(c.flags, AB_BCTL_IC_PENDING);
  } else {
    c.pending[k] = 0;
  }
}

__global__ void k_ic_check(ab_bctl c, const int* inertia) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.ninst || !c.pending[k]) return;
  if (inertia[2 * k] != c.np_each[k] || inertia[2 * k + 1] != c.nc_each[k])
    flag(c.flags, AB_BCTL_MISMATCH);
}

__global__ void k_ic_end(ab_bctl c) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.ninst) return;
  if (c.live[k] && c.dw[k] > 0.0) c.dw_last[k] = c.dw[k];
}

__global__ void k_ref_init(ab_bctl c, const double* seg) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.ninst) return;
  c.nrm[k] = seg[k];
  c.ratio_old[k] = 1e30;
  c.ratio[k] = 0.0;
  c.on[k] = c.live[k];
}

__global__ void k_ref_step(ab_bctl c, const double* seg, int step) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.ninst) return;
  const double nrm = c.nrm[k];
  const double r = seg[2 * k] / (fmin(seg[2 * k + 1], 1e6 * nrm) + nrm);
  int on = c.on[k];
  if (on) c.ratio[k] = r;
  if (step >= 1 && on && (r < 1e-10 || r > 0.999999999 * c.ratio_old[k])) on = 0;
  c.on[k] = on;
  if (on) {
    c.ratio_old[k] = r;
    flag(c.flags, AB_BCTL_REFINING);
  }
}

__global__ void k_ref_stalled(ab_bctl c) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.ninst) return;
  if (c.live[k] && c.ratio[k] > 1e-10) flag(c.flags, AB_BCTL_STALLED);
}

__global__ void k_mask_update(ab_bctl c, int n, int np, const int* vinst, const int* pinst,
                              double* dx, double* dzl, double* dzu) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    if (!c.live[vinst[i]]) dx[i] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += stride)
    if (!c.live[pinst[i]]) dzl[i] = dzu[i] = 0.0;
}

__global__ void k_ls_begin(ab_bctl c, const double* q, const double* obj) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.ninst) return;
  const double* qk = q + (size_t)k * kQ;
  const int live = c.live[k];
  double nu = c.nu[k];
  if (live) nu = fmax(nu, 1.1 * qk[8]);
  c.nu[k] = nu;
  const double theta0 = qk[3];
  c.phi0[k] = (obj[k] + qk[4]) + nu * theta0;
  c.dphi[k] = qk[7] - nu * theta0;
  c.alpha[k] = live ? qk[5] : 0.0;
  c.az[k] = live ? qk[6] : 0.0;
  c.search[k] = live;
}

__global__ void k_ls_test(ab_bctl c, ab_bctl_opts o, const double* q, const double* obj) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.ninst || !c.search[k]) return;
  const double* qk = q + (size_t)k * kQ;
  const double phi = (obj[k] + qk[4]) + c.nu[k] * qk[3];
  const double alpha = c.alpha[k];
  const double dphi = c.dphi[k];
  const bool accept = phi <= c.phi0[k] + o.armijo * alpha * dphi || !isfinite(dphi);
  if (accept) {
    c.search[k] = 0;
  } else {
    c.alpha[k] = 0.5 * alpha;
    flag(c.flags, AB_BCTL_SEARCHING);
  }
}

__global__ void k_end(ab_bctl c) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.ninst) return;
  if (c.live[k]) c.its[k] += 1;
}

inline int grid(int n) { return n <= 0 ? 1 : (n + kT - 1) / kT; }

inline int done() { return cudaGetLastError() == cudaSuccess ? AB_OK : AB_ERR_CUDA; }

bool bad(const ab_bctl* c) { return !c || c->ninst < 0 || (c->ninst > 0 && !c->flags); }

}  // namespace

extern "C" {

int ab_bctl_clear_flags(const ab_bctl* c, void* stream) {
  if (bad(c)) return AB_ERR_ARG;
  return cudaMemsetAsync(c->flags, 0, AB_BCTL_NFLAGS * sizeof(int), (cudaStream_t)stream) ==
                 cudaSuccess
             ? AB_OK
             : AB_ERR_CUDA;
}

int ab_bctl_converge_barrier(const ab_bctl* c, const ab_bctl_opts* o, const double* q,
                             void* stream) {
  if (bad(c) || !o || !q) return AB_ERR_ARG;
  if (!c->ninst) return AB_OK;
  k_converge_barrier<<<grid(c->ninst), kT, 0, (cudaStream_t)stream>>>(*c, *o, q);
  ab::count_launch();
  return done();
}

int ab_bctl_ic_begin(const ab_bctl* c, void* stream) {
  if (bad(c)) return AB_ERR_ARG;
  if (!c->ninst) return AB_OK;
  k_ic_begin<<<grid(c->ninst), kT, 0, (cudaStream_t)stream>>>(*c);
  ab::count_launch();
  return done();
}

int ab_bctl_shift_diag(const ab_bctl* c, int n, const int* vinst, const double* primal,
                       const double* diag, double* dtot, void* stream) {
  if (bad(c) || n < 0 || (n > 0 && (!vinst || !primal || !diag || !dtot))) return AB_ERR_ARG;
  if (!n) return AB_OK;
  const int g = grid(n) < 4 * 148 ? grid(n) : 4 * 148;
  k_shift_diag<<<g, kT, 0, (cudaStream_t)stream>>>(*c, n, vinst, primal, diag, dtot);
  ab::count_launch();
  return done();
}

int ab_bctl_ic_step(const ab_bctl* c, const ab_bctl_opts* o, const int* inertia,
                    void* stream) {
  if (bad(c) || !o || !inertia) return AB_ERR_ARG;
  if (!c->ninst) return AB_OK;
  k_ic_step<<<grid(c->ninst), kT, 0, (cudaStream_t)stream>>>(*c, *o, inertia);
  ab::count_launch();
  return done();
}

int ab_bctl_ic_check(const ab_bctl* c, const int* inertia, void* stream) {
  if (bad(c) || !inertia) return AB_ERR_ARG;
  if (!c->ninst) return AB_OK;
  k_ic_check<<<grid(c->ninst), kT, 0, (cudaStream_t)stream>>>(*c, inertia);
  ab::count_launch();
  return done();
}

int ab_bctl_ic_end(const ab_bctl* c, void* stream) {
  if (bad(c)) return AB_ERR_ARG;
  if (!c->ninst) return AB_OK;
  k_ic_end<<<grid(c->ninst), kT, 0, (cudaStream_t)stream>>>(*c);
  ab::count_launch();
  return done();
}

int ab_bctl_refine_init(const ab_bctl* c, const double* seg, void* stream) {
  if (bad(c) || !seg) return AB_ERR_ARG;
  if (!c->ninst) return AB_OK;
  k_ref_init<<<grid(c->ninst), kT, 0, (cudaStream_t)stream>>>(*c, seg);
  ab::count_launch();
  return done();
}

int ab_bctl_refine_step(const ab_bctl* c, const double* seg, int step, void* stream) {
  if (bad(c) || !seg) return AB_ERR_ARG;
  if (!c->ninst) return AB_OK;
  k_ref_step<<<grid(c->ninst), kT, 0, (cudaStream_t)stream>>>(*c, seg, step);
  ab::count_launch();
  return done();
}

int ab_bctl_refine_stalled(const ab_bctl* c, void* stream) {
  if (bad(c)) return AB_ERR_ARG;
  if (!c->ninst) return AB_OK;
  k_ref_stalled<<<grid(c->ninst), kT, 0, (cudaStream_t)stream>>>(*c);
  ab::count_launch();
  return done();
}

int ab_bctl_mask_update(const ab_bctl* c, int n, int np, const int* vinst, const int* pinst,
                        double* dx, double* dzl, double* dzu, void* stream) {
  if (bad(c) || n < 0 || np < 0 || !vinst || (np > 0 && !pinst) || !dx ||
      (np > 0 && (!dzl || !dzu)))
    return AB_ERR_ARG;
  const int m = n > np ? n : np;
  if (!m) return AB_OK;
  const int g = grid(m) < 4 * 148 ? grid(m) : 4 * 148;
  k_mask_update<<<g, kT, 0, (cudaStream_t)stream>>>(*c, n, np, vinst, pinst, dx, dzl, dzu);
  ab::count_launch();
  return done();
}

int ab_bctl_ls_begin(const ab_bctl* c, const double* q, const double* obj, void* stream) {
  if (bad(c) || !q || !obj) return AB_ERR_ARG;
  if (!c->ninst) return AB_OK;
  k_ls_begin<<<grid(c->ninst), kT, 0, (cudaStream_t)stream>>>(*c, q, obj);
  ab::count_launch();
  return done();
}

int ab_bctl_ls_test(const ab_bctl* c, const ab_bctl_opts* o, const double* q,
                    const double* obj, void* stream) {
  if (bad(c) || !o || !q || !obj) return AB_ERR_ARG;
  if (!c->ninst) return AB_OK;
  k_ls_test<<<grid(c->ninst), kT, 0, (cudaStream_t)stream>>>(*c, *o, q, obj);
  ab::count_launch();
  return done();
}

int ab_bctl_end(const ab_bctl* c, void* stream) {
  if (bad(c)) return AB_ERR_ARG;
  if (!c->ninst) return AB_OK;
  k_end<<<grid(c->ninst), kT, 0, (cudaStream_t)stream>>>(*c);
  ab::count_launch();
  return done();
}

}  // extern "C"

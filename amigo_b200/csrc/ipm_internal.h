// Host launchers of the IPM vector kernels (ipm_kernels.cu).  `scratch` is
// device memory of at least ipm_scratch_doubles() doubles that holds the
// per-block partial results of the deterministic reductions.
#pragma once
#include <cuda_runtime.h>

#include "../../include/amigo_b200.h"

namespace ab {

// Argument check shared by every IPM entry point: sizes non-negative and
// the index, bound and state arrays present for the sizes given.
inline bool ipm_args_bad(const ab_ipm_problem* p, const ab_ipm_state* s) {
  if (!p || !s) return true;
  if (p->n < 0 || p->np < 0 || p->nc < 0) return true;
  if (p->np > 0 && (!p->pidx || !p->lbx || !p->ubx || !s->zl || !s->zu ||
                    !s->sl || !s->su))
    return true;
  if (p->nc > 0 && (!p->cidx || !p->lbh)) return true;
  return false;
}

__device__ void block_sum2(double a, double b, double* partial);
__device__ void block_max2(double a, double b, double* partial);

long long ipm_scratch_doubles();
int ipm_residual(const ab_ipm_problem* p, const ab_ipm_state* s, double mu,
                 const double* grad, double* res, double* out2,
                 cudaStream_t st, double* scratch);
int ipm_diagonal(const ab_ipm_problem* p, const ab_ipm_state* s, double* diag,
                 cudaStream_t st);
int ipm_bound_dual_step(const ab_ipm_problem* p, const ab_ipm_state* s,
                        double mu, const double* px, double* dzl, double* dzu,
                        cudaStream_t st);
int ipm_max_step(const ab_ipm_problem* p, const ab_ipm_state* s, double tau,
                 const double* px, const double* dzl, const double* dzu,
                 double* out, int* iout, cudaStream_t st, double* scratch);
int ipm_apply_step(const ab_ipm_problem* p, const ab_ipm_state* s, double ax,
                   double az, const double* dxlam, const double* dzl,
                   const double* dzu, double* xlam_new, double* zl_new,
                   double* zu_new, double* sl_new, double* su_new,
                   cudaStream_t st);
int ipm_reductions(const ab_ipm_problem* p, const ab_ipm_state* s, double mu,
                   const double* grad, double* out, cudaStream_t st,
                   double* scratch);
int ipm_barrier_dphi(const ab_ipm_problem* p, const ab_ipm_state* s,
                     double mu, const double* grad, const double* px,
                     double* out, cudaStream_t st, double* scratch);
int ipm_reset_bound_multipliers(const ab_ipm_problem* p,
                                const ab_ipm_state* s, double mu,
                                double kappa, double* zl_out, double* zu_out,
                                cudaStream_t st);
int ipm_affine_start_point(const ab_ipm_problem* p, const ab_ipm_state* s,
                           double beta_min, const double* dzl,
                           const double* dzu, double* zl_out, double* zu_out,
                           cudaStream_t st);

int ipm_barrier_dphi_kkt(const ab_ipm_problem* p, const ab_ipm_state* s,
                         const double* res, const double* px,
                         const double* diag, double* out, cudaStream_t st,
                         double* scratch);
int ipm_relax_bounds(int np, const double* lbx, const double* ubx,
                     double* lo, double* hi, double factor, double tol,
                     cudaStream_t st);
int ipm_initialize(const ab_ipm_problem* p, double* xlam, double* zl,
                   double* zu, double* sl, double* su, double kappa1,
                   double kappa2, cudaStream_t st);

int ipm_seg_reduce(const ab_ipm_problem* p, const ab_ipm_state* s,
                   double tau, const double* grad, const double* px,
                   const double* dzl, const double* dzu, const double* gf,
                   double* out, cudaStream_t st);
int ipm_apply_step_seg(const ab_ipm_problem* p, const ab_ipm_state* s,
                       const double* ax, const double* az, const double* dxlam,
                       const double* dzl, const double* dzu, double* xlam_new,
                       double* zl_new, double* zu_new, double* sl_new,
                       double* su_new, cudaStream_t st);
int ipm_refine_init(const ab_ipm_problem* p, const ab_ipm_state* s,
                    double mu, const double* grad, const double* rhs_saved,
                    const double* px, double* dzl, double* dzu, double* out,
                    cudaStream_t st, double* scratch, double* seg = nullptr);
int ipm_refine_residual(const ab_ipm_problem* p, const ab_ipm_state* s,
                        double mu, const double* grad, const double* rhs_saved,
                        const double* kpx, const double* px, const double* dzl,
                        const double* dzu, double* e_cond, double* e_zl,
                        double* e_zu, double* out, cudaStream_t st,
                        double* scratch, double* seg = nullptr);
int ipm_refine_update(const ab_ipm_problem* p, const ab_ipm_state* s,
                      const double* corr, const double* e_zl,
                      const double* e_zu, double* px, double* dzl,
                      double* dzu, cudaStream_t st,
                      const int* active = nullptr);

int csr_add_diagonal(int n, const int* diag_pos, const double* d,
                     double* vals, cudaStream_t st);
int csr_matvec(int n, const int* rowp, const int* cols, const double* vals,
               const double* x, double* y, cudaStream_t st);

}  // namespace ab

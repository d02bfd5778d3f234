// extern "C" entry points for the IPM vector kernels and CSR utilities
// (include/amigo_b200.h).  The deterministic reductions need a small
// scratch array for block partials.  There is one per (device, stream):
// calls on different streams may overlap, calls on one stream are ordered
// by it.  Each is allocated on first use and kept until process exit.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

#include "../../include/amigo_b200.h"
#include "ipm_internal.h"

namespace {

std::mutex g_scratch_mu;
std::map<std::pair<int, void*>, double*> g_scratch;

double* device_scratch(void* stream) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return nullptr;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  double*& slot = g_scratch[std::make_pair(dev, stream)];
  if (!slot) {
    void* p = nullptr;
    if (cudaMalloc(&p, (size_t)ab::ipm_scratch_doubles() * sizeof(double)) !=
        cudaSuccess)
      return nullptr;
    slot = static_cast<double*>(p);
  }
  return slot;
}

bool bad(const ab_ipm_problem* p, const ab_ipm_state* s) {
  return ab::ipm_args_bad(p, s);
}

}  // namespace

extern "C" {

int ab_ipm_residual(const ab_ipm_problem* p, const ab_ipm_state* s, double mu,
                    const double* grad, double* res, double* out2,
                    void* stream) {
  if (bad(p, s) || (p->n > 0 && (!grad || !res))) return AB_ERR_ARG;
  double* scratch = nullptr;
  if (out2 && !(scratch = device_scratch(stream))) return AB_ERR_CUDA;
  return ab::ipm_residual(p, s, mu, grad, res, out2, (cudaStream_t)stream,
                          scratch);
}

int ab_ipm_diagonal(const ab_ipm_problem* p, const ab_ipm_state* s,
                    double* diag, void* stream) {
  if (bad(p, s) || (p->n > 0 && !diag)) return AB_ERR_ARG;
  return ab::ipm_diagonal(p, s, diag, (cudaStream_t)stream);
}

int ab_ipm_bound_dual_step(const ab_ipm_problem* p, const ab_ipm_state* s,
                           double mu, const double* px, double* dzl,
                           double* dzu, void* stream) {
  if (bad(p, s) || (p->np > 0 && (!px || !dzl || !dzu))) return AB_ERR_ARG;
  return ab::ipm_bound_dual_step(p, s, mu, px, dzl, dzu, (cudaStream_t)stream);
}

int ab_ipm_max_step(const ab_ipm_problem* p, const ab_ipm_state* s,
                    double tau, const double* px, const double* dzl,
                    const double* dzu, double* out, int* iout, void* stream) {
  if (bad(p, s) || !out || !iout || (p->np > 0 && (!px || !dzl || !dzu)))
    return AB_ERR_ARG;
  double* scratch = device_scratch(stream);
  if (!scratch) return AB_ERR_CUDA;
  return ab::ipm_max_step(p, s, tau, px, dzl, dzu, out, iout,
                          (cudaStream_t)stream, scratch);
}

int ab_ipm_apply_step(const ab_ipm_problem* p, const ab_ipm_state* s,
                      double ax, double az, const double* dxlam,
                      const double* dzl, const double* dzu, double* xlam_new,
                      double* zl_new, double* zu_new, double* sl_new,
                      double* su_new, void* stream) {
  if (bad(p, s) || (p->n > 0 && (!s->xlam || !dxlam || !xlam_new)) ||
      (p->np > 0 && (!dzl || !dzu || !zl_new || !zu_new || !sl_new || !su_new)))
    return AB_ERR_ARG;
  return ab::ipm_apply_step(p, s, ax, az, dxlam, dzl, dzu, xlam_new, zl_new,
                            zu_new, sl_new, su_new, (cudaStream_t)stream);
}

int ab_ipm_reductions(const ab_ipm_problem* p, const ab_ipm_state* s,
                      double mu, const double* grad, double* out,
                      void* stream) {
  if (bad(p, s) || !out) return AB_ERR_ARG;
  double* scratch = device_scratch(stream);
  if (!scratch) return AB_ERR_CUDA;
  return ab::ipm_reductions(p, s, mu, grad, out, (cudaStream_t)stream,
                            scratch);
}

int ab_ipm_barrier_dphi(const ab_ipm_problem* p, const ab_ipm_state* s,
                        double mu, const double* grad, const double* px,
                        double* out, void* stream) {
  if (bad(p, s) || !out || (p->np > 0 && (!grad || !px))) return AB_ERR_ARG;
  double* scratch = device_scratch(stream);
  if (!scratch) return AB_ERR_CUDA;
  return ab::ipm_barrier_dphi(p, s, mu, grad, px, out, (cudaStream_t)stream,
                              scratch);
}

int ab_ipm_reset_bound_multipliers(const ab_ipm_problem* p,
                                   const ab_ipm_state* s, double mu,
                                   double kappa, double* zl_out,
                                   double* zu_out, void* stream) {
  if (bad(p, s) || (p->np > 0 && (!zl_out || !zu_out))) return AB_ERR_ARG;
  return ab::ipm_reset_bound_multipliers(p, s, mu, kappa, zl_out, zu_out,
                                         (cudaStream_t)stream);
}

int ab_ipm_affine_start_point(const ab_ipm_problem* p, const ab_ipm_state* s,
                              double beta_min, const double* dzl,
                              const double* dzu, double* zl_out,
                              double* zu_out, void* stream) {
  if (bad(p, s) || (p->np > 0 && (!dzl || !dzu || !zl_out || !zu_out)))
    return AB_ERR_ARG;
  return ab::ipm_affine_start_point(p, s, beta_min, dzl, dzu, zl_out, zu_out,
                                    (cudaStream_t)stream);
}

int ab_ipm_barrier_dphi_kkt(const ab_ipm_problem* p, const ab_ipm_state* s,
                            const double* res, const double* px,
                            const double* diag, double* out, void* stream) {
  if (bad(p, s) || !res || !px || !diag || !out ||
      (p->nc > 0 && !s->xlam))
    return AB_ERR_ARG;
  double* scratch = device_scratch(stream);
  if (!scratch) return AB_ERR_CUDA;
  return ab::ipm_barrier_dphi_kkt(p, s, res, px, diag, out,
                                  (cudaStream_t)stream, scratch);
}

int ab_ipm_relax_bounds(int np, const double* lbx, const double* ubx,
                        double* lbx_out, double* ubx_out, double factor,
                        double constr_viol_tol, void* stream) {
  if (np < 0 || (np > 0 && (!lbx || !ubx || !lbx_out || !ubx_out)))
    return AB_ERR_ARG;
  return ab::ipm_relax_bounds(np, lbx, ubx, lbx_out, ubx_out, factor,
                              constr_viol_tol, (cudaStream_t)stream);
}

int ab_ipm_initialize(const ab_ipm_problem* p, double* xlam, double* zl,
                      double* zu, double* sl, double* su, double kappa1,
                      double kappa2, void* stream) {
  if (!p || p->np < 0 ||
      (p->np > 0 && (!p->pidx || !p->lbx || !p->ubx || !xlam || !zl || !zu ||
                     !sl || !su)))
    return AB_ERR_ARG;
  return ab::ipm_initialize(p, xlam, zl, zu, sl, su, kappa1, kappa2,
                            (cudaStream_t)stream);
}

int ab_ipm_seg_reduce(const ab_ipm_problem* p, const ab_ipm_state* s,
                      double tau, const double* grad, const double* px,
                      const double* dzl, const double* dzu, const double* gf,
                      double* out, void* stream) {
  if (bad(p, s) || !out || p->ninst < 1 || !p->mu_inst || !p->poff ||
      !p->coff)
    return AB_ERR_ARG;
  return ab::ipm_seg_reduce(p, s, tau, grad, px, dzl, dzu, gf, out,
                            (cudaStream_t)stream);
}

int ab_ipm_apply_step_seg(const ab_ipm_problem* p, const ab_ipm_state* s,
                          const double* ax, const double* az,
                          const double* dxlam, const double* dzl,
                          const double* dzu, double* xlam_new, double* zl_new,
                          double* zu_new, double* sl_new, double* su_new,
                          void* stream) {
  if (bad(p, s) || !ax || !az || !p->pinst || !p->vinst || !s->xlam ||
      !dxlam || !xlam_new ||
      (p->np > 0 && (!dzl || !dzu || !zl_new || !zu_new || !sl_new || !su_new)))
    return AB_ERR_ARG;
  return ab::ipm_apply_step_seg(p, s, ax, az, dxlam, dzl, dzu, xlam_new,
                                zl_new, zu_new, sl_new, su_new,
                                (cudaStream_t)stream);
}

int ab_ipm_refine_init(const ab_ipm_problem* p, const ab_ipm_state* s,
                       double mu, const double* grad, const double* rhs_saved,
                       const double* px, double* dzl, double* dzu, double* out,
                       void* stream) {
  if (bad(p, s) || !out || (p->n > 0 && (!grad || !rhs_saved || !px)) ||
      (p->np > 0 && (!dzl || !dzu)))
    return AB_ERR_ARG;
  double* scratch = device_scratch(stream);
  if (!scratch) return AB_ERR_CUDA;
  return ab::ipm_refine_init(p, s, mu, grad, rhs_saved, px, dzl, dzu, out,
                             (cudaStream_t)stream, scratch);
}

int ab_ipm_refine_residual(const ab_ipm_problem* p, const ab_ipm_state* s,
                           double mu, const double* grad,
                           const double* rhs_saved, const double* kpx,
                           const double* px, const double* dzl,
                           const double* dzu, double* e_cond, double* e_zl,
                           double* e_zu, double* out, void* stream) {
  if (bad(p, s) || !out ||
      (p->n > 0 && (!grad || !rhs_saved || !kpx || !px || !e_cond)) ||
      (p->np > 0 && (!dzl || !dzu || !e_zl || !e_zu)))
    return AB_ERR_ARG;
  double* scratch = device_scratch(stream);
  if (!scratch) return AB_ERR_CUDA;
  return ab::ipm_refine_residual(p, s, mu, grad, rhs_saved, kpx, px, dzl, dzu,
                                 e_cond, e_zl, e_zu, out, (cudaStream_t)stream,
                                 scratch);
}

int ab_ipm_refine_update(const ab_ipm_problem* p, const ab_ipm_state* s,
                         const double* corr, const double* e_zl,
                         const double* e_zu, double* px, double* dzl,
                         double* dzu, void* stream) {
  if (bad(p, s) || (p->n > 0 && (!corr || !px)) ||
      (p->np > 0 && (!e_zl || !e_zu || !dzl || !dzu)))
    return AB_ERR_ARG;
  return ab::ipm_refine_update(p, s, corr, e_zl, e_zu, px, dzl, dzu,
                               (cudaStream_t)stream);
}

static bool bad_seg(const ab_ipm_problem* p) {
  return p->ninst < 1 || !p->mu_inst || !p->pinst || !p->vinst;
}

int ab_ipm_refine_init_seg(const ab_ipm_problem* p, const ab_ipm_state* s,
                           const double* grad, const double* rhs_saved,
                           const double* px, double* dzl, double* dzu,
                           double* seg_out, void* stream) {
  if (bad(p, s) || bad_seg(p) || !seg_out ||
      (p->n > 0 && (!grad || !rhs_saved || !px)) ||
      (p->np > 0 && (!dzl || !dzu)))
    return AB_ERR_ARG;
  double* scratch = device_scratch(stream);
  if (!scratch) return AB_ERR_CUDA;
  return ab::ipm_refine_init(p, s, 0.0, grad, rhs_saved, px, dzl, dzu,
                             scratch + ab::ipm_scratch_doubles() - 8,
                             (cudaStream_t)stream, scratch, seg_out);
}

int ab_ipm_refine_residual_seg(const ab_ipm_problem* p, const ab_ipm_state* s,
                               const double* grad, const double* rhs_saved,
                               const double* kpx, const double* px,
                               const double* dzl, const double* dzu,
                               double* e_cond, double* e_zl, double* e_zu,
                               double* seg_out, void* stream) {
  if (bad(p, s) || bad_seg(p) || !seg_out ||
      (p->n > 0 && (!grad || !rhs_saved || !kpx || !px || !e_cond)) ||
      (p->np > 0 && (!dzl || !dzu || !e_zl || !e_zu)))
    return AB_ERR_ARG;
  double* scratch = device_scratch(stream);
  if (!scratch) return AB_ERR_CUDA;
  return ab::ipm_refine_residual(p, s, 0.0, grad, rhs_saved, kpx, px, dzl,
                                 dzu, e_cond, e_zl, e_zu,
                                 scratch + ab::ipm_scratch_doubles() - 8,
                                 (cudaStream_t)stream, scratch, seg_out);
}

int ab_ipm_refine_update_seg(const ab_ipm_problem* p, const ab_ipm_state* s,
                             const int* active, const double* corr,
                             const double* e_zl, const double* e_zu,
                             double* px, double* dzl, double* dzu,
                             void* stream) {
  if (bad(p, s) || bad_seg(p) || !active || (p->n > 0 && (!corr || !px)) ||
      (p->np > 0 && (!e_zl || !e_zu || !dzl || !dzu)))
    return AB_ERR_ARG;
  return ab::ipm_refine_update(p, s, corr, e_zl, e_zu, px, dzl, dzu,
                               (cudaStream_t)stream, active);
}

int ab_csr_add_diagonal(int n, const int* diag_pos, const double* d,
                        double* vals, void* stream) {
  if (n < 0 || (n > 0 && (!diag_pos || !d || !vals))) return AB_ERR_ARG;
  return ab::csr_add_diagonal(n, diag_pos, d, vals, (cudaStream_t)stream);
}

int ab_csr_matvec(int n, const int* rowp, const int* cols, const double* vals,
                  const double* x, double* y, void* stream) {
  if (n < 0 || (n > 0 && (!rowp || !cols || !vals || !x || !y)))
    return AB_ERR_ARG;
  return ab::csr_matvec(n, rowp, cols, vals, x, y, (cudaStream_t)stream);
}

}  // extern "C"

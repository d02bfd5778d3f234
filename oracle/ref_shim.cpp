/*
 * ref_shim.cpp -- C entry points around the reference's own CPU code, built
 * only as the parity checker (test infrastructure, never the product).
 *
 * This file is compiled against the reference's unmodified header-only
 * sources (include/sparse_ldl.h, include/block_amd.h, include/ordering_utils.h,
 * include/csr_matrix.h, include/interior_point_backend.h) by
 * oracle/build_ref.sh, with the single-rank stubs in oracle/ref_stub/ and
 * the BLAS/LAPACK forwarding shim oracle/blas_shim.c.  The output goes to
 * oracle/_ref/libamigo_ref.so, which is git-ignored.
 *
 * The wrappers expose the reference's private symbolic arrays (node_ptr,
 * node_to_var, node_children(_ptr), contrib_ptr/rows, invperm) so that the
 * product's own symbolic analysis can be compared with them bit for bit.
 */
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <deque>
#include <iomanip>
#include <iostream>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <string>
#include <vector>

// The symbolic arrays are private members of SparseLDL; the checker needs to
// read them, so widen access for this translation unit only.
#define private public
#define protected public
#include "sparse_ldl.h"
#include "interior_point_backend.h"
#undef private
#undef protected

using amigo::CSRMat;
using amigo::MemoryLocation;
using amigo::OrderingType;
using LDL = amigo::SparseLDL<double>;

namespace {
struct RefHandle {
  std::shared_ptr<CSRMat<double>> mat;
  std::unique_ptr<LDL> ldl;
  int n = 0, nnz = 0;
};

OrderingType to_order(int order) {
  switch (order) {
    case 0: return OrderingType::NESTED_DISSECTION;
    case 1: return OrderingType::AMD;
    case 2: return OrderingType::MULTI_COLOR;
    default: return OrderingType::NATURAL;
  }
}
}  // namespace

extern "C" {

// Thread count of the bundled OpenBLAS (its pthread pool must not be nested
// inside the reference's OpenMP task region, so the checker runs BLAS
// single-threaded unless asked otherwise).
void scipy_openblas_set_num_threads(int);
void ref_set_blas_threads(int n) { scipy_openblas_set_num_threads(n); }

// order: 0 = NESTED_DISSECTION (identity without METIS), 1 = AMD,
// 2 = MULTI_COLOR, 3 = NATURAL.  solver: 0 = LDL, 1 = CHOLESKY.
void* ref_ldl_create(int n, const int* rowp, const int* cols, int order,
                     double ustab, double pivot_tol, double delay_growth,
                     int solver) {
  auto* h = new RefHandle;
  h->n = n;
  h->nnz = rowp[n];
  h->mat = CSRMat<double>::create_from_csr_data(n, n, h->nnz, rowp, cols,
                                                MemoryLocation::HOST_ONLY);
  h->ldl.reset(new LDL(h->mat, solver ? LDL::SolverType::CHOLESKY
                                       : LDL::SolverType::LDL,
                       ustab, pivot_tol, delay_growth, to_order(order)));
  return h;
}

void ref_ldl_destroy(void* p) { delete static_cast<RefHandle*>(p); }

int ref_ldl_num_nodes(void* p) {
  return static_cast<RefHandle*>(p)->ldl->num_nodes;
}

int ref_ldl_contrib_total(void* p) {
  auto* h = static_cast<RefHandle*>(p);
  return h->ldl->contrib_ptr[h->ldl->num_nodes];
}

// Copies the symbolic arrays.  invperm may be null (NATURAL has none).
int ref_ldl_symbolic(void* p, int* node_ptr, int* node_to_var,
                     int* children_ptr, int* children, int* contrib_ptr,
                     int* contrib_rows, int* invperm) {
  auto* h = static_cast<RefHandle*>(p);
  LDL& s = *h->ldl;
  int nn = s.num_nodes;
  std::copy(s.node_ptr, s.node_ptr + nn + 1, node_ptr);
  std::copy(s.node_to_var, s.node_to_var + h->n, node_to_var);
  std::copy(s.node_children_ptr, s.node_children_ptr + nn + 2, children_ptr);
  std::copy(s.node_children, s.node_children + nn, children);
  std::copy(s.contrib_ptr, s.contrib_ptr + nn + 1, contrib_ptr);
  std::copy(s.contrib_rows, s.contrib_rows + s.contrib_ptr[nn], contrib_rows);
  if (invperm) {
    if (s.invperm) {
      std::copy(s.invperm, s.invperm + h->n, invperm);
    } else {
      for (int i = 0; i < h->n; i++) invperm[i] = i;
    }
  }
  return nn;
}

void ref_ldl_set_values(void* p, const double* vals) {
  auto* h = static_cast<RefHandle*>(p);
  double* data = h->mat->get_data_ptr();
  std::copy(vals, vals + h->nnz, data);
}

int ref_ldl_factor(void* p) { return static_cast<RefHandle*>(p)->ldl->factor(); }

void ref_ldl_inertia(void* p, int* npos, int* nneg) {
  static_cast<RefHandle*>(p)->ldl->get_inertia(npos, nneg);
}

void ref_ldl_solve(void* p, int nrhs, double* x, int ldx) {
  static_cast<RefHandle*>(p)->ldl->solve(nrhs, x, ldx);
}

// Per-node pivot and delay counts of the last numeric factorization.
void ref_ldl_node_pivots(void* p, int* num_pivots, int* num_delayed) {
  auto* h = static_cast<RefHandle*>(p);
  LDL& s = *h->ldl;
  for (int ks = 0; ks < s.num_nodes; ks++) {
    int np = 0, nd = 0;
    s.fact.get_factor(ks, &np, nullptr, &nd, nullptr, nullptr);
    num_pivots[ks] = np;
    num_delayed[ks] = nd;
  }
}

// Standalone ordering (the matrix pattern is copied as SparseLDL does).
void ref_order(int n, const int* rowp, const int* cols, int order, int* perm,
               int* iperm) {
  int *rc = nullptr, *cc = nullptr, *pp = nullptr, *ip = nullptr;
  OrderingType ot = to_order(order);
  amigo::OrderingUtils::copy_for_reorder(ot, n, rowp, cols, &rc, &cc);
  amigo::OrderingUtils::reorder(ot, n, rc, cc, &pp, &ip);
  std::copy(pp, pp + n, perm);
  std::copy(ip, ip + n, iperm);
  delete[] rc;
  delete[] cc;
  delete[] pp;
  delete[] ip;
}

/* ------------------------------------------------------------------ */
/* IPM vector functions (interior_point_backend.h) on raw arrays.      */
/* ------------------------------------------------------------------ */
namespace {
amigo::ipm::ProblemInfo<double> make_info(int np, int nc, const int* pidx,
                                          const int* cidx, const double* lbx,
                                          const double* ubx,
                                          const double* lbh) {
  amigo::ipm::ProblemInfo<double> p;
  p.n_primal = np;
  p.n_constraints = nc;
  p.primal_indices = pidx;
  p.constraint_indices = cidx;
  p.lbx = lbx;
  p.ubx = ubx;
  p.lbh = lbh;
  return p;
}
amigo::ipm::State<const double> make_state(const double* xlam,
                                           const double* zl, const double* zu,
                                           const double* sl,
                                           const double* su) {
  amigo::ipm::State<const double> s;
  s.xlam = xlam;
  s.zl = zl;
  s.zu = zu;
  s.sl = sl;
  s.su = su;
  return s;
}
}  // namespace

#define REF_IPM_ARGS                                                     \
  int np, int nc, const int *pidx, const int *cidx, const double *lbx,   \
      const double *ubx, const double *lbh, const double *xlam,          \
      const double *zl, const double *zu, const double *sl, const double *su
#define REF_IPM_SETUP                                       \
  auto P = make_info(np, nc, pidx, cidx, lbx, ubx, lbh);   \
  auto S = make_state(xlam, zl, zu, sl, su);

void ref_ipm_compute_residual(double mu, REF_IPM_ARGS, const double* grad,
                              double* res) {
  REF_IPM_SETUP
  amigo::ipm::compute_residual(mu, P, S, grad, res);
}

void ref_ipm_compute_residual_and_infeasibility(double mu, REF_IPM_ARGS,
                                                const double* grad,
                                                double* res, double* dual_sq,
                                                double* primal_sq) {
  REF_IPM_SETUP
  amigo::ipm::compute_residual_and_infeasibility(mu, P, S, grad, res, *dual_sq,
                                                 *primal_sq);
}

void ref_ipm_compute_diagonal(REF_IPM_ARGS, double* diag) {
  REF_IPM_SETUP
  amigo::ipm::compute_diagonal(P, S, diag);
}

void ref_ipm_compute_bound_dual_step(double mu, REF_IPM_ARGS,
                                     const double* px, double* dzl,
                                     double* dzu) {
  REF_IPM_SETUP
  amigo::ipm::compute_bound_dual_step(mu, P, S, px, dzl, dzu);
}

void ref_ipm_compute_max_step(double tau, REF_IPM_ARGS, const double* px,
                              const double* dzl, const double* dzu,
                              double* ax, int* xi, double* az, int* zi) {
  REF_IPM_SETUP
  amigo::ipm::compute_max_step(tau, P, S, px, dzl, dzu, *ax, *xi, *az, *zi);
}

void ref_ipm_apply_step(double ax, double az, REF_IPM_ARGS,
                        const double* dxlam, const double* dzl,
                        const double* dzu, double* xlam_new, int n_xlam,
                        double* zl_new, double* zu_new, double* sl_new,
                        double* su_new) {
  REF_IPM_SETUP
  amigo::ipm::apply_step(ax, az, P, S, dxlam, dzl, dzu, xlam_new, n_xlam,
                         zl_new, zu_new, sl_new, su_new);
}

void ref_ipm_compute_complementarity(REF_IPM_ARGS, double* partial_sum,
                                     double* local_min) {
  REF_IPM_SETUP
  amigo::ipm::compute_complementarity(P, S, partial_sum, *local_min);
}

void ref_ipm_compute_kkt_error(double mu, REF_IPM_ARGS, const double* grad,
                               double* dual, double* primal, double* comp) {
  REF_IPM_SETUP
  amigo::ipm::compute_kkt_error(mu, P, S, grad, *dual, *primal, *comp);
}

double ref_ipm_compute_barrier_log_sum(double mu, REF_IPM_ARGS) {
  REF_IPM_SETUP
  return amigo::ipm::compute_barrier_log_sum(mu, P, S);
}

double ref_ipm_compute_barrier_dphi(double mu, REF_IPM_ARGS,
                                    const double* grad, const double* px) {
  REF_IPM_SETUP
  return amigo::ipm::compute_barrier_dphi(mu, P, S, grad, px);
}

void ref_ipm_reset_bound_multipliers(double mu, double kappa, REF_IPM_ARGS,
                                     double* zl_out, double* zu_out) {
  REF_IPM_SETUP
  amigo::ipm::reset_bound_multipliers(mu, kappa, P, S, zl_out, zu_out);
}

void ref_ipm_compute_affine_start_point(double beta_min, REF_IPM_ARGS,
                                        const double* dzl, const double* dzu,
                                        double* zl_out, double* zu_out) {
  REF_IPM_SETUP
  amigo::ipm::compute_affine_start_point(beta_min, P, S, dzl, dzu, zl_out,
                                         zu_out);
}

void ref_ipm_compute_max_comp_deviation(REF_IPM_ARGS, double mu,
                                        double* max_dev) {
  REF_IPM_SETUP
  amigo::ipm::compute_max_comp_deviation(P, S, mu, *max_dev);
}

void ref_ipm_compute_complementarity_sq(REF_IPM_ARGS, double mu, double* sq) {
  REF_IPM_SETUP
  amigo::ipm::compute_complementarity_sq(P, S, mu, *sq);
}

double ref_ipm_compute_constraint_violation_1norm(REF_IPM_ARGS,
                                                  const double* grad) {
  REF_IPM_SETUP
  return amigo::ipm::compute_constraint_violation_1norm(P, S, grad);
}


// The remaining backend functions the reference's InteriorPointOptimizer
// calls (include/interior_point_backend.h:82-201, 539-611).
void ref_ipm_relax_bounds(int np, int nc, const int* pidx, const int* cidx,
                          const double* lbx, const double* ubx,
                          const double* lbh, double* lb_out, double* ub_out,
                          double factor, double tol) {
  auto P = make_info(np, nc, pidx, cidx, lbx, ubx, lbh);
  amigo::ipm::relax_bounds(P, lb_out, ub_out, factor, tol);
}

void ref_ipm_initialize(int np, int nc, const int* pidx, const int* cidx,
                        const double* lbx, const double* ubx, const double* lbh,
                        double mu, double* xlam, double* zl, double* zu,
                        double* sl, double* su) {
  auto P = make_info(np, nc, pidx, cidx, lbx, ubx, lbh);
  amigo::ipm::project_primals_into_interior(P, xlam);
  amigo::ipm::initialize_bound_duals(mu, P, xlam, zl, zu);
  amigo::ipm::initialize_slacks(P, xlam, sl, su);
}

void ref_ipm_compute_kkt_error_sq(REF_IPM_ARGS, const double* grad, double* d,
                                  double* p, double* c) {
  REF_IPM_SETUP
  amigo::ipm::compute_kkt_error_sq(P, S, grad, *d, *p, *c);
}

double ref_ipm_compute_barrier_dphi_from_kkt(REF_IPM_ARGS, const double* res,
                                             const double* px,
                                             const double* diag) {
  REF_IPM_SETUP
  return amigo::ipm::compute_barrier_dphi_from_kkt(P, S, res, px, diag);
}

void ref_ipm_compute_dual_residual_vector(REF_IPM_ARGS, const double* grad,
                                          double* out, int size) {
  REF_IPM_SETUP
  amigo::ipm::compute_dual_residual_vector(P, S, grad, out, size);
}

}  // extern "C"

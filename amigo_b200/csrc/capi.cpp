// extern "C" entry points declared in include/amigo_b200.h (LDL part).
#include <cuda_runtime.h>

#include <cstdio>
#include <new>

#include "../../include/amigo_b200.h"
#include "ldl_internal.h"

struct ab_ldl {
  ab::LdlHandle h;
};

extern "C" {

int ab_ldl_create(int n, const int* rowp, const int* cols, int order,
                  int solver_type, double ustab, double pivot_tol,
                  double delay_growth, ab_ldl_t* out) {
  if (!out || n < 0 || (n > 0 && (!rowp || !cols))) return AB_ERR_ARG;
  *out = nullptr;
  if (solver_type != 0) return AB_ERR_UNSUPPORTED;
  if (order != ab::ORDER_ND && order != ab::ORDER_AMD &&
      order != ab::ORDER_NATURAL)
    return AB_ERR_UNSUPPORTED;
  ab_ldl* H = new (std::nothrow) ab_ldl;
  if (!H) return AB_ERR_CAPACITY;
  ab::LdlHandle& h = H->h;
  // Same clamping as the reference constructor (sparse_ldl.h:73-93).
  if (ustab > 0.5) ustab = 0.5;
  if (ustab < 0.0) ustab = 0.0;
  if (delay_growth < 1.0) delay_growth = 1.0;
  if (delay_growth > 10.0) delay_growth = 10.0;
  h.ustab = ustab;
  h.pivot_tol = pivot_tol;
  h.delay_growth = delay_growth;
  h.order = order;
  if (cudaGetDevice(&h.device) != cudaSuccess) {
    delete H;
    return AB_ERR_CUDA;
  }
  for (int i = 0; i < n; i++)
    for (int p = rowp[i]; p < rowp[i + 1]; p++)
      if (cols[p] < 0 || cols[p] >= n) {
        delete H;
        return AB_ERR_ARG;
      }
  ab::analyze(order, n, rowp, cols, h.sym);
  h.has_plan = true;
  int rc = ab::build_plan(h, rowp, cols);
  if (rc != 0) {
    ab::free_plan(h);
    delete H;
    return rc;
  }
  *out = H;
  return AB_OK;
}

int ab_ldl_analyze(int n, const int* rowp, const int* cols, int order,
                   ab_ldl_t* out) {
  if (!out || n < 0 || (n > 0 && (!rowp || !cols))) return AB_ERR_ARG;
  *out = nullptr;
  if (order != ab::ORDER_ND && order != ab::ORDER_AMD &&
      order != ab::ORDER_NATURAL)
    return AB_ERR_UNSUPPORTED;
  for (int i = 0; i < n; i++)
    for (int p = rowp[i]; p < rowp[i + 1]; p++)
      if (cols[p] < 0 || cols[p] >= n) return AB_ERR_ARG;
  ab_ldl* H = new (std::nothrow) ab_ldl;
  if (!H) return AB_ERR_CAPACITY;
  H->h.order = order;
  ab::analyze(order, n, rowp, cols, H->h.sym);
  H->h.has_plan = false;
  *out = H;
  return AB_OK;
}

int ab_ldl_destroy(ab_ldl_t H) {
  if (!H) return AB_OK;
  if (H->h.has_plan) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(H->h.device);
    ab::free_plan(H->h);
    cudaSetDevice(prev);
  }
  delete H;
  return AB_OK;
}

int ab_ldl_symbolic_sizes(ab_ldl_t H, int* num_nodes, int* contrib_total) {
  if (!H) return AB_ERR_ARG;
  if (num_nodes) *num_nodes = H->h.sym.num_nodes;
  if (contrib_total) *contrib_total = (int)H->h.sym.contrib_rows.size();
  return AB_OK;
}

int ab_ldl_symbolic_arrays(ab_ldl_t H, int* node_ptr, int* node_to_var,
                           int* children_ptr, int* children, int* contrib_ptr,
                           int* contrib_rows, int* invperm) {
  if (!H) return AB_ERR_ARG;
  const ab::SymbolicTree& T = H->h.sym;
  auto cp = [](const std::vector<int>& v, int* dst) {
    if (dst)
      for (size_t i = 0; i < v.size(); i++) dst[i] = v[i];
  };
  cp(T.node_ptr, node_ptr);
  cp(T.node_to_var, node_to_var);
  cp(T.children_ptr, children_ptr);
  cp(T.children, children);
  cp(T.contrib_ptr, contrib_ptr);
  cp(T.contrib_rows, contrib_rows);
  cp(T.invperm, invperm);
  return AB_OK;
}

int ab_ldl_factor(ab_ldl_t H, const double* d_vals, void* stream) {
  if (!H || (!d_vals && H->h.d.nnz > 0)) return AB_ERR_ARG;
  if (!H->h.has_plan) return AB_ERR_UNSUPPORTED;
  if (H->h.sym.n == 0) {
    H->h.factored = true;
    return AB_OK;
  }
  H->h.factored = false;
  return ab::factor_numeric(H->h, d_vals, (cudaStream_t)stream);
}

int ab_ldl_inertia(ab_ldl_t H, void* stream, int* npos, int* nneg) {
  if (!H || !npos || !nneg) return AB_ERR_ARG;
  if (!H->h.factored) return AB_ERR_NOT_FACTORED;
  if (H->h.sym.n == 0) {
    *npos = *nneg = 0;
    return AB_OK;
  }
  int v[2];
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(v, H->h.d.inertia, 2 * sizeof(int),
                      cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return AB_ERR_CUDA;
  *npos = v[0];
  *nneg = v[1];
  return AB_OK;
}

int ab_ldl_solve(ab_ldl_t H, double* d_x, int nrhs, int ldx, void* stream) {
  if (!H || nrhs < 0 || ldx < H->h.sym.n) return AB_ERR_ARG;
  if (!H->h.factored) return AB_ERR_NOT_FACTORED;
  if (nrhs == 0 || H->h.sym.n == 0) return AB_OK;
  if (!d_x) return AB_ERR_ARG;
  return ab::solve_numeric(H->h, d_x, nrhs, ldx, (cudaStream_t)stream);
}

int ab_ldl_stats(ab_ldl_t H, void* stream, double* flops,
                 double* factor_entries, int* max_front, int* num_delayed,
                 int* levels) {
  (void)stream;
  if (!H) return AB_ERR_ARG;
  if (!H->h.factored) return AB_ERR_NOT_FACTORED;
  const ab::LdlHandle& h = H->h;
  double fl = 0.0, fe = 0.0;
  int mf = 0, nd = 0;
  for (size_t k = 0; k < h.h_f.size(); k++) {
    double p = h.h_npiv[k], c = h.h_f[k] - h.h_npiv[k];
    fl += p * p * p / 3.0 + p * p * c + p * c * c;
    fe += (double)h.h_f[k] * p;
    if (h.h_f[k] > mf) mf = h.h_f[k];
    nd += h.h_ndel[k];
  }
  if (flops) *flops = fl;
  if (factor_entries) *factor_entries = fe;
  if (max_front) *max_front = mf;
  if (num_delayed) *num_delayed = nd;
  if (levels) *levels = h.d.num_levels;
  return AB_OK;
}

int ab_ldl_node_pivots(ab_ldl_t H, void* stream, int* num_pivots,
                       int* num_delayed) {
  (void)stream;
  if (!H) return AB_ERR_ARG;
  if (!H->h.factored) return AB_ERR_NOT_FACTORED;
  for (size_t k = 0; k < H->h.h_npiv.size(); k++) {
    if (num_pivots) num_pivots[k] = H->h.h_npiv[k];
    if (num_delayed) num_delayed[k] = H->h.h_ndel[k];
  }
  return AB_OK;
}

}  // extern "C"

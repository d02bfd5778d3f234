// Static device plan of the multifrontal factorization (host side).
//
// From the symbolic tree this builds, once per sparsity pattern:
//   * the level schedule (height in the assembly tree: leaves are level 0),
//     so that all fronts of one level are factored by one launch;
//   * for each node, the list of CSR entries A(i, var) with var a node
//     variable and i at or below it in the elimination order, together with
//     the static front row of i (node variables first, then contribution
//     rows) -- the same entries the reference assembles in
//     assemble_front_matrix (include/sparse_ldl.h:1004-1074);
//   * for each node, the static position of every contribution row inside
//     its parent's front, used by extend-add (include/sparse_ldl.h:1076-1150).
// Front rows shift at run time by the number of delayed pivots a front
// receives; the device adds that shift.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "../../include/amigo_b200.h"
#include "ldl_internal.h"

namespace ab {

#define PLAN_CUDA(call)                                             \
  do {                                                              \
    cudaError_t e__ = (call);                                       \
    if (e__ != cudaSuccess) {                                       \
      std::fprintf(stderr, "amigo_b200: %s failed: %s\n", #call,    \
                   cudaGetErrorString(e__));                        \
      return -2;                                                    \
    }                                                               \
  } while (0)

template <typename T>
static int upload(T** dptr, const std::vector<T>& v) {
  size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(T);
  PLAN_CUDA(cudaMalloc((void**)dptr, bytes));
  if (!v.empty())
    PLAN_CUDA(cudaMemcpy(*dptr, v.data(), v.size() * sizeof(T),
                         cudaMemcpyHostToDevice));
  return 0;
}

template <typename T>
static int zalloc(T** dptr, size_t count) {
  PLAN_CUDA(cudaMalloc((void**)dptr, std::max<size_t>(count, 1) * sizeof(T)));
  PLAN_CUDA(cudaMemset(*dptr, 0, std::max<size_t>(count, 1) * sizeof(T)));
  return 0;
}

int build_plan(LdlHandle& h, const int* rowp, const int* cols) {
  const SymbolicTree& T = h.sym;
  const int n = T.n, nn = T.num_nodes;
  DevicePlan& d = h.d;
  d.nprob = std::max(1, (int)h.prob_node_ptr.size() - 1);
  if (d.nprob > 1) {
    std::vector<int> np(nn);
    for (int p = 0; p < d.nprob; p++)
      for (int k = h.prob_node_ptr[p]; k < h.prob_node_ptr[p + 1]; k++) np[k] = p;
    if (upload(&d.node_prob, np)) return -2;
  }
  d.n = n;
  d.nn = nn;
  d.nnz = rowp[n];

  // Reject repeated column indices inside a row: the device assembly adds
  // each CSR entry with a plain store-add, one thread per target.
  {
    std::vector<int> seen(n, -1);
    for (int i = 0; i < n; i++)
      for (int p = rowp[i]; p < rowp[i + 1]; p++) {
        int j = cols[p];
        if (j < 0 || j >= n) return -1;
        if (seen[j] == i) return -4;
        seen[j] = i;
      }
  }

  h.h_ns.resize(nn);
  h.h_nc.resize(nn);
  std::vector<int> level(nn, 0);
  for (int k = 0; k < nn; k++) {
    h.h_ns[k] = T.node_ptr[k + 1] - T.node_ptr[k];
    h.h_nc[k] = T.contrib_ptr[k + 1] - T.contrib_ptr[k];
    int lv = 0;
    for (int q = T.children_ptr[k]; q < T.children_ptr[k + 1]; q++)
      lv = std::max(lv, level[T.children[q]] + 1);
    level[k] = lv;
  }
  int L = 0;
  for (int k = 0; k < nn; k++) L = std::max(L, level[k] + 1);
  d.num_levels = L;
  h.level_ptr.assign(L + 1, 0);
  for (int k = 0; k < nn; k++) h.level_ptr[level[k] + 1]++;
  for (int l = 0; l < L; l++) h.level_ptr[l + 1] += h.level_ptr[l];
  h.level_nodes.assign(nn, 0);
  {
    std::vector<int> fill(h.level_ptr.begin(), h.level_ptr.end() - 1);
    for (int k = 0; k < nn; k++) h.level_nodes[fill[level[k]]++] = k;
  }
  h.level_max_f.assign(L, 0);
  h.f_static_total = 0;
  h.i_static_total = 0;
  for (int k = 0; k < nn; k++) {
    long long f = h.h_ns[k] + h.h_nc[k];
    h.level_max_f[level[k]] = std::max<int>(h.level_max_f[level[k]], (int)f);
    h.f_static_total += f * f + f * kPanel + 8;
    h.i_static_total += 4 * f + 16;
  }

  // Assembly map of A and the extend-add map.
  std::vector<int> pos_of(n, -1);
  std::vector<int> amap_ptr(nn + 1, 0), amap_pos, amap_row, amap_col;
  std::vector<int> cmap(T.contrib_ptr[nn], -1);
  const int* ip = T.invperm.data();
  auto mark_front = [&](int k, int val_sign) {
    const int ns = T.node_ptr[k + 1] - T.node_ptr[k];
    for (int j = 0; j < ns; j++)
      pos_of[T.node_to_var[T.node_ptr[k] + j]] = val_sign ? j : -1;
    for (int t = T.contrib_ptr[k]; t < T.contrib_ptr[k + 1]; t++)
      pos_of[T.contrib_rows[t]] = val_sign ? ns + (t - T.contrib_ptr[k]) : -1;
  };
  for (int k = 0; k < nn; k++) {
    mark_front(k, 1);
    const int ns = h.h_ns[k];
    for (int j = 0; j < ns; j++) {
      const int var = T.node_to_var[T.node_ptr[k] + j];
      const int pj = ip[var];
      for (int p = rowp[var]; p < rowp[var + 1]; p++) {
        const int i = cols[p];
        if (ip[i] < pj) continue;
        const int r = pos_of[i];
        if (r < 0) continue;
        amap_pos.push_back(p);
        amap_row.push_back(r);
        amap_col.push_back(j);
      }
    }
    amap_ptr[k + 1] = (int)amap_pos.size();
    // Children map into this front.
    for (int q = T.children_ptr[k]; q < T.children_ptr[k + 1]; q++) {
      const int c = T.children[q];
      for (int t = T.contrib_ptr[c]; t < T.contrib_ptr[c + 1]; t++) {
        int r = pos_of[T.contrib_rows[t]];
        if (r < 0) {
          std::fprintf(stderr, "amigo_b200: contribution row outside parent\n");
          mark_front(k, 0);
          return -1;
        }
        cmap[t] = r;
      }
    }
    mark_front(k, 0);
  }

  // Launch schedule: per level, the fronts that fit the shared-memory kernel
  // (by static size) first, then the large ones.
  std::vector<int> sched_nodes;
  sched_nodes.reserve(nn);
  h.sched.assign(L, LevelSchedule());
  for (int l = 0; l < L; l++) {
    LevelSchedule& S = h.sched[l];
    std::vector<int> small, big;
    for (int q = h.level_ptr[l]; q < h.level_ptr[l + 1]; q++) {
      const int k = h.level_nodes[q];
      const long long f = h.h_ns[k] + h.h_nc[k];
      const long long fm = f + 16;
      if ((fm * fm + fm * kPanel) * 8 <= kMaxDynSmem) {
        small.push_back(k);
        S.small_max_f = std::max<int>(S.small_max_f, (int)f);
      } else {
        big.push_back(k);
        S.big_max_f = std::max<int>(S.big_max_f, (int)f);
        S.big_max_fs = std::max<int>(S.big_max_fs, h.h_ns[k]);
        S.big_max_kids = std::max<int>(
            S.big_max_kids, T.children_ptr[k + 1] - T.children_ptr[k]);
        S.big_max_amap = std::max<long long>(
            S.big_max_amap, (long long)amap_ptr[k + 1] - amap_ptr[k]);
      }
    }
    S.small_begin = (int)sched_nodes.size();
    S.nsmall = (int)small.size();
    sched_nodes.insert(sched_nodes.end(), small.begin(), small.end());
    S.big_begin = (int)sched_nodes.size();
    S.nbig = (int)big.size();
    sched_nodes.insert(sched_nodes.end(), big.begin(), big.end());
  }

  std::vector<int> ns_v(h.h_ns), nc_v(h.h_nc);
  std::vector<int> kid_ptr(T.children_ptr.begin(), T.children_ptr.begin() + nn + 1);
  int rc = 0;
  rc |= upload(&d.ns, ns_v);
  rc |= upload(&d.nc, nc_v);
  rc |= upload(&d.var_ptr, T.node_ptr);
  rc |= upload(&d.vars, T.node_to_var);
  rc |= upload(&d.cptr, T.contrib_ptr);
  rc |= upload(&d.crows, T.contrib_rows);
  rc |= upload(&d.cmap, cmap);
  rc |= upload(&d.kid_ptr, kid_ptr);
  rc |= upload(&d.kids, T.children);
  rc |= upload(&d.amap_ptr, amap_ptr);
  rc |= upload(&d.amap_pos, amap_pos);
  rc |= upload(&d.amap_row, amap_row);
  rc |= upload(&d.amap_col, amap_col);
  rc |= upload(&d.level_nodes, h.level_nodes);
  rc |= upload(&d.sched_nodes, sched_nodes);
  rc |= zalloc(&d.pstate, 4 * (size_t)nn);
  rc |= zalloc(&d.scratch_int, 4);
  rc |= zalloc(&d.f, nn);
  rc |= zalloc(&d.npiv, nn);
  rc |= zalloc(&d.ndel, nn);
  rc |= zalloc(&d.ndin, nn);
  rc |= zalloc(&d.foff, nn);
  rc |= zalloc(&d.ioff, nn);
  rc |= zalloc(&d.inertia, 2 * (size_t)std::max(d.nprob, 1));
  rc |= zalloc(&d.status, 1);
  rc |= zalloc(&d.counters, 2);
  if (rc) return -2;

  // Pools: delay_growth times the static front sizes, capped by what the
  // device has free (keeping a reserve for the caller's vectors); the
  // static size itself must fit.
  double g = std::max(1.0, h.delay_growth);
  d.icap = (long long)(g * (double)h.i_static_total) + 4096;
  size_t free_b = 0, total_b = 0;
  PLAN_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const long long reserve = (long long)(total_b / 20) + d.icap * 4;
  const long long budget = ((long long)free_b - reserve) / 8;
  const long long fmin = h.f_static_total + 4096;
  if (fmin > budget) {
    std::fprintf(stderr, "amigo_b200: the fronts need %.1f GB, %.1f GB free\n",
                 fmin * 8e-9, free_b * 1e-9);
    return AB_ERR_CAPACITY;
  }
  d.fcap = std::min<long long>((long long)(g * (double)h.f_static_total) + 4096,
                               budget);
  PLAN_CUDA(cudaMalloc((void**)&d.fpool, (size_t)d.fcap * sizeof(double)));
  PLAN_CUDA(cudaMalloc((void**)&d.ipool, (size_t)d.icap * sizeof(int)));
  PLAN_CUDA(cudaMalloc((void**)&h.uoff, (size_t)std::max(nn, 1) * sizeof(long long)));
  return 0;
}

void free_plan(LdlHandle& h) {
  DevicePlan& d = h.d;
  void* ptrs[] = {d.ns, d.nc, d.var_ptr, d.vars, d.cptr, d.crows, d.cmap,
                  d.kid_ptr, d.kids, d.amap_ptr, d.amap_pos, d.amap_row,
                  d.amap_col, d.level_nodes, d.sched_nodes, d.pstate,
                  d.scratch_int, d.f, d.npiv, d.ndel, d.ndin,
                  d.foff, d.ioff, d.inertia, d.node_prob, d.status,
                  d.counters, d.fpool,
                  d.ipool, h.ubuf, h.uoff, h.sv_nodes, h.sv_state, h.cl_scratch,
                  h.sv_bq, h.sv_dep, h.sv_done, h.sv_ctr, h.sv_err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  d = DevicePlan();
  h.cl_scratch = nullptr;
  h.cl_scratch_bytes = 0;
  h.sv_bq = h.sv_dep = h.sv_err = nullptr;
  h.sv_done = h.sv_ctr = nullptr;
  h.sv_qlevels = h.sv_qcount = 0;
  h.ubuf = nullptr;
  h.uoff = nullptr;
  h.sv_nodes = nullptr;
  h.sv_state = nullptr;
  h.solve_epoch = -1;
}

}  // namespace ab

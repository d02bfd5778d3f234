// extern "C" entry points declared in include/amigo_b200.h (LDL part).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <unordered_map>
#include <cstdio>
#include <new>
#include <vector>

#include "../../include/amigo_b200.h"
#include "launch_count.h"
#include "ldl_internal.h"

namespace ab {
namespace {
std::atomic<long long> g_launches{0};
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace ab

struct ab_ldl {
  ab::LdlHandle h;
};

// Symbolic analyses of the batched handles are cached by pattern: a
// request stream of problems that share a pattern (e.g. trajectories with
// the same number of intervals) analyses each pattern once.  Keyed by the
// ordering, n, nnz and a 64-bit FNV-1a hash of rowp and cols; the stored
// pattern is compared in full before a hit is used.
namespace {
struct SymKey {
  int order, n;
  long long nnz;
  unsigned long long hash;
  bool operator==(const SymKey& o) const {
    return order == o.order && n == o.n && nnz == o.nnz && hash == o.hash;
  }
};
struct SymKeyHash {
  size_t operator()(const SymKey& k) const {
    return (size_t)(k.hash ^ ((unsigned long long)k.n << 1) ^
                    (unsigned long long)k.order);
  }
};
struct SymEntry {
  std::vector<int> rowp, cols;
  ab::SymbolicTree tree;
};
std::mutex g_sym_mutex;
std::unordered_map<SymKey, SymEntry, SymKeyHash> g_sym_cache;
constexpr size_t kSymCacheMax = 4096;

unsigned long long fnv1a(const int* a, long long len, unsigned long long h) {
  for (long long i = 0; i < len; i++) {
    h ^= (unsigned int)a[i];
    h *= 1099511628211ull;
  }
  return h;
}

void cached_analyze(int order, int n, const int* rowp, const int* cols,
                    ab::SymbolicTree& out) {
  const long long nnz = rowp[n];
  unsigned long long hh = fnv1a(rowp, n + 1, 1469598103934665603ull);
  hh = fnv1a(cols, nnz, hh);
  const SymKey key{order, n, nnz, hh};
  {
    std::lock_guard<std::mutex> lock(g_sym_mutex);
    auto it = g_sym_cache.find(key);
    if (it != g_sym_cache.end() &&
        std::equal(rowp, rowp + n + 1, it->second.rowp.begin()) &&
        std::equal(cols, cols + nnz, it->second.cols.begin())) {
      out = it->second.tree;
      return;
    }
  }
  ab::analyze(order, n, rowp, cols, out);
  std::lock_guard<std::mutex> lock(g_sym_mutex);
  if (g_sym_cache.size() >= kSymCacheMax) g_sym_cache.clear();
  SymEntry e;
  e.rowp.assign(rowp, rowp + n + 1);
  e.cols.assign(cols, cols + nnz);
  e.tree = out;
  g_sym_cache[key] = std::move(e);
}
}  // namespace

extern "C" {

long long ab_launch_count(void) { return ab::g_launches.load(); }

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

int ab_ldl_mem_estimate(ab_ldl_t H, int precision, double delay_growth,
                        int nrhs, long long* bytes) {
  if (!H || !bytes || (precision != 32 && precision != 64) || nrhs < 0)
    return AB_ERR_ARG;
  const ab::SymbolicTree& T = H->h.sym;
  const double g = delay_growth > 1.0 ? delay_growth : 1.0;
  const long long el = precision == 32 ? 4 : 8;
  long long fronts = 0, ints = 0, fsum = 0, csum = 0;
  for (int k = 0; k < T.num_nodes; k++) {
    const long long ns = T.node_ptr[k + 1] - T.node_ptr[k];
    const long long nc = T.contrib_ptr[k + 1] - T.contrib_ptr[k];
    const long long f = ns + nc;
    fronts += f * f + f * ab::kPanel + 8;
    ints += 4 * f + 16;
    fsum += f;
    csum += nc;
  }
  // front pool (in its element size, with room for delayed pivots), the
  // int pool, the static plan (per-node arrays, contribution rows and their
  // parent map, the assembly map of A: three ints per entry of the
  // supernodes' columns, bounded by the fronts' fully-summed areas) and
  // the solve's update vectors
  long long plan = 64LL * (T.num_nodes + 1) + 8LL * csum + 4LL * T.n;
  long long amap = 0;
  for (int k = 0; k < T.num_nodes; k++) {
    const long long ns = T.node_ptr[k + 1] - T.node_ptr[k];
    const long long nc = T.contrib_ptr[k + 1] - T.contrib_ptr[k];
    amap += ns * (ns + nc);
  }
  plan += 12LL * amap;
  const long long solve = 8LL * fsum * (nrhs > 0 ? nrhs : 1);
  // global scratch of the cluster panel for fronts past shared memory: W
  // and L rows of NB columns for every CTA of a cluster of up to 16, with
  // each CTA's rows rounded up to whole 32-row groups (bounded by the sum
  // over those fronts)
  long long clg = 0;
  for (int k = 0; k < T.num_nodes; k++) {
    const long long f = (T.node_ptr[k + 1] - T.node_ptr[k]) +
                        (T.contrib_ptr[k + 1] - T.contrib_ptr[k]);
    if (f + 64 > 3072) clg += 2LL * ab::kPanel * (f + 64 + 16 * 32) * el;
  }
  *bytes = (long long)(g * (double)(fronts * el)) + (long long)(g * (double)(ints * 4)) +
           plan + solve + clg;
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

int ab_ldl_set_solve_queue(ab_ldl_t H, int mode) {
  if (!H || mode < 0 || mode > 3) return AB_ERR_ARG;
  H->h.solve_queue = mode;
  return AB_OK;
}

int ab_ldl_solve_status(ab_ldl_t H, void* stream) {
  if (!H) return AB_ERR_ARG;
  if (!H->h.sv_err) return AB_OK;
  int e = 0;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(&e, H->h.sv_err, sizeof(int), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return AB_ERR_CUDA;
  if (e) {
    cudaMemsetAsync(H->h.sv_err, 0, sizeof(int), s);
    return AB_ERR_CUDA;
  }
  return AB_OK;
}

int ab_ldl_inertia_device(ab_ldl_t H, const int** out) {
  if (!H || !out) return AB_ERR_ARG;
  if (!H->h.factored) return AB_ERR_NOT_FACTORED;
  if (!H->h.has_plan) return AB_ERR_UNSUPPORTED;
  *out = H->h.d.inertia;
  return AB_OK;
}

int ab_ldl_batch_inertia(ab_ldl_t H, void* stream, int* npos, int* nneg) {
  if (!H || !npos || !nneg) return AB_ERR_ARG;
  if (!H->h.factored) return AB_ERR_NOT_FACTORED;
  const int np = H->h.d.nprob;
  if (H->h.sym.n == 0) {
    for (int p = 0; p < np; p++) npos[p] = nneg[p] = 0;
    return AB_OK;
  }
  std::vector<int> v(2 * (size_t)np);
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(v.data(), H->h.d.inertia, 2 * sizeof(int) * np,
                      cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return AB_ERR_CUDA;
  for (int p = 0; p < np; p++) {
    npos[p] = v[2 * p];
    nneg[p] = v[2 * p + 1];
  }
  return AB_OK;
}

int ab_ldl_inertia(ab_ldl_t H, void* stream, int* npos, int* nneg) {
  if (!H || !npos || !nneg) return AB_ERR_ARG;
  if (!H->h.factored) return AB_ERR_NOT_FACTORED;
  const int np = H->h.has_plan ? H->h.d.nprob : 1;
  std::vector<int> a(np), b(np);
  int rc = ab_ldl_batch_inertia(H, stream, a.data(), b.data());
  if (rc != AB_OK) return rc;
  *npos = *nneg = 0;
  for (int p = 0; p < np; p++) {
    *npos += a[p];
    *nneg += b[p];
  }
  return AB_OK;
}

// Merge per-problem symbolic trees into one block-diagonal tree: node,
// variable and contribution indices are offset, every problem keeps its own
// (reference-identical) ordering and supernodes, and the roots of all
// problems are listed at the tail of the children array.
static void merge_trees(const std::vector<ab::SymbolicTree>& P,
                        ab::SymbolicTree& M, std::vector<int>& node_ptr_p,
                        std::vector<int>& var_ptr_p) {
  M = ab::SymbolicTree();
  int n = 0, nn = 0, nc = 0;
  node_ptr_p.assign(1, 0);
  var_ptr_p.assign(1, 0);
  for (const auto& T : P) {
    n += T.n;
    nn += T.num_nodes;
    nc += (int)T.contrib_rows.size();
    node_ptr_p.push_back(nn);
    var_ptr_p.push_back(n);
  }
  M.n = n;
  M.num_nodes = nn;
  M.permuted = true;
  M.invperm.reserve(n);
  M.node_ptr.assign(1, 0);
  M.node_to_var.reserve(n);
  M.contrib_ptr.assign(1, 0);
  M.contrib_rows.reserve(nc);
  M.node_parent.reserve(nn);
  std::vector<int> kids_of(nn + 1, 0);  // counts per parent
  std::vector<int> roots;
  for (size_t p = 0; p < P.size(); p++) {
    const auto& T = P[p];
    const int vo = var_ptr_p[p], no = node_ptr_p[p];
    for (int i = 0; i < T.n; i++) M.invperm.push_back(vo + T.invperm[i]);
    for (int k = 0; k < T.num_nodes; k++)
      M.node_ptr.push_back(vo + T.node_ptr[k + 1]);
    for (int v : T.node_to_var) M.node_to_var.push_back(vo + v);
    const int cbase = M.contrib_ptr.back();
    for (int k = 0; k < T.num_nodes; k++)
      M.contrib_ptr.push_back(cbase + T.contrib_ptr[k + 1]);
    for (int r : T.contrib_rows) M.contrib_rows.push_back(vo + r);
    for (int k = 0; k < T.num_nodes; k++) {
      const int par = T.node_parent[k];
      M.node_parent.push_back(par >= 0 ? no + par : -1);
    }
  }
  // children lists: same construction as the per-problem ones
  M.children_ptr.assign(nn + 2, 0);
  M.children.assign(nn, 0);
  for (int i = 0; i < nn; i++)
    M.children_ptr[(M.node_parent[i] != -1 ? M.node_parent[i] : nn) + 1]++;
  for (int i = 0; i < nn + 1; i++) M.children_ptr[i + 1] += M.children_ptr[i];
  std::vector<int> fill(M.children_ptr.begin(), M.children_ptr.end() - 1);
  for (int i = 0; i < nn; i++) {
    const int slot = M.node_parent[i] != -1 ? M.node_parent[i] : nn;
    M.children[fill[slot]++] = i;
  }
  (void)kids_of;
  (void)roots;
}

int ab_ldl_batch_create(int nprob, const int* n, const int* const* rowp,
                        const int* const* cols, int order, int solver_type,
                        double ustab, double pivot_tol, double delay_growth,
                        ab_ldl_t* out) {
  if (!out || nprob < 1 || !n || !rowp || !cols) return AB_ERR_ARG;
  *out = nullptr;
  if (solver_type != 0) return AB_ERR_UNSUPPORTED;
  if (order != ab::ORDER_ND && order != ab::ORDER_AMD &&
      order != ab::ORDER_NATURAL)
    return AB_ERR_UNSUPPORTED;
  for (int p = 0; p < nprob; p++) {
    if (n[p] < 1 || !rowp[p] || !cols[p]) return AB_ERR_ARG;
    for (int i = 0; i < n[p]; i++)
      for (int q = rowp[p][i]; q < rowp[p][i + 1]; q++)
        if (cols[p][q] < 0 || cols[p][q] >= n[p]) return AB_ERR_ARG;
  }
  ab_ldl* H = new (std::nothrow) ab_ldl;
  if (!H) return AB_ERR_CAPACITY;
  ab::LdlHandle& h = H->h;
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
  std::vector<ab::SymbolicTree> trees(nprob);
  for (int p = 0; p < nprob; p++)
    cached_analyze(order, n[p], rowp[p], cols[p], trees[p]);
  merge_trees(trees, h.sym, h.prob_node_ptr, h.prob_var_ptr);
  // block-diagonal CSR of all problems
  std::vector<int> mr(1, 0), mc;
  h.prob_nnz_ptr.assign(1, 0);
  for (int p = 0; p < nprob; p++) {
    const int vo = h.prob_var_ptr[p];
    const int base = mr.back();
    for (int i = 0; i < n[p]; i++) mr.push_back(base + rowp[p][i + 1]);
    for (int q = 0; q < rowp[p][n[p]]; q++) mc.push_back(vo + cols[p][q]);
    h.prob_nnz_ptr.push_back(mr.back());
  }
  h.has_plan = true;
  int rc = ab::build_plan(h, mr.data(), mc.data());
  if (rc != 0) {
    ab::free_plan(h);
    delete H;
    return rc;
  }
  *out = H;
  return AB_OK;
}

int ab_ldl_batch_sizes(ab_ldl_t H, int* nprob, int* n_total,
                       long long* nnz_total) {
  if (!H) return AB_ERR_ARG;
  if (nprob) *nprob = H->h.has_plan ? H->h.d.nprob : 1;
  if (n_total) *n_total = H->h.sym.n;
  if (nnz_total) *nnz_total = H->h.has_plan ? H->h.d.nnz : 0;
  return AB_OK;
}

int ab_ldl_solve(ab_ldl_t H, double* d_x, int nrhs, int ldx, void* stream) {
  if (!H || nrhs < 0 || ldx < H->h.sym.n) return AB_ERR_ARG;
  if (!H->h.factored) return AB_ERR_NOT_FACTORED;
  if (nrhs == 0 || H->h.sym.n == 0) return AB_OK;
  if (!d_x) return AB_ERR_ARG;
  return ab::solve_numeric(H->h, d_x, nrhs, ldx, (cudaStream_t)stream);
}

int ab_ldl_set_precision(ab_ldl_t h, int bits) {
  if (!h || (bits != 32 && bits != 64)) return AB_ERR_ARG;
  h->h.precision = bits;
  return AB_OK;
}

int ab_ldl_set_tensor_cores(ab_ldl_t h, int on) {
  if (!h) return AB_ERR_ARG;
  h->h.tensor_cores = on != 0;
  return AB_OK;
}

int ab_ldl_set_panel_cache(ab_ldl_t h, int bytes) {
  if (!h || bytes < 0 || bytes > 200 * 1024) return AB_ERR_ARG;
  h->h.panel_cache_bytes = bytes;
  return AB_OK;
}

int ab_ldl_set_wide_threshold(ab_ldl_t h, long long entries) {
  if (!h || entries < 1) return AB_ERR_ARG;
  h->h.wide_entries = entries;
  h->h.solve_epoch = -1;
  return AB_OK;
}

int ab_ldl_set_cluster_threshold(ab_ldl_t h, long long entries) {
  if (!h || entries < 1) return AB_ERR_ARG;
  h->h.cluster_entries = entries;
  h->h.solve_epoch = -1;
  return AB_OK;
}

int ab_ldl_set_panel_mode(ab_ldl_t h, int mode, int min_rows) {
  if (!h || mode < 0 || mode > 3) return AB_ERR_ARG;
  h->h.panel_mode = mode;
  if (min_rows > 0) h->h.cl_min_rows = min_rows;
  return AB_OK;
}

// ---- autotuner ----------------------------------------------------------
extern "C++" {
namespace {

struct Tuning {
  int panel_mode, cl_min_rows, panel_cache;
  long long cluster_entries, wide_entries;
  int solve_queue;
};

Tuning get_tuning(const ab::LdlHandle& h) {
  return {h.panel_mode, h.cl_min_rows, h.panel_cache_bytes, h.cluster_entries,
          h.wide_entries, h.solve_queue};
}

void set_tuning(ab::LdlHandle& h, const Tuning& t) {
  h.panel_mode = t.panel_mode;
  h.cl_min_rows = t.cl_min_rows;
  h.panel_cache_bytes = t.panel_cache;
  if (h.cluster_entries != t.cluster_entries || h.wide_entries != t.wide_entries ||
      h.solve_queue != t.solve_queue)
    h.solve_epoch = -1;   // the solve schedule is rebuilt on the next solve
  h.cluster_entries = t.cluster_entries;
  h.wide_entries = t.wide_entries;
  h.solve_queue = t.solve_queue;
}

// Best of `reps` event-timed runs of f() on stream s (after one untimed
// run), in ms; the first non-zero status of f is returned in *rc.
template <class F>
double best_ms(cudaStream_t s, int reps, cudaEvent_t e0, cudaEvent_t e1, int* rc, F f) {
  *rc = f();
  if (*rc) return 0.0;
  double best = 1e300;
  for (int r = 0; r < reps; r++) {
    if (cudaEventRecord(e0, s) != cudaSuccess) { *rc = AB_ERR_CUDA; return 0.0; }
    *rc = f();
    if (*rc) return 0.0;
    float ms = 0.f;
    if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
      *rc = AB_ERR_CUDA;
      return 0.0;
    }
    best = std::min(best, (double)ms);
  }
  return best;
}

}  // namespace
}  // extern "C++"

int ab_ldl_autotune(ab_ldl_t H, const double* d_vals, int reps, void* stream,
                    ab_ldl_tuning* out) {
  if (!H || reps < 1 || (!d_vals && H->h.d.nnz > 0)) return AB_ERR_ARG;
  if (!H->h.has_plan) return AB_ERR_UNSUPPORTED;
  ab::LdlHandle& h = H->h;
  cudaStream_t s = (cudaStream_t)stream;
  const Tuning start = get_tuning(h);
  ab_ldl_tuning rep{};
  if (h.sym.n == 0) {
    h.factored = true;
    if (out) *out = rep;
    return AB_OK;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double* x = nullptr;
  int rc = AB_OK;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
      cudaMalloc((void**)&x, (size_t)h.sym.n * sizeof(double)) != cudaSuccess) {
    rc = AB_ERR_CUDA;
  }
  // the timed solves run on a zero right-hand side (their arithmetic does
  // not depend on the values)
  if (!rc && cudaMemsetAsync(x, 0, (size_t)h.sym.n * sizeof(double), s) != cudaSuccess)
    rc = AB_ERR_CUDA;
  auto factor = [&]() {
    h.factored = false;
    return ab::factor_numeric(h, d_vals, s);
  };
  auto solve = [&]() { return ab::solve_numeric(h, x, 1, h.sym.n, s); };
  int timed = 0;
  Tuning best = start;
  double fbest = 0.0, f0 = 0.0;
  bool factored_best = false;   // the handle's factor is of `best`
  if (!rc) {
    fbest = f0 = best_ms(s, reps, e0, e1, &rc, factor);
    factored_best = true;
    timed++;
  }
  // factor candidates: only patterns with a level of large fronts (the
  // small-front kernel has no setting here)
  int big_max = 0;
  for (const auto& L : h.sched)
    if (L.nbig > 0) big_max = std::max(big_max, L.big_max_f);
  if (!rc && big_max > 0) {
    std::vector<Tuning> cand;
    // the one-CTA panel, then the cluster panels' row threshold
    Tuning t = start;
    t.panel_mode = 1;
    cand.push_back(t);
    const int rows[] = {512, 768, 1024, 1536, 2048};
    for (int r : rows) {
      t = start;
      t.panel_mode = 0;
      t.cl_min_rows = r;
      cand.push_back(t);
    }
    // a threshold matters only through the levels it moves: keep one
    // candidate per distinct set of large-front levels on cluster panels
    auto signature = [&](const Tuning& c) {
      std::vector<char> sig;
      for (const auto& L : h.sched)
        sig.push_back(L.nbig > 0 && c.panel_mode == 0 && L.big_max_f >= c.cl_min_rows);
      return sig;
    };
    std::vector<std::vector<char>> seen{signature(start)};
    for (const Tuning& c : cand) {
      if (rc) break;
      const auto sg = signature(c);
      if (c.panel_mode == start.panel_mode &&
          std::find(seen.begin(), seen.end(), sg) != seen.end())
        continue;
      if (c.panel_mode == 0) seen.push_back(sg);
      set_tuning(h, c);
      const double ms = best_ms(s, reps, e0, e1, &rc, factor);
      timed++;
      if (!rc && ms < 0.98 * fbest) {
        fbest = ms;
        best = c;
        factored_best = true;
      } else {
        factored_best = false;
      }
    }
    // the shared-memory copy of the panel's columns, on the chosen form
    if (!rc) {
      Tuning c = best;
      c.panel_cache = best.panel_cache ? 0 : 96 * 1024;
      set_tuning(h, c);
      const double ms = best_ms(s, reps, e0, e1, &rc, factor);
      timed++;
      if (!rc && ms < 0.98 * fbest) {
        fbest = ms;
        best = c;
        factored_best = true;
      } else {
        factored_best = false;
      }
    }
    if (!rc) {
      set_tuning(h, best);
      if (!factored_best) rc = factor();
    }
  }
  // solve candidates, one knob at a time on the chosen factorization
  double sbest = 0.0, s0 = 0.0;
  if (!rc) {
    set_tuning(h, best);
    sbest = s0 = best_ms(s, reps, e0, e1, &rc, solve);
    timed++;
  }
  auto try_solve = [&](const Tuning& c) {
    if (rc) return;
    set_tuning(h, c);
    const double ms = best_ms(s, reps, e0, e1, &rc, solve);
    timed++;
    if (!rc && ms < 0.98 * sbest) {
      sbest = ms;
      best = c;
    }
  };
  {
    const long long wide[] = {1LL << 20, 1LL << 21, 1LL << 22, 1LL << 23, 1LL << 24, 1LL << 26};
    const Tuning base = best;
    for (long long w : wide)
      if (w != base.wide_entries) {
        Tuning c = base;
        c.wide_entries = w;
        try_solve(c);
      }
  }
  {
    const long long clu[] = {1LL << 12, 1LL << 13, 1LL << 14, 1LL << 15, 1LL << 16};
    const Tuning base = best;
    for (long long v : clu)
      if (v != base.cluster_entries) {
        Tuning c = base;
        c.cluster_entries = v;
        try_solve(c);
      }
  }
  {
    const int modes[] = {0, 1, 3};
    const Tuning base = best;
    for (int m : modes)
      if (m != base.solve_queue) {
        Tuning c = base;
        c.solve_queue = m;
        try_solve(c);
      }
  }
  if (!rc && h.sv_err) {
    // a work-queue sweep whose dependency wait ran out: report it
    int e = 0;
    if (cudaMemcpyAsync(&e, h.sv_err, sizeof(int), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess || e) {
      if (e) cudaMemsetAsync(h.sv_err, 0, sizeof(int), s);
      rc = AB_ERR_CUDA;
    }
  }
  if (!rc) {
    set_tuning(h, best);
    if (out) {
      rep.panel_mode = best.panel_mode;
      rep.cl_min_rows = best.cl_min_rows;
      rep.panel_cache_bytes = best.panel_cache;
      rep.cluster_entries = best.cluster_entries;
      rep.wide_entries = best.wide_entries;
      rep.solve_queue = best.solve_queue;
      rep.factor_ms = fbest;
      rep.solve_ms = sbest;
      rep.factor_ms_initial = f0;
      rep.solve_ms_initial = s0;
      rep.configurations = timed;
      *out = rep;
    }
  } else {
    set_tuning(h, start);
  }
  if (x) cudaFree(x);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return rc;
}

int ab_ldl_apply_tuning(ab_ldl_t H, const ab_ldl_tuning* t) {
  if (!H || !t || t->panel_mode < 0 || t->panel_mode > 3 || t->cl_min_rows < 1 ||
      t->panel_cache_bytes < 0 || t->panel_cache_bytes > 200 * 1024 ||
      t->cluster_entries < 1 || t->wide_entries < 1 || t->solve_queue < 0 ||
      t->solve_queue > 3)
    return AB_ERR_ARG;
  set_tuning(H->h, {t->panel_mode, t->cl_min_rows, t->panel_cache_bytes,
                    t->cluster_entries, t->wide_entries, t->solve_queue});
  return AB_OK;
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

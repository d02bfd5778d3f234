// Internal structures of the multifrontal LDL^T handle.
//
// Layout in HBM (device):
//   * static plan (uploaded once per pattern): per-node sizes, the level
//     schedule, the CSR-entry -> front-position map for assembling A, and the
//     child-contribution-row -> parent-front-position map for extend-add;
//   * per-factorization pools: every front F (f x f, column-major, ld = f)
//     plus its panel workspace W (f x NB) is carved (in FP64 or, for the
//     mixed-precision form, FP32 elements) from one pool with
//     an atomic bump pointer, so fronts whose size grows with delayed pivots
//     need no host round trip; after factorization the first npiv columns of
//     F hold L (unit lower, D on the diagonal / 2x2 blocks) and the trailing
//     block F[npiv:, npiv:] holds the contribution passed to the parent;
//   * an int pool with each front's variable list (pivots first, 2x2 pivots
//     encoded as -(var+1), then delayed, then contribution rows) followed by
//     the fully-summed permutation used by the forward solve.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "symbolic.h"

namespace ab {

// Panel width of the blocked in-front factorization.  The panel loop takes
// columns while kw < kPanel - 1 so that a 2x2 pivot still fits.
constexpr int kPanel = 32;
constexpr int kThreads = 256;
// Dynamic shared memory of the one-CTA-per-front kernel; a front is
// scheduled on that kernel when (f + 16)^2 + (f + 16) * kPanel doubles fit
// (16 rows of slack for delayed pivots), otherwise on the multi-CTA path.
constexpr int kMaxDynSmem = 190 * 1024;

// Status bits written by device code.
enum : int {
  ST_POOL_F = 1,     // FP64 front pool exhausted
  ST_POOL_I = 2,     // int pool exhausted
  ST_NAN = 4,        // non-finite pivot met
};

struct DevicePlan {
  int n = 0, nn = 0, nnz = 0, num_levels = 0;
  // per node
  int* ns = nullptr;           // node width (static fully-summed count)
  int* nc = nullptr;           // static contribution rows
  int* var_ptr = nullptr;      // node_ptr
  int* vars = nullptr;         // node_to_var
  int* cptr = nullptr;         // contrib_ptr
  int* crows = nullptr;        // contrib_rows (original numbering)
  int* cmap = nullptr;         // contrib row -> parent static index
  int* kid_ptr = nullptr;      // children_ptr (first nn+1 entries)
  int* kids = nullptr;         // children
  int* amap_ptr = nullptr;     // per node range into amap
  int* amap_pos = nullptr;     // CSR position
  int* amap_row = nullptr;     // static front row
  int* amap_col = nullptr;     // front column (< ns)
  int* level_nodes = nullptr;  // nodes sorted by level
  int* sched_nodes = nullptr;  // per level: small fronts, then large fronts
  // dynamic, per factorization
  int* f = nullptr;            // front size
  int* npiv = nullptr;         // pivots eliminated
  int* ndel = nullptr;         // delayed pivots passed to parent
  int* ndin = nullptr;         // delayed pivots received from children
  long long* foff = nullptr;   // offset of F in the FP64 pool
  long long* ioff = nullptr;   // offset of the var list in the int pool
  int* inertia = nullptr;      // [npos, nneg] per problem
  int* node_prob = nullptr;    // problem of each node (batched handles)
  int nprob = 1;
  int* status = nullptr;       // ST_* bits
  int* pstate = nullptr;       // per node: k, candidates left, kstart, kw
  int* scratch_int = nullptr;  // small device scratch for host queries
  unsigned long long* counters = nullptr;  // [F pool top, int pool top]
  double* fpool = nullptr;
  int* ipool = nullptr;
  long long fcap = 0, icap = 0;
};

// Per-level launch schedule (host side).
struct LevelSchedule {
  int small_begin = 0, nsmall = 0, big_begin = 0, nbig = 0;
  int small_max_f = 0, big_max_f = 0, big_max_fs = 0, big_max_kids = 0;
  long long big_max_amap = 0;
};

struct LdlHandle {
  int device = 0;
  double ustab = 0.01, pivot_tol = 1e-14, delay_growth = 2.0;
  int order = ORDER_AMD;
  SymbolicTree sym;
  std::vector<int> level_ptr;     // host copy: level boundaries
  std::vector<int> level_nodes;   // host copy
  std::vector<int> h_ns, h_nc;    // host copies of static sizes
  std::vector<int> level_max_f;   // static max front per level
  std::vector<LevelSchedule> sched;
  // Batched handles: node, variable and CSR-entry ranges of every problem
  // (empty for a single problem).
  std::vector<int> prob_node_ptr, prob_var_ptr;
  std::vector<long long> prob_nnz_ptr;
  long long f_static_total = 0;   // sum of static (f^2 + f*kPanel)
  long long i_static_total = 0;
  DevicePlan d;
  bool has_plan = false;   // false for analysis-only handles
  bool factored = false;
  int last_status = 0;
  // per-factorization host copies (filled at the end of factor)
  std::vector<int> h_f, h_npiv, h_ndel;
  // solve scratch
  double* ubuf = nullptr;         // update vectors passed up the tree
  long long ubuf_cap = 0;
  long long* uoff = nullptr;      // per node offset into ubuf (device)
  std::vector<long long> h_uoff;
  int uoff_nrhs = 0;
  // solve schedule, rebuilt after each factorization: per level the fronts
  // solved one per CTA ("narrow") and the wide fronts solved by the
  // cooperative multi-CTA kernels, concatenated level by level
  long long factor_epoch = 0, solve_epoch = -1;
  // f * npiv from which a front is solved by a cluster of CTAs, and from
  // which by the cooperative grid
  long long cluster_entries = 1 << 14;
  // large-front panels: 0 cluster panels for levels whose largest front has
  // at least cl_min_rows rows, 1 one-CTA panels only, 2 cluster panels
  // with the one-CTA panel's widths
  int panel_mode = 0;
  int cl_min_rows = 768;
  // global scratch of the cluster panel for fronts past shared memory
  void* cl_scratch = nullptr;
  size_t cl_scratch_bytes = 0;
  long long wide_entries = 1 << 22;
  // front storage / arithmetic of the next factorization (64: FP64, 32:
  // FP32 fronts for mixed precision) and of the last one
  int precision = 64, factor_precision = 64;
  bool tensor_cores = true;   // FP32 fronts: Schur updates on tcgen05
  // large-front panel: bytes of shared memory for a copy of the panel's L
  // columns (0: read them from HBM; measured faster on the 2D KKT)
  int panel_cache_bytes = 0;
  int* sv_nodes = nullptr;        // device, nn entries
  int* sv_state = nullptr;        // device, 2 ints per wide front of a level
  std::vector<int> sv_narrow_ptr, sv_clu_ptr, sv_wide_ptr, sv_narrow_smem, sv_clu_smem;
  std::vector<int> sv_host, sv_f, sv_npiv;   // schedule and the sizes it is for
  int sv_max_wide = 0, sv_state_cap = 0;
  long long sv_wide_entries = 0;
  std::vector<int> sv_fwd_grid, sv_bwd_grid;   // cooperative grid per level
  int sv_grid_cap = 0;
  // work-queue sweeps over the all-narrow levels [0, sv_qlevels): the
  // backward queue and its dependencies (parent in the queue, or -1), done
  // flags per node with an epoch per sweep, the queue counters and the
  // wait-ran-out word
  // bit 0: work-queue sweeps (default on); bit 1: fronts of at most 128
  // rows on 128-thread CTAs (off: measured slower)
  int solve_queue = 1;
  int sv_qlevels = 0, sv_qcount = 0, sv_qsmem = 0, sv_qgrid = 0, sv_qsmall_smem = 0;
  bool sv_qsmall = false, sv_qgrid_small = false;
  std::vector<int> sv_small_cnt;   // per level: narrow fronts of <= 128 rows
  std::vector<int> sv_small_smem;  // per level: their front vector bytes
  std::vector<int> sv_bq_host, sv_dep_host;
  int* sv_bq = nullptr;
  int* sv_dep = nullptr;
  unsigned* sv_done = nullptr;   // 2 x nn: forward, backward
  unsigned* sv_ctr = nullptr;    // 4: forward and backward counters, epoch, pad
  int* sv_err = nullptr;
};

int build_plan(LdlHandle& h, const int* rowp, const int* cols);
void free_plan(LdlHandle& h);
int factor_numeric(LdlHandle& h, const double* d_vals, cudaStream_t s);
int solve_numeric(LdlHandle& h, double* d_x, int nrhs, int ldx,
                  cudaStream_t s);

}  // namespace ab

/*
 * amigo_b200.h -- C ABI of the B200-native numeric core of amigo's
 * interior-point iteration.
 *
 * Plain C types only: host arrays are passed as pointers + sizes, device
 * buffers as raw device pointers (for example torch.Tensor.data_ptr()),
 * CUDA streams as `void*` (a cudaStream_t; NULL = the legacy default stream).
 * No call frees a caller buffer; handles own their device workspaces.
 * Every entry point returns an int status: 0 = OK, < 0 = error (see
 * AB_ERR_*), > 0 = warning.  No C++ exception crosses this boundary.
 *
 * Each entry point names the reference interface it replaces (file:line in
 * smdogroup/amigo).
 */
#ifndef AMIGO_B200_H
#define AMIGO_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define AB_OK 0
#define AB_ERR_ARG -1         /* bad argument (null pointer, size, order) */
#define AB_ERR_CUDA -2        /* a CUDA runtime call failed */
#define AB_ERR_NOT_FACTORED -3 /* solve/inertia before a successful factor */
#define AB_ERR_UNSUPPORTED -4 /* option not provided by this library */
#define AB_ERR_NUMERIC -5     /* NaN/Inf met in the factorization */
#define AB_ERR_CAPACITY -6    /* workspace could not be grown */

typedef struct ab_ldl* ab_ldl_t;

/* ----------------------------------------------------------------------
 * Sparse LDL^T (multifrontal, threshold 1x1/2x2 pivoting, exact inertia)
 * -------------------------------------------------------------------- */

/* Symbolic analysis + device plan.  Replaces the SparseLDL constructor
 * (include/sparse_ldl.h:65-118; binding amigo/amigo.cpp:616-625).
 * rowp[n+1], cols[nnz]: host CSR pattern of the full symmetric matrix.
 * order: 0 NESTED_DISSECTION, 1 AMD, 3 NATURAL (include/ordering_utils.h:21).
 * solver_type: 0 LDL (1 CHOLESKY is rejected with AB_ERR_UNSUPPORTED).
 * ustab is clamped to [0, 0.5] and delay_growth to [1, 10] as in the
 * reference.  The CUDA device current at this call is used for the handle. */
int ab_ldl_create(int n, const int* rowp, const int* cols, int order,
                  int solver_type, double ustab, double pivot_tol,
                  double delay_growth, ab_ldl_t* out);
int ab_ldl_destroy(ab_ldl_t h);

/* Device bytes a factorization of this pattern needs, from its symbolic
 * analysis alone (works on analysis-only handles, no GPU needed): the front
 * pool at `precision` (64 or 32) bits times delay_growth (room for fronts
 * grown by delayed pivots), the integer pools, the static plan and the
 * solve's update vectors for nrhs right-hand sides.  The admission budget
 * of a request loop adds the caller's own vectors.  No counterpart call in
 * the reference, whose SparseLDL sizes its pools from the same symbolic
 * data (include/sparse_ldl.h:62-93, 3162-3220). */
int ab_ldl_mem_estimate(ab_ldl_t h, int precision, double delay_growth,
                        int nrhs, long long* bytes);

/* Symbolic analysis only (host; makes no CUDA call).  The handle answers
 * ab_ldl_symbolic_sizes / ab_ldl_symbolic_arrays and must be released with
 * ab_ldl_destroy; ab_ldl_factor on it returns AB_ERR_UNSUPPORTED.  Mirrors
 * SparseLDL::symbolic_analysis (include/sparse_ldl.h:2204-2358). */
int ab_ldl_analyze(int n, const int* rowp, const int* cols, int order,
                   ab_ldl_t* out);

/* Sizes and copies of the symbolic arrays, for bit-exact comparison with
 * the reference's private members node_ptr, node_to_var,
 * node_children_ptr, node_children, contrib_ptr, contrib_rows, invperm
 * (include/sparse_ldl.h:3240-3262). */
int ab_ldl_symbolic_sizes(ab_ldl_t h, int* num_nodes, int* contrib_total);
int ab_ldl_symbolic_arrays(ab_ldl_t h, int* node_ptr, int* node_to_var,
                           int* children_ptr, int* children, int* contrib_ptr,
                           int* contrib_rows, int* invperm);

/* Numeric factorization of device CSR values d_vals[nnz] (FP64) on the
 * pattern given at create time.  Replaces SparseLDL::factor
 * (include/sparse_ldl.h:136-151).  Asynchronous on `stream` except when a
 * workspace must grow, which needs one synchronisation. */
int ab_ldl_factor(ab_ldl_t h, const double* d_vals, void* stream);

/* Inertia (npos, nneg) of the last factorization; synchronises `stream`.
 * Replaces SparseLDL::get_inertia (include/sparse_ldl.h:198-206). */
int ab_ldl_inertia(ab_ldl_t h, void* stream, int* npos, int* nneg);

/* In-place solve L D L^T x = b for nrhs right-hand sides stored column-major
 * with leading dimension ldx >= n in device memory.  Replaces
 * SparseLDL::solve (include/sparse_ldl.h:162-190). */
int ab_ldl_solve(ab_ldl_t h, double* d_x, int nrhs, int ldx, void* stream);

/* Batched handle: nprob independent problems factored and solved together,
 * one launch per elimination-tree level for all of them (fronts of every
 * problem at the same level share the launch).  Each problem keeps its own
 * symbolic analysis (identical to the reference's for that problem); the
 * values and right-hand sides are the concatenation of the problems' in
 * order (problem p's CSR values start at the sum of the earlier nnz, its
 * rows at the sum of the earlier n).  ab_ldl_factor / ab_ldl_solve /
 * ab_ldl_destroy apply to the batch; ab_ldl_inertia returns the sums and
 * ab_ldl_batch_inertia the per-problem values (arrays of nprob).  No single
 * reference counterpart: the reference factors one SparseLDL at a time. */
int ab_ldl_batch_create(int nprob, const int* n, const int* const* rowp,
                        const int* const* cols, int order, int solver_type,
                        double ustab, double pivot_tol, double delay_growth,
                        ab_ldl_t* out);
int ab_ldl_batch_inertia(ab_ldl_t h, void* stream, int* npos, int* nneg);
int ab_ldl_batch_sizes(ab_ldl_t h, int* nprob, int* n_total,
                       long long* nnz_total);

/* Precision of the fronts of the following factorizations: 64 (default,
 * FP64, the reference's arithmetic) or 32 (mixed precision: fronts
 * assembled from the FP64 values, stored and updated in FP32; the pivot
 * tests compare FP64 copies of the FP32 values and the solves accumulate in
 * FP64 while reading the FP32 factor.  Accuracy is recovered by iterative
 * refinement against the FP64 KKT).  No reference counterpart. */
int ab_ldl_set_precision(ab_ldl_t h, int bits);

/* FP32 fronts only: 1 (default) applies the large fronts' Schur updates on
 * the tensor cores (3xTF32 tcgen05, see ab_tc_syrk_tf32x3), 0 on the FP32
 * CUDA cores.  No reference counterpart. */
int ab_ldl_set_tensor_cores(ab_ldl_t h, int on);

/* Large-front panel knob: bytes of shared memory (0 .. 204800, default 0)
 * for a copy of the panel's L columns that the pivot-column builds read;
 * 0 reads them from the front in HBM (on the 2D SIMP KKT the copy measured
 * 7% slower: the shared-memory carve-out takes L1 from the other reads).
 * No reference counterpart. */
int ab_ldl_set_panel_cache(ab_ldl_t h, int bytes);

/* Solve schedule knobs: fronts with f * npiv >= the wide threshold
 * (default 2^22) are solved by the cooperative grid-wide kernels; fronts
 * from the cluster threshold (default 2^14) up to it by one thread-block
 * cluster of 8 CTAs each (when the front vector fits in shared memory);
 * smaller ones by one CTA per front.  All give the same result to
 * rounding.  No reference counterpart (the reference solves every front on
 * one thread). */
int ab_ldl_set_wide_threshold(ab_ldl_t h, long long entries);
int ab_ldl_set_cluster_threshold(ab_ldl_t h, long long entries);

/* Large-front panel knob.  mode 0 (default): levels whose largest front
 * has at least min_rows rows (default 768) factor their panels on one
 * thread-block cluster of 8 CTAs per front, NB = 32 columns a panel;
 * fronts past what shared memory holds (> 3,008 rows) keep W and L in a
 * global scratch region, on clusters of 8 CTAs to 16,320 rows and of 16
 * (where the device schedules them) to 32,704;
 * mode 1: one CTA per front for every level; mode 2: cluster panels with
 * the one-CTA panel's widths, whose results are the one-CTA panel's bit
 * for bit (a test mode); mode 3: the global-scratch form on clusters of 16
 * for every level from min_rows, bit-identical to mode 0 (a test mode).
 * min_rows <= 0 keeps the current value.  No reference counterpart (the
 * reference factors each front on one thread). */
int ab_ldl_set_panel_mode(ab_ldl_t h, int mode, int min_rows);

/* Solve schedule of the fronts solved without a cluster or the
 * cooperative grid ("narrow"), mode bits (default 1):
 *   bit 0: the sweeps over the levels whose fronts are all narrow (from
 *          the leaves) are one work-queue launch each -- fronts are taken
 *          in dependency order from an atomic counter and each waits
 *          (bounded) for the fronts it depends on; without it, one launch
 *          per level;
 *   bit 1: fronts of at most 128 rows run on 128-thread CTAs instead of
 *          256-thread ones (twice as many fronts in flight per SM;
 *          measured slower on the batched cart-pole and 2D SIMP KKTs).
 * All modes give the same result bit for bit.  ab_ldl_solve_status
 * reports (AB_ERR_CUDA) and clears a wait that ran out since the last
 * check; ab_ldl_factor also reports it.  No reference counterpart (the
 * reference solves front by front on the host). */
int ab_ldl_set_solve_queue(ab_ldl_t h, int mode);
int ab_ldl_solve_status(ab_ldl_t h, void* stream);

/* Launch forms and thresholds picked by ab_ldl_autotune for one pattern. */
typedef struct {
  int panel_mode, cl_min_rows, panel_cache_bytes; /* factor: large-front panels */
  long long cluster_entries, wide_entries;        /* solve: front classes */
  int solve_queue;                                /* solve: narrow-front schedule */
  double factor_ms, solve_ms;                 /* chosen settings, best of reps */
  double factor_ms_initial, solve_ms_initial; /* settings on entry */
  int configurations;                         /* settings timed */
} ab_ldl_tuning;

/* Autotuner: times the factorization of the KKT values d_vals (device, as
 * for ab_ldl_factor) under the large-front panel forms (one-CTA panels,
 * or cluster panels from 512 / 768 / 1,024 / 1,536 / 2,048 rows, with and
 * without the shared-memory column copy), then one solve under the solve
 * knobs (cooperative-grid threshold, cluster threshold, work-queue and
 * 128-thread schedules), one knob at a time, best of `reps` (>= 1) each on
 * `stream`, and keeps the fastest (a setting replaces the current one only
 * when it is at least 2% faster).  Patterns without large fronts skip the
 * factor candidates.  The chosen settings stay on the handle, which is
 * left factored with them; *out (may be NULL) reports them.  Panel forms
 * change the factorization to rounding (different panel widths; the same
 * pivot tests); the solve thresholds change the solution to rounding (a
 * front's class sets its reduction order) and the narrow-front schedules
 * not at all.  On an error the settings on entry are restored.
 * Allocates one n-vector of device memory for the timed solves.  No
 * reference counterpart (the reference has one fixed host schedule). */
int ab_ldl_autotune(ab_ldl_t h, const double* d_vals, int reps, void* stream,
                    ab_ldl_tuning* out);
/* Applies settings from ab_ldl_autotune (e.g. of another handle with the
 * same pattern). */
int ab_ldl_apply_tuning(ab_ldl_t h, const ab_ldl_tuning* t);

/* The tensor-core Schur update on plain device arrays (column-major, FP32):
 * lower(C) -= A B^T for n x kw panels A, B (kw <= 31), as 3xTF32 tcgen05
 * products accumulated in FP32 in tensor memory -- the update the
 * mixed-precision factorization applies to its large fronts.  *d_status
 * (device int) gets bit 8 if an MMA completion wait ran out.  No reference
 * counterpart (the reference updates fronts with FP64 dgemm,
 * include/sparse_ldl.h:1172-1197). */
int ab_tc_syrk_tf32x3(int n, int kw, const float* A, int lda, const float* B,
                      int ldb, float* C, int ldc, int* d_status, void* stream);

/* Number of kernels this library has launched in the process so far (every
 * kernel of every entry point; library memsets excluded).  No reference
 * counterpart: it lets callers count the device launches of a region. */
long long ab_launch_count(void);

/* Statistics of the last factorization (host values; synchronises).
 * flops: sum over fronts of p^3/3 + p^2 c + p c^2 with p = pivots, c =
 * contribution size; factor_entries: sum f*p; max_front; num_delayed:
 * total delayed pivots; levels: elimination-tree levels. */
int ab_ldl_stats(ab_ldl_t h, void* stream, double* flops,
                 double* factor_entries, int* max_front, int* num_delayed,
                 int* levels);

/* Per-node pivot and delayed-pivot counts of the last factorization
 * (host arrays of num_nodes ints; synchronises).  Mirrors the
 * reference's MatrixFactor::get_factor counts (include/sparse_ldl.h:418-445). */
int ab_ldl_node_pivots(ab_ldl_t h, void* stream, int* num_pivots,
                       int* num_delayed);

/* ----------------------------------------------------------------------
 * IPM vector kernels (include/interior_point_backend.h).  All array
 * arguments are device pointers; index arrays are int32.  The problem
 * description (ProblemInfo, interior_point_backend.h:55-63):
 *   np, nc: number of primal / constraint entries
 *   pidx[np], cidx[nc]: their positions in the n-vector xlam
 *   lbx[np], ubx[np]: bounds (+-inf allowed), lbh[nc]: constraint targets
 * The state (State, interior_point_backend.h:67-77):
 *   xlam[n], zl[np], zu[np], sl[np], su[np]
 * Scalar results are written to a device array `out` and are ready when
 * `stream` reaches the end of the call.
 * -------------------------------------------------------------------- */
typedef struct ab_ipm_problem {
  int n, np, nc;
  const int* pidx;
  const int* cidx;
  const double* lbx;
  const double* ubx;
  const double* lbh;
  /* Batched problems (all NULL / 0 for a single problem): instances are
   * stored one after another; mu_inst[k] is instance k's barrier parameter
   * (used instead of the `mu` argument wherever it is set), pinst / vinst
   * the instance of every primal entry / n-vector entry, and the primal and
   * constraint entries of instance k are [poff[k], poff[k+1]) and
   * [coff[k], coff[k+1]). */
  const double* mu_inst;
  const int* pinst;
  const int* vinst;
  int ninst;
  const int* poff;
  const int* coff;
} ab_ipm_problem;

typedef struct ab_ipm_state {
  const double* xlam;
  const double* zl;
  const double* zu;
  const double* sl;
  const double* su;
} ab_ipm_state;

/* compute_residual (interior_point_backend.h:203-229); when out2 != NULL
 * also the squared dual/primal infeasibilities of
 * compute_residual_and_infeasibility (:234-266) -> out2[0..1]. */
int ab_ipm_residual(const ab_ipm_problem* p, const ab_ipm_state* s, double mu,
                    const double* grad, double* res, double* out2,
                    void* stream);
/* compute_diagonal (:277-288) */
int ab_ipm_diagonal(const ab_ipm_problem* p, const ab_ipm_state* s,
                    double* diag, void* stream);
/* compute_bound_dual_step (:303-321) */
int ab_ipm_bound_dual_step(const ab_ipm_problem* p, const ab_ipm_state* s,
                           double mu, const double* px, double* dzl,
                           double* dzu, void* stream);
/* compute_max_step (:329-369), seeded ax = az = 1, xi = zi = -1 as the
 * binding does (amigo/amigo.cpp:768-775).  out[0] = ax, out[1] = az,
 * iout[0] = xi, iout[1] = zi.  Ties resolve to the first index in primal
 * order, which is what the sequential reference loop returns. */
int ab_ipm_max_step(const ab_ipm_problem* p, const ab_ipm_state* s,
                    double tau, const double* px, const double* dzl,
                    const double* dzu, double* out, int* iout, void* stream);
/* The same step-length computation as ab_ipm_max_step, for callers that
 * cannot let the library allocate device memory (a host whose caching
 * allocator owns the device, a loop that must not allocate once running,
 * an embedding in which the caller owns every device buffer).  No
 * counterpart in the reference.  Its reduction scratch is a fixed array
 * compiled into the library (192 KiB, held on every GPU that loads the
 * library until process exit) instead of a cudaMalloc'd buffer, which caps
 * np at 2,097,152 primal entries; larger problems return AB_ERR_CAPACITY.
 * The first call on a device looks up the array's device address (a CUDA
 * runtime query), so make that call before any stream capture.  All calls
 * share the one array: calls that can overlap on the GPU (different
 * streams, or different host threads) race and must be serialised by the
 * caller.  Arguments and results as for ab_ipm_max_step. */
int ab_ipm_max_step_noalloc(const ab_ipm_problem* p, const ab_ipm_state* s,
                            double tau, const double* px, const double* dzl,
                            const double* dzu, double* out, int* iout,
                            void* stream);
/* apply_step (:376-392) into new-state arrays */
int ab_ipm_apply_step(const ab_ipm_problem* p, const ab_ipm_state* s,
                      double ax, double az, const double* dxlam,
                      const double* dzl, const double* dzu, double* xlam_new,
                      double* zl_new, double* zu_new, double* sl_new,
                      double* su_new, void* stream);
/* Reductions, written to out[]:
 *  compute_complementarity (:397-413): out[0] = sum, out[1] = count,
 *    out[2] = min;
 *  compute_kkt_error (:450-466): out[3] = dual, out[4] = primal,
 *    out[5] = comp;
 *  compute_barrier_log_sum (:471-484): out[6];
 *  compute_constraint_violation_1norm (:565-573): out[7];
 *  compute_max_comp_deviation (:417-426): out[8];
 *  compute_complementarity_sq (:430-443): out[9];
 *  compute_kkt_error_sq (:539-561): out[10] = dual_sq, out[11] = primal_sq,
 *    out[12] = comp_sq.
 * out must hold 13 doubles.  grad may be NULL (then out[3], out[4],
 * out[7], out[10], out[11] are 0). */
int ab_ipm_reductions(const ab_ipm_problem* p, const ab_ipm_state* s,
                      double mu, const double* grad, double* out,
                      void* stream);
/* compute_barrier_dphi (:491-502) -> out[0] */
int ab_ipm_barrier_dphi(const ab_ipm_problem* p, const ab_ipm_state* s,
                        double mu, const double* grad, const double* px,
                        double* out, void* stream);
/* compute_barrier_dphi_from_kkt (:597-611) -> out[0]; res, px, diag are
 * n-vectors. */
int ab_ipm_barrier_dphi_kkt(const ab_ipm_problem* p, const ab_ipm_state* s,
                            const double* res, const double* px,
                            const double* diag, double* out, void* stream);
/* relax_bounds (:126-146): lbx_out/ubx_out may alias lbx/ubx. */
int ab_ipm_relax_bounds(int np, const double* lbx, const double* ubx,
                        double* lbx_out, double* ubx_out, double factor,
                        double constr_viol_tol, void* stream);
/* project_primals_into_interior (:156-177), initialize_bound_duals
 * (:182-188) and initialize_slacks (:82-88) in one pass, as
 * InteriorPointOptimizer::initialize_multipliers_and_slacks does
 * (include/interior_point_optimizer.h:202-212).  Uses p->lbx/ubx. */
int ab_ipm_initialize(const ab_ipm_problem* p, double* xlam, double* zl,
                      double* zu, double* sl, double* su, double kappa1,
                      double kappa2, void* stream);
/* Iterative refinement on the unreduced 8-block Newton system, the device
 * form of DirectSparseSolver.iterative_refinement
 * (amigo/algorithm/solvers/linear_solver.py:109-264).  rhs_saved is the
 * condensed right-hand side of the first solve; grad, rhs_saved, px, kpx,
 * e_cond, corr are n-vectors; dzl, dzu, e_zl, e_zu are np-vectors.
 *  refine_init: initial dzl/dzu by back-substitution, out[0] = ||rhs||_inf
 *    over the four blocks;
 *  refine_residual: given kpx = K px, the block residuals, the condensed
 *    correction rhs e_cond, out[0] = ||residual||_inf,
 *    out[1] = max(||px||, ||dzl||, ||dzu||)_inf;
 *  refine_update: dzl/dzu corrections from corr = K^-1 e_cond, px += corr. */
int ab_ipm_refine_init(const ab_ipm_problem* p, const ab_ipm_state* s,
                       double mu, const double* grad, const double* rhs_saved,
                       const double* px, double* dzl, double* dzu, double* out,
                       void* stream);
int ab_ipm_refine_residual(const ab_ipm_problem* p, const ab_ipm_state* s,
                           double mu, const double* grad,
                           const double* rhs_saved, const double* kpx,
                           const double* px, const double* dzl,
                           const double* dzu, double* e_cond, double* e_zl,
                           double* e_zu, double* out, void* stream);
int ab_ipm_refine_update(const ab_ipm_problem* p, const ab_ipm_state* s,
                         const double* corr, const double* e_zl,
                         const double* e_zu, double* px, double* dzl,
                         double* dzu, void* stream);
/* Batched problems: the refinement steps above with the barrier parameter
 * of each entry's instance (p->mu_inst) and per-instance norms, so every
 * instance applies the reference's stopping rule
 * (amigo/algorithm/solvers/linear_solver.py:203-239) on its own:
 *  refine_init_seg:     seg_out[k] = instance k's right-hand-side norm;
 *  refine_residual_seg: seg_out[2k] = residual norm, seg_out[2k+1] =
 *                       solution norm of instance k;
 *  refine_update_seg:   applies the correction only to instances with
 *                       active[k] != 0 (device array of ninst ints). */
int ab_ipm_refine_init_seg(const ab_ipm_problem* p, const ab_ipm_state* s,
                           const double* grad, const double* rhs_saved,
                           const double* px, double* dzl, double* dzu,
                           double* seg_out, void* stream);
int ab_ipm_refine_residual_seg(const ab_ipm_problem* p, const ab_ipm_state* s,
                               const double* grad, const double* rhs_saved,
                               const double* kpx, const double* px,
                               const double* dzl, const double* dzu,
                               double* e_cond, double* e_zl, double* e_zu,
                               double* seg_out, void* stream);
int ab_ipm_refine_update_seg(const ab_ipm_problem* p, const ab_ipm_state* s,
                             const int* active, const double* corr,
                             const double* e_zl, const double* e_zu,
                             double* px, double* dzl, double* dzu,
                             void* stream);
/* Batched problems: per-instance reductions, one block per instance
 * (deterministic).  out[k * 12 + q] for instance k: 0 dual, 1 primal,
 * 2 complementarity inf-norms of compute_kkt_error (:450-466, with
 * mu_inst[k]); 3 constraint violation 1-norm (:565-573); 4 barrier log-sum
 * (:471-484); 5, 6 primal / dual fraction-to-boundary steps
 * (compute_max_step :329-369, seeded at 1); 7 barrier directional
 * derivative (:491-502, with gf); 8 max |lam + dlam| over the
 * constraints; 9 / 10 the largest / smallest gap product s z over the
 * bounded entries (-/+inf without any), from which the complementarity
 * norm for any barrier parameter m is max(0, q9 - m, m - q10) exactly.
 * Null inputs skip the quantities that need them.  tau < 0 selects the
 * per-instance fraction max(-tau, 1 - mu_inst[k]). */
int ab_ipm_seg_reduce(const ab_ipm_problem* p, const ab_ipm_state* s,
                      double tau, const double* grad, const double* px,
                      const double* dzl, const double* dzu, const double* gf,
                      double* out, void* stream);
/* apply_step (:376-392) with step lengths ax[k], az[k] per instance. */
int ab_ipm_apply_step_seg(const ab_ipm_problem* p, const ab_ipm_state* s,
                          const double* ax, const double* az,
                          const double* dxlam, const double* dzl,
                          const double* dzu, double* xlam_new, double* zl_new,
                          double* zu_new, double* sl_new, double* su_new,
                          void* stream);
/* reset_bound_multipliers (:508-522) */
int ab_ipm_reset_bound_multipliers(const ab_ipm_problem* p,
                                   const ab_ipm_state* s, double mu,
                                   double kappa, double* zl_out,
                                   double* zu_out, void* stream);
/* compute_affine_start_point (:526-535) */
int ab_ipm_affine_start_point(const ab_ipm_problem* p, const ab_ipm_state* s,
                              double beta_min, const double* dzl,
                              const double* dzu, double* zl_out,
                              double* zu_out, void* stream);

/* ----------------------------------------------------------------------
 * KKT matrix utilities (CSR values on the device)
 * -------------------------------------------------------------------- */

/* ---- NLP scaling, slacks, dual residual (InteriorPointOptimizer,
 * include/interior_point_optimizer.h:476-598; interior_point_backend.h:
 * 99-121, 579-586).  Device pointers; asynchronous on `stream`. ---- */

/* *d_out = max_j |x[idx[j]]| (0 for m = 0): the objective-gradient norm of
 * compute_nlp_scaling (interior_point_optimizer.h:508-518). */
int ab_vec_absmax_gather(int m, const int* idx, const double* x,
                         double* d_out, void* stream);
/* Constraint scaling of compute_nlp_scaling (interior_point_optimizer.h:
 * 520-560): dc[j] = min(1, max_gradient / max_k |H[cidx[j], k]|) floored
 * at min_value, lbh[j] *= dc[j] where dc[j] != 1, scale[i] = 1 for every
 * variable and dc[j] at cidx[j] (the D of D H D). */
int ab_ipm_constraint_scale(int n, int nc, const int* cidx, const int* rowp,
                            const double* hess_vals, double max_gradient,
                            double min_value, double* dc, double* lbh,
                            double* scale, void* stream);
/* vals[k] *= scale[i] * scale[cols[k]] (apply_hessian_scaling,
 * interior_point_optimizer.h:573-584). */
int ab_csr_scale_symmetric(int n, const int* rowp, const int* cols,
                           const double* scale, double* vals, void* stream);
/* x[idx[j]] *= s[j], or /= s[j] when divide != 0 (apply_gradient_scaling,
 * scale_multipliers, unscale_multipliers, interior_point_optimizer.h:
 * 566-597). */
int ab_vec_scale_gather(int m, const int* idx, const double* s, double* x,
                        int divide, void* stream);
/* xlam[slack_idx[k]] = grad[constr_idx[k]] + xlam[slack_idx[k]]
 * (initialize_slacks, interior_point_optimizer.h:476-489). */
int ab_ipm_initialize_slacks(int nslack, const int* slack_idx,
                             const int* constr_idx, const double* grad,
                             double* xlam, void* stream);
/* out = 0, then out[pidx[i]] = grad[pidx[i]] - zl[i] + zu[i]
 * (compute_dual_residual_vector, interior_point_backend.h:579-586). */
int ab_ipm_dual_residual_vector(int n, int np, const int* pidx,
                                const double* grad, const double* zl,
                                const double* zu, double* out, void* stream);
/* dst[idx[j]] = src[idx[j]] (copy_primals / copy_constraints,
 * interior_point_backend.h:106-121). */
int ab_vec_copy_gather(int m, const int* idx, const double* src, double* dst,
                       void* stream);

/* vals[diag_pos[i]] += d[i] for i < n.  Replaces CSRMat::add_diagonal
 * (include/csr_matrix.h:508-528). */
int ab_csr_add_diagonal(int n, const int* diag_pos, const double* d,
                        double* vals, void* stream);
/* y = K x for the symmetric CSR matrix (both triangles stored), nrhs
 * columns with leading dimension ld.  Used by iterative refinement
 * (amigo/algorithm/solvers/linear_solver.py:196-200). */
int ab_csr_matvec(int n, const int* rowp, const int* cols, const double* vals,
                  const double* x, double* y, void* stream);

/* ----------------------------------------------------------------------
 * Component evaluation for the 2D SIMP full-space model: gradient of the
 * Lagrangian and its Hessian scattered into the CSR KKT values.  Replaces
 * OptimizationProblem::gradient / hessian (include/optimization_problem.h:
 * 742-762, 801-818) for that model's components.  All pointers are device
 * pointers except color_ptr, which is held in the struct.
 * -------------------------------------------------------------------- */
typedef struct ab_simp2d {
  int n, nnz, nelems, nnodes;
  int u0, rt0, re0, s_index, lam0, mu0, nu_index;
  int color_ptr[5];          /* element colour boundaries in color_elems */
  const int* color_elems;    /* elements sorted by colour */
  const int* ev;             /* [nelems x 20] u(8) rt(4) lam(8) indices */
  const int* fv;             /* [nelems x 9] rt(4) re mu(4) indices */
  const int* epos;           /* [nelems x 400] CSR positions of ev x ev */
  const int* fpos;           /* [nelems x 81] CSR positions of fv x fv */
  const int* vpos;           /* [nelems x 2] (re,nu), (nu,re) positions */
  const int* spos;           /* [2] (s,nu), (nu,s) positions */
  const int* fixed;          /* fixed variable indices */
  const int* fixed_zero_pos; /* off-diagonal positions in fixed rows/cols */
  const int* fixed_diag_pos; /* diagonal positions of fixed variables */
  const int* load_idx;       /* load dof (relative to u0 / lam0) */
  const double* load_val;
  const double* K0;          /* 8x8 unit-modulus element stiffness */
  const double* A;           /* 4x4 filter matrix M + r^2 K_lap */
  int nfixed, nfixed_zero, nload;
  double Bq, vcoef, volfrac, E0, Emin, penalty;
} ab_simp2d;

/* grad = nabla_x L(x) with objective weight alpha (fixed rows zeroed). */
int ab_simp2d_gradient(const ab_simp2d* m, const double* x, double alpha,
                       double* grad, void* stream);
/* vals = nabla^2 L(x) on the KKT pattern (fixed rows/columns zeroed, unit
 * diagonal). */
int ab_simp2d_hessian(const ab_simp2d* m, const double* x, double alpha,
                      double* vals, void* stream);

/* The 3D SIMP full-space model (48 x 24 x 24 trilinear hexahedra): the
 * same Lagrangian and field meanings as ab_simp2d with 8-node elements,
 * 3 displacement components per node and 8 element colours:
 *   ev   [nelems x 56]   u(24) rt(8) lam(24) indices
 *   fv   [nelems x 17]   rt(8) re mu(8) indices
 *   epos [nelems x 3136] CSR positions of ev x ev
 *   fpos [nelems x 289]  CSR positions of fv x fv
 *   K0   24 x 24 unit-modulus stiffness, A 8 x 8 filter matrix. */
typedef struct ab_simp3d {
  int n, nnz, nelems, nnodes;
  int u0, rt0, re0, s_index, lam0, mu0, nu_index;
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
} ab_simp3d;
int ab_simp3d_gradient(const ab_simp3d* m, const double* x, double alpha,
                       double* grad, void* stream);
int ab_simp3d_hessian(const ab_simp3d* m, const double* x, double alpha,
                      double* vals, void* stream);

/* ----------------------------------------------------------------------
 * Component evaluation for the cart-pole trapezoidal-collocation model
 * (gradient and Hessian of the Lagrangian; exact derivatives by hyper-dual
 * numbers).  Replaces OptimizationProblem::gradient / hessian for that
 * model.  Device pointers except where noted.
 * -------------------------------------------------------------------- */
typedef struct ab_cartpole {
  int n, nnz, N;
  double h, M, m, l, g;
  const int* iv;    /* [N x 14]: z_k (5), z_k+1 (5), defect multipliers (4) */
  const int* ipos;  /* [N x 196] CSR positions of iv x iv */
  const int* bv;    /* [nbc x 8]: boundary states (4), multipliers (4) */
  const int* bpos;  /* [nbc x 64] CSR positions of bv x bv */
  /* Batches of instances stored one after another (NULL / 0 for a single
   * model): per-interval step and pole mass, the number of boundary
   * components, and each instance's interval range [inst_iv[b],
   * inst_iv[b+1]) (objective per instance). */
  const double* h_iv;
  const double* m_iv;
  int nbc;
  int ninst;
  const int* inst_iv;
} ab_cartpole;

int ab_cartpole_gradient(const ab_cartpole* m, const double* x, double alpha,
                         double* grad, void* stream);
int ab_cartpole_hessian(const ab_cartpole* m, const double* x, double alpha,
                        double* vals, void* stream);
/* objective value (trapezoidal integral of u^2) -> out[0], or out[b] per
 * instance of a batch */
int ab_cartpole_objective(const ab_cartpole* m, const double* x, double* out,
                          void* stream);

/* ----------------------------------------------------------------------
 * Device-side decisions of the batched interior-point loop (one thread per
 * instance).  The loop is ipm_driver's (amigo_b200/ipm_driver.py): the
 * convergence test E_0 <= tol and the monotone barrier update (the
 * reference's monotone strategy, amigo/algorithm/barrier_strategy/:
 * mu <- max(mu_min, min(kappa_mu mu, mu^theta_mu)) while
 * E_mu <= kappa_eps mu), inertia correction (Algorithm IC,
 * amigo/algorithm/inertia_correction.py:261-402: delta_w from dw_first,
 * dw_last kw_minus, growth kw_plus_first / kw_plus; delta_c = dc mu^kappa_c
 * on singular matrices), the 8-block refinement stopping rule (ratio below
 * 1e-10 or no longer decreasing), and the l1-merit backtracking line
 * search (Armijo on phi = f + barrier + nu theta, alpha halved).  All
 * arrays are device arrays of ninst entries; mu is the barrier array the
 * batched IPM kernels read (ab_ipm_problem.mu_inst).  Each call sets bits
 * of flags[] (cleared by ab_bctl_clear_flags) that the host reads to end
 * its loops; no other per-instance data needs to leave the device inside
 * an iteration.  No single reference counterpart: the reference takes
 * these decisions in Python for one problem at a time. */
enum {
  AB_BCTL_RETIRED = 0,     /* an instance converged or ran out of iterations */
  AB_BCTL_LIVE = 1,        /* an instance continues this iteration */
  AB_BCTL_IC_PENDING = 2,  /* an instance needs another factorization */
  AB_BCTL_REFINING = 3,    /* an instance takes another refinement step */
  AB_BCTL_STALLED = 4,     /* an instance's refinement ended above 1e-10 */
  AB_BCTL_SEARCHING = 5,   /* an instance's line search continues */
  AB_BCTL_MISMATCH = 6,    /* a pending instance's inertia is not the wanted one */
  AB_BCTL_NFLAGS = 8
};

typedef struct ab_bctl {
  int ninst;
  double *mu, *nu, *dw, *dc, *dwf, *dcf, *dw_last, *alpha, *az, *phi0, *dphi;
  double *ratio, *ratio_old, *nrm, *e0;
  int *live, *pending, *search, *on, *its, *n_ic, *retire;
  const int *np_each, *nc_each, *n_each; /* wanted inertia and sizes */
  int* flags;                            /* AB_BCTL_NFLAGS ints */
} ab_bctl;

typedef struct ab_bctl_opts {
  double tol, mu_min, kappa_eps, kappa_mu, theta_mu, dw_first, dw_min, dw_max;
  double kw_plus_first, kw_plus, kw_minus, dc, kappa_c, armijo;
  int max_iter;
} ab_bctl_opts;

int ab_bctl_clear_flags(const ab_bctl* c, void* stream);
/* q: ab_ipm_seg_reduce output (grad given, current mu).  Retires converged
 * (retire = 1) and exhausted (retire = 2) instances, e0 = E_0; updates mu
 * of the others by the monotone rule, with E_mu from the gap-product
 * extremes (q slots 9, 10). */
int ab_bctl_converge_barrier(const ab_bctl* c, const ab_bctl_opts* o, const double* q,
                             void* stream);
/* delta_w = delta_c = 0, pending = live */
int ab_bctl_ic_begin(const ab_bctl* c, void* stream);
/* dtot = diag + dwf[inst] primal - dcf[inst] (1 - primal) */
int ab_bctl_shift_diag(const ab_bctl* c, int n, const int* vinst, const double* primal,
                       const double* diag, double* dtot, void* stream);
/* inertia: the batched factorization's [npos, nneg] per instance (device,
 * ab_ldl_inertia_device) */
int ab_bctl_ic_step(const ab_bctl* c, const ab_bctl_opts* o, const int* inertia,
                    void* stream);
/* sets AB_BCTL_MISMATCH when a pending instance's inertia differs from
 * (np_each, nc_each); changes nothing else (the mixed-precision loop
 * refactors in FP64 before deciding) */
int ab_bctl_ic_check(const ab_bctl* c, const int* inertia, void* stream);
/* dw_last = dw where an instance is live and dw > 0 */
int ab_bctl_ic_end(const ab_bctl* c, void* stream);
/* seg: ab_ipm_refine_init_seg's right-hand-side norms */
int ab_bctl_refine_init(const ab_bctl* c, const double* seg, void* stream);
/* seg: ab_ipm_refine_residual_seg's per-instance pairs; `on` is the active
 * mask ab_ipm_refine_update_seg takes */
int ab_bctl_refine_step(const ab_bctl* c, const double* seg, int step, void* stream);
int ab_bctl_refine_stalled(const ab_bctl* c, void* stream);
/* zero the update of instances that are not live */
int ab_bctl_mask_update(const ab_bctl* c, int n, int np, const int* vinst, const int* pinst,
                        double* dx, double* dzl, double* dzu, void* stream);
/* q: seg_reduce with the update, gf and tau < 0; obj: objective per
 * instance.  Sets nu, phi0, dphi, alpha (primal step), az, search. */
int ab_bctl_ls_begin(const ab_bctl* c, const double* q, const double* obj, void* stream);
/* q, obj at the trial point: accept, or halve alpha and keep searching */
int ab_bctl_ls_test(const ab_bctl* c, const ab_bctl_opts* o, const double* q,
                    const double* obj, void* stream);
/* its += 1 for live instances */
int ab_bctl_end(const ab_bctl* c, void* stream);

/* Device pointer of a factorization's per-problem inertia, [npos, nneg]
 * per problem (valid after ab_ldl_factor, until the next one). */
int ab_ldl_inertia_device(ab_ldl_t h, const int** out);

#ifdef __cplusplus
}
#endif
#endif /* AMIGO_B200_H */

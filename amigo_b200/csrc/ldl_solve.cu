// Triangular solves with the multifrontal LDL^T factor (FP64).
//
// Forward sweep (levels ascending, one CTA per front): the front vector is
// assembled from the right-hand side of the node's own variables plus the
// update vectors of its children, placed by the same row map as the
// factorization's extend-add; L11 is applied in column blocks (one warp
// solves a block, the CTA updates the rows below it), the tail is kept as
// this front's update vector for the parent, and D^{-1} (1x1 / 2x2 blocks)
// gives the pivots' values.  Backward sweep (levels descending): the front
// gathers the final values of its delayed and contribution rows, applies
// L21^T and L11^T and writes its pivots.  The arithmetic is that of the
// reference's solve_ldl (include/sparse_ldl.h:1807-1908,
// solve_pivot_lower/diagonal/transpose 1550-1669) reorganised so that fronts
// of one level run concurrently without atomics.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "ldl_internal.h"
#include "launch_count.h"

namespace ab {
namespace {

constexpr int NT = kThreads;
constexpr int SB = 32;  // column block of the triangular solves

__device__ __forceinline__ int decode_var(int v) { return v >= 0 ? v : -v - 1; }

// Block end for pivot columns starting at jb: at most SB columns and never
// splitting a 2x2 pair (kind 1 = first column of a pair).
__device__ __forceinline__ int block_end(const int* kind, int jb, int npiv) {
  int je = jb + SB < npiv ? jb + SB : npiv;
  if (je < npiv && kind[je - 1] == 1) je++;
  return je;
}

// sum_{j < n} col[j * ld] * v(j), accumulated in the order of j, with the
// loads issued 16 at a time so that they overlap (the factor streams from
// HBM / L2 with hundreds of cycles of latency per load).
template <class T, class VF>
__device__ __forceinline__ double dot_strided(const T* __restrict__ col, size_t ld,
                                              int n, VF v) {
  double acc = 0.0;
  int j = 0;
  for (; j + 16 <= n; j += 16) {
    T a[16];
#pragma unroll
    for (int u = 0; u < 16; u++) a[u] = col[(size_t)(j + u) * ld];
#pragma unroll
    for (int u = 0; u < 16; u++) acc = __fma_rn((double)a[u], v(j + u), acc);
  }
  for (; j < n; j++) acc = __fma_rn((double)col[(size_t)j * ld], v(j), acc);
  return acc;
}

// One lane's share of sum_{i0 <= i < i1} col[i] v(i): rows i0 + lane + 32 t
// in the order of t, with the loads issued 8 at a time.
template <class T, class VF>
__device__ __forceinline__ double lane_dot(const T* __restrict__ col, int i0, int i1,
                                           int lane, VF v) {
  double acc = 0.0;
  int i = i0 + lane;
  for (; i + 7 * 32 < i1; i += 8 * 32) {
    T a[8];
    double b[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      a[u] = col[i + 32 * u];
      b[u] = v(i + 32 * u);
    }
#pragma unroll
    for (int u = 0; u < 8; u++) acc = __fma_rn((double)a[u], b[u], acc);
  }
  for (; i < i1; i += 32) acc = __fma_rn((double)col[i], v(i), acc);
  return acc;
}

// The 2x2 block of D applied to (x1, x2): every product and difference
// rounded on its own (no contraction), so that every kernel that solves
// with a 2x2 pivot gives the same bits.
__device__ __forceinline__ double inv2x2(double d11, double d21, double d22) {
  return __ddiv_rn(1.0, __dsub_rn(__dmul_rn(d11, d22), __dmul_rn(d21, d21)));
}
__device__ __forceinline__ double piv2_first(double inv, double d21, double d22,
                                             double x1, double x2) {
  return __dmul_rn(inv, __dsub_rn(__dmul_rn(d22, x1), __dmul_rn(d21, x2)));
}
__device__ __forceinline__ double piv2_second(double inv, double d11, double d21,
                                              double x1, double x2) {
  return __dmul_rn(inv, __dsub_rn(__dmul_rn(d11, x2), __dmul_rn(d21, x1)));
}

__device__ __forceinline__ double warp_sum_down(double a) {
  for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
  return a;
}

// The value of row j of a block held R rows per lane (row lane + 32 r in
// v[r]), broadcast to the warp.
template <int R>
__device__ __forceinline__ double warp_row(const double (&v)[R], int j) {
  double s = v[0];
#pragma unroll
  for (int r = 1; r < R; r++)
    if ((j >> 5) == r) s = v[r];
  return __shfl_sync(0xffffffffu, s, j & 31);
}

// One warp solves the unit lower triangle of a diagonal block (bw <= 32 R
// rows, column-major in sL with leading dimension lds, pivot kinds in sK)
// in place on V[0:bw], with the block's values in registers: each step is
// one broadcast and one multiply-add per row.  A 2x2 pair (kind 1, 2)
// eliminates both columns at once; its off-diagonal entry belongs to D.
template <int R>
__device__ __forceinline__ void warp_lower_solve(const double* sL, int lds,
                                                 const int* sK, int bw, double* V,
                                                 int lane) {
  double v[R];
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = lane + 32 * r;
    v[r] = i < bw ? V[i] : 0.0;
  }
  for (int j = 0; j < bw;) {
    const bool two = sK[j] == 1;
    const double v0 = warp_row<R>(v, j);
    const double v1 = two ? warp_row<R>(v, j + 1) : 0.0;
    const int i0 = j + (two ? 2 : 1);
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int i = lane + 32 * r;
      if (i >= i0 && i < bw) {
        double t = __dmul_rn(sL[i + j * lds], v0);
        if (two) t = __fma_rn(sL[i + (j + 1) * lds], v1, t);
        v[r] = __dsub_rn(v[r], t);
      }
    }
    j = i0;
  }
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = lane + 32 * r;
    if (i < bw) V[i] = v[r];
  }
}

// One warp solves the unit upper triangle L^T of a diagonal block in place
// on V[0:bw], from the last pivot backwards: once a pivot's value is final
// it is broadcast and every earlier row subtracts its term.
template <int R>
__device__ __forceinline__ void warp_upper_solve(const double* sL, int lds,
                                                 const int* sK, int bw, double* V,
                                                 int lane) {
  double v[R];
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = lane + 32 * r;
    v[r] = i < bw ? V[i] : 0.0;
  }
  for (int j = bw - 1; j >= 0;) {
    const bool two = sK[j] == 2;
    const int jl = two ? j - 1 : j;
    const double xj = warp_row<R>(v, j);
    const double xl = two ? warp_row<R>(v, jl) : 0.0;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int i = lane + 32 * r;
      if (i < jl) {
        double t = __dmul_rn(sL[j + i * lds], xj);
        if (two) t = __fma_rn(sL[jl + i * lds], xl, t);
        v[r] = __dsub_rn(v[r], t);
      }
    }
    j = jl - 1;
  }
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = lane + 32 * r;
    if (i < bw) V[i] = v[r];
  }
}

// Programmatic dependent launch (see the factorization's pdl_enter): wait
// for the previous kernel of the stream, then let the next be scheduled.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Front vector of `node` for one right-hand side: the node's own entries
// of the right-hand side plus the update vectors of its children, placed
// by the same row map as the factorization's extend-add.  Called by a
// whole CTA; V may be shared or global memory.
template <int NTH = NT>
__device__ void assemble_front_vector(const DevicePlan& d, int node, double* V,
                                      const double* xr, const double* ubuf,
                                      const long long* uoff, int rhs,
                                      int* s_choff) {
  const int tid = threadIdx.x;
  const int f = d.f[node];
  const int ns = d.ns[node], ndin = d.ndin[node];
  const int fs = ns + ndin;
  const int* fsinv = d.ipool + d.ioff[node] + 2 * f;
  for (int r = tid; r < f; r += NTH) V[r] = 0.0;
  __syncthreads();
  const int vb = d.var_ptr[node];
  for (int r = tid; r < ns; r += NTH) V[fsinv[r]] = xr[d.vars[vb + r]];
  __syncthreads();
  if (tid == 0) *s_choff = ns;
  __syncthreads();
  for (int q = d.kid_ptr[node]; q < d.kid_ptr[node + 1]; q++) {
    const int c = d.kids[q];
    const int fc = d.f[c], npc = d.npiv[c], ndc = d.ndel[c];
    const int cc = fc - npc;
    const double* uc = ubuf + uoff[c] + (long long)rhs * fc + npc;
    const int cb = d.cptr[c];
    const int choff = *s_choff;
    for (int a = tid; a < cc; a += NTH) {
      int pos;
      if (a < ndc) {
        pos = choff + a;
      } else {
        int r0 = d.cmap[cb + a - ndc];
        pos = r0 < ns ? r0 : r0 + ndin;
      }
      if (pos < fs) pos = fsinv[pos];
      V[pos] += __ldcg(uc + a);  // written by another CTA (queue sweeps)
    }
    __syncthreads();
    if (tid == 0) *s_choff = choff + ndc;
    __syncthreads();
  }
}

// Shared scratch of the one-CTA front solves.
struct NarrowSmem {
  int choff;
  double L[(SB + 1) * (SB + 1)];
  int K[SB + 1];  // the block's pivot kinds
};

// Forward solve of one front by the whole CTA (sV: dynamic shared memory
// of smem_doubles).
template <class T, int NTH = NT>
__device__ void forward_front(const DevicePlan& d, int node, double* x, int nrhs,
                              int ldx, double* ubuf, const long long* uoff,
                              int smem_doubles, double* sV, NarrowSmem& sm) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int f = d.f[node], npiv = d.npiv[node];
  const int* fvars = d.ipool + d.ioff[node];
  const int* kind = fvars + 3 * f;
  const T* L = reinterpret_cast<const T*>(d.fpool) + d.foff[node];
  int& s_choff = sm.choff;
  double* sL = sm.L;
  int* sK = sm.K;

  for (int rhs = 0; rhs < nrhs; rhs++) {
    // The front vector is worked on in shared memory when it fits (every
    // step of the in-block triangular solve depends on the previous one);
    // its tail is stored in ubuf for the parent.
    double* G = ubuf + uoff[node] + (long long)rhs * f;
    double* V = f <= smem_doubles ? sV : G;
    double* xr = x + (long long)rhs * ldx;
    assemble_front_vector<NTH>(d, node, V, xr, ubuf, uoff, rhs, &s_choff);

    // Forward elimination with the unit lower factor.  The diagonal block
    // of each column block is staged in shared memory first, so that the
    // dependent steps of the warp's triangular solve read no global memory.
    for (int jb = 0; jb < npiv;) {
      const int je = block_end(kind, jb, npiv);
      const int bw = je - jb;
      for (int t = tid; t < bw * bw; t += NTH) {
        const int i = t % bw, j = t / bw;
        sL[i + j * (SB + 1)] = L[jb + i + (size_t)(jb + j) * f];
      }
      for (int t = tid; t < bw; t += NTH) sK[t] = kind[jb + t];
      __syncthreads();
      if (warp == 0) warp_lower_solve<2>(sL, SB + 1, sK, bw, V + jb, lane);
      __syncthreads();
      for (int i = je + tid; i < f; i += NTH)
        V[i] -= dot_strided(L + i + (size_t)jb * f, (size_t)f, bw,
                            [&](int j) { return V[jb + j]; });
      __syncthreads();
      jb = je;
    }
    // D^{-1} and the pivots' forward values.
    for (int j = tid; j < npiv; j += NTH) {
      const int kd = kind[j];
      if (kd == 0) {
        V[j] = V[j] / L[j + (size_t)j * f];
      } else if (kd == 1) {
        const double d11 = L[j + (size_t)j * f];
        const double d21 = L[j + 1 + (size_t)j * f];
        const double d22 = L[j + 1 + (size_t)(j + 1) * f];
        const double inv = inv2x2(d11, d21, d22);
        const double x1 = V[j], x2 = V[j + 1];
        V[j] = piv2_first(inv, d21, d22, x1, x2);
        V[j + 1] = piv2_second(inv, d11, d21, x1, x2);
      }
    }
    __syncthreads();
    for (int j = tid; j < npiv; j += NTH) xr[decode_var(fvars[j])] = V[j];
    if (V != G)
      for (int r = npiv + tid; r < f; r += NTH) G[r] = V[r];
    __syncthreads();
  }
}

template <class T, int NTH = NT>
__global__ void __launch_bounds__(NTH)
k_solve_forward(DevicePlan d, const int* __restrict__ nodes, double* x,
                int nrhs, int ldx, double* ubuf, const long long* uoff,
                int smem_doubles) {
  pdl_enter();
  extern __shared__ double sV[];
  __shared__ NarrowSmem sm;
  forward_front<T, NTH>(d, nodes[blockIdx.x], x, nrhs, ldx, ubuf, uoff, smem_doubles, sV, sm);
}

// Backward solve of one front by the whole CTA.
template <class T, int NTH = NT>
__device__ void backward_front(const DevicePlan& d, int node, double* x, int nrhs,
                               int ldx, double* ubuf, const long long* uoff,
                               int smem_doubles, double* sV, NarrowSmem& sm) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NWARP = NTH / 32;
  const int f = d.f[node], npiv = d.npiv[node];
  const int* fvars = d.ipool + d.ioff[node];
  const int* kind = fvars + 3 * f;
  const T* L = reinterpret_cast<const T*>(d.fpool) + d.foff[node];
  double* sL = sm.L;
  int* sK = sm.K;
  for (int rhs = 0; rhs < nrhs; rhs++) {
    double* V = f <= smem_doubles ? sV : ubuf + uoff[node] + (long long)rhs * f;
    double* xr = x + (long long)rhs * ldx;
    // pivots: their forward values (written to x by the forward sweep);
    // delayed and contribution rows: final values of the ancestors (from
    // L2: another CTA of the same sweep may have written them)
    for (int r = tid; r < npiv; r += NTH) V[r] = xr[decode_var(fvars[r])];
    for (int r = npiv + tid; r < f; r += NTH) V[r] = __ldcg(xr + fvars[r]);
    __syncthreads();
    // Column blocks from the last one backwards.
    int je = npiv;
    while (je > 0) {
      int jb = je - SB > 0 ? je - SB : 0;
      if (jb > 0 && kind[jb] == 2) jb--;  // keep 2x2 pairs together
      // t[j] -= sum_{i >= je} L[i, j] t[i] for j in [jb, je): one warp per
      // column, lanes over rows.
      for (int j = jb + warp; j < je; j += NWARP) {
        const double acc = warp_sum_down(
            lane_dot(L + (size_t)j * f, je, f, lane, [&](int i) { return V[i]; }));
        if (lane == 0) V[j] -= acc;
      }
      const int bw = je - jb;
      for (int t = tid; t < bw * bw; t += NTH) {
        const int i = t % bw, j = t / bw;
        sL[i + j * (SB + 1)] = L[jb + i + (size_t)(jb + j) * f];
      }
      for (int t = tid; t < bw; t += NTH) sK[t] = kind[jb + t];
      __syncthreads();
      // within the block, backwards: column j (or pair j-1, j)
      if (warp == 0) warp_upper_solve<2>(sL, SB + 1, sK, bw, V + jb, lane);
      __syncthreads();
      je = jb;
    }
    for (int j = tid; j < npiv; j += NTH) xr[decode_var(fvars[j])] = V[j];
    __syncthreads();
  }
}

template <class T, int NTH = NT>
__global__ void __launch_bounds__(NTH)
k_solve_backward(DevicePlan d, const int* __restrict__ nodes, double* x,
                 int nrhs, int ldx, double* ubuf, const long long* uoff,
                 int smem_doubles) {
  pdl_enter();
  extern __shared__ double sV[];
  __shared__ NarrowSmem sm;
  backward_front<T, NTH>(d, nodes[blockIdx.x], x, nrhs, ldx, ubuf, uoff, smem_doubles, sV, sm);
}

// Narrow fronts of at most kSmallRows rows run on CTAs of kSmallThreads
// threads (more fronts in flight per SM; the same steps in the same order,
// so the same bits).
constexpr int kSmallRows = 128;
constexpr int kSmallThreads = 128;

// ---------------------------------------------------------------------------
// Work-queue sweeps over the levels whose fronts are all narrow: one launch
// per sweep instead of one per level.  `nodes` lists the fronts in the
// order of a sweep (forward: level by level from the leaves; backward: the
// reverse); each CTA takes the next front from an atomic counter, waits
// until the fronts it depends on are done (forward: its children;
// backward: its parent, when the parent is in the queue), solves it and
// marks it done with this sweep's epoch.  Fronts are handed out in
// dependency order and a CTA takes a front only while it runs, so the
// earliest unfinished front always has its dependencies done: the waits
// end.  Each wait is still bounded; when one runs out the kernel records
// it in *err (the host reports it) and goes on.
constexpr long long kQueuePolls = 1ll << 22;

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void wait_done(const unsigned* flag, unsigned epoch, int* err) {
  for (long long it = 0; it < kQueuePolls; it++) {
    if (ld_acquire(flag) == epoch) return;
    __nanosleep(64);
  }
  atomicOr(err, 1);
}

// Take the next queue entry (-1 when the queue is exhausted).
__device__ __forceinline__ int queue_next(unsigned* ctr, int count, int* s_idx) {
  __syncthreads();
  if (threadIdx.x == 0) *s_idx = (int)atomicAdd(ctr, 1u);
  __syncthreads();
  const int idx = *s_idx;
  return idx < count ? idx : -1;
}

// This front's results are visible GPU-wide before its done flag.
__device__ __forceinline__ void mark_done(unsigned* flag, unsigned epoch) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) st_release(flag, epoch);
}

// Start of a solve's two queued sweeps: zero both queue counters and move
// to the next epoch (ctr[2]).  The epoch lives in device memory, so a
// captured CUDA graph of a solve takes a new epoch on every replay.
__global__ void k_sweep_begin(unsigned* ctr) {
  if (threadIdx.x == 0) {
    ctr[0] = 0u;
    ctr[1] = 0u;
    ctr[2] = ctr[2] + 1u;
  }
}

template <class T, int NTH = NT>
__global__ void __launch_bounds__(NTH)
k_solve_forward_q(DevicePlan d, const int* __restrict__ nodes, int count, double* x,
                  int nrhs, int ldx, double* ubuf, const long long* uoff,
                  int smem_doubles, unsigned* ctr, unsigned* done, const unsigned* ep,
                  int* err) {
  pdl_enter();
  extern __shared__ double sV[];
  __shared__ NarrowSmem sm;
  __shared__ int s_idx;
  const unsigned epoch = *ep;
  for (;;) {
    const int idx = queue_next(ctr, count, &s_idx);
    if (idx < 0) break;
    const int node = nodes[idx];
    for (int q = d.kid_ptr[node] + threadIdx.x; q < d.kid_ptr[node + 1]; q += NTH)
      wait_done(done + d.kids[q], epoch, err);
    __syncthreads();
    forward_front<T, NTH>(d, node, x, nrhs, ldx, ubuf, uoff, smem_doubles, sV, sm);
    mark_done(done + node, epoch);
  }
}

template <class T, int NTH = NT>
__global__ void __launch_bounds__(NTH)
k_solve_backward_q(DevicePlan d, const int* __restrict__ nodes,
                   const int* __restrict__ dep, int count, double* x, int nrhs,
                   int ldx, double* ubuf, const long long* uoff, int smem_doubles,
                   unsigned* ctr, unsigned* done, const unsigned* ep, int* err) {
  pdl_enter();
  extern __shared__ double sV[];
  __shared__ NarrowSmem sm;
  __shared__ int s_idx;
  const unsigned epoch = *ep;
  for (;;) {
    const int idx = queue_next(ctr, count, &s_idx);
    if (idx < 0) break;
    const int node = nodes[idx];
    if (threadIdx.x == 0 && dep[idx] >= 0) wait_done(done + dep[idx], epoch, err);
    __syncthreads();
    backward_front<T, NTH>(d, node, x, nrhs, ldx, ubuf, uoff, smem_doubles, sV, sm);
    mark_done(done + node, epoch);
  }
}


// ---------------------------------------------------------------------------
// Mid-size fronts: one thread-block cluster of CS CTAs per front.  CTA 0
// solves the pivot block (the blocked triangular solve of the narrow
// kernel, over the pivot rows only, with the front vector's pivot part in
// its shared memory); the contribution rows' product with the pivot block
// (the update vector passed to the parent, forward; the pivots' right-hand
// side correction, backward) is spread over all CS CTAs, which read the
// front's L21 once.  The cluster barrier orders CTA 0's results before the
// other CTAs read them from HBM (cluster-scope release / acquire).
constexpr int CS = 8;

// dst[0:n] = src[0:n] from L2 (src may have been written by another CTA).
__device__ __forceinline__ void copy_cg(double* dst, const double* src, int n) {
  for (int t = threadIdx.x; t < n; t += NT) dst[t] = __ldcg(src + t);
}

template <class T>
__global__ void __launch_bounds__(NT, 1)
k_clu_forward(DevicePlan d, const int* __restrict__ nodes, double* x,
              int nrhs, int ldx, double* ubuf, const long long* uoff) {
  pdl_enter();
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ double sm[];
  __shared__ double sL[(SB + 1) * (SB + 1)];
  __shared__ int sK[SB + 1];
  __shared__ int s_choff;
  const int cr = (int)cluster.block_rank();
  const int node = nodes[blockIdx.x / CS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NWARP = NT / 32;
  const int f = d.f[node], npiv = d.npiv[node];
  const int* fvars = d.ipool + d.ioff[node];
  const int* kind = fvars + 3 * f;
  const T* L = reinterpret_cast<const T*>(d.fpool) + d.foff[node];
  double* sv = sm;                 // CTA 0: pivot values; others: y1 copy
  double* part = sm + npiv;        // NWARP x 32 partial sums
  for (int rhs = 0; rhs < nrhs; rhs++) {
    double* G = ubuf + uoff[node] + (long long)rhs * f;
    double* xr = x + (long long)rhs * ldx;
    if (cr == 0) {
      assemble_front_vector(d, node, G, xr, ubuf, uoff, rhs, &s_choff);
      __syncthreads();
      for (int t = tid; t < npiv; t += NT) sv[t] = G[t];
      __syncthreads();
      for (int jb = 0; jb < npiv;) {
        const int je = block_end(kind, jb, npiv);
        const int bw = je - jb;
        for (int t = tid; t < bw * bw; t += NT) {
          const int i = t % bw, j = t / bw;
          sL[i + j * (SB + 1)] = L[jb + i + (size_t)(jb + j) * f];
        }
        for (int t = tid; t < bw; t += NT) sK[t] = kind[jb + t];
        __syncthreads();
        if (warp == 0) warp_lower_solve<2>(sL, SB + 1, sK, bw, sv + jb, lane);
        __syncthreads();
        // the pivot rows below the block
        for (int i = je + tid; i < npiv; i += NT)
          sv[i] -= dot_strided(L + i + (size_t)jb * f, (size_t)f, bw,
                               [&](int j) { return sv[jb + j]; });
        __syncthreads();
        jb = je;
      }
      for (int t = tid; t < npiv; t += NT) G[t] = sv[t];
    }
    cluster.sync();
    // contribution rows: G[i] -= L21[i, :] y1, 32-row strips over the
    // cluster's CTAs, the pivot columns split over the CTA's warps and the
    // warps' partial sums added in a fixed order
    if (cr != 0) copy_cg(sv, G, npiv);
    __syncthreads();
    const int ncr = f - npiv;
    const int nstrip = (ncr + 31) / 32;
    const int jc = (npiv + NWARP - 1) / NWARP;
    const int j0 = warp * jc, j1 = min(npiv, j0 + jc);
    for (int st = cr; st < nstrip; st += CS) {
      const int i = npiv + st * 32 + lane;
      double acc = 0.0;
      if (i < f && j1 > j0)
        acc = dot_strided(L + i + (size_t)j0 * f, (size_t)f, j1 - j0,
                          [&](int j) { return sv[j0 + j]; });
      part[warp * 32 + lane] = acc;
      __syncthreads();
      if (warp == 0 && i < f) {
        double s = 0.0;
        for (int w = 0; w < NWARP; w++) s += part[w * 32 + lane];
        G[i] = __ldcg(G + i) - s;
      }
      __syncthreads();
    }
    // D^{-1} and the pivots' values (CTA 0, from its shared copy)
    if (cr == 0) {
      for (int j = tid; j < npiv; j += NT) {
        const int kd = kind[j];
        double v = sv[j];
        if (kd == 0) {
          v = sv[j] / (double)L[j + (size_t)j * f];
        } else if (kd == 1) {
          const double d11 = L[j + (size_t)j * f];
          const double d21 = L[j + 1 + (size_t)j * f];
          const double d22 = L[j + 1 + (size_t)(j + 1) * f];
          const double inv = inv2x2(d11, d21, d22);
          v = piv2_first(inv, d21, d22, sv[j], sv[j + 1]);
        } else {
          const double d11 = L[j - 1 + (size_t)(j - 1) * f];
          const double d21 = L[j + (size_t)(j - 1) * f];
          const double d22 = L[j + (size_t)j * f];
          const double inv = inv2x2(d11, d21, d22);
          v = piv2_second(inv, d11, d21, sv[j - 1], sv[j]);
        }
        xr[decode_var(fvars[j])] = v;
      }
    }
    cluster.sync();
  }
}

template <class T>
__global__ void __launch_bounds__(NT, 1)
k_clu_backward(DevicePlan d, const int* __restrict__ nodes, double* x,
               int nrhs, int ldx, double* ubuf, const long long* uoff) {
  pdl_enter();
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ double sm[];
  __shared__ double sL[(SB + 1) * (SB + 1)];
  __shared__ int sK[SB + 1];
  const int cr = (int)cluster.block_rank();
  const int node = nodes[blockIdx.x / CS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NWARP = NT / 32;
  const int f = d.f[node], npiv = d.npiv[node];
  const int* fvars = d.ipool + d.ioff[node];
  const int* kind = fvars + 3 * f;
  const T* L = reinterpret_cast<const T*>(d.fpool) + d.foff[node];
  const int ncr = f - npiv;
  double* sx = sm;            // contribution rows' final values
  double* sv = sm + ncr;      // CTA 0: pivot values
  for (int rhs = 0; rhs < nrhs; rhs++) {
    double* G = ubuf + uoff[node] + (long long)rhs * f;
    double* xr = x + (long long)rhs * ldx;
    for (int r = tid; r < ncr; r += NT) sx[r] = xr[fvars[npiv + r]];
    __syncthreads();
    // t[j] = z[j] - L21[:, j]^T x2 for every pivot column, one warp per
    // column over the cluster's warps
    for (int j = cr * NWARP + warp; j < npiv; j += CS * NWARP) {
      const double acc = warp_sum_down(lane_dot(L + (size_t)j * f + npiv, 0, ncr, lane,
                                                [&](int i) { return sx[i]; }));
      if (lane == 0) G[j] = xr[decode_var(fvars[j])] - acc;
    }
    cluster.sync();
    if (cr == 0) {
      for (int t = tid; t < npiv; t += NT) sv[t] = __ldcg(G + t);
      __syncthreads();
      int je = npiv;
      while (je > 0) {
        int jb = je - SB > 0 ? je - SB : 0;
        if (jb > 0 && kind[jb] == 2) jb--;  // keep 2x2 pairs together
        // t[j] -= sum_{je <= i < npiv} L[i, j] t[i] for j in [jb, je)
        for (int j = jb + warp; j < je; j += NWARP) {
          const double acc = warp_sum_down(lane_dot(L + (size_t)j * f, je, npiv, lane,
                                                    [&](int i) { return sv[i]; }));
          if (lane == 0) sv[j] -= acc;
        }
        const int bw = je - jb;
        for (int t = tid; t < bw * bw; t += NT) {
          const int i = t % bw, j = t / bw;
          sL[i + j * (SB + 1)] = L[jb + i + (size_t)(jb + j) * f];
        }
        for (int t = tid; t < bw; t += NT) sK[t] = kind[jb + t];
        __syncthreads();
        if (warp == 0) warp_upper_solve<2>(sL, SB + 1, sK, bw, sv + jb, lane);
        __syncthreads();
        je = jb;
      }
      for (int j = tid; j < npiv; j += NT) xr[decode_var(fvars[j])] = sv[j];
    }
    cluster.sync();
  }
}

// ---------------------------------------------------------------------------
// Wide fronts (f * npiv large): one cooperative launch per level solves all
// of the level's wide fronts with every CTA of the GPU.  The front vectors
// live in ubuf (global memory).  Each column block of WB pivots alternates
// a sequential phase (one CTA per front solves the block's diagonal
// triangle in shared memory) with a parallel phase (all CTAs apply the
// block to the rows below it, forward, or to the columns left of it,
// backward), separated by grid-wide barriers.  Values other CTAs wrote
// since the last barrier are read with ld.global.cg (L2), never through
// the non-coherent L1.  Sums run in a fixed order: the result does not
// depend on the grid size.
constexpr int WB = 128;

__device__ __forceinline__ int block_end_w(const int* kind, int jb, int npiv) {
  int je = jb + WB < npiv ? jb + WB : npiv;
  if (je < npiv && kind[je - 1] == 1) je++;
  return je;
}

template <class T>
struct WideFront {
  int f, npiv;
  const int* fvars;
  const int* kind;
  const T* L;
  double* G;
};

template <class T>
__device__ __forceinline__ WideFront<T> wide_front(const DevicePlan& d, int node,
                                                double* ubuf,
                                                const long long* uoff,
                                                int rhs) {
  WideFront<T> w;
  w.f = d.f[node];
  w.npiv = d.npiv[node];
  w.fvars = d.ipool + d.ioff[node];
  w.kind = w.fvars + 3 * w.f;
  w.L = reinterpret_cast<const T*>(d.fpool) + d.foff[node];
  w.G = ubuf + uoff[node] + (long long)rhs * w.f;
  return w;
}

// Flattened work distribution: item g of a sequence in which front c owns
// cnt_c consecutive items goes to CTA g mod gridDim.x.  Returns this CTA's
// first item of front c, given the number of items before it.
__device__ __forceinline__ long long first_item(long long base) {
  const long long G = gridDim.x;
  long long r = ((long long)blockIdx.x - base) % G;
  return r < 0 ? r + G : r;
}

template <class T>
__global__ void __launch_bounds__(NT)
k_wide_forward(DevicePlan d, const int* __restrict__ nodes, int count,
               double* x, int nrhs, int ldx, double* ubuf,
               const long long* uoff, int* wst) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ double sm[];
  double* sL = sm;                         // (WB + 1)^2 diagonal block
  double* sv = sm + (WB + 1) * (WB + 1);   // WB + 1 block values
  __shared__ int sK[WB + 1];               // the block's pivot kinds
  __shared__ int s_choff;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int rhs = 0; rhs < nrhs; rhs++) {
    double* xr = x + (long long)rhs * ldx;
    for (int c = blockIdx.x; c < count; c += gridDim.x) {
      const WideFront<T> w = wide_front<T>(d, nodes[c], ubuf, uoff, rhs);
      assemble_front_vector(d, nodes[c], w.G, xr, ubuf, uoff, rhs, &s_choff);
      if (tid == 0) {
        wst[2 * c] = 0;
        wst[2 * c + 1] = 0;
      }
    }
    grid.sync();
    for (;;) {
      // sequential phase: next diagonal block of every front
      for (int c = blockIdx.x; c < count; c += gridDim.x) {
        const WideFront<T> w = wide_front<T>(d, nodes[c], ubuf, uoff, rhs);
        const int jb = __ldcg(wst + 2 * c + 1);
        if (jb >= w.npiv) {
          if (tid == 0) wst[2 * c] = jb;
          continue;
        }
        const int je = block_end_w(w.kind, jb, w.npiv);
        const int bw = je - jb;
        for (int t = tid; t < bw * bw; t += NT) {
          const int i = t % bw, j = t / bw;
          sL[i + j * (WB + 1)] = w.L[jb + i + (size_t)(jb + j) * w.f];
        }
        for (int t = tid; t < bw; t += NT) {
          sv[t] = __ldcg(w.G + jb + t);
          sK[t] = w.kind[jb + t];
        }
        __syncthreads();
        if (warp == 0) warp_lower_solve<(WB + 32) / 32>(sL, WB + 1, sK, bw, sv, lane);
        __syncthreads();
        for (int t = tid; t < bw; t += NT) w.G[jb + t] = sv[t];
        if (tid == 0) {
          wst[2 * c] = jb;
          wst[2 * c + 1] = je;
        }
        __syncthreads();
      }
      grid.sync();
      bool any = false;
      for (int c = 0; c < count && !any; c++)
        any = __ldcg(wst + 2 * c) < __ldcg(wst + 2 * c + 1);
      if (!any) break;
      // parallel phase: rows below the block, NT rows per item
      long long base = 0;
      for (int c = 0; c < count; c++) {
        const int jb = __ldcg(wst + 2 * c), je = __ldcg(wst + 2 * c + 1);
        if (jb >= je) continue;
        const WideFront<T> w = wide_front<T>(d, nodes[c], ubuf, uoff, rhs);
        const long long items = (w.f - je + NT - 1) / NT;
        const int bw = je - jb;
        bool staged = false;
        for (long long it = first_item(base); it < items; it += gridDim.x) {
          if (!staged) {
            __syncthreads();
            for (int t = tid; t < bw; t += NT) sv[t] = __ldcg(w.G + jb + t);
            __syncthreads();
            staged = true;
          }
          const int i = je + (int)it * NT + tid;
          if (i < w.f) {
            const double acc = dot_strided(w.L + i + (size_t)jb * w.f, (size_t)w.f, bw,
                                           [&](int j) { return sv[j]; });
            w.G[i] = __ldcg(w.G + i) - acc;
          }
        }
        base += items;
      }
      grid.sync();
    }
    // D^{-1} and the pivots' forward values
    for (int c = blockIdx.x; c < count; c += gridDim.x) {
      const WideFront<T> w = wide_front<T>(d, nodes[c], ubuf, uoff, rhs);
      for (int j = tid; j < w.npiv; j += NT) {
        const int kd = w.kind[j];
        const T* L = w.L;
        const size_t f = w.f;
        if (kd == 0) {
          w.G[j] = __ldcg(w.G + j) / L[j + j * f];
        } else if (kd == 1) {
          const double d11 = L[j + j * f];
          const double d21 = L[j + 1 + j * f];
          const double d22 = L[j + 1 + (j + 1) * f];
          const double inv = inv2x2(d11, d21, d22);
          const double x1 = __ldcg(w.G + j), x2 = __ldcg(w.G + j + 1);
          w.G[j] = piv2_first(inv, d21, d22, x1, x2);
          w.G[j + 1] = piv2_second(inv, d11, d21, x1, x2);
        }
      }
      __syncthreads();
      for (int j = tid; j < w.npiv; j += NT)
        xr[decode_var(w.fvars[j])] = __ldcg(w.G + j);
    }
    grid.sync();
  }
}

template <class T>
__global__ void __launch_bounds__(NT)
k_wide_backward(DevicePlan d, const int* __restrict__ nodes, int count,
                double* x, int nrhs, int ldx, double* ubuf,
                const long long* uoff, int* wst) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ double sm[];
  double* sL = sm;
  double* sv = sm + (WB + 1) * (WB + 1);
  __shared__ int sK[WB + 1];  // the block's pivot kinds
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NWARP = NT / 32;
  const long long gwarps = (long long)gridDim.x * NWARP;
  for (int rhs = 0; rhs < nrhs; rhs++) {
    double* xr = x + (long long)rhs * ldx;
    for (int c = blockIdx.x; c < count; c += gridDim.x) {
      const WideFront<T> w = wide_front<T>(d, nodes[c], ubuf, uoff, rhs);
      for (int r = tid; r < w.npiv; r += NT) w.G[r] = xr[decode_var(w.fvars[r])];
      for (int r = w.npiv + tid; r < w.f; r += NT) w.G[r] = xr[w.fvars[r]];
      if (tid == 0) {
        wst[2 * c] = w.npiv;
        wst[2 * c + 1] = w.npiv;
      }
    }
    grid.sync();
    // t[j] -= sum_{i >= npiv} L[i, j] t[i]: one warp per pivot column
    {
      long long base = 0;
      for (int c = 0; c < count; c++) {
        const WideFront<T> w = wide_front<T>(d, nodes[c], ubuf, uoff, rhs);
        const long long gw = (long long)blockIdx.x * NWARP + warp;
        long long r = (gw - base) % gwarps;
        if (r < 0) r += gwarps;
        for (long long j = r; j < w.npiv; j += gwarps) {
          const double acc = warp_sum_down(lane_dot(w.L + (size_t)j * w.f, w.npiv, w.f,
                                                    lane,
                                                    [&](int i) { return __ldcg(w.G + i); }));
          if (lane == 0) w.G[j] = __ldcg(w.G + j) - acc;
        }
        base += w.npiv;
      }
    }
    grid.sync();
    for (;;) {
      // sequential phase: the next diagonal block from the end
      for (int c = blockIdx.x; c < count; c += gridDim.x) {
        const WideFront<T> w = wide_front<T>(d, nodes[c], ubuf, uoff, rhs);
        const int je = __ldcg(wst + 2 * c);
        if (je <= 0) {
          if (tid == 0) wst[2 * c + 1] = je;
          continue;
        }
        int jb = je - WB > 0 ? je - WB : 0;
        if (jb > 0 && w.kind[jb] == 2) jb--;  // keep 2x2 pairs together
        const int bw = je - jb;
        for (int t = tid; t < bw * bw; t += NT) {
          const int i = t % bw, j = t / bw;
          sL[i + j * (WB + 1)] = w.L[jb + i + (size_t)(jb + j) * w.f];
        }
        for (int t = tid; t < bw; t += NT) {
          sv[t] = __ldcg(w.G + jb + t);
          sK[t] = w.kind[jb + t];
        }
        __syncthreads();
        if (warp == 0) warp_upper_solve<(WB + 32) / 32>(sL, WB + 1, sK, bw, sv, lane);
        __syncthreads();
        for (int t = tid; t < bw; t += NT) w.G[jb + t] = sv[t];
        if (tid == 0) {
          wst[2 * c] = jb;
          wst[2 * c + 1] = je;
        }
        __syncthreads();
      }
      grid.sync();
      bool any = false;
      for (int c = 0; c < count && !any; c++)
        any = __ldcg(wst + 2 * c) < __ldcg(wst + 2 * c + 1);
      if (!any) break;
      // parallel phase: t[j] -= sum_{i in block} L[i, j] t[i] for j < jb,
      // one warp per column
      long long base = 0;
      for (int c = 0; c < count; c++) {
        const int jb = __ldcg(wst + 2 * c), je = __ldcg(wst + 2 * c + 1);
        if (jb >= je) continue;
        const WideFront<T> w = wide_front<T>(d, nodes[c], ubuf, uoff, rhs);
        const long long gw = (long long)blockIdx.x * NWARP + warp;
        long long r = (gw - base) % gwarps;
        if (r < 0) r += gwarps;
        for (long long j = r; j < jb; j += gwarps) {
          const double acc = warp_sum_down(lane_dot(w.L + (size_t)j * w.f, jb, je, lane,
                                                    [&](int i) { return __ldcg(w.G + i); }));
          if (lane == 0) w.G[j] = __ldcg(w.G + j) - acc;
        }
        base += jb;
      }
      grid.sync();
    }
    for (int c = blockIdx.x; c < count; c += gridDim.x) {
      const WideFront<T> w = wide_front<T>(d, nodes[c], ubuf, uoff, rhs);
      for (int j = tid; j < w.npiv; j += NT)
        xr[decode_var(w.fvars[j])] = __ldcg(w.G + j);
    }
    grid.sync();
  }
}

}  // namespace

#define SCUDA(call)                                                       \
  do {                                                                    \
    cudaError_t e__ = (call);                                             \
    if (e__ != cudaSuccess) {                                             \
      std::fprintf(stderr, "amigo_b200: %s: %s\n", #call,                 \
                   cudaGetErrorString(e__));                              \
      return -2;                                                          \
    }                                                                     \
  } while (0)

// A launch that may start while the previous kernel of the stream drains
// (programmatic stream serialization; the kernel waits in pdl_enter).
template <class... KArgs, class... Args>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block,
                              size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// One cluster of CS CTAs per front (cudaLaunchKernelEx with a cluster
// dimension).
template <class K>
static int launch_cluster(K kernel, int fronts, int smem, cudaStream_t s,
                          const DevicePlan& d, const int* nodes, double* x,
                          int nrhs, int ldx, double* ubuf, const long long* uoff) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(fronts * CS);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CS;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 2;
  SCUDA(cudaLaunchKernelEx(&cfg, kernel, d, nodes, x, nrhs, ldx, ubuf, uoff));
  ab::count_launch();
  return 0;
}

// Per level: narrow fronts (one CTA each), cluster fronts (CS CTAs each)
// and wide fronts, from the sizes of the last factorization.
static int build_solve_schedule(LdlHandle& h, cudaStream_t s) {
  const int L = h.d.num_levels, nn = h.d.nn;
  // unchanged front sizes (the usual case between IPM iterations): keep it
  if (h.sv_f == h.h_f && h.sv_npiv == h.h_npiv && !h.sv_narrow_ptr.empty() &&
      h.sv_wide_entries == h.wide_entries) {
    h.solve_epoch = h.factor_epoch;
    return 0;
  }
  std::vector<int>& nodes = h.sv_host;
  nodes.clear();
  nodes.reserve(nn);
  h.sv_narrow_ptr.assign(L + 1, 0);
  h.sv_clu_ptr.assign(L + 1, 0);
  h.sv_wide_ptr.assign(L + 1, 0);
  h.sv_narrow_smem.assign(L, 0);
  h.sv_clu_smem.assign(L, 0);
  h.sv_max_wide = 0;
  // a front's class: narrow (one CTA), cluster (CS CTAs) or wide (the
  // cooperative grid), from f * npiv and, for clusters, the front vector
  // fitting in shared memory
  auto cls = [&](int k) {
    const long long e = (long long)h.h_f[k] * h.h_npiv[k];
    if (e >= h.wide_entries) return 2;
    if (e >= h.cluster_entries && ((long long)h.h_f[k] + NT) * 8 <= kMaxDynSmem) return 1;
    return 0;
  };
  h.sv_small_cnt.assign(L, 0);
  h.sv_small_smem.assign(L, 0);
  for (int l = 0; l < L; l++) {
    h.sv_narrow_ptr[l] = (int)nodes.size();
    int fm = 0, fsm = 0;
    // narrow fronts: the small ones (kSmallThreads-thread CTAs) first
    for (int pass = 0; pass < 2; pass++)
      for (int q = h.level_ptr[l]; q < h.level_ptr[l + 1]; q++) {
        const int k = h.level_nodes[q];
        if (cls(k) == 0 && (h.h_f[k] <= kSmallRows) == (pass == 0)) {
          nodes.push_back(k);
          if (pass == 0) {
            h.sv_small_cnt[l]++;
            fsm = std::max(fsm, h.h_f[k]);
          } else {
            fm = std::max(fm, h.h_f[k]);
          }
        }
      }
    h.sv_small_smem[l] = fsm * 8;
    h.sv_narrow_smem[l] =
        (int)std::min<long long>((long long)fm * 8, kMaxDynSmem);
    h.sv_clu_ptr[l] = (int)nodes.size();
    int cm = 0;
    for (int q = h.level_ptr[l]; q < h.level_ptr[l + 1]; q++) {
      const int k = h.level_nodes[q];
      if (cls(k) == 1) {
        nodes.push_back(k);
        cm = std::max(cm, h.h_f[k]);
      }
    }
    h.sv_clu_smem[l] = (int)std::min<long long>(((long long)cm + NT) * 8, kMaxDynSmem);
    h.sv_wide_ptr[l] = (int)nodes.size();
    for (int q = h.level_ptr[l]; q < h.level_ptr[l + 1]; q++) {
      const int k = h.level_nodes[q];
      if (cls(k) == 2) nodes.push_back(k);
    }
    h.sv_max_wide = std::max(h.sv_max_wide,
                             (int)nodes.size() - h.sv_wide_ptr[l]);
  }
  h.sv_narrow_ptr[L] = h.sv_clu_ptr[L] = h.sv_wide_ptr[L] = (int)nodes.size();
  if (!h.sv_nodes) SCUDA(cudaMalloc((void**)&h.sv_nodes, std::max(nn, 1) * sizeof(int)));
  if (h.sv_max_wide > h.sv_state_cap) {
    if (h.sv_state) SCUDA(cudaFree(h.sv_state));
    h.sv_state = nullptr;
    h.sv_state_cap = std::max(h.sv_max_wide, 16);
    SCUDA(cudaMalloc((void**)&h.sv_state, 2 * h.sv_state_cap * sizeof(int)));
  }
  // nodes is a member: it outlives the asynchronous copy
  SCUDA(cudaMemcpyAsync(h.sv_nodes, nodes.data(), nodes.size() * sizeof(int),
                        cudaMemcpyHostToDevice, s));
  // the all-narrow levels from the leaves, swept by one work-queue launch
  // each way (worth it from two levels)
  int ql = 0;
  while (ql < L && h.sv_clu_ptr[ql] == h.sv_narrow_ptr[ql + 1]) ql++;
  h.sv_qlevels = ql >= 2 ? ql : 0;
  h.sv_qcount = h.sv_qlevels ? h.sv_narrow_ptr[h.sv_qlevels] : 0;
  h.sv_qsmall = true;
  int qsm = 0;
  for (int l = 0; l < h.sv_qlevels; l++) {
    if (h.sv_small_cnt[l] != h.sv_clu_ptr[l] - h.sv_narrow_ptr[l]) h.sv_qsmall = false;
    qsm = std::max(qsm, h.sv_small_smem[l]);
  }
  h.sv_qsmall_smem = qsm;
  if (h.sv_qcount) {
    const int qc = h.sv_qcount;
    // position of each queued node in the forward order
    std::vector<int> pos(nn, -1);
    for (int i = 0; i < qc; i++) pos[nodes[i]] = i;
    std::vector<int>& bq = h.sv_bq_host;
    std::vector<int>& dep = h.sv_dep_host;
    bq.resize(qc);
    dep.resize(qc);
    int sm = 0;
    for (int l = 0; l < h.sv_qlevels; l++) sm = std::max(sm, h.sv_narrow_smem[l]);
    h.sv_qsmem = sm;
    for (int i = 0; i < qc; i++) {
      const int k = nodes[qc - 1 - i];
      const int par = h.sym.node_parent[k];
      bq[i] = k;
      dep[i] = (par >= 0 && pos[par] >= 0) ? par : -1;
    }
    if (!h.sv_bq) {
      SCUDA(cudaMalloc((void**)&h.sv_bq, std::max(nn, 1) * sizeof(int)));
      SCUDA(cudaMalloc((void**)&h.sv_dep, std::max(nn, 1) * sizeof(int)));
      SCUDA(cudaMalloc((void**)&h.sv_done, 2 * (size_t)std::max(nn, 1) * sizeof(unsigned)));
      SCUDA(cudaMalloc((void**)&h.sv_ctr, 4 * sizeof(unsigned)));
      SCUDA(cudaMalloc((void**)&h.sv_err, sizeof(int)));
      SCUDA(cudaMemsetAsync(h.sv_done, 0, 2 * (size_t)std::max(nn, 1) * sizeof(unsigned), s));
      SCUDA(cudaMemsetAsync(h.sv_ctr, 0, 4 * sizeof(unsigned), s));
      SCUDA(cudaMemsetAsync(h.sv_err, 0, sizeof(int), s));
    }
    SCUDA(cudaMemcpyAsync(h.sv_bq, bq.data(), qc * sizeof(int), cudaMemcpyHostToDevice, s));
    SCUDA(cudaMemcpyAsync(h.sv_dep, dep.data(), qc * sizeof(int), cudaMemcpyHostToDevice, s));
  }
  h.sv_qgrid = 0;
  h.sv_f = h.h_f;
  h.sv_npiv = h.h_npiv;
  h.sv_fwd_grid.clear();
  h.sv_wide_entries = h.wide_entries;
  h.solve_epoch = h.factor_epoch;
  return 0;
}

template <class T>
static int launch_solve(LdlHandle& h, double* d_x, int nrhs, int ldx,
                        cudaStream_t s) {
  DevicePlan& d = h.d;
  static bool attr_set = false;
  static int wide_grid = 0;
  const size_t wide_smem = ((WB + 1) * (WB + 1) + WB + 1) * sizeof(double);
  if (!attr_set) {
    SCUDA(cudaFuncSetAttribute(k_solve_forward<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kMaxDynSmem));
    SCUDA(cudaFuncSetAttribute(k_solve_backward<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kMaxDynSmem));
    SCUDA(cudaFuncSetAttribute(k_solve_forward_q<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kMaxDynSmem));
    SCUDA(cudaFuncSetAttribute(k_solve_backward_q<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kMaxDynSmem));
    SCUDA(cudaFuncSetAttribute(k_clu_forward<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kMaxDynSmem));
    SCUDA(cudaFuncSetAttribute(k_clu_backward<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kMaxDynSmem));
    SCUDA(cudaFuncSetAttribute(k_wide_forward<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)wide_smem));
    SCUDA(cudaFuncSetAttribute(k_wide_backward<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)wide_smem));
    int dev = 0, sms = 0, bf = 0, bb = 0;
    SCUDA(cudaGetDevice(&dev));
    SCUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf, k_wide_forward<T>, NT,
                                                        wide_smem));
    SCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bb, k_wide_backward<T>,
                                                        NT, wide_smem));
    wide_grid = sms * std::max(1, std::min(bf, bb));
    attr_set = true;
  }
  if ((int)h.sv_fwd_grid.size() != d.num_levels || h.sv_grid_cap != wide_grid) {
    // Cooperative grids sized to the level's work (a grid-wide barrier
    // costs more the more CTAs it spans): forward, one CTA per NT rows of
    // the level's wide fronts; backward, one per 8 pivot columns (one warp
    // each); at least one per front, at most what is co-resident.
    h.sv_fwd_grid.assign(d.num_levels, 1);
    h.sv_bwd_grid.assign(d.num_levels, 1);
    for (int l = 0; l < d.num_levels; l++) {
      long long fr = 0, bc = 0;
      const int wc = h.sv_narrow_ptr[l + 1] - h.sv_wide_ptr[l];
      for (int q = h.sv_wide_ptr[l]; q < h.sv_narrow_ptr[l + 1]; q++) {
        const int k = h.sv_host[q];
        fr += (h.h_f[k] + NT - 1) / NT;
        bc += (h.h_npiv[k] + 7) / 8;
      }
      h.sv_fwd_grid[l] = (int)std::min<long long>(wide_grid, std::max<long long>(fr, wc));
      h.sv_bwd_grid[l] = (int)std::min<long long>(wide_grid, std::max<long long>(bc, wc));
      h.sv_fwd_grid[l] = std::max(h.sv_fwd_grid[l], 1);
      h.sv_bwd_grid[l] = std::max(h.sv_bwd_grid[l], 1);
    }
    h.sv_grid_cap = wide_grid;
  }
  int* wst = h.sv_state;
  // AMIGO_B200_TRACE=1: device time of every level's sweeps (diagnostics)
  static const bool trace = std::getenv("AMIGO_B200_TRACE") != nullptr;
  std::vector<cudaEvent_t> ev;
  if (trace) {
    ev.resize(2 * d.num_levels + 2);
    for (auto& e : ev) cudaEventCreate(&e);
  }
  const bool queue = (h.solve_queue & 1) && h.sv_qcount > 0;
  const bool small = (h.solve_queue & 2) != 0;
  const bool qsmall = queue && small && h.sv_qsmall;
  const int qth = qsmall ? kSmallThreads : NT;
  const int qsm = qsmall ? h.sv_qsmall_smem : h.sv_qsmem;
  const unsigned* ep = h.sv_ctr + 2;   // this solve's epoch, set on the device
  if (queue) {
    if (h.sv_qgrid == 0 || h.sv_qgrid_small != qsmall) {
      // CTAs resident at once, at most one per queued front
      int dev = 0, sms = 0, per = 0;
      SCUDA(cudaGetDevice(&dev));
      SCUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      if (qsmall)
        SCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per, k_solve_forward_q<T, kSmallThreads>, kSmallThreads, (size_t)qsm));
      else
        SCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_solve_forward_q<T>, NT,
                                                            (size_t)qsm));
      h.sv_qgrid = std::max(1, std::min(h.sv_qcount, sms * std::max(per, 1)));
      h.sv_qgrid_small = qsmall;
    }
    { k_sweep_begin<<<1, 32, 0, s>>>(h.sv_ctr); ab::count_launch(); }
    SCUDA(cudaGetLastError());
    if (qsmall)
      SCUDA(launch_pdl(k_solve_forward_q<T, kSmallThreads>, dim3(h.sv_qgrid), dim3(qth),
                       (size_t)qsm, s, d, (const int*)h.sv_nodes, h.sv_qcount, d_x, nrhs,
                       ldx, h.ubuf, (const long long*)h.uoff, qsm / 8, h.sv_ctr, h.sv_done,
                       ep, h.sv_err));
    else
      SCUDA(launch_pdl(k_solve_forward_q<T>, dim3(h.sv_qgrid), dim3(qth), (size_t)qsm, s, d,
                       (const int*)h.sv_nodes, h.sv_qcount, d_x, nrhs, ldx, h.ubuf,
                       (const long long*)h.uoff, qsm / 8, h.sv_ctr, h.sv_done, ep,
                       h.sv_err));
    ab::count_launch();
  }
  for (int l = queue ? h.sv_qlevels : 0; l < d.num_levels; l++) {
    if (trace) cudaEventRecord(ev[l], s);
    int b = h.sv_narrow_ptr[l], cnt = h.sv_clu_ptr[l] - b;
    if (small && h.sv_small_cnt[l]) {
      const int sc = h.sv_small_cnt[l];
      SCUDA(launch_pdl(k_solve_forward<T, kSmallThreads>, dim3(sc), dim3(kSmallThreads),
                       (size_t)h.sv_small_smem[l], s, d, (const int*)(h.sv_nodes + b), d_x,
                       nrhs, ldx, h.ubuf, (const long long*)h.uoff, h.sv_small_smem[l] / 8));
      ab::count_launch();
      b += sc;
      cnt -= sc;
    }
    if (cnt) {
      SCUDA(launch_pdl(k_solve_forward<T>, dim3(cnt), dim3(NT), (size_t)h.sv_narrow_smem[l],
                       s, d, h.sv_nodes + b, d_x, nrhs, ldx, h.ubuf, h.uoff,
                       h.sv_narrow_smem[l] / 8));
      ab::count_launch();
    }
    const int cb = h.sv_clu_ptr[l], ccnt = h.sv_wide_ptr[l] - cb;
    if (ccnt) {
      int rc = launch_cluster(k_clu_forward<T>, ccnt, h.sv_clu_smem[l], s, d,
                              h.sv_nodes + cb, d_x, nrhs, ldx, h.ubuf, h.uoff);
      if (rc) return rc;
    }
    const int wb = h.sv_wide_ptr[l], wc = h.sv_narrow_ptr[l + 1] - wb;
    if (wc) {
      const int* wn = h.sv_nodes + wb;
      double* ub = h.ubuf;
      const long long* uo = h.uoff;
      void* args[] = {(void*)&d, (void*)&wn, (void*)&wc, (void*)&d_x,
                      (void*)&nrhs, (void*)&ldx, (void*)&ub, (void*)&uo,
                      (void*)&wst};
      SCUDA(cudaLaunchCooperativeKernel((const void*)k_wide_forward<T>,
                                        dim3(h.sv_fwd_grid[l]), dim3(NT), args,
                                        wide_smem, s));
      ab::count_launch();
    }
  }
  if (trace) cudaEventRecord(ev[d.num_levels], s);
  for (int l = d.num_levels - 1; l >= (queue ? h.sv_qlevels : 0); l--) {
    if (trace) cudaEventRecord(ev[d.num_levels + 1 + (d.num_levels - 1 - l)], s);
    int b = h.sv_narrow_ptr[l], cnt = h.sv_clu_ptr[l] - b;
    if (small && h.sv_small_cnt[l]) {
      const int sc = h.sv_small_cnt[l];
      SCUDA(launch_pdl(k_solve_backward<T, kSmallThreads>, dim3(sc), dim3(kSmallThreads),
                       (size_t)h.sv_small_smem[l], s, d, (const int*)(h.sv_nodes + b), d_x,
                       nrhs, ldx, h.ubuf, (const long long*)h.uoff, h.sv_small_smem[l] / 8));
      ab::count_launch();
      b += sc;
      cnt -= sc;
    }
    if (cnt) {
      SCUDA(launch_pdl(k_solve_backward<T>, dim3(cnt), dim3(NT), (size_t)h.sv_narrow_smem[l],
                       s, d, h.sv_nodes + b, d_x, nrhs, ldx, h.ubuf, h.uoff,
                       h.sv_narrow_smem[l] / 8));
      ab::count_launch();
    }
    const int cb = h.sv_clu_ptr[l], ccnt = h.sv_wide_ptr[l] - cb;
    if (ccnt) {
      int rc = launch_cluster(k_clu_backward<T>, ccnt, h.sv_clu_smem[l], s, d,
                              h.sv_nodes + cb, d_x, nrhs, ldx, h.ubuf, h.uoff);
      if (rc) return rc;
    }
    const int wb = h.sv_wide_ptr[l], wc = h.sv_narrow_ptr[l + 1] - wb;
    if (wc) {
      const int* wn = h.sv_nodes + wb;
      double* ub = h.ubuf;
      const long long* uo = h.uoff;
      void* args[] = {(void*)&d, (void*)&wn, (void*)&wc, (void*)&d_x,
                      (void*)&nrhs, (void*)&ldx, (void*)&ub, (void*)&uo,
                      (void*)&wst};
      SCUDA(cudaLaunchCooperativeKernel((const void*)k_wide_backward<T>,
                                        dim3(h.sv_bwd_grid[l]), dim3(NT), args,
                                        wide_smem, s));
      ab::count_launch();
    }
  }
  if (queue) {
    if (qsmall)
      SCUDA(launch_pdl(k_solve_backward_q<T, kSmallThreads>, dim3(h.sv_qgrid), dim3(qth),
                       (size_t)qsm, s, d, (const int*)h.sv_bq, (const int*)h.sv_dep,
                       h.sv_qcount, d_x, nrhs, ldx, h.ubuf, (const long long*)h.uoff,
                       qsm / 8, h.sv_ctr + 1, h.sv_done + d.nn, ep, h.sv_err));
    else
      SCUDA(launch_pdl(k_solve_backward_q<T>, dim3(h.sv_qgrid), dim3(qth), (size_t)qsm, s, d,
                       (const int*)h.sv_bq, (const int*)h.sv_dep, h.sv_qcount, d_x, nrhs,
                       ldx, h.ubuf, (const long long*)h.uoff, qsm / 8, h.sv_ctr + 1,
                       h.sv_done + d.nn, ep, h.sv_err));
    ab::count_launch();
  }
  if (trace && queue) {
    // the queued levels ran as one launch each way: no per-level times
    for (int l = 0; l < h.sv_qlevels; l++) {
      cudaEventRecord(ev[l], s);
      cudaEventRecord(ev[d.num_levels + 1 + (d.num_levels - 1 - l)], s);
    }
  }
  if (trace) {
    const int L = d.num_levels;
    cudaEventRecord(ev[2 * L + 1], s);
    cudaEventSynchronize(ev[2 * L + 1]);
    float tf = 0.f, tb = 0.f;
    for (int l = 0; l < L; l++) {
      float a = 0.f, b = 0.f;
      cudaEventElapsedTime(&a, ev[l], ev[l + 1]);
      const int bi = L + 1 + (L - 1 - l);
      cudaEventElapsedTime(&b, ev[bi], ev[bi + 1]);
      tf += a;
      tb += b;
      int fm = 0;
      for (int q = h.level_ptr[l]; q < h.level_ptr[l + 1]; q++)
        fm = std::max(fm, h.h_f[h.level_nodes[q]]);
      std::fprintf(stderr,
                   "solve level %d: narrow %d cluster %d wide %d max f %d  fwd %.3f ms  "
                   "bwd %.3f ms\n",
                   l, h.sv_clu_ptr[l] - h.sv_narrow_ptr[l], h.sv_wide_ptr[l] - h.sv_clu_ptr[l],
                   h.sv_narrow_ptr[l + 1] - h.sv_wide_ptr[l], fm, a, b);
    }
    std::fprintf(stderr, "solve total: fwd %.3f ms, bwd %.3f ms\n", tf, tb);
    for (auto& e : ev) cudaEventDestroy(e);
  }
  SCUDA(cudaGetLastError());
  return 0;
}

int solve_numeric(LdlHandle& h, double* d_x, int nrhs, int ldx,
                  cudaStream_t s) {
  DevicePlan& d = h.d;
  const int nn = d.nn;
  if (h.uoff_nrhs != nrhs ||
      (h.solve_epoch != h.factor_epoch && h.sv_f != h.h_f)) {
    // offsets of the update vectors (front sizes change with the delayed
    // pivots of each factorization)
    h.h_uoff.resize(nn);
    long long tot = 0;
    for (int k = 0; k < nn; k++) {
      h.h_uoff[k] = tot;
      tot += (long long)h.h_f[k] * nrhs;
    }
    if (tot + 8 > h.ubuf_cap) {
      if (h.ubuf) SCUDA(cudaFree(h.ubuf));
      h.ubuf = nullptr;
      h.ubuf_cap = tot + 8;
      SCUDA(cudaMalloc((void**)&h.ubuf, (size_t)h.ubuf_cap * sizeof(double)));
    }
    SCUDA(cudaMemcpyAsync(h.uoff, h.h_uoff.data(), nn * sizeof(long long),
                          cudaMemcpyHostToDevice, s));
    h.uoff_nrhs = nrhs;
  }
  if (h.solve_epoch != h.factor_epoch) {
    int rc = build_solve_schedule(h, s);
    if (rc) return rc;
  }
  return h.factor_precision == 32 ? launch_solve<float>(h, d_x, nrhs, ldx, s)
                                   : launch_solve<double>(h, d_x, nrhs, ldx, s);
}

}  // namespace ab

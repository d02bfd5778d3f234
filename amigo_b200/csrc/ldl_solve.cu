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
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
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

__global__ void __launch_bounds__(NT)
k_solve_forward(DevicePlan d, const int* __restrict__ nodes, double* x,
                int nrhs, int ldx, double* ubuf, const long long* uoff,
                int smem_doubles) {
  extern __shared__ double sV[];
  const int node = nodes[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int f = d.f[node], npiv = d.npiv[node];
  const int ns = d.ns[node], ndin = d.ndin[node];
  const int fs = ns + ndin;
  const int* fvars = d.ipool + d.ioff[node];
  const int* fsinv = fvars + 2 * f;
  const int* kind = fvars + 3 * f;
  const double* L = d.fpool + d.foff[node];
  __shared__ int s_choff;
  __shared__ double sL[(SB + 1) * (SB + 1)];

  for (int rhs = 0; rhs < nrhs; rhs++) {
    // The front vector is worked on in shared memory when it fits (every
    // step of the in-block triangular solve depends on the previous one);
    // its tail is stored in ubuf for the parent.
    double* G = ubuf + uoff[node] + (long long)rhs * f;
    double* V = f <= smem_doubles ? sV : G;
    double* xr = x + (long long)rhs * ldx;
    for (int r = tid; r < f; r += NT) V[r] = 0.0;
    __syncthreads();
    const int vb = d.var_ptr[node];
    for (int r = tid; r < ns; r += NT) V[fsinv[r]] = xr[d.vars[vb + r]];
    __syncthreads();
    if (tid == 0) s_choff = ns;
    __syncthreads();
    for (int q = d.kid_ptr[node]; q < d.kid_ptr[node + 1]; q++) {
      const int c = d.kids[q];
      const int fc = d.f[c], npc = d.npiv[c], ndc = d.ndel[c];
      const int cc = fc - npc;
      const double* uc = ubuf + uoff[c] + (long long)rhs * fc + npc;
      const int cb = d.cptr[c];
      const int choff = s_choff;
      for (int a = tid; a < cc; a += NT) {
        int pos;
        if (a < ndc) {
          pos = choff + a;
        } else {
          int r0 = d.cmap[cb + a - ndc];
          pos = r0 < ns ? r0 : r0 + ndin;
        }
        if (pos < fs) pos = fsinv[pos];
        V[pos] += uc[a];
      }
      __syncthreads();
      if (tid == 0) s_choff = choff + ndc;
      __syncthreads();
    }

    // Forward elimination with the unit lower factor.  The diagonal block
    // of each column block is staged in shared memory first, so that the
    // dependent steps of the warp's triangular solve read no global memory.
    for (int jb = 0; jb < npiv;) {
      const int je = block_end(kind, jb, npiv);
      const int bw = je - jb;
      for (int t = tid; t < bw * bw; t += NT) {
        const int i = t % bw, j = t / bw;
        sL[i + j * (SB + 1)] = L[jb + i + (size_t)(jb + j) * f];
      }
      __syncthreads();
      if (warp == 0) {
        for (int j = jb; j < je;) {
          const bool two = kind[j] == 1;
          const double v0 = V[j];
          const double v1 = two ? V[j + 1] : 0.0;
          const int i0 = j + (two ? 2 : 1);
          for (int i = i0 + lane; i < je; i += 32) {
            double t = sL[(i - jb) + (j - jb) * (SB + 1)] * v0;
            if (two) t += sL[(i - jb) + (j + 1 - jb) * (SB + 1)] * v1;
            V[i] -= t;
          }
          __syncwarp();
          j = i0;
        }
      }
      __syncthreads();
      for (int i = je + tid; i < f; i += NT) {
        double acc = 0.0;
        for (int j = jb; j < je; j++) acc += L[i + (size_t)j * f] * V[j];
        V[i] -= acc;
      }
      __syncthreads();
      jb = je;
    }
    // D^{-1} and the pivots' forward values.
    for (int j = tid; j < npiv; j += NT) {
      const int kd = kind[j];
      if (kd == 0) {
        V[j] = V[j] / L[j + (size_t)j * f];
      } else if (kd == 1) {
        const double d11 = L[j + (size_t)j * f];
        const double d21 = L[j + 1 + (size_t)j * f];
        const double d22 = L[j + 1 + (size_t)(j + 1) * f];
        const double inv = 1.0 / (d11 * d22 - d21 * d21);
        const double x1 = V[j], x2 = V[j + 1];
        V[j] = inv * (d22 * x1 - d21 * x2);
        V[j + 1] = inv * (d11 * x2 - d21 * x1);
      }
    }
    __syncthreads();
    for (int j = tid; j < npiv; j += NT) xr[decode_var(fvars[j])] = V[j];
    if (V != G)
      for (int r = npiv + tid; r < f; r += NT) G[r] = V[r];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(NT)
k_solve_backward(DevicePlan d, const int* __restrict__ nodes, double* x,
                 int nrhs, int ldx, double* ubuf, const long long* uoff,
                 int smem_doubles) {
  extern __shared__ double sV[];
  const int node = nodes[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NWARP = NT / 32;
  const int f = d.f[node], npiv = d.npiv[node];
  const int* fvars = d.ipool + d.ioff[node];
  const int* kind = fvars + 3 * f;
  const double* L = d.fpool + d.foff[node];
  __shared__ double sL[(SB + 1) * (SB + 1)];
  for (int rhs = 0; rhs < nrhs; rhs++) {
    double* V = f <= smem_doubles ? sV : ubuf + uoff[node] + (long long)rhs * f;
    double* xr = x + (long long)rhs * ldx;
    // pivots: their forward values (written to x by the forward sweep);
    // delayed and contribution rows: final values of the ancestors
    for (int r = tid; r < npiv; r += NT) V[r] = xr[decode_var(fvars[r])];
    for (int r = npiv + tid; r < f; r += NT) V[r] = xr[fvars[r]];
    __syncthreads();
    // Column blocks from the last one backwards.
    int je = npiv;
    while (je > 0) {
      int jb = je - SB > 0 ? je - SB : 0;
      if (jb > 0 && kind[jb] == 2) jb--;  // keep 2x2 pairs together
      // t[j] -= sum_{i >= je} L[i, j] t[i] for j in [jb, je): one warp per
      // column, lanes over rows.
      for (int j = jb + warp; j < je; j += NWARP) {
        double acc = 0.0;
        for (int i = je + lane; i < f; i += 32) acc += L[i + (size_t)j * f] * V[i];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) V[j] -= acc;
      }
      const int bw = je - jb;
      for (int t = tid; t < bw * bw; t += NT) {
        const int i = t % bw, j = t / bw;
        sL[i + j * (SB + 1)] = L[jb + i + (size_t)(jb + j) * f];
      }
      __syncthreads();
      if (warp == 0) {
        // within the block, backwards: column j (or pair j-1, j)
        for (int j = je - 1; j >= jb;) {
          const bool two = kind[j] == 2;
          const int jl = two ? j - 1 : j;
          // rows strictly inside the block below this pivot
          double a0 = 0.0, a1 = 0.0;
          for (int i = j + 1 + lane; i < je; i += 32) {
            a0 += sL[(i - jb) + (jl - jb) * (SB + 1)] * V[i];
            if (two) a1 += sL[(i - jb) + (j - jb) * (SB + 1)] * V[i];
          }
          for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_down_sync(0xffffffffu, a0, o);
            a1 += __shfl_down_sync(0xffffffffu, a1, o);
          }
          if (lane == 0) {
            V[jl] -= a0;
            if (two) V[j] -= a1;
          }
          __syncwarp();
          j = jl - 1;
        }
      }
      __syncthreads();
      je = jb;
    }
    for (int j = tid; j < npiv; j += NT) xr[decode_var(fvars[j])] = V[j];
    __syncthreads();
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

int solve_numeric(LdlHandle& h, double* d_x, int nrhs, int ldx,
                  cudaStream_t s) {
  DevicePlan& d = h.d;
  const int nn = d.nn;
  if (h.uoff_nrhs != nrhs) {
    h.h_uoff.resize(nn);
    long long tot = 0;
    for (int k = 0; k < nn; k++) {
      h.h_uoff[k] = tot;
      tot += (long long)h.h_f[k] * nrhs;
    }
    if (tot + 8 > h.ubuf_cap) {
      if (h.ubuf) SCUDA(cudaFree(h.ubuf));
      h.ubuf_cap = tot + 8;
      SCUDA(cudaMalloc((void**)&h.ubuf, (size_t)h.ubuf_cap * sizeof(double)));
    }
    SCUDA(cudaMemcpyAsync(h.uoff, h.h_uoff.data(), nn * sizeof(long long),
                          cudaMemcpyHostToDevice, s));
    h.uoff_nrhs = nrhs;
  }
  static bool attr_set = false;
  if (!attr_set) {
    SCUDA(cudaFuncSetAttribute(k_solve_forward,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kMaxDynSmem));
    SCUDA(cudaFuncSetAttribute(k_solve_backward,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kMaxDynSmem));
    attr_set = true;
  }
  // shared memory per level: the largest front vector of the level
  std::vector<int> smem(d.num_levels, 0);
  for (int l = 0; l < d.num_levels; l++) {
    int fm = 0;
    for (int q = h.level_ptr[l]; q < h.level_ptr[l + 1]; q++)
      fm = std::max(fm, h.h_f[h.level_nodes[q]]);
    long long bytes = (long long)fm * 8;
    smem[l] = (int)std::min<long long>(bytes, kMaxDynSmem);
  }
  for (int l = 0; l < d.num_levels; l++) {
    const int b = h.level_ptr[l], cnt = h.level_ptr[l + 1] - b;
    if (cnt)
      { k_solve_forward<<<cnt, NT, smem[l], s>>>(d, d.level_nodes + b, d_x, nrhs,
                                               ldx, h.ubuf, h.uoff, smem[l] / 8); ab::count_launch(); }
  }
  for (int l = d.num_levels - 1; l >= 0; l--) {
    const int b = h.level_ptr[l], cnt = h.level_ptr[l + 1] - b;
    if (cnt)
      { k_solve_backward<<<cnt, NT, smem[l], s>>>(d, d.level_nodes + b, d_x,
                                                nrhs, ldx, h.ubuf, h.uoff,
                                                smem[l] / 8); ab::count_launch(); }
  }
  SCUDA(cudaGetLastError());
  return 0;
}

}  // namespace ab

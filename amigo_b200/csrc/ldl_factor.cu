// Multifrontal LDL^T numeric factorization on the device (FP64).
//
// One launch per elimination-tree level; one CTA per front.  A CTA
//   1. sizes its front from the delayed pivots its children passed up and
//      carves F (f x f) and the panel workspace W (f x kPanel) out of the
//      FP64 pool with an atomic bump pointer;
//   2. assembles A's entries and the children's contribution blocks
//      (extend-add), in shared memory when the front fits, else in HBM;
//   3. factors the fully-summed block with the reference's blocked,
//      left-looking-in-panel threshold pivoting (include/sparse_ldl.h:
//      1298-1535): 1x1 pivots need |a_kk| >= pivot_tol and
//      |a_kk| >= ustab * colmax; else the row of the largest candidate entry
//      is tried as a 1x1 pivot, then the 2x2 (k, imax) pivot with the Duff
//      test; a column that passes none is delayed to the parent.  Root fronts
//      (no contribution rows) use Bunch-Kaufman partial pivoting instead, as
//      the reference's LAPACK dsytrf does (include/sparse_ldl.h:1208-1230);
//   4. applies the trailing update after every panel and counts the inertia
//      of its D blocks with the reference's rule (sparse_ldl.h:1917-1969).
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>

#include "ldl_internal.h"

namespace ab {
namespace {

constexpr int NT = kThreads;
constexpr int NB = kPanel;
constexpr int NWARP = NT / 32;
constexpr int kMaxDynSmem = 190 * 1024;
constexpr int kTile = 64;

struct Ctl {
  double wrow[NB];     // row k (or imax) of W, columns 0..kw-1
  double red_v[NWARP];
  int red_i[NWARP];
  double red_v2[NWARP];
  double abswik, ctail, rowmax;
  int imax;
  int f, fs, ns, ndin, npiv;
  long long foff, ioff;
  int skip;
};

// Lexicographic "larger |value|, then smaller index" -- the first maximum,
// which is what BLAS idamax returns.
__device__ __forceinline__ void argmax_merge(double& v, int& i, double v2,
                                             int i2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

// Block-wide first-argmax of (v, i) plus a max of v2.  Result is written to
// ctl.red_v[0], ctl.red_i[0], ctl.red_v2[0].
__device__ void block_argmax(Ctl& ctl, double v, int i, double v2) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    double ov = __shfl_down_sync(0xffffffffu, v, o);
    int oi = __shfl_down_sync(0xffffffffu, i, o);
    double ov2 = __shfl_down_sync(0xffffffffu, v2, o);
    argmax_merge(v, i, ov, oi);
    v2 = fmax(v2, ov2);
  }
  if (lane == 0) {
    ctl.red_v[warp] = v;
    ctl.red_i[warp] = i;
    ctl.red_v2[warp] = v2;
  }
  __syncthreads();
  if (warp == 0) {
    v = lane < NWARP ? ctl.red_v[lane] : -1.0;
    i = lane < NWARP ? ctl.red_i[lane] : 0x7fffffff;
    v2 = lane < NWARP ? ctl.red_v2[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_down_sync(0xffffffffu, v, o);
      int oi = __shfl_down_sync(0xffffffffu, i, o);
      double ov2 = __shfl_down_sync(0xffffffffu, v2, o);
      argmax_merge(v, i, ov, oi);
      v2 = fmax(v2, ov2);
    }
    if (lane == 0) {
      ctl.red_v[0] = v;
      ctl.red_i[0] = i;
      ctl.red_v2[0] = v2;
    }
  }
  __syncthreads();
}

// Symmetric interchange of rows/columns a < b of the lower triangle of F,
// of the variable list and of the fully-summed permutation record
// (reference: symm_swap, include/sparse_ldl.h:1252-1274).
__device__ void symm_swap(double* F, int ld, int n, int* vars, int* fsperm,
                          int a, int b) {
  const int tid = threadIdx.x;
  // rows a and b over columns [0, a)
  for (int j = tid; j < a; j += NT) {
    double t = F[a + (size_t)j * ld];
    F[a + (size_t)j * ld] = F[b + (size_t)j * ld];
    F[b + (size_t)j * ld] = t;
  }
  // F[j, a] <-> F[b, j] for a < j < b
  for (int j = a + 1 + tid; j < b; j += NT) {
    double t = F[j + (size_t)a * ld];
    F[j + (size_t)a * ld] = F[b + (size_t)j * ld];
    F[b + (size_t)j * ld] = t;
  }
  // F[j, a] <-> F[j, b] for j > b
  for (int j = b + 1 + tid; j < n; j += NT) {
    double t = F[j + (size_t)a * ld];
    F[j + (size_t)a * ld] = F[j + (size_t)b * ld];
    F[j + (size_t)b * ld] = t;
  }
  if (tid == 0) {
    double t = F[a + (size_t)a * ld];
    F[a + (size_t)a * ld] = F[b + (size_t)b * ld];
    F[b + (size_t)b * ld] = t;
    int tv = vars[a];
    vars[a] = vars[b];
    vars[b] = tv;
    tv = fsperm[a];
    fsperm[a] = fsperm[b];
    fsperm[b] = tv;
  }
}

// Swap rows a and b of W over columns [0, ncol).
__device__ void swap_wrows(double* W, int ldw, int ncol, int a, int b) {
  for (int j = threadIdx.x; j < ncol; j += NT) {
    double t = W[a + (size_t)j * ldw];
    W[a + (size_t)j * ldw] = W[b + (size_t)j * ldw];
    W[b + (size_t)j * ldw] = t;
  }
}

// Trailing update C -= A * B^T on the lower triangle of the (n-k) x (n-k)
// block starting at (k, k):  A = F[k:, kstart:kstart+kw], B = W[k:, 0:kw].
// `tiles` (>= 2 * kTile * NB doubles of shared memory) enables the tiled
// form used for fronts kept in HBM.
__device__ void trailing_update(double* F, int ld, const double* W, int ldw,
                                int n, int k, int kstart, int kw,
                                double* tiles) {
  const int m = n - k;
  if (m <= 0 || kw <= 0) return;
  const int tid = threadIdx.x;
  if (tiles == nullptr) {
    for (int c = 0; c < m; c++) {
      double* Fc = F + (size_t)(k + c) * ld + k;
      for (int r = c + tid; r < m; r += NT) {
        double acc = Fc[r];
        for (int j = 0; j < kw; j++)
          acc -= F[k + r + (size_t)(kstart + j) * ld] * W[k + c + (size_t)j * ldw];
        Fc[r] = acc;
      }
    }
    __syncthreads();
    return;
  }
  // Tiled: kTile x kTile output tiles over the lower triangle; A and B tiles
  // are staged in shared memory (kw <= NB).
  double* As = tiles;                 // kTile x NB, row-major by tile row
  double* Bs = tiles + kTile * NB;    // kTile x NB
  const int nt = (m + kTile - 1) / kTile;
  const int tr = tid % 16, tc = tid / 16;  // 16 x 16 threads, 4x4 each
  for (int tj = 0; tj < nt; tj++) {
    for (int ti = tj; ti < nt; ti++) {
      const int r0 = k + ti * kTile, c0 = k + tj * kTile;
      for (int idx = tid; idx < kTile * kw; idx += NT) {
        int rr = idx % kTile, jj = idx / kTile;
        As[rr * NB + jj] = (r0 + rr < n) ? F[r0 + rr + (size_t)(kstart + jj) * ld] : 0.0;
        Bs[rr * NB + jj] = (c0 + rr < n) ? W[c0 + rr + (size_t)jj * ldw] : 0.0;
      }
      __syncthreads();
      double acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
      for (int jj = 0; jj < kw; jj++) {
        double av[4], bv[4];
#pragma unroll
        for (int a = 0; a < 4; a++) av[a] = As[(tr + 16 * a) * NB + jj];
#pragma unroll
        for (int b = 0; b < 4; b++) bv[b] = Bs[(tc + 16 * b) * NB + jj];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int b = 0; b < 4; b++) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
      }
#pragma unroll
      for (int a = 0; a < 4; a++) {
        int r = r0 + tr + 16 * a;
#pragma unroll
        for (int b = 0; b < 4; b++) {
          int c = c0 + tc + 16 * b;
          if (r < n && c < n && r >= c) F[r + (size_t)c * ld] -= acc[a][b];
        }
      }
      __syncthreads();
    }
  }
}

// W[r, col] = src(r) - F[r, kstart:kstart+kw] . ctl.wrow  for r in [k, n),
// and the reductions the pivot tests need.
//   mode 0: candidate column k; src(r) = F[r, k]; reduces first-argmax of
//           |W| over (k, nc) -> ctl.imax / ctl.abswik and max over [nc, n)
//           -> ctl.ctail.
//   mode 1: column imax; src(r) = F[imax, r] for r < imax else F[r, imax];
//           reduces max over [k, n) \ {imax} -> ctl.rowmax.
__device__ void build_column(double* F, int ld, double* W, int ldw, int n,
                             int k, int kstart, int kw, int col, int mode,
                             int imax, int nc, Ctl& ctl) {
  const int tid = threadIdx.x;
  double bestv = -1.0, tailv = 0.0;
  int besti = 0x7fffffff;
  for (int r = k + tid; r < n; r += NT) {
    double acc;
    if (mode == 0) {
      acc = F[r + (size_t)k * ld];
    } else {
      acc = (r < imax) ? F[imax + (size_t)r * ld] : F[r + (size_t)imax * ld];
    }
    for (int j = 0; j < kw; j++)
      acc -= F[r + (size_t)(kstart + j) * ld] * ctl.wrow[j];
    W[r + (size_t)col * ldw] = acc;
    const double a = fabs(acc);
    if (mode == 0) {
      if (r > k && r < nc) argmax_merge(bestv, besti, a, r);
      if (r >= nc) tailv = fmax(tailv, a);
    } else {
      if (r != imax) tailv = fmax(tailv, a);
    }
  }
  block_argmax(ctl, bestv, besti, tailv);
  if (tid == 0) {
    if (mode == 0) {
      ctl.imax = ctl.red_i[0];
      ctl.abswik = ctl.red_v[0] < 0.0 ? 0.0 : ctl.red_v[0];
      ctl.ctail = ctl.red_v2[0];
    } else {
      ctl.rowmax = ctl.red_v2[0];
    }
  }
  __syncthreads();
}

// Load row `row` of W (columns 0..kw-1) into ctl.wrow.
__device__ void load_wrow(const double* W, int ldw, int row, int kw, Ctl& ctl) {
  for (int j = threadIdx.x; j < kw; j += NT) ctl.wrow[j] = W[row + (size_t)j * ldw];
  __syncthreads();
}

// Factor the fully-summed columns [0, fs) of the n x n front F (lower
// triangle valid).  Returns the number of pivots (== fs for a root front).
__device__ int factor_front(double* F, int ld, double* W, int ldw, int n,
                            int fs, bool root, int* vars, int* fsperm,
                            double ustab, double pivot_tol, double* tiles,
                            int* status, Ctl& ctl) {
  const int tid = threadIdx.x;
  const double bk_alpha = (1.0 + sqrt(17.0)) / 8.0;
  int nc = fs;
  int k = 0;
  while (k < nc) {
    const int kstart = k;
    int kw = 0;
    while (kw < NB - 1 && k < nc) {
      load_wrow(W, ldw, k, kw, ctl);
      build_column(F, ld, W, ldw, n, k, kstart, kw, kw, 0, 0, nc, ctl);
      const double wkk = W[k + (size_t)kw * ldw];
      const double abswkk = fabs(wkk);
      const int imax = ctl.imax;
      const double abswik = ctl.abswik;
      int step = 0, kpiv = -1;
      bool zero_pivot = false;
      if (!root) {
        const double colmax = fmax(abswik, ctl.ctail);
        if (abswkk >= pivot_tol && abswkk >= ustab * colmax) {
          step = 1;
          kpiv = k;
        } else if (k + 1 < nc) {
          load_wrow(W, ldw, imax, kw, ctl);
          build_column(F, ld, W, ldw, n, k, kstart, kw, kw + 1, 1, imax, nc, ctl);
          const double rowmax = ctl.rowmax;
          const double wii = W[imax + (size_t)(kw + 1) * ldw];
          const double abswii = fabs(wii);
          if (abswii >= pivot_tol && abswii >= ustab * rowmax) {
            for (int r = k + tid; r < n; r += NT)
              W[r + (size_t)kw * ldw] = W[r + (size_t)(kw + 1) * ldw];
            __syncthreads();
            step = 1;
            kpiv = imax;
          } else {
            const double wik = W[imax + (size_t)kw * ldw];
            const double det = fabs(wkk * wii - wik * wik);
            if (det >= pivot_tol) {
              const double delta = det / fmax(abswii + abswik, abswkk + abswik);
              if (delta >= ustab * colmax && delta >= ustab * rowmax) {
                step = 2;
                kpiv = imax;
              }
            }
          }
        }
      } else {
        // Bunch-Kaufman (LAPACK dsytf2/dlasyf, lower): every column is
        // eliminated, by a 1x1 or a 2x2 pivot.
        const double colmax = abswik;  // nc == n: all rows are candidates
        if (!(fmax(abswkk, colmax) > 0.0)) {
          step = 1;
          kpiv = k;
          zero_pivot = true;
        } else if (abswkk >= bk_alpha * colmax) {
          step = 1;
          kpiv = k;
        } else {
          load_wrow(W, ldw, imax, kw, ctl);
          build_column(F, ld, W, ldw, n, k, kstart, kw, kw + 1, 1, imax, nc, ctl);
          const double rowmax = ctl.rowmax;
          const double abswii = fabs(W[imax + (size_t)(kw + 1) * ldw]);
          if (abswkk >= bk_alpha * colmax * (colmax / rowmax)) {
            step = 1;
            kpiv = k;
          } else if (abswii >= bk_alpha * rowmax) {
            for (int r = k + tid; r < n; r += NT)
              W[r + (size_t)kw * ldw] = W[r + (size_t)(kw + 1) * ldw];
            __syncthreads();
            step = 1;
            kpiv = imax;
          } else {
            step = 2;
            kpiv = imax;
          }
        }
      }

      if (step == 0) {
        // Delay candidate k: move it to the end of the candidate set.
        if (k < nc - 1) {
          symm_swap(F, ld, n, vars, fsperm, k, nc - 1);
          swap_wrows(W, ldw, kw, k, nc - 1);
          __syncthreads();
        }
        nc -= 1;
        continue;
      }
      const int ksrc = k + step - 1;
      if (kpiv != ksrc) {
        symm_swap(F, ld, n, vars, fsperm, ksrc, kpiv);
        swap_wrows(W, ldw, kw + step, ksrc, kpiv);
        __syncthreads();
      }
      if (step == 1) {
        const double d = W[k + (size_t)kw * ldw];
        if (!isfinite(d) && tid == 0) atomicOr(status, ST_NAN);
        const double dinv = zero_pivot ? 0.0 : 1.0 / d;
        for (int r = k + tid; r < n; r += NT) {
          double w = W[r + (size_t)kw * ldw];
          F[r + (size_t)k * ld] = (r == k) ? w : w * dinv;
        }
      } else {
        const double d11 = W[k + (size_t)kw * ldw];
        const double d21 = W[k + 1 + (size_t)kw * ldw];
        const double d22 = W[k + 1 + (size_t)(kw + 1) * ldw];
        const double detinv = 1.0 / (d11 * d22 - d21 * d21);
        if (!isfinite(detinv) && tid == 0) atomicOr(status, ST_NAN);
        const double i00 = d22 * detinv, i10 = -d21 * detinv,
                     i01 = -d21 * detinv, i11 = d11 * detinv;
        for (int r = k + 2 + tid; r < n; r += NT) {
          double w0 = W[r + (size_t)kw * ldw], w1 = W[r + (size_t)(kw + 1) * ldw];
          F[r + (size_t)k * ld] = w0 * i00 + w1 * i10;
          F[r + (size_t)(k + 1) * ld] = w0 * i01 + w1 * i11;
        }
        if (tid == 0) {
          F[k + (size_t)k * ld] = d11;
          F[k + 1 + (size_t)k * ld] = d21;
          F[k + 1 + (size_t)(k + 1) * ld] = d22;
          vars[k] = -(vars[k] + 1);
          vars[k + 1] = -(vars[k + 1] + 1);
        }
      }
      __syncthreads();
      k += step;
      kw += step;
    }
    trailing_update(F, ld, W, ldw, n, k, kstart, kw, tiles);
    __syncthreads();
  }
  return nc;
}

// Per-level kernel: set up, assemble and factor one front per CTA.
__global__ void __launch_bounds__(NT)
k_factor_level(DevicePlan d, const int* __restrict__ nodes, int count,
               const double* __restrict__ vals, double ustab,
               double pivot_tol, int smem_doubles) {
  extern __shared__ double smem[];
  __shared__ Ctl ctl;
  const int tid = threadIdx.x;
  const int node = nodes[blockIdx.x];

  if (tid == 0) {
    ctl.skip = (*((volatile int*)d.status) & (ST_POOL_F | ST_POOL_I)) ? 1 : 0;
    const int ns = d.ns[node], nc = d.nc[node];
    int ndin = 0;
    for (int q = d.kid_ptr[node]; q < d.kid_ptr[node + 1]; q++)
      ndin += d.ndel[d.kids[q]];
    const int f = ns + ndin + nc;
    ctl.ns = ns;
    ctl.ndin = ndin;
    ctl.f = f;
    ctl.fs = ns + ndin;
    if (!ctl.skip) {
      // F followed by W, rounded to 8 doubles (64-byte alignment)
      const unsigned long long need =
          (((unsigned long long)f * f + (unsigned long long)f * NB) + 15) & ~7ull;
      unsigned long long off = atomicAdd(&d.counters[0], need);
      unsigned long long ioff = atomicAdd(&d.counters[1], (4ull * f + 15) & ~7ull);
      if (off + need > (unsigned long long)d.fcap) {
        atomicOr(d.status, ST_POOL_F);
        ctl.skip = 1;
      }
      if (ioff + ((4ull * f + 15) & ~7ull) > (unsigned long long)d.icap) {
        atomicOr(d.status, ST_POOL_I);
        ctl.skip = 1;
      }
      ctl.foff = (long long)off;
      ctl.ioff = (long long)ioff;
    }
    d.f[node] = f;
    d.ndin[node] = ndin;
    d.foff[node] = ctl.skip ? 0 : ctl.foff;
    d.ioff[node] = ctl.skip ? 0 : ctl.ioff;
    if (ctl.skip) {
      d.npiv[node] = 0;
      d.ndel[node] = 0;
    }
  }
  __syncthreads();
  if (ctl.skip) return;

  const int f = ctl.f, fs = ctl.fs, ns = ctl.ns, ndin = ctl.ndin;
  int* fvars = d.ipool + ctl.ioff;
  int* fsperm = fvars + f;
  double* Fg = d.fpool + ctl.foff;
  const bool in_smem = (long long)f * f + (long long)f * NB <= smem_doubles;
  double* F = in_smem ? smem : Fg;
  double* W = in_smem ? smem + (size_t)f * f : Fg + (size_t)f * f;
  double* tiles = nullptr;
  if (!in_smem && smem_doubles >= 2 * kTile * NB) tiles = smem;

  // Variable list: node vars, delayed pivots of the children, contribution
  // rows (include/sparse_ldl.h:957-987, 596-616).
  {
    const int vbase = d.var_ptr[node];
    for (int r = tid; r < ns; r += NT) fvars[r] = d.vars[vbase + r];
    int choff = ns;
    for (int q = d.kid_ptr[node]; q < d.kid_ptr[node + 1]; q++) {
      const int c = d.kids[q];
      const int ndc = d.ndel[c];
      const int* cv = d.ipool + d.ioff[c] + d.npiv[c];
      for (int t = tid; t < ndc; t += NT) fvars[choff + t] = cv[t];
      choff += ndc;
    }
    const int cb = d.cptr[node];
    for (int t = tid; t < d.nc[node]; t += NT) fvars[fs + t] = d.crows[cb + t];
    for (int r = tid; r < fs; r += NT) fsperm[r] = r;
  }

  // Assemble: zero, add A, extend-add the children.
  for (size_t idx = tid; idx < (size_t)f * f; idx += NT) F[idx] = 0.0;
  __syncthreads();
  for (int t = d.amap_ptr[node] + tid; t < d.amap_ptr[node + 1]; t += NT) {
    const int r0 = d.amap_row[t];
    const int r = r0 < ns ? r0 : r0 + ndin;
    F[r + (size_t)d.amap_col[t] * f] += vals[d.amap_pos[t]];
  }
  __syncthreads();
  {
    int* rmap = reinterpret_cast<int*>(W);  // W is free until factoring
    int choff = ns;
    for (int q = d.kid_ptr[node]; q < d.kid_ptr[node + 1]; q++) {
      const int c = d.kids[q];
      const int fc = d.f[c], npc = d.npiv[c], ndc = d.ndel[c];
      const int cc = fc - npc;
      const double* C = d.fpool + d.foff[c];
      const int cb = d.cptr[c];
      for (int a = tid; a < cc; a += NT) {
        int pos;
        if (a < ndc) {
          pos = choff + a;
        } else {
          int r0 = d.cmap[cb + a - ndc];
          pos = r0 < ns ? r0 : r0 + ndin;
        }
        rmap[a] = pos;
      }
      __syncthreads();
      for (int b = 0; b < cc; b++) {
        const int pb = rmap[b];
        const double* Cb = C + (size_t)(npc + b) * fc + npc;
        for (int a = b + tid; a < cc; a += NT) {
          const int pa = rmap[a];
          const double v = Cb[a];
          if (pa >= pb) F[pa + (size_t)pb * f] += v;
          else F[pb + (size_t)pa * f] += v;
        }
      }
      __syncthreads();
      choff += ndc;
    }
  }

  const bool root = (fs == f);
  const int npiv = factor_front(F, f, W, f, f, fs, root, fvars, fsperm, ustab,
                                pivot_tol, tiles, d.status, ctl);

  if (in_smem) {
    for (size_t idx = tid; idx < (size_t)f * f; idx += NT) Fg[idx] = F[idx];
  }
  // Inertia of the D blocks, scanned in pivot order as the reference does
  // (include/sparse_ldl.h:1937-1968).
  // Also records the pivot kinds (0: 1x1, 1/2: first/second column of a
  // 2x2 block) and the inverse of the fully-summed permutation, both used
  // by the solves.
  __syncthreads();
  int* fsinv = fvars + 2 * f;
  int* kind = fvars + 3 * f;
  for (int r = tid; r < fs; r += NT) fsinv[fsperm[r]] = r;
  if (tid == 0) {
    int pos = 0, neg = 0;
    for (int j = 0; j < npiv;) {
      if (fvars[j] >= 0) {
        if (F[j + (size_t)j * f] >= 0.0) pos++; else neg++;
        kind[j] = 0;
        j += 1;
      } else {
        kind[j] = 1;
        kind[j + 1] = 2;
        const double d11 = F[j + (size_t)j * f];
        const double d21 = F[j + 1 + (size_t)j * f];
        const double d22 = F[j + 1 + (size_t)(j + 1) * f];
        const double det = d11 * d22 - d21 * d21;
        if (det >= 0.0) {
          if (d11 >= 0.0) pos += 2; else neg += 2;
        } else {
          pos++;
          neg++;
        }
        j += 2;
      }
    }
    atomicAdd(&d.inertia[0], pos);
    atomicAdd(&d.inertia[1], neg);
    d.npiv[node] = npiv;
    d.ndel[node] = fs - npiv;
  }
}

}  // namespace

#define FCUDA(call)                                                       \
  do {                                                                    \
    cudaError_t e__ = (call);                                             \
    if (e__ != cudaSuccess) {                                             \
      std::fprintf(stderr, "amigo_b200: %s: %s\n", #call,                 \
                   cudaGetErrorString(e__));                              \
      return -2;                                                          \
    }                                                                     \
  } while (0)

static int launch_factor(LdlHandle& h, const double* d_vals, cudaStream_t s) {
  DevicePlan& d = h.d;
  static bool attr_set = false;
  if (!attr_set) {
    FCUDA(cudaFuncSetAttribute(k_factor_level,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kMaxDynSmem));
    attr_set = true;
  }
  FCUDA(cudaMemsetAsync(d.counters, 0, 2 * sizeof(unsigned long long), s));
  FCUDA(cudaMemsetAsync(d.inertia, 0, 2 * sizeof(int), s));
  FCUDA(cudaMemsetAsync(d.status, 0, sizeof(int), s));
  for (int l = 0; l < d.num_levels; l++) {
    const int b = h.level_ptr[l], cnt = h.level_ptr[l + 1] - b;
    if (cnt == 0) continue;
    long long fm = h.level_max_f[l] + 16;
    long long want = (fm * fm + fm * NB) * 8;
    long long need_tiles = 2LL * kTile * NB * 8;
    long long bytes = want < need_tiles ? need_tiles : want;
    if (bytes > kMaxDynSmem) bytes = kMaxDynSmem;
    k_factor_level<<<cnt, NT, (size_t)bytes, s>>>(
        d, d.level_nodes + b, cnt, d_vals, h.ustab, h.pivot_tol,
        (int)(bytes / 8));
  }
  FCUDA(cudaGetLastError());
  return 0;
}

int factor_numeric(LdlHandle& h, const double* d_vals, cudaStream_t s) {
  DevicePlan& d = h.d;
  for (int attempt = 0; attempt < 6; attempt++) {
    int rc = launch_factor(h, d_vals, s);
    if (rc) return rc;
    int status = 0;
    FCUDA(cudaMemcpyAsync(&status, d.status, sizeof(int),
                          cudaMemcpyDeviceToHost, s));
    FCUDA(cudaStreamSynchronize(s));
    h.last_status = status;
    if (status & (ST_POOL_F | ST_POOL_I)) {
      // Delayed pivots made fronts larger than the pool allows: grow it.
      if (status & ST_POOL_F) {
        FCUDA(cudaFree(d.fpool));
        d.fcap = d.fcap * 2;
        FCUDA(cudaMalloc((void**)&d.fpool, (size_t)d.fcap * sizeof(double)));
      }
      if (status & ST_POOL_I) {
        FCUDA(cudaFree(d.ipool));
        d.icap = d.icap * 2;
        FCUDA(cudaMalloc((void**)&d.ipool, (size_t)d.icap * sizeof(int)));
      }
      continue;
    }
    // Host copies of the per-node sizes (stats and solve offsets).
    const int nn = d.nn;
    h.h_f.resize(nn);
    h.h_npiv.resize(nn);
    h.h_ndel.resize(nn);
    FCUDA(cudaMemcpyAsync(h.h_f.data(), d.f, nn * sizeof(int),
                          cudaMemcpyDeviceToHost, s));
    FCUDA(cudaMemcpyAsync(h.h_npiv.data(), d.npiv, nn * sizeof(int),
                          cudaMemcpyDeviceToHost, s));
    FCUDA(cudaMemcpyAsync(h.h_ndel.data(), d.ndel, nn * sizeof(int),
                          cudaMemcpyDeviceToHost, s));
    FCUDA(cudaStreamSynchronize(s));
    h.factored = true;
    h.uoff_nrhs = 0;  // solve offsets must be rebuilt
    return (status & ST_NAN) ? -5 : 0;
  }
  return -6;
}

}  // namespace ab

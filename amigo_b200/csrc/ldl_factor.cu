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
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../include/amigo_b200.h"
#include "ldl_internal.h"
#include "launch_count.h"
#include "tc_update.cuh"

namespace ab {
namespace {

constexpr int NT = kThreads;
constexpr int NB = kPanel;
// Threads of the one-CTA panel kernel of the large-front path.  Each
// candidate column is brought up to date by one thread per row.  Measured
// on the 2D SIMP 128x64 KKT (fronts up to 1221 rows) one factorization
// takes 31.4 ms with 256 threads, 27.2 ms with 512 and 31.3 ms with 1024;
// the 3D SIMP 48x24x24 KKT (fronts up to 25216 rows) takes 4.9 s with 1024
// and 5.75 s with 512 (the same from 1280 to 4096 rows as the switch
// point).  Levels whose largest front has more than kPanelWideRows rows
// take the wide kernel.
constexpr int kPanelThreads = 512;
constexpr int kPanelThreadsWide = 1024;
constexpr int kPanelWideRows = 2048;
// Shared memory of the large-front panel kernel for its copy of the
// panel's L columns (the static control block aside).
constexpr int kPanelCacheBytes = 200 * 1024;
// Shared-W panel (k_big_panel_sw): threads, rows per thread, and the
// dynamic shared memory for the panel's W columns.  Levels whose largest
// static front has at most kSwThreads * kSwRows rows take it.
constexpr int kSwThreads = 512;
constexpr int kSwRows = 4;
constexpr int kSwSmemBytes = 200 * 1024;
constexpr int kTile = 64;
// Right-looking small-front kernel: rows of room for delayed pivots, and
// its block size (measured on 68-row fronts: 32 threads 11.9 ms, 64 9.7,
// 128 8.5, 256 8.25 for one factorization of 512 cart-pole problems).
constexpr int kRlSlack = 8;
constexpr int kRlThreads = 256;

template <int BT>
struct CtlT {
  double wrow[NB];     // row k (or imax) of W, columns 0..kw-1
  double red_v[(BT / 32)];   // per-warp results of the column reductions
  int red_i[(BT / 32)];
  double red_v2[(BT / 32)];
  int f, fs, ns, ndin;       // front set-up (setup_front)
  long long foff, ioff;
  int skip;
};
using Ctl = CtlT<NT>;

// Lexicographic "larger |value|, then smaller index" -- the first maximum,
// which is what BLAS idamax returns.
__device__ __forceinline__ void argmax_merge(double& v, int& i, double v2,
                                             int i2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

// Programmatic dependent launch: the large-front panel and update kernels
// are launched so that the next one may be scheduled while the previous one
// drains; each waits here for its predecessor's completion and memory
// before touching the front, then lets its own successor be scheduled.
// (Both are no-ops for a kernel launched without the attribute.)
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Symmetric interchange of rows/columns a < b of the lower triangle of F,
// of the variable list and of the fully-summed permutation record
// (reference: symm_swap, include/sparse_ldl.h:1252-1274).
template <class T, bool CG>
__device__ __forceinline__ T ldf(const T* p) {
  if constexpr (CG) return __ldcg(p);
  else return *p;
}

// (CG: loads from L2, for entries another CTA of a cluster may have
// written in the same launch.)
template <class T, int BT, bool CG = false>
__device__ void symm_swap(T* F, int ld, int n, int* vars, int* fsperm,
                          int a, int b) {
  const int tid = threadIdx.x;
  // rows a and b over columns [0, a)
  for (int j = tid; j < a; j += BT) {
    T t = ldf<T, CG>(F + a + (size_t)j * ld);
    F[a + (size_t)j * ld] = ldf<T, CG>(F + b + (size_t)j * ld);
    F[b + (size_t)j * ld] = t;
  }
  // F[j, a] <-> F[b, j] for a < j < b
  for (int j = a + 1 + tid; j < b; j += BT) {
    T t = ldf<T, CG>(F + j + (size_t)a * ld);
    F[j + (size_t)a * ld] = ldf<T, CG>(F + b + (size_t)j * ld);
    F[b + (size_t)j * ld] = t;
  }
  // F[j, a] <-> F[j, b] for j > b
  for (int j = b + 1 + tid; j < n; j += BT) {
    T t = ldf<T, CG>(F + j + (size_t)a * ld);
    F[j + (size_t)a * ld] = ldf<T, CG>(F + j + (size_t)b * ld);
    F[j + (size_t)b * ld] = t;
  }
  if (tid == 0) {
    T t = ldf<T, CG>(F + a + (size_t)a * ld);
    F[a + (size_t)a * ld] = ldf<T, CG>(F + b + (size_t)b * ld);
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
template <class T, int BT>
__device__ void swap_wrows(T* W, int ldw, int ncol, int a, int b) {
  for (int j = threadIdx.x; j < ncol; j += BT) {
    T t = W[a + (size_t)j * ldw];
    W[a + (size_t)j * ldw] = W[b + (size_t)j * ldw];
    W[b + (size_t)j * ldw] = t;
  }
}

// Row stride of the staged A/B tiles: one double of padding makes the
// 16 rows a warp reads in one step fall on distinct shared-memory banks.
constexpr int TP = NB + 1;
constexpr int kTileSmem = 2 * kTile * TP;  // doubles

// C tile (ti, tj) of the trailing block F[k:, k:] -= A * B^T with
// A = F[k:, kstart:kstart+kw] (L columns of the panel) and
// B = W[k:, 0:kw] (their L*D columns); only the lower triangle is written.
template <class T>
__device__ void update_tile(T* F, int ld, const T* W, int ldw,
                            int n, int k, int kstart, int kw, int ti, int tj,
                            T* As, T* Bs) {
  const int tid = threadIdx.x;
  const int r0 = k + ti * kTile, c0 = k + tj * kTile;
  const int tr = tid % 16, tc = tid / 16;  // 16 x 16 threads, 4 x 4 outputs each
  // C first, then A and B with all loads in flight before the shared stores
  T cv[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int r = r0 + tr + 16 * a, c = c0 + tc + 16 * b;
      cv[a][b] = (r < n && c < n && r >= c) ? F[r + (size_t)c * ld] : T(0);
    }
  constexpr int kSt = kTile * NB / NT;
  T av[kSt], bv[kSt];
#pragma unroll
  for (int u = 0; u < kSt; u++) {
    const int idx = tid + u * NT;
    const int rr = idx % kTile, jj = idx / kTile;
    const bool in = jj < kw;
    av[u] = (in && r0 + rr < n) ? F[r0 + rr + (size_t)(kstart + jj) * ld] : T(0);
    bv[u] = (in && c0 + rr < n) ? W[c0 + rr + (size_t)jj * ldw] : T(0);
  }
#pragma unroll
  for (int u = 0; u < kSt; u++) {
    const int idx = tid + u * NT;
    const int rr = idx % kTile, jj = idx / kTile;
    if (jj < kw) {
      As[rr * TP + jj] = av[u];
      Bs[rr * TP + jj] = bv[u];
    }
  }
  __syncthreads();
  T acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = T(0);
  for (int jj = 0; jj < kw; jj++) {
    T av[4], bv[4];
#pragma unroll
    for (int a = 0; a < 4; a++) av[a] = As[(tr + 16 * a) * TP + jj];
#pragma unroll
    for (int b = 0; b < 4; b++) bv[b] = Bs[(tc + 16 * b) * TP + jj];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
  }
#pragma unroll
  for (int a = 0; a < 4; a++) {
    const int r = r0 + tr + 16 * a;
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int c = c0 + tc + 16 * b;
      if (r < n && c < n && r >= c) F[r + (size_t)c * ld] = cv[a][b] - acc[a][b];
    }
  }
  __syncthreads();
}

// FP64 C tile on the FP64 tensor path: mma.sync m8n8k4 (DMMA), the same
// tile and operands as update_tile.  A and B are staged row-major with a
// row stride of TPD = 36 doubles, which puts the 4 x 4 (row, k) pattern of
// each half-warp's fragment loads on 16 distinct bank pairs; k is padded
// with zeros to a multiple of 4.  8 warps as 2 x 4, each a 32 x 16 block of
// the 64 x 64 tile: 4 x 2 MMA tiles of 8 x 8.  Fragment layouts (PTX ISA,
// mma.m8n8k4 .f64): a0 at (lane / 4, lane % 4), b0 at (k = lane % 4,
// n = lane / 4), c0 / c1 at (lane / 4, 2 (lane % 4) + 0 / 1).
constexpr int TPD = 36;

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a,
                                           double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, "
      "{%0, %1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// Lower-triangle tile index t -> (ti, tj), ti >= tj.
__device__ __forceinline__ void tile_coords(int t, int& ti, int& tj) {
  int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) i++;
  while (i * (i + 1) / 2 > t) i--;
  ti = i;
  tj = t - i * (i + 1) / 2;
}

// 8-byte asynchronous global -> shared copy; a false predicate writes zeros
// (source size 0, nothing read).
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool pred) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
               "r"(pred ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Shared A and B tiles of the FP64 update, column-major (k-major) with a
// column stride of APD = 68 doubles: the staging stores (consecutive rows
// in consecutive lanes) and the fragment loads ((row g, k q) for lane
// 4 g + q) both fall on distinct bank pairs within each half-warp.
constexpr int APD = 68;
constexpr int kUpdSmemD = 3 * NB * APD;  // doubles: B and two A buffers
constexpr int kStD = kTile * NB / NT;    // staged entries of A (and of B) per thread
static_assert(kTile * NB % NT == 0 && NT % kTile == 0, "staging split");

// Tiles [tbeg, tend) of the trailing update C -= A * B^T, in column-major
// order of the lower triangle of nt x nt tiles (column tj holds tiles
// ti = tj .. nt - 1), on the FP64 tensor path (DMMA m8n8k4); A =
// F[r0:r0+64, kstart:kstart+kw], B = W[c0:c0+64, 0:kw].  8 warps as 2 x 4,
// each a 32 x 16 block of the 64 x 64 tile.  B is staged once per column;
// the next tile's A is in flight to the other shared buffer (cp.async) and
// its C entries to registers while the current tile's products run.  The
// products accumulate from zero in k order and C - A B^T goes back (lower
// triangle).  Offsets inside a tile are 32-bit and computed once; interior
// tiles skip the bounds tests.
__device__ void update_tiles_dmma(double* F, int ld, const double* W, int ldw,
                                  int n, int k, int kstart, int kw, int nt, int tbeg,
                                  int tend, double* smem) {
  if (tbeg >= tend) return;
  double* Bs = smem;
  double* As = smem + NB * APD;
  const int tid = threadIdx.x;
  const int kp = (kw + 3) & ~3;
  const int lane = tid & 31, warp = tid >> 5;
  const int wr = (warp & 1) * 32, wc = (warp >> 1) * 16;
  const int g = lane >> 2, q = lane & 3;
  // accumulator (a, b, e) sits at row wr + 8 a + g, column wc + 8 b + 2 q + e
  int coff[2][2];
#pragma unroll
  for (int b = 0; b < 2; b++)
#pragma unroll
    for (int e = 0; e < 2; e++) coff[b][e] = (wc + 8 * b + 2 * q + e) * ld;
  const int rrow = wr + g;
  // staging: this thread's row rr and columns jj0 + kJs u of A and B
  constexpr int kJs = NT / kTile;
  const int rr = tid % kTile, jj0 = tid / kTile;
  const int aoff = rr + (kstart + jj0) * ld, boff = rr + jj0 * ldw;
  auto load_c = [&](double (&cv)[4][2][2], int ti, int tj) {
    const int r0 = k + ti * kTile, c0 = k + tj * kTile;
    const double* Ct = F + r0 + (size_t)c0 * ld;
    if (ti != tj && r0 + kTile <= n) {
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
          for (int e = 0; e < 2; e++) cv[a][b][e] = Ct[rrow + 8 * a + coff[b][e]];
    } else {
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int r = r0 + rrow + 8 * a;
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int c = c0 + wc + 8 * b + 2 * q + e;
            cv[a][b][e] = (r < n && c < n && r >= c) ? Ct[rrow + 8 * a + coff[b][e]] : 0.0;
          }
      }
    }
  };
  auto stage_a = [&](double* dst, int ti) {
    const int r0 = k + ti * kTile;
    const bool ra = r0 + rr < n;
    const double* Fa = F + r0;
#pragma unroll
    for (int u = 0; u < kStD; u++) {
      const int jj = jj0 + kJs * u;
      if (jj < kp) {
        const bool p = ra && jj < kw;
        cp_async8(dst + jj * APD + rr, p ? Fa + aoff + kJs * u * ld : F, p);
      }
    }
    cp_async_commit();
  };
  auto stage_b = [&](int tj) {
    const int c0 = k + tj * kTile;
    const bool rb = c0 + rr < n;
    const double* Wb = W + c0;
    double bv[kStD];
#pragma unroll
    for (int u = 0; u < kStD; u++)
      bv[u] = (rb && jj0 + kJs * u < kw) ? Wb[boff + kJs * u * ldw] : 0.0;
#pragma unroll
    for (int u = 0; u < kStD; u++)
      if (jj0 + kJs * u < kp) Bs[(jj0 + kJs * u) * APD + rr] = bv[u];
  };
  // (tj, ti) of tile tbeg: the largest tj whose column starts at or before it
  int tj, ti;
  {
    const double b2 = 2.0 * nt + 1.0;
    int c = (int)((b2 - sqrt(b2 * b2 - 8.0 * tbeg)) * 0.5);
    auto start = [&](int cc) { return cc * nt - cc * (cc - 1) / 2; };
    while (c > 0 && start(c) > tbeg) c--;
    while (c + 1 < nt && start(c + 1) <= tbeg) c++;
    tj = c;
    ti = tj + (tbeg - start(c));
  }
  stage_b(tj);
  stage_a(As, ti);
  double cv[4][2][2];
  load_c(cv, ti, tj);
  int buf = 0;
  for (int t = tbeg;; t++) {
    cp_async_wait_all();
    __syncthreads();  // A[buf] and B are in place; nobody reads A[buf ^ 1]
    const bool more = t + 1 < tend;
    int tin = ti + 1, tjn = tj;
    if (tin == nt) {
      tjn = tj + 1;
      tin = tjn;
    }
    double cvn[4][2][2];
    if (more) {
      if (tjn == tj) stage_a(As + (buf ^ 1) * NB * APD, tin);
      load_c(cvn, tin, tjn);
    }
    const double* A = As + buf * NB * APD;
    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 2; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < NB; kk += 4) {
      if (kk < kp) {
        double af[4], bf[2];
#pragma unroll
        for (int a = 0; a < 4; a++) af[a] = A[(kk + q) * APD + rrow + 8 * a];
#pragma unroll
        for (int b = 0; b < 2; b++) bf[b] = Bs[(kk + q) * APD + wc + 8 * b + g];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int b = 0; b < 2; b++) dmma_8x8x4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
      }
    }
    {
      const int r0 = k + ti * kTile, c0 = k + tj * kTile;
      double* Ct = F + r0 + (size_t)c0 * ld;
      if (ti != tj && r0 + kTile <= n) {
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int b = 0; b < 2; b++)
#pragma unroll
            for (int e = 0; e < 2; e++)
              Ct[rrow + 8 * a + coff[b][e]] = cv[a][b][e] - acc[a][b][e];
      } else {
#pragma unroll
        for (int a = 0; a < 4; a++) {
          const int r = r0 + rrow + 8 * a;
#pragma unroll
          for (int b = 0; b < 2; b++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
              const int c = c0 + wc + 8 * b + 2 * q + e;
              if (r < n && c < n && r >= c)
                Ct[rrow + 8 * a + coff[b][e]] = cv[a][b][e] - acc[a][b][e];
            }
        }
      }
    }
    if (!more) break;
    if (tjn != tj) {
      // a new column: its B, and the next A, after every warp is done
      // with the current ones
      __syncthreads();
      stage_b(tjn);
      stage_a(As + (buf ^ 1) * NB * APD, tin);
    }
    ti = tin;
    tj = tjn;
    buf ^= 1;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 2; b++) {
        cv[a][b][0] = cvn[a][b][0];
        cv[a][b][1] = cvn[a][b][1];
      }
  }
  cp_async_wait_all();
}

// Column imax as the pivot search sees it: the largest |entry| off its
// diagonal over rows [k, n), its diagonal and its entry in row k.
struct ImaxColumn {
  double rowmax, wii, wik;
};

struct PivotChoice {
  int step;       // 0: delay candidate k; 1 or 2: size of the pivot block
  int kpiv;       // k or imax
  bool zero;      // Bunch-Kaufman zero column: D = 0, L column 0
  bool imax_1x1;  // 1x1 pivot on column imax
};

// The pivot rule for candidate k of a front (reference: the 1x1 / 2x2
// threshold tests of the front factorization, include/sparse_ldl.h, and
// LAPACK dsytf2 Bunch-Kaufman for the root front): `wkk` is the candidate's
// current diagonal, `abswik` = |entry| at imax (largest over the other
// candidates), `ctail` = largest |entry| over the non-candidate rows.
// `imax_column()` evaluates column imax; it is called only when the 1x1
// test on k fails, and by every thread of the block together.
template <class ImaxFn>
__device__ __forceinline__ PivotChoice choose_pivot(bool root, int k, int nc,
                                                    double wkk, int imax,
                                                    double abswik, double ctail,
                                                    double ustab, double pivot_tol,
                                                    ImaxFn imax_column) {
  const double bk_alpha = (1.0 + sqrt(17.0)) / 8.0;
  const double abswkk = fabs(wkk);
  PivotChoice p{0, -1, false, false};
  if (!root) {
    const double colmax = fmax(abswik, ctail);
    if (abswkk >= pivot_tol && abswkk >= ustab * colmax) {
      p.step = 1;
      p.kpiv = k;
    } else if (k + 1 < nc) {
      const ImaxColumn c = imax_column();
      const double abswii = fabs(c.wii);
      if (abswii >= pivot_tol && abswii >= ustab * c.rowmax) {
        p.step = 1;
        p.kpiv = imax;
        p.imax_1x1 = true;
      } else {
        const double det = fabs(wkk * c.wii - c.wik * c.wik);
        if (det >= pivot_tol) {
          const double delta = det / fmax(abswii + abswik, abswkk + abswik);
          if (delta >= ustab * colmax && delta >= ustab * c.rowmax) {
            p.step = 2;
            p.kpiv = imax;
          }
        }
      }
    }
  } else {
    // Bunch-Kaufman (LAPACK dsytf2/dlasyf, lower): every column is
    // eliminated, by a 1x1 or a 2x2 pivot.
    const double colmax = abswik;  // nc == n: all rows are candidates
    if (!(fmax(abswkk, colmax) > 0.0)) {
      p.step = 1;
      p.kpiv = k;
      p.zero = true;
    } else if (abswkk >= bk_alpha * colmax) {
      p.step = 1;
      p.kpiv = k;
    } else {
      const ImaxColumn c = imax_column();
      const double abswii = fabs(c.wii);
      if (abswkk >= bk_alpha * colmax * (colmax / c.rowmax)) {
        p.step = 1;
        p.kpiv = k;
      } else if (abswii >= bk_alpha * c.rowmax) {
        p.step = 1;
        p.kpiv = imax;
        p.imax_1x1 = true;
      } else {
        p.step = 2;
        p.kpiv = imax;
      }
    }
  }
  return p;
}

// W[r, col] = src(r) - F[r, kstart:kstart+kw] . ctl.wrow  for r in [k, n),
// and the reductions the pivot tests need, returned to every thread.
//   mode 0: candidate column k; src(r) = F[r, k]; first-argmax of |W| over
//           (k, nc) -> imax / abswik, max over [nc, n) -> ctail.
//   mode 1: column imax; src(r) = F[imax, r] for r < imax else F[r, imax];
//           max over [k, n) \ {imax} -> rowmax.
// Below 1024 threads the W values of the thread's first two rows
// (k + tid, k + tid + BT) are also left in keep0 / keep1 (at 1024 threads
// the registers go to the memory-bound row loop).  One barrier, after all
// W stores.
struct ColScan {
  int imax;
  double abswik, ctail, rowmax;
};
template <class T, int BT>
__device__ ColScan build_column(T* F, int ld, T* W, int ldw, int n,
                                int k, int kstart, int kw, int col, int mode,
                                int imax, int nc, CtlT<BT>& ctl, int* status,
                                const T* cache, int cld, T& keep0, T& keep1) {
  const int tid = threadIdx.x;
  double bestv = -1.0, tailv = 0.0;
  int besti = 0x7fffffff;
  int it = 0;
  for (int r = k + tid; r < n; r += BT, it++) {
    T acc;
    if (mode == 0) {
      acc = F[r + (size_t)k * ld];
    } else {
      acc = (r < imax) ? F[imax + (size_t)r * ld] : F[r + (size_t)imax * ld];
    }
    // the panel's L columns: from the shared-memory copy for its rows
    const bool inc = cache && (r - kstart) < cld;
    const T* Lr = inc ? cache + (r - kstart) : F + r + (size_t)kstart * ld;
    const size_t ls = inc ? (size_t)cld : (size_t)ld;
    // the row's panel entries QB at a time, all loads before the FMAs
    // (same summation order as one at a time).  The 1024-thread kernel
    // (64 registers a thread) keeps the plain loop, which the compiler
    // unrolls with its loads ahead on its own.
    constexpr int QB = BT >= 1024 ? 1 : 8;
    int j = 0;
    if (QB == 1)
      for (; j < kw; j++) acc -= Lr[j * ls] * T(ctl.wrow[j]);
    for (; j + QB <= kw; j += QB) {
      T v[QB];
#pragma unroll
      for (int u = 0; u < QB; u++) v[u] = Lr[(j + u) * ls];
#pragma unroll
      for (int u = 0; u < QB; u++) acc -= v[u] * T(ctl.wrow[j + u]);
    }
    if (j < kw) {
      T v[QB];
#pragma unroll
      for (int u = 0; u < QB; u++)
        if (j + u < kw) v[u] = Lr[(j + u) * ls];
#pragma unroll
      for (int u = 0; u < QB; u++)
        if (j + u < kw) acc -= v[u] * T(ctl.wrow[j + u]);
    }
    W[r + (size_t)col * ldw] = acc;
    if (BT < 1024) {
      if (it == 0) keep0 = acc;
      else if (it == 1) keep1 = acc;
    }
    const double a = fabs((double)acc);
    if (mode == 0) {
      if (r > k && r < nc) argmax_merge(bestv, besti, a, r);
      if (r >= nc) tailv = fmax(tailv, a);
    } else {
      if (r != imax) tailv = fmax(tailv, a);
    }
  }
  // warp trees, then every warp folds the warp results itself (inputs are
  // never NaN, so all threads agree)
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, bestv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, besti, o);
    const double ov2 = __shfl_xor_sync(0xffffffffu, tailv, o);
    argmax_merge(bestv, besti, ov, oi);
    tailv = fmax(tailv, ov2);
  }
  const int lane = tid & 31, warp = tid >> 5;
  if (lane == 0) {
    ctl.red_v[warp] = bestv;
    ctl.red_i[warp] = besti;
    ctl.red_v2[warp] = tailv;
  }
  __syncthreads();
  bestv = lane < BT / 32 ? ctl.red_v[lane] : -1.0;
  besti = lane < BT / 32 ? ctl.red_i[lane] : 0x7fffffff;
  tailv = lane < BT / 32 ? ctl.red_v2[lane] : 0.0;
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, bestv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, besti, o);
    const double ov2 = __shfl_xor_sync(0xffffffffu, tailv, o);
    argmax_merge(bestv, besti, ov, oi);
    tailv = fmax(tailv, ov2);
  }
  ColScan cs{0, 0.0, 0.0, 0.0};
  if (mode == 0) {
    int im = besti;
    if (im >= nc || im <= k) {
      // No finite candidate entry (all NaN, or no candidates): keep the
      // index in range; NaN is reported through the status word.
      if (k + 1 < nc && tid == 0) atomicOr(status, ST_NAN);
      im = (k + 1 < n) ? k + 1 : k;
    }
    cs.imax = im;
    cs.abswik = bestv < 0.0 ? 0.0 : bestv;
    cs.ctail = tailv;
  } else {
    cs.rowmax = tailv;
  }
  return cs;
}

// Load row `row` of W (columns 0..kw-1) into ctl.wrow.
template <class T, int BT>
__device__ void load_wrow(const T* W, int ldw, int row, int kw, CtlT<BT>& ctl) {
  for (int j = threadIdx.x; j < kw; j += BT) ctl.wrow[j] = W[row + (size_t)j * ldw];
  __syncthreads();
}

// One panel of the blocked factorization of the fully-summed columns of the
// n x n front F (lower triangle valid): candidates are taken from column k
// on while kw < NB - 1, each either eliminated (1x1 or 2x2, its L column(s)
// written to F and its L*D column(s) kept in W) or delayed to the end of the
// candidate set.  The trailing update of F[k:, k:] is left to the caller.
// `cache` (shared memory, cache_rows x NB, leading dimension cache_rows)
// keeps a copy of the panel's L columns for rows [k_, k_ + cache_rows) for
// the column builds; the other rows (and all rows when cache is nullptr)
// are read from F, which always holds the values.
template <class T, int BT>
__device__ void refresh_cache_rows(const T* F, int ld, T* cache, int cld,
                                   int kstart, int kw, int a, int b) {
  for (int t = threadIdx.x; t < 2 * kw; t += BT) {
    const int row = (t & 1) ? b : a, j = t >> 1;
    if (row - kstart < cld)
      cache[(row - kstart) + (size_t)j * cld] = F[row + (size_t)(kstart + j) * ld];
  }
}

template <class T, int BT>
__device__ void panel_factor(T* F, int ld, T* W, int ldw, int n,
                             bool root, int* vars, int* fsperm, double ustab,
                             double pivot_tol, int* status, CtlT<BT>& ctl, int& k_,
                             int& nc_, int& kw_, T* cache = nullptr,
                             int cache_rows = 0) {
  const int tid = threadIdx.x;
  int k = k_, nc = nc_, kw = 0;
  const int kstart = k;
  const int cld = cache ? (n - kstart < cache_rows ? n - kstart : cache_rows) : 0;
  // ctl.wrow holds row k of W: staged by the previous pivot step
  bool wrow_ready = true;  // kw == 0: no columns
  while (kw < NB - 1 && k < nc) {
    if (!wrow_ready) load_wrow<T, BT>(W, ldw, k, kw, ctl);
    T keep0 = T(0), keep1 = T(0), spare0, spare1;
    const ColScan cs = build_column<T, BT>(F, ld, W, ldw, n, k, kstart, kw, kw, 0, 0,
                                           nc, ctl, status, cache, cld, keep0, keep1);
    const double wkk = W[k + (size_t)kw * ldw];
    const int imax = cs.imax;
    const PivotChoice pc = choose_pivot(
        root, k, nc, wkk, imax, cs.abswik, cs.ctail, ustab, pivot_tol, [&]() {
          const double wik = W[imax + (size_t)kw * ldw];
          load_wrow<T, BT>(W, ldw, imax, kw, ctl);
          const ColScan c1 = build_column<T, BT>(F, ld, W, ldw, n, k, kstart, kw,
                                                 kw + 1, 1, imax, nc, ctl, status,
                                                 cache, cld, spare0, spare1);
          const ImaxColumn c{c1.rowmax, (double)W[imax + (size_t)(kw + 1) * ldw],
                             wik};
          // every thread holds its decision inputs before the interchange
          // or the column copy that follow rewrite them
          __syncthreads();
          return c;
        });
    if (pc.imax_1x1) {
      // column imax is the pivot column: its W column replaces column k's
      for (int r = k + tid; r < n; r += BT)
        W[r + (size_t)kw * ldw] = W[r + (size_t)(kw + 1) * ldw];
      __syncthreads();
    }
    const int step = pc.step, kpiv = pc.kpiv;
    const bool zero_pivot = pc.zero;

    if (step == 0) {
      // Delay candidate k: move it to the end of the candidate set.
      if (k < nc - 1) {
        symm_swap<T, BT>(F, ld, n, vars, fsperm, k, nc - 1);
        swap_wrows<T, BT>(W, ldw, kw, k, nc - 1);
        __syncthreads();
        if (cache) {
          refresh_cache_rows<T, BT>(F, ld, cache, cld, kstart, kw, k, nc - 1);
          __syncthreads();
        }
      }
      nc -= 1;
      wrow_ready = false;
      continue;
    }
    const int ksrc = k + step - 1;
    if (kpiv != ksrc) {
      symm_swap<T, BT>(F, ld, n, vars, fsperm, ksrc, kpiv);
      swap_wrows<T, BT>(W, ldw, kw + step, ksrc, kpiv);
      __syncthreads();
      if (cache) {
        refresh_cache_rows<T, BT>(F, ld, cache, cld, kstart, kw, ksrc, kpiv);
        __syncthreads();
      }
    }
    if (step == 1) {
      const T d = W[k + (size_t)kw * ldw];
      if (!isfinite((double)d) && tid == 0) atomicOr(status, ST_NAN);
      const T dinv = zero_pivot ? T(0) : T(1) / d;
      if (tid == 0) vars[3 * ld + k] = 0;  // 1x1 pivot
      // column k as built: no interchange or copy since, so this thread's
      // first two rows are still in keep0 / keep1
      const bool kept = BT < 1024 && kpiv == k;
      int it = 0;
      for (int r = k + tid; r < n; r += BT, it++) {
        T w = (kept && it < 2) ? (it == 0 ? keep0 : keep1) : W[r + (size_t)kw * ldw];
        const T l = (r == k) ? w : w * dinv;
        F[r + (size_t)k * ld] = l;
        if (r - kstart < cld) cache[(r - kstart) + (size_t)kw * cld] = l;
      }
    } else {
      const T d11 = W[k + (size_t)kw * ldw];
      const T d21 = W[k + 1 + (size_t)kw * ldw];
      const T d22 = W[k + 1 + (size_t)(kw + 1) * ldw];
      const T detinv = T(1) / (d11 * d22 - d21 * d21);
      if (!isfinite((double)detinv) && tid == 0) atomicOr(status, ST_NAN);
      const T i00 = d22 * detinv, i10 = -d21 * detinv,
              i01 = -d21 * detinv, i11 = d11 * detinv;
      for (int r = k + 2 + tid; r < n; r += BT) {
        T w0 = W[r + (size_t)kw * ldw], w1 = W[r + (size_t)(kw + 1) * ldw];
        const T l0 = w0 * i00 + w1 * i10, l1 = w0 * i01 + w1 * i11;
        F[r + (size_t)k * ld] = l0;
        F[r + (size_t)(k + 1) * ld] = l1;
        if (r - kstart < cld) {
          cache[(r - kstart) + (size_t)kw * cld] = l0;
          cache[(r - kstart) + (size_t)(kw + 1) * cld] = l1;
        }
      }
      if (tid == 0) {
        F[k + (size_t)k * ld] = d11;
        F[k + 1 + (size_t)k * ld] = d21;
        F[k + 1 + (size_t)(k + 1) * ld] = d22;
        vars[k] = -(vars[k] + 1);
        vars[k + 1] = -(vars[k + 1] + 1);
        // pivot kinds (first / second column of a 2x2 block), used by the
        // inertia count and the solves; vars has ld rows per section
        vars[3 * ld + k] = 1;
        vars[3 * ld + k + 1] = 2;
      }
    }
    // stage row k + step of W for the next candidate; published by the
    // barrier below (nothing reads ctl.wrow between here and there)
    if (k + step < n)
      for (int j = tid; j < kw + step; j += BT)
        ctl.wrow[j] = W[(k + step) + (size_t)j * ldw];
    wrow_ready = true;
    __syncthreads();
    k += step;
    kw += step;
  }
  k_ = k;
  nc_ = nc;
  kw_ = kw;
}

// ---------------------------------------------------------------------------
// Unblocked right-looking factorization for fronts held in shared memory.
// Every pivot's rank-1 (2x2: rank-2) update is applied to the trailing
// lower triangle at once, so each candidate column is current when it is
// examined: a pivot step is one column scan with a block reduction, the
// pivot rule, an optional interchange and the update -- two barriers for
// the common 1x1 case and no W panel.  Entries are updated as
// F[r, c] -= L[r, j] * W[c, j] in pivot order, the operands and order of
// the blocked factorization's updates.

// Reduction slots: two sets, so the column-imax reduction can follow the
// column-k one without a barrier between them; and the next candidate
// column's scan, made during the update, by step parity.
template <int BT>
struct RedSlots {
  double v[2][BT / 32];
  int i[2][BT / 32];
  double v2[2][BT / 32];
  double nv[2], nt[2];
  int ni[2];
};

// Block-wide first-argmax of (v, i) and max of v2, result in every thread.
// Per-thread inputs are never NaN (they start at -1 / 0 and only take
// larger values), so the merge is commutative and all threads agree.
template <int BT>
__device__ __forceinline__ void block_argmax_all(RedSlots<BT>& rs, int set,
                                                 double& v, int& i, double& v2) {
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    const double ov2 = __shfl_xor_sync(0xffffffffu, v2, o);
    argmax_merge(v, i, ov, oi);
    v2 = fmax(v2, ov2);
  }
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    rs.v[set][warp] = v;
    rs.i[set][warp] = i;
    rs.v2[set][warp] = v2;
  }
  __syncthreads();
  v = rs.v[set][0];
  i = rs.i[set][0];
  v2 = rs.v2[set][0];
  for (int w = 1; w < BT / 32; w++) {
    argmax_merge(v, i, rs.v[set][w], rs.i[set][w]);
    v2 = fmax(v2, rs.v2[set][w]);
  }
}

// L column(s) of the pivot at k: rows (k + step, n) of column k (and k+1)
// scaled by D^-1 from the unscaled L*D values left there by the update.
template <class T, int BT>
__device__ __forceinline__ void rl_scale(T* F, int ld, int n, int k, int step,
                                         T dinv, T i00, T i10, T i01, T i11) {
  if (step == 1) {
    T* Fk = F + (size_t)k * ld;
    for (int r = k + 1 + threadIdx.x; r < n; r += BT) Fk[r] = Fk[r] * dinv;
  } else {
    T* F0 = F + (size_t)k * ld;
    T* F1 = F0 + ld;
    for (int r = k + 2 + threadIdx.x; r < n; r += BT) {
      const T w0 = F0[r], w1 = F1[r];
      F0[r] = w0 * i00 + w1 * i10;
      F1[r] = w0 * i01 + w1 * i11;
    }
  }
}

// Rank-1 (STEP 1) or rank-2 (STEP 2) update of the trailing triangle
// F[c0:, c0:] by the pivot at k: F[r, c] -= L[r, j] * W[c, j], j = k (and
// k+1), with L = W D^-1 (coefficients d00..d11).  Warp 0 takes column c0,
// one lane per row, and leaves its scan for the next pivot search
// (first-argmax over the candidates c0 < r < nc, max over r >= nc) in slot
// `par`: that column is the next step's critical path, so no other work
// shares the warp.  The other warps form a 16 x TC grid over columns
// c0+1 .. n-1: thread (tr, tc) takes columns c0 + 1 + tc + TC j and, in
// each, the rows on or below the diagonal congruent to c0 + 1 + tr modulo
// 16.  Returns whether the scan was left (c0 < n).
constexpr int kRlRows = 16;

template <class T, int BT, int STEP>
__device__ __forceinline__ bool rl_update(T* F, int ld, int n, int k, int c0,
                                          int nc, T d00, T d10, T d01, T d11,
                                          int par, RedSlots<BT>& rs) {
  static_assert(BT >= 64, "one warp for column c0 and at least one more");
  constexpr int TR = kRlRows, TC = (BT - 32) / TR;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const T* W0 = F + (size_t)k * ld;
  const T* W1 = W0 + ld;
  if (c0 >= n) return false;
  if (warp == 0) {
    double bv = -1.0, tv = 0.0;
    int bi = 0x7fffffff;
    const T y0 = W0[c0];
    const T y1 = STEP == 2 ? W1[c0] : T(0);
    T* Fc = F + (size_t)c0 * ld;
    for (int r = c0 + lane; r < n; r += 32) {
      T acc = Fc[r];
      if (STEP == 1) {
        acc -= (W0[r] * d00) * y0;
      } else {
        const T w0 = W0[r], w1 = W1[r];
        const T l0 = w0 * d00 + w1 * d10, l1 = w0 * d01 + w1 * d11;
        acc -= l0 * y0;
        acc -= l1 * y1;
      }
      Fc[r] = acc;
      const double av = fabs((double)acc);
      if (r > c0 && r < nc) argmax_merge(bv, bi, av, r);
      else if (r >= nc) tv = fmax(tv, av);
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      const double ot = __shfl_xor_sync(0xffffffffu, tv, o);
      argmax_merge(bv, bi, ov, oi);
      tv = fmax(tv, ot);
    }
    if (lane == 0) {
      rs.nv[par] = bv;
      rs.ni[par] = bi;
      rs.nt[par] = tv;
    }
    return true;
  }
  const int t = threadIdx.x - 32;
  const int tr = t % TR, tc = t / TR;
  const int b0 = c0 + 1;
  for (int c = b0 + tc; c < n; c += TC) {
    const T y0 = W0[c];
    const T y1 = STEP == 2 ? W1[c] : T(0);
    T* Fc = F + (size_t)c * ld;
    int r = b0 + tr;
    if (r < c) r += ((c - r + TR - 1) / TR) * TR;
    for (; r < n; r += TR) {
      T acc = Fc[r];
      if (STEP == 1) {
        acc -= (W0[r] * d00) * y0;
      } else {
        const T w0 = W0[r], w1 = W1[r];
        const T l0 = w0 * d00 + w1 * d10, l1 = w0 * d01 + w1 * d11;
        acc -= l0 * y0;
        acc -= l1 * y1;
      }
      Fc[r] = acc;
    }
  }
  return true;
}

// Factor the fully-summed columns [0, fs) of the n x n front F (lower
// triangle, leading dimension ld) in one CTA; `vars` holds 4 sections of ld
// ints (variables, fully-summed permutation, -, pivot kinds).  Same pivot
// rule, interchanges and output layout as the blocked panel factorization
// of the large fronts.  Returns the number of pivots.
template <class T, int BT>
__device__ int factor_front_rl(T* F, int ld, int n, int fs, bool root,
                               int* vars, int* fsperm, double ustab,
                               double pivot_tol, int* status, RedSlots<BT>& rs) {
  const int tid = threadIdx.x;
  int k = 0, nc = fs;
  int par = 0;          // parity of the scan slot the next step reads
  bool have = false;    // the update left the scan of column k in slot par
  // the last pivot, whose L column(s) are scaled at the next step
  int pk = -1, pstep = 0;
  T pd = T(0), p00 = T(0), p10 = T(0), p01 = T(0), p11 = T(0);
  while (k < nc) {
    if (pk >= 0) {
      rl_scale<T, BT>(F, ld, n, pk, pstep, pd, p00, p10, p01, p11);
      pk = -1;
    }
    const T* Fk = F + (size_t)k * ld;
    double bv, tv;
    int bi;
    if (have) {
      bv = rs.nv[par];
      bi = rs.ni[par];
      tv = rs.nt[par];
    } else {
      // candidate column k: first-argmax of |F[r, k]| over candidates
      // r > k, max over the non-candidate rows
      bv = -1.0;
      tv = 0.0;
      bi = 0x7fffffff;
      for (int r = k + 1 + tid; r < n; r += BT) {
        const double a = fabs((double)Fk[r]);
        if (r < nc) argmax_merge(bv, bi, a, r);
        else tv = fmax(tv, a);
      }
      block_argmax_all<BT>(rs, 0, bv, bi, tv);
    }
    int imax = bi;
    if (imax >= nc || imax <= k) {
      // no finite candidate entry (all NaN, or no candidates)
      if (k + 1 < nc && tid == 0) atomicOr(status, ST_NAN);
      imax = (k + 1 < n) ? k + 1 : k;
    }
    const PivotChoice pc = choose_pivot(
        root, k, nc, (double)Fk[k], imax, bv < 0.0 ? 0.0 : bv, tv, ustab,
        pivot_tol, [&]() {
          // read before the reduction's barrier: past it, other threads may
          // interchange or update these entries
          const double wii = F[imax + (size_t)imax * ld], wik = F[imax + (size_t)k * ld];
          double rv = -1.0, rt = 0.0;
          int ri = 0x7fffffff;
          for (int r = k + tid; r < n; r += BT) {
            if (r == imax) continue;
            const T x = r < imax ? F[imax + (size_t)r * ld] : F[r + (size_t)imax * ld];
            rt = fmax(rt, fabs((double)x));
          }
          block_argmax_all<BT>(rs, 1, rv, ri, rt);
          return ImaxColumn{rt, wii, wik};
        });
    if (pc.step == 0) {
      // delay candidate k: move it to the end of the candidate set
      if (k < nc - 1) {
        symm_swap<T, BT>(F, ld, n, vars, fsperm, k, nc - 1);
        __syncthreads();
      }
      nc -= 1;
      have = false;
      continue;
    }
    const int step = pc.step;
    const int ksrc = k + step - 1;
    if (pc.kpiv != ksrc) {
      symm_swap<T, BT>(F, ld, n, vars, fsperm, ksrc, pc.kpiv);
      __syncthreads();
    }
    const int c0 = k + step;
    const int npar = par ^ 1;
    if (step == 1) {
      const T d = Fk[k];
      if (!isfinite((double)d) && tid == 0) atomicOr(status, ST_NAN);
      const T dinv = pc.zero ? T(0) : T(1) / d;
      if (tid == 0) vars[3 * ld + k] = 0;  // 1x1 pivot
      have = rl_update<T, BT, 1>(F, ld, n, k, c0, nc, dinv, T(0), T(0), T(0), npar, rs);
      pd = dinv;
    } else {
      const T* W1 = Fk + ld;
      const T d11 = Fk[k], d21 = Fk[k + 1], d22 = W1[k + 1];
      const T detinv = T(1) / (d11 * d22 - d21 * d21);
      if (!isfinite((double)detinv) && tid == 0) atomicOr(status, ST_NAN);
      const T i00 = d22 * detinv, i10 = -d21 * detinv,
              i01 = -d21 * detinv, i11 = d11 * detinv;
      if (tid == 0) {
        vars[k] = -(vars[k] + 1);
        vars[k + 1] = -(vars[k + 1] + 1);
        vars[3 * ld + k] = 1;
        vars[3 * ld + k + 1] = 2;
      }
      have = rl_update<T, BT, 2>(F, ld, n, k, c0, nc, i00, i10, i01, i11, npar, rs);
      p00 = i00; p10 = i10; p01 = i01; p11 = i11;
    }
    pk = k;
    pstep = step;
    par = npar;
    __syncthreads();
    k += step;
  }
  if (pk >= 0) rl_scale<T, BT>(F, ld, n, pk, pstep, pd, p00, p10, p01, p11);
  __syncthreads();
  return nc;
}

// Front set-up shared by both paths (thread 0 sizes and allocates; all
// threads fill the variable list and the fully-summed permutation record).
// Returns false when the front must be skipped (a pool ran out earlier).
template <class T, int BT>
__device__ bool setup_front(const DevicePlan& d, int node, CtlT<BT>& ctl) {
  const int tid = threadIdx.x;
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
      // F followed by W in elements of T, rounded to 64 bytes; the pool
      // holds fcap doubles
      constexpr unsigned long long al = 64 / sizeof(T);
      const unsigned long long need =
          (((unsigned long long)f * f + (unsigned long long)f * NB) + 2 * al - 1) &
          ~(al - 1);
      const unsigned long long cap =
          (unsigned long long)d.fcap * (sizeof(double) / sizeof(T));
      const unsigned long long ineed = (4ull * f + 15) & ~7ull;
      unsigned long long off = atomicAdd(&d.counters[0], need);
      unsigned long long ioff = atomicAdd(&d.counters[1], ineed);
      if (off + need > cap) {
        atomicOr(d.status, ST_POOL_F);
        ctl.skip = 1;
      }
      if (ioff + ineed > (unsigned long long)d.icap) {
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
    d.pstate[4 * node + 0] = 0;          // k
    d.pstate[4 * node + 1] = ns + ndin;  // candidates left
    d.pstate[4 * node + 2] = 0;          // kstart of the last panel
    d.pstate[4 * node + 3] = 0;          // kw of the last panel
    if (ctl.skip) {
      d.npiv[node] = 0;
      d.ndel[node] = 0;
      d.pstate[4 * node + 1] = 0;
    }
  }
  __syncthreads();
  if (ctl.skip) return false;
  const int f = ctl.f, fs = ctl.fs, ns = ctl.ns;
  int* fvars = d.ipool + ctl.ioff;
  int* fsperm = fvars + f;
  // Variable list: node vars, delayed pivots of the children, contribution
  // rows (include/sparse_ldl.h:957-987, 596-616).
  const int vbase = d.var_ptr[node];
  for (int r = tid; r < ns; r += BT) fvars[r] = d.vars[vbase + r];
  int choff = ns;
  for (int q = d.kid_ptr[node]; q < d.kid_ptr[node + 1]; q++) {
    const int c = d.kids[q];
    const int ndc = d.ndel[c];
    const int* cv = d.ipool + d.ioff[c] + d.npiv[c];
    for (int t = tid; t < ndc; t += BT) fvars[choff + t] = cv[t];
    choff += ndc;
  }
  const int cb = d.cptr[node];
  for (int t = tid; t < d.nc[node]; t += BT) fvars[fs + t] = d.crows[cb + t];
  for (int r = tid; r < fs; r += BT) fsperm[r] = r;
  __syncthreads();
  return true;
}

// Static position of a child's contribution row `a` in the parent front.
__device__ __forceinline__ int child_row_pos(const DevicePlan& d, int cb,
                                             int ndc, int choff, int ns,
                                             int ndin, int a) {
  if (a < ndc) return choff + a;
  const int r0 = d.cmap[cb + a - ndc];
  return r0 < ns ? r0 : r0 + ndin;
}

// Inertia of the D blocks with the reference's rule
// (include/sparse_ldl.h:1937-1968), from the pivot kinds recorded when each
// pivot was accepted (0: 1x1, 1/2: first/second column of a 2x2 block),
// plus the inverse of the fully-summed permutation used by the solves.
template <class T>
__device__ void finish_front(const DevicePlan& d, int node, const T* F,
                             int f, int fs, int npiv, int* fvars) {
  __shared__ int s_pos, s_neg;
  const int tid = threadIdx.x;
  const int* fsperm = fvars + f;
  int* fsinv = fvars + 2 * f;
  const int* kind = fvars + 3 * f;
  if (tid == 0) {
    s_pos = 0;
    s_neg = 0;
  }
  for (int r = tid; r < fs; r += blockDim.x) fsinv[fsperm[r]] = r;
  __syncthreads();
  int pos = 0, neg = 0;
  for (int j = tid; j < npiv; j += blockDim.x) {
    const int kd = kind[j];
    if (kd == 0) {
      if ((double)F[j + (size_t)j * f] >= 0.0) pos++; else neg++;
    } else if (kd == 1) {
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
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    pos += __shfl_down_sync(0xffffffffu, pos, o);
    neg += __shfl_down_sync(0xffffffffu, neg, o);
  }
  if ((tid & 31) == 0 && (pos || neg)) {
    atomicAdd(&s_pos, pos);
    atomicAdd(&s_neg, neg);
  }
  __syncthreads();
  if (tid == 0) {
    const int pb = d.node_prob ? d.node_prob[node] : 0;
    atomicAdd(&d.inertia[2 * pb], s_pos);
    atomicAdd(&d.inertia[2 * pb + 1], s_neg);
    d.npiv[node] = npiv;
    d.ndel[node] = fs - npiv;
  }
}

// Assemble front `node` (f x f, leading dimension f) in F: zero, add the
// entries of A, extend-add the children's contribution blocks.  `rmap`
// holds f ints of scratch.
template <class T, int BT>
__device__ void assemble_front(const DevicePlan& d, int node, T* F, int f,
                               int ns, int ndin, const double* __restrict__ vals,
                               int* rmap) {
  const int tid = threadIdx.x;
  const T* pool = reinterpret_cast<const T*>(d.fpool);
  for (size_t idx = tid; idx < (size_t)f * f; idx += BT) F[idx] = T(0);
  __syncthreads();
  // each entry of A lands on its own front position: the index loads of a
  // thread's next entries are issued before its adds
  {
    const int a0 = d.amap_ptr[node], a1 = d.amap_ptr[node + 1];
    for (int t0 = a0 + tid; t0 < a1; t0 += 4 * BT) {
      long long pos[4];
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int t = t0 + u * BT;
        pos[u] = -1;
        if (t < a1) {
          const int r0 = d.amap_row[t];
          const int r = r0 < ns ? r0 : r0 + ndin;
          pos[u] = r + (long long)d.amap_col[t] * f;
          v[u] = vals[d.amap_pos[t]];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (pos[u] >= 0) F[pos[u]] += T(v[u]);
    }
  }
  __syncthreads();
  int choff = ns;
  for (int q = d.kid_ptr[node]; q < d.kid_ptr[node + 1]; q++) {
    const int c = d.kids[q];
    const int fc = d.f[c], npc = d.npiv[c], ndc = d.ndel[c];
    const int cc = fc - npc;
    const T* C = pool + d.foff[c];
    const int cb = d.cptr[c];
    for (int a = tid; a < cc; a += BT)
      rmap[a] = child_row_pos(d, cb, ndc, choff, ns, ndin, a);
    __syncthreads();
    for (int b = 0; b < cc; b++) {
      const int pb = rmap[b];
      const T* Cb = C + (size_t)(npc + b) * fc + npc;
      for (int a = b + tid; a < cc; a += BT) {
        const int pa = rmap[a];
        const T v = Cb[a];
        if (pa >= pb) F[pa + (size_t)pb * f] += v;
        else F[pb + (size_t)pa * f] += v;
      }
    }
    __syncthreads();
    choff += ndc;
  }
}

// Small fronts with the unblocked right-looking factorization: the front
// and its four integer sections (variables, fully-summed permutation,
// inverse permutation, pivot kinds) in shared memory when they fit, else in
// the pools; `smem_bytes` is the dynamic shared memory of the launch.
// Four CTAs per SM (64 registers a thread at 256 threads): as many fronts
// as shared memory holds for 70-row fronts.
template <class T, int BT>
__global__ void __launch_bounds__(BT, 4)
k_factor_level_rl(DevicePlan d, const int* __restrict__ nodes, int count,
                  const double* __restrict__ vals, double ustab,
                  double pivot_tol, int smem_bytes) {
  extern __shared__ double smem_raw[];
  __shared__ CtlT<BT> ctl;
  __shared__ RedSlots<BT> rs;
  const int tid = threadIdx.x;
  const int node = nodes[blockIdx.x];
  if (!setup_front<T, BT>(d, node, ctl)) return;
  T* pool = reinterpret_cast<T*>(d.fpool);
  const int f = ctl.f, fs = ctl.fs, ns = ctl.ns, ndin = ctl.ndin;
  int* fvars = d.ipool + ctl.ioff;
  T* Fg = pool + ctl.foff;
  const long long fbytes = ((long long)f * f * (long long)sizeof(T) + 15) & ~15ll;
  const bool in_smem = fbytes + 5ll * f * (long long)sizeof(int) <= smem_bytes;
  T* F = in_smem ? reinterpret_cast<T*>(smem_raw) : Fg;
  int* iv = in_smem ? reinterpret_cast<int*>(reinterpret_cast<char*>(smem_raw) + fbytes)
                    : fvars;
  // scratch for the child row map: shared memory, or the front's W area
  int* rmap = in_smem ? iv + 4 * f : reinterpret_cast<int*>(Fg + (size_t)f * f);
  if (in_smem)
    for (int t = tid; t < 2 * f; t += BT) iv[t] = fvars[t];
  assemble_front<T, BT>(d, node, F, f, ns, ndin, vals, rmap);
  const int npiv = factor_front_rl<T, BT>(F, f, f, fs, fs == f, iv, iv + f,
                                          ustab, pivot_tol, d.status, rs);
  if (in_smem) {
    for (size_t idx = tid; idx < (size_t)f * f; idx += BT) Fg[idx] = F[idx];
    for (int t = tid; t < 2 * f; t += BT) fvars[t] = iv[t];
    for (int t = tid; t < npiv; t += BT) fvars[3 * f + t] = iv[3 * f + t];
  }
  __syncthreads();
  finish_front(d, node, F, f, fs, npiv, fvars);
}

// ---------------------------------------------------------------------------
// Large fronts: one CTA sets each front up, grids of CTAs assemble it, then
// the factorization alternates a one-CTA panel kernel with a multi-CTA
// trailing-update kernel over 64 x 64 tiles.

template <class T>
__global__ void __launch_bounds__(NT)
k_big_setup(DevicePlan d, const int* __restrict__ nodes) {
  __shared__ Ctl ctl;
  setup_front<T, NT>(d, nodes[blockIdx.x], ctl);
}

__device__ __forceinline__ bool big_skip(const DevicePlan& d) {
  return (*((volatile int*)d.status) & (ST_POOL_F | ST_POOL_I)) != 0;
}

template <class T>
__global__ void __launch_bounds__(NT)
k_big_zero(DevicePlan d, const int* __restrict__ nodes) {
  if (big_skip(d)) return;
  const int node = nodes[blockIdx.x];
  const size_t f = d.f[node];
  T* F = reinterpret_cast<T*>(d.fpool) + d.foff[node];
  for (size_t idx = (size_t)blockIdx.y * NT + threadIdx.x; idx < f * f;
       idx += (size_t)gridDim.y * NT)
    F[idx] = T(0);
}

template <class T>
__global__ void __launch_bounds__(NT)
k_big_add_A(DevicePlan d, const int* __restrict__ nodes,
            const double* __restrict__ vals) {
  if (big_skip(d)) return;
  const int node = nodes[blockIdx.x];
  const int f = d.f[node], ns = d.ns[node], ndin = d.ndin[node];
  T* F = reinterpret_cast<T*>(d.fpool) + d.foff[node];
  for (int t = d.amap_ptr[node] + blockIdx.y * NT + threadIdx.x;
       t < d.amap_ptr[node + 1]; t += gridDim.y * NT) {
    const int r0 = d.amap_row[t];
    const int r = r0 < ns ? r0 : r0 + ndin;
    F[r + (size_t)d.amap_col[t] * f] += T(vals[d.amap_pos[t]]);
  }
}

// Extend-add of the q-th child of every front (one launch per child rank,
// so that no two writers of a launch touch the same parent entry).
template <class T>
__global__ void __launch_bounds__(NT)
k_big_extend(DevicePlan d, const int* __restrict__ nodes, int q) {
  if (big_skip(d)) return;
  const int node = nodes[blockIdx.x];
  const int q0 = d.kid_ptr[node];
  if (q0 + q >= d.kid_ptr[node + 1]) return;
  const int f = d.f[node], ns = d.ns[node], ndin = d.ndin[node];
  int choff = ns;
  for (int t = 0; t < q; t++) choff += d.ndel[d.kids[q0 + t]];
  const int c = d.kids[q0 + q];
  const int fc = d.f[c], npc = d.npiv[c], ndc = d.ndel[c];
  const int cc = fc - npc, cb = d.cptr[c];
  const T* C = reinterpret_cast<const T*>(d.fpool) + d.foff[c];
  T* F = reinterpret_cast<T*>(d.fpool) + d.foff[node];
  for (int b = blockIdx.y; b < cc; b += gridDim.y) {
    const int pb = child_row_pos(d, cb, ndc, choff, ns, ndin, b);
    const T* Cb = C + (size_t)(npc + b) * fc + npc;
    for (int a = b + threadIdx.x; a < cc; a += NT) {
      const int pa = child_row_pos(d, cb, ndc, choff, ns, ndin, a);
      const T v = Cb[a];
      if (pa >= pb) F[pa + (size_t)pb * f] += v;
      else F[pb + (size_t)pa * f] += v;
    }
  }
}

template <class T, int PT>
__global__ void __launch_bounds__(PT)
k_big_panel(DevicePlan d, const int* __restrict__ nodes, double ustab,
            double pivot_tol, int cache_bytes) {
  pdl_enter();
  __shared__ CtlT<PT> ctl;
  extern __shared__ double cache_raw[];
  if (big_skip(d)) return;
  const int node = nodes[blockIdx.x];
  int* st = d.pstate + 4 * node;
  int k = st[0], nc = st[1];
  if (k >= nc) {
    if (threadIdx.x == 0) st[3] = 0;
    return;
  }
  const int f = d.f[node];
  const int fs = d.ns[node] + d.ndin[node];
  T* F = reinterpret_cast<T*>(d.fpool) + d.foff[node];
  T* W = F + (size_t)f * f;
  int* fvars = d.ipool + d.ioff[node];
  const int kstart = k;
  int kw = 0;
  // the panel's L columns in shared memory for as many rows as fit
  const int cache_rows = cache_bytes / (NB * (int)sizeof(T));
  T* cache = cache_rows > 0 ? reinterpret_cast<T*>(cache_raw) : nullptr;
  panel_factor<T, PT>(F, f, W, f, f, fs == f, fvars, fvars + f, ustab, pivot_tol,
               d.status, ctl, k, nc, kw, cache, cache_rows);
  if (threadIdx.x == 0) {
    st[0] = k;
    st[1] = nc;
    st[2] = kstart;
    st[3] = kw;
  }
}

// ---------------------------------------------------------------------------
// Large-front panel with the panel's W columns in shared memory.
//
// The same pivot rule, candidate order, interchanges and outputs as
// panel_factor (the reference's left-looking-in-panel scheme), arranged so
// that one candidate column costs one block reduction and one barrier in
// the common case (a 1x1 pivot without interchange):
//   * W[kstart:, 0:kw] (the panel's unscaled L*D columns) lives in shared
//     memory, column-major with leading dimension cld = f - kstart, so a
//     column build reads only shared memory: L[r, j] is recomputed from W
//     with the same expression that writes it to F (W[r, j] * dinv_j for a
//     1x1 pivot; the D^-1 combination of the two W columns of a 2x2 pivot);
//   * each thread owns the rows kstart + tid + PT * i (i < RPT) for the
//     whole panel and keeps their entries of the next candidate column of
//     F, loaded one step ahead (reloaded after an interchange or a delay);
//   * the L columns are written to F and the W rows to HBM once, at the end
//     of the panel (the trailing-update kernel reads both there).
// The panel width adapts to the shared memory: nbe = min(kPanel,
// smem / (cld * sizeof(T))) columns, at least 4.
template <int PT>
struct SwCtl {
  // reduction slots by step parity and kind (candidate column, column
  // imax): a step's slots are written again two steps later, after the
  // next step's barrier, so no barrier is needed at the end of a step
  double red_v[4][PT / 32];
  int red_i[4][PT / 32];
  double red_v2[4][PT / 32];
  double wkk[2], wii;
  double cA[NB], cB[NB];   // L[r, j] = W[r, j] cA[j] + W[r, cP[j]] cB[j]
  int cP[NB];              // the column's partner (itself for a 1x1 pivot)
  int kind[NB];            // 0: 1x1, 1 / 2: first / second column of a 2x2
  // row interchanges of the panel's pivots not yet applied to the columns
  // left of the panel, and their composition (rows[t] <- src[t])
  int swa[NB], swb[NB], nsw;
  int rows[2 * NB], src[2 * NB], nrows;
};

// The pending interchanges of a panel composed into one row map (rows[t]
// takes the value of row src[t]); run by one thread.  The count c.nsw is
// left for the caller to reset after a barrier: every thread reads it to
// decide whether to join the barriers of the flush.
template <class C>
__device__ void compose_swaps(C& c) {
  int nr = 0;
  for (int s = 0; s < c.nsw; s++) {
    const int pr[2] = {c.swa[s], c.swb[s]};
    int at[2];
    for (int u = 0; u < 2; u++) {
      at[u] = -1;
      for (int t = 0; t < nr; t++)
        if (c.rows[t] == pr[u]) at[u] = t;
      if (at[u] < 0) {
        c.rows[nr] = pr[u];
        c.src[nr] = pr[u];
        at[u] = nr++;
      }
    }
    const int tmp = c.src[at[0]];
    c.src[at[0]] = c.src[at[1]];
    c.src[at[1]] = tmp;
  }
  c.nrows = nr;
}

// Row map applied to the columns [0, kstart) of F by warps gw, gw + gws,
// ...: a warp takes 8 columns at a time, its lanes load the mapped rows of
// all 8 before storing any (nr <= 64 rows).  L2 loads (CG) where another
// CTA may have written the entries in the same launch.
template <class T, bool CG>
__device__ void apply_row_map(T* F, int ld, int kstart, const int* rows,
                              const int* src, int nr, int gw, int gws) {
  const int lane = threadIdx.x & 31;
  const bool h0 = lane < nr, h1 = lane + 32 < nr;
  const int s0 = h0 ? src[lane] : 0, s1 = h1 ? src[lane + 32] : 0;
  const int d0 = h0 ? rows[lane] : 0, d1 = h1 ? rows[lane + 32] : 0;
  constexpr int CB = 8;
  for (int j0 = gw * CB; j0 < kstart; j0 += gws * CB) {
    T v0[CB], v1[CB];
#pragma unroll
    for (int u = 0; u < CB; u++) {
      const T* Fj = F + (size_t)(j0 + u) * ld;
      const bool in = j0 + u < kstart;
      if constexpr (CG) {
        v0[u] = in && h0 ? __ldcg(Fj + s0) : T(0);
        v1[u] = in && h1 ? __ldcg(Fj + s1) : T(0);
      } else {
        v0[u] = in && h0 ? Fj[s0] : T(0);
        v1[u] = in && h1 ? Fj[s1] : T(0);
      }
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < CB; u++) {
      if (j0 + u >= kstart) break;
      T* Fj = F + (size_t)(j0 + u) * ld;
      if (h0) Fj[d0] = v0[u];
      if (h1) Fj[d1] = v1[u];
    }
  }
}

// Apply the pending interchanges to the columns [0, kstart) left of the
// panel: thread 0 composes them into one row map, then the CTA's warps
// move the rows of the map.
template <class T, int PT>
__device__ void sw_flush_left(T* F, int ld, int kstart, SwCtl<PT>& c) {
  __syncthreads();
  // every thread takes the count before any thread changes it
  if (c.nsw == 0) return;
  if (threadIdx.x == 0) compose_swaps(c);
  __syncthreads();
  apply_row_map<T, false>(F, ld, kstart, c.rows, c.src, c.nrows, threadIdx.x >> 5,
                          PT / 32);
  __syncthreads();
  if (threadIdx.x == 0) c.nsw = 0;
}

// Interchange a < b for a pivot taken at position a (an imax 1x1 pivot,
// or the second column of a 2x2 pivot): only the entries that stay live
// are written -- column b and row b of the trailing part from column a's
// values, which each thread holds for its rows in colA -- since column a
// becomes a pivot column whose values come from the shared W.  The row
// interchange of the columns left of the panel is recorded for
// sw_flush_left; the panel's own columns are written at its end from W.
template <class T, int PT, int RPT>
__device__ __forceinline__ void sw_pivot_swap(T* F, int ld, int n, int kstart,
                                              int a, int b, const int (&rr)[RPT],
                                              const bool (&on)[RPT],
                                              const T (&colA)[RPT], int* vars,
                                              int* fsperm, SwCtl<PT>& c) {
#pragma unroll
  for (int i = 0; i < RPT; i++) {
    if (!on[i]) continue;
    const int r = kstart + rr[i];
    if (r > a && r < b) F[b + (size_t)r * ld] = colA[i];
    else if (r > b) F[r + (size_t)b * ld] = colA[i];
    else if (r == a) F[b + (size_t)b * ld] = colA[i];
  }
  if (threadIdx.x == 0) {
    int tv = vars[a];
    vars[a] = vars[b];
    vars[b] = tv;
    tv = fsperm[a];
    fsperm[a] = fsperm[b];
    fsperm[b] = tv;
    c.swa[c.nsw] = a;
    c.swb[c.nsw] = b;
    c.nsw++;
  }
}

// Block-wide first-argmax of (v, i) and max of v2 in every thread, in
// reduction slot `set`.
template <int PT>
__device__ __forceinline__ void sw_reduce(SwCtl<PT>& c, int set, double& v,
                                          int& i, double& v2) {
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    const double ov2 = __shfl_xor_sync(0xffffffffu, v2, o);
    argmax_merge(v, i, ov, oi);
    v2 = fmax(v2, ov2);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    c.red_v[set][warp] = v;
    c.red_i[set][warp] = i;
    c.red_v2[set][warp] = v2;
  }
  __syncthreads();
  v = lane < PT / 32 ? c.red_v[set][lane] : -1.0;
  i = lane < PT / 32 ? c.red_i[set][lane] : 0x7fffffff;
  v2 = lane < PT / 32 ? c.red_v2[set][lane] : 0.0;
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    const double ov2 = __shfl_xor_sync(0xffffffffu, v2, o);
    argmax_merge(v, i, ov, oi);
    v2 = fmax(v2, ov2);
  }
}

// The D^-1 of a 2x2 pivot block [d11 d21; d21 d22] as the coefficients of
// its two L columns in terms of their W columns: l0 = w0 i00 + w1 i10,
// l1 = w1 i11 + w0 i01.
struct Coef2 {
  double i00, i10, i11, i01;
  bool finite;
};
template <class T>
__device__ __forceinline__ Coef2 pivot2_coeffs(T d11, T d21, T d22) {
  const T detinv = T(1) / (d11 * d22 - d21 * d21);
  return Coef2{(double)(d22 * detinv), (double)(-d21 * detinv),
               (double)(d11 * detinv), (double)(-d21 * detinv),
               (bool)isfinite((double)detinv)};
}

// acc[i] -= sum_j L[r_i, j] * y[j] over the panel's columns j < kw, with
// L recomputed from the shared W columns; y[j] = W[yrow, j] of the column
// being built.  Every column is L[r, j] = W[r, j] cA[j] + W[r, cP[j]] cB[j]
// (cB = 0 and cP = j for a 1x1 pivot: the product W[r, j] cA[j] exactly).
// The sum runs in four partial sums, column j into partial j mod 4 in the
// order of j, added as (s0 + s1) + (s2 + s3): four independent chains of
// multiply-adds instead of one (the cluster panel sums in the same order).
template <class T>
__device__ __forceinline__ T sw_l(T w, T wp, T a, T b) {
  return fma(wp, b, w * a);
}

template <class T, int RPT>
__device__ __forceinline__ void sum4_apply(T (&acc)[RPT], const T (&s)[RPT][4]) {
#pragma unroll
  for (int i = 0; i < RPT; i++) acc[i] -= (s[i][0] + s[i][1]) + (s[i][2] + s[i][3]);
}

template <class T, int PT, int RPT>
__device__ __forceinline__ void sw_apply_panel(const T* __restrict__ Ws, int cld,
                                               int kw, int yrow, const SwCtl<PT>& c,
                                               const int (&rr)[RPT],
                                               const bool (&on)[RPT], T (&acc)[RPT]) {
  T s[RPT][4];
#pragma unroll
  for (int i = 0; i < RPT; i++)
#pragma unroll
    for (int q = 0; q < 4; q++) s[i][q] = T(0);
  int j = 0;
  for (; j + 4 <= kw; j += 4) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const T* w0 = Ws + (size_t)(j + q) * cld;
      const T* p0 = Ws + (size_t)c.cP[j + q] * cld;
      const T a0 = T(c.cA[j + q]), b0 = T(c.cB[j + q]), y0 = w0[yrow];
#pragma unroll
      for (int i = 0; i < RPT; i++)
        if (on[i]) s[i][q] += sw_l(w0[rr[i]], p0[rr[i]], a0, b0) * y0;
    }
  }
  // the last kw mod 4 columns (j is a multiple of 4 here: column j + q goes
  // to partial q)
#pragma unroll
  for (int q = 0; q < 3; q++) {
    if (j + q >= kw) break;
    const T* w0 = Ws + (size_t)(j + q) * cld;
    const T* p0 = Ws + (size_t)c.cP[j + q] * cld;
    const T a0 = T(c.cA[j + q]), b0 = T(c.cB[j + q]), y0 = w0[yrow];
#pragma unroll
    for (int i = 0; i < RPT; i++)
      if (on[i]) s[i][q] += sw_l(w0[rr[i]], p0[rr[i]], a0, b0) * y0;
  }
#pragma unroll
  for (int i = 0; i < RPT; i++)
    if (!on[i]) s[i][0] = s[i][1] = s[i][2] = s[i][3] = T(0);
  sum4_apply<T, RPT>(acc, s);
}

// Rows a and b interchanged in the shared W columns [0, ncol).
template <class T, int PT>
__device__ __forceinline__ void sw_swap_rows(T* Ws, int cld, int ncol, int a,
                                             int b) {
  for (int j = threadIdx.x; j < ncol; j += PT) {
    T t = Ws[a + (size_t)j * cld];
    Ws[a + (size_t)j * cld] = Ws[b + (size_t)j * cld];
    Ws[b + (size_t)j * cld] = t;
  }
}

template <class T, int PT, int RPT>
__device__ void panel_factor_sw(T* F, int ld, T* Wg, int n, bool root,
                                int* vars, int* fsperm, double ustab,
                                double pivot_tol, int* status, SwCtl<PT>& c,
                                T* Ws, int nbe, int& k_, int& nc_, int& kw_,
                                int* dbg) {
  const int tid = threadIdx.x;
  if (tid == 0) c.nsw = 0;
  int k = k_, nc = nc_, kw = 0;
  const int kstart = k;
  const int cld = n - kstart;
  int rr[RPT];       // owned rows relative to kstart
  bool on[RPT];
  T cur[RPT];        // F[r, k] of the candidate column
#pragma unroll
  for (int i = 0; i < RPT; i++) rr[i] = tid + PT * i;
  auto load_col = [&](int col, T (&dst)[RPT]) {
#pragma unroll
    for (int i = 0; i < RPT; i++) {
      const int r = kstart + rr[i];
      dst[i] = (r >= col && r < n) ? F[r + (size_t)col * ld] : T(0);
    }
  };
  load_col(k, cur);
  int par = 0;
  unsigned long long* cyc =
      dbg ? reinterpret_cast<unsigned long long*>(dbg + 8) : nullptr;
  long long tc0 = 0, tc1 = 0, tc2 = 0, tc3 = 0;
  while (kw < nbe - 1 && k < nc) {
    if (cyc && tid == 0) tc0 = clock64();
    par ^= 1;
    // F[r, k + 1] for the next step, valid unless this step interchanges
    // rows or delays the candidate
    T nxt[RPT];
    load_col(k + 1, nxt);
    // --- candidate column k: W[:, kw] = F[:, k] - L_panel W[k, :]^T
    T acc[RPT];
#pragma unroll
    for (int i = 0; i < RPT; i++) {
      acc[i] = cur[i];
      on[i] = kstart + rr[i] >= k && kstart + rr[i] < n;
    }
    const int krow = k - kstart;
    sw_apply_panel<T, PT, RPT>(Ws, cld, kw, krow, c, rr, on, acc);
    double bv = -1.0, tv = 0.0;
    int bi = 0x7fffffff;
    T* wcol = Ws + (size_t)kw * cld;
#pragma unroll
    for (int i = 0; i < RPT; i++)
      if (on[i]) {
        const int r = kstart + rr[i];
        wcol[rr[i]] = acc[i];
        const double a = fabs((double)acc[i]);
        if (r == k) c.wkk[par] = (double)acc[i];
        else if (r < nc) argmax_merge(bv, bi, a, r);
        else tv = fmax(tv, a);
      }
    if (cyc && tid == 0) tc1 = clock64();
    sw_reduce<PT>(c, 2 * par, bv, bi, tv);
    if (cyc && tid == 0) tc2 = clock64();
    int imax = bi;
    if (imax >= nc || imax <= k) {
      if (k + 1 < nc && tid == 0) atomicOr(status, ST_NAN);
      imax = (k + 1 < n) ? k + 1 : k;
    }
    const double wkk = c.wkk[par];
    const PivotChoice pc = choose_pivot(
        root, k, nc, wkk, imax, bv < 0.0 ? 0.0 : bv, tv, ustab, pivot_tol, [&]() {
          // column imax: F[imax, r] for r < imax, F[r, imax] below, minus
          // the panel's update with W row imax, into W[:, kw + 1]
          const double wik = (double)wcol[imax - kstart];
          T a2[RPT];
#pragma unroll
          for (int i = 0; i < RPT; i++) {
            const int r = kstart + rr[i];
            a2[i] = !on[i] ? T(0)
                           : (r < imax ? F[imax + (size_t)r * ld] : F[r + (size_t)imax * ld]);
          }
          sw_apply_panel<T, PT, RPT>(Ws, cld, kw, imax - kstart, c, rr, on, a2);
          double rv = -1.0, rt = 0.0;
          int ri = 0x7fffffff;
          T* w2 = Ws + (size_t)(kw + 1) * cld;
#pragma unroll
          for (int i = 0; i < RPT; i++)
            if (on[i]) {
              const int r = kstart + rr[i];
              w2[rr[i]] = a2[i];
              if (r == imax) c.wii = (double)a2[i];
              else rt = fmax(rt, fabs((double)a2[i]));
            }
          sw_reduce<PT>(c, 2 * par + 1, rv, ri, rt);
          return ImaxColumn{rt, c.wii, wik};
        });
    // every thread holds its decision inputs: the writes below may follow
    if (cyc && tid == 0) {
      tc3 = clock64();
      atomicAdd(cyc + 0, (unsigned long long)(tc1 - tc0));
      atomicAdd(cyc + 1, (unsigned long long)(tc2 - tc1));
      atomicAdd(cyc + 2, (unsigned long long)(tc3 - tc2));
    }
    if (pc.step == 0) {
      if (dbg && tid == 0) atomicAdd(dbg + 4, 1);
      // delay candidate k: move it to the end of the candidate set (both
      // positions stay live: the full interchange, after the pending ones)
      if (k < nc - 1) {
        sw_flush_left<T, PT>(F, ld, kstart, c);
        symm_swap<T, PT>(F, ld, n, vars, fsperm, k, nc - 1);
        sw_swap_rows<T, PT>(Ws, cld, kw, krow, nc - 1 - kstart);
        __syncthreads();
      }
      nc -= 1;
      load_col(k, cur);
      continue;
    }
    const int step = pc.step, kpiv = pc.kpiv;
    const int ksrc = k + step - 1;
    bool swapped = false;
    if (dbg && tid == 0)
      atomicAdd(dbg + (step == 1 ? (pc.imax_1x1 ? 1 : 0) : (kpiv != ksrc ? 3 : 2)), 1);
    if (pc.imax_1x1) {
      // column imax is the pivot column: its W column replaces column k's
      // (own rows; the imax build's reduction already separated every read
      // of W from these writes)
      T* w2 = Ws + (size_t)(kw + 1) * cld;
#pragma unroll
      for (int i = 0; i < RPT; i++)
        if (on[i]) wcol[rr[i]] = w2[rr[i]];
    }
    if (kpiv != ksrc) {
      // the global interchange from column ksrc's values (cur for a 1x1 at
      // k, nxt for the second column of a 2x2)
      if (step == 1) sw_pivot_swap<T, PT, RPT>(F, ld, n, kstart, ksrc, kpiv, rr, on, cur,
                                               vars, fsperm, c);
      else sw_pivot_swap<T, PT, RPT>(F, ld, n, kstart, ksrc, kpiv, rr, on, nxt,
                                     vars, fsperm, c);
      __syncthreads();   // the W copy above, before the W row interchange
      sw_swap_rows<T, PT>(Ws, cld, kw + step, ksrc - kstart, kpiv - kstart);
      swapped = true;
    }
    if (swapped || step == 2 || pc.imax_1x1) __syncthreads();
    if (step == 1 && !swapped) {
      // the common step: every thread sets the column's coefficients (the
      // same value), so the next step needs no barrier before reading them
      const T d = Ws[(size_t)kw * cld + krow];
      if (!isfinite((double)d) && tid == 0) atomicOr(status, ST_NAN);
      c.kind[kw] = 0;
      c.cA[kw] = pc.zero ? 0.0 : (double)(T(1) / d);
      c.cB[kw] = 0.0;
      c.cP[kw] = kw;
      if (tid == 0) vars[3 * ld + k] = 0;
    } else if (tid == 0) {
      if (step == 1) {
        const T d = Ws[(size_t)kw * cld + krow];
        if (!isfinite((double)d)) atomicOr(status, ST_NAN);
        c.kind[kw] = 0;
        c.cA[kw] = pc.zero ? 0.0 : (double)(T(1) / d);
        c.cB[kw] = 0.0;
        c.cP[kw] = kw;
        vars[3 * ld + k] = 0;
      } else {
        const Coef2 q = pivot2_coeffs<T>(Ws[(size_t)kw * cld + krow],
                                         Ws[(size_t)kw * cld + krow + 1],
                                         Ws[(size_t)(kw + 1) * cld + krow + 1]);
        if (!q.finite) atomicOr(status, ST_NAN);
        c.kind[kw] = 1;
        c.kind[kw + 1] = 2;
        c.cA[kw] = q.i00;
        c.cB[kw] = q.i10;
        c.cA[kw + 1] = q.i11;
        c.cB[kw + 1] = q.i01;
        c.cP[kw] = kw + 1;
        c.cP[kw + 1] = kw;
        vars[k] = -(vars[k] + 1);
        vars[k + 1] = -(vars[k + 1] + 1);
        vars[3 * ld + k] = 1;
        vars[3 * ld + k + 1] = 2;
      }
    }
    if (swapped || step == 2) __syncthreads();
    k += step;
    kw += step;
    if (!swapped && step == 1) {
#pragma unroll
      for (int i = 0; i < RPT; i++) cur[i] = nxt[i];
    } else {
      load_col(k, cur);
    }
    if (cyc && tid == 0) atomicAdd(cyc + 3, (unsigned long long)(clock64() - tc3));
  }
  // --- the pending interchanges left of the panel; the panel's L columns
  // to F and its W rows below k to HBM
  if (cyc && tid == 0) tc0 = clock64();
  sw_flush_left<T, PT>(F, ld, kstart, c);
  for (int j = 0; j < kw; j++) {
    const int col = kstart + j;
    const int kd = c.kind[j];
    const T* w0 = Ws + (size_t)j * cld;
    T* Fc = F + (size_t)col * ld;
    const T* wp = Ws + (size_t)c.cP[j] * cld;
    const T a = T(c.cA[j]), b = T(c.cB[j]);
    if (kd == 0) {
      if (tid == 0) Fc[col] = w0[j];
      for (int r = col + 1 + tid; r < n; r += PT)
        Fc[r] = sw_l(w0[r - kstart], wp[r - kstart], a, b);
    } else {
      const int j0 = kd == 1 ? j : j - 1;
      const T* wa = Ws + (size_t)j0 * cld;
      const T* wb = wa + cld;
      const int c0 = kstart + j0;
      if (tid == 0) {
        if (kd == 1) {
          Fc[col] = wa[j0];
          Fc[col + 1] = wa[j0 + 1];
        } else {
          Fc[col] = wb[j0 + 1];
        }
      }
      for (int r = c0 + 2 + tid; r < n; r += PT)
        Fc[r] = sw_l(w0[r - kstart], wp[r - kstart], a, b);
    }
    for (int r = k + tid; r < n; r += PT) Wg[r + (size_t)j * ld] = w0[r - kstart];
  }
  if (cyc && tid == 0) atomicAdd(cyc + 4, (unsigned long long)(clock64() - tc0));
  k_ = k;
  nc_ = nc;
  kw_ = kw;
}

template <class T, int PT, int RPT>
__global__ void __launch_bounds__(PT)
k_big_panel_sw(DevicePlan d, const int* __restrict__ nodes, double ustab,
               double pivot_tol, int smem_bytes, int* dbg) {
  pdl_enter();
  __shared__ SwCtl<PT> c;
  __shared__ CtlT<PT> ctl;
  extern __shared__ double sw_raw[];
  if (big_skip(d)) return;
  const int node = nodes[blockIdx.x];
  int* st = d.pstate + 4 * node;
  int k = st[0], nc = st[1];
  if (k >= nc) {
    if (threadIdx.x == 0) st[3] = 0;
    return;
  }
  const int f = d.f[node];
  const int fs = d.ns[node] + d.ndin[node];
  T* F = reinterpret_cast<T*>(d.fpool) + d.foff[node];
  T* W = F + (size_t)f * f;
  int* fvars = d.ipool + d.ioff[node];
  const int kstart = k;
  int kw = 0;
  // the panel width depends on the front alone (not on the launch), so a
  // front is factored the same way alone and in a batch
  const long long cld = f - kstart;
  const long long fit = (long long)kSwSmemBytes / (cld * (long long)sizeof(T));
  const int nbe = (int)(fit < NB ? fit : NB);
  if (nbe >= 4 && cld <= (long long)PT * RPT &&
      (long long)nbe * cld * (long long)sizeof(T) <= smem_bytes) {
    long long tk0 = 0;
    if (dbg && threadIdx.x == 0) {
      atomicAdd(dbg + 5, 1);
      tk0 = clock64();
    }
    panel_factor_sw<T, PT, RPT>(F, f, W, f, fs == f, fvars, fvars + f, ustab,
                                pivot_tol, d.status, c, reinterpret_cast<T*>(sw_raw),
                                nbe, k, nc, kw, dbg);
    if (dbg && threadIdx.x == 0)
      atomicAdd(reinterpret_cast<unsigned long long*>(dbg + 8) + 5,
                (unsigned long long)(clock64() - tk0));
  } else {
    // front grown past what this launch's shared memory holds (delayed
    // pivots): the HBM-panel form
    panel_factor<T, PT>(F, f, W, f, f, fs == f, fvars, fvars + f, ustab,
                        pivot_tol, d.status, ctl, k, nc, kw);
  }
  if (threadIdx.x == 0) {
    st[0] = k;
    st[1] = nc;
    st[2] = kstart;
    st[3] = kw;
  }
}

// ---------------------------------------------------------------------------
// Cluster panel: the shared-W panel with the front's rows spread over a
// thread-block cluster of CS CTAs, for levels of a few large fronts (the
// top-of-tree chain of a 2D KKT is a sequence of single ~1,100-row fronts,
// which the one-CTA panel leaves to one SM).  The pivot rule, candidate
// order, interchanges and the arithmetic of every row are those of
// panel_factor_sw; what changes is where the rows live:
//   * rows are dealt to the CTAs in groups of 32 (relative row group g to
//     CTA g mod CS), so that every warp's global accesses stay coalesced
//     and the rows still live as k advances stay balanced over the CTAs;
//   * each CTA keeps the W entries of its own rows in its shared memory,
//     so a column build reads local shared memory only, plus the W row of
//     the column being built, which each warp reads once from the owning
//     CTA (distributed shared memory) and broadcasts by shuffles;
//   * a reduction stores each warp's partial into every CTA's copy of the
//     slots and one cluster barrier publishes them, so that every CTA takes
//     the same decision from the same values -- and so passes the same
//     sequence of cluster barriers;
//   * an interchange moves W rows between CTAs through distributed shared
//     memory; F entries another CTA may have written in the same launch are
//     read from L2.
// With the one-CTA panel's widths (width_rule 1) the results are the one-
// CTA panel's bit for bit; by default every panel takes NB columns.
constexpr int kClThreads = 256;
constexpr int kClRows = 2;
constexpr int kClCS = 8;
// Rows a cluster panel takes: up to its threads' rows, capped so that W
// and L of NB columns fit in a CTA's shared memory.
constexpr int kClMaxRows = 3072;
constexpr int kClSlack = 64;
// Global-scratch cluster panel (GL): rows per thread; clusters of 8 take
// fronts to 8 x 256 x 8 rows, of 16 to twice that.
constexpr int kClRowsG = 8;
constexpr int kClMaxRowsG8 = kClThreads * kClRowsG * 8;
constexpr int kClMaxRowsG16 = kClThreads * kClRowsG * 16;
constexpr int kClSmemMax = 2 * NB * (kClMaxRows / kClCS) * 8;
static_assert(kClMaxRows <= kClThreads * kClRows * kClCS, "cluster panel rows");

template <int PT, int CS>
struct ClCtl {
  static constexpr int NS = CS * (PT / 32);  // warps of the cluster
  double rv[4][NS];   // reduction slots by step parity and kind, as SwCtl
  int ri[4][NS];
  double rv2[4][NS];
  double wkk[2], wii[2], wik[2];  // from the owners of rows k and imax
  double cA[NB], cB[NB];
  int cP[NB], kind[NB];
  int swa[NB], swb[NB], nsw;
  int rows[2 * NB], src[2 * NB], nrows;
  double xw[2][NB], xl[2][NB];  // W and L rows received in an interchange
  double ys[PT / 32][32];       // each warp's copy of the W row being applied
  int u[4];                     // launch-uniform values published by CTA 0
};

template <int CS>
__device__ __forceinline__ int cl_owner(int q) { return (q >> 5) % CS; }
template <int CS>
__device__ __forceinline__ int cl_lrow(int q) { return (((q >> 5) / CS) << 5) | (q & 31); }

// Warp fold of (v, i) -- the first argmax of v >= 0 (v < 0: no entry, index
// 0x7fffffff) -- and of the maximum of v2 >= 0, with warp reductions on the
// doubles' bit patterns (for non-negative doubles their order): high word,
// then low word among the lanes holding the maximal high word, then the
// smallest index among the maximal keys.  argmax_merge's result, exactly,
// and the same in every lane.
__device__ __forceinline__ void warp_fold_redux(double& v, int& i, double& v2) {
  const unsigned FULL = 0xffffffffu;
  const unsigned long long kv =
      v < 0.0 ? 0ull : (unsigned long long)__double_as_longlong(v);
  const unsigned hi = (unsigned)(kv >> 32), lo = (unsigned)kv;
  const unsigned mh = __reduce_max_sync(FULL, hi);
  const unsigned ml = __reduce_max_sync(FULL, hi == mh ? lo : 0u);
  const unsigned mi =
      __reduce_min_sync(FULL, (hi == mh && lo == ml) ? (unsigned)i : 0xffffffffu);
  i = (int)mi;
  v = mi == 0x7fffffffu
          ? -1.0
          : __longlong_as_double((long long)(((unsigned long long)mh << 32) | ml));
  const unsigned long long k2 = (unsigned long long)__double_as_longlong(v2);
  const unsigned h2 = (unsigned)(k2 >> 32), l2 = (unsigned)k2;
  const unsigned m2h = __reduce_max_sync(FULL, h2);
  const unsigned m2l = __reduce_max_sync(FULL, h2 == m2h ? l2 : 0u);
  v2 = __longlong_as_double((long long)(((unsigned long long)m2h << 32) | m2l));
}

// Block-wide reductions of sw_reduce over the whole cluster: every warp's
// fold goes into every CTA's copy of the slots (distributed shared memory
// stores), one cluster barrier, every warp folds the slots.  (ts: trace
// only, the clock after the warp fold, the barrier and the final fold.)
template <int PT, int CS, class Cl>
__device__ __forceinline__ void cl_reduce(ClCtl<PT, CS>& c, Cl& cluster, int set,
                                          double& v, int& i, double& v2,
                                          long long* ts = nullptr) {
  warp_fold_redux(v, i, v2);
  if (ts) ts[0] = clock64() + (v != v ? 1 : 0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = (int)cluster.block_rank() * (PT / 32) + warp;
  if (lane < CS) {
    ClCtl<PT, CS>* dst = cluster.map_shared_rank(&c, lane);
    dst->rv[set][slot] = v;
    dst->ri[set][slot] = i;
    dst->rv2[set][slot] = v2;
  }
  cluster.sync();
  if (ts) ts[1] = clock64();
  constexpr int NS = ClCtl<PT, CS>::NS;
  static_assert(NS <= 128, "cluster warps");
  v = lane < NS ? c.rv[set][lane] : -1.0;
  i = lane < NS ? c.ri[set][lane] : 0x7fffffff;
  v2 = lane < NS ? c.rv2[set][lane] : 0.0;
#pragma unroll
  for (int q = lane + 32; q < NS; q += 32) {
    argmax_merge(v, i, c.rv[set][q], c.ri[set][q]);
    v2 = fmax(v2, c.rv2[set][q]);
  }
  warp_fold_redux(v, i, v2);
  if (ts) ts[2] = clock64() + (v != v ? 1 : 0);
}

// *slot = v in every CTA of the cluster (one thread).
template <int CS, class Cl>
__device__ __forceinline__ void cl_bcast(Cl& cluster, double* slot, double v) {
#pragma unroll
  for (int r = 0; r < CS; r++) *cluster.map_shared_rank(slot, r) = v;
}

// W rows a and b (relative) interchanged over the columns [0, nw) and L
// rows over [0, nl): warp 0 of each row's CTA sends the row (a lane per
// column) to the other row's CTA, a cluster barrier, warp 0 stores what it
// received, a second barrier before any thread reads either row again
// (the barriers also publish the caller's F writes made before the call).
template <class T, int PT, int CS, class Cl>
__device__ void cl_swap_rows(T* Wl, T* Ll, int lld, int nw, int nl, int a, int b,
                             ClCtl<PT, CS>& c, Cl& cluster) {
  const int cr = (int)cluster.block_rank();
  const int lane = threadIdx.x & 31;
  const int oa = cl_owner<CS>(a), ob = cl_owner<CS>(b);
  const int la = cl_lrow<CS>(a), lb = cl_lrow<CS>(b);
  __syncthreads();  // this CTA's writes to rows a and b, before warp 0 reads
  if (threadIdx.x < 32) {
    if (cr == oa) {
      ClCtl<PT, CS>* dst = cluster.map_shared_rank(&c, ob);
      if (lane < nw) dst->xw[1][lane] = (double)Wl[(size_t)lane * lld + la];
      if (lane < nl) dst->xl[1][lane] = (double)Ll[(size_t)lane * lld + la];
    }
    if (cr == ob) {
      ClCtl<PT, CS>* dst = cluster.map_shared_rank(&c, oa);
      if (lane < nw) dst->xw[0][lane] = (double)Wl[(size_t)lane * lld + lb];
      if (lane < nl) dst->xl[0][lane] = (double)Ll[(size_t)lane * lld + lb];
    }
  }
  cluster.sync();
  if (threadIdx.x < 32) {
    if (cr == oa) {
      if (lane < nw) Wl[(size_t)lane * lld + la] = T(c.xw[0][lane]);
      if (lane < nl) Ll[(size_t)lane * lld + la] = T(c.xl[0][lane]);
    }
    if (cr == ob) {
      if (lane < nw) Wl[(size_t)lane * lld + lb] = T(c.xw[1][lane]);
      if (lane < nl) Ll[(size_t)lane * lld + lb] = T(c.xl[1][lane]);
    }
  }
  cluster.sync();
}

// The composed row map (rows[t] <- src[t], nr <= 64) applied to the
// variable list and the fully-summed permutation by one warp: loads before
// stores.
__device__ __forceinline__ void cl_map_vars(int* vars, int* fsperm, const int* rows,
                                            const int* src, int nr) {
  const int lane = threadIdx.x & 31;
  int v0 = 0, v1 = 0, p0 = 0, p1 = 0;
  if (lane < nr) {
    v0 = vars[src[lane]];
    p0 = fsperm[src[lane]];
  }
  if (lane + 32 < nr) {
    v1 = vars[src[lane + 32]];
    p1 = fsperm[src[lane + 32]];
  }
  __syncwarp();
  if (lane < nr) {
    vars[rows[lane]] = v0;
    fsperm[rows[lane]] = p0;
  }
  if (lane + 32 < nr) {
    vars[rows[lane + 32]] = v1;
    fsperm[rows[lane + 32]] = p1;
  }
}

// (GL: the panel's W and L rows of each CTA in a global scratch region --
// CTA r's at Wcl + r * stride -- instead of its shared memory, for fronts
// past what shared memory holds; rows of other CTAs are read from L2.)
template <class T, int PT, int RPT, int CS, bool TR, bool GL, class Cl>
__device__ void panel_factor_cl(T* F, int ld, T* Wg, int n, bool root,
                                int* vars, int* fsperm, double ustab,
                                double pivot_tol, int* status, ClCtl<PT, CS>& c,
                                T* Wl, T* Ll, int lld, int nbe, int& k_, int& nc_,
                                int& kw_, int* dbg, Cl& cluster, const T* Wcl,
                                size_t stride) {
  constexpr int NW = PT / 32;
  const unsigned FULL = 0xffffffffu;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cr = (int)cluster.block_rank();
  const bool lead = cr == 0 && tid == 0;
  if (tid == 0) c.nsw = 0;
  int k = k_, nc = nc_, kw = 0;
  const int kstart = k;
  int rel[RPT], lr[RPT];  // owned rows: relative to kstart, and local
  bool on[RPT];
  T cur[RPT];
#pragma unroll
  for (int i = 0; i < RPT; i++) {
    lr[i] = 32 * (warp + NW * i) + lane;
    rel[i] = 32 * (CS * (warp + NW * i) + cr) + lane;
  }
  auto load_col = [&](int col, T (&dst)[RPT]) {
#pragma unroll
    for (int i = 0; i < RPT; i++) {
      const int r = kstart + rel[i];
      dst[i] = (r >= col && r < n) ? __ldcg(F + r + (size_t)col * ld) : T(0);
    }
  };
  // lanes j < ncol: W[q, j] (q relative), from the row's CTA
  auto wrow = [&](int q, int ncol) -> T {
    if constexpr (GL) {
      const T* p = Wcl + (size_t)cl_owner<CS>(q) * stride + cl_lrow<CS>(q);
      return lane < ncol ? __ldcg(p + (size_t)lane * lld) : T(0);
    } else {
      const T* p = cluster.map_shared_rank(Wl + cl_lrow<CS>(q), cl_owner<CS>(q));
      return lane < ncol ? p[(size_t)lane * lld] : T(0);
    }
  };
  long long ts[10];  // trace only: clocks of the phases of a step (lead)
  unsigned long long acc_t[16] = {};
  // (TR: the trace build, with the step counters and phase clocks)
  const bool tr = TR && dbg != nullptr && lead;
  // acc[i] -= sum_{j < kw} L[r_i, j] y_j (the order of sw_apply_panel), y_j
  // in lane j of yv; the L entries of 8 columns are loaded before their
  // multiply-adds
  // the rows in chunks of RC (the partial sums and the loaded L entries of
  // one chunk in registers); y from the warp's shared copy
  constexpr int RC = RPT < 2 ? RPT : 2;
  double* ys = c.ys[warp];
  auto apply = [&](T yv, T (&acc)[RPT]) {
    ys[lane] = (double)yv;
    __syncwarp();
#pragma unroll
    for (int i0 = 0; i0 < RPT; i0 += RC) {
      T sm4[RC][4];
#pragma unroll
      for (int i = 0; i < RC; i++)
#pragma unroll
        for (int q = 0; q < 4; q++) sm4[i][q] = T(0);
      bool any = false;
#pragma unroll
      for (int i = 0; i < RC; i++) any |= on[i0 + i];
      if (__any_sync(FULL, any)) {
        for (int j0 = 0; j0 < kw; j0 += 8) {
          T lv[RC][8];
#pragma unroll
          for (int u = 0; u < 8; u++)
#pragma unroll
            for (int i = 0; i < RC; i++)
              lv[i][u] = (on[i0 + i] && j0 + u < kw)
                             ? Ll[(size_t)(j0 + u) * lld + lr[i0 + i]] : T(0);
#pragma unroll
          for (int u = 0; u < 8; u++) {
            const T yj = T(ys[(j0 + u) & 31]);
            if (j0 + u < kw) {
#pragma unroll
              for (int i = 0; i < RC; i++)
                if (on[i0 + i]) sm4[i][u & 3] += lv[i][u] * yj;
            }
          }
        }
      }
#pragma unroll
      for (int i = 0; i < RC; i++)
        if (on[i0 + i]) acc[i0 + i] -= (sm4[i][0] + sm4[i][1]) + (sm4[i][2] + sm4[i][3]);
    }
    __syncwarp();
    if (tr) ts[2] = clock64() + (acc[0] != acc[0] ? 1 : 0);
  };
  load_col(k, cur);
  int par = 0;
  bool have_y = false;  // ynext holds the next candidate's W row
  T ynext = T(0);
  while (kw < nbe - 1 && k < nc) {
    if (tr) ts[0] = clock64();
    par ^= 1;
    T nxt[RPT];
    load_col(k + 1, nxt);
    T acc[RPT];
#pragma unroll
    for (int i = 0; i < RPT; i++) {
      const int r = kstart + rel[i];
      acc[i] = cur[i];
      on[i] = r >= k && r < n;
    }
    const T yv = have_y ? ynext : wrow(k - kstart, kw);
    if (tr) ts[1] = clock64() + (yv != yv ? 1 : 0);
    apply(yv, acc);
    double bv = -1.0, tv = 0.0;
    int bi = 0x7fffffff;
    T* wcol = Wl + (size_t)kw * lld;
#pragma unroll
    for (int i = 0; i < RPT; i++)
      if (on[i]) {
        const int r = kstart + rel[i];
        wcol[lr[i]] = acc[i];
        const double a = fabs((double)acc[i]);
        if (r == k) cl_bcast<CS>(cluster, &c.wkk[par], (double)acc[i]);
        else if (r < nc) argmax_merge(bv, bi, a, r);
        else tv = fmax(tv, a);
      }
    if (tr) ts[3] = clock64();
    long long tb[3];
    cl_reduce<PT, CS>(c, cluster, 2 * par, bv, bi, tv, tr ? tb : nullptr);
    // the next candidate's W row, in case this step takes a 1x1 pivot
    // without an interchange (its entry in column kw is published now)
    have_y = false;
    if (k + 1 < n) ynext = wrow(k + 1 - kstart, kw + 1);
    int imax = bi;
    if (imax >= nc || imax <= k) {
      if (k + 1 < nc && lead) atomicOr(status, ST_NAN);
      imax = (k + 1 < n) ? k + 1 : k;
    }
    // column imax (F[imax, r] left of it, F[r, imax] below), loaded before
    // the decision on whether the pivot test needs it
    T a2[RPT];
#pragma unroll
    for (int i = 0; i < RPT; i++) {
      const int r = kstart + rel[i];
      a2[i] = !on[i] ? T(0)
                     : (r < imax ? __ldcg(F + imax + (size_t)r * ld)
                                 : __ldcg(F + r + (size_t)imax * ld));
    }
    const double wkk = c.wkk[par];
    const T dinv = T(1) / T(wkk);  // the 1x1 pivot's, ahead of the decision
    long long tl[7];  // trace only: phases of the column-imax evaluation
    const PivotChoice pc = choose_pivot(
        root, k, nc, wkk, imax, bv < 0.0 ? 0.0 : bv, tv, ustab, pivot_tol, [&]() {
          // column imax into W[:, kw + 1]; its owner publishes its diagonal
          // and the candidate column's entry in row imax
          if (tr) tl[0] = clock64() + (a2[0] != a2[0] || a2[RPT - 1] != a2[RPT - 1] ? 1 : 0);
          apply(wrow(imax - kstart, kw), a2);
          if (tr) tl[1] = ts[2];
          double rv = -1.0, rt = 0.0;
          int ri = 0x7fffffff;
          T* w2 = Wl + (size_t)(kw + 1) * lld;
#pragma unroll
          for (int i = 0; i < RPT; i++)
            if (on[i]) {
              const int r = kstart + rel[i];
              w2[lr[i]] = a2[i];
              if (r == imax) {
                cl_bcast<CS>(cluster, &c.wii[par], (double)a2[i]);
                cl_bcast<CS>(cluster, &c.wik[par], (double)wcol[lr[i]]);
              } else {
                rt = fmax(rt, fabs((double)a2[i]));
              }
            }
          if (tr) tl[2] = clock64();
          cl_reduce<PT, CS>(c, cluster, 2 * par + 1, rv, ri, rt, tr ? tl + 3 : nullptr);
          return ImaxColumn{rt, c.wii[par], c.wik[par]};
        });
    if (tr) tl[6] = clock64();
    if (tr) {
      ts[4] = tb[0];
      ts[5] = tb[1];
      ts[6] = tb[2];
      ts[7] = clock64();
    }
    if (pc.step == 0) {
      if (tr) atomicAdd(dbg + 4, 1);
      // delay candidate k (the full interchange with nc - 1 after the
      // pending ones, by CTA 0; the W and L rows by their CTAs)
      if (k < nc - 1) {
        if (cr == 0) {
          __syncthreads();
          // every thread takes the count before thread 0 changes it
          const int nsw = c.nsw;
          if (nsw > 0) {
            if (tid == 0) compose_swaps(c);
            __syncthreads();
            apply_row_map<T, true>(F, ld, kstart, c.rows, c.src, c.nrows, warp, NW);
            if (warp == 0) cl_map_vars(vars, fsperm, c.rows, c.src, c.nrows);
          }
          __syncthreads();
          if (tid == 0) c.nsw = 0;
          symm_swap<T, PT, true>(F, ld, n, vars, fsperm, k, nc - 1);
        } else if (tid == 0) {
          c.nsw = 0;
        }
        cl_swap_rows<T, PT, CS>(Wl, Ll, lld, kw, kw, k - kstart, nc - 1 - kstart, c,
                                cluster);
      }
      nc -= 1;
      load_col(k, cur);
      continue;
    }
    const int step = pc.step, kpiv = pc.kpiv;
    const int ksrc = k + step - 1;
    const bool swapped = kpiv != ksrc;
    if (tr)
      atomicAdd(dbg + (step == 1 ? (pc.imax_1x1 ? 1 : 0) : (swapped ? 3 : 2)), 1);
    if (pc.imax_1x1) {
      // column imax is the pivot column (own rows)
      T* w2 = Wl + (size_t)(kw + 1) * lld;
#pragma unroll
      for (int i = 0; i < RPT; i++)
        if (on[i]) wcol[lr[i]] = w2[lr[i]];
    }
    if (swapped) {
      // the entries of the interchange that stay live, from the registers
      // of column ksrc (own rows); the record for the columns left of the
      // panel; the W and L rows by their CTAs
      const int a = ksrc, b = kpiv;
#pragma unroll
      for (int i = 0; i < RPT; i++) {
        if (!on[i]) continue;
        const int r = kstart + rel[i];
        const T v = step == 1 ? cur[i] : nxt[i];
        if (r > a && r < b) F[b + (size_t)r * ld] = v;
        else if (r > b) F[r + (size_t)b * ld] = v;
        else if (r == a) F[b + (size_t)b * ld] = v;
      }
      if (tid == 0) {
        c.swa[c.nsw] = a;
        c.swb[c.nsw] = b;
        c.nsw++;
      }
      // (the variable list and the fully-summed permutation follow the
      // recorded interchanges at the end of the panel)
      if (tr) ts[9] = clock64();
      cl_swap_rows<T, PT, CS>(Wl, Ll, lld, kw + step, kw, a - kstart, b - kstart, c,
                              cluster);
      if (tr) acc_t[14] += (unsigned long long)(clock64() - ts[9]);
    }
    // the pivot block after the interchange: W[k, kw] is the candidate's
    // diagonal (column imax's for an imax 1x1 pivot); for a 2x2 pivot
    // W[k + 1, kw] and W[k + 1, kw + 1] are the entry of row imax and the
    // diagonal of column imax.  The L columns of the pivot (own rows) from
    // their W columns, with the expression that writes them to F.
    if (step == 1) {
      const T d = pc.imax_1x1 ? T(c.wii[par]) : T(wkk);
      if (!isfinite((double)d) && lead) atomicOr(status, ST_NAN);
      const T ainv = pc.zero ? T(0) : (pc.imax_1x1 ? T(1) / d : dinv);
      c.kind[kw] = 0;
      c.cA[kw] = (double)ainv;
      c.cB[kw] = 0.0;
      c.cP[kw] = kw;
      T* lc = Ll + (size_t)kw * lld;
#pragma unroll
      for (int i = 0; i < RPT; i++)
        if (on[i]) lc[lr[i]] = sw_l(wcol[lr[i]], wcol[lr[i]], ainv, T(0));
    } else {
      const Coef2 q = pivot2_coeffs<T>(T(wkk), T(c.wik[par]), T(c.wii[par]));
      if (!q.finite && lead) atomicOr(status, ST_NAN);
      c.kind[kw] = 1;
      c.kind[kw + 1] = 2;
      c.cA[kw] = q.i00;
      c.cB[kw] = q.i10;
      c.cA[kw + 1] = q.i11;
      c.cB[kw + 1] = q.i01;
      c.cP[kw] = kw + 1;
      c.cP[kw + 1] = kw;
      const T* w0 = wcol;
      const T* w1 = wcol + lld;
      T* l0 = Ll + (size_t)kw * lld;
      T* l1 = l0 + lld;
#pragma unroll
      for (int i = 0; i < RPT; i++)
        if (on[i]) {
          l0[lr[i]] = sw_l(w0[lr[i]], w1[lr[i]], T(q.i00), T(q.i10));
          l1[lr[i]] = sw_l(w1[lr[i]], w0[lr[i]], T(q.i11), T(q.i01));
        }
    }
    const bool plain = step == 1 && !swapped;
    k += step;
    kw += step;
    if (plain) {
#pragma unroll
      for (int i = 0; i < RPT; i++) cur[i] = nxt[i];
      have_y = true;
    } else {
      load_col(k, cur);
    }
    if (tr) {
      // fine phases of the steps without an interchange or a second column
      // (y row, column build, W stores, warp fold, barrier, final fold,
      // decision, rest); then all other steps' cycles and count
      ts[8] = clock64() + (cur[0] != cur[0] ? 1 : 0);
      if (plain && !pc.imax_1x1) {
        for (int q = 0; q < 8; q++) acc_t[q] += (unsigned long long)(ts[q + 1] - ts[q]);
        acc_t[10] += 1;
      } else {
        acc_t[8] += (unsigned long long)(ts[8] - ts[0]);
        acc_t[9] += 1;
        if (step == 2) {
          // 2x2 steps: to the end of the first reduction, column imax's
          // loads, build, stores, reduction, and the rest (the interchange
          // separately in acc_t[14])
          acc_t[11] += (unsigned long long)(ts[6] - ts[0]);
          acc_t[12] += (unsigned long long)(tl[0] - ts[6]);
          acc_t[13] += (unsigned long long)(tl[1] - tl[0]);
          acc_t[15] += (unsigned long long)(tl[5] - tl[1]);
        }
      }
    }
  }
  // --- the pending interchanges left of the panel (every CTA composes the
  // same map; the cluster's warps share the columns); the panel's L columns
  // to F and its W rows below k to HBM, each CTA for its own rows
  long long tw = tr ? clock64() : 0;
  __syncthreads();
  // every thread takes the count before thread 0 composes the map
  const int nsw = c.nsw;
  if (nsw > 0) {
    if (tid == 0) compose_swaps(c);
    __syncthreads();
    apply_row_map<T, true>(F, ld, kstart, c.rows, c.src, c.nrows, cr * NW + warp, CS * NW);
  }
  // the panel's interchanges of the variable list and the fully-summed
  // permutation, then its pivot kinds (2x2 pivots' variables encoded
  // -(v + 1)), by warp 0 of CTA 0
  if (cr == 0 && warp == 0) {
    if (nsw > 0) cl_map_vars(vars, fsperm, c.rows, c.src, c.nrows);
    __syncwarp();
    if (lane < kw) {
      const int col = kstart + lane, kd = c.kind[lane];
      vars[3 * ld + col] = kd;
      if (kd != 0) vars[col] = -(vars[col] + 1);
    }
  }
  for (int j = 0; j < kw; j++) {
    const int col = kstart + j;
    const int kd = c.kind[j];
    const T* w0 = Wl + (size_t)j * lld;
    const T* l0 = Ll + (size_t)j * lld;
    T* Fc = F + (size_t)col * ld;
    T* Wc = Wg + (size_t)j * ld;
#pragma unroll
    for (int i = 0; i < RPT; i++) {
      const int r = kstart + rel[i];
      if (r < col || r >= n) continue;
      const T w = w0[lr[i]];
      // the pivot block's own entries are D; below it, L
      if (r == col || (kd == 1 && r == col + 1)) Fc[r] = w;
      else Fc[r] = l0[lr[i]];
      if (r >= k) Wc[r] = w;
    }
  }
  if (tr) {
    unsigned long long* fine = reinterpret_cast<unsigned long long*>(dbg + 32);
    for (int q = 0; q < 16; q++) atomicAdd(fine + q, acc_t[q]);
    atomicAdd(reinterpret_cast<unsigned long long*>(dbg + 8) + 4,
              (unsigned long long)(clock64() - tw));
  }
  k_ = k;
  nc_ = nc;
  kw_ = kw;
}

// W local rows of a CTA for a panel of cld rows: the CTA's share of the
// 32-row groups.
template <int CS>
__host__ __device__ __forceinline__ int cl_local_rows(int cld) {
  return 32 * (((cld + 31) / 32 + CS - 1) / CS);
}

template <class T, int PT, int RPT, int CS, bool TR, bool GL>
__global__ void __launch_bounds__(PT, 1)
k_big_panel_cl(DevicePlan d, const int* __restrict__ nodes, double ustab,
               double pivot_tol, int smem_bytes, int width_rule, int fit_rows,
               int* dbg, T* scratch, long long stride) {
  pdl_enter();
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  __shared__ ClCtl<PT, CS> c;
  __shared__ CtlT<PT> ctl;
  extern __shared__ double cl_raw[];
  const int cr = (int)cluster.block_rank();
  const int node = nodes[blockIdx.x / CS];
  int* st = d.pstate + 4 * node;
  // every CTA of the cluster has started before any distributed shared
  // memory access; CTA 0 then publishes the values that steer the launch
  cluster.sync();
  if (cr == 0 && threadIdx.x == 0) {
    const int u0 = big_skip(d) ? 1 : 0, u1 = st[0], u2 = st[1];
    for (int r = 0; r < CS; r++) {
      ClCtl<PT, CS>* dst = cluster.map_shared_rank(&c, r);
      dst->u[0] = u0;
      dst->u[1] = u1;
      dst->u[2] = u2;
    }
  }
  cluster.sync();
  if (c.u[0]) return;
  int k = c.u[1], nc = c.u[2];
  if (k >= nc) {
    if (cr == 0 && threadIdx.x == 0) st[3] = 0;
    return;
  }
  const int f = d.f[node];
  const int fs = d.ns[node] + d.ndin[node];
  T* F = reinterpret_cast<T*>(d.fpool) + d.foff[node];
  T* W = F + (size_t)f * f;
  int* fvars = d.ipool + d.ioff[node];
  const int kstart = k;
  int kw = 0;
  const int cld = f - kstart;
  const int lld = cl_local_rows<CS>(cld);
  // the panel width depends on the front alone: NB, or the one-CTA
  // panel's (width_rule 1)
  int nbe = NB;
  int max_rows = GL ? CS * PT * RPT : kClMaxRows;
  if (width_rule == 1) {
    // the one-CTA panel's widths and its row limit (beyond which it takes
    // the HBM-panel form, as below)
    const long long fit = (long long)kSwSmemBytes / ((long long)cld * (long long)sizeof(T));
    nbe = (int)(fit < NB ? fit : NB);
    max_rows = kSwThreads * kSwRows;
  }
  // full-width panels: fronts of up to fit_rows rows (the level's largest
  // static front plus the slack its W and L rows were sized for, whatever
  // the cluster size); the one-CTA widths: as long as W and L fit
  const bool fits = width_rule == 0
                        ? cld <= fit_rows
                        : 2ll * nbe * lld * (long long)sizeof(T) <= smem_bytes;
  if (nbe >= 4 && cld <= max_rows && fits) {
    long long tk0 = 0;
    if (TR && dbg && cr == 0 && threadIdx.x == 0) {
      atomicAdd(dbg + 5, 1);
      tk0 = clock64();
    }
    T* Wcl = GL ? scratch + (size_t)(blockIdx.x / CS) * CS * (size_t)stride : nullptr;
    T* Wl = GL ? Wcl + (size_t)cr * (size_t)stride : reinterpret_cast<T*>(cl_raw);
    panel_factor_cl<T, PT, RPT, CS, TR, GL>(F, f, W, f, fs == f, fvars, fvars + f, ustab,
                                            pivot_tol, d.status, c, Wl,
                                            Wl + (size_t)nbe * lld, lld, nbe, k, nc, kw,
                                            dbg, cluster, Wcl, (size_t)stride);
    if (TR && dbg && cr == 0 && threadIdx.x == 0)
      atomicAdd(reinterpret_cast<unsigned long long*>(dbg + 8) + 5,
                (unsigned long long)(clock64() - tk0));
    // no CTA leaves while another may still read its shared memory
    cluster.sync();
  } else {
    // a front grown past the launch's shared memory (delayed pivots): the
    // HBM-panel form on CTA 0 (no distributed shared memory is used)
    if (cr != 0) return;
    panel_factor<T, PT>(F, f, W, f, f, fs == f, fvars, fvars + f, ustab,
                        pivot_tol, d.status, ctl, k, nc, kw);
  }
  if (cr == 0 && threadIdx.x == 0) {
    st[0] = k;
    st[1] = nc;
    st[2] = kstart;
    st[3] = kw;
  }
}

template <class T>
__global__ void __launch_bounds__(NT, 2)
k_big_update(DevicePlan d, const int* __restrict__ nodes) {
  pdl_enter();
  extern __shared__ double tiles_raw[];
  T* tiles = reinterpret_cast<T*>(tiles_raw);
  if (big_skip(d)) return;
  const int node = nodes[blockIdx.x];
  const int* st = d.pstate + 4 * node;
  const int k = st[0], kstart = st[2], kw = st[3];
  if (kw == 0) return;
  const int f = d.f[node];
  const int m = f - k;
  if (m <= 0) return;
  T* F = reinterpret_cast<T*>(d.fpool) + d.foff[node];
  const T* W = F + (size_t)f * f;
  const int nt = (m + kTile - 1) / kTile;
  const int ntiles = nt * (nt + 1) / 2;
  if constexpr (sizeof(T) == 8) {
    // a contiguous run of tiles per CTA (column-major), so that B is
    // staged once per column
    const int per = (ntiles + (int)gridDim.y - 1) / (int)gridDim.y;
    const int tb = (int)blockIdx.y * per;
    update_tiles_dmma(F, f, W, f, f, k, kstart, kw, nt, tb, min(ntiles, tb + per), tiles);
  } else {
    for (int t = blockIdx.y; t < ntiles; t += gridDim.y) {
      int ti, tj;
      tile_coords(t, ti, tj);
      update_tile(F, f, W, f, f, k, kstart, kw, ti, tj, tiles, tiles + kTile * TP);
    }
  }
}

// The same update for FP32 fronts on the tensor cores (tc_update.cuh):
// 128 x 128 tiles of the trailing block, 3xTF32 products in TMEM.
__global__ void __launch_bounds__(tc::kThreads)
k_big_update_tc(DevicePlan d, const int* __restrict__ nodes) {
  extern __shared__ __align__(1024) char tc_smem[];
  if (big_skip(d)) return;
  const int node = nodes[blockIdx.x];
  const int* st = d.pstate + 4 * node;
  const int k = st[0], kstart = st[2], kw = st[3];
  if (kw == 0) return;
  const int f = d.f[node];
  const int m = f - k;
  if (m <= 0) return;
  const int nt = (m + tc::TM - 1) / tc::TM;
  const int ntiles = nt * (nt + 1) / 2;
  if ((int)blockIdx.y >= ntiles) return;
  float* F = reinterpret_cast<float*>(d.fpool) + d.foff[node];
  const float* W = F + (size_t)f * f;
  tc::TcCta c = tc::tc_begin(tc_smem);
  for (int t = blockIdx.y; t < ntiles && c.ok; t += gridDim.y) {
    int ti, tj;
    tile_coords(t, ti, tj);
    tc::tc_tile(c, F + k + (size_t)k * f, f, F + k + (size_t)kstart * f, f,
                W + k, f, m, kw, ti * tc::TM, tj * tc::TN, d.status);
  }
  tc::tc_end(c);
}

template <class T>
__global__ void __launch_bounds__(NT)
k_big_finalize(DevicePlan d, const int* __restrict__ nodes) {
  if (big_skip(d)) return;
  const int node = nodes[blockIdx.x];
  const int f = d.f[node];
  const int fs = d.ns[node] + d.ndin[node];
  const int npiv = d.pstate[4 * node + 1];
  finish_front(d, node, reinterpret_cast<const T*>(d.fpool) + d.foff[node], f,
               fs, npiv, d.ipool + d.ioff[node]);
}

// Number of large fronts of the level still holding candidates; 0 when a
// pool ran out (the fronts stopped and the host grows the pool and
// restarts the factorization).
__global__ void k_big_remaining(DevicePlan d, const int* __restrict__ nodes,
                                int count, int* out) {
  int r = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    const int* st = d.pstate + 4 * nodes[i];
    r += st[0] < st[1] ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  if (threadIdx.x == 0) *out = big_skip(d) ? 0 : r;
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

// Streaming multiprocessors of the current device.
static int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    n = v;
  }
  return n;
}

// Whether clusters of 16 CTAs of the global-scratch panel can be scheduled
// on this device (set once, with the kernels' attributes).
template <class T>
static bool& cl16_ok() {
  static bool ok = false;
  return ok;
}

// One cluster of CS CTAs per front (cudaLaunchKernelEx with a cluster
// dimension).
template <class T, int RPT = kClRows, int CS = kClCS, bool GL = false>
static int launch_panel_cl(int fronts, int smem, cudaStream_t s, const DevicePlan& d,
                           const int* nodes, double ustab, double pivot_tol,
                           int width_rule, int fit_rows, int* dbg, T* scratch = nullptr,
                           long long stride = 0) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(fronts * CS);
  cfg.blockDim = dim3(kClThreads);
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
  if (dbg)
    FCUDA(cudaLaunchKernelEx(&cfg, k_big_panel_cl<T, kClThreads, RPT, CS, true, GL>, d,
                             nodes, ustab, pivot_tol, smem, width_rule, fit_rows, dbg,
                             scratch, stride));
  else
    FCUDA(cudaLaunchKernelEx(&cfg, k_big_panel_cl<T, kClThreads, RPT, CS, false, GL>, d,
                             nodes, ustab, pivot_tol, smem, width_rule, fit_rows,
                             (int*)nullptr, scratch, stride));
  return 0;
}

template <class T>
static int launch_factor(LdlHandle& h, const double* d_vals, cudaStream_t s) {
  DevicePlan& d = h.d;
  static bool attr_set = false;
  if (!attr_set) {
    FCUDA(cudaFuncSetAttribute(k_factor_level_rl<T, 256>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kMaxDynSmem));
    FCUDA(cudaFuncSetAttribute(k_big_update<T>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (sizeof(T) == 8 ? kUpdSmemD : kTileSmem) * sizeof(T)));
    FCUDA(cudaFuncSetAttribute(k_big_panel<T, kPanelThreads>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kPanelCacheBytes));
    FCUDA(cudaFuncSetAttribute(k_big_panel<T, kPanelThreadsWide>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kPanelCacheBytes));
    FCUDA(cudaFuncSetAttribute(k_big_panel_sw<T, kSwThreads, kSwRows>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kSwSmemBytes));
    FCUDA(cudaFuncSetAttribute(k_big_update_tc,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               tc::kSmemBytes));
    FCUDA(cudaFuncSetAttribute(k_big_panel_cl<T, kClThreads, kClRows, kClCS, false, false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kClSmemMax));
    FCUDA(cudaFuncSetAttribute(k_big_panel_cl<T, kClThreads, kClRows, kClCS, true, false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kClSmemMax));
    // the global-scratch cluster panel for the largest fronts: clusters of
    // 16 CTAs (a non-portable size) where the device schedules them
    FCUDA(cudaFuncSetAttribute(k_big_panel_cl<T, kClThreads, kClRowsG, 16, false, true>,
                               cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    FCUDA(cudaFuncSetAttribute(k_big_panel_cl<T, kClThreads, kClRowsG, 16, true, true>,
                               cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    {
      cudaLaunchConfig_t q = {};
      q.gridDim = dim3(16);
      q.blockDim = dim3(kClThreads);
      q.dynamicSmemBytes = 0;
      cudaLaunchAttribute a[1];
      a[0].id = cudaLaunchAttributeClusterDimension;
      a[0].val.clusterDim.x = 16;
      a[0].val.clusterDim.y = 1;
      a[0].val.clusterDim.z = 1;
      q.attrs = a;
      q.numAttrs = 1;
      int nclu = 0;
      if (cudaOccupancyMaxActiveClusters(
              &nclu, k_big_panel_cl<T, kClThreads, kClRowsG, 16, false, true>, &q) !=
          cudaSuccess)
        nclu = 0;
      cudaGetLastError();
      cl16_ok<T>() = nclu > 0;
    }
    attr_set = true;
  }
  FCUDA(cudaMemsetAsync(d.counters, 0, 2 * sizeof(unsigned long long), s));
  FCUDA(cudaMemsetAsync(d.inertia, 0, 2 * sizeof(int) * d.nprob, s));
  FCUDA(cudaMemsetAsync(d.status, 0, sizeof(int), s));
  // AMIGO_B200_TRACE=1 prints the device time of every level's small- and
  // large-front phases to stderr (diagnostics only).
  static const bool trace = std::getenv("AMIGO_B200_TRACE") != nullptr;
  std::vector<cudaEvent_t> ev;
  // trace only: per level, counts of the shared-W panel's steps (fast 1x1,
  // imax 1x1, 2x2 in place, 2x2 with interchange, delay, panels)
  int* dbg = nullptr;
  std::vector<int> dbg_h;
  std::vector<float> tpan(d.num_levels, 0.f), tupd(d.num_levels, 0.f);
  cudaEvent_t te[3];
  if (trace)
    for (auto& e : te) cudaEventCreate(&e);
  if (trace) {
    ev.resize(3 * d.num_levels);
    for (auto& e : ev) cudaEventCreate(&e);
    cudaMalloc((void**)&dbg, 64 * sizeof(int) * (size_t)d.num_levels);
    cudaMemsetAsync(dbg, 0, 64 * sizeof(int) * (size_t)d.num_levels, s);
    dbg_h.assign(64 * d.num_levels, 0);
  }
  for (int l = 0; l < d.num_levels; l++) {
    const LevelSchedule& L = h.sched[l];
    if (trace) cudaEventRecord(ev[3 * l], s);
    if (L.nsmall) {
      // front + 5 int sections, sized for a few delayed pivots more than
      // the static front; larger fronts run in the pools
      const long long fm = L.small_max_f + kRlSlack;
      long long bytes = ((fm * fm * (long long)sizeof(T) + 15) & ~15ll) + 5 * fm * 4;
      if (bytes > kMaxDynSmem) bytes = kMaxDynSmem;
      k_factor_level_rl<T, kRlThreads><<<L.nsmall, kRlThreads, (size_t)bytes, s>>>(
          d, d.sched_nodes + L.small_begin, L.nsmall, d_vals, h.ustab,
          h.pivot_tol, (int)bytes);
      ab::count_launch();
    }
    if (trace) cudaEventRecord(ev[3 * l + 1], s);
    if (L.nbig) {
      int* dbg_l = dbg ? dbg + 64 * l : nullptr;
      const int* nodes = d.sched_nodes + L.big_begin;
      const int B = L.nbig;
      const long long fm = L.big_max_f;
      int gz = (int)std::min<long long>(512, (fm * fm + 4095) / 4096);
      int ga = (int)std::min<long long>(256, (L.big_max_amap + NT - 1) / NT);
      int ge = (int)std::min<long long>(1024, fm);
      { k_big_setup<T><<<B, NT, 0, s>>>(d, nodes); ab::count_launch(); }
      { k_big_zero<T><<<dim3(B, std::max(gz, 1)), NT, 0, s>>>(d, nodes); ab::count_launch(); }
      { k_big_add_A<T><<<dim3(B, std::max(ga, 1)), NT, 0, s>>>(d, nodes, d_vals); ab::count_launch(); }
      for (int q = 0; q < L.big_max_kids; q++)
        { k_big_extend<T><<<dim3(B, std::max(ge, 1)), NT, 0, s>>>(d, nodes, q); ab::count_launch(); }
      const long long ntl = (fm + kTile - 1) / kTile;
      int gu = (int)std::min<long long>(4 * 148, ntl * (ntl + 1) / 2);
      // shared-memory copy of the panel's L columns: as many rows as fit
      const int panel_cache = (int)std::min<long long>(
          h.panel_cache_bytes, (long long)fm * NB * (long long)sizeof(T));
      // FP32 fronts of at least one 128-row tile: tensor-core update
      const bool use_tc = sizeof(T) == 4 && h.tensor_cores && fm >= tc::TM;
      const long long ntc = (fm + tc::TM - 1) / tc::TM;
      const int gtc = (int)std::max<long long>(
          1, std::min<long long>(3 * 148, ntc * (ntc + 1) / 2));
      // shared-W panel for levels whose fronts fit its rows; its shared
      // memory holds up to NB columns of W for the largest static front
      // (fronts grown by delayed pivots get fewer columns)
      // cluster panel for levels of large fronts (mode 0: full-width
      // panels; mode 2: the one-CTA panel's widths); its shared memory
      // holds NB columns of W for kClSlack rows more than the largest
      // static front
      const bool use_cl = (h.panel_mode == 0 || h.panel_mode == 2) && fm >= h.cl_min_rows &&
                          fm + kClSlack <= kClMaxRows;
      const int cl_rule = h.panel_mode == 2 ? 1 : 0;
      const int cl_smem =
          use_cl ? 2 * NB * cl_local_rows<kClCS>((int)fm + kClSlack) * (int)sizeof(T) : 0;
      // past shared memory: the cluster panel with its W and L rows in a
      // global scratch region (clusters of 8, or 16 for the largest fronts;
      // mode 3, a test mode: clusters of 16 on every level they can take,
      // bit-identical to mode 0)
      const long long gmax = cl16_ok<T>() ? kClMaxRowsG16 : kClMaxRowsG8;
      const bool force16 = h.panel_mode == 3 && cl16_ok<T>();
      const bool use_clg = ((h.panel_mode == 0 && !use_cl && fm + kClSlack > kClMaxRows) ||
                            force16) &&
                           fm >= h.cl_min_rows && fm + kClSlack <= gmax;
      const bool g16 = use_clg && (force16 || fm + kClSlack > kClMaxRowsG8);
      long long g_stride = 0;
      if (use_clg) {
        const int gcs = g16 ? 16 : 8;
        const long long glld = g16 ? cl_local_rows<16>((int)fm + kClSlack)
                                   : cl_local_rows<8>((int)fm + kClSlack);
        g_stride = 2ll * NB * glld;
        const size_t need = (size_t)B * gcs * (size_t)g_stride * sizeof(T);
        if (need > h.cl_scratch_bytes) {
          if (h.cl_scratch) FCUDA(cudaFree(h.cl_scratch));
          h.cl_scratch = nullptr;
          h.cl_scratch_bytes = 0;
          FCUDA(cudaMalloc(&h.cl_scratch, need));
          h.cl_scratch_bytes = need;
        }
      }
      const bool use_sw = !use_cl && !use_clg && fm <= (long long)kSwThreads * kSwRows;
      const int sw_smem = kSwSmemBytes;
      // panels a front of big_max_fs candidates needs without delays: each
      // takes nbe - 1 pivots, nbe growing as the remaining rows shrink
      int panels = 0;
      if (use_sw || (use_cl && cl_rule == 1)) {
        for (long long kk = 0; kk < L.big_max_fs; panels++) {
          const long long rows = std::max<long long>(fm - kk, 1);
          const long long nbe = std::min<long long>(
              NB, sw_smem / (rows * (long long)sizeof(T)));
          kk += std::max<long long>(nbe - 1, 1);
        }
        panels += 2;
      } else {
        panels = (int)((L.big_max_fs + NB - 2) / (NB - 1)) + 2;
      }
      // Every panel consumes at least one candidate of every unfinished
      // front, so no front needs more panels than it has rows.
      long long budget = 0;
      const long long max_panels = (long long)d.n + 8;
      for (;;) {
        budget += panels;
        for (int it = 0; it < panels; it++) {
          if (trace) cudaEventRecord(te[0], s);
          if (use_cl) {
            const int rc = launch_panel_cl<T>(B, cl_smem, s, d, nodes, h.ustab,
                                              h.pivot_tol, cl_rule, (int)fm + kClSlack,
                                              dbg_l);
            if (rc) return rc;
          } else if (use_clg) {
            T* scr = reinterpret_cast<T*>(h.cl_scratch);
            const int fr = (int)fm + kClSlack;
            const int rc =
                g16 ? launch_panel_cl<T, kClRowsG, 16, true>(B, 0, s, d, nodes, h.ustab,
                                                             h.pivot_tol, 0, fr, dbg_l, scr,
                                                             g_stride)
                    : launch_panel_cl<T, kClRowsG, 8, true>(B, 0, s, d, nodes, h.ustab,
                                                            h.pivot_tol, 0, fr, dbg_l, scr,
                                                            g_stride);
            if (rc) return rc;
          } else if (use_sw) {
            FCUDA(launch_pdl(k_big_panel_sw<T, kSwThreads, kSwRows>, dim3(B),
                             dim3(kSwThreads), (size_t)sw_smem, s, d, nodes, h.ustab,
                             h.pivot_tol, sw_smem, dbg_l));
          } else if (fm > kPanelWideRows) {
            FCUDA(launch_pdl(k_big_panel<T, kPanelThreadsWide>, dim3(B),
                             dim3(kPanelThreadsWide), (size_t)panel_cache, s, d, nodes,
                             h.ustab, h.pivot_tol, panel_cache));
          } else {
            FCUDA(launch_pdl(k_big_panel<T, kPanelThreads>, dim3(B), dim3(kPanelThreads),
                             (size_t)panel_cache, s, d, nodes, h.ustab, h.pivot_tol,
                             panel_cache));
          }
          ab::count_launch();
          if (trace) cudaEventRecord(te[1], s);
          if (use_tc) {
            { k_big_update_tc<<<dim3(B, gtc), tc::kThreads, tc::kSmemBytes, s>>>(
                d, nodes); ab::count_launch(); }
          } else {
            FCUDA(launch_pdl(k_big_update<T>, dim3(B, std::max(gu, 1)), dim3(NT),
                             (size_t)((sizeof(T) == 8 ? kUpdSmemD : kTileSmem) * sizeof(T)),
                             s, d, nodes));
            ab::count_launch();
          }
          if (trace) {
            cudaEventRecord(te[2], s);
            cudaEventSynchronize(te[2]);
            float a = 0.f, b = 0.f;
            cudaEventElapsedTime(&a, te[0], te[1]);
            cudaEventElapsedTime(&b, te[1], te[2]);
            tpan[l] += a;
            tupd[l] += b;
          }
        }
        // Delayed pivots received from the children can make a front need
        // more panels than its static size implies: check and continue.
        { k_big_remaining<<<1, 32, 0, s>>>(d, nodes, B, d.scratch_int); ab::count_launch(); }
        int left = 0;
        FCUDA(cudaMemcpyAsync(&left, d.scratch_int, sizeof(int),
                              cudaMemcpyDeviceToHost, s));
        FCUDA(cudaStreamSynchronize(s));
        if (left == 0) break;
        if (budget > max_panels) {
          std::fprintf(stderr, "amigo_b200: large-front panels did not finish\n");
          return -6;
        }
        panels = 4;
      }
      { k_big_finalize<T><<<B, NT, 0, s>>>(d, nodes); ab::count_launch(); }
    }
    if (trace) cudaEventRecord(ev[3 * l + 2], s);
  }
  if (trace) {
    cudaStreamSynchronize(s);
    cudaMemcpy(dbg_h.data(), dbg, 64 * sizeof(int) * (size_t)d.num_levels,
               cudaMemcpyDeviceToHost);
    cudaFree(dbg);
    float tot_s = 0.f, tot_b = 0.f;
    for (int l = 0; l < d.num_levels; l++) {
      float a = 0.f, b = 0.f;
      cudaEventElapsedTime(&a, ev[3 * l], ev[3 * l + 1]);
      cudaEventElapsedTime(&b, ev[3 * l + 1], ev[3 * l + 2]);
      tot_s += a;
      tot_b += b;
      std::fprintf(stderr,
                   "level %3d: small %5d (fmax %5d) %8.3f ms | large %4d "
                   "(fmax %5d) %8.3f ms\n",
                   l, h.sched[l].nsmall, h.sched[l].small_max_f, a,
                   h.sched[l].nbig, h.sched[l].big_max_f, b);
      const int* q = dbg_h.data() + 64 * l;
      const unsigned long long* cy = reinterpret_cast<const unsigned long long*>(q + 8);
      const unsigned long long* fi = reinterpret_cast<const unsigned long long*>(q + 32);
      if (!q[5] && (tpan[l] > 0.f || tupd[l] > 0.f))
        std::fprintf(stderr, "           panel launches %.3f ms update launches %.3f ms\n",
                     tpan[l], tupd[l]);
      if (q[5])
        std::fprintf(stderr, "           panel steps: fast %d imax %d 2x2 %d "
                             "2x2-swap %d delay %d panels %d | kcyc: build %llu "
                             "reduce %llu decide %llu post %llu wb %llu kernel %llu "
                             "| panel launches %.3f ms update launches %.3f ms\n",
                     q[0], q[1], q[2], q[3], q[4], q[5], cy[0] / 1000, cy[1] / 1000,
                     cy[2] / 1000, cy[3] / 1000, cy[4] / 1000, cy[5] / 1000,
                     tpan[l], tupd[l]);
      const unsigned long long nf = fi[10];
      if (fi[0] && nf)
        std::fprintf(stderr, "           plain-step cycles: yrow %llu build %llu stores %llu "
                             "fold %llu barrier %llu fold2 %llu decide %llu rest %llu | "
                             "other steps %llu cycles each (%llu)\n",
                     fi[0] / nf, fi[1] / nf, fi[2] / nf, fi[3] / nf, fi[4] / nf, fi[5] / nf,
                     fi[6] / nf, fi[7] / nf, fi[9] ? fi[8] / fi[9] : 0ull, fi[9]);
      const unsigned long long n2 = (unsigned long long)(q[2] + q[3]);
      const unsigned long long nsw = (unsigned long long)(q[1] + q[3]);
      if (fi[0] && n2)
        std::fprintf(stderr, "           2x2-step cycles: to first reduction %llu "
                             "imax loads %llu imax build %llu imax stores+reduce %llu | "
                             "interchange %llu per swap\n",
                     fi[11] / n2, fi[12] / n2, fi[13] / n2, fi[15] / n2,
                     nsw ? fi[14] / nsw : 0ull);
    }
    std::fprintf(stderr, "total: small %.3f ms, large %.3f ms\n", tot_s, tot_b);
    for (auto& e : ev) cudaEventDestroy(e);
  }
  FCUDA(cudaGetLastError());
  return 0;
}

int factor_numeric(LdlHandle& h, const double* d_vals, cudaStream_t s) {
  DevicePlan& d = h.d;
  for (int attempt = 0; attempt < 6; attempt++) {
    int rc = h.precision == 32 ? launch_factor<float>(h, d_vals, s)
                               : launch_factor<double>(h, d_vals, s);
    if (rc) return rc;
    int status = 0, solve_err = 0;
    FCUDA(cudaMemcpyAsync(&status, d.status, sizeof(int),
                          cudaMemcpyDeviceToHost, s));
    if (h.sv_err)
      FCUDA(cudaMemcpyAsync(&solve_err, h.sv_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    FCUDA(cudaStreamSynchronize(s));
    h.last_status = status;
    if (solve_err) {
      // a work-queue solve sweep since the last factorization gave up
      // waiting for a front (its result was wrong)
      std::fprintf(stderr, "amigo_b200: a solve sweep's dependency wait ran out\n");
      FCUDA(cudaMemsetAsync(h.sv_err, 0, sizeof(int), s));
      return AB_ERR_CUDA;
    }
    if (status & tc::kStatusTimeout) {
      std::fprintf(stderr, "amigo_b200: tensor-core update wait ran out\n");
      return AB_ERR_CUDA;
    }
    if (status & (ST_POOL_F | ST_POOL_I)) {
      // Delayed pivots made fronts larger than the pool allows: grow it.
      if (status & ST_POOL_F) {
        // double the pool, within what the device has free
        FCUDA(cudaFree(d.fpool));
        d.fpool = nullptr;
        size_t free_b = 0, total_b = 0;
        FCUDA(cudaMemGetInfo(&free_b, &total_b));
        const long long budget =
            ((long long)free_b - (long long)(total_b / 20)) / 8;
        const long long grown = std::min<long long>(2 * d.fcap, budget);
        if (grown <= d.fcap) {
          std::fprintf(stderr, "amigo_b200: delayed pivots need more than "
                               "the %.1f GB front pool\n", d.fcap * 8e-9);
          FCUDA(cudaMalloc((void**)&d.fpool, (size_t)d.fcap * sizeof(double)));
          return AB_ERR_CAPACITY;
        }
        d.fcap = grown;
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
    h.factor_epoch++;
    h.factor_precision = h.precision;
    return (status & ST_NAN) ? -5 : 0;
  }
  return -6;
}

}  // namespace ab

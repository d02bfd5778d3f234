// Kernels shared by every generated component module (amigo_b200.codegen).
//
// A generated module defines, per component group, an evaluator struct C
// (NQ variables, ND data entries, a straight-line `eval` calling
// out.grad(i, v) and out.hess(i, j, v) for j <= i, and `objective`) and
// expands AB_GEN_ENTRY_POINTS(C), which instantiates the kernels below:
//   * gradient: one thread per component instance of one colour (instances
//     of a colour share no variable, so the scatter g[idx] += dL/dq needs no
//     atomics and the sums are deterministic; colours are launched in turn
//     by the host, the role of the colour-serialised OpenMP backend,
//     include/component_group.h:432-528);
//   * Hessian: the same, scattering each entry of the lower triangle and
//     its mirror into the KKT CSR values through positions precomputed per
//     instance (the CUDA backend's position map, cuda/component_group_
//     backend.cuh:143-188);
//   * objective: per-instance values, summed on the device in a fixed
//     order.
// When compiled by a host compiler (the CPU tests), only `<C>_eval_host` is
// defined: the same evaluator on the host.
#pragma once
#include <cmath>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

#ifdef __CUDACC__
#include <cuda_runtime.h>

namespace abgen {

inline long long& launches() {
  static long long n = 0;
  return n;
}

// Local variable `kred` (or -1) is one global variable shared by every
// instance of the group (a global multiplier or slack): its gradient entry
// and Hessian diagonal go to a per-instance slot, summed afterwards in a
// fixed order, so instances of one colour never add to the same place.
template <class C>
struct DevGrad {
  static constexpr bool kHess = false;
  double* g;
  const int* ix;
  int kred;
  double* red;   // this instance's slot
  __device__ __forceinline__ void grad(int i, double v) {
    if (i == kred) *red = v;
    else g[ix[i]] += v;
  }
  __device__ __forceinline__ void hess(int, int, double) {}
};

template <class C>
struct DevHess {
  static constexpr bool kHess = true;
  double* vals;
  const int* pos;   // NQ x NQ CSR positions of this instance
  int kred;
  double* red;
  __device__ __forceinline__ void grad(int, double) {}
  __device__ __forceinline__ void hess(int i, int j, double v) {
    if (i == kred && j == kred) {
      *red = v;
      return;
    }
    vals[pos[i * C::NQ + j]] += v;
    if (i != j) vals[pos[j * C::NQ + i]] += v;
  }
};

template <class C>
__device__ __forceinline__ void gather(int e, const int* __restrict__ idx,
                                       const double* __restrict__ data,
                                       const double* __restrict__ x, double* q,
                                       double* d) {
  const int* ix = idx + (size_t)e * C::NQ;
#pragma unroll
  for (int i = 0; i < C::NQ; i++) q[i] = x[ix[i]];
#pragma unroll
  for (int i = 0; i < C::ND; i++) d[i] = data[(size_t)e * C::ND + i];
}

template <class C>
__global__ void k_gen_gradient(int ne, const int* __restrict__ elems,
                               const int* __restrict__ idx,
                               const double* __restrict__ data,
                               const double* __restrict__ x, double alpha,
                               double* __restrict__ g, int kred,
                               double* __restrict__ red) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ne;
       t += gridDim.x * blockDim.x) {
    const int e = elems ? elems[t] : t;
    double q[C::NQ], d[C::ND > 0 ? C::ND : 1];
    gather<C>(e, idx, data, x, q, d);
    DevGrad<C> o{g, idx + (size_t)e * C::NQ, kred, red + e};
    C::eval(q, d, alpha, o);
  }
}

template <class C>
__global__ void k_gen_hessian(int ne, const int* __restrict__ elems,
                              const int* __restrict__ idx,
                              const double* __restrict__ data,
                              const int* __restrict__ pos,
                              const double* __restrict__ x, double alpha,
                              double* __restrict__ vals, int kred,
                              double* __restrict__ red) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ne;
       t += gridDim.x * blockDim.x) {
    const int e = elems ? elems[t] : t;
    double q[C::NQ], d[C::ND > 0 ? C::ND : 1];
    gather<C>(e, idx, data, x, q, d);
    DevHess<C> o{vals, pos + (size_t)e * C::NQ * C::NQ, kred, red + e};
    C::eval(q, d, alpha, o);
  }
}

template <class C>
__global__ void k_gen_objective(int ne, const int* __restrict__ idx,
                                const double* __restrict__ data,
                                const double* __restrict__ x,
                                double* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne;
       e += gridDim.x * blockDim.x) {
    double q[C::NQ], d[C::ND > 0 ? C::ND : 1];
    gather<C>(e, idx, data, x, q, d);
    out[e] = C::objective(q, d);
  }
}

// Sum of n values by one 1024-thread block in a fixed order (strided
// per-thread sums, then a fixed tree): the same result on every run.
__global__ void k_gen_sum(int n, const double* __restrict__ in, double* out,
                          int accumulate) {
  __shared__ double s[1024];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += 1024) v += in[i];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int w = 512; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = accumulate ? *out + s[0] : s[0];
}

__global__ void k_gen_fill_at(int n, const int* __restrict__ pos, double v,
                              double* __restrict__ a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    a[pos[i]] = v;
}

inline int grid(long long n) {
  long long g = (n + 127) / 128;
  if (g > 148 * 16) g = 148 * 16;
  return g < 1 ? 1 : (int)g;
}

inline int status() { return cudaGetLastError() == cudaSuccess ? 0 : -2; }

}  // namespace abgen

extern "C" {
// Launches made by this module since it was loaded.
long long abgen_launch_count() { return abgen::launches(); }
// a[pos[i]] = v: the fixed-variable rows and columns of the KKT and the
// gradient (include/fixed_variables.h:56-72).
int abgen_fill_at(int n, const int* pos, double v, double* a, void* stream) {
  if (n <= 0) return 0;
  abgen::k_gen_fill_at<<<abgen::grid(n), 128, 0, (cudaStream_t)stream>>>(n, pos, v, a);
  abgen::launches()++;
  return abgen::status();
}
// *out = sum(in[0:n]) (accumulate: *out += sum), fixed order.
int abgen_sum(int n, const double* in, double* out, int accumulate,
              void* stream) {
  abgen::k_gen_sum<<<1, 1024, 0, (cudaStream_t)stream>>>(n, in, out, accumulate);
  abgen::launches()++;
  return abgen::status();
}
}

#define AB_GEN_ENTRY_POINTS(C)                                                 \
  extern "C" int C##_gradient(int ne, const int* elems, const int* idx,        \
                              const double* data, const double* x,             \
                              double alpha, double* g, int kred, double* red,  \
                              void* stream) {                                  \
    if (ne <= 0) return 0;                                                     \
    abgen::k_gen_gradient<C><<<abgen::grid(ne), 128, 0, (cudaStream_t)stream>>>( \
        ne, elems, idx, data, x, alpha, g, kred, red);                         \
    abgen::launches()++;                                                       \
    return abgen::status();                                                    \
  }                                                                            \
  extern "C" int C##_hessian(int ne, const int* elems, const int* idx,         \
                             const double* data, const int* pos,               \
                             const double* x, double alpha, double* vals,      \
                             int kred, double* red, void* stream) {            \
    if (ne <= 0) return 0;                                                     \
    abgen::k_gen_hessian<C><<<abgen::grid(ne), 128, 0, (cudaStream_t)stream>>>( \
        ne, elems, idx, data, pos, x, alpha, vals, kred, red);                 \
    abgen::launches()++;                                                       \
    return abgen::status();                                                    \
  }                                                                            \
  extern "C" int C##_objective(int ne, const int* idx, const double* data,     \
                               const double* x, double* out, void* stream) {   \
    if (ne <= 0) return 0;                                                     \
    abgen::k_gen_objective<C><<<abgen::grid(ne), 128, 0, (cudaStream_t)stream>>>( \
        ne, idx, data, x, out);                                                \
    abgen::launches()++;                                                       \
    return abgen::status();                                                    \
  }

#else  // host compiler: the evaluator on the host, for tests

namespace abgen {
template <int NQ>
struct HostOut {
  static constexpr bool kHess = true;
  double* g;
  double* h;   // NQ x NQ, both triangles
  void grad(int i, double v) { g[i] += v; }
  void hess(int i, int j, double v) {
    h[i * NQ + j] += v;
    if (i != j) h[j * NQ + i] += v;
  }
};
}  // namespace abgen

#define AB_GEN_ENTRY_POINTS(C)                                                 \
  extern "C" int C##_eval_host(const double* q, const double* d, double alpha, \
                               double* grad, double* hess, double* obj) {      \
    for (int i = 0; i < C::NQ; i++) grad[i] = 0.0;                             \
    for (int i = 0; i < C::NQ * C::NQ; i++) hess[i] = 0.0;                     \
    abgen::HostOut<C::NQ> o{grad, hess};                                       \
    C::eval(q, d, alpha, o);                                                   \
    *obj = C::objective(q, d);                                                 \
    return 0;                                                                  \
  }                                                                            \
  extern "C" int C##_sizes(int* nq, int* nd) {                                 \
    *nq = C::NQ;                                                               \
    *nd = C::ND;                                                               \
    return 0;                                                                  \
  }

#endif

// Post-optimality sensitivities of every instance of a group, on the host
// (dense per-instance blocks; see <C>_sens in the generated source):
// out[E x NO], dgd[E x NQ x ND], doq[E x NO x NQ], dod[E x NO x ND] at the
// global iterate x gathered through idx[E x NQ].
#define AB_GEN_SENS(C)                                                         \
  extern "C" int C##_sens_batch(int ne, const int* idx, const double* x,       \
                                const double* data, double alpha, double* out, \
                                double* dgd, double* doq, double* dod) {       \
    constexpr int NQ = C::NQ, ND = C::ND, NO = C##_sens::NO;                   \
    double q[NQ > 0 ? NQ : 1];                                                 \
    for (int e = 0; e < ne; e++) {                                             \
      for (int i = 0; i < NQ; i++) q[i] = x[idx[(long long)e * NQ + i]];       \
      C##_sens::eval(q, data + (long long)e * ND, alpha,                       \
                     out + (long long)e * NO, dgd + (long long)e * NQ * ND,    \
                     doq + (long long)e * NO * NQ, dod + (long long)e * NO * ND); \
    }                                                                          \
    return 0;                                                                  \
  }                                                                            \
  extern "C" int C##_sens_sizes(int* nq, int* nd, int* no) {                   \
    *nq = C::NQ;                                                               \
    *nd = C::ND;                                                               \
    *no = C##_sens::NO;                                                        \
    return 0;                                                                  \
  }


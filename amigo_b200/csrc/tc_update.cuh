// Schur-complement updates of FP32 fronts on the 5th-generation tensor
// cores (tcgen05, kind::tf32): lower(C) -= A * B^T for one rank-kw panel
// (kw <= 31), where A holds the panel's L columns and B their L*D columns.
//
// Every operand is split into a TF32 head and the TF32 of its remainder
// (a = hi + lo), and C is updated with hi*hi + hi*lo + lo*hi ("3xTF32"),
// accumulated in FP32 in tensor memory: the dropped lo*lo term is below
// FP32 resolution, so the update carries FP32 accuracy at tensor-core rate.
//
// One CTA of 128 threads owns a 128 x 128 accumulator in TMEM (128
// columns) and walks over lower-triangle tiles of the trailing block:
//   1. the 128 threads stage the A and B tiles (128 rows x 32 K, zero-padded)
//      as hi/lo pairs in shared memory in the K-major 128-byte-swizzled
//      layout the MMA descriptors describe;
//   2. one thread issues 3 x 4 tcgen05.mma (K = 8 each) and commits them to
//      an mbarrier;
//   3. while the MMAs run, every thread loads the first 32 entries of its
//      row of the C tile; after the (bounded) wait each warp reads its 32
//      TMEM lanes with tcgen05.ld chunk by chunk (the next chunk of C
//      already loading) and writes C - A B^T, lower triangle only.
// Descriptor encodings follow the sm_100 shared-memory and instruction
// descriptor formats (PTX ISA, tcgen05 "Matrix Descriptors" / "Instruction
// Descriptor"; the same fields as CUTLASS's UMMA::SmemDescriptor and
// UMMA::InstrDescriptor).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace ab {
namespace tc {

constexpr int TM = 128;                       // tile rows (MMA M)
constexpr int TN = 128;                       // tile columns (MMA N)
constexpr int TK = 32;                        // K of one panel, padded
constexpr int kTileBytes = TM * TK * 4;       // one 128 x 32 FP32 operand
constexpr int kSmemBytes = 4 * kTileBytes + 1024 + 64;
constexpr int kThreads = 128;
// Status bit set when the MMA completion wait ran out (the kernel then
// stops updating and returns; the host reports an error).
constexpr int kStatusTimeout = 8;
constexpr long long kWaitLimit = 1ll << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (row, k) of a 128-row x 32-float K-major tile
// with the 128-byte swizzle: 16-byte chunk k/4 of row `row` is stored at
// chunk (k/4) xor (row mod 8).
__device__ __forceinline__ uint32_t sw128(int row, int k) {
  return (uint32_t)row * 128u + ((uint32_t)(((k >> 2) ^ row) & 7) << 4) +
         ((uint32_t)(k & 3) << 2);
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), version 1, base offset 0 (tiles 1024-aligned).
__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;                  // LBO (unused for this layout)
  d |= (uint64_t)(1024u >> 4) << 32;        // SBO
  d |= (uint64_t)1u << 46;                  // descriptor version
  d |= (uint64_t)2u << 61;                  // SWIZZLE_128B
  return d;
}

// Instruction descriptor: D = F32, A = B = TF32, both K-major, N = 128,
// M = 128, dense, no negation.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) |
                            ((uint32_t)(TN >> 3) << 17) |
                            ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
      "[%0];" ::"r"(mbar)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(phase)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 32 lanes x 32 consecutive FP32 columns of TMEM into v[0..31].
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, "
      "%29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]),
        "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
        "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
        "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; j++) v[j] = __uint_as_float(r[j]);
}

// Per-CTA state of the tile loop.
struct TcCta {
  char* tiles;      // 4 x 16 KB, 1024-aligned: A hi, A lo, B hi, B lo
  uint32_t tiles_s; // their shared-space address
  uint32_t mbar;    // shared-space address of the MMA completion barrier
  uint32_t tmem;    // TMEM base of the 128 x 128 FP32 accumulator
  uint32_t phase;
  bool ok;
};

// Allocates TMEM (warp 0), initialises the mbarrier.  Whole CTA.
__device__ __forceinline__ TcCta tc_begin(char* smem_raw) {
  TcCta c;
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  c.tiles = smem_raw + (base - raw);
  c.tiles_s = base;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(c.tiles + 4 * kTileBytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(c.tiles + 4 * kTileBytes + 16);
  c.mbar = smem_u32(mbar);
  if (threadIdx.x < 32) {
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
            smem_u32(tslot)),
        "r"(TN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(c.mbar), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  c.tmem = *tslot;
  c.phase = 0;
  c.ok = true;
  return c;
}

__device__ __forceinline__ void tc_end(TcCta& c) {
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(
                     c.tmem),
                 "r"(TN));
}

// One tile: C[r0:r0+128, c0:c0+128] -= A[r0:, :kw] B[c0:, :kw]^T (lower
// triangle of the n x n block only).  A(r, j) = A[r + j * lda].  Whole
// CTA; returns false (and sets the status bit) if the MMA wait ran out.
__device__ __forceinline__ bool tc_tile(TcCta& c, float* C, long long ldc,
                                        const float* A, long long lda,
                                        const float* B, long long ldb, int n,
                                        int kw, int r0, int c0, int* status) {
  const int t = threadIdx.x;
  char* Ahi = c.tiles;
  char* Alo = c.tiles + kTileBytes;
  char* Bhi = c.tiles + 2 * kTileBytes;
  char* Blo = c.tiles + 3 * kTileBytes;
  {
    // all 64 loads first (in flight together), then split and store
    const int ra = r0 + t, rb = c0 + t;
    float av[TK], bv[TK];
#pragma unroll
    for (int j = 0; j < TK; j++) {
      av[j] = (ra < n && j < kw) ? A[ra + (long long)j * lda] : 0.f;
      bv[j] = (rb < n && j < kw) ? B[rb + (long long)j * ldb] : 0.f;
    }
#pragma unroll
    for (int j = 0; j < TK; j++) {
      const float ah = __uint_as_float(__float_as_uint(av[j]) & 0xffffe000u);
      const float bh = __uint_as_float(__float_as_uint(bv[j]) & 0xffffe000u);
      const uint32_t o = sw128(t, j);
      *reinterpret_cast<float*>(Ahi + o) = ah;
      *reinterpret_cast<float*>(Alo + o) = av[j] - ah;
      *reinterpret_cast<float*>(Bhi + o) = bh;
      *reinterpret_cast<float*>(Blo + o) = bv[j] - bh;
    }
  }
  // make the generic-proxy stores visible to the tensor core's async proxy
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (t == 0) {
    const uint32_t ah = c.tiles_s, al = c.tiles_s + kTileBytes;
    const uint32_t bh = c.tiles_s + 2 * kTileBytes, bl = c.tiles_s + 3 * kTileBytes;
    const uint32_t as[3] = {ah, ah, al}, bs[3] = {bh, bl, bh};
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int kk = 0; kk < TK / 8; kk++)
        mma_tf32(c.tmem, desc_sw128(as[p] + kk * 32), desc_sw128(bs[p] + kk * 32),
                 (p | kk) ? 1u : 0u);
    mma_commit(c.mbar);
  }
  // this thread's row of the C tile: chunk 0 is loaded while the MMAs run,
  // each later chunk while the previous one is updated
  const int warp = t >> 5, lane = t & 31;
  const int r = r0 + warp * 32 + lane;
  float cv[32];
  auto load_chunk = [&](int cc, float* dst) {
#pragma unroll
    for (int j = 0; j < 32; j++) {
      const int col = c0 + cc * 32 + j;
      dst[j] = (r < n && col < n && r >= col) ? C[r + (long long)col * ldc] : 0.f;
    }
  };
  load_chunk(0, cv);
  bool done = false;
  for (long long it = 0; it < kWaitLimit && !done; it++)
    done = mbar_try_wait(c.mbar, c.phase);
  c.phase ^= 1u;
  // every thread takes the same branch: one that ran out fails them all
  const bool failed = __syncthreads_or(!done) != 0;
  fence_after_sync();
  if (failed) {
    if (t == 0) atomicOr(status, kStatusTimeout);
    c.ok = false;
    return false;
  }
#pragma unroll 1
  for (int cc = 0; cc < TN / 32; cc++) {
    float nv[32];
    if (cc + 1 < TN / 32) load_chunk(cc + 1, nv);
    float v[32];
    tmem_ld32(c.tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cc * 32), v);
#pragma unroll
    for (int j = 0; j < 32; j++) {
      const int col = c0 + cc * 32 + j;
      if (r < n && col < n && r >= col) C[r + (long long)col * ldc] = cv[j] - v[j];
    }
    if (cc + 1 < TN / 32) {
#pragma unroll
      for (int j = 0; j < 32; j++) cv[j] = nv[j];
    }
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  return true;
}

}  // namespace tc
}  // namespace ab

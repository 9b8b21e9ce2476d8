// fb_tc.cuh -- asynchronous-copy and fifth-generation tensor core (tcgen05)
// building blocks for sm_100a, and the radix-16 DFT stage they compute.
//
//  * mbarrier and bulk-copy helpers (cp.async.bulk global -> shared), with a
//    bounded wait (about a second) that reports failure instead of hanging;
//  * tensor-memory allocation, shared-memory matrix descriptors, the BF16 MMA
//    with FP32 accumulation, its commit to an mbarrier, accumulator loads;
//  * tc_dft16: the first (twiddle-free) radix-16 stage of a Stockham program
//    as a GEMM on the tensor cores with split-BF16 operands.
//
// Operands live in shared memory in the K-major, no-swizzle canonical layout:
// element (row m, k) of a matrix with K_total columns sits at byte
//   (m / 8) * SBO + (k / 8) * LBO + (m % 8) * 16 + (k % 8) * 2,
// i.e. 8x8 "core matrices" of 128 contiguous bytes, LBO = 128 between core
// matrices adjacent along K, SBO = K_total / 8 * 128 between 8-row groups.
// An MMA with K = 16 consumes two core matrices along K starting at the
// descriptor's address.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "fb_device.cuh"
#include "fb_internal.h"

namespace fb {

// ------------------------------------------------- mbarrier / bulk copy
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return done != 0;
}
// Non-blocking: has phase `parity` of *b completed?  (try_wait above may
// suspend the thread for a while before it answers.)
__device__ __forceinline__ bool mbar_peek(uint64_t* b, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for phase `parity` of *b for at most `limit_ns` (0: kWaitNsDefault);
// false if it gave up.  The iteration count is bounded as well.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, uint64_t limit_ns = 0) {
  if (mbar_peek(b, parity)) return true;
  const uint64_t lim = limit_ns ? limit_ns : kWaitNsDefault;
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < (1u << 30); ++it) {
    if (global_ns() - t0 >= lim) return false;
    if (mbar_test(b, parity)) return true;
  }
  return false;
}
// The limit of a drain: the wait for a block's own copies or products still
// in flight after an earlier wait gave up -- never shorter than the default.
__device__ __forceinline__ uint64_t drain_limit(uint64_t limit_ns) {
  return limit_ns > kWaitNsDefault ? limit_ns : kWaitNsDefault;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* b) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(b))
      : "memory");
}


namespace tc {

// Byte offset of element (m, k) in the canonical layout above.
__host__ __device__ constexpr uint32_t kmajor_offset(int m, int k, int ktotal) {
  return (uint32_t)((m >> 3) * (ktotal / 8) * 128 + (k >> 3) * 128 + (m & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (sm_100 format: start address, leading and
// stride byte offsets in 16-byte units, version 1, no swizzle).
__device__ __forceinline__ uint64_t smem_desc(const void* p, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr(p) >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16 with BF16 A and B (both K-major) and
// an FP32 accumulator, shape M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// Warp-wide: allocate `ncols` (a power of two >= 32) tensor-memory columns;
// the address is written to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(dst)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
          dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
// Arrive on *bar once every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Make this thread's shared-memory stores visible to the tensor core.
__device__ __forceinline__ void fence_smem_to_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Warp-wide: lane i of the warp reads tensor-memory lane (lane field of
// taddr) + i, columns col .. col+31 of taddr, into v[0..31].
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// As tmem_ld32 for 16 columns.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// FP32 -> three BF16 terms whose sum reproduces x to about 2^-24 (round to
// nearest at each step; the second and third terms carry the residuals).
__device__ __forceinline__ void split3(float x, __nv_bfloat16& h, __nv_bfloat16& m,
                                       __nv_bfloat16& l) {
  h = __float2bfloat16_rn(x);
  const float r1 = __fsub_rn(x, __bfloat162float(h));
  m = __float2bfloat16_rn(r1);
  const float r2 = __fsub_rn(r1, __bfloat162float(m));
  l = __float2bfloat16_rn(r2);
}

// ------------------------------------------------- split-BF16 DFT-16 stage
// Layout of the radix-16 stage as a GEMM D = A * B^T (M = butterflies):
//   A row t (96 BF16): the butterfly's inputs [re_0..re_15, im_0..im_15]
//     split three ways, blocks h | m | l of 32 columns each;
//   B row o (96 BF16): output o (o < 16: Re y_o, else Im y_(o-16)) as the
//     matching row of the real form of the 16-point DFT matrix, split the same
//     way (made on the host from FP64 values, `kTcTableBytes` per direction);
//   D row t (32 FP32 in tensor memory): [Re y_0..Re y_15, Im y_0..Im y_15].
// Six block products h*h, h*m, m*h, h*l, l*h, m*m accumulate in FP32: h*h
// in one accumulator, the five correction products in a second, added in
// FP32 at the end, so the stage keeps about 24 significant bits like the FP32
// butterflies it replaces.
constexpr int kTcK = 96;                          // BF16 columns of A and B
constexpr uint32_t kTcSbo = kTcK / 8 * 128;       // 8-row group stride
constexpr int kTcTableBytes = 32 * kTcK * 2;      // B, one direction
constexpr int kTcRowBytes = kTcK * 2;             // A bytes per butterfly

// Shared state of one block's stage: A region (NT rows), B table, mbarrier,
// tensor-memory address, error flag.
struct TcCtx {
  unsigned char* a;
  const unsigned char* b;
  uint64_t* bar;
  uint32_t taddr;
  int* err;
  int t;   // block-linear thread id (= row of A and D)
  int nt;  // threads of the block: a multiple of 128, at most 512
  uint64_t wait_ns;  // limit of the wait for the products (0: default)
};

// Tensor-memory columns a block of NT threads allocates: two 32-column
// accumulators per 128-row tile, rounded up to a power of two.
__host__ __device__ constexpr uint32_t tc_cols(int NT) {
  return NT <= 128 ? 64u : (NT <= 256 ? 128u : 256u);
}

// The radix-16 DFT of v (this thread's butterfly).  Every thread of the
// block calls it once.  If the MMAs do not complete within the wait limit
// (about a second by default) the error flag is set to kErrWaitTimeout and v
// becomes zero -- but only after a second, longer wait (drain_limit) for the
// products in flight, so that the block never rewrites the A region (its
// line buffers) or frees tensor memory while the tensor core may still use
// them.
__device__ __forceinline__ void tc_dft16(cplx<float> (&v)[16], const TcCtx& c) {
  const int t = c.t;
  // 1. A row t, 16 bytes (8 BF16) per store
#pragma unroll
  for (int q = 0; q < 4; ++q) {  // re 0-7, re 8-15, im 0-7, im 8-15
    __nv_bfloat16 h[8], m[8], l[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int r = (q & 1) * 8 + i;
      split3(q < 2 ? v[r].x : v[r].y, h[i], m[i], l[i]);
    }
    *(uint4*)(c.a + kmajor_offset(t, 0 + q * 8, kTcK)) = *(const uint4*)h;
    *(uint4*)(c.a + kmajor_offset(t, 32 + q * 8, kTcK)) = *(const uint4*)m;
    *(uint4*)(c.a + kmajor_offset(t, 64 + q * 8, kTcK)) = *(const uint4*)l;
  }
  fence_smem_to_async();
  __syncthreads();
  // 2. one thread issues the MMAs: per 128-row tile, six block products of
  //    K = 32 (two K = 16 steps each), then commits to the mbarrier
  if (t == 0) {
    fence_after_sync();
    constexpr uint32_t id = idesc_bf16(128, 32);
    const int pa[6] = {0, 0, 1, 0, 2, 1}, pb[6] = {0, 1, 0, 2, 0, 1};
    for (int tile = 0; tile < c.nt / 128; ++tile) {
#pragma unroll
      for (int p = 0; p < 6; ++p) {
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          const uint64_t ad =
              smem_desc(c.a + (size_t)tile * 16 * kTcSbo + pa[p] * 512 + s * 256, 128, kTcSbo);
          const uint64_t bd = smem_desc(c.b + pb[p] * 512 + s * 256, 128, kTcSbo);
          // h*h into columns [64 tile, +32), corrections into [64 tile + 32, +32)
          const uint32_t col = (uint32_t)(tile * 64 + (p == 0 ? 0 : 32));
          mma_bf16(c.taddr + col, ad, bd, id, p == 0 ? s : (p > 1 || s > 0));
        }
      }
    }
    mma_commit(c.bar);
  }
  // 3. wait for the products, then each warp reads its 32 rows
  const bool got = mbar_wait(c.bar, 0, c.wait_ns);
  const bool ok = __syncthreads_and(got);
  fence_after_sync();
  if (ok) {
    const int w = t >> 5;
    const uint32_t base = c.taddr + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)(64 * (w >> 2));
    float d[16], e[16];
    tmem_ld16(base, d);       // Re, main products
    tmem_ld16(base + 32, e);  // Re, corrections
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r].x = __fadd_rn(d[r], e[r]);
    tmem_ld16(base + 16, d);  // Im
    tmem_ld16(base + 48, e);
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r].y = __fadd_rn(d[r], e[r]);
  } else {
    if (t == 0 && c.err) atomicExch(c.err, kErrWaitTimeout);
    // drain: the products complete before anyone reuses A or the columns
    mbar_wait(c.bar, 0, drain_limit(c.wait_ns));
    __syncthreads();
    fence_after_sync();
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = Sc<float>::mk(0.f, 0.f);
  }
  fence_before_sync();
}

// Block set-up and tear-down around tc_dft16.  tc_begin: copy the B table
// (global, 16-byte aligned) into shared memory, initialise the mbarrier,
// allocate tensor memory (warp 0); every thread calls it.  tc_end: after the
// last tensor-memory load of the block, free the columns (warp 0).
__device__ __forceinline__ TcCtx tc_begin(unsigned char* a, unsigned char* b, uint64_t* bar,
                                          uint32_t* taddr_slot, const void* table, int* err,
                                          int t, int nt, uint64_t wait_ns) {
  for (int i = t; i < kTcTableBytes / 16; i += nt) ((uint4*)b)[i] = ((const uint4*)table)[i];
  if (t == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (t < 32) {
    tmem_alloc(taddr_slot, tc_cols(nt));
    tmem_relinquish();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  return TcCtx{a, b, bar, *taddr_slot, err, t, nt, wait_ns};
}
__device__ __forceinline__ void tc_end(const TcCtx& c) {
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (c.t < 32) tmem_dealloc(c.taddr, tc_cols(c.nt));
}

}  // namespace tc
}  // namespace fb

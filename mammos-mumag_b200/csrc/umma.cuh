#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "mlp.cuh"

namespace mumag {

// The warm-start network on the 5th-generation tensor cores (tcgen05, accumulators in TMEM),
// shared by the stand-alone inference kernel (mlp.cu) and the solver's learned start
// (solver.cu).
//
// One CTA of 256 threads takes 128-row tiles (M = 128).  The three hidden layers are
// tcgen05.mma kind::f16 products, M = 128, N = 128, BF16 operands from shared memory, FP32
// accumulation in 128 TMEM columns; one thread issues them and commits to an mbarrier.
// Between layers warp w reads TMEM lanes 32 (w % 4) .. +31 (its rows) and columns
// 64 (w / 4) .. +63 (tcgen05.ld 32x32b), adds the bias, applies GELU, rounds to BF16 and
// writes them into the next layer's operand buffer; two warps per lane quarter split the
// CUDA-core epilogue.  The 128 -> 1 head is a per-thread dot product over its 64 columns,
// the two halves summed through shared memory.  The weights are copied into shared memory
// once per CTA, into a shared-memory region of kSmTc bytes (16-byte aligned).
//
// Operand layout (K-major, no swizzle): 8-row x 16-byte core matrices, 128 contiguous bytes
// each; the K/8 core matrices of an 8-row group are adjacent (leading byte offset 128), the
// groups K/8 * 128 bytes apart (stride byte offset).  One MMA consumes K = 16, i.e. two
// core matrices: the descriptors of step ks start 256 * ks bytes in.
constexpr int kTcRows = 128;     // rows per tile (M)
constexpr int kTcThreads = 256;  // two warps per TMEM lane quarter
constexpr uint32_t kSmW1 = 0;                                            // [128][16]  bf16
constexpr uint32_t kSmW2 = kSmW1 + kMlpHidden * kMlpInPad * 2;           // [128][128]
constexpr uint32_t kSmW3 = kSmW2 + kMlpHidden * kMlpHidden * 2;
constexpr uint32_t kSmA0 = kSmW3 + kMlpHidden * kMlpHidden * 2;          // [128][16] layer-1 input
constexpr uint32_t kSmA = kSmA0 + kTcRows * kMlpInPad * 2;               // [128][128] hidden rows
constexpr uint32_t kSmHead = kSmA + kTcRows * kMlpHidden * 2;            // [128] head partials
constexpr uint32_t kSmBar = kSmHead + kTcRows * 4;                       // mbarrier, TMEM address
constexpr uint32_t kSmTc = kSmBar + 16;
constexpr uint32_t kTmemCols = 128;
constexpr unsigned kTcWaitLimit = 1u << 22;

// byte offset of element (r, k) of a K-major [rows][kdim] BF16 operand
__device__ __forceinline__ uint32_t umma_off(int r, int k, int kdim) {
  return (uint32_t)(((r >> 3) * (kdim >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
// shared-memory matrix descriptor: start, leading and stride byte offsets (>> 4), the
// Blackwell descriptor version 1 (bit 46), no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N = 128, M = 128
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(128 >> 3) << 17) |
                              ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kTcIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// bounded wait for the mbarrier phase; false after the limit
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t phase) {
  for (unsigned it = 0; it < kTcWaitLimit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    if (ok) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// Copy a [128][kdim] BF16 weight matrix (row-major [out][in]) into the operand layout.
__device__ __forceinline__ void tc_stage_weights(unsigned char* sm, uint32_t off, const __nv_bfloat16* W, int kdim) {
  const int chunks = kMlpHidden * kdim / 8;
  for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
    const int r = c / (kdim / 8), k = (c % (kdim / 8)) * 8;
    *reinterpret_cast<uint4*>(sm + off + umma_off(r, k, kdim)) =
        __ldg(reinterpret_cast<const uint4*>(W + (size_t)r * kdim + k));
  }
}


// Per-CTA set-up (all 256 threads call it): TMEM columns (warp 0), the mbarrier, the
// weights in the region.  Returns the TMEM address.
__device__ __forceinline__ uint32_t tc_net_setup(unsigned char* sm, const MlpDev& M) {
  const int warp = threadIdx.x >> 5;
  const uint32_t bar = (uint32_t)__cvta_generic_to_shared(sm) + kSmBar;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(bar + 8),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_stage_weights(sm, kSmW1, M.W1, kMlpInPad);
  tc_stage_weights(sm, kSmW2, M.W2, kMlpHidden);
  tc_stage_weights(sm, kSmW3, M.W3, kMlpHidden);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return *reinterpret_cast<const volatile uint32_t*>(sm + kSmBar + 8);
}

// Release the TMEM columns (all threads call it).  After a failed tile, `pending` makes it
// first wait (bounded) for the product still in flight.
__device__ __forceinline__ void tc_net_teardown(unsigned char* sm, uint32_t tmem, bool pending, uint32_t phase) {
  if (pending) tc_wait((uint32_t)__cvta_generic_to_shared(sm) + kSmBar, phase);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// One 128-row tile through the network.  feat(r, col) gives raw feature col of tile row r
// (0 for rows past the valid ones); out(r, y) receives y = out_scale * network(row r), called
// by one thread per row.  Returns false, the same in every thread, if a product did not
// complete within the wait limit (the tile's outputs are then not written).
template <class F, class O>
__device__ __forceinline__ bool tc_net_tile(unsigned char* sm, uint32_t tmem, uint32_t& phase, const MlpDev& M, F feat,
                                            O out) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int rloc = 32 * (warp & 3) + lane;  // this thread's row in the tile (its TMEM lane)
  const int cbase = 64 * (warp >> 2);       // its 64 columns
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
  const uint32_t bar = sbase + kSmBar;
  const uint32_t trow = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)cbase;
  float* head = reinterpret_cast<float*>(sm + kSmHead);
  {  // layer-1 operand: the row's normalised features, BF16 (8 per thread)
    const int c = warp >> 2;
    float f[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) f[q] = (feat(rloc, 8 * c + q) - __ldg(M.fmean + 8 * c + q)) * __ldg(M.fscale + 8 * c + q);
    uint4 v;
    v.x = pack_bf16(f[0], f[1]);
    v.y = pack_bf16(f[2], f[3]);
    v.z = pack_bf16(f[4], f[5]);
    v.w = pack_bf16(f[6], f[7]);
    *reinterpret_cast<uint4*>(sm + kSmA0 + umma_off(rloc, 8 * c, kMlpInPad)) = v;
  }
  float yacc = 0.f;
  for (int layer = 0; layer < 3; ++layer) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t aoff = layer == 0 ? kSmA0 : kSmA;
      const uint32_t woff = layer == 0 ? kSmW1 : layer == 1 ? kSmW2 : kSmW3;
      const int kdim = layer == 0 ? kMlpInPad : kMlpHidden;
      const uint32_t sbo = (uint32_t)(kdim / 8) * 128;
      for (int ks = 0; ks < kdim / 16; ++ks)
        tc_mma(tmem, umma_desc(sbase + aoff + 256 * ks, 128, sbo), umma_desc(sbase + woff + 256 * ks, 128, sbo),
               ks > 0 ? 1u : 0u);
      tc_commit(bar);
    }
    const bool got = tc_wait(bar, phase);
    if (__syncthreads_or(!got)) return false;  // every thread leaves together
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const float* bias = (layer == 0 ? M.b1 : layer == 1 ? M.b2 : M.b3) + cbase;
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
      float v[16];
      tc_ld16(trow + 16 * j, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = gelu_f(v[q] + __ldg(bias + 16 * j + q));
      if (layer < 2) {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          uint4 w;
          w.x = pack_bf16(v[8 * c + 0], v[8 * c + 1]);
          w.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
          w.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
          w.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
          *reinterpret_cast<uint4*>(sm + kSmA + umma_off(rloc, cbase + 16 * j + 8 * c, kMlpHidden)) = w;
        }
      } else {  // head: the BF16-rounded activations against w4
#pragma unroll
        for (int q = 0; q < 16; ++q)
          yacc += __bfloat162float(__float2bfloat16(v[q])) * __ldg(M.w4 + cbase + 16 * j + q);
      }
    }
  }
  // the two column halves of each row's head
  if (warp >= 4) head[rloc] = yacc;
  __syncthreads();
  if (warp < 4) out(rloc, (yacc + head[rloc] + __ldg(M.b4)) * M.out_scale);
  return true;
}

}  // namespace mumag

#pragma once
// One training step's gradient of the warm-start network on the 5th-generation tensor cores:
// k_train_tc, one CTA of 256 threads per 128-row tile of the batch (mlp.cu launches it).
//
// Forward: the three hidden layers as in tc_net_tile (umma.cuh), but each layer's FP32
// accumulator stays in its own 128 TMEM columns (Z1 in 0..127, Z2 in 128..255, Z3 in
// 256..383; the bias is added when read), and every BF16 activation is written twice into
// shared memory: K-major by row (the next layer's A operand) and K-major by neuron (the
// transposed operand of the weight gradient, K = the batch rows).
// Backward, per layer from the top: dZ = dH * gelu'(Z) (dH3 = dy w4) rounded to BF16 and
// written the same two ways; then two products in one commit -- dH_below = dZ W (B operand
// W^T, staged over the forward weights once they are consumed) into columns 384..511, and
// dW = dZ^T H into the columns of the Z that dZ was just made from -- and the FP32 weight
// gradients added to the global gradient.  Bias gradients are column sums of the BF16 dZ,
// dw4 = sum dy H3, db4 = sum dy.  The rounding points are those of the warp-level kernels this
// replaces and of the oracle (oracle/mlp_oracle.py).
//
// Rows past the batch (a partial last tile) carry zero features and dy = 0, so they add
// nothing.  Every wait is bounded; a wait that runs out sets *err and the CTA leaves after
// releasing its tensor memory.
#include "umma.cuh"

namespace mumag {

constexpr uint32_t kTrW1 = 0;                                   // [128][16]  W1 (B, layer 1)
constexpr uint32_t kTrW2 = kTrW1 + kMlpHidden * kMlpInPad * 2;  // [128][128] W2, then W3^T
constexpr uint32_t kTrW3 = kTrW2 + kMlpHidden * kMlpHidden * 2; // [128][128] W3, then W2^T
constexpr uint32_t kTrA0 = kTrW3 + kMlpHidden * kMlpHidden * 2; // [128][16]  H0 by row
constexpr uint32_t kTrA = kTrA0 + kTcRows * kMlpInPad * 2;       // [128][128] H1, H2, then dZ3, dZ2 by row
constexpr uint32_t kTrT0 = kTrA + kTcRows * kMlpHidden * 2;      // [16][128]  H0 by feature
constexpr uint32_t kTrT1 = kTrT0 + kMlpInPad * kTcRows * 2;      // [128][128] H1 by neuron
constexpr uint32_t kTrT2 = kTrT1 + kMlpHidden * kTcRows * 2;     // [128][128] H2 by neuron
constexpr uint32_t kTrD = kTrT2 + kMlpHidden * kTcRows * 2;      // [128][128] dZ3, dZ2, dZ1 by neuron
constexpr uint32_t kTrDy = kTrD + kMlpHidden * kTcRows * 2;      // [128] dy
constexpr uint32_t kTrHead = kTrDy + kTcRows * 4;                // [128] head partials
constexpr uint32_t kTrW4 = kTrHead + kTcRows * 4;                // [128] dw4 partials
constexpr uint32_t kTrBar = kTrW4 + kMlpHidden * 4;              // mbarrier, TMEM address
constexpr uint32_t kSmTrain = kTrBar + 16;
constexpr uint32_t kTrCols = 512;

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void tc_mma_d(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}
// C[tmem] (+)= A [128][K] . B [n][K]^T, both K-major (kdim K) at byte offsets aoff, boff
__device__ __forceinline__ void tc_gemm(uint32_t sbase, uint32_t tmem, uint32_t aoff, uint32_t boff, int kdim, int n) {
  const uint32_t sbo = (uint32_t)(kdim / 8) * 128;
  for (int ks = 0; ks < kdim / 16; ++ks)
    tc_mma_d(tmem, umma_desc(sbase + aoff + 256 * ks, 128, sbo), umma_desc(sbase + boff + 256 * ks, 128, sbo),
             tc_idesc(n), ks > 0 ? 1u : 0u);
}
__device__ __forceinline__ void tc_sync_for_mma() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void st_bf16(unsigned char* sm, uint32_t off, float v) {
  *reinterpret_cast<__nv_bfloat16*>(sm + off) = __float2bfloat16(v);
}

__global__ void __launch_bounds__(kTcThreads, 1)
    k_train_tc(MlpDev M, const __nv_bfloat16* __restrict__ W2t, const __nv_bfloat16* __restrict__ W3t,
               const float* __restrict__ feat, const float* __restrict__ target, int B, float* __restrict__ g,
               int offW1, int offB1, int offW2, int offB2, int offW3, int offB3, int offW4, int offB4,
               float* __restrict__ loss, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int rloc = 32 * (warp & 3) + lane;  // this thread's tile row = its TMEM lane
  const int cbase = 64 * (warp >> 2);       // its 64 columns
  const int row = blockIdx.x * kTcRows + rloc;
  const bool live = row < B;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
  const uint32_t bar = sbase + kTrBar;
  float* dys = reinterpret_cast<float*>(sm + kTrDy);
  float* head = reinterpret_cast<float*>(sm + kTrHead);
  float* dw4s = reinterpret_cast<float*>(sm + kTrW4);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(bar + 8), "r"(kTrCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < kMlpHidden) dw4s[tid] = 0.f;
  tc_stage_weights(sm, kTrW1, M.W1, kMlpInPad);
  tc_stage_weights(sm, kTrW2, M.W2, kMlpHidden);
  tc_stage_weights(sm, kTrW3, M.W3, kMlpHidden);
  {  // normalised features, BF16, by row and by feature (8 per thread)
    const int c = warp >> 2;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int f = 8 * c + q;
      const float x = live ? (feat[(size_t)row * kMlpIn + f] - __ldg(M.fmean + f)) * __ldg(M.fscale + f) : 0.f;
      st_bf16(sm, kTrA0 + umma_off(rloc, f, kMlpInPad), x);
      st_bf16(sm, kTrT0 + umma_off(f, rloc, kTcRows), x);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *reinterpret_cast<const volatile uint32_t*>(sm + kTrBar + 8);
  const uint32_t tlane = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
  uint32_t phase = 0;
  bool ok = true;
  auto wait = [&]() {  // the phase advances only when the product completed
    const bool got = tc_wait(bar, phase);
    ok = !__syncthreads_or(!got);
    if (ok) phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return ok;
  };
  auto issue = [&](uint32_t col, uint32_t aoff, uint32_t boff, int kdim, int n, bool commit) {
    if (tid == 0) {
      tc_gemm(sbase, tmem + col, aoff, boff, kdim, n);
      if (commit) tc_commit(bar);
    }
  };
  // ---- forward
  float yacc = 0.f;
  for (int layer = 0; layer < 3 && ok; ++layer) {
    tc_sync_for_mma();
    issue(128u * layer, layer == 0 ? kTrA0 : kTrA, layer == 0 ? kTrW1 : layer == 1 ? kTrW2 : kTrW3,
          layer == 0 ? kMlpInPad : kMlpHidden, kMlpHidden, true);
    if (!wait()) break;
    const float* bias = layer == 0 ? M.b1 : layer == 1 ? M.b2 : M.b3;
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
      float v[16];
      tc_ld16(tlane + 128u * layer + cbase + 16 * j, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int col = cbase + 16 * j + q;
        const float h = gelu_f(v[q] + __ldg(bias + col));
        if (layer < 2) {
          st_bf16(sm, kTrA + umma_off(rloc, col, kMlpHidden), h);
          st_bf16(sm, (layer == 0 ? kTrT1 : kTrT2) + umma_off(col, rloc, kTcRows), h);
        } else {
          yacc += __bfloat162float(__float2bfloat16(h)) * __ldg(M.w4 + col);
        }
      }
    }
    // the forward weight just consumed makes room for a backward one
    if (layer == 1) tc_stage_weights(sm, kTrW2, W3t, kMlpHidden);
    if (layer == 2) tc_stage_weights(sm, kTrW3, W2t, kMlpHidden);
  }
  if (ok) {  // head, loss and dy
    if (warp >= 4) head[rloc] = yacc;
    __syncthreads();
    if (warp < 4) {
      float dy = 0.f;
      if (live) {
        const float y = yacc + head[rloc] + __ldg(M.b4);
        const float e = y - target[row] / M.out_scale;
        dy = 2.f * e / B;
        atomicAdd(loss, e * e / B);
        atomicAdd(g + offB4, dy);
      }
      dys[rloc] = dy;
    }
    __syncthreads();
  }
  // ---- backward: layer 3 (Z3 in 256..383), then 2 (128..255), then 1 (0..127)
  for (int layer = 2; layer >= 0 && ok; --layer) {
    const float* bias = layer == 0 ? M.b1 : layer == 1 ? M.b2 : M.b3;
    const float dy = dys[rloc];
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
      float z[16], dh[16];
      tc_ld16(tlane + 128u * layer + cbase + 16 * j, z);
      if (layer < 2) tc_ld16(tlane + 384u + cbase + 16 * j, dh);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int col = cbase + 16 * j + q;
        const float zz = z[q] + __ldg(bias + col);
        float d;
        if (layer == 2) {
          d = dy * __ldg(M.w4 + col);
          atomicAdd(dw4s + col, dy * __bfloat162float(__float2bfloat16(gelu_f(zz))));
        } else {
          d = dh[q];
        }
        d = live ? d * gelu_grad_f(zz) : 0.f;
        if (layer > 0) st_bf16(sm, kTrA + umma_off(rloc, col, kMlpHidden), d);
        st_bf16(sm, kTrD + umma_off(col, rloc, kTcRows), d);
      }
    }
    tc_sync_for_mma();
    // dH of the layer below (B = W^T, staged over the consumed forward weight) into 384..511,
    // dW = dZ^T H into this layer's Z columns; one commit for both
    if (layer > 0) issue(384u, kTrA, layer == 2 ? kTrW2 : kTrW3, kMlpHidden, kMlpHidden, false);
    issue(128u * layer, kTrD, layer == 2 ? kTrT2 : layer == 1 ? kTrT1 : kTrT0, kTcRows,
          layer == 0 ? kMlpInPad : kMlpHidden, true);
    // bias gradient: column sums of the BF16 dZ (read while the products run)
    if (tid < kMlpHidden) {
      float s = 0.f;
      for (int b = 0; b < kTcRows; ++b)
        s += __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(sm + kTrD + umma_off(tid, b, kTcRows)));
      atomicAdd(g + (layer == 0 ? offB1 : layer == 1 ? offB2 : offB3) + tid, s);
    }
    if (!wait()) break;
    // weight gradient rows = TMEM lanes (output neurons), columns = inputs
    const int nin = layer == 0 ? kMlpInPad : kMlpHidden;
    float* gw = g + (layer == 0 ? offW1 : layer == 1 ? offW2 : offW3) + (size_t)rloc * nin;
    if (layer > 0) {
#pragma unroll 1
      for (int j = 0; j < 4; ++j) {
        float v[16];
        tc_ld16(tlane + 128u * layer + cbase + 16 * j, v);
#pragma unroll
        for (int q = 0; q < 16; ++q) atomicAdd(gw + cbase + 16 * j + q, v[q]);
      }
    } else {
      float v[16];
      tc_ld16(tlane, v);  // every warp loads (the instruction is warp-collective); half add
      if (cbase == 0) {
#pragma unroll
        for (int q = 0; q < 16; ++q) atomicAdd(gw + q, v[q]);
      }
    }
  }
  if (ok) {
    __syncthreads();
    if (tid < kMlpHidden) atomicAdd(g + offW4 + tid, dw4s[tid]);
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  if (!ok) tc_wait(bar, phase);  // a product still in flight finishes before the columns go
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTrCols));
}

}  // namespace mumag

// The learned warm start for the magnetostatic Poisson solve: a per-node MLP
//   12 features -> 128 -> 128 -> 128 -> 1, GELU (tanh form), BF16 weights, FP32 accumulation,
// on the tensor cores with mma.sync m16n8k16.  One warp evaluates a tile of 16 nodes; each
// layer's accumulator fragments are re-packed in registers as the next layer's A fragments
// (the m16n8 C layout of two adjacent n-tiles is the m16n8k16 A layout of one k-step), so
// activations never leave the registers.
//
// Features of node i (the 1-ring = the node's row of the SELL pattern, itself included):
//   0-11  m_i (3), u_i (1), mean over the ring of m (3) and of u (1), max over the ring of
//         m (3) and of u (1); m the trial magnetisation, u the potential of the previous
//         evaluation (the solve's warm start);
//   12-15 the Jacobi-scaled initial residual z = (b - S u) / diag(S) over sigma: z_i, and its
//         ring mean, max and min.  sigma = rms of z over the mesh's nodes.
// The first input layer is one k16 step of the tensor-core product, so the four residual
// features ride in what would otherwise be zero padding of the twelve.  Inputs are
// normalised with the model's per-feature mean/scale; the output y gives the correction
// du_i = out_scale * y in units of sigma (the solve's equation is linear in the residual).
// The solve adds alpha du to u with the step alpha = du.r0 / du.S du that minimises the
// S-norm of the error along du, so a poor prediction cannot make the start worse than
// the previous potential in that norm.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace mumag {

constexpr int kMlpIn = 16;       // features
constexpr int kMlpInPad = 16;    // one k16 step
constexpr int kMlpHidden = 128;

// Device view of a model.  Weight matrices are [out][in] (K-major rows), BF16; the
// transposed copies serve the backward pass.
struct MlpDev {
  const __nv_bfloat16* W1;  // [128][16]
  const __nv_bfloat16* W2;  // [128][128]
  const __nv_bfloat16* W3;  // [128][128]
  const float* b1;          // [128]
  const float* b2;
  const float* b3;
  const float* w4;          // [128]
  const float* b4;          // [1]
  float out_scale;
  const float* fmean;       // [16]
  const float* fscale;      // [16]  (1/std)
};

__device__ __forceinline__ float gelu_f(float x) {
  const float k0 = 0.7978845608028654f, k1 = 0.044715f;  // sqrt(2/pi)
  return 0.5f * x * (1.0f + tanhf(k0 * (x + k1 * x * x * x)));
}
__device__ __forceinline__ float gelu_grad_f(float x) {
  const float k0 = 0.7978845608028654f, k1 = 0.044715f;
  const float t = tanhf(k0 * (x + k1 * x * x * x));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * k0 * (1.0f + 3.0f * k1 * x * x);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// B fragment of W[n][k] (K-major rows of length ldk) for n-tile nt and k-step ks.
__device__ __forceinline__ void load_b_frag(const __nv_bfloat16* W, int ldk, int nt, int ks, int lane, uint32_t& b0,
                                            uint32_t& b1) {
  const int g = lane >> 2, t = lane & 3;
  const __nv_bfloat16* p = W + (size_t)(nt * 8 + g) * ldk + ks * 16 + 2 * t;
  b0 = __ldg(reinterpret_cast<const unsigned int*>(p));
  b1 = __ldg(reinterpret_cast<const unsigned int*>(p + 8));
}

// One hidden layer on a 16-row tile: out = act(A . W^T + b), A as k16 fragments
// ain[ks][4] (K = 16 * nks), output as k16 fragments aout[8][4] of the 128 outputs.
// If zout != nullptr the pre-activations are returned in C layout (zout[16][4]).  The 16
// n-tiles are done four at a time (16 accumulator registers live), which keeps the layer
// within the register budget of the persistent solver kernel.
template <int NKS>
__device__ __forceinline__ void mlp_layer(const uint32_t (&ain)[NKS][4], const __nv_bfloat16* W, const float* b,
                                          int lane, uint32_t (&aout)[8][4], float (*zout)[4] = nullptr) {
  const int t = lane & 3;
#pragma unroll
  for (int quarter = 0; quarter < 4; ++quarter) {
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int nt = quarter * 4 + j;
      const float bl = __ldg(b + nt * 8 + 2 * t), bh = __ldg(b + nt * 8 + 2 * t + 1);
      acc[j][0] = bl;
      acc[j][1] = bh;
      acc[j][2] = bl;
      acc[j][3] = bh;
#pragma unroll
      for (int ks = 0; ks < NKS; ++ks) {
        uint32_t b0, b1;
        load_b_frag(W, NKS * 16, nt, ks, lane, b0, b1);
        mma_bf16_16816(acc[j], ain[ks], b0, b1);
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (zout) {
#pragma unroll
        for (int q = 0; q < 4; ++q) zout[quarter * 4 + j][q] = acc[j][q];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[j][q] = gelu_f(acc[j][q]);
    }
    // n-tiles (2p, 2p+1) of this quarter form k-step (quarter*2 + p) of the next layer
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const int ks = quarter * 2 + p;
      aout[ks][0] = pack_bf16(acc[2 * p][0], acc[2 * p][1]);
      aout[ks][1] = pack_bf16(acc[2 * p][2], acc[2 * p][3]);
      aout[ks][2] = pack_bf16(acc[2 * p + 1][0], acc[2 * p + 1][1]);
      aout[ks][3] = pack_bf16(acc[2 * p + 1][2], acc[2 * p + 1][3]);
    }
  }
}

// Final 128 -> 1 layer from k16 fragments: y for rows g (lo) and g+8 (hi), in every lane
// of the row's group of four.
__device__ __forceinline__ void mlp_head(const uint32_t (&h)[8][4], const float* w4, float b4, int lane, float& ylo,
                                         float& yhi) {
  const int t = lane & 3;
  float lo = 0.f, hi = 0.f;
#pragma unroll
  for (int ks = 0; ks < 8; ++ks) {
    const int c0 = ks * 16 + 2 * t;
    const float w0 = __ldg(w4 + c0), w1 = __ldg(w4 + c0 + 1), w8 = __ldg(w4 + c0 + 8), w9 = __ldg(w4 + c0 + 9);
    const __nv_bfloat162 r0 = *reinterpret_cast<const __nv_bfloat162*>(&h[ks][0]);
    const __nv_bfloat162 r1 = *reinterpret_cast<const __nv_bfloat162*>(&h[ks][1]);
    const __nv_bfloat162 r2 = *reinterpret_cast<const __nv_bfloat162*>(&h[ks][2]);
    const __nv_bfloat162 r3 = *reinterpret_cast<const __nv_bfloat162*>(&h[ks][3]);
    lo += __low2float(r0) * w0 + __high2float(r0) * w1 + __low2float(r2) * w8 + __high2float(r2) * w9;
    hi += __low2float(r1) * w0 + __high2float(r1) * w1 + __low2float(r3) * w8 + __high2float(r3) * w9;
  }
  lo += __shfl_xor_sync(0xffffffffu, lo, 1);
  lo += __shfl_xor_sync(0xffffffffu, lo, 2);
  hi += __shfl_xor_sync(0xffffffffu, hi, 1);
  hi += __shfl_xor_sync(0xffffffffu, hi, 2);
  ylo = lo + b4;
  yhi = hi + b4;
}

// A fragment (k16) of 16 normalised feature rows: feat(row, col) gives the raw feature.
template <class F>
__device__ __forceinline__ void feature_frag(const MlpDev& M, int lane, F feat, uint32_t (&a)[1][4]) {
  const int g = lane >> 2, t = lane & 3;
  auto nf = [&](int row, int col) -> float {
    return col < kMlpIn ? (feat(row, col) - __ldg(M.fmean + col)) * __ldg(M.fscale + col) : 0.f;
  };
  a[0][0] = pack_bf16(nf(g, 2 * t), nf(g, 2 * t + 1));
  a[0][1] = pack_bf16(nf(g + 8, 2 * t), nf(g + 8, 2 * t + 1));
  a[0][2] = pack_bf16(nf(g, 2 * t + 8), nf(g, 2 * t + 9));
  a[0][3] = pack_bf16(nf(g + 8, 2 * t + 8), nf(g + 8, 2 * t + 9));
}

// Forward pass of one 16-row tile: returns y * out_scale for rows g and g+8.
template <class F>
__device__ __forceinline__ void mlp_tile_forward(const MlpDev& M, int lane, F feat, float& du_lo, float& du_hi) {
  uint32_t a0[1][4];
  feature_frag(M, lane, feat, a0);
  uint32_t h1[8][4], h2[8][4];
  mlp_layer<1>(a0, M.W1, M.b1, lane, h1);
  mlp_layer<8>(h1, M.W2, M.b2, lane, h2);
  mlp_layer<8>(h2, M.W3, M.b3, lane, h1);
  float ylo, yhi;
  mlp_head(h1, M.w4, __ldg(M.b4), lane, ylo, yhi);
  du_lo = ylo * M.out_scale;
  du_hi = yhi * M.out_scale;
}

}  // namespace mumag

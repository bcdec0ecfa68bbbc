// Training and stand-alone inference of the warm-start MLP (mlp.cuh), plus its C ABI.
//
// One training step on a batch of B samples (B a multiple of 16):
//   k_fwd    per warp, 16 samples: normalised features -> three GELU layers (pre-activations
//            Z kept in FP32, activations stored transposed in BF16 for the weight gradients)
//            -> head y; loss 1/B sum (y - t/out_scale)^2 and dL/dy
//   k_bwd    per warp, 16 samples: dZ3 = dy w4 . gelu'(Z3), dZ2 = (dZ3 W3) . gelu'(Z2),
//            dZ1 = (dZ2 W2) . gelu'(Z1) on the tensor cores (B operands W^T), dZ stored
//            transposed in BF16; dw4, db4 by warp reductions
//   k_wgrad  dW = dZ^T H on the tensor cores (K = the batch), one 16x8 tile per warp
//   k_bsum   db = column sums of dZ
//   k_adam   Adam on FP32 master weights, then BF16 copies and transposes
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "device_mesh.h"
#include "mlp.cuh"
#include "umma.cuh"

namespace mumag {

// parameter offsets in the FP32 master vector
constexpr int kOffW1 = 0;                                   // [128][16]
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpInPad;     // [128]
constexpr int kOffW2 = kOffB1 + kMlpHidden;                 // [128][128]
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpHidden * kMlpHidden;
constexpr int kOffW4 = kOffB3 + kMlpHidden;                 // [128]
constexpr int kOffB4 = kOffW4 + kMlpHidden;                 // [1]
constexpr int kNumParams = kOffB4 + 1;

namespace {

__global__ void k_fwd(MlpDev M, const float* __restrict__ feat, const float* __restrict__ target, int B,
                      float* Z1, float* Z2, float* Z3, __nv_bfloat16* H0t, __nv_bfloat16* H1t, __nv_bfloat16* H2t,
                      __nv_bfloat16* H3t, float* dy, float* loss) {
  const int lane = threadIdx.x & 31;
  const int tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (tile * 16 >= B) return;
  const int r0 = tile * 16, g = lane >> 2, t = lane & 3;
  auto F = [&](int row, int col) { return feat[(size_t)(r0 + row) * kMlpIn + col]; };
  uint32_t a0[1][4];
  feature_frag(M, lane, F, a0);
  // store the normalised input transposed (its BF16 values are what layer 1 consumed)
  auto store_t = [&](__nv_bfloat16* Ht, const uint32_t(&a)[4], int ks) {
    const __nv_bfloat162 v0 = *reinterpret_cast<const __nv_bfloat162*>(&a[0]);
    const __nv_bfloat162 v1 = *reinterpret_cast<const __nv_bfloat162*>(&a[1]);
    const __nv_bfloat162 v2 = *reinterpret_cast<const __nv_bfloat162*>(&a[2]);
    const __nv_bfloat162 v3 = *reinterpret_cast<const __nv_bfloat162*>(&a[3]);
    const int c = ks * 16 + 2 * t;
    Ht[(size_t)c * B + r0 + g] = v0.x;
    Ht[(size_t)(c + 1) * B + r0 + g] = v0.y;
    Ht[(size_t)c * B + r0 + g + 8] = v1.x;
    Ht[(size_t)(c + 1) * B + r0 + g + 8] = v1.y;
    Ht[(size_t)(c + 8) * B + r0 + g] = v2.x;
    Ht[(size_t)(c + 9) * B + r0 + g] = v2.y;
    Ht[(size_t)(c + 8) * B + r0 + g + 8] = v3.x;
    Ht[(size_t)(c + 9) * B + r0 + g + 8] = v3.y;
  };
  store_t(H0t, a0[0], 0);
  auto store_z = [&](float* Z, const float (*z)[4]) {
    for (int nt = 0; nt < 16; ++nt) {
      const int c = nt * 8 + 2 * t;
      *reinterpret_cast<float2*>(Z + (size_t)(r0 + g) * kMlpHidden + c) = make_float2(z[nt][0], z[nt][1]);
      *reinterpret_cast<float2*>(Z + (size_t)(r0 + g + 8) * kMlpHidden + c) = make_float2(z[nt][2], z[nt][3]);
    }
  };
  uint32_t h1[8][4], h2[8][4];
  float z[16][4];
  mlp_layer<1>(a0, M.W1, M.b1, lane, h1, z);
  store_z(Z1, z);
  for (int ks = 0; ks < 8; ++ks) store_t(H1t, h1[ks], ks);
  mlp_layer<8>(h1, M.W2, M.b2, lane, h2, z);
  store_z(Z2, z);
  for (int ks = 0; ks < 8; ++ks) store_t(H2t, h2[ks], ks);
  mlp_layer<8>(h2, M.W3, M.b3, lane, h1, z);
  store_z(Z3, z);
  for (int ks = 0; ks < 8; ++ks) store_t(H3t, h1[ks], ks);
  float ylo, yhi;
  mlp_head(h1, M.w4, __ldg(M.b4), lane, ylo, yhi);
  if (t == 0) {
    const float elo = ylo - target[r0 + g] / M.out_scale, ehi = yhi - target[r0 + g + 8] / M.out_scale;
    dy[r0 + g] = 2.f * elo / B;
    dy[r0 + g + 8] = 2.f * ehi / B;
    atomicAdd(loss, (elo * elo + ehi * ehi) / B);
  }
}

// dZ of one layer from dH in C layout: dz = dh * gelu'(Z); stored transposed (BF16) and
// returned as k16 A fragments for the next product
__device__ __forceinline__ void dz_from_dh(float (*dh)[4], const float* Z, int B, int r0, int lane,
                                           __nv_bfloat16* dZt, uint32_t (&a)[8][4]) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) {
    const int c = nt * 8 + 2 * t;
    const float2 zl = *reinterpret_cast<const float2*>(Z + (size_t)(r0 + g) * kMlpHidden + c);
    const float2 zh = *reinterpret_cast<const float2*>(Z + (size_t)(r0 + g + 8) * kMlpHidden + c);
    dh[nt][0] *= gelu_grad_f(zl.x);
    dh[nt][1] *= gelu_grad_f(zl.y);
    dh[nt][2] *= gelu_grad_f(zh.x);
    dh[nt][3] *= gelu_grad_f(zh.y);
  }
#pragma unroll
  for (int p = 0; p < 8; ++p) {
    a[p][0] = pack_bf16(dh[2 * p][0], dh[2 * p][1]);
    a[p][1] = pack_bf16(dh[2 * p][2], dh[2 * p][3]);
    a[p][2] = pack_bf16(dh[2 * p + 1][0], dh[2 * p + 1][1]);
    a[p][3] = pack_bf16(dh[2 * p + 1][2], dh[2 * p + 1][3]);
    const __nv_bfloat162 v0 = *reinterpret_cast<const __nv_bfloat162*>(&a[p][0]);
    const __nv_bfloat162 v1 = *reinterpret_cast<const __nv_bfloat162*>(&a[p][1]);
    const __nv_bfloat162 v2 = *reinterpret_cast<const __nv_bfloat162*>(&a[p][2]);
    const __nv_bfloat162 v3 = *reinterpret_cast<const __nv_bfloat162*>(&a[p][3]);
    const int c = p * 16 + 2 * t;
    dZt[(size_t)c * B + r0 + g] = v0.x;
    dZt[(size_t)(c + 1) * B + r0 + g] = v0.y;
    dZt[(size_t)c * B + r0 + g + 8] = v1.x;
    dZt[(size_t)(c + 1) * B + r0 + g + 8] = v1.y;
    dZt[(size_t)(c + 8) * B + r0 + g] = v2.x;
    dZt[(size_t)(c + 9) * B + r0 + g] = v2.y;
    dZt[(size_t)(c + 8) * B + r0 + g + 8] = v3.x;
    dZt[(size_t)(c + 9) * B + r0 + g + 8] = v3.y;
  }
}

// dH = dZ . W (W [out][in]), B operand W^T stored [in][out]
__device__ __forceinline__ void back_product(const uint32_t (&a)[8][4], const __nv_bfloat16* Wt, int lane,
                                             float (*dh)[4]) {
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) {
    dh[nt][0] = dh[nt][1] = dh[nt][2] = dh[nt][3] = 0.f;
#pragma unroll
    for (int ks = 0; ks < 8; ++ks) {
      uint32_t b0, b1;
      load_b_frag(Wt, kMlpHidden, nt, ks, lane, b0, b1);
      mma_bf16_16816(dh[nt], a[ks], b0, b1);
    }
  }
}

__global__ void k_bwd(MlpDev M, const __nv_bfloat16* W2t, const __nv_bfloat16* W3t, int B, const float* Z1,
                      const float* Z2, const float* Z3, const __nv_bfloat16* H3t, const float* dy,
                      __nv_bfloat16* dZ1t, __nv_bfloat16* dZ2t, __nv_bfloat16* dZ3t, float* gw4, float* gb4) {
  const int lane = threadIdx.x & 31;
  const int tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (tile * 16 >= B) return;
  const int r0 = tile * 16, g = lane >> 2, t = lane & 3;
  const float dlo = dy[r0 + g], dhi = dy[r0 + g + 8];
  float dh[16][4];
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) {
    const int c = nt * 8 + 2 * t;
    const float w0 = M.w4[c], w1 = M.w4[c + 1];
    dh[nt][0] = dlo * w0;
    dh[nt][1] = dlo * w1;
    dh[nt][2] = dhi * w0;
    dh[nt][3] = dhi * w1;
    // dw4 partials: sum over the 16 rows of dy * H3
    float p0 = dlo * __bfloat162float(H3t[(size_t)c * B + r0 + g]) + dhi * __bfloat162float(H3t[(size_t)c * B + r0 + g + 8]);
    float p1 = dlo * __bfloat162float(H3t[(size_t)(c + 1) * B + r0 + g]) +
               dhi * __bfloat162float(H3t[(size_t)(c + 1) * B + r0 + g + 8]);
    for (int o = 4; o < 32; o <<= 1) {
      p0 += __shfl_xor_sync(0xffffffffu, p0, o);
      p1 += __shfl_xor_sync(0xffffffffu, p1, o);
    }
    if (g == 0) {
      atomicAdd(gw4 + c, p0);
      atomicAdd(gw4 + c + 1, p1);
    }
  }
  if (lane == 0) {
    float s = 0.f;
    for (int r = 0; r < 16; ++r) s += dy[r0 + r];
    atomicAdd(gb4, s);
  }
  uint32_t a[8][4];
  dz_from_dh(dh, Z3, B, r0, lane, dZ3t, a);
  back_product(a, W3t, lane, dh);
  dz_from_dh(dh, Z2, B, r0, lane, dZ2t, a);
  back_product(a, W2t, lane, dh);
  dz_from_dh(dh, Z1, B, r0, lane, dZ1t, a);
}

// dW[m][n] = sum_b At[m][b] Bt[n][b]  (At [M][K], Bt [N][K] rows of length K = batch)
__global__ void k_wgrad(const __nv_bfloat16* At, const __nv_bfloat16* Bt, int M, int N, int K, float* dW) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int ntn = N / 8;
  if (w >= (M / 16) * ntn) return;
  const int mt = w / ntn, nt = w % ntn;
  const int g = lane >> 2, t = lane & 3;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int ks = 0; ks < K / 16; ++ks) {
    uint32_t a[4];
    const __nv_bfloat16* p = At + (size_t)(mt * 16 + g) * K + ks * 16 + 2 * t;
    a[0] = *reinterpret_cast<const unsigned int*>(p);
    a[1] = *reinterpret_cast<const unsigned int*>(p + (size_t)8 * K);
    a[2] = *reinterpret_cast<const unsigned int*>(p + 8);
    a[3] = *reinterpret_cast<const unsigned int*>(p + (size_t)8 * K + 8);
    uint32_t b0, b1;
    load_b_frag(Bt, K, nt, ks, lane, b0, b1);
    mma_bf16_16816(acc, a, b0, b1);
  }
  const int r = mt * 16 + g, c = nt * 8 + 2 * t;
  dW[(size_t)r * N + c] = acc[0];
  dW[(size_t)r * N + c + 1] = acc[1];
  dW[(size_t)(r + 8) * N + c] = acc[2];
  dW[(size_t)(r + 8) * N + c + 1] = acc[3];
}

__global__ void k_bsum(const __nv_bfloat16* dZt, int B, float* db) {  // one warp per output neuron
  const int lane = threadIdx.x & 31;
  const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (j >= kMlpHidden) return;
  float s = 0.f;
  for (int b = lane; b < B; b += 32) s += __bfloat162float(dZt[(size_t)j * B + b]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) db[j] = s;
}

__global__ void k_adam(float* p, const float* gr, float* m1, float* m2, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = gr[i];
    m1[i] = b1 * m1[i] + (1.f - b1) * g;
    m2[i] = b2 * m2[i] + (1.f - b2) * g * g;
    p[i] -= lr * (m1[i] / c1) / (sqrtf(m2[i] / c2) + eps);
  }
}

// batch rows by index: dst[r] = src[idx[r]]
__global__ void k_gather(const float* __restrict__ feat, const float* __restrict__ tgt, const int64_t* __restrict__ idx,
                         int B, float* bf, float* bt) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B * kMlpIn; k += gridDim.x * blockDim.x) {
    const int r = k / kMlpIn, c = k % kMlpIn;
    const int64_t src = idx[r];
    bf[k] = feat[src * kMlpIn + c];
    if (c == 0) bt[r] = tgt[src];
  }
}

// BF16 copies of W1, W2, W3 and transposes of W2, W3
__global__ void k_publish(const float* p, __nv_bfloat16* W1, __nv_bfloat16* W2, __nv_bfloat16* W3, __nv_bfloat16* W2t,
                          __nv_bfloat16* W3t) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpHidden * kMlpHidden; i += gridDim.x * blockDim.x) {
    const int r = i / kMlpHidden, c = i % kMlpHidden;
    W2[i] = __float2bfloat16(p[kOffW2 + i]);
    W3[i] = __float2bfloat16(p[kOffW3 + i]);
    W2t[c * kMlpHidden + r] = __float2bfloat16(p[kOffW2 + i]);
    W3t[c * kMlpHidden + r] = __float2bfloat16(p[kOffW3 + i]);
    if (i < kMlpHidden * kMlpInPad) W1[i] = __float2bfloat16(p[kOffW1 + i]);
  }
}

// ---- stand-alone inference on tcgen05 (umma.cuh): 128-row tiles over the CTAs ----------
__global__ void __launch_bounds__(kTcThreads, 1) k_mlp_tc(MlpDev M, const float* __restrict__ feat, int n,
                                                          float* __restrict__ y, int* err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const uint32_t tmem = tc_net_setup(sm, M);
  uint32_t phase = 0;
  bool ok = true;
  const int ntiles = (n + kTcRows - 1) / kTcRows;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int r0 = tile * kTcRows;
    ok = tc_net_tile(
        sm, tmem, phase, M,
        [&](int r, int col) { return r0 + r < n ? feat[(size_t)(r0 + r) * kMlpIn + col] : 0.f; },
        [&](int r, float v) {
          if (r0 + r < n) y[r0 + r] = v;
        });
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
  }
  tc_net_teardown(sm, tmem, !ok, phase);
}

}  // namespace

// ---- host model ---------------------------------------------------------------------------
struct Model {
  int device = 0;
  float* p = nullptr;   // FP32 master parameters
  float* g = nullptr;   // gradients
  float* m1 = nullptr;  // Adam moments
  float* m2 = nullptr;
  __nv_bfloat16 *W1 = nullptr, *W2 = nullptr, *W3 = nullptr, *W2t = nullptr, *W3t = nullptr;
  float* norm = nullptr;  // fmean[16], fscale[16]
  float out_scale = 1.f;
  int64_t steps = 0;
  cudaStream_t stream = nullptr;

  MlpDev view() const {
    MlpDev d;
    d.W1 = W1;
    d.W2 = W2;
    d.W3 = W3;
    d.b1 = p + kOffB1;
    d.b2 = p + kOffB2;
    d.b3 = p + kOffB3;
    d.w4 = p + kOffW4;
    d.b4 = p + kOffB4;
    d.out_scale = out_scale;
    d.fmean = norm;
    d.fscale = norm + kMlpIn;
    return d;
  }
  void publish() {
    k_publish<<<64, 256, 0, stream>>>(p, W1, W2, W3, W2t, W3t);
    MM_CK(cudaGetLastError());
  }
  ~Model() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (void* q : {(void*)p, (void*)g, (void*)m1, (void*)m2, (void*)W1, (void*)W2, (void*)W3, (void*)W2t, (void*)W3t,
                    (void*)norm})
      if (q) cudaFree(q);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

template <class T>
void dal(T*& p, size_t n) {
  MM_CK(cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * (n ? n : 1)));
}

// Activations and gradients of one batch of B rows, allocated once per call.
struct Scratch {
  int B = 0;
  float *Z1 = nullptr, *Z2 = nullptr, *Z3 = nullptr, *dy = nullptr, *loss = nullptr;
  __nv_bfloat16 *H0t = nullptr, *H1t = nullptr, *H2t = nullptr, *H3t = nullptr;
  __nv_bfloat16 *dZ1t = nullptr, *dZ2t = nullptr, *dZ3t = nullptr;
  explicit Scratch(int b) : B(b) {
    const size_t H = kMlpHidden;
    dal(Z1, H * B);
    dal(Z2, H * B);
    dal(Z3, H * B);
    dal(dy, B);
    dal(loss, 1);
    dal(H0t, (size_t)kMlpInPad * B);
    dal(H1t, H * B);
    dal(H2t, H * B);
    dal(H3t, H * B);
    dal(dZ1t, H * B);
    dal(dZ2t, H * B);
    dal(dZ3t, H * B);
  }
  ~Scratch() {
    for (void* q : {(void*)Z1, (void*)Z2, (void*)Z3, (void*)dy, (void*)loss, (void*)H0t, (void*)H1t, (void*)H2t,
                    (void*)H3t, (void*)dZ1t, (void*)dZ2t, (void*)dZ3t})
      if (q) cudaFree(q);
  }
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
};

// Gradient of the batch loss (mean squared error in units of out_scale) into md.g; the
// loss is added to sc.loss.  All on md.stream, no host synchronisation.
void grad_batch(Model& md, Scratch& sc, const float* dfeat, const float* dtarget) {
  cudaStream_t st = md.stream;
  const int B = sc.B;
  MM_CK(cudaMemsetAsync(md.g, 0, sizeof(float) * kNumParams, st));
  const MlpDev M = md.view();
  const int warps = B / 16, tpb = 128;
  k_fwd<<<(warps * 32 + tpb - 1) / tpb, tpb, 0, st>>>(M, dfeat, dtarget, B, sc.Z1, sc.Z2, sc.Z3, sc.H0t, sc.H1t, sc.H2t,
                                                     sc.H3t, sc.dy, sc.loss);
  MM_CK(cudaGetLastError());
  k_bwd<<<(warps * 32 + tpb - 1) / tpb, tpb, 0, st>>>(M, md.W2t, md.W3t, B, sc.Z1, sc.Z2, sc.Z3, sc.H3t, sc.dy, sc.dZ1t,
                                                     sc.dZ2t, sc.dZ3t, md.g + kOffW4, md.g + kOffB4);
  MM_CK(cudaGetLastError());
  auto wg = [&](const __nv_bfloat16* At, const __nv_bfloat16* Bt, int Mr, int N, float* dW) {
    const int tiles = (Mr / 16) * (N / 8);
    k_wgrad<<<(tiles * 32 + 127) / 128, 128, 0, st>>>(At, Bt, Mr, N, B, dW);
    MM_CK(cudaGetLastError());
  };
  wg(sc.dZ3t, sc.H2t, kMlpHidden, kMlpHidden, md.g + kOffW3);
  wg(sc.dZ2t, sc.H1t, kMlpHidden, kMlpHidden, md.g + kOffW2);
  wg(sc.dZ1t, sc.H0t, kMlpHidden, kMlpInPad, md.g + kOffW1);
  k_bsum<<<(kMlpHidden * 32) / 128, 128, 0, st>>>(sc.dZ3t, B, md.g + kOffB3);
  k_bsum<<<(kMlpHidden * 32) / 128, 128, 0, st>>>(sc.dZ2t, B, md.g + kOffB2);
  k_bsum<<<(kMlpHidden * 32) / 128, 128, 0, st>>>(sc.dZ1t, B, md.g + kOffB1);
  MM_CK(cudaGetLastError());
}

void check_samples(const float* f, const float* t, int64_t n) {
  if (!f || n <= 0) throw std::runtime_error("empty sample set");
  for (int64_t i = 0; i < n * kMlpIn; ++i)
    if (!std::isfinite(f[i])) throw std::runtime_error("non-finite feature");
  if (t)
    for (int64_t i = 0; i < n; ++i)
      if (!std::isfinite(t[i])) throw std::runtime_error("non-finite target");
}

template <class T>
struct DevBuf {
  T* p = nullptr;
  explicit DevBuf(size_t n) { dal(p, n); }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

mm_status mfail(mm_status st, const std::string& s) {
  set_error(s);
  return st;
}
}  // namespace

MlpDev model_view(const mm_model* m);

}  // namespace mumag

struct mm_model {
  mumag::Model md;
};

mumag::MlpDev mumag::model_view(const mm_model* m) { return m->md.view(); }

using namespace mumag;

#define MAPI_BEGIN try {
#define MAPI_END                                \
  }                                             \
  catch (const mumag::CudaFailure& e) {         \
    return mfail(MM_CUDA_ERROR, e.what());      \
  }                                             \
  catch (const std::bad_alloc&) {               \
    return mfail(MM_BAD_INPUT, "host allocation failed"); \
  }                                             \
  catch (const std::exception& e) {             \
    return mfail(MM_BAD_INPUT, e.what());       \
  }

extern "C" {

mm_status mm_model_create(int32_t device, uint64_t seed, mm_model** out) {
  MAPI_BEGIN
  if (!out) throw std::runtime_error("NULL output");
  *out = nullptr;
  int ndev = 0;
  MM_CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) throw std::runtime_error("no such CUDA device");
  std::unique_ptr<mm_model> mo(new mm_model());
  Model& md = mo->md;
  md.device = device;
  MM_CK(cudaSetDevice(device));
  MM_CK(cudaStreamCreateWithFlags(&md.stream, cudaStreamNonBlocking));
  dal(md.p, kNumParams);
  dal(md.g, kNumParams);
  dal(md.m1, kNumParams);
  dal(md.m2, kNumParams);
  dal(md.W1, kMlpHidden * kMlpInPad);
  dal(md.W2, kMlpHidden * kMlpHidden);
  dal(md.W3, kMlpHidden * kMlpHidden);
  dal(md.W2t, kMlpHidden * kMlpHidden);
  dal(md.W3t, kMlpHidden * kMlpHidden);
  dal(md.norm, 2 * kMlpIn);
  // He initialisation of the hidden layers; a small head
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  std::vector<float> hp(kNumParams, 0.f);
  for (int r = 0; r < kMlpHidden; ++r)
    for (int c = 0; c < kMlpIn; ++c) hp[kOffW1 + r * kMlpInPad + c] = nd(rng) * std::sqrt(2.f / kMlpIn);
  for (int i = 0; i < kMlpHidden * kMlpHidden; ++i) {
    hp[kOffW2 + i] = nd(rng) * std::sqrt(2.f / kMlpHidden);
    hp[kOffW3 + i] = nd(rng) * std::sqrt(2.f / kMlpHidden);
  }
  for (int i = 0; i < kMlpHidden; ++i) hp[kOffW4 + i] = nd(rng) * std::sqrt(1.f / kMlpHidden) * 0.1f;
  std::vector<float> hn(2 * kMlpIn);
  for (int i = 0; i < kMlpIn; ++i) {
    hn[i] = 0.f;
    hn[kMlpIn + i] = 1.f;
  }
  MM_CK(cudaMemcpy(md.p, hp.data(), sizeof(float) * kNumParams, cudaMemcpyHostToDevice));
  MM_CK(cudaMemcpy(md.norm, hn.data(), sizeof(float) * 2 * kMlpIn, cudaMemcpyHostToDevice));
  MM_CK(cudaMemset(md.m1, 0, sizeof(float) * kNumParams));
  MM_CK(cudaMemset(md.m2, 0, sizeof(float) * kNumParams));
  md.publish();
  MM_CK(cudaStreamSynchronize(md.stream));
  *out = mo.release();
  return MM_OK;
  MAPI_END
}

mm_status mm_model_destroy(mm_model* m) {
  delete m;
  return MM_OK;
}

int64_t mm_model_num_params(void) { return kNumParams; }

mm_status mm_model_set_normalization(mm_model* mo, const float* fmean, const float* fscale, float out_scale) {
  MAPI_BEGIN
  if (!mo || !fmean || !fscale || !(out_scale > 0) || !std::isfinite(out_scale))
    throw std::runtime_error("invalid normalisation");
  std::vector<float> hn(2 * kMlpIn);
  for (int i = 0; i < kMlpIn; ++i) {
    if (!std::isfinite(fmean[i]) || !std::isfinite(fscale[i])) throw std::runtime_error("non-finite normalisation");
    hn[i] = fmean[i];
    hn[kMlpIn + i] = fscale[i];
  }
  Model& md = mo->md;
  md.out_scale = out_scale;
  MM_CK(cudaSetDevice(md.device));
  MM_CK(cudaStreamSynchronize(md.stream));
  MM_CK(cudaMemcpy(md.norm, hn.data(), sizeof(float) * 2 * kMlpIn, cudaMemcpyHostToDevice));
  return MM_OK;
  MAPI_END
}

mm_status mm_model_get_normalization(const mm_model* mo, float* fmean, float* fscale, float* out_scale) {
  MAPI_BEGIN
  if (!mo || !fmean || !fscale || !out_scale) throw std::runtime_error("NULL argument");
  const Model& md = mo->md;
  std::vector<float> hn(2 * kMlpIn);
  MM_CK(cudaSetDevice(md.device));
  MM_CK(cudaStreamSynchronize(md.stream));
  MM_CK(cudaMemcpy(hn.data(), md.norm, sizeof(float) * 2 * kMlpIn, cudaMemcpyDeviceToHost));
  for (int i = 0; i < kMlpIn; ++i) {
    fmean[i] = hn[i];
    fscale[i] = hn[kMlpIn + i];
  }
  *out_scale = md.out_scale;
  return MM_OK;
  MAPI_END
}

mm_status mm_model_fit_normalization(mm_model* mo, const float* feats, const float* target, int64_t n) {
  MAPI_BEGIN
  if (!mo || !target) throw std::runtime_error("NULL argument");
  check_samples(feats, target, n);
  std::vector<double> s(kMlpIn, 0.0), s2(kMlpIn, 0.0);
  double t2 = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    for (int c = 0; c < kMlpIn; ++c) {
      const double v = feats[i * kMlpIn + c];
      s[c] += v;
      s2[c] += v * v;
    }
    t2 += (double)target[i] * target[i];
  }
  float mean[kMlpIn], scale[kMlpIn];
  for (int c = 0; c < kMlpIn; ++c) {
    const double mu = s[c] / n, var = std::max(s2[c] / n - mu * mu, 0.0);
    mean[c] = (float)mu;
    scale[c] = var > 1e-24 ? (float)(1.0 / std::sqrt(var)) : 1.f;
  }
  const double rms = std::sqrt(t2 / n);
  return mm_model_set_normalization(mo, mean, scale, rms > 0 ? (float)rms : 1.f);
  MAPI_END
}

mm_status mm_model_get_params(mm_model* mo, float* params) {
  MAPI_BEGIN
  if (!mo || !params) throw std::runtime_error("NULL argument");
  MM_CK(cudaSetDevice(mo->md.device));
  MM_CK(cudaStreamSynchronize(mo->md.stream));
  MM_CK(cudaMemcpy(params, mo->md.p, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost));
  return MM_OK;
  MAPI_END
}

mm_status mm_model_set_params(mm_model* mo, const float* params) {
  MAPI_BEGIN
  if (!mo || !params) throw std::runtime_error("NULL argument");
  for (int i = 0; i < kNumParams; ++i)
    if (!std::isfinite(params[i])) throw std::runtime_error("non-finite parameter");
  Model& md = mo->md;
  MM_CK(cudaSetDevice(md.device));
  MM_CK(cudaStreamSynchronize(md.stream));
  MM_CK(cudaMemcpy(md.p, params, sizeof(float) * kNumParams, cudaMemcpyHostToDevice));
  MM_CK(cudaMemset(md.m1, 0, sizeof(float) * kNumParams));
  MM_CK(cudaMemset(md.m2, 0, sizeof(float) * kNumParams));
  md.steps = 0;
  md.publish();
  MM_CK(cudaStreamSynchronize(md.stream));
  return MM_OK;
  MAPI_END
}

mm_status mm_model_grad(mm_model* mo, const float* feats, const float* target, int32_t n, float* grads, float* loss) {
  MAPI_BEGIN
  if (!mo || !target || n <= 0 || n % 16) throw std::runtime_error("n must be a positive multiple of 16");
  check_samples(feats, target, n);
  Model& md = mo->md;
  MM_CK(cudaSetDevice(md.device));
  DevBuf<float> df((size_t)n * kMlpIn), dt(n);
  Scratch sc(n);
  MM_CK(cudaMemcpyAsync(df.p, feats, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice, md.stream));
  MM_CK(cudaMemcpyAsync(dt.p, target, sizeof(float) * n, cudaMemcpyHostToDevice, md.stream));
  MM_CK(cudaMemsetAsync(sc.loss, 0, sizeof(float), md.stream));
  grad_batch(md, sc, df.p, dt.p);
  float l = 0.f;
  MM_CK(cudaMemcpyAsync(&l, sc.loss, sizeof(float), cudaMemcpyDeviceToHost, md.stream));
  if (grads) MM_CK(cudaMemcpyAsync(grads, md.g, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost, md.stream));
  MM_CK(cudaStreamSynchronize(md.stream));
  if (loss) *loss = l;
  return MM_OK;
  MAPI_END
}

mm_status mm_model_train(mm_model* mo, const float* feats, const float* target, int64_t n, int32_t epochs,
                         int32_t batch, float lr, uint64_t seed, float* final_loss) {
  MAPI_BEGIN
  if (!mo || !target || n < 16 || epochs < 1 || batch < 16 || batch % 16 || !(lr > 0))
    throw std::runtime_error("invalid training arguments");
  check_samples(feats, target, n);
  Model& md = mo->md;
  MM_CK(cudaSetDevice(md.device));
  const int B = (int)std::min<int64_t>(batch, (n / 16) * 16);
  const int64_t nb = n / B;  // full batches per epoch
  DevBuf<float> df((size_t)n * kMlpIn), dt(n), bf((size_t)B * kMlpIn), bt(B);
  DevBuf<int64_t> didx((size_t)nb * B);
  Scratch sc(B);
  MM_CK(cudaMemcpyAsync(df.p, feats, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice, md.stream));
  MM_CK(cudaMemcpyAsync(dt.p, target, sizeof(float) * n, cudaMemcpyHostToDevice, md.stream));
  std::mt19937_64 rng(seed);
  std::vector<int64_t> order(n);
  for (int64_t i = 0; i < n; ++i) order[i] = i;
  float last = 0.f;
  const float b1 = 0.9f, b2 = 0.999f;
  for (int e = 0; e < epochs; ++e) {
    std::shuffle(order.begin(), order.end(), rng);
    MM_CK(cudaStreamSynchronize(md.stream));  // the previous epoch's index upload is consumed
    MM_CK(cudaMemcpyAsync(didx.p, order.data(), sizeof(int64_t) * nb * B, cudaMemcpyHostToDevice, md.stream));
    MM_CK(cudaMemsetAsync(sc.loss, 0, sizeof(float), md.stream));
    for (int64_t bi = 0; bi < nb; ++bi) {
      k_gather<<<64, 256, 0, md.stream>>>(df.p, dt.p, didx.p + bi * B, B, bf.p, bt.p);
      MM_CK(cudaGetLastError());
      grad_batch(md, sc, bf.p, bt.p);
      md.steps += 1;
      const float c1 = 1.f - std::pow(b1, (float)md.steps), c2 = 1.f - std::pow(b2, (float)md.steps);
      k_adam<<<64, 256, 0, md.stream>>>(md.p, md.g, md.m1, md.m2, kNumParams, lr, b1, b2, 1e-8f, c1, c2);
      MM_CK(cudaGetLastError());
      md.publish();
    }
    float l = 0.f;
    MM_CK(cudaMemcpyAsync(&l, sc.loss, sizeof(float), cudaMemcpyDeviceToHost, md.stream));
    MM_CK(cudaStreamSynchronize(md.stream));
    last = l / (float)nb;
    if (!std::isfinite(last)) throw std::runtime_error("training diverged (non-finite loss)");
  }
  if (final_loss) *final_loss = last;
  return MM_OK;
  MAPI_END
}

mm_status mm_model_predict(mm_model* mo, const float* feats, int64_t n, float* y) {
  MAPI_BEGIN
  if (!mo || !y) throw std::runtime_error("NULL argument");
  check_samples(feats, nullptr, n);
  if (n > (int64_t)1 << 30) throw std::runtime_error("too many rows");
  Model& md = mo->md;
  MM_CK(cudaSetDevice(md.device));
  DevBuf<float> df((size_t)n * kMlpIn), dd(n);
  DevBuf<int> derr(1);
  MM_CK(cudaMemsetAsync(derr.p, 0, sizeof(int), md.stream));
  MM_CK(cudaMemcpyAsync(df.p, feats, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice, md.stream));
  static bool attr_set[64] = {};
  if (md.device < 64 && !attr_set[md.device]) {
    MM_CK(cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmTc));
    attr_set[md.device] = true;
  }
  cudaDeviceProp prop;
  MM_CK(cudaGetDeviceProperties(&prop, md.device));
  const int64_t tiles = (n + kTcRows - 1) / kTcRows;
  const int grid = (int)std::min<int64_t>(tiles, 2 * (int64_t)prop.multiProcessorCount);
  k_mlp_tc<<<grid, kTcThreads, kSmTc, md.stream>>>(md.view(), df.p, (int)n, dd.p, derr.p);
  MM_CK(cudaGetLastError());
  int herr = 0;
  MM_CK(cudaMemcpyAsync(y, dd.p, sizeof(float) * n, cudaMemcpyDeviceToHost, md.stream));
  MM_CK(cudaMemcpyAsync(&herr, derr.p, sizeof(int), cudaMemcpyDeviceToHost, md.stream));
  MM_CK(cudaStreamSynchronize(md.stream));
  if (herr) return mfail(MM_TIMEOUT, "the tensor-core inference kernel timed out waiting for its products");
  return MM_OK;
  MAPI_END
}

}  // extern "C"

// Training and stand-alone inference of the warm-start MLP (mlp.cuh), plus its C ABI.
//
// One training step on a batch of B samples (B a multiple of 16):
//   k_train_tc  the gradient on the 5th-generation tensor cores (mlp_train_tc.cuh): one CTA
//               per 128-row tile, forward with the pre-activations kept in TMEM, backward
//               products dZ W and weight gradients dZ^T H as tcgen05 MMAs, loss
//               1/B sum (y - t/out_scale)^2
//   k_adam      Adam on FP32 master weights, then BF16 copies and transposes (k_publish)
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
#include "mlp_train_tc.cuh"
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

// A tensor-core product of the training kernel did not complete within its wait limit.
struct TrainTimeout : std::runtime_error {
  TrainTimeout() : std::runtime_error("the tensor-core training kernel timed out waiting for its products") {}
};

namespace {

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

// Per-call buffers of the training kernels: the loss accumulator and the error flag of the
// bounded tensor-core waits.
struct Scratch {
  int B = 0;
  float* loss = nullptr;
  int* err = nullptr;
  explicit Scratch(int b) : B(b) {
    dal(loss, 1);
    dal(err, 1);
    MM_CK(cudaMemset(err, 0, sizeof(int)));
  }
  ~Scratch() {
    if (loss) cudaFree(loss);
    if (err) cudaFree(err);
  }
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
};

// Gradient of the batch loss (mean squared error in units of out_scale) into md.g on the
// tensor cores (k_train_tc, one CTA per 128 rows); the loss is added to sc.loss.  All on
// md.stream, no host synchronisation.
void grad_batch(Model& md, Scratch& sc, const float* dfeat, const float* dtarget) {
  cudaStream_t st = md.stream;
  const int B = sc.B;
  static bool attr_set[64] = {};
  if (md.device < 64 && !attr_set[md.device]) {
    MM_CK(cudaFuncSetAttribute(k_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmTrain));
    attr_set[md.device] = true;
  }
  MM_CK(cudaMemsetAsync(md.g, 0, sizeof(float) * kNumParams, st));
  k_train_tc<<<(B + kTcRows - 1) / kTcRows, kTcThreads, kSmTrain, st>>>(
      md.view(), md.W2t, md.W3t, dfeat, dtarget, B, md.g, kOffW1, kOffB1, kOffW2, kOffB2, kOffW3, kOffB3, kOffW4,
      kOffB4, sc.loss, sc.err);
  MM_CK(cudaGetLastError());
}

// The training kernels' bounded waits: a product that did not complete is reported.
void check_train(Scratch& sc, cudaStream_t st) {
  int e = 0;
  MM_CK(cudaMemcpyAsync(&e, sc.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MM_CK(cudaStreamSynchronize(st));
  if (e) throw TrainTimeout();
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
  catch (const mumag::TrainTimeout& e) {        \
    return mfail(MM_TIMEOUT, e.what());         \
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
  check_train(sc, md.stream);
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
    check_train(sc, md.stream);
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

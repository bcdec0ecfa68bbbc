// mm_poisson_pcg_noalloc: the Jacobi-preconditioned CG solve of the magnetostatic Poisson
// system for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at all: plug-ins living inside a host application
// that owns every device byte through its own pool (a cudaMalloc of theirs would take memory
// the host has already promised elsewhere, or fail), and long-running services that
// pre-allocate at start-up and then forbid allocation on the serving path (an allocation
// there can stall every stream of the device and fragments memory over hours).  They hold their matrix and vectors in memory they already own and need
// a solve that takes nothing more.  This entry point takes a CSR matrix, a right-hand side
// and an initial guess (all device pointers the caller owns) and keeps every intermediate
// vector, reduction partial and barrier counter in one file-scope static device array,
// g_pcg_scratch below.
//
// Limits and sharing rules:
//  * at most kMaxRows = 65,536 rows (about 4.8 MB of static device memory, held by every
//    GPU that loads the library until the process exits); larger systems are rejected
//    with MM_BAD_INPUT;
//  * every call on a device uses the same array and leaves its contents behind; the call
//    clears what must start at zero (barrier counter, status, iteration count) itself;
//  * calls whose work overlaps on the GPU (two host threads, or two streams, at once) race
//    on the array and produce garbage; serialise them;
//  * the first call on a device does a one-time set-up on that device (looks up the array's
//    device address with cudaGetSymbolAddress and queries the occupancy of the kernel); make
//    that first call before any stream capture;
//  * the call is synchronous: it waits for its work on `stream` to finish and returns the
//    status, the iteration count and the result in x.
//
// Bad input is reported, never dereferenced: a row pointer or column outside the matrix,
// and a row whose diagonal is missing, zero or not finite (the Jacobi preconditioner
// divides by it), make the call return MM_BAD_INPUT before any iteration.
//
// The iteration is the same as the mesh path's Poisson PCG (the reference's
// jax.scipy.sparse.linalg.cg, scripts/solvers.py:221-231): z = r * (1/diag A), stop when
// r.r <= tol^2 b.b or after max_iter iterations, in the single-reduction Chronopoulos-Gear
// arrangement, one thread per CSR row.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <mutex>
#include <string>

#include "../../include/mumag_b200.h"
#include "mumag_internal.h"

namespace mumag {
namespace {

constexpr int kMaxRows = 65536;
constexpr int kMaxCtas = 256;
constexpr int kRed = 4;
constexpr int kThreads = 256;
constexpr unsigned kSpin = 1u << 23;

// layout of the scratch array (byte offsets, every part 256-byte aligned)
constexpr size_t kOffCtl = 0;                                        // u64 bar, int flags[2], ll iters
constexpr size_t kOffRed = 256;                                      // double [2][kRed][kMaxCtas]
constexpr size_t kOffRec = kOffRed + sizeof(double) * 2 * kRed * kMaxCtas;  // double4 [2][kMaxRows]
constexpr size_t kOffP = kOffRec + sizeof(double) * 4 * 2 * kMaxRows;       // double [kMaxRows]
constexpr size_t kScratchBytes = kOffP + sizeof(double) * kMaxRows;

static __device__ __align__(256) unsigned char g_pcg_scratch[kScratchBytes];

struct Ctl {
  unsigned long long bar;
  int flags[2];  // abort, status
  long long iters;  // iterations completed (kept current, so a timed-out call reports them too)
  int bad;          // kind of bad input: 1 = row pointers or columns, 2 = diagonal
  int pad;
};
static_assert(sizeof(Ctl) <= kOffRed, "control block overlaps the reduction partials");

// Test hook: extra arrivals every barrier of the next calls waits for (0 = none; 1 makes
// every wait run out, so a call returns MM_TIMEOUT without a fault).  Set through
// mm_debug_stall_barriers(NULL, stall).
int g_noalloc_stall = 0;

__device__ __forceinline__ unsigned long long ld_acq(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_rel(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

struct GridSync {
  Ctl* ctl;
  double* red;
  unsigned long long epoch;
  int slot;
  int stall;
};

__device__ bool barrier(GridSync& g) {
  __shared__ int ab;
  __syncthreads();
  if (threadIdx.x == 0) {
    g.epoch += 1;
    const unsigned long long target = g.epoch * gridDim.x + (unsigned long long)g.stall;
    red_rel(&g.ctl->bar, 1ull);
    int a = 0;
    for (unsigned it = 0; ld_acq(&g.ctl->bar) < target; ++it) {
      if ((it & 63) == 63 && *((volatile int*)&g.ctl->flags[0])) {
        a = 1;
        break;
      }
      if (it > kSpin) {
        atomicCAS(&g.ctl->flags[1], 0, (int)MM_TIMEOUT);
        atomicExch(&g.ctl->flags[0], 1);
        a = 1;
        break;
      }
      if (it > 64) __nanosleep(it > 8192 ? 256 : 16);
    }
    ab = a;
  }
  __syncthreads();
  return ab == 0;
}

// deterministic sum of K values over the grid (CTA order), also a barrier
template <int K>
__device__ bool reduce(GridSync& g, double (&v)[K]) {
  __shared__ double sh[kThreads / 32][kRed];
  __shared__ double res[kRed];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < K; ++k) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sh[warp][k] = x;
  }
  __syncthreads();
  double* set = g.red + (size_t)g.slot * kRed * kMaxCtas;
  if (threadIdx.x < K) {
    double a = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) a += sh[w][threadIdx.x];
    set[threadIdx.x * kMaxCtas + blockIdx.x] = a;
  }
  if (!barrier(g)) return false;
  if (warp < K) {
    double a = 0.0;
    for (int b = lane; b < (int)gridDim.x; b += 32) a += __ldcg(set + warp * kMaxCtas + b);
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) res[warp] = a;
  }
  __syncthreads();
  for (int k = 0; k < K; ++k) v[k] = res[k];
  g.slot ^= 1;
  return true;
}

struct Rec {
  double r, w, s, invd;  // r_i, w_i = A z_i, s_{i-1}, 1/diag
};

__device__ __forceinline__ double znext(const Rec& q, double alpha, double beta, double* s_out, double* r_out) {
  const double s = q.w + beta * q.s;
  const double r = q.r - alpha * s;
  if (s_out) *s_out = s;
  if (r_out) *r_out = r;
  return r * q.invd;
}

__global__ void __launch_bounds__(kThreads, 1)
    k_pcg_csr(int n, int nnz, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
              const double* __restrict__ av, const double* __restrict__ b, double* x, double tol, int max_iter,
              unsigned char* scratch, int stall) {
  Ctl* ctl = reinterpret_cast<Ctl*>(scratch + kOffCtl);
  Rec* rec[2] = {reinterpret_cast<Rec*>(scratch + kOffRec), reinterpret_cast<Rec*>(scratch + kOffRec) + kMaxRows};
  double* pv = reinterpret_cast<double*>(scratch + kOffP);
  GridSync g{ctl, reinterpret_cast<double*>(scratch + kOffRed), 0ull, 0, stall};
  const int r0 = (int)(((long long)n * blockIdx.x) / gridDim.x);
  const int r1 = (int)(((long long)n * (blockIdx.x + 1)) / gridDim.x);
  // validate this CTA's rows: 0 <= rp[i] <= rp[i+1] <= nnz, every column in [0, n), and a
  // diagonal (the sum of the row's entries in column i) that is present, nonzero and finite;
  // rows that fail are skipped and reported as MM_BAD_INPUT
  for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const int e0 = rp[i], e1 = rp[i + 1];
    bool ok = 0 <= e0 && e0 <= e1 && e1 <= nnz;
    for (int e = ok ? e0 : 0; ok && e < e1; ++e) ok = 0 <= ci[e] && ci[e] < n;
    if (!ok) {
      atomicCAS(&ctl->bad, 0, 1);
      atomicCAS(&ctl->flags[1], 0, (int)MM_BAD_INPUT);
      continue;
    }
    double d = 0.0;
    bool has = false;
    for (int e = e0; e < e1; ++e)
      if (ci[e] == i) {
        d += av[e];
        has = true;
      }
    if (!has || !(d != 0.0) || !isfinite(d)) {
      atomicCAS(&ctl->bad, 0, 2);
      atomicCAS(&ctl->flags[1], 0, (int)MM_BAD_INPUT);
    }
  }
  // r0 = b - A x0, z0 = r0 / diag
  double gamma, rr, bb;
  {
    double v[3] = {0, 0, 0};
    if (!barrier(g)) return;
    if (*((volatile int*)&ctl->flags[1]) != 0) return;  // same decision in every CTA after the barrier
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      double ax = 0.0, d = 0.0;
      for (int e = rp[i]; e < rp[i + 1]; ++e) {
        const int j = ci[e];
        ax += av[e] * x[j];
        if (j == i) d += av[e];
      }
      const double invd = 1.0 / d;
      const double r = b[i] - ax;
      rec[0][i] = Rec{r, 0.0, 0.0, invd};
      pv[i] = 0.0;
      v[0] += r * (r * invd);
      v[1] += r * r;
      v[2] += b[i] * b[i];
    }
    if (!reduce<3>(g, v)) return;
    gamma = v[0];
    rr = v[1];
    bb = v[2];
  }
  const double atol2 = tol * tol * bb;
  int k = 0;
  if (rr > atol2 && k < max_iter) {
    double delta;
    {
      double v[1] = {0};
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        double w = 0.0;
        for (int e = rp[i]; e < rp[i + 1]; ++e) {
          const int j = ci[e];
          w += av[e] * (rec[0][j].r * rec[0][j].invd);
        }
        rec[0][i].w = w;
        v[0] += w * (rec[0][i].r * rec[0][i].invd);
      }
      if (!reduce<1>(g, v)) return;
      delta = v[0];
    }
    double alpha = gamma / delta, beta = 0.0;
    for (int it = 0;; ++it) {
      const int cur = it & 1, nxt = cur ^ 1;
      double v[3] = {0, 0, 0};
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        double w = 0.0;
        for (int e = rp[i]; e < rp[i + 1]; ++e) w += av[e] * znext(rec[cur][ci[e]], alpha, beta, nullptr, nullptr);
        const Rec q = rec[cur][i];
        double s, r;
        const double z = znext(q, alpha, beta, &s, &r);
        const double p = q.r * q.invd + beta * pv[i];
        pv[i] = p;
        x[i] = x[i] + alpha * p;
        rec[nxt][i] = Rec{r, w, s, q.invd};
        v[0] += r * z;
        v[1] += w * z;
        v[2] += r * r;
      }
      if (!reduce<3>(g, v)) return;
      ++k;
      if (blockIdx.x == 0 && threadIdx.x == 0) ctl->iters = k;
      rr = v[2];
      if (!(rr > atol2 && k < max_iter)) break;
      const double bn = v[0] / gamma;
      alpha = v[0] / (v[1] - bn * v[0] / alpha);
      beta = bn;
      gamma = v[0];
    }
  }
}

// one-time set-up per device: the scratch array's device address and the launch shape
struct DeviceSetup {
  bool done = false;
  unsigned char* scratch = nullptr;
  int grid = 0;
};
std::mutex g_setup_mu;
DeviceSetup g_setup[64];

mm_status setup_device(int dev, DeviceSetup*& out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (dev < 0 || dev >= 64) {
    set_error("device ordinal out of range");
    return MM_BAD_INPUT;
  }
  DeviceSetup& s = g_setup[dev];
  if (!s.done) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_pcg_scratch);
    if (e != cudaSuccess) {
      set_error(std::string("cudaGetSymbolAddress(g_pcg_scratch): ") + cudaGetErrorString(e));
      return MM_CUDA_ERROR;
    }
    int sms = 0, occ = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pcg_csr, kThreads, 0);
    if (e != cudaSuccess || occ < 1) {
      set_error(std::string("occupancy query of the no-alloc PCG kernel failed: ") + cudaGetErrorString(e));
      return MM_CUDA_ERROR;
    }
    s.scratch = static_cast<unsigned char*>(p);
    s.grid = std::min(kMaxCtas, sms * occ);
    s.done = true;
  }
  out = &s;
  return MM_OK;
}

}  // namespace
}  // namespace mumag

extern "C" mm_status mm_poisson_pcg_noalloc(int32_t n, int32_t nnz, const int32_t* row_ptr, const int32_t* col,
                                            const double* val, const double* b, double* x, double tol,
                                            int32_t max_iter, int32_t* iters, void* stream) {
  using namespace mumag;
  if (iters) *iters = 0;
  if (n <= 0 || n > kMaxRows) {
    set_error("mm_poisson_pcg_noalloc: n = " + std::to_string(n) + " rows is outside [1, " +
              std::to_string(kMaxRows) + "], the size of its static scratch");
    return MM_BAD_INPUT;
  }
  if (nnz < 0 || !row_ptr || !col || !val || !b || !x) {
    set_error("mm_poisson_pcg_noalloc: NULL device pointer");
    return MM_BAD_INPUT;
  }
  if (!(tol >= 0.0) || max_iter < 0) {
    set_error("mm_poisson_pcg_noalloc: tol must be >= 0 and max_iter >= 0");
    return MM_BAD_INPUT;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return MM_CUDA_ERROR;
  }
  DeviceSetup* ds = nullptr;
  mm_status st = setup_device(dev, ds);
  if (st != MM_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int grid = std::max(1, std::min(ds->grid, (n + 31) / 32));
  // clear what must start at zero: barrier counter, abort/status flags, iteration count
  e = cudaMemsetAsync(ds->scratch + kOffCtl, 0, sizeof(Ctl), s);
  if (e == cudaSuccess) {
    unsigned char* sc = ds->scratch;
    int stall = g_noalloc_stall;
    void* args[] = {&n, &nnz, (void*)&row_ptr, (void*)&col, (void*)&val, (void*)&b, &x, &tol, &max_iter, &sc, &stall};
    e = cudaLaunchCooperativeKernel((const void*)k_pcg_csr, dim3(grid), dim3(kThreads), args, 0, s);
  }
  Ctl ctl{};
  if (e == cudaSuccess) e = cudaMemcpyAsync(&ctl, ds->scratch + kOffCtl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_error(std::string("mm_poisson_pcg_noalloc: ") + cudaGetErrorString(e));
    return MM_CUDA_ERROR;
  }
  if (iters) *iters = (int32_t)ctl.iters;
  if (ctl.flags[1] == MM_TIMEOUT) {
    set_error("mm_poisson_pcg_noalloc: a grid barrier timed out after " + std::to_string(ctl.iters) +
              " iterations");
    return MM_TIMEOUT;
  }
  if (ctl.flags[1] == MM_BAD_INPUT) {
    set_error(ctl.bad == 2 ? "mm_poisson_pcg_noalloc: a row's diagonal is missing, zero or not finite"
                           : "mm_poisson_pcg_noalloc: CSR row pointers or column indices out of range");
    return MM_BAD_INPUT;
  }
  if (ctl.flags[1] != MM_OK) {
    set_error("mm_poisson_pcg_noalloc: the kernel left an invalid status word");
    return MM_CUDA_ERROR;
  }
  return MM_OK;
}

namespace mumag {
void set_noalloc_stall(int stall) { g_noalloc_stall = stall; }
}  // namespace mumag

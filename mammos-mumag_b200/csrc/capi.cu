// C ABI of libmumag_b200.so (include/mumag_b200.h): mesh lifecycle, state transfer between
// the reference's layout (interleaved m, mesh-file node order) and the device layout
// (component planes, reverse Cuthill-McKee order), and the field-sweep driver that
// replaces scripts/loop.py:71-142.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <tuple>
#include <stdexcept>
#include <string>
#include <vector>

#include "device_mesh.h"

struct mm_mesh {
  mumag::DevMesh dm;
};

struct mm_batch {
  std::vector<mm_mesh*> meshes;
  mumag::BatchPlan plan;
  int device = 0;
  cudaStream_t stream = nullptr;
  mumag::SolveArgs* d_args = nullptr;
  int* d_group = nullptr;
  std::vector<mumag::SolveArgs> h_args;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace mumag {

namespace {
thread_local std::string g_error;

template <class T>
void dalloc(T*& p, size_t n) {
  MM_CK(cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * (n ? n : 1)));
}
template <class T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}
template <class T>
void upload(T* d, const std::vector<T>& h, cudaStream_t st) {
  if (!h.empty()) MM_CK(cudaMemcpyAsync(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, st));
}

// file-order interleaved [3N] <-> device planes [3][Npad]
void to_planes(const DevMesh& m, const double* in, std::vector<double>& out) {
  const auto& h = m.h;
  out.assign(3 * h.Npad, 0.0);
  for (int64_t i = 0; i < h.N; ++i)
    for (int q = 0; q < 3; ++q) out[q * h.Npad + h.iperm[i]] = in[3 * i + q];
}
void from_planes(const DevMesh& m, const std::vector<double>& in, double* out) {
  const auto& h = m.h;
  for (int64_t i = 0; i < h.N; ++i)
    for (int q = 0; q < 3; ++q) out[3 * i + q] = in[q * h.Npad + h.iperm[i]];
}
void to_nodes(const DevMesh& m, const double* in, std::vector<double>& out) {
  out.assign(m.h.Npad, 0.0);
  for (int64_t i = 0; i < m.h.N; ++i) out[m.h.iperm[i]] = in[i];
}
void from_nodes(const DevMesh& m, const std::vector<double>& in, double* out) {
  for (int64_t i = 0; i < m.h.N; ++i) out[i] = in[m.h.iperm[i]];
}
void d2h(std::vector<double>& h, const double* d, size_t n, cudaStream_t st) {
  h.resize(n);
  MM_CK(cudaMemcpyAsync(h.data(), d, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  MM_CK(cudaStreamSynchronize(st));
}

// Device-resident state transfers: the reference's layout (interleaved m [3N], u [N], mesh-file
// order) to the device layout (component planes, device row order) and back, one thread per
// node.  A non-finite input value raises *bad (the host form refuses it the same way).
__global__ void k_state_in(const double* __restrict__ m, const double* __restrict__ u,
                           const double* __restrict__ mb, const int32_t* __restrict__ iperm, int64_t N, int64_t np,
                           double* x, double* ud, double* mbd, int* bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = iperm[i];
    for (int q = 0; q < 3; ++q) {
      const double v = m[3 * i + q], w = mb ? mb[3 * i + q] : v;
      if (!isfinite(v) || !isfinite(w)) *bad = 1;
      x[q * np + j] = v;
      mbd[q * np + j] = w;
    }
    const double uv = u ? u[i] : 0.0;
    if (!isfinite(uv)) *bad = 1;
    ud[j] = uv;
  }
}
__global__ void k_state_out(const double* __restrict__ x, const double* __restrict__ ud,
                            const double* __restrict__ gf, const int32_t* __restrict__ iperm, int64_t N, int64_t np,
                            double* m, double* u, double* g) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = iperm[i];
    for (int q = 0; q < 3; ++q) {
      if (m) m[3 * i + q] = x[q * np + j];
      if (g) g[3 * i + q] = gf[q * np + j];
    }
    if (u) u[i] = ud[j];
  }
}

void ensure_iperm(DevMesh& m) {
  if (m.d_iperm) return;
  dalloc(m.d_iperm, m.h.N);
  dalloc(m.d_bad, 1);
  upload(m.d_iperm, m.h.iperm, m.stream);
}

void release(DevMesh& m) {
  if (m.device >= 0) cudaSetDevice(m.device);
  dfree(m.sl_off);
  dfree(m.sl_w);
  dfree(m.col);
  dfree(m.rowlen);
  dfree(m.vals);
  dfree(m.vals32);
  dfree(m.diagS);
  dfree(m.invdS);
  dfree(m.Dex);
  dfree(m.meas);
  dfree(m.bnd);
  dfree(m.Xd);
  dfree(m.econn);
  dfree(m.etag);
  dfree(m.dmats);
  dfree(m.ws);
  dfree(m.bar);
  dfree(m.red);
  dfree(m.flags);
  dfree(m.resd);
  dfree(m.resi);
  dfree(m.prof);
  dfree(m.feat);
  dfree(m.du);
  dfree(m.rs_feat);
  dfree(m.rs_tgt);
  dfree(m.rs_u0);
  dfree(m.rs_node);
  dfree(m.rs_slot);
  dfree(m.rs_count);
  dfree(m.rbox);
  dfree(m.Ainv);
  dfree(m.Ainv32);
  dfree(m.bslots);
  dfree(m.bslot);
  dfree(m.ctabox);
  dfree(m.d_iperm);
  dfree(m.d_bad);
  if (m.h_resd) cudaFreeHost(m.h_resd);
  if (m.h_resi) cudaFreeHost(m.h_resi);
  if (m.h_flags) cudaFreeHost(m.h_flags);
  m.h_resd = nullptr;
  m.h_resi = nullptr;
  m.h_flags = nullptr;
  if (m.evk0) cudaEventDestroy(m.evk0);
  if (m.evk1) cudaEventDestroy(m.evk1);
  m.evk0 = m.evk1 = nullptr;
  if (m.ev0) cudaEventDestroy(m.ev0);
  if (m.ev1) cudaEventDestroy(m.ev1);
  m.ev0 = m.ev1 = nullptr;
  if (m.stream) cudaStreamDestroy(m.stream);
  m.stream = nullptr;
}

// Process-wide cache of the host preprocessing (node order, SELL pattern, element colouring,
// boundary branch, aggregate boxes) and of the coarse inverse, keyed by the exact mesh input
// and the options that shape it -- the counterpart of the reference's scripts/store.py,
// which pickles escript's assembled arrays so a rerun skips the set-up.  Entries compare the
// full input (a 64-bit hash first), so a hit is exact; the last kPrepCache meshes are kept.
constexpr size_t kPrepCache = 4;
struct PrepEntry {
  uint64_t hash = 0;
  int reorder = 0, coarse = 0;
  std::vector<double> X;
  std::vector<int32_t> T, tag;
  HostMesh h;
  std::vector<double> Ainv;  // filled by the first build_coarse of this mesh
};
std::mutex g_prep_mu;
std::list<std::shared_ptr<PrepEntry>> g_prep;  // most recent first

uint64_t hash_bytes(uint64_t h, const void* p, size_t n) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  size_t k = 0;
  for (; k + 8 <= n; k += 8) {
    uint64_t w;
    std::memcpy(&w, b + k, 8);
    h = (h ^ w) * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
  }
  for (; k < n; ++k) h = (h ^ b[k]) * 0x100000001B3ull;
  return h;
}

std::shared_ptr<PrepEntry> prep_find(uint64_t hash, const double* X, int64_t N, const int32_t* T, const int32_t* tag,
                                     int64_t E, int reorder, int coarse) {
  std::lock_guard<std::mutex> lk(g_prep_mu);
  for (auto it = g_prep.begin(); it != g_prep.end(); ++it) {
    const PrepEntry& e = **it;
    if (e.hash != hash || e.reorder != reorder || e.coarse != coarse || (int64_t)e.X.size() != 3 * N ||
        (int64_t)e.tag.size() != E)
      continue;
    if (std::memcmp(e.X.data(), X, sizeof(double) * 3 * N) || std::memcmp(e.T.data(), T, sizeof(int32_t) * 4 * E) ||
        std::memcmp(e.tag.data(), tag, sizeof(int32_t) * E))
      continue;
    auto hit = *it;
    g_prep.erase(it);
    g_prep.push_front(hit);
    return hit;
  }
  return nullptr;
}

void prep_store(std::shared_ptr<PrepEntry> e) {
  std::lock_guard<std::mutex> lk(g_prep_mu);
  g_prep.push_front(std::move(e));
  while (g_prep.size() > kPrepCache) g_prep.pop_back();
}

// The two-level preconditioner's coarse operator: Ac = P^T S P summed on the host from the
// assembled Poisson plane (rows in device order, so the sums are deterministic), inverted
// densely (banded Cholesky; Ac couples only neighbouring boxes), uploaded in FP64 and FP32.
void build_coarse(DevMesh& m, std::vector<double>* cached) {
  const HostMesh& h = m.h;
  const int nc = h.nc;
  m.nc = nc;
  if (nc <= 0) return;
  std::vector<double> A;
  {
    std::lock_guard<std::mutex> lk(g_prep_mu);
    if (cached && cached->size() == (size_t)nc * nc) A = *cached;
  }
  if (A.empty()) {
    std::vector<double> S;
    d2h(S, m.vals + (size_t)P_S * h.nent, h.nent, m.stream);
    A.assign((size_t)nc * nc, 0.0);
    int32_t bw = 0;
    for (int64_t s = 0; s < h.nslices; ++s)
      for (int l = 0; l < kSlice; ++l) {
        const int64_t i = s * kSlice + l;
        if (i >= h.N || h.rbox[i] < 0) continue;
        const int32_t ci = h.rbox[i];
        for (int32_t k = 0; k < h.rowlen[i]; ++k) {
          const int64_t e = h.sl_off[s] + (int64_t)k * kSlice + l;
          const int32_t cj = h.rbox[h.col[e]];
          if (cj < 0) continue;
          A[(size_t)ci * nc + cj] += S[e];
          bw = std::max(bw, std::abs(ci - cj));
        }
      }
    spd_inverse(nc, bw, A);
    if (cached) {
      std::lock_guard<std::mutex> lk(g_prep_mu);
      *cached = A;
    }
  }
  std::vector<float> A32(A.size());
  for (size_t q = 0; q < A.size(); ++q) A32[q] = (float)A[q];
  dalloc(m.rbox, h.Npad);
  dalloc(m.Ainv, A.size());
  dalloc(m.Ainv32, A32.size());
  dalloc(m.bslots, (size_t)nc + kMaxGrid);
  dalloc(m.bslot, (size_t)nc + 1);
  dalloc(m.ctabox, (size_t)3 * kMaxGrid);
  upload(m.rbox, h.rbox, m.stream);
  upload(m.Ainv, A, m.stream);
  upload(m.Ainv32, A32, m.stream);
  MM_CK(cudaStreamSynchronize(m.stream));
}

mm_status fail(mm_status st, const std::string& msg) {
  g_error = msg;
  return st;
}

#define API_BEGIN try {
#define API_END                                                \
  }                                                            \
  catch (const mumag::CudaFailure& e) {                        \
    return mumag::fail(MM_CUDA_ERROR, e.what());               \
  }                                                            \
  catch (const std::bad_alloc&) {                              \
    return mumag::fail(MM_BAD_INPUT, "host allocation failed"); \
  }                                                            \
  catch (const std::exception& e) {                            \
    return mumag::fail(MM_BAD_INPUT, e.what());                \
  }

void check_mesh(const mm_mesh* mesh) {
  if (!mesh) throw std::runtime_error("mesh handle is NULL");
}

void check_params(const mm_solver_params* sp) {
  if (!sp) throw std::runtime_error("solver parameters are NULL");
  if (!(sp->tol_fun > 0) || !(sp->tol_u >= 0)) throw std::runtime_error("tolerances must be positive");
  if (sp->max_pcg_iter < 0 || sp->max_ncg_iter < 1) throw std::runtime_error("iteration caps must be positive");
}

// The sample-recording hash seed of the next launch (an LCG step).
unsigned next_seed(unsigned s) { return s * 1664525u + 1013904223u; }

// Run one persistent launch and collect its status.
mm_status run(DevMesh& m, const SolveArgs& a) {
  MM_CK(cudaSetDevice(m.device));
  if (!m.evk0) MM_CK(cudaEventCreate(&m.evk0));
  if (!m.evk1) MM_CK(cudaEventCreate(&m.evk1));
  MM_CK(solver_launch(m, a));
  MM_CK(cudaMemcpyAsync(m.h_resd, m.resd, 2 * sizeof(double), cudaMemcpyDeviceToHost, m.stream));
  MM_CK(cudaMemcpyAsync(m.h_resi, m.resi, kResI * sizeof(long long), cudaMemcpyDeviceToHost, m.stream));
  MM_CK(cudaMemcpyAsync(m.h_flags, m.flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, m.stream));
  MM_CK(cudaStreamSynchronize(m.stream));
  MM_CK(cudaEventElapsedTime(&m.last_launch_ms, m.evk0, m.evk1));
  m.rec_seed = next_seed(m.rec_seed);
  const int st = m.h_flags[FLAG_STATUS];
  if (st == MM_TIMEOUT) return fail(MM_TIMEOUT, "a grid barrier of the persistent solver kernel timed out");
  if (st != MM_OK && st != MM_NONFINITE)
    return fail(MM_CUDA_ERROR, "the solver kernel left an invalid status word (" + std::to_string(st) + ")");
  return st;
}

}  // namespace

void set_error(const std::string& msg) { g_error = msg; }

}  // namespace mumag

using namespace mumag;

extern "C" {

const char* mm_version(void) { return "mumag_b200 0.1.0 (sm_100a)"; }

const char* mm_last_error(void) { return g_error.c_str(); }

void mm_default_options(mm_options* opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->size = 1e-9;
  opt->dirichlet_rhs = MM_DIRICHLET_RHS_REFERENCE;
  opt->precision = MM_PREC_FP64;
  opt->device = 0;
  opt->grid_ctas = 0;
  opt->block_threads = 0;
  opt->reorder = 1;
  opt->pcg_variant = 0;
  opt->ctas_per_sm = 0;
  opt->stage_operators = 1;
  opt->coarse_box_nodes = 0;
}

void mm_default_solver_params(mm_solver_params* sp) {
  if (!sp) return;
  std::memset(sp, 0, sizeof(*sp));
  sp->hdir[2] = 1.0;
  sp->tol_fun = 1e-10;
  sp->tol_u = 1e-10;
  sp->precond_iter = 10;
  sp->hmag_on = 1;
  sp->mbar_mode = 0;
  sp->max_pcg_iter = 10000;
  sp->max_ncg_iter = 100000;
}

int mm_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int ok = 0;
  for (int d = 0; d < n; ++d) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10) ++ok;
  }
  return ok;
}

mm_status mm_rcm_permutation(int64_t N, const int32_t* T, int64_t E, int32_t* perm) {
  API_BEGIN
  if (!T || !perm) throw std::runtime_error("NULL array");
  auto p = rcm_order(N, T, E);
  std::memcpy(perm, p.data(), sizeof(int32_t) * N);
  return MM_OK;
  API_END
}

mm_status mm_color_elements(int64_t N, const int32_t* T, int64_t E, int32_t* colour, int32_t* ncolours) {
  API_BEGIN
  if (!T || !colour || !ncolours) throw std::runtime_error("NULL array");
  if (N <= 0 || E <= 0) throw std::runtime_error("mesh needs N > 0 nodes and E > 0 elements");
  for (int64_t k = 0; k < 4 * E; ++k)
    if (T[k] < 0 || T[k] >= N) throw std::runtime_error("element node index out of range");
  *ncolours = greedy_colour(N, T, E, nullptr, colour);
  return MM_OK;
  API_END
}

mm_status mm_mesh_create(const double* X, int64_t N, const int32_t* T, const int32_t* tag, int64_t E,
                         const mm_material* mats, int32_t nmats, const mm_options* opt, mm_mesh** out) {
  API_BEGIN
  if (!out) throw std::runtime_error("output handle pointer is NULL");
  *out = nullptr;
  if (!X || !T || !tag || !mats) throw std::runtime_error("NULL input array");
  mm_options o;
  mm_default_options(&o);
  if (opt) o = *opt;
  if (!(o.size > 0)) throw std::runtime_error("options.size must be positive");
  if (o.pcg_variant < 0 || o.pcg_variant > 2) throw std::runtime_error("options.pcg_variant must be 0, 1 or 2");
  if (o.ctas_per_sm != 0 && o.ctas_per_sm != 2 && o.ctas_per_sm != 3)
    throw std::runtime_error("options.ctas_per_sm must be 0, 2 or 3");
  if (o.stage_operators != 0 && o.stage_operators != 1)
    throw std::runtime_error("options.stage_operators must be 0 or 1");
  if (o.coarse_box_nodes < 0) throw std::runtime_error("options.coarse_box_nodes must be >= 0");
  for (int64_t i = 0; i < 3 * N; ++i)
    if (!std::isfinite(X[i])) throw std::runtime_error("non-finite node coordinate");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(MM_NO_DEVICE, "no CUDA device");
  }
  if (o.device < 0 || o.device >= ndev) throw std::runtime_error("options.device out of range");
  cudaDeviceProp prop;
  MM_CK(cudaGetDeviceProperties(&prop, o.device));
  if (prop.major != 10) return fail(MM_NO_DEVICE, "device is not sm_100 (B200): " + std::string(prop.name));
  std::unique_ptr<mm_mesh> mesh(new mm_mesh());
  DevMesh& m = mesh->dm;
  m.device = o.device;
  m.opt = o;
  // host preprocessing, from the cache when this exact mesh was prepared before
  uint64_t key = hash_bytes(0x6D756D6167ull, X, sizeof(double) * 3 * (size_t)std::max<int64_t>(N, 0));
  key = hash_bytes(key, T, sizeof(int32_t) * 4 * (size_t)std::max<int64_t>(E, 0));
  key = hash_bytes(key, tag, sizeof(int32_t) * (size_t)std::max<int64_t>(E, 0));
  std::shared_ptr<PrepEntry> prep =
      N > 0 && E > 0 ? prep_find(key, X, N, T, tag, E, o.reorder != 0, o.coarse_box_nodes) : nullptr;
  if (prep) {
    m.h = prep->h;
    if ((int32_t)m.h.tags.size() > nmats)
      throw std::runtime_error("materials file has " + std::to_string(nmats) + " rows for " +
                               std::to_string(m.h.tags.size()) + " element tags");
  } else {
    preprocess(X, N, T, tag, E, nmats, o.reorder != 0, o.coarse_box_nodes, m.h);
    prep = std::make_shared<PrepEntry>();
    prep->hash = key;
    prep->reorder = o.reorder != 0;
    prep->coarse = o.coarse_box_nodes;
    prep->X.assign(X, X + 3 * N);
    prep->T.assign(T, T + 4 * E);
    prep->tag.assign(tag, tag + E);
    prep->h = m.h;
    prep_store(prep);
  }
  // PCG arrangement: fixed by the caller, else by size until mm_autotune times both; the
  // two-level preconditioner runs in the two-sync arrangement only
  m.pcg2 = o.pcg_variant == 2 ? 1 : o.pcg_variant == 1 ? 0 : (m.h.N >= kPcg2Nodes ? 1 : 0);
  if (m.h.nc > 0) {
    if (o.pcg_variant == 1)
      throw std::runtime_error("the two-level preconditioner runs in the two-sync PCG arrangement (pcg_variant 0 or 2)");
    m.pcg2 = 1;
  }
  m.kernel_mb = o.ctas_per_sm == 3 ? 3 : 2;
  HostMesh& h = m.h;
  m.ncolours = (int32_t)h.colour_off.size() - 1;
  // materials, scripts/materials.py:17-35
  const double mu0 = 4e-7 * M_PI;
  m.mats.resize(h.tags.size());
  for (size_t t = 0; t < h.tags.size(); ++t) {
    const mm_material& r = mats[t];
    MatRow mr{};
    if (r.Js > 0) {
      mr.u[0] = std::sin(r.theta) * std::cos(r.phi);
      mr.u[1] = std::sin(r.theta) * std::sin(r.phi);
      mr.u[2] = std::cos(r.theta);
      mr.K = mu0 * r.K1;
      mr.Js = r.Js;
      mr.A = mu0 * r.A / (o.size * o.size);
    }
    m.mats[t] = mr;
  }
  try {
    MM_CK(cudaSetDevice(m.device));
    MM_CK(cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking));
    dalloc(m.sl_off, h.sl_off.size());
    dalloc(m.sl_w, h.sl_w.size());
    dalloc(m.col, h.col.size());
    dalloc(m.rowlen, h.rowlen.size());
    dalloc(m.vals, (size_t)kNumPlanes * h.nent);
    dalloc(m.diagS, h.Npad);
    dalloc(m.invdS, h.Npad);
    dalloc(m.Dex, h.Npad);
    dalloc(m.meas, h.Npad);
    dalloc(m.bnd, h.Npad);
    dalloc(m.Xd, h.Xd.size());
    dalloc(m.econn, h.econn.size());
    dalloc(m.etag, h.etag.size());
    dalloc(m.dmats, m.mats.size());
    if (o.precision == MM_PREC_MIXED) dalloc(m.vals32, (size_t)kNumPlanes32 * h.nent);
    upload(m.sl_off, h.sl_off, m.stream);
    upload(m.sl_w, h.sl_w, m.stream);
    upload(m.col, h.col, m.stream);
    upload(m.rowlen, h.rowlen, m.stream);
    upload(m.bnd, h.bnd, m.stream);
    upload(m.Xd, h.Xd, m.stream);
    upload(m.econn, h.econn, m.stream);
    upload(m.etag, h.etag, m.stream);
    upload(m.dmats, m.mats, m.stream);
    assemble_operators(m);
    build_coarse(m, &prep->Ainv);
    // solver state: 12 three-vectors, 2 node vectors, 2 x Npad PCG records (4 doubles each);
    // the total is computed from the same list that carves the buffer
    const size_t np = h.Npad;
    double** v3[] = {&m.x, &m.x1, &m.g, &m.g1, &m.d, &m.gf, &m.mbar, &m.zp, &m.tr, &m.tz, &m.td, &m.tBd};
    double** v1[] = {&m.u, &m.pp, &m.r64};
    constexpr int kRecDoubles = (int)(sizeof(PcgRec) / sizeof(double));
    constexpr int kRec32Doubles = (int)(sizeof(PcgRec32) / sizeof(double));
    // + 2 x Npad FP32 records and the FP32 inner vectors pp32, e32 (one Npad of doubles)
    const size_t total = (sizeof(v3) / sizeof(v3[0])) * 3 * np + (sizeof(v1) / sizeof(v1[0])) * np +
                         2 * kRecDoubles * np + 2 * kRec32Doubles * np + np;
    dalloc(m.ws, total);
    MM_CK(cudaMemsetAsync(m.ws, 0, sizeof(double) * total, m.stream));
    double* p = m.ws;
    for (double** q : v3) {
      *q = p;
      p += 3 * np;
    }
    for (double** q : v1) {
      *q = p;
      p += np;
    }
    for (int q = 0; q < 2; ++q) {  // 32-byte aligned: every preceding part is a multiple of 256 bytes
      m.rec[q] = reinterpret_cast<PcgRec*>(p);
      p += kRecDoubles * np;
    }
    for (int q = 0; q < 2; ++q) {
      m.rec32[q] = reinterpret_cast<PcgRec32*>(p);
      p += kRec32Doubles * np;
    }
    m.pp32 = reinterpret_cast<float*>(p);
    m.e32 = m.pp32 + np;
    p += np;
    if (p != m.ws + total) throw std::logic_error("solver workspace carve does not match its size");
    solver_configure(m);
    dalloc(m.bar, 1);
    dalloc(m.red, (size_t)2 * kMaxRed * kMaxGrid);  // any grid the autotuner may choose
    dalloc(m.flags, 2);
    dalloc(m.resd, 2);
    dalloc(m.resi, kResI);
    if (std::getenv("MUMAG_PROFILE")) {  // diagnostic per-CTA phase timers
      dalloc(m.prof, (size_t)kProfCols * kMaxGrid);  // any grid the autotuner may choose
      MM_CK(cudaMemsetAsync(m.prof, 0, sizeof(long long) * kProfCols * kMaxGrid, m.stream));
    }
    MM_CK(cudaHostAlloc(reinterpret_cast<void**>(&m.h_resd), 2 * sizeof(double), cudaHostAllocDefault));
    MM_CK(cudaHostAlloc(reinterpret_cast<void**>(&m.h_resi), kResI * sizeof(long long), cudaHostAllocDefault));
    MM_CK(cudaHostAlloc(reinterpret_cast<void**>(&m.h_flags), 2 * sizeof(int), cudaHostAllocDefault));
    MM_CK(cudaStreamSynchronize(m.stream));
  } catch (...) {
    release(m);
    throw;
  }
  *out = mesh.release();
  return MM_OK;
  API_END
}

mm_status mm_mesh_destroy(mm_mesh* mesh) {
  if (!mesh) return MM_OK;
  release(mesh->dm);
  delete mesh;
  return MM_OK;
}

mm_status mm_mesh_get_info(const mm_mesh* mesh, mm_mesh_info* info) {
  API_BEGIN
  check_mesh(mesh);
  if (!info) throw std::runtime_error("info is NULL");
  const DevMesh& m = mesh->dm;
  info->nodes = m.h.N;
  info->elements = m.h.E;
  info->sell_slices = m.h.nslices;
  info->sell_entries = m.h.nent;
  info->nnz = m.h.nnz;
  info->colours = m.ncolours;
  info->airbox = m.h.airbox;
  info->grid_ctas = m.grid;
  info->block_threads = m.block;
  int64_t nb = 0;
  for (auto b : m.h.bnd) nb += b;
  info->dirichlet_nodes = nb;
  info->volume = m.V;
  info->bandwidth_before = (double)m.h.bandwidth_before;
  info->bandwidth_after = (double)m.h.bandwidth_after;
  info->pcg_variant = m.pcg2 ? 2 : 1;
  info->kernel_ctas_per_sm = m.kernel_mb;
  info->staged = m.stage;
  info->coarse_boxes = m.nc;
  return MM_OK;
  API_END
}

mm_status mm_mesh_get_coarse(const mm_mesh* mesh, int32_t* box, int32_t* nboxes) {
  API_BEGIN
  check_mesh(mesh);
  if (!nboxes) throw std::runtime_error("nboxes is NULL");
  const DevMesh& m = mesh->dm;
  *nboxes = m.nc;
  if (box && m.nc > 0)
    for (int64_t i = 0; i < m.h.N; ++i) box[i] = m.h.rbox[m.h.iperm[i]];
  return MM_OK;
  API_END
}

mm_status mm_get_meas(mm_mesh* mesh, double* meas, double* volume) {
  API_BEGIN
  check_mesh(mesh);
  DevMesh& m = mesh->dm;
  MM_CK(cudaSetDevice(m.device));
  if (meas) {
    std::vector<double> t;
    d2h(t, m.meas, m.h.Npad, m.stream);
    from_nodes(m, t, meas);
  }
  if (volume) *volume = m.V;
  return MM_OK;
  API_END
}

mm_status mm_get_operator(mm_mesh* mesh, int32_t which, int64_t* nnz, int32_t* rows, int32_t* cols, double* vals) {
  API_BEGIN
  check_mesh(mesh);
  if (which < 0 || which >= kNumPlanes) throw std::runtime_error("operator index out of range");
  if (!nnz) throw std::runtime_error("nnz is NULL");
  DevMesh& m = mesh->dm;
  const HostMesh& h = m.h;
  *nnz = h.nnz;
  if (!rows) return MM_OK;
  if (!cols || !vals) throw std::runtime_error("NULL output array");
  MM_CK(cudaSetDevice(m.device));
  std::vector<double> pv;
  d2h(pv, m.vals + (size_t)which * h.nent, h.nent, m.stream);
  int64_t q = 0;
  for (int64_t s = 0; s < h.nslices; ++s)
    for (int l = 0; l < kSlice; ++l) {
      const int64_t i = s * kSlice + l;
      if (i >= h.N) continue;
      for (int32_t k = 0; k < h.rowlen[i]; ++k) {
        const int64_t e = h.sl_off[s] + (int64_t)k * kSlice + l;
        rows[q] = h.perm[i];
        cols[q] = h.perm[h.col[e]];
        vals[q] = pv[e];
        ++q;
      }
    }
  return MM_OK;
  API_END
}

mm_status mm_set_state(mm_mesh* mesh, const double* mv, const double* uv, const double* mbar) {
  API_BEGIN
  check_mesh(mesh);
  if (!mv) throw std::runtime_error("m is NULL");
  DevMesh& m = mesh->dm;
  const size_t np = m.h.Npad;
  for (int64_t i = 0; i < 3 * m.h.N; ++i)
    if (!std::isfinite(mv[i]) || (mbar && !std::isfinite(mbar[i]))) throw std::runtime_error("non-finite magnetisation");
  MM_CK(cudaSetDevice(m.device));
  std::vector<double> t;
  to_planes(m, mv, t);
  MM_CK(cudaMemcpyAsync(m.x, t.data(), sizeof(double) * 3 * np, cudaMemcpyHostToDevice, m.stream));
  if (mbar) to_planes(m, mbar, t);
  MM_CK(cudaMemcpyAsync(m.mbar, t.data(), sizeof(double) * 3 * np, cudaMemcpyHostToDevice, m.stream));
  std::vector<double> tu(np, 0.0);
  if (uv) {
    for (int64_t i = 0; i < m.h.N; ++i)
      if (!std::isfinite(uv[i])) throw std::runtime_error("non-finite potential");
    to_nodes(m, uv, tu);
  }
  MM_CK(cudaMemcpyAsync(m.u, tu.data(), sizeof(double) * np, cudaMemcpyHostToDevice, m.stream));
  MM_CK(cudaMemsetAsync(m.gf, 0, sizeof(double) * 3 * np, m.stream));
  MM_CK(cudaStreamSynchronize(m.stream));
  return MM_OK;
  API_END
}

mm_status mm_set_state_device(mm_mesh* mesh, const double* mv, const double* uv, const double* mbar) {
  API_BEGIN
  check_mesh(mesh);
  if (!mv) throw std::runtime_error("m is NULL");
  DevMesh& m = mesh->dm;
  const size_t np = m.h.Npad;
  MM_CK(cudaSetDevice(m.device));
  ensure_iperm(m);
  MM_CK(cudaMemsetAsync(m.x, 0, sizeof(double) * 3 * np, m.stream));
  MM_CK(cudaMemsetAsync(m.mbar, 0, sizeof(double) * 3 * np, m.stream));
  MM_CK(cudaMemsetAsync(m.u, 0, sizeof(double) * np, m.stream));
  MM_CK(cudaMemsetAsync(m.gf, 0, sizeof(double) * 3 * np, m.stream));
  MM_CK(cudaMemsetAsync(m.d_bad, 0, sizeof(int), m.stream));
  const int grid = (int)std::min<int64_t>((m.h.N + 255) / 256, 1184);
  k_state_in<<<grid, 256, 0, m.stream>>>(mv, uv, mbar, m.d_iperm, m.h.N, (int64_t)np, m.x, m.u, m.mbar, m.d_bad);
  MM_CK(cudaGetLastError());
  MM_CK(cudaMemcpyAsync(m.h_flags, m.d_bad, sizeof(int), cudaMemcpyDeviceToHost, m.stream));
  MM_CK(cudaStreamSynchronize(m.stream));
  if (m.h_flags[0]) throw std::runtime_error("non-finite magnetisation or potential");
  return MM_OK;
  API_END
}

mm_status mm_get_state_device(mm_mesh* mesh, double* mv, double* uv, double* gfull) {
  API_BEGIN
  check_mesh(mesh);
  DevMesh& m = mesh->dm;
  MM_CK(cudaSetDevice(m.device));
  ensure_iperm(m);
  const int grid = (int)std::min<int64_t>((m.h.N + 255) / 256, 1184);
  k_state_out<<<grid, 256, 0, m.stream>>>(m.x, m.u, m.gf, m.d_iperm, m.h.N, (int64_t)m.h.Npad, mv, uv, gfull);
  MM_CK(cudaGetLastError());
  MM_CK(cudaStreamSynchronize(m.stream));
  return MM_OK;
  API_END
}

mm_status mm_get_state(mm_mesh* mesh, double* mv, double* uv, double* gfull) {
  API_BEGIN
  check_mesh(mesh);
  DevMesh& m = mesh->dm;
  const size_t np = m.h.Npad;
  MM_CK(cudaSetDevice(m.device));
  std::vector<double> t;
  if (mv) {
    d2h(t, m.x, 3 * np, m.stream);
    from_planes(m, t, mv);
  }
  if (uv) {
    d2h(t, m.u, np, m.stream);
    from_nodes(m, t, uv);
  }
  if (gfull) {
    d2h(t, m.gf, 3 * np, m.stream);
    from_planes(m, t, gfull);
  }
  return MM_OK;
  API_END
}

mm_status mm_energy_grad(mm_mesh* mesh, double h, const mm_solver_params* sp, double* energy, double* gproj,
                         int64_t* pcg_iters) {
  API_BEGIN
  check_mesh(mesh);
  check_params(sp);
  DevMesh& m = mesh->dm;
  mm_status st = run(m, solver_args(m, MODE_EVAL, h, *sp));
  if (energy) *energy = m.h_resd[0];
  if (pcg_iters) *pcg_iters = m.h_resi[2];
  if (gproj) {
    std::vector<double> t;
    d2h(t, m.g, 3 * m.h.Npad, m.stream);
    from_planes(m, t, gproj);
  }
  if (st == MM_NONFINITE) return fail(st, "energy is not finite");
  return st;
  API_END
}

mm_status mm_apply_minv(mm_mesh* mesh, const mm_solver_params* sp, const double* g, double* z, int64_t* iters) {
  API_BEGIN
  check_mesh(mesh);
  check_params(sp);
  if (!g || !z) throw std::runtime_error("NULL vector");
  DevMesh& m = mesh->dm;
  const size_t np = m.h.Npad;
  MM_CK(cudaSetDevice(m.device));
  std::vector<double> t;
  to_planes(m, g, t);
  MM_CK(cudaMemcpyAsync(m.g, t.data(), sizeof(double) * 3 * np, cudaMemcpyHostToDevice, m.stream));
  mm_status st = run(m, solver_args(m, MODE_MINV, 0.0, *sp));
  d2h(t, m.zp, 3 * np, m.stream);
  from_planes(m, t, z);
  if (iters) *iters = m.h_resi[4];
  return st;
  API_END
}

mm_status mm_minimize(mm_mesh* mesh, double h, const mm_solver_params* sp, mm_step_result* res) {
  API_BEGIN
  check_mesh(mesh);
  check_params(sp);
  DevMesh& m = mesh->dm;
  mm_status st = run(m, solver_args(m, MODE_MINIMIZE, h, *sp));
  if (res) {
    res->energy = m.h_resd[0];
    res->mh = m.h_resd[1];
    res->ncg_iters = m.h_resi[0];
    res->evals = m.h_resi[1];
    res->pcg_iters = m.h_resi[2];
    res->ls_shrinks = m.h_resi[3];
    res->minv_iters = m.h_resi[4];
    res->kernel_ns = m.h_resi[5];
    res->sync_ns = m.h_resi[6];
    res->barriers = m.h_resi[7];
    res->learned_starts = m.h_resi[8];
    res->device_ms = m.last_launch_ms;
    res->status = st;
  }
  if (st == MM_NONFINITE) return fail(st, "energy is not finite");
  return st;
  API_END
}

mm_status mm_loop(mm_mesh* mesh, const mm_loop_params* lp, const mm_solver_params* sp, mm_record* rec,
                  int32_t* nrec, mm_step_result* steps, mm_snapshot_cb cb, void* user) {
  API_BEGIN
  check_mesh(mesh);
  check_params(sp);
  if (!lp || !rec || !nrec) throw std::runtime_error("NULL loop argument");
  if (!(lp->hstep != 0.0) || !std::isfinite(lp->hstart) || !std::isfinite(lp->hfinal))
    throw std::runtime_error("invalid field sweep");
  DevMesh& m = mesh->dm;
  // scripts/loop.py:126-131
  int64_t nmax = (int64_t)(std::fabs(lp->hfinal - lp->hstart) / std::fabs(lp->hstep)) + 1;
  if (lp->max_steps > 0) nmax = std::min<int64_t>(nmax, lp->max_steps);
  *nrec = 0;
  double mh = 1.7976931348623157e308, last_saved = mh;
  int counter = 0;
  double hext = lp->hstart;
  std::vector<double> tm, tu, fm, fu;
  for (int64_t idx = 0; idx < nmax && mh > lp->mfinal; ++idx) {
    mm_step_result r{};
    mm_status st = run(m, solver_args(m, MODE_MINIMIZE, hext, *sp));
    r.energy = m.h_resd[0];
    r.mh = m.h_resd[1];
    r.ncg_iters = m.h_resi[0];
    r.evals = m.h_resi[1];
    r.pcg_iters = m.h_resi[2];
    r.ls_shrinks = m.h_resi[3];
    r.minv_iters = m.h_resi[4];
    r.kernel_ns = m.h_resi[5];
    r.sync_ns = m.h_resi[6];
    r.barriers = m.h_resi[7];
    r.learned_starts = m.h_resi[8];
    r.device_ms = m.last_launch_ms;
    r.status = st;
    if (st != MM_OK) {
      if (steps) steps[idx] = r;
      return st == MM_NONFINITE ? fail(st, "energy is not finite at field " + std::to_string(hext)) : st;
    }
    mh = r.mh;
    if ((last_saved - mh) > lp->mstep) {  // scripts/loop.py:103-116
      counter += 1;
      last_saved = mh;
      if (cb) {
        d2h(tm, m.x, 3 * m.h.Npad, m.stream);
        d2h(tu, m.u, m.h.Npad, m.stream);
        fm.resize(3 * m.h.N);
        fu.resize(m.h.N);
        from_planes(m, tm, fm.data());
        from_nodes(m, tu, fu.data());
        if (cb(counter, fm.data(), fu.data(), m.h.N, user) != 0)
          return fail(MM_BAD_INPUT, "snapshot callback aborted the loop");
      }
    }
    rec[idx].counter = counter;
    rec[idx].hext = hext;
    rec[idx].mh = mh;
    rec[idx].energy = r.energy;
    if (steps) steps[idx] = r;
    *nrec = (int32_t)(idx + 1);
    hext = hext + lp->hstep;
  }
  return MM_OK;
  API_END
}

mm_status mm_profile_read(mm_mesh* mesh, long long* out, int32_t* nctas) {
  API_BEGIN
  check_mesh(mesh);
  DevMesh& m = mesh->dm;
  if (!nctas) throw std::runtime_error("nctas is NULL");
  *nctas = m.prof ? m.grid : 0;
  if (!m.prof || !out) return MM_OK;
  MM_CK(cudaSetDevice(m.device));
  MM_CK(cudaMemcpy(out, m.prof, sizeof(long long) * kProfCols * m.grid, cudaMemcpyDeviceToHost));
  MM_CK(cudaMemset(m.prof, 0, sizeof(long long) * kProfCols * kMaxGrid));
  return MM_OK;
  API_END
}

mm_status mm_timer_start(mm_mesh* mesh) {
  API_BEGIN
  check_mesh(mesh);
  DevMesh& m = mesh->dm;
  MM_CK(cudaSetDevice(m.device));
  if (!m.ev0) MM_CK(cudaEventCreate(&m.ev0));
  if (!m.ev1) MM_CK(cudaEventCreate(&m.ev1));
  MM_CK(cudaEventRecord(m.ev0, m.stream));
  return MM_OK;
  API_END
}

mm_status mm_timer_stop(mm_mesh* mesh, double* elapsed_ms) {
  API_BEGIN
  check_mesh(mesh);
  if (!elapsed_ms) throw std::runtime_error("elapsed_ms is NULL");
  DevMesh& m = mesh->dm;
  if (!m.ev0) throw std::runtime_error("mm_timer_start was not called");
  MM_CK(cudaSetDevice(m.device));
  MM_CK(cudaEventRecord(m.ev1, m.stream));
  MM_CK(cudaEventSynchronize(m.ev1));
  float ms = 0.f;
  MM_CK(cudaEventElapsedTime(&ms, m.ev0, m.ev1));
  *elapsed_ms = ms;
  return MM_OK;
  API_END
}

namespace {
void batch_release(mm_batch* b) {
  cudaSetDevice(b->device);
  if (b->d_args) cudaFree(b->d_args);
  if (b->d_group) cudaFree(b->d_group);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
}

// One batched launch: args[q] with mode MINIMIZE (h[q]) or IDLE (active[q] == 0).
mm_status batch_run(mm_batch* b, const double* h, const mm_solver_params* sp, const std::vector<char>& active) {
  const int count = (int)b->meshes.size();
  MM_CK(cudaSetDevice(b->device));
  for (int q = 0; q < count; ++q) {
    DevMesh& m = b->meshes[q]->dm;
    SolveArgs a = solver_args(m, active[q] ? MODE_MINIMIZE : MODE_IDLE, h[q], sp[q]);
    a.stage = b->plan.stage[q];
    a.stage_max = b->plan.stage_max[q];
    a.meta_max = b->plan.meta_max[q];
    a.prof = nullptr;
    a.tc_off = -1;  // batched launches run the network on mma.sync
    a.nc = 0;       // and the Jacobi preconditioner
    b->h_args[q] = a;
    MM_CK(launch_prep(m, b->stream));
  }
  MM_CK(cudaMemcpyAsync(b->d_args, b->h_args.data(), sizeof(SolveArgs) * count, cudaMemcpyHostToDevice, b->stream));
  MM_CK(batch_launch(b->plan, b->d_args, b->d_group, count, b->stream));
  for (int q = 0; q < count; ++q) {
    DevMesh& m = b->meshes[q]->dm;
    MM_CK(cudaMemcpyAsync(m.h_resd, m.resd, 2 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    MM_CK(cudaMemcpyAsync(m.h_resi, m.resi, kResI * sizeof(long long), cudaMemcpyDeviceToHost, b->stream));
    MM_CK(cudaMemcpyAsync(m.h_flags, m.flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  }
  MM_CK(cudaStreamSynchronize(b->stream));
  for (int q = 0; q < count; ++q) b->meshes[q]->dm.rec_seed = next_seed(b->meshes[q]->dm.rec_seed);
  mm_status worst = MM_OK;
  for (int q = 0; q < count; ++q) {
    const int st = b->meshes[q]->dm.h_flags[FLAG_STATUS];
    if (st == MM_TIMEOUT) return fail(MM_TIMEOUT, "a grid barrier of the batched solver kernel timed out");
    if (st != MM_OK && st != MM_NONFINITE)
      return fail(MM_CUDA_ERROR, "the batched solver kernel left an invalid status word");
    if (st == MM_NONFINITE) worst = MM_NONFINITE;
  }
  return worst;
}

void fill_result(const DevMesh& m, mm_status st, mm_step_result& r) {
  r.energy = m.h_resd[0];
  r.mh = m.h_resd[1];
  r.ncg_iters = m.h_resi[0];
  r.evals = m.h_resi[1];
  r.pcg_iters = m.h_resi[2];
  r.ls_shrinks = m.h_resi[3];
  r.minv_iters = m.h_resi[4];
  r.kernel_ns = m.h_resi[5];
  r.sync_ns = m.h_resi[6];
  r.barriers = m.h_resi[7];
  r.learned_starts = m.h_resi[8];
  r.device_ms = 0.0;
  r.status = st;
}
}  // namespace

mm_status mm_batch_create(mm_mesh* const* meshes, int32_t count, mm_batch** out) {
  API_BEGIN
  if (!out || !meshes || count < 1) throw std::runtime_error("invalid batch arguments");
  *out = nullptr;
  std::unique_ptr<mm_batch> b(new mm_batch());
  std::vector<DevMesh*> ms;
  for (int q = 0; q < count; ++q) {
    check_mesh(meshes[q]);
    b->meshes.push_back(meshes[q]);
    ms.push_back(&meshes[q]->dm);
  }
  b->device = ms[0]->device;
  try {
    MM_CK(cudaSetDevice(b->device));
    batch_configure(ms, b->plan);
    MM_CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    MM_CK(cudaMalloc(reinterpret_cast<void**>(&b->d_args), sizeof(SolveArgs) * count));
    MM_CK(cudaMalloc(reinterpret_cast<void**>(&b->d_group), sizeof(int) * (count + 1)));
    MM_CK(cudaMemcpy(b->d_group, b->plan.group.data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice));
    b->h_args.resize(count);
  } catch (...) {
    batch_release(b.get());
    throw;
  }
  *out = b.release();
  return MM_OK;
  API_END
}

mm_status mm_batch_destroy(mm_batch* batch) {
  if (!batch) return MM_OK;
  batch_release(batch);
  delete batch;
  return MM_OK;
}

mm_status mm_batch_groups(const mm_batch* batch, int32_t* group) {
  API_BEGIN
  if (!batch || !group) throw std::runtime_error("NULL batch or output");
  for (size_t q = 0; q < batch->plan.group.size(); ++q) group[q] = batch->plan.group[q];
  return MM_OK;
  API_END
}

mm_status mm_batch_minimize(mm_batch* batch, const double* h, const mm_solver_params* sp, mm_step_result* res) {
  API_BEGIN
  if (!batch || !h || !sp) throw std::runtime_error("NULL batch argument");
  const int count = (int)batch->meshes.size();
  for (int q = 0; q < count; ++q) check_params(&sp[q]);
  std::vector<char> active(count, 1);
  mm_status st = batch_run(batch, h, sp, active);
  if (res)
    for (int q = 0; q < count; ++q) fill_result(batch->meshes[q]->dm, st, res[q]);
  return st;
  API_END
}

mm_status mm_batch_loop(mm_batch* batch, const mm_loop_params* lp, const mm_solver_params* sp, int32_t max_steps,
                        mm_record* rec, int32_t* nrec, mm_step_result* steps) {
  API_BEGIN
  if (!batch || !lp || !sp || !rec || !nrec || max_steps < 1) throw std::runtime_error("invalid batch loop arguments");
  if (!(lp->hstep != 0.0) || !std::isfinite(lp->hstart) || !std::isfinite(lp->hfinal))
    throw std::runtime_error("invalid field sweep");
  const int count = (int)batch->meshes.size();
  for (int q = 0; q < count; ++q) check_params(&sp[q]);
  int64_t nmax = (int64_t)(std::fabs(lp->hfinal - lp->hstart) / std::fabs(lp->hstep)) + 1;
  if (lp->max_steps > 0) nmax = std::min<int64_t>(nmax, lp->max_steps);
  nmax = std::min<int64_t>(nmax, max_steps);
  for (int q = 0; q < count; ++q) nrec[q] = 0;
  MM_CK(cudaSetDevice(batch->device));
  // per mesh: rows [nmax][4] doubles, counters [nmax][8] int64, one row count
  const size_t per = (size_t)nmax * (4 * sizeof(double) + 8 * sizeof(long long)) + 256;
  char* buf = nullptr;
  MM_CK(cudaMalloc(reinterpret_cast<void**>(&buf), per * count));
  std::vector<char> host(per * count);
  try {
    MM_CK(cudaMemsetAsync(buf, 0, per * count, batch->stream));
    for (int q = 0; q < count; ++q) {
      DevMesh& m = batch->meshes[q]->dm;
      SolveArgs a = solver_args(m, MODE_SWEEP, lp->hstart, sp[q]);
      char* b = buf + per * q;
      a.sw_rec = reinterpret_cast<double*>(b);
      a.sw_stat = reinterpret_cast<long long*>(b + (size_t)nmax * 4 * sizeof(double));
      a.sw_nrec = reinterpret_cast<int*>(b + (size_t)nmax * (4 * sizeof(double) + 8 * sizeof(long long)));
      a.sw_hstep = lp->hstep;
      a.sw_mstep = lp->mstep;
      a.sw_mfinal = lp->mfinal;
      a.sw_nmax = (int)nmax;
      a.stage = batch->plan.stage[q];
      a.stage_max = batch->plan.stage_max[q];
      a.meta_max = batch->plan.meta_max[q];
      a.prof = nullptr;
      a.tc_off = -1;  // batched launches run the network on mma.sync
      a.nc = 0;       // and the Jacobi preconditioner
      batch->h_args[q] = a;
      MM_CK(launch_prep(m, batch->stream));
    }
    MM_CK(cudaMemcpyAsync(batch->d_args, batch->h_args.data(), sizeof(SolveArgs) * count, cudaMemcpyHostToDevice,
                          batch->stream));
    MM_CK(batch_launch(batch->plan, batch->d_args, batch->d_group, count, batch->stream));
    MM_CK(cudaMemcpyAsync(host.data(), buf, per * count, cudaMemcpyDeviceToHost, batch->stream));
    for (int q = 0; q < count; ++q) {
      DevMesh& m = batch->meshes[q]->dm;
      MM_CK(cudaMemcpyAsync(m.h_flags, m.flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, batch->stream));
    }
    MM_CK(cudaStreamSynchronize(batch->stream));
  } catch (...) {
    cudaFree(buf);
    throw;
  }
  cudaFree(buf);
  for (int q = 0; q < count; ++q) batch->meshes[q]->dm.rec_seed = next_seed(batch->meshes[q]->dm.rec_seed);
  mm_status worst = MM_OK;
  for (int q = 0; q < count; ++q) {
    const int st = batch->meshes[q]->dm.h_flags[FLAG_STATUS];
    if (st == MM_TIMEOUT) return fail(MM_TIMEOUT, "a grid barrier of the batched solver kernel timed out");
    if (st != MM_OK && st != MM_NONFINITE)
      return fail(MM_CUDA_ERROR, "the batched solver kernel left an invalid status word");
    if (st == MM_NONFINITE) worst = MM_NONFINITE;
    const char* b = host.data() + per * q;
    const double* rows = reinterpret_cast<const double*>(b);
    const long long* stat = reinterpret_cast<const long long*>(b + (size_t)nmax * 4 * sizeof(double));
    const int k = *reinterpret_cast<const int*>(b + (size_t)nmax * (4 * sizeof(double) + 8 * sizeof(long long)));
    if (k < 0 || k > nmax) return fail(MM_CUDA_ERROR, "the batched solver kernel left an invalid row count");
    for (int i = 0; i < k; ++i) {
      mm_record& r = rec[(size_t)q * max_steps + i];
      r.counter = rows[4 * i + 0];
      r.hext = rows[4 * i + 1];
      r.mh = rows[4 * i + 2];
      r.energy = rows[4 * i + 3];
      if (steps) {
        mm_step_result& t = steps[(size_t)q * max_steps + i];
        t = mm_step_result{};
        t.energy = r.energy;
        t.mh = r.mh;
        t.ncg_iters = stat[8 * i + 0];
        t.evals = stat[8 * i + 1];
        t.pcg_iters = stat[8 * i + 2];
        t.ls_shrinks = stat[8 * i + 3];
        t.minv_iters = stat[8 * i + 4];
        t.kernel_ns = stat[8 * i + 5];
        t.sync_ns = stat[8 * i + 6];
        t.barriers = stat[8 * i + 7];
        t.device_ms = 0.0;
        t.status = MM_OK;
      }
    }
    nrec[q] = k;
  }
  if (worst == MM_NONFINITE) return fail(MM_NONFINITE, "energy is not finite in a batched sweep");
  return MM_OK;
  API_END
}

mm_status mm_batch_timer_start(mm_batch* batch) {
  API_BEGIN
  if (!batch) throw std::runtime_error("NULL batch");
  MM_CK(cudaSetDevice(batch->device));
  if (!batch->ev0) MM_CK(cudaEventCreate(&batch->ev0));
  if (!batch->ev1) MM_CK(cudaEventCreate(&batch->ev1));
  MM_CK(cudaEventRecord(batch->ev0, batch->stream));
  return MM_OK;
  API_END
}

mm_status mm_batch_timer_stop(mm_batch* batch, double* elapsed_ms) {
  API_BEGIN
  if (!batch || !elapsed_ms || !batch->ev0) throw std::runtime_error("timer not started");
  MM_CK(cudaSetDevice(batch->device));
  MM_CK(cudaEventRecord(batch->ev1, batch->stream));
  MM_CK(cudaEventSynchronize(batch->ev1));
  float ms = 0.f;
  MM_CK(cudaEventElapsedTime(&ms, batch->ev0, batch->ev1));
  *elapsed_ms = ms;
  return MM_OK;
  API_END
}

namespace {
// Launch shapes already chosen for meshes of the same shape and precision (process-wide).
std::mutex g_tune_mu;
std::map<std::tuple<int64_t, int64_t, int, int, int>, std::tuple<int, int, int>> g_tune_cache;
}  // namespace

mm_status mm_autotune(mm_mesh* mesh, const mm_solver_params* sp, int32_t* grid_out) {
  API_BEGIN
  check_mesh(mesh);
  check_params(sp);
  DevMesh& m = mesh->dm;
  MM_CK(cudaSetDevice(m.device));
  cudaDeviceProp prop;
  MM_CK(cudaGetDeviceProperties(&prop, m.device));
  const auto key = std::make_tuple(m.h.nslices, m.h.nent,
                                   (m.vals32 ? 1 : 0) + (m.warm == WARM_LEARNED ? 2 : 0) + 4 * m.nc,
                                   m.device, (m.opt.pcg_variant * 4 + m.opt.ctas_per_sm) * 2 + m.opt.stage_operators);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      m.opt.grid_ctas = std::get<0>(it->second);
      m.pcg2 = std::get<1>(it->second);
      m.kernel_mb = std::get<2>(it->second);
      solver_configure(m);
      if (grid_out) *grid_out = m.grid;
      return MM_OK;
    }
  }
  // candidates (kernel build, CTAs): the two-CTA-per-SM build with one CTA per SM (or one
  // slice per warp), one and a half and two per SM; the three-CTA build with two and three
  // per SM; each with both PCG arrangements unless the options fix one
  const int64_t ns = m.h.nslices;
  const int sms = prop.multiProcessorCount;
  std::vector<std::pair<int, int>> cand;
  auto add = [&](int mb, int64_t g, int64_t per) {
    const int gg = (int)std::min<int64_t>(g, (ns + per - 1) / per);
    if (gg >= 1 && std::find(cand.begin(), cand.end(), std::make_pair(mb, gg)) == cand.end()) cand.emplace_back(mb, gg);
  };
  if (m.opt.ctas_per_sm != 3) {
    add(2, sms, 8);
    add(2, 3 * sms / 2, 6);
    add(2, 2 * sms, 4);
  }
  if (m.opt.ctas_per_sm != 2) {
    add(3, 2 * sms, 4);
    add(3, 3 * sms, 3);
  }
  std::vector<int> variants;
  if (m.nc > 0)
    variants = {1};
  else if (m.opt.pcg_variant == 1)
    variants = {0};
  else if (m.opt.pcg_variant == 2)
    variants = {1};
  else
    variants = {0, 1};
  // time a cold Poisson solve + energy evaluation at the current state for each shape
  std::vector<double> u0, gf0;
  d2h(u0, m.u, m.h.Npad, m.stream);
  d2h(gf0, m.gf, 3 * m.h.Npad, m.stream);
  int best = -1, best_v = m.pcg2, best_mb = m.kernel_mb;
  float best_ms = 0.f;
  const int saved = m.opt.grid_ctas, saved_v = m.pcg2, saved_mb = m.kernel_mb;
  for (const auto& [mb, g] : cand) {
    m.opt.grid_ctas = g;
    m.kernel_mb = mb;
    solver_configure(m);
    if (m.grid != g) continue;  // not resident
    for (int v : variants) {
      m.pcg2 = v;
      float ms = 0.f;
      for (int rep = 0; rep < 2; ++rep) {
        MM_CK(cudaMemsetAsync(m.u, 0, sizeof(double) * m.h.Npad, m.stream));
        mm_status st = run(m, solver_args(m, MODE_EVAL, 0.0, *sp));
        if (st != MM_OK && st != MM_NONFINITE) {
          m.opt.grid_ctas = saved;
          m.pcg2 = saved_v;
          m.kernel_mb = saved_mb;
          solver_configure(m);
          return st;
        }
        ms = m.last_launch_ms;
      }
      if (best < 0 || ms < best_ms) {
        best = g;
        best_v = v;
        best_mb = mb;
        best_ms = ms;
      }
    }
  }
  m.opt.grid_ctas = best > 0 ? best : saved;
  m.pcg2 = best > 0 ? best_v : saved_v;
  m.kernel_mb = best > 0 ? best_mb : saved_mb;
  solver_configure(m);
  MM_CK(cudaMemcpyAsync(m.u, u0.data(), sizeof(double) * m.h.Npad, cudaMemcpyHostToDevice, m.stream));
  MM_CK(cudaMemcpyAsync(m.gf, gf0.data(), sizeof(double) * 3 * m.h.Npad, cudaMemcpyHostToDevice, m.stream));
  MM_CK(cudaStreamSynchronize(m.stream));
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = std::make_tuple(m.grid, m.pcg2, m.kernel_mb);
  }
  if (grid_out) *grid_out = m.grid;
  return MM_OK;
  API_END
}

}  // extern "C"

// ---- learned warm start and sample recording --------------------------------------------
namespace mumag {
MlpDev model_view(const mm_model* m);
void set_noalloc_stall(int stall);  // noalloc.cu
}

extern "C" {

mm_status mm_debug_stall_barriers(mm_mesh* mesh, int32_t stall) {
  API_BEGIN
  if (stall < 0 || stall > 1024) throw std::runtime_error("stall must be in [0, 1024]");
  if (!mesh) {  // the allocation-free Poisson solve's barriers
    set_noalloc_stall(stall);
    return MM_OK;
  }
  mesh->dm.bar_stall = stall;
  return MM_OK;
  API_END
}

mm_status mm_mesh_set_warm_start(mm_mesh* mesh, int32_t mode, const mm_model* model) {
  API_BEGIN
  check_mesh(mesh);
  DevMesh& m = mesh->dm;
  if (mode != MM_WARM_PREVIOUS && mode != MM_WARM_ZERO && mode != MM_WARM_LEARNED)
    throw std::runtime_error("unknown warm-start mode");
  if (mode == MM_WARM_LEARNED && !model) throw std::runtime_error("the learned warm start needs a model");
  MM_CK(cudaSetDevice(m.device));
  if (mode == MM_WARM_LEARNED) {
    if (!m.feat) dalloc(m.feat, (size_t)m.h.Npad * kMlpIn);
    if (!m.du) dalloc(m.du, (size_t)m.h.Npad);
    m.mlp = model_view(model);
  } else {
    m.mlp = MlpDev{};
  }
  m.warm = mode;
  solver_configure(m);  // the learned start's network region changes the shared-memory plan
  return MM_OK;
  API_END
}

mm_status mm_mesh_set_learned_gate(mm_mesh* mesh, double ratio) {
  API_BEGIN
  check_mesh(mesh);
  if (!(ratio >= 0.0) || !std::isfinite(ratio)) throw std::runtime_error("the gate ratio must be finite and >= 0");
  mesh->dm.warm_gate = ratio;
  return MM_OK;
  API_END
}

mm_status mm_mesh_record_samples(mm_mesh* mesh, int64_t capacity, int32_t stride, uint64_t seed) {
  API_BEGIN
  check_mesh(mesh);
  DevMesh& m = mesh->dm;
  if (capacity < 0 || capacity > ((int64_t)1 << 31) - 1 || stride < 1) throw std::runtime_error("invalid recording arguments");
  MM_CK(cudaSetDevice(m.device));
  MM_CK(cudaStreamSynchronize(m.stream));
  dfree(m.rs_feat);
  dfree(m.rs_tgt);
  dfree(m.rs_u0);
  dfree(m.rs_node);
  dfree(m.rs_slot);
  dfree(m.rs_count);
  m.rec_cap = 0;
  if (capacity == 0) return MM_OK;
  dalloc(m.rs_feat, (size_t)capacity * kMlpIn);
  dalloc(m.rs_tgt, (size_t)capacity);
  dalloc(m.rs_u0, (size_t)capacity);
  dalloc(m.rs_node, (size_t)capacity);
  dalloc(m.rs_slot, (size_t)m.h.Npad);
  dalloc(m.rs_count, 1);
  MM_CK(cudaMemsetAsync(m.rs_slot, 0xFF, sizeof(int32_t) * m.h.Npad, m.stream));
  MM_CK(cudaMemsetAsync(m.rs_count, 0, sizeof(unsigned long long), m.stream));
  MM_CK(cudaMemsetAsync(m.rs_tgt, 0, sizeof(float) * capacity, m.stream));
  MM_CK(cudaStreamSynchronize(m.stream));
  m.rec_cap = capacity;
  m.rec_stride = stride;
  m.rec_seed = (unsigned)(seed ^ (seed >> 32));
  return MM_OK;
  API_END
}

mm_status mm_mesh_read_samples(mm_mesh* mesh, float* feats, float* target, int32_t* node, int64_t cap,
                               int64_t* count) {
  API_BEGIN
  check_mesh(mesh);
  if (!feats || !target || !count || cap < 0) throw std::runtime_error("invalid arguments");
  DevMesh& m = mesh->dm;
  *count = 0;
  if (m.rec_cap == 0) return MM_OK;
  MM_CK(cudaSetDevice(m.device));
  unsigned long long c = 0;
  MM_CK(cudaMemcpyAsync(&c, m.rs_count, sizeof(c), cudaMemcpyDeviceToHost, m.stream));
  MM_CK(cudaStreamSynchronize(m.stream));
  const int64_t k = std::min<int64_t>(std::min<int64_t>((int64_t)c, m.rec_cap), cap);
  if (k == 0) return MM_OK;
  MM_CK(cudaMemcpyAsync(feats, m.rs_feat, sizeof(float) * k * kMlpIn, cudaMemcpyDeviceToHost, m.stream));
  MM_CK(cudaMemcpyAsync(target, m.rs_tgt, sizeof(float) * k, cudaMemcpyDeviceToHost, m.stream));
  std::vector<int32_t> rows(k);
  MM_CK(cudaMemcpyAsync(rows.data(), m.rs_node, sizeof(int32_t) * k, cudaMemcpyDeviceToHost, m.stream));
  MM_CK(cudaStreamSynchronize(m.stream));
  if (node)
    for (int64_t q = 0; q < k; ++q) node[q] = m.h.perm[rows[q]];
  *count = k;
  return MM_OK;
  API_END
}

}  // extern "C"

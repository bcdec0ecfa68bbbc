// P1-tetrahedron element kernels that assemble every operator of the hot path on the
// device, replacing escript/finley's assembly (scripts/matrix.py:9-74,
// scripts/escript_tools.py:13-17, scripts/materials.py:36-41, scripts/trafo.py:24-45):
//
//   V      = sum of |det J|/6 over tets with Js > 0         (warp-shuffle block partials)
//   meas_i = sum_e Js vol/4                                   (node scatter)
//   S      = sum_e vol grad Na . k . grad Nb, k = I or the shell tensor averaged over the
//            4-point Tet4 rule in the last tag; Dirichlet rows/cols -> identity
//   Aex    = (2A/V) vol grad Na . grad Nb                     (exchange, per component)
//   K      = (-2K/V) vol/20 (1+d_ab) u u^T                    (anisotropy, consistent mass)
//   dk     = Js vol/4 d_k Na  (row a, col b)                  (divergence)
//   gk     = Js vol/(4V) d_k Nb                               (gradient = dk^T / V)
//
// Elements are processed one colour at a time; within a colour no two tets share a node,
// so each thread owns the row of its node and the scatter needs no atomics.
#include <cuda_runtime.h>

#include <cmath>
#include <stdexcept>
#include <string>

#include "device_mesh.h"

namespace mumag {

#define CK(call) MM_CK(call)

namespace {

constexpr double kQuadA = 0.5854101966249685;  // 4-point Tet4 rule (barycentric)
constexpr double kQuadB = 0.1381966011250105;

struct Tet {
  double G[4][3];  // gradients of the barycentric shape functions
  double vol;
  double P[4][3];
};

__device__ __forceinline__ void tet_geometry(const double* __restrict__ X, const int32_t* n, Tet& t) {
  for (int a = 0; a < 4; ++a)
    for (int c = 0; c < 3; ++c) t.P[a][c] = X[3 * n[a] + c];
  double J[3][3];  // columns: P1-P0, P2-P0, P3-P0
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) J[r][c] = t.P[c + 1][r] - t.P[0][r];
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const double inv = 1.0 / det;
  // rows of J^-1 are the gradients of barycentric coordinates 1..3
  double Ji[3][3];
  Ji[0][0] = c00 * inv;
  Ji[1][0] = c01 * inv;
  Ji[2][0] = c02 * inv;
  Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * inv;
  Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * inv;
  Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * inv;
  Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * inv;
  Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * inv;
  Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * inv;
  for (int c = 0; c < 3; ++c) {
    t.G[1][c] = Ji[0][c];
    t.G[2][c] = Ji[1][c];
    t.G[3][c] = Ji[2][c];
    t.G[0][c] = -(Ji[0][c] + Ji[1][c] + Ji[2][c]);
  }
  t.vol = fabs(det) / 6.0;
}

// Magnetic volume: per-block partial sums (warp shuffles, then warps in order).
__global__ void k_volume(const double* __restrict__ X, const int32_t* __restrict__ econn,
                         const int32_t* __restrict__ etag, const MatRow* __restrict__ mats,
                         int64_t E, double* __restrict__ part) {
  __shared__ double sw[32];
  double v = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
       e += (int64_t)gridDim.x * blockDim.x) {
    if (mats[etag[e]].Js > 0.0) {
      Tet t;
      tet_geometry(X, econn + 4 * e, t);
      v += t.vol;
    }
  }
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sw[w];
    part[blockIdx.x] = s;
  }
}

struct ScatterArgs {
  const double* X;
  const int32_t* econn;
  const int32_t* etag;
  const MatRow* mats;
  const int64_t* sl_off;
  const int32_t* col;
  const int32_t* rowlen;
  double* vals;
  int64_t nent;
  double* meas;
  double V, R, Rinf;
  int shell_tag;  // tag index carrying the shell tensor, -1 for none (airbox)
};

__device__ __forceinline__ void shell_tensor(const double xq[3], double R, double Rinf, double k[3][3]) {
  // scripts/trafo.py:24-45 (get_T3D)
  const double x = sqrt(xq[0] * xq[0] + xq[1] * xq[1] + xq[2] * xq[2]);
  const double a2 = R * (Rinf - R);
  const double ax = Rinf / x;
  const double a2x2 = a2 / (x * x);
  const double f = ax * (2.0 - ax) / ((ax - 1.0) * (ax - 1.0));
  const double xh[3] = {xq[0] / x, xq[1] / x, xq[2] / x};
  for (int i = 0; i < 3; ++i) k[i][i] = a2x2 * (1.0 + f * (1.0 - xh[i] * xh[i]));
  k[0][1] = k[1][0] = -a2x2 * (f * xh[0] * xh[1]);
  k[0][2] = k[2][0] = -a2x2 * (f * xh[0] * xh[2]);
  k[1][2] = k[2][1] = -a2x2 * (f * xh[1] * xh[2]);
}

// One thread per (element, local node a) of one colour: adds the element's row-a
// contributions into the node's SELL row.
__global__ void k_scatter(ScatterArgs A, int64_t e0, int64_t e1) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t e = e0 + t / 4;
  const int a = (int)(t & 3);
  if (e >= e1) return;
  const int32_t* n = A.econn + 4 * e;
  Tet T;
  tet_geometry(A.X, n, T);
  const MatRow mr = A.mats[A.etag[e]];
  const double vol = T.vol, V = A.V;
  double kb[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  if (A.etag[e] == A.shell_tag) {
    double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int q = 0; q < 4; ++q) {
      double xq[3];
      for (int c = 0; c < 3; ++c) {
        double s = 0.0;
        for (int i = 0; i < 4; ++i) s += (i == q ? kQuadA : kQuadB) * T.P[i][c];
        xq[c] = s;
      }
      double k[3][3];
      shell_tensor(xq, A.R, A.Rinf, k);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) acc[r][c] += k[r][c];
    }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) kb[r][c] = acc[r][c] / 4.0;
  }
  const int32_t row = n[a];
  const int64_t s = row >> 5;
  const int lane = row & 31;
  const int64_t off = A.sl_off[s] + lane;
  const int len = A.rowlen[row];
  const double cex = 2.0 * mr.A / V, cani = -2.0 * mr.K / V;
  const double wd = mr.Js * vol / 4.0;
  double kGa[3];
  for (int c = 0; c < 3; ++c) kGa[c] = kb[c][0] * T.G[a][0] + kb[c][1] * T.G[a][1] + kb[c][2] * T.G[a][2];
  for (int b = 0; b < 4; ++b) {
    int64_t pos = -1;
    for (int k = 0; k < len; ++k)
      if (A.col[off + 32 * (int64_t)k] == n[b]) {
        pos = off + 32 * (int64_t)k;
        break;
      }
    if (pos < 0) continue;  // cannot happen: the pattern holds every element pair
    const double gg = T.G[a][0] * T.G[b][0] + T.G[a][1] * T.G[b][1] + T.G[a][2] * T.G[b][2];
    const double gkg = kGa[0] * T.G[b][0] + kGa[1] * T.G[b][1] + kGa[2] * T.G[b][2];
    double* v = A.vals + pos;
    const int64_t ps = A.nent;
    v[P_S * ps] += gkg * vol;
    v[P_AEX * ps] += (gg * vol) * cex;
    const double mk = ((a == b ? 2.0 : 1.0) * (vol / 20.0)) * cani;
    v[(P_K + 0) * ps] += mk * (mr.u[0] * mr.u[0]);
    v[(P_K + 1) * ps] += mk * (mr.u[0] * mr.u[1]);
    v[(P_K + 2) * ps] += mk * (mr.u[0] * mr.u[2]);
    v[(P_K + 3) * ps] += mk * (mr.u[1] * mr.u[1]);
    v[(P_K + 4) * ps] += mk * (mr.u[1] * mr.u[2]);
    v[(P_K + 5) * ps] += mk * (mr.u[2] * mr.u[2]);
    for (int c = 0; c < 3; ++c) {
      v[(P_D + c) * ps] += T.G[a][c] * wd;
      v[(P_G + c) * ps] += (T.G[b][c] * wd) / V;
    }
  }
  A.meas[row] += wd;
}

// Dirichlet rows/columns of S -> identity (escript nullifyRowsAndCols with diagonal 1),
// diagonals, the M_inv preconditioner D (exchange diagonal, 1 where meas = 0,
// scripts/mapping.py:207-209), and optionally a zero right-hand side on Dirichlet rows.
__global__ void k_finalize(const int64_t* __restrict__ sl_off, const int32_t* __restrict__ sl_w,
                           const int32_t* __restrict__ col, const int32_t* __restrict__ rowlen,
                           const uint8_t* __restrict__ bnd, double* vals, int64_t nent,
                           const double* __restrict__ meas, double* diagS, double* invdS,
                           double* Dex, int Npad, int zero_rhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Npad) return;
  const int64_t s = i >> 5;
  const int lane = i & 31;
  const int w = sl_w[s];
  double dS = 1.0, dA = 1.0;
  for (int k = 0; k < w; ++k) {
    const int64_t e = sl_off[s] + 32 * (int64_t)k + lane;
    const int j = col[e];
    if (k >= rowlen[i]) continue;
    if (bnd[i] || bnd[j]) vals[P_S * nent + e] = (i == j && bnd[i]) ? 1.0 : 0.0;
    if (zero_rhs && bnd[i])
      for (int c = 0; c < 3; ++c) vals[(P_D + c) * nent + e] = 0.0;
    if (j == i) {
      dS = vals[P_S * nent + e];
      dA = vals[P_AEX * nent + e];
    }
  }
  if (rowlen[i] == 0) dS = 1.0;
  diagS[i] = dS;
  invdS[i] = 1.0 / dS;
  Dex[i] = (meas[i] == 0.0) ? 1.0 : dA;
}

// FP32 copies of every operator plane (mixed precision reads them, accumulating in FP64).
__global__ void k_to_f32(const double* __restrict__ vals, float* __restrict__ v32, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    v32[t] = (float)vals[t];
}

}  // namespace

void assemble_operators(DevMesh& m) {
  const HostMesh& h = m.h;
  cudaStream_t st = m.stream;
  // magnetic volume
  const int vb = 256;
  int vg = (int)std::min<int64_t>((h.E + vb - 1) / vb, 4096);
  double* part = nullptr;
  CK(cudaMalloc(&part, sizeof(double) * vg));
  k_volume<<<vg, vb, 0, st>>>(m.Xd, m.econn, m.etag, m.dmats, h.E, part);
  CK(cudaGetLastError());
  std::vector<double> hp(vg);
  CK(cudaMemcpyAsync(hp.data(), part, sizeof(double) * vg, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  CK(cudaFree(part));
  double V = 0.0;
  for (double p : hp) V += p;
  if (!(V > 0.0)) throw std::runtime_error("no magnetic material (every Js <= 0)");
  m.V = V;
  // element scatter, one launch per colour
  CK(cudaMemsetAsync(m.vals, 0, sizeof(double) * kNumPlanes * h.nent, st));
  CK(cudaMemsetAsync(m.meas, 0, sizeof(double) * h.Npad, st));
  ScatterArgs A;
  A.X = m.Xd;
  A.econn = m.econn;
  A.etag = m.etag;
  A.mats = m.dmats;
  A.sl_off = m.sl_off;
  A.col = m.col;
  A.rowlen = m.rowlen;
  A.vals = m.vals;
  A.nent = h.nent;
  A.meas = m.meas;
  A.V = V;
  A.R = h.R;
  A.Rinf = h.Rinf;
  A.shell_tag = h.airbox ? -1 : (int)h.tags.size() - 1;
  for (size_t c = 0; c + 1 < h.colour_off.size(); ++c) {
    const int64_t e0 = h.colour_off[c], e1 = h.colour_off[c + 1];
    const int64_t nt = 4 * (e1 - e0);
    if (nt == 0) continue;
    const int tb = 128;
    k_scatter<<<(unsigned)((nt + tb - 1) / tb), tb, 0, st>>>(A, e0, e1);
    CK(cudaGetLastError());
  }
  k_finalize<<<(unsigned)((h.Npad + 255) / 256), 256, 0, st>>>(
      m.sl_off, m.sl_w, m.col, m.rowlen, m.bnd, m.vals, h.nent, m.meas, m.diagS, m.invdS, m.Dex,
      (int)h.Npad, m.opt.dirichlet_rhs == MM_DIRICHLET_RHS_ZERO);
  CK(cudaGetLastError());
  if (m.vals32) {
    static_assert(kNumPlanes32 == kNumPlanes, "FP32 planes mirror the FP64 planes");
    k_to_f32<<<592, 256, 0, st>>>(m.vals, m.vals32, (int64_t)kNumPlanes * h.nent);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(st));
}

}  // namespace mumag

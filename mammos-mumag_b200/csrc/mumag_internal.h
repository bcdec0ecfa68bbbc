// Internal declarations shared by the host preprocessing (preprocess.cpp), the device
// kernels (assemble.cu, solver.cu) and the C ABI (capi.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mumag_b200.h"

namespace mumag {

constexpr int kSlice = 32;      // SELL slice height = one warp, lane = row
constexpr int kMaxRed = 8;      // values per grid reduction
constexpr int kNumPlanes = 14;  // S, Aex, K[6], D[3], G[3]
constexpr int kMaxGrid = 480;   // CTAs a persistent launch may use (reduction coverage)
constexpr int64_t kPcg2Nodes = 100000;  // default to the two-sync PCG from this many nodes
constexpr int kMaxCoarse = 2048;        // aggregates of the two-level Poisson preconditioner
constexpr int kMinBoxNodes = 32;        // smallest aggregate box (so a SELL slice meets <= 2 boxes)

// Value planes of the node-pair operators, all on one SELL-32 pattern.
enum Plane {
  P_S = 0,     // Poisson stiffness (with Dirichlet rows/cols -> identity)
  P_AEX = 1,   // exchange scalar (2A/V) int grad Ni . grad Nj
  P_K = 2,     // 6 planes: anisotropy block (-2K/V) int Ni Nj u u^T, xx xy xz yy yz zz
  P_D = 8,     // 3 planes: divergence dk_ij = int Js Nj d_k Ni
  P_G = 11     // 3 planes: gradient gk_ij = (1/V) int Js Ni d_k Nj
};

// Host-side result of preprocessing one mesh.
struct HostMesh {
  int64_t N = 0, E = 0, Npad = 0, nslices = 0, nent = 0, nnz = 0;
  std::vector<int32_t> perm;     // perm[new] = old
  std::vector<int32_t> iperm;    // iperm[old] = new
  std::vector<int64_t> sl_off;   // [nslices+1] entry offset of each slice
  std::vector<int32_t> sl_w;     // [nslices] slice width
  std::vector<int32_t> col;      // [nent]
  std::vector<int32_t> rowlen;   // [Npad]
  std::vector<int32_t> econn;    // [E*4] colour-sorted elements, device node ids
  std::vector<int32_t> etag;     // [E] tag index of each colour-sorted element
  std::vector<int64_t> colour_off;  // [ncolours+1]
  std::vector<uint8_t> bnd;      // [Npad] Dirichlet mask (device order)
  std::vector<double> Xd;        // [Npad*3] coordinates in device order
  std::vector<int32_t> tags;     // sorted unique element tags
  int airbox = 0;
  double R = 0.0, Rinf = 0.0;    // shell radii (shell branch)
  int64_t bandwidth_before = 0, bandwidth_after = 0;
  // two-level Poisson preconditioner: aggregate ("box") of each device row, -1 for Dirichlet
  // and padding rows; nc aggregates, numbered in device-row order
  int32_t nc = 0;
  std::vector<int32_t> rbox;     // [Npad]
};

// Build everything the device needs. Throws std::runtime_error on bad input.
// coarse_nodes > 0 also groups the interior nodes into spatial boxes of about that many nodes
// for the two-level preconditioner and numbers the nodes box by box (reverse Cuthill-McKee
// order inside a box).
void preprocess(const double* X, int64_t N, const int32_t* T, const int32_t* tag, int64_t E,
                int32_t nmats, bool reorder, int32_t coarse_nodes, HostMesh& out);

// In place: A [n][n] (symmetric positive definite, nonzero only within `bw` of the
// diagonal) becomes A^-1, by a banded Cholesky factorisation and one pair of triangular
// solves per column (columns on host threads).  Throws if A is not positive definite.
void spd_inverse(int32_t n, int32_t bw, std::vector<double>& A);

std::vector<int32_t> rcm_order(int64_t N, const int32_t* T, int64_t E);
int32_t greedy_colour(int64_t N, const int32_t* T, int64_t E, const int64_t* order,
                      int32_t* colour);

void set_error(const std::string& msg);

}  // namespace mumag

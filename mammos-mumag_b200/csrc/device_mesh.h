// Device-resident mesh, operators and solver state, plus the launchers of the CUDA
// kernels (assemble.cu, solver.cu).  Host code only; no device code here.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "mlp.cuh"
#include "mumag_internal.h"

namespace mumag {

// A failed CUDA runtime call (mapped to MM_CUDA_ERROR at the C ABI).
struct CudaFailure : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// On failure the runtime's last-error state is cleared too, so a failed (non-sticky) call
// does not resurface in a later, unrelated cudaGetLastError().
#define MM_CK(call)                                                                          \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      (void)cudaGetLastError();                                                              \
      throw ::mumag::CudaFailure(std::string(#call) + ": " + cudaGetErrorString(e_) + " (" + \
                                 __FILE__ + ":" + std::to_string(__LINE__) + ")");           \
    }                                                                                        \
  } while (0)

// Materials per element tag, scripts/materials.py:17-35: Js [T], K = mu0*K1,
// A = mu0*A/size^2, easy axis u.  All zero for Js <= 0.
struct MatRow {
  double Js, K, A, u[3];
};

// One node's Poisson-PCG state in the Chronopoulos-Gear iteration: r_i, w_i = S z_i,
// s_{i-1} and 1/diag S.  Stored as four planes of a buffer (solver.cu rec_load/rec_store).
struct __align__(32) PcgRec {
  double r, w, s, invd;
};

// The same record in FP32, for the inner iterations of the mixed-precision solve.
struct __align__(16) PcgRec32 {
  float r, w, s, invd;
};

constexpr int kResI = 9;       // integer results of a launch (SolveArgs::resi)
constexpr int kProfCols = 12;  // per-CTA timers of SolveArgs::prof
constexpr int kNumPlanes32 = kNumPlanes;  // FP32 copies of every plane (mixed precision)

// Arguments of the persistent solver kernel (passed by value, __grid_constant__).
struct SolveArgs {
  // SELL-32 pattern and operator planes (plane stride nent)
  const int64_t* sl_off;
  const int32_t* sl_w;
  const int32_t* col;
  const double* vals;  // [kNumPlanes][nent]
  int64_t nent;
  const double* invdS;
  const double* Dex;
  const double* meas;
  int32_t nslices, Npad;
  double V;
  // vectors; 3-vectors are 3 planes of Npad
  double *x, *x1, *g, *g1, *d, *gf, *mbar, *zp, *tr, *tz, *td, *tBd;
  double* u;        // magnetostatic potential (PCG solution)
  PcgRec* rec[2];   // PCG records, double-buffered by iteration parity
  double* pp;       // PCG search direction
  // mixed precision: FP32 operator planes and inner-solve state
  int mixed;
  const float* vals32;  // [kNumPlanes32][nent]: FP32 copies of the planes of vals
  PcgRec32* rec32[2];
  float *pp32, *e32;    // inner search direction and correction
  double* r64;          // FP64 residual of the outer refinement
  int pcg2;             // 1: two-sync PCG iteration (z gathered alone), 0: one-sync
  // Poisson warm start (MM_WARM_*): previous u, zero, or previous u + the learned correction
  int warm;
  double warm_gate2;    // the learned start runs only when r.r > warm_gate2 * tol_u^2 b.b
  int32_t nreal;        // real (non-padding) rows
  MlpDev mlp;           // learned warm start: the model
  float* feat;          // [Npad][kMlpIn] node features of the learned start
  float* du;            // [Npad] its predicted correction (units of sigma)
  int tc_off;           // >= 0: dynamic shared-memory offset of the tensor-core network's
                        // region (learned start on tcgen05); -1: the network runs on mma.sync
  // two-level Poisson preconditioner (nc > 0; 0 = Jacobi): z = r/diag + P Ac^-1 P^T r with P
  // constant on aggregates ("boxes") of rows and Ac = P^T S P
  int nc;
  const int32_t* rbox;  // [Npad] box of each row, -1 for Dirichlet and padding rows
  const double* Ainv;   // [nc][nc] Ac^-1
  const float* Ainv32;  // [nc][nc] Ac^-1 in FP32 (mixed precision's inner iterations)
  double* bslots;       // box partial sums, one slot per (CTA, box it holds rows of)
  const int32_t* bslot; // [nc+1] box c's partial sums are slots [bslot[c], bslot[c+1])
  const int32_t* ctabox;  // [grid][3] first box, number of boxes and first slot of each CTA
  int co_off;           // dynamic shared-memory offset of the coarse vectors
  int co_rows;          // > 0: each CTA keeps its rows of Ainv32 in shared memory (capacity)
  // training-sample recording (rec_cap > 0): at a hash-selected 1/rec_stride of the
  // (node, solve) pairs, the node's features at the warm start and, after the solve,
  // the target (u - u0) / sigma
  float* rs_feat;       // [rec_cap][kMlpIn]
  float* rs_tgt;        // [rec_cap]
  double* rs_u0;        // [rec_cap]
  int32_t* rs_node;     // [rec_cap] device row
  int32_t* rs_slot;     // [Npad] sample slot of the row in the current solve, -1 = none
  unsigned long long* rs_count;
  long long rec_cap;
  int rec_stride;
  unsigned rec_seed;
  // grid synchronisation
  unsigned long long* bar;    // barrier arrival counter, zeroed before each launch
  int bar_stall;              // test hook: extra arrivals each barrier waits for (0 = normal)
  double* red;                // [2][kMaxRed][gridDim.x] reduction partials
  int* flags;                 // [0] abort, [1] status
  int stage;                  // 1: the CTA's SELL columns + Poisson values live in shared memory
  int64_t stage_max;          // entries of the largest CTA (shared-memory layout)
  int64_t meta_max;           // slices of the largest CTA (shared-memory slice metadata)
  // control
  int mode;  // 0 energy+gradient, 1 M_inv, 2 minimise (one field step), 3 idle, 4 field sweep
  double h, hdir[3], tol_fun, sqrt_tol, cbrt_tol, tol_u;
  int precond_iter, hmag_on, mbar_current, max_pcg, max_ncg;
  // field sweep inside one launch (MODE_SWEEP): from h by sw_hstep, scripts/loop.py:71-124
  double sw_hstep, sw_mstep, sw_mfinal;
  int sw_nmax;
  double* sw_rec;       // [sw_nmax][4] counter, hext, mh, energy
  long long* sw_stat;   // [sw_nmax][8] ncg, evals, pcg, shrinks, minv, ns, sync ns, barriers
  int* sw_nrec;         // rows written
  // optional per-CTA timing [gridDim.x][kProfCols] ns (null = off): PCG row phases, reduction
  // before the barrier, barrier wait, partial read after the barrier, whole Poisson solves,
  // M_inv applications, energy evaluations (solves included), the launch, and the
  // two-level preconditioner's publish, gather and own-box solve steps
  long long* prof;
  // results
  double* resd;     // [0] energy, [1] mh
  long long* resi;  // [kResI]: ncg iters, evals, pcg iters, ls shrinks, minv iters, kernel ns,
                    // sync ns, barriers, learned starts applied
};

enum { WARM_PREV = 0, WARM_ZERO = 1, WARM_LEARNED = 2 };
enum { MODE_EVAL = 0, MODE_MINV = 1, MODE_MINIMIZE = 2, MODE_IDLE = 3, MODE_SWEEP = 4 };
enum { FLAG_ABORT = 0, FLAG_STATUS = 1 };

struct DevMesh {
  int device = 0;
  HostMesh h;
  mm_options opt{};
  cudaStream_t stream = nullptr;
  std::vector<MatRow> mats;
  int32_t ncolours = 0;
  double V = 0.0;
  // pattern + operators
  int64_t* sl_off = nullptr;
  int32_t* sl_w = nullptr;
  int32_t* col = nullptr;
  int32_t* rowlen = nullptr;
  double* vals = nullptr;
  double *diagS = nullptr, *invdS = nullptr, *Dex = nullptr, *meas = nullptr;
  uint8_t* bnd = nullptr;
  double* Xd = nullptr;
  int32_t *econn = nullptr, *etag = nullptr;
  MatRow* dmats = nullptr;
  // state and workspace
  double* ws = nullptr;  // all solver vectors
  double *x, *x1, *g, *g1, *d, *gf, *mbar, *zp, *tr, *tz, *td, *tBd;
  double *u, *pp;
  PcgRec* rec[2];
  float* vals32 = nullptr;
  PcgRec32* rec32[2] = {nullptr, nullptr};
  float *pp32 = nullptr, *e32 = nullptr;
  double* r64 = nullptr;
  int pcg2 = 0;  // PCG arrangement (SolveArgs::pcg2)
  int bar_stall = 0;  // test hook (SolveArgs::bar_stall)
  // warm start and sample recording (SolveArgs)
  int warm = 0;
  double warm_gate = 0.0;  // mm_mesh_set_learned_gate
  MlpDev mlp{};
  float *feat = nullptr, *du = nullptr;
  float *rs_feat = nullptr, *rs_tgt = nullptr;
  double* rs_u0 = nullptr;
  int32_t *rs_node = nullptr, *rs_slot = nullptr;
  unsigned long long* rs_count = nullptr;
  long long rec_cap = 0;
  int rec_stride = 1;
  unsigned rec_seed = 0;
  unsigned long long* bar = nullptr;
  double* red = nullptr;
  int* flags = nullptr;
  double* resd = nullptr;
  long long* resi = nullptr;
  long long* prof = nullptr;  // [grid][4] when MUMAG_PROFILE is set
  // pinned host mirrors of the results
  double* h_resd = nullptr;
  long long* h_resi = nullptr;
  int* h_flags = nullptr;
  // launch shape of the persistent kernel and its build (resident CTAs per SM, 2 or 3)
  int grid = 0, block = 0;
  int kernel_mb = 2;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;    // mm_timer_*
  cudaEvent_t evk0 = nullptr, evk1 = nullptr;  // around each persistent launch
  float last_launch_ms = 0.f;
  int stage = 0;
  int64_t stage_max = 0, meta_max = 0;
  size_t smem = 0;
  int tc_off = -1;  // SolveArgs::tc_off
  // two-level preconditioner (SolveArgs): nc boxes, 0 = Jacobi
  int nc = 0;
  int32_t* rbox = nullptr;
  double* Ainv = nullptr;
  float* Ainv32 = nullptr;
  double* bslots = nullptr;
  int32_t* bslot = nullptr;
  int32_t* ctabox = nullptr;
  int32_t* d_iperm = nullptr;  // iperm on the device (device-resident state transfers)
  int* d_bad = nullptr;
  int co_off = -1;
  int co_rows = 0;
};

// A batched persistent launch over several meshes: mesh q runs on CTAs
// [group[q], group[q+1]) with its own staging decision for that group size.
struct BatchPlan {
  std::vector<int> group;
  std::vector<int> stage;
  std::vector<int64_t> stage_max, meta_max;
  int grid = 0, block = 256;
  size_t smem = 0;
};

// assemble.cu
void assemble_operators(DevMesh& m);
// solver.cu
void solver_configure(DevMesh& m);
cudaError_t solver_launch(DevMesh& m, const SolveArgs& a);
SolveArgs solver_args(const DevMesh& m, int mode, double h, const mm_solver_params& sp);
cudaError_t launch_prep(DevMesh& m, cudaStream_t st);
void batch_configure(const std::vector<DevMesh*>& ms, BatchPlan& plan);
cudaError_t batch_launch(const BatchPlan& plan, const SolveArgs* d_args, const int* d_group, int count,
                         cudaStream_t st);

}  // namespace mumag

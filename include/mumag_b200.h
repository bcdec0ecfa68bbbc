/*
 * mumag_b200.h -- C ABI of libmumag_b200.so, the B200 (sm_100a) back end of the
 * hysteresis-loop hot path of mammos-mumag.
 *
 * The reference runs its hot path as a subprocess, `run-escript scripts/loop.py <name>`
 * (src/mammos_mumag/simulation.py:88-113 run_script, :258-305 run_loop), whose solver core is a set of
 * jitted JAX functions over escript-assembled sparse operators.  This library replaces
 * that subprocess: the Python host (mammos_mumag.Simulation.run_loop) calls it in process.
 * Plain C types only; host arrays are owned by the caller; device state lives behind an
 * opaque mesh handle.  Every call returns an mm_status; on failure mm_last_error() holds
 * a message.
 *
 * Layouts at this boundary are the reference's:
 *   X    [N][3]  node coordinates in mesh-file order (nm), double
 *   T    [E][4]  tetrahedra, 0-based node indices, int32
 *   tag  [E]     element tags, int32; material row i belongs to the i-th tag in
 *                ascending order (scripts/materials.py:22-25)
 *   m    [3N]    interleaved magnetisation [mx0,my0,mz0,mx1,...] (scripts/converters.py:36-37)
 *   u    [N]     magnetostatic scalar potential
 * Energies are in the reference's internal units (J/m^3 times mu0); divide by
 * scipy.constants.mu_0 for the .dat column (scripts/tools.py:20-24).
 */
#ifndef MUMAG_B200_H
#define MUMAG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int mm_status;
enum {
  MM_OK = 0,
  MM_BAD_INPUT = 1,    /* invalid sizes, indices, materials, or a missing mesh handle */
  MM_CUDA_ERROR = 2,   /* a CUDA runtime call failed (message in mm_last_error) */
  MM_NONFINITE = 3,    /* the energy became NaN/Inf during a solve */
  MM_TIMEOUT = 4,      /* a device-side grid barrier gave up waiting (kernel returned early) */
  MM_NO_DEVICE = 5     /* no usable sm_100 device */
};

/* One .krn row (src/mammos_mumag/templates/krn.jinja:1-3): theta phi K1 K2 Js A.
 * Js in T, K1/K2 in J/m^3, A in J/m.  K2 is carried but, as in the reference
 * (scripts/materials.py:28-34), not used. */
typedef struct {
  double theta, phi, K1, K2, Js, A;
} mm_material;

enum { MM_PREC_FP64 = 0, MM_PREC_MIXED = 1 };
enum { MM_DIRICHLET_RHS_REFERENCE = 0, MM_DIRICHLET_RHS_ZERO = 1 };

typedef struct {
  double size;         /* length unit of X in m; the reference fixes 1e-9 (scripts/materials.py:13) */
  int dirichlet_rhs;   /* MM_DIRICHLET_RHS_*: Poisson right-hand side on Dirichlet nodes */
  int precision;       /* MM_PREC_*: arithmetic of the operator kernels */
  int device;          /* CUDA device ordinal */
  int grid_ctas;       /* persistent-kernel CTAs; 0 = autotuned */
  int block_threads;   /* threads per CTA; 0 = autotuned */
  int reorder;         /* 1 = reverse Cuthill-McKee node order on the device (default), 0 = file order */
  int pcg_variant;     /* Poisson PCG arrangement: 0 = chosen by size and mm_autotune (default),
                          1 = one grid synchronisation per iteration (neighbour z recomputed
                          from gathered r, w, s), 2 = two (z stored, gathered alone); both
                          give the same iterates */
  int ctas_per_sm;     /* build of the persistent kernel: 0 = chosen by mm_autotune (2 until
                          then), 2 or 3 resident CTAs per SM (128 or 80 registers per thread) */
  int stage_operators; /* 1 (default): each CTA keeps its SELL columns and Poisson values in
                          shared memory when they fit; 0: always read them from HBM (the
                          large-mesh path, selectable on any mesh; results are identical) */
  int coarse_box_nodes; /* Poisson preconditioner: 0 (default) = Jacobi, the reference's
                          (scripts/solvers.py:221-231); > 0 = two-level additive
                          M^-1 = D^-1 + P (P^T S P)^-1 P^T with P constant on spatial boxes
                          of about this many interior nodes (at most 2,048 boxes; nodes are
                          then numbered box by box).  No counterpart in the reference: only
                          the path to the solution changes, the stop test r.r <= tol_u^2 b.b
                          stays.  Batched launches always use Jacobi. */
} mm_options;

/* Solver settings of one field step (scripts/tools.py:64-120, scripts/minimizers.py:140-190). */
typedef struct {
  double hdir[3];      /* unit field direction (the .p2 [field] hx,hy,hz normalised) */
  double tol_fun;      /* NCG tolerance (tol_fun) */
  double tol_u;        /* Poisson PCG relative residual tolerance (tol_fun * tol_hmag_factor) */
  int precond_iter;    /* truncated-CG iterations of the M_inv preconditioner */
  int hmag_on;         /* 0 disables the magnetostatic term */
  int mbar_mode;       /* 0: M_inv projects with the loop's initial m (the reference,
                          scripts/loop.py:50-52); 1: with the current iterate */
  int max_pcg_iter;    /* Poisson PCG cap (reference 10000, scripts/solvers.py:222) */
  int max_ncg_iter;    /* NCG cap (reference 100000, scripts/minimizers.py:142) */
} mm_solver_params;

/* Result of one field step. */
typedef struct {
  double energy;       /* total energy at the minimiser (internal units) */
  double mh;           /* magnetic polarisation along hdir, T (scripts/loop.py:25-38) */
  int64_t ncg_iters;   /* NCG iterations k as returned by hestenes_stiefel_ncg */
  int64_t evals;       /* energy+gradient evaluations */
  int64_t pcg_iters;   /* Poisson PCG iterations summed over the evaluations */
  int64_t ls_shrinks;  /* line-search step halvings */
  int64_t minv_iters;  /* truncated-CG iterations inside M_inv */
  int64_t kernel_ns;   /* device time of the persistent launch (CTA 0, %globaltimer) */
  int64_t sync_ns;     /* of which spent in grid barriers / reductions */
  int64_t barriers;    /* grid barriers executed */
  double device_ms;    /* duration of the launch from CUDA events on the launching stream */
  int status;          /* MM_OK, MM_NONFINITE or MM_TIMEOUT */
  int64_t learned_starts;  /* Poisson solves that took the learned warm start */
} mm_step_result;

typedef struct {
  int64_t nodes, elements;
  int64_t sell_slices, sell_entries;   /* SELL-32 Poisson/operator pattern */
  int64_t nnz;                         /* unpadded node-pair entries */
  int32_t colours;                     /* element colours used by the assembly kernels */
  int32_t airbox;                      /* 1: bare-box Dirichlet branch, 0: spherical shell */
  int32_t grid_ctas, block_threads;    /* persistent-kernel launch shape in use */
  int64_t dirichlet_nodes;
  double volume;                       /* magnetic volume V, nm^3 */
  double bandwidth_before, bandwidth_after;  /* max |i-j| over node pairs, file vs device order */
  int32_t pcg_variant;                 /* PCG arrangement in use: 1 one-sync, 2 two-sync */
  int32_t kernel_ctas_per_sm;          /* build of the persistent kernel in use: 2 or 3 resident
                                          CTAs per SM (128 or 80 registers per thread) */
  int32_t staged;                      /* 1: SELL columns + Poisson values in shared memory */
  int32_t coarse_boxes;                /* boxes of the two-level preconditioner (0 = Jacobi) */
} mm_mesh_info;

/* Field-sweep parameters (the .p2 [field] section; scripts/loop.py:71-142). */
typedef struct {
  double hstart, hfinal, hstep, mstep, mfinal;
  int32_t max_steps;   /* <= 0: int(|hfinal-hstart|/|hstep|)+1 as the reference */
} mm_loop_params;

/* One .dat row: vtk counter, mu0*Hext [T], polarisation [T], energy (internal units). */
typedef struct {
  double counter, hext, mh, energy;
} mm_record;

/* Called where the reference writes <name>_<counter:04d>.vtu (scripts/loop.py:103-116):
 * m [3N] and u [N] in mesh-file order, valid for the duration of the call.
 * A non-zero return aborts the loop with MM_BAD_INPUT. */
typedef int (*mm_snapshot_cb)(int counter, const double* m, const double* u, int64_t n, void* user);

typedef struct mm_mesh mm_mesh;

/* Library version string. */
const char* mm_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char* mm_last_error(void);

/* Default options / solver parameters (the reference's defaults). */
void mm_default_options(mm_options* opt);
void mm_default_solver_params(mm_solver_params* sp);

/* Number of usable sm_100 devices (0 without a GPU; never fails). */
int mm_device_count(void);

/* ---- host-only mesh utilities (no GPU needed) ---------------------------------------- */

/* Reverse Cuthill-McKee order of the node graph of T: perm[new] = old.
 * Replaces nothing in the reference (escript keeps its own DOF order); used to make the
 * device gathers local. */
mm_status mm_rcm_permutation(int64_t N, const int32_t* T, int64_t E, int32_t* perm);

/* Greedy element colouring: no two elements of one colour share a node.  colour[e] in
 * [0, *ncolours).  Used so the assembly scatters are atomic-free. */
mm_status mm_color_elements(int64_t N, const int32_t* T, int64_t E, int32_t* colour,
                            int32_t* ncolours);

/* ---- mesh handle ---------------------------------------------------------------------- */

/* Build the device operators of one mesh: replaces escript2arrays
 * (scripts/mapping.py:171-236) -- materials (scripts/materials.py:12-41), meas
 * (scripts/escript_tools.py:13-17), exchange+anisotropy C and its exchange diagonal D
 * (scripts/matrix.py:37-47, scripts/mapping.py:203-210), divergence dk and gradient gk
 * (scripts/matrix.py:9-35), and the Poisson matrix with its boundary treatment
 * (scripts/matrix.py:49-74, scripts/trafo.py:4-45). */
/* The host preprocessing (node order, SELL pattern, element colouring, boundary branch,
 * aggregate boxes) and the two-level preconditioner's coarse inverse are cached per process
 * for the last four meshes, keyed by the exact X, T, tag and the reorder / coarse_box_nodes
 * options (the counterpart of the reference's scripts/store.py pickles, scripts/store.py:8-23):
 * creating the same mesh again repeats only the device assembly. */
mm_status mm_mesh_create(const double* X, int64_t N, const int32_t* T, const int32_t* tag,
                         int64_t E, const mm_material* mats, int32_t nmats,
                         const mm_options* opt, mm_mesh** out);
mm_status mm_mesh_destroy(mm_mesh* mesh);
mm_status mm_mesh_get_info(const mm_mesh* mesh, mm_mesh_info* info);

/* The two-level preconditioner's aggregates: box [N] (mesh-file order) receives the box of
 * every node (-1 for Dirichlet nodes), *nboxes their number (0 = Jacobi, box untouched).
 * No counterpart in the reference; for checks of the preconditioner. */
mm_status mm_mesh_get_coarse(const mm_mesh* mesh, int32_t* box, int32_t* nboxes);

/* Node measure meas [N] (mesh-file order) and the magnetic volume. */
mm_status mm_get_meas(mm_mesh* mesh, double* meas, double* volume);

/* Export the assembled operators as COO triplets in mesh-file order (parity checks).
 * which: 0 S (Poisson, Dirichlet-modified), 1 exchange scalar (2A/V)K, 2..7 anisotropy
 * blocks xx,xy,xz,yy,yz,zz, 8..10 dx,dy,dz, 11..13 gx,gy,gz.
 * With rows == NULL only *nnz is returned. */
mm_status mm_get_operator(mm_mesh* mesh, int32_t which, int64_t* nnz, int32_t* rows,
                          int32_t* cols, double* vals);

/* Set the solver state: m [3N] (required), u [N] (NULL: zeros), mbar [3N] the
 * magnetisation M_inv projects with (NULL: m).  The full gradient carried between
 * steps is reset to 0 as at scripts/loop.py:84. */
mm_status mm_set_state(mm_mesh* mesh, const double* m, const double* u, const double* mbar);
/* Read the state back; any pointer may be NULL. gfull [3N] is the last full gradient. */
mm_status mm_get_state(mm_mesh* mesh, double* m, double* u, double* gfull);

/* Device-resident forms of mm_set_state / mm_get_state: the same arrays and layouts
 * (interleaved m [3N] and mbar [3N], u [N], gfull [3N], mesh-file order), but as pointers to
 * memory on the mesh's device, so a caller whose state already lives on the GPU (as the
 * reference's total_eg takes JAX device arrays, scripts/energies.py:67-99) avoids the host
 * round trip.  The permutation to the device layout runs on the mesh's stream; both calls
 * return when it has finished.  A non-finite input is refused with MM_BAD_INPUT (the state
 * is then undefined: set it again). */
mm_status mm_set_state_device(mm_mesh* mesh, const double* m, const double* u, const double* mbar);
mm_status mm_get_state_device(mm_mesh* mesh, double* m, double* u, double* gfull);

/* One energy + gradient evaluation, total_eg (scripts/energies.py:67-99), at the state's
 * m with the state's u as PCG warm start; u and gfull in the state are updated.
 * Outputs (NULL allowed): *energy, gproj [3N] = m x (g x m), *pcg_iters. */
mm_status mm_energy_grad(mm_mesh* mesh, double h, const mm_solver_params* sp, double* energy,
                         double* gproj, int64_t* pcg_iters);

/* The M_inv preconditioner (scripts/loop.py:40-55) applied to g [3N]: z [3N]. Uses the
 * state's mbar and gfull. */
mm_status mm_apply_minv(mm_mesh* mesh, const mm_solver_params* sp, const double* g, double* z,
                        int64_t* iters);

/* One field step: hestenes_stiefel_ncg (scripts/minimizers.py:140-190) on the resident
 * state at applied field h (T), then mh.  One persistent launch. */
mm_status mm_minimize(mm_mesh* mesh, double h, const mm_solver_params* sp, mm_step_result* res);

/* The field sweep, solve() + loop() (scripts/loop.py:71-142): starts from the state set by
 * mm_set_state.  rec must hold max_steps rows; *nrec receives the rows written.  steps
 * (NULL allowed) receives one mm_step_result per row.  cb may be NULL. */
mm_status mm_loop(mm_mesh* mesh, const mm_loop_params* lp, const mm_solver_params* sp,
                  mm_record* rec, int32_t* nrec, mm_step_result* steps, mm_snapshot_cb cb,
                  void* user);

/* Autotune the persistent launch shape of this mesh (no counterpart in the reference): times
 * a cold Poisson solve + energy evaluation at the current state for a few launch shapes --
 * the kernel built for two resident CTAs per SM at one, one and a half and two CTAs per SM,
 * the build for three at two and three per SM -- each with both PCG arrangements unless
 * options.pcg_variant fixes one, and keeps the fastest; u and the full gradient are
 * restored.  Results are cached per mesh shape, precision, warm-start kind and the
 * pcg_variant / ctas_per_sm options for the process.  *grid_out (may be NULL) receives the
 * CTA count chosen. */
mm_status mm_autotune(mm_mesh* mesh, const mm_solver_params* sp, int32_t* grid_out);

/* ---- batched persistent launch ----------------------------------------------------------
 *
 * Several independent meshes stepped together in ONE cooperative launch: mesh q runs on a
 * group of CTAs sized in proportion to its rows, with barriers and reductions local to the
 * group, so the meshes' iterations proceed independently inside the launch.  This is the
 * batched form of mm_minimize / mm_loop (no counterpart in the reference, which runs one
 * loop per process); each mesh keeps its own state (mm_set_state / mm_get_state). */
typedef struct mm_batch mm_batch;

/* The meshes must live on one device; count <= number of SMs.  The handles stay owned by
 * the caller and must outlive the batch. */
mm_status mm_batch_create(mm_mesh* const* meshes, int32_t count, mm_batch** out);
mm_status mm_batch_destroy(mm_batch* batch);
/* CTAs assigned to mesh q (group[q+1]-group[q]); group has count+1 entries. */
mm_status mm_batch_groups(const mm_batch* batch, int32_t* group);

/* One field step of every mesh: h[q], sp[q], res[q] (count each). */
mm_status mm_batch_minimize(mm_batch* batch, const double* h, const mm_solver_params* sp, mm_step_result* res);

/* The field sweep of every mesh (all share lp; sp[q] per mesh), each mesh's whole sweep
 * inside ONE launch: its CTA group runs the reference's loop (scripts/loop.py:71-124: field
 * steps, cumulative field update, mfinal stop, snapshot counter) on the device, independent
 * of the other groups, so a mesh never waits for another mesh's field step.  rec holds
 * count x max_steps rows (mesh-major), nrec[q] the rows written for mesh q, steps (may be
 * NULL) count x max_steps results (device_ms 0; kernel_ns is the step's device time).
 * No snapshot callback. */
mm_status mm_batch_loop(mm_batch* batch, const mm_loop_params* lp, const mm_solver_params* sp, int32_t max_steps,
                        mm_record* rec, int32_t* nrec, mm_step_result* steps);

/* Device timing on the mesh's CUDA stream: mm_timer_start records an event; mm_timer_stop
 * records a second one, waits for it and returns the elapsed milliseconds between them.
 * Used to time field sweeps with CUDA events on the stream the kernels run on. */
mm_status mm_timer_start(mm_mesh* mesh);
/* The same for a batch's stream. */
mm_status mm_batch_timer_start(mm_batch* batch);
mm_status mm_batch_timer_stop(mm_batch* batch, double* elapsed_ms);

/* Diagnostic per-CTA phase timers, collected only when the environment variable
 * MUMAG_PROFILE is set at mm_mesh_create: out [nctas][12] ns accumulated since the last read
 * (Poisson-PCG row phases, reduction before the grid barrier, barrier wait, partial read
 * after the barrier, whole Poisson solves, M_inv applications, energy evaluations with their
 * solves, whole launches, and the two-level preconditioner's box-sum publish, box-sum
 * gather and own-box coarse solve); the counters are reset.  *nctas = 0 when profiling is
 * off. */
mm_status mm_profile_read(mm_mesh* mesh, long long* out, int32_t* nctas);
mm_status mm_timer_stop(mm_mesh* mesh, double* elapsed_ms);

/* ---- learned warm start of the magnetostatic Poisson solve --------------------------------
 *
 * No counterpart in the reference, whose PCG always starts from the previous potential
 * (scripts/solvers.py:221-231, x0 = u).  A per-node network
 *   16 features -> 128 -> 128 -> 128 -> 1, GELU (tanh form), BF16 weights, FP32 accumulation
 * corrects that start: u0 = u_prev + alpha * y(features), with the step alpha = y.r0 / y.S y
 * that minimises the S-norm of the error along the prediction (a one-dimensional Galerkin
 * projection: the start is never worse than u_prev in that norm).  The features of node i over its
 * 1-ring (its row of the Poisson pattern): m_i (3), u_i, ring mean of m (3) and u, ring max of
 * m (3) and u, then the Jacobi-scaled initial residual z = (b - S u_prev)/diag(S) in units of
 * sigma = rms(z): z_i and its ring mean, max and min.  The PCG then runs from u0 to the
 * reference's tolerance, so the solution criterion is unchanged.  Training and inference
 * run on the tensor cores (mma.sync m16n8k16 BF16 -> FP32) in this library's own kernels.
 *
 * A model holds FP32 master parameters (mm_model_num_params floats: W1 [128][16], b1 [128],
 * W2 [128][128], b2, W3 [128][128], b3, w4 [128], b4 [1]; W as [out][in]) with BF16 copies
 * for the products, per-feature normalisation (x - mean) * scale, and the output scale. */
typedef struct mm_model mm_model;

#define MM_MLP_FEATURES 16

mm_status mm_model_create(int32_t device, uint64_t seed, mm_model** out);
mm_status mm_model_destroy(mm_model* model);
int64_t mm_model_num_params(void);
mm_status mm_model_get_params(mm_model* model, float* params);
/* Also resets the Adam moments. */
mm_status mm_model_set_params(mm_model* model, const float* params);
mm_status mm_model_set_normalization(mm_model* model, const float* fmean, const float* fscale, float out_scale);
mm_status mm_model_get_normalization(const mm_model* model, float* fmean, float* fscale, float* out_scale);
/* mean / (1/std) of each feature and the rms of the targets, from n samples. */
mm_status mm_model_fit_normalization(mm_model* model, const float* feats, const float* target, int64_t n);
/* Loss (1/n) sum (y - t/out_scale)^2 and its gradient w.r.t. the FP32 parameters (layout of
 * mm_model_get_params), for n (a multiple of 16) samples feats [n][16], target [n]. */
mm_status mm_model_grad(mm_model* model, const float* feats, const float* target, int32_t n, float* grads,
                        float* loss);
/* Adam (beta 0.9/0.999, eps 1e-8) on shuffled mini-batches of `batch` rows (a multiple of 16);
 * *final_loss = the last epoch's mean batch loss. */
mm_status mm_model_train(mm_model* model, const float* feats, const float* target, int64_t n, int32_t epochs,
                         int32_t batch, float lr, uint64_t seed, float* final_loss);
/* y [n] = out_scale * network(feats [n][16]) (the correction in units of sigma). */
mm_status mm_model_predict(mm_model* model, const float* feats, int64_t n, float* y);

/* Warm start of the mesh's Poisson solves: the reference's previous u (default), zero, or
 * the learned correction of the previous u (model required; it must outlive its use).
 * With the learned start and a launch of at most one CTA per SM the network runs on
 * tcgen05 from its own shared-memory region (the launch shape is re-planned here; run
 * mm_autotune after this call to tune for it); larger launches run it on mma.sync. */
typedef enum { MM_WARM_PREVIOUS = 0, MM_WARM_ZERO = 1, MM_WARM_LEARNED = 2 } mm_warm_mode;
mm_status mm_mesh_set_warm_start(mm_mesh* mesh, int32_t mode, const mm_model* model);

/* Gate of the learned start: it runs only on Poisson solves whose initial residual exceeds
 * `ratio` times the stop tolerance (r.r > ratio^2 tol_u^2 b.b), i.e. solves with at least
 * log10(ratio) decades to go, where a better start can save more iterations than the
 * network costs; other solves start from the previous u.  ratio <= 1 (the default 0): every
 * solve.  No counterpart in the reference. */
mm_status mm_mesh_set_learned_gate(mm_mesh* mesh, double ratio);

/* Training-sample recording: from now on, in every Poisson solve of the mesh (of any entry
 * point), a hash-selected 1/stride of the nodes record their features
 * at the warm start and, after the solve, the target (u - u0)/sigma, into a device buffer of
 * `capacity` samples (later samples are dropped).  capacity 0 stops recording. */
mm_status mm_mesh_record_samples(mm_mesh* mesh, int64_t capacity, int32_t stride, uint64_t seed);
/* Copies out up to `cap` recorded samples: feats [cap][16], target [cap], node [cap] (input
 * node ids; may be NULL); *count = the samples copied. */
mm_status mm_mesh_read_samples(mm_mesh* mesh, float* feats, float* target, int32_t* node, int64_t cap,
                               int64_t* count);

/* ---- failure path test hook ----------------------------------------------------------------
 *
 * Every wait of the persistent kernel is bounded: a grid barrier that has not seen all CTAs
 * arrive after its spin limit (about two seconds) records MM_TIMEOUT, raises the abort flag
 * that releases the other CTAs, and the kernel returns; the call then returns MM_TIMEOUT and
 * the mesh stays usable.  This hook makes that happen on purpose, without a fault: with
 * stall > 0 every barrier of the mesh's later launches waits for `stall` arrivals that never
 * come.  stall = 0 restores normal operation.  With mesh == NULL the setting applies to the
 * barriers of mm_poisson_pcg_noalloc instead (its later calls then return MM_TIMEOUT after
 * about two seconds).  For tests of the failure path only. */
mm_status mm_debug_stall_barriers(mm_mesh* mesh, int32_t stall);

/* ---- allocation-free Poisson solve ------------------------------------------------------
 *
 * No counterpart in the reference: an extra entry point of this library for callers that
 * cannot allocate device memory -- plug-ins whose host application owns every device byte
 * through its own pool, services that allocate everything at start-up and forbid
 * allocation on their serving path.  It solves A x = b (A symmetric positive
 * definite, CSR) by Jacobi-preconditioned CG with the mesh path's iteration (the
 * reference's jax.scipy.sparse.linalg.cg: stop when r.r <= tol^2 b.b or after max_iter
 * iterations), x holding the initial guess on entry and the solution on return.
 *
 * row_ptr [n+1], col [nnz], val [nnz], b [n], x [n] are device pointers the caller owns;
 * iters (may be NULL) is a host pointer.  The call allocates nothing: every intermediate
 * lives in one static device array sized for at most 65,536 rows (about 4.8 MB, held by each
 * GPU that loads the library until exit); n outside [1, 65536] is rejected with
 * MM_BAD_INPUT, as is a CSR structure with out-of-range row pointers or columns or a row
 * whose diagonal is missing, zero or not finite (nothing is iterated then).  Reaching
 * max_iter before the tolerance is not an error: x holds the last iterate, as in the
 * reference's cg.  *iters receives the iterations completed on every return (0 when
 * nothing was iterated).  All calls on a device share that array, which keeps the last
 * call's contents; each call clears what must start at zero.  Calls that overlap on the
 * GPU race on the array: serialise them.  The first call on a device does a one-time
 * set-up there (the array's device address, the kernel's occupancy); make it before any
 * stream capture.  The call runs on `stream` (a cudaStream_t; NULL = the legacy default
 * stream) of the current device and is synchronous: it waits for its own work on that
 * stream and returns when the solve has finished. */
mm_status mm_poisson_pcg_noalloc(int32_t n, int32_t nnz, const int32_t* row_ptr, const int32_t* col,
                                 const double* val, const double* b, double* x, double tol,
                                 int32_t max_iter, int32_t* iters, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MUMAG_B200_H */

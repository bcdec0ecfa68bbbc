"""ctypes binding of ``libmumag_b200.so`` (C ABI declared in ``include/mumag_b200.h``).

The library is the only compute path: there is no CPU fallback.  If the shared object is
missing or no sm_100 device is present, the calls raise.
"""

from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

import os

LIB_PATH = pathlib.Path(os.environ.get("MUMAG_LIB") or pathlib.Path(__file__).resolve().parent / "lib" / "libmumag_b200.so")

MM_OK, MM_BAD_INPUT, MM_CUDA_ERROR, MM_NONFINITE, MM_TIMEOUT, MM_NO_DEVICE = range(6)
STATUS_NAMES = {
    MM_OK: "OK",
    MM_BAD_INPUT: "BAD_INPUT",
    MM_CUDA_ERROR: "CUDA_ERROR",
    MM_NONFINITE: "NONFINITE",
    MM_TIMEOUT: "TIMEOUT",
    MM_NO_DEVICE: "NO_DEVICE",
}
PREC_FP64, PREC_MIXED = 0, 1

# every symbol include/mumag_b200.h declares
EXPORTED = (
    "mm_version",
    "mm_last_error",
    "mm_default_options",
    "mm_default_solver_params",
    "mm_device_count",
    "mm_rcm_permutation",
    "mm_color_elements",
    "mm_mesh_create",
    "mm_mesh_destroy",
    "mm_mesh_get_info",
    "mm_get_meas",
    "mm_get_operator",
    "mm_set_state",
    "mm_get_state",
    "mm_energy_grad",
    "mm_apply_minv",
    "mm_minimize",
    "mm_loop",
    "mm_timer_start",
    "mm_timer_stop",
    "mm_autotune",
    "mm_batch_create",
    "mm_batch_destroy",
    "mm_batch_groups",
    "mm_batch_minimize",
    "mm_batch_loop",
    "mm_batch_timer_start",
    "mm_batch_timer_stop",
    "mm_profile_read",
    "mm_poisson_pcg_noalloc",
    "mm_model_create",
    "mm_model_destroy",
    "mm_model_num_params",
    "mm_model_get_params",
    "mm_model_set_params",
    "mm_model_set_normalization",
    "mm_model_get_normalization",
    "mm_model_fit_normalization",
    "mm_model_grad",
    "mm_model_train",
    "mm_model_predict",
    "mm_mesh_set_warm_start",
    "mm_mesh_record_samples",
    "mm_mesh_read_samples",
    "mm_debug_stall_barriers",
    "mm_mesh_get_coarse",
    "mm_mesh_set_learned_gate",
    "mm_set_state_device",
    "mm_get_state_device",
)
WARM_PREVIOUS, WARM_ZERO, WARM_LEARNED = 0, 1, 2
MLP_FEATURES = 16


class Material(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("theta", "phi", "K1", "K2", "Js", "A")]


class Options(C.Structure):
    _fields_ = [
        ("size", C.c_double),
        ("dirichlet_rhs", C.c_int),
        ("precision", C.c_int),
        ("device", C.c_int),
        ("grid_ctas", C.c_int),
        ("block_threads", C.c_int),
        ("reorder", C.c_int),
        ("pcg_variant", C.c_int),
        ("ctas_per_sm", C.c_int),
        ("stage_operators", C.c_int),
        ("coarse_box_nodes", C.c_int),
    ]


class SolverParams(C.Structure):
    _fields_ = [
        ("hdir", C.c_double * 3),
        ("tol_fun", C.c_double),
        ("tol_u", C.c_double),
        ("precond_iter", C.c_int),
        ("hmag_on", C.c_int),
        ("mbar_mode", C.c_int),
        ("max_pcg_iter", C.c_int),
        ("max_ncg_iter", C.c_int),
    ]


class StepResult(C.Structure):
    _fields_ = [
        ("energy", C.c_double),
        ("mh", C.c_double),
        ("ncg_iters", C.c_int64),
        ("evals", C.c_int64),
        ("pcg_iters", C.c_int64),
        ("ls_shrinks", C.c_int64),
        ("minv_iters", C.c_int64),
        ("kernel_ns", C.c_int64),
        ("sync_ns", C.c_int64),
        ("barriers", C.c_int64),
        ("device_ms", C.c_double),
        ("status", C.c_int),
        ("learned_starts", C.c_int64),
    ]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class MeshInfo(C.Structure):
    _fields_ = [
        ("nodes", C.c_int64),
        ("elements", C.c_int64),
        ("sell_slices", C.c_int64),
        ("sell_entries", C.c_int64),
        ("nnz", C.c_int64),
        ("colours", C.c_int32),
        ("airbox", C.c_int32),
        ("grid_ctas", C.c_int32),
        ("block_threads", C.c_int32),
        ("dirichlet_nodes", C.c_int64),
        ("volume", C.c_double),
        ("bandwidth_before", C.c_double),
        ("bandwidth_after", C.c_double),
        ("pcg_variant", C.c_int32),
        ("kernel_ctas_per_sm", C.c_int32),
        ("staged", C.c_int32),
        ("coarse_boxes", C.c_int32),
    ]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class LoopParams(C.Structure):
    _fields_ = [
        ("hstart", C.c_double),
        ("hfinal", C.c_double),
        ("hstep", C.c_double),
        ("mstep", C.c_double),
        ("mfinal", C.c_double),
        ("max_steps", C.c_int32),
    ]


class Record(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("counter", "hext", "mh", "energy")]


SNAPSHOT_CB = C.CFUNCTYPE(C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64, C.c_void_p)

_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_I64 = C.POINTER(C.c_int64)
_F = C.POINTER(C.c_float)
_lib = None


def load():
    """Load the shared library (once) and declare the signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python mammos-mumag_b200/build.py` "
            "(the CUDA path has no CPU fallback)"
        )
    lib = C.CDLL(str(LIB_PATH))
    sig = {
        "mm_version": (C.c_char_p, []),
        "mm_last_error": (C.c_char_p, []),
        "mm_default_options": (None, [C.POINTER(Options)]),
        "mm_default_solver_params": (None, [C.POINTER(SolverParams)]),
        "mm_device_count": (C.c_int, []),
        "mm_rcm_permutation": (C.c_int, [C.c_int64, _I32, C.c_int64, _I32]),
        "mm_color_elements": (C.c_int, [C.c_int64, _I32, C.c_int64, _I32, _I32]),
        "mm_mesh_create": (
            C.c_int,
            [_D, C.c_int64, _I32, _I32, C.c_int64, C.POINTER(Material), C.c_int32, C.POINTER(Options), C.POINTER(C.c_void_p)],
        ),
        "mm_mesh_destroy": (C.c_int, [C.c_void_p]),
        "mm_mesh_get_info": (C.c_int, [C.c_void_p, C.POINTER(MeshInfo)]),
        "mm_get_meas": (C.c_int, [C.c_void_p, _D, _D]),
        "mm_get_operator": (C.c_int, [C.c_void_p, C.c_int32, _I64, _I32, _I32, _D]),
        "mm_set_state": (C.c_int, [C.c_void_p, _D, _D, _D]),
        "mm_get_state": (C.c_int, [C.c_void_p, _D, _D, _D]),
        "mm_energy_grad": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(SolverParams), _D, _D, _I64]),
        "mm_apply_minv": (C.c_int, [C.c_void_p, C.POINTER(SolverParams), _D, _D, _I64]),
        "mm_minimize": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(SolverParams), C.POINTER(StepResult)]),
        "mm_poisson_pcg_noalloc": (
            C.c_int,
            [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
             C.c_int32, _I32, C.c_void_p],
        ),
        "mm_profile_read": (C.c_int, [C.c_void_p, _I64, _I32]),
        "mm_autotune": (C.c_int, [C.c_void_p, C.POINTER(SolverParams), _I32]),
        "mm_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)]),
        "mm_batch_destroy": (C.c_int, [C.c_void_p]),
        "mm_batch_groups": (C.c_int, [C.c_void_p, _I32]),
        "mm_batch_minimize": (C.c_int, [C.c_void_p, _D, C.POINTER(SolverParams), C.POINTER(StepResult)]),
        "mm_batch_loop": (
            C.c_int,
            [C.c_void_p, C.POINTER(LoopParams), C.POINTER(SolverParams), C.c_int32, C.POINTER(Record), _I32,
             C.POINTER(StepResult)],
        ),
        "mm_batch_timer_start": (C.c_int, [C.c_void_p]),
        "mm_batch_timer_stop": (C.c_int, [C.c_void_p, _D]),
        "mm_timer_start": (C.c_int, [C.c_void_p]),
        "mm_timer_stop": (C.c_int, [C.c_void_p, _D]),
        "mm_loop": (
            C.c_int,
            [C.c_void_p, C.POINTER(LoopParams), C.POINTER(SolverParams), C.POINTER(Record), _I32,
             C.POINTER(StepResult), SNAPSHOT_CB, C.c_void_p],
        ),
        "mm_model_create": (C.c_int, [C.c_int32, C.c_uint64, C.POINTER(C.c_void_p)]),
        "mm_model_destroy": (C.c_int, [C.c_void_p]),
        "mm_model_num_params": (C.c_int64, []),
        "mm_model_get_params": (C.c_int, [C.c_void_p, _F]),
        "mm_model_set_params": (C.c_int, [C.c_void_p, _F]),
        "mm_model_set_normalization": (C.c_int, [C.c_void_p, _F, _F, C.c_float]),
        "mm_model_get_normalization": (C.c_int, [C.c_void_p, _F, _F, _F]),
        "mm_model_fit_normalization": (C.c_int, [C.c_void_p, _F, _F, C.c_int64]),
        "mm_model_grad": (C.c_int, [C.c_void_p, _F, _F, C.c_int32, _F, _F]),
        "mm_model_train": (
            C.c_int, [C.c_void_p, _F, _F, C.c_int64, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _F]),
        "mm_model_predict": (C.c_int, [C.c_void_p, _F, C.c_int64, _F]),
        "mm_mesh_set_warm_start": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
        "mm_mesh_record_samples": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_uint64]),
        "mm_mesh_read_samples": (C.c_int, [C.c_void_p, _F, _F, _I32, C.c_int64, _I64]),
        "mm_debug_stall_barriers": (C.c_int, [C.c_void_p, C.c_int32]),
        "mm_mesh_get_coarse": (C.c_int, [C.c_void_p, _I32, _I32]),
        "mm_mesh_set_learned_gate": (C.c_int, [C.c_void_p, C.c_double]),
        "mm_set_state_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "mm_get_state_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class NativeError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"libmumag_b200 {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status):
    if status != MM_OK:
        raise NativeError(status, load().mm_last_error().decode())


def _dp(a):
    return a.ctypes.data_as(_D) if a is not None else None


def _fp(a):
    return a.ctypes.data_as(_F) if a is not None else None


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape[1:] != shape:
        raise ValueError(f"expected rows of shape {shape}, got {a.shape}")
    return a


def device_count() -> int:
    return load().mm_device_count()


def default_options(**kw) -> Options:
    o = Options()
    load().mm_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def solver_params(hdir=(0.0, 0.0, 1.0), tol_fun=1e-10, tol_u=None, precond_iter=10, hmag_on=1,
                  mbar_mode=0, max_pcg_iter=10000, max_ncg_iter=100000) -> SolverParams:
    sp = SolverParams()
    load().mm_default_solver_params(C.byref(sp))
    for q in range(3):
        sp.hdir[q] = float(hdir[q])
    sp.tol_fun = tol_fun
    sp.tol_u = tol_fun if tol_u is None else tol_u
    sp.precond_iter = precond_iter
    sp.hmag_on = hmag_on
    sp.mbar_mode = mbar_mode
    sp.max_pcg_iter = max_pcg_iter
    sp.max_ncg_iter = max_ncg_iter
    return sp


def poisson_pcg_noalloc(n, nnz, row_ptr, col, val, b, x, tol=1e-10, max_iter=10000, stream=0, raise_error=True):
    """Allocation-free Jacobi-PCG solve (``mm_poisson_pcg_noalloc``) on device pointers
    (integers); ``x`` holds the initial guess and receives the solution.  Returns the
    iteration count, or ``(status, iterations)`` without raising when ``raise_error`` is
    false."""
    it = C.c_int32(-1)
    st = load().mm_poisson_pcg_noalloc(n, nnz, C.c_void_p(row_ptr), C.c_void_p(col), C.c_void_p(val),
                                       C.c_void_p(b), C.c_void_p(x), float(tol), int(max_iter), C.byref(it),
                                       C.c_void_p(stream))
    if not raise_error:
        return st, it.value
    check(st)
    return it.value


def noalloc_stall_barriers(stall: int):
    """Test hook of the failure path of ``poisson_pcg_noalloc``: with stall > 0 every grid
    barrier of its later calls waits for arrivals that never come, gives up after its
    bounded wait and the call returns MM_TIMEOUT.  0 restores normal operation."""
    check(load().mm_debug_stall_barriers(None, int(stall)))


def rcm_permutation(T: np.ndarray, N: int) -> np.ndarray:
    T = np.ascontiguousarray(T, dtype=np.int32)
    perm = np.empty(N, dtype=np.int32)
    check(load().mm_rcm_permutation(N, T.ctypes.data_as(_I32), T.shape[0], perm.ctypes.data_as(_I32)))
    return perm


def color_elements(T: np.ndarray, N: int):
    T = np.ascontiguousarray(T, dtype=np.int32)
    col = np.empty(T.shape[0], dtype=np.int32)
    n = C.c_int32()
    check(load().mm_color_elements(N, T.ctypes.data_as(_I32), T.shape[0], col.ctypes.data_as(_I32), C.byref(n)))
    return col, n.value


class Mesh:
    """Device operators of one mesh (an ``mm_mesh`` handle)."""

    def __init__(self, X, T, tag, materials, size=1e-9, dirichlet_rhs=0, precision=PREC_FP64, device=0,
                 grid_ctas=0, block_threads=0, reorder=1, pcg_variant=0, ctas_per_sm=0, stage_operators=1,
                 coarse_box_nodes=0):
        lib = load()
        self.X = np.ascontiguousarray(X, dtype=np.float64)
        self.T = np.ascontiguousarray(T, dtype=np.int32)
        self.tag = np.ascontiguousarray(tag, dtype=np.int32)
        self.N, self.E = self.X.shape[0], self.T.shape[0]
        rows = [tuple(float(v) for v in r[:6]) for r in materials]
        mats = (Material * max(1, len(rows)))(*[Material(*r) for r in rows])
        opt = default_options(size=size, dirichlet_rhs=dirichlet_rhs, precision=precision, device=device,
                              grid_ctas=grid_ctas, block_threads=block_threads, reorder=reorder,
                              pcg_variant=pcg_variant, ctas_per_sm=ctas_per_sm,
                              stage_operators=stage_operators, coarse_box_nodes=coarse_box_nodes)
        h = C.c_void_p()
        check(lib.mm_mesh_create(_dp(self.X), self.N, self.T.ctypes.data_as(_I32), self.tag.ctypes.data_as(_I32),
                                 self.E, mats, len(rows), C.byref(opt), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            load().mm_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_warm_start(self, mode: int, model: "Model | None" = None):
        """Warm start of the Poisson solves: WARM_PREVIOUS (the reference), WARM_ZERO or
        WARM_LEARNED (``model`` must stay alive while the mesh uses it)."""
        check(load().mm_mesh_set_warm_start(self._h, int(mode), model._h if model is not None else None))
        self._warm_model = model

    def set_learned_gate(self, ratio: float):
        """Run the learned start only on solves whose initial residual exceeds ``ratio`` times
        the stop tolerance (0 or 1: every solve)."""
        check(load().mm_mesh_set_learned_gate(self._h, float(ratio)))

    def record_samples(self, capacity: int, stride: int = 1, seed: int = 0):
        """Record (features, target) pairs of 1/stride of the (node, solve) pairs from now on."""
        check(load().mm_mesh_record_samples(self._h, int(capacity), int(stride), int(seed)))

    def read_samples(self, cap: int | None = None):
        """Recorded samples: ``(feats [k,16] float32, target [k] float32, node [k] int32)``."""
        cap = int(cap if cap is not None else 1 << 22)
        f = np.empty((cap, MLP_FEATURES), np.float32)
        t = np.empty(cap, np.float32)
        n = np.empty(cap, np.int32)
        k = C.c_int64()
        check(load().mm_mesh_read_samples(self._h, _fp(f), _fp(t), n.ctypes.data_as(_I32), cap, C.byref(k)))
        k = k.value
        return f[:k].copy(), t[:k].copy(), n[:k].copy()

    def coarse(self):
        """The two-level preconditioner's aggregates: ``(box [N] int32 in mesh-file order,
        -1 for Dirichlet nodes; number of boxes)``; ``(None, 0)`` with the Jacobi preconditioner."""
        box = np.empty(self.N, np.int32)
        nb = C.c_int32()
        check(load().mm_mesh_get_coarse(self._h, box.ctypes.data_as(_I32), C.byref(nb)))
        return (box, nb.value) if nb.value > 0 else (None, 0)

    def debug_stall_barriers(self, stall: int):
        """Test hook of the failure path: with stall > 0 every grid barrier of later launches
        waits for arrivals that never come, gives up after its bounded wait and the call
        raises NativeError with status MM_TIMEOUT.  0 restores normal operation."""
        check(load().mm_debug_stall_barriers(self._h, int(stall)))

    def autotune(self, sp) -> int:
        """Pick the persistent launch shape by timing candidates; returns the CTA count."""
        g = C.c_int32()
        check(load().mm_autotune(self._h, C.byref(sp), C.byref(g)))
        return g.value

    def timer_start(self):
        check(load().mm_timer_start(self._h))

    def timer_stop(self) -> float:
        """Milliseconds of device time on the mesh's stream since timer_start."""
        ms = C.c_double()
        check(load().mm_timer_stop(self._h, C.byref(ms)))
        return ms.value

    def profile(self):
        """Per-CTA phase timers [nctas, 12] ns (MUMAG_PROFILE set at creation), else None:
        PCG row phases, reduction before the barrier, barrier wait, partial read after it,
        whole Poisson solves, M_inv, energy evaluations (solves included), whole launches,
        the two-level preconditioner's publish, gather and own-box solve."""
        n = C.c_int32()
        check(load().mm_profile_read(self._h, None, C.byref(n)))
        if n.value == 0:
            return None
        out = np.zeros((n.value, 12), np.int64)
        check(load().mm_profile_read(self._h, out.ctypes.data_as(_I64), C.byref(n)))
        return out

    def info(self) -> dict:
        i = MeshInfo()
        check(load().mm_mesh_get_info(self._h, C.byref(i)))
        return i.as_dict()

    def meas(self):
        out = np.empty(self.N)
        v = C.c_double()
        check(load().mm_get_meas(self._h, _dp(out), C.byref(v)))
        return out, v.value

    def operator(self, which: int):
        nnz = C.c_int64()
        lib = load()
        check(lib.mm_get_operator(self._h, which, C.byref(nnz), None, None, None))
        r = np.empty(nnz.value, np.int32)
        c = np.empty(nnz.value, np.int32)
        v = np.empty(nnz.value)
        check(lib.mm_get_operator(self._h, which, C.byref(nnz), r.ctypes.data_as(_I32), c.ctypes.data_as(_I32), _dp(v)))
        return r, c, v

    def set_state(self, m, u=None, mbar=None):
        m = np.ascontiguousarray(m, dtype=np.float64).ravel()
        u = None if u is None else np.ascontiguousarray(u, dtype=np.float64).ravel()
        mbar = None if mbar is None else np.ascontiguousarray(mbar, dtype=np.float64).ravel()
        if m.size != 3 * self.N or (u is not None and u.size != self.N) or (mbar is not None and mbar.size != 3 * self.N):
            raise ValueError("state arrays have the wrong size")
        check(load().mm_set_state(self._h, _dp(m), _dp(u), _dp(mbar)))

    def set_state_device(self, m_ptr: int, u_ptr: int = 0, mbar_ptr: int = 0):
        """``set_state`` from device memory: pointers (integers, 0 = NULL) to float64 arrays on
        the mesh's device in the reference's layout (m, mbar [3N] interleaved, u [N])."""
        check(load().mm_set_state_device(self._h, C.c_void_p(m_ptr or None), C.c_void_p(u_ptr or None),
                                         C.c_void_p(mbar_ptr or None)))

    def get_state_device(self, m_ptr: int = 0, u_ptr: int = 0, g_ptr: int = 0):
        """``get_state`` into device memory (pointers as in ``set_state_device``; 0 = skip)."""
        check(load().mm_get_state_device(self._h, C.c_void_p(m_ptr or None), C.c_void_p(u_ptr or None),
                                         C.c_void_p(g_ptr or None)))

    def get_state(self):
        m = np.empty(3 * self.N)
        u = np.empty(self.N)
        g = np.empty(3 * self.N)
        check(load().mm_get_state(self._h, _dp(m), _dp(u), _dp(g)))
        return m, u, g

    def energy_grad(self, h, sp):
        e = C.c_double()
        g = np.empty(3 * self.N)
        it = C.c_int64()
        check(load().mm_energy_grad(self._h, float(h), C.byref(sp), C.byref(e), _dp(g), C.byref(it)))
        return e.value, g, it.value

    def apply_minv(self, g, sp):
        g = np.ascontiguousarray(g, dtype=np.float64).ravel()
        z = np.empty(3 * self.N)
        it = C.c_int64()
        check(load().mm_apply_minv(self._h, C.byref(sp), _dp(g), _dp(z), C.byref(it)))
        return z, it.value

    def minimize(self, h, sp) -> dict:
        r = StepResult()
        check(load().mm_minimize(self._h, float(h), C.byref(sp), C.byref(r)))
        return r.as_dict()

    def loop(self, hstart, hfinal, hstep, mstep, mfinal, sp, snapshot=None, max_steps=0):
        """Field sweep from the current state. Returns (rows [n,4], per-step dicts)."""
        lp = LoopParams(hstart, hfinal, hstep, mstep, mfinal, max_steps)
        nmax = int(abs(hfinal - hstart) / abs(hstep)) + 1
        if max_steps > 0:
            nmax = min(nmax, max_steps)
        rec = (Record * nmax)()
        steps = (StepResult * nmax)()
        nrec = C.c_int32()
        err = []

        def _cb(counter, mp, up, n, _user):
            try:
                m = np.ctypeslib.as_array(mp, shape=(3 * n,)).copy()
                u = np.ctypeslib.as_array(up, shape=(n,)).copy()
                snapshot(counter, m, u)
                return 0
            except Exception as e:  # surfaced after the call
                err.append(e)
                return 1

        cb = SNAPSHOT_CB(_cb) if snapshot is not None else SNAPSHOT_CB()
        st = load().mm_loop(self._h, C.byref(lp), C.byref(sp), rec, C.byref(nrec), steps, cb, None)
        if err:
            raise err[0]
        check(st)
        n = nrec.value
        rows = np.array([[rec[i].counter, rec[i].hext, rec[i].mh, rec[i].energy] for i in range(n)]).reshape(n, 4)
        return rows, [steps[i].as_dict() for i in range(n)]


class Batch:
    """Several meshes stepped together in one persistent launch (``mm_batch_*``)."""

    def __init__(self, meshes):
        self.meshes = list(meshes)
        arr = (C.c_void_p * len(self.meshes))(*[m._h for m in self.meshes])
        h = C.c_void_p()
        check(load().mm_batch_create(arr, len(self.meshes), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            load().mm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def groups(self):
        g = np.zeros(len(self.meshes) + 1, np.int32)
        check(load().mm_batch_groups(self._h, g.ctypes.data_as(_I32)))
        return g

    def timer_start(self):
        check(load().mm_batch_timer_start(self._h))

    def timer_stop(self) -> float:
        ms = C.c_double()
        check(load().mm_batch_timer_stop(self._h, C.byref(ms)))
        return ms.value

    def minimize(self, h, sps):
        n = len(self.meshes)
        hv = np.ascontiguousarray(np.broadcast_to(np.asarray(h, np.float64), (n,)))
        spa = (SolverParams * n)(*sps) if isinstance(sps, (list, tuple)) else (SolverParams * n)(*([sps] * n))
        res = (StepResult * n)()
        check(load().mm_batch_minimize(self._h, _dp(hv), spa, res))
        return [r.as_dict() for r in res]

    def loop(self, hstart, hfinal, hstep, mstep, mfinal, sps, max_steps=0):
        """Every mesh's whole sweep in one launch; returns per mesh (rows [n,4], per-step dicts)."""
        n = len(self.meshes)
        nmax = int(abs(hfinal - hstart) / abs(hstep)) + 1
        if max_steps > 0:
            nmax = min(nmax, max_steps)
        lp = LoopParams(hstart, hfinal, hstep, mstep, mfinal, max_steps)
        spa = (SolverParams * n)(*sps) if isinstance(sps, (list, tuple)) else (SolverParams * n)(*([sps] * n))
        rec = (Record * (n * nmax))()
        steps = (StepResult * (n * nmax))()
        nrec = np.zeros(n, np.int32)
        check(load().mm_batch_loop(self._h, C.byref(lp), spa, nmax, rec, nrec.ctypes.data_as(_I32), steps))
        out = []
        for q in range(n):
            k = int(nrec[q])
            rows = np.array([[rec[q * nmax + i].counter, rec[q * nmax + i].hext, rec[q * nmax + i].mh,
                              rec[q * nmax + i].energy] for i in range(k)]).reshape(k, 4)
            out.append((rows, [steps[q * nmax + i].as_dict() for i in range(k)]))
        return out


class Model:
    """The warm-start network (an ``mm_model`` handle): 16 -> 128 -> 128 -> 128 -> 1, GELU,
    BF16 weights with FP32 accumulation, trained and evaluated by this library's kernels."""

    def __init__(self, device: int = 0, seed: int = 0):
        h = C.c_void_p()
        check(load().mm_model_create(int(device), int(seed), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            load().mm_model_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def num_params() -> int:
        return int(load().mm_model_num_params())

    def get_params(self) -> np.ndarray:
        p = np.empty(self.num_params(), np.float32)
        check(load().mm_model_get_params(self._h, _fp(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.shape != (self.num_params(),):
            raise ValueError("wrong parameter count")
        check(load().mm_model_set_params(self._h, _fp(p)))

    def set_normalization(self, fmean, fscale, out_scale: float):
        fm, fs = _f32(fmean), _f32(fscale)
        if fm.shape != (MLP_FEATURES,) or fs.shape != (MLP_FEATURES,):
            raise ValueError("normalisation vectors have 16 entries")
        check(load().mm_model_set_normalization(self._h, _fp(fm), _fp(fs), float(out_scale)))

    def get_normalization(self):
        fm = np.empty(MLP_FEATURES, np.float32)
        fs = np.empty(MLP_FEATURES, np.float32)
        o = np.empty(1, np.float32)
        check(load().mm_model_get_normalization(self._h, _fp(fm), _fp(fs), _fp(o)))
        return fm, fs, float(o[0])

    def fit_normalization(self, feats, target):
        f, t = _f32(feats, (MLP_FEATURES,)), _f32(target)
        check(load().mm_model_fit_normalization(self._h, _fp(f), _fp(t), f.shape[0]))

    def grad(self, feats, target):
        """(loss, gradient) of one batch (rows a multiple of 16)."""
        f, t = _f32(feats, (MLP_FEATURES,)), _f32(target)
        g = np.empty(self.num_params(), np.float32)
        loss = np.empty(1, np.float32)
        check(load().mm_model_grad(self._h, _fp(f), _fp(t), f.shape[0], _fp(g), _fp(loss)))
        return float(loss[0]), g

    def train(self, feats, target, epochs=30, batch=256, lr=1e-3, seed=0) -> float:
        f, t = _f32(feats, (MLP_FEATURES,)), _f32(target)
        loss = np.empty(1, np.float32)
        check(load().mm_model_train(self._h, _fp(f), _fp(t), f.shape[0], int(epochs), int(batch), float(lr),
                                    int(seed), _fp(loss)))
        return float(loss[0])

    def predict(self, feats) -> np.ndarray:
        f = _f32(feats, (MLP_FEATURES,))
        y = np.empty(f.shape[0], np.float32)
        check(load().mm_model_predict(self._h, _fp(f), f.shape[0], _fp(y)))
        return y

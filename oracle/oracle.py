"""ctypes loaders of the oracle libraries under oracle/ -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py (CPU-baseline leg and
``--impl reference``); never by the library.

  * ``run_f32`` / ``run_f64``: the CPU restatement of the reference step
    (vof_oracle.cpp), FP32 without FMA contraction, or FP64.
  * ``run_conv_f64``: FP64 steps with the pressure solved to a tolerance (CG).
  * ``adjoint`` / ``SwitchTape``: the host adjoint of the step (vof_adjoint.cpp)
    and the switch-frozen forward that checks it by finite differences.
  * ``ref_run`` / ``ref_time``: the reference's own kernels (voftrial1.cu
    compiled with ref_harness.cu into oracle/_ref/); GPU only.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
ORACLE_LIB = ORACLE_DIR / "_build" / "liboracle.so"
REF_LIBS = {
    "sm100a": ORACLE_DIR / "_ref" / "libvofref_sm100a.so",   # nvcc -O3 sm_100a (default -fmad=true)
    "nofma": ORACLE_DIR / "_ref" / "libvofref_nofma.so",     # same, -fmad=false
    "readme": ORACLE_DIR / "_ref" / "libvofref_readme.so",   # README flags, PTX JIT
}
# The reference checkout (the directory holding voftrial1.cu), for building
# the harness only: given by VOF_REFERENCE_DIR or by the caller of build().
REFERENCE_SRC = Path(os.environ["VOF_REFERENCE_DIR"]) if os.environ.get("VOF_REFERENCE_DIR") else None

STATE = ("F", "u", "v", "w", "p")

_oracle = None
_refs = {}


def build(ref: bool | None = None, ref_dir=None) -> None:
    """make the oracle (always) and the reference harness from the reference
    checkout `ref_dir` (or VOF_REFERENCE_DIR) when it holds voftrial1.cu."""
    targets = ["oracle"]
    src = Path(ref_dir) if ref_dir else REFERENCE_SRC
    if ref is None:
        ref = src is not None and (src / "voftrial1.cu").exists()
    if ref:
        if src is None or not (src / "voftrial1.cu").exists():
            raise FileNotFoundError("reference harness: set VOF_REFERENCE_DIR (or pass ref_dir) to the directory "
                                    "holding voftrial1.cu")
        targets.append("ref")
    extra = [f"REF_DIR={src}"] if ref else []
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), *extra, *targets], check=True)


def _params_type():
    sys.path.insert(0, str(ORACLE_DIR.parent / "cuda-lbm-ibm-fvm_b200"))
    from vof_b200 import Params  # the ctypes mirror of vof_params
    return Params


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not ORACLE_LIB.exists():
            build(ref=False)
        Params = _params_type()
        lib = C.CDLL(str(ORACLE_LIB))
        for name, T in (("oracle_run_f32", C.c_float), ("oracle_run_f64", C.c_double)):
            fn = getattr(lib, name)
            fn.restype = C.c_int
            fn.argtypes = [C.POINTER(Params)] + [C.POINTER(T)] * 5 + [C.c_int, C.c_int] + \
                [C.POINTER(T)] * 4 + [C.c_int]
        lib.oracle_run_conv_f64.restype = C.c_int
        lib.oracle_run_conv_f64.argtypes = [C.POINTER(Params)] + [C.POINTER(C.c_double)] * 5 + \
            [C.c_int, C.c_int, C.c_double, C.c_int]
        D = C.POINTER(C.c_double)
        for name, T in (("oracle_adjoint_f32", C.c_float), ("oracle_adjoint_f64", C.c_double)):
            fn = getattr(lib, name)
            fn.restype = C.c_int
            fn.argtypes = [C.POINTER(Params)] + [C.POINTER(T)] * 5 + [C.c_int, C.c_int, D] + [D] * 7 + [C.c_int]
        for name, T in (("oracle_adjoint_conv_f32", C.c_float), ("oracle_adjoint_conv_f64", C.c_double)):
            fn = getattr(lib, name)
            fn.restype = C.c_int
            fn.argtypes = [C.POINTER(Params)] + [C.POINTER(T)] * 5 + [C.c_int, C.c_int, D] + [D] * 7 + \
                [C.c_double, C.c_int]
        lib.oracle_tangent_f64.restype = C.c_int
        lib.oracle_tangent_f64.argtypes = [C.POINTER(Params)] + [D] * 11 + [C.c_int, C.c_int, D, D, D, C.c_int]
        lib.oracle_tape_new.restype = C.c_void_p
        lib.oracle_tape_new.argtypes = []
        lib.oracle_tape_free.restype = None
        lib.oracle_tape_free.argtypes = [C.c_void_p]
        lib.oracle_tape_size.restype = C.c_longlong
        lib.oracle_tape_size.argtypes = [C.c_void_p]
        for name, T in (("oracle_tape_run_f32", C.c_float), ("oracle_tape_run_f64", C.c_double)):
            fn = getattr(lib, name)
            fn.restype = C.c_int
            fn.argtypes = [C.c_void_p, C.c_int, C.POINTER(Params)] + [C.POINTER(T)] * 5 + [C.c_int, C.c_int, D, D]
        lib.oracle_apply_bc_f32.restype = C.c_int
        lib.oracle_apply_bc_f32.argtypes = [C.POINTER(Params)] + [C.POINTER(C.c_float)] * 6
        lib.oracle_clamp01f.restype = C.c_float
        lib.oracle_clamp01f.argtypes = [C.c_float]
        lib.oracle_clamp01d.restype = C.c_double
        lib.oracle_clamp01d.argtypes = [C.c_double]
        lib.oracle_max_threads.restype = C.c_int
        _oracle = lib
    return _oracle


def _ptr(a, T):
    return a.ctypes.data_as(C.POINTER(T)) if a is not None else None


def _run(fn, T, dtype, prm, state, istep0, nsteps, nthreads, extras):
    st = {k: np.ascontiguousarray(state[k], dtype=dtype).copy() for k in STATE}
    ex = {k: np.zeros(prm.shape, dtype=dtype) for k in ("ustar", "vstar", "wstar", "rhs")} if extras else {}
    rc = fn(C.byref(prm), *(_ptr(st[k], T) for k in STATE), istep0, nsteps,
            *(_ptr(ex.get(k), T) for k in ("ustar", "vstar", "wstar", "rhs")), int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle run failed: {rc}")
    st.update(ex)
    return st


def run_f32(prm, state, istep0: int, nsteps: int, nthreads: int = 0, extras: bool = False) -> dict:
    """nsteps reference steps in FP32 (IEEE, no FMA) on a copy of `state`."""
    return _run(oracle_lib().oracle_run_f32, C.c_float, np.float32, prm, state, istep0, nsteps, nthreads, extras)


def run_f64(prm, state, istep0: int, nsteps: int, nthreads: int = 0, extras: bool = False) -> dict:
    """nsteps reference steps in FP64 on a copy of `state` (promoted to float64)."""
    return _run(oracle_lib().oracle_run_f64, C.c_double, np.float64, prm, state, istep0, nsteps, nthreads, extras)


def run_conv_f64(prm, state, istep0: int, nsteps: int, tol: float = 1e-12, nthreads: int = 0) -> dict:
    """FP64 steps with the pressure solved to ||r|| <= tol ||b|| (CG), mean(p) = 0."""
    st = {k: np.ascontiguousarray(state[k], dtype=np.float64).copy() for k in STATE}
    rc = oracle_lib().oracle_run_conv_f64(C.byref(prm), *(_ptr(st[k], C.c_double) for k in STATE), istep0,
                                          nsteps, float(tol), int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle conv run failed: {rc}")
    return st


def _box(box):
    b = np.asarray(box if box is not None else (-1e300, 1e300) * 3, dtype=np.float64)
    assert b.shape == (6,)
    return b


def adjoint(prm, state, istep0: int, nsteps: int, box, precision: str = "f32", nthreads: int = 0,
            conv_tol: float = 0.0) -> dict:
    """Host adjoint of L = sum over `box` (x0, x1, y0, y1, z0, z1; strict bounds
    on cell centres) of F dV after nsteps steps: dL/d(F, u, v, w, p) of the
    initial state (float64, reference layout) as "lF", "lu", ..., dL/dg as
    "grad_g" and the loss as "loss".  The forward runs in FP32 ("f32", the
    CUDA plain path's arithmetic) or FP64 ("f64"); conv_tol > 0 solves every
    step's pressure to that tolerance instead of the Jacobi sweeps."""
    T, dt = (C.c_float, np.float32) if precision == "f32" else (C.c_double, np.float64)
    if conv_tol > 0:
        base = oracle_lib().oracle_adjoint_conv_f32 if precision == "f32" else oracle_lib().oracle_adjoint_conv_f64
        fn = lambda *a: base(*a[:-1], float(conv_tol), a[-1])  # noqa: E731
    else:
        fn = oracle_lib().oracle_adjoint_f32 if precision == "f32" else oracle_lib().oracle_adjoint_f64
    st = {k: np.ascontiguousarray(state[k], dtype=dt) for k in STATE}
    out = {k: np.zeros(prm.shape, dtype=np.float64) for k in ("lF", "lu", "lv", "lw", "lp")}
    g = np.zeros(3)
    loss = np.zeros(1)
    b = _box(box)
    D = C.POINTER(C.c_double)
    rc = fn(C.byref(prm), *(_ptr(st[k], T) for k in STATE), istep0, nsteps, _ptr(b, C.c_double),
            *(_ptr(out[k], C.c_double) for k in ("lF", "lu", "lv", "lw", "lp")), _ptr(g, C.c_double),
            _ptr(loss, C.c_double), int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle adjoint failed: {rc}")
    out["grad_g"] = g
    out["loss"] = float(loss[0])
    return out


def tangent(prm, state, direction: dict, istep0: int, nsteps: int, box, dg=None, nthreads: int = 0):
    """(loss, dloss): the FP64 box loss and its derivative along `direction`
    (arrays for any of F, u, v, w, p) and dg (body force), by the dual-number
    tangent of the FP64 step with the adjoint's switch convention."""
    st = {k: np.ascontiguousarray(state[k], dtype=np.float64) for k in STATE}
    dd = {k: (np.ascontiguousarray(direction[k], dtype=np.float64) if k in direction else None) for k in STATE}
    g = None if dg is None else np.ascontiguousarray(dg, dtype=np.float64)
    loss, dloss = np.zeros(1), np.zeros(1)
    b = _box(box)
    rc = oracle_lib().oracle_tangent_f64(C.byref(prm), *(_ptr(st[k], C.c_double) for k in STATE),
                                         *(_ptr(dd[k], C.c_double) for k in STATE), _ptr(g, C.c_double), istep0,
                                         nsteps, _ptr(b, C.c_double), _ptr(loss, C.c_double),
                                         _ptr(dloss, C.c_double), int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle tangent failed: {rc}")
    return float(loss[0]), float(dloss[0])


class SwitchTape:
    """The switches of one forward run: record() runs the base point and keeps
    every non-smooth choice; replay() runs another state with those choices
    frozen (the base point's piecewise-smooth map).  Both return the final
    state and the box loss."""

    def __init__(self, prm, istep0: int, nsteps: int, box, precision: str = "f64"):
        self.prm, self.istep0, self.nsteps, self.box = prm, istep0, nsteps, _box(box)
        self.T, self.dt = (C.c_float, np.float32) if precision == "f32" else (C.c_double, np.float64)
        self.fn = oracle_lib().oracle_tape_run_f32 if precision == "f32" else oracle_lib().oracle_tape_run_f64
        self.h = oracle_lib().oracle_tape_new()

    def _run(self, state, replay):
        st = {k: np.ascontiguousarray(state[k], dtype=self.dt).copy() for k in STATE}
        loss = np.zeros(1)
        rc = self.fn(self.h, int(replay), C.byref(self.prm), *(_ptr(st[k], self.T) for k in STATE), self.istep0,
                     self.nsteps, _ptr(self.box, C.c_double), _ptr(loss, C.c_double))
        if rc != 0:
            raise RuntimeError(f"tape run failed: {rc} (replay={replay})")
        return st, float(loss[0])

    def record(self, state):
        return self._run(state, False)

    def replay(self, state):
        return self._run(state, True)

    def size(self) -> int:
        return int(oracle_lib().oracle_tape_size(self.h))

    def close(self):
        if self.h:
            oracle_lib().oracle_tape_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


BC_FIELDS = ("u", "v", "w", "F", "p", "rho")  # apply_bc's argument order (voftrial1.cu:943)


def apply_bc(prm, fields: dict) -> dict:
    """The reference's apply_bc (voftrial1.cu:943-956) on copies of the six
    fields (reference layout): set_bc_j, then set_bc_i, then set_bc_k."""
    st = {k: np.ascontiguousarray(fields[k], dtype=np.float32).copy() for k in BC_FIELDS}
    rc = oracle_lib().oracle_apply_bc_f32(C.byref(prm), *(_ptr(st[k], C.c_float) for k in BC_FIELDS))
    if rc != 0:
        raise RuntimeError(f"oracle apply_bc failed: {rc}")
    return st


def clamp01f(x: float) -> float:
    return oracle_lib().oracle_clamp01f(x)


def max_threads() -> int:
    return oracle_lib().oracle_max_threads()


# ---- the reference's own kernels (GPU) ------------------------------------
def ref_available(variant: str = "sm100a") -> bool:
    return REF_LIBS[variant].exists()


def ref_lib(variant: str = "sm100a"):
    if variant not in _refs:
        path = REF_LIBS[variant]
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (needs the reference source; see oracle/Makefile)")
        Params = _params_type()
        lib = C.CDLL(str(path))
        F = C.POINTER(C.c_float)
        lib.ref_run.restype = C.c_int
        lib.ref_run.argtypes = [C.POINTER(Params)] + [F] * 5 + [C.c_int, C.c_int] + [F] * 3
        lib.ref_time.restype = C.c_int
        lib.ref_time.argtypes = [C.POINTER(Params)] + [F] * 5 + [C.c_int, C.c_int, C.c_int,
                                                                 C.POINTER(C.c_double), F]
        lib.ref_kernels_per_step.restype = C.c_int
        lib.ref_kernels_per_step.argtypes = [C.c_int]
        lib.ref_initial_F.restype = C.c_int
        lib.ref_initial_F.argtypes = [C.POINTER(Params), C.c_int, F]
        lib.ref_write_vtk.restype = C.c_int
        lib.ref_write_vtk.argtypes = [C.c_char_p, F, C.c_int, C.c_int, C.c_int]
        lib.ref_apply_bc.restype = C.c_int
        lib.ref_apply_bc.argtypes = [C.POINTER(Params)] + [F] * 6
        _refs[variant] = lib
    return _refs[variant]


def ref_initial_F(prm, ic: int = 1, variant: str = "sm100a") -> np.ndarray:
    """set_init_F_kernel + apply_bc_F of the reference (GPU), reference layout."""
    F = np.zeros(prm.shape, dtype=np.float32)
    rc = ref_lib(variant).ref_initial_F(C.byref(prm), int(ic), _ptr(F, C.c_float))
    if rc != 0:
        raise RuntimeError(f"ref_initial_F failed: {rc}")
    return F


def ref_write_vtk(path, F: np.ndarray, variant: str = "sm100a") -> None:
    """The reference's write_legacy_vtk on a host field (host code; no GPU)."""
    F = np.ascontiguousarray(F, dtype=np.float32)
    nz, ny, nx = F.shape
    rc = ref_lib(variant).ref_write_vtk(str(path).encode(), _ptr(F, C.c_float), nx, ny, nz)
    if rc != 0:
        raise RuntimeError(f"ref_write_vtk failed: {rc}")


def ref_apply_bc(prm, fields: dict, variant: str = "sm100a") -> dict:
    """The reference's own apply_bc kernels (GPU) on copies of the six fields."""
    st = {k: np.ascontiguousarray(fields[k], dtype=np.float32).copy() for k in BC_FIELDS}
    rc = ref_lib(variant).ref_apply_bc(C.byref(prm), *(_ptr(st[k], C.c_float) for k in BC_FIELDS))
    if rc != 0:
        raise RuntimeError(f"ref_apply_bc failed: {rc}")
    return st


def ref_run(prm, state, istep0: int, nsteps: int, variant: str = "sm100a", extras: bool = False) -> dict:
    lib = ref_lib(variant)
    st = {k: np.ascontiguousarray(state[k], dtype=np.float32).copy() for k in STATE}
    ex = {k: np.zeros(prm.shape, dtype=np.float32) for k in ("ustar", "vstar", "wstar")} if extras else {}
    rc = lib.ref_run(C.byref(prm), *(_ptr(st[k], C.c_float) for k in STATE), istep0, nsteps,
                     *(_ptr(ex.get(k), C.c_float) for k in ("ustar", "vstar", "wstar")))
    if rc != 0:
        raise RuntimeError(f"ref_run failed: {rc}")
    st.update(ex)
    return st


def ref_time(prm, state, istep0: int, warmup: int, nsteps: int, variant: str = "sm100a",
             want_F: bool = False):
    """Milliseconds of nsteps reference steps (CUDA events), and F if asked."""
    lib = ref_lib(variant)
    st = {k: np.ascontiguousarray(state[k], dtype=np.float32) for k in STATE}
    ms = C.c_double()
    Fo = np.zeros(prm.shape, dtype=np.float32) if want_F else None
    rc = lib.ref_time(C.byref(prm), *(_ptr(st[k], C.c_float) for k in STATE), istep0, warmup, nsteps,
                      C.byref(ms), _ptr(Fo, C.c_float))
    if rc != 0:
        raise RuntimeError(f"ref_time failed: {rc}")
    return ms.value, Fo

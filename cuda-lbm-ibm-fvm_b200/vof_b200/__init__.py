"""Python binding of libvof_b200.so, the C-ABI of include/vof.h.

The binding is a thin ctypes layer: every call goes to the CUDA library, and
importing this module on a machine where the library is missing raises
immediately (there is no CPU fallback).  Fields cross the boundary in the
reference's layout, a C-contiguous float32 array of shape (nz+2, ny+2, nx+2)
(index [k, j, i], i fastest, voftrial1.cu:66-70).

Typical use, the drop-in for the time loop of voftrial1.cu:1361-1401::

    prm = vof_b200.default_params(200, 200, 200, gz=-9.81, gy=0.0)
    with vof_b200.Solver(prm) as s:
        s.upload_state(F=F0, u=u0, v=v0, w=w0, p=p0)
        s.run(istep0=1, nsteps=2000)       # steps 1..2000
        F = s.download("F")
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("VOF_B200_LIB", str(_PKG / "libvof_b200.so")))

# ---- constants mirrored from include/vof.h -------------------------------
OK = 0
E_INVALID, E_SIZE, E_NOMEM, E_CUDA, E_NOT_CONVERGED, E_NONFINITE, E_STATE, E_UNSUPPORTED, E_TIMEOUT = (
    -1, -2, -3, -4, -5, -6, -7, -8, -9)
MODE_PLAIN, MODE_MIXED, MODE_FP64 = 0, 1, 2
ADJ_AUTO, ADJ_RECOMPUTE, ADJ_KEEP = 0, 1, 2
FIELDS = {"F": 0, "u": 1, "v": 2, "w": 3, "p": 4, "ustar": 5, "vstar": 6, "wstar": 7, "rhs": 8}
REDUCTIONS = {"volume": 0, "div_l2": 1, "div_max": 2, "pres_resid": 3, "nonfinite": 4,
              "f_min": 5, "f_max": 6}
STATE_FIELDS = ("F", "u", "v", "w", "p")


class Params(C.Structure):
    """Mirror of vof_params (include/vof.h) == Params of voftrial1.cu:27-41 + additions."""
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("imin", C.c_int), ("imax", C.c_int), ("jmin", C.c_int), ("jmax", C.c_int),
        ("kmin", C.c_int), ("kmax", C.c_int),
        ("Lx", C.c_float), ("Ly", C.c_float), ("Lz", C.c_float),
        ("rho_l", C.c_float), ("rho_g", C.c_float),
        ("nu_l", C.c_float), ("nu_g", C.c_float),
        ("sigma", C.c_float),
        ("gx", C.c_float), ("gy", C.c_float), ("gz", C.c_float),
        ("dt", C.c_float),
        ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
        ("dxi", C.c_float), ("dyi", C.c_float), ("dzi", C.c_float),
        ("nTot", C.c_int),
        ("jacobi_iters", C.c_int), ("mode", C.c_int), ("inner_sweeps", C.c_int),
        ("max_outer", C.c_int), ("tol", C.c_double),
        ("surface_tension", C.c_int),
    ]

    @property
    def shape(self):
        return (self.nz + 2, self.ny + 2, self.nx + 2)

    def copy(self) -> "Params":
        q = Params()
        C.pointer(q)[0] = self
        return q

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class VofError(RuntimeError):
    def __init__(self, status: int, what: str, cuda_error: int = 0):
        self.status = status
        self.cuda_error = cuda_error
        msg = f"{what}: status {status}"
        try:
            msg += f" ({lib().vof_error_string(status).decode()})"
        except Exception:  # pragma: no cover - library unavailable
            pass
        if cuda_error:
            msg += f", cudaError {cuda_error}"
        super().__init__(msg)


_lib = None


def _declare(lib):
    P = C.POINTER
    vp = C.c_void_p
    sig = {
        "vof_abi_version": (C.c_int, []),
        "vof_error_string": (C.c_char_p, [C.c_int]),
        "vof_params_init": (C.c_int, [P(Params), C.c_int, C.c_int, C.c_int]),
        "vof_params_finalize": (C.c_int, [P(Params)]),
        "vof_create": (C.c_int, [P(Params), vp, P(vp)]),
        "vof_destroy": (None, [vp]),
        "vof_get_params": (C.c_int, [vp, P(Params)]),
        "vof_upload": (C.c_int, [vp, C.c_int, vp, C.c_int]),
        "vof_download": (C.c_int, [vp, C.c_int, vp, C.c_int]),
        "vof_step": (C.c_int, [vp, C.c_int]),
        "vof_run": (C.c_int, [vp, C.c_int, C.c_int]),
        "vof_sync": (C.c_int, [vp]),
        "vof_reduce": (C.c_int, [vp, C.c_int, P(C.c_double)]),
        "vof_reduce_async": (C.c_int, [vp, C.c_int, vp]),
        "vof_last_cuda_error": (C.c_int, [vp]),
        "vof_kernels_per_step": (C.c_int, [vp]),
        "vof_device_bytes": (C.c_size_t, [vp]),
        "vof_step_timed": (C.c_int, [vp, C.c_int, P(C.c_float), P(C.c_int), C.c_int]),
        "vof_phase_name": (C.c_char_p, [C.c_int]),
        "vof_solver_stats": (C.c_int, [vp, P(C.c_int), P(C.c_double), P(C.c_double)]),
        "vof_step_noalloc": (C.c_int, [P(Params), vp, vp, vp, vp, vp, C.c_int, vp]),
        "vof_forward_record": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
        "vof_backward": (C.c_int, [vp, P(C.c_double), P(C.c_double), P(C.c_double)]),
        "vof_adjoint_download": (C.c_int, [vp, C.c_int, vp]),
        "vof_adjoint_kernels_per_step": (C.c_int, [vp]),
        "vof_adjoint_storage": (C.c_int, [vp, C.c_int]),
        "vof_adjoint_keeps": (C.c_int, [vp]),
        "vof_debug_fail_alloc": (C.c_int, [C.c_int]),
        "vof_debug_wait_timeout": (C.c_int, [vp, C.c_uint]),
        "vof_get_planes": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, C.c_int]),
        "vof_put_planes": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, C.c_int]),
        "vof_reduce_range": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, P(C.c_double)]),
        "vof_reduce_range_async": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp]),
        "vof_apply_bc": (C.c_int, [vp]),
        "vof_apply_bc_fields": (C.c_int, [P(Params), vp, vp, vp, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def lib():
    """Load libvof_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} not found: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
                " (the CUDA library is required; there is no CPU fallback)")
        _lib = _declare(C.CDLL(str(LIB_PATH)))
    return _lib


def exported_symbols():
    """Names declared in include/vof.h that the loaded library must export."""
    return ["vof_abi_version", "vof_error_string", "vof_params_init", "vof_params_finalize",
            "vof_create", "vof_destroy", "vof_get_params", "vof_upload", "vof_download",
            "vof_step", "vof_run", "vof_sync", "vof_reduce", "vof_reduce_async",
            "vof_last_cuda_error", "vof_kernels_per_step", "vof_device_bytes",
            "vof_step_timed", "vof_phase_name", "vof_solver_stats", "vof_step_noalloc",
            "vof_forward_record", "vof_backward", "vof_adjoint_download", "vof_adjoint_kernels_per_step",
            "vof_adjoint_storage", "vof_adjoint_keeps", "vof_debug_fail_alloc", "vof_debug_wait_timeout",
            "vof_get_planes", "vof_put_planes", "vof_reduce_range", "vof_reduce_range_async",
            "vof_apply_bc", "vof_apply_bc_fields"]


BC_FIELDS = ("u", "v", "w", "F", "p", "rho")  # apply_bc's argument order (voftrial1.cu:943)


def apply_bc_fields(prm, stream: int = 0, **device_ptrs):
    """The reference's apply_bc on caller-owned device buffers in the reference
    layout, given as device pointers by name (u, v, w, F, p, rho; a name left
    out is skipped), enqueued on `stream` (0: the legacy default stream)."""
    unknown = set(device_ptrs) - set(BC_FIELDS)
    if unknown:
        raise ValueError(f"unknown fields {sorted(unknown)}")
    ptrs = [C.c_void_p(device_ptrs[k]) if device_ptrs.get(k) else None for k in BC_FIELDS]
    st = lib().vof_apply_bc_fields(C.byref(prm), *ptrs, C.c_void_p(stream) if stream else None)
    if st != OK:
        raise VofError(st, "vof_apply_bc_fields")


def default_params(nx: int, ny: int | None = None, nz: int | None = None, **overrides) -> Params:
    """vof_params_init (the reference's constants), then `overrides`, then finalize."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = Params()
    st = lib().vof_params_init(C.byref(p), nx, ny, nz)
    if st != OK:
        raise VofError(st, "vof_params_init")
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    st = lib().vof_params_finalize(C.byref(p))
    if st != OK:
        raise VofError(st, "vof_params_finalize")
    return p


def zeros(prm: Params, dtype=np.float32) -> np.ndarray:
    return np.zeros(prm.shape, dtype=dtype)


class Solver:
    """One vof_ctx.  `stream` is a cudaStream_t as an int (0 = legacy default)."""

    def __init__(self, prm: Params, stream: int = 0):
        self._lib = lib()
        self.prm = prm.copy()
        self._ctx = C.c_void_p()
        st = self._lib.vof_create(C.byref(self.prm), C.c_void_p(stream or None), C.byref(self._ctx))
        if st != OK:
            raise VofError(st, "vof_create")

    # -- lifecycle -----------------------------------------------------------
    def close(self):
        if self._ctx:
            self._lib.vof_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str):
        if st != OK:
            raise VofError(st, what, self._lib.vof_last_cuda_error(self._ctx))

    # -- data ----------------------------------------------------------------
    def _fid(self, field) -> int:
        return FIELDS[field] if isinstance(field, str) else int(field)

    def upload(self, field, arr=None, device_ptr: int | None = None):
        """Host array (reference layout) or a raw device pointer."""
        fid = self._fid(field)
        if device_ptr is not None:
            self._check(self._lib.vof_upload(self._ctx, fid, C.c_void_p(device_ptr), 1), "vof_upload")
            return
        a = np.ascontiguousarray(arr, dtype=np.float32)
        if a.size != self.prm.nTot:
            raise ValueError(f"field {field}: {a.size} values, expected {self.prm.nTot}")
        self._check(self._lib.vof_upload(self._ctx, fid, a.ctypes.data_as(C.c_void_p), 0), "vof_upload")
        self._check(self._lib.vof_sync(self._ctx), "vof_sync")  # `a` may be a temporary

    def upload_state(self, **fields):
        for name, arr in fields.items():
            self.upload(name, arr)

    def download(self, field, out: np.ndarray | None = None) -> np.ndarray:
        fid = self._fid(field)
        if out is None:
            out = np.empty(self.prm.shape, dtype=np.float32)
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.size == self.prm.nTot
        self._check(self._lib.vof_download(self._ctx, fid, out.ctypes.data_as(C.c_void_p), 0),
                    "vof_download")
        return out

    def download_device(self, field, device_ptr: int):
        self._check(self._lib.vof_download(self._ctx, self._fid(field), C.c_void_p(device_ptr), 1),
                    "vof_download")

    def state(self) -> dict:
        return {f: self.download(f) for f in STATE_FIELDS}

    def get_planes(self, field, k0: int, nk: int, out=None, device_ptr: int | None = None):
        """Planes k0 .. k0+nk-1 of a field (reference layout): into `out` (a
        host float32 array of nk (ny+2)(nx+2) values, allocated when None) or
        to a device pointer (stream-ordered)."""
        fid = self._fid(field)
        if device_ptr is not None:
            self._check(self._lib.vof_get_planes(self._ctx, fid, k0, nk, C.c_void_p(device_ptr), 1), "vof_get_planes")
            return None
        if out is None:
            out = np.empty((nk, self.prm.ny + 2, self.prm.nx + 2), dtype=np.float32)
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.size == nk * (self.prm.ny + 2) * (self.prm.nx + 2)
        self._check(self._lib.vof_get_planes(self._ctx, fid, k0, nk, out.ctypes.data_as(C.c_void_p), 0),
                    "vof_get_planes")
        return out

    def put_planes(self, field, k0: int, arr=None, device_ptr: int | None = None, nk: int | None = None):
        """Write planes k0 .. from a host array (nk, ny+2, nx+2) or a device pointer (nk given)."""
        fid = self._fid(field)
        if device_ptr is not None:
            self._check(self._lib.vof_put_planes(self._ctx, fid, k0, int(nk), C.c_void_p(device_ptr), 1),
                        "vof_put_planes")
            return
        a = np.ascontiguousarray(arr, dtype=np.float32)
        nk = a.size // ((self.prm.ny + 2) * (self.prm.nx + 2))
        self._check(self._lib.vof_put_planes(self._ctx, fid, k0, nk, a.ctypes.data_as(C.c_void_p), 0),
                    "vof_put_planes")
        self._check(self._lib.vof_sync(self._ctx), "vof_sync")  # `a` may be a temporary

    def reduce_range(self, what, k0: int, k1: int) -> float:
        out = C.c_double()
        w = REDUCTIONS[what] if isinstance(what, str) else int(what)
        self._check(self._lib.vof_reduce_range(self._ctx, w, k0, k1, C.byref(out)), "vof_reduce_range")
        return out.value

    def reduce_range_async(self, what, k0: int, k1: int, host_ptr: int):
        """reduce_range written to host_ptr (pinned) in stream order; sync before reading."""
        w = REDUCTIONS[what] if isinstance(what, str) else int(what)
        self._check(self._lib.vof_reduce_range_async(self._ctx, w, k0, k1, C.c_void_p(host_ptr)),
                    "vof_reduce_range_async")

    # -- stepping ------------------------------------------------------------
    def step(self, istep: int):
        self._check(self._lib.vof_step(self._ctx, istep), "vof_step")

    def run(self, istep0: int, nsteps: int):
        self._check(self._lib.vof_run(self._ctx, istep0, nsteps), "vof_run")

    def sync(self):
        self._check(self._lib.vof_sync(self._ctx), "vof_sync")

    def apply_bc(self):
        """The reference's apply_bc on the current state (stream-ordered)."""
        self._check(self._lib.vof_apply_bc(self._ctx), "vof_apply_bc")

    def reduce(self, what) -> float:
        out = C.c_double()
        w = REDUCTIONS[what] if isinstance(what, str) else int(what)
        self._check(self._lib.vof_reduce(self._ctx, w, C.byref(out)), "vof_reduce")
        return out.value

    def reduce_async(self, what, host_ptr: int):
        w = REDUCTIONS[what] if isinstance(what, str) else int(what)
        self._check(self._lib.vof_reduce_async(self._ctx, w, C.c_void_p(host_ptr)), "vof_reduce_async")

    def step_timed(self, istep: int) -> dict:
        """One step with CUDA events around each phase: {phase: (ms, launches)}."""
        n = 7
        ms = (C.c_float * n)()
        la = (C.c_int * n)()
        st = self._lib.vof_step_timed(self._ctx, istep, ms, la, n)
        if st < 0:
            self._check(st, "vof_step_timed")
        return {self._lib.vof_phase_name(q).decode(): (ms[q], la[q]) for q in range(st)}

    def solver_stats(self) -> dict:
        """Convergent modes: {'outer', 'rel_initial', 'rel_final'} of the last solve."""
        o, a, b = C.c_int(), C.c_double(), C.c_double()
        self._check(self._lib.vof_solver_stats(self._ctx, C.byref(o), C.byref(a), C.byref(b)), "vof_solver_stats")
        return {"outer": o.value, "rel_initial": a.value, "rel_final": b.value}

    # ---- adjoint ----------------------------------------------------------
    def forward_record(self, istep0: int, nsteps: int, checkpoint_every: int = 0):
        """nsteps plain steps from istep0, with checkpoints for backward()."""
        self._check(self._lib.vof_forward_record(self._ctx, istep0, nsteps, checkpoint_every), "vof_forward_record")

    def backward(self, box) -> dict:
        """Reverse pass of the recorded run for L = sum over `box` (x0, x1, y0,
        y1, z0, z1; strict bounds on cell centres) of F dV: {'loss', 'grad_g'}."""
        b = np.ascontiguousarray(box, dtype=np.float64)
        if b.shape != (6,):
            raise ValueError("box must be (x0, x1, y0, y1, z0, z1)")
        loss = C.c_double()
        g = np.zeros(3)
        self._check(self._lib.vof_backward(self._ctx, b.ctypes.data_as(C.POINTER(C.c_double)), C.byref(loss),
                                           g.ctypes.data_as(C.POINTER(C.c_double))), "vof_backward")
        return {"loss": loss.value, "grad_g": g}

    def adjoint(self, field) -> np.ndarray:
        """dL/d(field) of the recorded run's initial state (float64, reference layout)."""
        out = np.empty(self.prm.shape, dtype=np.float64)
        self._check(self._lib.vof_adjoint_download(self._ctx, self._fid(field), out.ctypes.data), "vof_adjoint_download")
        return out

    @property
    def adjoint_kernels_per_step(self) -> int:
        return self._lib.vof_adjoint_kernels_per_step(self._ctx)

    def adjoint_storage(self, policy: int):
        """ADJ_AUTO / ADJ_RECOMPUTE / ADJ_KEEP: where the reverse pass takes
        each step's intermediates from (next forward_record)."""
        self._check(self._lib.vof_adjoint_storage(self._ctx, policy), "vof_adjoint_storage")

    @property
    def adjoint_keeps(self) -> bool:
        """True when the recorded tape keeps the steps' intermediates."""
        r = self._lib.vof_adjoint_keeps(self._ctx)
        self._check(min(r, 0), "vof_adjoint_keeps")
        return r == 1

    @property
    def kernels_per_step(self) -> int:
        return self._lib.vof_kernels_per_step(self._ctx)

    @property
    def device_bytes(self) -> int:
        return self._lib.vof_device_bytes(self._ctx)

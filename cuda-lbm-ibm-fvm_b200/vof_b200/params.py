"""vof_params filled on the host without the CUDA library (numpy float32).

The same values as vof_params_init + vof_params_finalize (include/vof.h):
the constants of voftrial1.cu:1272-1283 and the derived members of
voftrial1.cu:1262-1270, 1285-1291 with the reference's float expressions
(dx = Lx / (float)nx, dxi = 1.0f / dx; numpy float32 division is the IEEE
correctly rounded one, as on the host and the device).  Used where a process
must not map libvof_b200.so: the reference arm of the benchmark, which runs
only the reference's own kernels.  A CPU test checks it against the library's
vof_params_init field by field.
"""
from __future__ import annotations

import numpy as np

from . import MODE_PLAIN, Params

f32 = np.float32


def finalize(p: Params) -> Params:
    """Recompute imin..kmax, dx..dzi and nTot from nx, ny, nz and Lx, Ly, Lz."""
    if p.nx < 1 or p.ny < 1 or p.nz < 1:
        raise ValueError("grid size out of range")
    p.imin, p.jmin, p.kmin = 1, 1, 1
    p.imax, p.jmax, p.kmax = p.nx, p.ny, p.nz
    dx = f32(f32(p.Lx) / f32(p.nx))
    dy = f32(f32(p.Ly) / f32(p.ny))
    dz = f32(f32(p.Lz) / f32(p.nz))
    p.dx, p.dy, p.dz = float(dx), float(dy), float(dz)
    p.dxi, p.dyi, p.dzi = float(f32(1.0) / dx), float(f32(1.0) / dy), float(f32(1.0) / dz)
    tot = (p.nx + 2) * (p.ny + 2) * (p.nz + 2)
    if tot > 0x7FFFFFFF:
        raise ValueError("grid size out of range (nTot is an int)")
    p.nTot = tot
    return p


def host_params(nx: int, ny: int | None = None, nz: int | None = None, **overrides) -> Params:
    """vof_params_init's values, then `overrides`, then finalize()."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = Params()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.Lx = p.Ly = p.Lz = float(f32(0.1))
    p.rho_l, p.rho_g = 1000.0, 50.0
    p.nu_l, p.nu_g = float(f32(1.0e-6)), float(f32(1.5e-5))
    p.sigma = float(f32(0.007))
    p.gx, p.gy, p.gz = 0.0, -5.0, 0.0
    p.dt = float(f32(4.0e-6))
    p.jacobi_iters = 10
    p.mode = MODE_PLAIN
    p.inner_sweeps = 32
    p.max_outer = 200
    p.tol = 1e-8
    p.surface_tension = 0
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return finalize(p)

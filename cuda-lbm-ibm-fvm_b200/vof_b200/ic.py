"""Host-side initial conditions for the dam-break workloads (numpy, float32).

The reference builds its initial field on the device with set_init_F_kernel
(voftrial1.cu:72-93): liquid where the cell-corner coordinate
``clampi(i-1, 0, nx) * dx`` (and likewise in y, z) lies inside the block,
then one apply_bc_F.  The generators here keep that corner convention and the
clamped ghost coordinates, and add the perturbed interface heights of the
benchmark workloads.  Random numbers come from splitmix64 (Steele, Lea and
Flood, 2014; the seeding generator of xoshiro), evaluated counter-style so the
n-th draw of a seed is ``mix(seed + (n+1) * 0x9E3779B97F4A7C15)``.
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """The first n outputs of splitmix64 seeded with `seed` (uint64 array)."""
    with np.errstate(over="ignore"):
        ctr = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + ctr * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, n: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
    """n float64 draws in [lo, hi) from the top 53 bits of splitmix64."""
    u = (splitmix64(seed, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return lo + (hi - lo) * u


def normal(seed: int, n: int, std: float = 1.0) -> np.ndarray:
    """n float64 N(0, std^2) draws, Box-Muller on consecutive uniform pairs."""
    m = (n + 1) // 2
    u = uniform(seed, 2 * m)
    u1 = np.maximum(u[0::2], 1e-300)
    u2 = u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.concatenate([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)])
    out = np.empty(2 * m)
    out[0::2] = z[:m]
    out[1::2] = z[m:]
    return std * out[:n]


def apply_bc_F(F: np.ndarray) -> np.ndarray:
    """Zero-gradient ghosts in the order j, i, k (voftrial1.cu:1122-1135)."""
    F[:, 0, :] = F[:, 1, :]
    F[:, -1, :] = F[:, -2, :]
    F[:, :, 0] = F[:, :, 1]
    F[:, :, -1] = F[:, :, -2]
    F[0, :, :] = F[1, :, :]
    F[-1, :, :] = F[-2, :, :]
    return F


def _nominal(length) -> float:
    # The box lengths are float32 parameters (0.1f); geometry is laid out in
    # cell units against the decimal length they were written as.
    return float(f"{float(length):.7g}")


def _cell_coords(n: int) -> np.ndarray:
    # clampi(i-1, 0, n) for i = 0..n+1: the corner index of set_init_F_kernel
    return np.clip(np.arange(n + 2) - 1, 0, n).astype(np.float64)


def dam_break(prm, h0: float = 0.06, xw: float = 0.04, yw: float = 0.04, height=None) -> np.ndarray:
    """Liquid block x < xw, y < yw, z < h(x, y), tested at cell corners.

    `height` is None (flat h0), or an array of shape (ny+2, nx+2) giving h at
    every column (ghost columns included).  Lengths are converted to cell
    units, (i-1) < xw/Lx*nx; the cell straddling the interface gets the
    fraction clamp(h/dz - (k-1), 0, 1), with fractions within 1e-9 of 0 or 1
    snapped, so a flat h on a cell face gives a binary field.
    """
    nx, ny, nz = prm.nx, prm.ny, prm.nz
    Lx, Ly, Lz = _nominal(prm.Lx), _nominal(prm.Ly), _nominal(prm.Lz)
    x, y, z = _cell_coords(nx), _cell_coords(ny), _cell_coords(nz)
    if height is None:
        h = np.full((ny + 2, nx + 2), h0, dtype=np.float64)
    else:
        h = np.asarray(height, dtype=np.float64)
    hc = h * (nz / Lz)
    inside_xy = (x[None, :] < xw * nx / Lx) & (y[:, None] < yw * ny / Ly)
    frac = np.clip(hc[None, :, :] - z[:, None, None], 0.0, 1.0)
    frac[frac < 1e-9] = 0.0
    frac[frac > 1.0 - 1e-9] = 1.0
    F = np.where(inside_xy[None, :, :], frac, 0.0).astype(np.float32)
    return apply_bc_F(F)


def noisy_height(prm, seed: int = 1, h0: float = 0.06, amp_cells: float = 0.5) -> np.ndarray:
    """h(i,j) = h0 + amp_cells*dx*U(-1,1): the 200^3 benchmark interface (seed 1)."""
    n = (prm.ny + 2) * (prm.nx + 2)
    dx = _nominal(prm.Lx) / prm.nx
    return h0 + amp_cells * dx * uniform(seed, n, -1.0, 1.0).reshape(prm.ny + 2, prm.nx + 2)


def sinusoidal_height(prm, seed: int = 5, h0: float = 0.06, amp_cells: float = 1.0) -> np.ndarray:
    """h = h0 + dx*S/max|S|, S = sum_{m=1..4} sin(2 pi m x/L + phi_m) sin(2 pi m y/L + psi_m)."""
    ph = uniform(seed, 8, 0.0, 2 * np.pi)
    L = _nominal(prm.Lx)
    x = _cell_coords(prm.nx) * (L / prm.nx)
    y = _cell_coords(prm.ny) * (_nominal(prm.Ly) / prm.ny)
    S = np.zeros((prm.ny + 2, prm.nx + 2))
    for m in range(1, 5):
        S += np.sin(2 * np.pi * m * x[None, :] / L + ph[m - 1]) * np.sin(2 * np.pi * m * y[:, None] / L + ph[m + 3])
    return h0 + amp_cells * (L / prm.nx) * S / np.max(np.abs(S))


def rest_state(prm, F: np.ndarray) -> dict:
    """u = v = w = p = 0 with the given F (the reference's memset start)."""
    z = np.zeros(prm.shape, dtype=np.float32)
    return {"F": F.astype(np.float32), "u": z.copy(), "v": z.copy(), "w": z.copy(), "p": z.copy()}


def random_state(prm, seed: int, vel_scale: float = 1.0, p_scale: float = 1.0, zero_frac: float = 0.2) -> dict:
    """Arbitrary finite state for parity tests: F in [0,1] with exact 0/1 regions,
    velocities of both signs with exact zeros (ghosts and wall faces included),
    random pressure.  Nothing here respects the boundary conditions."""
    shape = prm.shape
    n = int(np.prod(shape))
    f = uniform(seed, n, -0.6, 1.6).reshape(shape)
    F = np.clip(f, 0.0, 1.0).astype(np.float32)
    out = {"F": F}
    for q, name in enumerate(("u", "v", "w")):
        a = normal(seed * 7 + q + 1, n, vel_scale)
        z = uniform(seed * 11 + q + 1, n) < zero_frac
        a[z] = 0.0
        out[name] = a.reshape(shape).astype(np.float32)
    out["p"] = normal(seed * 13 + 5, n, p_scale).reshape(shape).astype(np.float32)
    return out

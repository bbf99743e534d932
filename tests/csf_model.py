"""numpy FP32 restatement of the optional continuum-surface-force term
(vof_params.surface_tension = 1; Brackbill, Kothe & Zemach 1992), with the
kernels' operation order: normals and curvature by central differences,
mirror normals beyond a wall, face mean curvature, face density of the
correction.  The GPU test compares the library with it bit for bit; the CPU
test checks its physics on analytic interfaces.  Arrays are padded [k, j, i]
with one ghost layer."""
import numpy as np

from vof_b200 import ic

f32 = np.float32


def droplet(prm, R_cells=5.0):
    """A sphere of liquid centred in the box, the interface smeared over
    about two cells."""
    nx, ny, nz = prm.nx, prm.ny, prm.nz
    k, j, i = np.meshgrid(np.arange(nz + 2), np.arange(ny + 2), np.arange(nx + 2), indexing="ij")
    r = np.sqrt((i - 0.5 - nx / 2) ** 2 + (j - 0.5 - ny / 2) ** 2 + (k - 0.5 - nz / 2) ** 2)
    F = np.clip(0.5 - (r - R_cells) / 2.0, 0.0, 1.0).astype(np.float32)
    return ic.apply_bc_F(F)


def clamp01(v):
    one, zero = f32(1.0), f32(0.0)
    s = (zero + one) + v
    return (s - np.maximum(one, v)) - np.minimum(zero, v)


def rho_of(prm, F):
    f = clamp01(F)
    return f32(prm.rho_g) * (f32(1.0) - f) + f32(prm.rho_l) * f


def _neighbour(a, axis, step):
    """a shifted by `step` cells along `axis`, with mirror images beyond the
    walls (the wall-normal component negated)."""
    pad = [(0, 0)] * 3
    pad[axis] = (1, 1)
    e = np.pad(a, pad)
    lo = [slice(None)] * 3
    hi = [slice(None)] * 3
    lo[axis], hi[axis] = 0, -1
    first = [slice(None)] * 3
    last = [slice(None)] * 3
    first[axis], last[axis] = 0, -1
    e[tuple(lo)] = -a[tuple(first)]
    e[tuple(hi)] = -a[tuple(last)]
    sl = [slice(None)] * 3
    sl[axis] = slice(1 + step, e.shape[axis] - 1 + step)
    return e[tuple(sl)]


def csf_normals(prm, F):
    """Unit normals grad F / |grad F| of the interior cells (x, y, z
    components, each [nz, ny, nx]); zero where |grad F| <= 1e-6 dxi."""
    dxi, dyi, dzi = f32(prm.dxi), f32(prm.dyi), f32(prm.dzi)
    hx, hy, hz = f32(0.5) * dxi, f32(0.5) * dyi, f32(0.5) * dzi
    gx = (F[1:-1, 1:-1, 2:] - F[1:-1, 1:-1, :-2]) * hx
    gy = (F[1:-1, 2:, 1:-1] - F[1:-1, :-2, 1:-1]) * hy
    gz = (F[2:, 1:-1, 1:-1] - F[:-2, 1:-1, 1:-1]) * hz
    mag = np.sqrt(gx * gx + gy * gy + gz * gz)
    has = mag > f32(1e-6) * dxi
    with np.errstate(invalid="ignore", divide="ignore"):
        return [np.where(has, c / mag, f32(0.0)).astype(np.float32) for c in (gx, gy, gz)]


def csf_curvature(prm, F):
    """kappa = -div n on the interior cells, zero on the ghosts (padded)."""
    nx, ny, nz = prm.nx, prm.ny, prm.nz
    hx, hy, hz = f32(0.5) * f32(prm.dxi), f32(0.5) * f32(prm.dyi), f32(0.5) * f32(prm.dzi)
    n = csf_normals(prm, F)
    xe, xw = _neighbour(n[0], 2, 1), _neighbour(n[0], 2, -1)
    yn, ys = _neighbour(n[1], 1, 1), _neighbour(n[1], 1, -1)
    zu, zd = _neighbour(n[2], 0, 1), _neighbour(n[2], 0, -1)
    kap = np.zeros_like(F)
    kap[1:nz + 1, 1:ny + 1, 1:nx + 1] = -(((xe - xw) * hx + (yn - ys) * hy) + (zu - zd) * hz)
    return kap


def csf_face_forces(prm, F):
    """Face forces per volume sigma * kappa_face * dF/dh on u, v, w faces:
    [(force, mask)] for x, y, z; mask marks the faces the term updates (not
    the first interior layer along the axis: walls)."""
    nx, ny, nz = prm.nx, prm.ny, prm.nz
    kap = csf_curvature(prm, F)
    sigma = f32(prm.sigma)
    out = []
    for axis, hinv in ((2, f32(prm.dxi)), (1, f32(prm.dyi)), (0, f32(prm.dzi))):
        c = [slice(1, nz + 1), slice(1, ny + 1), slice(1, nx + 1)]
        m = list(c)
        m[axis] = slice(0, c[axis].stop - 1)  # the cell below along the axis
        f = np.zeros_like(F)
        f[tuple(c)] = (sigma * (f32(0.5) * (kap[tuple(m)] + kap[tuple(c)]))) * ((F[tuple(c)] - F[tuple(m)]) * hinv)
        mask = np.zeros(F.shape, dtype=bool)
        mask[tuple(c)] = True
        w = [slice(None)] * 3
        w[axis] = 1
        mask[tuple(w)] = False
        out.append((f, mask))
    return out


def csf_increments(prm, F):
    """dt * (face acceleration) on u, v, w faces: [(increment, mask)]."""
    nx, ny, nz = prm.nx, prm.ny, prm.nz
    rho = rho_of(prm, F)
    dt = f32(prm.dt)
    out = []
    for axis, (f, mask) in zip((2, 1, 0), csf_face_forces(prm, F)):
        c = [slice(1, nz + 1), slice(1, ny + 1), slice(1, nx + 1)]
        m = list(c)
        m[axis] = slice(0, c[axis].stop - 1)
        r = f32(0.5) * (rho[tuple(m)] + rho[tuple(c)])
        inc = np.zeros_like(F)
        inc[tuple(c)] = dt * (f[tuple(c)] / r)
        out.append((inc, mask))
    return out

"""The optional continuum-surface-force term (vof_params.surface_tension = 1;
an extension: the reference has no surface tension).

Its acceleration is restated here in numpy FP32 with the kernels' operation
order (normals and curvature by central differences, mirror normals beyond a
wall, face mean curvature, face density of the correction), so u*, v*, w* of
a step with the term must equal those of the plain step plus dt times that
acceleration bit for bit.  Off (the default), the step is the plain one.
"""
import numpy as np
import pytest

from vof_b200 import ic

pytestmark = pytest.mark.gpu

f32 = np.float32


def droplet(prm, R_cells=5.0):
    """A sphere of liquid, the interface smeared over about two cells."""
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


def csf_increments(prm, F):
    """dt * (face acceleration) on u, v, w faces of the padded arrays [k, j, i]."""
    nx, ny, nz = prm.nx, prm.ny, prm.nz
    dxi, dyi, dzi = f32(prm.dxi), f32(prm.dyi), f32(prm.dzi)
    hx, hy, hz = f32(0.5) * dxi, f32(0.5) * dyi, f32(0.5) * dzi
    I = (slice(1, nz + 1), slice(1, ny + 1), slice(1, nx + 1))
    gx = (F[1:-1, 1:-1, 2:] - F[1:-1, 1:-1, :-2]) * hx
    gy = (F[1:-1, 2:, 1:-1] - F[1:-1, :-2, 1:-1]) * hy
    gz = (F[2:, 1:-1, 1:-1] - F[:-2, 1:-1, 1:-1]) * hz
    mag = np.sqrt(gx * gx + gy * gy + gz * gz)
    has = mag > f32(1e-6) * dxi
    with np.errstate(invalid="ignore", divide="ignore"):
        n = [np.where(has, c / mag, f32(0.0)).astype(np.float32) for c in (gx, gy, gz)]
    # neighbours with mirror images beyond the walls (wall-normal component negated)
    def nb(a, axis, step):
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
    xe, xw = nb(n[0], 2, 1), nb(n[0], 2, -1)
    yn, ys = nb(n[1], 1, 1), nb(n[1], 1, -1)
    zu, zd = nb(n[2], 0, 1), nb(n[2], 0, -1)
    kap_i = -(((xe - xw) * hx + (yn - ys) * hy) + (zu - zd) * hz)
    kap = np.zeros_like(F)
    kap[I] = kap_i
    rho = rho_of(prm, F)
    sigma, dt = f32(prm.sigma), f32(prm.dt)
    out = []
    for axis, hinv in ((2, dxi), (1, dyi), (0, dzi)):
        c = [slice(1, nz + 1), slice(1, ny + 1), slice(1, nx + 1)]
        m = list(c)
        m[axis] = slice(0, c[axis].stop - 1)  # the cell below along the axis
        Fa, Fb = F[tuple(m)], F[tuple(c)]
        ka, kb = kap[tuple(m)], kap[tuple(c)]
        f = (sigma * (f32(0.5) * (ka + kb))) * ((Fb - Fa) * hinv)
        r = f32(0.5) * (rho[tuple(m)] + rho[tuple(c)])
        inc = np.zeros_like(F)
        inc[tuple(c)] = dt * (f / r)
        mask = np.zeros(F.shape, dtype=bool)
        mask[tuple(c)] = True
        # faces on the first interior layer along the axis are walls: no update
        w = [slice(None)] * 3
        w[axis] = 1
        mask[tuple(w)] = False
        out.append((inc, mask))
    return out


def run(V, prm, state):
    with V.Solver(prm) as s:
        s.upload_state(**state)
        s.step(1)
        out = s.state()
        for k in ("ustar", "vstar", "wstar"):
            out[k] = s.download(k)
    return out


@pytest.mark.parametrize("shape", [(20, 18, 16), (13, 9, 11)])
def test_surface_tension_adds_the_csf_acceleration(cuda, V, shape):
    prm0 = V.default_params(*shape, dt=1e-4, gy=0.0, gz=-9.81)
    prm1 = V.default_params(*shape, dt=1e-4, gy=0.0, gz=-9.81, surface_tension=1, sigma=0.07)
    F = droplet(prm0, R_cells=min(shape) / 3.0)
    state = ic.rest_state(prm0, F)
    rng = np.random.default_rng(2)
    for k in ("u", "v", "w"):
        state[k] = (0.01 * rng.standard_normal(prm0.shape)).astype(np.float32)
    plain = run(V, prm0, state)
    got = run(V, prm1, state)
    inc = csf_increments(prm1, F)
    for name, (d, mask) in zip(("ustar", "vstar", "wstar"), inc):
        want = np.where(mask, plain[name] + d, plain[name]).astype(np.float32)
        bad = np.argwhere(got[name].view(np.uint32) != want.view(np.uint32))
        assert bad.size == 0, (name, len(bad), bad[:3])
    assert any(np.abs(d[m]).max() > 0 for d, m in inc)


def test_surface_tension_is_off_by_default(cuda, V):
    prm = V.default_params(16, 12, 10, dt=1e-4)
    assert prm.surface_tension == 0
    state = ic.random_state(prm, seed=4)
    a = run(V, prm, state)
    prm_off = V.default_params(16, 12, 10, dt=1e-4, sigma=0.5)  # sigma alone changes nothing
    b = run(V, prm_off, state)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_surface_tension_refuses_the_adjoint(cuda, V):
    prm = V.default_params(12, 10, 8, surface_tension=1)
    with V.Solver(prm) as s:
        s.upload_state(**ic.rest_state(prm, droplet(prm, 3.0)))
        with pytest.raises(V.VofError) as e:
            s.forward_record(1, 2, 0)
        assert e.value.status == V.E_UNSUPPORTED

"""The surface-tension restatement (tests/csf_model.py), which the GPU test
holds the library to bit for bit, against the geometry it models: the
curvature of a sphere is 2/R and of a cylinder 1/R, a plane has none, and the
force on a droplet points inward and sums to zero.  The interfaces are tanh
profiles one cell wide (a clipped linear ramp leaves normals undefined at the
ramp's ends, where CSF's curvature is known to be wrong).  CPU only."""
import numpy as np
import pytest

import csf_model as M


def params(V, n):
    return V.default_params(n, n, n, dt=1e-4, sigma=0.07, surface_tension=1)


def smooth_interface(n, R, width=1.0, cylinder=False):
    """F = 1 inside radius R (cells) around the box centre, a tanh profile
    `width` cells wide; a cylinder along z when `cylinder`."""
    k, j, i = np.meshgrid(np.arange(n + 2), np.arange(n + 2), np.arange(n + 2), indexing="ij")
    r2 = (i - 0.5 - n / 2) ** 2 + (j - 0.5 - n / 2) ** 2
    if not cylinder:
        r2 = r2 + (k - 0.5 - n / 2) ** 2
    return (0.5 - 0.5 * np.tanh((np.sqrt(r2) - R) / width)).astype(np.float32)


def band_ratio(prm, F, R, per_radius):
    """kappa R / per_radius on the interior cells with 0.3 < F < 0.7."""
    kap = M.csf_curvature(prm, F)[1:-1, 1:-1, 1:-1]
    Fi = F[1:-1, 1:-1, 1:-1]
    band = (Fi > 0.3) & (Fi < 0.7)
    return kap[band] * np.float32(R * prm.dx) / per_radius


@pytest.mark.parametrize("R", [6.0, 8.0, 12.0])
def test_sphere_curvature_is_two_over_R(V, R):
    n = int(4 * R)
    prm = params(V, n)
    ratio = band_ratio(prm, smooth_interface(n, R), R, 2)
    assert abs(np.median(ratio) - 1) < 0.05, np.median(ratio)


@pytest.mark.parametrize("R", [6.0, 8.0, 12.0])
def test_cylinder_curvature_is_one_over_R(V, R):
    """F independent of z: the z normals vanish, kappa = 1/R."""
    n = int(4 * R)
    prm = params(V, n)
    F = smooth_interface(n, R, cylinder=True)
    assert not M.csf_normals(prm, F)[2].any()
    ratio = band_ratio(prm, F, R, 1)
    assert abs(np.median(ratio) - 1) < 0.05, np.median(ratio)


def test_plane_has_no_curvature_away_from_the_walls(V):
    """A smooth profile along x (0.1 < F < 0.9 everywhere): unit normals
    along -x, no curvature and no force two cells or more from the x walls
    (next to a wall the mirrored normal bends the plane)."""
    n = 24
    prm = params(V, n)
    x = np.arange(n + 2, dtype=np.float64)
    prof = (0.5 - 0.4 * np.tanh((x - n / 2) / 4.0)).astype(np.float32)
    F = np.broadcast_to(prof[None, None, :], prm.shape).copy()
    nx_, ny_, nz_ = M.csf_normals(prm, F)
    assert not ny_.any() and not nz_.any()
    assert np.allclose(nx_, -1.0, atol=1e-6)
    kap = M.csf_curvature(prm, F)
    assert np.abs(kap[1:-1, 1:-1, 3:-3]).max() <= 1e-5 * prm.dxi
    fx = M.csf_face_forces(prm, F)[0][0]
    assert np.abs(fx[1:-1, 1:-1, 4:-3]).max() <= 1e-5 * prm.sigma * prm.dxi * prm.dxi


@pytest.mark.parametrize("R", [6.0, 8.0])
def test_droplet_force_points_inward_and_sums_to_zero(V, R):
    n = int(4 * R)
    prm = params(V, n)
    F = smooth_interface(n, R)
    c = 0.5 + n / 2  # the droplet's centre in padded cell indices
    for axis, (f, mask) in zip((2, 1, 0), M.csf_face_forces(prm, F)):
        fm = f[mask].astype(np.float64)
        assert abs(fm.sum()) <= 1e-9 * np.abs(fm).sum()
        strong = mask & (np.abs(f) > 0.01 * np.abs(f).max())
        assert strong.sum() > 0
        pos = np.argwhere(strong)[:, axis] - 0.5  # face h lies between cells h - 1 and h
        assert np.all(np.sign(f[strong]) == -np.sign(pos - c))


def test_no_force_where_F_is_uniform(V):
    n = 32
    prm = params(V, n)
    F = M.droplet(prm, R_cells=8.0)
    for axis, (f, mask) in zip((2, 1, 0), M.csf_face_forces(prm, F)):
        flat = mask & (F == np.roll(F, 1, axis=axis))
        assert not f[flat].any()

"""The optional continuum-surface-force term (vof_params.surface_tension = 1;
an extension: the reference has no surface tension).

Its acceleration is restated in numpy FP32 with the kernels' operation order
(tests/csf_model.py: normals and curvature by central differences, mirror
normals beyond a wall, face mean curvature, face density of the correction),
so u*, v*, w* of a step with the term must equal those of the plain step plus
dt times that acceleration bit for bit.  Off (the default), the step is the
plain one.
"""
import numpy as np
import pytest

from csf_model import csf_increments, droplet
from vof_b200 import ic

pytestmark = pytest.mark.gpu


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

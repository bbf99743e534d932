"""The reference's apply_bc (voftrial1.cu:943-956; set_bc_{j,i,k}_kernel of
:105-228) through the C-ABI: vof_apply_bc_fields on device buffers in the
reference layout and vof_apply_bc on a context's state.  Both must equal the
oracle's literal three passes bit for bit (the boundary conditions are copies
and zeros).  The oracle itself is pinned against the reference's own kernels
here (oracle/_ref) and against the committed fixtures in the CPU suite."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BC = ("u", "v", "w", "F", "p", "rho")
SHAPES = [(1, 1, 1), (1, 3, 2), (4, 1, 3), (5, 6, 1), (7, 5, 4), (33, 9, 6), (200, 3, 2)]


def random_fields(prm, seed):
    rng = np.random.default_rng(seed)
    return {k: rng.standard_normal(prm.shape).astype(np.float32) for k in BC}


@pytest.mark.parametrize("shape", SHAPES)
def test_fields_entry_point_matches_the_oracle(cuda, V, orc, shape):
    import torch

    prm = V.default_params(*shape)
    inp = random_fields(prm, seed=sum(shape))
    want = orc.apply_bc(prm, inp)
    dev = {k: torch.from_numpy(inp[k]).cuda() for k in BC}
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    V.apply_bc_fields(prm, stream=s.cuda_stream, **{k: t.data_ptr() for k, t in dev.items()})
    s.synchronize()
    for k in BC:
        assert np.array_equal(dev[k].cpu().numpy(), want[k]), k


def test_skipped_fields_stay_as_they_were(cuda, V, orc):
    import torch

    prm = V.default_params(9, 7, 5)
    inp = random_fields(prm, seed=3)
    want = orc.apply_bc(prm, inp)
    dev = {k: torch.from_numpy(inp[k]).cuda() for k in BC}
    V.apply_bc_fields(prm, **{k: dev[k].data_ptr() for k in ("v", "F")})  # the legacy default stream
    torch.cuda.synchronize()
    for k in BC:
        assert np.array_equal(dev[k].cpu().numpy(), want[k] if k in ("v", "F") else inp[k]), k


def test_context_entry_point_matches_the_oracle(cuda, V, orc):
    prm = V.default_params(21, 13, 8, dt=5e-4)
    inp = random_fields(prm, seed=8)
    want = orc.apply_bc(prm, inp)
    with V.Solver(prm) as s:
        s.upload_state(**{k: inp[k] for k in ("F", "u", "v", "w", "p")})
        s.apply_bc()
        got = s.state()
        # idempotent: a second call changes nothing
        s.apply_bc()
        again = s.state()
    for k in ("F", "u", "v", "w", "p"):
        assert np.array_equal(got[k], want[k]), k
        assert np.array_equal(again[k], want[k]), k


def test_then_a_step_matches_the_oracle(cuda, V, orc):
    """apply_bc between steps, as a caller of the reference would place it."""
    from vof_b200 import ic

    prm = V.default_params(16, 12, 10, dt=2e-4, gy=0.0, gz=-9.81)
    st = ic.random_state(prm, seed=5, vel_scale=1.0)
    with V.Solver(prm) as s:
        s.upload_state(**st)
        s.step(1)
        s.apply_bc()
        s.step(2)
        got = s.state()
    mid = orc.run_f32(prm, st, 1, 1)
    mid = orc.apply_bc(prm, {**mid, "rho": np.zeros(prm.shape, np.float32)})
    want = orc.run_f32(prm, mid, 2, 1)
    for k in ("F", "u", "v", "w", "p"):
        assert np.array_equal(got[k], want[k]), k


def test_errors(cuda, V):
    import ctypes as C

    lib = V.lib()
    prm = V.default_params(6, 5, 4)
    assert lib.vof_apply_bc_fields(None, None, None, None, None, None, None, None) == V.E_INVALID
    bad = V.default_params(6, 5, 4)
    bad.nTot += 1
    assert lib.vof_apply_bc_fields(C.byref(bad), None, None, None, None, None, None, None) == V.E_INVALID
    bad = V.default_params(6, 5, 4)
    bad.nx = 0
    assert lib.vof_apply_bc_fields(C.byref(bad), None, None, None, None, None, None, None) == V.E_SIZE
    assert lib.vof_apply_bc(None) == V.E_INVALID
    # nothing to do: every field skipped
    assert lib.vof_apply_bc_fields(C.byref(prm), None, None, None, None, None, None, None) == V.OK
    mixed = V.default_params(16, 16, 16, mode=V.MODE_MIXED)
    with V.Solver(mixed) as s:
        with pytest.raises(V.VofError) as e:
            s.apply_bc()
        assert e.value.status == V.E_UNSUPPORTED


@pytest.mark.parametrize("shape", [(7, 5, 4), (1, 3, 2), (12, 9, 6)])
def test_oracle_matches_the_reference_kernels(cuda, orc, V, shape):
    if not orc.ref_available("sm100a"):
        pytest.skip("oracle/_ref not built (needs the reference source)")
    prm = V.default_params(*shape)
    inp = random_fields(prm, seed=11)
    ref = orc.ref_apply_bc(prm, inp)
    want = orc.apply_bc(prm, inp)
    for k in BC:
        assert np.array_equal(ref[k], want[k]), k

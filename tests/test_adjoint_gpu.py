"""The CUDA adjoint (vof_forward_record / vof_backward) against the host adjoint
(oracle/vof_adjoint.cpp) on the same FP32 trajectory.

The device forward is the plain FP32 step (bit-identical to the oracle's FP32
step), so both reverse passes see the same values and take the same switches;
they differ only in the order of FP64 sums (the device scatters with atomics).
Tolerance: relative L2 1e-9 on every gradient field, 1e-9 on dL/dg, the loss
to 1e-12.
"""
import numpy as np
import pytest

from vof_b200 import ic

pytestmark = pytest.mark.gpu

GRADS = (("lF", "F"), ("lu", "u"), ("lv", "v"), ("lw", "w"), ("lp", "p"))


def dam_state(V, nx, ny, nz, seed=3, amp=1e-2, **kw):
    prm = V.default_params(nx, ny, nz, dt=2e-4, gy=0.0, gz=-9.81, **kw)
    st = ic.rest_state(prm, ic.dam_break(prm))
    rng = np.random.default_rng(seed)
    for k in ("u", "v", "w"):
        st[k] = (st[k] + amp * rng.standard_normal(prm.shape)).astype(np.float32)
    return prm, st


def box_of(prm):
    return (0.3 * prm.Lx, 0.6 * prm.Lx, -1e9, 1e9, -1e9, 0.6 * prm.Lz)


def gpu_adjoint(V, prm, st, istep0, nsteps, box, every=0, policy=None):
    with V.Solver(prm) as s:
        if policy is not None:
            s.adjoint_storage(policy)
        s.upload_state(**st)
        s.forward_record(istep0, nsteps, every)
        final = s.state()
        r = s.backward(box)
        r.update({k: s.adjoint(f) for k, f in GRADS})
        r["keeps"] = s.adjoint_keeps
    r["final"] = final
    return r


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def check_against_host(orc, prm, st, istep0, nsteps, box, got, tol=1e-9):
    ref = orc.adjoint(prm, st, istep0, nsteps, box, "f32")
    assert got["loss"] == pytest.approx(ref["loss"], rel=1e-12, abs=1e-300)
    for k, _ in GRADS:
        assert rel(got[k], ref[k]) <= tol, (k, rel(got[k], ref[k]))
    assert np.allclose(got["grad_g"], ref["grad_g"], rtol=tol, atol=1e-30), (got["grad_g"], ref["grad_g"])


@pytest.mark.parametrize("sweep", ["march", "shared"])
@pytest.mark.parametrize("shape,nsteps,istep0", [((16, 14, 12), 6, 1), ((13, 17, 11), 5, 0), ((12, 12, 20), 4, 2),
                                                  ((70, 9, 8), 3, 1), ((7, 66, 9), 3, 2), ((9, 8, 75), 3, 0)])
def test_device_adjoint_matches_host(cuda, V, orc, shape, nsteps, istep0, sweep, monkeypatch):
    """Long lines along each axis split into several segments of the line march."""
    monkeypatch.setenv("VOF_ADJ_SWEEP", sweep)
    prm, st = dam_state(V, *shape)
    box = box_of(prm)
    got = gpu_adjoint(V, prm, st, istep0, nsteps, box)
    ref_final = orc.run_f32(prm, st, istep0, nsteps)
    for k in ("F", "u", "v", "w", "p"):  # the recorded run is the plain run, bit for bit
        assert np.array_equal(got["final"][k], ref_final[k]), k
    check_against_host(orc, prm, st, istep0, nsteps, box, got)


@pytest.mark.parametrize("sweep", ["march", "shared"])
@pytest.mark.parametrize("policy", ["ADJ_KEEP", "ADJ_RECOMPUTE"])
@pytest.mark.parametrize("every", [1, 3, 4, 0])
def test_checkpoint_spacing_does_not_change_the_gradient(cuda, V, orc, every, policy, sweep, monkeypatch):
    """Kept intermediates (from the segment replay) and recomputed ones (from
    each step's start state) are the forward's bits either way; both FCT sweep
    adjoint kernels (line march, shared memory) give the host's gradient."""
    monkeypatch.setenv("VOF_ADJ_SWEEP", sweep)
    prm, st = dam_state(V, 14, 12, 10, seed=5)
    box = box_of(prm)
    got = gpu_adjoint(V, prm, st, 1, 9, box, every=every, policy=getattr(V, policy))
    assert got["keeps"] == (policy == "ADJ_KEEP")
    check_against_host(orc, prm, st, 1, 9, box, got)


def test_storage_policy_auto_keeps_small_tapes(cuda, V):
    prm, st = dam_state(V, 10, 10, 10)
    with V.Solver(prm) as s:
        with pytest.raises(V.VofError) as e:
            s.adjoint_keeps
        assert e.value.status == V.E_STATE
        with pytest.raises(V.VofError) as e:
            s.adjoint_storage(7)
        assert e.value.status == V.E_INVALID
        s.upload_state(**st)
        s.forward_record(0, 4, 2)
        assert s.adjoint_keeps
        b0 = s.device_bytes
        s.adjoint_storage(V.ADJ_RECOMPUTE)
        s.upload_state(**st)
        s.forward_record(0, 4, 2)
        assert not s.adjoint_keeps
        assert s.device_bytes < b0  # kept: 5 more fields per segment step, one state fewer


@pytest.mark.parametrize("iters", [0, 1, 3])
def test_jacobi_iteration_counts(cuda, V, orc, iters):
    prm, st = dam_state(V, 12, 11, 10, jacobi_iters=iters)
    box = box_of(prm)
    got = gpu_adjoint(V, prm, st, 0, 4, box)
    check_against_host(orc, prm, st, 0, 4, box, got)


def test_velocity_perturbation_gradient_32(cuda, V, orc):
    """The gradient the adjoint is for: dL/d(initial velocity perturbation)
    on interior faces and dL/dg, loss = F dV over x > 0.06, z < 0.02 (cell
    centres), a 32^3 dam break with N(0, 1e-3^2) face perturbations."""
    prm = V.default_params(32, dt=1e-4, gy=0.0, gz=-9.81)
    st = ic.rest_state(prm, ic.dam_break(prm))
    rng = np.random.default_rng(3)
    for k, lo in (("u", (1, 1, 2)), ("v", (1, 2, 1)), ("w", (2, 1, 1))):
        d = np.zeros(prm.shape, dtype=np.float32)
        d[lo[0]:prm.nz + 1, lo[1]:prm.ny + 1, lo[2]:prm.nx + 1] = 1e-3 * rng.standard_normal(
            (prm.nz + 1 - lo[0], prm.ny + 1 - lo[1], prm.nx + 1 - lo[2]))
        st[k] = st[k] + d
    box = (0.06, 1e9, -1e9, 1e9, -1e9, 0.02)
    got = gpu_adjoint(V, prm, st, 1, 30, box, every=6)
    check_against_host(orc, prm, st, 1, 30, box, got)
    assert np.linalg.norm(got["lu"]) > 0


@pytest.mark.parametrize("every", [3, 7, 1])
def test_second_reverse_pass_replays_the_recorded_tail(cuda, V, every):
    """The record runs its last segment (segments align to the end of the run:
    7 steps in 3 give 1 + 3 + 3) as the reverse pass replays it, and the first
    reverse pass starts there without a replay; a second reverse pass of the
    same record replays every segment.  The recorded state is the plain run's
    bit for bit; the two passes agree to the order of their FP64 atomic sums."""
    prm, st = dam_state(V, 16, 14, 12)
    box = box_of(prm)
    with V.Solver(prm) as s:
        s.upload_state(**st)
        s.run(1, 7)
        plain = s.state()
    with V.Solver(prm) as s:
        s.adjoint_storage(V.ADJ_KEEP)
        s.upload_state(**st)
        s.forward_record(1, 7, every)
        rec = s.state()
        r1 = s.backward(box)
        a1 = {k: s.adjoint(f) for k, f in GRADS}
        r2 = s.backward(box)
        a2 = {k: s.adjoint(f) for k, f in GRADS}
    for k in ("F", "u", "v", "w", "p"):
        assert np.array_equal(rec[k], plain[k]), k
    assert r1["loss"] == r2["loss"]
    assert np.allclose(r1["grad_g"], r2["grad_g"], rtol=1e-11, atol=1e-30)
    for k in a1:
        assert rel(a1[k], a2[k]) <= 1e-11, (k, rel(a1[k], a2[k]))


def test_state_errors(cuda, V):
    prm, st = dam_state(V, 10, 10, 10)
    with V.Solver(prm) as s:
        s.upload_state(**st)
        with pytest.raises(V.VofError) as e:
            s.backward(box_of(prm))
        assert e.value.status == V.E_STATE


@pytest.mark.parametrize("policy", ["ADJ_KEEP", "ADJ_RECOMPUTE"])
@pytest.mark.parametrize("mode", ["MODE_MIXED", "MODE_FP64"])
def test_convergent_mode_adjoint_matches_host(cuda, V, orc, mode, policy):
    """MIXED / FP64 modes: the pressure is the solve of the mean-free system;
    its adjoint is the same solve on the pressure adjoint (device: the
    multigrid defect correction to 1e-10; host: CG to 1e-12 on the FP32
    trajectory).  The two forwards differ only by the solves' tolerances, so
    the comparison is at 1e-4 relative."""
    prm, st = dam_state(V, 16, 14, 12, mode=getattr(V, mode), tol=1e-10, max_outer=100)
    box = box_of(prm)
    with V.Solver(prm) as s:
        s.adjoint_storage(getattr(V, policy))
        s.upload_state(**st)
        s.forward_record(1, 6, 3)
        got = s.backward(box)
        got.update({k: s.adjoint(f) for k, f in GRADS})
    ref = orc.adjoint(prm, st, 1, 6, box, "f32", conv_tol=1e-12)
    assert got["loss"] == pytest.approx(ref["loss"], rel=1e-6)
    for k in ("lF", "lu", "lv", "lw"):
        assert rel(got[k], ref[k]) <= 1e-4, (k, rel(got[k], ref[k]))
    assert np.count_nonzero(got["lp"]) == 0
    assert np.allclose(got["grad_g"], ref["grad_g"], rtol=1e-4, atol=1e-30)

"""Convergent pressure modes (VOF_MODE_MIXED: BF16-stored/FP32 multigrid inside
FP64 defect correction; VOF_MODE_FP64: the same with FP64 multigrid) against the
FP64 oracle whose pressure is solved by conjugate gradients to 1e-12.

Tolerances (rel-L2 after the stated steps; p compared with mean(p) = 0, which
both sides impose): pressure relative residual <= 1e-8 at every step (the
target), F <= 1e-5 (the target), u, v, w <= 1e-4, p <= 1e-5.
"""
import numpy as np
import pytest

from vof_b200 import ic

pytestmark = pytest.mark.gpu

STATE = ("F", "u", "v", "w", "p")


def rel_l2(a, b, interior=False):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if interior:
        a, b = a[1:-1, 1:-1, 1:-1], b[1:-1, 1:-1, 1:-1]
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def run_mode(V, prm, state, istep0, nsteps):
    stats = []
    with V.Solver(prm) as s:
        s.upload_state(**state)
        for t in range(nsteps):
            s.step(istep0 + t)
            stats.append(s.solver_stats())
        out = s.state()
    return out, stats


@pytest.mark.parametrize("mode", ["MODE_MIXED", "MODE_FP64"])
def test_dam_break_32_vs_fp64_oracle(cuda, V, orc, mode):
    prm = V.default_params(32, gy=0.0, gz=-9.81, mode=getattr(V, mode), tol=1e-8, max_outer=60)
    state = ic.rest_state(prm, ic.dam_break(prm))
    got, stats = run_mode(V, prm, state, 1, 20)
    assert all(s["rel_final"] <= 1e-8 for s in stats), stats
    ref = orc.run_conv_f64(prm, state, 1, 20, tol=1e-12)
    assert rel_l2(got["F"], ref["F"]) <= 1e-5
    for k in ("u", "v", "w"):
        assert rel_l2(got[k], ref[k]) <= 1e-4, (k, rel_l2(got[k], ref[k]))
    assert rel_l2(got["p"], ref["p"], interior=True) <= 1e-5
    assert abs(np.mean(got["p"][1:-1, 1:-1, 1:-1].astype(np.float64))) <= 1e-6 * np.abs(ref["p"]).max()


@pytest.mark.parametrize("shape", [(30, 20, 18), (16, 16, 40), (5, 7, 9)])
def test_random_state_odd_factor_grids(cuda, V, orc, shape):
    """Grids whose multigrid hierarchy coarsens by 2, 3, 5 and 7 (or not at all)."""
    nx, ny, nz = shape
    prm = V.default_params(nx, ny, nz, dt=2e-4, mode=V.MODE_MIXED, tol=1e-8, max_outer=200)
    state = ic.random_state(prm, seed=sum(shape), vel_scale=0.5)
    got, stats = run_mode(V, prm, state, 1, 3)
    assert all(s["rel_final"] <= 1e-8 for s in stats), stats
    ref = orc.run_conv_f64(prm, state, 1, 3, tol=1e-12)
    assert rel_l2(got["F"], ref["F"]) <= 1e-5
    for k in ("u", "v", "w"):
        assert rel_l2(got[k], ref[k]) <= 1e-4, (k, rel_l2(got[k], ref[k]))


@pytest.mark.parametrize("mode", ["MODE_MIXED", "MODE_FP64"])
@pytest.mark.parametrize("shape", [(64, 64, 64), (60, 48, 40)])
def test_multi_block_levels_vs_fp64_oracle(cuda, V, orc, mode, shape):
    """Grids whose fine levels are smoothed by the multi-block kernels, with
    the fused residual / first sweep and last sweep / update kernels."""
    prm = V.default_params(*shape, dt=2e-4, mode=getattr(V, mode), tol=1e-8, max_outer=100)
    state = ic.random_state(prm, seed=3, vel_scale=0.5)
    got, stats = run_mode(V, prm, state, 1, 3)
    assert all(s["rel_final"] <= 1e-8 for s in stats), stats
    assert all(s["outer"] <= 25 for s in stats), stats
    ref = orc.run_conv_f64(prm, state, 1, 3, tol=1e-12)
    assert rel_l2(got["F"], ref["F"]) <= 1e-5
    for k in ("u", "v", "w"):
        assert rel_l2(got[k], ref[k]) <= 1e-4, (k, rel_l2(got[k], ref[k]))
    assert rel_l2(got["p"], ref["p"], interior=True) <= 1e-5


def test_large_prime_grid_without_coarsening(cuda, V, orc):
    """37^3 has no factor to coarsen by and is too large for the one-block
    kernel: the level is smoothed by mean-free damped sweeps only (slow but
    convergent)."""
    prm = V.default_params(37, 37, 37, dt=2e-4, mode=V.MODE_MIXED, tol=1e-6, max_outer=400)
    state = ic.random_state(prm, seed=8, vel_scale=0.5)
    got, stats = run_mode(V, prm, state, 1, 1)
    assert stats[0]["rel_final"] <= 1e-6, stats
    ref = orc.run_conv_f64(prm, state, 1, 1, tol=1e-12)
    assert rel_l2(got["F"], ref["F"]) <= 1e-5
    for k in ("u", "v", "w"):
        assert rel_l2(got[k], ref[k]) <= 1e-3, (k, rel_l2(got[k], ref[k]))


def test_mixed_and_fp64_modes_agree(cuda, V):
    prm_m = V.default_params(24, 24, 24, dt=1e-4, mode=V.MODE_MIXED, tol=1e-10, max_outer=80)
    prm_d = V.default_params(24, 24, 24, dt=1e-4, mode=V.MODE_FP64, tol=1e-10, max_outer=80)
    state = ic.random_state(prm_m, seed=5, vel_scale=0.3)
    a, _ = run_mode(V, prm_m, state, 1, 4)
    b, _ = run_mode(V, prm_d, state, 1, 4)
    for k in STATE:
        assert rel_l2(a[k], b[k], interior=(k == "p")) <= 1e-6, k


def test_warm_start_needs_fewer_cycles(cuda, V):
    prm = V.default_params(32, gy=0.0, gz=-9.81, mode=V.MODE_MIXED, tol=1e-8, max_outer=60)
    state = ic.rest_state(prm, ic.dam_break(prm))
    _, stats = run_mode(V, prm, state, 1, 6)
    assert stats[-1]["outer"] <= stats[0]["outer"]
    assert stats[-1]["rel_initial"] < 1.0


def test_not_converged_status_and_state_still_advanced(cuda, V):
    prm = V.default_params(20, 20, 20, dt=1e-4, mode=V.MODE_MIXED, tol=1e-14, max_outer=1)
    state = ic.random_state(prm, seed=9, vel_scale=0.3)
    with V.Solver(prm) as s:
        s.upload_state(**state)
        with pytest.raises(V.VofError) as e:
            s.step(1)
        assert e.value.status == V.E_NOT_CONVERGED
        assert s.solver_stats()["outer"] == 1
        F = s.download("F")
    assert not np.array_equal(F, state["F"])


def test_upload_of_pressure_seeds_the_solver(cuda, V):
    """Uploading the converged pressure of a step into a fresh context and
    repeating that step starts the solve at (almost) zero residual."""
    prm = V.default_params(16, 16, 16, dt=1e-4, mode=V.MODE_FP64, tol=1e-10, max_outer=80)
    state = ic.random_state(prm, seed=4, vel_scale=0.3)
    state["p"][:] = 0.0
    with V.Solver(prm) as s:
        s.upload_state(**state)
        s.step(1)
        st1 = s.solver_stats()
        p = s.download("p")
    seeded = dict(state, p=p)
    with V.Solver(prm) as s:
        s.upload_state(**seeded)
        s.step(1)
        st2 = s.solver_stats()
    assert st1["rel_initial"] == pytest.approx(1.0)
    assert st2["rel_initial"] < 1e-5 and st2["outer"] < st1["outer"]


@pytest.mark.parametrize("shape", [(64, 64, 64), (60, 48, 40), (30, 20, 18)])
def test_flat_paired_kernels_agree_with_row_kernels(cuda, V, monkeypatch, shape):
    """MIXED levels of even width are smoothed, restricted and prolongated by
    the flat paired kernels (packed FP32 on cell pairs); VOF_MG_PAIRS=0 selects
    the row kernels.  Both solve the same system to the same tolerance: the
    fields agree to the tolerance's level and the cycle counts match within 1."""
    prm = V.default_params(*shape, dt=2e-4, mode=V.MODE_MIXED, tol=1e-10, max_outer=100)
    state = ic.random_state(prm, seed=11, vel_scale=0.5)
    monkeypatch.setenv("VOF_MG_PAIRS", "0")
    rows, st_rows = run_mode(V, prm, state, 1, 3)
    monkeypatch.setenv("VOF_MG_PAIRS", "1")
    flat, st_flat = run_mode(V, prm, state, 1, 3)
    assert all(s["rel_final"] <= 1e-10 for s in st_rows + st_flat)
    for a, b in zip(st_rows, st_flat):
        assert abs(a["outer"] - b["outer"]) <= 1, (st_rows, st_flat)
    for k in STATE:
        assert rel_l2(flat[k], rows[k], interior=(k == "p")) <= 1e-6, (k, rel_l2(flat[k], rows[k], interior=(k == "p")))

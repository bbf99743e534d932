"""CPU checks of the oracle (the restatement of voftrial1.cu's step) and of the
host-side inputs: the reference's arithmetic quirks, step invariants, FP32 vs
FP64 agreement, and the golden vectors produced by the reference's own kernels."""
import json

import numpy as np
import pytest

from conftest import GOLDEN
from vof_b200 import ic

STATE = ("F", "u", "v", "w", "p")


# ---- clamp01f quirks (voftrial1.cu:52-60) -----------------------------------
@pytest.mark.parametrize("x,want", [
    (1e-9, 0.0),
    (0.1234567016, np.float32(0.1234567165)),
    (-1e-9, np.float32(1e-9)),
    (float(np.float32(1) + np.float32(2 ** -23)), np.float32(1 - 2 ** -23)),
    (float(np.float32(0.99999994)), 1.0),
    (0.5, 0.5),
    (2.0, 1.0),
    (-3.0, 0.0),
])
def test_clamp01f_quantisation(orc, x, want):
    assert np.float32(orc.clamp01f(x)) == np.float32(want)


def test_clamp01f_not_idempotent_on_tiny_negatives(orc):
    a = orc.clamp01f(-1e-9)
    assert a > 0 and orc.clamp01f(a) == 0.0


# ---- step invariants ---------------------------------------------------------
def test_oracle_step_invariants(V, orc):
    prm = V.default_params(14, 12, 10, dt=5e-4)
    st = orc.run_f32(prm, ic.random_state(prm, seed=4), 1, 2)
    u, v, w, F = st["u"], st["v"], st["w"], st["F"]
    assert np.all(u[:, :, 1] == 0) and np.all(u[:, :, -1] == 0)
    assert np.all(v[:, 1, :] == 0) and np.all(v[:, -1, :] == 0)
    assert np.all(w[1, :, :] == 0) and np.all(w[-1, :, :] == 0)
    ci = np.clip(np.arange(prm.nx + 2), 1, prm.nx)
    cj = np.clip(np.arange(prm.ny + 2), 1, prm.ny)
    ck = np.clip(np.arange(prm.nz + 2), 1, prm.nz)
    assert np.array_equal(F, F[np.ix_(ck, cj, ci)])
    # pressure ghosts are never written (the reference's apply_bc is dead code)
    p0 = ic.random_state(prm, seed=4)["p"]
    assert np.array_equal(st["p"][0], p0[0]) and np.array_equal(st["p"][:, :, 0], p0[:, :, 0])


def test_sweep_order_rotates_with_istep(V, orc):
    prm = V.default_params(12, 12, 12, dt=1e-3)
    s = ic.random_state(prm, seed=6, vel_scale=2.0)
    outs = [orc.run_f32(prm, s, i, 1)["F"] for i in (1, 2, 3)]
    assert not np.array_equal(outs[0], outs[1]) and not np.array_equal(outs[1], outs[2])
    assert np.array_equal(orc.run_f32(prm, s, 4, 1)["F"], outs[0])  # istep % 3


def test_oracle_threads_do_not_change_bits(V, orc):
    prm = V.default_params(20, 16, 12, dt=5e-4)
    s = ic.random_state(prm, seed=12)
    a = orc.run_f32(prm, s, 1, 3, nthreads=1)
    b = orc.run_f32(prm, s, 1, 3, nthreads=0)
    for k in STATE:
        assert np.array_equal(a[k], b[k])


def test_fp32_vs_fp64_dam_break_32(V, orc):
    prm = V.default_params(32, gy=0.0, gz=-9.81)
    s = ic.rest_state(prm, ic.dam_break(prm))
    a = orc.run_f32(prm, s, 1, 200)
    b = orc.run_f64(prm, s, 1, 200)
    for k in ("F", "u", "v", "w"):
        d = np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k])
        assert d < 1e-4, (k, d)
    v0 = s["F"][1:-1, 1:-1, 1:-1].sum(dtype=np.float64)
    assert abs(b["F"][1:-1, 1:-1, 1:-1].sum() / v0 - 1) < 1e-5
    assert abs(a["F"][1:-1, 1:-1, 1:-1].sum(dtype=np.float64) / v0 - 1) < 1e-5


# ---- golden vectors from the reference's own kernels --------------------------
def golden_cases():
    idx = GOLDEN / "index.json"
    if not idx.exists():
        return []
    return json.loads(idx.read_text())["cases"]


def load_case(V, case):
    data = np.load(GOLDEN / case["file"])
    prm = V.default_params(case["nx"], case["ny"], case["nz"], **case["overrides"])
    inp = {k: data["in_" + k] for k in STATE}
    return prm, inp, data


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c["name"])
def test_oracle_matches_reference_golden(V, orc, case):
    """The FP32 oracle reproduces the reference's -fmad=false kernels bit for bit
    and the default (FMA) build within the case's stated tolerance."""
    prm, inp, data = load_case(V, case)
    out = orc.run_f32(prm, inp, case["istep0"], case["nsteps"])
    for k in STATE:
        nof = data["nofma_" + k]
        assert np.array_equal(out[k], nof), (k, int(np.sum(out[k] != nof)))
    tol = case["fma_rel_l2"]
    for k in STATE:
        ref = data["fma_" + k].astype(np.float64)
        got = out[k].astype(np.float64)
        if k == "p":
            ref = ref[1:-1, 1:-1, 1:-1]
            got = got[1:-1, 1:-1, 1:-1]
            ref, got = ref - ref.mean(), got - got.mean()
        nr = np.linalg.norm(ref)
        d = np.linalg.norm(got - ref) / (nr if nr > 0 else 1.0)
        assert d <= tol, (k, d, tol)


def test_golden_index_present_when_fixtures_exist():
    files = sorted(p.name for p in GOLDEN.glob("*.npz"))
    if files:
        names = {c["file"] for c in golden_cases()} | {c["file"] for c in bc_cases()}
        assert set(files) <= names


# ---- apply_bc (voftrial1.cu:943-956) -------------------------------------
BC = ("u", "v", "w", "F", "p", "rho")


def bc_cases():
    idx = GOLDEN / "apply_bc.json"
    return json.loads(idx.read_text())["cases"] if idx.exists() else []


def bc_closed_form(inp):
    """What set_bc_j, set_bc_i and set_bc_k leave, in one numpy expression per
    field: ghosts of F, p, rho from the clamped interior cell; u, v, w zero on
    their first and last faces, their other ghosts clamped in the two
    tangential directions only."""
    nz2, ny2, nx2 = inp["F"].shape
    ci = np.clip(np.arange(nx2), 1, nx2 - 2)
    cj = np.clip(np.arange(ny2), 1, ny2 - 2)
    ck = np.clip(np.arange(nz2), 1, nz2 - 2)
    out = {k: inp[k][np.ix_(ck, cj, ci)] for k in ("F", "p", "rho")}
    out["u"] = inp["u"][np.ix_(ck, cj, np.arange(nx2))]
    out["u"][:, :, [1, nx2 - 1]] = 0
    out["v"] = inp["v"][np.ix_(ck, np.arange(ny2), ci)]
    out["v"][:, [1, ny2 - 1], :] = 0
    out["w"] = inp["w"][np.ix_(np.arange(nz2), cj, ci)]
    out["w"][[1, nz2 - 1], :, :] = 0
    return out


@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 3, 2), (4, 1, 3), (5, 6, 1), (9, 7, 5)])
def test_apply_bc_oracle_is_the_closed_form(V, orc, shape):
    prm = V.default_params(*shape)
    rng = np.random.default_rng(sum(shape))
    inp = {k: rng.standard_normal(prm.shape).astype(np.float32) for k in BC}
    got = orc.apply_bc(prm, inp)
    want = bc_closed_form(inp)
    for k in BC:
        assert np.array_equal(got[k], want[k]), k
    again = orc.apply_bc(prm, got)  # idempotent
    for k in BC:
        assert np.array_equal(again[k], got[k]), k


@pytest.mark.parametrize("case", bc_cases(), ids=lambda c: c["name"])
def test_apply_bc_oracle_matches_reference_golden(V, orc, case):
    """The oracle's apply_bc reproduces the reference's own kernels bit for bit."""
    data = np.load(GOLDEN / case["file"])
    prm = V.default_params(case["nx"], case["ny"], case["nz"])
    got = orc.apply_bc(prm, {k: data["in_" + k] for k in BC})
    for k in BC:
        assert np.array_equal(got[k], data["out_" + k]), k

"""The host adjoint (oracle/vof_adjoint.cpp) against the forward it reverses.

* The switch-policy forward (Taped) is the forward oracle bit for bit, and its
  replay reproduces the recorded run.
* Transpose test: <dL/dx0, d> from the adjoint equals the dual-number tangent
  dL(x0 + t d)/dt of the FP64 step with the same switch convention, for
  directions in every state field and in the body force (relative 1e-10).
* The tangent against central finite differences of the unfrozen FP64
  forward for the inputs the gradient is taken with respect to (initial
  velocity perturbations on interior faces, body force): relative 1e-4 at
  eps = 1e-7.  (F directions cross the clamps of pure cells, where the map is
  not differentiable, so they are not finite-difference checked.)
"""
import numpy as np
import pytest

from vof_b200 import ic

STATE = ("F", "u", "v", "w", "p")


def dam_state(V, nx, ny, nz, seed=3, amp=1e-2, **kw):
    prm = V.default_params(nx, ny, nz, dt=2e-4, gy=0.0, gz=-9.81, **kw)
    st = ic.rest_state(prm, ic.dam_break(prm))
    rng = np.random.default_rng(seed)
    for k in ("u", "v", "w"):
        st[k] = st[k] + amp * rng.standard_normal(prm.shape)
    return prm, st


def box_of(prm):
    return (0.3 * prm.Lx, 0.6 * prm.Lx, -1e9, 1e9, -1e9, 0.6 * prm.Lz)


def box_loss(prm, F, box):
    nz2, ny2, nx2 = F.shape
    k = np.arange(nz2)[:, None, None]
    j = np.arange(ny2)[None, :, None]
    i = np.arange(nx2)[None, None, :]
    xc, yc, zc = (i - 0.5) * np.float64(prm.dx), (j - 0.5) * np.float64(prm.dy), (k - 0.5) * np.float64(prm.dz)
    m = ((i >= 1) & (i <= nx2 - 2) & (j >= 1) & (j <= ny2 - 2) & (k >= 1) & (k <= nz2 - 2) & (xc > box[0]) &
         (xc < box[1]) & (yc > box[2]) & (yc < box[3]) & (zc > box[4]) & (zc < box[5]))
    return float(np.sum(F[m].astype(np.float64)) * np.float64(prm.dx) * np.float64(prm.dy) * np.float64(prm.dz))


def interior_faces(prm, comp, rng, sigma=1e-3):
    """N(0, sigma^2) on the interior faces of one velocity component, 0 elsewhere."""
    d = np.zeros(prm.shape)
    nz, ny, nx = prm.nz, prm.ny, prm.nx
    lo = {"u": (1, 1, 2), "v": (1, 2, 1), "w": (2, 1, 1)}[comp]  # (k, j, i) first interior face
    d[lo[0]:nz + 1, lo[1]:ny + 1, lo[2]:nx + 1] = sigma * rng.standard_normal(
        (nz + 1 - lo[0], ny + 1 - lo[1], nx + 1 - lo[2]))
    return d


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_taped_forward_is_the_oracle(V, orc, prec):
    prm, st = dam_state(V, 13, 11, 9)
    run = orc.run_f32 if prec == "f32" else orc.run_f64
    for istep0 in (0, 1, 2):
        ref = run(prm, st, istep0, 4)
        tp = orc.SwitchTape(prm, istep0, 4, box_of(prm), prec)
        got, _ = tp.record(st)
        for k in STATE:
            assert np.array_equal(got[k], ref[k]), (k, istep0)
        again, _ = tp.replay(st)
        for k in STATE:
            assert np.array_equal(again[k], ref[k]), (k, istep0)
        tp.close()


@pytest.mark.parametrize("shape,steps,istep0,iters", [
    ((12, 12, 12), 6, 1, 10),
    ((13, 9, 11), 5, 0, 10),
    ((10, 12, 8), 4, 2, 1),
    ((9, 9, 9), 3, 1, 0),
])
def test_adjoint_is_the_transpose_of_the_tangent(V, orc, shape, steps, istep0, iters):
    prm, st = dam_state(V, *shape, jacobi_iters=iters)
    box = box_of(prm)
    A = orc.adjoint(prm, st, istep0, steps, box, "f64")
    assert A["loss"] > 0
    rng = np.random.default_rng(7)
    for comp in STATE:
        d = rng.standard_normal(prm.shape)
        adj = float(np.sum(A["l" + comp] * d))
        L, tl = orc.tangent(prm, st, {comp: d}, istep0, steps, box)
        assert L == pytest.approx(A["loss"], rel=1e-15)
        assert abs(adj - tl) <= 1e-10 * max(abs(tl), 1e-30) + 1e-25, (comp, adj, tl)
    for q in range(3):
        dg = np.zeros(3)
        dg[q] = 1.0
        _, tl = orc.tangent(prm, st, {}, istep0, steps, box, dg=dg)
        assert abs(A["grad_g"][q] - tl) <= 1e-10 * max(abs(tl), 1e-30) + 1e-25, (q, A["grad_g"][q], tl)


def test_tangent_against_finite_differences(V, orc):
    prm, st = dam_state(V, 12, 12, 12)
    box = box_of(prm)
    steps, eps = 6, 1e-7
    rng = np.random.default_rng(4)
    for comp in ("u", "v", "w"):
        d = interior_faces(prm, comp, rng, sigma=1.0)
        _, tl = orc.tangent(prm, st, {comp: d}, 1, steps, box)
        sp, sm = dict(st), dict(st)
        sp[comp] = st[comp] + eps * d
        sm[comp] = st[comp] - eps * d
        fd = (box_loss(prm, orc.run_f64(prm, sp, 1, steps)["F"], box) -
              box_loss(prm, orc.run_f64(prm, sm, 1, steps)["F"], box)) / (2 * eps)
        assert abs(fd - tl) <= 1e-4 * abs(tl), (comp, fd, tl)
    for q, name in enumerate(("gx", "gy", "gz")):
        dg = np.zeros(3)
        dg[q] = 1.0
        _, tl = orc.tangent(prm, st, {}, 1, steps, box, dg=dg)
        h = 1e-4
        pp = V.default_params(12, 12, 12, dt=2e-4, gy=0.0, gz=-9.81)
        pm = V.default_params(12, 12, 12, dt=2e-4, gy=0.0, gz=-9.81)
        setattr(pp, name, getattr(prm, name) + h)
        setattr(pm, name, getattr(prm, name) - h)
        # the parameters are float32: divide by the step they actually took
        fd = (box_loss(prm, orc.run_f64(pp, st, 1, steps)["F"], box) -
              box_loss(prm, orc.run_f64(pm, st, 1, steps)["F"], box)) / (getattr(pp, name) - getattr(pm, name))
        assert abs(fd - tl) <= 1e-4 * abs(tl), (name, fd, tl)


def test_adjoint_against_finite_differences_along_sixteen_directions(V, orc):
    """The form of the 64^3 adjoint gradient check at a CPU size: the initial
    velocity perturbed by N(0, (1e-3 m/s)^2) on interior faces, 16 seeded
    directions (seed 4) in the joint u, v, w interior-face space with the same
    std, central differences with eps = 1e-4 (1e-7 m/s per face) of the
    unfrozen FP64 forward against the FP64 adjoint's <dL/du, d>: relative
    1e-4."""
    prm, st = dam_state(V, 12, 12, 12, amp=1e-3)
    box = box_of(prm)
    steps, eps = 6, 1e-4
    A = orc.adjoint(prm, st, 1, steps, box, "f64")
    assert A["loss"] > 0
    rng = np.random.default_rng(4)
    for n in range(16):
        d = {c: interior_faces(prm, c, rng, sigma=1e-3) for c in ("u", "v", "w")}
        adj = sum(float(np.sum(A["l" + c] * d[c])) for c in d)
        sp = {k: (st[k] + eps * d[k] if k in d else st[k]) for k in STATE}
        sm = {k: (st[k] - eps * d[k] if k in d else st[k]) for k in STATE}
        fd = (box_loss(prm, orc.run_f64(prm, sp, 1, steps)["F"], box) -
              box_loss(prm, orc.run_f64(prm, sm, 1, steps)["F"], box)) / (2 * eps)
        rel = abs(fd - adj) / abs(adj)
        assert rel <= 1e-4, (n, fd, adj, rel)


def test_fp32_and_fp64_trajectories_give_close_gradients(V, orc):
    prm, st = dam_state(V, 12, 12, 12)
    box = box_of(prm)
    a = orc.adjoint(prm, st, 1, 6, box, "f32")
    b = orc.adjoint(prm, st, 1, 6, box, "f64")
    for k in ("lu", "lv", "lw"):
        assert np.linalg.norm(a[k] - b[k]) <= 1e-3 * np.linalg.norm(b[k]), k
    assert np.allclose(a["grad_g"], b["grad_g"], rtol=1e-3)


def test_convergent_solve_adjoint_against_finite_differences(V, orc):
    """With the pressure solved to 1e-13 every step (the FP64 oracle of the
    MIXED / FP64 modes), the adjoint's solve step (mean-free solve of A mu =
    lp - mean(lp)) gives dL/du0, dL/dv0, dL/dw0 that match central
    differences of that forward; the state pressure gets no adjoint."""
    prm, st = dam_state(V, 12, 12, 12)
    box = box_of(prm)
    steps, eps = 6, 1e-7
    A = orc.adjoint(prm, st, 1, steps, box, "f64", conv_tol=1e-13)
    assert np.count_nonzero(A["lp"]) == 0
    rng = np.random.default_rng(11)
    for comp in ("u", "v", "w"):
        d = interior_faces(prm, comp, rng, sigma=1.0)
        adj = float(np.sum(A["l" + comp] * d))
        sp, sm = dict(st), dict(st)
        sp[comp] = st[comp] + eps * d
        sm[comp] = st[comp] - eps * d
        fd = (box_loss(prm, orc.run_conv_f64(prm, sp, 1, steps, tol=1e-13)["F"], box) -
              box_loss(prm, orc.run_conv_f64(prm, sm, 1, steps, tol=1e-13)["F"], box)) / (2 * eps)
        assert abs(fd - adj) <= 1e-4 * abs(fd), (comp, fd, adj)

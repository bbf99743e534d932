"""Parity of the CUDA step (through the C-ABI) with the oracle and the reference.

Tolerances:
  * vs the FP32 CPU restatement (oracle, no FMA): bit-identical (np.array_equal,
    so +0 == -0) for F, u, v, w, p, u*, v*, w* and rhs.
  * vs the reference's kernels built with -fmad=false: bit-identical.
  * vs the reference's kernels built with nvcc defaults (FMA contraction):
    max-abs and relative-L2 bounds stated in each test.
  * vs the FP64 oracle: relative-L2 bounds stated in each test.
"""
import numpy as np
import pytest

from vof_b200 import ic

pytestmark = pytest.mark.gpu

STATE = ("F", "u", "v", "w", "p")


def run_gpu(V, prm, state, istep0, nsteps, use_graph=False, extras=False):
    with V.Solver(prm) as s:
        s.upload_state(**state)
        if use_graph:
            s.run(istep0, nsteps)
        else:
            for t in range(nsteps):
                s.step(istep0 + t)
        out = s.state()
        if extras:
            for k in ("ustar", "vstar", "wstar", "rhs"):
                out[k] = s.download(k)
    return out


def assert_bitwise(got, want, keys, ctx=""):
    msgs = []
    for k in keys:
        g, w = got[k], want[k]
        if not np.array_equal(g, w):
            bad = np.argwhere(g != w)
            kk, jj, ii = bad[0]
            msgs.append(f"field {k}: {len(bad)} cells differ; first (k,j,i)=({kk},{jj},{ii}) "
                        f"got {g[kk, jj, ii]!r} want {w[kk, jj, ii]!r}")
    if msgs:
        raise AssertionError(f"{ctx}: " + " | ".join(msgs))


def rel_l2(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


CASES = [
    # (nx, ny, nz, seed, dt, vel_scale)
    (16, 12, 10, 1, 1e-3, 1.0),
    (17, 9, 13, 2, 5e-4, 2.0),
    (32, 32, 32, 3, 4e-6, 1.0),
    (1, 3, 2, 4, 1e-3, 1.0),
    (40, 33, 21, 5, 2e-4, 3.0),
]


@pytest.mark.parametrize("nx,ny,nz,seed,dt,vs", CASES)
def test_random_state_bitwise_vs_oracle(cuda, V, orc, nx, ny, nz, seed, dt, vs):
    prm = V.default_params(nx, ny, nz, dt=dt, gy=0.0, gz=-9.81)
    state = ic.random_state(prm, seed=seed, vel_scale=vs)
    got = run_gpu(V, prm, state, 1, 3, extras=True)  # istep 1,2,3: all sweep orders
    want = orc.run_f32(prm, state, 1, 3, extras=True)
    assert_bitwise(got, want, STATE + ("ustar", "vstar", "wstar", "rhs"), f"{nx}x{ny}x{nz}")


@pytest.mark.parametrize("env", [{"VOF_JACOBI": "pairs2"}, {"VOF_JACOBI": "ring"}, {"VOF_JACOBI": "tb"},
                                 {"VOF_JACOBI": "col"}, {"VOF_JACOBI": "ring", "VOF_JACOBI_KCHUNK": "1"},
                                 {"VOF_JACOBI": "ring", "VOF_JACOBI_KCHUNK": "3"},
                                 {"VOF_JACOBI": "pairs", "VOF_JACOBI_KCHUNK": "1"},
                                 {"VOF_JACOBI": "pairs", "VOF_JACOBI_KCHUNK": "5"},
                                 {"VOF_JACOBI": "tb1"}, {"VOF_JACOBI": "pairs"}, {"VOF_CORRECT": "1"}, {"VOF_RHS": "1"},
                                 {"VOF_PREDICT": "1"}, {"VOF_JACOBI": "quad"},
                                 {"VOF_JACOBI": "quad", "VOF_JACOBI_KCHUNK": "1"},
                                 {"VOF_JACOBI": "quad", "VOF_JACOBI_KCHUNK": "21"},
                                 {"VOF_JACOBI": "bulk"}, {"VOF_JACOBI": "bulk", "VOF_JACOBI_KCHUNK": "1"},
                                 {"VOF_JACOBI": "bulk", "VOF_JACOBI_KCHUNK": "7"},
                                 {"VOF_JACOBI": "bulk", "VOF_JACOBI_KCHUNK": "21"},
                                 {"VOF_JACOBI": "peel", "VOF_JP_UNROLL": "1"},
                                 {"VOF_JACOBI": "peel", "VOF_JP_UNROLL": "1", "VOF_JP_MINB": "4"},
                                 {"VOF_JACOBI": "peel", "VOF_JP_UNROLL": "2"},
                                 {"VOF_JACOBI": "peel", "VOF_JP_UNROLL": "2", "VOF_JP_MINB": "4"},
                                 {"VOF_JACOBI": "peel", "VOF_JP_UNROLL": "4"},
                                 {"VOF_JACOBI": "peel", "VOF_JP_UNROLL": "4", "VOF_JP_MINB": "4"},
                                 {"VOF_JACOBI": "peel", "VOF_JACOBI_KCHUNK": "1"},
                                 {"VOF_JACOBI": "peel", "VOF_JACOBI_KCHUNK": "2"},
                                 {"VOF_JACOBI": "peel", "VOF_JP_UNROLL": "4", "VOF_JACOBI_KCHUNK": "7"},
                                 {"VOF_JACOBI": "peel", "VOF_JP_UNROLL": "4", "VOF_JACOBI_KCHUNK": "21"},
                                 {"VOF_JACOBI_ALT": "0"}, {"VOF_JACOBI_ALT": "1", "VOF_JACOBI_KCHUNK": "1"},
                                 {"VOF_JACOBI_ALT": "1", "VOF_JACOBI_KCHUNK": "2"},
                                 {"VOF_JACOBI_ALT": "1", "VOF_JACOBI_KCHUNK": "7"}])
def test_jacobi_kernel_choices_give_the_same_bits(cuda, V, orc, tmp_path, env):
    """The kernels a process may select give the oracle's bits.  The defaults
    (the peeled paired Jacobi sweep, marching z down on every second sweep at
    these sizes, and the size-chosen predictor, rhs and correction kernels)
    run in every other test; here the other Jacobi kernels: the paired sweep,
    the peeled form at other unrolls and register caps and with every sweep
    marching up, the downward march over short z chunks, the four-cell sweep,
    the two-sweep paired kernel, the cp.async ring, the bulk-copy ring, the
    TMA-blocked kernels, the one-cell streaming sweep, and z chunks of
    several of them; and the one-cell predictor, rhs and correction.  The
    choice is read once per process, so each runs in a child process."""
    import os
    import subprocess
    import sys
    from pathlib import Path

    prm = V.default_params(40, 33, 21, dt=2e-4, gy=0.0, gz=-9.81)
    state = ic.random_state(prm, seed=5, vel_scale=3.0)
    np.savez(tmp_path / "in.npz", **state)
    root = Path(__file__).resolve().parent.parent
    code = (
        "import sys, numpy as np\n"
        f"sys.path.insert(0, {str(root / 'cuda-lbm-ibm-fvm_b200')!r})\n"
        "import vof_b200 as V\n"
        "prm = V.default_params(40, 33, 21, dt=2e-4, gy=0.0, gz=-9.81)\n"
        f"st = dict(np.load({str(tmp_path / 'in.npz')!r}))\n"
        "with V.Solver(prm) as s:\n"
        "    s.upload_state(**st)\n"
        "    for t in range(3):\n"
        "        s.step(1 + t)\n"
        f"    np.savez({str(tmp_path / 'out.npz')!r}, **s.state())\n")
    subprocess.run([sys.executable, "-c", code], env={**os.environ, **env}, check=True, timeout=600)
    got = dict(np.load(tmp_path / "out.npz"))
    want = orc.run_f32(prm, state, 1, 3)
    assert_bitwise(got, want, STATE, str(env))


@pytest.mark.parametrize("shape", [(1, 3, 2), (6, 5, 4), (17, 9, 13), (40, 33, 21), (64, 7, 5)])
def test_four_cell_kernels_on_odd_grids(cuda, V, orc, tmp_path, shape):
    """The four-cell right-hand side and correction (k_rhs4, k_correct4: the
    defaults from about 128^3 up) and the four-cell Jacobi sweep forced on
    small and odd grids -- rows that end inside a quad, warps that span rows,
    every edge and corner cell -- give the oracle's bits (child process: the
    switches are read once)."""
    import os
    import subprocess
    import sys
    from pathlib import Path

    prm = V.default_params(*shape, dt=2e-4, gy=0.0, gz=-9.81)
    state = ic.random_state(prm, seed=sum(shape), vel_scale=3.0)
    np.savez(tmp_path / "in.npz", **state)
    root = Path(__file__).resolve().parent.parent
    code = (
        "import sys, numpy as np\n"
        f"sys.path.insert(0, {str(root / 'cuda-lbm-ibm-fvm_b200')!r})\n"
        "import vof_b200 as V\n"
        f"prm = V.default_params(*{shape!r}, dt=2e-4, gy=0.0, gz=-9.81)\n"
        f"st = dict(np.load({str(tmp_path / 'in.npz')!r}))\n"
        "with V.Solver(prm) as s:\n"
        "    s.upload_state(**st)\n"
        "    for t in range(3):\n"
        "        s.step(1 + t)\n"
        "    out = s.state()\n"
        "    for k in ('ustar', 'vstar', 'wstar', 'rhs'):\n"
        "        out[k] = s.download(k)\n"
        f"    np.savez({str(tmp_path / 'out.npz')!r}, **out)\n")
    env = {**os.environ, "VOF_CORRECT": "4", "VOF_RHS": "4", "VOF_JACOBI": "quad"}
    subprocess.run([sys.executable, "-c", code], env=env, check=True, timeout=600)
    got = dict(np.load(tmp_path / "out.npz"))
    want = orc.run_f32(prm, state, 1, 3, extras=True)
    assert_bitwise(got, want, STATE + ("ustar", "vstar", "wstar", "rhs"), f"four-cell {shape}")


@pytest.mark.parametrize("shape,seed,vfrac", [((40, 36, 34), 41, 0.45), ((130, 17, 19), 42, 0.3),
                                              ((17, 130, 9), 43, 0.6), ((9, 11, 140), 44, 0.45),
                                              ((250, 12, 10), 45, 0.2)])
def test_sparse_interface_bitwise_vs_oracle(cuda, V, orc, shape, seed, vfrac):
    """F exactly 0 over irregular regions (runs of every length along every
    axis, lines longer than one x window of the x sweep, a gas slab covering
    whole x windows) next to mixed cells, velocities of both signs with a
    standard deviation of vfrac times the sweeps' quiet-window velocity bound
    (0.49 dx / dt), so some exceed it: the sweeps' zero-window shortcuts
    against the full arithmetic of the oracle, every sweep order, bit for bit."""
    prm = V.default_params(*shape, dt=1e-3, gy=0.0, gz=-9.81)
    vq = 0.49 * float(prm.dx) / float(prm.dt)
    st = ic.random_state(prm, seed=seed, vel_scale=vfrac * vq)
    nz, ny, nx = prm.shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ph = ic.uniform(seed, 6, 0.0, 2 * np.pi)
    wave = (np.sin(0.37 * i + ph[0]) * np.sin(0.23 * j + ph[1]) * np.sin(0.31 * k + ph[2]) +
            0.5 * np.sin(0.11 * (i + j + k) + ph[3]))
    st["F"] = np.where(wave < 0.15, 0.0, st["F"]).astype(np.float32)
    st["F"][:, :, nx // 2:] = 0.0  # gas slab
    got = run_gpu(V, prm, st, 1, 3, extras=True)
    want = orc.run_f32(prm, st, 1, 3, extras=True)
    assert_bitwise(got, want, STATE + ("ustar", "vstar", "wstar", "rhs"), f"sparse {shape}")


@pytest.mark.parametrize("istep", [1, 2, 3])
def test_each_sweep_order_bitwise(cuda, V, orc, istep):
    prm = V.default_params(20, 18, 16, dt=5e-4)
    state = ic.random_state(prm, seed=100 + istep, vel_scale=1.5)
    got = run_gpu(V, prm, state, istep, 1)
    want = orc.run_f32(prm, state, istep, 1)
    assert_bitwise(got, want, STATE, f"istep={istep}")


@pytest.mark.parametrize("iters", [0, 1, 7, 10])
def test_jacobi_iteration_counts(cuda, V, orc, iters):
    prm = V.default_params(12, 14, 10, dt=1e-3, jacobi_iters=iters)
    state = ic.random_state(prm, seed=7, vel_scale=1.0)
    got = run_gpu(V, prm, state, 1, 4)
    want = orc.run_f32(prm, state, 1, 4)
    assert_bitwise(got, want, STATE, f"iters={iters}")
    got_g = run_gpu(V, prm, state, 1, 4, use_graph=True)
    assert_bitwise(got_g, want, STATE, f"graph iters={iters}")


def test_graph_run_equals_steps(cuda, V):
    prm = V.default_params(24, 24, 24, dt=2e-4)
    state = ic.random_state(prm, seed=9, vel_scale=1.0)
    a = run_gpu(V, prm, state, 5, 7, use_graph=False)
    b = run_gpu(V, prm, state, 5, 7, use_graph=True)
    assert_bitwise(a, b, STATE, "graph vs step")


def test_dam_break_32_200_steps(cuda, V, orc):
    """The 32^3 dam break of 200 steps (gravity -9.81 along z)."""
    prm = V.default_params(32, gy=0.0, gz=-9.81)
    state = ic.rest_state(prm, ic.dam_break(prm))
    got = run_gpu(V, prm, state, 1, 200, use_graph=True)
    want = orc.run_f32(prm, state, 1, 200)
    assert_bitwise(got, want, STATE, "32^3 x 200")
    ref64 = orc.run_f64(prm, state, 1, 200)
    # FP32 vs FP64 after 200 steps (measured ~1e-5; bound 1e-4 rel-L2, p modulo its mean)
    for k in ("F", "u", "v", "w"):
        assert rel_l2(got[k], ref64[k]) < 1e-4, k
    pm = got["p"][1:-1, 1:-1, 1:-1].astype(np.float64)
    qm = ref64["p"][1:-1, 1:-1, 1:-1]
    assert rel_l2(pm - pm.mean(), qm - qm.mean()) < 1e-4
    vol0 = state["F"][1:-1, 1:-1, 1:-1].sum(dtype=np.float64)
    vol1 = got["F"][1:-1, 1:-1, 1:-1].sum(dtype=np.float64)
    assert abs(vol1 / vol0 - 1.0) < 1e-5  # measured -5.4e-7 in FP32


def test_invariants_after_step(cuda, V):
    prm = V.default_params(18, 16, 14, dt=5e-4)
    state = ic.random_state(prm, seed=21, vel_scale=1.0)
    got = run_gpu(V, prm, state, 2, 1)
    u, v, w, F = got["u"], got["v"], got["w"], got["F"]
    # wall-normal face velocities are exactly 0 (voftrial1.cu:980-986, 1012-1018, 1044-1050)
    assert np.all(u[:, :, 1] == 0) and np.all(u[:, :, -1] == 0)
    assert np.all(v[:, 1, :] == 0) and np.all(v[:, -1, :] == 0)
    assert np.all(w[1, :, :] == 0) and np.all(w[-1, :, :] == 0)
    # F ghosts equal the clamped interior index (apply_bc_F composition)
    ci = np.clip(np.arange(prm.nx + 2), 1, prm.nx)
    cj = np.clip(np.arange(prm.ny + 2), 1, prm.ny)
    ck = np.clip(np.arange(prm.nz + 2), 1, prm.nz)
    assert np.array_equal(F, F[np.ix_(ck, cj, ci)])
    assert F.min() >= -1e-6 and F.max() <= 1.0


def test_reductions_match_numpy(cuda, V):
    prm = V.default_params(30, 26, 22, dt=5e-4)
    state = ic.random_state(prm, seed=31, vel_scale=1.0)
    with V.Solver(prm) as s:
        s.upload_state(**state)
        s.step(1)
        st = s.state()
        rhs = s.download("rhs").astype(np.float64)
        red = {k: s.reduce(k) for k in V.REDUCTIONS}
    F = st["F"][1:-1, 1:-1, 1:-1].astype(np.float64)
    vol = F.sum() * float(prm.dx) * float(prm.dy) * float(prm.dz)
    assert red["volume"] == pytest.approx(vol, rel=1e-12)
    assert red["f_min"] == F.min() and red["f_max"] == F.max()
    u, v, w = (st[k].astype(np.float64) for k in "uvw")
    div = ((u[1:-1, 1:-1, 2:] - u[1:-1, 1:-1, 1:-1]) * float(prm.dxi)
           + (v[1:-1, 2:, 1:-1] - v[1:-1, 1:-1, 1:-1]) * float(prm.dyi)
           + (w[2:, 1:-1, 1:-1] - w[1:-1, 1:-1, 1:-1]) * float(prm.dzi))
    assert red["div_l2"] == pytest.approx(np.sqrt((div ** 2).sum()), rel=1e-10)
    assert red["div_max"] == pytest.approx(np.abs(div).max(), rel=1e-12)
    # residual of the pressure system with the mean-free rhs
    p = st["p"].astype(np.float64)
    b = rhs[1:-1, 1:-1, 1:-1] - rhs[1:-1, 1:-1, 1:-1].mean()
    Ap = np.zeros_like(b)
    c = p[1:-1, 1:-1, 1:-1]
    cx, cy, cz = float(prm.dxi) ** 2, float(prm.dyi) ** 2, float(prm.dzi) ** 2
    Ap[:, :, :-1] += cx * (p[1:-1, 1:-1, 2:-1] - c[:, :, :-1])
    Ap[:, :, 1:] += cx * (p[1:-1, 1:-1, 1:-2] - c[:, :, 1:])
    Ap[:, :-1, :] += cy * (p[1:-1, 2:-1, 1:-1] - c[:, :-1, :])
    Ap[:, 1:, :] += cy * (p[1:-1, 1:-2, 1:-1] - c[:, 1:, :])
    Ap[:-1, :, :] += cz * (p[2:-1, 1:-1, 1:-1] - c[:-1, :, :])
    Ap[1:, :, :] += cz * (p[1:-2, 1:-1, 1:-1] - c[1:, :, :])
    want = np.linalg.norm(b - Ap) / np.linalg.norm(b)
    assert red["pres_resid"] == pytest.approx(want, rel=1e-9)
    assert red["nonfinite"] == 0.0


def test_reductions_deterministic(cuda, V):
    prm = V.default_params(64, 48, 40, dt=5e-4)
    state = ic.random_state(prm, seed=41)
    with V.Solver(prm) as s:
        s.upload_state(**state)
        s.step(1)
        a = [s.reduce(k) for k in V.REDUCTIONS]
        b = [s.reduce(k) for k in V.REDUCTIONS]
    assert a == b


def test_async_reductions_into_mapped_and_pageable_memory(cuda, V):
    """vof_reduce_async into pinned (mapped) memory -- one kernel writes the
    value itself -- and into pageable memory -- a copy follows: the same bits
    as the blocking call, call after call (the completion counter resets)."""
    import torch

    prm = V.default_params(30, 26, 22, dt=5e-4)
    state = ic.random_state(prm, seed=32, vel_scale=1.0)
    names = ("volume", "f_min", "f_max", "div_l2")
    pinned = torch.zeros(4 * len(names), dtype=torch.float64).pin_memory()
    pageable = np.zeros(4 * len(names), dtype=np.float64)
    with V.Solver(prm) as s:
        s.upload_state(**state)
        s.step(1)
        want = [s.reduce(k) for k in names]
        for rep in range(4):
            for q, k in enumerate(names):
                s.reduce_async(k, pinned.data_ptr() + 8 * (rep * len(names) + q))
                s.reduce_async(k, pageable.ctypes.data + 8 * (rep * len(names) + q))
        s.sync()
    got_p = pinned.numpy().reshape(4, len(names))
    got_h = pageable.reshape(4, len(names))
    for rep in range(4):
        assert list(got_p[rep]) == want and list(got_h[rep]) == want, (rep, got_p[rep], got_h[rep], want)


@pytest.mark.parametrize("env", [{}, {"VOF_JACOBI_ALT": "0"}, {"VOF_JACOBI": "pairs"}])
def test_jacobi_ieee_division_cells(cuda, V, orc, tmp_path, env):
    """Pressures near 1e31 give Jacobi quotients above 2^96, outside the fast
    division's range: those cells take the IEEE division.  The pressure after
    one step is the sweeps' output and must be the oracle's bit for bit; the
    other fields (the correction and the sweeps then see huge gradients) must
    agree wherever they are not NaN and be NaN at the same cells."""
    import os
    import subprocess
    import sys
    from pathlib import Path

    shape = (12, 10, 9)
    prm = V.default_params(*shape, dt=2e-4, gy=0.0, gz=-9.81)
    state = ic.random_state(prm, seed=21, vel_scale=1.0)
    rng = np.random.default_rng(21)
    p = state["p"]
    idx = tuple(rng.integers(1, n + 1, 40) for n in (shape[2], shape[1], shape[0]))
    p[idx] = (rng.standard_normal(40) * 1e31).astype(np.float32)
    p[2, 3, 4], p[5, 5, 5], p[7, 1, 11] = 3.0e33, -2.0e33, 1.5e32
    np.savez(tmp_path / "in.npz", **state)
    root = Path(__file__).resolve().parent.parent
    code = (
        "import sys, numpy as np\n"
        f"sys.path.insert(0, {str(root / 'cuda-lbm-ibm-fvm_b200')!r})\n"
        "import vof_b200 as V\n"
        f"prm = V.default_params(*{shape!r}, dt=2e-4, gy=0.0, gz=-9.81)\n"
        f"st = dict(np.load({str(tmp_path / 'in.npz')!r}))\n"
        "with V.Solver(prm) as s:\n"
        "    s.upload_state(**st)\n"
        "    s.step(1)\n"
        f"    np.savez({str(tmp_path / 'out.npz')!r}, **s.state())\n")
    subprocess.run([sys.executable, "-c", code], env={**os.environ, **env}, check=True, timeout=600)
    got = dict(np.load(tmp_path / "out.npz"))
    want = orc.run_f32(prm, state, 1, 1)
    assert np.isfinite(want["p"]).all() and np.abs(want["p"]).max() > 1e24  # still far outside the fast range's reach
    assert_bitwise(got, want, ("p",), f"pressure {env}")
    for k in ("F", "u", "v", "w"):
        gn, wn = np.isnan(got[k]), np.isnan(want[k])
        assert np.array_equal(gn, wn), (k, int((gn != wn).sum()))
        g, w = got[k].copy(), want[k].copy()
        g[gn] = 0.0
        w[wn] = 0.0
        assert_bitwise({k: g}, {k: w}, (k,), f"{k} {env}")


def test_nonfinite_watchdog(cuda, V):
    prm = V.default_params(10, 10, 10)
    state = ic.random_state(prm, seed=3)
    state["u"][3, 4, 5] = np.nan
    state["F"][2, 2, 2] = np.inf
    with V.Solver(prm) as s:
        s.upload_state(**state)
        assert s.reduce("nonfinite") == 2.0


def test_upload_download_roundtrip_and_device_pointers(cuda, V):
    import torch

    prm = V.default_params(13, 11, 9)
    state = ic.random_state(prm, seed=5)
    with V.Solver(prm) as s:
        for k in STATE:
            s.upload(k, state[k])
        for k in STATE:
            assert np.array_equal(s.download(k), state[k])
        t = torch.from_numpy(state["w"] * 2).cuda()
        s.upload("w", device_ptr=t.data_ptr())
        o = torch.zeros_like(t)
        s.download_device("w", o.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(o, t)


def test_host_copies_pinned_pageable_and_full_size(cuda, V):
    """Host uploads and downloads go whole through the staging buffer and are
    repacked on the device: pageable and pinned memory, a grid whose row
    pitch is not a multiple of 16 bytes, and 200^3, round trip exactly; the
    context's other fields are untouched by a field's copy."""
    import torch

    for dims in ((13, 11, 9), (200, 200, 200)):
        prm = V.default_params(*dims)
        state = ic.random_state(prm, seed=7) if dims[0] < 100 else {
            k: (np.arange(prm.nTot, dtype=np.float32).reshape(prm.shape) * (q + 1)) for q, k in enumerate(STATE)}
        with V.Solver(prm) as s:
            pinned = {k: torch.from_numpy(state[k]).pin_memory() for k in STATE}
            for k in STATE:
                s._check(s._lib.vof_upload(s._ctx, V.FIELDS[k], pinned[k].data_ptr(), 0), "vof_upload")
            s.sync()
            for k in STATE:
                assert np.array_equal(s.download(k), state[k]), (dims, k)
                out = torch.empty(prm.shape, dtype=torch.float32).pin_memory()
                s._check(s._lib.vof_download(s._ctx, V.FIELDS[k], out.data_ptr(), 0), "vof_download")
                assert np.array_equal(out.numpy(), state[k]), (dims, k, "pinned")
            s.upload("u", state["v"])  # pageable
            assert np.array_equal(s.download("u"), state["v"])
            assert np.array_equal(s.download("w"), state["w"])


def test_bounded_wait_timeout_is_reported_and_cleared(cuda, V, orc):
    """A device-side wait that runs out (vof_debug_wait_timeout: an mbarrier
    armed for copy bytes that never come, polled a few times by the TMA
    kernels' bounded wait) sets the context's status word: vof_sync returns
    VOF_E_TIMEOUT once and clears it, for every limit; vof_reduce reports it
    too; the context keeps working (the next steps are still bit-identical
    to the oracle)."""
    prm = V.default_params(12, 10, 8, dt=5e-4)
    state = ic.random_state(prm, seed=21)
    lib = V.lib()
    with V.Solver(prm) as s:
        s.upload_state(**state)
        assert lib.vof_sync(s._ctx) == V.OK
        for limit in (0, 1, 1024):
            assert lib.vof_debug_wait_timeout(s._ctx, limit) == V.OK
            assert lib.vof_sync(s._ctx) == V.E_TIMEOUT, limit
            assert lib.vof_sync(s._ctx) == V.OK, limit  # cleared
        assert lib.vof_debug_wait_timeout(s._ctx, 4) == V.OK
        with pytest.raises(V.VofError) as e:
            s.reduce("volume")  # vof_reduce waits through vof_sync
        assert e.value.status == V.E_TIMEOUT
        s.run(1, 2)
        assert lib.vof_sync(s._ctx) == V.OK
        got = s.state()
    assert lib.vof_debug_wait_timeout(None, 1) == V.E_INVALID
    want = orc.run_f32(prm, state, 1, 2)
    assert_bitwise(got, want, STATE, "after timeouts")


def test_user_stream(cuda, V, orc):
    import torch

    prm = V.default_params(16, 16, 16, dt=5e-4)
    state = ic.random_state(prm, seed=8)
    st = torch.cuda.Stream()
    with V.Solver(prm, stream=st.cuda_stream) as s:
        s.upload_state(**state)
        s.run(1, 3)
        s.sync()
        got = s.state()
    want = orc.run_f32(prm, state, 1, 3)
    assert_bitwise(got, want, STATE, "user stream")


def test_argument_errors(cuda, V):
    prm = V.default_params(8, 8, 8)
    with V.Solver(prm) as s:
        with pytest.raises(V.VofError) as e:
            s._check(s._lib.vof_upload(s._ctx, 99, None, 0), "upload")
        assert e.value.status == V.E_INVALID
        assert s._lib.vof_reduce(s._ctx, 99, None) == V.E_INVALID
        assert s._lib.vof_run(s._ctx, 1, -1) == V.E_INVALID


# ---- golden vectors produced by the reference's own kernels -----------------
def _golden_cases():
    import json

    from conftest import GOLDEN

    idx = GOLDEN / "index.json"
    return json.loads(idx.read_text())["cases"] if idx.exists() else []


@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: c["name"])
def test_golden_vectors(cuda, V, case):
    """CUDA path vs the stored outputs of voftrial1.cu's kernels: bit-identical
    to the -fmad=false build, within the case's stated rel-L2 of the FMA build."""
    from conftest import GOLDEN

    data = np.load(GOLDEN / case["file"])
    prm = V.default_params(case["nx"], case["ny"], case["nz"], **case["overrides"])
    inp = {k: data["in_" + k] for k in STATE}
    got = run_gpu(V, prm, inp, case["istep0"], case["nsteps"], use_graph=True)
    assert_bitwise(got, {k: data["nofma_" + k] for k in STATE}, STATE, case["name"])
    for k in STATE:
        ref = data["fma_" + k].astype(np.float64)
        g = got[k].astype(np.float64)
        if k == "p":
            ref, g = ref[1:-1, 1:-1, 1:-1], g[1:-1, 1:-1, 1:-1]
            ref, g = ref - ref.mean(), g - g.mean()
        assert rel_l2(g, ref) <= case["fma_rel_l2"], k


# ---- the reference's own kernels (oracle/_ref) -------------------------------
def _need_ref(orc, variant):
    if not orc.ref_available(variant):
        pytest.skip(f"reference harness {variant} not built (needs the reference source at build time)")


@pytest.mark.parametrize("nx,ny,nz,seed,dt,vs", CASES[:3])
def test_bitwise_vs_reference_kernels_nofma(cuda, V, orc, nx, ny, nz, seed, dt, vs):
    _need_ref(orc, "nofma")
    prm = V.default_params(nx, ny, nz, dt=dt, gy=0.0, gz=-9.81)
    state = ic.random_state(prm, seed=seed, vel_scale=vs)
    ref = orc.ref_run(prm, state, 1, 3, variant="nofma", extras=True)
    got = run_gpu(V, prm, state, 1, 3, extras=True)
    assert_bitwise(got, ref, STATE + ("ustar", "vstar", "wstar"), "vs reference -fmad=false")


def test_dam_break_vs_reference_kernels(cuda, V, orc):
    """32^3 dam break, 200 steps, against the reference's default (FMA) build.
    Bounds: rel-L2 <= 1e-5 for F, u, v, w and for p modulo its mean;
    max-abs |dF| <= 1e-4."""
    _need_ref(orc, "sm100a")
    prm = V.default_params(32, gy=0.0, gz=-9.81)
    state = ic.rest_state(prm, ic.dam_break(prm))
    ref = orc.ref_run(prm, state, 1, 200, variant="sm100a")
    got = run_gpu(V, prm, state, 1, 200, use_graph=True)
    for k in ("F", "u", "v", "w"):
        assert rel_l2(got[k], ref[k]) <= 1e-5, (k, rel_l2(got[k], ref[k]))
    assert np.abs(got["F"].astype(np.float64) - ref["F"]).max() <= 1e-4
    pm = got["p"][1:-1, 1:-1, 1:-1].astype(np.float64)
    qm = ref["p"][1:-1, 1:-1, 1:-1].astype(np.float64)
    assert rel_l2(pm - pm.mean(), qm - qm.mean()) <= 1e-5
    if orc.ref_available("nofma"):
        ref_nf = orc.ref_run(prm, state, 1, 200, variant="nofma")
        assert_bitwise(got, ref_nf, STATE, "32^3 x 200 vs reference -fmad=false")


def test_full_size_dam_break_vs_reference_kernels(cuda, V, orc):
    """The benchmark workload at its full size: 200^3 dam break with the
    noisy interface (splitmix64 seed 1), 30 steps (every sweep order ten
    times), graph-captured.  Bit-identical to the reference's kernels built
    with -fmad=false; against its default (FMA) build rel-L2 <= 1e-5 for F,
    u, v, w and p modulo its mean, max-abs |dF| <= 1e-4, and the total liquid
    volume (FP64 sum of F) within 1e-7 relative."""
    _need_ref(orc, "nofma")
    prm = V.default_params(200, gy=0.0, gz=-9.81)
    state = ic.rest_state(prm, ic.dam_break(prm, height=ic.noisy_height(prm, seed=1)))
    got = run_gpu(V, prm, state, 1, 30, use_graph=True)
    ref_nf = orc.ref_run(prm, state, 1, 30, variant="nofma")
    assert_bitwise(got, ref_nf, STATE, "200^3 x 30 vs reference -fmad=false")
    if orc.ref_available("sm100a"):
        ref = orc.ref_run(prm, state, 1, 30, variant="sm100a")
        for k in ("F", "u", "v", "w"):
            assert rel_l2(got[k], ref[k]) <= 1e-5, (k, rel_l2(got[k], ref[k]))
        assert np.abs(got["F"].astype(np.float64) - ref["F"]).max() <= 1e-4
        pm = got["p"][1:-1, 1:-1, 1:-1].astype(np.float64)
        qm = ref["p"][1:-1, 1:-1, 1:-1].astype(np.float64)
        assert rel_l2(pm - pm.mean(), qm - qm.mean()) <= 1e-5
        vol = lambda F: float(F[1:-1, 1:-1, 1:-1].astype(np.float64).sum())  # noqa: E731
        assert abs(vol(got["F"]) - vol(ref["F"])) <= 1e-7 * vol(ref["F"])


def test_allocation_failure_in_create(cuda, V, tmp_path):
    """Each device allocation of vof_create (the multigrid solver's in the
    MIXED mode included) made to fail in turn (vof_debug_fail_alloc, a
    host-side fake of an out-of-memory cudaMalloc):
    VOF_E_NOMEM and no context, nothing left allocated (device free memory
    back to within 16 MiB of what it was: less than one 160^3 field, 19.2
    MiB), and the next vof_create, which finds no setting left, works.  In a child process, so
    that the free-memory count sees only these contexts."""
    import json
    import os
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    out = tmp_path / "alloc.json"
    code = f"""
import ctypes as C, json, sys
sys.path.insert(0, {str(root / 'cuda-lbm-ibm-fvm_b200')!r})
import torch
import vof_b200 as V
lib = V.lib()
torch.cuda.mem_get_info(0)  # (torch's own CUDA set-up before any count)
res = {{}}
for name, kw in (("plain", {{}}), ("csf", {{"surface_tension": 1}}), ("mixed", {{"mode": V.MODE_MIXED}})):
    prm = V.default_params(160, **kw)
    ctx = C.c_void_p()
    assert lib.vof_create(C.byref(prm), None, C.byref(ctx)) == 0
    if name == "plain":
        assert lib.vof_step(ctx, 1) == 0 and lib.vof_sync(ctx) == 0
    lib.vof_destroy(ctx)
    free0 = torch.cuda.mem_get_info(0)[0]
    n = 0
    while True:
        lib.vof_debug_fail_alloc(n)
        ctx = C.c_void_p()
        rc = lib.vof_create(C.byref(prm), None, C.byref(ctx))
        if rc == 0:
            break
        assert rc == V.E_NOMEM and not ctx.value, (name, n, rc)
        n += 1
        assert n < 64, name
    if name == "plain":
        assert lib.vof_step(ctx, 1) == 0 and lib.vof_sync(ctx) == 0
    lib.vof_destroy(ctx)
    ctx = C.c_void_p()
    assert lib.vof_create(C.byref(prm), None, C.byref(ctx)) == 0
    lib.vof_destroy(ctx)
    res[name] = [n, free0 - torch.cuda.mem_get_info(0)[0]]
json.dump(res, open({str(out)!r}, "w"))
"""
    subprocess.run([sys.executable, "-c", code], env=dict(os.environ), check=True, timeout=600)
    res = json.loads(out.read_text())
    n_plain = res["plain"][0]
    assert n_plain >= 10
    assert res["csf"][0] == n_plain + 4  # the four surface-tension fields
    # the FP64 pressure and the multigrid solver's buffers (three per level
    # over at least four levels at 160^3, its partials, result and level table)
    assert res["mixed"][0] >= n_plain + 1 + 3 * 4 + 3
    for name, (n, leaked) in res.items():
        assert leaked < 16 * 2**20, (name, leaked)

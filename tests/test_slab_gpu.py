"""z-slab decomposition on the GPU: the ranks of a decomposition as contexts
of one process on one GPU (vof_b200.slab.LocalGroup, with the halo planes
moved by vof_get_planes / vof_put_planes through device buffers), against
one context on the whole grid: every field bit for bit, the liquid volume
(vof_reduce_range over owned planes, summed) to 1e-12.  The plane copies and
range reductions are also checked on their own."""
import numpy as np
import pytest

from vof_b200 import ic, slab

pytestmark = pytest.mark.gpu

STATE = ("F", "u", "v", "w", "p")


def solver_factory(V):
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    return lambda prm: V.Solver(prm, stream=stream)


def test_plane_copies_and_range_reductions(cuda, V):
    import torch

    prm = V.default_params(14, 11, 23, dt=5e-4)
    st = ic.random_state(prm, seed=4)
    with V.Solver(prm, stream=torch.cuda.current_stream().cuda_stream) as s:
        s.upload_state(**st)
        for f in STATE:
            assert np.array_equal(s.get_planes(f, 0, prm.nz + 2), st[f])
            assert np.array_equal(s.get_planes(f, 5, 3), st[f][5:8])
        d = torch.zeros((4, prm.ny + 2, prm.nx + 2), dtype=torch.float32, device="cuda")
        s.get_planes("u", 9, 4, device_ptr=d.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy(), st["u"][9:13])
        s.put_planes("v", 2, device_ptr=d.data_ptr(), nk=4)
        s.put_planes("w", 20, st["F"][1:5])
        got = s.state()
        want_v = st["v"].copy()
        want_v[2:6] = st["u"][9:13]
        want_w = st["w"].copy()
        want_w[20:24] = st["F"][1:5]
        assert np.array_equal(got["v"], want_v) and np.array_equal(got["w"], want_w)
        F = st["F"].astype(np.float64)
        dv = float(prm.dx) * float(prm.dy) * float(prm.dz)
        assert s.reduce_range("volume", 3, 17) == pytest.approx(F[3:18, 1:-1, 1:-1].sum() * dv, rel=1e-12)
        assert s.reduce_range("f_max", 6, 6) == F[6, 1:-1, 1:-1].max()
        tot = sum(s.reduce_range("volume", a, b) for a, b in ((1, 8), (9, 9), (10, 23)))
        assert tot == pytest.approx(s.reduce("volume"), rel=1e-12)
        # stream-ordered: mapped pinned memory (written by the kernel) and an
        # ordinary host array (a copy in the stream), both equal to the blocking call
        ranges = (("volume", 3, 17), ("f_max", 6, 6), ("f_min", 1, 23), ("div_l2", 2, 9), ("div_max", 4, 12))
        pinned = torch.zeros(len(ranges), dtype=torch.float64).pin_memory()
        plain = np.zeros(len(ranges), dtype=np.float64)
        for i, (what, a, b) in enumerate(ranges):
            s.reduce_range_async(what, a, b, pinned.data_ptr() + 8 * i)
            s.reduce_range_async(what, a, b, plain.ctypes.data + 8 * i)
        s.sync()
        want = [s.reduce_range(what, a, b) for what, a, b in ranges]
        assert pinned.tolist() == want and plain.tolist() == want
        lib = s._lib
        assert lib.vof_reduce_range_async(s._ctx, 0, 0, 3, plain.ctypes.data) == V.E_INVALID
        assert lib.vof_reduce_range_async(s._ctx, 0, 1, 3, None) == V.E_INVALID
        with pytest.raises(V.VofError) as e:
            s.reduce_range_async("nonfinite", 1, 3, plain.ctypes.data)
        assert e.value.status == V.E_UNSUPPORTED
        assert lib.vof_get_planes(s._ctx, 0, -1, 2, d.data_ptr(), 1) == V.E_INVALID
        assert lib.vof_get_planes(s._ctx, 0, prm.nz + 1, 2, d.data_ptr(), 1) == V.E_INVALID
        assert lib.vof_reduce_range(s._ctx, 0, 0, 3, None) == V.E_INVALID
        with pytest.raises(V.VofError) as e:
            s.reduce_range("pres_resid", 1, 3)
        assert e.value.status == V.E_UNSUPPORTED


@pytest.mark.parametrize("nranks,shape,seed", [(2, (20, 18, 40), 1), (3, (17, 13, 60), 2), (4, (24, 24, 64), 3)])
def test_slabs_on_one_gpu_match_the_single_grid(cuda, V, nranks, shape, seed):
    prm = V.default_params(*shape, dt=2e-4, gy=0.0, gz=-9.81)
    st = ic.random_state(prm, seed=seed, vel_scale=0.5)  # (a state that stays finite over the steps)
    with V.Solver(prm) as s:
        s.upload_state(**st)
        s.run(1, 7)
        want = s.state()
        vol = s.reduce("volume")
    assert all(np.isfinite(want[k]).all() for k in STATE)
    grp = slab.LocalGroup(prm, nranks, solver_factory(V), device="cuda")
    grp.upload_global(st)
    grp.run(1, 7)
    got = grp.state()
    for k in STATE:
        assert np.array_equal(got[k], want[k]), k
    assert grp.volume() == pytest.approx(vol, rel=1e-12)
    for r in grp.ranks:
        r.engine.close()


def test_dam_break_slabs_match_the_single_grid(cuda, V):
    """The 64^3 dam break (quiet gas regions, the interface crossing a cut)
    over 2 slabs, 60 steps."""
    prm = V.default_params(64, gy=0.0, gz=-9.81)
    st = ic.rest_state(prm, ic.dam_break(prm, height=ic.noisy_height(prm, seed=1)))
    with V.Solver(prm) as s:
        s.upload_state(**st)
        s.run(1, 60)
        want = s.state()
    grp = slab.LocalGroup(prm, 2, solver_factory(V), device="cuda")
    grp.upload_global(st)
    grp.run(1, 60)
    got = grp.state()
    for k in STATE:
        assert np.array_equal(got[k], want[k]), k
    for r in grp.ranks:
        r.engine.close()

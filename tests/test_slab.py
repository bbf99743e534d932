"""z-slab decomposition (vof_b200.slab) on CPU: the plan, the halo exchange
over torch.distributed with the gloo backend (2 and 3 ranks, one process
each), and the ranks of one process (LocalGroup).  The ranks step with the
FP32 oracle (test infrastructure standing in for the CUDA library here); the
decomposed run must give the single-grid run's fields bit for bit, and the
liquid volume to 1e-12 (different summation order)."""
import os
import socket

import numpy as np
import pytest

from vof_b200 import ic, slab
from vof_b200.params import host_params

STATE = ("F", "u", "v", "w", "p")


class OracleEngine:
    """The Solver interface over the FP32 oracle (CPU), for the slab tests."""

    def __init__(self, prm):
        from oracle import oracle as orc

        self.orc = orc
        self.prm = prm
        self.st = None

    def upload_state(self, **st):
        self.st = {k: np.array(v, dtype=np.float32) for k, v in st.items()}

    def step(self, istep):
        self.st = self.orc.run_f32(self.prm, self.st, istep, 1)

    def run(self, istep0, n):
        for s in range(n):
            self.step(istep0 + s)

    def get_planes(self, f, k0, nk):
        return self.st[f][k0:k0 + nk].copy()

    def put_planes(self, f, k0, arr):
        self.st[f][k0:k0 + arr.shape[0]] = arr

    def reduce_range(self, what, a, b):
        assert what == "volume"
        F = self.st["F"][a:b + 1, 1:-1, 1:-1].astype(np.float64)
        return float(F.sum()) * float(self.prm.dx) * float(self.prm.dy) * float(self.prm.dz)

    def state(self):
        return self.st


def case(nz, seed):
    prm = host_params(12, 10, nz, dt=5e-4, gy=0.0, gz=-9.81)
    st = ic.random_state(prm, seed=seed, vel_scale=1.0)
    return prm, st


def test_plan_covers_the_grid_and_halos_come_from_one_neighbour():
    for nz, n in ((40, 2), (50, 3), (200, 8), (129, 4), (17, 1)):
        sl = slab.plan(nz, n)
        assert sl[0].own0 == 1 and sl[-1].own1 == nz and sl[0].lo == 1 and sl[-1].hi == nz
        for a, b in zip(sl, sl[1:]):
            assert b.own0 == a.own1 + 1
            assert b.lo == b.own0 - slab.HALO and a.hi == a.own1 + slab.HALO
            assert a.own1 - a.own0 + 1 >= slab.HALO and b.own1 - b.own0 + 1 >= slab.HALO
    with pytest.raises(ValueError):
        slab.plan(30, 2)  # 15-plane slabs: thinner than the halo
    assert slab.halo_for(10) == 16 and slab.halo_for(40) == 46


@pytest.mark.parametrize("world", [2, 4, 8])
def test_bench_slab_plans_for_the_scaling_run(world):
    """The plans `bench.py --gpus N` makes (200 planes per rank, the halo of
    ten Jacobi sweeps): every rank owns 200 planes, steps those plus one
    halo per cut, and exchanges exactly its halo depth with each neighbour."""
    import bench

    g = bench.slab_global_params(200, world)
    assert g.nz == 200 * world and g.nTot == 202 * 202 * (200 * world + 2)
    h = slab.halo_for(g.jacobi_iters)
    assert h == 16
    sl = slab.plan(g.nz, world, h)
    assert [s.own1 - s.own0 + 1 for s in sl] == [200] * world
    for r, s in enumerate(sl):
        cuts = (r > 0) + (r < world - 1)
        q = slab.local_params(g, s)
        assert q.nz == s.nz == 200 + h * cuts
        assert q.nTot == (q.nx + 2) * (q.ny + 2) * (q.nz + 2)
        ex = slab.Exchange(sl, r)
        assert sorted(p for p, _, _ in ex.sends) == sorted(p for p, _, _ in ex.recvs)
        assert [nk for _, _, nk in ex.sends] == [h] * cuts and [nk for _, _, nk in ex.recvs] == [h] * cuts


def test_exchange_pairs_match():
    sl = slab.plan(60, 3)
    ex = [slab.Exchange(sl, r) for r in range(3)]
    for r in range(3):
        for peer, k0, nk in ex[r].sends:
            back = [x for x in ex[peer].recvs if x[0] == r]
            assert len(back) == 1 and back[0][2] == nk
            # the planes sent are the ones the peer's halo stands for
            g_sent = sl[r].lo - 1 + k0
            g_recv = sl[peer].lo - 1 + back[0][1]
            assert g_sent == g_recv


@pytest.mark.parametrize("nranks,nz", [(2, 40), (3, 50)])
def test_local_group_matches_single_grid(orc, nranks, nz):
    prm, st = case(nz, seed=nranks)
    want = orc.run_f32(prm, st, 1, 6)
    assert all(np.isfinite(want[k]).all() for k in STATE)
    grp = slab.LocalGroup(prm, nranks, OracleEngine)
    grp.upload_global(st)
    grp.run(1, 6)  # every sweep order, twice
    got = grp.state()
    for k in STATE:
        assert got[k].shape == want[k].shape
        assert np.array_equal(got[k], want[k]), k
    vol = float(want["F"][1:-1, 1:-1, 1:-1].astype(np.float64).sum()) * float(prm.dx) * float(prm.dy) * float(prm.dz)
    assert grp.volume() == pytest.approx(vol, rel=1e-12)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nz, out_dir):
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "cuda-lbm-ibm-fvm_b200"), os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from test_slab import OracleEngine, case
    from vof_b200 import slab as sl

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        prm, st = case(nz, seed=world)
        r = sl.SlabRank(prm, sl.TorchComm(), OracleEngine, device="cpu")
        r.upload_global(st)
        r.run(1, 6)
        vol = r.volume()
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), vol=vol, **r.owned())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nz", [(2, 40), (3, 50)])
def test_gloo_ranks_match_single_grid(orc, tmp_path, world, nz):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_worker, args=(world, port, nz, str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    prm, st = case(nz, seed=world)
    want = orc.run_f32(prm, st, 1, 6)
    parts = [dict(np.load(tmp_path / f"rank{r}.npz")) for r in range(world)]
    for k in STATE:
        got = np.concatenate([p[k] for p in parts])
        assert np.array_equal(got, want[k]), k
    vol = float(want["F"][1:-1, 1:-1, 1:-1].astype(np.float64).sum()) * float(prm.dx) * float(prm.dy) * float(prm.dz)
    for p in parts:
        assert float(p["vol"]) == pytest.approx(vol, rel=1e-12)

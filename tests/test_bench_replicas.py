"""The multi-GPU path of bench.py (independent replicas, one per rank) on
CPU: two gloo ranks check the max-over-ranks timing, the whole-job value,
the barrier and the configuration label, and the reference arm's rank
gating (rank 1 does no work)."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "cuda-lbm-ibm-fvm_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_env() == (rank, world, rank)
        bench.barrier(world)
        # rank r timed 10 + r ms for 20 steps of a 1000-cell replica
        ms_max, value = bench.replica_throughput(world, 1000, 20, 10.0 + rank, None)
        bench.barrier(world)
        out[rank] = (ms_max, value)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_take_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        ms_max, value = out[r]
        assert ms_max == pytest.approx(11.0)
        # whole job: 2 replicas x 1000 cells x 20 steps in 11 ms
        assert value == pytest.approx(2 * 1000 * 20 / 11e-3 / 1e6)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.replica_throughput(1, 8_000_000, 100, 85.4) == (85.4, pytest.approx(8e6 * 100 / 0.0854 / 1e6))


def test_replica_config_label_and_reference_rank_gating(monkeypatch):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "cuda-lbm-ibm-fvm_b200"))
    import bench
    import vof_b200 as V

    prm = V.default_params(16)
    assert bench.workload_config(prm, 10, 4)["parallelism"] == "replicas x4"
    assert bench.workload_config(prm, 10, 1)["parallelism"] == "single"
    # the reference arm: a rank other than 0 returns before touching the GPU or the oracle
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")
    args = bench.parse_args(["--impl", "reference", "--gpus", "2"])
    assert bench.run_reference(args) is None


def test_clock_summary_flags_slowdowns():
    sys.path.insert(0, str(ROOT))
    import bench

    lines = ["0, 1965, 1965, 600.0, 0x0, Not Active, Not Active, Not Active, Not Active",
             "0, 1320, 1965, 1000.0, 0x4, Not Active, Not Active, Not Active, Active",
             "0, 1320, 1965, 1000.0, 0x8, Active, Not Active, Not Active, Active"]
    c = bench.summarize_clocks(lines)
    assert c["sm_mhz"] == 1320 and c["sm_max_mhz"] == 1965 and c["samples"] == 3
    assert c["reasons"] == ["hw_slowdown", "sw_power_cap"]


def test_slab_bench_grid_keeps_the_cell_size():
    """The multi-GPU bench's n x n x (n N) grid: the n^3 workload's constants
    and cell size (dz and dzi bit for bit), N slabs of n owned planes."""
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "cuda-lbm-ibm-fvm_b200"))
    import bench
    from vof_b200 import slab

    one = bench.workload_params(40)
    for world in (2, 3, 8):
        g = bench.slab_global_params(40, world)
        assert (g.nx, g.ny, g.nz) == (40, 40, 40 * world)
        assert (g.dz, g.dzi, g.dx, g.dt, g.gz) == (one.dz, one.dzi, one.dx, one.dt, one.gz)
        assert g.nTot == 42 * 42 * (40 * world + 2)
        sl = slab.plan(g.nz, world, slab.halo_for(g.jacobi_iters))
        assert all(s.own1 - s.own0 + 1 == 40 for s in sl)
    assert bench.parse_args(["--gpus", "2"]).decomp == "slab"

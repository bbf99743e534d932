"""bench.py's z-slab path -- the one `bench.py --gpus N` takes under torchrun
-- run as a single NCCL rank on one GPU: one slab, no exchange partner.  It
covers the path's set-up, timed regions, e2e loop and JSON line; the halo
exchange itself is covered by tests/test_slab.py (gloo ranks on CPU) and
tests/test_slab_gpu.py (local slabs on one GPU)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slab_bench_path_single_rank(cuda):
    code = (
        "import sys\n"
        f"sys.path.insert(0, {str(ROOT)!r})\n"
        f"sys.path.insert(0, {str(ROOT / 'cuda-lbm-ibm-fvm_b200')!r})\n"
        "import torch, torch.distributed as dist\n"
        "import bench\n"
        "import vof_b200 as V\n"
        "args = bench.parse_args(['--n', '64', '--steps', '5', '--warmup', '3'])\n"
        "dev = torch.device('cuda', 0)\n"
        "torch.cuda.set_device(dev)\n"
        "dist.init_process_group('nccl', device_id=dev, rank=0, world_size=1)\n"
        "try:\n"
        "    bench.run_slab(args, V, 0, 1, dev)\n"
        "finally:\n"
        "    dist.destroy_process_group()\n")
    env = {**os.environ, "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(free_port()), "RANK": "0",
           "WORLD_SIZE": "1", "LOCAL_RANK": "0"}
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600,
                         cwd=str(ROOT))
    assert out.returncode == 0, out.stderr[-3000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["n_gpus"] == 1 and line["steps"] == 5 and line["value"] > 0
    assert line["config"]["grid"] == [64, 64, 64]
    assert line["config"]["planes_per_rank"] == [[1, 64, 1, 64]]
    assert line["e2e"]["value"] > 0 and line["e2e"]["final_volume"] > 0
    assert line["halo_bytes_per_step_per_rank"] == 0  # no neighbour
    assert line["gpu_launches"] > 0

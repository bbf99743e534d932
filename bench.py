#!/usr/bin/env python
"""Benchmark of the two-phase VOF step on the 200^3 dam break (2000 steps).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A bench "step" is one solver time step (the loop body of voftrial1.cu:1361-1401)
over the whole 200^3 grid; the metric is Mcell-updates/s = cells * steps / s.

ours (default): the CUDA library through its C-ABI.
  value      device-resident throughput: W warm-up steps, then K steps through
             captured CUDA graphs bracketed by a barrier, synchronize and CUDA
             events on the library's stream; max over ranks.
  e2e        the same K steps through the public API with host buffers: upload
             of F,u,v,w,p from pinned memory, per step vof_run + an async FP64
             liquid-volume readback (8 bytes), final download of F; all inside
             the timed region.
  roofline   the dominant kernel (largest share of the step, timed live with
             CUDA events around each phase on the library's stream) against the
             measured HBM copy bandwidth in MEASURED_PEAKS.json.
  cpu_baseline  the FP64 CPU restatement (oracle/, OpenMP on every host core)
             on a bounded sample of the same workload.
reference: the reference's own voftrial1.cu kernels (oracle/_ref, built from
  the reference source; the reference has no CPU implementation of the path),
  sm_100a build and README build, better of the two; rank 0 only.

Multi-GPU (--decomp slab, the default): one n x n x (n N) grid cut into z
slabs of n planes per GPU, each rank stepping its slab plus a halo and
exchanging the halos with its neighbours over NCCL after every step
(vof_b200.slab; weak scaling); value = cells of the grid * steps / max-over-
ranks time.  --decomp replicas: N independent n^3 problems, no data-path
collective.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for _p in (str(ROOT), str(ROOT / "cuda-lbm-ibm-fvm_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "Mcell-updates/s at 200^3"
UNIT = "Mcell-updates/s"

# Algorithmic DRAM bytes per interior cell of one launch of each kernel
# (FP32 fields, stencil neighbours counted once).
ALG_BYTES = {
    "predict": 28,   # read F,u,v,w; write u*,v*,w*
    "rhs": 20,       # read F,u*,v*,w*; write rhs
    "jacobi": 12,    # read rhs,p; write p'
    "correct": 32,   # read u*,v*,w*,p,F; write u,v,w
    "sweep1": 12,    # read F, face velocity; write F
    "sweep2": 12,
    "sweep3": 12,
}
KERNEL_NAMES = {
    "predict": "k_predict2", "rhs": "k_rhs4", "jacobi": "k_jacobi_peel", "correct": "k_correct4",
    "sweep1": "k_fct_x|k_fct_march", "sweep2": "k_fct_x|k_fct_march", "sweep3": "k_fct_x|k_fct_march",
}
# the Jacobi kernel the library runs at the bench size (VOF_JACOBI=peel|pairs|ring|bulk|col|pairs2|tb|tb1;
# peel, one sweep per launch with two cells per thread, by default)
KERNEL_NAMES["jacobi"] = {"col": "k_jacobi_col", "tb": "k_jacobi_tb", "tb1": "k_jacobi_tb", "pairs2": "k_jacobi_pairs2",
                          "ring": "k_jacobi_ring", "bulk": "k_jacobi_bulk",
                          "pairs": "k_jacobi_pairs"}.get(os.environ.get("VOF_JACOBI", ""), "k_jacobi_peel")
if os.environ.get("VOF_CORRECT") == "1":
    KERNEL_NAMES["correct"] = "k_correct"
if os.environ.get("VOF_RHS") == "1":
    KERNEL_NAMES["rhs"] = "k_rhs"
if os.environ.get("VOF_PREDICT") == "1":
    KERNEL_NAMES["predict"] = "k_predict"
STEP_MODEL_BYTES = 188  # B per cell-step of the fused plain path (10 sweeps, FP32)
WARM_MS = 60.0  # least GPU time of warm-up steps run back to back before a timed region


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=200, help="grid cells per side (default 200)")
    ap.add_argument("--profile-steps", type=int, default=6)
    ap.add_argument("--repeats", type=int, default=3,
                    help="extra K-step regions timed after the reported one (diagnostic spread)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="target CPU time of the CPU-baseline sample (0 disables)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--ext-steps", type=int, default=10,
                    help="steps of each convergent-mode measurement at the bench size (0 disables)")
    ap.add_argument("--large-steps", type=int, default=8,
                    help="steps of the 320^3 mixed-solve + adjoint rollout (0: skip)")
    ap.add_argument("--adj-steps", type=int, default=400,
                    help="steps of the adjoint measurement at 64^3 (the bench size runs 1/8 of them; 0 disables)")
    ap.add_argument("--no-small", dest="small", action="store_false",
                    help="skip the 32^3 / 64^3 plain-step measurement")
    ap.add_argument("--decomp", choices=("slab", "replicas"), default="slab",
                    help="N > 1: one grid of n x n x (n N) cells cut into z slabs of n planes per GPU with a "
                         "halo exchange every step (slab), or N independent n^3 problems (replicas)")
    ap.add_argument("--drive-steps", type=int, default=300,
                    help="steps of the drop-in program run (voftrial1.cu's main at 200^3 with a dump every "
                         "100 steps), timed end to end (0 disables)")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []
        self._thr = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self._thr = threading.Thread(target=self._read, daemon=True)
        self._thr.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout: float = 3.0):
        """Block until the sampler has produced its first line (nvidia-smi
        start-up is done), so that it does not start inside a timed region."""
        t0 = time.perf_counter()
        while self.proc is not None and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self._thr:
            self._thr.join(timeout=2)
        return summarize_clocks(self.lines)


def summarize_clocks(lines) -> dict:
    sm, smax, power = [], [], []
    reasons = set()
    names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    for ln in lines:
        parts = [x.strip() for x in ln.split(",")]
        if len(parts) < 9:
            continue
        try:
            sm.append(float(parts[1]))
            smax.append(float(parts[2]))
            power.append(float(parts[3]))
        except ValueError:
            continue
        for name, val in zip(names, parts[5:9]):
            if val.lower().startswith("active"):
                reasons.add(name)
    if not sm:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
            "samples": len(sm), "power_w_max": max(power)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def workload_params(n, **over):
    """0.1 m box, rho 1000/50, nu 1e-6/1.5e-5, dt 4e-6, 10 Jacobi sweeps;
    gravity -9.81 along z (the reference's kernels add gx, gy, gz from the
    parameters).  Filled on the host (vof_b200.params, checked against the
    library's vof_params_init by a CPU test), so the reference arm never maps
    the library."""
    from vof_b200.params import host_params

    return host_params(n, gx=0.0, gy=0.0, gz=-9.81, **over)


def workload_state(prm):
    from vof_b200 import ic

    F = ic.dam_break(prm, height=ic.noisy_height(prm, seed=1))
    return ic.rest_state(prm, F)


def workload_config(prm, steps, world):
    return {
        "workload": f"dam_break_{prm.nx}^3_plain_fp32",
        "grid": [prm.nx, prm.ny, prm.nz],
        "steps_timed": steps,
        "dt": float(prm.dt),
        "jacobi_iters": prm.jacobi_iters,
        "gravity": [float(prm.gx), float(prm.gy), float(prm.gz)],
        "ic": "liquid x<0.04, y<0.04, z<0.06+0.5*dx*U(-1,1) (splitmix64 seed 1), u=v=w=p=0",
        "l2_policy": "inputs larger than L2: 10 resident fields x %.0f MB" % (prm.nTot * 4 / 1e6),
        "parallelism": "single" if world == 1 else f"replicas x{world}",
    }


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    return 6650.0, "fallback 6.65 TB/s"


def measured_traffic():
    """Per-launch DRAM bytes of each kernel at 200^3 from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic_200.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


# ---------------------------------------------------------------------------
# distributed plumbing (replicas: barrier + max over ranks only)
# ---------------------------------------------------------------------------
def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(x: float, world: int, device=None) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, cells: int, steps: int, ms: float, device=None):
    """(max over ranks of the timed milliseconds, whole-job Mcell-updates/s):
    every rank advanced its own `cells`-cell replica `steps` steps."""
    ms_max = max_over_ranks(ms, world, device)
    return ms_max, world * cells * steps / (ms_max / 1e3) / 1e6


def barrier(world: int, device=None):
    if world > 1:
        import torch.distributed as dist

        dist.barrier(device_ids=[device.index] if device is not None and device.type == "cuda" else None)


# ---------------------------------------------------------------------------
# CPU baseline
# ---------------------------------------------------------------------------
def cpu_baseline(prm, state, seconds: float) -> dict | None:
    """The FP64 CPU restatement (oracle) on the host: all cores on a bounded
    sample of the workload (steps after one warm-up step, about `seconds`),
    one core on one step, and the 32^3 dam break (200 steps) on all cores."""
    if seconds <= 0:
        return None
    from oracle import oracle as orc

    import vof_b200 as V
    from vof_b200 import ic

    cores = os.cpu_count() or 1
    cells = prm.nx * prm.ny * prm.nz
    st = {k: state[k] for k in ("F", "u", "v", "w", "p")}
    t0 = time.perf_counter()
    st = orc.run_f64(prm, st, 1, 1, nthreads=cores)
    t1 = time.perf_counter()
    per = max(t1 - t0, 1e-6)
    n = int(min(20, max(1, round(seconds / per))))
    t0 = time.perf_counter()
    st = orc.run_f64(prm, st, 2, n, nthreads=cores)
    el = time.perf_counter() - t0
    t0 = time.perf_counter()
    orc.run_f64(prm, st, 2 + n, 1, nthreads=1)
    el1 = time.perf_counter() - t0
    small = V.default_params(32, gx=0.0, gy=0.0, gz=-9.81)
    s_state = ic.rest_state(small, ic.dam_break(small))
    t0 = time.perf_counter()
    orc.run_f64(small, s_state, 1, 200, nthreads=cores)
    el32 = time.perf_counter() - t0
    cpu = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                cpu = ln.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return {"value": cells * n / el / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"FP64 CPU restatement (oracle/vof_oracle.cpp, OpenMP {cores} threads = nproc, {cpu}): "
                      f"steps 2..{n + 1} of the {prm.nx}^3 workload after 1 warm-up step, {el:.2f} s",
            "single_thread_value": cells / el1 / 1e6,
            "dam_break_32_200_steps": {"value": 32 ** 3 * 200 / el32 / 1e6, "seconds": round(el32, 3),
                                       "cores": cores}}


# ---------------------------------------------------------------------------
# convergent pressure modes (extension): MIXED vs FP64 solver, same tolerance
# ---------------------------------------------------------------------------
def measure_convergent(V, n, steps, stream, dev, tol=1e-8):
    """Time `steps` steps of the MIXED and FP64 modes (3 warm-up steps each) on the
    workload; each step solves the pressure to ||r|| <= tol ||b||.  The timed
    region includes the host synchronisations of the convergence checks."""
    import torch

    out = {}
    fields = {}
    state = None
    for name, mode in (("mixed", V.MODE_MIXED), ("fp64", V.MODE_FP64)):
        prm = V.default_params(n, gx=0.0, gy=0.0, gz=-9.81, mode=mode, tol=tol, max_outer=200)
        if state is None:
            state = workload_state(prm)
        s = V.Solver(prm, stream=stream.cuda_stream)
        s.upload_state(**state)
        for q in range(3):
            s.step(1 + q)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        outer, rel = [], []
        e0.record(stream)
        for q in range(steps):
            s.step(4 + q)
            st = s.solver_stats()
            outer.append(st["outer"])
            rel.append(st["rel_final"])
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        cells = prm.nx * prm.ny * prm.nz
        out[name] = {"value": round(cells * steps / (ms / 1e3) / 1e6, 1), "unit": UNIT,
                     "ms_per_step": round(ms / steps, 4), "vcycles_per_step": round(float(np.mean(outer)), 2),
                     "max_rel_residual": float(np.max(rel)), "steps": steps,
                     "inner": "BF16 storage / FP32 math" if name == "mixed" else "FP64"}
        fields[name] = s.state()
        s.close()
    a, b = fields["mixed"], fields["fp64"]
    diff = {}
    for k in ("F", "u", "v", "w", "p"):
        x = a[k].astype(np.float64)
        y = b[k].astype(np.float64)
        if k == "p":
            x, y = x[1:-1, 1:-1, 1:-1], y[1:-1, 1:-1, 1:-1]
        diff[k] = float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
    out["mixed_vs_fp64_rel_l2"] = diff
    out["speedup_mixed_over_fp64"] = round(out["mixed"]["value"] / out["fp64"]["value"], 3)
    out["tol"] = tol
    out["workload"] = f"dam_break_{n}^3, steps 4..{3 + steps} after 3 warm-up steps"
    return out


# ---------------------------------------------------------------------------
# adjoint (extension): gradient of a box loss w.r.t. the initial velocity
# perturbation and the body force; time of the reverse pass vs the forward
# ---------------------------------------------------------------------------
def measure_adjoint(V, n, steps, every, stream, dev, dense=False):
    """dam break n^3 with N(0, (1e-3)^2) perturbations of u, v, w on interior
    faces (splitmix64 seed 3), loss = sum of F dV over cells with centre
    x > 0.06 and z < 0.02; forward = `steps` plain steps through captured
    graphs, record = the same steps with a checkpoint every `every` steps,
    backward = the reverse pass (segment recompute + per-step recompute +
    FP64 adjoint kernels).  CUDA events on the library's stream.  dense: the
    loss box is the whole domain (every adjoint field dense; at 4e-6 s x 400
    steps no liquid reaches the x > 0.06, z < 0.02 box, whose loss and
    adjoint are then 0 almost everywhere)."""
    import torch

    from vof_b200 import ic

    prm = V.default_params(n, gx=0.0, gy=0.0, gz=-9.81)
    st = ic.rest_state(prm, ic.dam_break(prm))
    lo = {"u": (1, 1, 2), "v": (1, 2, 1), "w": (2, 1, 1)}
    for q, k in enumerate(("u", "v", "w")):
        a = lo[k]
        shape = (prm.nz + 1 - a[0], prm.ny + 1 - a[1], prm.nx + 1 - a[2])
        st[k][a[0]:prm.nz + 1, a[1]:prm.ny + 1, a[2]:prm.nx + 1] += (
            1e-3 * ic.normal(3 * 1000 + q, int(np.prod(shape))).reshape(shape)).astype(np.float32)
    box = (0.06, 1e300, -1e300, 1e300, -1e300, 0.02) if not dense else (-1e300, 1e300) * 3

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    with V.Solver(prm, stream=stream.cuda_stream) as s:
        s.upload_state(**st)
        s.run(1, 3)  # graphs captured
        s.upload_state(**st)
        fwd_ms, _ = timed(lambda: s.run(1, steps))
        s.upload_state(**st)
        s.forward_record(1, steps, every)  # engine and tape allocated outside the timed region
        s.upload_state(**st)
        rec_ms, _ = timed(lambda: s.forward_record(1, steps, every))
        bwd_ms, r = timed(lambda: s.backward(box))
        lu = s.adjoint("u")
        kps = s.adjoint_kernels_per_step
        nbytes = s.device_bytes
    return {"workload": f"dam_break_{n}^3 + N(0,1e-3^2) interior-face velocity perturbation (seed 3), "
                        f"{steps} steps, loss = sum F dV over " + ("the whole domain" if dense else "x>0.06, z<0.02"),
            "steps": steps, "checkpoint_every": every if every > 0 else int(np.ceil(np.sqrt(steps))),
            "forward_mcell_s": round(prm.nx * prm.ny * prm.nz * steps / fwd_ms / 1e3, 1),
            "backward_mcell_s": round(prm.nx * prm.ny * prm.nz * steps / bwd_ms / 1e3, 1),
            "forward_ms_per_step": round(fwd_ms / steps, 4),
            "record_ms_per_step": round(rec_ms / steps, 4),
            "backward_ms_per_step": round(bwd_ms / steps, 4),
            "backward_over_forward": round(bwd_ms / fwd_ms, 3),
            "record_plus_backward_over_forward": round((rec_ms + bwd_ms) / fwd_ms, 3),
            "loss": r["loss"], "dL_dg": [float(x) for x in r["grad_g"]],
            "dL_du_norm": float(np.linalg.norm(lu)),
            "kernels_per_reversed_step": kps, "device_bytes": int(nbytes),
            "precision": "FP32 forward (bit-identical to the plain step), FP64 adjoint fields"}


# ---------------------------------------------------------------------------
# large rollout (extension, opt-in): 320^3, sinusoidal interface, MIXED
# pressure solve, adjoint of the box loss with sqrt(N) checkpoints
# ---------------------------------------------------------------------------
def measure_large(V, steps, stream, dev, n=320, horizon=5000):
    """`steps` steps of the 320^3 rollout (h = 0.06 + dx S(x,y)/max|S|,
    S = sum_{m=1..4} sin(2 pi m x/L + phi_m) sin(2 pi m y/L + psi_m), phases
    from splitmix64 seed 5), MIXED solve to 1e-8: forward through vof_step,
    record + reverse pass with checkpoints every ceil(sqrt(steps)) steps; and
    the device memory the same tape takes for `horizon` steps (computed from
    the measured per-state and engine sizes)."""
    import torch

    from vof_b200 import ic

    prm = V.default_params(n, gx=0.0, gy=0.0, gz=-9.81, mode=V.MODE_MIXED, tol=1e-8, max_outer=200)
    st = ic.rest_state(prm, ic.dam_break(prm, height=ic.sinusoidal_height(prm, seed=5)))
    box = (0.06, 1e300, -1e300, 1e300, -1e300, 0.02)
    cells = prm.nx * prm.ny * prm.nz

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    with V.Solver(prm, stream=stream.cuda_stream) as s:
        base = s.device_bytes
        s.upload_state(**st)
        s.step(1)
        s.upload_state(**st)
        fwd_ms, _ = timed(lambda: [s.step(1 + q) for q in range(steps)])
        s.upload_state(**st)
        s.forward_record(1, steps, 0)  # engine and tape allocated outside the timed region
        with_tape = s.device_bytes
        s.upload_state(**st)
        rec_ms, _ = timed(lambda: s.forward_record(1, steps, 0))
        bwd_ms, r = timed(lambda: s.backward(box))
        free, total = torch.cuda.mem_get_info(dev)
        stats = s.solver_stats()
    every = int(np.ceil(np.sqrt(steps)))
    px = -(-(n + 2) // 32) * 32
    padded = px * (n + 2) * (n + 2)
    state_bytes = padded * (5 * 4 + 8)  # five FP32 fields + the FP64 warm start
    tape_now = (-(-steps // every) + every) * state_bytes
    engine = with_tape - base - tape_now
    every_h = int(np.ceil(np.sqrt(horizon)))
    tape_h = (-(-horizon // every_h) + every_h) * state_bytes
    return {"workload": f"{n}^3 sinusoidal interface (seed 5), MIXED solve to 1e-8, {steps} steps; "
                        "loss = sum F dV over x>0.06, z<0.02",
            "steps": steps, "checkpoint_every": every,
            "forward_mcell_s": round(cells * steps / fwd_ms / 1e3, 1),
            "forward_ms_per_step": round(fwd_ms / steps, 3),
            "record_ms_per_step": round(rec_ms / steps, 3),
            "backward_ms_per_step": round(bwd_ms / steps, 3),
            "backward_mcell_s": round(cells * steps / bwd_ms / 1e3, 1),
            "backward_over_forward": round(bwd_ms / fwd_ms, 3),
            "device_bytes_solver": int(base), "device_bytes_with_tape": int(with_tape),
            "peak_device_bytes": int(with_tape), "device_used_bytes_with_tape": int(total - free),
            "device_total_bytes": int(total), "last_solve": stats,
            "tape_bytes_for_horizon": {"steps": horizon, "checkpoint_every": every_h,
                                       "bytes": int(tape_h + engine + base),
                                       "fits": bool(tape_h + engine + base < total)},
            "loss": r["loss"], "dL_dg": [float(x) for x in r["grad_g"]]}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch

    import vof_b200 as V

    rank, world, local = dist_env()
    if world != args.gpus:
        print(f"warning: --gpus {args.gpus} but WORLD_SIZE {world}", file=sys.stderr)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        if args.decomp == "slab":
            try:
                run_slab(args, V, rank, world, dev)
            finally:
                dist.destroy_process_group()
            return

    prm = workload_params(args.n)
    state = workload_state(prm)
    cells = prm.nx * prm.ny * prm.nz
    K, W = args.steps, max(3, args.warmup)
    stream = torch.cuda.current_stream(dev)
    props = torch.cuda.get_device_properties(dev)
    gpu_id = None
    try:
        gpu_id = "GPU-" + str(props.uuid)
    except Exception:
        pass

    solver = V.Solver(prm, stream=stream.cuda_stream)
    solver.upload_state(**state)
    istep = 1
    solver.run(istep, 3)  # captures the three per-order graphs
    istep += 3
    # the clock sampler is up before the warm-up, so that the warm-up steps
    # run straight into the timed ones (an idle GPU lowers its clocks)
    clocks = ClockSampler(gpu_id)
    clocks.start()
    clocks.wait_first()
    barrier(world, dev)
    # warm-up: W steps, and more until about WARM_MS of them have run back to
    # back (a GPU that has idled runs its first milliseconds of work slower)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.run(istep, W)
    e1.record(stream)
    e1.synchronize()
    istep += W
    w_ms = e0.elapsed_time(e1)
    extra = max(0, int(np.ceil((WARM_MS - w_ms) / max(w_ms / W, 1e-3))))
    extra = int(max_over_ranks(float(extra), world, dev))  # the same count on every rank
    solver.run(istep, extra)
    istep += extra
    W_eff = W + extra
    barrier(world, dev)
    torch.cuda.synchronize(dev)
    timed_steps = [istep, istep + K - 1]
    e0.record(stream)
    solver.run(istep, K)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    barrier(world, dev)
    ms = e0.elapsed_time(e1)
    istep += K
    ms_max, value = replica_throughput(world, cells, K, ms, dev)
    # the same K-step region again (diagnostic: spread between regions) and
    # single steps one by one (launch-to-launch variation)
    repeats = []
    for _ in range(max(0, args.repeats)):
        torch.cuda.synchronize(dev)
        e0.record(stream)
        solver.run(istep, K)
        e1.record(stream)
        e1.synchronize()
        repeats.append(round(e0.elapsed_time(e1) / K, 5))
        istep += K
    singles = []
    for _ in range(25):
        e0.record(stream)
        solver.run(istep, 1)
        e1.record(stream)
        e1.synchronize()
        singles.append(round(e0.elapsed_time(e1), 4))
        istep += 1
    clk = clocks.stop()
    vol = solver.reduce("volume")
    nonfinite = solver.reduce("nonfinite")

    # per-phase CUDA-event timing on the library's stream (live, same state)
    phases = {}
    for q in range(max(3, args.profile_steps)):
        for name, (pms, nl) in solver.step_timed(istep).items():
            phases.setdefault(name, []).append((pms, nl))
        istep += 1
    phase_ms = {k: statistics.median(x[0] for x in v) for k, v in phases.items()}
    phase_launches = {k: v[0][1] for k, v in phases.items()}
    dom = max(phase_ms, key=lambda k: phase_ms[k])
    per_launch_s = phase_ms[dom] / phase_launches[dom] / 1e3
    peak, peak_src = measured_peaks()
    achieved = ALG_BYTES[dom] * cells / per_launch_s / 1e9
    traffic = measured_traffic().get(KERNEL_NAMES[dom] + ":" + dom)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "kernel": KERNEL_NAMES[dom],
                "phase": dom, "alg_bytes_per_cell": ALG_BYTES[dom], "units_per_launch": cells,
                "launch_ms": round(per_launch_s * 1e3, 5), "peak_source": peak_src}
    step_ms = ms_max / K
    step_gbs = STEP_MODEL_BYTES * cells / (step_ms / 1e3) / 1e9
    step_roofline = {"model_bytes_per_cell_step": STEP_MODEL_BYTES,
                     "achieved_gbs": round(step_gbs, 1),
                     "frac_of_peak": round(step_gbs / peak, 4), "peak_gbs": peak,
                     "frac_of_nominal_8tbs": round(step_gbs / 8000.0, 4)}

    # e2e through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        lib = V.lib()
        host = {k: torch.from_numpy(state[k]).pin_memory() for k in V.STATE_FIELDS}
        vols = torch.zeros(K, dtype=torch.float64).pin_memory()
        Fout = torch.empty(prm.shape, dtype=torch.float32).pin_memory()
        solver2 = V.Solver(prm, stream=stream.cuda_stream)
        solver2.run(1, 3)  # graph capture outside the timed region
        # the output buffer's first device write outside the timed region
        # (the first DMA into freshly pinned pages runs at a few GB/s)
        solver2.download("F", Fout.numpy())
        solver.run(istep, W_eff)  # the GPU busy right up to the timed region
        istep += W_eff
        barrier(world, dev)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        au = torch.cuda.Event(enable_timing=True)
        ad = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for k in V.STATE_FIELDS:
            solver2._check(lib.vof_upload(solver2._ctx, V.FIELDS[k], C.c_void_p(host[k].data_ptr()), 0),
                           "vof_upload")
        au.record(stream)
        vptr = vols.data_ptr()
        for s in range(K):
            solver2.run(1 + s, 1)
            solver2.reduce_async("volume", vptr + 8 * s)
        ad.record(stream)
        solver2.download("F", Fout.numpy())  # synchronizes the stream
        a1.record(stream)
        a1.synchronize()
        wall = time.perf_counter() - t0
        e2e_ms, e2e_value = replica_throughput(world, cells, K, a0.elapsed_time(a1), dev)
        up_ms, dn_ms = a0.elapsed_time(au), ad.elapsed_time(a1)
        solver2.close()
        nbytes = prm.nTot * 4
        e2e = {"value": round(e2e_value, 1), "unit": UNIT,
               "h2d_bytes_per_step": 5 * nbytes / K, "d2h_bytes_per_step": (nbytes + 8 * K) / K,
               "ms": round(e2e_ms, 3), "wall_ms": round(wall * 1e3, 3),
               "upload_ms": round(up_ms, 3), "upload_gbs": round(5 * nbytes / up_ms / 1e6, 1),
               "download_ms": round(dn_ms, 3), "download_gbs": round(nbytes / dn_ms / 1e6, 1),
               "api": "vof_upload x5 (pinned) + K x (vof_run 1 step + vof_reduce_async volume) + vof_download F",
               "final_volume": float(vols[-1])}

    cpu = cpu_baseline(prm, state, args.cpu_seconds) if (rank == 0 and world == 1) else None
    ext = {}
    if args.ext_steps > 0 and world == 1:
        ext["convergent_pressure"] = measure_convergent(V, args.n, args.ext_steps, stream, dev)
        ext["convergent_pressure"]["speedup_mixed_over_plain"] = round(
            ext["convergent_pressure"]["mixed"]["value"] / value, 3)
    if args.large_steps > 0 and world == 1:
        ext["large_mixed_adjoint"] = measure_large(V, args.large_steps, stream, dev)
    if args.small and world == 1:
        ext["small_grids"] = measure_small(V, stream, dev)
    if args.drive_steps > 0 and world == 1:
        ext["drive"] = measure_drive(args.drive_steps)
    if args.adj_steps > 0 and world == 1:
        ext["adjoint"] = [measure_adjoint(V, 64, args.adj_steps, 20, stream, dev),
                          measure_adjoint(V, 64, args.adj_steps, 20, stream, dev, dense=True),
                          measure_adjoint(V, args.n, max(1, args.adj_steps // 8), 0, stream, dev, dense=True)]

    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": W_eff, "ms_per_step": round(step_ms, 5), "higher_is_better": True,
        "timed_steps": timed_steps, "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": workload_config(prm, K, world),
        "roofline": roofline, "step_roofline": step_roofline,
        "cpu_baseline": cpu, "clocks": clk, "e2e": e2e,
        "gpu_launches": solver.kernels_per_step * K,
        "repeat_ms_per_step": repeats, "single_step_ms": singles,
        "native_so_loaded": mapped_libraries(),
        "phases_ms": {k: round(v, 5) for k, v in phase_ms.items()},
        "phase_launches": phase_launches,
        "check": {"volume_after": vol, "nonfinite": nonfinite},
        "extensions": ext,
        "device": props.name,
    }
    solver.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# N GPUs, one grid: z slabs with a halo exchange every step (vof_b200.slab)
# ---------------------------------------------------------------------------
def slab_global_params(n, world):
    """The n x n x (n world) dam break: the bench's constants, dz of the n^3
    grid (the box is world times as tall)."""
    prm = workload_params(n)
    g = prm.copy()
    g.nz = n * world
    g.kmax = g.nz
    g.nTot = (g.nx + 2) * (g.ny + 2) * (g.nz + 2)
    g.Lz = float(np.float32(prm.Lz) * np.float32(world))
    return g


def run_slab(args, V, rank, world, dev):
    """Weak scaling over one grid: each of the `world` ranks owns n planes of
    an n x n x (n world) dam break (interface height 0.06 + 0.5 dx U(-1, 1),
    seed 1: liquid in the lowest slab), steps them with a halo of
    slab.halo_for(10) planes, and exchanges the halos with its neighbours over
    NCCL (point-to-point) after every step.  value = owned cells of all ranks
    x K / max over ranks of the device time of K steps (halo exchange
    included)."""
    import torch
    import torch.distributed as dist

    from vof_b200 import ic, slab

    stream = torch.cuda.current_stream(dev)
    props = torch.cuda.get_device_properties(dev)
    prm = slab_global_params(args.n, world)
    state = ic.rest_state(prm, ic.dam_break(prm, height=ic.noisy_height(prm, seed=1)))
    comm = slab.TorchComm()
    r = slab.SlabRank(prm, comm, lambda q: V.Solver(q, stream=stream.cuda_stream), device=dev)
    r.upload_global(state)
    K, W = args.steps, max(3, args.warmup)
    gpu_id = None
    try:
        gpu_id = "GPU-" + str(props.uuid)
    except Exception:
        pass
    clocks = ClockSampler(gpu_id)
    clocks.start()
    clocks.wait_first()
    istep = 1
    r.run(istep, max(W, 20))
    istep += max(W, 20)
    W_eff = max(W, 20)
    barrier(world, dev)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r.run(istep, K)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    barrier(world, dev)
    istep += K
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world, dev)
    own_cells = prm.nx * prm.ny * (r.slab.own1 - r.slab.own0 + 1)
    cells_all = prm.nx * prm.ny * prm.nz
    value = cells_all * K / (ms_max / 1e3) / 1e6
    # the halo exchange alone (K of them) and the rank's step alone
    barrier(world, dev)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(K):
        r.exchange()
    e1.record(stream)
    e1.synchronize()
    ex_ms = max_over_ranks(e0.elapsed_time(e1), world, dev) / K
    barrier(world, dev)
    e0.record(stream)
    r.engine.run(istep, K)
    e1.record(stream)
    e1.synchronize()
    step_ms = max_over_ranks(e0.elapsed_time(e1), world, dev) / K
    istep += K
    r.upload_global(state)
    barrier(world, dev)
    # e2e: the local state from pinned host memory, K steps with each rank's
    # liquid volume (its owned planes) read on the host every step through
    # mapped pinned memory, the owned F back, then the K partial volumes
    # summed over the ranks
    host = {k: torch.from_numpy(v).pin_memory() for k, v in slab.local_state(state, r.slab).items()}
    Fout = torch.empty((r.slab.own1 - r.slab.own0 + 1, prm.ny + 2, prm.nx + 2), dtype=torch.float32).pin_memory()
    vols = torch.zeros(K, dtype=torch.float64).pin_memory()
    k_own = (r.slab.local(r.slab.own0), r.slab.local(r.slab.own1))

    def upload():
        for k in slab.STATE:
            r.engine._check(r.engine._lib.vof_upload(r.engine._ctx, V.FIELDS[k], C.c_void_p(host[k].data_ptr()), 0),
                            "vof_upload")

    # the pinned pages' first transfers outside the timed region
    upload()
    r.engine.reduce_range_async("volume", *k_own, vols.data_ptr())
    r.engine.get_planes("F", k_own[0], Fout.shape[0], out=Fout.numpy())
    torch.cuda.synchronize(dev)
    barrier(world, dev)
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    upload()
    for s in range(K):
        r.run(1 + s, 1)
        r.engine.reduce_range_async("volume", *k_own, vols.data_ptr() + 8 * s)
    r.engine.get_planes("F", k_own[0], Fout.shape[0], out=Fout.numpy())  # synchronizes the stream
    vol_all = vols.to(dev)
    if world > 1:
        dist.all_reduce(vol_all)
    vol_all = vol_all.cpu()
    a1.record(stream)
    a1.synchronize()
    e2e_ms = max_over_ranks(a0.elapsed_time(a1), world, dev)
    clk = clocks.stop()
    nbytes = sum(v.numel() * 4 for v in host.values())
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": W_eff, "ms_per_step": round(ms_max / K, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": f"dam_break_{prm.nx}x{prm.ny}x{prm.nz}_plain_fp32",
                   "grid": [prm.nx, prm.ny, prm.nz], "steps_timed": K, "dt": float(prm.dt),
                   "jacobi_iters": prm.jacobi_iters, "gravity": [float(prm.gx), float(prm.gy), float(prm.gz)],
                   "ic": "liquid x<0.04, y<0.04, z<0.06+0.5*dx*U(-1,1) (splitmix64 seed 1), u=v=w=p=0",
                   "l2_policy": "inputs larger than L2: 10 resident fields x %.0f MB per GPU"
                                % (r.lprm.nTot * 4 / 1e6),
                   "parallelism": f"z slabs x{world}, halo {slab.halo_for(prm.jacobi_iters)} planes, "
                                  "NCCL point-to-point halo exchange every step",
                   "planes_per_rank": [[s.own0, s.own1, s.lo, s.hi] for s in r.slabs]},
        "e2e": {"value": round(cells_all * K / (e2e_ms / 1e3) / 1e6, 1), "unit": UNIT,
                "h2d_bytes_per_step": world * nbytes / K, "d2h_bytes_per_step": world * (Fout.numel() * 4 + 8 * K) / K,
                "ms": round(e2e_ms, 3), "final_volume": float(vol_all[-1]),
                "api": "vof_upload x5 (pinned) + K x (vof_run 1 step + halo exchange + vof_reduce_range_async "
                       "volume) + vof_get_planes F (owned) + one all-reduce of the K partial volumes"},
        "halo_exchange_ms_per_step": round(ex_ms, 5), "rank_step_ms": round(step_ms, 5),
        "halo_bytes_per_step_per_rank": int(sum(b.numel() * 4 for b in r.sbuf.values())),
        "owned_cells_per_rank": own_cells, "clocks": clk,
        "gpu_launches": r.engine.kernels_per_step * K,
        "native_so_loaded": mapped_libraries(), "device": props.name,
    }
    for rr in (r.engine,):
        rr.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# small grids: the 32^3 dam break with a flat interface (200 steps) and 64^3
# ---------------------------------------------------------------------------
SMALL_GRIDS = ((32, 200), (64, 200))


def small_state(n):
    """The dam break with a flat interface (h0 = 0.06, no noise) at n^3."""
    from vof_b200 import ic

    prm = workload_params(n)
    return prm, ic.rest_state(prm, ic.dam_break(prm))


def measure_small(V, stream, dev):
    """Plain steps at 32^3 and 64^3 (the bench's physics, flat interface):
    3 warm-up steps, then the grid's step count through vof_run (captured
    graphs), CUDA events on the library's stream."""
    import torch

    out = {}
    for n, steps in SMALL_GRIDS:
        prm, st = small_state(n)
        with V.Solver(prm, stream=stream.cuda_stream) as s:
            s.upload_state(**st)
            s.run(1, 3)
            s.upload_state(**st)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            e0.record(stream)
            s.run(1, steps)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
        out[f"{n}^3"] = {"steps": steps, "ms_per_step": round(ms / steps, 5),
                         "value": round(n ** 3 * steps / ms / 1e3, 1), "unit": UNIT}
    return out


# ---------------------------------------------------------------------------
# the drop-in program: voftrial1.cu's main() end to end, dumps included
# ---------------------------------------------------------------------------
DRIVE_NSTEP = 100


def finished_seconds(out: str):
    """The "Finished at step N in T s" line of the reference's main()."""
    m = re.search(r">>> Finished at step (\d+) in ([0-9.eE+-]+) s", out)
    return (int(m.group(1)), float(m.group(2))) if m else (None, None)


def time_program(cmd, steps):
    """Run one drop-in program in a scratch directory (its dumps go to
    output/ there, removed afterwards); wall time from its own timing line."""
    import shutil
    import subprocess
    import tempfile

    d = tempfile.mkdtemp(prefix="vofdrive_")
    try:
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=1800)
        n, sec = finished_seconds(r.stdout)
        dumps = sorted(os.listdir(os.path.join(d, "output"))) if os.path.isdir(os.path.join(d, "output")) else []
        size = sum(os.path.getsize(os.path.join(d, "output", f)) for f in dumps)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    if r.returncode != 0 or n != steps:
        return {"error": (r.stderr or r.stdout)[-300:], "returncode": r.returncode}
    return {"seconds": sec, "mcell_s": round(200 ** 3 * steps / sec / 1e6, 1), "dumps": len(dumps),
            "dump_bytes": size}


def measure_drive(steps):
    """vof_drive (driver/vof_drive.cpp) with the reference program's own
    set-up (200^3, ic 1, g = (0, -5, 0), 10 Jacobi sweeps): `steps` steps with
    a dump of F every 100 steps as ASCII VTK (the reference's format), as
    binary VTK and with no dumps.  Seconds from the program's own
    "Finished at step N in T s" line (host wall clock around the loop,
    including the dumps still being written at the end)."""
    from vof_b200 import build as vb

    exe = str(vb.DRIVER_PATH)
    out = {"workload": f"voftrial1.cu main(): 200^3, ic 1, g=(0,-5,0), {steps} steps, F dumped every "
                       f"{DRIVE_NSTEP} steps", "nstep": DRIVE_NSTEP, "steps": steps}
    for kind in ("ascii", "binary", "none"):
        out[kind] = time_program([exe, "--max_steps", str(steps), "--nstep", str(DRIVE_NSTEP), "--vtk", kind], steps)
    return out


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    from oracle import oracle as orc

    variants = [v for v in ("sm100a", "readme") if orc.ref_available(v)]
    if not variants:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference harness oracle/_ref not built (needs the reference source at build time)"}))
        return
    import torch

    torch.cuda.set_device(local)
    props = torch.cuda.get_device_properties(local)
    gpu_id = None
    try:
        gpu_id = "GPU-" + str(props.uuid)
    except Exception:
        pass
    prm = workload_params(args.n)
    state = workload_state(prm)
    cells = prm.nx * prm.ny * prm.nz
    K, W = args.steps, max(3, args.warmup)
    results = {}
    clk = None
    for var in variants:
        clocks = ClockSampler(gpu_id)
        clocks.start()
        clocks.wait_first()
        # warm-up as in the library's arm: W steps, and more until about
        # WARM_MS of them have run (the timed steps then lie past the start-up
        # transient in both arms, and the clocks have ramped)
        w_ms, _ = orc.ref_time(prm, state, 1, 0, W, variant=var)
        W_eff = W + max(0, int(np.ceil((WARM_MS - w_ms) / max(w_ms / W, 1e-3))))
        ms, _ = orc.ref_time(prm, state, 1, W_eff, K, variant=var)
        c = clocks.stop()
        results[var] = {"ms": ms, "value": cells * K / (ms / 1e3) / 1e6, "clocks": c, "warmup": W_eff}
    best = max(results, key=lambda v: results[v]["value"])
    clk = results[best]["clocks"]
    value = results[best]["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": 1,
        "steps": K, "warmup": results[best]["warmup"], "ms_per_step": round(results[best]["ms"] / K, 5),
        "higher_is_better": True, "timed_steps": [1 + results[best]["warmup"], results[best]["warmup"] + K],
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": workload_config(prm, K, 1),
        "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": None, "kind": "reference",
                         "sample": f"voftrial1.cu's own kernels ({best} build) on {props.name}, "
                                   f"{K} steps after {W}; the reference has no CPU implementation of the path"},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "variants": {v: {"value": round(r["value"], 1), "ms_per_step": round(r["ms"] / K, 5)}
                     for v, r in results.items()},
        "clocks": clk, "gpu_launches": orc.ref_lib(best).ref_kernels_per_step(prm.jacobi_iters) * K,
        "device": props.name,
    }
    # small grids through the reference's own kernels (the faster build)
    if args.small:
        line["small_grids"] = {}
        for n, steps in SMALL_GRIDS:
            prm_s, st_s = small_state(n)
            ms_s, _ = orc.ref_time(prm_s, st_s, 1, 3, steps, variant=best)
            line["small_grids"][f"{n}^3"] = {"steps": steps, "ms_per_step": round(ms_s / steps, 5),
                                             "value": round(n ** 3 * steps / ms_s / 1e3, 1), "unit": UNIT,
                                             "build": best}
    # the reference program itself, end to end with its dumps (voftrial1.cu main())
    exe = orc.ORACLE_DIR / "_ref" / "vof3d_ref"
    if args.drive_steps > 0 and exe.exists():
        line["drive"] = {"workload": f"voftrial1.cu main() unmodified (sm_100a build): 200^3, ic 1, g=(0,-5,0), "
                                     f"{args.drive_steps} steps, F dumped every {DRIVE_NSTEP} steps (ASCII VTK)",
                         "nstep": DRIVE_NSTEP, "steps": args.drive_steps,
                         "ascii": time_program([str(exe), "--max_steps", str(args.drive_steps), "--nstep",
                                                str(DRIVE_NSTEP)], args.drive_steps)}
    # the arm must run the reference's code only: no library of this repository mapped
    line["native_so_loaded"] = mapped_libraries()
    own = [x for x in line["native_so_loaded"] if "libvof_b200" in x]
    if own:
        raise RuntimeError(f"reference arm mapped this repository's library: {own}")
    print(json.dumps(line), flush=True)


def mapped_libraries() -> list:
    """Shared objects of this repository mapped into the process (from
    /proc/self/maps): the oracle's and the reference harness's on the
    reference arm, the library's on ours."""
    out = set()
    try:
        with open("/proc/self/maps") as fh:
            for ln in fh:
                parts = ln.split()
                if len(parts) >= 6 and parts[-1].endswith(".so") and str(ROOT) in parts[-1]:
                    out.add(os.path.relpath(parts[-1], ROOT))
    except OSError:
        pass
    return sorted(out)


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

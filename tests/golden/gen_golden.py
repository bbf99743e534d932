"""Generate the golden vectors in tests/golden from the reference's own kernels.

Runs on a machine with a GPU and the reference harness built under
oracle/_ref (oracle/Makefile: voftrial1.cu compiled unmodified, once with
-fmad=false and once with nvcc's defaults).  For every case it stores the
inputs and the state after `nsteps` steps of both builds:

    in_{F,u,v,w,p}, nofma_{F,u,v,w,p}, fma_{F,u,v,w,p}

and writes index.json with the parameters, the tolerance the tests apply to
the FMA build (fma_rel_l2, a stated bound) and the measured difference
between the two builds.

It also runs the reference's apply_bc (voftrial1.cu:943-956, never called by
its time loop) on seeded random fields and stores in_/out_{u,v,w,F,p,rho} per
case in apply_bc_*.npz, listed in apply_bc.json.

    python tests/golden/gen_golden.py [outdir] [--only steps|apply_bc]
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "cuda-lbm-ibm-fvm_b200"))

import vof_b200 as V  # noqa: E402
from oracle import oracle as orc  # noqa: E402
from vof_b200 import ic  # noqa: E402

STATE = ("F", "u", "v", "w", "p")

CASES = [
    # name, grid, overrides, input, istep0, nsteps, stated rel-L2 bound vs the FMA build
    dict(name="rand_16x12x10_s1", nx=16, ny=12, nz=10, overrides=dict(dt=1e-3, gy=0.0, gz=-9.81),
         input=dict(kind="random", seed=1, vel_scale=1.0), istep0=1, nsteps=3, fma_rel_l2=1e-5),
    dict(name="rand_17x9x13_s2", nx=17, ny=9, nz=13, overrides=dict(dt=5e-4),
         input=dict(kind="random", seed=2, vel_scale=2.0), istep0=2, nsteps=3, fma_rel_l2=1e-5),
    dict(name="rand_8x8x8_iters7", nx=8, ny=8, nz=8, overrides=dict(dt=1e-3, jacobi_iters=7),
         input=dict(kind="random", seed=3, vel_scale=1.0), istep0=1, nsteps=4, fma_rel_l2=1e-5),
    dict(name="dam_32_200", nx=32, ny=32, nz=32, overrides=dict(gy=0.0, gz=-9.81),
         input=dict(kind="dam_break"), istep0=1, nsteps=200, fma_rel_l2=1e-5),
]


BC_CASES = [
    # name, grid, seed of the six standard-normal float32 input fields
    dict(name="apply_bc_7x5x4_s1", nx=7, ny=5, nz=4, seed=1),
    dict(name="apply_bc_1x3x2_s2", nx=1, ny=3, nz=2, seed=2),
    dict(name="apply_bc_16x12x10_s3", nx=16, ny=12, nz=10, seed=3),
]


def bc_input(prm, seed):
    rng = np.random.default_rng(seed)
    return {k: rng.standard_normal(prm.shape).astype(np.float32) for k in orc.BC_FIELDS}


def gen_apply_bc(outdir: Path):
    index = {"generator": "tests/golden/gen_golden.py --only apply_bc", "cases": []}
    for c in BC_CASES:
        prm = V.default_params(c["nx"], c["ny"], c["nz"])
        inp = bc_input(prm, c["seed"])
        out = orc.ref_apply_bc(prm, inp)
        arrays = {**{"in_" + k: inp[k] for k in orc.BC_FIELDS}, **{"out_" + k: out[k] for k in orc.BC_FIELDS}}
        fname = c["name"] + ".npz"
        np.savez_compressed(outdir / fname, **arrays)
        changed = {k: int((out[k] != inp[k]).sum()) for k in orc.BC_FIELDS}
        index["cases"].append({**c, "file": fname, "changed_cells": changed})
        print(c["name"], json.dumps(changed))
    (outdir / "apply_bc.json").write_text(json.dumps(index, indent=1) + "\n")


def make_input(prm, spec):
    if spec["kind"] == "random":
        return ic.random_state(prm, seed=spec["seed"], vel_scale=spec["vel_scale"])
    return ic.rest_state(prm, ic.dam_break(prm))


def rel_l2(a, b, interior_mean_free=False):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    if interior_mean_free:
        a = a[1:-1, 1:-1, 1:-1]
        b = b[1:-1, 1:-1, 1:-1]
        a, b = a - a.mean(), b - b.mean()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def main(outdir: Path):
    outdir.mkdir(parents=True, exist_ok=True)
    index = {"generator": "tests/golden/gen_golden.py", "cases": []}
    for c in CASES:
        prm = V.default_params(c["nx"], c["ny"], c["nz"], **c["overrides"])
        inp = make_input(prm, c["input"])
        nof = orc.ref_run(prm, inp, c["istep0"], c["nsteps"], variant="nofma")
        fma = orc.ref_run(prm, inp, c["istep0"], c["nsteps"], variant="sm100a")
        arrays = {}
        for k in STATE:
            arrays["in_" + k] = inp[k]
            arrays["nofma_" + k] = nof[k]
            arrays["fma_" + k] = fma[k]
        fname = c["name"] + ".npz"
        np.savez_compressed(outdir / fname, **arrays)
        measured = {k: rel_l2(nof[k], fma[k], interior_mean_free=(k == "p")) for k in STATE}
        entry = {kk: c[kk] for kk in ("name", "nx", "ny", "nz", "overrides", "input", "istep0", "nsteps",
                                       "fma_rel_l2")}
        entry["file"] = fname
        entry["measured_nofma_vs_fma_rel_l2"] = measured
        index["cases"].append(entry)
        print(c["name"], json.dumps(measured))
        worst = max(measured.values())
        if worst > c["fma_rel_l2"]:
            print(f"WARNING: {c['name']}: measured {worst:.3g} exceeds the stated bound {c['fma_rel_l2']}")
    (outdir / "index.json").write_text(json.dumps(index, indent=1) + "\n")


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("outdir", nargs="?", default=str(Path(__file__).resolve().parent))
    ap.add_argument("--only", choices=("steps", "apply_bc"))
    a = ap.parse_args()
    out = Path(a.outdir)
    out.mkdir(parents=True, exist_ok=True)
    if a.only in (None, "steps"):
        main(out)
    if a.only in (None, "apply_bc"):
        gen_apply_bc(out)

"""The C++ drop-in driver (driver/vof_drive.cpp) against the reference's main():
its initial condition (set_init_F_kernel + apply_bc_F, voftrial1.cu:72-93,
1122-1135) and dump format (write_legacy_vtk, voftrial1.cu:907-941) restated
in numpy, and a driven run against the FP32 oracle.

CPU tests use --ic-only (no GPU work); GPU tests run the time loop."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
DRIVE = ROOT / "cuda-lbm-ibm-fvm_b200" / "vof_b200" / "vof_drive"


def drive(*args, check=True, timeout=600):
    if not DRIVE.exists():
        pytest.fail(f"{DRIVE} not built (__graft_entry__.build())")
    r = subprocess.run([str(DRIVE), *map(str, args)], capture_output=True, text=True, timeout=timeout)
    if check:
        assert r.returncode == 0, r.stdout + r.stderr
    return r


def reference_ic(V, nx, ny, nz, ic=1):
    """set_init_F_kernel (ic 1) at every cell with the kernel's float32
    expressions, then apply_bc_F."""
    from vof_b200 import ic as icm

    prm = V.default_params(nx, ny, nz)
    F = np.zeros(prm.shape, dtype=np.float32)
    if ic == 1:
        f32 = np.float32
        cx = (np.clip(np.arange(nx + 2) - 1, 0, nx).astype(f32) * f32(prm.dx)).astype(f32)
        cy = (np.clip(np.arange(ny + 2) - 1, 0, ny).astype(f32) * f32(prm.dy)).astype(f32)
        cz = (np.clip(np.arange(nz + 2) - 1, 0, nz).astype(f32) * f32(prm.dz)).astype(f32)
        ix = (cx >= 0) & (cx <= f32(prm.Lx) / f32(3.0))
        iy = (cy >= 0) & (cy <= f32(prm.Ly) / f32(2.0))
        iz = (cz >= 0) & (cz <= f32(prm.Lz) / f32(3.0))
        F[iz[:, None, None] & iy[None, :, None] & ix[None, None, :]] = 1.0
    return icm.apply_bc_F(F)


def reference_vtk_text(F):
    """write_legacy_vtk's bytes: header (SPACING with the default 6 digits),
    then every value with setprecision(8), i.e. printf("%.8g")."""
    nzT, nyT, nxT = F.shape
    sx, sy, sz = (float(np.float32(1.0) / np.float32(n - 1)) for n in (nxT, nyT, nzT))
    head = ("# vtk DataFile Version 3.0\n3D VOF field\nASCII\nDATASET STRUCTURED_POINTS\n"
            f"DIMENSIONS {nxT} {nyT} {nzT}\nORIGIN 0 0 0\nSPACING {sx:g} {sy:g} {sz:g}\n"
            f"POINT_DATA {nxT * nyT * nzT}\nSCALARS VOF float 1\nLOOKUP_TABLE default\n")
    return head + "".join("%.8g\n" % float(v) for v in F.ravel())


def read_binary_vtk(path, shape):
    data = Path(path).read_bytes()
    lines = data.split(b"\n", 10)
    assert lines[2] == b"BINARY"
    body = lines[10]
    n = int(np.prod(shape))
    return np.frombuffer(body[:4 * n], dtype=">f4").astype(np.float32).reshape(shape)


@pytest.mark.parametrize("grid", [(8, 6, 5), (13, 9, 11), (30, 30, 30)])
def test_initial_condition_and_ascii_dump_match_the_reference(V, tmp_path, grid):
    nx, ny, nz = grid
    drive("--ic-only", "--grid", nx, ny, nz, "--out", tmp_path)
    got = (tmp_path / "step-00000.vtk").read_text()
    assert got == reference_vtk_text(reference_ic(V, nx, ny, nz))


@pytest.mark.parametrize("grid", [(8, 6, 5), (21, 17, 12)])
def test_ascii_dump_is_the_reference_writers_output(V, orc, tmp_path, grid):
    """The reference's own write_legacy_vtk (compiled from voftrial1.cu into
    oracle/_ref; host code) on the same field writes the same bytes."""
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference source)")
    from vof_b200 import ic as icm

    nx, ny, nz = grid
    prm = V.default_params(nx, ny, nz)
    F = icm.dam_break(prm, height=icm.noisy_height(prm, seed=7))
    rng = np.random.default_rng(1)
    F = np.where(F > 0, F, rng.random(F.shape) * (rng.random(F.shape) < 0.3)).astype(np.float32)
    F = icm.apply_bc_F(F)
    F.tofile(tmp_path / "F0.raw")
    drive("--ic-only", "--grid", nx, ny, nz, "--ic-file", tmp_path / "F0.raw", "--out", tmp_path)
    orc.ref_write_vtk(tmp_path / "ref.vtk", F)
    assert (tmp_path / "step-00000.vtk").read_bytes() == (tmp_path / "ref.vtk").read_bytes()


@pytest.mark.parametrize("ic", [2, 3])
def test_unimplemented_initial_conditions_leave_F_zero(V, tmp_path, ic):
    drive("--ic-only", "-ic", ic, "--grid", 6, 5, 4, "--out", tmp_path, "--vtk", "binary")
    F = read_binary_vtk(tmp_path / "step-00000.vtk", (6, 7, 8))
    assert not F.any()


def test_invalid_initial_condition_is_rejected(tmp_path):
    r = drive("--ic-only", "-ic", 4, "--out", tmp_path, check=False)
    assert r.returncode != 0 and "Invalid initial condition" in r.stderr


def test_binary_dump_and_ic_file(V, tmp_path):
    from vof_b200 import ic as icm

    prm = V.default_params(11, 7, 9)
    F = icm.dam_break(prm, height=icm.noisy_height(prm, seed=2))
    F[1:-1, 1:-1, 1:-1] += np.float32(0.25) * (F[1:-1, 1:-1, 1:-1] == 0)  # distinct interior values
    F.astype(np.float32).tofile(tmp_path / "F0.raw")
    drive("--ic-only", "--grid", 11, 7, 9, "--ic-file", tmp_path / "F0.raw", "--out", tmp_path, "--vtk", "binary")
    got = read_binary_vtk(tmp_path / "step-00000.vtk", prm.shape)
    want = icm.apply_bc_F(F.astype(np.float32).copy())
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_help_lists_the_reference_options():
    out = drive("--help").stdout
    for opt in ("-ic", "--nstep", "--max_steps", "--grid", "--vtk", "--mode", "--surface-tension"):
        assert opt in out


@pytest.mark.gpu
@pytest.mark.parametrize("grid", [(20, 18, 16), (31, 12, 25)])
def test_initial_condition_is_the_references(cuda, V, orc, tmp_path, grid):
    """The host IC of the driver against set_init_F_kernel + apply_bc_F run
    on the GPU by the reference's own code."""
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference source)")
    nx, ny, nz = grid
    drive("--ic-only", "--grid", nx, ny, nz, "--out", tmp_path, "--vtk", "binary")
    got = read_binary_vtk(tmp_path / "step-00000.vtk", (nz + 2, ny + 2, nx + 2))
    want = orc.ref_initial_F(V.default_params(nx, ny, nz), 1)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_driven_run_matches_the_oracle(cuda, V, orc, tmp_path):
    """12 steps of the reference's own set-up (ic 1, g = (0, -5, 0)) on a 20 x
    18 x 16 grid: dumps every 5 steps as the reference formats them, final
    fields bit for bit the FP32 oracle's."""
    nx, ny, nz = 20, 18, 16
    r = drive("--grid", nx, ny, nz, "--max_steps", 12, "--nstep", 5, "--out", tmp_path, "--final", tmp_path / "fin_")
    assert ">>> Finished at step 12 in" in r.stdout
    assert ">>> Exporting step-00005 result..." in r.stdout and ">>> Exporting step-00010 result..." in r.stdout
    prm = V.default_params(nx, ny, nz)
    from vof_b200 import ic as icm

    st = icm.rest_state(prm, reference_ic(V, nx, ny, nz))
    s5 = orc.run_f32(prm, st, 1, 5)
    s10 = orc.run_f32(prm, s5, 6, 5)
    s12 = orc.run_f32(prm, s10, 11, 2)
    assert (tmp_path / "step-00005.vtk").read_text() == reference_vtk_text(s5["F"])
    assert (tmp_path / "step-00010.vtk").read_text() == reference_vtk_text(s10["F"])
    for k, name in (("F", "F"), ("u", "U"), ("v", "V"), ("w", "W"), ("p", "P")):
        got = np.fromfile(tmp_path / f"fin_{name}.raw", dtype=np.float32).reshape(prm.shape)
        assert np.array_equal(got.view(np.uint32), s12[k].view(np.uint32)), k


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["mixed", "fp64"])
def test_driven_convergent_modes_match_the_library(cuda, V, tmp_path, mode):
    """The driver in a convergent mode gives the library's own result (same
    kernels, same calls), dumps in binary."""
    nx, ny, nz = 16, 16, 16
    drive("--grid", nx, ny, nz, "--max_steps", 6, "--nstep", 3, "--mode", mode, "--g", 0, 0, -9.81, "--vtk",
          "binary", "--out", tmp_path, "--final", tmp_path / "fin_")
    prm = V.default_params(nx, ny, nz, gx=0.0, gy=0.0, gz=-9.81, mode=getattr(V, "MODE_" + mode.upper()))
    with V.Solver(prm) as s:
        s.upload_state(**__import__("vof_b200").ic.rest_state(prm, reference_ic(V, nx, ny, nz)))
        s.run(1, 3)
        F3 = s.download("F")
        s.run(4, 3)
        fin = s.state()
    assert np.array_equal(read_binary_vtk(tmp_path / "step-00003.vtk", prm.shape), F3)
    for k, name in (("F", "F"), ("u", "U"), ("p", "P")):
        got = np.fromfile(tmp_path / f"fin_{name}.raw", dtype=np.float32).reshape(prm.shape)
        assert np.array_equal(got, fin[k]), k

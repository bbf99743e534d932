"""Build recipe for libvof_b200.so (sm_100a) -- nvcc only, no JIT cache.

The shared library is written next to this file, inside the source tree, so it
travels with the repository to the machine that runs it.  Object files go to
``cuda-lbm-ibm-fvm_b200/_build``.

``plain_step.cu`` (and the other FP32 step sources, and ``adjoint.cu``, which
recomputes the step's values) are compiled with ``-fmad=false``: the FP32 drop-in step keeps
the reference's per-point expressions without FMA contraction, which makes it
bit-identical to the CPU restatement (oracle/) and to the reference's kernels
compiled the same way.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
SRC_DIR = PKG_DIR.parent / "csrc"
BUILD_DIR = PKG_DIR.parent / "_build"
INCLUDE_DIR = PKG_DIR.parent.parent / "include"
LIB_PATH = PKG_DIR / "libvof_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + str(INCLUDE_DIR),
          "-Xptxas", "-warn-spills"]

# source -> extra flags
SOURCES = {
    "plain_step.cu": ["-fmad=false", "-DVOF_FMAD_FALSE"],
    "fct_sweep.cu": ["-fmad=false", "-DVOF_FMAD_FALSE"],
    "jacobi_tb.cu": ["-fmad=false", "-DVOF_FMAD_FALSE"],
    "adjoint.cu": ["-fmad=false", "-DVOF_FMAD_FALSE"],
    "tma_host.cu": [],
    "mg_solve.cu": [],
    "reduce.cu": [],
    "capi.cu": [],
    "noalloc.cu": [],
    "apply_bc.cu": [],
}
HEADERS = ["vof_device.cuh", "tma.cuh", "plain_step.h", "fct_sweep.h", "fct_line.cuh", "jacobi_tb.h", "mg_solve.h",
           "reduce.h", "adjoint.h", "apply_bc.h"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: cannot build libvof_b200.so")
    return exe


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra=(), lib_path: Path | None = None,
          build_dir: Path | None = None) -> Path:
    """Compile every CUDA source for sm_100a and link libvof_b200.so (or
    lib_path, with `extra` nvcc flags on every source, objects in build_dir)."""
    lib_out = LIB_PATH if lib_path is None else Path(lib_path)
    bdir = BUILD_DIR if build_dir is None else Path(build_dir)
    bdir.mkdir(parents=True, exist_ok=True)
    headers = [SRC_DIR / h for h in HEADERS] + [INCLUDE_DIR / "vof.h"]
    objs = []
    for src, flags in SOURCES.items():
        s = SRC_DIR / src
        o = bdir / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s, *headers, Path(__file__)]):
            cmd = [nvcc(), *ARCH, *COMMON, *flags, *extra, "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if force or _stale(lib_out, objs):
        tmp = lib_out.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(tmp)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(tmp, lib_out)
    return lib_out


DRIVER_SRC = PKG_DIR.parent / "driver" / "vof_drive.cpp"
DRIVER_PATH = PKG_DIR / "vof_drive"


def cuda_home() -> Path:
    return Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))


def build_driver(force: bool = False, verbose: bool = False) -> Path:
    """The C++ drop-in driver (driver/vof_drive.cpp) linked against
    libvof_b200.so (found next to it at run time) and the CUDA runtime."""
    lib = build(verbose=verbose)
    if force or _stale(DRIVER_PATH, [DRIVER_SRC, INCLUDE_DIR / "vof.h", lib]):
        cuda = cuda_home()
        tmp = DRIVER_PATH.with_name(DRIVER_PATH.name + ".tmp")
        cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", "-pthread", "-Wall", "-I", str(INCLUDE_DIR),
               "-I", str(cuda / "include"), str(DRIVER_SRC), "-o", str(tmp), "-L", str(lib.parent), "-lvof_b200",
               "-L", str(cuda / "lib64"), "-lcudart", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + str(cuda / "lib64")]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(tmp, DRIVER_PATH)
    return DRIVER_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

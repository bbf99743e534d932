"""C-ABI boundary checks that need no GPU: the library loads, exports every
entry point include/vof.h declares, fills parameters like the reference and
rejects bad arguments before touching the device."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import CUDA, ROOT


def declared_functions(header):
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vof_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(V):
    names = declared_functions(ROOT / "include" / "vof.h")
    assert "vof_step" in names and "vof_create" in names
    lib = V.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(V.exported_symbols()) <= set(names)


def test_abi_version(V):
    assert V.lib().vof_abi_version() == 2


def test_params_struct_layout(V):
    # vof_params: 9 int + 18 float + int nTot + 4 int + double + int, natural alignment
    assert C.sizeof(V.Params) == 144
    assert V.Params.tol.offset == 128
    assert V.Params.nTot.offset == 108
    assert V.Params.surface_tension.offset == 136


def test_params_init_leaves_surface_tension_off(V):
    assert V.default_params(8).surface_tension == 0


def test_params_init_matches_reference_constants(V):
    p = V.default_params(200, 200, 200)
    f32 = np.float32
    # voftrial1.cu:1262-1291
    assert (p.imin, p.imax, p.jmin, p.jmax, p.kmin, p.kmax) == (1, 200, 1, 200, 1, 200)
    assert p.dx == f32(f32(0.1) / f32(200))
    assert p.dxi == f32(f32(1.0) / f32(p.dx))
    assert p.rho_l == 1000.0 and p.rho_g == 50.0
    assert p.nu_l == f32(1e-6) and p.nu_g == f32(1.5e-5)
    assert p.sigma == f32(0.007)
    assert (p.gx, p.gy, p.gz) == (0.0, -5.0, 0.0)
    assert p.dt == f32(4e-6)
    assert p.nTot == 202 ** 3
    assert p.jacobi_iters == 10 and p.mode == V.MODE_PLAIN


def test_params_nonuniform(V):
    p = V.default_params(16, 12, 10, Lx=0.2)
    assert p.dx == np.float32(np.float32(0.2) / np.float32(16))
    assert p.dy == np.float32(np.float32(0.1) / np.float32(12))
    assert p.nTot == 18 * 14 * 12


@pytest.mark.parametrize("dims,over", [((200, 200, 200), {}), ((200, 200, 200), {"gy": 0.0, "gz": -9.81}),
                                       ((32, 32, 32), {"gy": 0.0, "gz": -9.81}), ((17, 9, 13), {"Lx": 0.2}),
                                       ((320, 320, 320), {"gy": 0.0, "gz": -9.81, "dt": 2e-6})])
def test_host_params_match_the_library(V, dims, over):
    """The numpy fill used where the library must not be loaded (the
    benchmark's reference arm) gives vof_params_init's values bit for bit."""
    from vof_b200.params import host_params

    a = V.default_params(*dims, **over)
    b = host_params(*dims, **over)
    assert bytes(a) == bytes(b)


def test_params_finalize_rejects_bad_sizes(V):
    p = V.Params()
    assert V.lib().vof_params_init(C.byref(p), 0, 4, 4) == V.E_SIZE
    assert V.lib().vof_params_init(C.byref(p), 2000, 2000, 2000) == V.E_SIZE  # nTot > INT_MAX
    assert V.lib().vof_params_finalize(None) == V.E_INVALID


def test_create_rejects_invalid_params_without_touching_device(V):
    lib = V.lib()
    ctx = C.c_void_p()
    assert lib.vof_create(None, None, C.byref(ctx)) == V.E_INVALID
    p = V.default_params(8, 8, 8)
    p.imax = 7  # inconsistent with nx
    assert lib.vof_create(C.byref(p), None, C.byref(ctx)) == V.E_INVALID
    p = V.default_params(8, 8, 8)
    p.dt = 0.0
    assert lib.vof_create(C.byref(p), None, C.byref(ctx)) == V.E_INVALID
    p = V.default_params(8, 8, 8)
    p.jacobi_iters = -1
    assert lib.vof_create(C.byref(p), None, C.byref(ctx)) == V.E_INVALID
    p = V.default_params(8, 8, 8)
    p.mode = 7
    assert lib.vof_create(C.byref(p), None, C.byref(ctx)) == V.E_INVALID
    assert not ctx.value


def test_null_context_calls_return_invalid(V):
    lib = V.lib()
    assert lib.vof_step(None, 1) == V.E_INVALID
    assert lib.vof_run(None, 1, 3) == V.E_INVALID
    assert lib.vof_sync(None) == V.E_INVALID
    assert lib.vof_upload(None, 0, None, 0) == V.E_INVALID
    assert lib.vof_download(None, 0, None, 0) == V.E_INVALID
    assert lib.vof_kernels_per_step(None) == V.E_INVALID
    assert lib.vof_reduce_range(None, 0, 1, 2, None) == V.E_INVALID
    assert lib.vof_reduce_range_async(None, 0, 1, 2, None) == V.E_INVALID
    assert lib.vof_apply_bc(None) == V.E_INVALID
    lib.vof_destroy(None)  # no-op


def test_apply_bc_fields_rejects_bad_params_without_touching_device(V):
    """vof_apply_bc_fields checks its parameters before any CUDA call."""
    lib = V.lib()
    nulls = [None] * 7
    assert lib.vof_apply_bc_fields(None, *nulls) == V.E_INVALID
    p = V.default_params(6, 5, 4)
    p.nTot += 1
    assert lib.vof_apply_bc_fields(C.byref(p), *nulls) == V.E_INVALID
    p = V.default_params(6, 5, 4)
    p.imax = 5
    assert lib.vof_apply_bc_fields(C.byref(p), *nulls) == V.E_INVALID
    p = V.default_params(6, 5, 4)
    p.nz = 0
    assert lib.vof_apply_bc_fields(C.byref(p), *nulls) == V.E_SIZE
    p = V.default_params(6, 5, 4)
    p.nx = p.ny = p.nz = 1300  # (nx+2)(ny+2)(nz+2) beyond the cell limit
    assert lib.vof_apply_bc_fields(C.byref(p), *nulls) == V.E_SIZE


def test_error_strings(V):
    lib = V.lib()
    for code in (0, -1, -2, -3, -4, -5, -6, -7, -8, -9):
        assert lib.vof_error_string(code)
    assert lib.vof_error_string(-99) == b"unknown status"


@pytest.mark.skipif(CUDA, reason="checks the behaviour on a machine without a GPU")
def test_create_without_gpu_returns_cuda_error(V):
    ctx = C.c_void_p()
    p = V.default_params(8, 8, 8)
    st = V.lib().vof_create(C.byref(p), None, C.byref(ctx))
    assert st == V.E_CUDA and not ctx.value


def test_binding_refuses_missing_library(tmp_path, monkeypatch):
    import vof_b200

    monkeypatch.setattr(vof_b200, "LIB_PATH", tmp_path / "nope.so")
    monkeypatch.setattr(vof_b200, "_lib", None)
    with pytest.raises(ImportError):
        vof_b200.lib()

"""vof_step_noalloc: the plain step for callers that must not allocate device
memory while they step -- their GPU memory is owned up front by their own
pool or allocator, or they cannot afford cudaMalloc's device-wide
synchronisation.  The caller keeps F, u, v, w, p in its own device buffers;
the step's scratch is a fixed device array inside the library.

Checked through the C-ABI against the context entry point (vof_step), bit
for bit, on two calls in a row; and the size limit is checked.  This file
sorts last so a run that stops at the first failure has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

from vof_b200 import ic

pytestmark = pytest.mark.gpu

STATE = ("F", "u", "v", "w", "p")


def noalloc_fn(V):
    fn = V.lib().vof_step_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(V.Params)] + [C.c_void_p] * 5 + [C.c_int, C.c_void_p]
    return fn


def test_noalloc_step_matches_context_on_two_calls(cuda, V):
    import torch

    prm = V.default_params(24, 20, 18, dt=5e-4, gy=0.0, gz=-9.81)
    state = ic.random_state(prm, seed=77, vel_scale=1.0)
    ref = []
    with V.Solver(prm) as s:
        s.upload_state(**state)
        for istep in (1, 2):
            s.step(istep)
            ref.append(s.state())
    dev = {k: torch.from_numpy(state[k].copy()).cuda() for k in STATE}
    torch.cuda.synchronize()
    fn = noalloc_fn(V)
    for n, istep in enumerate((1, 2)):
        rc = fn(C.byref(prm), *(C.c_void_p(dev[k].data_ptr()) for k in STATE), istep, None)
        assert rc == V.OK, rc
        torch.cuda.synchronize()
        for k in STATE:
            got = dev[k].cpu().numpy()
            assert np.array_equal(got, ref[n][k]), (n, k, int(np.sum(got != ref[n][k])))


def test_noalloc_rejects_grids_beyond_its_array(cuda, V):
    import torch

    prm = V.default_params(64, 64, 64)  # 11 padded fields of 96*66*66 floats > 2^21 floats
    buf = torch.zeros(prm.nTot, dtype=torch.float32, device="cuda")
    ptr = C.c_void_p(buf.data_ptr())
    rc = noalloc_fn(V)(C.byref(prm), ptr, ptr, ptr, ptr, ptr, 1, None)
    assert rc == V.E_SIZE
    assert float(buf.abs().sum()) == 0.0  # nothing was touched

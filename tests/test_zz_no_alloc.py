"""wf_pressure_noalloc: the pressure solve for callers that cannot allocate
device memory (frameworks that own all device memory through their own pool,
fixed device-memory budgets, allocation-free time-critical paths).

It must agree with the allocating entry point wf_pressure to the tolerance of
the operator tests (1e-11 of the largest pressure magnitude) on calls in a
row: the second call reuses the tables the first one left in the fixed
scratch array, the third changes grid (a Bluestein length in x instead of y)
and rebuilds them, the fourth changes back.  The device buffers are the
test's own; the entry point allocates nothing.  The host-side rejections are
in test_abi.py.  This file runs last so a failure here leaves every other test
already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_pressure_matches_allocating_entry_point(params_from_text):
    import torch
    from wildfires_b200 import Solver, _abi, configs

    torch.cuda.set_device(0)
    L = _abi.lib()
    results = []
    # (Nx, Ny, seed): x length 64 (power of two) and y length 47 (Bluestein),
    # then the same grid again, then the lengths swapped, then back
    for Nx, Ny, seed in ((65, 48, 11), (65, 48, 12), (48, 65, 13), (65, 48, 14)):
        case = configs.hill(Nx=Nx, Ny=Ny, Nz=24, Nt=1, L=100.0, H=20.0, jitter=0.3, seed=seed)
        P = params_from_text(configs.param_text(case.params))
        y0, p0 = case.fields(P)
        with Solver(P, "fp64") as s:
            p_ref, _ = s.pressure(y0, y0, p0)
        y_dev = torch.from_numpy(y0).to("cuda")
        p_dev = torch.from_numpy(p0.copy()).to("cuda")
        stream = torch.cuda.current_stream().cuda_stream
        st = L.wf_pressure_noalloc(C.byref(P.rec), C.c_void_p(y_dev.data_ptr()), C.c_void_p(p_dev.data_ptr()),
                                   C.c_void_p(stream))
        assert st == 0, L.wf_last_error().decode()
        torch.cuda.synchronize()
        p = p_dev.cpu().numpy()
        scale = np.max(np.abs(p_ref))
        assert np.max(np.abs(p - p_ref)) <= 1e-11 * scale, (Nx, Ny, seed)
        results.append(p)
    assert not np.array_equal(results[0], results[1])

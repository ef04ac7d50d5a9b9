"""Error paths of the context set-up, driven from the host (no GPU fault):
every device allocation wf_create makes is refused in turn by the library's
failure injection; each time wf_create returns WF_ERR_OOM with a message,
hands back no context, and frees what it had allocated (device memory in use
returns to where it was), and a context created afterwards works."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_every_refused_allocation_in_create_is_reported_and_cleaned_up(params_from_text):
    import torch
    from wildfires_b200 import Solver, _abi
    torch.cuda.set_device(0)
    L = _abi.lib()
    g = load_golden("hill_rk4")
    P = params_from_text(g["params"])
    for prec in (_abi.WF_FP64, _abi.WF_FP32_STENCIL):
        with Solver(P, "fp64" if prec == _abi.WF_FP64 else "fp32"):
            pass                                      # one-time set-up of the device
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        refused = 0
        for k in range(200):
            L.wf_inject_allocation_failure(k)
            h = C.c_void_p()
            st = L.wf_create(C.byref(P.rec), prec, C.byref(h))
            L.wf_inject_allocation_failure(-1)
            if st == 0:
                L.wf_destroy(h)
                break
            assert st == _abi.WF_ERR_OOM, (k, st)
            assert b"failure injection" in L.wf_last_error()
            assert not h.value
            refused += 1
        assert refused >= 10, refused                 # the context makes that many allocations
        torch.cuda.synchronize()
        assert abs(torch.cuda.mem_get_info()[0] - free0) <= 4 << 20
    with Solver(P, "fp32") as s:
        s.upload(g["y0"], g["p0"])
        s.step(2)
        y, _ = s.download()
    assert np.isfinite(y).all()

"""The C-ABI boundary on device buffers and caller streams.

* wf_phi_device / wf_rk_device / wf_pressure_device give the same bits as the
  host-buffer entry points (same kernels, no host copies), FP64 and FP32.
* wf_set_stream: steps enqueued on a caller's stream (a torch stream, and the
  legacy default stream) give the same bits as on the context's own stream,
  and order after the caller's earlier work on that stream.
* The drop-in's Phi (include/wf_dropin.h, the reference's signature) on
  device buffers: the result equals wf_phi's, and its event-timed duration is
  below that of one device-to-host copy of the state, so it cannot contain the
  host round trip it used to make (reference Phi: pde.cu:910-917).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
vp = C.c_void_p


def _case(params_from_text, Nx=33, Ny=40, Nz=16, seed=3):
    from wildfires_b200 import configs
    case = configs.hill(Nx=Nx, Ny=Ny, Nz=Nz, Nt=2, L=80.0, H=16.0, jitter=0.2, seed=seed)
    P = params_from_text(configs.param_text(case.params))
    y0, p0 = case.fields(P)
    return P, y0, p0


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_device_operators_match_host_operators(prec, params_from_text):
    import torch
    from wildfires_b200 import Solver, _abi
    L = _abi.lib()
    P, y0, p0 = _case(params_from_text)
    with Solver(P, prec) as s:
        R_host = s.phi(y0)
        y1_host = s.rk(y0) if hasattr(s, "rk") else None
        p_host, _ = s.pressure(y0, y0, p0)
    with Solver(P, prec) as s:
        a = torch.from_numpy(y0).to("cuda")
        b = torch.zeros_like(a)
        pd = torch.from_numpy(p0.copy()).to("cuda")
        _abi.check(L.wf_phi_device(s._h, vp(a.data_ptr()), vp(b.data_ptr())), "wf_phi_device")
        s.synchronize()
        assert np.array_equal(b.cpu().numpy(), R_host)
        if y1_host is not None:
            _abi.check(L.wf_rk_device(s._h, vp(a.data_ptr()), vp(b.data_ptr())), "wf_rk_device")
            s.synchronize()
            assert np.array_equal(b.cpu().numpy(), y1_host)
        _abi.check(L.wf_pressure_device(s._h, vp(a.data_ptr()), vp(a.data_ptr()), vp(pd.data_ptr())),
                   "wf_pressure_device")
        s.synchronize()
        assert np.array_equal(pd.cpu().numpy(), p_host)


@pytest.mark.parametrize("which", ["torch", "legacy"])
def test_steps_on_a_caller_stream(which, params_from_text):
    import torch
    from wildfires_b200 import Solver, _abi
    L = _abi.lib()
    P, y0, p0 = _case(params_from_text, seed=4)
    with Solver(P, "fp32") as s:
        s.upload(y0, p0)
        s.step(3)
        ref = s.download()
    with Solver(P, "fp32") as s:
        s.upload(y0, p0)
        if which == "torch":
            st = torch.cuda.Stream()
            handle = st.cuda_stream
        else:
            st = None
            handle = 1          # cudaStreamLegacy
        _abi.check(L.wf_set_stream(s._h, vp(handle)), "wf_set_stream")
        assert L.wf_stream(s._h) == handle
        if st is not None:
            # work of the caller enqueued first on its stream: the steps wait for it
            with torch.cuda.stream(st):
                big = torch.empty(1 << 26, device="cuda")
                for _ in range(4):
                    big.mul_(1.0001)
        s.step(3)
        s.synchronize()
        got = s.download()
        _abi.check(L.wf_set_stream(s._h, None), "wf_set_stream")
        s.step(1)
        s.synchronize()
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


DROPIN_LIB = os.path.join(ROOT, "wildfires_b200", "libwildfires_b200_dropin.a")


@pytest.mark.skipif(not os.path.exists(DROPIN_LIB), reason="drop-in archive not built")
def test_dropin_phi_runs_on_device_buffers(tmp_path, params_from_text):
    from wildfires_b200 import Solver, configs
    exe = str(tmp_path / "dropin_device_phi")
    libdir = os.path.join(ROOT, "wildfires_b200")
    cmd = ["/usr/local/cuda/bin/nvcc", "-O2", "-std=c++17", "-ccbin", "/usr/bin/g++", "-gencode",
           "arch=compute_100a,code=sm_100a",
           "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "dropin_device_phi.cu"),
           DROPIN_LIB, "-L" + libdir, "-lwildfires_b200", "-Xlinker", "-rpath", "-Xlinker", libdir, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    # 256 x 256 x 64 FP64: a 135 MB packed state
    case = configs.hill(Nx=256, Ny=256, Nz=64, Nt=1, L=400.0, H=25.0, jitter=0.1, seed=8)
    ppath = tmp_path / "parameters.txt"
    ppath.write_text(configs.param_text(case.params))
    P = params_from_text(configs.param_text(case.params))
    y0, _ = case.fields(P)
    y0.tofile(str(tmp_path / "y0.bin"))
    r = subprocess.run([exe, str(ppath), str(tmp_path / "y0.bin"), str(tmp_path / "R.bin")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    kv = dict(line.split("=") for line in r.stdout.split() if "=" in line)
    phi_ms, copy_ms = float(kv["PHI_MS"]), float(kv["COPY_MS"])
    R = np.fromfile(str(tmp_path / "R.bin"))
    with Solver(P, "fp64") as s:
        R_host = s.phi(y0)
    assert np.array_equal(R, R_host)
    # one device-to-host copy of the state takes longer than the whole Phi
    assert phi_ms < copy_ms, (phi_ms, copy_ms)

"""Full-size parity against the reference's own CUDA solver.

The reference's src/cu sources, built unmodified for sm_100a by oracle/Makefile
(oracle/_ref/ref_gpu), run the flat 128 x 128 x 64 workload and the
512 x 512 x 128 eight-hill workload on the same B200 from the same seeded
inputs.  Comparisons use the periodic cell set (the duplicate planes
i = Nx-1, j = Ny-1 are filled by the reference with an in-place copy that races
with the writes of plane 0, src/cu/pressure.cu:409-414; on these grids each
reference thread owns 16 or more cells, plane 0 is written long before the
copy, and the GPU build is reproducible -- on grids with one cell per thread
it is not, see tests/test_dropin_gpu.py).

The model amplifies rounding differences by about 1e12 between steps 50 and
100 of this workload (buoyant plume + stiff Arrhenius source): the reference's
own CPU and GPU builds of the same source differ by 1e-3 relative L2 in v
after 100 steps.  The 1e-10 gate is therefore applied within the predictable
horizon (50 steps); at the stated 200 steps the FP64 path must stay closer to
the reference than the model's own sensitivity to a 1e-15 relative change of
the initial temperature.
Skipped where the reference binaries were not built.
"""
import numpy as np
import pytest

import ref_runner
from conftest import _rel

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_runner.available("gpu"), reason="oracle/_ref/ref_gpu not built")]


def _errors(P, ours, ref):
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    out = {}
    for q, nm in enumerate("uvwT"):
        a = ours[q * N:(q + 1) * N].reshape(r.Nx, r.Ny, r.Nz)[:-1, :-1]
        b = ref[q * N:(q + 1) * N].reshape(r.Nx, r.Ny, r.Nz)[:-1, :-1]
        out[nm] = _rel(a.ravel(), b.ravel())
    nzy = P.nz_y()
    k = np.arange(r.Nz_Y_max)[None, None, :]
    m = (k < nzy[:, :, None])
    m[-1] = False
    m[:, -1] = False
    out["Y"] = _rel(ours[4 * N:][m.reshape(-1)], ref[4 * N:][m.reshape(-1)])
    return out


def _run(P, y0, p0, n):
    from wildfires_b200 import Solver
    with Solver(P, "fp64") as s:
        s.upload(y0, p0)
        s.step(n)
        y, _ = s.download()
        d = s.diagnostics(allow_nan=True)
    return y, d


def test_fp64_matches_reference_cuda_within_predictable_horizon():
    from wildfires_b200 import configs
    res = ref_runner.run(configs.flat(Nt=50), "step", flavour="gpu", timeout=1800)
    y, d = _run(res["P"], res["y0"], res["p0"], 50)
    assert d["nan_count"] == 0
    errs = _errors(res["P"], y, res["y"])
    bad = {f: e for f, e in errs.items() if e[0] > 1e-10 or e[1] > 1e-10}
    assert not bad, bad


def test_fp64_after_stated_steps_within_model_sensitivity():
    from wildfires_b200 import configs
    res = ref_runner.run(configs.flat(Nt=200), "step", flavour="gpu", timeout=1800)
    P = res["P"]
    y, d = _run(P, res["y0"], res["p0"], 200)
    assert d["nan_count"] == 0
    N = P.rec.Nx * P.rec.Ny * P.rec.Nz
    yp0 = res["y0"].copy()
    rng = np.random.default_rng(0)
    yp0[3 * N:4 * N] *= 1 + 1e-15 * rng.standard_normal(N)
    yp, _ = _run(P, yp0, res["p0"], 200)
    vs_ref = _errors(P, y, res["y"])
    own = _errors(P, yp, y)
    for f in "uvwT":
        assert vs_ref[f][1] <= own[f][1], (f, vs_ref[f], own[f])


def test_full_size_eight_hills_fp64_matches_reference_cuda():
    """The benchmark workload itself (512 x 512 x 128, terrain override), three
    FP64 steps against the reference's own GPU build at the 1e-10 gate."""
    from wildfires_b200 import configs
    res = ref_runner.run(configs.hills8(Nt=3), "step", flavour="gpu", timeout=1800)
    y, d = _run(res["P"], res["y0"], res["p0"], 3)
    assert d["nan_count"] == 0
    errs = _errors(res["P"], y, res["y"])
    bad = {f: e for f, e in errs.items() if e[0] > 1e-10 or e[1] > 1e-10}
    assert not bad, bad

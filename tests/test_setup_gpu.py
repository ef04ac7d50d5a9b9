"""Initial conditions generated on the GPU (wf_initial_conditions) against the
reference's own initial_conditions + create_y_0 (functions.cu:187-323,
solver.cu:41-56; fixtures tests/golden/ic_*.npz from its host build).

Tolerance: p, v, w, Y and every dead-node value bit-exact (no transcendental
in them; the products are rounded as the reference's host build rounds them);
u = u_r (z/z_r)^alpha_u and the gaussian T within 4e-16 of the field's
largest magnitude (CUDA's pow and exp against the host library's: an ulp or
two).  FP32 contexts hold the FP32 rounding of those values (one FP32 ulp)."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, field_errors

pytestmark = pytest.mark.gpu
IC = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "ic_*.npz")))


def _load(name, params_from_text):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    P = params_from_text(g["params"])
    if "topography" in g:
        P.set_topography(g["topography"])
    return g, P


def _solver(P, prec):
    from wildfires_b200 import Solver
    return Solver(P, prec)


@pytest.mark.parametrize("name", IC)
def test_initial_conditions_match_reference(name, params_from_text):
    g, P = _load(name, params_from_text)
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    with _solver(P, "fp64") as s:
        s.initial_conditions()
        y, p = s.download()
        assert s.time()[0] == 0
    ref = g["y0"]
    assert y.shape == ref.shape
    assert np.array_equal(p, g["p0"])
    for q in (1, 2):   # v, w
        assert np.array_equal(y[q * N:(q + 1) * N], ref[q * N:(q + 1) * N])
    assert np.array_equal(y[4 * N:], ref[4 * N:])   # Y
    cut = P.cut_nodes().reshape(-1)
    dead = (np.arange(r.Nz)[None, :] < cut[:, None]).reshape(-1)
    for q in (0, 3):   # u, T: transcendental away from dead nodes
        a, b = y[q * N:(q + 1) * N], ref[q * N:(q + 1) * N]
        assert np.array_equal(a[dead], b[dead])
        assert np.max(np.abs(a - b)) <= 4e-16 * np.max(np.abs(b))
    assert 0 < np.count_nonzero(y[4 * N:]) < r.Nx * r.Ny * r.Nz_Y_max   # the fuel shapes are exercised


@pytest.mark.parametrize("name", IC)
def test_initial_conditions_fp32(name, params_from_text):
    g, P = _load(name, params_from_text)
    with _solver(P, "fp32") as s:
        s.initial_conditions()
        y, p = s.download()
    ref32 = g["y0"].astype(np.float32).astype(np.float64)
    assert np.array_equal(p, g["p0"])
    assert np.all(np.abs(y - ref32) <= np.abs(ref32) * 2.0 ** -23)


@pytest.mark.parametrize("name", IC)
def test_steps_from_device_initial_conditions(name, params_from_text):
    """Stepping (the case's Nt steps) from the device-generated state equals
    stepping from the reference's uploaded state (to the 1e-12 the ulp-level
    start allows)."""
    g, P = _load(name, params_from_text)
    n = int(P.rec.Nt)
    with _solver(P, "fp64") as s:
        s.initial_conditions()
        s.step(n)
        a, pa = s.download()
    with _solver(P, "fp64") as s:
        s.upload(g["y0"], g["p0"])
        s.step(n)
        b, pb = s.download()
    bad = {f: e for f, e in field_errors(P, a, b).items() if e[0] > 1e-12 or e[1] > 1e-12}
    assert not bad, bad
    assert np.all(np.isfinite(pb))
    assert np.max(np.abs(pa - pb)) <= 1e-12 * max(np.max(np.abs(pb)), 1.0)

"""Tile shapes of the fused stage pass: every compiled shape gives bit-identical
states (a cell's arithmetic does not depend on the tiling, and the Van Driest
shortcut only skips factors that are exactly 1), and the per-context tuner
picks one of them."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu
SHAPES32 = [(8, 16, 512), (8, 16, 384), (8, 8, 256)]


def _run(P, g, prec, shape, n):
    from wildfires_b200 import Solver
    with Solver(P, prec) as s:
        if shape is not None:
            s.set_stage_tile(*shape)
        s.upload(g["y0"], g["p0"])
        s.step(n)
        return s.download(), s.stage_tile()


@pytest.mark.parametrize("name", ["hill_rk4", "flat_33x33x16_10", "stretched_rk2"])
def test_tile_shapes_give_identical_states(name, params_from_text):
    g = load_golden(name)
    P = params_from_text(g["params"])
    n = int(g["nsteps"])
    (y0, p0), _ = _run(P, g, "fp32", SHAPES32[0], n)
    for shape in SHAPES32[1:]:
        (y, p), used = _run(P, g, "fp32", shape, n)
        assert used == shape
        assert np.array_equal(y, y0) and np.array_equal(p, p0), shape


def test_tuner_picks_a_compiled_shape(params_from_text):
    g = load_golden("flat_33x33x16_10")
    P = params_from_text(g["params"])
    (y, p), used = _run(P, g, "fp32", None, 2)
    assert used in SHAPES32
    (yr, pr), _ = _run(P, g, "fp32", SHAPES32[0], 2)
    assert np.array_equal(y, yr) and np.array_equal(p, pr)
    (_, _), used64 = _run(P, g, "fp64", None, 1)
    assert used64[:2] == (8, 8)


def test_unknown_shape_is_rejected(params_from_text):
    from wildfires_b200 import Solver, WfError
    g = load_golden("hill_rk4")
    P = params_from_text(g["params"])
    with Solver(P, "fp32") as s:
        with pytest.raises(WfError):
            s.set_stage_tile(16, 16)
        with pytest.raises(WfError):
            s.set_stage_tile(8, 16, 256)


@pytest.mark.parametrize("name", ["hill_rk4", "vardens_rk4"])
def test_fp64_block_forms_give_identical_states(name, params_from_text):
    g = load_golden(name)
    P = params_from_text(g["params"])
    n = int(g["nsteps"])
    (y0, p0), _ = _run(P, g, "fp64", (8, 8, 256), n)
    for shape in [(8, 8, 512)]:
        (y, p), used = _run(P, g, "fp64", shape, n)
        assert used == shape
        assert np.array_equal(y, y0) and np.array_equal(p, p0), shape


@pytest.mark.parametrize("name", ["hill_rk4", "flat_33x33x16_10"])
def test_tma_and_cp_async_tile_loads_give_identical_states(name, params_from_text, monkeypatch):
    """FP32 tiles whose halo does not wrap arrive as one TMA box (re-packed into
    the tile's pair layout); WF_NO_TMA=1 loads every tile by cp.async.  Same
    bits either way, for every compiled form."""
    g = load_golden(name)
    P = params_from_text(g["params"])
    n = int(g["nsteps"])
    for shape in SHAPES32:
        monkeypatch.setenv("WF_NO_TMA", "0")
        (y0, p0), _ = _run(P, g, "fp32", shape, n)
        monkeypatch.setenv("WF_NO_TMA", "1")
        (y, p), _ = _run(P, g, "fp32", shape, n)
        assert np.array_equal(y, y0) and np.array_equal(p, p0), shape


def test_tma_tile_loads_on_a_grid_with_interior_tiles(params_from_text, monkeypatch):
    """A grid with many interior tiles of both widths (64 x 80 x 32, hill case):
    TMA and cp.async loads give bit-identical states after two steps, and all
    forms agree."""
    from wildfires_b200 import configs
    case = configs.hill(Nx=64, Ny=80, Nz=32, Nt=2, L=120.0, H=24.0, jitter=0.3, seed=6)
    P = params_from_text(configs.param_text(case.params))
    y0, p0 = case.fields(P)
    g = {"y0": y0, "p0": p0}
    out = []
    for flag in ("0", "1"):
        monkeypatch.setenv("WF_NO_TMA", flag)
        for shape in SHAPES32:
            (y, p), _ = _run(P, g, "fp32", shape, 2)
            out.append((y, p))
    for y, p in out[1:]:
        assert np.array_equal(y, out[0][0]) and np.array_equal(p, out[0][1])

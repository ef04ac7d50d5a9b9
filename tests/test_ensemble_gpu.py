"""Ensembles: members of different grid sizes stepped together must give
exactly what each member gives when stepped alone (the kernels are
deterministic, so the comparison is bitwise)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _members():
    from wildfires_b200 import configs
    kw = dict(Nz=32, z_max=31 * 0.3125, Nt=4, jitter=0.2)
    return [configs.scenario(33, 48, seed=1, **kw), configs.scenario(65, 40, seed=2, **kw),
            configs.scenario(48, 48, seed=3, **kw)]


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_ensemble_equals_members_alone(prec):
    from wildfires_b200 import Ensemble, Solver, configs
    built = [configs.materialize(c) for c in _members()]
    alone = []
    for P, y0, p0 in built:
        with Solver(P, prec) as s:
            s.upload(y0, p0)
            s.step(4)
            alone.append(s.download())
    with Ensemble([b[0] for b in built], prec) as ens:
        for i, (P, y0, p0) in enumerate(built):
            ens[i].upload(y0, p0)
        ens.step(2)
        ens.step(2)
        ens.synchronize()
        for i in range(len(built)):
            y, p = ens[i].download()
            assert np.array_equal(y, alone[i][0]) and np.array_equal(p, alone[i][1]), i
            assert ens[i].time()[0] == 4


def test_ensemble_members_out_of_step_fall_back_to_eager():
    from wildfires_b200 import Ensemble, Solver, configs
    built = [configs.materialize(c) for c in _members()[:2]]
    with Ensemble([b[0] for b in built], "fp32") as ens:
        for i, (P, y0, p0) in enumerate(built):
            ens[i].upload(y0, p0)
        ens[0].step(1)          # member 0 one step ahead: parities differ
        ens.step(2)
        ens.synchronize()
        n = [ens[i].time()[0] for i in range(2)]
        got = [ens[i].download() for i in range(2)]
    assert n == [3, 2]
    for i, k in enumerate(n):
        P, y0, p0 = built[i]
        with Solver(P, "fp32") as s:
            s.upload(y0, p0)
            s.step(k)
            y, p = s.download()
        assert np.array_equal(got[i][0], y) and np.array_equal(got[i][1], p)


def test_ensemble_with_pressure_tolerance_equals_members_alone():
    """Variable density with a tolerance: each member's fixed point runs as a
    CUDA graph WHILE node inside the ensemble graph (captured on the member's
    stream); results and iteration reports equal the members stepped alone."""
    from wildfires_b200 import Ensemble, Solver, configs
    kw = dict(Nz=32, z_max=31 * 0.3125, Nt=4, jitter=0.2, variable_density=1,
              pressure_solver_iter=20, pressure_solver_tol=1e-9)
    built = [configs.materialize(c) for c in (configs.scenario(33, 48, seed=4, **kw),
                                              configs.scenario(48, 40, seed=5, **kw))]
    alone = []
    for P, y0, p0 in built:
        with Solver(P, "fp64") as s:
            s.upload(y0, p0)
            s.step(3)
            alone.append((s.download(), s.pressure_report()))
    with Ensemble([b[0] for b in built], "fp64") as ens:
        for i, (P, y0, p0) in enumerate(built):
            ens[i].upload(y0, p0)
        ens.step(3)
        ens.synchronize()
        for i in range(len(built)):
            y, p = ens[i].download()
            (ya, pa), rep = alone[i]
            assert np.array_equal(y, ya) and np.array_equal(p, pa), i
            err, it = ens[i].pressure_report()
            assert (err, it) == rep and 0 <= it < 20

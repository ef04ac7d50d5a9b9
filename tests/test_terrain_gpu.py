"""Terrain and immersed-boundary tables on the device (wf_ibm_parameters_device,
wf_set_topography_hills) against the host computation (wf_set_topography,
the restatement of ibm_parameters, src/cu/ibm.cu:57-95, itself pinned to the
reference's parser output in test_parser_golden.py).

The tables are comparisons and one subtraction per node: bit-identical.  The
hill terrain is a sum of exp() terms: the device exp and numpy's may differ
in the last bit, so the terrain is held to 4 ulp-sized relative differences
and the tables to exact equality wherever the two terrains agree bitwise."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _record(params_from_text, case):
    from wildfires_b200 import configs
    return params_from_text(configs.param_text(case.params))


@pytest.mark.parametrize("which", ["hills8", "hill_fixture", "scenario"])
def test_device_ibm_tables_match_host(which, params_from_text):
    from wildfires_b200 import configs
    if which == "hills8":
        case = configs.hills8(Nt=1)
    elif which == "scenario":
        case = configs.ensemble(8)[0]
    else:
        case = None
    if case is None:
        g = load_golden("hill_rk4")
        A, B = params_from_text(g["params"]), params_from_text(g["params"])
    else:
        A, B = _record(params_from_text, case), _record(params_from_text, case)
        topo = case.topography(A)
        if topo is not None:
            A.set_topography(topo)   # host
            B.set_topography(topo)
    B.ibm_on_device()
    assert A.rec.Nz_Y_max == B.rec.Nz_Y_max
    assert np.array_equal(A.cut_nodes(), B.cut_nodes())
    assert np.array_equal(A.nz_y(), B.nz_y())
    assert np.array_equal(A.z_ibm(), B.z_ibm())


@pytest.mark.parametrize("which", ["hills8", "scenario"])
def test_device_hill_terrain_matches_numpy(which, params_from_text):
    from wildfires_b200 import configs
    case = configs.hills8(Nt=1) if which == "hills8" else configs.ensemble(8)[0]
    assert case.hills
    A, B = _record(params_from_text, case), _record(params_from_text, case)
    A.set_topography(case.topography(A))
    B.set_topography_hills(case.hills)
    ta, tb = A.topo(), B.topo()
    scale = np.max(np.abs(ta))
    assert np.max(np.abs(ta - tb)) <= 4 * np.finfo(float).eps * scale
    same = (ta == tb)
    assert same.mean() > 0.5
    assert np.array_equal(A.cut_nodes()[same], B.cut_nodes()[same])
    assert np.array_equal(A.nz_y()[same], B.nz_y()[same])

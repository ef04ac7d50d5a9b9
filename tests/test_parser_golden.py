"""The parser against the reference's own parser (read_parameters_file,
src/cu/parameters.cu:11-523): every scalar and string member of the record and
every derived array, on the files of tests/golden/make_golden_parser.py
(defaults only, every key set, and the line-matching quirks)."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN

# members that point into memory, hold open files, or carry the reference's
# run timestamp (sim_id, save_path: its output directory, parameters.cu:21-24)
SKIP = {"x", "y", "z", "t", "r", "s", "kx", "ky", "Nz_Y", "topography", "cut_nodes", "z_ibm", "log_files",
        "sim_id", "save_path"}

FIX = os.path.join(GOLDEN, "parser_records.npz")
CASES = sorted({k.split("/")[0] for k in np.load(FIX).files}) if os.path.exists(FIX) else []


def _members(rec, prefix=""):
    for name, typ in rec._fields_:
        if name in SKIP:
            continue
        v = getattr(rec, name)
        if isinstance(v, C.Structure):
            yield from _members(v, prefix + name + ".")
        else:
            yield prefix + name, v


@pytest.mark.parametrize("case", CASES)
def test_parser_record_equals_the_reference_parsers(case, params_from_text):
    from wildfires_b200._params import Parameters
    g = np.load(FIX)
    ref = Parameters.from_buffer_copy(g[case + "/record"].tobytes())
    P = params_from_text(str(g[case + "/text"]))
    ours = dict(_members(P.rec))
    theirs = dict(_members(ref))
    assert ours.keys() == theirs.keys()
    # the one deliberate difference: a file without NT leaves the reference's
    # NT at 0, and its time loop then takes n % 0 (solver.cu:245); here NT = Nt
    if theirs["NT"] == 0:
        theirs["NT"] = theirs["Nt"]
    bad = {k: (ours[k], theirs[k]) for k in ours
           if not (ours[k] == theirs[k] or (isinstance(ours[k], float) and np.isnan(ours[k]) and np.isnan(theirs[k])))}
    assert not bad, bad
    r = P.rec
    n = {"x": r.Nx, "y": r.Ny, "z": r.Nz, "t": r.Nt + 1, "kx": r.Nx - 1, "ky": r.Ny - 1, "topography": r.Nx * r.Ny}
    if ref.topo_shape not in (b"flat", b"hill"):
        # the reference fills its terrain only for these shapes (parameters.cu:489-492);
        # otherwise the array is fresh malloc memory, and zeros here
        del n["topography"]
        assert not np.any(np.ctypeslib.as_array(r.topography, shape=(r.Nx * r.Ny,)))
    for nm, size in n.items():
        mine = np.ctypeslib.as_array(getattr(r, nm), shape=(size,))
        np.testing.assert_array_equal(mine, g[case + "/" + nm], err_msg=nm)
    np.testing.assert_array_equal(P.cut_nodes().reshape(-1), g[case + "/cut_nodes"])
    np.testing.assert_array_equal(P.nz_y().reshape(-1), g[case + "/Nz_Y"])


DOMAIN = sorted({k.split("/")[0] for k in np.load(FIX).files if "/file_" in k}) if os.path.exists(FIX) else []


@pytest.mark.parametrize("case", DOMAIN)
def test_domain_files_equal_the_reference_writers(case, tmp_path, params_from_text):
    """wf_save_domain / wf_save_topography against the bytes the reference's
    save_domain / save_topography (output.cu:46-99) write for the same file."""
    from wildfires_b200 import save_domain, save_topography
    g = np.load(FIX)
    P = params_from_text(str(g[case + "/text"]))
    save_domain(P, tmp_path)
    save_topography(P, tmp_path)
    for nm in ("x", "y", "z", "t", "topography", "Nz_Y"):
        with open(tmp_path / (nm + ".bin"), "rb") as f:
            assert f.read() == g[case + "/file_" + nm].tobytes(), nm

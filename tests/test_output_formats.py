"""save_domain and save_topography (reference output.cu:46-99) through the
C-ABI: grid coordinates, the times of the saved steps (n % NT == 0 or
n == Nt), terrain heights and per-column fuel heights in the reference's raw
formats.  Host-only: no GPU needed."""
import numpy as np

from conftest import load_golden


def test_save_domain_and_topography(tmp_path, params_from_text):
    from wildfires_b200 import save_domain, save_topography
    g = load_golden("hill_rk4")
    text = str(g["params"]).replace("NT = 3", "NT = 2")
    P = params_from_text(text)
    r = P.rec
    save_domain(P, tmp_path)
    save_topography(P, tmp_path)
    x = np.ctypeslib.as_array(r.x, shape=(r.Nx,))
    y = np.ctypeslib.as_array(r.y, shape=(r.Ny,))
    t = np.ctypeslib.as_array(r.t, shape=(r.Nt + 1,))
    assert np.array_equal(np.fromfile(tmp_path / "x.bin"), x)
    assert np.array_equal(np.fromfile(tmp_path / "y.bin"), y)
    assert np.array_equal(np.fromfile(tmp_path / "z.bin"), P.z())
    saved = [n for n in range(r.Nt + 1) if n % r.NT == 0 or n == r.Nt]
    assert r.NT == 2 and saved == [0, 2, 3]
    assert np.array_equal(np.fromfile(tmp_path / "t.bin"), t[saved])
    topo = np.ctypeslib.as_array(r.topography, shape=(r.Nx * r.Ny,))
    assert np.array_equal(np.fromfile(tmp_path / "topography.bin"), topo)
    assert np.array_equal(np.fromfile(tmp_path / "Nz_Y.bin", dtype=np.int32), P.nz_y().reshape(-1))

import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_built():
    from wildfires_b200 import build
    build.build()
    import oracle_py
    oracle_py.build()


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    _ensure_built()


def golden_names():
    """Fixtures of the time step (the ic_* fixtures hold initial conditions
    only, parser_records the parsed records)."""
    names = (os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
    return sorted(n for n in names if not n.startswith(("ic_", "parser_")))


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.fixture
def params_from_text(tmp_path):
    """Parse parameter-file text with the library's parser."""
    from wildfires_b200 import read_parameters

    def make(text):
        p = tmp_path / "parameters.txt"
        p.write_text(str(text))
        return read_parameters(p)
    return make


def field_errors(P, a, b):
    """Per-field (max relative, L2 relative) errors; fuel compared where stored."""
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    out = {}
    for q, nm in enumerate("uvwT"):
        x, y = a[q * N:(q + 1) * N], b[q * N:(q + 1) * N]
        out[nm] = _rel(x, y)
    if r.Nz_Y_max:
        nzy = P.nz_y()
        k = np.arange(r.Nz_Y_max)[None, None, :]
        m = (k < nzy[:, :, None]).reshape(-1)
        out["Y"] = _rel(a[4 * N:][m], b[4 * N:][m])
    return out


def _rel(x, y):
    ny = np.linalg.norm(y)
    scale = max(np.max(np.abs(y)), 1e-300)
    linf = float(np.max(np.abs(x - y)) / scale) if x.size else 0.0
    l2 = float(np.linalg.norm(x - y) / max(ny, 1e-300)) if x.size else 0.0
    return linf, l2


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False

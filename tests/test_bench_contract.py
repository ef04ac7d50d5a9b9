"""The reference arm of bench.py prints the one JSON line the benchmark
contract asks for (it runs the reference's host build, so it needs no GPU)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def test_reference_arm_prints_the_contract_line():
    """The full workload (here the flat 128 x 128 x 64 one), W + K steps of the
    reference's own solver with the last K timed, and this repository's
    library never loaded in that process."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_host")):
        pytest.skip("reference host build not present (make -C oracle ref REF=<reference tree>)")
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--config', 'flat', '--steps', '3', "
            "'--warmup', '1']; runpy.run_path('bench.py', run_name='__main__'); "
            "print('LOADED', 'libwildfires_b200' in open('/proc/self/maps').read())")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    assert "LOADED False" in r.stdout, r.stdout[-500:]
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["metric"] == d["unit"] == "Mcell-steps/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 3 and d["warmup"] == 1
    assert d["n_gpus"] == 1
    assert "workload" in d["config"] and d["config"]["grid"] == [128, 128, 64]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and "128x128x64" in cb["sample"]
    assert abs(cb["value"] - d["value"]) <= 1e-4 * max(d["value"], 1.0)
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}

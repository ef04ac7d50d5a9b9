"""Run the REFERENCE's own solver (oracle/_ref/ref_host or ref_gpu, built by
oracle/Makefile from the reference sources) on a synthetic case and read its
outputs back.

TEST INFRASTRUCTURE ONLY: used to pin the oracle and to generate the golden
fixtures under tests/golden/ (tests/golden/make_golden.py), and by bench.py's
reference arm.  The binaries exist only where the reference tree was available
when oracle/Makefile ran.
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def binary(flavour="host"):
    return os.path.join(REF_DIR, "ref_host" if flavour == "host" else "ref_gpu")


def available(flavour="host"):
    return os.path.exists(binary(flavour))


def run(case, mode, flavour="host", parallel=False, timeout=3600, keep=None):
    """Write `case` into a fresh directory, run the driver in `mode` and return
    its outputs as a dict of numpy arrays (plus 'seconds' for step/time)."""
    from wildfires_b200.configs import write_case
    work = tempfile.mkdtemp(prefix="wf_ref_")
    try:
        ppath, P, y0, p0 = write_case(case, work)
        out = os.path.join(work, "out")
        os.makedirs(out)
        cmd = [binary(flavour), mode, "parameters.txt", "out"]
        if parallel:
            cmd.append("parallel")
        env = dict(os.environ)
        r = subprocess.run(cmd, cwd=work, capture_output=True, text=True, timeout=timeout, env=env)
        if r.returncode != 0:
            raise RuntimeError("reference driver failed (%d):\n%s\n%s" % (r.returncode, r.stdout[-2000:], r.stderr[-2000:]))
        res = {"P": P, "y0": y0, "p0": p0, "stdout": r.stdout}
        rec = P.rec
        N = rec.Nx * rec.Ny * rec.Nz
        S = P.state_size
        if mode == "phi":
            res["R"] = np.fromfile(os.path.join(out, "R.bin"))
        elif mode == "rk4":
            res["y1"] = np.fromfile(os.path.join(out, "y1.bin"))
        elif mode == "pressure":
            res["p"] = np.fromfile(os.path.join(out, "p.bin"))
        elif mode == "ic":
            res["ic_y"] = np.fromfile(os.path.join(out, "y0.bin"))
            res["ic_p"] = np.fromfile(os.path.join(out, "p0.bin"))
        elif mode == "params":
            with open(os.path.join(out, "params.bin"), "rb") as f:
                res["record"] = f.read()
            for nm in ("x", "y", "z", "t", "kx", "ky", "topography"):
                res[nm] = np.fromfile(os.path.join(out, nm + ".bin"))
            for nm in ("cut_nodes", "Nz_Y"):
                res[nm] = np.fromfile(os.path.join(out, nm + ".bin"), dtype=np.int32)
        else:
            kv = dict(line.split("=", 1) for line in r.stdout.splitlines() if "=" in line)
            res["seconds"] = float(kv.get("SECONDS", "nan"))
            if mode == "step":
                save = os.path.join(work, kv["SAVE_PATH"].strip())
                nsave = rec.Nt // rec.NT
                y = np.empty(S)
                for q, nm in enumerate("uvwT"):
                    y[q * N:(q + 1) * N] = np.fromfile(os.path.join(save, "%s.bin.%d" % (nm, nsave)))
                y[4 * N:] = np.fromfile(os.path.join(save, "Y.bin.%d" % nsave))
                res["y"] = y
                res["p"] = np.fromfile(os.path.join(save, "p.bin.%d" % nsave))
        if keep:
            shutil.copytree(work, keep, dirs_exist_ok=True)
        return res
    finally:
        shutil.rmtree(work, ignore_errors=True)

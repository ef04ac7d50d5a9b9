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


# ---- the reference's own parameter record, without this repository's library -----
class RefRecord:
    """The record the reference's read_parameters_file (+ ibm_parameters for a
    terrain override) built, read back from the driver's `params` mode, with
    the interface the case builders use (rec, z(), topo(), cut_nodes(),
    nz_y(), state_size).  Its pointer members are meaningless in this process
    (they were the driver's); the arrays come from the driver's files."""

    def __init__(self, outdir):
        from wildfires_b200._params import Parameters
        with open(os.path.join(outdir, "params.bin"), "rb") as f:
            raw = f.read()
        self.rec = Parameters.from_buffer_copy(raw)
        r = self.rec
        self._z = np.fromfile(os.path.join(outdir, "z.bin"))
        self._topo = np.fromfile(os.path.join(outdir, "topography.bin")).reshape(r.Nx, r.Ny)
        self._cut = np.fromfile(os.path.join(outdir, "cut_nodes.bin"), dtype=np.int32).reshape(r.Nx, r.Ny)
        self._nzy = np.fromfile(os.path.join(outdir, "Nz_Y.bin"), dtype=np.int32).reshape(r.Nx, r.Ny)

    @property
    def state_size(self):
        r = self.rec
        return 4 * r.Nx * r.Ny * r.Nz + r.Nx * r.Ny * r.Nz_Y_max

    def z(self):
        return self._z.copy()

    def topo(self):
        return self._topo.copy()

    def cut_nodes(self):
        return self._cut.copy()

    def nz_y(self):
        return self._nzy.copy()


def _driver(flavour, mode, work, parallel=False, timeout=3600):
    cmd = [binary(flavour), mode, "parameters.txt", "out"]
    if parallel:
        cmd.append("parallel")
    os.makedirs(os.path.join(work, "out"), exist_ok=True)
    r = subprocess.run(cmd, cwd=work, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("reference driver failed (%d):\n%s\n%s" % (r.returncode, r.stdout[-2000:], r.stderr[-2000:]))
    return r.stdout


def write_case_reference(case, work, **overrides):
    """Write `case` for the reference driver using the reference's own parser
    and immersed-boundary precompute (the driver's params mode) to build the
    record the fields are generated on -- this repository's library is not
    loaded.  Returns the RefRecord and the initial fields."""
    from wildfires_b200.configs import param_text
    params = dict(case.params)
    params["input_path"] = "in/"
    params.update(overrides)
    with open(os.path.join(work, "parameters.txt"), "w") as f:
        f.write(param_text(params))
    _driver("host", "params", work)
    P = RefRecord(os.path.join(work, "out"))
    topo = case.topography(P)
    if topo is not None:
        np.ascontiguousarray(topo, dtype=np.float64).tofile(os.path.join(work, "topography.bin"))
        _driver("host", "params", work)             # the driver applies topography.bin and ibm_parameters
        P = RefRecord(os.path.join(work, "out"))
    y0, p0 = case.fields(P)
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    ind = os.path.join(work, "in")
    os.makedirs(ind, exist_ok=True)
    for q, nm in enumerate("uvwT"):
        y0[q * N:(q + 1) * N].tofile(os.path.join(ind, nm + ".bin"))
    y0[4 * N:].tofile(os.path.join(ind, "Y.bin"))
    p0.tofile(os.path.join(ind, "p.bin"))
    return P


def time_steps(case, warmup, timeout=7200):
    """The reference's own solver (host build, all cores) on `case`, its Nt
    time steps in one run; the per-step times come from its own step timer
    (solver.cu:178-265 prints the running average every time_step_log steps;
    here every step).  Returns the seconds of the steps after the first
    `warmup` and the record."""
    work = tempfile.mkdtemp(prefix="wf_reftime_")
    try:
        n = int(case.params["Nt"])
        P = write_case_reference(case, work, time_step_log=1)
        out = _driver("host", "time", work, parallel=True, timeout=timeout)
        avg = {}
        for line in out.splitlines():
            if line.startswith("Time step:") and "Average time:" in line:
                a, b = line.split(",")
                avg[int(a.split(":")[1])] = float(b.split(":")[1].strip().split()[0])
        if n not in avg:
            raise RuntimeError("reference step times missing from its output:\n" + out[-2000:])
        cum_n = avg[n] * n
        cum_w = avg[warmup] * warmup if warmup > 0 else 0.0
        return cum_n - cum_w, P
    finally:
        shutil.rmtree(work, ignore_errors=True)

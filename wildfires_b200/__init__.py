"""B200 coupled atmosphere-wildfire solver: Python host API over the C-ABI.

The time step of the reference model (dsanmartinreyes' wildfires, src/cu) runs
as hand-written sm_100a CUDA kernels in libwildfires_b200.so; this module only
moves host buffers in and out.  Typical use::

    from wildfires_b200 import read_parameters, Solver
    P = read_parameters("parameters.txt")
    with Solver(P, precision="fp32") as s:
        s.upload(y0, p0)          # packed [u|v|w|T|Y] FP64 host state, pressure
        s.step(100)
        y, p = s.download()
"""
import ctypes as C

import numpy as np

from ._abi import WF_FP32_STENCIL, WF_FP64, WfDiag, WfError, WfReport, check, lib
from ._params import Parameters

__all__ = ["Params", "Solver", "Ensemble", "read_parameters", "WfError", "Parameters"]

_dp = C.POINTER(C.c_double)


def _ptr(a):
    return a.ctypes.data_as(_dp)


class Params:
    """A parsed parameter record whose host arrays are owned by the library."""

    def __init__(self, rec):
        self.rec = rec
        self._owned = True

    @property
    def shape(self):
        r = self.rec
        return r.Nx, r.Ny, r.Nz

    @property
    def state_size(self):
        return int(lib().wf_state_size(C.byref(self.rec)))

    def array(self, name, n):
        p = getattr(self.rec, name)
        return np.ctypeslib.as_array(p, shape=(n,)).copy()

    def z(self):
        return self.array("z", self.rec.Nz)

    def nz_y(self):
        r = self.rec
        return np.ctypeslib.as_array(r.Nz_Y, shape=(r.Nx * r.Ny,)).copy().reshape(r.Nx, r.Ny)

    def topo(self):
        """Terrain height, Nx x Ny."""
        r = self.rec
        return np.ctypeslib.as_array(r.topography, shape=(r.Nx * r.Ny,)).copy().reshape(r.Nx, r.Ny)

    def cut_nodes(self):
        r = self.rec
        return np.ctypeslib.as_array(r.cut_nodes, shape=(r.Nx * r.Ny,)).copy().reshape(r.Nx, r.Ny)

    def set_topography(self, topo):
        t = np.ascontiguousarray(topo, dtype=np.float64).reshape(-1)
        r = self.rec
        assert t.size == r.Nx * r.Ny
        check(lib().wf_set_topography(C.byref(r), _ptr(t)), "wf_set_topography")

    def set_topography_hills(self, hills):
        """Terrain of Gaussian hills [(cx, cy, height, width), ...] and its
        immersed-boundary tables, computed on the current GPU."""
        h = np.ascontiguousarray(np.asarray(hills, dtype=np.float64).reshape(-1))
        check(lib().wf_set_topography_hills(C.byref(self.rec), len(h) // 4, _ptr(h)), "wf_set_topography_hills")

    def ibm_on_device(self):
        """Recompute the immersed-boundary tables of the current terrain on the GPU."""
        check(lib().wf_ibm_parameters_device(C.byref(self.rec)), "wf_ibm_parameters_device")

    def z_ibm(self):
        r = self.rec
        return np.ctypeslib.as_array(r.z_ibm, shape=(r.Nx * r.Ny * r.Nz,)).copy()

    def free(self):
        if self._owned:
            lib().wf_free_parameters(C.byref(self.rec))
            self._owned = False

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def read_parameters(path):
    """Parse a reference-format parameter file (no output directory is created)."""
    rec = Parameters()
    check(lib().wf_read_parameters(str(path).encode(), C.byref(rec)), "wf_read_parameters")
    return Params(rec)


def _dir(directory):
    d = str(directory)
    return (d if d.endswith("/") else d + "/").encode()


def save_fields(params, directory, n, y, p):
    """Write <dir>u.bin.<n> ... p.bin.<n> (reference save_data format)."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    p = np.ascontiguousarray(p, dtype=np.float64)
    check(lib().wf_save_fields(C.byref(params.rec), _dir(directory), int(n), _ptr(y), _ptr(p)), "wf_save_fields")


def save_domain(params, directory):
    """Write <dir>x.bin, y.bin, z.bin, t.bin (reference save_domain format)."""
    check(lib().wf_save_domain(C.byref(params.rec), _dir(directory)), "wf_save_domain")


def save_topography(params, directory):
    """Write <dir>topography.bin and Nz_Y.bin (reference save_topography format)."""
    check(lib().wf_save_topography(C.byref(params.rec), _dir(directory)), "wf_save_topography")


def load_fields(params, directory):
    """Read <dir>u.bin ... p.bin into a packed state and p (reference input format)."""
    r = params.rec
    y = np.empty(params.state_size)
    p = np.empty(r.Nx * r.Ny * r.Nz)
    d = str(directory)
    if not d.endswith("/"):
        d += "/"
    check(lib().wf_load_fields(C.byref(r), d.encode(), _ptr(y), _ptr(p)), "wf_load_fields")
    return y, p


class Solver:
    """A solver context on the current CUDA device."""

    def __init__(self, params, precision="fp64"):
        self.params = params
        prec = {"fp64": WF_FP64, "fp32": WF_FP32_STENCIL}[precision]
        self.precision = precision
        h = C.c_void_p()
        check(lib().wf_create(C.byref(params.rec), prec, C.byref(h)), "wf_create")
        self._h = h
        r = params.rec
        self.N = r.Nx * r.Ny * r.Nz
        self.S = params.state_size

    def close(self):
        if self._h:
            lib().wf_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, y, p):
        y = np.ascontiguousarray(y, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        assert y.size == self.S and p.size == self.N
        check(lib().wf_upload_state(self._h, _ptr(y), _ptr(p)), "wf_upload_state")

    def download(self):
        y = np.empty(self.S)
        p = np.empty(self.N)
        check(lib().wf_download_state(self._h, _ptr(y), _ptr(p)), "wf_download_state")
        return y, p

    def step(self, n=1):
        check(lib().wf_step(self._h, int(n)), "wf_step")

    def synchronize(self):
        check(lib().wf_synchronize(self._h), "wf_synchronize")

    def time(self):
        n = C.c_int()
        t = C.c_double()
        check(lib().wf_time(self._h, C.byref(n), C.byref(t)), "wf_time")
        return n.value, t.value

    def diagnostics(self, allow_nan=False):
        d = WfDiag()
        s = lib().wf_diagnostics(self._h, C.byref(d))
        if not (allow_nan and s == 6):
            check(s, "wf_diagnostics")
        return {f: getattr(d, f) for f, _ in WfDiag._fields_}

    def stage_tile(self):
        """(TI, TJ, threads) of the fused stage pass (picked by the first step)."""
        ti, tj, nt = C.c_int(), C.c_int(), C.c_int()
        check(lib().wf_stage_tile(self._h, C.byref(ti), C.byref(tj), C.byref(nt)), "wf_stage_tile")
        return ti.value, tj.value, nt.value

    def set_stage_tile(self, ti, tj, threads=0):
        check(lib().wf_set_stage_tile(self._h, int(ti), int(tj), int(threads)), "wf_set_stage_tile")

    def initial_conditions(self):
        """The reference's initial conditions, generated on the GPU (time level 0)."""
        check(lib().wf_initial_conditions(self._h), "wf_initial_conditions")

    def timestep_reports(self):
        """The reference's checkpoint report (functions.cu:82-185) reduced on the GPU."""
        r = WfReport()
        check(lib().wf_timestep_reports(self._h, C.byref(r)), "wf_timestep_reports")
        return {f: getattr(r, f) for f, _ in WfReport._fields_}

    def dump_async(self, directory, n):
        """Checkpoint the current state to <dir>*.bin.<n> in the background."""
        check(lib().wf_dump_async(self._h, _dir(directory), int(n)), "wf_dump_async")

    def dump_wait(self):
        check(lib().wf_dump_wait(self._h), "wf_dump_wait")

    def phi(self, R_old):
        R_old = np.ascontiguousarray(R_old, dtype=np.float64)
        out = np.empty(self.S)
        check(lib().wf_phi(self._h, _ptr(R_old), _ptr(out)), "wf_phi")
        return out

    def rk(self, y_n):
        """The RK stages of one step (no pressure solve, no projection)."""
        y_n = np.ascontiguousarray(y_n, dtype=np.float64)
        out = np.empty(self.S)
        check(lib().wf_rk(self._h, _ptr(y_n), _ptr(out)), "wf_rk")
        return out

    def pressure_report(self):
        """(error, max_iter) as the reference's iterative pressure solve reports them."""
        e = C.c_double()
        m = C.c_int()
        check(lib().wf_pressure_report(self._h, C.byref(e), C.byref(m)), "wf_pressure_report")
        return e.value, m.value

    def pressure(self, y_np1, y_n, p):
        a = np.ascontiguousarray(y_np1, dtype=np.float64)
        b = np.ascontiguousarray(y_n, dtype=np.float64)
        pp = np.array(p, dtype=np.float64, copy=True)
        it = C.c_int()
        check(lib().wf_pressure(self._h, _ptr(a), _ptr(b), _ptr(pp), C.byref(it)), "wf_pressure")
        return pp, it.value

    def device_state(self):
        y = C.c_void_p()
        p = _dp()
        check(lib().wf_device_state(self._h, C.byref(y), C.byref(p)), "wf_device_state")
        return y.value, C.cast(p, C.c_void_p).value

    def stream(self):
        return lib().wf_stream(self._h)

    def launches_per_step(self):
        return lib().wf_launches_per_step(self._h)

    def profile(self, nsteps=1):
        """Per-kernel-kind device time over nsteps eager steps: {name: (total_ms, launches)}."""
        from ._abi import WF_NPHASES
        ms = (C.c_double * WF_NPHASES)()
        n = (C.c_int * WF_NPHASES)()
        check(lib().wf_profile_phases(self._h, int(nsteps), ms, n), "wf_profile_phases")
        return {lib().wf_phase_name(q).decode(): (ms[q], n[q]) for q in range(WF_NPHASES)}


class _Member(Solver):
    """A member context owned by an Ensemble (not destroyed on its own)."""

    def __init__(self, params, handle, precision):
        self.params = params
        self.precision = precision
        self._h = handle
        r = params.rec
        self.N = r.Nx * r.Ny * r.Nz
        self.S = params.state_size

    def close(self):
        self._h = None


class Ensemble:
    """Independent members stepped together (one CUDA graph per ensemble step,
    one concurrent branch per member)."""

    def __init__(self, params_list, precision="fp32"):
        prec = {"fp64": WF_FP64, "fp32": WF_FP32_STENCIL}[precision]
        self.params = list(params_list)
        recs = (Parameters * len(self.params))(*[p.rec for p in self.params])
        h = C.c_void_p()
        check(lib().wf_ensemble_create(recs, len(self.params), prec, C.byref(h)), "wf_ensemble_create")
        self._h = h
        self.members = [_Member(p, C.c_void_p(lib().wf_ensemble_member(h, i)), precision)
                        for i, p in enumerate(self.params)]

    def __len__(self):
        return len(self.members)

    def __getitem__(self, i):
        return self.members[i]

    def step(self, n=1):
        check(lib().wf_ensemble_step(self._h, int(n)), "wf_ensemble_step")

    def stream(self):
        """The cudaStream_t (as an int) ensemble steps are launched on."""
        return lib().wf_ensemble_stream(self._h) or 0

    def synchronize(self):
        check(lib().wf_ensemble_synchronize(self._h), "wf_ensemble_synchronize")

    def close(self):
        if self._h:
            lib().wf_ensemble_destroy(self._h)
            self._h = None
            for m in self.members:
                m.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""Learned subgrid closure: data from box-filtered fine runs, training on the
GPU with the library's own kernels, and evaluation against Smagorinsky.

The closure replaces C_s^2 in mu_sgs = rho C_s^2 Delta^2 |S| by c(x) =
softplus(MLP(x)), x = 12 resolved-scale features (strain rate, vorticity,
grad T; wildfires_b200/csrc/closure.cu).  Training data come from this
solver's own fine-grid runs:

* a fine run on a grid with Nf - 1 = 4 (Nc - 1) nodes per direction;
* every `every` steps its u, v, w, T are box-filtered (width 4 fine spacings,
  trapezoid weights 1,2,2,2,1 / 8 per direction, periodic in x and y) onto
  the coarse nodes;
* the target is the local coefficient that makes the Smagorinsky form carry
  the resolved-scale energy transfer of the true subgrid stress
  tau_ij = F(u_i u_j) - F(u_i) F(u_j):
      c* = -tau^d_ij S_ij / (2 S_kl S_kl) / (Delta_c^2 |S|),  clipped to [0, 0.3],
  with S the strain rate of the filtered velocity on the coarse grid and
  Delta_c the coarse filter width (the projection of tau on the eddy-viscosity
  form, evaluated a priori);
* features are those of the kernel, computed on the filtered fields.

Evaluation runs the coarse grid with Smagorinsky and with the trained network
and compares both with the filtered fine run: per-field relative L2, the
downwind fire-front position and the burned fuel fraction.
"""
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NIN, NH = 12, 64
NPARAM = NH * NIN + NH + NH * NH + NH + NH + 1
FACTOR = 4


# ---- parameter vectors --------------------------------------------------------
def smagorinsky_params(C_s=0.173):
    """Weights that give c = C_s^2 everywhere (the Smagorinsky closure)."""
    th = np.zeros(NPARAM + NIN, dtype=np.float32)
    c = C_s * C_s
    th[NPARAM - 1] = math.log(math.expm1(c))          # softplus^-1
    th[NPARAM:] = 1.0
    return th


def init_params(seed=0, scales=None, c0=0.03):
    """Xavier-uniform weights, zero biases, output bias at softplus^-1(c0)."""
    rng = np.random.default_rng(seed)
    th = np.zeros(NPARAM + NIN, dtype=np.float32)
    o = 0
    for fan_out, fan_in in ((NH, NIN), (NH, NH), (1, NH)):
        n = fan_out * fan_in
        lim = math.sqrt(6.0 / (fan_in + fan_out))
        th[o:o + n] = rng.uniform(-lim, lim, n)
        o += n + (fan_out if fan_out > 1 else 0)      # skip the bias block that follows
    th[NPARAM - 1] = math.log(math.expm1(c0))
    th[NPARAM:] = 1.0 if scales is None else scales
    return th


# ---- filtering and targets ------------------------------------------------------
def _box1d(f, axis, periodic):
    """Trapezoid box of width 4 spacings at every 4th node along `axis`."""
    w = np.array([1, 2, 2, 2, 1], dtype=np.float64) / 8.0
    f = np.moveaxis(f, axis, 0)
    n = f.shape[0]
    nc = (n - 1) // FACTOR + 1
    out = np.zeros((nc,) + f.shape[1:])
    for c in range(nc):
        for q, wq in enumerate(w):
            i = FACTOR * c + q - 2
            if periodic:
                i %= (n - 1)
            else:
                i = min(max(i, 0), n - 1)
            out[c] += wq * f[i]
    return np.moveaxis(out, 0, axis)


def box_filter(f):
    """Fine [Nfx, Nfy, Nfz] -> coarse [Nc...]: periodic in x, y, clamped in z."""
    return _box1d(_box1d(_box1d(f, 0, True), 1, True), 2, False)


def _grad(f, dx, dy, z):
    n0, n1 = f.shape[0] - 1, f.shape[1] - 1
    ip, im = np.r_[1:n0, 0, 1], np.r_[n0 - 1, 0:n0 - 1, n0 - 1]
    jp, jm = np.r_[1:n1, 0, 1], np.r_[n1 - 1, 0:n1 - 1, n1 - 1]
    gx = (f[ip] - f[im]) / (2 * dx)
    gy = (f[:, jp] - f[:, jm]) / (2 * dy)
    gz = np.zeros_like(f)
    gz[:, :, 1:-1] = (f[:, :, 2:] - f[:, :, :-2]) / (z[2:] - z[:-2])[None, None, :]
    return gx, gy, gz


def features(u, v, w, T, dx, dy, z):
    """The kernel's 12 features (walls zero) on a grid: [Nx, Ny, Nz, 12]."""
    dz = np.r_[z[1:] - z[:-1], z[-1] - z[-2]]
    delta = np.cbrt(dx * dy * dz)[None, None, :]
    (ux, uy, uz), (vx, vy, vz), (wx, wy, wz), (Tx, Ty, Tz) = (_grad(q, dx, dy, z) for q in (u, v, w, T))
    sv, st = delta, delta * 0.01
    F = np.stack([ux * sv, vy * sv, wz * sv, 0.5 * (uy + vx) * sv, 0.5 * (uz + wx) * sv, 0.5 * (vz + wy) * sv,
                  (wy - vz) * sv, (uz - wx) * sv, (vx - uy) * sv, Tx * st, Ty * st, Tz * st], axis=-1)
    F[:, :, 0] = 0.0
    F[:, :, -1] = 0.0
    return F


def targets(uf, vf, wf, dxc, dyc, zc):
    """c* at the coarse nodes from fine velocities (see the module text)."""
    U = [box_filter(q) for q in (uf, vf, wf)]
    g = [_grad(q, dxc, dyc, zc) for q in U]                # g[i][j] = d U_i / d x_j
    S = [[0.5 * (g[i][j] + g[j][i]) for j in range(3)] for i in range(3)]
    tau = [[box_filter(a * b) - U[i] * U[j] for j, b in enumerate((uf, vf, wf))] for i, a in enumerate((uf, vf, wf))]
    tr = (tau[0][0] + tau[1][1] + tau[2][2]) / 3.0
    SS = sum(S[i][j] * S[i][j] for i in range(3) for j in range(3))
    tS = sum((tau[i][j] - (tr if i == j else 0.0)) * S[i][j] for i in range(3) for j in range(3))
    dz = np.r_[zc[1:] - zc[:-1], zc[-1] - zc[-2]]
    d2 = np.cbrt(dxc * dyc * dz) ** 2
    modS = np.sqrt(2.0 * SS)
    nu = -tS / np.maximum(2.0 * SS, 1e-30)
    c = nu / np.maximum(d2[None, None, :] * modS, 1e-30)
    c = np.clip(c, 0.0, 0.3)
    c[:, :, 0] = c[:, :, -1] = 0.0
    return c


# ---- cases ----------------------------------------------------------------------
def study_case(Nc=(33, 33, 9), fine=False, seed=0, Nt=120, dt=0.002, L=100.0, H=20.0, gust=1.0, Y_h=0.1, **kw):
    """The closure study family: flat terrain, log wind with seeded velocity
    fluctuations (`gust` m/s, on the fine grid's scale so that the coarse grid
    does not resolve them), one hot spot; the fine grid has 4x the intervals
    of the coarse one on the same box.  The fuel layer (Y_h = 0.1 m) is
    thinner than one cell on both grids, so the cut-node rule removes it and
    the case is a buoyant thermal (800 K, 2 m deep) carried by the wind: the
    stiff Arrhenius source of a burning layer limits RK4 to temperatures below
    about 950 K at these steps, which a burning fine grid exceeds.  The coarse
    case starts from the box-filtered fine initial state."""
    from . import configs
    N = tuple(FACTOR * (n - 1) + 1 for n in Nc) if fine else Nc
    rng = np.random.default_rng(seed)
    params = configs.base_params(N[0], N[1], N[2], Nt, L, L, H, Nt * dt, Y_h=Y_h, **kw)
    u_r = rng.uniform(3, 6)
    xc, yc = rng.uniform(0.2, 0.4) * L, rng.uniform(0.35, 0.65) * L

    def fine_fields(P):
        x, y, z = configs._grid(P)
        X, Yg, Z = np.meshgrid(x, y, z, indexing="ij")
        u = configs.log_wind(Z, u_r)
        v = np.zeros_like(u)
        w = np.zeros_like(u)
        frng = np.random.default_rng(seed + 7)
        shape = u.shape
        for f in (u, v, w):
            f += gust * frng.standard_normal(shape) * (Z > 0)
        T = configs.T_AMB + np.where(Z < 2.0, 500.0 * np.exp(-((X - xc) ** 2 + (Yg - yc) ** 2) / 18.0), 0.0)
        Y = np.ones_like(u)
        return u, v, w, T, Y

    def fields(P):
        if fine:
            return configs._finish(P, *fine_fields(P), None, 0.0)
        Pf, _, _ = configs.materialize(study_case(Nc, True, seed, Nt, dt, L, H, gust, Y_h, **kw))
        u, v, w, T, Y = (box_filter(q) for q in fine_fields(Pf))
        return configs._finish(P, u, v, w, T, np.ones_like(u), None, 0.0)

    return configs.Case("closure_study", params, fields)


def _unpack(P, y):
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    sh = (r.Nx, r.Ny, r.Nz)
    return [y[q * N:(q + 1) * N].reshape(sh) for q in range(4)]


def fine_snapshots(seed, Nc, steps, every, precision="fp32", **kw):
    """Yield (step, u, v, w, T) of the fine run every `every` steps (kw: study_case)."""
    from . import Solver, configs
    P, y0, p0 = configs.materialize(study_case(Nc, fine=True, seed=seed, Nt=steps, **kw))
    with Solver(P, precision) as s:
        s.upload(y0, p0)
        for n in range(every, steps + 1, every):
            s.step(every)
            y, _ = s.download()
            yield n, P, y


def dataset(seeds, Nc=(33, 33, 9), steps=120, every=12, **kw):
    """Features (unnormalised) and targets at interior coarse nodes (samples
    with a non-finite value are dropped; kw: study_case)."""
    from . import configs
    Pc, _, _ = configs.materialize(study_case(Nc, seed=0, Nt=1, **kw))
    r = Pc.rec
    zc = Pc.z()
    X, Yt = [], []
    for sd in seeds:
        for n, Pf, y in fine_snapshots(sd, Nc, steps, every, **kw):
            uf, vf, wf, Tf = _unpack(Pf, y)
            F = features(box_filter(uf), box_filter(vf), box_filter(wf), box_filter(Tf), r.dx, r.dy, zc)
            c = targets(uf, vf, wf, r.dx, r.dy, zc)
            X.append(F[:-1, :-1, 1:-1].reshape(-1, NIN))
            Yt.append(c[:-1, :-1, 1:-1].reshape(-1))
    X, Yt = np.concatenate(X), np.concatenate(Yt)
    ok = np.isfinite(X).all(axis=1) & np.isfinite(Yt)
    return X[ok].astype(np.float32), Yt[ok].astype(np.float32)


# ---- training -------------------------------------------------------------------
def train(X, y, steps=3000, batch=8192, lr=1e-3, seed=0):
    """Train with the library's kernels; returns (params, loss history)."""
    import ctypes as C
    from ._abi import check, lib
    scales = (1.0 / np.maximum(X.std(0), 1e-12)).astype(np.float32)
    th = init_params(seed, scales, c0=float(np.mean(y)))
    xn = np.ascontiguousarray(X * scales, dtype=np.float32)
    yy = np.ascontiguousarray(y, dtype=np.float32)
    hist = np.zeros(steps)
    fp = C.POINTER(C.c_float)
    check(lib().wf_mlp_train(th.ctypes.data_as(fp), xn.ctypes.data_as(fp), yy.ctypes.data_as(fp), len(yy), steps,
                             batch, lr, seed, hist.ctypes.data_as(C.POINTER(C.c_double))), "wf_mlp_train")
    return th, hist


def predict(th, X):
    """The network's coefficient for rows of unnormalised features X (n x 12),
    evaluated by the solver's own BF16 tensor-core inference kernel on the
    current GPU (wf_closure_predict)."""
    import ctypes as C
    from ._abi import check, lib
    th32 = np.ascontiguousarray(th, dtype=np.float32)
    X32 = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, NIN)
    out = np.empty(len(X32), dtype=np.float32)
    fp = C.POINTER(C.c_float)
    check(lib().wf_closure_predict(th32.ctypes.data_as(fp), X32.ctypes.data_as(fp), len(X32), out.ctypes.data_as(fp)),
          "wf_closure_predict")
    return out.astype(np.float64)


# ---- evaluation -----------------------------------------------------------------
def front_position(P, y, T_thr=500.0):
    """Largest x at which any ground-adjacent cell (k = 1) exceeds T_thr."""
    T = _unpack(P, y)[3]
    hot = np.where((T[:-1, :-1, 1] > T_thr).any(axis=1))[0]
    return float(hot.max() * P.rec.dx) if hot.size else float("nan")


def burned_fraction(P, y, y0):
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    return float(1.0 - y[4 * N:].sum() / y0[4 * N:].sum())


def evaluate(th, seed=100, Nc=(33, 33, 9), steps=120, precision="fp32", **kw):
    """Coarse runs with Smagorinsky and with the network against the filtered
    fine run (kw: study_case)."""
    import ctypes as C
    from . import Solver, configs
    from ._abi import check, lib
    Pf, yf0, pf0 = configs.materialize(study_case(Nc, fine=True, seed=seed, Nt=steps, **kw))
    t0 = time.perf_counter()
    with Solver(Pf, precision) as s:
        s.upload(yf0, pf0)
        s.step(steps)
        yf, _ = s.download()
    t_fine = time.perf_counter() - t0
    Pc, yc0, pc0 = configs.materialize(study_case(Nc, seed=seed, Nt=steps, **kw))
    truth = np.concatenate([box_filter(q).reshape(-1) for q in _unpack(Pf, yf)])
    rc = Pc.rec
    Nc_ = rc.Nx * rc.Ny * rc.Nz
    out = {"fine_seconds": t_fine, "dx_coarse": rc.dx}
    for name, params in (("smagorinsky", None), ("mlp", th)):
        with Solver(Pc, precision) as s:
            if params is not None:
                p = np.ascontiguousarray(params, dtype=np.float32)
                check(lib().wf_set_closure(s._h, 1, p.ctypes.data_as(C.POINTER(C.c_float))), "wf_set_closure")
            s.upload(yc0, pc0)
            t0 = time.perf_counter()
            s.step(steps)
            y, _ = s.download()
            tc = time.perf_counter() - t0
        errs = {f: float(np.linalg.norm(y[q * Nc_:(q + 1) * Nc_] - truth[q * Nc_:(q + 1) * Nc_]) /
                         max(np.linalg.norm(truth[q * Nc_:(q + 1) * Nc_]), 1e-30)) for q, f in enumerate("uvwT")}
        yt = np.concatenate([truth, y[4 * Nc_:]])
        out[name] = {"rel_l2": errs, "front_m": front_position(Pc, y), "seconds": tc,
                     "burned": burned_fraction(Pc, y, yc0)}
    out["filtered_fine"] = {"front_m": front_position(Pc, np.concatenate([truth, yc0[4 * Nc_:]])),
                            "burned_fine": burned_fraction(Pf, yf, yf0)}
    return out


def cost_study(th, Nc=(65, 65, 17), steps=40, precision="fp32", **kw):
    """Cost of the 4x refinement at a size where the GPU, not launch latency,
    sets the pace: seconds per step of the fine run and of the coarse run
    with Smagorinsky and with the network, the same time step for both (the
    study's setting), timed around device synchronisations after a warm-up
    that also records the step graphs.  Only cost is measured here; the
    accuracy comparison is `evaluate`."""
    import ctypes as C
    from . import Solver, configs
    from ._abi import check, lib
    out = {"coarse_grid": list(Nc), "fine_grid": [FACTOR * (n - 1) + 1 for n in Nc], "steps": steps}
    runs = (("fine", True, None), ("smagorinsky", False, None), ("mlp", False, th))
    for name, fine, params in runs:
        P, y0, p0 = configs.materialize(study_case(Nc, fine=fine, seed=100, Nt=steps, **kw))
        with Solver(P, precision) as s:
            if params is not None:
                p = np.ascontiguousarray(params, dtype=np.float32)
                check(lib().wf_set_closure(s._h, 1, p.ctypes.data_as(C.POINTER(C.c_float))), "wf_set_closure")
            s.upload(y0, p0)
            s.step(4)
            s.synchronize()
            t0 = time.perf_counter()
            s.step(steps)
            s.synchronize()
            out[name + "_ms_per_step"] = (time.perf_counter() - t0) / steps * 1e3
    out["fine_over_mlp"] = out["fine_ms_per_step"] / out["mlp_ms_per_step"]
    out["fine_over_smagorinsky"] = out["fine_ms_per_step"] / out["smagorinsky_ms_per_step"]
    return out


def main(argv=None):
    """python -m wildfires_b200.closure [out.npy] [--coarse NX,NY,NZ] [--steps N]
    [--gust G]: build the dataset from fine runs (seeds 0-2, a snapshot every
    tenth of the horizon), train, score a priori and a posteriori on seed 100,
    time the refinement at the same size, save the parameters."""
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m wildfires_b200.closure")
    ap.add_argument("out", nargs="?", default="closure_params.npy")
    ap.add_argument("--coarse", default="33,33,9", help="coarse grid nodes; the fine grid has 4x the intervals")
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--gust", type=float, default=1.0, help="fine-scale velocity fluctuations, m/s")
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=8192)
    args = ap.parse_args(sys.argv[1:] if argv is None else argv)
    Nc = tuple(int(v) for v in args.coarse.split(","))
    every = max(args.steps // 10, 1)
    kw = {"gust": args.gust}
    X, y = dataset([0, 1, 2], Nc, args.steps, every, **kw)
    th, hist = train(X, y, steps=args.train_steps, batch=args.batch)
    np.save(args.out, th)
    # a priori on the held-out seed: the solver's tensor-core inference against c*
    Xh, yh = dataset([100], Nc, args.steps, every, **kw)
    c = predict(th, Xh)
    cs2 = float(configs_C_s()) ** 2
    res = evaluate(th, 100, Nc, args.steps, **kw)
    res["apriori"] = {"mse_network": float(np.mean((c - yh) ** 2)), "mse_smagorinsky": float(np.mean((cs2 - yh) ** 2)),
                      "mse_best_constant": float(np.var(yh)), "samples": int(len(yh))}
    res["cost"] = cost_study(th, Nc, **kw)
    res["train"] = {"samples": int(len(y)), "loss_first": float(hist[0]), "loss_last": float(np.mean(hist[-50:])),
                    "target_mean": float(y.mean())}
    res["case"] = {"coarse": list(Nc), "steps": args.steps, "gust": args.gust}
    print(json.dumps(res))
    return res


def configs_C_s():
    """The Smagorinsky constant of the study cases."""
    from . import configs
    return configs.base_params(9, 9, 9, 1, 1.0, 1.0, 1.0, 1.0)["C_s"]


if __name__ == "__main__":
    main()

"""CPU oracle of the learned subgrid closure (TEST INFRASTRUCTURE ONLY).

A float64 numpy statement of the closure network and its training step, used
to check the GPU kernels (wildfires_b200/csrc/closure.cu): features, forward
pass, loss, gradients and the Adam update.  The closure has no counterpart in
the reference; it replaces the Smagorinsky coefficient C_s^2 of
mu_sgs = rho (C_s Delta)^2 |S| (reference pde.cu:745) by a learned local
coefficient c(x) = softplus(MLP(x)).

Parameter vector (float32 on the device), in this order:
  W1 [64][12], b1 [64], W2 [64][64], b2 [64], W3 [64], b3 [1]   (5057 values)
followed by 12 feature scales (x_hat = x * scale).
"""
import numpy as np

NIN, NH = 12, 64
SIZES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH,)), ("b3", (1,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)
NTOTAL = NPARAM + NIN
GELU_K = np.sqrt(2.0 / np.pi)


def unpack(theta):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).reshape(-1) for name, _ in SIZES])


def gelu(x):
    """tanh form of GELU (Hendrycks & Gimpel)."""
    return 0.5 * x * (1.0 + np.tanh(GELU_K * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(GELU_K * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_K * (1.0 + 3 * 0.044715 * x * x)


def softplus(x):
    return np.where(x > 20.0, x, np.log1p(np.exp(np.minimum(x, 20.0))))


def sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def forward(theta, xhat):
    """Coefficient c = softplus(o) for normalised features xhat [n, 12]."""
    p = unpack(theta)
    a1 = xhat @ p["W1"].T + p["b1"]
    h1 = gelu(a1)
    a2 = h1 @ p["W2"].T + p["b2"]
    h2 = gelu(a2)
    o = h2 @ p["W3"] + p["b3"][0]
    return softplus(o), (a1, h1, a2, h2, o)


def loss_and_grad(theta, xhat, y):
    """Mean squared error of c against y and its gradient (same packing)."""
    p = unpack(theta)
    n = xhat.shape[0]
    c, (a1, h1, a2, h2, o) = forward(theta, xhat)
    r = c - y
    loss = np.mean(r * r)
    g_o = 2.0 * r / n * sigmoid(o)
    g = {"W3": h2.T @ g_o, "b3": np.array([g_o.sum()])}
    g_a2 = np.outer(g_o, p["W3"]) * gelu_grad(a2)
    g["W2"] = g_a2.T @ h1
    g["b2"] = g_a2.sum(0)
    g_a1 = (g_a2 @ p["W2"]) * gelu_grad(a1)
    g["W1"] = g_a1.T @ xhat
    g["b1"] = g_a1.sum(0)
    return loss, pack(g)


def adam(theta, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba) at step count t >= 1."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v


def features(u, v, w, T, dx, dy, z, delta, u0=1.0, t0=100.0):
    """The 12 closure features at interior nodes of fields shaped [Nx, Ny, Nz]
    (periodic x, y with period N-1; central differences in z on the grid z):
    S11, S22, S33, S12, S13, S23, the vorticity (3) and grad T (3); velocity
    gradients scaled by delta/u0, temperature gradients by delta/t0.  Returns
    [Nx, Ny, Nz, 12] (z walls: 0)."""
    def px(f):
        n = f.shape[0] - 1
        ip = np.r_[1:n, 0, 1]
        im = np.r_[n - 1, 0:n - 1, n - 1]
        return (f[ip] - f[im]) / (2 * dx)

    def py(f):
        n = f.shape[1] - 1
        jp = np.r_[1:n, 0, 1]
        jm = np.r_[n - 1, 0:n - 1, n - 1]
        return (f[:, jp] - f[:, jm]) / (2 * dy)

    def pz(f):
        d = np.zeros_like(f)
        d[:, :, 1:-1] = (f[:, :, 2:] - f[:, :, :-2]) / (z[2:] - z[:-2])
        return d

    ux, uy, uz = px(u), py(u), pz(u)
    vx, vy, vz = px(v), py(v), pz(v)
    wx, wy, wz = px(w), py(w), pz(w)
    Tx, Ty, Tz = px(T), py(T), pz(T)
    sv = delta / u0
    st = delta / t0
    F = np.stack([ux * sv, vy * sv, wz * sv, 0.5 * (uy + vx) * sv, 0.5 * (uz + wx) * sv, 0.5 * (vz + wy) * sv,
                  (wy - vz) * sv, (uz - wx) * sv, (vx - uy) * sv, Tx * st, Ty * st, Tz * st], axis=-1)
    F[:, :, 0] = 0.0
    F[:, :, -1] = 0.0
    return F

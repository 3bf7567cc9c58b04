"""CPU oracle of the learned subgrid-stress MLP (TEST INFRASTRUCTURE ONLY).

The learned closure has no counterpart in the reference; this restates the
network that pyspectral_b200 evaluates and trains on tensor cores, so that its
forward pass and gradients can be checked.  NumPy, FP64 accumulation, with the
same BF16 rounding of the tensor-core operands (features, weights, hidden
activations and back-propagated errors) as the GPU kernels; biases, pre-
activations and bias gradients stay in full precision.

Network: 10 -> H -> H -> 6 (H = 32 or 64, read from the length of the
parameter block), hidden activation exact GELU ("gelu") or ReLU ("relu",
derivative 0 at 0), MSE on normalised outputs.
Parameter block (row-major [out][in]): W1[64][10] b1[64] W2[64][64] b2[64]
W3[6][64] b3[6].  Normalisation block: xmean[10] xistd[10] ymean[6] ystd[6].
"""
from __future__ import annotations

import math

import numpy as np

NIN, NH, NOUT = 10, 64, 6
NNORM = 32


def sizes(h=NH):
    """(name, shape) of the parameter blocks of a width-h network."""
    return [("W1", (h, NIN)), ("b1", (h,)), ("W2", (h, h)), ("b2", (h,)), ("W3", (NOUT, h)), ("b3", (NOUT,))]


def nparams(h=NH):
    return sum(int(np.prod(s)) for _, s in sizes(h))


SIZES = sizes()
NPARAMS = nparams()


def width_of(P):
    """Hidden width of a parameter block (h^2 + 18 h + 6 floats)."""
    for h in (32, 64):
        if len(P) == nparams(h):
            return h
    raise ValueError(f"{len(P)} parameters: not a width-32 or width-64 network")


def unpack(P):
    out, o = {}, 0
    for name, shp in sizes(width_of(P)):
        n = int(np.prod(shp))
        out[name] = np.asarray(P[o:o + n], dtype=np.float64).reshape(shp)
        o += n
    return out


def pack(d):
    h = d["b1"].shape[0]
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in sizes(h)])


def bf16(x):
    """Round to bfloat16 (round to nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_d(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def act_fn(act):
    """(activation, derivative) by name."""
    if act == "gelu":
        return gelu, gelu_d
    if act == "relu":
        return (lambda x: np.maximum(x, 0.0)), (lambda x: (x > 0).astype(np.float64))
    raise ValueError(act)


def init_params(seed=0, hidden=NH):
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases."""
    rs = np.random.RandomState(seed)
    d = {}
    for name, shp in sizes(hidden):
        if name.startswith("W"):
            b = 1.0 / math.sqrt(shp[1])
            d[name] = rs.uniform(-b, b, size=shp)
        else:
            d[name] = np.zeros(shp)
    return pack(d)


def forward(P, norm, X, keep=False, act="gelu"):
    f, _ = act_fn(act)
    p = unpack(P)
    xm, xi = norm[0:NIN], norm[NIN:2 * NIN]
    ym, ys = norm[2 * NIN:2 * NIN + NOUT], norm[2 * NIN + NOUT:2 * NIN + 2 * NOUT]
    Xn = bf16((np.asarray(X, np.float64) - xm) * xi)
    Z1 = Xn @ bf16(p["W1"]).T + p["b1"]
    H1 = bf16(f(Z1))
    Z2 = H1 @ bf16(p["W2"]).T + p["b2"]
    H2 = bf16(f(Z2))
    Y = H2 @ bf16(p["W3"]).T + p["b3"]
    if keep:
        return Y, (Xn, Z1, H1, Z2, H2)
    return Y * ys + ym


def rhs_learned(g, state, nu, P, norm, delta, act="gelu"):
    """LES right-hand side with the MLP stress on the 3/2-padded grid: the
    DNS formula of PySpectral/src/RHSfunctions.py:3-50 applied to the summed
    products u_i u_j + tau_ij / s^2 (real-space scaling physical / s)."""
    from oracle import spectral_oracle as orc
    u = [orc.nyquist_zero(state[i]) for i in range(3)]
    s = orc.scale_32(g)
    k = (g.k1, g.k2, g.k3)
    ur = [orc.ifft32(g, orc.pad(x)) * s for x in u]
    grads = [orc.ifft32(g, orc.pad(1j * k[j] * u[i])) * s * s for i in range(3) for j in range(3)]
    X = np.stack([a.ravel() for a in grads] + [np.full(ur[0].size, delta)], axis=1)
    tau = forward(P, norm, X, act=act).T.reshape((6,) + ur[0].shape)
    pairs = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
    prods = [orc.unpad(orc.fft32(ur[a] * ur[b] + tau[m] / (s * s))) for m, (a, b) in enumerate(pairs)]
    k1, k2, k3 = k
    phat = orc._pressure(k1, k2, k3, g.ksqr_i, *prods)
    return np.stack(orc._advection(k1, k2, k3, nu, g.ksqr, phat, prods, *u))


def loss_and_grad(P, norm, X, T, act="gelu"):
    """MSE of the normalised outputs and its gradient w.r.t. the FP32 master
    parameters (straight through the BF16 casts)."""
    p = unpack(P)
    ym, ys = norm[2 * NIN:2 * NIN + NOUT], norm[2 * NIN + NOUT:2 * NIN + 2 * NOUT]
    _, fd = act_fn(act)
    Y, (Xn, Z1, H1, Z2, H2) = forward(P, norm, X, keep=True, act=act)
    Tn = (np.asarray(T, np.float64) - ym) / ys
    B = X.shape[0]
    D = Y - Tn
    loss = float(np.mean(D * D))
    dY = 2.0 * D / (NOUT * B)
    dYb = bf16(dY)
    dZ2 = (dYb @ bf16(p["W3"])) * fd(Z2)
    dZ2b = bf16(dZ2)
    dZ1 = (dZ2b @ bf16(p["W2"])) * fd(Z1)
    dZ1b = bf16(dZ1)
    g = {"W3": dYb.T @ H2, "b3": dY.sum(0), "W2": dZ2b.T @ H1, "b2": dZ2.sum(0), "W1": dZ1b.T @ Xn,
         "b1": dZ1.sum(0)}
    return loss, pack(g)

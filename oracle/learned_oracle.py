"""CPU oracle of the learned coarse-mesh correction -- TEST INFRASTRUCTURE ONLY.

The learned form has no counterpart in ParticleDynamics.jl (it is an added force term compared
with the plain fine-mesh PME), so there is no reference code or golden vector to restate:
parity unpinned against the reference.  The restatement below is pinned instead by

* central finite differences of the exact-arithmetic network (``mlp_grads`` with
  ``bf16=False``) in tests/test_oracle.py,
* the closed form of Adam (Kingma & Ba, 2015, Algorithm 1),
* a direct double loop over all minimum-image pairs for the descriptors.

With ``bf16=True`` the functions round at the points where the tensor-core kernels do
(x, W1, W2, h1 and the backward operands dz2, dz1 in bfloat16, round to nearest even; every
product accumulated exactly here, in FP32 on the device), so device results agree to
accumulation-order and ulp-of-bf16 differences.  Only ``tests/`` and ``bench.py``'s CPU legs use
this module.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H = 32, 128


def bf16(a) -> np.ndarray:
    """Round FP32 values to bfloat16 (nearest, ties to even), returned as float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(flat):
    flat = np.asarray(flat, np.float64)
    o = 0
    out = {}
    for name, shape in (("w1", (N_H, N_IN)), ("b1", (N_H,)), ("w2", (N_H, N_H)), ("b2", (N_H,)), ("w3", (N_H,)),
                        ("b3", (1,))):
        k = int(np.prod(shape))
        out[name] = flat[o:o + k].reshape(shape)
        o += k
    return out


def pack(d) -> np.ndarray:
    return np.concatenate([np.ravel(d[k]) for k in ("w1", "b1", "w2", "b2", "w3", "b3")])


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def mlp_forward(flat, X, bf16_points: bool = True):
    """s (n,) and the intermediates of s = w3 . silu(W2 h1 + b2) + b3, h1 = silu(W1 x + b1)."""
    p = unpack(flat)
    r = bf16 if bf16_points else (lambda a: np.asarray(a, np.float64))
    x = r(X)
    W1, W2 = r(p["w1"]), r(p["w2"])
    z1 = x @ W1.T + p["b1"]
    h1 = r(_silu(z1))
    z2 = h1 @ W2.T + p["b2"]
    h2 = _silu(z2)
    s = h2 @ p["w3"] + p["b3"][0]
    return s, dict(x=x, W1=W1, W2=W2, z1=z1, h1=h1, z2=z2, h2=h2)


def mlp_grads(flat, X, ds, bf16_points: bool = True) -> np.ndarray:
    """Gradient (flat layout) of sum_r ds_r s_r with respect to the parameters."""
    p = unpack(flat)
    r = bf16 if bf16_points else (lambda a: np.asarray(a, np.float64))
    _, c = mlp_forward(flat, X, bf16_points)
    ds = np.asarray(ds, np.float64)
    g = {}
    g["w3"] = c["h2"].T @ ds
    g["b3"] = np.array([ds.sum()])
    dz2 = ds[:, None] * p["w3"][None, :] * _dsilu(c["z2"])
    g["b2"] = dz2.sum(0)
    dz2r = r(dz2)
    g["w2"] = dz2r.T @ c["h1"]
    dh1 = dz2r @ c["W2"]
    dz1 = dh1 * _dsilu(c["z1"])
    g["b1"] = dz1.sum(0)
    g["w1"] = r(dz1).T @ c["x"]
    return pack(g)


def residual_loss_grads(flat, X, ab, scale, bf16_points: bool = True):
    """Loss sum_r (s^2 a - 2 s b) scale / 2 and its gradient (the training kernel's objective)."""
    s, _ = mlp_forward(flat, X, bf16_points)
    a, b = np.asarray(ab, np.float64)[:, 0], np.asarray(ab, np.float64)[:, 1]
    loss = 0.5 * scale * float((s * (s * a - 2.0 * b)).sum())
    ds = scale * (s * a - b)
    return loss, mlp_grads(flat, X, ds, bf16_points)


def adam(p, g, m, v, t, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba, 2015, Algorithm 1) on float64 copies: (p, m, v)."""
    p, g, m, v = (np.asarray(a, np.float64).copy() for a in (p, g, m, v))
    m = beta1 * m + (1 - beta1) * g
    v = beta2 * v + (1 - beta2) * g * g
    p = p - lr * (m / (1 - beta1 ** t)) / (np.sqrt(v / (1 - beta2 ** t)) + eps)
    return p, m, v


def descriptors(pos, q, typ, box, *, rcut, mu0, dmu, sigma, nb, nu0, dnu, tau, coef=None):
    """Features (n, 32), V (n, 3) and the radial-term vectors Vb (nb, n, 3) by a direct pair loop.

    Species 0 is type id 1, species 1 every other id; f_c(r) = (1 - r^2 / rcut^2)^2."""
    pos = np.asarray(pos, np.float64)
    q = np.asarray(q, np.float64)
    L = np.asarray(box, np.float64)
    n = len(pos)
    X = np.zeros((n, 32))
    Vb = np.zeros((nb, n, 3))
    mu = mu0 + dmu * np.arange(16)
    nu = nu0 + dnu * np.arange(nb)
    for i in range(n):
        d = pos[i] - pos
        d -= L * np.round(d / L)
        r2 = (d * d).sum(1)
        sel = (r2 < rcut * rcut) & (r2 > 0)
        j = np.nonzero(sel)[0]
        r = np.sqrt(r2[j])
        fc = (1.0 - (r / rcut) ** 2) ** 2
        g = np.exp(-((r[:, None] - mu[None, :]) ** 2) / (2 * sigma * sigma))
        w = (q[j] * fc)[:, None] * g
        s1 = np.asarray(typ)[j] > 1
        X[i, :16] = w[~s1].sum(0)
        X[i, 16:] = w[s1].sum(0)
        e = np.exp(-((r[:, None] - nu[None, :]) ** 2) / (2 * tau * tau)) * (q[i] * q[j] * fc)[:, None]
        Vb[:, i, :] = (e[:, :, None] * d[j][:, None, :]).sum(0)
    V = np.zeros((n, 3)) if coef is None else np.einsum("m,mnc->nc", np.asarray(coef, np.float64)[:nb], Vb)
    return X, V, Vb

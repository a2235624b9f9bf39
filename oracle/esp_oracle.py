"""CPU oracle of Ewald summation with prolates (ESP) -- TEST INFRASTRUCTURE ONLY.

Restates in FP64 numpy what ParticleDynamics.jl computes for an ESP solver, from the definitions
rather than from the library's setup code:

* psi_0^c by the Nystrom method on the finite Fourier transform, whose eigenfunction it is
  (int_{-1}^{1} cos(c x t) psi(t) dt = lambda psi(x) for the even eigenfunction; Slepian's
  characterisation, which src/electrostatics/Prolates.jl:4-9 states) -- a different algorithm from the
  library's Legendre-basis eigenproblem, normalised the same way (psi(0) = 1);
* the prolate split (src/electrostatics/Splits.jl:37-60, 169-225): E_s(t) = 1 - int_0^t chi,
  chi = psi / int_0^1 psi, short-range pair energy C q q E_s / r and force factor
  C q q (E_s / r - E_s'(t) / r_c) / r^2 (pair_kernel, Splits.jl:118-128), self energy
  -(C/2) chi(0) / r_c q^2, background -C pi r_c^2 m_2 Q^2 / V;
* the prolate window W(y) = psi(y) - psi(1), y = 2 (k - u) / P, exact (Windows.jl:26-37) with the
  stencil base of _prolate_cell (Windows.jl:158-167);
* the spectral transform g(k) = 4 pi c_hat(k r_c) / k^2, c_hat(u) = int_0^1 chi(x) cos(u x) dx by
  Gauss-Legendre quadrature, and the influence functions :esp_deconvolution (G = C/V g D1 D2 D3) and
  :esp (optimal AD influence with alias sums), with the virial coefficients
  (src/electrostatics/Influence.jl:35-181);
* spread, R2C, solve, C2R and the AD gather (src/electrostatics/MeshKernels.jl, Solver.jl:305-393).

Only tests use it.
"""
from __future__ import annotations

import math

import numpy as np


def gl(n, a=-1.0, b=1.0):
    x, w = np.polynomial.legendre.leggauss(n)
    return 0.5 * (b + a) + 0.5 * (b - a) * x, 0.5 * (b - a) * w


class Psi:
    """psi_0^c from the Nystrom discretisation of the even finite Fourier transform."""

    def __init__(self, c, n=200):
        x, w = gl(n)
        A = np.cos(c * np.outer(x, x)) * w[None, :]
        vals, vecs = np.linalg.eig(A)
        k = int(np.argmax(vals.real))
        self.c, self.x, self.w = float(c), x, w
        self.lam = float(vals[k].real)
        v = vecs[:, k].real
        self.v = v / self._raw(0.0, v)

    def _raw(self, t, v):
        return float((self.w * np.cos(self.c * t * self.x) * v).sum() / self.lam)

    def __call__(self, t):
        t = np.asarray(t, float)
        return (np.cos(self.c * np.multiply.outer(t, self.x)) @ (self.w * self.v)) / self.lam

    def deriv(self, t):
        t = np.asarray(t, float)
        return (-(np.sin(self.c * np.multiply.outer(t, self.x)) * (self.c * self.x)) @ (self.w * self.v)) / self.lam

    def integral(self, t):
        """int_0^t psi, in closed form from the Nystrom representation (the integral of each cosine)."""
        t = np.atleast_1d(np.asarray(t, float))
        return (np.sin(self.c * np.multiply.outer(t, self.x)) / (self.c * self.x)) @ (self.w * self.v) / self.lam

    def l2_norm(self):
        return math.sqrt(float((self.w * self(self.x) ** 2).sum()))


def shape_for_tolerance(eps, lo=0.5, hi=80.0):
    """c with psi(1) / ||psi|| = eps (bisection on the Nystrom psi)."""
    def f(c):
        p = Psi(c)
        return math.log(abs(float(p(1.0))) / p.l2_norm()) - math.log(eps)
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if f(mid) > 0:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


class Split:
    def __init__(self, rc, shape):
        self.rc = float(rc)
        self.psi = Psi(shape)
        self.norm = float(self.psi.integral(1.0)[0])
        self.chi0 = 1.0 / self.norm
        xq, wq = gl(128, 0.0, 1.0)
        chi = self.psi(xq) / self.norm
        self.m2 = float((wq * xq ** 2 * chi).sum())
        self.xq, self.wchi = xq, wq * chi

    def Es(self, t):
        return 1.0 - self.psi.integral(t) / self.norm

    def pair(self, r):
        """(e, f) per unit C q q: e = E_s / r, f = (E_s / r + chi(t) / r_c) / r^2 (zero beyond r_c)."""
        r = np.asarray(r, float)
        t = np.minimum(r / self.rc, 1.0)
        Es = self.Es(t)
        chi = self.psi(t) / self.norm
        e = np.where(r < self.rc, Es / r, 0.0)
        f = np.where(r < self.rc, (Es / r + chi / self.rc) / (r * r), 0.0)
        return e, f

    def g(self, k):
        """g(k) and g'(k)/k (spectral_g, Splits.jl:209-225)."""
        k = np.asarray(k, float)
        u = k * self.rc
        ux = np.multiply.outer(u, self.xq)
        c = np.cos(ux) @ self.wchi
        dc = -(np.sin(ux) * self.xq) @ self.wchi
        k2 = k * k
        g = 4 * math.pi * c / k2
        gp = 4 * math.pi * (self.rc * dc / k2 - 2 * c / (k2 * k))
        return g, gp / k


class Window:
    def __init__(self, P, shape):
        self.P = int(P)
        self.psi = Psi(shape)
        self.edge = float(self.psi(1.0))

    def stencil(self, u):
        """(k0, w, dw/du) for grid coordinates u (arrays)."""
        P = self.P
        u = np.asarray(u, float)
        if P % 2 == 0:
            k0 = np.floor(u).astype(np.int64) - (P // 2 - 1)
        else:
            k0 = np.floor(u + 0.5).astype(np.int64) - (P - 1) // 2
        k = k0[:, None] + np.arange(P)[None, :]
        y = (k - u[:, None]) * (2.0 / P)
        inside = np.abs(y) <= 1.0
        yc = np.clip(y, -1, 1)
        w = np.where(inside, self.psi(yc) - self.edge, 0.0)
        dw = np.where(inside, -(2.0 / P) * self.psi.deriv(yc), 0.0)
        return k0, w, dw

    def phat(self, theta, n=256):
        x, wq = gl(n)
        vals = self.psi(x) - self.edge
        half = 0.5 * self.P
        return (np.cos(np.multiply.outer(np.asarray(theta, float), half * x)) @ (wq * vals)) * half


def _signed(m, K):
    return np.where(m <= K // 2, m, m - K)


def influence(kind, window, split, K, box, C, nmax=2):
    """G and Vc (6, modes) on the R2C half spectrum in the (m1 fastest) order of the device."""
    K = [int(k) for k in K]
    L = [float(b) for b in box]
    CoverV = C / (L[0] * L[1] * L[2])
    m1 = np.arange(K[0] // 2 + 1)
    m2 = np.arange(K[1])
    m3 = np.arange(K[2])
    M3, M2, M1 = np.meshgrid(m3, m2, m1, indexing="ij")
    s = [_signed(M1, K[0]), _signed(M2, K[1]), _signed(M3, K[2])]
    ny = [(K[d] % 2 == 0) & ([M1, M2, M3][d] == K[d] // 2) for d in range(3)]
    zero = (s[0] == 0) & (s[1] == 0) & (s[2] == 0)
    kv = [2 * math.pi * s[d] / L[d] for d in range(3)]
    if kind == "esp_deconvolution":
        D = [1.0 / window.phat(2 * math.pi * _signed(np.arange(K[d]), K[d]) / K[d]) ** 2 for d in range(3)]
        kk = np.sqrt(kv[0] ** 2 + kv[1] ** 2 + kv[2] ** 2)
        kk = np.where(zero, 1.0, kk)
        g, gpk = split.g(kk)
        Dm = D[0][M1] * D[1][M2] * D[2][M3]
        G = CoverV * g * Dm
        c = CoverV * Dm * gpk
        Vc = [G + c * kv[0] ** 2, G + c * kv[1] ** 2, G + c * kv[2] ** 2, c * kv[0] * kv[1], c * kv[0] * kv[2],
              c * kv[1] * kv[2]]
    else:
        A = np.zeros(G_shape := M1.shape)
        B = np.zeros(G_shape)
        Cc = np.zeros(G_shape)
        a = [np.zeros(G_shape) for _ in range(6)]
        cc = [np.zeros(G_shape) for _ in range(6)]
        Ut = [None] * 3
        for d in range(3):
            sd = _signed(np.arange(K[d]), K[d])
            Ut[d] = np.array([window.phat(2 * math.pi * (sd + K[d] * n) / K[d]) for n in range(-nmax, nmax + 1)])
        for n1 in range(-nmax, nmax + 1):
            U1 = Ut[0][n1 + nmax][M1]
            q1 = 2 * math.pi * (s[0] + K[0] * n1) / L[0]
            for n2 in range(-nmax, nmax + 1):
                U2 = Ut[1][n2 + nmax][M2]
                q2 = 2 * math.pi * (s[1] + K[1] * n2) / L[1]
                for n3 in range(-nmax, nmax + 1):
                    U3 = Ut[2][n3 + nmax][M3]
                    q3 = 2 * math.pi * (s[2] + K[2] * n3) / L[2]
                    U2t = (U1 * U2 * U3) ** 2
                    B += U2t
                    qq = q1 * q1 + q2 * q2 + q3 * q3
                    ok = qq != 0
                    g, gpk = split.g(np.sqrt(np.where(ok, qq, 1.0)))
                    g = np.where(ok, g, 0.0)
                    gpk = np.where(ok, gpk, 0.0)
                    A += U2t * g * qq
                    Cc += U2t * qq
                    h = U2t * (gpk * qq + 2 * g)
                    q = (q1, q2, q3)
                    pairs = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
                    for j, (p1, p2) in enumerate(pairs):
                        a[j] += h * q[p1] * q[p2]
                        cc[j] += 2 * U2t * q[p1] * q[p2]
        with np.errstate(divide="ignore", invalid="ignore"):
            G = CoverV * A / (B * Cc)
            f = CoverV / (B * Cc)
            r = CoverV * A / (B * Cc * Cc)
            Vc = [G + f * a[0] - r * cc[0], G + f * a[1] - r * cc[1], G + f * a[2] - r * cc[2],
                  f * a[3] - r * cc[3], f * a[4] - r * cc[4], f * a[5] - r * cc[5]]
    G = np.where(zero, 0.0, G)
    Vc = [np.where(zero, 0.0, v) for v in Vc]
    Vc[3] = np.where(ny[0] | ny[1], 0.0, Vc[3])
    Vc[4] = np.where(ny[0] | ny[2], 0.0, Vc[4])
    Vc[5] = np.where(ny[1] | ny[2], 0.0, Vc[5])
    return G.reshape(-1), np.stack([v.reshape(-1) for v in Vc])


def mesh(pos, q, box, K, window, split, kind="esp", C=1.0, nmax=2, background=False):
    """Mesh forces, per-particle energies q phi / 2 (+ background), mesh energy and virial."""
    pos = np.asarray(pos, float)
    q = np.asarray(q, float)
    n = len(q)
    K = [int(k) for k in K]
    L = np.asarray(box, float)
    u = []
    for d in range(3):
        s = pos[:, d] / L[d]
        s = s - np.floor(s)
        ud = s * K[d]
        ud = np.where(ud >= K[d], ud - K[d], ud)
        u.append(ud)
    st = [window.stencil(u[d]) for d in range(3)]
    P = window.P
    idx = [(st[d][0][:, None] + np.arange(P)[None, :]) % K[d] for d in range(3)]
    grid = np.zeros((K[2], K[1], K[0]))
    w1, w2, w3 = st[0][1], st[1][1], st[2][1]
    for j3 in range(P):
        for j2 in range(P):
            np.add.at(grid, (idx[2][:, j3][:, None], idx[1][:, j2][:, None], idx[0]),
                      (q * w3[:, j3] * w2[:, j2])[:, None] * w1)
    spec = np.fft.rfftn(grid)
    G, Vc = influence(kind, window, split, K, box, C, nmax)
    G3 = G.reshape(spec.shape)
    K1h = K[0] // 2 + 1
    m1 = np.arange(K1h)
    wgt = np.where((m1 == 0) | ((K[0] % 2 == 0) & (m1 == K[0] // 2)), 0.5, 1.0)[None, None, :]
    a2 = wgt * np.abs(spec) ** 2
    Emesh = float((a2 * G3).sum())
    Wm = np.array([float((a2 * Vc[c].reshape(spec.shape)).sum()) for c in range(6)])
    pot = np.fft.irfftn(spec * G3, s=(K[2], K[1], K[0]), axes=(0, 1, 2)) * (K[0] * K[1] * K[2])
    d1, d2, d3 = st[0][2], st[1][2], st[2][2]
    phi = np.zeros(n)
    gx = np.zeros(n)
    gy = np.zeros(n)
    gz = np.zeros(n)
    for j3 in range(P):
        for j2 in range(P):
            row = pot[idx[2][:, j3][:, None], idx[1][:, j2][:, None], idx[0]]   # (n, P)
            phi += w3[:, j3] * w2[:, j2] * (row * w1).sum(1)
            gx += w3[:, j3] * w2[:, j2] * (row * d1).sum(1)
            gy += w3[:, j3] * d2[:, j2] * (row * w1).sum(1)
            gz += d3[:, j3] * w2[:, j2] * (row * w1).sum(1)
    F = -np.stack([q * gx * K[0] / L[0], q * gy * K[1] / L[1], q * gz * K[2] / L[2]], 1)
    V = float(np.prod(L))
    bgc = math.pi * split.rc ** 2 * split.m2
    bg = -C * bgc * q.sum() / V if background else 0.0
    ubg = -C * bgc * q.sum() ** 2 / V if background else 0.0
    Wm[:3] += ubg
    return dict(F=F, E=0.5 * q * phi + bg * q, Emesh=Emesh, W=Wm, phi=phi)


def pairs(pos, q, box, split, C=1.0):
    """Short-range prolate pair sums (minimum image, r < r_c < L/2): forces, per-particle energies
    (half per pair) and the pair virial (6)."""
    pos = np.asarray(pos, float)
    q = np.asarray(q, float)
    n = len(q)
    L = np.asarray(box, float)
    F = np.zeros((n, 3))
    E = np.zeros(n)
    W = np.zeros(6)
    for a in range(0, n, 256):
        d = pos[a:a + 256, None, :] - pos[None, :, :]
        d -= L * np.round(d / L)
        r2 = (d * d).sum(-1)
        ii, jj = np.nonzero((r2 > 0) & (r2 < split.rc ** 2))
        dij = d[ii, jj]
        e, f = split.pair(np.sqrt(r2[ii, jj]))
        qq = C * q[a + ii] * q[jj]
        e, f = e * qq, f * qq
        np.add.at(F, a + ii, f[:, None] * dij)
        np.add.at(E, a + ii, 0.5 * e)
        for j, (p1, p2) in enumerate(((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))):
            W[j] += 0.5 * (f * dij[:, p1] * dij[:, p2]).sum()
    return dict(F=F, E=E, W=W)


def total(pos, q, box, K, window, split, kind="esp", C=1.0, nmax=2):
    """Real space + mesh + self of an ESP solver: forces, energy, virial."""
    pr = pairs(pos, q, box, split, C)
    ms = mesh(pos, q, box, K, window, split, kind, C, nmax)
    self_e = -0.5 * C * split.chi0 / split.rc * np.asarray(q, float) ** 2
    E = pr["E"] + ms["E"] + self_e
    return dict(F=pr["F"] + ms["F"], E=E, Etot=float(E.sum()), W=pr["W"] + ms["W"], F_mesh=ms["F"],
                E_mesh=ms["E"], W_mesh=ms["W"])

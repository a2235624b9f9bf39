"""Host-side (FP64) setup of Ewald summation with prolates (ESP).

Restates the once-per-solver setup code of ParticleDynamics.jl for the prolate split and window:

* the order-zero prolate spheroidal wave function psi_0^c by Bouwkamp's method (a symmetric
  tridiagonal eigenproblem in normalised even Legendre polynomials), its derivative, integral and
  L2 norm, and the tolerance -> shape bisection (src/electrostatics/Prolates.jl:1-129);
* the prolate split: chi(0), the second moment, the long-range correction by Gauss-Legendre
  quadrature and the spectral transform c_hat(u) (src/electrostatics/Splits.jl:37-60, 96-132,
  169-240);
* the prolate window: the per-node polynomials of the device stencil, the continuum window
  transform, its deconvolution and alias tables, the Nyquist attenuation bound
  (src/electrostatics/Windows.jl:38-185, 329-411);
* the workflow's parameter rules (width from the tolerance, window shape resolved in the state's
  precision, mesh spacing pi r_c / c) (src/workflow/Electrostatics.jl:176-272);
* Gauss-Legendre nodes and the Legendre recurrences (src/electrostatics/Quadrature.jl:1-50).

The device evaluates what these produce: the node polynomials (spread and gather), the tabulated
spectral transform (influence function) and the polynomial fit of the long-range correction (the
cluster-pair kernel).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

F32_EPS = float(np.finfo(np.float32).eps)
F64_EPS = float(np.finfo(np.float64).eps)


def gauss_legendre(n: int, a: float = -1.0, b: float = 1.0):
    """n-point Gauss-Legendre nodes and weights on [a, b] (Quadrature.jl:10-24)."""
    x, w = np.polynomial.legendre.leggauss(int(n))
    half, mid = 0.5 * (b - a), 0.5 * (b + a)
    return mid + half * x, half * w


def legendre_all(x, nmax: int) -> np.ndarray:
    """P_0 .. P_{nmax+1} at x (array), shape (nmax + 2, len(x)) (Quadrature.jl:27-36)."""
    x = np.atleast_1d(np.asarray(x, float))
    P = np.empty((nmax + 2, x.size))
    P[0] = 1.0
    P[1] = x
    for n in range(1, nmax + 1):
        P[n + 1] = ((2 * n + 1) * x * P[n] - n * P[n - 1]) / (n + 1)
    return P


class ProlateFunction:
    """psi_0^c on [-1, 1] normalised to psi(0) = 1, as coefficients of P_0, P_2, P_4, ...
    (ProlateFunction, Prolates.jl:19-54)."""

    def __init__(self, c: float, nterms: int | None = None):
        if not c > 0:
            raise ValueError("Prolate bandlimit c must be positive.")
        from scipy.linalg import eigh_tridiagonal
        nterms = int(math.ceil(c)) + 48 if nterms is None else int(nterms)
        cc = float(c) ** 2
        n = 2.0 * np.arange(nterms)
        diag = n * (n + 1) + cc * (2.0 * n * (n + 1) - 1.0) / ((2 * n + 3) * (2 * n - 1))
        nn = n[:-1]
        off = cc * (nn + 2) * (nn + 1) / ((2 * nn + 3) * np.sqrt((2.0 * nn + 1) * (2.0 * nn + 5)))
        _, v = eigh_tridiagonal(diag, off, select="i", select_range=(0, 0))
        beta = v[:, 0] * np.sqrt(n + 0.5)
        # P_{2m}(0) = (-1)^m (2m-1)!! / (2m)!!
        p0 = np.ones(nterms)
        for m in range(1, nterms):
            p0[m] = p0[m - 1] * (-(2 * m - 1) / (2 * m))
        self.c = float(c)
        self.coeffs = beta / float((beta * p0).sum())

    @property
    def nmax(self) -> int:
        return 2 * len(self.coeffs) - 1

    def __call__(self, x):
        P = legendre_all(x, self.nmax)
        out = self.coeffs @ P[0:2 * len(self.coeffs):2]
        return out if np.ndim(x) else float(out[0])

    def derivative(self, x):
        """psi'(x) via P'_{n+1} = P'_{n-1} + (2n + 1) P_n (Prolates.jl:71-79)."""
        P = legendre_all(x, self.nmax)
        dP = np.zeros((self.nmax + 1, P.shape[1]))
        if self.nmax >= 1:
            dP[1] = 1.0
        for n in range(1, self.nmax):
            dP[n + 1] = dP[n - 1] + (2 * n + 1) * P[n]
        out = self.coeffs @ dP[0:2 * len(self.coeffs):2]
        return out if np.ndim(x) else float(out[0])

    def integral(self, x):
        """int_0^x psi (Prolates.jl:84-95): int_0^x P_n = (P_{n+1}(x) - P_{n-1}(x)) / (2n + 1)."""
        xa = np.atleast_1d(np.asarray(x, float))
        P = legendre_all(xa, self.nmax)
        acc = self.coeffs[0] * xa
        for k in range(1, len(self.coeffs)):
            n = 2 * k
            acc = acc + self.coeffs[k] * (P[n + 1] - P[n - 1]) / (2 * n + 1)
        return acc if np.ndim(x) else float(acc[0])

    def l2_norm(self) -> float:
        n = 2.0 * np.arange(len(self.coeffs))
        return float(np.sqrt((self.coeffs ** 2 * 2.0 / (2 * n + 1)).sum()))


def prolate_shape_for_tolerance(eps: float) -> float:
    """c with psi_0^c(1) = eps for the L2-normalised prolate function (Prolates.jl:108-129)."""
    if not 0.0 < eps < 1.0:
        raise ValueError("Prolate tolerance must lie in (0, 1).")
    target = math.log(float(eps))

    def f(c):
        pf = ProlateFunction(c)
        with np.errstate(divide="ignore"):   # psi(1) rounds to 0 for large c: log gives -inf
            return float(np.log(abs(pf(1.0)) / pf.l2_norm())) - target

    lo, hi = 0.5, 80.0
    if not f(lo) > 0:
        raise ValueError(f"Tolerance {eps} is too loose for a prolate split.")
    if not f(hi) < 0:
        raise ValueError(f"Tolerance {eps} is too tight for a prolate split.")
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid) > 0:
            lo = mid
        else:
            hi = mid
        if hi - lo < 1e-12 * hi:
            break
    return 0.5 * (lo + hi)


# ----------------------------------------------------------------------------- split

@dataclass
class ProlateSplit:
    """chi(x) proportional to psi_0^c(x) on [0, 1], zero beyond (ProlateSplit, Splits.jl:37-60).

    The short-range part vanishes at r = cutoff; E_s(t) = 1 - a(t), a(t) = int_0^t chi."""
    cutoff: float
    shape: float
    nquad: int = 128
    pf: ProlateFunction = field(init=False, repr=False)
    norm: float = field(init=False)
    chi0: float = field(init=False)
    m2: float = field(init=False)
    xq: np.ndarray = field(init=False, repr=False)
    wchi: np.ndarray = field(init=False, repr=False)

    def __post_init__(self):
        if not (math.isfinite(self.cutoff) and self.cutoff > 0):
            raise ValueError("ESP cutoff must be finite and positive.")
        if not (math.isfinite(self.shape) and self.shape > 0):
            raise ValueError("ESP split shape must be finite and positive.")
        self.pf = ProlateFunction(self.shape)
        self.norm = self.pf.integral(1.0)
        xq, wq = gauss_legendre(self.nquad, 0.0, 1.0)
        chi = self.pf(xq) / self.norm
        self.chi0 = 1.0 / self.norm
        self.m2 = float((wq * xq ** 2 * chi).sum())
        self.xq, self.wchi = xq, wq * chi

    def self_coefficient(self) -> float:
        """chi(0) / r_c (Splits.jl:68)."""
        return self.chi0 / self.cutoff

    def background_coefficient(self) -> float:
        """pi r_c^2 m_2 (Splits.jl:86)."""
        return math.pi * self.cutoff ** 2 * self.m2

    def short_range(self, r):
        """E_s(r / r_c) for r < r_c (0 beyond), the short-range fraction of 1/r."""
        t = np.minimum(np.asarray(r, float) / self.cutoff, 1.0)
        return 1.0 - self.pf.integral(t) / self.norm

    def chat(self, u):
        """c_hat(u) = int chi(x) cos(u x) dx and its u-derivative (the quadrature of spectral_g,
        Splits.jl:209-225); g(k) = 4 pi c_hat(k r_c) / k^2."""
        ux = np.multiply.outer(np.atleast_1d(np.asarray(u, float)), self.xq)
        return np.cos(ux) @ self.wchi, -(np.sin(ux) * self.xq) @ self.wchi

    def spectral_table(self, u_max: float, du: float = 0.01):
        """c_hat and dc_hat/du at u = j du, j = 0 .. ceil(u_max / du) + 2 (the device interpolates them
        by cubic Hermite, as TabulatedSpectral does, Splits.jl:233-268)."""
        nodes = int(math.ceil(u_max / du)) + 3
        u = du * np.arange(nodes)
        c, dc = self.chat(u)
        return float(du), c, dc


class ProlateCorrection:
    """Long-range part of the prolate split at s = r^2 (ProlateCorrection, Splits.jl:163-200):
    corr = a(t)/r = (1/r_c) int_0^1 chi(t u) du, fcorr = -(1/r) dcorr/dr
    = (1/(r_c r^2)) int_0^1 (chi(t u) - chi(t)) du, by Gauss-Legendre quadrature."""

    def __init__(self, split: ProlateSplit, nquad: int = 96):
        self.rc = split.cutoff
        self.pf = split.pf
        self.inv_norm = 1.0 / split.norm
        self.u, self.w = gauss_legendre(nquad, 0.0, 1.0)

    def __call__(self, s: float):
        rc = self.rc
        r = math.sqrt(s)
        t = min(r / rc, 1.0)
        chit = self.pf(t) * self.inv_norm
        chiu = self.pf(t * self.u) * self.inv_norm
        corr = float((self.w * chiu).sum()) / rc
        if t < 1e-4:
            # the limit of int (chi(tu) - chi(t)) du / r^2: chi''(0) (1/3 - 1) / 2 / r_c^2
            h = 1e-3
            d2 = (self.pf(h) - 2 * self.pf(0.0) + self.pf(-h)) * self.inv_norm / h ** 2
            return corr, d2 * (1.0 / 3.0 - 1.0) / 2.0 / rc ** 3
        return corr, float((self.w * (chiu - chit)).sum()) / (rc * r * r)


# ----------------------------------------------------------------------------- window

def _lobatto_monomials(f, d: int) -> np.ndarray:
    """Monomial coefficients in s in [-1, 1] of the degree-d interpolant of f at the Chebyshev-Lobatto
    points (Windows.jl:79-97); the points include s = +-1, so neighbouring node polynomials agree where
    a particle crosses a cell boundary."""
    i = np.arange(d + 1)
    v = np.array([f(math.cos(math.pi * k / d)) for k in range(d + 1)])
    wt = np.where((i == 0) | (i == d), 0.5, 1.0)
    a = np.array([(2.0 / d) * (wt * v * np.cos(np.pi * i * k / d)).sum() for k in range(d + 1)])
    a[0] *= 0.5
    a[-1] *= 0.5
    m = np.zeros(d + 1)
    tp = np.zeros(d + 1)
    tp[0] = 1.0
    tc = np.zeros(d + 1)
    tc[1] = 1.0
    m += a[0] * tp
    for k in range(1, d + 1):
        m += a[k] * tc
        tn = np.zeros(d + 1)
        tn[1:] = 2.0 * tc[:-1]
        tn -= tp
        tp, tc = tc, tn
    return m


@dataclass
class ProlateWindow:
    """W(x) = psi_0^c(2x/P) - psi_0^c(1) for |x| <= P/2 grid spacings, centred on the particle
    (ProlateWindow, Windows.jl:38-54)."""
    order: int
    shape: float
    pf: ProlateFunction = field(init=False, repr=False)
    edge: float = field(init=False)

    def __post_init__(self):
        if not 2 <= int(self.order) <= 16:
            raise ValueError(f"Prolate window width must be between 2 and 16 grid points; got {self.order}.")
        if not (math.isfinite(self.shape) and self.shape > 0):
            raise ValueError("Prolate window shape must be finite and positive.")
        self.order = int(self.order)
        self.pf = ProlateFunction(self.shape)
        self.edge = self.pf(1.0)

    def weights(self, y):
        """W at y = 2 x / P (zero outside [-1, 1])."""
        y = np.asarray(y, float)
        return np.where(np.abs(y) <= 1.0, self.pf(np.clip(y, -1, 1)) - self.edge, 0.0)

    def node_polynomials(self, precision=np.float32) -> np.ndarray:
        """C[h, k], the coefficient of tau^k of node h (h < ceil(P/2), tau in [-1/2, 1/2]) at the lowest
        even degree whose weights lie within eps/64 (not below 4e-15) of psi and whose derivatives lie
        within eps/4 (not below 1e-12) of the largest derivative (prolate_node_polynomials,
        Windows.jl:99-135)."""
        P = self.order
        H = (P + 1) // 2
        eps = float(np.finfo(precision).eps)

        def y(h, tau):
            return (h - (P - 1) / 2.0 - tau) * 2.0 / P

        check = np.linspace(-0.5, 0.5, 97)
        wref = np.array([self.pf(y(h, check)) - self.edge for h in range(H)])
        dref = np.array([-(2.0 / P) * self.pf.derivative(y(h, check)) for h in range(H)])
        tolw = max(eps / 64, 4e-15)
        told = max(eps / 4, 1e-12) * np.max(np.abs(dref))
        for d in range(6, 25, 2):
            C = np.empty((H, d + 1))
            for h in range(H):
                C[h] = _lobatto_monomials(lambda s: self.pf(y(h, s / 2.0)) - self.edge, d) * 2.0 ** np.arange(d + 1)
            if P % 2 == 1:
                C[H - 1, 1::2] = 0.0   # the centre node is its own mirror image: even in tau
            p = np.zeros((H, check.size))
            dp = np.zeros((H, check.size))
            for k in range(d, -1, -1):
                dp = dp * check + (p if k < d else 0.0)
                p = p * check + C[:, k][:, None]
            if np.max(np.abs(p - wref)) <= tolw and np.max(np.abs(dp - dref)) <= told:
                return C
        raise ValueError("no node polynomial up to degree 24 reaches the precision of the window")

    def transform(self, theta, nquad: int = 192):
        """phi_hat(theta) = (P/2) int_{-1}^{1} (psi(t) - psi(1)) cos(theta P t / 2) dt (Windows.jl:315-321)."""
        x, wq = gauss_legendre(nquad)
        vals = self.pf(x) - self.edge
        half = 0.5 * self.order
        th = np.atleast_1d(np.asarray(theta, float))
        return half * (np.cos(np.multiply.outer(th, half * x)) @ (wq * vals))

    def deconvolution(self, K: int) -> np.ndarray:
        """1 / phi_hat(2 pi m' / K)^2 for m = 0 .. K-1, m' the signed mode (Windows.jl:367-381)."""
        if self.order > K:
            raise ValueError(f"Mesh dimension {K} is smaller than the window width {self.order}.")
        m = np.arange(K)
        s = np.where(m <= K // 2, m, m - K)
        ph = self.transform(2 * np.pi * s / K)
        if not np.all(ph > 0):
            raise ValueError("Prolate window transform vanishes inside the mesh band; increase the window "
                             "shape or width.")
        return 1.0 / ph ** 2

    def alias_table(self, K: int, nmax: int) -> np.ndarray:
        """U[n + nmax, m] = phi_hat(theta_m + 2 pi n), theta_m = 2 pi m' / K (Windows.jl:400-411)."""
        m = np.arange(K)
        s = np.where(m <= K // 2, m, m - K)
        out = np.empty((2 * nmax + 1, K))
        for n in range(-nmax, nmax + 1):
            out[n + nmax] = self.transform(2 * np.pi * (s + K * n) / K, nquad=256)
        return out

    def nyquist_attenuation(self) -> float:
        """(phi_hat(pi) / phi_hat(0))^2 (window_nyquist_attenuation, Windows.jl:334-342)."""
        t = self.transform([math.pi, 0.0])
        return float((t[0] / t[1]) ** 2)


def min_nyquist_attenuation(precision=np.float32) -> float:
    """0.02 eps^(2/3): the smallest Nyquist attenuation a mesh solve in this precision resolves
    (Windows.jl:345-356)."""
    return 0.02 * float(np.finfo(precision).eps) ** (2.0 / 3.0)


def max_prolate_order(shape: float) -> int:
    """Widest window for shape c: P <= 2c/pi - 1/2 (Spec.jl:113)."""
    return int(math.floor(2 * shape / math.pi - 0.5 + 1e-9))


def esp_order_for_tolerance(eps: float) -> int:
    """Window width from the tolerance (esp_order_for_tolerance, src/workflow/Electrostatics.jl:183-192)."""
    d = -math.log10(float(eps))
    if d <= 3.35:
        return 5
    if d <= 4.05:
        return 6
    if d <= 4.35:
        return 7
    if d <= 5.05:
        return 8
    c1 = prolate_shape_for_tolerance(float(eps) / 2)
    return min(max(int(math.floor(2 * c1 / math.pi - 1)), 8), 16)


def esp_window_shape(eps: float, P: int, precision=np.float32) -> float:
    """c(eps/2), or the smallest larger shape whose window the precision resolves
    (esp_window_shape, src/workflow/Electrostatics.jl:202-218)."""
    def resolved(c):
        return ProlateWindow(P, c).nyquist_attenuation() >= min_nyquist_attenuation(precision)

    c1 = prolate_shape_for_tolerance(float(eps) / 2)
    if resolved(c1):
        return c1
    lo, hi = c1, c1 + 0.5
    while not resolved(hi):
        lo = hi
        hi += 0.5
        if hi >= 80:
            raise ValueError(f"No prolate window of width {P} is resolved in {np.dtype(precision).name}.")
    while hi - lo > 1e-3:
        mid = 0.5 * (lo + hi)
        if resolved(mid):
            hi = mid
        else:
            lo = mid
    return hi

"""Host-side (FP64) setup math of the electrostatics and pair kernels.

Restates the setup code of ParticleDynamics.jl that runs once per solver:
the Gaussian split constants (src/electrostatics/Splits.jl:67-86, 142-161),
the real-space tolerance -> alpha bisection and FFT-friendly mesh sizes
(src/electrostatics/Spec.jl:122-187), the adaptive Chebyshev fit
(src/electrostatics/Quadrature.jl:58-122) and the Coulomb polynomial of the
cluster-pair kernel (src/clusterpairs/PairFunctor.jl:37-84).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

SQRT_PI = math.sqrt(math.pi)


def self_coefficient(alpha: float) -> float:
    """chi(0)/r_c of the Gaussian split: 2 alpha / sqrt(pi) (Splits.jl:67)."""
    return 2.0 * alpha / SQRT_PI


def background_coefficient(alpha: float) -> float:
    """pi r_c^2 m_2 of the Gaussian split: pi / (2 alpha^2) (Splits.jl:85)."""
    return math.pi / (2.0 * alpha * alpha)


def cutoff_energy(alpha: float, rc: float) -> float:
    """erfc(alpha r_c) / r_c, the potential-shift constant (Splits.jl:77)."""
    return math.erfc(alpha * rc) / rc


def alpha_from_tolerance(cutoff: float, tol: float) -> float:
    """alpha with erfc(alpha r_c) = tol by bisection on [0, 10] (Spec.jl:154-163)."""
    if not (0.0 < tol < 1.0):
        raise ValueError("real_space_tolerance must lie in (0, 1).")
    lo, hi = 0.0, 10.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if math.erfc(mid) - tol > 0:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi) / cutoff


def fft_friendly(n: int) -> int:
    """Smallest integer >= n whose prime factors are all in {2, 3, 5, 7} (Spec.jl:122-134)."""
    m = max(int(n), 1)
    while True:
        r = m
        for p in (2, 3, 5, 7):
            while r % p == 0:
                r //= p
        if r == 1:
            return m
        m += 1


def resolve_mesh(mesh, mesh_spacing, box, order: int) -> tuple[int, int, int]:
    """Explicit mesh, or FFT-friendly sizes from the spacing (Spec.jl:141-146)."""
    if mesh is not None:
        return tuple(int(k) for k in mesh)
    h = float(mesh_spacing)
    return tuple(max(fft_friendly(math.ceil(float(box[d]) / h - 1e-9)), order) for d in range(3))


def long_range_correction(alpha: float, s: float) -> tuple[float, float]:
    """(corr, fcorr) at s = r^2: corr = erf(alpha r)/r and fcorr = -(1/r) d corr/dr (Splits.jl:142-161).

    Small arguments use the power series of the reference (no cancellation near
    r = 0); larger ones the closed forms.
    """
    z = alpha * alpha * s
    pre = 2.0 * alpha / SQRT_PI
    if z < 0.5:
        ce, cf, prev = 1.0, 0.0, 1.0
        for n in range(1, 200):
            term = prev * z / n
            sgn = -1.0 if n % 2 else 1.0
            ce += sgn * term / (2 * n + 1)
            cf -= 2.0 * sgn * alpha * alpha * prev / (2 * n + 1)
            prev = term
            if n > 10 and abs(term) < 1e-30:
                break
        return pre * ce, pre * cf
    r = math.sqrt(s)
    corr = math.erf(alpha * r) / r
    fcorr = math.erf(alpha * r) / (r * s) - pre * math.exp(-z) / s
    return corr, fcorr


def chebyshev_fit(f, degree: int) -> np.ndarray:
    """Interpolant coefficients at the Chebyshev points of the first kind (Quadrature.jl:58-71)."""
    n = degree + 1
    k = np.arange(n)
    xs = np.cos(np.pi * (k + 0.5) / n)
    fs = np.array([f(x) for x in xs])
    j = np.arange(n)[:, None]
    c = 2.0 * (np.cos(np.pi * j * (k[None, :] + 0.5) / n) @ fs) / n
    c[0] *= 0.5
    return c


def chebyshev_eval(c, s: float) -> float:
    b1 = b2 = 0.0
    for j in range(len(c) - 1, 0, -1):
        b0 = 2.0 * s * b1 - b2 + c[j]
        b2, b1 = b1, b0
    return s * b1 - b2 + c[0]


def chebyshev_fit_adaptive(f, tol: float = 2e-14, max_degree: int = 96) -> np.ndarray:
    """Smallest even-degree interpolant within tol * max|f| on a dense grid (Quadrature.jl:107-122)."""
    check = np.cos(np.pi * (np.arange(1024) + 0.25) / 1024)
    fcheck = np.array([f(x) for x in check])
    scale = max(np.max(np.abs(fcheck)), np.finfo(float).tiny)
    best = None
    for degree in range(8, max_degree + 1, 2):
        c = chebyshev_fit(f, degree)
        # Clenshaw on the whole grid at once
        b1 = np.zeros_like(check)
        b2 = np.zeros_like(check)
        for j in range(len(c) - 1, 0, -1):
            b0 = 2.0 * check * b1 - b2 + c[j]
            b2, b1 = b1, b0
        vals = check * b1 - b2 + c[0]
        err = np.max(np.abs(vals - fcheck))
        best = c
        if err <= tol * scale:
            break
    best = list(best)
    while len(best) > 2 and abs(best[-1]) <= 0.01 * tol * scale:
        best.pop()
    return np.array(best)


def chebyshev_to_monomial(c) -> np.ndarray:
    """Chebyshev series in x -> monomial coefficients in x (PairFunctor.jl:37-52)."""
    n = len(c)
    t0 = np.zeros(n)
    t0[0] = 1.0
    m = c[0] * t0
    if n == 1:
        return m
    t1 = np.zeros(n)
    t1[1] = 1.0
    m = m + c[1] * t1
    for k in range(2, n):
        t2 = np.zeros(n)
        t2[1:] = 2.0 * t1[:-1]
        t2 -= t0
        m = m + c[k] * t2
        t0, t1 = t1, t2
    return m


@dataclass
class CoulombPolynomial:
    """Device description of the short-range Coulomb term (PairFunctor.jl:21-29).

    e = C qq (1/r + P_e(x) - eshift), f/r = C qq (1/r^3 - P_f(x)) inside r_c,
    x = r^2 sx - 1; pe/pf are monomial coefficients (constant first).
    """
    C: float
    rc2: float
    sx: float
    eshift: float
    has_mesh: bool
    pe: np.ndarray
    pf: np.ndarray


def coulomb_polynomial(alpha, C: float, cutoff: float, eshift: float = 0.0,
                       tol: float | None = None, energy_tol: float | None = None) -> CoulombPolynomial:
    """Fit the long-range correction of the split on [0, r_c^2] for Float32 kernels (PairFunctor.jl:65-84).

    ``alpha`` is the Gaussian split's parameter (the erf correction), or a callable s -> (corr, fcorr)
    giving another split's correction (the prolate split's ProlateCorrection)."""
    ftol = 1e-7 if tol is None else float(tol)
    etol = 1e-8 if energy_tol is None else float(energy_tol)
    rc2 = float(cutoff) ** 2
    corr = alpha if callable(alpha) else (lambda s: long_range_correction(alpha, s))

    def s_of(x):
        return (x + 1.0) * rc2 / 2.0

    ce = chebyshev_fit_adaptive(lambda x: -corr(s_of(x))[0], tol=etol)
    cf = chebyshev_fit_adaptive(lambda x: corr(s_of(x))[1], tol=ftol)
    if max(len(ce), len(cf)) > 20:
        raise ValueError("Coulomb correction needs more than 20 coefficients at Float32 tolerances")
    return CoulombPolynomial(C=float(C), rc2=rc2, sx=2.0 / rc2, eshift=float(eshift), has_mesh=True,
                             pe=chebyshev_to_monomial(ce), pf=chebyshev_to_monomial(cf))


def lj_type_table(sigma, epsilon, rcut, shift: bool = False, wca: bool = False) -> np.ndarray:
    """(c6, c12, rc^2, e_shift) per type pair, row-major (PairFunctor.jl:166-179)."""
    sigma = np.atleast_2d(np.asarray(sigma, float))
    epsilon = np.atleast_2d(np.asarray(epsilon, float))
    rcut = np.atleast_2d(np.asarray(rcut, float))
    n = sigma.shape[0]
    out = np.zeros((n * n, 4))
    for a in range(n):
        for b in range(n):
            s6 = sigma[a, b] ** 6
            e = epsilon[a, b]
            rc = rcut[a, b]
            if wca:
                esh = -e
            elif shift and rc > 0:
                esh = 4 * e * s6 * (s6 / rc ** 12 - 1 / rc ** 6)
            else:
                esh = 0.0
            out[a * n + b] = (4 * e * s6, 4 * e * s6 * s6, rc * rc, esh)
    return out


WCA_RC_FACTOR = 1.2599211 ** 0.5   # r_c = 2^(1/6) sigma, written as the reference's sqrt(1.2599211)


def lj_cutoff_energy(sigma: float, epsilon: float, rc: float) -> float:
    """4 eps ((sigma/rc)^12 - (sigma/rc)^6), the potential-shift constant (lj_cutoff_energy,
    src/engine/PairModels.jl:27-32)."""
    if rc <= 0:
        return 0.0
    s2 = sigma * sigma / (rc * rc)
    s6 = s2 * s2 * s2
    return 4.0 * epsilon * (s6 * s6 - s6)

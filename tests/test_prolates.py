"""Host-side ESP setup (prolate function, split, window, parameter rules) against the reference's own
known answers and against the ESP oracle's independent prolate function (CPU)."""
import importlib.util
import math
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def eo():
    spec = importlib.util.spec_from_file_location("pdb200_esp_oracle", ROOT / "oracle" / "esp_oracle.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_shape_table(pd, kats):
    # Table 2 of Liang et al. as the reference tests it (test/test_electrostatics.jl:55-58)
    k = kats["esp"]
    for eps, c in k["shape_table"]:
        assert math.isclose(pd.prolates.prolate_shape_for_tolerance(eps), c, rel_tol=k["shape_rtol"]), eps


def test_prolate_function_properties(pd, eo):
    # finite Fourier eigenfunction (test/test_electrostatics.jl:59-63): the ratio of transform to value is
    # constant; the derivative matches a central difference; the Legendre-basis psi equals the oracle's
    # Nystrom psi
    pf = pd.prolates.ProlateFunction(10.0)
    x, w = pd.prolates.gauss_legendre(160)

    def ratio(t):
        return (w * pf(x) * np.cos(10.0 * t * x)).sum() / pf(t)

    assert math.isclose(ratio(0.2), ratio(0.9), rel_tol=1e-10)
    assert math.isclose(pf.derivative(0.3), (pf(0.3 + 1e-6) - pf(0.3 - 1e-6)) / 2e-6, rel_tol=1e-7)
    for c in (8.0, 12.024, 15.2):
        a, b = pd.prolates.ProlateFunction(c), eo.Psi(c)
        t = np.linspace(-1, 1, 201)
        assert np.max(np.abs(a(t) - b(t))) < 1e-10, c
        assert np.max(np.abs(a.derivative(t) - b.deriv(t))) < 1e-9, c
    # the oracle's own shape bisection on its psi agrees with the table rule
    assert math.isclose(eo.shape_for_tolerance(1e-4), pd.prolates.prolate_shape_for_tolerance(1e-4), rel_tol=1e-8)


def test_window_symmetric_value(pd, kats):
    # test/test_electrostatics.jl:88-91: width 6, shape 12 at u = 10.5 -> k0 = 8, the two middle nodes
    # carry psi(1/6) - psi(1)
    k = kats["esp"]["window"]
    w = pd.prolates.ProlateWindow(k["order"], k["shape"])
    C = w.node_polynomials(np.float64)
    P = k["order"]
    H = (P + 1) // 2
    u = k["u"]
    fl = math.floor(u)
    assert fl - (P // 2 - 1) == k["k0"]
    tau = (u - fl) - 0.5
    vals = [np.polynomial.polynomial.polyval(tau if j < H else -tau, C[j if j < H else P - 1 - j]) for j in range(P)]
    assert math.isclose(vals[2], vals[3], rel_tol=1e-12)
    assert math.isclose(vals[2], w.pf(1 / 6) - w.edge, rel_tol=1e-12)


@pytest.mark.parametrize("P,eps", [(4, 2.5e-4), (5, 5e-4), (6, 5e-5), (8, 5e-6), (8, 5e-7)])
def test_node_polynomials(pd, eo, P, eps):
    # the per-node polynomials reproduce W = psi(y) - psi(1) and dW/du of the oracle's psi within the FP32
    # bounds of prolate_node_polynomials (Windows.jl:99-135), and the window is continuous where the stencil
    # base changes (test/test_electrostatics.jl:98-122)
    c = pd.prolates.prolate_shape_for_tolerance(eps)
    w = pd.prolates.ProlateWindow(P, c)
    Cp = w.node_polynomials(np.float32)
    H = (P + 1) // 2
    ow = eo.Window(P, c)
    rng = np.random.default_rng(P)
    u = rng.uniform(0.0, 40.0, 400)

    def stencil(u):
        if P % 2 == 0:
            fl = np.floor(u)
            k0, tau = fl - (P // 2 - 1), (u - fl) - 0.5
        else:
            fl = np.floor(u + 0.5)
            k0, tau = fl - (P - 1) // 2, u - fl
        W = np.zeros((len(u), P))
        D = np.zeros((len(u), P))
        for j in range(P):
            h, t = (j, tau) if j < H else (P - 1 - j, -tau)
            W[:, j] = np.polynomial.polynomial.polyval(t, Cp[h])
            d = np.polynomial.polynomial.polyval(t, np.polynomial.polynomial.polyder(Cp[h]))
            D[:, j] = d if j < H else -d
        return k0.astype(int), W, D

    k0, W, D = stencil(u)
    ok0, oW, oD = ow.stencil(u)
    assert np.array_equal(k0, ok0)
    eps32 = float(np.finfo(np.float32).eps)
    assert np.max(np.abs(W - oW)) < max(eps32 / 16, 4e-14)
    assert np.max(np.abs(D - oD)) < eps32 * np.max(np.abs(oD))
    # continuity across the base change: u0 - tiny and u0 share node weights (a missing node weighs 0)
    u0 = 7.0 if P % 2 == 0 else 7.5
    kl, wl, _ = stencil(np.array([u0 - 1e-13]))
    kr, wr, _ = stencil(np.array([u0 + 1e-13]))
    nodes_l = {int(kl[0]) + j: wl[0, j] for j in range(P)}
    nodes_r = {int(kr[0]) + j: wr[0, j] for j in range(P)}
    assert int(kl[0]) != int(kr[0])
    assert max(abs(nodes_l.get(k, 0.0) - nodes_r.get(k, 0.0)) for k in set(nodes_l) | set(nodes_r)) < 1e-10


def test_split_constants_and_correction(pd, eo):
    # chi(0), the second moment and the long-range correction of the prolate split against the oracle's
    # direct integrals: corr = (1 - E_s(t)) / r and fcorr = -(1/r) d corr / dr
    rc, c = 3.0, 11.0
    sp = pd.prolates.ProlateSplit(rc, c)
    osp = eo.Split(rc, c)
    assert math.isclose(sp.chi0, osp.chi0, rel_tol=1e-10)
    assert math.isclose(sp.m2, osp.m2, rel_tol=1e-10)
    corr = pd.prolates.ProlateCorrection(sp)
    for r in (0.01, 0.5, 1.3, 2.2, 2.9):
        e, f = osp.pair(np.array([r]))
        ce, cf = corr(r * r)
        assert math.isclose(ce, 1.0 / r - e[0], rel_tol=1e-9, abs_tol=1e-12), r
        assert math.isclose(cf, 1.0 / r ** 3 - f[0], rel_tol=1e-7, abs_tol=1e-10), r
    assert np.allclose(sp.short_range(np.array([3.0, 3.5])), 0.0, atol=1e-12)   # zero from the cutoff on
    # E_s(t) = 1 - chi(0) t + O(t^3) near the origin (test/test_electrostatics.jl:295-297)
    r = 1e-3
    assert math.isclose(float(sp.short_range(r)), 1 - sp.chi0 * r / rc, abs_tol=1e-9)


def test_parameter_rules(pd):
    # width from the tolerance (5, 5, 6, 7, 8 for 1e-3, 5e-4, 1e-4, 5e-5, 1e-5), the width bound, spacing
    P = pd.prolates
    assert [P.esp_order_for_tolerance(e) for e in (1e-3, 5e-4, 1e-4, 5e-5, 1e-5)] == [5, 5, 6, 7, 8]
    for eps in (1e-3, 1e-4, 1e-5):
        assert P.esp_order_for_tolerance(eps) <= P.max_prolate_order(P.prolate_shape_for_tolerance(eps / 2))
    spec = pd.electrostatics_spec(pd.ESP(coulomb_prefactor=14.4, real_cutoff=9.0, tolerance=1e-5))
    assert spec.influence == "esp" and spec.order == 8
    assert math.isclose(spec.mesh_spacing, math.pi * 9.0 / spec.split_shape)
    assert P.ProlateWindow(8, spec.window_shape).nyquist_attenuation() >= P.min_nyquist_attenuation(np.float32)
    with pytest.raises(ValueError, match="supports at most"):
        pd.ElectrostaticsSpec(coulomb_prefactor=1.0, real_cutoff=3.0, influence="esp", order=12, mesh=(32, 32, 32),
                              split_shape=10.0, window_shape=10.0)
    with pytest.raises(ValueError, match="optimal or deconvolution"):
        pd.electrostatics_spec(pd.ESP(coulomb_prefactor=1.0, real_cutoff=3.0, influence="fast"))


def test_esp_oracle_against_ewald(pd, ora, eo, kats):
    # pins the ESP oracle: the reference's ESP case (test/test_electrostatics.jl:299-341, C = 1.7, r_c = 4,
    # 120 ions in 14 x 15 x 16, eps 1e-6, mesh 32 x 32 x 36, width 8) reproduces the Ewald sum within the
    # reference's FP64 tolerances (force 1e-5, energy 1e-6)
    k = kats["esp"]["solver"]
    e = kats["electrostatics"]
    rng = np.random.default_rng(3)
    L = tuple(e["box"])
    R = rng.uniform(0, 1, (e["n"], 3)) * np.array(L)
    q = np.where(np.arange(e["n"]) % 2 == 0, 1.0, -1.0)
    c = pd.prolates.prolate_shape_for_tolerance(k["eps"])
    c1 = pd.prolates.prolate_shape_for_tolerance(k["eps"] / 2)
    tot = eo.total(R, q, L, k["mesh"], eo.Window(k["order"], c1), eo.Split(e["rc"], c), "esp", C=e["C"], nmax=2)
    E, F, W = ora.ewald(R, q, L, C=e["C"])
    assert np.linalg.norm(tot["F"] - F) / np.linalg.norm(F) < k["ftol"]
    assert abs(tot["Etot"] - E) < k["etol"] * abs(E)
    assert np.max(np.abs(tot["W"][:3] - np.diag(W))) < 10 * max(k["ftol"], k["etol"]) * abs(np.trace(W))

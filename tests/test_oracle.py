"""The CPU oracle pinned on the reference's known answers (no GPU needed)."""
import math
from pathlib import Path

import numpy as np
import pytest


def test_two_atom_lj_known_answers(ora, kats):
    # test/test_force_precision_gpu.jl:7-20
    for case in kats["two_atom_lj"]:
        pos = np.array([[0.0, 0.0, 0.0], [case["separation"], 0.0, 0.0]])
        r = ora.pairs_direct(pos, (10.0, 10.0, 10.0), kind=1, sigma=1.0, eps=1.0, rc_lj=2.5)
        assert np.allclose(r["F"][:, 0], case["F_x"], rtol=0, atol=1e-14)
        assert np.allclose(r["F"][:, 1:], 0.0)
        assert np.allclose(r["E"], case["energy"], rtol=0, atol=1e-15)
        assert np.allclose(r["W"].sum(0), case["virial_sum"], rtol=0, atol=1e-14)
        assert np.all(r["count"] == 1)


def _rows_py(coords, box, radii):
    """Pure-Python restatement of reference_neighbor_rows for the small known answers."""
    n = len(coords[0])
    out = []
    for i in range(n):
        row = []
        for j in range(n):
            if j == i:
                continue
            d2 = 0.0
            for d in range(len(coords)):
                dd = coords[d][j] - coords[d][i]
                dd -= box[d] * round(dd / box[d])
                d2 += dd * dd
            if d2 <= radii[i] ** 2:
                row.append(j + 1)   # 1-based as the reference's rows
        out.append(row)
    return out


def test_neighbor_rows_known_answers(kats, ora):
    # test/test_neighbor_reference.jl:2-4
    for case in kats["neighbor_rows"]:
        assert _rows_py(case["coords"], case["box"], case["radii"]) == case["rows"]
    # the C restatement agrees with the Python one on a random 3D case
    rng = np.random.default_rng(3)
    pos = rng.uniform(0, 6.0, size=(300, 3))
    rows = ora.neighbor_rows(pos, (6.0, 6.0, 6.0), 1.3)
    py = _rows_py([pos[:, d].tolist() for d in range(3)], (6.0, 6.0, 6.0), [1.3] * 300)
    assert [[j + 1 for j in r] for r in rows] == py


@pytest.mark.parametrize("P", [3, 4, 5, 6, 7, 8])
def test_bspline_partition_and_base(ora, P):
    # test/test_electrostatics.jl:54-96
    rng = np.random.default_rng(5)
    for _ in range(20):
        u = 40 * rng.random()
        k0, w, dw = ora.bspline(P, u)
        assert abs(w.sum() - 1.0) < 1e-14
        assert abs(dw.sum()) < 1e-13
        assert k0 == math.floor(u) - P + 1
        h = 1e-7
        if math.floor(u + h) == math.floor(u - h):
            _, wp, _ = ora.bspline(P, u + h)
            _, wm, _ = ora.bspline(P, u - h)
            assert np.max(np.abs((wp - wm) / (2 * h) - dw)) < 1e-6
    kL, wL, _ = ora.bspline(P, 7.0 - 1e-12)
    kR, wR, _ = ora.bspline(P, 7.0)
    nodes = {}
    for k, w in ((kL, wL), (kR, wR)):
        for j in range(P):
            nodes.setdefault(k + j, []).append(w[j])
    for k, ws in nodes.items():
        ws = ws + [0.0] * (2 - len(ws))
        assert abs(ws[0] - ws[1]) < 1e-10


def test_fft_conventions():
    # test/test_electrostatics.jl:260-279: impulse -> flat spectrum, constant -> M value at m = 0,
    # single mode -> M/2, backward transform unnormalised
    import sys
    ora = sys.modules["pdb200_oracle"]
    K = np.array([8, 6, 5], np.int32)
    g = np.zeros(240)
    g[0] = 1.0
    s = ora._rfft(g, K, 1)
    assert s.shape == (5, 6, 5) and np.allclose(s, 1.0, atol=1e-14)
    s = ora._rfft(np.full(240, 2.0), K, 1)
    assert abs(s[0, 0, 0] - 480.0) < 1e-10 and np.max(np.abs(s.reshape(-1)[1:])) < 1e-10
    i, j, k = np.meshgrid(np.arange(8), np.arange(6), np.arange(5), indexing="ij")
    gm = np.cos(2 * np.pi * (1 * i / 8 + 2 * j / 6 + 1 * k / 5))
    flat = gm.transpose(2, 1, 0).reshape(-1)   # node n1 + K1 (n2 + K2 n3)
    s = ora._rfft(flat, K, 1)
    assert abs(s[1, 2, 1] - 120.0) < 1e-10
    back = ora._irfft(s, K, 1)
    assert np.max(np.abs(back / 240 - flat)) < 1e-13


def _cloud(n, L, seed):
    rng = np.random.default_rng(seed)
    R = rng.random((n, 3)) * np.array(L) - np.array(L) / 2
    q = rng.standard_normal(n)
    q -= q.sum() / n
    return R, q


def test_mesh_oracle_against_ewald(ora, kats):
    # the reference's solver cases and tolerances (test/test_electrostatics.jl:299-341) applied to the
    # FP64 restatement: real space + mesh + self against the independent Ewald sum
    e = kats["electrostatics"]
    C, rc, L = e["C"], e["rc"], tuple(e["box"])
    R, q = _cloud(e["n"], L, 3)
    Eref, Fref, Wref = ora.ewald(R, q, L, C=C)
    for case in e["cases"]:
        tot = ora.pme_total(R, q, L, C=C, alpha=case["alpha"], rc=rc, K=case["mesh"], P=case["order"],
                            kind=case["influence"])
        rel = np.sqrt(((tot["F"] - Fref) ** 2).sum() / (Fref ** 2).sum())
        assert rel < case["ftol"], (case["name"], rel)
        assert abs(tot["Etot"] - Eref) / abs(Eref) < case["etol"], case["name"]
        W = tot["W"]
        Wm = np.array([[W[0], W[3], W[4]], [W[3], W[1], W[5]], [W[4], W[5], W[2]]])
        assert np.max(np.abs(Wm - Wref)) / abs(np.trace(Wref)) < 10 * max(case["ftol"], case["etol"]), case["name"]


def test_self_and_background_energy(ora):
    # test/test_electrostatics.jl:321 and :409
    R, q = _cloud(60, (9.0, 9.5, 10.0), 11)
    qn = q + 0.05
    C, a = 1.3, 0.9
    E0, _, _ = ora.ewald(R, qn, (9.0, 9.5, 10.0), C=C, alpha=a, background=False)
    E1, _, W1 = ora.ewald(R, qn, (9.0, 9.5, 10.0), C=C, alpha=a, background=True)
    V = 9.0 * 9.5 * 10.0
    Ebg = -C * math.pi * qn.sum() ** 2 / (2 * a * a * V)
    assert abs((E1 - E0) - Ebg) < 1e-12 * abs(E0)


def test_cluster_list_pair_set(ora):
    """Every pair inside the list radius lies in exactly one tile of the oracle's outer list."""
    rng = np.random.default_rng(1)
    L = (5.3, 5.6, 6.1)
    n = 1201
    pos = (rng.random((n, 3)) * np.array(L) - np.array(L) / 2).astype(np.float32)
    rl = 1.05
    b = ora.cluster_build(pos, L, rl)
    pairs = ora.tile_pairs(b["perm"], b["scio"], dict(cjo=b["cjo"]), working=False)
    assert len(pairs) == len(set(pairs)), "a pair appears in two tiles"
    rows = ora.neighbor_rows(pos.astype(float), L, 1.0)
    need = {(min(i, j), max(i, j)) for i, r in enumerate(rows) for j in r}
    assert need <= set(pairs)
    perm = b["perm"]
    assert sorted(perm[perm >= 0].tolist()) == list(range(n))


def test_coulomb_polynomial_against_erfc(pd, ora):
    # PairFunctor.jl:65-84 fit (Float32 tolerances) against the exact correction; the reference's FP64
    # fit is checked at 1e-12 (test/test_cluster_pairs.jl:203-211)
    for alpha, rc in ((0.347046, 9.0), (3.0, 1.2), (0.9, 4.0)):
        cp = pd.splits.coulomb_polynomial(alpha, 1.0, rc)
        for r in np.linspace(0.05 * rc, 0.999 * rc, 200):
            x = r * r * cp.sx - 1.0
            pf = np.polyval(cp.pf[::-1], x)
            pe = np.polyval(cp.pe[::-1], x)
            f_ref = (math.erfc(alpha * r) / r + 2 * alpha / math.sqrt(math.pi) * math.exp(-(alpha * r) ** 2)) / r ** 2
            e_ref = math.erfc(alpha * r) / r
            f = 1 / r ** 3 - pf
            e = 1 / r + pe
            assert abs(f - f_ref) < 2e-6 / r ** 3
            assert abs(e - e_ref) < 2e-7 / r


def test_setup_math(pd):
    s = pd.splits
    a = s.alpha_from_tolerance(9.0, 1e-5)
    assert abs(math.erfc(9.0 * a) - 1e-5) < 1e-12
    assert abs(a - 0.34705) < 5e-5
    assert s.fft_friendly(119) == 120 and s.fft_friendly(121) == 125 and s.fft_friendly(11) == 12
    assert s.resolve_mesh(None, 1.0, (119.5, 119.5, 119.5), 5) == (120, 120, 120)
    assert s.resolve_mesh(None, 2.0, (119.5,) * 3, 4) == (60, 60, 60)
    t = s.lj_type_table(1.0, 1.0, 2 ** (1 / 6), wca=True)
    assert t[0, 3] == -1.0


def _learned_oracle():
    import importlib.util
    import sys
    name = "pdb200_learned_oracle"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, Path(__file__).resolve().parent.parent / "oracle" /
                                                      "learned_oracle.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def test_learned_oracle_gradients_against_finite_differences():
    """Pins the network restatement: exact-arithmetic gradients vs central differences."""
    lo = _learned_oracle()
    rng = np.random.default_rng(5)
    flat = rng.normal(0, 0.3, 4096 + 128 + 16384 + 128 + 128 + 1)
    X = rng.normal(0, 1, (6, 32))
    ab = np.abs(rng.normal(0, 1, (6, 2)))
    scale = 0.37
    loss, g = lo.residual_loss_grads(flat, X, ab, scale, bf16_points=False)
    idx = np.concatenate([rng.choice(4096, 6, replace=False), 4096 + rng.choice(128, 3, replace=False),
                          4224 + rng.choice(16384, 6, replace=False), 20608 + rng.choice(128, 3, replace=False),
                          20736 + rng.choice(128, 3, replace=False), [20864]])
    h = 1e-6
    for k in idx:
        p, m = flat.copy(), flat.copy()
        p[k] += h
        m[k] -= h
        fd = (lo.residual_loss_grads(p, X, ab, scale, False)[0] - lo.residual_loss_grads(m, X, ab, scale, False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_learned_oracle_bf16_and_adam():
    lo = _learned_oracle()
    # round to nearest, ties to even, on the 8-bit bfloat16 mantissa
    a = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5, 3.0e-3], np.float32)
    r = lo.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 * 2.0 ** -7 and r[3] == 1.0 and r[4] == -2.5
    assert abs(r[5] - 3.0e-3) <= 2.0 ** -8 * 3.0e-3
    p, m, v = lo.adam(np.ones(3), np.array([1.0, -2.0, 0.0]), np.zeros(3), np.zeros(3), 1, lr=0.1)
    # first step: m_hat = g, v_hat = g^2, so the step is lr * sign(g) (up to eps)
    assert np.allclose(p, [0.9, 1.1, 1.0], atol=1e-7)

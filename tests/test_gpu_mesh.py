"""PME / P3M mesh engine on the GPU against the FP64 oracle and the Ewald sum."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cloud(n, L, seed):
    rng = np.random.default_rng(seed)
    R = rng.random((n, 3)) * np.array(L) - np.array(L) / 2
    q = rng.standard_normal(n)
    q -= q.sum() / n
    return R.astype(np.float32).astype(np.float64), q.astype(np.float32).astype(np.float64)


def _solver(pd, influence, alpha, mesh, order, C, rc, box, q, nmax=None, background=False):
    spec = pd.ElectrostaticsSpec(coulomb_prefactor=C, real_cutoff=rc, alpha=alpha, influence=influence, order=order,
                                 mesh=tuple(mesh), net_charge="background" if background else "error")
    return pd.ElectrostaticsSolver(spec, box, q, nmax=nmax)


def _mesh_gpu(pd, s, R, q, order_perm=None, energy=True):
    import torch
    n = len(q)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")
    x, y, z, qq = d(R[:, 0]), d(R[:, 1]), d(R[:, 2]), d(q)
    o = None if order_perm is None else torch.tensor(order_perm, dtype=torch.int32, device="cuda")
    fx, fy, fz, e = (torch.zeros(n, device="cuda") for _ in range(4))
    vg = torch.zeros(6, device="cuda")
    s.transform(x, y, z, qq, order=o, energy=energy)
    s.gather(x, y, z, qq, fx, fy, fz, e, vg, order=o, energy=energy, set=True)
    torch.cuda.synchronize()
    F = torch.stack([fx, fy, fz], 1).double().cpu().numpy()
    return F, e.double().cpu().numpy(), vg.double().cpu().numpy(), s.mesh_energy()


CASES = [("spme", (48, 48, 54), 6), ("spme", (64, 64, 72), 8), ("p3m_ad", (48, 48, 54), 6),
         ("p3m_ik", (48, 48, 54), 6), ("spme", (24, 25, 27), 5), ("p3m_ad", (24, 25, 27), 5)]


@pytest.mark.parametrize("influence,mesh,order", CASES)
def test_mesh_matches_fp64_oracle(pd, ora, cuda, influence, mesh, order):
    L = (14.0, 15.0, 16.0)
    C, rc, alpha = 1.7, 4.0, 0.9
    R, q = _cloud(120, L, 3)
    s = _solver(pd, influence, alpha, mesh, order, C, rc, L, q)
    G, Vc = s.influence()
    Go, Vco = ora.influence(influence, order, mesh, L, C, alpha)
    assert np.max(np.abs(G - Go)) <= 2e-7 * np.max(np.abs(Go))
    assert np.max(np.abs(Vc - Vco)) <= 2e-7 * np.max(np.abs(Vco))
    F, E, vg, acc = _mesh_gpu(pd, s, R, q)
    ref = ora.mesh(R, q, L, mesh, order, kind=influence, alpha=alpha, C=C)
    rel = np.linalg.norm(F - ref["F"]) / np.linalg.norm(ref["F"])
    assert rel < 1e-5, rel                                    # FP32 mesh vs FP64 (test_electrostatics.jl:553-565)
    assert abs(acc[0] - ref["Emesh"]) < 1e-6 * abs(ref["Emesh"])   # FP64 reduction of the mesh energy
    assert abs(E.sum() - ref["E"].sum()) < 1e-5 * abs(ref["E"].sum())
    assert np.max(np.abs(vg - ref["W"])) < 1e-5 * abs(ref["W"][:3].sum())
    s.close()


@pytest.mark.parametrize("influence,mesh,order,ftol", [("spme", (48, 48, 54), 6, 1e-4), ("p3m_ad", (48, 48, 54), 6, 1e-4),
                                                       ("p3m_ik", (48, 48, 54), 6, 1e-4)])
def test_solver_against_ewald(pd, ora, cuda, influence, mesh, order, ftol):
    # FP32 solver (real space on the cluster kernel + mesh + self) against the Ewald oracle, the reference's
    # FP32 bound 1e-4 (test/test_electrostatics.jl:553-565)
    import torch
    L = (14.0, 15.0, 16.0)
    C, rc, alpha = 1.7, 4.0, 0.9
    R, q = _cloud(120, L, 3)
    Eref, Fref, Wref = ora.ewald(R, q, L, C=C)
    s = _solver(pd, influence, alpha, mesh, order, C, rc, L, q)
    cp = s.coulomb_polynomial()
    eng = pd.ClusterPairEngine(120, L, rmax=rc, skin=0.3, prune_buffer=0.0, coulomb=cp, selfc=s.selfc)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")
    x, y, z, qq = d(R[:, 0]), d(R[:, 1]), d(R[:, 2]), d(q)
    f = [torch.zeros(120, device="cuda") for _ in range(4)]
    w = torch.zeros((120, 6), device="cuda")
    vg = torch.zeros(6, device="cuda")
    s.transform(x, y, z, qq, energy=True)
    s.gather(x, y, z, qq, f[0], f[1], f[2], f[3], vg, energy=True, set=True)
    fx2, fy2, fz2, e2 = (torch.zeros(120, device="cuda") for _ in range(4))
    eng.compute(x, y, z, qq, torch.ones(120, dtype=torch.int32, device="cuda"), fx2, fy2, fz2, e2, w, energy=True)
    torch.cuda.synchronize()
    F = (torch.stack(f[:3], 1) + torch.stack([fx2, fy2, fz2], 1)).double().cpu().numpy()
    E = float(f[3].double().sum() + e2.double().sum())
    rel = np.linalg.norm(F - Fref) / np.linalg.norm(Fref)
    assert rel < ftol, rel
    assert abs(E - Eref) / abs(Eref) < 1e-4
    W6 = w.double().sum(0).cpu().numpy() + vg.double().cpu().numpy()
    Wm = np.array([[W6[0], W6[3], W6[4]], [W6[3], W6[1], W6[5]], [W6[4], W6[5], W6[2]]])
    assert np.max(np.abs(Wm - Wref)) / abs(np.trace(Wref)) < 1e-3
    eng.close()
    s.close()


def test_order_and_background(pd, ora, cuda):
    L = (13.0, 13.5, 14.0)
    R, q = _cloud(300, L, 9)
    qn = q + 0.05
    s = _solver(pd, "spme", 0.9, (24, 25, 27), 5, 1.3, 3.8, L, qn, background=True)
    perm = np.random.default_rng(1).permutation(300).astype(np.int32)
    F0, E0, vg0, _ = _mesh_gpu(pd, s, R, qn)
    F1, E1, vg1, _ = _mesh_gpu(pd, s, R, qn, order_perm=perm)
    assert np.max(np.abs(F1 - F0)) < 1e-5 * np.max(np.abs(F0))
    ref = ora.mesh(R, qn, L, (24, 25, 27), 5, alpha=0.9, C=1.3, background=True)
    assert abs(E0.sum() - ref["E"].sum()) < 1e-5 * abs(ref["E"].sum())
    assert np.max(np.abs(vg0 - ref["W"])) < 1e-5 * abs(ref["W"][:3].sum())
    Ebg = -1.3 * math.pi * qn.sum() ** 2 / (2 * 0.81 * np.prod(L))
    assert abs(s.background_energy() - Ebg) < 1e-12 * abs(Ebg)
    s.close()


def test_zero_charges_and_validation(pd, cuda):
    L = (13.0, 13.5, 14.0)
    R, q = _cloud(100, L, 2)
    s = _solver(pd, "spme", 0.9, (24, 25, 27), 5, 1.0, 3.8, L, np.zeros(100))
    F, E, vg, acc = _mesh_gpu(pd, s, R, np.zeros(100))
    assert np.all(F == 0) and np.all(E == 0) and np.all(vg == 0) and acc[0] == 0
    with pytest.raises(ValueError):
        _solver(pd, "spme", 0.9, (24, 25, 27), 5, 1.0, 3.8, L, q + 0.05)    # net charge rejected
    with pytest.raises(ValueError):
        _solver(pd, "spme", 0.9, (24, 25, 27), 5, 1.0, 7.0, L, q)           # r_c >= L/2
    with pytest.raises(ValueError):
        pd.ElectrostaticsSpec(coulomb_prefactor=1.0, real_cutoff=3.0, alpha=1.0, order=2, mesh=(16, 16, 16))


def _melt(pd, L, seed):
    n = int(0.0375 * L ** 3) // 2 * 2
    pos, q, _ = pd.synthetic.ionic_melt(n, L, seed=seed)
    return np.asarray(pos, np.float32).astype(np.float64), np.asarray(q, np.float64)


@pytest.mark.parametrize("influence", ["spme", "p3m_ad"])
def test_self_force_table_and_removal(pd, ora, cuda, influence):
    # the table equals the self force of a lone unit charge through the FP64 oracle mesh; the gather
    # subtracts q^2 times its trilinear interpolation; removing it lowers the coarse mesh's error
    # against a fine mesh; 0 turns it off again
    C, alpha, L, K, P = 14.399645, 0.34705, 30.0, 15, 4
    box = (L, L, L)
    R, q = _melt(pd, L, 21)
    s = _solver(pd, influence, alpha, (K, K, K), P, C, 9.0, box, q)
    F_off, _, _, _ = _mesh_gpu(pd, s, R, q, energy=False)
    s.set_self_force_removal(16)
    tab = s.self_force_table().astype(np.float64)
    assert tab.shape == (16, 16, 16, 3)
    tables = ora.influence(influence, P, (K, K, K), box, C, alpha)
    rng = np.random.default_rng(0)
    for t in rng.integers(0, 16, (24, 3)):
        pos = (t[::-1] / 16.0 * L / K)[None, :]          # table index (t3, t2, t1) -> grid coordinate (t1, t2, t3)/T
        ex = ora.mesh_source_forces(pos, np.array([1.0]), box, (K, K, K), P, tables, [0])[0, 0]
        assert np.abs(tab[t[0], t[1], t[2]] - ex).max() <= 1e-3 * np.abs(tab).max() + 1e-9, (t, ex)
    F_on, _, _, _ = _mesh_gpu(pd, s, R, q, energy=False)
    u = (R / L - np.floor(R / L)) * K
    f = (u - np.floor(u)) * 16
    i0 = np.minimum(f.astype(int), 15)
    w = f - i0
    S = np.zeros_like(R)
    for c in range(8):
        b = [(c >> d) & 1 for d in range(3)]
        idx = [(i0[:, d] + b[d]) % 16 for d in range(3)]
        wt = np.prod([w[:, d] if b[d] else 1 - w[:, d] for d in range(3)], axis=0)
        S += wt[:, None] * tab[idx[2], idx[1], idx[0]]
    expect = F_off - (q * q)[:, None] * S
    assert np.linalg.norm(F_on - expect) <= 2e-5 * np.linalg.norm(F_off)
    fine = ora.mesh(R, q, box, (30, 30, 30), 5, kind=influence, alpha=alpha, C=C)["F"]
    e_off, e_on = np.linalg.norm(F_off - fine), np.linalg.norm(F_on - fine)
    assert e_on < 0.95 * e_off, (e_on, e_off)
    # a new box recomputes the table; 0 turns the removal off
    s.set_box((L + 1.0,) * 3)
    tab2 = s.self_force_table()
    assert np.abs(tab2 - tab).max() > 1e-3 * np.abs(tab).max()
    s.set_box(box)
    s.set_self_force_removal(0)
    assert s.self_force_table().size == 0
    F_again, _, _, _ = _mesh_gpu(pd, s, R, q, energy=False)
    assert np.linalg.norm(F_again - F_off) <= 1e-6 * np.linalg.norm(F_off)   # spread atomics: order varies
    with pytest.raises(Exception):
        s.set_self_force_removal(3)
    s.close()


def test_self_force_removal_refused_for_ik(pd, cuda):
    R, q = _cloud(64, (14.0, 15.0, 16.0), 5)
    s = _solver(pd, "p3m_ik", 0.9, (24, 25, 27), 5, 1.7, 4.0, (14.0, 15.0, 16.0), q)
    with pytest.raises(Exception):
        s.set_self_force_removal(16)
    s.close()

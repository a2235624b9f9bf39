"""Learned coarse-mesh correction on the GPU: tensor-core network forward / training gradients /
Adam against the CPU restatement, descriptors against a direct pair loop, the FP64 Ewald oracle
against the CPU Ewald sum, the step engine with the correction attached, and the gain of the
trained network over the coarse mesh alone."""
import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def lo():
    name = "pdb200_learned_oracle"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, ROOT / "oracle" / "learned_oracle.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def _params(pd, seed):
    rng = np.random.default_rng(seed)
    flat = pd.learned.init_params(seed, s0=0.3, out_scale=1.0)
    p = pd.learned.split_params(flat)
    p["b1"][:] = rng.normal(0, 0.3, 128)
    p["b2"][:] = rng.normal(0, 0.3, 128)
    return flat


def _bf16_input(n, seed, cuda):
    import torch
    g = torch.Generator().manual_seed(seed)
    X = (torch.randn((n, 32), generator=g) * 1.5).to(torch.bfloat16)
    return X.to(cuda), X.float().numpy()


@pytest.mark.parametrize("n", [1, 127, 1000, 5 * 128, 100_000])
def test_mlp_forward_matches_oracle(pd, lo, cuda, n):
    # 100 000 rows: 782 tiles, more than the 4 x 148 warpgroup slots, so warpgroups take several tiles
    import torch
    net = pd.learned.MLPNetwork(_params(pd, 3))
    X, Xh = _bf16_input(n, 11 + n, cuda)
    s = net.forward(X).cpu().numpy()
    ref, _ = lo.mlp_forward(net.params(), Xh, bf16_points=True)
    err = np.abs(s - ref)
    scale = np.sqrt(np.mean(ref ** 2))
    assert np.sqrt(np.mean(err ** 2)) <= 1e-4 * scale, (np.sqrt(np.mean(err ** 2)), scale)
    assert err.max() <= 1e-2 * scale
    V = torch.randn((n, 4), device=cuda)
    corr = net.forward(X, V=V).cpu().numpy()
    sv = corr[:, 3]
    assert np.array_equal(sv, s)
    assert np.allclose(corr[:, :3], sv[:, None] * V[:, :3].cpu().numpy(), rtol=1e-6, atol=0)
    assert net.error() == 0


@pytest.mark.parametrize("n", [300, 148 * 128 + 300])
def test_mlp_training_gradients_match_oracle(pd, lo, cuda, n):
    """Fused forward + backward on the tensor cores vs the restatement with the same BF16 rounding
    points; n above 148 tiles makes CTAs accumulate several tiles in tensor memory."""
    import torch
    net = pd.learned.MLPNetwork(_params(pd, 5))
    X, Xh = _bf16_input(n, 21, cuda)
    rng = np.random.default_rng(9)
    ab = np.stack([np.abs(rng.normal(0, 1, n)), rng.normal(0, 1, n)], 1).astype(np.float32)
    scale = 2.0 / (3 * n)
    net.loss(reset=True)
    net.train_batch(X, torch.tensor(ab, device=cuda), scale)
    torch.cuda.synchronize()
    g = net.grads()
    loss = net.loss(reset=True)
    rloss, rg = lo.residual_loss_grads(net.params(), Xh, ab, scale, bf16_points=True)
    assert abs(loss - rloss) <= 1e-4 * abs(rloss) + 1e-12
    P = pd.learned.split_params(g.astype(np.float64))
    R = pd.learned.split_params(rg)
    for k in P:
        num = np.linalg.norm(P[k] - R[k])
        den = np.linalg.norm(R[k])
        assert num <= 5e-3 * den + 1e-9, (k, num / max(den, 1e-30))
    assert net.error() == 0


def test_adam_matches_oracle(pd, lo, cuda):
    import torch
    net = pd.learned.MLPNetwork(_params(pd, 7))
    X, Xh = _bf16_input(512, 5, cuda)
    ab = torch.stack([torch.rand(512, device=cuda), torch.randn(512, device=cuda)], 1).contiguous()
    p0 = net.params()
    m = np.zeros_like(p0, dtype=np.float64)
    v = np.zeros_like(p0, dtype=np.float64)
    p = p0.astype(np.float64)
    for t in (1, 2):
        net.train_batch(X, ab, 1e-3)
        torch.cuda.synchronize()
        g = net.grads().astype(np.float64)
        net.adam(lr=1e-3)
        torch.cuda.synchronize()
        p, m, v = lo.adam(p, g, m, v, t, lr=1e-3)
        got = net.params()
        assert np.allclose(got, p, rtol=1e-5, atol=1e-7)
        assert not net.grads().any()   # cleared by the step


def _ions(pd, n, L, seed):
    pos, q, box = pd.synthetic.ionic_melt(n, L, 2.2, seed=seed)
    pos = pos - L * np.floor(pos / L + 0.5)
    typ = np.where(q > 0, 1, 2).astype(np.int32)
    return pos, q, typ, box


def test_descriptors_match_oracle(pd, lo, cuda):
    import torch
    n, L = 700, 26.0
    pos, q, typ, box = _ions(pd, n, L, 4)
    lc = pd.learned.LearnedCorrection(n, box)
    coef = np.random.default_rng(2).normal(0, 1, lc.nb)
    lc.set_radial(coef)
    t = {k: torch.tensor(pos[:, d], dtype=torch.float32, device=cuda) for d, k in enumerate("xyz")}
    qd = torch.tensor(q, dtype=torch.float32, device=cuda)
    td = torch.tensor(typ, device=cuda)
    X, V = lc.descriptors(t["x"], t["y"], t["z"], qd, td)
    Vb = lc.radial_basis(t["x"], t["y"], t["z"], qd, td).cpu().numpy()
    cfg = lc.cfg
    Xr, Vr, Vbr = lo.descriptors(pos.astype(np.float32), q, typ, box, rcut=cfg["rcut"], mu0=cfg["mu0"],
                                 dmu=cfg["dmu"], sigma=cfg["sigma"], nb=cfg["nb"], nu0=cfg["nu0"], dnu=cfg["dnu"],
                                 tau=cfg["tau"], coef=lc.coef)
    Xg = X.float().cpu().numpy()
    assert np.all(np.abs(Xg - Xr) <= 2.0 ** -7 * np.abs(Xr) + 1e-4)
    assert np.any(np.abs(Xr) > 0.5)
    rel = lambda a, b: np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2))   # noqa: E731
    assert rel(V.cpu().numpy()[:, :3], Vr) < 2e-5
    assert rel(Vb[..., :3], Vbr) < 2e-5
    st = lc.status()
    assert st["error"] == 0 and st["valid"] == 1


def test_ewald_oracle_matches_cpu(pd, ora, cuda):
    import torch
    n, L = 120, 16.0
    pos, q, typ, box = _ions(pd, n, L, 8)
    C, alpha, digits = 14.399645, 0.7, 12.0
    E0, F0, _ = ora.ewald(pos, q, box, C=C, alpha=alpha, digits=digits)
    rq = torch.tensor(np.concatenate([pos, q[:, None]], 1), dtype=torch.float64, device=cuda).contiguous()
    F, E = pd.learned.ewald_oracle(rq, box, C, alpha, digits=digits, parts=7)
    F = F.cpu().numpy()
    assert abs(E - E0) <= 1e-10 * abs(E0)
    assert np.sqrt(np.sum((F - F0) ** 2) / np.sum(F0 ** 2)) < 1e-10
    # the parts add up
    Fr, Er = pd.learned.ewald_oracle(rq, box, C, alpha, digits=digits, parts=1)
    Fk, Ek = pd.learned.ewald_oracle(rq, box, C, alpha, digits=digits, parts=2)
    assert np.allclose(Fr.cpu().numpy() + Fk.cpu().numpy(), F, rtol=0, atol=1e-10 * np.abs(F).max())


def _melt_trainer(pd, n, seed=0):
    import torch
    L = (n / 0.0375) ** (1.0 / 3.0)
    pos, q, typ, box = _ions(pd, n, L, 100)
    spec = pd.ElectrostaticsSpec(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=9.0,
                                 alpha=pd.splits.alpha_from_tolerance(9.0, 1e-5), order=5, mesh_spacing=1.0)
    qd = torch.tensor(q, dtype=torch.float32, device="cuda")
    td = torch.tensor(typ, device="cuda")
    tr = pd.learned.CoarseMeshTrainer(n, box, qd, td, spec, seed=seed)
    return tr, box, q, spec


def test_step_engine_adds_the_correction(pd, cuda):
    """Forces of an evaluation with the correction attached = forces without + s V; graph == eager."""
    import torch
    n = 4000
    L = (n / 0.0375) ** (1.0 / 3.0)
    pos, q, typ, box = _ions(pd, n, L, 12)
    m = pd.synthetic.melt_masses(q)
    v = pd.synthetic.maxwell_boltzmann(m, 1200.0, seed=3, kB=pd.synthetic.KB_EV)
    system = pd.ParticleSystem(pos, box, types=["Na", "Cl"], typeids=typ, masses=m, charges=q, velocities=v)
    lj = pd.LennardJones(epsilon=0.01, sigma=2.8, cutoff=9.0, pairs="neighborlist",
                         neighborlist=pd.ClusterPairList(buffer=2.0, prune_buffer=0.6))
    el = pd.PME(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=9.0, real_space_tolerance=1e-5,
                mesh_spacing=2.0, order=4)
    dt = 1.0 / pd.synthetic.TIME_UNIT_FS

    def make():
        sim = pd.Simulation(system, pd.Integrator(dt=dt, forces=[lj, el]))
        return sim.state

    st0 = make()
    st0.evaluate_forces_into_f(False)
    f0 = st0.forces()
    st1 = make()
    lc = pd.learned.LearnedCorrection(n, box)
    lc.set_radial(np.linspace(0.01, -0.02, lc.nb))
    net = pd.learned.MLPNetwork(_params(pd, 1))
    st1.engine.set_learned(lc, net)
    st1.evaluate_forces_into_f(False)
    f1 = st1.forces()
    corr = lc.correction(net, st1.x, st1.y, st1.z, st1.q, st1.typ).cpu().numpy()
    assert np.abs(corr[:, :3]).max() > 0
    assert np.allclose(f1 - f0, corr[:, :3], rtol=1e-4, atol=1e-5 * np.abs(f0).max())
    # a few steps: graph replay and eager launches agree
    st2 = make()
    lc2 = pd.learned.LearnedCorrection(n, box)
    lc2.set_radial(lc.coef)
    net2 = pd.learned.MLPNetwork(net.params())
    st2.engine.set_learned(lc2, net2)
    st2.evaluate_forces_into_f(False)
    st1.step(5, use_graph=True)
    st2.step(5, use_graph=False)
    st1.synchronize()
    st2.synchronize()
    assert np.allclose(st1.positions(), st2.positions(), rtol=0, atol=1e-4)
    assert net.error() == 0 and lc.status()["error"] == 0
    # the radial term alone (no network): the forces gain V, the correction at s = 1
    st3 = make()
    lc3 = pd.learned.LearnedCorrection(n, box)
    lc3.set_radial(lc.coef)
    st3.engine.set_learned(lc3, None)
    st3.evaluate_forces_into_f(False)
    f3 = st3.forces()
    ones = pd.learned.MLPNetwork(pd.learned.init_params(0, s0=1.0, out_scale=0.0))
    V = lc3.correction(ones, st3.x, st3.y, st3.z, st3.q, st3.typ).cpu().numpy()
    assert np.abs(V[:, :3]).max() > 0
    assert np.allclose(f3 - f0, V[:, :3], rtol=1e-4, atol=1e-5 * np.abs(f0).max())


def test_trained_network_beats_the_coarse_mesh(pd, cuda):
    """What the learned part gains: held-out reciprocal-space force error against the FP64 Ewald sum
    of the coarse mesh alone, with its self force removed, with the fitted radial term (s = 1) and
    with the trained network."""
    import torch
    n = 4000
    tr, box, q, spec = _melt_trainer(pd, n)
    L = box[0]
    train_seeds, test_seeds = range(200, 248), range(900, 904)

    def coords(seed):
        pos, _, _, _ = _ions(pd, n, L, seed)
        return [torch.tensor(pos[:, d], dtype=torch.float32, device="cuda") for d in range(3)], pos

    # same composition in every configuration (ionic_melt alternates +1 / -1 by index)
    for s in train_seeds:
        tr.add_snapshot(*coords(s)[0])
    tr.fit_radial()
    tr.build_dataset()
    losses = tr.train(epochs=6, lr=2e-3)
    assert losses[-1] < losses[0]
    errs = {"fine": [], "raw": [], "coarse": [], "radial": [], "learned": []}
    ones = pd.learned.MLPNetwork(pd.learned.init_params(0, s0=1.0, out_scale=0.0))
    raw = pd.ElectrostaticsSolver(tr.coarse_spec, box, q, nmax=n)   # coarse mesh, self force kept
    for s in test_seeds:
        (x, y, z), pos = coords(s)
        rq = torch.tensor(np.concatenate([pos, q[:, None]], 1), dtype=torch.float64, device="cuda").contiguous()
        Fk, _ = pd.learned.ewald_oracle(rq, box, spec.C, spec.alpha, digits=10, parts=2)
        Ft, _ = pd.learned.ewald_oracle(rq, box, spec.C, spec.alpha, digits=10, parts=3)
        fine = tr.mesh_forces(tr.fine, x, y, z).double()
        coarse = tr.mesh_forces(tr.coarse, x, y, z).double()
        rad = coarse + tr.corr.correction(ones, x, y, z, tr.q, tr.typ)[:, :3].double()
        lea = coarse + tr.corr.correction(tr.net, x, y, z, tr.q, tr.typ)[:, :3].double()
        den = torch.sqrt((Ft ** 2).sum())
        forms = (("fine", fine), ("raw", tr.mesh_forces(raw, x, y, z).double()), ("coarse", coarse),
                 ("radial", rad), ("learned", lea))
        for k, f in forms:
            errs[k].append(float(torch.sqrt(((f - Fk) ** 2).sum()) / den))
    e = {k: float(np.mean(v)) for k, v in errs.items()}
    print("held-out relative RMS reciprocal-force error:", e)
    assert e["fine"] < e["coarse"] < 0.95 * e["raw"]
    assert e["learned"] < 0.95 * e["coarse"]
    assert e["learned"] <= 1.02 * e["radial"]


def test_descriptors_of_isolated_and_sparse_ions(pd, lo, cuda):
    # an ion with no neighbour inside the cutoff has zero features and a zero residual direction; a
    # sparse system (few ions per row) still matches the direct pair loop
    import torch
    L = 40.0
    pos = np.array([[0.0, 0.0, 0.0], [15.0, 15.0, 15.0], [17.5, 15.0, 15.0], [-15.0, 12.0, 3.0],
                    [-13.0, 13.0, 4.0], [5.0, -18.0, 9.0]])
    q = np.array([1.0, -1.0, 1.0, -1.0, 1.0, -1.0])
    typ = np.where(q > 0, 1, 2).astype(np.int32)
    box = (L, L, L)
    n = len(pos)
    lc = pd.learned.LearnedCorrection(n, box, cap=8)
    lc.set_radial(np.linspace(0.5, -0.5, lc.nb))
    t = [torch.tensor(pos[:, d], dtype=torch.float32, device=cuda) for d in range(3)]
    X, V = lc.descriptors(*t, torch.tensor(q, dtype=torch.float32, device=cuda), torch.tensor(typ, device=cuda))
    cfg = lc.cfg
    Xr, Vr, _ = lo.descriptors(pos.astype(np.float32), q, typ, box, rcut=cfg["rcut"], mu0=cfg["mu0"],
                               dmu=cfg["dmu"], sigma=cfg["sigma"], nb=cfg["nb"], nu0=cfg["nu0"], dnu=cfg["dnu"],
                               tau=cfg["tau"], coef=lc.coef)
    Xg, Vg = X.float().cpu().numpy(), V.cpu().numpy()[:, :3]
    for i in (0, 5):   # no neighbour within 6 A
        assert not Xg[i].any() and not Vg[i].any()
    assert np.all(np.abs(Xg - Xr) <= 2.0 ** -7 * np.abs(Xr) + 1e-4)
    assert np.allclose(Vg, Vr, rtol=2e-5, atol=1e-6)

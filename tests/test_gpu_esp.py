"""ESP (prolate split and window) on the mesh engine against the FP64 ESP oracle and the Ewald sum
(GPU, through the C ABI).

The oracle (oracle/esp_oracle.py) evaluates the prolate function by a Nystrom discretisation of the
finite Fourier transform, independently of the library's host setup, and reproduces the Ewald sum of
the reference's ESP case (test/test_electrostatics.jl:309) to 1e-6.  Bounds here: the FP32 mesh
against the FP64 oracle mesh 1e-5 relative RMS force (the parity bound of the other meshes); the full
FP32 solver against the Ewald sum 1e-4 (the reference's FP32 bound, test/test_electrostatics.jl:553-565).
"""
import importlib.util
import math
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def eo():
    spec = importlib.util.spec_from_file_location("pdb200_esp_oracle", ROOT / "oracle" / "esp_oracle.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _cloud(n, L, seed):
    rng = np.random.default_rng(seed)
    R = rng.uniform(0, 1, (n, 3)) * np.asarray(L)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    return R.astype(np.float32).astype(np.float64), q


def _spec(pd, C, rc, eps, mesh, P, kind="esp"):
    c = pd.prolates.prolate_shape_for_tolerance(eps)
    c1 = pd.prolates.prolate_shape_for_tolerance(eps / 2)
    return pd.ElectrostaticsSpec(coulomb_prefactor=C, real_cutoff=rc, influence=kind, order=P, mesh=mesh,
                                 split_shape=c, window_shape=c1), c, c1


def _dev(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")


def _mesh_forces(pd, solver, R, q):
    import torch
    n = len(q)
    x, y, z = (_dev(R[:, d]) for d in range(3))
    qq = _dev(q)
    f = [torch.zeros(n, device="cuda") for _ in range(3)]
    e = torch.zeros(n, device="cuda")
    vg = torch.zeros(6, device="cuda")
    solver.transform(x, y, z, qq, energy=True)
    solver.gather(x, y, z, qq, *f, epot=e, vglobal=vg, energy=True, set=True)
    torch.cuda.synchronize()
    acc = solver.mesh_energy()
    return torch.stack(f, 1).double().cpu().numpy(), e.double().cpu().numpy(), acc, vg.double().cpu().numpy()


@pytest.mark.parametrize("kind", ["esp", "esp_deconvolution"])
def test_influence_matches_oracle(pd, eo, cuda, kind):
    C, rc, L = 1.7, 4.0, (14.0, 15.0, 16.0)
    spec, c, c1 = _spec(pd, C, rc, 1e-5, (16, 18, 20), 8, kind)
    q = np.array([1.0, -1.0])
    solver = pd.ElectrostaticsSolver(spec, L, q, nmax=2)
    G, Vc = solver.influence()
    Gr, Vr = eo.influence(kind, eo.Window(8, c1), eo.Split(rc, c), (16, 18, 20), L, C, nmax=2)
    assert np.max(np.abs(G - Gr)) < 2e-6 * np.max(np.abs(Gr))
    assert np.max(np.abs(Vc - Vr)) < 2e-6 * np.max(np.abs(Vr))
    solver.close()


@pytest.mark.parametrize("kind", ["esp", "esp_deconvolution"])
def test_mesh_forces_match_oracle(pd, eo, cuda, kind):
    # the reference's ESP case (C = 1.7, r_c = 4, 120 ions in 14 x 15 x 16, eps 1e-6, mesh 32 x 32 x 36,
    # width 8): FP32 mesh forces, energy and virial against the FP64 oracle mesh
    C, rc, L = 1.7, 4.0, (14.0, 15.0, 16.0)
    R, q = _cloud(120, L, 3)
    spec, c, c1 = _spec(pd, C, rc, 1e-6, (32, 32, 36), 8, kind)
    solver = pd.ElectrostaticsSolver(spec, L, q, nmax=len(q))
    F, E, acc, vg = _mesh_forces(pd, solver, R, q)
    ref = eo.mesh(R, q, L, (32, 32, 36), eo.Window(8, c1), eo.Split(rc, c), kind, C=C, nmax=2)
    rel = np.linalg.norm(F - ref["F"]) / np.linalg.norm(ref["F"])
    assert rel < 1e-5, rel
    assert math.isclose(acc[0], ref["Emesh"], rel_tol=1e-5)
    assert math.isclose(E.sum(), ref["E"].sum(), rel_tol=1e-5)
    assert np.max(np.abs(vg - ref["W"])) < 1e-5 * abs(ref["W"][:3].sum())
    solver.close()


def test_solver_against_ewald(pd, ora, cuda, kats):
    # the whole ESP solver (cluster-pair real space through the fitted prolate correction, mesh, self)
    # through the workflow against the Ewald sum, at the reference's ESP case
    k = kats["esp"]["solver"]
    C, rc, L = 1.7, 4.0, (14.0, 15.0, 16.0)
    R, q = _cloud(120, L, 3)
    system = pd.ParticleSystem(R, L, charges=q, masses=np.ones(len(q)))
    f = pd.ESP(coulomb_prefactor=C, real_cutoff=rc, tolerance=k["eps"], order=k["order"], mesh=tuple(k["mesh"]),
               neighborlist=pd.ClusterPairList(buffer=0.5))
    sim = pd.Simulation(system, pd.Integrator(dt=1e-3, forces=[f]))
    pd.evaluate_forces_into_f(sim, energy=True)
    st = sim.state
    E0, F0, W0 = ora.ewald(st.positions(), q, L, C=C)
    F = st.forces()
    rel = np.linalg.norm(F - F0) / np.linalg.norm(F0)
    assert rel < 1e-4, rel
    assert abs(st.potential_energy() - E0) < 1e-5 * abs(E0)
    W = st.virial_tensor()
    assert np.max(np.abs(np.array([W["xx"], W["yy"], W["zz"]]) - np.diag(W0))) < 1e-4 * abs(np.trace(W0))


def test_melt_and_step(pd, ora, eo, cuda):
    # a 4000-ion LJ + ESP melt (tolerance 1e-5 rules: width 8, spacing pi r_c / c) through the workflow:
    # total forces, energy and virial against the FP64 oracle (LJ pairs + ESP real space + mesh + self),
    # then 20 captured NVE steps and the forces again
    n = 4000
    L = (n / 0.0375) ** (1 / 3)
    pos, q, box = pd.synthetic.ionic_melt(n, L, 2.2, seed=7)
    m = pd.synthetic.melt_masses(q)
    v = pd.synthetic.maxwell_boltzmann(m, 1200.0, seed=8, kB=pd.synthetic.KB_EV)
    system = pd.ParticleSystem(pos, box, types=["Na", "Cl"], typeids=np.where(q > 0, 1, 2), masses=m, charges=q,
                               velocities=v)
    Cc = pd.synthetic.COULOMB_EV_A
    lj = pd.LennardJones(epsilon=0.01, sigma=2.8, cutoff=9.0, pairs="neighborlist",
                         neighborlist=pd.ClusterPairList(buffer=1.0, prune_buffer=0.3))
    el = pd.ESP(coulomb_prefactor=Cc, real_cutoff=9.0, tolerance=1e-5)
    sim = pd.Simulation(system, pd.Integrator(dt=1.0 / pd.synthetic.TIME_UNIT_FS, forces=[lj, el]))
    st = sim.state
    spec = st.solver.spec
    win, split = eo.Window(spec.order, spec.window_shape), eo.Split(9.0, spec.split_shape)

    def check():
        pd.evaluate_forces_into_f(sim, energy=True)
        P = st.positions()
        ref = eo.total(P, q, box, st.solver.mesh, win, split, "esp", C=Cc, nmax=2)
        ljr = ora.pairs_cells(P, box, kind=1, sigma=2.8, eps=0.01, rc_lj=9.0)
        Fr = ref["F"] + ljr["F"]
        F = st.forces()
        rel = np.linalg.norm(F - Fr) / np.linalg.norm(Fr)
        assert rel < 1e-5, rel
        Er = ref["Etot"] + ljr["E"].sum()
        assert abs(st.potential_energy() - Er) < 1e-5 * abs(Er)
        W = st.virial_tensor()
        Wr = ref["W"] + ljr["W"].sum(0)
        W6 = np.array([W[k] for k in ("xx", "yy", "zz", "xy", "xz", "yz")])
        assert np.max(np.abs(W6 - Wr)) < 1e-4 * abs(Wr[:3].sum())

    check()
    st.step(20, use_graph=True)
    st.synchronize()
    assert np.isfinite(st.positions()).all() and st.cluster.statistics()["error"] == 0
    check()

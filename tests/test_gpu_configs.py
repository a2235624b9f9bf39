"""The uncharged configurations at their full sizes against the FP64 oracle (GPU, through the C ABI).

* 3D LJ fluid, 1 048 576 atoms (fcc 64^3 x 4 at rho 0.8442, T 0.72, r_c 2.5, skin 0.3, NVE dt 0.005) on
  the ELL route: every atom's force, the energy and the virial, at the start and after 100 steps of
  device list maintenance.
* 2D WCA disks, 1 048 576 (packing 0.7, eps 10, Langevin gamma 50, kT 1, dt 2e-4): the same checks.
* 512 LJ / WCA replicas (2.7 M atoms, N log-uniform in [500, 20 000]) as one batch: a spread of 24
  replicas against the all-pairs FP64 sum, at the start and after 50 batched steps.

Tolerance: the reference's FP32 bound, 2e-5 relative RMS force (test/test_cluster_pairs.jl:79-86,
test/test_force_precision_gpu.jl:39), and 2e-5 of the total energy and virial.  In the dense replicas
(rho up to 0.9) close contacts make the net forces much smaller than the pair forces they sum, so there
every particle's force is held to the FP32 precision of that sum instead: |F_i - F_i(FP64)| <= 64 eps_32
sum_j (|f_rep| + |f_att|)_ij (each pair force to a few ulps of its repulsive and attractive terms, the
r^-13 power included; the terms cancel at the WCA cutoff) plus the force of any pair within a relative
1e-6 of the truncated LJ cutoff (FP32 rounding of r^2 may count it on either side), and the energy to 2e-5
or, where the WCA pair energies u + eps nearly vanish, to the same multiple of
eps_32 sum (|u_rep| + |u_att| + eps).
"""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

TOL = 2e-5


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _embed(pos, box, height):
    p3 = np.zeros((len(pos), 3))
    p3[:, :2] = pos
    return p3, (box[0], box[1], height)


def _check_state(pd, ora, st, kind, **kw):
    pos = st.positions()
    if st.dim == 2:
        p3, b3 = _embed(pos, st.box, 8.0)
        ref = ora.pairs_cells(p3, b3, kind=kind, **kw)
        Fref, Wref = ref["F"][:, :2], ref["W"].sum(0)[[0, 1, 3]]
        W = st.virial_tensor()
        W = np.array([W["xx"], W["yy"], W["xy"]])
    else:
        ref = ora.pairs_cells(pos, st.box, kind=kind, **kw)
        Fref, Wref = ref["F"], ref["W"].sum(0)
        W = st.virial_tensor()
        W = np.array([W[k] for k in ("xx", "yy", "zz", "xy", "xz", "yz")])
    F = st.forces()
    assert _rel(F, Fref) < TOL, _rel(F, Fref)
    E, Eref = st.potential_energy(), ref["E"].sum()
    assert abs(E - Eref) < TOL * abs(Eref), (E, Eref)
    assert np.max(np.abs(W - Wref)) < TOL * np.abs(Wref[:st.dim]).sum(), (W, Wref)


def test_lj_fluid_1m(pd, ora, cuda):
    pos, box = pd.synthetic.fcc_lattice(64, 0.8442, 0.05)
    assert len(pos) == 1048576
    m = np.ones(len(pos))
    v = pd.synthetic.maxwell_boltzmann(m, 0.72, seed=2026)
    force = pd.LennardJones(epsilon=1.0, sigma=1.0, cutoff=2.5, pairs="neighborlist",
                            neighborlist=pd.CellList(buffer=0.3, capacity=96, rebuild_interval=10))
    sim = pd.Simulation(pd.ParticleSystem(pos, box, masses=m, velocities=v),
                        pd.Integrator(dt=0.005, forces=[force], methods=[pd.ConstantVolume()]))
    st = sim.state
    kw = dict(sigma=1.0, eps=1.0, rc_lj=2.5)
    pd.evaluate_forces_into_f(sim, energy=True)
    _check_state(pd, ora, st, 1, **kw)
    st.step(100)
    st.synchronize()
    s = st._ell_check()
    assert s["step"] == 100 and s["builds"] >= 2
    pd.evaluate_forces_into_f(sim, energy=True)
    _check_state(pd, ora, st, 1, **kw)


def test_wca_disks_1m(pd, ora, cuda):
    pos, box = pd.synthetic.hex_random_2d(1024, 0.7, 1.0, 0.25, seed=2026)
    assert len(pos) == 1048576
    m = np.ones(len(pos))
    v = pd.synthetic.maxwell_boltzmann(m, 1.0, seed=2026, dim=2)
    force = pd.WCA(epsilon=10.0, sigma=1.0, pairs="neighborlist",
                   neighborlist=pd.CellList(buffer=0.4, capacity=32, rebuild_interval=10))
    sim = pd.Simulation(pd.ParticleSystem(pos, box, masses=m, velocities=v),
                        pd.Integrator(dt=2e-4, forces=[force], methods=[pd.Langevin(gamma=50.0, kT=1.0)]), seed=2026)
    st = sim.state
    kw = dict(sigma=1.0, eps=10.0, rc_lj=float(np.sqrt(np.float32(1.2599211))))
    pd.evaluate_forces_into_f(sim, energy=True)
    _check_state(pd, ora, st, 2, **kw)
    st.step(100)
    st.synchronize()
    s = st._ell_check()
    assert s["step"] == 100 and s["builds"] >= 2
    pd.evaluate_forces_into_f(sim, energy=True)
    _check_state(pd, ora, st, 2, **kw)


def test_replica_set_512(pd, ora, cuda):
    import torch
    specs = pd.synthetic.replica_set(512, seed=2026)
    systems = pd.batch.make_systems(specs)
    b = pd.batch.BatchedReplicas(systems, skin=0.3)
    ns = np.array([s["n"] for s in systems])
    pick = sorted(set(np.linspace(0, len(systems) - 1, 22).astype(int).tolist()
                      + [int(np.argmin(ns)), int(np.argmax(ns))]))

    def check():
        b.evaluate(energy=True)
        st = b.status()
        assert st["error"] == 0 and st["valid"]
        for k in pick:
            s = systems[k]
            pos = np.stack([b.replica(k, t).double().cpu().numpy() for t in (b.x, b.y, b.z)], 1)
            kw = dict(kind=1, sigma=1.0, eps=1.0, rc_lj=2.5) if s["kind"] == "lj" else \
                dict(kind=2, sigma=1.0, eps=1.0, rc_lj=float(np.sqrt(np.float32(1.2599211))))
            ref = ora.pairs_direct(pos, s["box"], **kw)
            F = torch.stack([b.replica(k, t) for t in (b.fx, b.fy, b.fz)], 1).double().cpu().numpy()
            S, SE, A = ora.pair_term_scales(pos, s["box"], **kw)
            eps32 = float(np.finfo(np.float32).eps)
            dev = np.linalg.norm(F - ref["F"], axis=1)
            bound = 64 * eps32 * S + A + 1e-9
            assert np.all(dev <= bound), (k, s["kind"], s["n"], float(np.max(dev / bound)), _rel(F, ref["F"]))
            E, Eref = float(b.replica(k, b.epot).double().sum()), float(ref["E"].sum())
            assert abs(E - Eref) < max(TOL * abs(Eref), 64 * eps32 * SE), (k, E, Eref, SE)

    check()
    b.step(50, 0.005)
    b.synchronize()
    assert b.status()["step"] == 50
    check()

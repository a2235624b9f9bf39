"""Batched charged melts on the GPU: one launch per force stage over every replica (the real-space
Coulomb polynomial in the row pair kernel, one SPME mesh per replica spread, multiplied and gathered over
all replicas, batched cuFFT per mesh size).  Each replica's forces and energy against the FP64 oracle's
PME sum at the replica's own mesh; the spread tiles and lanes against each other; the captured step
against the eager one and against each replica's single-system engine."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ALPHA_TOL = 1e-5
RC = 9.0


def _batch(pd, ns, seed=5, skin=1.0, lanes=4, tile=64, kind="spme"):
    systems = pd.batch.melt_systems(ns, seed=seed)
    alpha = pd.splits.alpha_from_tolerance(RC, ALPHA_TOL)
    el = dict(alpha=alpha, C=pd.synthetic.COULOMB_EV_A, rc=RC, order=5, kind=kind, spacing=1.0)
    b = pd.batch.BatchedReplicas(systems, skin=skin, lanes=lanes, electrostatics=el)
    b.set_spread_tile(tile)
    return b, systems, alpha


def _oracle(pd, ora, s, K, alpha, pos, kind="spme"):
    return ora.pme_total(pos, s["charges"], s["box"], C=pd.synthetic.COULOMB_EV_A, alpha=alpha, rc=RC, K=K, P=5,
                         kind=kind, lj=dict(sigma=2.8, eps=0.01, rc=RC))


@pytest.mark.parametrize("kind", ["spme", "p3m_ad"])
def test_batched_melts_match_the_oracle(pd, ora, cuda, kind):
    ns = [600, 1000, 1400, 2200, 3000]
    b, systems, alpha = _batch(pd, ns, kind=kind)
    info = b.mesh_info()
    assert info["groups"] == len({tuple(m) for m in b.meshes})
    b.evaluate(energy=True)
    st = b.status()
    assert st["valid"] and st["error"] == 0
    for k, s in enumerate(systems):
        pos = np.stack([b.replica(k, t).cpu().numpy() for t in (b.x, b.y, b.z)], 1).astype(float)
        F = np.stack([b.replica(k, t).cpu().numpy() for t in (b.fx, b.fy, b.fz)], 1).astype(float)
        E = float(b.replica(k, b.epot).double().sum())
        ref = _oracle(pd, ora, s, b.meshes[k], alpha, pos, kind=kind)
        rel = np.linalg.norm(F - ref["F"]) / np.linalg.norm(ref["F"])
        assert rel < 1e-5, (k, rel)   # the parity bound: 1e-5 relative RMS force
        assert abs(E - ref["Etot"]) < 1e-5 * abs(ref["Etot"]), (k, E, ref["Etot"])


def test_spread_tiles_and_lanes_agree(pd, cuda):
    b, systems, _ = _batch(pd, [800, 1700, 2500], seed=9)
    results = []
    for lanes, tile in ((1, (32, 2)), (4, (64, 2)), (8, (32, 2)), (2, (64, 4)), (1, (64, 4))):
        b.set_lanes(lanes)
        b.set_spread_tile(*tile)
        b.evaluate(energy=True)
        results.append((np.stack([t.cpu().numpy() for t in (b.fx, b.fy, b.fz)], 1), b.epot.double().sum().item()))
    F0, E0 = results[0]
    for F, E in results[1:]:
        assert np.linalg.norm(F - F0) / np.linalg.norm(F0) < 2e-6
        assert abs(E - E0) < 1e-6 * abs(E0)


def test_batched_steps_match_single_system_engines(pd, cuda):
    """30 captured batched NVE steps against each replica's own single-system engine (cluster list + SPME,
    the same mesh), from the same start: positions within 1e-4 A."""
    ns = [700, 1600, 2600]
    b, systems, alpha = _batch(pd, ns, seed=13)
    dt = 1.0 / pd.synthetic.TIME_UNIT_FS
    b.evaluate()
    b.step(30, dt, use_graph=True)
    b.synchronize()
    assert b.status()["error"] == 0
    for k, s in enumerate(systems):
        system = pd.ParticleSystem(s["positions"], s["box"], types=["Na", "Cl"],
                                   typeids=np.where(s["charges"] > 0, 1, 2), masses=s["masses"],
                                   charges=s["charges"], velocities=s["velocities"])
        lj = pd.LennardJones(epsilon=0.01, sigma=2.8, cutoff=RC, pairs="neighborlist",
                             neighborlist=pd.ClusterPairList(buffer=1.0, prune_buffer=0.3))
        el = pd.PME(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=RC, alpha=alpha, mesh=b.meshes[k],
                    order=5)
        sim = pd.Simulation(system, pd.Integrator(dt=dt, forces=[lj, el]))
        pd.run(sim, pd.Stage(steps=30))
        P1 = sim.state.positions()
        P2 = np.stack([b.replica(k, t).cpu().numpy() for t in (b.x, b.y, b.z)], 1).astype(float)
        L = np.asarray(s["box"])
        d = P2 - P1
        d -= L * np.round(d / L)
        assert np.abs(d).max() < 1e-4, (k, np.abs(d).max())


def test_graph_equals_eager_and_energy_is_conserved(pd, cuda):
    ns = [900, 1900]
    dt = 1.0 / pd.synthetic.TIME_UNIT_FS
    a, systems, _ = _batch(pd, ns, seed=17)
    c, _, _ = _batch(pd, ns, seed=17)
    for bb in (a, c):
        bb.evaluate()
    a.step(20, dt, use_graph=True)
    c.step(20, dt, use_graph=False)
    a.synchronize()
    c.synchronize()
    Pa = np.stack([t.cpu().numpy() for t in (a.x, a.y, a.z)], 1)
    Pc = np.stack([t.cpu().numpy() for t in (c.x, c.y, c.z)], 1)
    assert np.abs(Pa - Pc).max() < 1e-4

    def total_energy(bb):
        bb.evaluate(energy=True)
        m = np.concatenate([np.broadcast_to(s["masses"], (s["n"],)) for s in systems])
        v2 = sum(t.double().cpu().numpy() ** 2 for t in (bb.vx, bb.vy, bb.vz))
        return 0.5 * float((m * v2).sum()) + float(bb.epot.double().sum())

    E0 = total_energy(a)
    a.step(200, dt, use_graph=True)
    a.synchronize()
    E1 = total_energy(a)
    assert abs(E1 - E0) < 1e-3 * abs(E0), (E0, E1)   # over 200 fs at 1 fs


def test_batched_melt_errors(pd, cuda):
    systems = pd.batch.melt_systems([600, 900], seed=3)
    alpha = pd.splits.alpha_from_tolerance(RC, ALPHA_TOL)
    b = pd.batch.BatchedReplicas(systems, skin=1.0)
    arr = (C.c_int * 6)(*([40] * 6))
    with pytest.raises(pd._native.NativeError, match="Coulomb terms first"):
        pd._native.call("pd_batch_set_mesh", b.handle, 1, 5, alpha, 14.4, arr)
    with pytest.raises(pd._native.NativeError, match="32 or 64"):
        b.set_spread_tile(48)
    with pytest.raises(pd._native.NativeError, match="4 with tiles of 64"):
        b.set_spread_tile(32, 4)
    systems[0]["charges"] = systems[0]["charges"].copy()
    systems[0]["charges"][0] += 1.0
    with pytest.raises(ValueError, match="net charge"):
        pd.batch.BatchedReplicas(systems, skin=1.0, electrostatics=dict(alpha=alpha, C=14.4, rc=RC, spacing=1.0))


@pytest.mark.slow
def test_the_64_melt_set_at_full_size(pd, ora, cuda):
    """The benchmark's 64 melts (760 278 ions) as one batch: every melt's forces equal its own
    single-system engine's (cluster list + SPME at the same mesh) within 1e-5 relative RMS, and the
    smallest, a middle and the largest melt equal the FP64 oracle's PME sum within 1e-5."""
    ns = pd.batch.melt_sizes(64, 2026 + 64)
    systems = pd.batch.melt_systems(ns, seed=2026)
    alpha = pd.splits.alpha_from_tolerance(RC, ALPHA_TOL)
    el = dict(alpha=alpha, C=pd.synthetic.COULOMB_EV_A, rc=RC, order=5, kind="spme", spacing=1.0)
    b = pd.batch.BatchedReplicas(systems, skin=1.2, lanes=1, electrostatics=el)
    b.evaluate()
    assert b.status()["error"] == 0 and b.mesh_info()["groups"] == len({tuple(m) for m in b.meshes})
    for k, s in enumerate(systems):
        F = np.stack([b.replica(k, t).cpu().numpy() for t in (b.fx, b.fy, b.fz)], 1).astype(float)
        system = pd.ParticleSystem(s["positions"], s["box"], types=["Na", "Cl"],
                                   typeids=np.where(s["charges"] > 0, 1, 2), masses=s["masses"],
                                   charges=s["charges"], velocities=s["velocities"])
        lj = pd.LennardJones(epsilon=0.01, sigma=2.8, cutoff=RC, pairs="neighborlist",
                             neighborlist=pd.ClusterPairList(buffer=1.0, prune_buffer=0.3))
        pme = pd.PME(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=RC, alpha=alpha, mesh=b.meshes[k],
                     order=5)
        sim = pd.Simulation(system, pd.Integrator(dt=1.0 / pd.synthetic.TIME_UNIT_FS, forces=[lj, pme]))
        pd.evaluate_forces_into_f(sim)
        Fs = sim.state.forces()
        rel = np.linalg.norm(F - Fs) / np.linalg.norm(Fs)
        assert rel < 1e-5, (k, s["n"], rel)
        del sim
    order = np.argsort(ns)
    for k in (order[0], order[len(order) // 2], order[-1]):
        s = systems[k]
        pos = np.stack([b.replica(k, t).cpu().numpy() for t in (b.x, b.y, b.z)], 1).astype(float)
        F = np.stack([b.replica(k, t).cpu().numpy() for t in (b.fx, b.fy, b.fz)], 1).astype(float)
        ref = _oracle(pd, ora, s, b.meshes[k], alpha, pos)
        assert np.linalg.norm(F - ref["F"]) / np.linalg.norm(ref["F"]) < 1e-5, (k, s["n"])

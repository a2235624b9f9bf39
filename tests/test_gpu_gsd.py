"""GSD snapshot I/O on the GPU: the device frame packing against the state's arrays, the reference's own GSD
cases (test/test_io_gsd.jl: a 2D frame, chemical properties, append, the virial chunks), scheduled writer
frames against the state after each run, and restarts from a frame (ParticleSystem.from_gsd +
electrostatics_from_gsd) that reproduce the original solver and forces."""
import importlib.util
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def gsdo():
    spec = importlib.util.spec_from_file_location("pdb200_gsd_oracle", ROOT / "oracle" / "gsd_oracle.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _tiny(pd, dim, typeids, seed=0, n=8):
    rng = np.random.default_rng(seed)
    box = (20.0,) * dim
    # a loose lattice plus jitter keeps the WCA pairs apart
    side = int(np.ceil(n ** (1 / dim)))
    grid = np.stack(np.meshgrid(*[np.arange(side)] * dim, indexing="ij"), -1).reshape(-1, dim)[:n]
    pos = grid * (20.0 / side) - 10.0 + rng.uniform(-0.3, 0.3, (n, dim))
    system = pd.ParticleSystem(pos, box, types=["A", "B"], typeids=typeids, masses=1.0,
                               velocities=rng.normal(0, 0.4, (n, dim)))
    wca = pd.WCA(epsilon=1.0, sigma=1.0, pairs="neighborlist", neighborlist=pd.CellList(buffer=0.3, capacity=32))
    return pd.Simulation(system, pd.Integrator(dt=1e-3, forces=[wca]))


def _melt(pd, n=4000, kind="PME", seed=7, exclude=False):
    L = (n / 0.0375) ** (1 / 3)
    pos, q, box = pd.synthetic.ionic_melt(n, L, 2.2, seed=seed)
    m = pd.synthetic.melt_masses(q)
    v = pd.synthetic.maxwell_boltzmann(m, 1200.0, seed=seed + 1, kB=pd.synthetic.KB_EV)
    topo = pd.Topology(exclusions=[(1, 2), (5, 9)]) if exclude else None
    system = pd.ParticleSystem(pos, box, types=["Na", "Cl"], typeids=np.where(q > 0, 1, 2), masses=m, charges=q,
                               velocities=v, topology=topo)
    lj = pd.LennardJones(epsilon=0.01, sigma=2.8, cutoff=9.0, pairs="neighborlist",
                         neighborlist=pd.ClusterPairList(buffer=1.0, prune_buffer=0.3))
    common = dict(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=9.0)
    if kind == "PME":
        el = pd.PME(**common, real_space_tolerance=1e-5, mesh_spacing=1.0, order=5,
                    scaled_pairs=((3, 4, 0.5),) if exclude else ())
    elif kind == "PPPM_ik":
        el = pd.PPPM(**common, real_space_tolerance=1e-5, mesh_spacing=1.0, order=5, differentiation="ik")
    else:
        el = pd.ESP(**common, tolerance=1e-4)
    sim = pd.Simulation(system, pd.Integrator(dt=1.0 / pd.synthetic.TIME_UNIT_FS, forces=[lj, el]))
    return sim, lj


def test_snapshot_pack_equals_the_state(pd, cuda):
    import torch

    sim, _ = _melt(pd, 1000)
    st = sim.state
    pd.evaluate_forces_into_f(sim, energy=True)
    stager = pd.gsdio.FrameStager(st, forces=True, virial=True)
    fr = stager.take(stager.stage())
    pos = torch.stack([st.x, st.y, st.z], 1).cpu().numpy()
    vel = torch.stack([st.vx, st.vy, st.vz], 1).cpu().numpy()
    frc = torch.stack([st.fx, st.fy, st.fz], 1).cpu().numpy()
    np.testing.assert_array_equal(fr["position"], pos)     # bit-exact: a copy, no arithmetic
    np.testing.assert_array_equal(fr["velocity"], vel)
    np.testing.assert_array_equal(fr["force"], frc)
    np.testing.assert_array_equal(fr["virial"], st.vir6.cpu().numpy())
    np.testing.assert_array_equal(fr["typeid"], st.typ.cpu().numpy() - 1)
    # 2D: z columns are zero, 3 virial columns
    sim2 = _tiny(pd, 2, np.array([1, 2] * 4))
    pd.evaluate_forces_into_f(sim2, energy=True)
    s2 = sim2.state
    st2 = pd.gsdio.FrameStager(s2, forces=True, virial=True)
    f2 = st2.take(st2.stage())
    assert (f2["position"][:, 2] == 0).all() and (f2["force"][:, 2] == 0).all()
    np.testing.assert_array_equal(f2["position"][:, :2], torch.stack([s2.x, s2.y], 1).cpu().numpy())
    np.testing.assert_array_equal(f2["virial"], s2.vir6.cpu().numpy())
    assert f2["virial"].shape == (8, 3)


def test_reference_tiny_2d_frame(pd, cuda, tmp_path):
    """test_io_gsd.jl:3-38: step, N, D, positions and type ids of a 2D frame."""
    tid = np.array([1, 2, 1, 2, 1, 2, 1, 2])
    sim = _tiny(pd, 2, tid)
    st = sim.state
    path = tmp_path / "tiny_traj.gsd"
    h = pd.gsd_open(path)
    try:
        pd.write_gsd_frame(h, st, step=7, types_names=["A", "B"])
    finally:
        pd.gsd_close(h)
    fr = pd.read_gsd_frame(path)
    assert fr.step == 7 and fr.N == 8 and fr.D == 2
    assert len(fr.rx) == 8 and len(fr.ry) == 8 and fr.rz is None
    assert fr.types == ["A", "B"]
    P = st.positions()
    assert abs(fr.rx.sum() - P[:, 0].sum()) < 1e-5 + 1e-6 * abs(P[:, 0].sum())
    assert abs(fr.ry.sum() - P[:, 1].sum()) < 1e-5 + 1e-6 * abs(P[:, 1].sum())
    assert list(fr.typeid) == list(tid)


def test_reference_chemical_properties(pd, cuda, tmp_path):
    """test_io_gsd.jl:39-58: element diameters from type names, state masses, per-type charges."""
    tid = np.array([1, 2, 2, 1, 2, 2, 1, 2])
    sim = _tiny(pd, 3, tid)
    path = tmp_path / "chemical_properties.gsd"
    with pd.gsd_open(path) as h:
        pd.write_gsd_frame(h, sim.state, types_names=["O", "H"], charge=np.float32([-0.8, 0.4]), step=1)
    fr = pd.read_gsd_frame(path)
    np.testing.assert_allclose(fr.particle_properties["diameter"],
                               np.float32([1.32, 0.62, 0.62, 1.32, 0.62, 0.62, 1.32, 0.62]), rtol=1e-6)
    np.testing.assert_allclose(fr.particle_properties["mass"], np.ones(8, np.float32))
    np.testing.assert_allclose(fr.particle_properties["charge"],
                               np.float32([-0.8, 0.4, 0.4, -0.8, 0.4, 0.4, -0.8, 0.4]), rtol=1e-6)


def test_reference_append(pd, gsdo, cuda, tmp_path):
    """test_io_gsd.jl:60-95: a second handle appends; first and last frames by step, two frames in all."""
    sim = _tiny(pd, 2, np.ones(8, int))
    path = tmp_path / "tiny_traj_append.gsd"
    h1 = pd.gsd_open(path)
    pd.write_gsd_frame(h1, sim.state, step=7, types_names=["A"])
    pd.gsd_close(h1)
    h2 = pd.gsd_open(path, append=True)
    pd.write_gsd_frame(h2, sim.state, step=8, types_names=["A"])
    pd.gsd_close(h2)
    assert pd.read_gsd_frame(path).step == 8
    assert pd.read_gsd_frame(path, step=1).step == 7
    assert gsdo.Reader(path).nframes == 2


def test_reference_virial_chunks(pd, gsdo, cuda, tmp_path):
    """test_io_gsd.jl:97-146: write_virial stores the state's per-particle virial rows under
    particles/virial and particles/property/virial, float32 (type 9), N x 3 in 2D."""
    sim = _tiny(pd, 2, np.ones(8, int))
    pd.step(sim, compute_energy=True)
    st = sim.state
    expected = st.vir6.cpu().numpy()
    path = tmp_path / "tiny_traj_virial.gsd"
    with pd.gsd_open(path) as h:
        pd.write_gsd_frame(h, st, step=st.step_count, types_names=["A"], write_virial=True)
    fr = pd.read_gsd_frame(path)
    assert fr.particle_properties["virial"].shape == expected.shape
    np.testing.assert_allclose(fr.particle_properties["virial"], expected, atol=1e-6, rtol=1e-6)
    r = gsdo.Reader(path)
    for name in ("particles/virial", "particles/property/virial"):
        e = r.entry(0, name)
        assert e is not None and e["type"] == 9 and (e["N"], e["M"]) == expected.shape
        np.testing.assert_allclose(r.chunk(0, name), expected, atol=1e-6, rtol=1e-6)


def test_scheduled_writer_frames_equal_the_state(pd, gsdo, cuda, tmp_path):
    """GSDWriter(every=5) over four runs of 5 steps: each frame holds the state after its run, bit for bit;
    the runs append to one file (frames written while the next steps run)."""
    sim, _ = _melt(pd, 2000)
    path = tmp_path / "traj.gsd"
    sim.writers.append(pd.GSDWriter(str(path), every=5, write_start=False, write_forces=True))
    seen = []
    for _ in range(4):
        pd.run(sim, pd.Stage(steps=5))
        seen.append((sim.state.step_count, sim.state.positions().astype(np.float32),
                     sim.state.velocities().astype(np.float32), sim.state.forces().astype(np.float32)))
    r = gsdo.Reader(path)
    assert r.nframes == 4
    for f, (step, P, V, F) in enumerate(seen):
        assert r.chunk(f, "configuration/step")[0] == step
        np.testing.assert_array_equal(r.chunk(f, "particles/position"), P)
        np.testing.assert_array_equal(r.chunk(f, "particles/velocity"), V)
        np.testing.assert_array_equal(r.chunk(f, "particles/force"), F)
    assert r.chunk(0, "log/electrostatics/settings") is not None
    # one run of 20 steps with every=5 and a start frame writes 5 frames at steps 20, 25, ..., 40
    path2 = tmp_path / "traj2.gsd"
    sim.writers[:] = [pd.GSDWriter(str(path2), every=5)]
    pd.run(sim, pd.Stage(steps=20))
    r2 = gsdo.Reader(path2)
    assert [int(r2.chunk(f, "configuration/step")[0]) for f in range(r2.nframes)] == [20, 25, 30, 35, 40]
    np.testing.assert_array_equal(r2.chunk(4, "particles/position"), sim.state.positions().astype(np.float32))


@pytest.mark.parametrize("kind", ["PME", "PPPM_ik", "ESP"])
def test_restart_from_gsd(pd, cuda, kind, tmp_path):
    """ParticleSystem.from_gsd + electrostatics_from_gsd (src/workflow/System.jl:518-531,
    src/workflow/Electrostatics.jl:347-360): the restored solver has the original's settings and exceptions,
    and the restored simulation's forces equal the original's at the frame's coordinates."""
    sim, lj = _melt(pd, 2000, kind=kind, exclude=(kind == "PME"))
    pd.run(sim, pd.Stage(steps=10))
    st = sim.state
    path = tmp_path / "restart.gsd"
    with pd.gsd_open(path) as h:
        pd.write_gsd_frame(h, st, types_names=sim.system.types, step=st.step_count)
    system = pd.ParticleSystem.from_gsd(path)
    el = pd.electrostatics_from_gsd(path)
    assert el is not None
    sim2 = pd.Simulation(system, pd.Integrator(dt=sim.integrator.dt, forces=[lj, el]))
    s2 = sim2.state
    np.testing.assert_array_equal(pd.settings_record(s2.solver), pd.settings_record(st.solver))
    assert s2.exceptions == st.exceptions
    np.testing.assert_array_equal(s2.positions(), st.positions())
    np.testing.assert_array_equal(s2.velocities(), st.velocities())
    np.testing.assert_array_equal(s2.masses, st.masses.astype(np.float32))
    pd.evaluate_forces_into_f(sim, energy=True)
    pd.evaluate_forces_into_f(sim2, energy=True)
    F1, F2 = st.forces(), s2.forces()
    assert np.linalg.norm(F2 - F1) / np.linalg.norm(F1) < 1e-6
    assert abs(s2.potential_energy() - st.potential_energy()) < 1e-6 * abs(st.potential_energy())

"""ELL route (cell list, neighbour rows, row pair kernels, NVE and Langevin steps) against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")


def _engine(pd, pos, box, **kw):
    return pd.ELLEngine(len(pos), box, dim=len(box), **kw)


def _forces(pd, eng, pos, energy=True):
    import torch
    n, dim = pos.shape
    xs = [_dev(pos[:, d]) for d in range(dim)] + [None] * (3 - dim)
    fs = [torch.zeros(n, device="cuda") for _ in range(dim)] + [None] * (3 - dim)
    e = torch.zeros(n, device="cuda")
    w = torch.zeros((n, 6 if dim == 3 else 3), device="cuda")
    eng.update(*xs)
    eng.forces(*xs, *fs, e, w, energy=energy)
    torch.cuda.synchronize()
    F = torch.stack(fs[:dim], 1).double().cpu().numpy()
    return F, e.double().cpu().numpy(), w.double().cpu().numpy()


def _embed(pos, box, rl):
    """2D positions and box as 3D for the oracle (z = 0, a box height above three list radii)."""
    if len(box) == 3:
        return np.asarray(pos, np.float64), tuple(box)
    p3 = np.zeros((len(pos), 3))
    p3[:, :2] = pos
    return p3, (box[0], box[1], 4.0 * rl)


def _lj_fluid(pd, ncell=10, rho=0.8442):
    pos, box = pd.synthetic.fcc_lattice(ncell, rho, 0.05)
    return pos.astype(np.float32).astype(np.float64), box


def _disks(pd, n_side=48, phi=0.7):
    pos, box = pd.synthetic.hex_random_2d(n_side, phi, 1.0, 0.25, seed=3)
    return pos.astype(np.float32).astype(np.float64), box


def _rows_match(pd, ora, eng, pos, box, rl):
    rows, counts = eng.rows_host()
    p3, b3 = _embed(pos, box, rl)
    # pairs within a relative 1e-5 of the list radius may fall either side in FP32
    inner = ora.neighbor_rows(p3, b3, rl * (1 - 1e-5))
    outer = ora.neighbor_rows(p3, b3, rl * (1 + 1e-5))
    for i in range(len(pos)):
        got = set(rows[i].tolist())
        assert len(got) == len(rows[i]) == counts[i]
        assert set(inner[i]) <= got <= set(outer[i]), i


@pytest.mark.parametrize("case", ["lj3d", "wca2d"])
def test_rows_match_oracle(pd, ora, cuda, case):
    # reference_neighbor_rows (test/neighbor_reference.jl:6-16): every j within the list radius, once
    if case == "lj3d":
        pos, box = _lj_fluid(pd, 8)
        eng = _engine(pd, pos, box, model="lj", cutoff=2.5, skin=0.3, capacity=128)
        rl = 2.8
    else:
        pos, box = _disks(pd)
        eng = _engine(pd, pos, box, model="wca", epsilon=10.0, skin=0.4, capacity=32)
        rl = float(np.sqrt(np.float32(1.2599211))) + 0.4
    _forces(pd, eng, pos)
    st = eng.status()
    assert st["valid"] and st["error"] == 0 and st["builds"] == 1
    _rows_match(pd, ora, eng, pos, box, rl)
    eng.close()


def test_known_answer_rows(pd, cuda, kats):
    # test/test_neighbor_reference.jl:2-4 through the device rows: each row i with its own radius
    # (the first case crosses the periodic seam of a 10-cell 2D grid)
    for case in kats["neighbor_rows"]:
        coords = np.asarray(case["coords"], np.float64).T
        L = np.asarray(case["box"], np.float64)
        coords = coords - L * np.round(coords / L)   # the device rows take centred coordinates
        for i, (radius, want) in enumerate(zip(case["radii"], case["rows"])):
            eng = _engine(pd, coords, tuple(case["box"]), model="lj", cutoff=radius, skin=0.0, capacity=4)
            _forces(pd, eng, coords)
            rows, _ = eng.rows_host()
            assert sorted(rows[i].tolist()) == [j - 1 for j in want], (case["source"], i)
            eng.close()


def _check_forces(F, E, W, ref, tol=2e-5):
    nF = np.linalg.norm(ref["F"])
    assert np.linalg.norm(F - ref["F"]) / nF < tol
    assert abs(E.sum() - ref["E"].sum()) / max(abs(ref["E"].sum()), 1e-30) < tol
    assert np.max(np.abs(W.sum(0) - ref["W"])) / max(np.abs(ref["W"][:2]).sum(), 1e-30) < tol


@pytest.mark.parametrize("shift", [False, True])
def test_lj3d_forces(pd, ora, cuda, shift):
    # _lj3_ell_kernel_virial! (LJELLEngineKernels.jl:45-79): C0 state point, FP32 tolerance 2e-5
    pos, box = _lj_fluid(pd, 10)
    eng = _engine(pd, pos, box, model="lj", cutoff=2.5, skin=0.3, shift=shift)
    F, E, W = _forces(pd, eng, pos)
    esh = pd.splits.lj_cutoff_energy(1.0, 1.0, 2.5) if shift else 0.0
    ref = ora.pairs_cells(pos, box, kind=1, sigma=1.0, eps=1.0, rc_lj=2.5, eshift_lj=esh)
    _check_forces(F, E, W, dict(F=ref["F"], E=ref["E"], W=ref["W"].sum(0)))
    F2, _, _ = _forces(pd, eng, pos, energy=False)
    assert np.max(np.abs(F - F2)) < 1e-5 * np.max(np.abs(F))   # the variants differ in contraction only
    eng.close()


@pytest.mark.parametrize("dim", [2, 3])
def test_wca_forces(pd, ora, cuda, dim):
    # UniformWCA (PairModels.jl:13-49): rc^2 = 1.2599211 sigma^2, u + eps; 2D disks at packing 0.7
    if dim == 3:
        pos, box = _lj_fluid(pd, 8)
        eps = 1.0
    else:
        pos, box = _disks(pd)
        eps = 10.0
    rc = float(np.sqrt(np.float32(1.2599211)))
    eng = _engine(pd, pos, box, model="wca", epsilon=eps, skin=0.4)
    F, E, W = _forces(pd, eng, pos)
    p3, b3 = _embed(pos, box, rc + 0.4)
    ref = ora.pairs_direct(p3, b3, kind=2, sigma=1.0, eps=eps, rc_lj=rc)
    Wref = ref["W"].sum(0)
    if dim == 2:
        Wref = Wref[[0, 1, 3]]
    _check_forces(F, E, W, dict(F=ref["F"][:, :dim], E=ref["E"], W=Wref))
    eng.close()


def test_lanes_agree(pd, cuda):
    # the cooperative traversal's lane count changes only the summation order
    pos, box = _lj_fluid(pd, 6)
    out = []
    for lanes in (1, 2, 4, 8):
        eng = _engine(pd, pos, box, model="lj", cutoff=2.5, skin=0.3, lanes=lanes)
        out.append(_forces(pd, eng, pos)[0])
        eng.close()
    for F in out[1:]:
        assert np.max(np.abs(F - out[0])) < 1e-4 * np.max(np.abs(out[0]))


def test_two_atom_known_answers(pd, cuda, kats):
    # test/test_force_precision_gpu.jl:7-20 through the ELL route
    for case in kats["two_atom_lj"]:
        pos = np.array([[0.0, 0.0, 0.0], [case["separation"], 0.0, 0.0]])
        eng = _engine(pd, pos, (10.0, 10.0, 10.0), model="lj", cutoff=2.5, skin=0.3, capacity=4)
        F, E, W = _forces(pd, eng, pos)
        assert np.allclose(F[:, 0], case["F_x"], rtol=1e-6, atol=0)
        assert np.all(F[:, 1:] == 0)
        assert np.allclose(E, case["energy"], rtol=1e-6, atol=1e-7)
        assert np.allclose(W.sum(0), case["virial_sum"], rtol=1e-6, atol=1e-6)
        eng.close()


def test_face_crossing_precision(pd, ora, cuda, kats):
    # test/test_force_precision_gpu.jl:22-75 on the ELL route: compensated periodic differences
    face = kats["face"]
    L = float(np.float32(face["L"]))
    R = np.asarray(face["positions"], np.float64).T.astype(np.float32).astype(np.float64)
    eng = _engine(pd, R, (L, L, L), model="lj", cutoff=2.5, skin=0.4, capacity=16)
    F, E, W = _forces(pd, eng, R)
    ref = ora.pairs_direct(R, (L, L, L), kind=1, sigma=1.0, eps=1.0, rc_lj=2.5)
    _check_forces(F, E, W, dict(F=ref["F"], E=ref["E"], W=ref["W"].sum(0)), tol=face["tol_f32"])
    eng.close()


def test_capacity_error_and_resize(pd, ora, cuda):
    # capacity latch (_device_commit_kernel!, DeviceNeighborCUDA.jl:345-404) and resize_capacity! +
    # rearm (:606-620): rows longer than cap latch error 1 with the required length, no forces are
    # written; after a resize the rebuild succeeds and forces match the oracle
    pos, box = _lj_fluid(pd, 6)
    eng = _engine(pd, pos, box, model="lj", cutoff=2.5, skin=0.3, capacity=8)
    _forces(pd, eng, pos)
    st = eng.status()
    assert st["error"] == 1 and not st["valid"] and st["required"] > 8
    eng.resize(int(st["required"]))
    F, E, W = _forces(pd, eng, pos)
    st = eng.status()
    assert st["error"] == 0 and st["valid"] and st["cap"] == st["required"]
    ref = ora.pairs_cells(pos, box, kind=1, sigma=1.0, eps=1.0, rc_lj=2.5)
    assert np.linalg.norm(F - ref["F"]) / np.linalg.norm(ref["F"]) < 2e-5
    eng.close()


def test_rebuild_decision_and_adaptive_interval(pd, cuda):
    # _device_decide_kernel! (DeviceNeighborCUDA.jl:198-238): rebuild when a particle moved more than
    # skin/2 (interval x0.9, at least 5) or the list aged past the interval; non-finite or uncentred
    # coordinates latch error 2
    import torch
    pos, box = _lj_fluid(pd, 6)
    eng = _engine(pd, pos, box, model="lj", cutoff=2.5, skin=0.3, interval=20)
    xs = [_dev(pos[:, d]) for d in range(3)]
    k = int(np.argmin(np.abs(pos[:, 0])))   # a particle far from the faces
    eng.update(*xs)
    st = eng.status()
    assert st["builds"] == 1 and st["interval"] == 20
    xs[0][k] += 0.1          # below skin/2: keep
    eng.update(*xs)
    assert eng.status()["builds"] == 1
    xs[0][k] += 0.1          # 0.2 > skin/2 = 0.15: rebuild, interval round(0.9 * 20) = 18
    eng.update(*xs)
    st = eng.status()
    assert st["builds"] == 2 and st["interval"] == 18
    xs[1][7] = float("nan")
    eng.update(*xs)
    torch.cuda.synchronize()
    st = eng.status()
    assert st["error"] == 2 and not st["valid"]
    eng.close()


def _system(pd, dim, methods, dt, seed=0, n_side=40):
    if dim == 3:
        pos, box = _lj_fluid(pd, 8)
        m = np.ones(len(pos))
        v = pd.synthetic.maxwell_boltzmann(m, 0.72, seed=1)
        force = pd.LennardJones(epsilon=1.0, sigma=1.0, cutoff=2.5, pairs="neighborlist",
                                neighborlist=pd.CellList(buffer=0.3))
    else:
        pos, box = _disks(pd, n_side)
        m = np.ones(len(pos))
        v = pd.synthetic.maxwell_boltzmann(m, 1.0, seed=1, dim=2)
        force = pd.WCA(epsilon=10.0, sigma=1.0, pairs="neighborlist", neighborlist=pd.CellList(buffer=0.4,
                                                                                                  capacity=32))
    system = pd.ParticleSystem(pos, box, masses=m, velocities=v)
    return pd.Simulation(system, pd.Integrator(dt=dt, forces=[force], methods=methods), seed=seed)


def test_nve_lj_fluid(pd, ora, cuda):
    # C0: fcc 10^3 x 4 at rho 0.8442, T = 0.72, rc 2.5, skin 0.3, velocity Verlet dt = 0.005
    sim = _system(pd, 3, [pd.ConstantVolume()], 0.005)
    st = sim.state
    assert st.ell is not None
    pd.evaluate_forces_into_f(sim, energy=True)
    ref = ora.pairs_cells(st.positions(), st.box, kind=1, sigma=1.0, eps=1.0, rc_lj=2.5)
    F = st.forces()
    assert np.linalg.norm(F - ref["F"]) / np.linalg.norm(ref["F"]) < 2e-5
    E0 = st.potential_energy() + st.kinetic_energy()
    pd.run(sim, pd.Stage(steps=400))
    E1 = st.potential_energy() + st.kinetic_energy()
    s = st._ell_check()
    assert s["builds"] >= 2 and s["step"] == 400
    assert abs(E1 - E0) / abs(E0) < 2e-3
    # forces after 400 steps of device list maintenance still match the oracle
    pd.evaluate_forces_into_f(sim)
    ref = ora.pairs_cells(st.positions(), st.box, kind=1, sigma=1.0, eps=1.0, rc_lj=2.5)
    assert np.linalg.norm(st.forces() - ref["F"]) / np.linalg.norm(ref["F"]) < 2e-5


def test_graph_equals_eager(pd, cuda):
    a = _system(pd, 3, [pd.ConstantVolume()], 0.005)
    b = _system(pd, 3, [pd.ConstantVolume()], 0.005)
    a.state.step(60, use_graph=True)
    b.state.step(60, use_graph=False)
    assert np.max(np.abs(a.state.positions() - b.state.positions())) < 1e-5
    assert a.state._ell_check()["builds"] == b.state._ell_check()["builds"]


def test_langevin_step_matches_oracle(pd, ora, cuda):
    # _baoa_kernel! (Langevin.jl:58-88): B1 A1 O A2 in FP64 with Philox noise keyed on (particle, step)
    sim = _system(pd, 2, [pd.Langevin(gamma=50.0, kT=1.0)], 2e-4, seed=12345)
    st = sim.state
    pd.evaluate_forces_into_f(sim)
    p0, v0, f0 = st.positions(), st.velocities(), st.forces()
    st.step(1, use_graph=False)
    p1, v1, f1 = st.positions(), st.velocities(), st.forces()
    pr, vr = ora.baoab_drift(p0, v0, f0, 1.0, st.box, dt=2e-4, gamma=50.0, kT=1.0, seed=12345, step=0)
    assert np.max(np.abs(p1 - pr)) < 1e-5
    vfull = vr + 0.5 * 2e-4 * f1    # B2 with the new forces
    assert np.max(np.abs(v1 - vfull)) < 1e-4 * max(1.0, np.max(np.abs(vfull)))


def test_langevin_temperature(pd, cuda):
    # C1b physics at small N: 2D WCA disks at packing 0.7, eps 10, gamma 50, kT 1, dt 2e-4; the
    # kinetic temperature settles at kT
    sim = _system(pd, 2, [pd.Langevin(gamma=50.0, kT=1.0)], 2e-4, seed=7, n_side=32)
    st = sim.state
    pd.evaluate_forces_into_f(sim)
    st.step(3000)   # the lattice start releases potential energy; gamma removes it within ~0.5 time units
    temps = []
    for _ in range(20):
        st.step(100)
        temps.append(st.kinetic_energy() / st.n)   # per particle: kT (2 dof x kT/2)
    st._ell_check()
    assert abs(np.mean(temps) - 1.0) < 0.05


def test_philox_normals(pd, ora, cuda):
    # the device noise equals the oracle's Philox4x32-10 + Box-Muller draws (via one BAOAB step of a
    # force-free particle set with zero velocities: v' = r * noise * xi)
    import torch
    n = 64
    pos = np.zeros((n, 2))
    pos[:, 0] = np.linspace(-20, 20, n)
    box = (50.0, 50.0)
    system = pd.ParticleSystem(pos, box, masses=np.ones(n), velocities=np.zeros((n, 2)))
    force = pd.WCA(epsilon=1.0, sigma=0.1, pairs="neighborlist", neighborlist=pd.CellList(buffer=0.1, capacity=4))
    sim = pd.Simulation(system, pd.Integrator(dt=1e-3, forces=[force], methods=[pd.Langevin(gamma=2.0, kT=0.5)]),
                        seed=99)
    st = sim.state
    pd.evaluate_forces_into_f(sim)
    st.step(1, use_graph=False)
    v = st.velocities()
    c = np.exp(-2.0 * 1e-3)
    r = np.sqrt((1 - c * c) / (2 * 2.0 * 1e-3))
    noise = np.float32(np.sqrt(2 * 2.0 * 0.5 * np.float32(1e-3)))
    xi = np.array([ora.philox_normals4(99, 0, i + 1)[0][:2] for i in range(n)])
    assert np.max(np.abs(v - r * noise * xi)) < 1e-5
    torch.cuda.synchronize()


def _gjf(pd, seed, n_side=40):
    """The 2D WCA disks of _system under Langevin with the velocity-Verlet scheme (GJF)."""
    base = _system(pd, 2, [pd.Langevin(gamma=50.0, kT=1.0)], 2e-4, seed=seed, n_side=n_side)
    return pd.Simulation(base.system, pd.Integrator(dt=2e-4, forces=base.integrator.forces,
                                                    methods=[pd.Langevin(gamma=50.0, kT=1.0)],
                                                    scheme=pd.VelocityVerlet), seed=seed)


def test_gjf_step_matches_oracle(pd, ora, cuda):
    # _gjf_pos_kernel! / _gjf_vel_kernel! (Langevin.jl:164-208): Langevin under the velocity-Verlet scheme
    sim = _gjf(pd, 321)
    st = sim.state
    assert st.langevin_scheme == "gjf"
    pd.evaluate_forces_into_f(sim)
    p0, v0, f0 = st.positions(), st.velocities(), st.forces()
    st.step(1, use_graph=False)
    p1, v1, f1 = st.positions(), st.velocities(), st.forces()
    pr, beta = ora.gjf_step_parts(p0, v0, f0, 1.0, st.box, dt=2e-4, gamma=50.0, kT=1.0, seed=321, step=0)
    assert np.max(np.abs(p1 - pr)) < 1e-5
    vr = ora.gjf_velocity(v0, f0, f1, 1.0, beta, dt=2e-4, gamma=50.0)
    assert np.max(np.abs(v1 - vr)) < 1e-5 * max(1.0, np.max(np.abs(vr)))
    assert st._ell_check()["step"] == 1


def test_gjf_temperature_and_graph(pd, cuda):
    make = lambda seed: _gjf(pd, seed, n_side=32)   # noqa: E731
    a, b = make(7), make(7)
    for s in (a, b):
        pd.evaluate_forces_into_f(s)
    a.state.step(40, use_graph=True)
    b.state.step(40, use_graph=False)
    assert np.max(np.abs(a.state.positions() - b.state.positions())) < 1e-5
    st = a.state
    st.step(3000)
    temps = []
    for _ in range(20):
        st.step(100)
        temps.append(st.kinetic_energy() / st.n)
    st._ell_check()
    assert abs(np.mean(temps) - 1.0) < 0.05


def test_baoa_step_matches_oracle(pd, ora, cuda):
    # BAOA (_baoa_kernel! with kick = 2 dt, no trailing B): equal to the BAOAB drift started from
    # v + dt/2 f/m, without the closing half kick
    base = _system(pd, 2, [pd.Langevin(gamma=50.0, kT=1.0)], 2e-4, seed=77)
    sim = pd.Simulation(base.system, pd.Integrator(dt=2e-4, forces=base.integrator.forces,
                                                   methods=[pd.Langevin(gamma=50.0, kT=1.0)], scheme=pd.BAOA),
                        seed=77)
    st = sim.state
    assert st.langevin_scheme == "baoa"
    pd.evaluate_forces_into_f(sim)
    p0, v0, f0 = st.positions(), st.velocities(), st.forces()
    st.step(1, use_graph=False)
    p1, v1 = st.positions(), st.velocities()
    vh = (v0 + np.float32(0.5 * 2e-4) * f0).astype(np.float32)
    pr, vr = ora.baoab_drift(p0, vh, f0, 1.0, st.box, dt=2e-4, gamma=50.0, kT=1.0, seed=77, step=0)
    assert np.max(np.abs(p1 - pr)) < 1e-5
    assert np.max(np.abs(v1 - vr)) < 1e-4 * max(1.0, np.max(np.abs(vr)))


def test_langevin_bookkeeping(pd, ora, cuda):
    # dq, dU, Ekin of one BAOAB step (_baoa_kernel! and _b2_kernel!, Langevin.jl:58-78, 141-160)
    import torch
    sim = _system(pd, 2, [pd.Langevin(gamma=50.0, kT=1.0)], 2e-4, seed=5)
    st = sim.state
    pd.evaluate_forces_into_f(sim)
    n = st.n
    dq, dU, ek = (torch.zeros(n, device="cuda") for _ in range(3))
    st.engine.bookkeeping(dq, dU, ek)
    p0, v0, f0 = st.positions(), st.velocities().astype(np.float64), st.forces().astype(np.float64)
    st.step(1, use_graph=False)
    v1f, f1 = st.velocities().astype(np.float64), st.forces().astype(np.float64)
    dt, g, kT = 2e-4, 50.0, 1.0
    noise = np.float32(np.sqrt(2.0 * g * kT * float(np.float32(dt))))
    xi = np.stack([ora.philox_normals4(5, 0, i + 1, 0)[0][:2] for i in range(n)])
    beta = (noise * xi.astype(np.float32)).astype(np.float64)
    dt64 = float(np.float32(dt))
    vb1 = v0 + 0.5 * dt64 * f0
    c = np.exp(-g * dt64)
    rr = np.sqrt((1.0 - c * c) / (2.0 * g * dt64))
    v2 = c * vb1 + rr * beta
    vbar = 0.5 * (vb1 + v2)
    dq_ref = -g * (vbar * vbar).sum(1) + (vbar * beta).sum(1) / dt64
    dU_ref = (vb1 * f0).sum(1) + (v1f * f1).sum(1)
    ek_ref = 0.5 * (v1f * v1f).sum(1)
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)   # noqa: E731
    assert rel(dq.double().cpu().numpy(), dq_ref) < 1e-4
    assert rel(dU.double().cpu().numpy(), dU_ref) < 1e-4
    assert rel(ek.double().cpu().numpy(), ek_ref) < 1e-5
    # GJF: the kinetic energy after the velocity update
    sim2 = _gjf(pd, 9)
    st2 = sim2.state
    pd.evaluate_forces_into_f(sim2)
    q2, u2, k2 = (torch.zeros(st2.n, device="cuda") for _ in range(3))
    st2.engine.bookkeeping(q2, u2, k2)
    st2.step(3, use_graph=False)
    v = st2.velocities().astype(np.float64)
    assert rel(k2.double().cpu().numpy(), 0.5 * (v * v).sum(1)) < 1e-5
    assert np.all(np.isfinite(q2.cpu().numpy())) and np.abs(u2.cpu().numpy()).sum() > 0

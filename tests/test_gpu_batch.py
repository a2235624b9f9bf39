"""Batched replicas on the GPU: rows of each replica against the neighbour-row oracle, batch forces
and energies against the single-system ELL engine replica by replica, the captured step against
the eager one, energy conservation, and the lanes autotuner."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems(pd, nrep=6, seed=11, n_hi=3000):
    specs = pd.synthetic.replica_set(nrep, n_lo=500, n_hi=n_hi, seed=seed)
    return pd.batch.make_systems(specs)


def test_batch_rows_match_oracle(pd, ora, cuda):
    systems = _systems(pd, nrep=4, n_hi=1500)
    b = pd.batch.BatchedReplicas(systems, skin=0.3, cap=128)
    b.evaluate()
    st = b.status()
    assert st["valid"] and st["error"] == 0 and st["builds"] == 1
    import ctypes as C
    rows_p, counts_p, order_p = C.c_void_p(), C.c_void_p(), C.c_void_p()
    pd._native.call("pd_batch_rows", b.handle, C.byref(rows_p), C.byref(counts_p), C.byref(order_p))
    import torch
    n = b.n
    rows = torch.empty(128 * n, dtype=torch.int32, device="cuda")
    counts = torch.empty(n, dtype=torch.int32, device="cuda")
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    pd.engine._memcpy_d2d(rows.data_ptr(), rows_p.value, 4 * 128 * n)
    pd.engine._memcpy_d2d(counts.data_ptr(), counts_p.value, 4 * n)
    pd.engine._memcpy_d2d(order.data_ptr(), order_p.value, 4 * n)
    # rows by cell-order position -> rows by particle index
    order = order.cpu().numpy()
    pos_of = np.empty(n, np.int64)
    pos_of[order] = np.arange(n)
    rows_k = rows.view(128, n).t().cpu().numpy()
    counts_k = counts.cpu().numpy()
    rows = order[rows_k[pos_of]]
    counts = counts_k[pos_of]
    rl = 2.5 + 0.3
    for k, s in enumerate(systems):
        a = int(b.first[k])
        pos = np.stack([b.replica(k, t).double().cpu().numpy() for t in (b.x, b.y, b.z)], 1)
        inner = ora.neighbor_rows(pos, s["box"], rl * (1 - 1e-5))
        outer = ora.neighbor_rows(pos, s["box"], rl * (1 + 1e-5))
        for i in range(s["n"]):
            c = counts[a + i]
            got = set((rows[a + i, :c] - a).tolist())
            assert len(got) == c
            assert set(inner[i]) <= got <= set(outer[i]), (k, i)


def test_batch_forces_match_single_systems(pd, cuda):
    import torch
    systems = _systems(pd)
    b = pd.batch.BatchedReplicas(systems, skin=0.3, cap=128, lanes=4)
    b.evaluate(energy=True)
    for k, s in enumerate(systems):
        pos = np.stack([b.replica(k, t).cpu().numpy() for t in (b.x, b.y, b.z)], 1)
        kw = dict(model="lj", cutoff=2.5) if s["kind"] == "lj" else dict(model="wca")
        eng = pd.ELLEngine(s["n"], s["box"], skin=0.3, capacity=128, lanes=4, **kw)
        xs = [torch.tensor(pos[:, d], device="cuda") for d in range(3)]
        fs = [torch.zeros(s["n"], device="cuda") for _ in range(3)]
        e = torch.zeros(s["n"], device="cuda")
        w = torch.zeros((s["n"], 6), device="cuda")
        eng.update(*xs)
        eng.forces(*xs, *fs, e, w, energy=True)
        torch.cuda.synchronize()
        Fr = torch.stack(fs, 1).double().cpu().numpy()
        F = torch.stack([b.replica(k, t) for t in (b.fx, b.fy, b.fz)], 1).double().cpu().numpy()
        rel = np.sqrt(((F - Fr) ** 2).sum() / (Fr ** 2).sum())
        assert rel < 1e-5, (k, s["kind"], rel)
        E, Er = float(b.replica(k, b.epot).double().sum()), float(e.double().sum())
        assert abs(E - Er) <= 1e-5 * abs(Er), (k, E, Er)
        eng.close()


def test_batch_graph_matches_eager_and_conserves_energy(pd, cuda):
    systems = _systems(pd, nrep=5, seed=3)
    dt = 0.005
    g = pd.batch.BatchedReplicas(systems, skin=0.3, cap=128)
    e = pd.batch.BatchedReplicas(systems, skin=0.3, cap=128)
    g.evaluate(energy=True)
    e.evaluate()

    def total(b):
        b.evaluate(energy=True)
        m = 1.0 / b.inv_mass.double()
        ke = 0.5 * (m * (b.vx.double() ** 2 + b.vy.double() ** 2 + b.vz.double() ** 2)).sum()
        return float(ke + b.epot.double().sum()), float(ke + b.epot.double().abs().sum())

    E0, scale = total(g)
    g.step(60, dt, use_graph=True)
    e.step(60, dt, use_graph=False)
    g.synchronize()
    e.synchronize()
    for a, c in ((g.x, e.x), (g.y, e.y), (g.z, e.z)):
        assert float((a - c).abs().max()) < 1e-4
    st = g.status()
    assert st["error"] == 0 and st["builds"] >= 1 and st["step"] == 60
    E1, _ = total(g)
    assert abs(E1 - E0) <= 1e-3 * scale, (E0, E1, scale)


def test_batch_autotuner_picks_a_candidate(pd, cuda):
    systems = _systems(pd, nrep=8, seed=7)
    b = pd.batch.BatchedReplicas(systems, skin=0.3, cap=128)
    b.evaluate()
    res = b.autotune_lanes()
    assert res["lanes"] in (1, 2, 4, 8) and set(res["ms"]) == {1, 2, 4, 8}
    assert b.lanes == res["lanes"]


def test_batch_sparse_and_small_replicas(pd, ora, cuda):
    # a dilute replica (a few particles per cell) and the smallest box the list radius allows (three
    # cells per dimension, the stencil spans the whole box) next to a dense one
    import torch
    rng = np.random.default_rng(3)
    systems = []
    for n, L, kind in ((40, 12.0, "lj"), (60, 5.7, "wca"), (700, 9.5, "lj")):
        pos = rng.uniform(-L / 2, L / 2, (n, 3))
        if n == 700:
            pos, box = pd.synthetic.fcc_fill(n, 0.8, seed=4)
            L = box[0]
        systems.append(dict(n=n, box=(L, L, L), kind=kind, positions=pos, velocities=np.zeros((n, 3)), masses=1.0))
    b = pd.batch.BatchedReplicas(systems, skin=0.3, cap=160)
    b.evaluate(energy=True)
    st = b.status()
    assert st["error"] == 0 and st["valid"] == 1
    for k, s in enumerate(systems):
        pos = np.stack([b.replica(k, t).cpu().numpy() for t in (b.x, b.y, b.z)], 1).astype(np.float64)
        kw = dict(kind=1, sigma=1.0, eps=1.0, rc_lj=2.5) if s["kind"] == "lj" else \
            dict(kind=2, sigma=1.0, eps=1.0, rc_lj=float(np.sqrt(np.float32(1.2599211))))
        ref = ora.pairs_direct(pos, s["box"], **kw)
        F = torch.stack([b.replica(k, t) for t in (b.fx, b.fy, b.fz)], 1).double().cpu().numpy()
        scale = max(np.linalg.norm(ref["F"]), 1e-12)
        assert np.linalg.norm(F - ref["F"]) <= 2e-5 * scale + 1e-6, (k, s["kind"])

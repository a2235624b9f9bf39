"""Cluster-route rebuild / prune decision against the reference's rule (GPU, through the C ABI).

The rule (_displacement_kernel! + _decide_kernel!, src/clusterpairs/List.jl:799-825 and
src/clusterpairs/Engine.jl:301-324), restated in the oracle as ``list_decision``: with displacement
triggers the list is rebuilt when a particle has moved more than skin/2 (minimum image) since the
build, or on request, and pruned after a rebuild or when a particle has moved more than
prune_buffer/2 since the last prune; with fixed intervals (nstlist, nstprune) decision k rebuilds at
k % nstlist == 0, on request or on non-finite motion, and prunes after a rebuild or at
k % nstprune == 0.  Displacements sit well clear of the thresholds, so FP32 and FP64 agree.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SKIN, PRUNE = 1.0, 0.4


def _fluid(pd):
    pos, box = pd.synthetic.fcc_lattice(6, 0.8442, 0.05)
    L = np.asarray(box)
    pos = pos - L * np.floor(pos / L + 0.5)
    return pos.astype(np.float32).astype(np.float64), box


def _engine(pd, n, box, **kw):
    table = pd.splits.lj_type_table(1.0, 1.0, 2.5)
    return pd.ClusterPairEngine(n, box, rmax=2.5, skin=SKIN, prune_buffer=PRUNE, lj=dict(table=table), **kw)


class _Arrays:
    def __init__(self, n):
        import torch
        f32 = dict(dtype=torch.float32, device="cuda")
        self.xyz = [torch.zeros(n, **f32) for _ in range(3)]
        self.f = [torch.zeros(n, **f32) for _ in range(3)]
        self.typ = torch.ones(n, dtype=torch.int32, device="cuda")

    def load(self, pos):
        import torch
        for d in range(3):
            self.xyz[d].copy_(torch.tensor(pos[:, d], dtype=torch.float32))
        torch.cuda.synchronize()


def test_displacement_triggers(pd, ora, cuda):
    import torch
    pos0, box = _fluid(pd)
    L = np.asarray(box)
    n = len(pos0)
    eng = _engine(pd, n, box)
    a = _Arrays(n)
    a.load(pos0)
    eng.compute(*a.xyz, None, a.typ, *a.f)
    st = eng.statistics()
    assert st["last_build"] == 1 and st["builds"] == 1   # the setup request
    ref_b, ref_p = pos0.copy(), pos0.copy()
    k = int(np.argmin((pos0 ** 2).sum(1)))    # near the centre
    f = int(np.argmax(pos0[:, 0]))            # next to the +x face
    # (particle, x offset from its start): below both thresholds, past prune/2, unchanged, past prune/2
    # again since the prune, past skin/2; then across the periodic face (minimum image) and past prune/2
    moves = [(k, 0.0), (k, 0.15), (k, 0.25), (k, 0.25), (k, 0.48), (k, 0.55), (f, 0.1), (f, 0.35)]
    want_seq = [(False, False), (False, False), (False, True), (False, False), (False, True), (True, True),
                (False, False), (False, True)]
    pos = pos0.copy()
    for (i, dx), want in zip(moves, want_seq):
        pos[i, 0] = pos0[i, 0] + dx
        pos[i, 0] -= L[0] * np.floor(pos[i, 0] / L[0] + 0.5)   # stay in the centred image
        pos = pos.astype(np.float32).astype(np.float64)
        a.load(pos)
        rb, ra = ora.displacement_ratios(pos, ref_b, ref_p, box, SKIN, PRUNE)
        exp = ora.list_decision(rb, ra)
        assert exp == want, (i, dx, rb, ra)
        before = eng.statistics()
        eng.compute(*a.xyz, None, a.typ, *a.f)
        st = eng.statistics()
        got = (bool(st["last_build"]), bool(st["last_prune"]))
        assert got == exp, (i, dx, rb, ra, got)
        assert st["builds"] - before["builds"] == int(exp[0]) and st["prunes"] - before["prunes"] == int(exp[1])
        if exp[0]:
            ref_b = pos.copy()
        if exp[1]:
            ref_p = pos.copy()
    # a request rebuilds without motion; non-finite motion rebuilds
    pd._native.call("pd_cluster_request_build", eng.handle, torch.cuda.current_stream().cuda_stream)
    eng.decide(*a.xyz)
    st = eng.statistics()
    assert (st["last_build"], st["last_prune"]) == (1, 1)
    eng.compute(*a.xyz, None, a.typ, *a.f)
    bad = pos.copy()
    bad[3, 1] = np.nan
    a.load(bad)
    eng.decide(*a.xyz)
    st = eng.statistics()
    assert ora.list_decision(float("inf"), float("inf")) == (True, True)
    assert (st["last_build"], st["last_prune"]) == (1, 1)
    eng.close()


def test_fixed_intervals(pd, ora, cuda):
    import torch
    pos, box = _fluid(pd)
    n = len(pos)
    nstlist, nstprune = 4, 2
    eng = _engine(pd, n, box, list_intervals=(nstlist, nstprune))
    a = _Arrays(n)
    a.load(pos)
    eng.compute(*a.xyz, None, a.typ, *a.f)   # a trigger decision: consumes the setup request, k stays 0
    rng = np.random.default_rng(4)
    for k in range(11):
        # motion does not matter with fixed intervals (here up to skin, far past both thresholds)
        moved = pos + rng.uniform(-0.5, 0.5, size=pos.shape) * (k % 3 == 1)
        a.load(moved.astype(np.float32).astype(np.float64))
        request = k == 5
        if request:
            pd._native.call("pd_cluster_request_build", eng.handle, torch.cuda.current_stream().cuda_stream)
        eng.decide(*a.xyz, fixed=True)
        st = eng.statistics()
        exp = ora.list_decision(0.0, 0.0, request=request, nstlist=nstlist, nstprune=nstprune, k=k)
        assert (bool(st["last_build"]), bool(st["last_prune"])) == exp, (k, st)
    eng.close()


def test_fixed_intervals_in_the_captured_step(pd, cuda):
    # the step engine takes the same decision inside its graph: over 20 steps with (nstlist, nstprune) =
    # (5, 1) it builds at steps 0, 5, 10, 15 and prunes every step
    import torch
    pos, box = _fluid(pd)
    n = len(pos)
    eng = _engine(pd, n, box, list_intervals=(5, 1))
    m = np.ones(n)
    v = pd.synthetic.maxwell_boltzmann(m, 0.72, seed=3)
    f32 = dict(dtype=torch.float32, device="cuda")
    state = {k: torch.tensor(pos[:, d], **f32) for d, k in enumerate("xyz")}
    state.update({k: torch.tensor(v[:, d], **f32) for d, k in enumerate(("vx", "vy", "vz"))})
    state.update({k: torch.zeros(n, **f32) for k in ("fx", "fy", "fz", "epot")})
    state.update(vir6=torch.zeros((n, 6), **f32), vglobal=torch.zeros(6, **f32), inv_mass=1.0,
                 type=torch.ones(n, dtype=torch.int32, device="cuda"))
    md = pd.DeviceEngine(eng, None, state, box)
    s = torch.cuda.Stream()   # captured steps replay on a non-default stream
    torch.cuda.synchronize()
    md.evaluate(stream=s)
    s0 = eng.statistics(stream=s)
    md.step(20, 0.005, use_graph=True, stream=s)
    s1 = eng.statistics(stream=s)
    assert s1["error"] == 0
    assert s1["builds"] - s0["builds"] == 4 and s1["prunes"] - s0["prunes"] == 20, (s0, s1)
    md.close()
    eng.close()

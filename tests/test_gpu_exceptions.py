"""Coulomb exceptions (exclusions, scaled pairs) and LJ bond exclusions on the cluster route against the
FP64 oracle (GPU, through the C ABI and the workflow API).

The reference's semantics: the excluded branch of pair_force (src/clusterpairs/PairFunctor.jl:127-156),
_scaled_pairs_kernel!, _lj_restore_kernel!, _coulomb_shift_kernel! (src/clusterpairs/Kernels.jl:244-339)
and bond_exclusion_rows (src/clusterpairs/Engine.jl:274-290): an exception pair's Coulomb term becomes
scale * C qi qj / r wherever the pair lies (same cluster, inside the cutoff, in the list beyond it, or
beyond the list), which changes the forces by exactly oracle.exception_terms."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

C_EV = 14.399645


def _dev(a, dtype=None):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype or torch.float32, device="cuda")


def _compute(eng, pos, q, energy=True):
    import torch
    n = len(pos)
    x, y, z = (_dev(pos[:, d]) for d in range(3))
    fx, fy, fz, e = (torch.zeros(n, device="cuda") for _ in range(4))
    w = torch.zeros((n, 6), device="cuda")
    typ = torch.ones(n, dtype=torch.int32, device="cuda")
    eng.compute(x, y, z, _dev(q), typ, fx, fy, fz, e, w, energy=energy)
    torch.cuda.synchronize()
    F = torch.stack([fx, fy, fz], 1).double().cpu().numpy()
    return F, e.double().cpu().numpy(), w.double().cpu().numpy()


def _pick_pairs(pos, box, rc, rlist, seed, scales=(0.0, 0.5, 0.8333333)):
    """Exception pairs of every kind: nearest neighbours (often in one cluster), pairs between r_c and the
    list radius, and pairs well beyond the list; 0-based (i, j, scale)."""
    rng = np.random.default_rng(seed)
    L = np.asarray(box, float)
    n = len(pos)
    out = {}
    kinds = {"near": 0, "band": 0, "far": 0}
    for i in rng.choice(n, 240, replace=False):
        d = pos - pos[i]
        d -= L * np.round(d / L)
        r = np.sqrt((d * d).sum(1))
        r[i] = np.inf
        which = ("near", "band", "far")[len(out) % 3]
        if which == "near":
            j = int(np.argmin(r))
        elif which == "band":
            c = np.flatnonzero((r > rc + 0.05) & (r < rlist - 0.05))
            if len(c) == 0:
                continue
            j = int(rng.choice(c))
        else:
            c = np.flatnonzero(r > rlist + 3.0)
            j = int(rng.choice(c))
        key = (min(i, j), max(i, j))
        if key in out:
            continue
        out[key] = float(scales[len(out) % len(scales)])
        kinds[which] += 1
    assert min(kinds.values()) >= 40, kinds
    return [(i, j, s) for (i, j), s in out.items()]


def _melt(pd, n=3000, Lb=39.6, seed=5):
    pos, q, box = pd.synthetic.ionic_melt(n, Lb, 2.2, seed=seed)
    return pos.astype(np.float32).astype(np.float64), q, box


def _engine(pd, n, box, rc, eshift=0.0, lj=True, skin=1.0, prune=0.3):
    alpha = pd.splits.alpha_from_tolerance(rc, 1e-5)
    cp = pd.splits.coulomb_polynomial(alpha, C_EV, rc, eshift=eshift)
    table = pd.splits.lj_type_table(2.8, 0.01, rc, shift=True)
    return pd.ClusterPairEngine(n, box, rmax=rc, skin=skin, prune_buffer=prune,
                                lj=dict(table=table) if lj else None, coulomb=cp,
                                selfc=pd.splits.self_coefficient(alpha))


def _check_delta(F1, F0, E1, E0, W1, W0, d, ftol=1e-4, etol=5e-4):
    dF = F1 - F0 - d["F"]
    assert np.max(np.abs(dF)) < ftol, np.max(np.abs(dF))
    assert np.linalg.norm(dF) < 1e-4 * np.linalg.norm(d["F"])
    if E1 is not None:
        assert np.max(np.abs(E1 - E0 - d["E"])) < etol
        assert np.max(np.abs(W1 - W0 - d["W"])) < etol


@pytest.mark.parametrize("eshift", [0.0, 0.0123])
def test_exceptions_every_pair_kind(pd, ora, cuda, eshift):
    # excluded (scale 0) and scaled pairs next to each other, between the cutoff and the list radius and
    # beyond the list: the change of forces, per-particle energies and virial rows is the oracle's
    rc = 9.0
    pos, q, box = _melt(pd)
    eng = _engine(pd, len(pos), box, rc, eshift=eshift)
    F0, E0, W0 = _compute(eng, pos, q)
    pairs = _pick_pairs(pos, box, rc, rc + 1.0, seed=11)
    eng.set_exceptions(pairs)
    F1, E1, W1 = _compute(eng, pos, q)
    d = ora.exception_terms(pos, q, box, pairs, C=C_EV, rc=rc, eshift=eshift)
    _check_delta(F1, F0, E1, E0, W1, W0, d)
    st = eng.statistics()
    assert st["error"] == 0 and st["mask_entries"] > 0
    nonzero = sum(1 for p in pairs if p[2] != 0.0)
    assert nonzero <= st["outside_pairs"] <= len(pairs)
    # force-only pass with the masks
    F2, _, _ = _compute(eng, pos, q, energy=False)
    assert np.max(np.abs(F2 - F1)) < 1e-4
    # removing the exceptions restores the plain engine
    eng.set_exceptions([])
    F3, E3, _ = _compute(eng, pos, q)
    assert np.max(np.abs(F3 - F0)) < 1e-4 and np.max(np.abs(E3 - E0)) < 5e-4
    eng.close()


def test_exceptions_survive_list_maintenance(pd, ora, cuda):
    # rebuilds re-derive the masks and the outside pairs, prunes keep the masked tiles: coordinates moved
    # by up to a few tenths of an angstrom after a build at the old ones
    rc = 9.0
    pos, q, box = _melt(pd, seed=8)
    eng = _engine(pd, len(pos), box, rc)
    pairs = _pick_pairs(pos, box, rc, rc + 1.0, seed=3)
    rng = np.random.default_rng(1)
    for it in range(4):
        p = pos + rng.normal(0, 0.05 * it, pos.shape)
        p -= np.array(box) * np.floor(p / np.array(box) + 0.5)
        p = p.astype(np.float32).astype(np.float64)
        eng.set_exceptions([])
        F0, E0, W0 = _compute(eng, p, q)
        eng.set_exceptions(pairs)
        _compute(eng, pos, q)            # build at the old coordinates, then evaluate at the moved ones
        F1, E1, W1 = _compute(eng, p, q)
        d = ora.exception_terms(p, q, box, pairs, C=C_EV, rc=rc)
        _check_delta(F1, F0, E1, E0, W1, W0, d)
    eng.close()


def test_bond_exclusions(pd, ora, cuda):
    # bonded pairs lose their LJ term; bonded pairs that are no Coulomb exception keep their whole Coulomb
    # term including the potential shift; Coulomb exceptions that are not bonded keep their LJ term
    rc, eshift = 9.0, 0.0123
    pos, q, box = _melt(pd, seed=6)
    eng = _engine(pd, len(pos), box, rc, eshift=eshift)
    F0, E0, W0 = _compute(eng, pos, q)
    pairs = _pick_pairs(pos, box, rc, rc + 1.0, seed=5)
    near = [(i, j) for i, j, s in pairs[::3]]             # nearest-neighbour pairs: bonded
    bonded = near[: len(near) // 2] + [(i, j) for i, j, s in pairs[1::3]][:10]
    exc = [p for p in pairs if (p[0], p[1]) not in set(near[len(near) // 2:])]
    eng.set_exceptions(exc, bonds=bonded)
    F1, E1, W1 = _compute(eng, pos, q)
    tab = pd.splits.lj_type_table(2.8, 0.01, rc, shift=True)[0]
    lj = dict(c6=tab[0], c12=tab[1], rc2=tab[2], esh=tab[3])
    d = ora.exception_terms(pos, q, box, exc, C=C_EV, rc=rc, eshift=eshift, bonded=bonded, lj=lj)
    _check_delta(F1, F0, E1, E0, W1, W0, d)
    eng.close()


def test_bond_exclusions_without_coulomb(pd, ora, cuda):
    # a plain LJ fluid with bonds: the masked pairs lose their LJ term and nothing else changes
    n, rc = 4000, 2.5
    pos, box = pd.synthetic.fcc_fill(n, 0.8442, seed=3)
    pos = pos.astype(np.float32).astype(np.float64)
    table = pd.splits.lj_type_table(1.0, 1.0, rc)
    eng = pd.ClusterPairEngine(n, box, rmax=rc, skin=0.3, prune_buffer=0.1, lj=dict(table=table))
    q = np.zeros(n)
    F0, E0, W0 = _compute(eng, pos, q)
    pairs = _pick_pairs(pos, box, rc, rc + 0.3, seed=2)
    bonded = [(i, j) for i, j, _ in pairs]
    eng.set_exceptions([], bonds=bonded)
    F1, E1, W1 = _compute(eng, pos, q)
    lj = dict(c6=table[0][0], c12=table[0][1], rc2=table[0][2], esh=table[0][3])
    d = ora.exception_terms(pos, q, box, [], C=0.0, rc=rc, bonded=bonded, lj=lj)
    _check_delta(F1, F0, E1, E0, W1, W0, d, ftol=2e-4)
    with pytest.raises(pd._native.NativeError, match="Coulomb term"):
        eng.set_exceptions([(0, 1, 0.0)])
    eng.close()


def test_exception_errors(pd, cuda):
    # normalize_exceptions (src/electrostatics/Spec.jl:200-227) messages
    pos, q, box = _melt(pd, n=600, Lb=24.0)
    eng = _engine(pd, len(pos), box, 9.0, lj=False, skin=0.5, prune=0.2)
    NE = pd._native.NativeError
    with pytest.raises(NE, match="out of range"):
        eng.set_exceptions([(0, 600)])
    with pytest.raises(NE, match="single particle"):
        eng.set_exceptions([(3, 3)])
    with pytest.raises(NE, match="finite and nonnegative"):
        eng.set_exceptions([(1, 2, -0.5)])
    with pytest.raises(NE, match="conflicting scales"):
        eng.set_exceptions([(1, 2, 0.5), (2, 1, 0.0)])
    with pytest.raises(NE, match="no"):
        eng.set_exceptions([], bonds=[(1, 2)])         # no LJ term to exclude
    eng.set_exceptions([(1, 2, 0.5), (2, 1, 0.5), (4, 5, 1.0)])   # duplicates agree; scale 1 is dropped
    F, _, _ = _compute(eng, pos, q)
    assert np.all(np.isfinite(F))
    eng.close()


def _melt_sim(pd, n, seed, exclusions, scaled):
    L = (n / 0.0375) ** (1 / 3)
    pos, q, box = pd.synthetic.ionic_melt(n, L, 2.2, seed=seed)
    m = pd.synthetic.melt_masses(q)
    v = pd.synthetic.maxwell_boltzmann(m, 1200.0, seed=seed + 1, kB=pd.synthetic.KB_EV)
    topo = pd.Topology(exclusions=exclusions)
    system = pd.ParticleSystem(pos, box, types=["Na", "Cl"], typeids=np.where(q > 0, 1, 2), masses=m, charges=q,
                               velocities=v, topology=topo)
    lj = pd.LennardJones(epsilon=0.01, sigma=2.8, cutoff=9.0, pairs="neighborlist",
                         neighborlist=pd.ClusterPairList(buffer=1.0, prune_buffer=0.3))
    el = pd.PME(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=9.0, real_space_tolerance=1e-5,
                mesh_spacing=1.0, order=5, scaled_pairs=tuple(scaled))
    sim = pd.Simulation(system, pd.Integrator(dt=1.0 / pd.synthetic.TIME_UNIT_FS, forces=[lj, el]))
    return sim, q, box


def test_workflow_exceptions_through_steps(pd, ora, cuda):
    # topology exclusions and scaled pairs of a PME descriptor through the step engine: the forces,
    # energy and virial after 40 graph steps (list rebuilds and prunes on the way) are the oracle's
    n = 4000
    L = (n / 0.0375) ** (1 / 3)
    pos, q, box = pd.synthetic.ionic_melt(n, L, 2.2, seed=12)
    pairs = _pick_pairs(pos, box, 9.0, 10.0, seed=4)
    excl = [(i + 1, j + 1) for i, j, s in pairs if s == 0.0]
    scaled = [(i + 1, j + 1, s) for i, j, s in pairs if s != 0.0]
    sim, q, box = _melt_sim(pd, n, 12, excl, scaled)
    st = sim.state
    assert len(st.exceptions) == len(pairs)
    st.step(40, energy_last=False, use_graph=True)
    pd.evaluate_forces_into_f(sim, energy=True)
    R = st.positions()
    ref = ora.pme_total(R, q, box, C=pd.synthetic.COULOMB_EV_A, alpha=st.solver.spec.alpha, rc=9.0,
                        K=st.solver.mesh, P=5, kind="spme", lj=dict(sigma=2.8, eps=0.01, rc=9.0))
    d = ora.exception_terms(R, q, box, pairs, C=pd.synthetic.COULOMB_EV_A, rc=9.0)
    F = st.forces()
    Fref = ref["F"] + d["F"]
    rel = np.linalg.norm(F - Fref) / np.linalg.norm(Fref)
    assert rel < 1e-5, rel
    E = st.potential_energy()
    Eref = ref["Etot"] + d["E"].sum()
    assert abs(E - Eref) / abs(Eref) < 1e-5
    W = st.virial_tensor()
    W6 = np.array([W[k] for k in ("xx", "yy", "zz", "xy", "xz", "yz")])
    assert np.max(np.abs(W6 - (ref["W"] + d["W"].sum(0)))) / abs(ref["W"][:3].sum()) < 1e-4
    s = st.cluster.statistics()
    assert s["builds"] >= 2 and s["error"] == 0 and s["mask_entries"] > 0
    assert math.isfinite(E)

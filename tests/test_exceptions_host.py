"""Host side of the exceptions (CPU): the workflow's exception list (electrostatic_exceptions,
src/workflow/Electrostatics.jl:281-306), the topology checks (src/workflow/System.jl:39-50) and the oracle's
exception terms against a direct restatement."""
import math

import numpy as np
import pytest


def test_electrostatic_exceptions_rules(pd):
    topo = pd.Topology(bonds=[(1, 2), (3, 2)], exclusions=[(5, 4), (1, 3)])
    sysm = pd.ParticleSystem(np.zeros((6, 3)), (10.0, 10.0, 10.0), topology=topo)
    el = pd.PME(coulomb_prefactor=1.0, real_cutoff=3.0, alpha=1.0)
    assert pd.electrostatic_exceptions(sysm, el) == [(1, 3, 0.0), (4, 5, 0.0)]
    el = pd.PME(coulomb_prefactor=1.0, real_cutoff=3.0, alpha=1.0, exclude_bonded=True,
                scaled_pairs=((2, 1, 0.5), (6, 1, 0.8)))
    # bonded pairs are excluded, scaled pairs override (sorted by pair)
    assert pd.electrostatic_exceptions(sysm, el) == [(1, 2, 0.5), (1, 3, 0.0), (1, 6, 0.8), (2, 3, 0.0),
                                                      (4, 5, 0.0)]
    el = pd.PME(coulomb_prefactor=1.0, real_cutoff=3.0, alpha=1.0, exclusions=None)
    assert pd.electrostatic_exceptions(sysm, el) == []
    el = pd.PME(coulomb_prefactor=1.0, real_cutoff=3.0, alpha=1.0, exclusions=[(2, 6)])
    assert pd.electrostatic_exceptions(sysm, el) == [(2, 6, 0.0)]
    with pytest.raises(ValueError, match=r"\(i, j, scale\)"):
        pd.electrostatic_exceptions(sysm, pd.PME(coulomb_prefactor=1.0, real_cutoff=3.0, alpha=1.0,
                                                 scaled_pairs=((1, 2),)))
    # descriptors with exceptions are valid solver specs
    pd.electrostatics_spec(pd.PME(coulomb_prefactor=1.0, real_cutoff=3.0, alpha=1.0, mesh_spacing=1.0,
                                  exclude_bonded=True))


def test_topology_checks(pd):
    with pytest.raises(ValueError, match="length 2"):
        pd.Topology(bonds=[(1, 2, 3)])
    with pytest.raises(ValueError, match="must be positive"):
        pd.Topology(exclusions=[(0, 2)])
    assert pd.ParticleSystem(np.zeros((2, 3)), (5.0, 5.0, 5.0)).topology.bonds == []


def test_oracle_exception_terms(ora):
    # one excluded and one scaled pair, one inside and one beyond the cutoff, by hand
    box = (20.0, 20.0, 20.0)
    R = np.array([[0.0, 0.0, 0.0], [2.0, 0.0, 0.0], [0.0, 0.0, 19.0 - 12.0], [1.0, 1.0, 1.0]])
    q = np.array([1.0, -1.0, 0.5, 2.0])
    C, rc, es = 2.0, 5.0, 0.1
    d = ora.exception_terms(R, q, box, [(0, 1, 0.0), (0, 2, 0.25)], C=C, rc=rc, eshift=es)
    # (0, 1): r = 2 inside r_c, scale 0: e = -C q0 q1 / r + C q0 q1 eshift, f = -C q0 q1 / r^3
    e01 = -C * (1 * -1) / 2.0 + C * (1 * -1) * es
    # (0, 2): minimum image r = 7 beyond r_c, scale 0.25: e = -0.75 C q0 q2 / r
    e02 = -0.75 * C * 0.5 / 7.0
    assert math.isclose(d["E"][0], 0.5 * (e01 + e02), rel_tol=1e-14)
    assert math.isclose(d["E"][1], 0.5 * e01, rel_tol=1e-14)
    f01 = -C * -1.0 / 8.0 * np.array([-2.0, 0.0, 0.0])
    f02 = -0.75 * C * 0.5 / 343.0 * np.array([0.0, 0.0, -7.0])
    assert np.allclose(d["F"][0], f01 + f02, rtol=1e-14)
    assert np.allclose(d["F"].sum(0), 0.0, atol=1e-15)
    assert np.all(d["F"][3] == 0) and d["E"][3] == 0
    # bonded LJ removal: the negative of the pair's LJ force and energy
    lj = dict(c6=1.0, c12=1.0, rc2=6.25, esh=0.0)
    d = ora.exception_terms(R, q, box, [], C=C, rc=rc, bonded=[(0, 3)], lj=lj)
    r2 = 3.0
    ir6 = 1 / r2 ** 3
    assert math.isclose(d["E"].sum(), -((ir6 - 1) * ir6), rel_tol=1e-14)

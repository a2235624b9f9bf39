"""Cluster-pair force kernel against the FP64 oracle (GPU, through the C ABI)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a, dtype=None):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype or torch.float32, device="cuda")


def _lj_engine(pd, n, box, sigma, eps, rc, skin=0.4, prune=0.05, wca=False, shift=False):
    table = pd.splits.lj_type_table(sigma, eps, rc, wca=wca, shift=shift)
    return pd.ClusterPairEngine(n, box, rmax=rc, skin=skin, prune_buffer=prune, lj=dict(table=table))


def _compute(pd, eng, pos, q=None, energy=True):
    import torch
    n = len(pos)
    x, y, z = (_dev(pos[:, d]) for d in range(3))
    fx, fy, fz, e = (torch.zeros(n, device="cuda") for _ in range(4))
    w = torch.zeros((n, 6), device="cuda")
    qq = None if q is None else _dev(q)
    typ = torch.ones(n, dtype=torch.int32, device="cuda")
    eng.compute(x, y, z, qq, typ, fx, fy, fz, e, w, energy=energy)
    torch.cuda.synchronize()
    F = torch.stack([fx, fy, fz], 1).double().cpu().numpy()
    return F, e.double().cpu().numpy(), w.double().cpu().numpy()


def test_two_atom_known_answers(pd, cuda, kats):
    # test/test_force_precision_gpu.jl:7-20 through the cluster route (FP32 is exact for these values)
    for case in kats["two_atom_lj"]:
        eng = _lj_engine(pd, 2, (10.0, 10.0, 10.0), 1.0, 1.0, 2.5)
        pos = np.array([[0.0, 0.0, 0.0], [case["separation"], 0.0, 0.0]])
        F, E, W = _compute(pd, eng, pos)
        assert np.allclose(F[:, 0], case["F_x"], rtol=1e-6, atol=0)
        assert np.all(F[:, 1:] == 0)
        assert np.allclose(E, case["energy"], rtol=1e-6, atol=1e-7)
        assert np.allclose(W.sum(0), case["virial_sum"], rtol=1e-6, atol=1e-6)
        eng.close()


@pytest.mark.parametrize("image", ["centered", "positive"])
def test_face_crossing_precision(pd, ora, cuda, kats, image):
    # test/test_force_precision_gpu.jl:22-75: ten near-face particles, phases initial / small move /
    # crossing, forces, energy and virial within 2e-5 of the FP64 direct sum
    face = kats["face"]
    L = np.float32(face["L"])
    R = np.asarray(face["positions"], np.float64).T.astype(np.float32)
    if image == "positive":
        R = R + L / np.float32(2)
    n = len(R)
    eng = _lj_engine(pd, n, (float(L),) * 3, 1.0, 1.0, 2.5, skin=0.4, prune=0.05)
    ids = np.arange(1, n + 1, dtype=np.float64)
    tol = face["tol_f32"]
    for phase in ("initial", "small_move", "crossing"):
        if phase == "small_move":
            for d in range(3):
                R[:, d] = R[:, d] + (0.017 * np.sin(ids * (0.73 + 0.11 * (d + 1)))).astype(np.float32)
        elif phase == "crossing":
            R = R + np.float32(0.33)
            R = (R - L * np.floor(R / L + np.float32(0.5))).astype(np.float32)
        F, E, W = _compute(pd, eng, R.astype(np.float64))
        ref = ora.pairs_direct(R.astype(np.float64), (float(L),) * 3, kind=1, sigma=1.0, eps=1.0, rc_lj=2.5)
        nF = np.linalg.norm(ref["F"])
        assert np.linalg.norm(F - ref["F"]) / nF < tol, phase
        assert np.linalg.norm(F.sum(0)) / nF < tol
        assert abs(E.sum() - ref["E"].sum()) / max(abs(ref["E"].sum()), 1) < tol
        assert np.linalg.norm(W.sum(0) - ref["W"].sum(0)) / max(np.linalg.norm(ref["W"].sum(0)), 1) < tol
        Fno, _, _ = _compute(pd, eng, R.astype(np.float64), energy=False)
        assert np.linalg.norm(Fno - ref["F"]) / nF < tol
    eng.close()


def test_random_lj_matches_oracle(pd, ora, cuda):
    # test/test_cluster_pairs.jl:64-86: uniform LJ, N = 2501 (not a multiple of 8), FP32 tolerance 2e-5
    rng = np.random.default_rng(11)
    L = (5.3, 5.6, 6.1)
    n = 2501
    pos = rng.random((n, 3)) * np.array(L) - np.array(L) / 2
    pos = pos.astype(np.float32).astype(np.float64)
    eng = _lj_engine(pd, n, L, 0.32, 0.8, 1.0, skin=0.1, prune=0.05)
    F, E, W = _compute(pd, eng, pos)
    ref = ora.pairs_cells(pos, L, kind=1, sigma=0.32, eps=0.8, rc_lj=1.0)
    assert np.linalg.norm(F - ref["F"]) / np.linalg.norm(ref["F"]) < 2e-5
    assert abs(E.sum() - ref["E"].sum()) / abs(ref["E"].sum()) < 2e-5
    assert np.linalg.norm(W.sum(0) - ref["W"].sum(0)) / np.linalg.norm(ref["W"].sum(0)) < 2e-5
    # Newton's third law within FP32 summation noise
    assert np.linalg.norm(F.sum(0)) < 1e-4 * np.linalg.norm(ref["F"])
    eng.close()


def test_wca_and_shifted_lj(pd, ora, cuda):
    rng = np.random.default_rng(2)
    L = (6.0, 6.0, 6.0)
    n = 900
    pos = (rng.random((n, 3)) * 6.0 - 3.0).astype(np.float32).astype(np.float64)
    rcw = 1.0 * pd.splits.WCA_RC_FACTOR
    eng = _lj_engine(pd, n, L, 0.5, 10.0, rcw, wca=True)
    F, E, _ = _compute(pd, eng, pos)
    ref = ora.pairs_cells(pos, L, kind=2, sigma=0.5, eps=10.0, rc_lj=rcw)
    assert np.linalg.norm(F - ref["F"]) / np.linalg.norm(ref["F"]) < 2e-5
    assert abs(E.sum() - ref["E"].sum()) / abs(ref["E"].sum()) < 2e-5
    eng.close()
    eng = _lj_engine(pd, n, L, 0.5, 1.0, 1.25, shift=True)
    F, E, _ = _compute(pd, eng, pos)
    sh = 4 * 1.0 * ((0.5 / 1.25) ** 12 - (0.5 / 1.25) ** 6)
    ref = ora.pairs_cells(pos, L, kind=1, sigma=0.5, eps=1.0, rc_lj=1.25, eshift_lj=sh)
    assert np.linalg.norm(F - ref["F"]) / np.linalg.norm(ref["F"]) < 2e-5
    assert abs(E.sum() - ref["E"].sum()) / abs(ref["E"].sum()) < 2e-5
    eng.close()


def test_lj_coulomb_real_space(pd, ora, cuda):
    # LJ + real-space Ewald Coulomb through the fitted polynomial against exact erfc pairs
    n, Lb = 3000, 39.6
    pos, q, box = pd.synthetic.ionic_melt(n, Lb, 2.2, seed=5)
    pos = pos.astype(np.float32).astype(np.float64)
    C, rc = pd.synthetic.COULOMB_EV_A, 9.0
    alpha = pd.splits.alpha_from_tolerance(rc, 1e-5)
    cp = pd.splits.coulomb_polynomial(alpha, C, rc)
    table = pd.splits.lj_type_table(2.8, 0.01, rc)
    eng = pd.ClusterPairEngine(n, box, rmax=rc, skin=1.0, prune_buffer=0.3, lj=dict(table=table), coulomb=cp,
                               selfc=pd.splits.self_coefficient(alpha))
    F, E, W = _compute(pd, eng, pos, q=q)
    ref = ora.pairs_cells(pos, box, q=q, kind=1, sigma=2.8, eps=0.01, rc_lj=rc, C=C, alpha=alpha, rc_coul=rc)
    rel = np.linalg.norm(F - ref["F"]) / np.linalg.norm(ref["F"])
    assert rel < 1e-5, rel
    selfE = -C * alpha / math.sqrt(math.pi) * (q * q)
    assert abs(E.sum() - (ref["E"] + selfE).sum()) / abs((ref["E"] + selfE).sum()) < 1e-5
    assert np.linalg.norm(W.sum(0) - ref["W"].sum(0)) / np.linalg.norm(ref["W"].sum(0)) < 1e-5
    eng.close()


def test_nonfinite_coordinates_are_reported(pd, cuda):
    import torch
    n = 64
    eng = _lj_engine(pd, n, (8.0, 8.0, 8.0), 1.0, 1.0, 2.5)
    pos = np.random.default_rng(0).random((n, 3)) * 8 - 4
    pos[5, 1] = np.nan
    with pytest.raises(pd._native.NativeError) as ei:
        _compute(pd, eng, pos)
    assert ei.value.code == pd._native.PD_ENONFINITE
    eng.close()


def test_rejects_small_box(pd, cuda):
    with pytest.raises(pd._native.NativeError) as ei:
        _lj_engine(pd, 10, (4.0, 4.0, 4.0), 1.0, 1.0, 2.5)
    assert ei.value.code == pd._native.PD_EINVAL


@pytest.mark.parametrize("nsplit,warps", [(1, 1), (3, 4), (7, 2), (2, 1)])
def test_pair_shapes_agree(pd, cuda, nsplit, warps):
    # every CTA shape of the pair kernel (parts per super-cluster x warps per part) gives the same forces,
    # energies and virials (up to the order of the float reductions)
    n, Lb = 3000, 39.6
    pos, q, box = pd.synthetic.ionic_melt(n, Lb, 2.2, seed=6)
    C, rc = pd.synthetic.COULOMB_EV_A, 9.0
    alpha = pd.splits.alpha_from_tolerance(rc, 1e-5)
    cp = pd.splits.coulomb_polynomial(alpha, C, rc)
    table = pd.splits.lj_type_table(2.8, 0.01, rc)

    def run(shape):
        eng = pd.ClusterPairEngine(n, box, rmax=rc, skin=1.0, prune_buffer=0.3, lj=dict(table=table), coulomb=cp,
                                   selfc=pd.splits.self_coefficient(alpha))
        if shape is not None:
            eng.set_pair_shape(*shape)
            assert eng.pair_shape() == shape
        out = _compute(pd, eng, pos, q=q)
        eng.close()
        return out

    F0, E0, W0 = run(None)
    F1, E1, W1 = run((nsplit, warps))
    assert np.linalg.norm(F1 - F0) <= 1e-6 * np.linalg.norm(F0)
    assert np.linalg.norm(E1 - E0) <= 1e-6 * np.linalg.norm(E0)
    assert np.linalg.norm(W1 - W0) <= 1e-6 * np.linalg.norm(W0)

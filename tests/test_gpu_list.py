"""Cluster-pair list built on the GPU against the oracle's Float32 restatement, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _build(pd, pos, box, rc, skin, prune, q=None):
    import torch
    n = len(pos)
    table = pd.splits.lj_type_table(1.0, 1.0, rc)
    eng = pd.ClusterPairEngine(n, box, rmax=rc, skin=skin, prune_buffer=prune, lj=dict(table=table))
    x, y, z = (torch.tensor(np.ascontiguousarray(pos[:, d]), dtype=torch.float32, device="cuda") for d in range(3))
    f = [torch.zeros(n, device="cuda") for _ in range(4)]
    typ = torch.ones(n, dtype=torch.int32, device="cuda")
    eng.compute(x, y, z, None, typ, f[0], f[1], f[2], f[3], None, energy=False)
    torch.cuda.synchronize()
    return eng


@pytest.mark.parametrize("n,box,rc,skin,prune,seed", [
    (2501, (5.3, 5.6, 6.1), 1.0, 0.1, 0.05, 11),
    (4000, (16.796, 16.796, 16.796), 2.5, 0.3, 0.15, 3),
    (777, (9.0, 7.5, 12.0), 1.2, 0.4, 0.0, 9),
])
def test_list_bit_exact(pd, ora, cuda, n, box, rc, skin, prune, seed):
    rng = np.random.default_rng(seed)
    pos = (rng.random((n, 3)) * np.array(box) - np.array(box) / 2).astype(np.float32)
    eng = _build(pd, pos.astype(np.float64), box, rc, skin, prune)
    gpu = eng.list_host()
    ref = ora.cluster_build(pos, box, rc + skin)
    assert gpu["ns"] == ref["ns"]
    assert np.array_equal(gpu["perm"][:64 * ref["ns"]], ref["perm"][:64 * ref["ns"]])
    assert np.array_equal(gpu["scio"], ref["scio"])
    assert np.array_equal(gpu["cjo"], ref["cjo"])
    # packed force coordinates equal the storage coordinates (centred image) bit for bit
    perm = gpu["perm"][:64 * ref["ns"]]
    occ = perm >= 0
    for d in range(3):
        fc = ora.force_coordinate(pos[perm[occ], d], box[d])
        assert np.array_equal(gpu["xq"][:64 * ref["ns"]][occ, d], fc)
    pad = gpu["xq"][:64 * ref["ns"]][~occ]
    assert np.all(pad[:, :3] > 1e6) and np.all(pad[:, 3] == 0)
    assert len(np.unique(pad[:, :3], axis=0)) == len(pad)
    # pruned working list from the GPU's packed coordinates
    cjw, nw = ora.cluster_prune(ref["ns"], gpu["xq"][:64 * ref["ns"]].reshape(-1), ref["scio"], ref["cjo"], box,
                                rc + prune, prune)
    assert np.array_equal(gpu["nw"], nw)
    for S in range(ref["ns"]):
        a, k = ref["scio"][S], nw[S]
        assert np.array_equal(gpu["cjw"][a:a + k], cjw[a:a + k])
    # every pair inside the cutoff lies in exactly one live tile of the working list
    pairs = ora.tile_pairs(gpu["perm"], gpu["scio"], dict(cjw=gpu["cjw"], nw=gpu["nw"]), working=True)
    assert len(pairs) == len(set(pairs))
    rows = ora.neighbor_rows(pos.astype(np.float64), box, rc * (1 - 1e-6))
    need = {(min(i, j), max(i, j)) for i, r in enumerate(rows) for j in r}
    assert need <= set(pairs)
    eng.close()


def test_far_coordinates_stay_in_range(pd, ora, cuda):
    # Finite coordinates billions of box lengths away wrap with a rounding error of up to half an
    # ulp (here 128), so the wrapped value can fall below 0 or above L; the column and z-bin
    # indices are clamped, and the list still equals the oracle's bit for bit.
    rng = np.random.default_rng(5)
    box = (12.0, 12.0, 12.0)
    n = 2000
    pos = (rng.random((n, 3)) * 12 - 6).astype(np.float32)
    far = rng.choice(n, 200, replace=False)
    pos[far] = (rng.uniform(-1, 1, (200, 3)) * 3e9).astype(np.float32)
    wrapped = pos[far] - np.float32(12.0) * np.floor(pos[far] / np.float32(12.0))
    assert (wrapped < 0).any() or (wrapped >= 12.0).any()
    eng = _build(pd, pos.astype(np.float64), box, 1.5, 0.3, 0.1)
    gpu = eng.list_host()
    ref = ora.cluster_build(pos, box, 1.8)
    assert gpu["ns"] == ref["ns"]
    perm = gpu["perm"][:64 * ref["ns"]]
    assert np.array_equal(perm, ref["perm"][:64 * ref["ns"]])
    assert np.array_equal(np.sort(perm[perm >= 0]), np.arange(n))
    assert np.array_equal(gpu["scio"], ref["scio"]) and np.array_equal(gpu["cjo"], ref["cjo"])
    eng.close()


def test_list_is_reproducible(pd, cuda):
    rng = np.random.default_rng(4)
    box = (12.0, 12.0, 12.0)
    pos = rng.random((3000, 3)) * 12 - 6
    a = _build(pd, pos, box, 1.5, 0.3, 0.1).list_host()
    b = _build(pd, pos, box, 1.5, 0.3, 0.1).list_host()
    for k in ("perm", "scio", "cjo", "nw"):
        assert np.array_equal(a[k], b[k])


def test_statistics(pd, cuda):
    rng = np.random.default_rng(4)
    box = (12.0, 12.0, 12.0)
    eng = _build(pd, rng.random((3000, 3)) * 12 - 6, box, 1.5, 0.3, 0.1)
    s = eng.statistics()
    assert s["superclusters"] > 0 and s["outer_entries"] >= s["working_entries"] > 0
    assert s["error"] == 0 and s["builds"] >= 1
    # pairs evaluated per particle: 32 x live (i-atom, j-half) bits / N, at least the pairs inside r_c
    assert s["pairs_per_particle"] > 0.5 * 3000 / 1728 * 4 / 3 * np.pi * 1.5 ** 3

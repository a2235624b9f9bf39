"""Host side of the batched charged melts (CPU): the melt generator (sizes, neutrality, centred image,
minimum separation, masses) and the per-melt meshes at the shared 1 Å spacing (resolve_mesh,
src/electrostatics/Spec.jl:141-146), and the bench's melt sizes (N log-uniform in [2 000, 32 000])."""
import numpy as np


def test_melt_systems(pd):
    ns = [600, 1002, 2400]
    systems = pd.batch.melt_systems(ns, seed=3)
    for n, s in zip(ns, systems):
        assert s["n"] == n and s["positions"].shape == (n, 3)
        L = np.asarray(s["box"])
        assert np.allclose(L, (n / 0.0375) ** (1 / 3))
        assert (s["positions"] >= -L / 2).all() and (s["positions"] < L / 2).all()
        q = s["charges"]
        assert set(np.unique(q)) == {-1.0, 1.0} and q.sum() == 0
        assert np.allclose(s["masses"], np.where(q > 0, 22.99, 35.45))
        d = s["positions"][:, None, :] - s["positions"][None, :, :]
        d -= L * np.round(d / L)
        r = np.sqrt((d ** 2).sum(-1)) + np.eye(n) * 1e9
        assert r.min() >= 2.2 - 1e-9
        assert (s["eps"], s["sigma"], s["rc"]) == (0.01, 2.8, 9.0)
    # seeded: the same call gives the same melts
    again = pd.batch.melt_systems(ns, seed=3)
    assert all(np.array_equal(a["positions"], b["positions"]) for a, b in zip(systems, again))


def test_melt_meshes_follow_the_box(pd):
    systems = pd.batch.melt_systems([2000, 32000], seed=1)
    meshes = [pd.splits.resolve_mesh(None, 1.0, s["box"], 5) for s in systems]
    for s, K in zip(systems, meshes):
        for k, L in zip(K, s["box"]):
            assert k == pd.splits.fft_friendly(int(np.ceil(L / 1.0)))
    assert meshes[0] != meshes[1]


def test_melt_sizes(pd):
    ns = pd.batch.melt_sizes(64, 2090)
    assert len(ns) == 64 and all(n % 2 == 0 for n in ns)
    assert min(ns) >= 2000 and max(ns) <= 32002
    assert ns == pd.batch.melt_sizes(64, 2090) and ns != pd.batch.melt_sizes(64, 2091)

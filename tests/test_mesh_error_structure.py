"""Structure of the coarse-mesh force error that the learned form corrects (CPU, FP64 oracle).

The mesh part is linear in the charges, so the residual R_i = F_fine,i - F_coarse,i of the ionic
melt splits exactly into source terms E_ij (the fine-minus-coarse force on i from charge j alone).
The test states three facts about E_ij on a small melt at the melt's density and Ewald splitting
(alpha = 0.34705 / A, SPME 2 A order 4 against 1 A order 5):

* the error is local: source terms within 8 A of the ion carry all but a few per cent of |R|^2;
* the self term E_ii (the mesh's spurious self force, a function of the ion's position relative to
  the nodes) carries a fifth of |R|^2 or more;
* the best radial pair model E_ij ~ q_i q_j b(r_ij) r_ij (b averaged over all pairs at each
  distance, the most a rotation-invariant pair term can reach) leaves more than half of |R|^2.

So what a local model must learn depends on where both ions sit relative to the mesh nodes, which
rotation-invariant charge descriptors cannot see.
"""
import numpy as np
import pytest

ALPHA, COUL = 0.34705, 14.399645


@pytest.fixture(scope="module")
def decomposition(pd, ora):
    L = 30.0
    n = int(0.0375 * L ** 3) // 2 * 2
    pos, q, _ = pd.synthetic.ionic_melt(n, L, seed=17)
    pos = np.asarray(pos, np.float64)
    q = np.asarray(q, np.float64)
    box = (L, L, L)
    tc = ora.influence("spme", 4, (15, 15, 15), box, COUL, ALPHA)
    tf = ora.influence("spme", 5, (30, 30, 30), box, COUL, ALPHA)
    Fc = ora.mesh(pos, q, box, (15, 15, 15), 4, alpha=ALPHA, C=COUL, tables=tc)["F"]
    Ff = ora.mesh(pos, q, box, (30, 30, 30), 5, alpha=ALPHA, C=COUL, tables=tf)["F"]
    src = np.arange(n)
    E = (ora.mesh_source_forces(pos, q, box, (30, 30, 30), 5, tf, src)
         - ora.mesh_source_forces(pos, q, box, (15, 15, 15), 4, tc, src))    # E[j, i] = force on i from j
    d = pos[:, None, :] - pos[None, :, :]
    d -= L * np.round(d / L)
    r = np.sqrt((d * d).sum(-1))
    return dict(n=n, q=q, R=Ff - Fc, E=np.transpose(E, (1, 0, 2)), d=d, r=r, Ff=Ff)


def test_source_terms_sum_to_the_residual(decomposition):
    D = decomposition
    assert np.abs(D["E"].sum(1) - D["R"]).max() <= 1e-9 * np.abs(D["R"]).max()
    rel = np.sqrt((D["R"] ** 2).sum() / (D["Ff"] ** 2).sum())
    assert 5e-3 < rel < 3e-2, rel


def test_coarse_mesh_error_is_local(decomposition):
    D = decomposition
    tot = (D["R"] ** 2).sum()
    left = {}
    for rc in (0.0, 4.0, 8.0):
        part = (D["E"] * (D["r"] <= rc)[..., None]).sum(1)
        left[rc] = ((D["R"] - part) ** 2).sum() / tot
    assert left[8.0] < 0.03, left
    assert left[4.0] < 0.5 < left[0.0], left


def test_self_term_and_radial_model_shares(decomposition):
    D = decomposition
    tot = (D["R"] ** 2).sum()
    n, E, d, r, q = D["n"], D["E"], D["d"], D["r"], D["q"]
    self_share = (E[np.arange(n), np.arange(n)] ** 2).sum() / tot
    assert 0.15 < self_share < 0.5, self_share
    qq = q[:, None] * q[None, :]
    off = (r > 0) & (r < 10.0)
    proj = (E * d).sum(-1) / np.where(r > 0, r * r, 1.0) * qq
    edges = np.linspace(0.0, 10.0, 101)
    k = np.digitize(r[off], edges)
    mean = np.zeros(len(edges) + 1)
    for b in np.unique(k):
        mean[b] = proj[off][k == b].mean()
    b_r = np.zeros_like(r)
    b_r[off] = mean[k]
    radial = ((qq * b_r)[..., None] * d).sum(1)
    left = ((D["R"] - radial) ** 2).sum() / tot
    assert left > 0.5, left

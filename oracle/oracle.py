"""CPU oracle of the force hot path -- TEST INFRASTRUCTURE ONLY.

Restates ParticleDynamics.jl's algorithms on the CPU in FP64 (the cluster list
in the reference's Float32 geometry) to check libpdb200's CUDA results, and
serves as the timed CPU baseline of ``bench.py``.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs use it; the product
never calls it.

Parity pins: the known-answer tests of the reference's own suite
(test/test_force_precision_gpu.jl:7-20 two-atom LJ values,
test/test_electrostatics.jl:54-96 B-spline partition of unity and node base,
:260-279 FFT normalisation, :321 and :409 self and background energies) are
checked against this oracle in tests/test_oracle.py; the reference itself
(Julia + CUDA.jl) cannot run here, so no further golden vectors exist.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_lib = None

_d = C.POINTER(C.c_double)
_f = C.POINTER(C.c_float)
_i = C.POINTER(C.c_int)
_u = C.POINTER(C.c_uint32)


def _load():
    global _lib
    if _lib is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location("_oracle_build", HERE / "build.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        path = mod.build()
        L = C.CDLL(str(path))
        L.ora_pairs_direct.argtypes = [C.c_int, _d, _d, _d, _d, _d, C.c_int, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_double, _i, C.c_int, _d]
        L.ora_pairs_cells.argtypes = [C.c_int, _d, _d, _d, _d, _d, C.c_int, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_double, C.c_double, _d, _d, _d, _d, _d]
        L.ora_neighbor_rows.argtypes = [C.c_int, _d, _d, _d, _d, C.c_double, C.c_int, _i, _i]
        L.ora_neighbor_rows.restype = C.c_int
        L.ora_ewald.argtypes = [C.c_int, _d, _d, _d, C.c_double, C.c_double, C.c_double, C.c_int, _d, _d, _d]
        L.ora_bspline.argtypes = [C.c_int, C.c_double, _d, _d]
        L.ora_bspline.restype = C.c_int
        L.ora_spread.argtypes = [C.c_int, _d, _d, _d, _d, _d, _i, C.c_int, _d]
        L.ora_gather_ad.argtypes = [C.c_int, _d, _d, _d, _d, _d, _i, C.c_int, _d, _d, _d]
        L.ora_gather_ik.argtypes = [C.c_int, _d, _d, _d, _d, _d, _i, C.c_int, _d, _d, _d, _d, _d, _d]
        L.ora_influence.argtypes = [C.c_int, C.c_int, C.c_int, _i, _d, C.c_double, C.c_double, _d, _d]
        L.ora_cluster_geometry.argtypes = [C.c_int, _d, C.c_double, _i]
        L.ora_cluster_geometry.restype = C.c_int
        L.ora_cluster_build.argtypes = [C.c_int, _f, _f, _f, _d, C.c_double, C.c_int, _i, _i, _u]
        L.ora_cluster_build.restype = C.c_int
        L.ora_cluster_prune.argtypes = [C.c_int, _f, _i, _u, _d, C.c_double, C.c_double, _u, _i]
        L.ora_force_coordinate.argtypes = [C.c_float, C.c_float]
        L.ora_force_coordinate.restype = C.c_float
        L.ora_philox_normals4.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, _f, _u]
        L.ora_baoab_drift.argtypes = [C.c_int, C.c_int, _f, _f, _f, _f, _f, _f, _f, _f, _f, _f, C.c_float,
                                      C.c_float, C.c_float, C.c_uint64, C.c_uint64, _d]
        _lib = L
    return _lib


def _p(a, t=_d):
    return a.ctypes.data_as(t)


def _box(box):
    return np.ascontiguousarray(box, np.float64)


def _xyz(pos):
    pos = np.asarray(pos, np.float64)
    return [np.ascontiguousarray(pos[:, d]) for d in range(3)]


# ------------------------------------------------------------------ pair sums

def pairs_direct(pos, box, *, q=None, kind=1, sigma=1.0, eps=1.0, rc_lj=2.5, eshift_lj=0.0, C=0.0, alpha=0.0,
                 rc_coul=0.0, ids=None):
    """All-pairs FP64 sums at the sampled particles (gpu_force_reference.jl:38-80, pair_reference_gpu.jl)."""
    L = _load()
    x, y, z = _xyz(pos)
    n = len(x)
    qq = None if q is None else np.ascontiguousarray(q, np.float64)
    idx = None if ids is None else np.ascontiguousarray(ids, np.int32)
    nids = n if ids is None else len(idx)
    out = np.zeros((nids, 11))
    L.ora_pairs_direct(n, _p(x), _p(y), _p(z), None if qq is None else _p(qq), _p(_box(box)), int(kind),
                       float(sigma), float(eps), float(rc_lj), float(eshift_lj), float(C), float(alpha),
                       float(rc_coul), None if idx is None else _p(idx, _i), nids, _p(out))
    return dict(F=out[:, :3], E=out[:, 3], W=out[:, 4:10], count=out[:, 10])


def pairs_cells(pos, box, *, q=None, kind=1, sigma=1.0, eps=1.0, rc_lj=2.5, eshift_lj=0.0, C=0.0, alpha=0.0,
                rc_coul=0.0):
    """Every particle's FP64 pair force, energy and virial row with a cell grid."""
    L = _load()
    x, y, z = _xyz(pos)
    n = len(x)
    qq = None if q is None else np.ascontiguousarray(q, np.float64)
    fx, fy, fz, e = (np.zeros(n) for _ in range(4))
    w = np.zeros((n, 6))
    L.ora_pairs_cells(n, _p(x), _p(y), _p(z), None if qq is None else _p(qq), _p(_box(box)), int(kind),
                      float(sigma), float(eps), float(rc_lj), float(eshift_lj), float(C), float(alpha),
                      float(rc_coul), _p(fx), _p(fy), _p(fz), _p(e), _p(w))
    return dict(F=np.stack([fx, fy, fz], 1), E=e, W=w)


def pair_term_scales(pos, box, *, kind=1, sigma=1.0, eps=1.0, rc_lj=2.5, band=1e-6):
    """(S_i, S_E, A_i): S_i = sum_j (|f_rep| + |f_att|)_ij per particle and S_E = sum over pairs of
    |u_rep| + |u_att| + |e_shift| (WCA: e_shift = -eps), the scales of the FP32 rounding error of the
    force and energy sums of LJ (kind 1) or WCA (kind 2) pairs inside r_c (see pair_force_abs_sums);
    A_i = sum of |f_ij| over the pairs within a relative ``band`` of r_c, which FP32 rounding of r^2 may
    put on either side of the cutoff (the truncated LJ force does not vanish there)."""
    S = pair_force_abs_sums(pos, box, kind=kind, sigma=sigma, eps=eps, rc_lj=rc_lj)
    from scipy.spatial import cKDTree
    L = np.asarray(box, float)
    p = np.asarray(pos, float) % L
    tree = cKDTree(p, boxsize=L)
    ij = tree.query_pairs(rc_lj * (1.0 + band), output_type="ndarray")
    d = p[ij[:, 0]] - p[ij[:, 1]]
    d -= L * np.round(d / L)
    r2 = (d * d).sum(1)
    inside = r2 < rc_lj * rc_lj
    ir6 = (sigma * sigma / r2) ** 3
    esh = eps if kind == 2 else 0.0
    SE = float((4.0 * eps * (ir6 * ir6 + ir6) + esh)[inside].sum())
    edge = np.abs(np.sqrt(r2) - rc_lj) <= band * rc_lj
    fe = np.abs(24.0 * eps * (2.0 * ir6 - 1.0) * ir6 / np.sqrt(r2)) * edge
    A = np.zeros(len(p))
    np.add.at(A, ij[:, 0], fe)
    np.add.at(A, ij[:, 1], fe)
    return S, SE, A


def pair_force_abs_sums(pos, box, *, kind=1, sigma=1.0, eps=1.0, rc_lj=2.5):
    """S_i = sum_j (|f_rep| + |f_att|)_ij over the LJ (kind 1) or WCA (kind 2) pairs inside r_c, in FP64:
    the scale of the rounding error of an FP32 sum of pair forces.  Each pair force is the difference of
    a repulsive 48 eps sigma^12 / r^13 and an attractive 24 eps sigma^6 / r^7 term, computed to a few ulps
    of their magnitudes (they cancel where the force changes sign, at the WCA cutoff), so
    |F_i(FP32) - F_i| stays within a small multiple of eps_32 S_i however much the terms cancel."""
    from scipy.spatial import cKDTree
    L = np.asarray(box, float)
    p = np.asarray(pos, float) % L
    tree = cKDTree(p, boxsize=L)
    ij = tree.query_pairs(rc_lj, output_type="ndarray")
    d = p[ij[:, 0]] - p[ij[:, 1]]
    d -= L * np.round(d / L)
    r2 = (d * d).sum(1)
    ir2 = sigma * sigma / r2
    ir6 = ir2 * ir2 * ir2
    f = 24.0 * eps * (2.0 * ir6 + 1.0) * ir6 / np.sqrt(r2)
    S = np.zeros(len(p))
    np.add.at(S, ij[:, 0], f)
    np.add.at(S, ij[:, 1], f)
    return S


def neighbor_rows(pos, box, radius, cap=512):
    """reference_neighbor_rows (test/neighbor_reference.jl:6-16): sorted rows of j within radius."""
    L = _load()
    x, y, z = _xyz(pos)
    n = len(x)
    counts = np.zeros(n, np.int32)
    rows = np.zeros(n * cap, np.int32)
    mx = L.ora_neighbor_rows(n, _p(x), _p(y), _p(z), _p(_box(box)), float(radius), cap, _p(counts, _i),
                             _p(rows, _i))
    if mx > cap:
        return neighbor_rows(pos, box, radius, cap=mx)
    return [sorted(rows[i * cap:i * cap + counts[i]].tolist()) for i in range(n)]


def ewald(pos, q, box, C=1.0, alpha=None, digits=16, background=False):
    """ewald_reference (test/ewald_reference.jl:50-127) for an orthorhombic box: (E, F (n,3), W (3,3))."""
    L = _load()
    R = np.ascontiguousarray(np.asarray(pos, np.float64).reshape(-1, 3))
    qq = np.ascontiguousarray(q, np.float64)
    n = len(qq)
    E = np.zeros(1)
    F = np.zeros(3 * n)
    W = np.zeros(9)
    L.ora_ewald(n, _p(R), _p(qq), _p(_box(box)), float(C), -1.0 if alpha is None else float(alpha), float(digits),
                int(bool(background)), _p(E), _p(F), _p(W))
    return float(E[0]), F.reshape(n, 3), W.reshape(3, 3)


# ------------------------------------------------------------------ mesh

def bspline(P: int, u: float):
    """window_stencil(BSplineStencil{P}, u) (Windows.jl:209-223): (k0, w, dw)."""
    L = _load()
    w = np.zeros(P)
    dw = np.zeros(P)
    k0 = L.ora_bspline(int(P), float(u), _p(w), _p(dw))
    return k0, w, dw


KINDS = {"spme": 1, "p3m_ad": 2, "p3m_ik": 3}


def influence(kind, P, K, box, C, alpha, nmax=2):
    """G and Vc on the R2C half spectrum (Influence.jl:35-181)."""
    L = _load()
    K = np.ascontiguousarray(K, np.int32)
    nm = (K[0] // 2 + 1) * K[1] * K[2]
    G = np.zeros(nm)
    Vc = np.zeros(6 * nm)
    L.ora_influence(KINDS[kind], int(P), int(nmax), _p(K, _i), _p(_box(box)), float(C), float(alpha), _p(G), _p(Vc))
    return G, Vc.reshape(6, nm)


def _rfft(grid, K, workers):
    try:
        import scipy.fft as sf
        return sf.rfftn(grid.reshape(K[2], K[1], K[0]), workers=workers)
    except Exception:  # pragma: no cover
        return np.fft.rfftn(grid.reshape(K[2], K[1], K[0]))


def _irfft(spec, K, workers):
    M = K[0] * K[1] * K[2]
    try:
        import scipy.fft as sf
        out = sf.irfftn(spec, s=(K[2], K[1], K[0]), workers=workers)
    except Exception:  # pragma: no cover
        out = np.fft.irfftn(spec, s=(K[2], K[1], K[0]))
    return np.ascontiguousarray(out.reshape(-1) * M)   # the reference's backward transform is unnormalised


def hermitian_weight(K):
    K1h = K[0] // 2 + 1
    m1 = np.arange(K1h)
    w = np.where((m1 == 0) | ((K[0] % 2 == 0) & (m1 == K[0] // 2)), 0.5, 1.0)
    return np.broadcast_to(w[None, None, :], (K[2], K[1], K1h))


def mesh(pos, q, box, K, P, kind="spme", alpha=1.0, C=1.0, nmax=2, background=False, tables=None, workers=1):
    """Mesh part in FP64 (Solver.jl:305-393): spread, FFT, influence solve, inverse, gather.

    Returns per-particle forces F (n,3), energies E_i = q phi/2 + bg q, the mesh
    energy, the mesh virial (6, background included) and phi.
    """
    L = _load()
    K = np.ascontiguousarray(K, np.int32)
    x, y, z = _xyz(pos)
    n = len(x)
    qq = np.ascontiguousarray(q, np.float64)
    b = _box(box)
    grid = np.zeros(int(K[0]) * int(K[1]) * int(K[2]))
    L.ora_spread(n, _p(x), _p(y), _p(z), _p(qq), _p(b), _p(K, _i), int(P), _p(grid))
    spec = _rfft(grid, K, workers)
    G, Vc = tables if tables is not None else influence(kind, P, K, box, C, alpha, nmax)
    G3 = G.reshape(spec.shape)
    wgt = hermitian_weight(K)
    a = wgt * np.abs(spec) ** 2
    Emesh = float((a * G3).sum())
    Wm = np.array([float((a * Vc[c].reshape(spec.shape)).sum()) for c in range(6)])
    spec = spec * G3
    V = float(np.prod(box))
    bg = -C * (math.pi / (2 * alpha * alpha)) * qq.sum() / V if background else 0.0
    ubg = -C * (math.pi / (2 * alpha * alpha)) * qq.sum() ** 2 / V if background else 0.0
    F = np.zeros(3 * n)
    phi = np.zeros(n)
    if kind == "p3m_ik":
        fields = []
        Ls = box
        K1h = K[0] // 2 + 1
        m = [np.arange(K1h), np.arange(K[1]), np.arange(K[2])]
        for d in range(3):
            Kd = K[d]
            md = m[d]
            s = np.where((Kd % 2 == 0) & (md == Kd // 2), 0, np.where(md <= Kd // 2, md, md - Kd))
            kd = 2 * math.pi * s / Ls[d]
            shape = [1, 1, 1]
            shape[2 - d] = len(kd)
            fld = -1j * kd.reshape(shape) * spec
            fields.append(_irfft(fld, K, workers))
        pot = _irfft(spec, K, workers)
        L.ora_gather_ik(n, _p(x), _p(y), _p(z), _p(qq), _p(b), _p(K, _i), int(P), _p(fields[0]), _p(fields[1]),
                        _p(fields[2]), _p(pot), _p(F), _p(phi))
    else:
        pot = _irfft(spec, K, workers)
        L.ora_gather_ad(n, _p(x), _p(y), _p(z), _p(qq), _p(b), _p(K, _i), int(P), _p(pot), _p(F), _p(phi))
    E = 0.5 * qq * phi + bg * qq
    Wm[:3] += ubg
    return dict(F=F.reshape(n, 3), E=E, Emesh=Emesh, W=Wm, phi=phi, ubg=ubg)


def mesh_source_forces(pos, q, box, K, P, tables, sources, workers=1):
    """Mesh force (AD gather) on every particle from each source charge alone: (len(sources), n, 3).

    The mesh part is linear in the charges, so summing over all sources gives ``mesh(...)["F"]``; the
    source's own row entry is its self force through the mesh (zero for the exact reciprocal sum).
    """
    L = _load()
    K = np.ascontiguousarray(K, np.int32)
    x, y, z = _xyz(pos)
    n = len(x)
    qq = np.ascontiguousarray(q, np.float64)
    b = _box(box)
    G = tables[0]
    out = np.zeros((len(sources), n, 3))
    for s, j in enumerate(sources):
        grid = np.zeros(int(K[0]) * int(K[1]) * int(K[2]))
        xs, ys, zs = (np.ascontiguousarray(a[j:j + 1]) for a in (x, y, z))
        L.ora_spread(1, _p(xs), _p(ys), _p(zs), _p(np.ascontiguousarray(qq[j:j + 1])), _p(b), _p(K, _i), int(P),
                     _p(grid))
        spec = _rfft(grid, K, workers)
        pot = _irfft(spec * G.reshape(spec.shape), K, workers)
        F = np.zeros(3 * n)
        phi = np.zeros(n)
        L.ora_gather_ad(n, _p(x), _p(y), _p(z), _p(qq), _p(b), _p(K, _i), int(P), _p(pot), _p(F), _p(phi))
        out[s] = F.reshape(n, 3)
    return out


def pme_total(pos, q, box, *, C, alpha, rc, K, P, kind="spme", nmax=2, lj=None, workers=1):
    """Total (real space + mesh + self) forces, energy and virial of a charged system in FP64.

    lj: None or dict(sigma, eps, rc, kind) for a Lennard-Jones term on the same pairs.
    """
    kw = {}
    if lj is not None:
        kw = dict(kind=lj.get("kind", 1), sigma=lj["sigma"], eps=lj["eps"], rc_lj=lj["rc"],
                  eshift_lj=lj.get("eshift", 0.0))
    else:
        kw = dict(kind=0)
    pr = pairs_cells(pos, box, q=q, C=C, alpha=alpha, rc_coul=rc, **kw)
    ms = mesh(pos, q, box, K, P, kind=kind, alpha=alpha, C=C, nmax=nmax, workers=workers)
    q = np.asarray(q, float)
    selfE = -C * alpha / math.sqrt(math.pi) * q * q
    E = pr["E"] + ms["E"] + selfE
    W = pr["W"].sum(0) + ms["W"]
    return dict(F=pr["F"] + ms["F"], E=E, Etot=float(E.sum()), W=W, F_pair=pr["F"], F_mesh=ms["F"])


def exception_terms(pos, q, box, pairs, *, C, rc, eshift=0.0, bonded=(), lj=None):
    """Change of the forces, per-particle energies and per-particle virial rows (xx, yy, zz, xy, xz, yz)
    that exceptions make, in FP64, minimum image.

    pairs: 0-based (i, j, scale).  The pair's Coulomb term becomes scale * C qi qj / r in place of the
    full 1/r that the real-space sum and the mesh carry together (the excluded branch of pair_force,
    PairFunctor.jl:127-156, with _scaled_pairs_kernel!, Kernels.jl:307-339): a change of
    (scale - 1) C qi qj / r, and inside the real-space cutoff the ordinary pair's potential shift
    -C qi qj eshift goes too.  bonded: pairs whose LJ term is dropped (bond_exclusion_rows,
    Engine.jl:274-290); lj = dict(c6, c12, rc2, esh).  A bonded pair that is no Coulomb exception keeps
    its whole Coulomb term, so only its LJ term changes."""
    R = np.asarray(pos, float)
    q = np.asarray(q, float)
    L = np.asarray(box, float)
    n = len(R)
    F = np.zeros((n, 3))
    E = np.zeros(n)
    W = np.zeros((n, 6))

    def add(i, j, f, e, d):
        F[i] += f * d
        F[j] -= f * d
        E[i] += 0.5 * e
        E[j] += 0.5 * e
        w = 0.5 * f * np.array([d[0] * d[0], d[1] * d[1], d[2] * d[2], d[0] * d[1], d[0] * d[2], d[1] * d[2]])
        W[i] += w
        W[j] += w

    for i, j, s in pairs:
        if s == 1.0:
            continue
        d = R[i] - R[j]
        d -= L * np.round(d / L)
        r2 = float(d @ d)
        r = math.sqrt(r2)
        cq = C * q[i] * q[j]
        e = (s - 1.0) * cq / r + (cq * eshift if r2 < rc * rc else 0.0)
        add(i, j, (s - 1.0) * cq / (r2 * r), e, d)
    for i, j in bonded:
        d = R[i] - R[j]
        d -= L * np.round(d / L)
        r2 = float(d @ d)
        if r2 >= lj["rc2"]:
            continue
        ir6 = 1.0 / r2 ** 3
        f = (12.0 * lj["c12"] * ir6 - 6.0 * lj["c6"]) * ir6 / r2
        e = (lj["c12"] * ir6 - lj["c6"]) * ir6 - lj["esh"]
        add(i, j, -f, -e, d)
    return dict(F=F, E=E, W=W)


# ------------------------------------------------------------------ cluster list

def displacement_ratios(pos, ref_build, ref_prune, box, skin, prune_buffer):
    """Largest minimum-image |r - r_build|^2 / (skin/2)^2 and the larger of that and
    |r - r_prune|^2 / (prune_buffer/2)^2 over the particles (_displacement_kernel!,
    src/clusterpairs/List.jl:799-825; a zero threshold gives inf for any motion)."""
    L = np.asarray(box, float)

    def ratio(ref, half):
        d = np.asarray(pos, float) - np.asarray(ref, float)
        d -= L * np.round(d / L)
        d2 = (d * d).sum(1)
        if half == 0.0:
            return np.where(d2 > 0, np.inf, 0.0)
        r = d2 / (half * half)
        return np.where(np.isfinite(r), r, np.inf)

    rb = ratio(ref_build, 0.5 * skin)
    rp = ratio(ref_prune, 0.5 * prune_buffer)
    return float(rb.max()), float(np.maximum(rb, rp).max())


def list_decision(build_ratio, any_ratio, *, request=False, nstlist=0, nstprune=0, k=0):
    """(build, prune) of the device decision (_decide_kernel!, src/clusterpairs/Engine.jl:301-324).

    Triggers (nstlist = 0): rebuild when a particle moved more than skin/2 since the build or on
    request, prune after a rebuild or when one moved more than prune_buffer/2 since the prune.
    Fixed intervals: rebuild at decision k % nstlist == 0, on request or on non-finite motion; prune
    after a rebuild or at k % nstprune == 0."""
    if nstlist > 0:
        build = (k % nstlist == 0) or request or not math.isfinite(build_ratio)
        prune = build or (nstprune > 0 and k % nstprune == 0)
    else:
        build = build_ratio > 1.0 or request
        prune = build or any_ratio > 1.0
    return bool(build), bool(prune)


def force_coordinate(x, L):
    """force_coordinate (PeriodicDisplacement.jl:21-25) in Float32."""
    lib_ = _load()
    return np.array([lib_.ora_force_coordinate(float(v), float(L)) for v in np.asarray(x, np.float32)], np.float32)


def cluster_geometry(n, box, rlist):
    L = _load()
    g = np.zeros(10, np.int32)
    if L.ora_cluster_geometry(int(n), _p(_box(box)), float(rlist), _p(g, _i)):
        raise ValueError("box below twice the list radius")
    return dict(zip(("ncx", "ncy", "nzb", "mx", "my", "ncol", "nbin", "nsmax", "nslot", "ncs"), g.tolist()))


def cluster_build(pos32, box, rlist):
    """build! (List.jl:979-1051) in Float32 geometry: perm, scio, outer entries (cj << 8 | imask)."""
    L = _load()
    pos32 = np.asarray(pos32, np.float32)
    x, y, z = (np.ascontiguousarray(pos32[:, d]) for d in range(3))
    n = len(x)
    g = cluster_geometry(n, box, rlist)
    perm = np.zeros(g["nslot"], np.int32)
    scio = np.zeros(g["nsmax"] + 1, np.int32)
    necap = max(1024, 64 * g["nsmax"])
    while True:
        cjo = np.zeros(necap, np.uint32)
        ns = L.ora_cluster_build(n, _p(x, _f), _p(y, _f), _p(z, _f), _p(_box(box)), float(rlist), necap,
                                 _p(perm, _i), _p(scio, _i), _p(cjo, _u))
        if ns >= 0:
            break
        necap = -ns
    ne = int(scio[ns])
    return dict(ns=ns, perm=perm, scio=scio[:ns + 1].copy(), cjo=cjo[:ne].copy(), geom=g)


def cluster_prune(ns, xq, scio, cjo, box, rp, pbuf):
    """Prune + compaction (Kernels.jl:349-394, List.jl:719-759): working entries per super-cluster.

    The second word of an entry holds the two 8-bit warp masks and, in bit 16, the periodic-path
    mark (an atom within pbuf/2 of a face or a separation component above L/2 - pbuf)."""
    L = _load()
    xq = np.ascontiguousarray(xq, np.float32)
    scio = np.ascontiguousarray(scio, np.int32)
    cjo = np.ascontiguousarray(cjo, np.uint32)
    cjw = np.zeros((max(len(cjo), 1), 2), np.uint32)
    nw = np.zeros(max(ns, 1), np.int32)
    L.ora_cluster_prune(int(ns), _p(xq, _f), _p(scio, _i), _p(cjo, _u), _p(_box(box)), float(rp), float(pbuf), _p(cjw, _u),
                        _p(nw, _i))
    return cjw[:len(cjo)], nw[:ns]


def tile_pairs(perm, scio, entries, working: bool):
    """Particle pairs (i < j as sorted tuple set) covered by the live tiles of a list, and the multiset count.

    Newton-3 rule of the pair kernel: in a diagonal tile (cj == ci) only tj > ti.
    """
    pairs = []
    ns = len(scio) - 1
    for S in range(ns):
        for e in range(scio[S], scio[S + 1] if not working else scio[S] + entries["nw"][S]):
            if working:
                cj = int(entries["cjw"][e, 0])
                m = int(entries["cjw"][e, 1])
                masks = [(m & 0xff), (m >> 8) & 0xff]
            else:
                cj = int(entries["cjo"][e] >> 8)
                mm = int(entries["cjo"][e] & 0xff)
                masks = [mm, mm]
            for half in range(2):
                for a in range(8):
                    if not (masks[half] >> a) & 1:
                        continue
                    ci = 8 * S + a
                    for ti in range(8):
                        i = perm[8 * ci + ti]
                        if i < 0:
                            continue
                        for tj in range(4 * half, 4 * half + 4):
                            if cj == ci and not tj > ti:
                                continue
                            j = perm[8 * cj + tj]
                            if j < 0:
                                continue
                            pairs.append((min(i, j), max(i, j)))
    return pairs


# ------------------------------------------------------------------ CPU step (baseline)

class CpuMelt:
    """Velocity-Verlet NVE of an LJ + PME system on the host cores (FP64): the CPU baseline.

    Short-range forces from the cell-grid pair sums, the mesh from the FP64
    restatement with multithreaded FFTs; one step = kick, drift, forces, kick.
    """

    def __init__(self, pos, vel, q, masses, box, *, C, alpha, rc, K, P, lj, kind="spme", workers=-1):
        self.pos = np.array(pos, float)
        self.vel = np.array(vel, float)
        self.q = np.asarray(q, float)
        self.im = 1.0 / np.asarray(masses, float)
        self.box = tuple(box)
        self.kw = dict(C=C, alpha=alpha, rc=rc, K=K, P=P, kind=kind, lj=lj, workers=workers)
        self.tables = influence(kind, P, K, box, C, alpha)
        self.F = self.forces()

    def forces(self):
        kw = self.kw
        lj = kw["lj"]
        pr = pairs_cells(self.pos, self.box, q=self.q, C=kw["C"], alpha=kw["alpha"], rc_coul=kw["rc"],
                         kind=lj.get("kind", 1), sigma=lj["sigma"], eps=lj["eps"], rc_lj=lj["rc"])
        ms = mesh(self.pos, self.q, self.box, kw["K"], kw["P"], kind=kw["kind"], alpha=kw["alpha"], C=kw["C"],
                  tables=self.tables, workers=kw["workers"])
        return pr["F"] + ms["F"]

    def step(self, dt):
        self.vel += 0.5 * dt * self.im[:, None] * self.F
        self.pos += dt * self.vel
        L = np.array(self.box)
        self.pos -= L * np.floor(self.pos / L + 0.5)
        self.F = self.forces()
        self.vel += 0.5 * dt * self.im[:, None] * self.F


# ------------------------------------------------------------------ Langevin

def philox_normals4(seed: int, step: int, pid: int, stream: int = 0):
    """Four Float32 normals and the four Philox4x32-10 words for (pid, stream, step) under seed
    (src/engine/Philox.jl:20-67)."""
    L = _load()
    out = np.zeros(4, np.float32)
    words = np.zeros(4, np.uint32)
    L.ora_philox_normals4(int(seed) & 0xFFFFFFFFFFFFFFFF, int(step), int(pid), int(stream), _p(out, _f),
                          _p(words, _u))
    return out, words


def baoab_drift(pos, vel, force, inv_mass, box, *, dt, gamma, kT, seed, step):
    """One BAOAB drift (B1 A1 O A2) of Float32 state arrays (N x D) with FP64 intermediates
    (_baoa_kernel!, src/engine/Langevin.jl:58-88); returns new (pos, vel)."""
    L = _load()
    pos = np.asarray(pos, np.float32)
    n, dim = pos.shape
    comp = lambda a, d: np.ascontiguousarray(np.asarray(a, np.float32)[:, d])  # noqa: E731
    p = [comp(pos, d) for d in range(dim)]
    v = [comp(vel, d) for d in range(dim)]
    f = [comp(force, d) for d in range(dim)]
    if dim == 2:
        p.append(np.zeros(n, np.float32)); v.append(np.zeros(n, np.float32)); f.append(np.zeros(n, np.float32))
    im = np.ascontiguousarray(np.broadcast_to(np.asarray(inv_mass, np.float32), (n,)))
    noise = np.float32(np.sqrt(2.0 * float(gamma) * float(kT) * float(np.float32(dt))))
    b = np.array(list(box) + [1.0] * (3 - len(box)), np.float64)
    L.ora_baoab_drift(n, dim, *[_p(a, _f) for a in p], *[_p(a, _f) for a in v], *[_p(a, _f) for a in f],
                      _p(im, _f), float(dt), float(gamma), float(noise), int(seed) & 0xFFFFFFFFFFFFFFFF, int(step),
                      _p(b))
    return np.stack(p[:dim], 1), np.stack(v[:dim], 1)


def gjf_step_parts(pos, vel, force, inv_mass, box, *, dt, gamma, kT, seed, step):
    """Grønbech-Jensen-Farago positions (_gjf_pos_kernel!, src/engine/Langevin.jl:164-181) of Float32 state
    arrays (N x D): returns (new positions, the draw beta per particle) -- the velocity update
    (gjf_velocity) takes the same beta.  Coefficients in Float32 as the reference (gjf_pos_coefs,
    src/engine/Masses.jl:47-56)."""
    f32 = np.float32
    pos = np.asarray(pos, f32)
    n, dim = pos.shape
    vel = np.asarray(vel, f32)
    force = np.asarray(force, f32)
    im = np.broadcast_to(np.asarray(inv_mass, f32), (n,))
    dt32, g32 = f32(dt), f32(gamma)
    noise = f32(np.sqrt(2.0 * float(gamma) * float(kT) * float(dt32)))
    L = np.asarray(box, f32)
    out = pos.copy()
    beta = np.zeros((n, dim), f32)
    for i in range(n):
        q = f32(g32 * dt32 * im[i] / f32(2))
        b = f32(f32(1) / (f32(1) + q))
        coef = f32(b * dt32 * im[i] / f32(2))
        xi, _ = philox_normals4(seed, step, i + 1, 0)
        for d in range(dim):
            beta[i, d] = f32(noise * xi[d])
            dp = f32(f32(b * dt32) * vel[i, d] + coef * f32(dt32 * force[i, d] + beta[i, d]))
            x = f32(pos[i, d] + dp)
            x = f32(x - L[d]) if x >= f32(0.5) * L[d] else x
            x = f32(x + L[d]) if x < -f32(0.5) * L[d] else x
            out[i, d] = x
    return out, beta


def gjf_velocity(vel, f_old, f_new, inv_mass, beta, *, dt, gamma):
    """Grønbech-Jensen-Farago velocities (_gjf_vel_kernel!, src/engine/Langevin.jl:183-208):
    v = a v + dt/(2m) (a f_old + f_new) + (b/m) beta in FP64 with a, b from Float32 q."""
    f32 = np.float32
    vel = np.asarray(vel, np.float64)
    n = vel.shape[0]
    im32 = np.broadcast_to(np.asarray(inv_mass, f32), (n,))
    q = (f32(gamma) * f32(dt) * im32 / f32(2)).astype(f32)
    a = ((f32(1) - q) / (f32(1) + q)).astype(f32).astype(np.float64)[:, None]
    b = (f32(1) / (f32(1) + q)).astype(f32).astype(np.float64)[:, None]
    kf = (float(f32(dt)) * im32.astype(np.float64) / 2.0)[:, None]
    nf = b * im32.astype(np.float64)[:, None]
    return (a * vel + kf * (a * np.asarray(f_old, np.float64) + np.asarray(f_new, np.float64))
            + nf * np.asarray(beta, np.float64)).astype(f32)


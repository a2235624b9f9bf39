"""Seeded synthetic inputs of the benchmark shapes.

The reference has no public dataset on this path; its own generators
(``fcc_random_3d``, ``hex_random_2d``, src/InitGenerators.jl:191-203, 478-485)
build lattices with random perturbations.  These generators produce systems of
the same shapes from numpy PCG64 streams, so every input is reproducible from
its seed.  Units of the ionic melt: Angstrom, eV, amu, elementary charge; the
time unit is then Angstrom * sqrt(amu / eV) = 10.1805 fs.
"""
from __future__ import annotations

import math

import numpy as np

KB_EV = 8.617333262e-5                 # Boltzmann constant in eV / K
TIME_UNIT_FS = 10.180505305645         # Angstrom sqrt(amu / eV) in fs
COULOMB_EV_A = 14.399645               # e^2 / (4 pi eps0) in eV Angstrom


def fcc_lattice(ncell: int, rho: float, jitter: float = 0.05, seed: int = 0xC0FFEE00):
    """fcc ncell^3 x 4 sites at reduced density rho, +-jitter uniform per component, centred box."""
    rng = np.random.default_rng(seed)
    a = (4.0 / rho) ** (1.0 / 3.0)
    L = a * ncell
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(ncell), np.arange(ncell), np.arange(ncell), indexing="ij"), -1).reshape(-1, 3)
    pos = ((g[:, None, :] + base[None, :, :]).reshape(-1, 3) + 0.25) * a
    pos += rng.uniform(-jitter, jitter, size=pos.shape)
    pos -= L / 2
    pos -= L * np.floor(pos / L + 0.5)
    return pos, (L, L, L)


def hex_random_2d(n_side: int, phi: float, sigma: float = 1.0, displacement: float = 0.25, seed: int = 0):
    """n_side^2 disks of diameter sigma on a hexagonal lattice (rows shifted by half a spacing)
    in a square box at packing fraction phi, each displaced uniformly by up to `displacement`
    sigma per component; centred coordinates."""
    rng = np.random.default_rng(seed)
    n = n_side * n_side
    L = math.sqrt(n * math.pi * sigma * sigma / (4.0 * phi))
    a = L / n_side
    i, j = np.meshgrid(np.arange(n_side), np.arange(n_side), indexing="ij")
    x = (i + 0.5 * (j % 2) + 0.25) * a
    y = (j + 0.5) * a
    pos = np.stack([x.ravel(), y.ravel()], 1)
    pos += rng.uniform(-displacement, displacement, size=pos.shape) * sigma
    pos -= L / 2
    pos -= L * np.floor(pos / L + 0.5)
    return pos, (L, L)


def maxwell_boltzmann(masses, T: float, seed: int = 0, kB: float = 1.0, remove_com: bool = True, dim: int = 3):
    """Velocities at temperature T (COM momentum removed, rescaled to exactly T)."""
    rng = np.random.default_rng(seed)
    m = np.asarray(masses, float)
    v = rng.normal(size=(m.size, dim)) * np.sqrt(kB * T / m)[:, None]
    if remove_com:
        v -= (m[:, None] * v).sum(0) / m.sum()
    dof = dim * m.size - (dim if remove_com else 0)
    ke = 0.5 * (m[:, None] * v * v).sum()
    if ke > 0:
        v *= math.sqrt(0.5 * dof * kB * T / ke)
    return v


def ionic_melt(n: int, L: float, min_sep: float = 2.2, seed: int = 2026, batch: int = 4096):
    """n ions (half +1, half -1) uniformly random in a cubic box with a minimum separation.

    Seeded rejection sampling accelerated by a cell grid: candidates come in
    batches and are accepted in order when no accepted ion (earlier in the
    same batch included) lies within min_sep.
    """
    rng = np.random.default_rng(seed)
    ncell = max(3, int(L // min_sep))
    h = L / ncell
    cap = 8
    grid = np.full((ncell, ncell, ncell, cap), -1, np.int64)
    fill = np.zeros((ncell, ncell, ncell), np.int64)
    pos = np.empty((n, 3))
    m = 0
    offs = np.stack(np.meshgrid([-1, 0, 1], [-1, 0, 1], [-1, 0, 1], indexing="ij"), -1).reshape(-1, 3)
    d2min = min_sep * min_sep
    while m < n:
        cand = rng.uniform(0.0, L, size=(min(batch, 2 * (n - m) + 64), 3))
        cell = np.minimum((cand // h).astype(np.int64), ncell - 1)
        ok = np.ones(len(cand), bool)
        if m > 0:
            nb = (cell[:, None, :] + offs[None, :, :]) % ncell
            ids = grid[nb[..., 0], nb[..., 1], nb[..., 2]].reshape(len(cand), -1)
            valid = ids >= 0
            pj = pos[np.where(valid, ids, 0)]
            d = cand[:, None, :] - pj
            d -= L * np.round(d / L)
            close = (np.einsum("ijk,ijk->ij", d, d) < d2min) & valid
            ok &= ~close.any(1)
        idx = np.nonzero(ok)[0]
        c = cand[idx]
        d = c[:, None, :] - c[None, :, :]
        d -= L * np.round(d / L)
        conflict = np.triu(np.einsum("ijk,ijk->ij", d, d) < d2min, 1)
        keep = np.ones(len(idx), bool)
        for a, b in zip(*np.nonzero(conflict)):
            if keep[a] and keep[b]:
                keep[b] = False
        for k in idx[keep]:
            if m >= n:
                break
            cx, cy, cz = cell[k]
            if fill[cx, cy, cz] >= cap:
                continue
            grid[cx, cy, cz, fill[cx, cy, cz]] = m
            fill[cx, cy, cz] += 1
            pos[m] = cand[k]
            m += 1
    pos -= L / 2
    q = np.where(np.arange(n) < n // 2, 1.0, -1.0)
    perm = rng.permutation(n)
    return pos[perm].copy(), q, (L, L, L)


def melt_masses(q, m_plus: float = 22.99, m_minus: float = 35.45):
    q = np.asarray(q)
    return np.where(q > 0, m_plus, m_minus)


def fcc_fill(n: int, rho: float, jitter: float = 0.05, seed: int = 0):
    """n particles on the sites of the smallest cubic fcc lattice with at least n sites (a seeded
    random subset), scaled to number density rho, plus uniform jitter; centred coordinates."""
    rng = np.random.default_rng(seed)
    m = int(math.ceil((n / 4.0) ** (1.0 / 3.0) - 1e-9))
    L = (n / rho) ** (1.0 / 3.0)
    a = L / m
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
    sites = ((g[:, None, :] + basis[None, :, :]).reshape(-1, 3) + 0.25) * a
    pick = np.sort(rng.choice(len(sites), n, replace=False))
    pos = sites[pick] + rng.uniform(-jitter, jitter, (n, 3))
    pos -= L * np.floor(pos / L + 0.5)
    return pos, (L, L, L)


def replica_set(nrep: int, n_lo: int = 500, n_hi: int = 20000, rho=(0.70, 0.90), T=(0.6, 1.2), seed: int = 4):
    """Independent 3D LJ / WCA systems (even replicas LJ, odd WCA): N log-uniform in [n_lo, n_hi],
    reduced density and temperature uniform in the given ranges, seeded per replica."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(nrep):
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        out.append(dict(n=n, rho=float(rng.uniform(*rho)), T=float(rng.uniform(*T)),
                        kind="lj" if r % 2 == 0 else "wca", seed=int(rng.integers(1 << 31))))
    return out

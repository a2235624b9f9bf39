"""Batched replicas: host side of ``batch.cu`` and ``batch_mesh.cu``.

Hundreds of independent 3D LJ / WCA systems of uneven size run as one device batch: their
particles are concatenated, every stage of the NVE step is one launch over all replicas and the
step is captured into one CUDA graph.  Charged replicas (ionic melts) add the real-space Coulomb
polynomial to the pair kernel and one SPME / P3M-AD mesh per replica, spread, multiplied and
gathered in one launch each over all replicas, transformed by one batched cuFFT plan per mesh size.
``autotune_lanes`` picks the pair kernel's lanes per row, ``autotune`` the lanes per row and the
spread tile of charged batches, by timing the candidates on the batch itself.  The reference steps
one system per engine; looping the single-system engines is the comparison.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N
from . import splits, synthetic
from .engine import WCA_RC2_FACTOR, _destroy, _ptr, _stream

LJ_RC = 2.5


def replica_params(kind: str, box, n: int, eps: float = 1.0, sigma: float = 1.0, rc: float = LJ_RC):
    """One ``pd_batch_replica``: LJ cut at rc (unshifted) or WCA (rc^2 = 1.2599211 sigma^2, +eps)."""
    r = N.BatchReplica()
    for d in range(3):
        r.box[d] = float(box[d])
    r.n = int(n)
    r.eps, r.sigma = float(eps), float(sigma)
    if kind == "lj":
        r.kind, r.rc2, r.eshift = N.PD_PAIR_LJ, float(rc * rc), 0.0
    elif kind == "wca":
        r.kind, r.rc2, r.eshift = N.PD_PAIR_WCA, float(WCA_RC2_FACTOR * sigma * sigma), 0.0
    else:
        raise ValueError(f"unknown pair model {kind}")
    return r


class BatchedReplicas:
    """Device batch of replicas (``pd_batch``) with its concatenated step state."""

    def __init__(self, systems, *, skin: float = 0.3, cap: int | None = None, lanes: int = 4, device="cuda",
                 electrostatics: dict | None = None):
        """``systems``: list of dicts with n, box, kind, positions (n, 3) centred, velocities (n, 3),
        masses (n,) or a float, and optionally eps, sigma, rc (default 1, 1, 2.5) and charges (n,).
        ``cap`` (row capacity) defaults to 1.4x the mean row length at the densest replica, plus 16.
        ``electrostatics`` (charged replicas): dict with alpha, C, rc (real-space cutoff), order,
        kind ("spme" or "p3m_ad") and spacing (mesh spacing; each replica's mesh follows its box)."""
        self.systems = systems
        rcut = max(float(s.get("rc", LJ_RC)) for s in systems)
        if cap is None:
            rl = rcut + skin
            rho = max(s["n"] / float(np.prod(s["box"])) for s in systems)
            cap = int(1.4 * rho * 4.18879 * rl ** 3) + 16
        reps = (N.BatchReplica * len(systems))()
        for k, s in enumerate(systems):
            reps[k] = replica_params(s["kind"], s["box"], s["n"], eps=s.get("eps", 1.0), sigma=s.get("sigma", 1.0),
                                     rc=s.get("rc", LJ_RC))
        h = C.c_void_p()
        N.call("pd_batch_create", C.byref(h), reps, len(systems), float(skin), int(cap), int(lanes))
        self.cap = int(cap)
        self.handle = h
        n, nc = C.c_int(), C.c_int()
        N.call("pd_batch_count", h, C.byref(n), C.byref(nc))
        self.n, self.ncell = n.value, nc.value
        self.first = np.concatenate([[0], np.cumsum([s["n"] for s in systems])])[:-1]
        f32 = dict(dtype=torch.float32, device=device)
        pos = np.concatenate([s["positions"] for s in systems])
        vel = np.concatenate([s["velocities"] for s in systems])
        mass = np.concatenate([np.broadcast_to(np.asarray(s.get("masses", 1.0), float), (s["n"],)) for s in systems])
        self.x, self.y, self.z = (torch.tensor(pos[:, d], **f32) for d in range(3))
        self.vx, self.vy, self.vz = (torch.tensor(vel[:, d], **f32) for d in range(3))
        self.fx, self.fy, self.fz = (torch.zeros(self.n, **f32) for _ in range(3))
        self.epot = torch.zeros(self.n, **f32)
        self.inv_mass = torch.tensor(1.0 / mass, **f32)
        charged = any("charges" in s for s in systems)
        self.q = (torch.tensor(np.concatenate([np.asarray(s.get("charges", np.zeros(s["n"])), float) for s in systems]),
                               **f32) if charged else None)
        st = N.MDState()
        st.n = self.n
        for k in ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "epot", "inv_mass", "q"):
            setattr(st, k, _ptr(getattr(self, k)))
        self._state = st
        N.call("pd_batch_bind", h, C.byref(st))
        self.lanes = int(lanes)
        self.stream = torch.cuda.Stream(device=device)
        self.electrostatics = None
        self.spread_tile = (64, 2)
        if electrostatics is not None:
            self._set_electrostatics(electrostatics)

    def _set_electrostatics(self, el: dict):
        """Real-space Coulomb polynomial (the cluster route's fit) and one mesh per replica."""
        if self.q is None:
            raise ValueError("electrostatics needs per-particle charges in the systems")
        for k, s in enumerate(self.systems):
            qt = float(np.sum(s["charges"]))
            if abs(qt) > 1e-8 * max(1.0, float(np.abs(s["charges"]).sum())):
                raise ValueError(f"replica {k} has net charge {qt}; batched meshes take neutral replicas")
        alpha, Cc, rc = float(el["alpha"]), float(el["C"]), float(el["rc"])
        order = int(el.get("order", 5))
        kind = {"spme": N.PD_MESH_SPME, "p3m_ad": N.PD_MESH_P3M_AD}[el.get("kind", "spme")]
        poly = splits.coulomb_polynomial(alpha, Cc, rc, eshift=0.0)
        c = N.BatchCoulomb()
        c.C, c.rc2, c.sx, c.eshift = poly.C, poly.rc2, poly.sx, poly.eshift
        c.ne, c.nf = len(poly.pe), len(poly.pf)
        for k, v in enumerate(poly.pe):
            c.pe[k] = float(v)
        for k, v in enumerate(poly.pf):
            c.pf[k] = float(v)
        c.selfc = 2.0 * alpha / np.sqrt(np.pi)
        N.call("pd_batch_set_coulomb", self.handle, C.byref(c))
        meshes = [splits.resolve_mesh(el.get("mesh"), el.get("spacing"), s["box"], order) for s in self.systems]
        arr = (C.c_int * (3 * len(meshes)))(*[int(v) for m in meshes for v in m])
        N.call("pd_batch_set_mesh", self.handle, kind, order, alpha, Cc, arr)
        self.meshes = meshes
        self.electrostatics = dict(el, order=order, meshes=meshes)

    def set_spread_tile(self, tile: int, threads_per_ion: int = 2):
        """Ions per spread / gather CTA (32 or 64) and threads per ion (2, or 4 with 64)."""
        N.call("pd_batch_set_spread_tile", self.handle, int(tile), int(threads_per_ion))
        self.spread_tile = (int(tile), int(threads_per_ion))

    def mesh_info(self) -> dict:
        g, ch, nc = C.c_int(), C.c_int(), C.c_int()
        nn, nm = C.c_longlong(), C.c_longlong()
        N.call("pd_batch_mesh_info", self.handle, C.byref(g), C.byref(nn), C.byref(nm), C.byref(ch), C.byref(nc))
        return dict(groups=g.value, nodes=nn.value, modes=nm.value, tile=ch.value, tiles=nc.value)

    def close(self, _destroy=_destroy):
        if getattr(self, "handle", None):
            _destroy("pd_batch_destroy", self.handle)
            self.handle = None

    __del__ = close

    def set_lanes(self, lanes: int):
        N.call("pd_batch_set_lanes", self.handle, int(lanes))
        self.lanes = int(lanes)

    def evaluate(self, energy=False):
        N.call("pd_batch_evaluate", self.handle, int(bool(energy)), _stream(self.stream))
        self.stream.synchronize()

    def step(self, nsteps: int, dt: float, use_graph=True):
        N.call("pd_batch_step", self.handle, int(nsteps), float(dt), int(bool(use_graph)), _stream(self.stream))

    def synchronize(self):
        self.stream.synchronize()

    def status(self) -> dict:
        st = N.EllStats()
        N.call("pd_batch_status", self.handle, C.byref(st))
        return {k: getattr(st, k) for k, _ in N.EllStats._fields_}

    def replica(self, k: int, arr):
        """Slice of a concatenated per-particle array for replica k."""
        a = int(self.first[k])
        return arr[a:a + self.systems[k]["n"]]

    def autotune_lanes(self, candidates=(1, 2, 4, 8), reps: int = 20) -> dict:
        """Time the force pass for each lanes-per-row choice on this batch and keep the fastest."""
        times = {}
        s = self.stream
        for g in candidates:
            self.set_lanes(g)
            with torch.cuda.stream(s):
                for _ in range(3):
                    N.call("pd_batch_forces", self.handle, _ptr(self.x), _ptr(self.y), _ptr(self.z), _ptr(self.fx),
                           _ptr(self.fy), _ptr(self.fz), 0, 0, _stream(s))
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(s)
                for _ in range(reps):
                    N.call("pd_batch_forces", self.handle, _ptr(self.x), _ptr(self.y), _ptr(self.z), _ptr(self.fx),
                           _ptr(self.fy), _ptr(self.fz), 0, 0, _stream(s))
                b.record(s)
            b.synchronize()
            times[g] = a.elapsed_time(b) / reps
        best = min(times, key=times.get)
        self.set_lanes(best)
        self.evaluate()   # forces of the current positions again
        return {"lanes": best, "ms": times}


    def autotune(self, dt: float, lanes=(1, 2, 4, 8), tiles=((32, 2), (64, 2), (64, 4)), steps: int = 10) -> dict:
        """Time the captured step for every (lanes per row, spread tile) pair on this batch and keep the
        fastest (the step's pair pass and mesh branch overlap, so whole steps are timed); a spread tile is
        (ions per CTA, threads per ion).  The state is restored afterwards."""
        saved = [t.clone() for t in (self.x, self.y, self.z, self.vx, self.vy, self.vz, self.fx, self.fy, self.fz)]
        s = self.stream
        times = {}
        for g in lanes:
            for tile in (tiles if self.electrostatics is not None else (self.spread_tile,)):
                self.set_lanes(g)
                if self.electrostatics is not None:
                    self.set_spread_tile(*tile)
                self.step(2, dt)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                with torch.cuda.stream(s):
                    a.record(s)
                    self.step(steps, dt)
                    b.record(s)
                b.synchronize()
                times[(g, tile)] = a.elapsed_time(b) / steps
        best = min(times, key=times.get)
        self.set_lanes(best[0])
        if self.electrostatics is not None:
            self.set_spread_tile(*best[1])
        torch.cuda.synchronize()
        for t, v in zip((self.x, self.y, self.z, self.vx, self.vy, self.vz, self.fx, self.fy, self.fz), saved):
            t.copy_(v)
        torch.cuda.synchronize()
        self.evaluate()
        tag = lambda k: f"lanes {k[0]}, tile {k[1][0]}x{k[1][1]}" if isinstance(k[1], tuple) else f"lanes {k[0]}"
        return {"lanes": best[0], "spread_tile": list(best[1]) if isinstance(best[1], tuple) else best[1],
                "ms": {tag(k): v for k, v in times.items()}}


def make_systems(specs, mass: float = 1.0):
    """Positions (fcc fill at the replica's density) and Maxwell-Boltzmann velocities for replica specs
    (``synthetic.replica_set``)."""
    out = []
    for sp in specs:
        pos, box = synthetic.fcc_fill(sp["n"], sp["rho"], seed=sp["seed"])
        vel = synthetic.maxwell_boltzmann(np.full(sp["n"], mass), sp["T"], seed=sp["seed"] + 1)
        out.append(dict(n=sp["n"], box=box, kind=sp["kind"], positions=pos, velocities=vel, masses=mass,
                        T=sp["T"], rho=sp["rho"]))
    return out


def melt_sizes(nmelts: int, seed: int, n_lo: int = 2000, n_hi: int = 32000):
    """Sizes of a set of charged melts: N log-uniform in [n_lo, n_hi], rounded to even (half +1, half -1)."""
    import math
    rng = np.random.default_rng(seed)
    ns = [int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi))))) for _ in range(nmelts)]
    return [n + (n % 2) for n in ns]


def melt_systems(ns, rho: float = 0.0375, T: float = 1200.0, seed: int = 0, min_sep: float = 2.2):
    """Charged melts of the given sizes (half +1, half -1) at number density rho, seeded rejection
    placement with min_sep, Na/Cl masses, Maxwell-Boltzmann velocities at T (eV units, A/fs scaled by
    the synthetic module's time unit), LJ eps 0.01 eV, sigma 2.8 A, r_c 9 A; positions centred."""
    out = []
    for k, n in enumerate(ns):
        L = (n / rho) ** (1.0 / 3.0)
        pos, q, box = synthetic.ionic_melt(int(n), L, min_sep, seed=seed + 1000 + k)
        Lb = np.asarray(box, float)
        pos = pos - Lb * np.floor(pos / Lb + 0.5)   # centred image
        m = synthetic.melt_masses(q)
        v = synthetic.maxwell_boltzmann(m, T, seed=seed + 2000 + k, kB=synthetic.KB_EV)
        out.append(dict(n=int(n), box=box, kind="lj", positions=pos, velocities=v, masses=m, charges=q, eps=0.01,
                        sigma=2.8, rc=9.0))
    return out


def replica_cost(spec) -> float:
    """Work estimate of one replica per step: N times its neighbours per particle (N rho r_list^3)."""
    return float(spec["n"]) * float(spec["rho"]) * (LJ_RC + 0.3) ** 3


def partition_by_cost(specs, world: int):
    """Replicas split across `world` ranks by cost (longest-processing-time greedy): every rank gets a
    list of replica indices; the lists are disjoint, cover every replica and depend only on the specs,
    so every rank computes the same partition without communication."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(specs)), key=lambda k: (-replica_cost(specs[k]), k))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += replica_cost(specs[k])
    return [sorted(p) for p in parts]


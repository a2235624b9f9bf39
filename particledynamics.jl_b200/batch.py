"""Batched replicas: host side of ``batch.cu``.

Hundreds of independent 3D LJ / WCA systems of uneven size run as one device batch: their
particles are concatenated, every stage of the NVE step is one launch over all replicas and the
step is captured into one CUDA graph.  ``autotune_lanes`` picks the pair kernel's lanes per row by
timing the candidates on the batch itself.  The reference steps one system per engine; looping
the single-system ELL engines (``ELLDeviceEngine``) is the comparison.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N
from . import synthetic
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

    def __init__(self, systems, *, skin: float = 0.3, cap: int | None = None, lanes: int = 4, device="cuda"):
        """``systems``: list of dicts with n, box, kind, positions (n, 3) centred, velocities (n, 3),
        masses (n,) or a float.  ``cap`` (row capacity) defaults to 1.4x the mean row length at the
        densest replica, plus 16."""
        self.systems = systems
        if cap is None:
            rl = LJ_RC + skin
            rho = max(s["n"] / float(np.prod(s["box"])) for s in systems)
            cap = int(1.4 * rho * 4.18879 * rl ** 3) + 16
        reps = (N.BatchReplica * len(systems))()
        for k, s in enumerate(systems):
            reps[k] = replica_params(s["kind"], s["box"], s["n"])
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
        st = N.MDState()
        st.n = self.n
        for k in ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "epot", "inv_mass"):
            setattr(st, k, _ptr(getattr(self, k)))
        self._state = st
        N.call("pd_batch_bind", h, C.byref(st))
        self.lanes = int(lanes)
        self.stream = torch.cuda.Stream(device=device)

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


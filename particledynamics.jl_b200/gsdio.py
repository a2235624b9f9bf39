"""GSD snapshot I/O: trajectory frames, restart reads and the electrostatics settings record.

Mirrors the reference's GSD layer (src/io/GSDIO.jl, src/io/RestartIO.jl,
src/workflow/Writers.jl:50-90, src/workflow/System.jl:455-531,
src/workflow/Electrostatics.jl:318-360, src/electrostatics/Solver.jl:432-466): ``gsd_open`` /
``gsd_close``, ``write_gsd_frame``, ``read_gsd_frame``, ``read_gsd_log``, ``GSDFrameData``,
``settings_record``, ``exceptions_record``, ``electrostatics_from_settings`` and
``electrostatics_from_gsd`` (``write_gsd_frame!`` and ``read_gsd_frame!`` in Julia).

The file layer (GSD 2.0, HOOMD schema 1.4) is libpdb200's native ``pd_gsd_*`` code; a frame's
per-particle chunks leave the GPU through one packing kernel (``pd_snapshot_pack``) and one copy.
:class:`FrameStager` keeps that copy asynchronous: a frame is packed and copied on the state's
stream after the steps that produced it, and written to the file while the next steps run.
"""
from __future__ import annotations

import ctypes as C
import os
import warnings
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

HOOMD_SCHEMA = (1, 4)

# GSD type codes (RestartIO.jl:27-39) and the numpy types they hold
_TYPES = {1: np.uint8, 2: np.uint16, 3: np.uint32, 4: np.uint64, 5: np.int8, 6: np.int16, 7: np.int32, 8: np.int64,
          9: np.float32, 10: np.float64, 11: np.uint8}
_CODES = {np.dtype(np.uint8): 1, np.dtype(np.uint16): 2, np.dtype(np.uint32): 3, np.dtype(np.uint64): 4,
          np.dtype(np.int8): 5, np.dtype(np.int16): 6, np.dtype(np.int32): 7, np.dtype(np.int64): 8,
          np.dtype(np.float32): 9, np.dtype(np.float64): 10}

# covalent diameters of recognised element names, the default particles/diameter (GSDIO.jl:318-326)
ELEMENT_COVALENT_DIAMETER = {
    "H": 0.62, "He": 0.56, "Li": 2.56, "Be": 1.92, "B": 1.68, "C": 1.52, "N": 1.42, "O": 1.32, "F": 1.14,
    "Ne": 1.16, "Na": 3.32, "Mg": 2.82, "Al": 2.42, "Si": 2.22, "P": 2.14, "S": 2.10, "Cl": 2.04, "Ar": 2.12,
    "K": 4.06, "Ca": 3.52, "Fe": 2.64, "Ni": 2.48, "Cu": 2.64, "Zn": 2.44, "Br": 2.40, "Ag": 2.90, "I": 2.78,
    "Au": 2.72, "Hg": 2.64, "Pb": 2.92,
}

_ABSENT = (1 << 64) - 1


def _version(v) -> int:
    return (int(v[0]) << 16) | int(v[1])


class GSDFile:
    """An open GSD file (the handle of ``gsd_open``).  ``mode``: ``"w"`` create or truncate, ``"a"`` append
    after the last committed frame, ``"r"`` read."""

    def __init__(self, path, mode="r", application="ParticleDynamics", schema="hoomd", schema_version=HOOMD_SCHEMA):
        modes = {"w": 0, "a": 1, "r": 2}
        if mode not in modes:
            raise ValueError(f"GSD mode must be w, a or r; got {mode}")
        self.path = os.fspath(path)
        self.mode = mode
        h = C.c_void_p()
        N.call("pd_gsd_open", self.path.encode(), modes[mode], application.encode(), schema.encode(),
               _version(schema_version), C.byref(h))
        self._h = h
        self._names = None

    # -- lifetime
    def close(self):
        if self._h:
            h, self._h = self._h, None
            N.call("pd_gsd_close", h)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _handle(self):
        if not self._h:
            raise ValueError(f"GSD file {self.path} is closed")
        return self._h

    # -- writing
    def write_chunk(self, name: str, data, dtype=None):
        """write_chunk_raw!(h, name; type_code, N, M, data): an N-vector or N x M matrix, row-major."""
        a = np.asarray(data, dtype=dtype)
        if a.dtype == np.bool_:
            a = a.astype(np.uint8)
        code = _CODES.get(a.dtype)
        if code is None:
            raise TypeError(f"GSD chunk {name}: unsupported element type {a.dtype}")
        if a.ndim == 0:
            a = a.reshape(1)
        if a.ndim > 2:
            raise ValueError(f"GSD chunk {name}: data must be a vector or a matrix")
        a = np.ascontiguousarray(a)
        n = a.shape[0]
        m = 1 if a.ndim == 1 else a.shape[1]
        N.call("pd_gsd_write_chunk", self._handle(), name.encode(), code, n, max(m, 1),
               a.ctypes.data if a.size else None)

    def write_raw(self, name: str, code: int, n: int, m: int, ptr):
        """A chunk straight from host memory at ``ptr`` (n x m values of GSD type ``code``)."""
        N.call("pd_gsd_write_chunk", self._handle(), name.encode(), code, n, m, ptr)

    def end_frame(self):
        N.call("pd_gsd_end_frame", self._handle())
        self._names = None

    def flush(self):
        N.call("pd_gsd_flush", self._handle())

    # -- reading
    @property
    def nframes(self) -> int:
        return int(N.lib().pd_gsd_nframes(self._handle()))

    def header(self) -> dict:
        gv, sv = C.c_uint32(), C.c_uint32()
        app, sch = C.create_string_buffer(64), C.create_string_buffer(64)
        N.call("pd_gsd_header", self._handle(), C.byref(gv), C.byref(sv), app, sch)
        return dict(gsd_version=(gv.value >> 16, gv.value & 0xFFFF), schema_version=(sv.value >> 16, sv.value & 0xFFFF),
                    application=app.value.decode(), schema=sch.value.decode())

    def find(self, frame: int, name: str):
        e, found = N.GsdIndexEntry(), C.c_int()
        N.call("pd_gsd_find_chunk", self._handle(), int(frame), name.encode(), C.byref(e), C.byref(found))
        return e if found.value else None

    def read(self, entry) -> np.ndarray:
        """read_chunk(entry) (RestartIO.jl:41-52): a vector (M = 1) or an N x M matrix."""
        t = _TYPES.get(int(entry.type))
        if t is None:
            raise ValueError(f"Unsupported dtype code {entry.type} for chunk {self.name(entry.id)} in {self.path}")
        n, m = int(entry.N), max(1, int(entry.M))
        out = np.empty(n * m, t)
        if out.size:
            N.call("pd_gsd_read_chunk", self._handle(), C.byref(entry), out.ctypes.data, out.nbytes)
        return out if m == 1 else out.reshape(n, m)

    def name(self, cid: int) -> str:
        buf = C.create_string_buffer(4096)
        N.call("pd_gsd_name", self._handle(), int(cid), buf, len(buf))
        return buf.value.decode()

    def entries(self, frame: int) -> list:
        count = C.c_int()
        N.call("pd_gsd_frame_entries", self._handle(), int(frame), None, 0, C.byref(count))
        arr = (N.GsdIndexEntry * max(count.value, 1))()
        N.call("pd_gsd_frame_entries", self._handle(), int(frame), arr, count.value, C.byref(count))
        return list(arr[:count.value])

    def frame_names(self, frame: int) -> list:
        return [self.name(e.id) for e in self.entries(frame)]

    def latest(self, name: str, frame: int):
        """The chunk of the closest frame <= ``frame`` holding it (the GSD default-value rule)."""
        for f in range(int(frame), -1, -1):
            e = self.find(f, name)
            if e is not None:
                return e
        return None

    def find_one_of(self, frame: int, names):
        for nm in names:
            e = self.find(frame, nm)
            if e is not None:
                return e
        return None


def gsd_open(path, application="ParticleDynamics", schema="hoomd", schema_version=HOOMD_SCHEMA,
             append: bool = False) -> GSDFile:
    """gsd_open(path; application, schema, schema_version, append) (GSDIO.jl:167-175): a new file, or with
    ``append`` and an existing non-empty file, the continuation after its last frame."""
    path = os.fspath(path)
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    if append and os.path.isfile(path) and os.path.getsize(path) > 0:
        return GSDFile(path, "a")
    return GSDFile(path, "w", application=application, schema=schema, schema_version=schema_version)


def gsd_close(h: GSDFile) -> None:
    h.close()


def _encode_types(names) -> np.ndarray:
    """particles/types as int8 rows of the names, null-padded to the longest name + 1 (HOOMD schema)."""
    enc = [str(t).encode() for t in names]
    width = max([len(e) for e in enc] + [0]) + 1
    out = np.zeros((len(enc), width), np.int8)
    for k, e in enumerate(enc):
        out[k, :len(e)] = np.frombuffer(e, np.int8)
    return out


def _decode_types(a: np.ndarray) -> list:
    a = np.atleast_2d(np.asarray(a)).view(np.uint8)
    return [bytes(row).split(b"\0", 1)[0].decode() for row in a]


def _property_values(value, typeid1, types_names, n, default_by_type=None):
    """_particle_property_values (GSDIO.jl:328-346): None (per-type default), a scalar, a per-type or a
    per-particle vector."""
    if value is None:
        if default_by_type is None:
            return None
        per_type = np.array([default_by_type.get(str(t), 1.0) for t in types_names], np.float32)
        return per_type[typeid1 - 1]
    if np.ndim(value) == 0:
        return np.full(n, float(value), np.float32)
    vals = np.asarray(value, np.float32).reshape(-1)
    if len(vals) == n:
        return vals
    if len(vals) == len(types_names):
        return vals[typeid1 - 1]
    raise ValueError(f"property vector length {len(vals)} must equal N={n} or number of types={len(types_names)}")


# ----------------------------------------------------------------------------- device frames

class FrameStager:
    """Packs a state's per-particle chunks on the device and copies them to pinned host memory on the
    state's stream; :meth:`take` waits for the copy.  Two host buffers let one frame be written to
    the file while the next is being copied."""

    def __init__(self, st, forces=False, virial=False):
        import torch

        self.st = st
        self.src = N.SnapshotSrc()
        self.src.n, self.src.dim = st.n, st.dim
        keep = [st.x, st.y, st.z, st.vx, st.vy, st.vz] + ([st.fx, st.fy, st.fz] if forces else [None] * 3)
        for name, t in zip(("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz"), keep):
            setattr(self.src, name, t.data_ptr() if t is not None else None)
        self.src.type = st.typ.data_ptr()
        self.src.vir = st.vir6.data_ptr() if virial else None
        self.off = N.SnapshotOffsets()
        N.call("pd_snapshot_layout", C.byref(self.src), C.byref(self.off))
        nbytes = int(self.off.bytes)
        self.dev = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=st.dev)
        self.host = [torch.empty(max(nbytes, 16), dtype=torch.uint8, pin_memory=True) for _ in range(2)]
        self.events = [None, None]
        self.slot = 0
        self._keep = keep

    def stage(self) -> int:
        """Enqueue pack + copy of the current state after the work already on its stream; returns the slot."""
        import torch

        s = self.st.stream
        k = self.slot
        self.slot ^= 1
        if self.events[k] is not None:
            self.events[k].synchronize()   # the slot's previous frame has left the host buffer
        with torch.cuda.stream(s):
            N.call("pd_snapshot_pack", C.byref(self.src), self.dev.data_ptr(), self.dev.numel(), C.c_void_p(s.cuda_stream))
            self.host[k].copy_(self.dev, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
        self.events[k] = ev
        return k

    def take(self, k: int) -> dict:
        """The staged frame of slot ``k`` as numpy views of the pinned buffer (valid until the slot is reused)."""
        self.events[k].synchronize()
        buf = self.host[k].numpy()
        n, dim = self.st.n, self.st.dim

        def view(off, dtype, cols):
            if int(off) == _ABSENT:
                return None
            a = buf[int(off):int(off) + n * cols * np.dtype(dtype).itemsize].view(dtype)
            return a.reshape(n, cols) if cols > 1 else a

        return dict(position=view(self.off.position, np.float32, 3), velocity=view(self.off.velocity, np.float32, 3),
                    force=view(self.off.force, np.float32, 3), typeid=view(self.off.typeid, np.uint32, 1),
                    virial=view(self.off.virial, np.float32, int(self.off.virial_columns)))


def settings_record(solver) -> np.ndarray:
    """settings_record(solver) (Solver.jl:432-458): every setting needed to rebuild the solver exactly.
    [version 1, method (1 SPME, 2 P3M-AD, 3 P3M-ik, 4 ESP, 5 ESP with plain deconvolution),
    coulomb_prefactor, relative_permittivity, real_cutoff, alpha or split shape, order, window shape
    (0 for B-splines), K1, K2, K3, alias_order, net_charge (1 background), precision bits,
    real_space_modifier (1 potential shift)]."""
    spec = solver.spec
    code = {"spme": 1.0, "p3m_ad": 2.0, "p3m_ik": 3.0, "esp": 4.0, "esp_deconvolution": 5.0}[spec.influence]
    esp = spec.influence in ("esp", "esp_deconvolution")
    shape = float(spec.split_shape) if esp else float(spec.alpha)
    wshape = float(spec.window_shape) if esp else 0.0
    K = solver.mesh
    return np.array([1.0, code, spec.coulomb_prefactor, spec.relative_permittivity, spec.real_cutoff, shape,
                     float(spec.order), wshape, float(K[0]), float(K[1]), float(K[2]), float(spec.alias_order),
                     1.0 if spec.net_charge == "background" else 0.0, 32.0,
                     1.0 if spec.real_space_modifier == "potential_shift" else 0.0], np.float64)


def exceptions_record(exceptions) -> np.ndarray:
    """exceptions_record(solver) (Solver.jl:460-466): the (i, j, scale) triples, stable 1-based ids."""
    return np.array([v for t in exceptions for v in (float(t[0]), float(t[1]), float(t[2]))], np.float64)


def write_gsd_frame(h: GSDFile, st, diameter=None, mass=None, charge=None, types_names=("A",), step: int = 0,
                    write_forces: bool = False, write_virial: bool = False, sync_on_write: bool = False, logs=(),
                    stager: FrameStager | None = None, staged: int | None = None, topology=None):
    """write_gsd_frame!(h, st; ...) (GSDIO.jl:380-612): one HOOMD-schema frame of the state.

    Positions and velocities are always written; ``diameter``, ``mass`` and ``charge`` take None
    (defaults: element covalent diameters by type name, the state's masses and charges), a scalar,
    a per-type or a per-particle vector.  With an electrostatics solver attached the frame records
    ``log/electrostatics/settings`` and ``log/electrostatics/exceptions``.  ``write_forces`` and
    ``write_virial`` add the forces and the per-particle virial rows (``particles/virial`` and
    ``particles/property/virial``, float32 N x 6 in 3D, N x 3 in 2D).  ``logs`` adds float64 chunks
    ``name => values``.  The state has no unwrapped positions, so the frame carries no image chunk.

    A frame already staged by a :class:`FrameStager` (slot ``staged``) is written from its pinned
    buffer; otherwise the state is packed and copied now."""
    own = stager is None
    if own:
        stager = FrameStager(st, forces=write_forces, virial=write_virial)
    if staged is None:
        staged = stager.stage()
    fr = stager.take(staged)
    n, D = st.n, st.dim
    types_names = [str(t) for t in types_names]
    tid1 = fr["typeid"].astype(np.int32) + 1
    if tid1.size and (tid1.max() > len(types_names) or tid1.min() < 1):
        raise ValueError(f"type ids run to {int(tid1.max())} but types_names has {len(types_names)} names")
    box6 = np.zeros(6, np.float32)
    box6[:D] = st.box
    h.write_chunk("configuration/step", np.array([step], np.uint64))
    h.write_chunk("configuration/dimensions", np.array([D], np.uint8))
    h.write_chunk("configuration/box", box6)
    h.write_chunk("particles/N", np.array([n], np.uint32))
    h.write_chunk("particles/types", _encode_types(types_names))
    h.write_chunk("particles/typeid", fr["typeid"])
    h.write_chunk("particles/diameter",
                  _property_values(diameter, tid1, types_names, n, default_by_type=ELEMENT_COVALENT_DIAMETER))
    masses = (np.asarray(st.masses, np.float32).reshape(n) if mass is None
              else _property_values(mass, tid1, types_names, n))
    h.write_chunk("particles/mass", masses)
    charges = _property_values(charge, tid1, types_names, n)
    if charges is None and st.q is not None:
        charges = st.q.detach().float().cpu().numpy()
    if charges is not None:
        h.write_chunk("particles/charge", charges)
    if getattr(st, "solver", None) is not None:
        h.write_chunk("log/electrostatics/settings", settings_record(st.solver))
        exc = exceptions_record(getattr(st, "exceptions", []) or [])
        if exc.size:
            h.write_chunk("log/electrostatics/exceptions", exc.reshape(-1, 3))
    h.write_chunk("particles/position", fr["position"])
    h.write_chunk("particles/velocity", fr["velocity"])
    if write_forces:
        if fr["force"] is None:
            raise ValueError("write_forces needs a stager that packs the forces")
        h.write_chunk("particles/force", fr["force"])
    if write_virial:
        if fr["virial"] is None:
            raise ValueError("write_virial needs a stager that packs the virial rows")
        h.write_chunk("particles/virial", fr["virial"])
        h.write_chunk("particles/property/virial", fr["virial"])
    bonds = list(topology.bonds) if topology is not None else []
    if bonds:
        pairs = sorted({(min(i, j) - 1, max(i, j) - 1) for i, j in bonds if i != j})
        h.write_chunk("bonds/N", np.array([len(pairs)], np.uint32))
        h.write_chunk("bonds/types", _encode_types(["bond"]))
        h.write_chunk("bonds/typeid", np.zeros(len(pairs), np.uint32))
        h.write_chunk("bonds/group", np.array(pairs, np.uint32).reshape(-1, 2))
    for name, values in (logs.items() if isinstance(logs, dict) else logs):
        h.write_chunk(str(name), np.asarray(values, np.float64).reshape(-1))
    h.end_frame()
    if sync_on_write:
        h.flush()
    return h


# ----------------------------------------------------------------------------- reading

@dataclass
class GSDTopology:
    """Bonds, angles, dihedrals, impropers, constraints and special pairs of a frame (GSDIO.jl:12-19):
    each a dict with ``N``, ``types``, ``typeid0`` / ``typeid`` (0- / 1-based) and ``group0`` / ``group``."""
    bonds: dict
    angles: dict
    dihedrals: dict
    impropers: dict
    constraints: dict
    special_pairs: dict


@dataclass
class GSDFrameData:
    """Container of ``read_gsd_frame`` (GSDIO.jl:22-60); iterates as the legacy tuple
    ``(step, rx, ry, rz, vx, vy, vz, typeid, types, box, force)``."""
    step: int
    N: int
    D: int
    rx: np.ndarray
    ry: np.ndarray
    rz: np.ndarray | None
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray | None
    typeid: np.ndarray
    types: list
    box: tuple
    forceM: np.ndarray | None
    particle_properties: dict = field(default_factory=dict)
    per_type_properties: dict = field(default_factory=dict)
    topology: GSDTopology | None = None
    configuration: dict = field(default_factory=dict)

    def __iter__(self):
        return iter((self.step, self.rx, self.ry, self.rz, self.vx, self.vy, self.vz, self.typeid, self.types,
                     self.box, self.forceM))

    def __len__(self):
        return 11


def _scalar(a):
    a = np.asarray(a)
    return a.reshape(-1)[0] if a.size == 1 else a


def _topology_section(r: GSDFile, fid: int, prefix: str, cols: int, group_names) -> dict:
    ne = r.latest(f"{prefix}/N", fid)
    n = int(_scalar(r.read(ne))) if ne is not None else 0
    te = r.latest(f"{prefix}/types", fid)
    types = _decode_types(r.read(te)) if te is not None else []
    group0 = np.zeros((0, cols), np.uint32)
    typeid0 = np.zeros(0, np.uint32)
    if n > 0:
        ge = None
        for nm in group_names:
            ge = r.latest(nm, fid)
            if ge is not None:
                break
        if ge is not None:
            group0 = r.read(ge).astype(np.uint32).reshape(-1, cols)
        tie = r.latest(f"{prefix}/typeid", fid)
        typeid0 = r.read(tie).astype(np.uint32).reshape(-1) if tie is not None else np.zeros(n, np.uint32)
    return dict(N=n, types=types, typeid0=typeid0, typeid=typeid0.astype(np.int32) + 1, group0=group0,
                group=group0.astype(np.int32) + 1, tuples=[tuple(int(v) + 1 for v in row) for row in group0])


def _read_frame(r: GSDFile, fid: int, path: str) -> GSDFrameData:
    step_e = r.latest("configuration/step", fid)
    dim_e = r.latest("configuration/dimensions", fid)
    box_e = r.latest("configuration/box", fid)
    if step_e is None or dim_e is None or box_e is None:
        raise ValueError("configuration chunks missing")
    frame_step = int(_scalar(r.read(step_e)))
    D = int(_scalar(r.read(dim_e)))
    if D not in (2, 3):
        raise ValueError(f"Unsupported configuration/dimensions={D}")
    box6 = r.read(box_e).astype(np.float64).reshape(-1)
    n_e = r.latest("particles/N", fid)
    if n_e is None:
        raise ValueError("particles/N missing")
    n = int(_scalar(r.read(n_e)))
    pos_e = r.find_one_of(fid, ["particles/position", "particles/positions"]) or r.latest("particles/position", fid)
    if pos_e is None:
        raise ValueError("particles/position missing")
    pos = r.read(pos_e)
    if pos.ndim != 2:
        raise ValueError("particles/position expected matrix data")
    if not np.issubdtype(pos.dtype, np.floating):
        raise ValueError("particles/position must be floating-point")
    T = pos.dtype
    rx, ry = pos[:, 0].copy(), pos[:, 1].copy()
    rz = pos[:, 2].copy() if D == 3 else None
    vel_e = r.find_one_of(fid, ["particles/velocity", "particles/velocities"])
    if vel_e is None:
        vx, vy = np.zeros(n, T), np.zeros(n, T)
        vz = np.zeros(n, T) if D == 3 else None
        warnings.warn(f"Velocities missing in GSD frame {fid + 1} of {path}; using zeros")
    else:
        vel = r.read(vel_e).astype(T)
        vx, vy = vel[:, 0].copy(), vel[:, 1].copy()
        vz = vel[:, 2].copy() if D == 3 else None
    types_e = r.latest("particles/types", fid)
    types = _decode_types(r.read(types_e)) if types_e is not None else []
    tid_e = r.find_one_of(fid, ["particles/typeid", "particles/typeids"]) or r.latest("particles/typeid", fid)
    if tid_e is None:
        typeid = np.ones(n, np.int32)
    else:
        tid0 = r.read(tid_e).astype(np.uint32).reshape(-1)
        if len(tid0) != n:
            warnings.warn(f"particles/typeid length {len(tid0)} != N={n}")
        typeid = tid0.astype(np.int32) + 1
    if not types:
        types = ["A"]
    props: dict = {}
    skip = set()
    frc_e = r.find_one_of(fid, ["particles/force", "particles/forces", "particles/net_force",
                                "particles/property/force"])
    forceM = None
    if frc_e is not None:
        f = r.read(frc_e)
        nm = r.name(frc_e.id)
        if f.ndim == 2:
            forceM = f.astype(T)
        elif f.size == 3 * n:
            forceM = f.reshape(n, 3).astype(T)
        else:
            warnings.warn(f"Unexpected force chunk shape in {nm}; skipping forceM")
        if nm.startswith("particles/property/"):
            skip.add(nm)

    def vec(key, names, dtype):
        e = r.find_one_of(fid, names)
        if e is not None:
            a = r.read(e)
            if a.ndim != 1:
                raise ValueError(f"Chunk {r.name(e.id)} expected to be a vector")
            props[key] = a.astype(dtype)

    def mat(key, names, dtype):
        e = r.find_one_of(fid, names)
        if e is not None:
            a = r.read(e)
            if a.ndim != 2:
                raise ValueError(f"Chunk {r.name(e.id)} expected to be a matrix")
            props[key] = a.astype(dtype)

    vec("diameter", ["particles/diameter"], T)
    vec("mass", ["particles/mass"], T)
    vec("charge", ["particles/charge"], T)
    vec("body", ["particles/body"], np.int32)
    mat("image", ["particles/image"], np.int32)
    for key in ("orientation", "angmom", "moment_inertia", "acceleration", "momentum", "torque"):
        mat(key, [f"particles/{key}"], T)
    if forceM is not None:
        props["force"] = forceM
    vir_e = r.find_one_of(fid, ["particles/virial", "particles/property/virial"])
    if vir_e is not None:
        v = r.read(vir_e)
        nm = r.name(vir_e.id)
        if v.ndim == 2:
            props["virial"] = v.astype(T)
        elif v.size in (3 * n, 6 * n):
            props["virial"] = v.reshape(n, -1).astype(T)
        else:
            warnings.warn(f"Unexpected virial chunk shape in {nm}; skipping virial")
        if nm.startswith("particles/property/"):
            skip.add(nm)
    names = r.frame_names(fid)
    entries = r.entries(fid)
    extra = {}
    for e, nm in zip(entries, names):
        if nm.startswith("particles/property/") and nm not in skip:
            suffix = nm[len("particles/property/"):]
            if suffix:
                extra[suffix.replace("/", "_")] = _scalar(r.read(e))
    if extra:
        props["property"] = extra
    per_type = {}
    for e, nm in zip(entries, names):
        if nm == "particles/type_shapes":
            raw = r.read(e)
            per_type["shapes"] = ([s for s in bytes(raw.view(np.uint8)).decode(errors="replace").split("\0") if s]
                                  if raw.dtype in (np.uint8, np.int8) else raw)
        elif nm.startswith("particles/type_") and nm != "particles/types":
            per_type[nm[len("particles/type_"):].replace("/", "_")] = _scalar(r.read(e))
    extras = {}
    for e, nm in zip(entries, names):
        if nm.startswith("configuration/") and nm not in ("configuration/step", "configuration/dimensions",
                                                          "configuration/box"):
            extras[nm[len("configuration/"):].replace("/", "_")] = _scalar(r.read(e))
    topo = GSDTopology(
        bonds=_topology_section(r, fid, "bonds", 2, ["bonds/group"]),
        angles=_topology_section(r, fid, "angles", 3, ["angles/group"]),
        dihedrals=_topology_section(r, fid, "dihedrals", 4, ["dihedrals/group"]),
        impropers=_topology_section(r, fid, "impropers", 4, ["impropers/group"]),
        constraints=_topology_section(r, fid, "constraints", 2, ["constraints/group", "constraints/constraint"]),
        special_pairs=_topology_section(r, fid, "pairs", 2, ["pairs/pair", "pairs/group"]),
    )
    box = tuple(float(T.type(b)) for b in box6[:D])
    configuration = dict(metadata=dict(step=frame_step, N=n, dimension=D, box=box, box6=tuple(box6), extras=extras),
                         particles=dict(rx=rx, ry=ry, rz=rz, vx=vx, vy=vy, vz=vz, typeid=typeid, types=types,
                                        force=forceM, properties=props, per_type=per_type),
                         topology=topo)
    return GSDFrameData(frame_step, n, D, rx, ry, rz, vx, vy, vz, typeid, types, box, forceM, props, per_type, topo,
                        configuration)


def read_gsd_frame(path, step: int | None = None) -> GSDFrameData:
    """read_gsd_frame!(file_path; step) (RestartIO.jl:20-419).  ``step=None``: the last readable frame
    (earlier ones if the last is incomplete); otherwise the frame whose configuration/step equals
    ``step``, or, when none does, the ``step``-th frame (1-based)."""
    path = os.fspath(path)
    with GSDFile(path, "r") as r:
        nf = r.nframes
        if nf == 0:
            raise ValueError(f"No frames in GSD: {path}")
        if step is None:
            candidates = list(range(nf, 0, -1))
        else:
            candidates = []
            for i in range(1, nf + 1):
                e = r.find(i - 1, "configuration/step")
                if e is not None and int(_scalar(r.read(e))) == step:
                    candidates.append(i)
            if not candidates and 1 <= step <= nf:
                candidates = [int(step)]
        if not candidates:
            raise ValueError(f"Requested step={step} not found in {path}")
        last_error = None
        for idx in candidates:
            try:
                fr = _read_frame(r, idx - 1, path)
                if idx != nf and step is None:
                    warnings.warn(f"Last frame appears incomplete; using frame {idx} of {path}")
                return fr
            except ValueError as err:
                last_error = err
        raise last_error if last_error is not None else ValueError(f"Failed to read any valid frame from {path}")


def read_gsd_log(path, name: str, frame: int = -1):
    """read_gsd_log(path, name; frame) (RestartIO.jl:421-447): the float64 chunk ``name`` of the 1-based
    ``frame`` (-1 = last), inherited from the closest earlier frame; None when absent."""
    with GSDFile(os.fspath(path), "r") as r:
        nf = r.nframes
        if nf == 0:
            return None
        idx = nf if frame == -1 else int(frame)
        if not 1 <= idx <= nf:
            raise ValueError(f"Frame {frame} is out of range for {path}.")
        e = r.latest(name, idx - 1)
        if e is None:
            return None
        if int(e.type) != 10:
            raise ValueError(f"GSD chunk {name} is not Float64.")
        return r.read(e).reshape(-1).astype(np.float64)


def electrostatics_from_settings(rec, exceptions=()):
    """electrostatics_from_settings(record, exceptions) (Electrostatics.jl:318-344): the exact workflow
    descriptor of a settings record; the stored mesh is used verbatim."""
    from .workflow import ESP, PME, PPPM

    rec = np.asarray(rec, np.float64).reshape(-1)
    if not (len(rec) >= 14 and rec[0] == 1.0):
        raise ValueError("Unsupported electrostatics settings record.")
    method = int(rec[1])
    mesh = (int(rec[8]), int(rec[9]), int(rec[10]))
    net = "background" if rec[12] == 1.0 else "error"
    modifier = "potential_shift" if (len(rec) >= 15 and rec[14] == 1.0) else "none"
    pairs = tuple((int(e[0]), int(e[1]), float(e[2])) for e in exceptions)
    common = dict(coulomb_prefactor=float(rec[2]), relative_permittivity=float(rec[3]), real_cutoff=float(rec[4]),
                  mesh=mesh, net_charge=net, real_space_modifier=modifier, exclusions="none", scaled_pairs=pairs)
    if method == 1:
        return PME(**common, alpha=float(rec[5]), order=int(rec[6]))
    if method in (2, 3):
        return PPPM(**common, alpha=float(rec[5]), order=int(rec[6]), differentiation="ad" if method == 2 else "ik",
                    alias_order=int(rec[11]))
    if method in (4, 5):
        return ESP(**common, tolerance=None, split_shape=float(rec[5]), order=int(rec[6]), window_shape=float(rec[7]),
                   alias_order=int(rec[11]), influence="optimal" if method == 4 else "deconvolution")
    raise ValueError(f"Unknown electrostatics method code {method}.")


def electrostatics_from_gsd(path, frame: int = -1):
    """electrostatics_from_gsd(path; frame) (Electrostatics.jl:347-360): the descriptor recorded in a frame
    written while electrostatics was attached, or None."""
    rec = read_gsd_log(path, "log/electrostatics/settings", frame=frame)
    if rec is None:
        return None
    exc = read_gsd_log(path, "log/electrostatics/exceptions", frame=frame)
    triples = [] if exc is None else [tuple(exc[3 * k:3 * k + 3]) for k in range(len(exc) // 3)]
    return electrostatics_from_settings(rec, triples)

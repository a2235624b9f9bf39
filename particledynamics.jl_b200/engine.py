"""Device engines over the C ABI: cluster-pair engine, mesh solver, step engine.

These mirror the reference's engine objects: ``ClusterPairEngine``
(src/clusterpairs/Engine.jl:15-97), ``ElectrostaticsSpec`` /
``ElectrostaticsSolver`` (src/electrostatics/Spec.jl:31-102,
src/electrostatics/Solver.jl:75-158) and the device step of the engine
(src/engine/ClusterBackend.jl:90-220).  Device arrays are torch CUDA tensors;
only raw pointers cross into libpdb200.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from . import prolates, splits


def _ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


def _destroy(name: str, handle, _native=N) -> None:
    """Release a native handle; a no-op during interpreter shutdown (module globals already cleared)."""
    try:
        getattr(_native.lib(), name)(handle)
    except Exception:
        pass


def _stream(stream=None) -> int:
    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream)


def _require_cuda(*ts):
    for t in ts:
        if t is not None and (not t.is_cuda or not t.is_contiguous()):
            raise ValueError("device arrays must be contiguous CUDA tensors")


# ----------------------------------------------------------------------------- cluster pairs

class ClusterPairEngine:
    """Cluster-pair nonbonded engine (ClusterPairEngine, Engine.jl:54-97).

    ``lj`` is None or a dict with either ``c6, c12, rc2, esh`` (uniform) or
    ``table`` (ntypes^2 x 4 array from :func:`splits.lj_type_table`).  ``coulomb``
    is None or a :class:`splits.CoulombPolynomial`.
    """

    def __init__(self, n: int, box, *, rmax: float, skin: float, prune_buffer: float | None = None,
                 lj: dict | None = None, coulomb: splits.CoulombPolynomial | None = None, selfc: float = 0.0,
                 list_intervals: tuple[int, int] | None = None):
        if prune_buffer is None:
            prune_buffer = 0.5 * skin
        p = N.ClusterParams()
        p.n = int(n)
        p.rmax, p.skin, p.prune_buffer = float(rmax), float(skin), float(prune_buffer)
        if lj is None:
            p.lj_kind = N.PD_LJ_NONE
        elif "table" in lj and np.asarray(lj["table"]).shape[0] > 1:
            tab = np.asarray(lj["table"], np.float32)
            nt = int(round(math.sqrt(tab.shape[0])))
            if nt * nt != tab.shape[0] or nt > N.PD_MAX_TYPES:
                raise ValueError(f"LJ table needs ntypes^2 rows with ntypes <= {N.PD_MAX_TYPES}")
            p.lj_kind = N.PD_LJ_TABLE
            p.ntypes = nt
            flat = tab.reshape(-1)
            for k, v in enumerate(flat):
                p.lj_table[k] = float(v)
        else:
            if "table" in lj:
                c6, c12, rc2, esh = (float(v) for v in np.asarray(lj["table"]).reshape(-1)[:4])
            else:
                c6, c12, rc2, esh = (float(lj[k]) for k in ("c6", "c12", "rc2", "esh"))
            p.lj_kind = N.PD_LJ_UNIFORM
            p.lj_c6, p.lj_c12, p.lj_rc2, p.lj_esh = c6, c12, rc2, esh
            p.ntypes = 1
        if coulomb is not None:
            p.coulomb = 1
            p.coul_C, p.coul_rc2, p.coul_sx, p.coul_eshift = coulomb.C, coulomb.rc2, coulomb.sx, coulomb.eshift
            p.coul_has_mesh = int(coulomb.has_mesh)
            p.coul_ne, p.coul_nf = len(coulomb.pe), len(coulomb.pf)
            for k, v in enumerate(coulomb.pe):
                p.coul_pe[k] = float(v)
            for k, v in enumerate(coulomb.pf):
                p.coul_pf[k] = float(v)
            p.selfc = float(selfc)
        if list_intervals is not None:
            p.nstlist, p.nstprune = (int(v) for v in list_intervals)
        self.params = p
        self.n = int(n)
        self.coulomb = coulomb
        self.selfc = float(selfc)
        h = C.c_void_p()
        N.call("pd_cluster_create", C.byref(h), C.byref(p), N.dbl3(box))
        self.handle = h
        self.box = tuple(float(b) for b in box)

    def close(self, _destroy=_destroy):
        if getattr(self, "handle", None):
            _destroy("pd_cluster_destroy", self.handle)
            self.handle = None

    __del__ = close

    def setup(self, box):
        N.call("pd_cluster_setup", self.handle, N.dbl3(box))
        self.box = tuple(float(b) for b in box)

    def compute(self, x, y, z, q, typ, fx, fy, fz, epot=None, vir6=None, energy=False, stream=None):
        """compute!(eng, ...) (Engine.jl:185-190): overwrite the forces (and energies, virial rows)."""
        _require_cuda(x, y, z, q, typ, fx, fy, fz, epot, vir6)
        N.call("pd_cluster_compute", self.handle, _ptr(x), _ptr(y), _ptr(z), _ptr(q), _ptr(typ), _ptr(fx),
               _ptr(fy), _ptr(fz), _ptr(epot), _ptr(vir6), int(bool(energy)), _stream(stream))

    def decide(self, x, y, z, fixed=False, stream=None):
        N.call("pd_cluster_decide", self.handle, _ptr(x), _ptr(y), _ptr(z), int(fixed), _stream(stream))

    def build(self, x, y, z, q=None, typ=None, conditional=False, stream=None):
        N.call("pd_cluster_build", self.handle, _ptr(x), _ptr(y), _ptr(z), _ptr(q), _ptr(typ), int(conditional),
               _stream(stream))

    def pack(self, x, y, z, q=None, typ=None, stream=None):
        N.call("pd_cluster_pack", self.handle, _ptr(x), _ptr(y), _ptr(z), _ptr(q), _ptr(typ), _stream(stream))

    def prune(self, conditional=False, stream=None):
        N.call("pd_cluster_prune", self.handle, 0, 0, 0, int(conditional), _stream(stream))

    def pairs(self, energy=False, stream=None):
        N.call("pd_cluster_pairs", self.handle, int(bool(energy)), _stream(stream))

    def scatter(self, fx, fy, fz, epot=None, vir6=None, q=None, energy=False, add=False, stream=None):
        N.call("pd_cluster_scatter", self.handle, _ptr(fx), _ptr(fy), _ptr(fz), _ptr(epot), _ptr(vir6), _ptr(q),
               int(bool(energy)), int(bool(add)), _stream(stream))

    def pair_shape(self) -> tuple[int, int]:
        a, b = C.c_int(), C.c_int()
        N.call("pd_cluster_pair_shape", self.handle, C.byref(a), C.byref(b))
        return a.value, b.value

    def set_pair_shape(self, nsplit: int, warps: int):
        N.call("pd_cluster_set_pair_shape", self.handle, int(nsplit), int(warps))

    def autotune_pairs(self, stream=None, reps: int = 20, warps=(1, 2, 4)) -> dict:
        """Time the pair pass (force only) over CTA shapes -- parts per super-cluster (the default and
        half / twice it) x warps per part -- and keep the fastest.  The pair pass accumulates into the slot
        forces, so the caller re-evaluates the forces afterwards."""
        n0, w0 = self.pair_shape()
        splits = sorted({max(1, n0 // 2), n0, min(64, 2 * n0)})
        s = stream if stream is not None else torch.cuda.current_stream()
        times = {}
        for ns in splits:
            for w in warps:
                self.set_pair_shape(ns, w)
                with torch.cuda.stream(s):
                    for _ in range(3):
                        self.pairs(energy=False, stream=s)
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(s)
                    for _ in range(reps):
                        self.pairs(energy=False, stream=s)
                    b.record(s)
                b.synchronize()
                times[(ns, w)] = a.elapsed_time(b) / reps
        best = min(times, key=times.get)
        self.set_pair_shape(*best)
        return {"nsplit": best[0], "warps": best[1], "default": [n0, w0],
                "ms": {f"{k[0]}x{k[1]}": v for k, v in times.items()}}

    def set_exceptions(self, exceptions=(), bonds=()):
        """Coulomb exceptions and bond exclusions (0-based storage indices).

        ``exceptions``: ``(i, j)`` (excluded) or ``(i, j, scale)`` items, normalised as
        ``normalize_exceptions`` (Spec.jl:200-227) does; ``bonds``: ``(i, j)`` pairs whose LJ term is
        dropped, with the corrections of ``bond_exclusion_rows`` (Engine.jl:274-290).  Empty lists
        remove every exception.  The next evaluation rebuilds the list."""
        pi, pj, sc = [], [], []
        for item in exceptions:
            if len(item) not in (2, 3):
                raise ValueError("Each electrostatic exception must be (i, j) or (i, j, scale).")
            pi.append(int(item[0]))
            pj.append(int(item[1]))
            sc.append(float(item[2]) if len(item) == 3 else 0.0)
        bi, bj = [], []
        for item in bonds:
            if len(item) != 2:
                raise ValueError("Each bonded pair must be (i, j).")
            bi.append(int(item[0]))
            bj.append(int(item[1]))
        a = np.array(pi, np.int32)
        b = np.array(pj, np.int32)
        s = np.array(sc, np.float64)
        c = np.array(bi, np.int32)
        d = np.array(bj, np.int32)
        N.call("pd_cluster_set_exceptions", self.handle, len(a), a.ctypes.data, b.ctypes.data, s.ctypes.data,
               len(c), c.ctypes.data, d.ctypes.data)

    def grow(self):
        N.call("pd_cluster_grow", self.handle)

    def statistics(self, stream=None) -> dict:
        """statistics(eng) (Engine.jl:402-412)."""
        s = N.ClusterStats()
        N.call("pd_cluster_status", self.handle, C.byref(s), _stream(stream))
        d = {k: getattr(s, k) for k, _ in N.ClusterStats._fields_}
        d["pairs_per_particle"] = 32.0 * s.tile_bits / max(self.n, 1)
        return d

    def order_ptr(self) -> int:
        return int(N.lib().pd_cluster_order(self.handle) or 0)

    def buffers(self) -> dict:
        ptrs = [C.c_void_p() for _ in range(6)]
        N.call("pd_cluster_buffers", self.handle, *[C.byref(p) for p in ptrs])
        return dict(zip(("perm", "xq", "scio", "cjo", "cjw", "nw"), [p.value or 0 for p in ptrs]))

    def list_host(self) -> dict:
        """Host copies of the list (tests): perm, packed xyzq, outer and working entries per super-cluster."""
        st = self.statistics()
        b = self.buffers()
        ns, nslot, nsmax = st["superclusters"], st["nslot"], st["nsmax"]
        dev = torch.device("cuda")

        def fetch(ptr, count, dtype):
            out = torch.empty(count, dtype=dtype, device=dev)
            torch.cuda.synchronize()
            _memcpy_d2d(out.data_ptr(), ptr, out.numel() * out.element_size())
            return out.cpu().numpy()

        perm = fetch(b["perm"], nslot, torch.int32)
        xq = fetch(b["xq"], 4 * nslot, torch.float32).reshape(-1, 4)
        scio = fetch(b["scio"], nsmax + 1, torch.int32)
        nw = fetch(b["nw"], nsmax, torch.int32)
        ne = int(scio[ns]) if ns > 0 else 0
        cjo = fetch(b["cjo"], max(ne, 1), torch.int32).view(np.uint32)[:ne]
        cjw = fetch(b["cjw"], 2 * max(ne, 1), torch.int32).view(np.uint32).reshape(-1, 2)[:ne]
        return dict(ns=ns, perm=perm, xq=xq, scio=scio[:ns + 1], nw=nw[:ns], cjo=cjo, cjw=cjw, stats=st)


def _memcpy_d2d(dst: int, src: int, nbytes: int):
    cudart = _cudart()
    rc = cudart.cudaMemcpy(C.c_void_p(dst), C.c_void_p(src), C.c_size_t(nbytes), 3)
    if rc != 0:
        raise RuntimeError(f"cudaMemcpy failed ({rc})")


_CUDART = None


def _cudart():
    """The CUDA runtime torch already loaded (for device-to-device copies of list buffers in tests)."""
    global _CUDART
    if _CUDART is None:
        torch.cuda.init()
        for name in ("libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so.12"):
            try:
                _CUDART = C.CDLL(name)
                break
            except OSError:
                continue
        if _CUDART is None:
            raise RuntimeError("libcudart.so.12 not found")
        _CUDART.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
        _CUDART.cudaMemcpy.restype = C.c_int
    return _CUDART


# ----------------------------------------------------------------------------- electrostatics

_KINDS = {"spme": N.PD_MESH_SPME, "p3m_ad": N.PD_MESH_P3M_AD, "p3m_ik": N.PD_MESH_P3M_IK, "esp": N.PD_MESH_ESP,
          "esp_deconvolution": N.PD_MESH_ESP_DECONV}
_ESP = ("esp", "esp_deconvolution")


@dataclass
class ElectrostaticsSpec:
    """Validated description of a mesh Coulomb solver (ElectrostaticsSpec, Spec.jl:31-102).

    Gaussian split + B-spline window (``spme``, ``p3m_ad``, ``p3m_ik``: ``alpha``, ``order`` = B-spline
    order) or prolate split + prolate window (``esp``, ``esp_deconvolution``: ``split_shape`` c,
    ``window_shape`` c_1, ``order`` = window width in grid points)."""
    coulomb_prefactor: float
    real_cutoff: float
    alpha: float | None = None
    influence: str = "spme"
    order: int = 4
    mesh: tuple | None = None
    mesh_spacing: float | None = None
    alias_order: int = 2
    relative_permittivity: float = 1.0
    net_charge: str = "error"
    real_space_modifier: str = "none"
    net_charge_tolerance: float = 1e-8
    split_shape: float | None = None
    window_shape: float | None = None

    def __post_init__(self):
        if not (math.isfinite(self.coulomb_prefactor) and self.coulomb_prefactor > 0):
            raise ValueError("coulomb_prefactor must be finite and positive.")
        if not (math.isfinite(self.relative_permittivity) and self.relative_permittivity > 0):
            raise ValueError("relative_permittivity must be finite and positive.")
        if not (math.isfinite(self.real_cutoff) and self.real_cutoff > 0):
            raise ValueError("real_cutoff must be finite and positive.")
        if self.influence not in _KINDS:
            raise ValueError(f"Unknown influence kind {self.influence}.")
        if self.influence in _ESP:
            if self.split_shape is None or self.window_shape is None:
                raise ValueError("ESP requires a prolate split and a prolate window.")
            if not (math.isfinite(self.split_shape) and self.split_shape > 0 and math.isfinite(self.window_shape)
                    and self.window_shape > 0):
                raise ValueError("Prolate shapes must be finite and positive.")
            if not (3 <= self.order <= 12):
                raise ValueError(f"Prolate window width must be between 3 and 12 grid points in this build; "
                                 f"got {self.order}.")
            pmax = prolates.max_prolate_order(self.window_shape)
            if self.order > pmax:
                raise ValueError(f"A prolate window of shape {self.window_shape:.3f} supports at most {pmax} grid "
                                 f"points (P <= 2c/pi - 1/2); got {self.order}. Use a larger window shape (tighter "
                                 "tolerance) or a narrower window.")
        else:
            if self.alpha is None or not (math.isfinite(self.alpha) and self.alpha > 0):
                raise ValueError("Ewald alpha must be finite and positive.")
            if not (3 <= self.order <= 12):
                raise ValueError(f"B-spline assignment order must be between 3 and 12; got {self.order}.")
        if not (0 <= self.alias_order <= 6):
            raise ValueError("alias_order must be between 0 and 6.")
        if self.net_charge not in ("error", "background"):
            raise ValueError(f"net_charge must be error or background; got {self.net_charge}.")
        if self.real_space_modifier not in ("none", "potential_shift"):
            raise ValueError("real_space_modifier must be none or potential_shift.")
        if self.mesh is None and self.mesh_spacing is None:
            raise ValueError("Provide either `mesh=(K1,K2,K3)` or `mesh_spacing`.")
        if self.mesh is not None:
            if len(self.mesh) != 3:
                raise ValueError("mesh must have three dimensions.")
            if any(k < self.order for k in self.mesh):
                raise ValueError(f"Every mesh dimension must be at least the assignment order {self.order}.")

    @property
    def C(self) -> float:
        return self.coulomb_prefactor / self.relative_permittivity

    @property
    def prolate(self) -> bool:
        return self.influence in _ESP


class ElectrostaticsSolver:
    """Mesh part of a PME/P3M solver on the device (ElectrostaticsSolver, Solver.jl:129-158).

    ``charges`` (host) set the net-charge policy and the background term
    (set_solver_charges!, Solver.jl:166-177).
    """

    def __init__(self, spec: ElectrostaticsSpec, box, charges, nmax: int | None = None):
        box = tuple(float(b) for b in box)
        if not 2 * spec.real_cutoff < min(box):
            raise ValueError(f"real_cutoff={spec.real_cutoff} must be smaller than half the shortest box length "
                             f"{min(box)} (minimum-image real space).")
        q = np.asarray(charges, float)
        if not np.all(np.isfinite(q)):
            raise ValueError("Charges must be finite.")
        Q = float(q.sum())
        qabs = float(np.abs(q).sum())
        if spec.net_charge == "error" and abs(Q) > spec.net_charge_tolerance * max(qabs, 1.0):
            raise ValueError(f"The system carries net charge {Q}. Neutralise it, or select net_charge=background.")
        self.spec = spec
        self.box = box
        self.mesh = splits.resolve_mesh(spec.mesh, spec.mesh_spacing, box, spec.order)
        self.qtotal = Q
        self.qsq = float((q * q).sum())
        self.C = spec.C
        if spec.prolate:
            self.split = prolates.ProlateSplit(spec.real_cutoff, spec.split_shape)
            self.window = prolates.ProlateWindow(spec.order, spec.window_shape)
            if self.window.nyquist_attenuation() < prolates.min_nyquist_attenuation(np.float32):
                raise ValueError(f"The prolate window (width {spec.order}, shape {spec.window_shape:.3f}) decays "
                                 "below what an FP32 mesh solve resolves at the mesh Nyquist frequency; use a "
                                 "larger window shape.")
            self.selfc = self.split.self_coefficient()
            self.eshift = 0.0    # the prolate split vanishes at the cutoff (cutoff_energy, Splits.jl:77-78)
        else:
            self.selfc = splits.self_coefficient(spec.alpha)
            self.eshift = splits.cutoff_energy(spec.alpha, spec.real_cutoff) \
                if spec.real_space_modifier == "potential_shift" else 0.0
        p = N.MeshParams()
        p.kind = _KINDS[spec.influence]
        p.order = spec.order
        p.alias_order = spec.alias_order
        for d in range(3):
            p.mesh[d] = self.mesh[d]
        p.alpha = spec.alpha if spec.alpha is not None else 0.0
        p.C = self.C
        p.background = 1 if spec.net_charge == "background" else 0
        p.qtotal = Q
        p.nmax = int(nmax if nmax is not None else len(q))
        self.params = p
        h = C.c_void_p()
        if spec.prolate:
            self._prolate = self._prolate_tables(p)
            N.call("pd_mesh_create_prolate", C.byref(h), C.byref(p), C.byref(self._prolate[0]), N.dbl3(box))
        else:
            N.call("pd_mesh_create", C.byref(h), C.byref(p), N.dbl3(box))
        self.handle = h

    def _prolate_tables(self, p):
        """pd_prolate of this solver: the split's quadrature of c_hat, the window's node polynomials (fitted
        to FP32 round-off) and, per axis, the deconvolution (esp_deconvolution) or the alias table (esp)."""
        w = N.Prolate()
        sp, win = self.split, self.window
        w.cutoff = sp.cutoff
        w.nquad = len(sp.xq)
        for i, (x, c) in enumerate(zip(sp.xq, sp.wchi)):
            w.xq[i], w.wchi[i] = float(x), float(c)
        w.background_coefficient = sp.background_coefficient()
        Cp = win.node_polynomials(np.float32)
        H, D1 = Cp.shape
        w.deg = D1 - 1
        for k in range(D1):
            for hh in range(H):
                w.poly[k][hh] = float(Cp[hh, k])
        tabs = []
        for d in range(3):
            K = int(self.mesh[d])
            if self.spec.influence == "esp":
                t = np.ascontiguousarray(win.alias_table(K, self.spec.alias_order).T)   # m-major
            else:
                t = np.ascontiguousarray(win.deconvolution(K))
            tabs.append(t)
            w.table[d] = t.ctypes.data
        return w, tabs

    def close(self, _destroy=_destroy):
        if getattr(self, "handle", None):
            _destroy("pd_mesh_destroy", self.handle)
            self.handle = None

    __del__ = close

    @property
    def ik(self) -> bool:
        return self.spec.influence == "p3m_ik"

    def set_box(self, box):
        """refresh_geometry! (Solver.jl:193-209)."""
        N.call("pd_mesh_set_box", self.handle, N.dbl3(box))
        self.box = tuple(float(b) for b in box)

    def transform(self, x, y, z, q, order=None, n=None, energy=False, stream=None):
        n = x.numel() if n is None else n
        N.call("pd_mesh_transform", self.handle, _ptr(x), _ptr(y), _ptr(z), _ptr(q),
               0 if order is None else (order if isinstance(order, int) else _ptr(order)), int(n),
               int(bool(energy)), _stream(stream))

    def gather(self, x, y, z, q, fx, fy, fz, epot=None, vglobal=None, order=None, n=None, energy=False, set=False,
               stream=None):
        n = x.numel() if n is None else n
        N.call("pd_mesh_gather", self.handle, _ptr(x), _ptr(y), _ptr(z), _ptr(q),
               0 if order is None else (order if isinstance(order, int) else _ptr(order)), int(n), _ptr(fx),
               _ptr(fy), _ptr(fz), _ptr(epot), _ptr(vglobal), int(bool(energy)), int(bool(set)), _stream(stream))

    def mesh_energy(self, stream=None) -> np.ndarray:
        out = (C.c_double * 7)()
        N.call("pd_mesh_energy", self.handle, out, _stream(stream))
        return np.array(out[:])

    def self_energy(self) -> float:
        """-(C/2) chi(0)/r_c sum q^2 (Solver.jl:421)."""
        return -0.5 * self.C * self.selfc * self.qsq

    def background_energy(self) -> float:
        if self.spec.net_charge != "background":
            return 0.0
        coef = self.split.background_coefficient() if self.spec.prolate else \
            splits.background_coefficient(self.spec.alpha)
        return -self.C * coef * self.qtotal ** 2 / np.prod(self.box)

    def influence(self) -> tuple[np.ndarray, np.ndarray]:
        dims = (C.c_int * 3)()
        nm = C.c_int()
        N.call("pd_mesh_dims", self.handle, dims, C.byref(nm))
        G = np.empty(nm.value, np.float32)
        Vc = np.empty(6 * nm.value, np.float32)
        N.call("pd_mesh_influence", self.handle, G.ctypes.data_as(C.c_void_p), Vc.ctypes.data_as(C.c_void_p))
        return G, Vc.reshape(6, -1)

    def coulomb_polynomial(self) -> splits.CoulombPolynomial:
        corr = prolates.ProlateCorrection(self.split) if self.spec.prolate else self.spec.alpha
        return splits.coulomb_polynomial(corr, self.C, self.spec.real_cutoff, eshift=self.eshift)

    def set_self_force_removal(self, table_size: int = 16):
        """Subtract each charge's own force through the mesh (AD gathers; 0 turns it off).

        Not part of the reference's solver, whose mesh forces keep the spurious self force; the
        learned coarse-mesh form uses it on its coarse mesh."""
        N.call("pd_mesh_set_self_force_removal", self.handle, int(table_size))
        self.self_force_T = int(table_size)

    def self_force_table(self) -> np.ndarray:
        """(T, T, T, 3) array S[t3, t2, t1] of the self force per unit charge squared (empty when off)."""
        T = C.c_int()
        N.call("pd_mesh_self_force_table", self.handle, None, C.byref(T))
        out = np.empty((T.value, T.value, T.value, 4), np.float32)
        if T.value:
            N.call("pd_mesh_self_force_table", self.handle, out.ctypes.data_as(C.c_void_p), C.byref(T))
        return out[..., :3]


# ----------------------------------------------------------------------------- step engine

class DeviceEngine:
    """Captured NVE step over a cluster engine and an optional mesh (ClusterBackend.jl:90-220).

    ``state`` is a dict of CUDA tensors: x, y, z, vx, vy, vz, fx, fy, fz, q, type,
    inv_mass (or a float), epot, vir6 (N x 6), vglobal (6).
    """

    def __init__(self, cluster: ClusterPairEngine, mesh: ElectrostaticsSolver | None, state: dict, box):
        s = N.MDState()
        s.n = int(state["x"].numel())
        for k in ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz"):
            setattr(s, k, _ptr(state[k]))
        s.q = _ptr(state.get("q"))
        s.type = _ptr(state.get("type"))
        im = state.get("inv_mass", 1.0)
        if isinstance(im, torch.Tensor):
            s.inv_mass = _ptr(im)
            s.inv_mass_uniform = 0.0
        else:
            s.inv_mass = 0
            s.inv_mass_uniform = float(im)
        s.epot = _ptr(state.get("epot"))
        s.vir6 = _ptr(state.get("vir6"))
        s.vglobal6 = _ptr(state.get("vglobal"))
        self.state = state
        self.cluster = cluster
        self.mesh = mesh
        h = C.c_void_p()
        N.call("pd_md_create", C.byref(h), cluster.handle, mesh.handle if mesh is not None else None, C.byref(s),
               N.dbl3(box))
        self.handle = h
        self._keep = s

    def close(self, _destroy=_destroy):
        if getattr(self, "handle", None):
            _destroy("pd_md_destroy", self.handle)
            self.handle = None

    __del__ = close

    def evaluate(self, energy=False, stream=None):
        N.call("pd_md_evaluate", self.handle, int(bool(energy)), _stream(stream))

    def set_learned(self, correction=None, net=None):
        """Attach the learned coarse-mesh correction (``learned.LearnedCorrection`` + ``learned.MLPNetwork``):
        every force pass then adds s_i V_i before the closing kick.  A correction without a network adds the
        radial term V_i alone (s = 1); None detaches it."""
        N.call("pd_md_set_learned", self.handle, correction.handle if correction is not None else None,
               net.handle if net is not None else None)
        self._learned = (correction, net)

    def set_schedule(self, pair_wait: int):
        """Start the pair pass after the prune (0), the mesh spread (1) or the forward transform (2)."""
        N.call("pd_md_set_schedule", self.handle, int(pair_wait))
        self.pair_wait = int(pair_wait)

    def step(self, nsteps: int, dt: float, energy_last=False, use_graph=True, stream=None):
        N.call("pd_md_step", self.handle, int(nsteps), float(dt), int(bool(energy_last)), int(bool(use_graph)),
               _stream(stream))

    def step_host(self, host_xyz: np.ndarray, host_v: np.ndarray, nsteps: int, dt: float, stream=None,
                  energy: bool = True):
        """Steps from and back to host buffers (3n floats each); the potential energy of the last step
        when energy is set, else None."""
        e = C.c_double()
        N.call("pd_md_step_host", self.handle, host_xyz.ctypes.data_as(C.c_void_p),
               host_v.ctypes.data_as(C.c_void_p), int(nsteps), float(dt), C.byref(e) if energy else None,
               _stream(stream))
        return e.value if energy else None


# ----------------------------------------------------------------------------- ELL route

WCA_RC2_FACTOR = 1.2599211   # rc^2 / sigma^2 of the WCA model (src/engine/PairModels.jl:25)


class ELLEngine:
    """Cell-list neighbour rows with a fixed capacity and the row pair kernels (the reference's default
    `CellList` route for Lennard-Jones and WCA: DeviceNeighborWorkspace, DeviceNeighborCUDA.jl:64-88;
    UniformLJ / UniformWCA, src/engine/PairModels.jl:13-49).

    ``dim`` is 2 or 3; coordinates are centred (|x| <= L/2).  ``capacity`` and ``interval`` are the
    CellList ``capacity`` and ``rebuild_interval``; ``skin`` is its ``buffer``.
    """

    def __init__(self, n: int, box, *, dim: int = 3, model: str = "lj", epsilon: float = 1.0, sigma: float = 1.0,
                 cutoff: float | None = None, skin: float = 0.4, capacity: int = 96, interval: int = 20,
                 shift: bool = False, lanes: int = 0):
        if model not in ("lj", "wca"):
            raise ValueError(f"unknown pair model {model!r}")
        eps, sig = float(epsilon), float(sigma)
        if model == "wca":
            rc2 = np.float32(WCA_RC2_FACTOR) * np.float32(sig * sig)
            rc = float(np.sqrt(rc2)) if cutoff is None else float(cutoff)
            eshift = 0.0
        else:
            if cutoff is None:
                raise ValueError("LennardJones requires an explicit cutoff.")
            rc = float(cutoff)
            rc2 = np.float32(rc) * np.float32(rc)
            eshift = splits.lj_cutoff_energy(sig, eps, rc) if shift else 0.0
        p = N.EllParams()
        p.dim, p.n = int(dim), int(n)
        p.cutoff, p.skin = rc, float(skin)
        p.cap, p.interval = int(capacity), int(interval)
        p.model = N.PD_PAIR_LJ if model == "lj" else N.PD_PAIR_WCA
        p.eps, p.sigma, p.rc2, p.eshift = eps, sig, float(rc2), float(eshift)
        p.lanes = int(lanes)
        self.params = p
        self.n, self.dim, self.model = int(n), int(dim), model
        self.box = tuple(float(b) for b in box) + (1.0,) * (3 - len(box))
        h = C.c_void_p()
        N.call("pd_ell_create", C.byref(h), C.byref(p), N.dbl3(self.box))
        self.handle = h

    def close(self, _destroy=_destroy):
        if getattr(self, "handle", None):
            _destroy("pd_ell_destroy", self.handle)
            self.handle = None

    __del__ = close

    def update(self, x, y, z=None, stream=None):
        N.call("pd_ell_update", self.handle, _ptr(x), _ptr(y), _ptr(z), _stream(stream))

    def request(self, stream=None):
        N.call("pd_ell_request", self.handle, _stream(stream))

    def forces(self, x, y, z, fx, fy, fz, epot=None, vir=None, energy=False, stream=None):
        N.call("pd_ell_forces", self.handle, _ptr(x), _ptr(y), _ptr(z), _ptr(fx), _ptr(fy), _ptr(fz), _ptr(epot),
               _ptr(vir), int(bool(energy)), _stream(stream))

    def status(self) -> dict:
        st = N.EllStats()
        N.call("pd_ell_status", self.handle, C.byref(st))
        return {k: getattr(st, k) for k, _ in N.EllStats._fields_}

    def resize(self, capacity: int):
        N.call("pd_ell_resize", self.handle, int(capacity))

    def counts_host(self) -> np.ndarray:
        """Host copy of the row lengths."""
        r, c = C.c_void_p(), C.c_void_p()
        N.call("pd_ell_rows", self.handle, C.byref(r), C.byref(c))
        counts = torch.empty(self.n, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        _memcpy_d2d(counts.data_ptr(), c.value, 4 * self.n)
        return counts.cpu().numpy()

    def rows_host(self):
        """Host copies of the rows (as a list of neighbour-id arrays, truncated at the capacity)."""
        r, c = C.c_void_p(), C.c_void_p()
        N.call("pd_ell_rows", self.handle, C.byref(r), C.byref(c))
        st = self.status()
        cap, n = st["cap"], self.n
        rows = torch.empty(cap * n, dtype=torch.int32, device="cuda")
        counts = torch.empty(n, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        _memcpy_d2d(rows.data_ptr(), r.value, 4 * cap * n)
        _memcpy_d2d(counts.data_ptr(), c.value, 4 * n)
        R = rows.cpu().numpy().reshape(cap, n)
        cnt = counts.cpu().numpy()
        return [R[:min(cnt[i], cap), i].copy() for i in range(n)], cnt


class ELLDeviceEngine:
    """Captured NVE / Langevin (BAOAB) steps on the ELL route (src/engine/Run.jl:162-294,
    src/engine/Langevin.jl:58-88).  ``state``: dict of CUDA tensors x, y, (z), vx, vy, (vz), fx, fy,
    (fz), inv_mass (or a float), epot, vir (N x 6 in 3D, N x 3 in 2D)."""

    def __init__(self, ell: ELLEngine, state: dict):
        s = N.MDState()
        s.n = int(state["x"].numel())
        for k in ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz"):
            setattr(s, k, _ptr(state.get(k)))
        im = state.get("inv_mass", 1.0)
        if isinstance(im, torch.Tensor):
            s.inv_mass, s.inv_mass_uniform = _ptr(im), 0.0
        else:
            s.inv_mass, s.inv_mass_uniform = 0, float(im)
        s.epot = _ptr(state.get("epot"))
        s.vir6 = _ptr(state.get("vir"))
        self.state, self.ell = state, ell
        h = C.c_void_p()
        N.call("pd_ell_md_create", C.byref(h), ell.handle, C.byref(s))
        self.handle = h
        self._keep = s

    def close(self, _destroy=_destroy):
        if getattr(self, "handle", None):
            _destroy("pd_ell_md_destroy", self.handle)
            self.handle = None

    __del__ = close

    def evaluate(self, energy=False, stream=None):
        N.call("pd_ell_md_evaluate", self.handle, int(bool(energy)), _stream(stream))

    def step(self, nsteps: int, dt: float, energy_last=False, use_graph=True, stream=None):
        N.call("pd_ell_md_step", self.handle, int(nsteps), float(dt), int(bool(energy_last)), int(bool(use_graph)),
               _stream(stream))

    def bookkeeping(self, dq=None, dU=None, ekin=None):
        """Attach (or detach) the Langevin bookkeeping arrays: heat dq, force work dU (accumulated) and the
        kinetic energy after each step, n floats each."""
        N.call("pd_ell_md_bookkeeping", self.handle, _ptr(dq), _ptr(dU), _ptr(ekin))
        self._bookkeeping = (dq, dU, ekin)

    def langevin(self, nsteps: int, dt: float, gamma: float, kT: float, seed: int, energy_last=False,
                 use_graph=True, stream=None, scheme: str = "baoab"):
        """Langevin steps: ``scheme`` "baoab" (BAOAB splitting), "baoa" (BAOA) or "gjf" (Grønbech-Jensen-Farago)."""
        name = {"baoab": "pd_ell_md_langevin", "baoa": "pd_ell_md_baoa", "gjf": "pd_ell_md_gjf"}.get(scheme)
        if name is None:
            raise ValueError(f"unknown Langevin scheme {scheme!r}")
        N.call(name, self.handle, int(nsteps), float(dt), float(gamma), float(kT),
               int(seed) & 0xFFFFFFFFFFFFFFFF, int(bool(energy_last)), int(bool(use_graph)), _stream(stream))

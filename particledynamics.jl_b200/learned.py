"""Learned coarse-mesh correction: host side of ``mlp.cu``, ``learned.cu`` and ``ewald.cu``.

The reference has no learned form; this is an added force term compared with the plain
fine-mesh PME of the same system.  PME runs on a mesh twice as coarse (2.0 A, order 4 instead of
1.0 A, order 5) and the force residual of the coarse mesh is predicted per particle:

* descriptors ``x_i`` (32 features): 2 species x 16 Gaussian radial bases of neighbour charge
  within ``rcut`` (6 A), with the smooth cutoff ``(1 - r^2 / rcut^2)^2``;
* a scalar ``s_i`` from a 32-128-128-1 SiLU network (BF16 weights and activations, FP32
  accumulation, tcgen05 tensor cores);
* the residual ``F_i = s_i V_i`` with ``V_i = sum_j q_i q_j b(r_ij) (r_i - r_j)``: the network's
  scalar times a per-neighbour radial weight multiplies each displacement vector, so the residual
  rotates with the configuration.

Before anything is learned, the coarse mesh's spurious self force (the force each ion receives
through the mesh from its own charge, a known function of its position relative to the nodes) is
removed exactly (``ElectrostaticsSolver.set_self_force_removal``).

Training (``CoarseMeshTrainer``): snapshots from a fine-mesh run give the target
``R_i = F_fine_mesh - F_coarse_mesh`` (the real-space part is identical for both meshes), the radial
function ``b`` is fitted by linear least squares, then the network is trained by Adam on the mean
squared error of ``s_i V_i - R_i`` with the fused forward/backward tensor-core kernel.  Held-out
errors are stated against the FP64 Ewald sum on the GPU (``ewald_oracle``).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _native as N
from .engine import ElectrostaticsSolver, ElectrostaticsSpec, _destroy, _ptr, _stream

N_IN, N_H = 32, 128
PARAM_COUNT = N_H * N_IN + N_H + N_H * N_H + N_H + N_H + 1
_SLICES = {}
_o = 0
for _name, _shape in (("w1", (N_H, N_IN)), ("b1", (N_H,)), ("w2", (N_H, N_H)), ("b2", (N_H,)), ("w3", (N_H,)),
                      ("b3", (1,))):
    _SLICES[_name] = (_o, _shape)
    _o += int(np.prod(_shape))
assert _o == PARAM_COUNT


def split_params(flat) -> dict:
    """Views of the flat parameter vector: w1 (128, 32), b1, w2 (128, 128), b2, w3 (128,), b3 (1,)."""
    return {k: flat[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in _SLICES.items()}


def init_params(seed: int = 0, s0: float = 1.0, out_scale: float = 1e-2) -> np.ndarray:
    """He-style initial weights, zero biases, a small output layer and b3 = s0 (so that s starts near s0)."""
    rng = np.random.default_rng(seed)
    flat = np.zeros(PARAM_COUNT, np.float32)
    p = split_params(flat)
    p["w1"][:] = rng.normal(0.0, math.sqrt(2.0 / N_IN), (N_H, N_IN))
    p["w2"][:] = rng.normal(0.0, math.sqrt(2.0 / N_H), (N_H, N_H))
    p["w3"][:] = rng.normal(0.0, out_scale / math.sqrt(N_H), N_H)
    p["b3"][:] = s0
    return flat


class MLPNetwork:
    """The 32-128-128-1 SiLU network on the device (``pd_mlp``)."""

    def __init__(self, params=None, seed: int = 0):
        if N.lib().pd_mlp_param_count() != PARAM_COUNT:
            raise RuntimeError("libpdb200 and the host disagree on the network layout")
        h = C.c_void_p()
        N.call("pd_mlp_create", C.byref(h))
        self.handle = h
        self.set_params(init_params(seed) if params is None else params)

    def close(self, _destroy=_destroy):
        if getattr(self, "handle", None):
            _destroy("pd_mlp_destroy", self.handle)
            self.handle = None

    __del__ = close

    def set_params(self, flat):
        a = np.ascontiguousarray(flat, np.float32)
        if a.size != PARAM_COUNT:
            raise ValueError(f"expected {PARAM_COUNT} parameters, got {a.size}")
        N.call("pd_mlp_set_params", self.handle, a.ctypes.data_as(C.c_void_p))

    def params(self) -> np.ndarray:
        a = np.empty(PARAM_COUNT, np.float32)
        N.call("pd_mlp_get_params", self.handle, a.ctypes.data_as(C.c_void_p))
        return a

    def grads(self) -> np.ndarray:
        a = np.empty(PARAM_COUNT, np.float32)
        N.call("pd_mlp_get_grads", self.handle, a.ctypes.data_as(C.c_void_p))
        return a

    def forward(self, X, V=None, s=None, corr=None, stream=None):
        """s (n,) and/or corr (n, 4) = (s V, s) for X (n, 32) bfloat16 on the device."""
        n = X.shape[0]
        if X.dtype != torch.bfloat16 or tuple(X.shape[1:]) != (N_IN,) or not X.is_contiguous():
            raise ValueError("X must be a contiguous (n, 32) bfloat16 tensor")
        if V is not None and corr is None:
            corr = torch.empty((n, 4), dtype=torch.float32, device=X.device)
        if V is None and s is None:
            s = torch.empty(n, dtype=torch.float32, device=X.device)
        N.call("pd_mlp_forward", self.handle, _ptr(X), int(n), _ptr(s), _ptr(V), _ptr(corr), _stream(stream))
        return corr if V is not None else s

    def train_batch(self, X, ab, scale: float, stream=None):
        """Fused forward + backward: gradients of sum (s^2 a - 2 s b) scale / 2 added to the network's."""
        n = X.shape[0]
        if ab.shape != (n, 2) or ab.dtype != torch.float32 or not ab.is_contiguous():
            raise ValueError("ab must be a contiguous (n, 2) float32 tensor")
        N.call("pd_mlp_train", self.handle, _ptr(X), _ptr(ab), int(n), float(scale), _stream(stream))

    def adam(self, lr: float, beta1=0.9, beta2=0.999, eps=1e-8, grad_scale=1.0, stream=None):
        N.call("pd_mlp_adam", self.handle, float(lr), float(beta1), float(beta2), float(eps), float(grad_scale),
               _stream(stream))

    def loss(self, reset: bool = True) -> float:
        out = C.c_double()
        N.call("pd_mlp_loss", self.handle, C.byref(out), int(bool(reset)))
        return out.value

    def zero_grads(self, stream=None):
        N.call("pd_mlp_zero_grads", self.handle, _stream(stream))

    def error(self) -> int:
        out = C.c_int()
        N.call("pd_mlp_error", self.handle, C.byref(out))
        return out.value


DEFAULT_DESCRIPTOR = dict(rcut=6.0, skin=1.0, mu0=0.5, dmu=5.5 / 15.0, sigma=0.35, nb=8, nu0=2.0, dnu=4.0 / 7.0,
                          tau=0.45)


class LearnedCorrection:
    """Descriptors and network residual over device neighbour rows (``pd_learned``)."""

    def __init__(self, n: int, box, *, cap: int | None = None, coef=None, **kw):
        cfg = dict(DEFAULT_DESCRIPTOR)
        cfg.update(kw)
        self.cfg = cfg
        self.n = int(n)
        self.box = tuple(float(b) for b in box)
        p = N.LearnedParams()
        p.rcut, p.skin = cfg["rcut"], cfg["skin"]
        if cap is None:
            rho = self.n / float(np.prod(self.box))
            cap = int(1.5 * rho * 4.18879 * (cfg["rcut"] + cfg["skin"]) ** 3) + 32
        p.cap = int(cap)
        p.mu0, p.dmu, p.sigma = cfg["mu0"], cfg["dmu"], cfg["sigma"]
        p.nb, p.nu0, p.dnu, p.tau = int(cfg["nb"]), cfg["nu0"], cfg["dnu"], cfg["tau"]
        c = np.zeros(N.PD_LEARNED_MAX_RADIAL) if coef is None else np.asarray(coef, float)
        for m in range(N.PD_LEARNED_MAX_RADIAL):
            p.coef[m] = float(c[m]) if m < len(c) else 0.0
        self.params = p
        h = C.c_void_p()
        N.call("pd_learned_create", C.byref(h), C.byref(p), self.n, N.dbl3(self.box))
        self.handle = h
        self.coef = np.array([p.coef[m] for m in range(p.nb)])

    def close(self, _destroy=_destroy):
        if getattr(self, "handle", None):
            _destroy("pd_learned_destroy", self.handle)
            self.handle = None

    __del__ = close

    @property
    def nb(self) -> int:
        return int(self.params.nb)

    def set_radial(self, coef):
        c = np.ascontiguousarray(coef, np.float32)
        N.call("pd_learned_set_radial", self.handle, c.ctypes.data_as(C.c_void_p), int(c.size))
        self.coef = c.astype(float)

    def descriptors(self, x, y, z, q, typ=None, X=None, V=None, stream=None):
        """(X (n, 32) bfloat16, V (n, 4) float32) at centred coordinates."""
        dev = x.device
        X = torch.empty((self.n, N_IN), dtype=torch.bfloat16, device=dev) if X is None else X
        V = torch.empty((self.n, 4), dtype=torch.float32, device=dev) if V is None else V
        N.call("pd_learned_descriptors", self.handle, _ptr(x), _ptr(y), _ptr(z), _ptr(q), _ptr(typ), _ptr(X),
               _ptr(V), 0, _stream(stream))
        return X, V

    def radial_basis(self, x, y, z, q, typ=None, stream=None):
        """V_i^(m) for the radial terms m < nb: (nb, n, 4) float32."""
        Vb = torch.empty((self.nb, self.n, 4), dtype=torch.float32, device=x.device)
        N.call("pd_learned_descriptors", self.handle, _ptr(x), _ptr(y), _ptr(z), _ptr(q), _ptr(typ), 0, 0,
               _ptr(Vb), _stream(stream))
        return Vb

    def correction(self, net: MLPNetwork, x, y, z, q, typ=None, out=None, stream=None):
        """(n, 4) = (s V, s) through the descriptors and the network."""
        out = torch.empty((self.n, 4), dtype=torch.float32, device=x.device) if out is None else out
        N.call("pd_learned_correction", self.handle, net.handle, _ptr(x), _ptr(y), _ptr(z), _ptr(q), _ptr(typ),
               _ptr(out), _stream(stream))
        return out

    def status(self) -> dict:
        st = N.EllStats()
        N.call("pd_learned_status", self.handle, C.byref(st))
        return {k: getattr(st, k) for k, _ in N.EllStats._fields_}

    def resize(self, cap: int):
        N.call("pd_learned_resize", self.handle, int(cap))
        self.params.cap = int(cap)


def fit_radial(Vb: torch.Tensor, R: torch.Tensor, ridge: float = 1e-9) -> np.ndarray:
    """Least-squares coefficients c of R_i ~ sum_m c_m V_i^(m) (FP64 normal equations, ridge-stabilised).

    ``Vb`` may stack several snapshots along its particle axis: (nb, rows, 4); ``R`` is (rows, 3)."""
    B = Vb[..., :3].double()
    A = torch.einsum("mrc,lrc->ml", B, B)
    b = torch.einsum("mrc,rc->m", B, R.double())
    A = A + ridge * torch.trace(A) / A.shape[0] * torch.eye(A.shape[0], dtype=A.dtype, device=A.device)
    return torch.linalg.solve(A, b).cpu().numpy()


def ewald_oracle(rq4: torch.Tensor, box, coulomb: float, alpha: float, digits: float = 12.0, parts: int = 7):
    """FP64 Ewald sum on the GPU: (F (n, 3) float64 on the device, E).  rq4 = (n, 4) float64 (x, y, z, q)."""
    if rq4.dtype != torch.float64 or rq4.shape[1:] != (4,) or not rq4.is_contiguous():
        raise ValueError("rq4 must be a contiguous (n, 4) float64 tensor")
    n = rq4.shape[0]
    F = torch.empty((n, 3), dtype=torch.float64, device=rq4.device)
    e = C.c_double()
    N.call("pd_ewald_oracle", int(n), _ptr(rq4), N.dbl3(box), float(coulomb), float(alpha), float(digits), int(parts),
           _ptr(F), C.byref(e))
    return F, e.value


def rms_error(F, Fref) -> float:
    """Relative RMS force error |F - Fref|_rms / |Fref|_rms over all components."""
    d = (F.double() - Fref.double())
    return float(torch.sqrt((d * d).sum() / (Fref.double() ** 2).sum()))


class CoarseMeshTrainer:
    """Training data, fit and training of the learned correction for one charged system.

    ``q`` and ``typ`` are the particles' charges and 1-based type ids (device tensors); ``spec`` is
    the fine-mesh electrostatics spec; the coarse mesh has ``coarse_spacing`` and ``coarse_order``.
    """

    def __init__(self, n, box, q, typ, spec: ElectrostaticsSpec, *, coarse_spacing=2.0, coarse_order=4, seed=0,
                 self_force_table: int = 16, correction: LearnedCorrection | None = None,
                 net: MLPNetwork | None = None, **desc):
        self.n = int(n)
        self.box = tuple(float(b) for b in box)
        self.q, self.typ = q, typ
        self.spec = spec
        qh = q.double().cpu().numpy()
        self.fine = ElectrostaticsSolver(spec, self.box, qh, nmax=self.n)
        cspec = ElectrostaticsSpec(coulomb_prefactor=spec.coulomb_prefactor, real_cutoff=spec.real_cutoff,
                                   alpha=spec.alpha, influence=spec.influence, order=int(coarse_order),
                                   mesh_spacing=float(coarse_spacing), alias_order=spec.alias_order,
                                   relative_permittivity=spec.relative_permittivity, net_charge=spec.net_charge,
                                   real_space_modifier=spec.real_space_modifier)
        self.coarse_spec = cspec
        self.coarse = ElectrostaticsSolver(cspec, self.box, qh, nmax=self.n)
        # the coarse mesh's spurious self force is known exactly (a function of each ion's position
        # relative to the nodes): it is removed before anything is learned
        self.self_force_table = int(self_force_table)
        if self.self_force_table:
            self.coarse.set_self_force_removal(self.self_force_table)
        self.corr = correction if correction is not None else LearnedCorrection(self.n, self.box, **desc)
        self.net = net if net is not None else MLPNetwork(seed=seed)
        self.snap_pos = []      # centred coordinates (3, n) float32 per snapshot
        self.snap_res = []      # residual targets (n, 3) float32
        self.X = None
        self.ab = None
        self.rr = None          # sum |R|^2 per snapshot (constant part of the loss)
        self.history = []

    def mesh_forces(self, solver, x, y, z):
        f = [torch.empty(self.n, dtype=torch.float32, device=x.device) for _ in range(3)]
        solver.transform(x, y, z, self.q)
        solver.gather(x, y, z, self.q, f[0], f[1], f[2], set=True)
        return torch.stack(f, 1)

    def residual(self, x, y, z):
        return self.mesh_forces(self.fine, x, y, z) - self.mesh_forces(self.coarse, x, y, z)

    def add_snapshot(self, x, y, z):
        self.snap_pos.append(torch.stack([x, y, z]).clone())
        self.snap_res.append(self.residual(x, y, z))

    def fit_radial(self, max_snapshots: int = 16) -> np.ndarray:
        k = min(max_snapshots, len(self.snap_pos))
        Vb = torch.cat([self.corr.radial_basis(*self.snap_pos[i], self.q, self.typ) for i in range(k)], 1)
        R = torch.cat(self.snap_res[:k], 0)
        coef = fit_radial(Vb, R)
        self.corr.set_radial(coef)
        return coef

    def build_dataset(self):
        """Descriptors X (rows, 32) bf16 and loss coefficients ab = (|V|^2, V . R) of every snapshot."""
        S, n = len(self.snap_pos), self.n
        dev = self.q.device
        self.X = torch.empty((S * n, N_IN), dtype=torch.bfloat16, device=dev)
        self.ab = torch.empty((S * n, 2), dtype=torch.float32, device=dev)
        self.rr = torch.empty(S, dtype=torch.float64, device=dev)
        V = torch.empty((n, 4), dtype=torch.float32, device=dev)
        for k in range(S):
            x, y, z = self.snap_pos[k]
            self.corr.descriptors(x, y, z, self.q, self.typ, X=self.X[k * n:(k + 1) * n], V=V)
            R = self.snap_res[k]
            v = V[:, :3]
            self.ab[k * n:(k + 1) * n, 0] = (v * v).sum(1)
            self.ab[k * n:(k + 1) * n, 1] = (v * R).sum(1)
            self.rr[k] = (R.double() ** 2).sum()
        st = self.corr.status()
        if st["error"]:
            raise RuntimeError(f"descriptor rows overflowed their capacity (status {st})")

    def train(self, epochs: int = 4, lr: float = 1e-3, batch_snapshots: int = 1, seed: int = 0, lr_decay=0.5):
        """Adam over shuffled snapshot batches; returns the mean loss (MSE per component) of each epoch."""
        S, n = len(self.snap_pos), self.n
        rng = np.random.default_rng(seed)
        out = []
        for ep in range(epochs):
            order = rng.permutation(S)
            self.net.loss(reset=True)
            lre = lr * (lr_decay ** ep if lr_decay else 1.0)
            for b0 in range(0, S, batch_snapshots):
                ks = order[b0:b0 + batch_snapshots]
                if len(ks) == 1:
                    k = int(ks[0])
                    X, ab = self.X[k * n:(k + 1) * n], self.ab[k * n:(k + 1) * n]
                else:
                    idx = torch.cat([torch.arange(int(k) * n, (int(k) + 1) * n, device=self.X.device) for k in ks])
                    X, ab = self.X[idx].contiguous(), self.ab[idx].contiguous()
                rows = X.shape[0]
                self.net.train_batch(X, ab, scale=2.0 / (3 * rows))
                self.net.adam(lr=lre)
            # the kernel adds sum (s^2 a - 2 s b) / (3 rows) per batch; the constant |R|^2 part completes
            # the mean squared error per force component
            nbatch = (S + batch_snapshots - 1) // batch_snapshots
            tot = self.net.loss(reset=True) / nbatch + float(self.rr.sum()) / (3.0 * n * S)
            out.append(tot)
            self.history.append(tot)
        if self.net.error():
            raise RuntimeError("a tensor-core wait timed out during training")
        return out

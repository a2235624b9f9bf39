"""Workflow API over the device engines.

Mirrors the reference's public force/integrator/simulation API
(src/workflow/Forces.jl:33-118, src/workflow/Electrostatics.jl:44-99,
src/workflow/RunLoop.jl:403-457): force descriptors ``LennardJones``, ``WCA``,
``PME``, ``PPPM``; list policies ``ClusterPairList`` and ``CellList``;
``Integrator``, ``Stage``, ``ParticleSystem``, ``Simulation`` and the
``run`` / ``step`` / ``evaluate_forces_into_f`` calls (``run!``, ``step!`` and
``evaluate_forces_into_f!`` in Julia).  Every force evaluation and step runs on
the GPU through libpdb200; there is no CPU path.

Routes follow the reference's user rules: charged systems run on the
cluster-pair backend (src/simulation/ElectrostaticsCoupling.jl:76-86), as do
LJ/WCA forces that ask for a ``ClusterPairList``; LJ/WCA forces with a
``CellList`` (the default) run on the ELL route (cell list + neighbour rows,
2D or 3D).  ``ConstantVolume`` integrates NVE; ``Langevin`` integrates BAOAB
(ELL route).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import prolates, splits
from .engine import (ClusterPairEngine, DeviceEngine, ELLDeviceEngine, ELLEngine, ElectrostaticsSolver,
                     ElectrostaticsSpec)


# ----------------------------------------------------------------------------- descriptors

@dataclass
class CellList:
    """Neighbor-list policy (Forces.jl:33-44): list buffer (skin), row capacity, rebuild interval."""
    buffer: float = 0.4
    capacity: int = 96
    rebuild_interval: int = 20


@dataclass
class ClusterPairList:
    """Cluster-pair traversal (Forces.jl:46-57): list radius = cutoff + buffer, pruned to cutoff + prune_buffer."""
    buffer: float = 0.1
    prune_buffer: float | None = None


@dataclass
class LennardJones:
    """Lennard-Jones force (Forces.jl:84-93); vdw_modifier 'none' truncates, 'potential_shift' shifts."""
    epsilon: float | None = None
    sigma: float | None = None
    cutoff: float | None = None
    pairs: str = "all"
    mode: str = "standard"
    pair_table: object = None
    neighborlist: object = None
    vdw_modifier: str = "none"


@dataclass
class WCA:
    """Weeks-Chandler-Andersen force (Forces.jl:100-108): LJ cut at 2^(1/6) sigma, shifted by +epsilon."""
    epsilon: float | None = None
    sigma: float | None = None
    cutoff: float | None = None
    pairs: str = "all"
    mode: str = "standard"
    pair_table: object = None
    neighborlist: object = None


@dataclass
class PME:
    """Smooth particle-mesh Ewald with analytic differentiation (Electrostatics.jl:44-61)."""
    coulomb_prefactor: float | None = None
    real_cutoff: float | None = None
    alpha: float | None = None
    real_space_tolerance: float | None = None
    mesh: tuple | None = None
    mesh_spacing: float | None = None
    order: int = 4
    relative_permittivity: float = 1.0
    net_charge: str = "error"
    boundary: str = "tin_foil"
    real_space_modifier: str = "none"
    exclusions: object = "topology"
    exclude_bonded: bool = False
    scaled_pairs: tuple = ()
    pairs: str = "neighborlist"
    neighborlist: object = None


@dataclass
class PPPM:
    """P3M with the optimal influence function, AD or ik differentiation (Electrostatics.jl:79-99)."""
    coulomb_prefactor: float | None = None
    real_cutoff: float | None = None
    alpha: float | None = None
    real_space_tolerance: float | None = None
    mesh: tuple | None = None
    mesh_spacing: float | None = None
    order: int = 5
    differentiation: str = "ad"
    alias_order: int = 2
    relative_permittivity: float = 1.0
    net_charge: str = "error"
    boundary: str = "tin_foil"
    real_space_modifier: str = "none"
    exclusions: object = "topology"
    exclude_bonded: bool = False
    scaled_pairs: tuple = ()
    pairs: str = "neighborlist"
    neighborlist: object = None


@dataclass
class ESP:
    """Ewald summation with prolates (Electrostatics.jl:101-155): the prolate split and a prolate window
    of width ``order`` grid points.  Defaults follow the selection rules for a target relative force
    error ``tolerance``: split shape c with psi(1) = tolerance, window shape from tolerance / 2 (the
    smallest larger shape an FP32 mesh resolves, where that one is not), width from the table
    (5, 5, 6, 7, 8 for 1e-3, 5e-4, 1e-4, 5e-5, 1e-5) and mesh spacing pi r_c / c."""
    coulomb_prefactor: float | None = None
    real_cutoff: float | None = None
    tolerance: float | None = 1e-4
    split_shape: float | None = None
    window_shape: float | None = None
    order: int | None = None
    influence: str = "optimal"
    alias_order: int = 2
    mesh: tuple | None = None
    mesh_spacing: float | None = None
    relative_permittivity: float = 1.0
    net_charge: str = "error"
    boundary: str = "tin_foil"
    real_space_modifier: str = "none"
    exclusions: object = "topology"
    exclude_bonded: bool = False
    scaled_pairs: tuple = ()
    pairs: str = "neighborlist"
    neighborlist: object = None


def _esp_spec(f: ESP) -> ElectrostaticsSpec:
    """electrostatics_spec(::ESP, Float32) (src/workflow/Electrostatics.jl:253-272)."""
    if f.split_shape is None or f.window_shape is None or f.order is None:
        if f.tolerance is None:
            raise ValueError("ESP needs `tolerance`, or explicit `split_shape`, `window_shape` and `order`.")
    eps = None if f.tolerance is None else float(f.tolerance)
    rc = float(f.real_cutoff)
    c = prolates.prolate_shape_for_tolerance(eps) if f.split_shape is None else float(f.split_shape)
    P = prolates.esp_order_for_tolerance(eps) if f.order is None else int(f.order)
    c1 = prolates.esp_window_shape(eps, P, np.float32) if f.window_shape is None else float(f.window_shape)
    spacing = math.pi * rc / c if (f.mesh is None and f.mesh_spacing is None) else f.mesh_spacing
    if f.influence not in ("optimal", "deconvolution"):
        raise ValueError(f"ESP influence must be optimal or deconvolution; got {f.influence}.")
    return ElectrostaticsSpec(coulomb_prefactor=float(f.coulomb_prefactor), real_cutoff=rc,
                              influence="esp" if f.influence == "optimal" else "esp_deconvolution", order=P,
                              mesh=f.mesh, mesh_spacing=spacing, alias_order=f.alias_order,
                              relative_permittivity=float(f.relative_permittivity), net_charge=f.net_charge,
                              real_space_modifier=f.real_space_modifier, split_shape=c, window_shape=c1)


def electrostatics_spec(f) -> ElectrostaticsSpec:
    """Validated solver spec of a PME, PPPM or ESP descriptor."""
    if f.coulomb_prefactor is None or f.real_cutoff is None:
        raise ValueError(f"{type(f).__name__} requires coulomb_prefactor and real_cutoff.")
    if f.boundary != "tin_foil":
        raise ValueError(f"Only conducting (tin-foil) boundary conditions are implemented; got {f.boundary}.")
    if isinstance(f, ESP):
        return _esp_spec(f)
    if (f.alpha is None) == (f.real_space_tolerance is None):
        raise ValueError("Provide exactly one of alpha and real_space_tolerance.")
    alpha = float(f.alpha) if f.alpha is not None else splits.alpha_from_tolerance(f.real_cutoff,
                                                                                    f.real_space_tolerance)
    if isinstance(f, PME):
        influence = "spme"
        alias = 2
    else:
        if f.differentiation not in ("ad", "ik"):
            raise ValueError("differentiation must be ad or ik.")
        influence = "p3m_ad" if f.differentiation == "ad" else "p3m_ik"
        alias = f.alias_order
    return ElectrostaticsSpec(coulomb_prefactor=float(f.coulomb_prefactor), real_cutoff=float(f.real_cutoff),
                              alpha=alpha, influence=influence, order=int(f.order), mesh=f.mesh,
                              mesh_spacing=f.mesh_spacing, alias_order=alias,
                              relative_permittivity=float(f.relative_permittivity), net_charge=f.net_charge,
                              real_space_modifier=f.real_space_modifier)


@dataclass
class ConstantVolume:
    """NVE velocity Verlet on a group (the whole system) (src/workflow/Integrator.jl:45-55)."""
    group: object = None
    thermostat: object = None


@dataclass
class Langevin:
    """Langevin method on a group (the whole system) with friction gamma and bath temperature kT
    (src/workflow/Integrator.jl:57-66), integrated by BAOAB, or by GJF under the VelocityVerlet scheme."""
    group: object = None
    gamma: float = 1.0
    kT: float = 1.0


class VelocityVerlet:
    """Velocity-Verlet stepping scheme (Integrator.jl:6-7)."""


class BAOAB:
    """BAOAB Langevin splitting (Integrator.jl:8-9)."""


class BAOA:
    """BAOA Langevin splitting, no trailing half kick (Integrator.jl:10-11)."""


@dataclass
class Integrator:
    dt: float
    forces: list = field(default_factory=list)
    methods: list = field(default_factory=lambda: [ConstantVolume()])
    scheme: object = None


@dataclass
class GSDWriter:
    """Scheduled GSD trajectory writer (src/workflow/Writers.jl:50-90): a frame every ``every`` steps
    (and at the stage start with ``write_start``); ``mode`` "replace" starts a new file, "append" (or
    ``append=True``) continues an existing one.  ``types`` and ``diameter`` "automatic" take the
    system's type names and the element covalent diameters.  Frames are packed and copied on the
    device after their steps and written to the file while the next steps run."""
    filename: str
    every: int | None = None
    schedule: object = None
    group: object = None
    write_start: bool = True
    mode: str = "replace"
    append: bool = False
    types: object = "automatic"
    diameter: object = "automatic"
    write_unwrapped: bool = False
    sync_on_write: bool = True
    write_forces: bool = False
    write_virial: bool = False
    observables: list = field(default_factory=list)

    def __post_init__(self):
        if self.mode not in ("replace", "append"):
            raise ValueError(f"GSDWriter mode must be replace or append; got {self.mode}")
        if self.every is not None and int(self.every) <= 0:
            raise ValueError("GSDWriter every must be positive")
        if self.schedule is not None:
            raise NotImplementedError("GSDWriter schedules other than `every` are not part of this build")
        if self.group is not None:
            raise NotImplementedError("GSDWriter groups other than the whole system are not part of this build")
        if self.write_unwrapped:
            raise ValueError("GSDWriter(write_unwrapped=true) requires unwrapped position buffers, which this "
                             "build's state does not keep")


@dataclass
class Stage:
    """A run stage (RunLoop.jl): name, steps, and how often energies are evaluated (0 = last step only)."""
    name: str = "run"
    steps: int = 0
    energy_every: int = 0
    progress: bool = False


def _pair_tuples(values, label):
    """_normalize_pair_tuples (src/workflow/System.jl:39-50): 1-based (i, j) pairs."""
    out = []
    for item in values:
        if len(item) != 2:
            raise ValueError(f"Each {label} entry must have length 2.")
        i, j = int(item[0]), int(item[1])
        if i <= 0 or j <= 0:
            raise ValueError(f"{label} indices must be positive.")
        out.append((i, j))
    return out


@dataclass
class Topology:
    """Bonds and exclusions of a system (Topology, src/workflow/System.jl:89-150), 1-based particle ids.

    The nonbonded path uses ``bonds`` (with ``exclude_bonded``) and ``exclusions`` (the default
    ``exclusions="topology"`` of the electrostatics descriptors); bonded force terms are not part of it."""
    bonds: list = field(default_factory=list)
    exclusions: list = field(default_factory=list)

    def __post_init__(self):
        self.bonds = _pair_tuples(self.bonds, "bond")
        self.exclusions = _pair_tuples(self.exclusions, "exclusion")


def electrostatic_exceptions(system, f) -> list:
    """Exception list implied by a descriptor's ``exclusions``, ``exclude_bonded`` and ``scaled_pairs``
    (electrostatic_exceptions, src/workflow/Electrostatics.jl:281-306): sorted 1-based (i, j, scale)."""
    scales = {}

    def key(i, j):
        i, j = int(i), int(j)
        return (i, j) if i < j else (j, i)

    topo = getattr(system, "topology", None) or Topology()
    excl = f.exclusions
    if isinstance(excl, str) and excl == "topology":
        for i, j in topo.exclusions:
            scales[key(i, j)] = 0.0
    elif excl is None or (isinstance(excl, str) and excl == "none"):
        pass
    else:
        for item in excl:
            scales[key(item[0], item[1])] = 0.0
    if f.exclude_bonded:
        for i, j in topo.bonds:
            scales[key(i, j)] = 0.0
    for item in f.scaled_pairs:
        if len(item) != 3:
            raise ValueError("scaled_pairs entries must be (i, j, scale).")
        scales[key(item[0], item[1])] = float(item[2])
    return [(k[0], k[1], s) for k, s in sorted(scales.items())]


class ParticleSystem:
    """Positions (N x D, D = 2 or 3 from the box), box, types, per-type masses and charges (host data),
    and an optional :class:`Topology`."""

    def __init__(self, positions, box, types=("A",), typeids=None, masses=None, charges=None, velocities=None,
                 topology=None):
        self.topology = topology if topology is not None else Topology()
        self.box = tuple(float(b) for b in box)
        if len(self.box) not in (2, 3):
            raise ValueError("periodic boxes are 2D or 3D")
        self.dim = len(self.box)
        self.positions = np.asarray(positions, float).reshape(-1, self.dim)
        n = len(self.positions)
        self.types = [str(t) for t in types]
        self.typeids = np.ones(n, np.int32) if typeids is None else np.asarray(typeids, np.int32)

        def per_particle(v, default):
            if v is None:
                return np.full(n, default, float)
            if isinstance(v, dict):
                return np.array([float(v[self.types[t - 1]]) for t in self.typeids])
            a = np.asarray(v, float)
            return np.full(n, float(a)) if a.ndim == 0 else a.reshape(n)

        self.masses = per_particle(masses, 1.0)
        self.charges = None if charges is None else per_particle(charges, 0.0)
        self.velocities = None if velocities is None else np.asarray(velocities, float).reshape(n, self.dim)

    @property
    def n(self) -> int:
        return len(self.positions)

    @staticmethod
    def from_gsd(path, frame: int = -1) -> "ParticleSystem":
        """ParticleSystem.from_gsd(path; frame=-1) (src/workflow/System.jl:455-531): positions, box, types,
        type ids, masses, charges, velocities and bonds of a GSD frame (-1 = the last)."""
        from .gsdio import read_gsd_frame

        fr = read_gsd_frame(path) if frame == -1 else read_gsd_frame(path, step=frame)
        cols = [fr.rx, fr.ry] + ([fr.rz] if fr.D == 3 else [])
        vcols = [fr.vx, fr.vy] + ([fr.vz] if fr.D == 3 else [])
        props = fr.particle_properties
        bonds = [tuple(int(v) for v in t) for t in fr.topology.bonds["tuples"]] if fr.topology else []
        system = ParticleSystem(np.stack(cols, 1).astype(float), fr.box, types=fr.types, typeids=fr.typeid,
                                masses=props.get("mass"), charges=props.get("charge"),
                                velocities=np.stack(vcols, 1).astype(float), topology=Topology(bonds=bonds))
        system.metadata = dict(step=fr.step, source_path=str(path), particle_properties=props,
                               per_type_properties=fr.per_type_properties)
        if "diameter" in props:
            system.metadata["diameters"] = props["diameter"]
        return system


# ----------------------------------------------------------------------------- state

class SimulationState:
    """Device state of one system and its engines (the SimulationState of the reference)."""

    def __init__(self, system: ParticleSystem, forces, dt: float, device="cuda", methods=None, seed: int = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("libpdb200 needs a CUDA device; there is no CPU force path")
        self.dev = torch.device(device)
        n = system.n
        self.n = n
        self.dim = system.dim
        self.box = system.box
        f32 = dict(dtype=torch.float32, device=self.dev)
        L = np.array(self.box)
        D = self.dim
        pos = system.positions - L * np.floor(system.positions / L + 0.5)   # centred image
        # positions and velocities as the rows of one (2D, n) block, so that host transfers of a whole
        # state are single copies
        v = system.velocities if system.velocities is not None else np.zeros((n, D))
        self._xv = torch.tensor(np.ascontiguousarray(np.concatenate([pos.T, np.asarray(v, float).T])), **f32)
        comp = [self._xv[d] for d in range(D)] + [None] * (3 - D)
        self.x, self.y, self.z = comp
        comp = [self._xv[D + d] for d in range(D)] + [None] * (3 - D)
        self.vx, self.vy, self.vz = comp
        comp = [torch.zeros(n, **f32) for _ in range(D)] + [None] * (3 - D)
        self.fx, self.fy, self.fz = comp
        self.epot = torch.zeros(n, **f32)
        self.vir6 = torch.zeros((n, 6 if D == 3 else 3), **f32)
        self.langevin = None
        self.langevin_scheme = "baoab"
        for m in methods or []:
            if isinstance(m, Langevin):
                if float(m.gamma) <= 0:
                    raise ValueError("Langevin gamma must be positive")
                self.langevin = (float(m.gamma), float(m.kT))
            elif not isinstance(m, ConstantVolume):
                raise NotImplementedError(f"integration method {type(m).__name__} is not part of this build")
        self.seed = int(seed)
        self.vglobal = torch.zeros(6, **f32)
        self.q = torch.tensor(system.charges, **f32) if system.charges is not None else None
        self.typ = torch.tensor(system.typeids, dtype=torch.int32, device=self.dev)
        self.inv_mass = torch.tensor(1.0 / system.masses, **f32)
        self.masses = system.masses
        self.dt = float(dt)
        self.step_count = 0
        self.stream = torch.cuda.Stream(device=self.dev)
        self._compile(system, forces)

    def _compile(self, system, forces):
        vdw = [f for f in forces if isinstance(f, (LennardJones, WCA))]
        elec = [f for f in forces if isinstance(f, (PME, PPPM, ESP))]
        if len(vdw) > 1 or len(elec) > 1:
            raise ValueError("at most one short-range vdW force and one electrostatics force")
        self.ell = None
        if vdw and not elec and not isinstance(vdw[0].neighborlist, ClusterPairList):
            self._compile_ell(vdw[0])
            return
        if self.dim != 3:
            raise ValueError("the cluster-pair backend needs a 3D box")
        if self.langevin is not None:
            raise NotImplementedError("Langevin runs on the CellList (ELL) route in this build")
        lj = None
        rlj = 0.0
        nl = None
        if vdw:
            f = vdw[0]
            if f.mode != "standard":
                raise ValueError(f"Only mode=standard is supported for {type(f).__name__}.")
            if f.epsilon is None or f.sigma is None:
                raise ValueError(f"{type(f).__name__} requires epsilon and sigma.")
            eps, sig = float(f.epsilon), float(f.sigma)
            if isinstance(f, WCA):
                rc = sig * splits.WCA_RC_FACTOR if f.cutoff is None else float(f.cutoff)
                table = splits.lj_type_table(sig, eps, rc, wca=True)
            else:
                if f.cutoff is None:
                    raise ValueError("LennardJones requires an explicit cutoff.")
                rc = float(f.cutoff)
                table = splits.lj_type_table(sig, eps, rc, shift=f.vdw_modifier == "potential_shift")
            lj = dict(table=table)
            rlj = rc
            nl = f.neighborlist
        self.solver = None
        coul = None
        selfc = 0.0
        rcoul = 0.0
        if elec:
            if self.q is None:
                raise ValueError("electrostatics requires per-particle charges")
            spec = electrostatics_spec(elec[0])
            self.solver = ElectrostaticsSolver(spec, self.box, system.charges, nmax=self.n)
            coul = self.solver.coulomb_polynomial()
            selfc = self.solver.selfc
            rcoul = spec.real_cutoff
            if nl is None:
                nl = elec[0].neighborlist
        rmax = max(rlj, rcoul)
        if rmax <= 0:
            raise ValueError("The cluster-pair backend needs a vdW term or an electrostatics solver.")
        if isinstance(nl, ClusterPairList):
            skin = nl.buffer
            pb = nl.prune_buffer if nl.prune_buffer is not None else 0.5 * skin
        else:
            skin = (nl.buffer if isinstance(nl, CellList) else CellList().buffer)
            pb = 0.5 * skin
        # small boxes: the list radius stays below half the box (_charged_backend!, ElectrostaticsCoupling.jl:76-86)
        skin = min(skin, max(0.999 * (min(self.box) / 2 - rmax), 0.0))
        pb = min(pb, skin)
        self.cluster = ClusterPairEngine(self.n, self.box, rmax=rmax, skin=skin, prune_buffer=pb, lj=lj,
                                         coulomb=coul, selfc=selfc)
        self.exceptions = electrostatic_exceptions(system, elec[0]) if elec else []
        if self.exceptions:
            # build-time ids are 1-based; the engine takes storage indices (the same order here)
            self.cluster.set_exceptions([(i - 1, j - 1, s) for i, j, s in self.exceptions])
        state = dict(x=self.x, y=self.y, z=self.z, vx=self.vx, vy=self.vy, vz=self.vz, fx=self.fx, fy=self.fy,
                     fz=self.fz, q=self.q if coul is not None else None, type=self.typ, inv_mass=self.inv_mass,
                     epot=self.epot, vir6=self.vir6, vglobal=self.vglobal)
        self.engine = DeviceEngine(self.cluster, self.solver, state, self.box)
        self.forces_valid = False

    def _compile_ell(self, f):
        """The ELL route: cell list + rows with the CellList policy (Forces.jl:255-283)."""
        if f.mode != "standard":
            raise ValueError(f"Only mode=standard is supported for {type(f).__name__}.")
        if f.pair_table is not None:
            raise NotImplementedError("type-dependent pair tables run on the cluster-pair route in this build")
        if f.epsilon is None or f.sigma is None:
            raise ValueError(f"{type(f).__name__} requires epsilon and sigma.")
        nl = f.neighborlist if isinstance(f.neighborlist, CellList) else CellList()
        if f.neighborlist is not None and not isinstance(f.neighborlist, CellList):
            raise ValueError(f"Neighbor specification must be CellList or ClusterPairList; got {type(f.neighborlist).__name__}.")
        if nl.capacity <= 0:
            raise ValueError("CellList capacity must be positive.")
        if nl.buffer < 0:
            raise ValueError("CellList buffer must be nonnegative.")
        if nl.rebuild_interval <= 0:
            raise ValueError("CellList rebuild_interval must be positive.")
        if isinstance(f, WCA):
            model, cutoff, shift = "wca", (None if f.cutoff is None else float(f.cutoff)), False
        else:
            if f.cutoff is None:
                raise ValueError("LennardJones requires an explicit cutoff.")
            model, cutoff, shift = "lj", float(f.cutoff), f.vdw_modifier == "potential_shift"
        self.solver = None
        self.cluster = None
        self.ell = ELLEngine(self.n, self.box, dim=self.dim, model=model, epsilon=f.epsilon, sigma=f.sigma,
                             cutoff=cutoff, skin=nl.buffer, capacity=nl.capacity,
                             interval=min(max(int(nl.rebuild_interval), 1), 100), shift=shift)
        state = dict(x=self.x, y=self.y, z=self.z, vx=self.vx, vy=self.vy, vz=self.vz, fx=self.fx, fy=self.fy,
                     fz=self.fz, inv_mass=self.inv_mass, epot=self.epot, vir=self.vir6)
        self.engine = ELLDeviceEngine(self.ell, state)
        self.forces_valid = False

    def _ell_check(self):
        st = self.ell.status()
        if st["error"] == 1:
            raise RuntimeError(f"Neighbor capacity {st['cap']} exceeded: a row needs {st['required']} entries; "
                               "raise CellList capacity")
        if st["error"] == 2:
            raise ValueError("Device ELL requires finite, centered coordinates; execution stopped before "
                             "rebuilding/forces")
        return st

    # -- force evaluation
    def evaluate_forces_into_f(self, energy: bool = False):
        """evaluate_forces_into_f!(st, energy) (ForceEvaluation.jl:40-44)."""
        with torch.cuda.stream(self.stream):
            if self.solver is None:
                self.vglobal.zero_()
            self.engine.evaluate(energy=energy, stream=self.stream)
            if self.ell is not None:
                self.stream.synchronize()
                st = self.ell.status()
                if st["error"] == 1:
                    # capacity recovery at a host boundary: larger rows, rebuild, evaluate again
                    self.ell.resize(max(int(st["required"] * 1.25) + 8, st["cap"] + 8))
                    self.engine.evaluate(energy=energy, stream=self.stream)
        self.stream.synchronize()
        if self.ell is not None:
            self._ell_check()
        self.forces_valid = True

    def step(self, nsteps: int = 1, energy_last: bool = False, use_graph: bool = True):
        if not self.forces_valid:
            self.evaluate_forces_into_f(False)
        if self.langevin is not None:
            self.engine.langevin(nsteps, self.dt, self.langevin[0], self.langevin[1], self.seed,
                                 energy_last=energy_last, use_graph=use_graph, stream=self.stream,
                                 scheme=self.langevin_scheme)
        else:
            self.engine.step(nsteps, self.dt, energy_last=energy_last, use_graph=use_graph, stream=self.stream)
        self.step_count += nsteps

    def synchronize(self):
        self.stream.synchronize()

    # -- observables (FP64 host reductions)
    def potential_energy(self) -> float:
        self.synchronize()
        return float(self.epot.double().sum())

    def _comps(self, a, b, c):
        return [a, b] + ([c] if self.dim == 3 else [])

    def kinetic_energy(self) -> float:
        self.synchronize()
        v2 = sum(t.double() ** 2 for t in self._comps(self.vx, self.vy, self.vz)).cpu().numpy()
        return 0.5 * float((self.masses * v2).sum())

    def virial_tensor(self) -> dict:
        """Pair virial rows plus the mesh virial (xx, yy, zz, xy, xz, yz; 2D: xx, yy, xy)."""
        self.synchronize()
        if self.dim == 2:
            return dict(zip(("xx", "yy", "xy"), self.vir6.double().sum(0).cpu().numpy()))
        w = self.vir6.double().sum(0).cpu().numpy() + self.vglobal.double().cpu().numpy()
        return dict(zip(("xx", "yy", "zz", "xy", "xz", "yz"), w))

    def forces(self) -> np.ndarray:
        self.synchronize()
        return torch.stack(self._comps(self.fx, self.fy, self.fz), 1).double().cpu().numpy()

    def velocities(self) -> np.ndarray:
        self.synchronize()
        return torch.stack(self._comps(self.vx, self.vy, self.vz), 1).double().cpu().numpy()

    def positions(self) -> np.ndarray:
        self.synchronize()
        return torch.stack(self._comps(self.x, self.y, self.z), 1).double().cpu().numpy()


class Simulation:
    """System + integrator on one GPU (the reference's Simulation, src/workflow)."""

    def __init__(self, system: ParticleSystem, integrator: Integrator, precision="f32", seed: int = 0,
                 writers=()):
        if precision not in ("f32", np.float32, "Float32"):
            raise ValueError("this build runs the Float32 force path")
        if len(integrator.methods) != 1:
            raise NotImplementedError("one integration method covering the whole system")
        m = integrator.methods[0]
        if isinstance(m, ConstantVolume) and m.thermostat is not None:
            raise NotImplementedError("thermostats other than Langevin are not part of this build")
        sch = integrator.scheme
        vv = sch is VelocityVerlet or isinstance(sch, VelocityVerlet)
        baoa = sch is BAOA or isinstance(sch, BAOA)
        if isinstance(m, Langevin) and not (sch is None or sch is BAOAB or isinstance(sch, BAOAB) or vv or baoa):
            raise NotImplementedError("Langevin integrates with the BAOAB, BAOA or velocity-Verlet (GJF) scheme")
        self.system = system
        self.integrator = integrator
        self.seed = seed
        self.state = SimulationState(system, integrator.forces, integrator.dt, methods=integrator.methods, seed=seed)
        # Langevin under the velocity-Verlet scheme is the Grønbech-Jensen-Farago integrator
        # (the reference's Langevin/GJF `velocityverlet` path, IntegratorSpecs.jl:158)
        self.state.langevin_scheme = "gjf" if vv else ("baoa" if baoa else "baoab")
        self.writers = list(writers)
        for w in self.writers:
            if not isinstance(w, GSDWriter):
                raise NotImplementedError(f"writer {type(w).__name__} is not part of this build")
        self._gsd = {}       # writer index -> (GSDFile, FrameStager, pending slot, pending step)
        self._opened = set()

    def _writer_handle(self, k: int):
        from .gsdio import FrameStager, gsd_open

        if k not in self._gsd:
            w = self.writers[k]
            # a file this simulation has written before is continued by later runs
            append = w.append or w.mode == "append" or w.filename in self._opened
            h = gsd_open(w.filename, append=append)
            self._opened.add(w.filename)
            stager = FrameStager(self.state, forces=w.write_forces, virial=w.write_virial)
            self._gsd[k] = [h, stager, None, None]
        return self._gsd[k]

    def _stage_frame(self, k: int):
        """Pack and copy the state's frame for writer k on the device; the previous pending frame of the
        writer is written to its file meanwhile."""
        rec = self._writer_handle(k)
        slot = rec[1].stage()
        self._write_pending(k)
        rec[2], rec[3] = slot, self.state.step_count

    def _write_pending(self, k: int):
        from .gsdio import write_gsd_frame

        rec = self._gsd.get(k)
        if rec is None or rec[2] is None:
            return
        w = self.writers[k]
        h, stager, slot, stp = rec
        types = self.system.types if w.types == "automatic" else list(w.types)
        diam = None if w.diameter == "automatic" else w.diameter
        write_gsd_frame(h, self.state, diameter=diam, types_names=types, step=int(stp),
                        write_forces=w.write_forces, write_virial=w.write_virial, sync_on_write=w.sync_on_write,
                        stager=stager, staged=slot, topology=self.system.topology)
        rec[2] = rec[3] = None

    def close_writers(self):
        """Write every pending frame and close the writers' files (a later run appends to them)."""
        for k in list(self._gsd):
            self._write_pending(k)
            self._gsd.pop(k)[0].close()


def state(sim: Simulation) -> SimulationState:
    return sim.state


def run(sim: Simulation, stage: Stage) -> Simulation:
    """run!(sim, stage) (RunLoop.jl:403-457): stage.steps steps on the device, with the writers' frames
    at the stage start (``write_start``) and every ``every`` steps of the running step count."""
    st = sim.state
    writers = getattr(sim, "writers", [])
    needs_forces = any(w.write_forces or w.write_virial for w in writers)
    if writers and needs_forces and not st.forces_valid:
        st.evaluate_forces_into_f(True)
    for k, w in enumerate(writers):
        if w.write_start:
            sim._stage_frame(k)
    if stage.steps > 0:
        every = stage.energy_every if stage.energy_every and stage.energy_every > 0 else 0
        marks = {stage.steps}
        if every:
            marks |= set(range(every, stage.steps, every))
        for w in writers:
            if w.every:
                e = int(w.every)
                first = e - st.step_count % e
                marks |= set(range(first, stage.steps + 1, e))
        done = 0
        base = st.step_count
        for m in sorted(marks):
            if m <= done:
                continue
            st.step(m - done, energy_last=True)
            done = m
            for k, w in enumerate(writers):
                if w.every and (base + done) % int(w.every) == 0:
                    sim._stage_frame(k)
    sim.close_writers()
    st.synchronize()
    return sim


def step(sim_or_state, compute_energy: bool = False):
    """step!(st, integ, dt; compute_energy) (SteppingEngine.jl:23)."""
    st = sim_or_state.state if isinstance(sim_or_state, Simulation) else sim_or_state
    st.step(1, energy_last=compute_energy)
    return st


def evaluate_forces_into_f(sim_or_state, energy: bool = False):
    st = sim_or_state.state if isinstance(sim_or_state, Simulation) else sim_or_state
    st.evaluate_forces_into_f(energy)
    return st

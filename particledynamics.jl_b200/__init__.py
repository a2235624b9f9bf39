"""B200 (sm_100a) implementation of ParticleDynamics.jl's per-step force hot path.

The compute path is libpdb200.so (CUDA, built in-tree by ``build.py``); this
package holds the host side above its C ABI: ctypes bindings, the FP64 setup
math, the engine objects and the workflow API.  Importing the package does
not require a GPU; creating an engine does, and there is no CPU fallback.
"""
from . import _native, batch, gsdio, learned, prolates, splits, synthetic  # noqa: F401
from .gsdio import (GSDFrameData, GSDTopology, electrostatics_from_gsd, electrostatics_from_settings,  # noqa: F401
                    exceptions_record, gsd_close, gsd_open, read_gsd_frame, read_gsd_log, settings_record,
                    write_gsd_frame)
from .engine import (ClusterPairEngine, DeviceEngine, ELLDeviceEngine, ELLEngine, ElectrostaticsSolver,  # noqa: F401
                     ElectrostaticsSpec)
from .workflow import (  # noqa: F401
    BAOA, BAOAB, ESP, PME, PPPM, WCA, CellList, ClusterPairList, ConstantVolume, GSDWriter, Integrator, Langevin,
    LennardJones,
    ParticleSystem, Simulation, SimulationState, Stage, Topology, VelocityVerlet, electrostatic_exceptions,
    electrostatics_spec, evaluate_forces_into_f, run, state, step,
)

__version__ = "0.1.0"


def build(force: bool = False):
    """Compile libpdb200.so for sm_100a (in-tree)."""
    from ._build import build as _b
    return _b(force=force)

"""B200-native BEADS: the per-step MD hot path on sm_100a behind the
reference's Python surface.

``System``, ``ForceField``, ``Dynamics`` and ``Simulation`` have the
reference's names, arguments and errors; ``Simulation.execute()`` runs on the
CUDA engine (``libbeads_b200.so``, C ABI in include/beads_b200.h) and writes
the reference's thermo CSV, trajectory, final-state and log files.
``beads_b200.engine.Engine`` is the in-process handle on a batch of replicas.
"""

from . import io
from .dynamics import Dynamics
from .forcefield import ForceField
from .simulation import Simulation
from .system import System

__version__ = "0.1.0"


def build_info() -> dict:
    """The engine's dtype configuration (the reference's beads.build_info)."""
    from . import _native

    return _native.build_info()


__all__ = ["Dynamics", "ForceField", "Simulation", "System", "__version__", "build_info", "io"]

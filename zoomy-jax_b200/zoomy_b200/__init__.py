"""zoomy_b200 -- B200-native drop-in for zoomy_jax's finite-volume time step.

Host side of the package: the reference's solver / mesh / model call shape
(``HyperbolicSolver``, ``MarchSolver`` and its blocks, ``create_2d``,
``timestepping.adaptive``), dispatching every compute step to libzb, the
sm_100a CUDA library declared in ``include/zb.h``.  Device memory and streams
come from PyTorch; nothing runs on the CPU.
"""
from . import timestepping  # noqa: F401
from .mesh import CartesianMesh, create_2d  # noqa: F401
from .trimesh import DeviceTriangleMesh, TriangleMesh, create_tri  # noqa: F401
from .model import (NumericalSystemModel, ReconstructionSpec,  # noqa: F401
                    ShallowWater2D)

__all__ = ["CartesianMesh", "TriangleMesh", "DeviceTriangleMesh", "create_2d", "create_tri", "NumericalSystemModel",
           "ReconstructionSpec", "ShallowWater2D", "timestepping"]

"""dt strategies with zoomy_core's ``timestepping`` call shape.

``adaptive(CFL, dimension)`` is the law the reference's tests pass to the
solver (``tests/conftest.py:285-295``):
``dt = min_f CFL 2 r_f / (d (2k+1) |lambda|_f)``, capped by ``dt_max``; a
wave-free face drops out.  ``constant(dt)`` is a fixed step.
"""
from __future__ import annotations

import math
from dataclasses import dataclass


@dataclass(frozen=True)
class Adaptive:
    CFL: float
    dimension: int = 2
    degree: int = 0
    dt_max: float = math.inf

    def with_dt_max(self, dt_max):
        """``apply_default_dt_max``: the explicit cap wins
        (``zoomy_jax/fvm/solver_jax.py:922-929``)."""
        if math.isfinite(self.dt_max) or dt_max is None:
            return self
        return Adaptive(self.CFL, self.dimension, self.degree, float(dt_max))


@dataclass(frozen=True)
class Constant:
    dt: float


def adaptive(CFL, dimension=2, degree=0, dt_max=None):
    if not (0.0 < CFL):
        raise ValueError("CFL must be positive")
    return Adaptive(float(CFL), int(dimension), int(degree),
                    math.inf if dt_max is None else float(dt_max))


def constant(dt):
    return Constant(float(dt))

"""The shallow-water model and its numerics, with the reference's call shape.

The reference derives SME(level=0) symbolically in zoomy_core (absent here):
state ``[b, h, q_x, q_y]``, flux ``(q.n, q (u.n) + g h^2 n / 2)``, bed term
``g h grad b``, eigenvalues ``u.n +- sqrt(g h)``, KP-desingularised ``hinv``
aux and the Manning friction closure (``tests/models.py:43-53``).  This module
states that model explicitly; ``NumericalSystemModel`` carries the numerics
(``ReconstructionSpec(order, limiter)`` and the Riemann solver) exactly as
``NumericalSystemModel.from_system_model(sm, reconstruction=..., riemann=...)``
does in the reference's tests.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

STATE = ("b", "h", "q_0", "q_1")
AUX = ("dq_0dx", "dhdx", "dq_1dy", "dhdy", "dbdx", "dbdy", "hinv")
RIEMANNS = ("rusanov", "rusanov_hr", "hll_hr")
LIMITERS = ("minmod", "barth_jespersen", "venkatakrishnan", "none")


@dataclass
class ShallowWater2D:
    """SME(level=0, dimension=3): 2-D horizontal shallow water."""
    g: float = 9.81
    manning_n: float = 0.0
    wet_dry_eps: float = 1e-8
    boundary_conditions: dict = field(default_factory=dict)
    initial_conditions: Optional[Callable] = None
    dt_max: Optional[float] = None
    state = STATE
    aux_state = AUX

    def bc_kinds(self):
        from .mesh import TAGS
        out = []
        for t in TAGS:
            k = self.boundary_conditions.get(t, "extrapolation")
            if k not in ("extrapolation", "wall", "periodic"):
                raise NotImplementedError(f"boundary condition {k!r} on {t}")
            out.append(k)
        if (out[0] == "periodic") != (out[1] == "periodic") or \
                (out[2] == "periodic") != (out[3] == "periodic"):
            raise ValueError("periodic boundaries come in left/right, bottom/top pairs")
        return out

    def initial_state(self, mesh):
        """Host ``(4, C)`` float64 initial state from ``initial_conditions``
        (a callable of the cell centre ``x (2,)`` returning the state, as the
        reference's ``IC.UserFunction``, or an array)."""
        ic = self.initial_conditions
        if ic is None:
            raise ValueError("the model has no initial_conditions")
        if callable(ic):
            xc = mesh.cell_centers()
            return np.stack([np.asarray(ic(xc[:, k]), dtype=np.float64)
                             for k in range(xc.shape[1])], axis=1)
        Q = np.asarray(ic, dtype=np.float64)
        if Q.shape != (4, mesh.n_cells):
            raise ValueError(f"initial state must be (4, {mesh.n_cells})")
        return Q


@dataclass(frozen=True)
class ReconstructionSpec:
    order: int = 1
    limiter: str = "minmod"


@dataclass
class NumericalSystemModel:
    model: ShallowWater2D
    reconstruction: ReconstructionSpec = ReconstructionSpec()
    riemann: str = "rusanov"

    @staticmethod
    def from_system_model(model, reconstruction=None, riemann=None):
        rs = reconstruction or ReconstructionSpec()
        rm = riemann or "rusanov"
        if rs.order not in (1, 2):
            raise NotImplementedError(f"reconstruction order {rs.order}")
        if rs.limiter not in LIMITERS:
            raise ValueError(f"unknown limiter {rs.limiter!r}")
        if rm not in RIEMANNS:
            raise NotImplementedError(f"riemann solver {rm!r}")
        return NumericalSystemModel(model, rs, rm)

    from_model = from_system_model

    @property
    def state(self):
        return STATE

    @property
    def aux_state(self):
        return AUX

    @property
    def dt_max(self):
        return self.model.dt_max

    @property
    def update_variables(self):
        return None

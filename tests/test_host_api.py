"""Host-side logic of the reference-facing API (no GPU needed)."""
import math

import numpy as np
import pytest

import zoomy_b200 as zb
from zoomy_b200 import _lib as L
from zoomy_b200.fvm.solver import HyperbolicSolver
from zoomy_b200.fvm.solver2 import (assert_dt_admissible, proceed, reduce_dt_clamp,
                                    should_write, MarchState)


def nsm(order=2, limiter="minmod", riemann="hll_hr", **model):
    return zb.NumericalSystemModel.from_system_model(
        zb.ShallowWater2D(**model), zb.ReconstructionSpec(order, limiter), riemann)


def test_create_2d_geometry():
    m = zb.create_2d((-1.0, 1.0, -1.0, 1.0), 32, 16)
    assert m.n_cells == 512
    assert m.dx == pytest.approx(1 / 16) and m.dy == pytest.approx(1 / 8)
    xc = m.cell_centers()
    assert xc.shape == (2, 512)
    # y fastest: cell 1 is (i=0, j=1)
    assert xc[0, 1] == xc[0, 0] and xc[1, 1] > xc[1, 0]
    assert m.cell_inradius == pytest.approx(m.dx * m.dy / (m.dx + m.dy))


def test_cfg_encodes_scheme():
    m = zb.create_2d((0, 1, 0, 1), 8, 8)
    s = HyperbolicSolver(time_end=0.3, compute_dt=zb.timestepping.adaptive(0.45, 2),
                         reconstruction_variables="eta", free_surface_h_index=1,
                         dtype="float32", eps_wet=1e-6)
    cfg = s._make_cfg(m, nsm(boundary_conditions={"left": "wall", "right": "wall"}))
    assert (cfg.order, cfg.recon, cfg.riemann) == (2, L.RECON["eta"], L.RIEMANN["hll_hr"])
    assert list(cfg.bc) == [1, 1, 0, 0]
    assert cfg.dtype == L.ZB_F32 and cfg.eps_wet == 1e-6
    assert cfg.cfl == 0.45 and cfg.dim_factor == 2 and cfg.t_end == 0.3


def test_eta_needs_h_index_and_hr_flux():
    m = zb.create_2d((0, 1, 0, 1), 8, 8)
    with pytest.raises(AssertionError):
        HyperbolicSolver(reconstruction_variables="eta")._make_cfg(m, nsm())
    with pytest.raises(NotImplementedError):
        HyperbolicSolver(reconstruction_variables="eta", free_surface_h_index=1) \
            ._make_cfg(m, nsm(riemann="rusanov"))


def test_mood_requires_eta():
    m = zb.create_2d((0, 1, 0, 1), 8, 8)
    with pytest.raises(NotImplementedError, match="per-cell"):
        HyperbolicSolver(mood=True)._make_cfg(m, nsm())


def test_periodic_pairs_and_unknown_bc():
    with pytest.raises(ValueError):
        zb.ShallowWater2D(boundary_conditions={"left": "periodic"}).bc_kinds()
    with pytest.raises(NotImplementedError):
        zb.ShallowWater2D(boundary_conditions={"top": "inflow"}).bc_kinds()


def test_dt_max_default_fill():
    a = zb.timestepping.adaptive(0.9, 2)
    assert a.with_dt_max(0.25).dt_max == 0.25
    assert zb.timestepping.adaptive(0.9, 2, dt_max=0.1).with_dt_max(0.25).dt_max == 0.1


def test_reduce_dt_clamp_is_xor():
    with pytest.raises(ValueError, match="XOR"):
        reduce_dt_clamp(1.0, 0.5)
    assert reduce_dt_clamp(None, 0.5) == 0.5
    assert reduce_dt_clamp(1.0, None) == 1.0


@pytest.mark.parametrize("dt", [0.0, -1.0, math.nan, math.inf])
def test_assert_dt_admissible_fatal(dt):
    with pytest.raises(FloatingPointError, match="FATAL"):
        assert_dt_admissible(dt, time=0.5, iteration=3)


def test_write_gate_and_proceed():
    S = MarchState(0.2, 1, 0, None, None)
    assert proceed(S, 0.3) and not proceed(S, 0.2)
    assert should_write(0.0, 0.1, 0, 0.5) == (True, 1)
    assert should_write(0.49, 0.1, 1, 0.5) == (False, 1)
    assert should_write(0.5 - 1e-15, 0.1, 1, 0.5) == (True, 2)


def test_initial_state_from_callable():
    m = zb.create_2d((-1, 1, -1, 1), 4, 4)
    mod = zb.ShallowWater2D(initial_conditions=lambda x: np.array([0, 1 + x[0], 0, 0]))
    Q = mod.initial_state(m)
    assert Q.shape == (4, 16)
    np.testing.assert_allclose(Q[1], 1 + m.cell_centers()[0])

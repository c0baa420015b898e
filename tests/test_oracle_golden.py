"""The oracle reproduces the reference's own golden end states.

Goldens: ``tests/golden/reference_goldens.npz`` (copied from the reference's
``tests/refs`` by ``tests/golden/make_golden.py``).  These pin the oracle's
first-order Rusanov march, the CFL law, KP ``hinv`` and the least-squares
derivative rows to round-off.
"""
import numpy as np
import pytest

from cases import gaussian_pulse_2d, lake_at_rest_ic, ritter_ic, stoker_ic, tilted_ic
from oracle import mesh as M
from oracle import swe as S

CFL = 0.9      # the reference's CFL law (tests/conftest.py:80-93)


def _march_1d(ic, n, t_end, **scheme):
    m = M.create_1d(0.0, 10.0, n)
    Q = np.stack([ic(x) for x in m.cell_centers[:, 0]], axis=1)
    return S.march(m, Q, S.Params(), S.Scheme(order=1, cfl=CFL, **scheme), t_end=t_end)


@pytest.mark.parametrize("name,ic,n,t_end", [
    ("parity", stoker_ic, 50, 0.5),
    ("stoker_wet", stoker_ic, 100, 1.0),
    ("ritter_dry", ritter_ic, 100, 1.0),
])
def test_oracle_1d_goldens(goldens, name, ic, n, t_end):
    Q, A, t, steps = _march_1d(ic, n, t_end)
    assert t == pytest.approx(t_end, abs=0)
    np.testing.assert_allclose(Q, goldens[f"{name}__Q"], rtol=0, atol=1e-15)
    # derivative rows to round-off; KP hinv (up to 1.4e3) to 1e-14 relative
    np.testing.assert_allclose(A[:3], goldens[f"{name}__Qaux"][:3], rtol=0, atol=1e-15)
    np.testing.assert_allclose(A[3], goldens[f"{name}__Qaux"][3], rtol=1e-13, atol=0)


def test_oracle_lake_at_rest_golden(goldens):
    """Hydrostatic-reconstruction Rusanov with walls keeps the lake at rest
    and matches the reference's ``wb_lake`` end state."""
    Q, A, t, steps = _march_1d(lake_at_rest_ic, 100, 1.0, riemann="rusanov_hr",
                               bc={"left": "wall", "right": "wall"})
    eta = Q[0] + Q[1]
    assert np.abs(eta - eta[0]).max() < 1e-12
    assert np.abs(Q[2] / Q[1]).max() < 1e-12
    np.testing.assert_allclose(Q, goldens["wb_lake__Q"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(A, goldens["wb_lake__Qaux"], rtol=0, atol=1e-14)


def test_oracle_2d_golden(goldens):
    m = M.create_2d(-1.0, 1.0, -1.0, 1.0, 32, 32)
    Q = np.stack([gaussian_pulse_2d(x) for x in m.cell_centers], axis=1)
    Q, A, t, steps = S.march(m, Q, S.Params(), S.Scheme(order=1, cfl=CFL), t_end=0.1)
    assert steps == 9
    np.testing.assert_allclose(Q, goldens["swe_2d__Q"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(A, goldens["swe_2d__Qaux"], rtol=0, atol=1e-14)


def test_bc_wall_golden(goldens):
    """Walls at both ends of the tilted surface (reference
    ``tests/runtime/test_bc_runtime.py:19-37``, kind "wall"): the end state
    and all four aux rows, including the end cells' derivative rows, whose
    least-squares stencil is the one-sided pair of cells plus the boundary
    ghost."""
    m = M.create_1d(0.0, 1.0, 40)
    Q = np.stack([tilted_ic(x) for x in m.cell_centers[:, 0]], axis=1)
    Q, A, t, steps = S.march(m, Q, S.Params(),
                             S.Scheme(order=1, cfl=CFL, bc={"left": "wall", "right": "wall"}),
                             t_end=0.2)
    np.testing.assert_allclose(Q, goldens["bc_wall__Q"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(A, goldens["bc_wall__Qaux"], rtol=0, atol=1e-13)


def test_bc_periodic_golden(goldens):
    """Periodic ends (kind "periodic").  Matched to 1.5e-7 absolute (3e-7
    relative on h ~ 0.5), not to round-off: the gap grows at the two wave
    fronts that leave the seam, and no per-step dt change explains it (a
    least-squares fit of 20 per-step dt perturbations leaves 1.1e-7), so one
    detail of the reference's seam flux is not restated here."""
    m = M.create_1d(0.0, 1.0, 40)
    Q = np.stack([tilted_ic(x) for x in m.cell_centers[:, 0]], axis=1)
    Q, A, t, steps = S.march(
        m, Q, S.Params(), S.Scheme(order=1, cfl=CFL,
                                   bc={"left": "periodic", "right": "periodic"}),
        t_end=0.2)
    gap = np.abs(Q - goldens["bc_periodic__Q"]).max()
    assert gap <= 2e-7, gap


def test_order2_goldens_gap_is_recorded(goldens):
    """The order-2 twins (20 cells, 2 steps) run zoomy_core numerics that are
    not in the reference tree.  The oracle's restatement of the readable
    order-2 pipeline (LSQ-MUSCL with the clip-min limiter, SSP-RK2 with the
    aux refreshed between stages, the cell-edge nonconservative term) differs
    from them by O(1e-4); the reference's momentum balance puts its time after
    two steps at 3.9655 against the oracle's 3.9291, so the state after the
    first step already differs.  Variants that were ruled out (none closes
    the gap below 1.5e-4): stale aux in stage 2, face-consistent hinv in the
    flux, cell-state wave speeds, hydrostatic-reconstruction Rusanov / HLL,
    the eta reconstruction with MOOD, other limiters, a rescaled gradient.
    This test keeps the gap visible so it cannot turn into a claim."""
    m = M.create_1d(0.0, 10.0, 20)
    for name, ic in (("stoker_wet_o2_small", stoker_ic), ("ritter_dry_o2_small", ritter_ic)):
        Q = np.stack([ic(x) for x in m.cell_centers[:, 0]], axis=1)
        scheme = S.Scheme(order=2, cfl=CFL)
        if name.startswith("ritter"):
            # the reference marches this twin with the eta reconstruction and
            # MOOD (``wet_dry_o2`` in its tests/conftest.py)
            scheme = S.Scheme(order=2, cfl=CFL, recon="eta", riemann="rusanov_hr", mood=True)
        Q, A, t, steps = S.march(m, Q, S.Params(), scheme, n_steps=2)
        gap = np.abs(Q - goldens[f"{name}__Q"]).max()
        assert 1e-6 < gap < 1e-3, (name, gap)

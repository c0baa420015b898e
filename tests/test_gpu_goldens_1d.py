"""The reference's own 1-D golden end states, reproduced through libzb.

The Cartesian kernels are two-dimensional; a 1-D case runs as its y-uniform
embedding: ``n x 4`` square cells, the 1-D boundary conditions on the left and
right sides, walls on the bottom and top (they mirror a zero ``q_y``, so the
y-faces carry only the hydrostatic pressure, which cancels in every cell), and
the reference's 1-D CFL law ``dt = CFL 2 r / (1 |lambda|)`` through
``adaptive(0.9, dimension=1)`` with ``r = dx / 2``.  Each run is
``HyperbolicSolver.solve`` in float64 to the reference's ``t_end``.

Checked per golden: every column of the state equals the golden end state to
1e-12 of the largest depth (the scale of every row: a lake at rest has
momentum ~1e-17; ``bc_periodic`` to 5e-7, the seam gap the oracle has too),
``q_y`` stays zero, and the aux rows that the 2-D
stencil shares with the 1-D one (KP ``hinv`` everywhere; the x-derivative rows
away from the two end cells, where the reference's 1-D mesh takes a one-sided
pair of cells) match to 1e-11 of the row's scale (1e-13 absolute at least).
"""
import numpy as np
import pytest

from cases import lake_at_rest_ic, ritter_ic, stoker_ic, tilted_ic

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import zoomy_b200 as zb  # noqa: E402
from zoomy_b200.fvm.solver import HyperbolicSolver  # noqa: E402

NY = 4
CASES = [
    # name, ic, domain, cells, t_end, left/right BC, riemann, tolerance
    ("parity", stoker_ic, (0.0, 10.0), 50, 0.5, "extrapolation", "rusanov", 1e-12),
    ("stoker_wet", stoker_ic, (0.0, 10.0), 100, 1.0, "extrapolation", "rusanov", 1e-12),
    ("ritter_dry", ritter_ic, (0.0, 10.0), 100, 1.0, "extrapolation", "rusanov", 1e-12),
    ("wb_lake", lake_at_rest_ic, (0.0, 10.0), 100, 1.0, "wall", "rusanov_hr", 1e-12),
    ("bc_wall", tilted_ic, (0.0, 1.0), 40, 0.2, "wall", "rusanov", 1e-12),
    ("bc_periodic", tilted_ic, (0.0, 1.0), 40, 0.2, "periodic", "rusanov", 5e-7),
]


def _embed(ic, xc1):
    q = np.stack([ic(x) for x in xc1], axis=1)           # (3, n)
    n = q.shape[1]
    Q = np.zeros((4, n * NY))
    Q[:3] = np.repeat(q, NY, axis=1)                     # cell (i, j) = i * NY + j
    return Q


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_gpu_reproduces_reference_1d_golden(goldens, case):
    name, ic, (x0, x1), n, t_end, side, riemann, tol = case
    dx = (x1 - x0) / n
    mesh = zb.create_2d((x0, x1, 0.0, NY * dx), n, NY)
    xc1 = x0 + (np.arange(n) + 0.5) * dx
    bcs = {"left": side, "right": side, "bottom": "wall", "top": "wall"}
    model = zb.ShallowWater2D(boundary_conditions=bcs, initial_conditions=_embed(ic, xc1))
    nsm = zb.NumericalSystemModel.from_system_model(
        model, zb.ReconstructionSpec(1, "minmod"), riemann)
    solver = HyperbolicSolver(time_end=t_end,
                              compute_dt=zb.timestepping.adaptive(0.9, dimension=1))
    Q, Qaux = solver.solve(mesh, nsm)
    assert solver.time == pytest.approx(t_end, abs=1e-15)
    q = Q.cpu().numpy().reshape(4, n, NY)
    a = Qaux.cpu().numpy().reshape(7, n, NY)
    G = goldens[f"{name}__Q"]
    GA = goldens[f"{name}__Qaux"]
    assert np.all(q[3] == 0.0)
    scale = np.abs(G[1]).max()
    for v in range(3):
        for j in range(NY):
            err = np.abs(q[v, :, j] - G[v]).max() / scale
            assert err <= tol, (name, v, j, err)
    # aux: 2-D rows [dq0/dx, dh/dx, dq1/dy, dh/dy, db/dx, db/dy, hinv] against
    # the 1-D rows [dq/dx, dh/dx, db/dx, hinv]
    inner = slice(1, n - 1)
    for row2, row1 in ((0, 0), (1, 1), (4, 2), (6, 3)):
        sl = slice(None) if row2 == 6 else inner
        ref = GA[row1, sl]
        scale = max(np.abs(GA[row1]).max(), 1e-300)
        atol = max(1e-11 * scale if tol <= 1e-12 else 1e-4 * scale, 1e-13)
        for j in range(NY):
            assert np.abs(a[row2, sl, j] - ref).max() <= atol, (name, row2, j)

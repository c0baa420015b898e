"""GPU parity of the unstructured-triangle SWE path against the oracle.

The mesh is built by the product's ``TriangleMesh``; the oracle rebuilds its
own connectivity, geometry and least-squares weights from the same vertices
and triangles (``oracle.mesh.tri_from_points``) and steps independently.
Tolerances as for the Cartesian path: float64 <= 1e-12 relative L-infinity
per step, dt <= 1e-14 relative, mass conserved to 1e-12 (float64 sums).
"""
import math

import numpy as np
import pytest

from oracle import mesh as OM
from oracle import swe as OS

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import zoomy_b200 as zb  # noqa: E402
from zoomy_b200 import _lib as L  # noqa: E402
from zoomy_b200.fvm.solver import HyperbolicSolver  # noqa: E402
from zoomy_b200.workloads import circular_dam_state  # noqa: E402

TAGS = ("left", "right", "bottom", "top")


def rel_err(a, b):
    return np.array([np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-14)
                     for v in range(a.shape[0])])


def setup(mesh, Q0, *, order=2, recon="eta", riemann="hll_hr", limiter="barth_jespersen",
          bc="wall", manning=0.0, eps_wet=None, dtype="float64", implicit=False,
          cfl=0.45, t_end=math.inf, oracle=True):
    bcs = {t: bc for t in TAGS}
    model = zb.ShallowWater2D(manning_n=manning, boundary_conditions=bcs,
                              initial_conditions=Q0)
    nsm = zb.NumericalSystemModel.from_system_model(
        model, zb.ReconstructionSpec(order, limiter), riemann)
    solver = HyperbolicSolver(
        time_end=t_end, compute_dt=zb.timestepping.adaptive(cfl, 2),
        reconstruction_variables="eta" if recon == "eta" else "conservative",
        free_surface_h_index=1 if recon == "eta" else None, eps_wet=eps_wet,
        dtype=dtype, implicit_source=implicit)
    Q, Qaux = solver.setup_simulation(mesh, nsm)
    om = OM.tri_from_points(mesh.vertices, mesh.triangles) if oracle else None
    scheme = OS.Scheme(order=order, limiter=limiter, recon="constant" if order == 1 else recon,
                       riemann=riemann, eps_wet=eps_wet, cfl=cfl, bc=bcs,
                       source="implicit" if implicit else "explicit")
    return solver, Q, Qaux, om, scheme, OS.Params(manning_n=manning)


def dam(mesh, wet=False, seed=4):
    xc = mesh.cell_centers()
    Q = circular_dam_state(xc, seed=seed, h_in=3.0 if wet else 2.0, h_out=2.0 if wet else 1.0)
    w = Q[1] > 0
    Q[2] = np.where(w, 0.1 * Q[1] * np.sin(3 * xc[1]), 0.0)
    Q[3] = np.where(w, -0.1 * Q[1] * np.cos(2 * xc[0]), 0.0)
    return Q


CONFIGS = [
    dict(order=1, recon="constant", riemann="rusanov", bc="extrapolation"),
    dict(order=1, recon="constant", riemann="hll_hr", bc="wall"),
    dict(order=2, recon="conservative", riemann="rusanov", bc="wall"),
    dict(order=2, recon="eta", riemann="hll_hr", bc="wall"),
    dict(order=2, recon="eta", riemann="hll_hr", bc="extrapolation", eps_wet=1e-6),
    dict(order=2, recon="eta", riemann="rusanov_hr", bc="wall", limiter="minmod"),
    dict(order=2, recon="eta", riemann="hll_hr", bc="wall", manning=0.03),
    dict(order=2, recon="eta", riemann="hll_hr", bc="wall", manning=0.03, implicit=True),
]


@pytest.fixture(scope="module")
def small_mesh():
    return zb.create_tri(36, seed=1)


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(str(v) for v in c.values()))
def test_tri_step_matches_oracle_per_step(small_mesh, cfg):
    Q0 = dam(small_mesh, wet=cfg["recon"] == "conservative")
    solver, Q, Qaux, om, scheme, params = setup(small_mesh, Q0, **cfg)
    solver.init_march(Q)
    for it in range(4):
        q = Q.double().cpu().numpy().copy()
        dt_ref = OS.compute_dt(om, q, params, scheme)
        solver.launch_steps(Q, 1)
        c = solver.read_ctrl()
        assert not (c.status & L.ZB_ST_DT_INVALID), c.status
        assert c.dt == pytest.approx(dt_ref, rel=1e-14, abs=0)
        ref, trouble = OS.step(om, q, c.dt, params, scheme, return_troubled=True)
        # without dry demotion or MOOD the order-2 scheme can leave h >= 0 at
        # CFL 0.45 (the reference needs 1/(2k+1) or MOOD for positivity); the
        # troubled flag must then agree with the oracle's predicate
        assert bool(c.status & L.ZB_ST_TROUBLED) == bool(trouble.any())
        err = rel_err(Q.double().cpu().numpy(), ref)
        assert err.max() <= 1e-12, f"step {it}: {err}"


def test_tri_host_dt_step_and_aux(small_mesh):
    Q0 = dam(small_mesh, seed=9)
    solver, Q, Qaux, om, scheme, params = setup(small_mesh, Q0, manning=0.03)
    q0 = Q.cpu().numpy()
    np.testing.assert_allclose(Qaux.cpu().numpy(), OS.derivative_aux(om, q0, params),
                               rtol=1e-12, atol=1e-12)
    dt = solver.compute_timestep(Q, Qaux)
    assert dt == pytest.approx(OS.compute_dt(om, q0, params, scheme), rel=1e-14)
    Qn = solver.step(dt, 0.0, Q, Qaux)
    assert rel_err(Qn.cpu().numpy(), OS.step(om, q0, dt, params, scheme)).max() <= 1e-12


@pytest.fixture(scope="module")
def big_mesh():
    return zb.create_tri(1415, seed=0)


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_tri_4m_cells_mass_and_lake(big_mesh, dtype):
    """About 4M triangles (config 3 size): a lake at rest over bumps with dry
    islands stays at rest, and a dam break with Manning n = 0.03 conserves
    mass (float64 sums) with walls."""
    mesh = big_mesh
    assert mesh.n_cells > 3_900_000
    xc = mesh.cell_centers()
    from zoomy_b200.workloads import bumps
    b = bumps(xc, seed=5)
    lake = np.stack([b, np.maximum(1.0 - b, 0.0), 0 * b, 0 * b])
    tol = 1e-12 if dtype == "float64" else 1e-5
    solver, Q, Qaux, *_ = setup(mesh, lake, dtype=dtype, eps_wet=1e-6, manning=0.03,
                                oracle=False)
    solver.init_march(Q)
    solver.launch_steps(Q, 5)
    assert solver.read_ctrl().status == 0
    q = Q.double().cpu().numpy()
    wet = lake[1] > 0
    assert np.abs((q[0] + q[1])[wet] - 1.0).max() <= 10 * tol
    assert np.abs(q[2:]).max() <= 10 * tol
    solver, Q, Qaux, *_ = setup(mesh, circular_dam_state(xc, seed=0), dtype=dtype,
                                eps_wet=1e-6, manning=0.03, oracle=False)
    m0 = solver.mass(Q)
    solver.init_march(Q)
    solver.launch_steps(Q, 10)
    c = solver.read_ctrl()
    assert c.status == 0 and c.steps == 10
    m1 = solver.mass(Q)
    assert abs(m1 - m0) / m0 <= (1e-12 if dtype == "float64" else 1e-6)

"""GPU parity of the Cartesian SWE path (libzb) against the float64 oracle.

Tolerances (stated here, checked below):
* float64 kernels: relative L-infinity error <= 1e-12 per step against the
  oracle fed the same state and dt (per state row, relative to the row's
  max-norm, with an absolute floor of 1e-14 for rows that are ~0);
* dt: relative error <= 1e-14;
* float32 kernels: after 1000 steps of the noisy dam break the float32 state
  agrees with float64 to relative L1 2e-3 (h) and 2e-2 (momentum) and
  relative L-infinity 2e-2 (h) -- see test_fp32_drift_after_1000_steps;
* mass (float64 sums) is conserved to 1e-12 relative per 10 steps in float64.
"""
import math

import numpy as np
import pytest

from cases import circular_dam_state, gaussian_pulse_2d
from oracle import mesh as OM
from oracle import swe as OS

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import zoomy_b200 as zb  # noqa: E402
from zoomy_b200 import _lib as L  # noqa: E402
from zoomy_b200.fvm.solver import HyperbolicSolver  # noqa: E402
from zoomy_b200.fvm.solver2 import MarchSolver  # noqa: E402

TAGS = ("left", "right", "bottom", "top")


def make(nx, ny, domain, state, *, order=2, recon="eta", riemann="hll_hr",
         limiter="minmod", bc="wall", manning=0.0, cfl=0.45, eps_wet=None,
         dtype="float64", implicit=False, t_end=math.inf, mood=False, oracle=True):
    bcs = {t: bc for t in TAGS} if isinstance(bc, str) else dict(zip(TAGS, bc))
    model = zb.ShallowWater2D(manning_n=manning, boundary_conditions=bcs,
                              initial_conditions=state)
    nsm = zb.NumericalSystemModel.from_system_model(
        model, zb.ReconstructionSpec(order, limiter), riemann)
    mesh = zb.create_2d(domain, nx, ny)
    solver = HyperbolicSolver(
        time_end=t_end, compute_dt=zb.timestepping.adaptive(cfl, 2),
        reconstruction_variables="eta" if recon == "eta" else "conservative",
        free_surface_h_index=1 if recon == "eta" else None, eps_wet=eps_wet,
        dtype=dtype, implicit_source=implicit, mood=mood)
    Q, Qaux = solver.setup_simulation(mesh, nsm)
    om = OM.create_2d(domain[0], domain[1], domain[2], domain[3], nx, ny) if oracle else None
    scheme = OS.Scheme(order=order, limiter=limiter,
                       recon="constant" if order == 1 else recon, riemann=riemann,
                       eps_wet=eps_wet, cfl=cfl, bc=bcs, mood=mood,
                       source="implicit" if implicit else "explicit")
    params = OS.Params(manning_n=manning)
    return solver, Q, Qaux, om, scheme, params


def rel_err(a, b):
    out = []
    for v in range(a.shape[0]):
        scale = max(np.abs(b[v]).max(), 1e-14)
        out.append(np.abs(a[v] - b[v]).max() / scale)
    return np.array(out)


def moving_dam(nx, ny, domain, seed=3, wet=False):
    """Circular dam break over seeded bumps (dry islands unless ``wet``) with
    a swirl so every flux term is non-zero from the first step.  ``wet``
    raises the water level so no cell is dry: the conservative LSQ-MUSCL path
    is not positivity preserving at a dry front (the reference measured
    negative depth there), so its parity cases run wet."""
    m = zb.create_2d(domain, nx, ny)
    xc = m.cell_centers()
    Q = circular_dam_state(xc, seed=seed, center=(0.5 * (domain[0] + domain[1]),
                                                 0.5 * (domain[2] + domain[3])),
                           h_in=3.0 if wet else 2.0, h_out=2.0 if wet else 1.0)
    wet = Q[1] > 0
    Q[2] = np.where(wet, 0.1 * Q[1] * np.sin(3 * xc[1]), 0.0)
    Q[3] = np.where(wet, -0.1 * Q[1] * np.cos(2 * xc[0]), 0.0)
    return Q


CONFIGS = [
    dict(order=1, recon="constant", riemann="rusanov", bc="extrapolation"),
    dict(order=1, recon="constant", riemann="rusanov", bc="wall"),
    dict(order=1, recon="constant", riemann="hll_hr", bc="periodic"),
    dict(order=2, recon="conservative", riemann="rusanov", bc="extrapolation"),
    dict(order=2, recon="conservative", riemann="hll_hr", bc="wall"),
    dict(order=2, recon="eta", riemann="hll_hr", bc="wall"),
    dict(order=2, recon="eta", riemann="hll_hr", bc="periodic"),
    dict(order=2, recon="eta", riemann="hll_hr", bc=("wall", "extrapolation",
                                                    "extrapolation", "wall")),
    dict(order=2, recon="eta", riemann="rusanov_hr", bc="extrapolation"),
    dict(order=2, recon="eta", riemann="hll_hr", bc="wall", eps_wet=1e-6),
    dict(order=2, recon="eta", riemann="hll_hr", bc="wall", limiter="venkatakrishnan"),
    dict(order=2, recon="eta", riemann="hll_hr", bc="wall", manning=0.03),
    dict(order=2, recon="eta", riemann="hll_hr", bc="wall", manning=0.03, implicit=True),
]


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(str(v) for v in c.values()))
def test_fused_step_matches_oracle_per_step(cfg):
    domain = (0.0, 1.0, 0.0, 1.5)
    nx, ny = 40, 48
    Q0 = moving_dam(nx, ny, domain, wet=cfg["recon"] == "conservative")
    solver, Q, Qaux, om, scheme, params = make(nx, ny, domain, Q0, **cfg)
    solver.init_march(Q)
    for it in range(4):
        q_before = Q.double().cpu().numpy().copy()
        dt_ref = OS.compute_dt(om, q_before, params, scheme)
        solver.launch_steps(Q, 1)
        c = solver.read_ctrl()
        assert c.status == 0, f"status {c.status} at step {it}"
        assert c.dt == pytest.approx(dt_ref, rel=1e-14, abs=0)
        ref = OS.step(om, q_before, c.dt, params, scheme)
        got = Q.double().cpu().numpy()
        err = rel_err(got, ref)
        assert err.max() <= 1e-12, f"step {it}: rel err per row {err}"
        assert np.array_equal(got[0], q_before[0]), "the b row must not change"


STRIP_CONFIGS = [
    dict(order=2, recon="eta", riemann="hll_hr", bc="wall", eps_wet=1e-6),
    dict(order=2, recon="conservative", riemann="rusanov", bc="periodic"),
    dict(order=2, recon="eta", riemann="rusanov_hr", bc="extrapolation",
         limiter="venkatakrishnan", manning=0.03),
]


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("cfg", STRIP_CONFIGS, ids=lambda c: "-".join(str(v) for v in c.values()))
def test_strip_kernel_matches_tiles(cfg, dtype):
    """The fused step hands the grid to the register-marching strip kernel:
    without a periodic side the strips cover every cell (items that reach a
    boundary run its EDGE body), with one the interior (two cells in from
    every side) -- here three 28-column strips and three row chunks of a
    150 x 100 grid -- and the tile kernel takes the frame.  The host-dt step
    runs the tile kernel everywhere.  Interior strips give the tile kernel's
    bits; the EDGE body (whose normal sign is a runtime value, so the compiler
    fuses a few products differently) agrees to rounding; and the float64
    result matches the oracle."""
    domain = (0.0, 1.5, 0.0, 1.0)
    nx, ny = 150, 100
    Q0 = moving_dam(nx, ny, domain, wet=cfg["recon"] == "conservative")
    solver, Q, Qaux, om, scheme, params = make(nx, ny, domain, Q0, dtype=dtype,
                                               oracle=dtype == "float64", **cfg)
    Qa = Q.clone()
    solver.init_march(Q)
    solver.launch_steps(Q, 1)
    c = solver.read_ctrl()
    assert c.status == 0
    dt = c.dt
    ref_tiles = solver.step(dt, 0.0, Qa, Qaux)
    if cfg["bc"] == "periodic":
        assert torch.equal(Q, ref_tiles)
    else:
        tol = 1e-13 if dtype == "float64" else 2e-6
        if cfg.get("manning", 0.0) != 0.0:   # the host-dt path applies friction afterwards
            tol = 1e-6
        err = rel_err(Q.double().cpu().numpy(), ref_tiles.double().cpu().numpy())
        assert err.max() <= tol, err
    if dtype == "float64":
        ref = OS.step(om, Q0, dt, params, scheme)
        assert rel_err(Q.cpu().numpy(), ref).max() <= 1e-12


def test_fused_steps_replay_from_a_cuda_graph():
    """Three fused steps captured into a CUDA graph -- each stage forks its
    boundary-strip launch onto the library's second stream and joins it back
    -- replay to the bits of the same steps launched eagerly."""
    domain = (0.0, 1.5, 0.0, 1.0)
    nx, ny = 150, 100
    Q0 = moving_dam(nx, ny, domain)
    solver, Q, Qaux, *_ = make(nx, ny, domain, Q0, dtype="float32", oracle=False, order=2,
                               recon="eta", riemann="hll_hr", bc="wall", eps_wet=1e-6)
    Qe = Q.clone()
    solver.init_march(Qe)
    solver.launch_steps(Qe, 3)
    torch.cuda.synchronize()
    Qg = Q.clone()
    solver.init_march(Qg)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        solver.launch_steps(Qg, 3)
    g.replay()
    torch.cuda.synchronize()
    assert solver.read_ctrl().status == 0
    assert torch.equal(Qg, Qe)


@pytest.mark.parametrize("nx,ny", [(4, 4), (5, 33), (37, 61), (70, 29), (130, 57), (67, 58)])
def test_full_coverage_strips_on_ragged_grids(nx, ny):
    """Full-coverage strip lists on grids whose sides are not multiples of the
    28-column strips or the 64-row chunks (a last strip of one column, middle
    strips that reach the right side, grids narrower than one strip): one
    float64 step against the oracle, walls on x and extrapolation on y."""
    domain = (0.0, 1.0, 0.0, 1.0)
    Q0 = moving_dam(nx, ny, domain)
    cfg = dict(order=2, recon="eta", riemann="hll_hr", bc=("wall", "wall", "extrapolation",
                                                           "extrapolation"), eps_wet=1e-6)
    solver, Q, Qaux, om, scheme, params = make(nx, ny, domain, Q0, dtype="float64",
                                               oracle=True, **cfg)
    solver.init_march(Q)
    solver.launch_steps(Q, 1)
    c = solver.read_ctrl()
    assert c.status == 0
    ref = OS.step(om, Q0, c.dt, params, scheme)
    assert rel_err(Q.cpu().numpy(), ref).max() <= 1e-12


@pytest.mark.parametrize("bc", ["wall", ("extrapolation", "extrapolation", "wall", "wall")],
                         ids=["walls", "y-walls"])
@pytest.mark.parametrize("nx,ny", [(5, 33), (37, 61), (70, 29), (130, 57), (67, 58)])
def test_float32_column_edge_strips_match_tiles(nx, ny, bc):
    """In float32 the strips whose lanes reach a y-boundary column march the
    rows between the boundary rows with the paired-float interior arithmetic
    and recompute the boundary column's slopes and its boundary y-face with the
    boundary expressions (walls mirror q_y there).  One fused step against the
    tile kernel's host-dt step with the same dt, on ragged grids."""
    domain = (0.0, 1.0, 0.0, 1.0)
    Q0 = moving_dam(nx, ny, domain)
    solver, Q, Qaux, *_ = make(nx, ny, domain, Q0, dtype="float32", oracle=False, bc=bc,
                               eps_wet=1e-6)
    Qa = Q.clone()
    solver.init_march(Q)
    solver.launch_steps(Q, 1)
    c = solver.read_ctrl()
    assert c.status == 0
    ref = solver.step(c.dt, 0.0, Qa, Qaux)
    err = rel_err(Q.double().cpu().numpy(), ref.double().cpu().numpy())
    assert err.max() <= 2e-6, err


@pytest.mark.parametrize("cfg", CONFIGS[3:7], ids=lambda c: "-".join(str(v) for v in c.values()))
def test_host_dt_step_matches_oracle(cfg):
    """``step(dt, t, Q, Qaux)`` with a host dt (the reference's call shape)."""
    domain = (0.0, 1.0, 0.0, 1.5)
    Q0 = moving_dam(40, 48, domain, seed=5, wet=cfg["recon"] == "conservative")
    solver, Q, Qaux, om, scheme, params = make(40, 48, domain, Q0, **cfg)
    dt = solver.compute_timestep(Q, Qaux)
    q0 = Q.double().cpu().numpy()
    assert dt == pytest.approx(OS.compute_dt(om, q0, params, scheme), rel=1e-14)
    Qn = solver.step(dt, 0.0, Q, Qaux)
    err = rel_err(Qn.double().cpu().numpy(), OS.step(om, q0, dt, params, scheme))
    assert err.max() <= 1e-12, err


def test_float64_newton_quotient_and_roots():
    """The float64 kernels divide and take square roots by Newton refinement
    of the hardware approximations with a final residual correction.  Against
    IEEE arithmetic over magnitudes 2^-40 .. 2^40: the quotient and the
    square root within 1 ulp of numpy's correctly rounded results, the
    reciprocal square root within 2 ulp of an 80-bit extended reference."""
    rng = np.random.default_rng(7)
    n = 1 << 20
    a = rng.uniform(-1.0, 1.0, n) * np.exp2(rng.integers(-40, 41, n))
    b = rng.uniform(0.5, 1.0, n) * np.exp2(rng.integers(-40, 41, n))
    da = torch.tensor(a, device="cuda")
    db = torch.tensor(b, device="cuda")
    out = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    assert L.load().zb_newton_check_f64(L.ptr(da), L.ptr(db), L.ptr(out), n,
                                        L.stream_ptr()) == 0
    o = out.cpu().numpy()

    def ulps(got, ref):
        return np.abs(got - ref) / np.spacing(np.abs(ref))

    assert ulps(o[:n], a / b).max() <= 1.0
    assert ulps(o[n:2 * n], np.sqrt(b)).max() <= 1.0
    rs = (1.0 / np.sqrt(b.astype(np.longdouble))).astype(np.float64)
    assert ulps(o[2 * n:], rs).max() <= 2.0


def test_aux_rows_match_oracle():
    domain = (0.0, 1.0, 0.0, 1.5)
    Q0 = moving_dam(40, 48, domain)
    solver, Q, Qaux, om, scheme, params = make(40, 48, domain, Q0)
    ref = OS.derivative_aux(om, Q.cpu().numpy(), params)
    np.testing.assert_allclose(Qaux.cpu().numpy(), ref, rtol=1e-13, atol=1e-13)


def test_gpu_reproduces_reference_golden_swe_2d(goldens):
    """The reference's own 2-D golden (32x32 Gaussian pulse, first order,
    extrapolation, CFL 0.9, t_end 0.1) through ``HyperbolicSolver.solve``."""
    model = zb.ShallowWater2D(boundary_conditions={t: "extrapolation" for t in TAGS},
                              initial_conditions=gaussian_pulse_2d)
    nsm = zb.NumericalSystemModel.from_system_model(
        model, zb.ReconstructionSpec(1, "minmod"))
    mesh = zb.create_2d((-1.0, 1.0, -1.0, 1.0), 32, 32)
    solver = HyperbolicSolver(time_end=0.1, compute_dt=zb.timestepping.adaptive(0.9, 2))
    Q, Qaux = solver.solve(mesh, nsm)
    assert solver.steps_taken == 9
    np.testing.assert_allclose(Q.cpu().numpy(), goldens["swe_2d__Q"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(Qaux.cpu().numpy(), goldens["swe_2d__Qaux"], rtol=0, atol=1e-13)


def _l1(a, b):
    return np.abs(a - b).sum() / np.abs(b).sum()


def test_fp32_drift_after_1000_steps():
    """float32 against float64 after 1000 steps of the noisy dam break over
    bumps (64^2).  Measured on B200: L1(h) 4.4e-4, L1(q) 6.1e-3, Linf(h)
    4.5e-3 -- the float64 GPU path itself drifts from the float64 oracle by
    5e-8 (L1) over 200 steps of this case, so the gap is float32 rounding
    amplified by limiter switching, not an arithmetic difference.  Stated
    tolerance: L1(h) <= 2e-3, L1(q) <= 2e-2, Linf(h) <= 2e-2, times within 1e-4.
    The per-step parity of the float64 kernels (1e-12) is the arithmetic gate."""
    domain = (0.0, 1.0, 0.0, 1.0)
    m = zb.create_2d(domain, 64, 64)
    Q0 = circular_dam_state(m.cell_centers(), seed=7)
    runs = {}
    for dt_ in ("float32", "float64"):
        solver, Q, Qaux, *_ = make(64, 64, domain, Q0, dtype=dt_, eps_wet=1e-6,
                                   oracle=False)
        solver.init_march(Q)
        solver.launch_steps(Q, 1000)
        c = solver.read_ctrl()
        assert c.status == 0
        runs[dt_] = (Q.double().cpu().numpy(), c.t[1000 % 3])
    (q32, t32), (q64, t64) = runs["float32"], runs["float64"]
    assert t32 == pytest.approx(t64, rel=1e-4)
    assert _l1(q32[1], q64[1]) <= 2e-3
    assert max(_l1(q32[2], q64[2]), _l1(q32[3], q64[3])) <= 2e-2
    assert np.abs(q32[1] - q64[1]).max() / np.abs(q64[1]).max() <= 2e-2


def test_fp32_1000_steps_against_the_float64_oracle():
    """The float32 GPU march of 1000 steps at 256^2 (the 2048^2 configuration's
    scheme and case family: noisy circular dam break over 16 seeded bumps,
    eta-MUSCL minmod + HR-HLL, SSP-RK2, walls, dry-cell demotion 1e-6, CFL
    0.45) against the float64 ORACLE's own march of the same 1000 steps
    (``tests/golden/march_256_1000.npz``, made by ``make_march_fixture.py``).
    Stated tolerance: relative L1 of h <= 2e-3, of each momentum row <= 2e-2,
    relative L-infinity of h <= 2e-2, end times within 1e-4 relative."""
    import pathlib
    fx = np.load(pathlib.Path(__file__).parent / "golden" / "march_256_1000.npz")
    n, steps = int(fx["n"]), int(fx["steps"])
    domain = (0.0, 1.0, 0.0, 1.0)
    m = zb.create_2d(domain, n, n)
    Q0 = circular_dam_state(m.cell_centers(), seed=int(fx["seed"]))
    solver, Q, Qaux, *_ = make(n, n, domain, Q0, dtype="float32", eps_wet=1e-6, oracle=False)
    solver.init_march(Q)
    solver.launch_steps(Q, steps)
    c = solver.read_ctrl()
    assert c.status == 0
    got = Q.double().cpu().numpy()[1:]
    ref = fx["Q"].astype(np.float64)
    assert c.t[steps % 3] == pytest.approx(float(fx["t"]), rel=1e-4)
    assert _l1(got[0], ref[0]) <= 2e-3
    assert max(_l1(got[1], ref[1]), _l1(got[2], ref[2])) <= 2e-2
    assert np.abs(got[0] - ref[0]).max() / np.abs(ref[0]).max() <= 2e-2


def test_fp64_short_march_tracks_oracle():
    """20 steps of the wet-dry dam break: float64 GPU against the oracle's
    own march (own dt each step) stays within 1e-9 relative L-infinity."""
    domain = (0.0, 1.0, 0.0, 1.0)
    m = zb.create_2d(domain, 48, 48)
    Q0 = circular_dam_state(m.cell_centers(), seed=11)
    solver, Q, Qaux, om, scheme, params = make(48, 48, domain, Q0, eps_wet=1e-6)
    solver.init_march(Q)
    solver.launch_steps(Q, 20)
    assert solver.read_ctrl().status == 0
    Qr, _, t, _ = OS.march(om, Q0, params, scheme, n_steps=20)
    assert rel_err(Q.double().cpu().numpy(), Qr).max() <= 1e-9


@pytest.mark.parametrize("dtype,tol", [("float64", 1e-12), ("float32", 1e-5)])
def test_full_size_mass_and_lake_at_rest(dtype, tol):
    """2048^2 with dry islands: a lake at rest stays at rest and a dam break
    conserves mass (float64 sums on the device)."""
    n = 2048
    domain = (0.0, 1.0, 0.0, 1.0)
    m = zb.create_2d(domain, n, n)
    xc = m.cell_centers()
    from cases import bumps
    b = bumps(xc, seed=0)
    lake = np.stack([b, np.maximum(1.0 - b, 0.0), 0 * b, 0 * b])
    solver, Q, Qaux, *_ = make(n, n, domain, lake, dtype=dtype, eps_wet=1e-6, oracle=False)
    solver.init_march(Q)
    solver.launch_steps(Q, 10)
    assert solver.read_ctrl().status == 0
    q = Q.double().cpu().numpy()
    wet = lake[1] > 0
    assert np.abs((q[0] + q[1])[wet] - 1.0).max() <= tol * 10
    assert np.abs(q[2:]).max() <= tol * 10
    assert np.all(q[1][~wet] == 0.0)
    dam = circular_dam_state(xc, seed=0)
    solver, Q, Qaux, *_ = make(n, n, domain, dam, dtype=dtype, eps_wet=1e-6, oracle=False)
    m0 = solver.mass(Q)
    solver.init_march(Q)
    solver.launch_steps(Q, 10)
    assert solver.read_ctrl().status == 0
    m1 = solver.mass(Q)
    assert abs(m1 - m0) / m0 <= (1e-12 if dtype == "float64" else 1e-6)


def test_steps_after_t_end_are_noops():
    domain = (0.0, 1.0, 0.0, 1.0)
    Q0 = moving_dam(32, 32, domain)
    solver, Q, Qaux, *_ = make(32, 32, domain, Q0, t_end=0.01)
    Q, Qaux = solver.run_simulation(Q, Qaux)
    assert solver.time == pytest.approx(0.01, abs=1e-15)
    before = Q.clone()
    solver.launch_steps(Q, 5)
    c = solver.read_ctrl()
    assert c.status == 0 and c.dt == 0.0
    assert torch.equal(Q, before)


def test_host_injected_nan_is_fatal():
    """Failure detection without a GPU fault: a NaN planted in the host state
    before upload makes dt non-finite; the march aborts with the reference's
    FloatingPointError and the troubled/dt status bits are set."""
    domain = (0.0, 1.0, 0.0, 1.0)
    Q0 = moving_dam(32, 32, domain)
    Q0[1, 100] = np.nan
    solver, Q, Qaux, *_ = make(32, 32, domain, Q0, t_end=1.0)
    with pytest.raises(FloatingPointError, match="FATAL"):
        solver.run_simulation(Q, Qaux)
    assert solver.read_ctrl().status & L.ZB_ST_DT_INVALID


def test_march_solver_matches_hyperbolic_solver():
    domain = (0.0, 1.0, 0.0, 1.0)
    Q0 = moving_dam(40, 40, domain)
    solver, Q, Qaux, om, scheme, params = make(40, 40, domain, Q0)
    solver.init_march(Q)
    solver.launch_steps(Q, 3)
    ms = MarchSolver(reconstruction_variables="eta", free_surface_h_index=1)
    model = solver.nsm
    S = ms.setup_march(solver.mesh, model, CFL=0.45)
    S, stats = ms.march(S, n_steps=3)
    assert stats["steps"] == 3
    err = rel_err(S.Q.double().cpu().numpy(), Q.double().cpu().numpy())
    assert err.max() <= 1e-13, err


def _island_under_flow(n):
    """A Gaussian island (peak 0.8) that emerges from a 0.5-deep layer moving
    in x: with the eta reconstruction and no dry-cell demotion the order-2
    candidate leaves negative depth at the island's shore at the plain CFL dt
    (the oracle troubles 32 cells of 48^2)."""
    m = zb.create_2d((0.0, 1.0, 0.0, 1.0), n, n)
    xc = m.cell_centers()
    Q0 = np.zeros((4, m.n_cells))
    Q0[0] = 0.8 * np.exp(-((xc[0] - 0.5) ** 2 + (xc[1] - 0.5) ** 2) / 0.02)
    Q0[1] = np.maximum(0.5 - Q0[0], 0.0)
    Q0[2] = 0.5 * Q0[1]
    return Q0


def test_mood_redo_matches_oracle():
    """Per-cell MOOD (production ``solver_jax.py:1055-1071``): the troubled
    cells of the order-2 candidate are demoted to first order and the step is
    re-run.  The case troubles cells by construction (asserted first)."""
    domain = (0.0, 1.0, 0.0, 1.0)
    Q0 = _island_under_flow(48)
    solver, Q, Qaux, om, scheme, params = make(48, 48, domain, Q0, mood=True)
    q0 = Q.double().cpu().numpy()
    dt = OS.compute_dt(om, q0, params, scheme)
    ref_plain, trouble = OS.step(om, q0, dt, params,
                                 OS.Scheme(**{**scheme.__dict__, "mood": False}),
                                 return_troubled=True)
    assert trouble.sum() > 0 and ref_plain[1].min() < 0.0
    got = solver.step(dt, 0.0, Q, Qaux).double().cpu().numpy()
    ref = OS.step(om, q0, dt, params, scheme)
    assert rel_err(got, ref).max() <= 1e-12
    assert got[1].min() >= 0.0
    assert not np.allclose(got, ref_plain)
    # mass is conserved through the redo (shared face fluxes)
    assert abs(got[1].sum() - q0[1].sum()) <= 1e-12 * q0[1].sum()


def test_march_solver_whole_step_redo_matches_oracle():
    """solver2's MOOD (``solver2/blocks.py:304-323``): when any cell is
    troubled the whole step is replayed with the constant reconstruction
    through the same SSP-RK2 stage loop."""
    domain = (0.0, 1.0, 0.0, 1.0)
    Q0 = _island_under_flow(48)
    _, _, _, om, scheme, params = make(48, 48, domain, Q0, mood=True)
    model = zb.ShallowWater2D(boundary_conditions={t: "wall" for t in TAGS},
                              initial_conditions=Q0)
    nsm = zb.NumericalSystemModel.from_system_model(
        model, zb.ReconstructionSpec(2, "minmod"), "hll_hr")
    ms = MarchSolver(mood_redo=True, reconstruction_variables="eta", free_surface_h_index=1)
    S = ms.setup_march(zb.create_2d(domain, 48, 48), nsm, CFL=0.45)
    _, _, dt = ms.step_head(S)
    assert dt == pytest.approx(OS.compute_dt(om, Q0, params, scheme), rel=1e-14)
    S1, troubled = ms.hyperbolic_step(S, dt)
    assert troubled
    ref = OS.step(om, Q0, dt, params, OS.Scheme(**{**scheme.__dict__, "mood_mode": "step"}))
    got = S1.Q.double().cpu().numpy()
    assert rel_err(got, ref).max() <= 1e-12
    assert got[1].min() >= 0.0

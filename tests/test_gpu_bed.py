"""Prepared bed slopes (``zb_swe2d_bed_prepare``) against the bed slope
evaluated in every stage.

The bathymetry row never changes, so the eta / HLL-HR fused step can read
b's interior gradient and limiter value from planes prepared once.  The
prepared planes repeat the strip body's own operations for b (the paired
float32 block, the scalar float64 one), so a march with them is the same
march bit for bit; these tests hold that over fused steps on square and
ragged grids, both precisions, every limiter, dry cells, periodic sides and
Manning friction, and check the planes against the float64 central
least-squares gradient.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from zoomy_b200 import _lib as L  # noqa: E402
from zoomy_b200.workloads import bumps, circular_dam_state, grf_dam_state  # noqa: E402


def _centers(nx, ny):
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    return np.stack([((i + 0.5) / nx).reshape(-1), ((j + 0.5) / ny).reshape(-1)])


def _cfg(nx, ny, limiter="minmod", bc="wall", manning=0.0, eps_wet=1e-6, dtype=torch.float32):
    c = L.ZbSwe2dCfg()
    c.nx, c.ny = nx, ny
    c.x0, c.y0, c.dx, c.dy = 0.0, 0.0, 1.0 / nx, 1.0 / ny
    c.order, c.recon, c.riemann = 2, L.RECON["eta"], L.RIEMANN["hll_hr"]
    c.limiter = L.LIMITER[limiter]
    for i in range(4):
        c.bc[i] = L.BC[bc]
    c.g, c.wet_dry_eps, c.eps_wet, c.manning_n = 9.81, 1e-6, eps_wet, manning
    c.implicit_source, c.dim_factor, c.cfl = 0, 2, 0.45
    c.dt_max, c.t_end, c.degree = float("inf"), float("inf"), 0
    c.dtype = L.ZB_F64 if dtype == torch.float64 else L.ZB_F32
    return c


def _march(lib, cfg, Q, steps):
    """``steps`` fused steps in place on ``Q``; returns the control block."""
    st = L.stream_ptr()
    ctrl = torch.zeros(L.CTRL_BYTES, dtype=torch.uint8, device="cuda")
    wsb = lib.zb_swe2d_workspace_bytes(C.byref(cfg))
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    assert lib.zb_swe2d_init(C.byref(cfg), L.ptr(Q), L.ptr(ctrl), 0, 0.0, st) == 0
    for k in range(steps):
        assert lib.zb_swe2d_step(C.byref(cfg), L.ptr(Q), L.ptr(ws), C.c_size_t(wsb),
                                 L.ptr(ctrl), k % 3, st) == 0
    torch.cuda.synchronize()
    return L.ZbCtrl.from_buffer_copy(ctrl.cpu().numpy().tobytes())


def _prepare(lib, cfg, Q):
    nb = lib.zb_swe2d_bed_bytes(C.byref(cfg))
    assert nb == 3 * cfg.nx * cfg.ny * (8 if cfg.dtype == L.ZB_F64 else 4)
    bed = torch.empty(nb, dtype=torch.uint8, device="cuda")
    assert lib.zb_swe2d_bed_prepare(C.byref(cfg), L.ptr(Q), L.ptr(bed), C.c_size_t(nb),
                                    L.stream_ptr()) == 0
    torch.cuda.synchronize()
    return bed


CASES = {
    "minmod-walls-256": dict(nx=256, ny=256),
    "minmod-ragged-131x77": dict(nx=131, ny=77),
    "minmod-ragged-70x300": dict(nx=70, ny=300),
    "barth-jespersen": dict(nx=160, ny=96, limiter="barth_jespersen"),
    "venkatakrishnan": dict(nx=96, ny=160, limiter="venkatakrishnan"),
    "unlimited": dict(nx=128, ny=128, limiter="none"),
    "periodic": dict(nx=128, ny=96, bc="periodic"),
    "extrapolation-manning": dict(nx=120, ny=120, bc="extrapolation", manning=0.03),
    "no-dry-demotion": dict(nx=100, ny=140, eps_wet=-1.0),
}


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("state", ["dam", "grf"])
@pytest.mark.parametrize("case", list(CASES))
def test_prepared_bed_march_is_bitwise_the_evaluated_one(case, state, dtype):
    kw = dict(CASES[case])
    nx, ny = kw.pop("nx"), kw.pop("ny")
    lib = L.load()
    xc = _centers(nx, ny)
    q = circular_dam_state(xc, seed=5) if state == "dam" else grf_dam_state(xc, seed=6)
    Q0 = torch.as_tensor(q, dtype=dtype, device="cuda").contiguous()
    cfg_a = _cfg(nx, ny, dtype=dtype, **kw)
    cfg_b = _cfg(nx, ny, dtype=dtype, **kw)
    bed = _prepare(lib, cfg_b, Q0)
    cfg_b.bed = bed.data_ptr()
    Qa, Qb = Q0.clone(), Q0.clone()
    ca = _march(lib, cfg_a, Qa, 20)
    cb = _march(lib, cfg_b, Qb, 20)
    # the dry islands of the random-field state trouble a few cells (h < 0
    # flagged, no MOOD here): the flags must agree as well
    # without the dry demotion the random-field state breaks down within the
    # 20 steps (a dt turns invalid and the remaining steps do nothing): the
    # two marches must still agree on where
    assert ca.status == cb.status
    assert ca.steps == cb.steps
    if state == "dam":
        assert ca.steps == 20
    bits = torch.int64 if dtype == torch.float64 else torch.int32
    assert torch.equal(Qa.view(bits), Qb.view(bits)), \
        (Qa - Qb).abs().max().item()
    assert ca.t[20 % 3] == cb.t[20 % 3]


def test_bed_planes_are_the_interior_least_squares_gradient():
    """Planes 0 and 1 against the float64 central least-squares gradient of b
    (``(b[i+1, j-1..j+1] - b[i-1, j-1..j+1]).sum() / (6 dx)`` and its y twin)
    on interior cells, plane 2 in [0, 1]; boundary cells hold zeros."""
    lib = L.load()
    nx, ny = 96, 64
    xc = _centers(nx, ny)
    b = bumps(xc, seed=3)
    q = np.stack([b, np.ones_like(b), np.zeros_like(b), np.zeros_like(b)])
    Q = torch.as_tensor(q, dtype=torch.float32, device="cuda").contiguous()
    cfg = _cfg(nx, ny)
    bed = _prepare(lib, cfg, Q).view(torch.float32).cpu().numpy().reshape(3, nx, ny)
    B = Q[0].double().cpu().numpy().reshape(nx, ny)
    gx = (B[2:, :-2] + B[2:, 1:-1] + B[2:, 2:] - B[:-2, :-2] - B[:-2, 1:-1] - B[:-2, 2:]) \
        * nx / 6.0
    gy = (B[:-2, 2:] + B[1:-1, 2:] + B[2:, 2:] - B[:-2, :-2] - B[1:-1, :-2] - B[2:, :-2]) \
        * ny / 6.0
    scale = max(np.abs(gx).max(), np.abs(gy).max())
    assert np.abs(bed[0, 1:-1, 1:-1] - gx).max() <= 1e-5 * scale
    assert np.abs(bed[1, 1:-1, 1:-1] - gy).max() <= 1e-5 * scale
    phi = bed[2, 1:-1, 1:-1]
    assert phi.min() >= 0.0 and phi.max() <= 1.0 and phi.min() < 1.0
    ring = np.ones((nx, ny), dtype=bool)
    ring[1:-1, 1:-1] = False
    assert not bed[:, ring].any()


def test_bed_prepare_rejects_schemes_that_do_not_read_it():
    lib = L.load()
    cfg = _cfg(64, 64)
    cfg.riemann = L.RIEMANN["rusanov_hr"]
    assert lib.zb_swe2d_bed_bytes(C.byref(cfg)) == 0
    Q = torch.zeros((4, 64 * 64), dtype=torch.float32, device="cuda")
    bed = torch.empty(3 * 64 * 64 * 4, dtype=torch.uint8, device="cuda")
    rc = lib.zb_swe2d_bed_prepare(C.byref(cfg), L.ptr(Q), L.ptr(bed), C.c_size_t(bed.numel()),
                                  L.stream_ptr())
    assert rc == L.ZB_E_ARG
    cfg = _cfg(64, 64)
    rc = lib.zb_swe2d_bed_prepare(C.byref(cfg), L.ptr(Q), L.ptr(bed), C.c_size_t(100),
                                  L.stream_ptr())
    assert rc == L.ZB_E_ARG


def test_solver_prepares_again_after_a_torch_edit_of_the_bed():
    """The solver's march re-prepares the planes when the state tensor was
    modified from torch (here: a new bump added to ``Q[0]``) and matches a
    march that evaluates b's slope every stage."""
    import zoomy_b200 as zb
    from zoomy_b200.fvm.solver import HyperbolicSolver
    n = 128
    xc = _centers(n, n)
    q = circular_dam_state(xc, seed=9)
    tags = ("left", "right", "bottom", "top")
    model = zb.ShallowWater2D(wet_dry_eps=1e-6, initial_conditions=q,
                              boundary_conditions={t: "wall" for t in tags})
    nsm = zb.NumericalSystemModel.from_system_model(model, zb.ReconstructionSpec(2, "minmod"),
                                                    "hll_hr")
    out = []
    for use_bed in (True, False):
        s = HyperbolicSolver(time_end=float("inf"), compute_dt=zb.timestepping.adaptive(0.45, 2),
                             reconstruction_variables="eta", free_surface_h_index=1,
                             eps_wet=1e-6, dtype="float32")
        s.use_bed = use_bed
        Q, _ = s.setup_simulation(zb.create_2d((0.0, 1.0, 0.0, 1.0), n, n), nsm)
        assert bool(s.cfg.bed) == use_bed
        s.init_march(Q)
        s.launch_steps(Q, 5)
        Q[0] += torch.as_tensor(0.3 * np.exp(-((xc[0] - 0.3) ** 2 + (xc[1] - 0.6) ** 2) / 0.01),
                                dtype=Q.dtype, device=Q.device)
        s.launch_steps(Q, 5)
        torch.cuda.synchronize()
        out.append(Q.clone())
    assert torch.equal(out[0], out[1])

"""The allocation-free step against the workspace step.

``zb_swe2d_step_noalloc`` serves callers that cannot allocate device memory
(a plugin inside a framework that owns all device memory and hands it only
its operands): its stage scratch is a fixed array inside libzb instead of a
caller workspace.  This file is named to be collected last
so that a run stopping at the first failure has run every other test; it
also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from zoomy_b200 import _lib as L  # noqa: E402
from zoomy_b200.workloads import cartesian_centers, circular_dam_state  # noqa: E402


def _cfg(nx, ny, dtype, order=2):
    c = L.ZbSwe2dCfg()
    c.nx, c.ny = nx, ny
    c.x0, c.y0, c.dx, c.dy = 0.0, 0.0, 1.0 / nx, 1.0 / ny
    c.order, c.riemann, c.limiter = order, L.RIEMANN["hll_hr"], 0
    c.recon = L.RECON["eta"] if order == 2 else L.RECON["constant"]
    for i in range(4):
        c.bc[i] = L.BC["wall"]
    c.g, c.wet_dry_eps, c.eps_wet, c.manning_n = 9.81, 1e-6, 1e-6, 0.03
    c.implicit_source, c.dim_factor, c.cfl = 0, 2, 0.45
    c.dt_max, c.t_end, c.degree = float("inf"), float("inf"), 0
    c.dtype = L.ZB_F64 if dtype == torch.float64 else L.ZB_F32
    return c


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-6)])
def test_noalloc_step_matches_workspace_step(dtype, tol):
    lib = L.load()
    n = 256
    cfg = _cfg(n, n, dtype)
    q0 = torch.as_tensor(circular_dam_state(cartesian_centers(n), seed=2),
                         dtype=dtype, device="cuda").contiguous()
    stream = L.stream_ptr()
    Qa, Qb = q0.clone(), q0.clone()
    ctrl_a = torch.zeros(L.CTRL_BYTES, dtype=torch.uint8, device="cuda")
    ctrl_b = torch.zeros_like(ctrl_a)
    wsb = lib.zb_swe2d_workspace_bytes(C.byref(cfg))
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    for Q, ctrl in ((Qa, ctrl_a), (Qb, ctrl_b)):
        assert lib.zb_swe2d_init(C.byref(cfg), L.ptr(Q), L.ptr(ctrl), 0, 0.0, stream) == 0
    for call in range(2):
        rc = lib.zb_swe2d_step(C.byref(cfg), L.ptr(Qa), L.ptr(ws), C.c_size_t(wsb),
                               L.ptr(ctrl_a), call % 3, stream)
        assert rc == 0
        rc = lib.zb_swe2d_step_noalloc(C.byref(cfg), L.ptr(Qb), L.ptr(ctrl_b), call % 3, stream)
        assert rc == 0
        torch.cuda.synchronize()
        a = Qa.double().cpu().numpy()
        b = Qb.double().cpu().numpy()
        scale = np.abs(a).max(axis=1, keepdims=True)
        assert (np.abs(a - b) / scale).max() <= tol, f"call {call}"
        ca = L.ZbCtrl.from_buffer_copy(ctrl_a.cpu().numpy().tobytes())
        cb = L.ZbCtrl.from_buffer_copy(ctrl_b.cpu().numpy().tobytes())
        assert ca.status == 0 and cb.status == 0
        assert cb.dt == pytest.approx(ca.dt, rel=tol)


@pytest.mark.parametrize("n,order", [(1024, 2), (256, 1)], ids=["at-the-cap", "order-1"])
def test_noalloc_step_is_bitwise_the_workspace_step(n, order):
    """A grid of exactly ZB_NOALLOC_MAX_CELLS cells (the fixed array full)
    and the order-1 step (whose Euler stage writes the scratch and copies it
    back into Q): two calls in a row, float64, bit for bit against the
    workspace step."""
    lib = L.load()
    cfg = _cfg(n, n, torch.float64, order)
    q0 = torch.as_tensor(circular_dam_state(cartesian_centers(n), seed=4),
                         dtype=torch.float64, device="cuda").contiguous()
    stream = L.stream_ptr()
    Qa, Qb = q0.clone(), q0.clone()
    ctrl_a = torch.zeros(L.CTRL_BYTES, dtype=torch.uint8, device="cuda")
    ctrl_b = torch.zeros_like(ctrl_a)
    wsb = lib.zb_swe2d_workspace_bytes(C.byref(cfg))
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    for Q, ctrl in ((Qa, ctrl_a), (Qb, ctrl_b)):
        assert lib.zb_swe2d_init(C.byref(cfg), L.ptr(Q), L.ptr(ctrl), 0, 0.0, stream) == 0
    for call in range(2):
        assert lib.zb_swe2d_step(C.byref(cfg), L.ptr(Qa), L.ptr(ws), C.c_size_t(wsb),
                                 L.ptr(ctrl_a), call % 3, stream) == 0
        assert lib.zb_swe2d_step_noalloc(C.byref(cfg), L.ptr(Qb), L.ptr(ctrl_b),
                                         call % 3, stream) == 0
        torch.cuda.synchronize()
        assert torch.equal(Qa, Qb), f"call {call}"
        assert not torch.equal(Qb, q0)
        assert torch.equal(ctrl_a, ctrl_b), f"call {call}"


def test_noalloc_rejects_grids_beyond_its_scratch():
    lib = L.load()
    side = 1025                       # 1025^2 > ZB_NOALLOC_MAX_CELLS = 2^20
    cfg = _cfg(side, side, torch.float32)
    Q = torch.zeros((4, 8), dtype=torch.float32, device="cuda")
    ctrl = torch.zeros(L.CTRL_BYTES, dtype=torch.uint8, device="cuda")
    rc = lib.zb_swe2d_step_noalloc(C.byref(cfg), L.ptr(Q), L.ptr(ctrl), 0, L.stream_ptr())
    assert rc == L.ZB_E_TOO_LARGE

"""GPU triangle-mesh preparation (zb_trimesh_match / zb_trimesh_fill) against
the host builder (TriangleMesh.from_points) and the oracle.

The device numbers faces by (owner cell, local edge) with the lower cell index
owning a shared edge, the host by sorted vertex pair, so face-indexed arrays
are compared after mapping both to a canonical form (the face's two cells,
its normal out of the lower one); per-cell arrays are compared slot by slot
after ordering each cell's three stencil slots by neighbour.  Geometry is
float64 on both sides: 1e-14 relative for lengths, normals and offsets, 1e-12
for least-squares weights (a 2x2 closed-form inverse against numpy's LU).
The SWE step on a device-prepared mesh matches the oracle to 1e-12 per step.
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
from zoomy_b200.trimesh import DeviceTriangleMesh, TriangleMesh, lattice_triangulation  # noqa: E402
from zoomy_b200.workloads import circular_dam_state  # noqa: E402

TAGS = ("left", "right", "bottom", "top")
KINDS = [L.BC["wall"], L.BC["extrapolation"], L.BC["wall"], L.BC["extrapolation"]]


def host_np(d):
    return {k: v.cpu().numpy() for k, v in d.items()}


def canonical_faces(a):
    """Rows (lo cell, hi cell or -1, length, normal out of lo, offsets from
    lo / hi, inradius), sorted."""
    A, B = a["face_a"].astype(np.int64), a["face_b"].astype(np.int64)
    inner = B >= 0
    swap = inner & (B < A)
    lo = np.where(swap, B, A)
    hi = np.where(inner, np.where(swap, A, B), -1)
    sg = np.where(swap, -1.0, 1.0)
    rlx = np.where(swap, a["face_rbx"], a["face_rax"])
    rly = np.where(swap, a["face_rby"], a["face_ray"])
    rhx = np.where(swap, a["face_rax"], a["face_rbx"])
    rhy = np.where(swap, a["face_ray"], a["face_rby"])
    rows = np.stack([lo, hi, a["face_len"], sg * a["face_nx"], sg * a["face_ny"], rlx, rly,
                     rhx, rhy, a["face_inr"]], axis=1)
    return rows[np.lexsort((rows[:, 6], rows[:, 5], rows[:, 1], rows[:, 0]))]


def canonical_cells(a):
    """Per cell, its three slots (neighbour or -1, offsets, weights) ordered by
    (neighbour, offset x, offset y)."""
    idx = a["lsq_idx"].astype(np.int64)
    nb = np.where(idx >= 0, idx, -1)
    vals = np.stack([nb, a["cf_rx"], a["cf_ry"], a["lsq_wx"], a["lsq_wy"]], axis=-1)  # (3, C, 5)
    vals = np.transpose(vals, (1, 0, 2))                                             # (C, 3, 5)
    key = vals[:, :, 0] * 1e6 + vals[:, :, 1] * 1e3 + vals[:, :, 2]
    o = np.argsort(key, axis=1)
    return np.take_along_axis(vals, o[:, :, None], axis=1)


def close(a, b, rtol):
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() <= rtol * scale


@pytest.mark.parametrize("n_side,seed", [(12, 0), (41, 3)])
def test_device_preparation_matches_the_host_builder(n_side, seed):
    P, T = lattice_triangulation(n_side, seed=seed)
    host = TriangleMesh.from_points(P, T)
    dev = DeviceTriangleMesh(P, T)
    assert (dev.n_faces, dev.n_bf) == (host.n_faces, host.n_bf)
    ah = host_np(host.device_arrays(torch.float64, "cuda", KINDS))
    ad = host_np(dev.device_arrays(torch.float64, "cuda", KINDS))
    assert close(ad["cell_inv_area"], ah["cell_inv_area"], 1e-14)
    fh, fd = canonical_faces(ah), canonical_faces(ad)
    assert np.array_equal(fd[:, :2], fh[:, :2])
    for col in range(2, fh.shape[1]):
        assert close(fd[:, col], fh[:, col], 1e-14), col
    ch, cd = canonical_cells(ah), canonical_cells(ad)
    assert np.array_equal(cd[:, :, 0], ch[:, :, 0])
    assert close(cd[:, :, 1:3], ch[:, :, 1:3], 1e-14)
    assert close(cd[:, :, 3:5], ch[:, :, 3:5], 1e-12)
    # boundary faces: the same (kind, normal) multiset
    bh = np.stack([ah["bf_kind"], ah["bf_nx"], ah["bf_ny"]], 1)
    bd = np.stack([ad["bf_kind"][:dev.n_bf], ad["bf_nx"][:dev.n_bf], ad["bf_ny"][:dev.n_bf]], 1)
    bh = bh[np.lexsort(bh.T[::-1])]
    bd = bd[np.lexsort(bd.T[::-1])]
    assert np.array_equal(bd[:, 0], bh[:, 0]) and close(bd[:, 1:], bh[:, 1:], 1e-14)
    # cell -> face links agree with face owner / neighbour, faces increasing
    C = dev.n_cells
    cf = ad["cell_face"]
    f, side = cf >> 1, cf & 1
    cells = np.broadcast_to(np.arange(C), (3, C))
    assert np.all(np.where(side == 0, ad["face_a"][f], ad["face_b"][f]) == cells)
    assert np.all(np.diff(f, axis=0) > 0)
    # boundary numbers in face order
    bf = np.nonzero(ad["face_b"] < 0)[0]
    assert np.array_equal(-(ad["face_b"][bf] + 1), np.arange(dev.n_bf))


def test_orientation_and_precision():
    """Clockwise input triangles give the mesh of the counter-clockwise ones
    (their local edges start elsewhere, so compare canonical forms); the
    float32 arrays are the float64 ones rounded."""
    P, T = lattice_triangulation(16, seed=5)
    a = host_np(DeviceTriangleMesh(P, T).device_arrays(torch.float64, "cuda", KINDS))
    b = host_np(DeviceTriangleMesh(P, T[:, ::-1]).device_arrays(torch.float64, "cuda", KINDS))
    fa, fb = canonical_faces(a), canonical_faces(b)
    assert np.array_equal(fa[:, :2], fb[:, :2]) and close(fb[:, 2:], fa[:, 2:], 1e-14)
    ca, cb = canonical_cells(a), canonical_cells(b)
    assert np.array_equal(ca[:, :, 0], cb[:, :, 0]) and close(cb[:, :, 1:], ca[:, :, 1:], 1e-12)
    c = host_np(DeviceTriangleMesh(P, T).device_arrays(torch.float32, "cuda", KINDS))
    for k in a:
        if a[k].dtype == np.float64 and c[k].dtype == np.float32:
            assert np.array_equal(c[k], a[k].astype(np.float32)), k


def test_invalid_meshes_are_rejected():
    P = np.array([[0, 0], [1, 0], [0, 1], [0, -1], [1, 1]], dtype=np.float64)
    with pytest.raises(L.ZbError):      # edge (0, 1) shared by three triangles
        DeviceTriangleMesh(P, np.array([[0, 1, 2], [0, 1, 3], [1, 0, 4]]))
    with pytest.raises(L.ZbError):      # vertex index out of range
        DeviceTriangleMesh(P, np.array([[0, 1, 7]]))
    with pytest.raises(L.ZbError):      # zero-area triangle
        DeviceTriangleMesh(np.array([[0, 0], [1, 0], [2, 0]], dtype=np.float64),
                           np.array([[0, 1, 2]]))


def test_step_on_a_device_prepared_mesh_matches_the_oracle():
    """Five float64 SSP-RK2 steps (eta-MUSCL + Barth-Jespersen + HR-HLL, walls
    and extrapolation) on the device-prepared mesh against the oracle, which
    builds its own mesh from the same vertices and triangles."""
    P, T = lattice_triangulation(30, seed=2)
    mesh = DeviceTriangleMesh(P, T)
    bcs = dict(zip(TAGS, ("wall", "extrapolation", "wall", "extrapolation")))
    xc = mesh.cell_centers()
    Q0 = circular_dam_state(xc, seed=4, h_in=3.0, h_out=2.0)     # wet everywhere
    model = zb.ShallowWater2D(boundary_conditions=bcs, initial_conditions=Q0)
    nsm = zb.NumericalSystemModel.from_system_model(
        model, zb.ReconstructionSpec(2, "barth_jespersen"), "hll_hr")
    solver = HyperbolicSolver(time_end=math.inf, compute_dt=zb.timestepping.adaptive(0.45, 2),
                              reconstruction_variables="eta", free_surface_h_index=1,
                              dtype="float64")
    Q, _ = solver.setup_simulation(mesh, nsm)
    om = OM.tri_from_points(P, T)
    scheme = OS.Scheme(order=2, limiter="barth_jespersen", recon="eta", riemann="hll_hr",
                       cfl=0.45, bc=bcs)
    params = OS.Params()
    solver.init_march(Q)
    q = Q0.copy()
    for _ in range(5):
        solver.launch_steps(Q, 1)
        c = solver.read_ctrl()
        assert c.status == 0
        q = OS.step(om, q, c.dt, params, scheme)
        got = Q.cpu().numpy()
        err = max(np.abs(got[v] - q[v]).max() / max(np.abs(q[v]).max(), 1e-14) for v in range(4))
        assert err <= 1e-12

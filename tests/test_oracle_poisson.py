"""CPU checks of the Poisson and U-Net oracles (the checkers of the GPU
pressure solve and of the learned smoother's kernels).

The reference's elliptic operator is VAM's (absent zoomy_core), so the
Poisson oracle's parity with the reference is unpinned; its arbiter is the
float64 sparse direct solve, and these tests pin the oracle's own
multigrid/FCG against it.  The U-Net oracle's backward pass is pinned by
central finite differences."""
import numpy as np
import pytest

from oracle import poisson as OP
from oracle import unet as OU


def _coef(n, seed=0):
    rng = np.random.default_rng(seed)
    h = rng.uniform(0.0, 2.5, (n, n))
    return OP.face_coefficients(h)


def test_operator_is_symmetric_positive_definite():
    cx, cy = _coef(12)
    A = OP.matrix(cx, cy, 1.0 / 12).toarray()
    assert np.allclose(A, A.T, rtol=0, atol=1e-12 * np.abs(A).max())
    assert np.linalg.eigvalsh(A).min() > 0
    p = np.random.default_rng(1).standard_normal((12, 12))
    assert np.allclose(A @ p.reshape(-1), OP.apply(cx, cy, p, 1.0 / 12).reshape(-1))
    assert np.allclose(np.diag(A), OP.diagonal(cx, cy, 1.0 / 12).reshape(-1))


def test_prolongation_interpolates_and_restriction_is_its_transpose():
    P = OP.prolongation(4, 6)
    # interior fine cells reproduce a constant coarse field exactly
    e = np.ones(4 * 6)
    f = (P @ e).reshape(8, 12)
    assert np.allclose(f[1:-1, 1:-1], 1.0)
    # a cell on the wall sees the odd reflection of its x-neighbour:
    # 9/16 - 3/16 (reflected) + 3/16 - 1/16 (reflected diagonal) = 1/2
    assert np.isclose(f[0, 5], 0.5)
    assert P.shape == (8 * 12, 4 * 6)


def test_vcycle_is_symmetric():
    n = 32
    cx, cy = _coef(n, 2)
    H = OP.Hierarchy(cx, cy, 1.0 / n, coarsest=4)
    rng = np.random.default_rng(3)
    a, b = rng.standard_normal((2, n, n))
    Ma, Mb = OP.vcycle(H, a), OP.vcycle(H, b)
    assert abs(np.vdot(Ma, b) - np.vdot(a, Mb)) <= 1e-12 * abs(np.vdot(Ma, b))


def test_fcg_matches_direct_solve():
    n = 64
    cx, cy = _coef(n, 4)
    H = OP.Hierarchy(cx, cy, 1.0 / n, coarsest=4)
    b = np.random.default_rng(5).standard_normal((n, n))
    x, it, rel = OP.fcg(H, b, tol=1e-10, precond="mg")
    assert rel <= 1e-10 and it <= 20
    xd = OP.direct_solve(cx, cy, b, 1.0 / n)
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
    x2, it2, _ = OP.fcg(H, b, tol=1e-10, precond="none", maxit=5000)
    assert it2 > 5 * it
    assert np.linalg.norm(x2 - xd) <= 1e-8 * np.linalg.norm(xd)


def test_coarse_coefficients_average_covered_faces():
    cx, cy = _coef(8, 6)
    cxc, cyc = OP.coarsen_coefficients(cx, cy)
    assert cxc.shape == (5, 4) and cyc.shape == (4, 5)
    assert np.isclose(cxc[2, 1], 0.5 * (cx[4, 2] + cx[4, 3]))
    assert np.isclose(cyc[1, 2], 0.5 * (cy[2, 4] + cy[3, 4]))


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(7)
    w = np.concatenate([rng.standard_normal(4096).astype(np.float32),
                        np.float32([1.00390625, 1.01171875, -3.0e-39, 65504.0])])
    ours = OU.bf16_round(w)
    theirs = torch.as_tensor(w).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(ours, theirs)


@pytest.mark.parametrize("energy", [False, True], ids=["residual_loss", "energy_loss"])
def test_unet_backward_matches_finite_differences(energy):
    c1, c2 = 8, 16
    rng = np.random.default_rng(8)
    nw, nb = OU.param_counts(c1, c2)
    Ws, bs = OU.split(OU.bf16_round(rng.normal(0, 0.3, nw)), rng.normal(0, 0.1, nb), c1, c2)
    B, n = 2, 8
    r = rng.standard_normal((B, n, n))
    cx = rng.uniform(0.1, 2, (B, n + 1, n))
    cy = rng.uniform(0.1, 2, (B, n, n + 1))
    dx = 1.0 / n
    tgt = rng.standard_normal((B, n, n)) * dx ** 2 if energy else None
    lg = lambda W_, b_: OU.loss_and_grads(W_, b_, r, cx, cy, dx, 2.0, target=tgt)  # noqa: E731
    _, dWs, dbs = lg(Ws, bs)
    eps = 1e-6
    for layer in range(6):
        idx = tuple(int(rng.integers(0, s)) for s in Ws[layer].shape)
        Wp = [W.copy() for W in Ws]
        Wm = [W.copy() for W in Ws]
        Wp[layer][idx] += eps
        Wm[layer][idx] -= eps
        fd = (lg(Wp, bs)[0] - lg(Wm, bs)[0]) / (2 * eps)
        assert abs(fd - dWs[layer][idx]) <= 1e-6 * max(1.0, abs(fd))
        j = int(rng.integers(0, bs[layer].shape[0]))
        bp = [b.copy() for b in bs]
        bm = [b.copy() for b in bs]
        bp[layer][j] += eps
        bm[layer][j] -= eps
        fd = (lg(Ws, bp)[0] - lg(Ws, bm)[0]) / (2 * eps)
        assert abs(fd - dbs[layer][j]) <= 1e-6 * max(1.0, abs(fd))


def test_unet_output_is_homogeneous_in_the_residual():
    c1, c2 = 8, 16
    rng = np.random.default_rng(9)
    nw, nb = OU.param_counts(c1, c2)
    Ws, bs = OU.split(OU.bf16_round(rng.normal(0, 0.3, nw)), rng.normal(0, 0.1, nb), c1, c2)
    r = rng.standard_normal((1, 8, 8))
    cx = rng.uniform(0.1, 2, (1, 9, 8))
    cy = rng.uniform(0.1, 2, (1, 8, 9))
    y1, _ = OU.forward(Ws, bs, r, cx, cy, 0.1, 2.0)
    y2, _ = OU.forward(Ws, bs, 7.0 * r, cx, cy, 0.1, 2.0)
    assert np.allclose(y2, 7.0 * y1, rtol=1e-12, atol=0)
    assert OU.param_counts(24, 48) == (52488, 169)


def test_coefficient_variation_costs_at_most_one_iteration():
    """How much room a coefficient-aware learned component has: on a Chorin
    pressure problem (the first stage of the seeded dam break over bumps,
    128^2, c = clip(h, 0.1, 2) from 0.21 to 1.97) multigrid FCG needs 8
    iterations to 1e-8, and the same right-hand side with the coefficient
    replaced by a constant still needs 7.  A smoother or transfer operator
    that learned the coefficient field perfectly could therefore save about
    one iteration of eight; halving the count needs a V-cycle that contracts
    ~100x instead of ~7x, i.e. a stronger cycle, not a coefficient-aware one."""
    import sys
    import pathlib
    sys.path.insert(0, str(pathlib.Path(__file__).resolve().parent.parent / "zoomy-jax_b200"))
    from oracle import mesh as OM
    from oracle import swe as OS
    from zoomy_b200.workloads import cartesian_centers, circular_dam_state
    n = 128
    tags = ("left", "right", "bottom", "top")
    Q0 = circular_dam_state(cartesian_centers(n), seed=0)
    om = OM.create_2d(0.0, 1.0, 0.0, 1.0, n, n)
    sc = OS.Scheme(order=2, recon="eta", riemann="hll_hr", cfl=0.45,
                   bc={t: "wall" for t in tags}, eps_wet=1e-6)
    p = OS.Params(wet_dry_eps=1e-6)
    dt = OS.compute_dt(om, Q0, p, sc)
    Qs = Q0 + dt * OS.flux_operator(om, Q0, sc, p, OS.bc_kinds(om, sc))
    dx = 1.0 / n
    b = OP.divergence_rhs(Qs[2].reshape(n, n), Qs[3].reshape(n, n), dt, dx)
    cx, cy = OP.face_coefficients(Qs[1].reshape(n, n))
    _, it_var, rel_var = OP.fcg(OP.Hierarchy(cx, cy, dx, coarsest=4), b, tol=1e-8)
    ones = (np.ones_like(cx), np.ones_like(cy))
    _, it_const, rel_const = OP.fcg(OP.Hierarchy(*ones, dx, coarsest=4), b, tol=1e-8)
    assert rel_var <= 1e-8 and rel_const <= 1e-8
    assert it_var == 8 and it_const == 7, (it_var, it_const)

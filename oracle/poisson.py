"""Float64 oracle of the Chorin pressure solve -- TEST INFRASTRUCTURE ONLY.

The reference's Chorin projection (``zoomy_jax/fvm/solver_chorin_vam_jax.py``:
``chorin_stage`` :524-572, ``_step_pressure_pure`` :673-883,
``_step_corrector_pure`` :885-907) runs hyperbolic Euler -> pressure solve ->
corrector, with VAM's elliptic operator generated by the absent zoomy_core and
solved by unpreconditioned restarted GMRES to ``pressure_tol``.  The operator
here is the variable-coefficient Poisson problem the configuration names
(coefficient from the depth, clipped to [0.1, 2]); parity with the reference's
operator is therefore unpinned and the arbiter of the solution is the float64
sparse direct solve below.

Discretisation on an ``nx x ny`` Cartesian grid with spacing ``dx = dy``:
* face coefficients: harmonic mean of ``c = clip(h, cmin, cmax)`` of the two
  cells; at a boundary face the boundary cell's ``c``;
* ``(A p)_i = sum_f c_f (p_i - p_j) / dx^2`` with the Dirichlet ghost
  ``p_j = -p_i`` (p = 0 on the boundary) -- symmetric positive definite;
* ``f = -div(q*) / dt`` with face fluxes ``(q*_L + q*_R) . n / 2`` and zero
  flux through walls;
* corrector ``q = q* - dt * (c_f (p_R - p_L) / dx averaged over the cell's two
  faces along each axis)``.

Multigrid: cell-centred, factor-2 coarsening, coarse face coefficient = mean
of the two fine face coefficients it covers, bilinear prolongation ``P`` (odd
reflection at the Dirichlet boundary), restriction ``R = P^T / 4``, red-black
Gauss-Seidel smoothing (pre: red, black; post: black, red), a symmetric
coarsest solve, V-cycle, flexible CG (one-term Notay FCG).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


# ── operator ────────────────────────────────────────────────────────────────

def face_coefficients(h, cmin=0.1, cmax=2.0):
    """``cx (nx+1, ny)``, ``cy (nx, ny+1)`` from the cell depth ``h (nx, ny)``."""
    c = np.clip(h, cmin, cmax)
    nx, ny = c.shape
    cx = np.empty((nx + 1, ny))
    cy = np.empty((nx, ny + 1))
    cx[1:-1] = 2.0 * c[:-1] * c[1:] / (c[:-1] + c[1:])
    cx[0] = c[0]
    cx[-1] = c[-1]
    cy[:, 1:-1] = 2.0 * c[:, :-1] * c[:, 1:] / (c[:, :-1] + c[:, 1:])
    cy[:, 0] = c[:, 0]
    cy[:, -1] = c[:, -1]
    return cx, cy


def diagonal(cx, cy, dx):
    """Diagonal of A: interior faces c_f / dx^2, boundary faces 2 c_f / dx^2."""
    nx, ny = cx.shape[0] - 1, cy.shape[1] - 1
    d = np.zeros((nx, ny))
    d += cx[1:] + cx[:-1]
    d += cy[:, 1:] + cy[:, :-1]
    d[0, :] += cx[0]
    d[-1, :] += cx[-1]
    d[:, 0] += cy[:, 0]
    d[:, -1] += cy[:, -1]
    return d / dx ** 2


def apply(cx, cy, p, dx):
    """``A p`` (Dirichlet zero ghost -p)."""
    pp = np.pad(p, 1)
    pp[0, :] = -pp[1, :]
    pp[-1, :] = -pp[-2, :]
    pp[:, 0] = -pp[:, 1]
    pp[:, -1] = -pp[:, -2]
    pc = pp[1:-1, 1:-1]
    out = (cx[1:] * (pc - pp[2:, 1:-1]) + cx[:-1] * (pc - pp[:-2, 1:-1])
           + cy[:, 1:] * (pc - pp[1:-1, 2:]) + cy[:, :-1] * (pc - pp[1:-1, :-2]))
    return out / dx ** 2


def matrix(cx, cy, dx):
    """Sparse CSR of A (for the direct solve that arbitrates)."""
    nx, ny = cx.shape[0] - 1, cy.shape[1] - 1
    N = nx * ny
    idx = np.arange(N).reshape(nx, ny)
    rows, cols, vals = [], [], []
    d = diagonal(cx, cy, dx).reshape(-1)
    rows.append(idx.reshape(-1)); cols.append(idx.reshape(-1)); vals.append(d)
    w = -cx[1:-1] / dx ** 2
    rows += [idx[:-1].reshape(-1), idx[1:].reshape(-1)]
    cols += [idx[1:].reshape(-1), idx[:-1].reshape(-1)]
    vals += [w.reshape(-1), w.reshape(-1)]
    w = -cy[:, 1:-1] / dx ** 2
    rows += [idx[:, :-1].reshape(-1), idx[:, 1:].reshape(-1)]
    cols += [idx[:, 1:].reshape(-1), idx[:, :-1].reshape(-1)]
    vals += [w.reshape(-1), w.reshape(-1)]
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(N, N))


def divergence_rhs(qx, qy, dt, dx):
    """``f = -div(q*) / dt`` with average face fluxes and walls."""
    fx = np.zeros((qx.shape[0] + 1, qx.shape[1]))
    fy = np.zeros((qy.shape[0], qy.shape[1] + 1))
    fx[1:-1] = 0.5 * (qx[:-1] + qx[1:])
    fy[:, 1:-1] = 0.5 * (qy[:, :-1] + qy[:, 1:])
    div = (fx[1:] - fx[:-1] + fy[:, 1:] - fy[:, :-1]) / dx
    return -div / dt


def corrector(qx, qy, p, cx, cy, dt, dx):
    """``q = q* - dt * cell average of the face terms c_f grad_f p``."""
    pp = np.pad(p, 1)
    pp[0, :] = -pp[1, :]
    pp[-1, :] = -pp[-2, :]
    pp[:, 0] = -pp[:, 1]
    pp[:, -1] = -pp[:, -2]
    gx = cx * (pp[1:, 1:-1] - pp[:-1, 1:-1]) / dx      # (nx+1, ny)
    gy = cy * (pp[1:-1, 1:] - pp[1:-1, :-1]) / dx      # (nx, ny+1)
    return (qx - dt * 0.5 * (gx[1:] + gx[:-1]), qy - dt * 0.5 * (gy[:, 1:] + gy[:, :-1]))


# ── multigrid ───────────────────────────────────────────────────────────────

def coarsen_coefficients(cx, cy):
    """Coarse face coefficient = mean of the two fine faces it covers."""
    return (0.5 * (cx[0::2, 0::2] + cx[0::2, 1::2]),
            0.5 * (cy[0::2, 0::2] + cy[1::2, 0::2]))


def prolongation(nxc, nyc):
    """Sparse bilinear cell-centred prolongation (coarse -> fine) with odd
    reflection (Dirichlet zero) at the boundary: fine cell (2I+a, 2J+b) takes
    9/16 of coarse (I, J), 3/16 of the x- and y-neighbour on its side and
    1/16 of the diagonal one; a neighbour outside the grid contributes its
    weight with a minus sign to (I, J) itself."""
    nxf, nyf = 2 * nxc, 2 * nyc
    rows, cols, vals = [], [], []
    for a in (0, 1):
        for b in (0, 1):
            I, J = np.meshgrid(np.arange(nxc), np.arange(nyc), indexing="ij")
            fi = (2 * I + a) * nyf + (2 * J + b)
            sx = -1 if a == 0 else 1
            sy = -1 if b == 0 else 1
            for di, dj, w in ((0, 0, 9 / 16), (sx, 0, 3 / 16), (0, sy, 3 / 16), (sx, sy, 1 / 16)):
                ci, cj = I + di, J + dj
                inside = (ci >= 0) & (ci < nxc) & (cj >= 0) & (cj < nyc)
                sign = np.ones_like(I, dtype=float)
                # a neighbour outside the grid is the odd reflection of the
                # in-range cell on that side: -e(I or clipped, J or clipped)
                outx = (ci < 0) | (ci >= nxc)
                outy = (cj < 0) | (cj >= nyc)
                ci = np.where(outx, I, ci)
                cj = np.where(outy, J, cj)
                sign = np.where(outx, -sign, sign)
                sign = np.where(outy, -sign, sign)
                rows.append(fi.reshape(-1))
                cols.append((ci * nyc + cj).reshape(-1))
                vals.append((w * sign).reshape(-1))
                del inside
    P = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(nxf * nyf, nxc * nyc))
    P.sum_duplicates()
    return P


class Hierarchy:
    """Levels of (cx, cy, dx) down to a ``coarsest`` side."""

    def __init__(self, cx, cy, dx, coarsest=8):
        self.levels = [(cx, cy, dx)]
        while True:
            cx, cy, dx = self.levels[-1]
            nx, ny = cx.shape[0] - 1, cy.shape[1] - 1
            if nx <= coarsest or ny <= coarsest or nx % 2 or ny % 2:
                break
            cxc, cyc = coarsen_coefficients(cx, cy)
            self.levels.append((cxc, cyc, 2 * dx))
        self.P = []
        for cx, cy, dx in self.levels[1:]:
            nxc, nyc = cx.shape[0] - 1, cy.shape[1] - 1
            self.P.append(prolongation(nxc, nyc))
        self.diag = [diagonal(cx, cy, dx) for cx, cy, dx in self.levels]


def rbgs(x, f, cx, cy, dx, diag, color):
    """One Gauss-Seidel half-sweep on cells with (i + j) % 2 == color."""
    nx, ny = x.shape
    I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    mask = ((I + J) % 2) == color
    r = f - apply(cx, cy, x, dx)
    x = x.copy()
    x[mask] += r[mask] / diag[mask]
    return x


DENSE_MAX_CELLS = 64


def vcycle(H, f, level=0, nu=2, coarse_sweeps=40, smoother=None):
    """Symmetric V-cycle for ``A x = f`` from x = 0: the coarsest level is
    solved exactly when it has at most 64 cells, else by ``coarse_sweeps``
    symmetric red-black sweep pairs.  ``smoother(x, f, pre)`` replaces the
    level-0 pre/post smoothing when given (the learned path)."""
    cx, cy, dx = H.levels[level]
    d = H.diag[level]
    x = np.zeros_like(f)
    if level == len(H.levels) - 1:
        if f.size <= DENSE_MAX_CELLS:
            # exact coarsest solve (the device inverts this level at set-up)
            return np.linalg.solve(matrix(cx, cy, dx).toarray(), f.reshape(-1)).reshape(f.shape)
        for _ in range(coarse_sweeps):
            x = rbgs(x, f, cx, cy, dx, d, 0)
            x = rbgs(x, f, cx, cy, dx, d, 1)
        for _ in range(coarse_sweeps):
            x = rbgs(x, f, cx, cy, dx, d, 1)
            x = rbgs(x, f, cx, cy, dx, d, 0)
        return x
    if smoother is not None and level == 0:
        x = smoother(x, f, pre=True)
    else:
        for _ in range(nu):
            x = rbgs(x, f, cx, cy, dx, d, 0)
            x = rbgs(x, f, cx, cy, dx, d, 1)
    r = f - apply(cx, cy, x, dx)
    P = H.P[level]
    nxc, nyc = H.levels[level + 1][0].shape[0] - 1, H.levels[level + 1][1].shape[1] - 1
    fc = (P.T @ r.reshape(-1) / 4.0).reshape(nxc, nyc)
    ec = vcycle(H, fc, level + 1, nu, coarse_sweeps, smoother)
    x = x + (P @ ec.reshape(-1)).reshape(x.shape)
    if smoother is not None and level == 0:
        x = smoother(x, f, pre=False)
    else:
        for _ in range(nu):
            x = rbgs(x, f, cx, cy, dx, d, 1)
            x = rbgs(x, f, cx, cy, dx, d, 0)
    return x


def fcg(H, b, tol=1e-8, maxit=200, precond="mg", smoother=None, x0=None):
    """Flexible CG (Notay, one-term) with the V-cycle preconditioner
    (``precond='none'`` = plain CG).  Returns ``(x, iterations, rel_res)``;
    the relative residual ``||b - A x|| / ||b||`` is evaluated in float64."""
    cx, cy, dx = H.levels[0]
    x = np.zeros_like(b) if x0 is None else x0.copy()
    r = b - apply(cx, cy, x, dx)
    nb = np.linalg.norm(b)
    if nb == 0.0:
        return x, 0, 0.0
    M = (lambda v: vcycle(H, v, smoother=smoother)) if precond == "mg" else (lambda v: v)
    z = M(r)
    p = z.copy()
    it = 0
    rel = np.linalg.norm(r) / nb
    while rel > tol and it < maxit:
        q = apply(cx, cy, p, dx)
        pq = np.vdot(p, q)
        alpha = np.vdot(p, r) / pq
        x = x + alpha * p
        r = r - alpha * q
        it += 1
        rel = np.linalg.norm(r) / nb
        if rel <= tol:
            break
        z = M(r)
        beta = np.vdot(z, q) / pq
        p = z - beta * p
    return x, it, rel


def direct_solve(cx, cy, b, dx):
    """The float64 sparse direct solve -- the arbiter of the pressure."""
    A = matrix(cx, cy, dx)
    return spla.spsolve(A.tocsc(), b.reshape(-1)).reshape(b.shape)

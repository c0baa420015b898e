"""Float64 NumPy restatement of zoomy_jax's explicit shallow-water step.

TEST INFRASTRUCTURE ONLY -- the checker the CUDA path is compared with.  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline legs
may import this module.

State layout is the reference's SME(level=0) state, cell axis last:
``Q (n_state, C)`` with rows ``[b, h, q_1, .., q_dim]``
(``tests/spmd/test_spmd_real_solver.py:49-58`` in the reference; the golden
``swe_2d.npz`` is ``(4, 1024)``).  ``Qaux`` for the derivative-aux diagnostics
has rows ``[dq_1/dx_1, dh/dx_1, (dq_2/dx_2, dh/dx_2,) db/dx_1(, db/dx_2), hinv]``
(pinned against ``swe_2d.npz`` (7 rows) and ``stoker_wet.npz`` (4 rows)).

Every function cites the reference lines it restates.  Where the arithmetic
lives in the absent ``zoomy_core`` (HLL, hydrostatic reconstruction, Manning),
the published method is named instead.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

EPS_LIM = 1e-30      # limiter branch threshold, reconstruction_jax.py:603-691


@dataclass
class Params:
    """Physical parameters of the derived SWE (zoomy_core owns the values;
    the goldens are reproduced with ``manning_n = 0``)."""
    g: float = 9.81
    manning_n: float = 0.0
    wet_dry_eps: float = 1e-8        # KP desingularisation (solver_jax.py:291-292)


@dataclass
class Scheme:
    """Numerical knobs (``HyperbolicSolver`` params, solver_jax.py:183-226, and
    the NSM ``ReconstructionSpec(order, limiter)``)."""
    order: int = 1
    limiter: str = "minmod"              # minmod | barth_jespersen | venkatakrishnan | none
    recon: str = "conservative"          # conservative | eta
    riemann: str = "rusanov"             # rusanov | rusanov_hr | hll_hr
    eps_wet: Optional[float] = None      # eta: dry-cell demotion (emitted wet_dry_eps)
    positivity: Optional[str] = None     # eta: None | "zhang_shu"
    front_tol: Optional[float] = None    # eta: front pre-detector
    mood: bool = False                   # a-posteriori order-1 redo
    mood_mode: str = "cell"              # cell: demote the troubled cells | step: whole step
    cfl: float = 0.9
    dt_max: float = np.inf
    degree: int = 0                      # (2k+1) factor of the CFL law
    bc: dict = field(default_factory=dict)   # tag -> extrapolation | wall | periodic
    source: str = "explicit"             # explicit | implicit (point-implicit Manning)


# ── aux ─────────────────────────────────────────────────────────────────────

def kp_hinv(h, eps):
    """KP-desingularised inverse depth ``hinv = sqrt(2) h / sqrt(h^4 +
    max(h, eps)^4)`` (``zoomy_jax/fvm/solver_jax.py:291-292``)."""
    return np.sqrt(2.0) * h / np.sqrt(h ** 4 + np.maximum(h, eps) ** 4)


def velocities(Q, hinv):
    """``u = hinv * q`` per momentum row (the emitted map of
    ``reconstruction_jax.py:1000-1010``: ``W = (b, b + h, hinv q)``)."""
    return Q[2:] * hinv[None, :]


# ── boundary conditions ─────────────────────────────────────────────────────

def bc_kinds(mesh, scheme):
    """Per-boundary-face BC kind (0 extrapolation, 1 wall, 2 periodic).  A
    periodic side is paired with its opposite side (``resolve_periodic_bcs``,
    ``zoomy_jax/fvm/solver_jax.py:931-941``) the first time it is seen."""
    kinds = []
    for t in mesh.tag_names:
        kinds.append(scheme.bc.get(t, "extrapolation"))
    out = np.array([{"extrapolation": 0, "wall": 1, "periodic": 2}[k]
                    for k in kinds])[mesh.bf_tag]
    per = out == 2
    if per.any() and (mesh.bf_partner is None or (mesh.bf_partner[per] < 0).any()):
        opposite = {"left": "right", "right": "left", "bottom": "top", "top": "bottom"}
        pairs = [(t, opposite[t]) for t, k in zip(mesh.tag_names, kinds)
                 if k == "periodic"]
        mesh.set_periodic(pairs)
    return out


def apply_bc(mesh, kind, q, normals):
    """Ghost state of the indexed BC kernel (``solver2/blocks.py:129-157``):
    extrapolation copies, a wall mirrors the normal momentum
    (``q -> q - 2 (q.n) n``, the reference's ``Wall`` "mirrors q -> -q").
    ``q`` is ``(n_state, n_bf)``, ``normals`` ``(dim, n_bf)``."""
    out = q.copy()
    wall = kind == 1
    if wall.any():
        mom = q[2:, wall]
        qn = (mom * normals[:, wall]).sum(axis=0)
        out[2:, wall] = mom - 2.0 * qn[None, :] * normals[:, wall]
    return out


def halo_bc(mesh, Q, kind):
    """``bf_values (n_state, n_bf)`` -- BC at the owner cell state; at a
    periodic seam the partner cell's state (``solver2/blocks.py:129-157``)."""
    nrm = mesh.face_normals[:, mesh.bf]
    bfv = apply_bc(mesh, kind, Q[:, mesh.bf_cell], nrm)
    per = kind == 2
    if per.any():
        bfv[:, per] = Q[:, mesh.bf_partner[per]]
    return bfv


# ── LSQ gradient, bounds, limiters ──────────────────────────────────────────

def lsq_gradient(mesh, u, u_bf=None):
    """Cell gradient ``(dim, C)`` from the stencil weights
    (``reconstruction_jax.py:433-522``; ``mesh/mesh.py:74-120``).  A boundary
    ghost enters as ``u_bf - u_i`` (already ghost semantics, no second lift,
    ``reconstruction_jax.py:475-498``); ``u_bf=None`` means extrapolation
    (zero delta)."""
    idx = mesh.lsq_idx
    C = mesh.n_cells
    rows = np.repeat(np.arange(C), np.diff(mesh.lsq_ptr))
    val = np.empty(len(idx))
    cell = idx >= 0
    val[cell] = u[idx[cell]]
    if u_bf is None:
        val[~cell] = u[rows[~cell]]
    else:
        val[~cell] = u_bf[-idx[~cell] - 1]
    delta = val - u[rows]
    g = np.zeros((mesh.dim, C))
    for d in range(mesh.dim):
        g[d] = np.bincount(rows, weights=mesh.lsq_w[d] * delta, minlength=C)
    return g


def neighbor_bounds(mesh, u, u_bf):
    """``(u_min, u_max)`` over face neighbours; a boundary face contributes
    the ghost value ``2 u_bf - u_cell`` (``reconstruction_jax.py:535-579``)."""
    fc = mesh.face_cells
    it = mesh.interior
    A, B = fc[0, it], fc[1, it]
    umax = u.copy()
    umin = u.copy()
    np.maximum.at(umax, A, u[B])
    np.maximum.at(umax, B, u[A])
    np.minimum.at(umin, A, u[B])
    np.minimum.at(umin, B, u[A])
    ghost = 2.0 * u_bf - u[mesh.bf_cell]
    np.maximum.at(umax, mesh.bf_cell, ghost)
    np.minimum.at(umin, mesh.bf_cell, ghost)
    return umin, umax


def _face_offsets(mesh):
    fc = mesh.face_cells
    it = mesh.interior
    xc = mesh.cell_centers
    fcen = mesh.face_centers
    rA = (fcen[it] - xc[fc[0, it]]).T           # (dim, F_int)
    rB = (fcen[it] - xc[fc[1, it]]).T
    rbnd = (fcen[mesh.bf] - xc[mesh.bf_cell]).T
    return it, rA, rB, rbnd


def _cand(limiter, delta, dpos, dneg, ev2):
    """Per-face limiter candidate (``reconstruction_jax.py:603-691``).  The
    reference's ``minmod`` and ``barth_jespersen`` are the same clip-min form."""
    if limiter in ("minmod", "barth_jespersen"):
        rp = dpos / np.maximum(delta, EPS_LIM)
        rn = dneg / np.minimum(delta, -EPS_LIM)
        return np.where(delta > EPS_LIM, np.clip(rp, 0.0, 1.0),
                        np.where(delta < -EPS_LIM, np.clip(rn, 0.0, 1.0), 1.0))
    if limiter == "venkatakrishnan":
        num_p = dpos ** 2 + ev2 + 2 * delta * dpos
        den_p = dpos ** 2 + 2 * delta ** 2 + delta * dpos + ev2
        cp = np.clip(num_p / np.maximum(den_p, EPS_LIM), 0.0, 1.0)
        num_n = dneg ** 2 + ev2 + 2 * delta * dneg
        den_n = dneg ** 2 + 2 * delta ** 2 + delta * dneg + ev2
        cn = np.clip(-num_n / np.minimum(den_n, -EPS_LIM), 0.0, 1.0)
        return np.where(delta > EPS_LIM, cp, np.where(delta < -EPS_LIM, cn, 1.0))
    raise ValueError(limiter)


def limiter_phi(mesh, limiter, u, grad, umin, umax):
    """``phi (C,)`` = min over the cell's faces of the per-face candidate,
    clipped to [0, 1] (``reconstruction_jax.py:603-706``)."""
    C = mesh.n_cells
    if limiter == "none":
        return np.ones(C)
    it, rA, rB, rbnd = _face_offsets(mesh)
    fc = mesh.face_cells
    ev2 = (mesh.cell_volumes ** (1.0 / mesh.dim)) ** 2   # reconstruction_jax.py:396-399
    phi = np.ones(C)
    for cells, r in ((fc[0, it], rA), (fc[1, it], rB), (mesh.bf_cell, rbnd)):
        delta = (grad[:, cells] * r).sum(axis=0)
        cand = _cand(limiter, delta, umax[cells] - u[cells],
                     umin[cells] - u[cells], ev2[cells])
        np.minimum.at(phi, cells, cand)
    return np.clip(phi, 0.0, 1.0)


def face_values(mesh, U, slope, bf_vals):
    """Linear extrapolation to face centres (``reconstruction_jax.py:710-740``).
    ``U (n, C)``, ``slope (n, dim, C)`` = phi * grad.  Returns ``(U_L, U_R)``
    of shape ``(n, F)``; boundary ``U_R`` = ``bf_vals``."""
    it, rA, rB, rbnd = _face_offsets(mesh)
    fc = mesh.face_cells
    n = U.shape[0]
    UL = np.zeros((n, mesh.n_faces))
    UR = np.zeros((n, mesh.n_faces))
    A, B = fc[0, it], fc[1, it]
    UL[:, it] = U[:, A] + (slope[:, :, A] * rA[None]).sum(axis=1)
    UR[:, it] = U[:, B] + (slope[:, :, B] * rB[None]).sum(axis=1)
    c = mesh.bf_cell
    UL[:, mesh.bf] = U[:, c] + (slope[:, :, c] * rbnd[None]).sum(axis=1)
    UR[:, mesh.bf] = bf_vals
    return UL, UR


def pp_theta(mesh, h_bar, h_slope, eps=1e-14):
    """Xing-Zhang-Shu indicator: theta so that ``min_face(h_bar + slope.r) >=
    0`` (``reconstruction_jax.py:816-850``)."""
    C = mesh.n_cells
    rows = np.repeat(np.arange(C), np.diff(mesh.cf_ptr))
    r = mesh.face_centers[mesh.cf_idx].T - mesh.cell_centers[rows].T
    delta = (h_slope[:, rows] * r).sum(axis=0)
    hmin = np.full(C, np.inf)
    np.minimum.at(hmin, rows, h_bar[rows] + delta)
    denom = np.maximum(h_bar - hmin, eps)
    return np.where(hmin < 0.0, np.clip(h_bar / denom, 0.0, 1.0), 1.0)


# ── reconstructions ─────────────────────────────────────────────────────────

@dataclass
class Faces:
    """Face traces.  ``b, h (F,)``, ``q, u (dim, F)`` per side."""
    bL: np.ndarray
    hL: np.ndarray
    qL: np.ndarray
    uL: np.ndarray
    bR: np.ndarray
    hR: np.ndarray
    qR: np.ndarray
    uR: np.ndarray


def reconstruct(mesh, Q, scheme, params, kind, force_o1=None):
    """Face traces for one flux evaluation, with the boundary ``Q_R`` already
    replaced by ``BC(Q_L)`` (partner cell at a periodic seam), as the flux pass
    does (``solver_jax.py:827-858``, ``solver2/blocks.py:160-238``).

    Velocities: on the constant / conservative paths ``u = q * hinv`` with the
    CELL aux of the face's owner / neighbour (the flux pass hands the numerical
    flux ``Qaux[:, iA]`` and ``Qaux[:, iB]``, and the inner cell's aux on both
    sides of a boundary face, ``solver_jax.py:790-802, 827-866``); on the
    eta path ``u`` is the reconstructed primitive velocity itself.
    """
    dim = mesh.dim
    fc = mesh.face_cells
    hinv = kp_hinv(Q[1], params.wet_dry_eps)
    bfv = halo_bc(mesh, Q, kind)
    nrm_b = mesh.face_normals[:, mesh.bf]
    per = kind == 2
    if scheme.order < 2 or scheme.recon == "constant":
        slope = None
        QL, QR = face_values(mesh, Q, np.zeros((Q.shape[0], dim, Q.shape[1])), bfv)
    elif scheme.recon == "conservative":
        n = Q.shape[0]
        slope = np.zeros((n, dim, mesh.n_cells))
        for v in range(n):
            g = lsq_gradient(mesh, Q[v], bfv[v])
            umin, umax = neighbor_bounds(mesh, Q[v], bfv[v])
            phi = limiter_phi(mesh, scheme.limiter, Q[v], g, umin, umax)
            slope[v] = phi[None, :] * g
        QL, QR = face_values(mesh, Q, slope, bfv)
    elif scheme.recon == "eta":
        return _reconstruct_eta(mesh, Q, scheme, params, kind, bfv, force_o1)
    else:
        raise ValueError(scheme.recon)
    # boundary Q_R = BC(Q_L) at the reconstructed face state; partner at seam
    QRb = apply_bc(mesh, kind, QL[:, mesh.bf], nrm_b)
    if per.any():
        QRb[:, per] = Q[:, mesh.bf_partner[per]]
    QR[:, mesh.bf] = QRb
    iB = mesh.iB_or_owner
    uL = QL[2:] * hinv[fc[0]][None]
    uR = QR[2:] * hinv[iB][None]
    return Faces(QL[0], QL[1], QL[2:], uL, QR[0], QR[1], QR[2:], uR), slope


def _reconstruct_eta(mesh, Q, scheme, params, kind, bfv, force_o1):
    """Emitted-W reconstruction ``EmittedWLSQMUSCLJAX._eta_core``
    (``reconstruction_jax.py:1134-1292``) for SWE: ``W = (b, eta = b + h,
    u = hinv q)``; limiter on W; optional dry demotion (``eps_wet``); tie
    ``phi_b, phi_u <= phi_eta``; front pre-detector; optional Zhang-Shu cap;
    MOOD ``force_o1``; Audusse clip ``eta_f = max(eta_f, b_f)``; inverse map
    ``h_f = eta_f - b_f``, ``q_f = u_f h_f``."""
    dim = mesh.dim
    eps = params.wet_dry_eps
    hinv = kp_hinv(Q[1], eps)
    W = np.concatenate([Q[0:1], (Q[0] + Q[1])[None], velocities(Q, hinv)])
    bhinv = kp_hinv(bfv[1], eps)
    bfW = np.concatenate([bfv[0:1], (bfv[0] + bfv[1])[None], bfv[2:] * bhinv[None]])
    n = W.shape[0]
    grads = np.zeros((n, dim, mesh.n_cells))
    phi = np.ones((n, mesh.n_cells))
    for v in range(n):
        grads[v] = lsq_gradient(mesh, W[v], bfW[v])
        umin, umax = neighbor_bounds(mesh, W[v], bfW[v])
        phi[v] = limiter_phi(mesh, scheme.limiter, W[v], grads[v], umin, umax)
    if scheme.eps_wet is not None:
        dry = Q[1] < scheme.eps_wet
        phi[:, dry] = 0.0
    for v in [0] + list(range(2, n)):
        phi[v] = np.minimum(phi[v], phi[1])
    o1 = None if force_o1 is None else force_o1.copy()
    if scheme.front_tol is not None:
        sh0 = phi[1][None] * grads[1] - phi[0][None] * grads[0]
        th = pp_theta(mesh, Q[1], sh0)
        front = th < scheme.front_tol
        o1 = front if o1 is None else (o1 | front)
    if scheme.positivity == "zhang_shu":
        bslope = phi[0][None] * grads[0]
        sh = phi[1][None] * grads[1] - bslope
        th = pp_theta(mesh, Q[1], sh)
        grads[1] = bslope + th[None] * sh
        phi[1] = 1.0
        for v in range(2, n):
            phi[v] = phi[v] * th
    if o1 is not None:
        phi[:, o1] = 0.0
    slope = phi[:, None, :] * grads
    WL, WR = face_values(mesh, W, slope, bfW)
    WL[1] = np.maximum(WL[1], WL[0])
    WR[1] = np.maximum(WR[1], WR[0])
    hL = WL[1] - WL[0]
    hR = WR[1] - WR[0]
    qL = WL[2:] * hL[None]
    qR = WR[2:] * hR[None]
    uL = WL[2:].copy()
    uR = WR[2:].copy()
    # boundary Q_R = BC(Q_L): same b and h, reflected momentum / velocity
    nrm_b = mesh.face_normals[:, mesh.bf]
    QLb = np.concatenate([WL[0:1, mesh.bf], hL[None, mesh.bf], qL[:, mesh.bf]])
    QRb = apply_bc(mesh, kind, QLb, nrm_b)
    ULb = apply_bc(mesh, kind, np.concatenate([QLb[:2], uL[:, mesh.bf]]), nrm_b)[2:]
    per = kind == 2
    if per.any():
        pc = mesh.bf_partner[per]
        QRb[:, per] = Q[:, pc]
        ULb[:, per] = velocities(Q[:, pc], hinv[pc])
    bR = WR[0].copy()
    bR[mesh.bf] = QRb[0]
    hR[mesh.bf] = QRb[1]
    qR[:, mesh.bf] = QRb[2:]
    uR[:, mesh.bf] = ULb
    return Faces(WL[0], hL, qL, uL, bR, hR, qR, uR), slope


# ── numerical fluxes ────────────────────────────────────────────────────────

def numerical_flux(fa, normals, riemann, g):
    """Per-face numerical flux ``F (n_state, F)`` and fluctuations ``Dp, Dm``.

    * ``rusanov``: ``F = 1/2 (F_L + F_R).n - 1/2 s (Q_R - Q_L)`` with
      ``s = max(|u.n| + c)`` of the two sides (``zoomy_jax/fvm/flux.py:72-82``);
      SWE flux ``(q.n, q (u.n) + 1/2 g h^2 n)``; no bed term (flat-bed form,
      pinned by the goldens).
    * ``rusanov_hr`` / ``hll_hr``: hydrostatic reconstruction (Audusse et al.
      2004): ``b* = max(b_L, b_R)``, ``h*_{L,R} = max(0, h + b - b*)``,
      ``q* = h* u``; the Rusanov / HLL flux (Harten-Lax-van Leer 1983, Davis
      wave speeds ``S_L = min(u_n - c)``, ``S_R = max(u_n + c)``) of the starred
      states; fluctuations carry the well-balancing pressure correction
      ``Dm = 1/2 g (h_L^2 - h_L*^2) n``, ``Dp = -1/2 g (h_R^2 - h_R*^2) n``
      (reference names: ``PositiveNonconservativeRusanov`` /
      ``PositiveNonconservativeHLL`` of zoomy_core, not in the reference tree).
    The b row has zero flux (the bed is stationary).
    """
    dim = normals.shape[0]
    nF = normals.shape[1]
    ns = 2 + dim
    Fn = np.zeros((ns, nF))
    Dp = np.zeros((ns, nF))
    Dm = np.zeros((ns, nF))
    if riemann == "rusanov":
        unL = (fa.uL * normals).sum(axis=0)
        unR = (fa.uR * normals).sum(axis=0)
        cL = np.sqrt(g * fa.hL)
        cR = np.sqrt(g * fa.hR)
        s = np.maximum(np.abs(unL) + cL, np.abs(unR) + cR)
        qnL = (fa.qL * normals).sum(axis=0)
        qnR = (fa.qR * normals).sum(axis=0)
        FL_h, FR_h = qnL, qnR
        FL_q = fa.qL * unL[None] + 0.5 * g * fa.hL[None] ** 2 * normals
        FR_q = fa.qR * unR[None] + 0.5 * g * fa.hR[None] ** 2 * normals
        Fn[1] = 0.5 * (FL_h + FR_h) - 0.5 * s * (fa.hR - fa.hL)
        Fn[2:] = 0.5 * (FL_q + FR_q) - 0.5 * s[None] * (fa.qR - fa.qL)
        return Fn, Dp, Dm
    bs = np.maximum(fa.bL, fa.bR)
    hLs = np.maximum(0.0, fa.hL + fa.bL - bs)
    hRs = np.maximum(0.0, fa.hR + fa.bR - bs)
    unL = (fa.uL * normals).sum(axis=0)
    unR = (fa.uR * normals).sum(axis=0)
    cL = np.sqrt(g * hLs)
    cR = np.sqrt(g * hRs)
    qLs = hLs[None] * fa.uL
    qRs = hRs[None] * fa.uR
    FL_h = hLs * unL
    FR_h = hRs * unR
    FL_q = qLs * unL[None] + 0.5 * g * hLs[None] ** 2 * normals
    FR_q = qRs * unR[None] + 0.5 * g * hRs[None] ** 2 * normals
    if riemann == "rusanov_hr":
        s = np.maximum(np.abs(unL) + cL, np.abs(unR) + cR)
        Fn[1] = 0.5 * (FL_h + FR_h) - 0.5 * s * (hRs - hLs)
        Fn[2:] = 0.5 * (FL_q + FR_q) - 0.5 * s[None] * (qRs - qLs)
    elif riemann == "hll_hr":
        SL = np.minimum(unL - cL, unR - cR)
        SR = np.maximum(unL + cL, unR + cR)
        sl = np.minimum(SL, 0.0)
        sr = np.maximum(SR, 0.0)
        den = sr - sl
        ok = den > 0.0
        inv = np.where(ok, 1.0 / np.where(ok, den, 1.0), 0.0)
        Fn[1] = (sr * FL_h - sl * FR_h + sl * sr * (hRs - hLs)) * inv
        Fn[2:] = (sr[None] * FL_q - sl[None] * FR_q
                  + (sl * sr)[None] * (qRs - qLs)) * inv[None]
    else:
        raise ValueError(riemann)
    Dm[2:] = 0.5 * g * (fa.hL ** 2 - hLs ** 2)[None] * normals
    Dp[2:] = -0.5 * g * (fa.hR ** 2 - hRs ** 2)[None] * normals
    return Fn, Dp, Dm


# ── the flux operator ───────────────────────────────────────────────────────

def flux_operator(mesh, Q, scheme, params, kind, force_o1=None):
    """``dQ (n_state, C)`` = the explicit residual of one stage
    (``solver_jax.py:722-895``; ``solver2/blocks.py:241-287``):

        dQ[A] -= (F + Dm) |f| / |A|,   dQ[B] -= (-F + Dp) |f| / |B|,

    boundary faces to their owner only, plus the order-2 cell-edge
    nonconservative integral (``solver_jax.py:811-825, 868-883``) which for the
    SWE bed term ``B[q, b] = g h`` over the straight path from the cell mean to
    the cell's own face trace is ``1/2 g (h_c + h_f) (b_f - b_c) n``.
    """
    fa, slope = reconstruct(mesh, Q, scheme, params, kind, force_o1)
    nrm = mesh.face_normals
    Fn, Dp, Dm = numerical_flux(fa, nrm, scheme.riemann, params.g)
    fc = mesh.face_cells
    it = mesh.interior
    C = mesh.n_cells
    fv = mesh.face_volumes
    cv = mesh.cell_volumes
    A, B = fc[0, it], fc[1, it]
    ns = Q.shape[0]
    dQ = np.zeros_like(Q)
    bnd = mesh.bf
    own = mesh.bf_cell
    cell_term = scheme.order >= 2
    if cell_term:
        gA = 0.5 * params.g * (Q[1, fc[0]] + fa.hL) * (fa.bL - Q[0, fc[0]])
        cesA = gA[None] * nrm                      # (dim, F)
        gB = 0.5 * params.g * (Q[1, mesh.iB_or_owner] + fa.hR) * (fa.bR - Q[0, mesh.iB_or_owner])
        cesB = -gB[None] * nrm
    for v in range(1, ns):
        wa = (Fn[v, it] + Dm[v, it]) * fv[it] / cv[A]
        wb = (-Fn[v, it] + Dp[v, it]) * fv[it] / cv[B]
        wbnd = (Fn[v, bnd] + Dm[v, bnd]) * fv[bnd] / cv[own]
        acc = np.bincount(A, weights=wa, minlength=C)
        acc += np.bincount(B, weights=wb, minlength=C)
        acc += np.bincount(own, weights=wbnd, minlength=C)
        if cell_term and v >= 2:
            d = v - 2
            acc += np.bincount(A, weights=cesA[d, it] * fv[it] / cv[A], minlength=C)
            acc += np.bincount(B, weights=cesB[d, it] * fv[it] / cv[B], minlength=C)
            acc += np.bincount(own, weights=cesA[d, bnd] * fv[bnd] / cv[own], minlength=C)
        dQ[v] = -acc
    return dQ


# ── dt, source, step ────────────────────────────────────────────────────────

def face_wave_speed(mesh, Q, params):
    """Per-face ``max(|lambda_A|, |lambda_B|)`` at the CELL states with the
    owner on both sides of a boundary face (``solver2/blocks.py:36-61``,
    ``context.py:111-117``); ``|lambda| = |u.n| + sqrt(g h)``."""
    hinv = kp_hinv(Q[1], params.wet_dry_eps)
    u = velocities(Q, hinv)
    c = np.sqrt(params.g * np.maximum(Q[1], 0.0))
    nrm = mesh.face_normals
    A = mesh.face_cells[0]
    B = mesh.iB_or_owner
    lA = np.abs((u[:, A] * nrm).sum(axis=0)) + c[A]
    lB = np.abs((u[:, B] * nrm).sum(axis=0)) + c[B]
    return np.maximum(lA, lB)


def compute_dt(mesh, Q, params, scheme, t_remaining=None):
    """``dt = min_f CFL 2 r_f / (d (2k+1) |lambda|_f)``, a wave-free face
    (``|lambda| = 0``) drops out, capped by ``dt_max`` and ``t_remaining``
    (``solver2/blocks.py:64-95``)."""
    amax = face_wave_speed(mesh, Q, params)
    with np.errstate(divide="ignore"):
        loc = scheme.cfl * 2.0 * mesh.inradius_f / (
            float(mesh.dim) * float(2 * scheme.degree + 1) * amax)
    dt = float(np.min(loc))
    dt = min(dt, scheme.dt_max)
    if t_remaining is not None:
        dt = min(dt, float(t_remaining))
    return dt


def manning_source(Q, hinv, params):
    """Manning friction ``S_q = -g n^2 q |q| hinv^{7/3}`` (the standard
    ``-g n^2 u |u| / h^{1/3}`` in conservative form; zoomy_core's
    ``ManningFriction`` closure, ``tests/models.py:47-53`` in the reference)."""
    S = np.zeros_like(Q)
    if params.manning_n == 0.0:
        return S
    qn = np.sqrt((Q[2:] ** 2).sum(axis=0))
    k = -params.g * params.manning_n ** 2 * qn * hinv ** 2 * np.cbrt(hinv)
    S[2:] = Q[2:] * k[None]
    return S


def troubled_cells(Q):
    """``h < 0`` or any non-finite component (``solver2/blocks.py:290-301``)."""
    return (Q[1] < 0.0) | ~np.isfinite(Q).all(axis=0)


def step(mesh, Q, dt, params, scheme, kind=None, return_troubled=False):
    """One ``HyperbolicSolver.step`` (``solver_jax.py:1095-1131``): the
    hyperbolic sub-step (SSP-RK2 at order 2 with the aux refreshed between the
    stages, Euler at order 1; ``solver_jax.py:990-1074``), MOOD redo when
    enabled, then the source as RK1 with the step's INPUT aux
    (``ode.RK1``, ``solver_jax.py:1129``)."""
    if kind is None:
        kind = bc_kinds(mesh, scheme)
    hinv0 = kp_hinv(Q[1], params.wet_dry_eps)

    def advance(force_o1):
        if scheme.order >= 2:
            Q1 = Q + dt * flux_operator(mesh, Q, scheme, params, kind, force_o1)
            Q2 = Q1 + dt * flux_operator(mesh, Q1, scheme, params, kind, force_o1)
            return 0.5 * (Q + Q2)
        return Q + dt * flux_operator(mesh, Q, scheme, params, kind, force_o1)

    Qn = advance(None)
    trouble = troubled_cells(Qn)
    if scheme.mood and trouble.any():
        # production MOOD demotes the troubled cells (solver_jax.py:1055-1071);
        # solver2's sanctioned body redoes the whole step at order 1 with the
        # same stage loop (solver2/blocks.py:304-323)
        Qn = advance(trouble if scheme.mood_mode == "cell"
                     else np.ones(Q.shape[1], dtype=bool))
    if params.manning_n != 0.0:
        if scheme.source == "implicit":
            # point-implicit Manning (IMEX local implicit source,
            # solver_imex_jax.py:269-342, closed form for the friction law)
            qn = np.sqrt((Qn[2:] ** 2).sum(axis=0))
            k = params.g * params.manning_n ** 2 * qn * hinv0 ** 2 * np.cbrt(hinv0)
            Qn = Qn.copy()
            Qn[2:] = Qn[2:] / (1.0 + dt * k)[None]
        else:
            Qn = Qn + dt * manning_source(Qn, hinv0, params)
    if return_troubled:
        return Qn, trouble
    return Qn


def derivative_aux(mesh, Q, params):
    """Post-step aux (``solver_jax.py:284-369``): the LSQ derivative rows with
    extrapolation ghosts, then KP ``hinv``.  Row order (pinned by the goldens):
    ``[dq_1/dx_1, dh/dx_1, dq_2/dx_2, dh/dx_2, db/dx_1, db/dx_2, hinv]`` in 2-D,
    ``[dq/dx, dh/dx, db/dx, hinv]`` in 1-D."""
    gq = [lsq_gradient(mesh, Q[2 + d]) for d in range(mesh.dim)]
    gh = lsq_gradient(mesh, Q[1])
    gb = lsq_gradient(mesh, Q[0])
    rows = []
    for d in range(mesh.dim):
        rows += [gq[d][d], gh[d]]
    rows += [gb[d] for d in range(mesh.dim)]
    rows.append(kp_hinv(Q[1], params.wet_dry_eps))
    return np.stack(rows)


def march(mesh, Q, params, scheme, t_end=None, n_steps=None, max_steps=10 ** 7):
    """Adaptive march to ``t_end`` or for exactly ``n_steps`` steps
    (``tests/conftest.py:138-186`` in the reference).  Returns
    ``(Q, Qaux, t, steps)``."""
    kind = bc_kinds(mesh, scheme)
    t = 0.0
    it = 0
    while (t < t_end) if n_steps is None else (it < n_steps):
        dt = compute_dt(mesh, Q, params, scheme,
                        None if t_end is None else t_end - t)
        if not (np.isfinite(dt) and dt > 0.0):
            raise FloatingPointError(f"dt = {dt!r} at t = {t} (iteration {it})")
        Q = step(mesh, Q, dt, params, scheme, kind)
        t += dt
        it += 1
        if it >= max_steps:
            raise FloatingPointError("march exceeded max_steps")
    return Q, derivative_aux(mesh, Q, params), t, it


def mass(mesh, Q):
    """``sum h |cell|`` (``tests/test_swe_2d_jax.py:159-168`` in the reference)."""
    return float(np.sum(Q[1] * mesh.cell_volumes))

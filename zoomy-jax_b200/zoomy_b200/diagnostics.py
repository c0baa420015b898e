"""Host-side diagnostics for the fatal-dt abort (only on the error path).

``assert_dt_admissible`` in the reference names the worst face
(``zoomy_jax/fvm/solver2/blocks.py:98-124``); the fused GPU step never stores
per-face wave speeds, so on failure the state is copied to the host once and
the face with the smallest local limit (or the first non-finite one) is
located here.
"""
from __future__ import annotations

import numpy as np


def face_speeds(mesh, Q, g, eps):
    """Per-face ``max(|lambda_A|, |lambda_B|)`` for x-faces ``(nx+1, ny)`` and
    y-faces ``(nx, ny+1)`` (owner on both sides at the boundary)."""
    b, h, qx, qy = (Q[k].reshape(mesh.nx, mesh.ny) for k in range(4))
    m = np.maximum(h, eps)
    hinv = np.sqrt(2.0) * h / np.sqrt(h ** 4 + m ** 4)
    c = np.sqrt(g * np.maximum(h, 0.0))
    lx = np.abs(qx * hinv) + c
    ly = np.abs(qy * hinv) + c
    fx = np.maximum(np.pad(lx, ((1, 0), (0, 0)), mode="edge"),
                    np.pad(lx, ((0, 1), (0, 0)), mode="edge"))
    fy = np.maximum(np.pad(ly, ((0, 0), (1, 0)), mode="edge"),
                    np.pad(ly, ((0, 0), (0, 1)), mode="edge"))
    return fx, fy


def worst_face(solver, Q):
    q = Q.detach().double().cpu().numpy()
    m = solver.nsm.model
    fx, fy = face_speeds(solver.mesh, q, m.g, m.wet_dry_eps)
    allf = np.concatenate([fx.reshape(-1), fy.reshape(-1)])
    r = solver.mesh.cell_inradius
    with np.errstate(divide="ignore", invalid="ignore"):
        loc = 2.0 * r / allf
    fin = np.isfinite(loc)
    bad = int(np.argmin(np.where(fin, loc, np.inf))) if fin.any() else \
        int(np.argmax(np.nan_to_num(allf, nan=np.inf)))
    return (f"Worst face f = {bad} (x-faces first, (nx+1)*ny of them): "
            f"|lambda| = {allf[bad]!r}, inradius = {r!r}.")

"""Seeded synthetic workloads of the benchmark configurations (host NumPy).

The reference measures on test cases rather than datasets; these seeded
generators stand in for them with the configured shapes and distributions.
"""
from __future__ import annotations

import numpy as np


def bumps(xc, seed=0, n=16, amp=(0.0, 0.8), width=(0.02, 0.1), domain=(0, 1, 0, 1)):
    """Sum of ``n`` seeded Gaussian bumps with amplitude U[amp], width
    U[width] and centre U[domain]; ``xc`` is ``(2, C)``."""
    rng = np.random.default_rng(seed)
    b = np.zeros(xc.shape[1])
    x0, x1, y0, y1 = domain
    for _ in range(n):
        A = rng.uniform(*amp)
        w = rng.uniform(*width)
        cx = rng.uniform(x0, x1)
        cy = rng.uniform(y0, y1)
        b += A * np.exp(-((xc[0] - cx) ** 2 + (xc[1] - cy) ** 2) / (2 * w * w))
    return b


def gaussian_random_field(xc, seed=0, modes=64, corr=0.05, std=0.35, dry_fraction=0.10,
                          level=1.0):
    """Seeded smooth Gaussian random field on the unit square, sampled at the
    points ``xc (2, C)``: a sum of ``modes`` random Fourier modes whose wave
    vectors are drawn from the Gaussian spectrum ``exp(-k^2 corr^2)`` (random
    phases; the spectral form of filtered white noise with correlation length
    ``corr``), scaled to standard deviation ``std`` and shifted so that a
    fraction ``dry_fraction`` of the points rises above ``level`` (the dry
    islands of a lake at that level)."""
    rng = np.random.default_rng(seed)
    k = rng.normal(0.0, 1.0 / (np.sqrt(2.0) * corr), size=(modes, 2))
    ph = rng.uniform(0.0, 2.0 * np.pi, size=modes)
    f = np.zeros(xc.shape[1])
    for m in range(modes):
        f += np.cos(k[m, 0] * xc[0] + k[m, 1] * xc[1] + ph[m])
    f *= std * np.sqrt(2.0 / modes)
    return f + (level - np.quantile(f, 1.0 - dry_fraction))


def grf_dam_state(xc, seed=0, r0=0.2, h_in=2.0, h_out=1.0):
    """The unstructured configuration's state: Gaussian-random-field
    bathymetry, a circular dam (level ``h_in`` inside ``r0``, ``h_out``
    outside), dry where the bed tops the level, fluid at rest."""
    b = gaussian_random_field(xc, seed)
    r = np.sqrt((xc[0] - 0.5) ** 2 + (xc[1] - 0.5) ** 2)
    level = np.where(r < r0, h_in, h_out)
    h = np.maximum(level - b, 0.0)
    return np.stack([b, h, np.zeros_like(b), np.zeros_like(b)])


def circular_dam_state(xc, seed=0, r0=0.2, h_in=2.0, h_out=1.0, noise=1e-3,
                       center=(0.5, 0.5), bathymetry=True):
    """Circular dam break over the seeded bumps: level ``h_in`` inside radius
    ``r0`` else ``h_out`` plus ``noise * N(0, 1)``; ``h = max(level - b, 0)``
    (dry where a bump tops the level); ``u = v = 0``.  Returns ``(4, C)``
    float64 ``[b, h, q_x, q_y]``."""
    b = bumps(xc, seed) if bathymetry else np.zeros(xc.shape[1])
    rng = np.random.default_rng(seed + 1)
    r = np.sqrt((xc[0] - center[0]) ** 2 + (xc[1] - center[1]) ** 2)
    level = np.where(r < r0, h_in, h_out) + noise * rng.standard_normal(xc.shape[1])
    h = np.maximum(level - b, 0.0)
    return np.stack([b, h, np.zeros_like(b), np.zeros_like(b)])


def cartesian_centers(n, domain=(0.0, 1.0, 0.0, 1.0)):
    """``(2, n*n)`` cell centres of the ``n x n`` grid in cell order."""
    x0, x1, y0, y1 = domain
    dx = (x1 - x0) / n
    dy = (y1 - y0) / n
    i, j = np.divmod(np.arange(n * n), n)
    return np.stack([x0 + (i + 0.5) * dx, y0 + (j + 0.5) * dy])


def dam_break_2048(n=2048, seed=0):
    """The 2048^2 configuration's initial state on the unit square."""
    return circular_dam_state(cartesian_centers(n), seed=seed)


def ensemble_512(n_inst=512, seed=0, side=(64, 512)):
    """Seeded ensemble of the batched configuration: sides log-uniform in
    ``side`` (``round(64 * 8**U)``), dam height U[1.1, 3] inside radius 0.2
    (depth 1 outside), Manning n U[0.01, 0.05], flat bed, fluid at rest.
    Returns ``(sides, heights, manning)`` arrays."""
    rng = np.random.default_rng(seed)
    lo, hi = side
    u = rng.uniform(0.0, 1.0, n_inst)
    sides = np.rint(lo * (hi / lo) ** u).astype(np.int64)
    heights = rng.uniform(1.1, 3.0, n_inst)
    manning = rng.uniform(0.01, 0.05, n_inst)
    return sides, heights, manning


def ensemble_state(n, height):
    """``(4, n*n)`` flat-bed circular dam of the given height on the unit
    square (the ensemble instance's initial state)."""
    xc = cartesian_centers(n)
    r = np.sqrt((xc[0] - 0.5) ** 2 + (xc[1] - 0.5) ** 2)
    h = np.where(r < 0.2, height, 1.0)
    z = np.zeros_like(h)
    return np.stack([z, h, z, z])

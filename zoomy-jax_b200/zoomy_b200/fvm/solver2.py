"""``MarchSolver`` and the solver2 blocks on libzb.

Mirrors ``zoomy_jax.fvm.solver2`` (``blocks.py:36-361``, ``march.py:44-250``,
``state.py:15-45``, ``context.py:34-35``): the step head (dt, frozen for the
step), the Shu-Osher stage loop in which each stage is one fused libzb launch
(halo_bc + reconstruct + flux_pass + gather_update, source inside the stage
residual, troubled predicate while writing), the whole-step first-order MOOD
redo, and the post-step aux.  The fused GPU stage never materialises the
per-face wave-speed bounds, so ``step_head`` returns ``(None, None, dt)`` and
the fatal-dt diagnostic recomputes the worst face on the host.
"""
from __future__ import annotations

import ctypes as C
import math
from time import perf_counter
from typing import Any, NamedTuple

from .. import _lib as L
from ..model import NumericalSystemModel, ReconstructionSpec
from ..timestepping import adaptive
from .solver import HyperbolicSolver

TABLEAU_EULER = ((0.0, 1.0),)
TABLEAU_SSPRK2 = ((0.0, 1.0), (0.5, 1.0))


class MarchState(NamedTuple):
    time: Any
    iteration: Any
    i_snapshot: Any
    Q: Any
    Qaux: Any


def proceed(S, time_end):
    """``time < time_end`` (``state.py:28-34``)."""
    return bool(S.time < time_end)


def should_write(time, dt, i_snapshot, write_interval):
    """Drift-free write gate (``state.py:37-46``)."""
    stamp = i_snapshot * write_interval
    write = bool(time + 1e-14 >= stamp)
    return write, (i_snapshot + 1 if write else i_snapshot)


def reduce_dt_clamp(t_remaining=None, dt_window=None):
    """The clamp rule of ``reduce_dt`` (``blocks.py:64-95``): ``t_remaining``
    XOR ``dt_window``, never min-combined."""
    if t_remaining is not None and dt_window is not None:
        raise ValueError(
            "reduce_dt takes t_remaining XOR dt_window: dt_window REPLACES the "
            "t_end clamp, it is never min-combined.")
    return t_remaining if t_remaining is not None else dt_window


def assert_dt_admissible(dt, *, time, iteration, diagnose=None):
    """``dt <= 0`` or non-finite is FATAL (``blocks.py:98-124``)."""
    dt_h = float(dt)
    if math.isfinite(dt_h) and dt_h > 0.0:
        return dt_h
    extra = diagnose() if diagnose is not None else ""
    raise FloatingPointError(
        f"reduce_dt returned dt = {dt_h!r} at t = {float(time)} (iteration "
        f"{int(iteration)}) -- FATAL. {extra} The march aborts: a non-positive "
        f"or non-finite dt is a reported FINDING, never a silent spin.")


class MarchSolver(HyperbolicSolver):
    """The solver2 march (``march.py:44-250``); ``mood_redo`` is the
    whole-step order-1 redo (``blocks.py:304-323``)."""

    def __init__(self, mood_redo=False, **kw):
        super().__init__(**kw)
        self.mood_redo = bool(mood_redo)

    def setup_march(self, mesh, model, *, CFL, dt_max=None, dt_dimension=None):
        self.compute_dt = adaptive(CFL, dt_dimension or mesh.dimension,
                                   dt_max=dt_max if dt_max is not None else model.dt_max)
        self.time_end = math.inf
        Q, Qaux = self.setup_simulation(mesh, model)
        self._cfl = float(CFL)
        self.tableau = TABLEAU_SSPRK2 if self.cfg.order >= 2 else TABLEAU_EULER
        # the order-1 configuration used by the MOOD redo (constant recon,
        # same Riemann solver, no cell-interior term)
        o1 = type(self.cfg).from_buffer_copy(bytes(self.cfg))
        o1.order, o1.recon = 1, L.RECON["constant"]
        self._cfg_o1 = o1
        return MarchState(0.0, 0, 0, Q, Qaux)

    def step_head(self, S, p=None, t_remaining=None, dt_window=None):
        clamp = reduce_dt_clamp(t_remaining, dt_window)
        cfg = self.cfg
        saved = cfg.t_end
        cfg.t_end = math.inf if clamp is None else float(S.time) + float(clamp)
        try:
            L.check(self.be.dt(C.byref(cfg), L.ptr(S.Q), L.ptr(self._ws),
                               C.c_size_t(self._ws_bytes), L.ptr(self._ctrl),
                               float(S.time), self._s()), "dt")
        finally:
            cfg.t_end = saved
        dt = float(self.read_ctrl().dt)
        return None, None, dt

    def stage_loop(self, Q0, Qaux, dt, o1=False):
        """Shu-Osher stages; returns ``(Q, troubled_any)``."""
        import torch
        cfg = self._cfg_o1 if o1 else self.cfg
        hinv = Qaux[6].contiguous() if self.cfg.manning_n != 0.0 else None
        mask = torch.zeros(Q0.shape[1], dtype=torch.uint8, device=Q0.device)
        Qk = Q0
        for alpha, beta in self.tableau:
            out = torch.empty_like(Q0)
            out[0].copy_(Q0[0])
            self._stage(cfg, Qk, Q0, out, alpha, beta, dt, hinv=hinv, tr=mask)
            Qk = out
        return Qk, bool(mask.any())

    def hyperbolic_step(self, S, dt, p=None):
        Q_cand, troubled = self.stage_loop(S.Q, S.Qaux, dt, False)
        Q_next = Q_cand
        if self.mood_redo and troubled:
            Q_next, _ = self.stage_loop(S.Q, S.Qaux, dt, True)
        t_new = S.time + dt
        Qaux_next = self.update_qaux(Q_next)
        return MarchState(t_new, S.iteration + 1, S.i_snapshot, Q_next, Qaux_next), troubled

    def march(self, S, *, time_end=None, n_steps=None, dt_window=None,
              write_interval=None, on_write=None, parameters=None, max_steps=1_000_000):
        time_end = self.time_end if time_end is None else time_end
        stats = {"steps": 0, "dt_min": math.inf, "dt_max": 0.0,
                 "troubled_steps": 0, "wall": 0.0}
        t0 = perf_counter()
        while (proceed(S, time_end) if n_steps is None else S.iteration < n_steps):
            _, _, dt = self.step_head(
                S, None, None if dt_window is not None else
                (time_end - S.time if math.isfinite(time_end) else None), dt_window)
            dt = assert_dt_admissible(
                dt, time=S.time, iteration=S.iteration,
                diagnose=lambda: __import__(
                    "zoomy_b200.diagnostics", fromlist=["worst_face"]).worst_face(self, S.Q))
            S, troubled = self.hyperbolic_step(S, dt)
            stats["steps"] += 1
            stats["dt_min"] = min(stats["dt_min"], dt)
            stats["dt_max"] = max(stats["dt_max"], dt)
            if troubled:
                stats["troubled_steps"] += 1
            if write_interval is not None:
                do_write, i_snap = should_write(float(S.time), dt, int(S.i_snapshot),
                                                write_interval)
                if do_write and on_write is not None:
                    on_write(S)
                S = S._replace(i_snapshot=i_snap)
            if stats["steps"] >= max_steps:
                raise FloatingPointError(
                    f"march exceeded max_steps = {max_steps} at t = {float(S.time)} "
                    f"/ {time_end} with dt = {dt:.6e} (dt_min so far "
                    f"{stats['dt_min']:.6e}) -- the timestep collapsed towards zero "
                    f"without ever becoming non-positive.")
        import torch
        torch.cuda.synchronize()
        stats["wall"] = perf_counter() - t0
        return S, stats

    def solve_march(self, mesh, model, *, CFL, time_end=None, n_steps=None,
                    dt_dimension=None):
        S = self.setup_march(mesh, model, CFL=CFL, dt_dimension=dt_dimension)
        return self.march(S, time_end=time_end, n_steps=n_steps)


__all__ = ["MarchSolver", "MarchState", "TABLEAU_EULER", "TABLEAU_SSPRK2",
           "assert_dt_admissible", "proceed", "reduce_dt_clamp", "should_write"]

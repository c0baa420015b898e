"""Chorin projection on the GPU: hyperbolic step -> pressure Poisson -> corrector.

Mirrors ``zoomy_jax/fvm/solver_chorin_vam_jax.py``: ``ChorinSplitVAMSolverJax``
(:105) with ``setup_simulation`` (:242), ``chorin_stage`` (:524-572),
``chorin_cycle`` (:574-615, ``time_order`` 1 or 2), ``step`` (:617-638),
``run_jit_steps`` (:640-671), the pressure solve ``_step_pressure_pure``
(:673-883) with its acceptance gate ``max(1e-6, 10 tol)`` (:72-91) and
``EllipticSolveError`` (:94-102), and the corrector (:885-907).

The reference's elliptic block is VAM's operator from the absent zoomy_core
split, solved by unpreconditioned restarted GMRES; here it is the
variable-coefficient pressure Poisson problem of the non-hydrostatic
configuration, ``-div(c grad p) = -div(q*) / dt`` with ``c = clip(h, 0.1, 2)``,
solved by float64 flexible CG preconditioned by a float32 geometric-multigrid
V-cycle (plain red-black Gauss-Seidel, or the learned U-Net smoother).  A
whole solve is one CUDA graph with a device-side WHILE loop; the host reads
the residual only where the gate needs it.
"""
from __future__ import annotations

import ctypes as C

from .. import _lib as L
from .solver import HyperbolicSolver
from ..mesh import CartesianMesh


class EllipticSolveError(RuntimeError):
    """The pressure solve missed its acceptance gate
    (``solver_chorin_vam_jax.py:94-102``)."""


def elliptic_accept(tol):
    """Residual above which the solve is declared failed
    (``solver_chorin_vam_jax.py:72-91``)."""
    return max(1e-6, 10.0 * float(tol))


class PoissonSolver:
    """``-div(c grad p) = f`` on an ``nx x ny`` grid (spacing ``dx``, p = 0
    on the walls), ``c`` from a depth field: float64 FCG with a float32
    V-cycle preconditioner; ``precond`` is ``'none'`` (plain CG), ``'mg'``,
    ``'learned'`` (the V-cycle followed by one learned smoothing step on the
    finest level) or ``'learned_replace'`` (the U-Net in place of the finest
    level's red-black sweeps).  ``coarsest``: coarsening stops at this side
    (a coarsest level of at most 64 cells is solved with its dense inverse,
    built at set-up).  An 8 x 8 end instead of the default 4 x 4 one saves
    20 us per 1024^2 solve but its 64 x 64 inverse costs about 150 us of
    set-up, which a Chorin step pays every step (its coefficients follow h)."""

    def __init__(self, nx, ny, dx, cmin=0.1, cmax=2.0, nu=2, coarse_sweeps=8, coarsest=4,
                 device=None):
        import torch
        L.require_cuda()
        self.lib = L.load()
        self.nx, self.ny, self.dx = int(nx), int(ny), float(dx)
        self.cfg = L.ZbPoissonCfg(self.nx, self.ny, self.dx, float(cmin), float(cmax), int(nu),
                                  int(coarse_sweeps), int(coarsest))
        nbytes = self.lib.zb_poisson_workspace_bytes(C.byref(self.cfg))
        if nbytes == 0:
            raise ValueError("invalid Poisson configuration")
        self.device = torch.device(device or "cuda")
        self.ws = torch.zeros(nbytes, dtype=torch.uint8, device=self.device)
        lay = (C.c_int64 * 11)()
        L.check(self.lib.zb_poisson_layout(C.byref(self.cfg), lay), "poisson_layout")
        self.layout = list(lay)
        self.n_levels = self.layout[7]
        n = self.nx * self.ny
        self.scal = self.ws[self.layout[4]:self.layout[4] + 16 * 8].view(torch.float64)
        self.cx32 = self.ws[self.layout[9]:self.layout[9] + 4 * (self.nx + 1) * self.ny].view(
            torch.float32)
        self.cy32 = self.ws[self.layout[10]:self.layout[10] + 4 * self.nx * (self.ny + 1)].view(
            torch.float32)
        self.r = self.ws[self.layout[0]:self.layout[0] + 8 * n].view(torch.float64)
        self.b = torch.zeros(n, dtype=torch.float64, device=self.device)
        self.x = torch.zeros(n, dtype=torch.float64, device=self.device)
        self._graphs = {}

    def close(self):
        for g in self._graphs.values():
            self.lib.zb_fcg_graph_destroy(g)
        self._graphs.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _s(self):
        return L.stream_ptr()

    def _smo(self, precond, smoother):
        if precond.startswith("learned"):
            if smoother is None:
                raise ValueError("precond='learned' needs a LearnedSmoother")
            return C.byref(smoother.struct(self.nx, self.ny))
        return None

    # ── operator pieces ────────────────────────────────────────────────────
    def setup(self, h):
        """Face coefficients of every level from the depth ``h`` (``nx*ny``,
        float32 or float64 device tensor)."""
        dt = L.ZB_F64 if h.dtype.itemsize == 8 else L.ZB_F32
        L.check(self.lib.zb_poisson_setup(C.byref(self.cfg), L.ptr(h), dt, L.ptr(self.ws),
                                          C.c_size_t(self.ws.numel()), self._s()),
                "poisson_setup")

    def apply(self, p, out=None):
        import torch
        out = torch.empty_like(p) if out is None else out
        L.check(self.lib.zb_poisson_apply(C.byref(self.cfg), L.ptr(self.ws), L.ptr(p),
                                          L.ptr(out), self._s()), "poisson_apply")
        return out

    def vcycle(self, r32, precond="mg", smoother=None):
        """``z = M r`` (float32): one V-cycle from zero."""
        import torch
        z = torch.empty_like(r32)
        L.check(self.lib.zb_poisson_vcycle(C.byref(self.cfg), L.ptr(self.ws), L.ptr(r32),
                                           L.ptr(z), L.PRECOND[precond],
                                           self._smo(precond, smoother), self._s()),
                "poisson_vcycle")
        return z

    def rhs(self, Q, dt, out=None):
        """``f = -div(q*) / dt`` from the state ``Q (4, C)``."""
        out = self.b if out is None else out
        L.check(self.lib.zb_poisson_rhs(C.byref(self.cfg), L.ptr(Q),
                                        L.ZB_F64 if Q.dtype.itemsize == 8 else L.ZB_F32,
                                        float(dt), L.ptr(out), self._s()), "poisson_rhs")
        return out

    def correct(self, Q, p, dt):
        """``q -= dt c grad p`` in place on ``Q``'s momentum rows."""
        L.check(self.lib.zb_poisson_correct(C.byref(self.cfg), L.ptr(self.ws), L.ptr(Q),
                                            L.ZB_F64 if Q.dtype.itemsize == 8 else L.ZB_F32,
                                            L.ptr(p), float(dt), self._s()), "poisson_correct")

    # ── solves ─────────────────────────────────────────────────────────────
    def graph(self, precond="mg", smoother=None, tol=1e-8, maxit=200):
        """The CUDA graph of a whole FCG solve of ``A x = b`` on the
        solver's own ``b`` and ``x`` buffers (created once per setting)."""
        key = (precond, id(smoother), float(tol), int(maxit))
        g = self._graphs.get(key)
        if g is None:
            h = C.c_void_p()
            L.check(self.lib.zb_fcg_graph_create(
                C.byref(self.cfg), L.ptr(self.ws), L.ptr(self.b), L.ptr(self.x),
                L.PRECOND[precond], self._smo(precond, smoother), float(tol), int(maxit),
                C.byref(h), self._s()), "fcg_graph_create")
            g = self._graphs[key] = h
        return g

    def launch(self, precond="mg", smoother=None, tol=1e-8, maxit=200):
        """Queue one whole solve (no host sync) from the current ``x``."""
        g = self.graph(precond, smoother, tol, maxit)
        L.check(self.lib.zb_fcg_graph_launch(g, self._s()), "fcg_graph_launch")

    def solve(self, b=None, x0=None, tol=1e-8, maxit=200, precond="mg", smoother=None):
        """Solve ``A x = b``; returns ``(x, iterations, relative residual)``
        (one host sync for the two scalars)."""
        if b is not None and b.data_ptr() != self.b.data_ptr():
            self.b.copy_(b.reshape(-1))
        if x0 is None:
            self.x.zero_()
        elif x0.data_ptr() != self.x.data_ptr():
            self.x.copy_(x0.reshape(-1))
        self.launch(precond, smoother, tol, maxit)
        s = self.scal[7:9].cpu()
        return self.x, int(s[1].item()), float(s[0].item())

    def post_vcycle_residual(self):
        """``r - A z`` (float32) for the residual ``r`` and the V-cycle output
        ``z = M r`` the last FCG start/iteration left in the workspace: what
        the preconditioner failed to remove."""
        import torch
        n = self.nx * self.ny
        z = self.ws[self.layout[5]:self.layout[5] + 4 * n].view(torch.float32)
        return (self.r - self.apply(z.double())).float()

    def solve_stepwise(self, b=None, x0=None, tol=1e-8, maxit=200, precond="mg",
                       smoother=None, record=None, record_post=None):
        """The same solve driven from the host one iteration at a time
        (a sync per iteration); ``record`` (a list) receives a float32 copy
        of the residual after the start and after every iteration,
        ``record_post`` the residual left by each preconditioner application
        (:meth:`post_vcycle_residual`)."""
        if b is not None and b.data_ptr() != self.b.data_ptr():
            self.b.copy_(b.reshape(-1))
        if x0 is None:
            self.x.zero_()
        elif x0.data_ptr() != self.x.data_ptr():
            self.x.copy_(x0.reshape(-1))
        smo = self._smo(precond, smoother)
        pc = L.PRECOND[precond]
        L.check(self.lib.zb_fcg_start(C.byref(self.cfg), L.ptr(self.ws), L.ptr(self.b),
                                      L.ptr(self.x), pc, smo, self._s()), "fcg_start")
        if record is not None:
            record.append(self.r.float().clone())
        if record_post is not None:
            record_post.append(self.post_vcycle_residual())
        it = 0
        rel = float(self.scal[7].item())
        while rel > tol and it < maxit:
            L.check(self.lib.zb_fcg_iterate(C.byref(self.cfg), L.ptr(self.ws), L.ptr(self.x),
                                            pc, smo, self._s()), "fcg_iterate")
            it += 1
            rel = float(self.scal[7].item())
            if record is not None:
                record.append(self.r.float().clone())
            if record_post is not None and rel > tol:
                record_post.append(self.post_vcycle_residual())
        self.scal[8].fill_(float(it))     # where the graph solve leaves its count
        return self.x, it, rel


class ChorinSolver(HyperbolicSolver):
    """Chorin projection march on a Cartesian grid (``dx == dy``, walls):
    each stage is one hyperbolic Euler step of the shallow-water predictor,
    the pressure solve and the corrector (``chorin_stage``); ``time_order``
    2 wraps two stages in the outer SSP-RK2 average (``chorin_cycle``).

    Extra parameters: ``pressure_tol`` (1e-8), ``pressure_maxit`` (FCG
    iterations, 200), ``time_order`` (1 or 2), ``precond`` (``'mg'`` |
    ``'learned'`` | ``'none'``), ``smoother`` (a LearnedSmoother), ``cmin``,
    ``cmax`` (coefficient clip, 0.1 and 2), ``nu`` (smoothing sweeps),
    ``use_graph`` (False: drive the FCG iterations from the host)."""

    def __init__(self, pressure_tol=1e-8, pressure_maxit=200, time_order=1, precond="mg",
                 smoother=None, cmin=0.1, cmax=2.0, nu=2, coarse_sweeps=8, coarsest=4,
                 use_graph=True, **kw):
        super().__init__(**kw)
        if time_order not in (1, 2):
            raise ValueError("time_order is 1 or 2")
        if precond not in L.PRECOND:
            raise ValueError(f"precond must be one of {sorted(L.PRECOND)}")
        self.pressure_tol = float(pressure_tol)
        self.pressure_maxit = int(pressure_maxit)
        self.time_order = int(time_order)
        self.precond = precond
        self.smoother = smoother
        self.cmin, self.cmax, self.nu = float(cmin), float(cmax), int(nu)
        self.coarse_sweeps, self.coarsest = int(coarse_sweeps), int(coarsest)
        self.use_graph = bool(use_graph)
        self.last_elliptic_rel_resid = None
        self.last_elliptic_iterations = None

    def setup_simulation(self, mesh, model):
        import torch
        if not isinstance(mesh, CartesianMesh):
            raise NotImplementedError("the Chorin pressure solve runs on Cartesian grids")
        if abs(mesh.dx - mesh.dy) > 1e-12 * mesh.dx:
            raise NotImplementedError("the Chorin pressure solve needs dx == dy")
        Q, Qaux = super().setup_simulation(mesh, model)
        self.poisson = PoissonSolver(mesh.nx, mesh.ny, mesh.dx, self.cmin, self.cmax, self.nu,
                                     self.coarse_sweeps, self.coarsest, device=Q.device)
        self.p = self.poisson.x
        self._max_rel = torch.zeros(1, dtype=torch.float64, device=Q.device)
        self._iters = torch.zeros(1, dtype=torch.float64, device=Q.device)
        return Q, Qaux

    # ── the three sub-steps ────────────────────────────────────────────────
    def _hyperbolic_stage(self, dt, time, Q):
        """One Euler step of the shallow-water predictor (plus Manning as
        RK1), ``solver_chorin_vam_jax.py:495-522``."""
        import torch
        # the stage writes rows 1..3 of every cell; only b is carried over
        Qn = torch.empty_like(Q)
        Qn[0].copy_(Q[0])
        self._stage(self.cfg, Q, None, Qn, 0.0, 1.0, dt)
        if self.cfg.manning_n != 0.0:
            hinv = self.update_qaux(Q)[6].contiguous()
            L.check(self.be.source(L.ptr(Qn), L.ptr(hinv), float(dt), self._s()), "source")
        return Qn

    def _step_pressure(self, Q, dt, time, sync=True):
        """Coefficients from h, right-hand side, one FCG graph launch; with
        ``sync`` the gate is checked on the host, else the residual is
        folded into a device maximum checked later."""
        import torch
        P = self.poisson
        P.setup(Q[1])
        P.rhs(Q, dt)
        P.x.zero_()
        if self.use_graph:
            P.launch(self.precond, self.smoother, self.pressure_tol, self.pressure_maxit)
        else:
            # host-driven iterations (one sync each): every kernel is an
            # ordinary launch, which profilers list one by one
            P.solve_stepwise(None, P.x, self.pressure_tol, self.pressure_maxit, self.precond,
                             self.smoother)
        if sync:
            s = P.scal[7:9].cpu()
            rel, it = float(s[0]), int(s[1])
            self.last_elliptic_rel_resid, self.last_elliptic_iterations = rel, it
            if not rel <= elliptic_accept(self.pressure_tol):
                self._abort(rel, time, dt, Q)
        else:
            torch.maximum(self._max_rel, P.scal[7:8], out=self._max_rel)
            self._iters.add_(P.scal[8:9])
        return P.x

    def _abort(self, rel, time, dt, Q):
        hmin = float(Q[1].min())
        raise EllipticSolveError(
            f"Chorin pressure solve did NOT converge (t={time:.6g}, dt={dt:.6g}): relative "
            f"residual {rel:.3e} > accept gate {elliptic_accept(self.pressure_tol):.1e} "
            f"(target {self.pressure_tol:.1e}) after {self.pressure_maxit} FCG iterations "
            f"(precond={self.precond}); min(h)={hmin:.6g}.  The march is aborted.")

    def _step_corrector(self, Q, dt):
        self.poisson.correct(Q, self.poisson.x, dt)
        return Q

    def chorin_stage(self, dt, time, Q, sync=True):
        """Hyperbolic Euler -> pressure -> corrector (``:524-572``)."""
        Q = self._hyperbolic_stage(dt, time, Q)
        self._step_pressure(Q, dt, time, sync=sync)
        return self._step_corrector(Q, dt)

    def chorin_cycle(self, dt, time, Q, sync=True):
        """One time step: ``time_order`` stages with the SSP-RK2 average
        (``:574-615``)."""
        if self.time_order == 1:
            return self.chorin_stage(dt, time, Q, sync)
        Q1 = self.chorin_stage(dt, time, Q, sync)
        Q2 = self.chorin_stage(dt, time + dt, Q1, sync)
        return 0.5 * (Q + Q2)

    def step(self, dt, time, Q, Qaux=None, parameters=None):
        return self.chorin_cycle(float(dt), float(time), Q)

    def run_jit_steps(self, dt, n_steps, Q, t_start=0.0):
        """``n_steps`` cycles queued without a host round trip; the gate is
        checked once at the end on the largest residual of the run
        (``:640-671``).  Returns ``(Q, t)``."""
        self._max_rel.zero_()
        self._iters.zero_()
        t = float(t_start)
        for _ in range(int(n_steps)):
            Q = self.chorin_cycle(float(dt), t, Q, sync=False)
            t += float(dt)
        rel = float(self._max_rel.item())
        self.last_elliptic_rel_resid = rel
        self.last_elliptic_iterations = float(self._iters.item())
        if not rel <= elliptic_accept(self.pressure_tol):
            self._abort(rel, t, dt, Q)
        return Q, t

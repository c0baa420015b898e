"""``HyperbolicSolver`` -- the reference's explicit FV solver API on libzb.

Same methods and knobs as ``zoomy_jax.fvm.solver_jax.HyperbolicSolver``
(``setup_simulation`` :901-988, ``compute_timestep`` :1222-1236, ``step``
:1095-1131, ``post_step`` :1133-1172, ``run_simulation`` :1238-1352,
``solve`` :1356-1368).  ``Q`` and ``Qaux`` are CUDA tensors in the reference
layout ``(n_state, n_cells)``; every operator is a libzb call on the current
torch stream.  The time loop of ``run_simulation`` is device-resident: dt,
time and the CFL reduction live in a device control block and the host only
polls it between batches of steps.

Two meshes are served through one backend interface: the Cartesian mesh
(``create_2d``; fused tile kernels) and the unstructured triangle mesh
(``trimesh.create_tri``; gradient / face / gather-update kernels).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from .. import _lib as L
from ..mesh import CartesianMesh
from ..timestepping import Adaptive, Constant, adaptive
from ..trimesh import DeviceTriangleMesh, TriangleMesh


class _CartBackend:
    """libzb calls of the Cartesian path (``zb_swe2d_*``)."""

    def __init__(self, lib, cfg):
        self.lib, self.cfg = lib, cfg
        self.ref = C.byref(cfg)

    def workspace_bytes(self):
        return int(self.lib.zb_swe2d_workspace_bytes(self.ref))

    def mass_partials(self):
        return int(self.lib.zb_swe2d_mass_partials(self.ref))

    def init(self, Q, ctrl, t0, st):
        return self.lib.zb_swe2d_init(self.ref, Q, ctrl, 0, t0, st)

    def step(self, Q, ws, wsb, ctrl, phase, st):
        return self.lib.zb_swe2d_step(self.ref, Q, ws, wsb, ctrl, phase, st)

    def stage(self, cfgref, Qk, Q0, Qo, a, b, dt, hinv, fo, tr, ws, wsb, ctrl, st):
        return self.lib.zb_swe2d_stage(cfgref, Qk, Q0, Qo, a, b, dt, hinv, fo, tr, ctrl, st)

    def dt(self, cfgref, Q, ws, wsb, ctrl, t, st):
        return self.lib.zb_swe2d_dt(cfgref, Q, ctrl, t, st)

    def source(self, Q, hinv, dt, st):
        return self.lib.zb_swe2d_source(self.ref, Q, hinv, dt, st)

    def mass(self, Q, part, ctrl, st):
        return self.lib.zb_swe2d_mass(self.ref, Q, part, ctrl, st)

    def aux(self, Q, A, st):
        return self.lib.zb_swe2d_aux(self.ref, Q, A, st)


class _TriBackend:
    """libzb calls of the triangle path (``zb_tri_*``)."""

    def __init__(self, lib, cfg, mesh_struct):
        self.lib, self.cfg, self.mesh = lib, cfg, mesh_struct
        self.ref = C.byref(cfg)
        self.mref = C.byref(mesh_struct)

    def workspace_bytes(self):
        return int(self.lib.zb_tri_workspace_bytes(self.ref, self.mref))

    def mass_partials(self):
        return int(self.lib.zb_tri_mass_partials())

    def init(self, Q, ctrl, t0, st):
        return self.lib.zb_tri_init(self.ref, self.mref, ctrl, 0, t0, st)

    def step(self, Q, ws, wsb, ctrl, phase, st):
        return self.lib.zb_tri_step(self.ref, self.mref, Q, ws, wsb, ctrl, phase, st)

    def stage(self, cfgref, Qk, Q0, Qo, a, b, dt, hinv, fo, tr, ws, wsb, ctrl, st):
        return self.lib.zb_tri_stage(cfgref, self.mref, Qk, Q0, Qo, a, b, dt, hinv, fo, tr,
                                     ws, wsb, ctrl, st)

    def dt(self, cfgref, Q, ws, wsb, ctrl, t, st):
        return self.lib.zb_tri_dt(cfgref, self.mref, Q, ws, wsb, ctrl, t, st)

    def source(self, Q, hinv, dt, st):
        return self.lib.zb_tri_source(self.ref, self.mref, Q, hinv, dt, st)

    def mass(self, Q, part, ctrl, st):
        return self.lib.zb_tri_mass(self.ref, self.mref, Q, part, ctrl, st)

    def aux(self, Q, A, st):
        return self.lib.zb_tri_aux(self.ref, self.mref, Q, A, st)


class HyperbolicSolver:
    """Explicit SSP-RK2 / Euler finite-volume solver for 2-D shallow water.

    Parameters follow the reference (``solver_jax.py:183-226``):
    ``time_end``, ``compute_dt``, ``free_surface_h_index``,
    ``free_surface_b_index``, ``reconstruction_variables`` (``conservative`` |
    ``eta``), ``positivity_method``, ``front_theta_tol``, ``mood``; plus
    ``dtype`` (``float64`` default, as the reference enables x64, or
    ``float32``), ``eps_wet`` (the emitted dry-cell demotion threshold of the
    eta reconstruction, ``None`` = off) and ``implicit_source`` (point-implicit
    Manning, the IMEX local solve); ``output_path`` and ``output_snapshots``
    (the reference's ``settings.output`` file and snapshot count) for
    ``run_simulation(write_output=True)``.  ``use_bed`` (attribute): with
    True the fused float32 eta / HLL-HR steps read the bathymetry's gradient
    and limiter value from planes prepared once per state tensor instead of
    evaluating them every stage (the same bits either way); ``"auto"`` (the
    default) does so in float64 (0.715 -> 0.643 ms per 2048^2 minmod step on a
    B200) and for the float32 Venkatakrishnan limiter, whose b evaluation is
    costly (0.422 -> 0.376 ms), and not for the float32 clip-min limiters,
    where the extra loads cost what the saved arithmetic gains (0.2068 ->
    0.2071 ms).  A caller that edits ``Q[0]`` through a raw
    pointer instead of torch clears ``solver.cfg.bed`` or sets ``use_bed =
    False``.
    """

    use_bed = "auto"

    def __init__(self, time_end=1.0, compute_dt=None, free_surface_h_index=None,
                 free_surface_b_index=0, free_surface_momentum_indices=None,
                 reconstruction_variables="conservative", positivity_method="",
                 front_theta_tol=None, mood=False, dtype="float64", eps_wet=None,
                 implicit_source=False, device=None, output_path=None, output_snapshots=2):
        self.time_end = float(time_end)
        self.compute_dt = compute_dt if compute_dt is not None else adaptive(0.45, 2)
        self.free_surface_h_index = free_surface_h_index
        self.free_surface_b_index = free_surface_b_index
        self.free_surface_momentum_indices = free_surface_momentum_indices
        if reconstruction_variables not in ("conservative", "eta", "xz"):
            raise ValueError(reconstruction_variables)
        self.reconstruction_variables = reconstruction_variables
        self.positivity_method = positivity_method
        self.front_theta_tol = front_theta_tol
        self.mood = bool(mood)
        if dtype not in ("float32", "float64"):
            raise ValueError("dtype must be float32 or float64")
        self.dtype = dtype
        self.eps_wet = eps_wet
        self.implicit_source = bool(implicit_source)
        self.device = device
        self.output_path = output_path
        self.output_snapshots = int(output_snapshots)

    # ── configuration ─────────────────────────────────────────────────────
    def _torch_dtype(self):
        import torch
        return torch.float64 if self.dtype == "float64" else torch.float32

    def _scheme(self, nsm):
        order = nsm.reconstruction.order
        recon = "constant" if order == 1 else (
            "eta" if self.reconstruction_variables == "eta" else "conservative")
        if order >= 2 and self.reconstruction_variables == "eta" \
                and self.free_surface_h_index is None:
            raise AssertionError("reconstruction_variables='eta' requires "
                                 "free_surface_h_index to be set")
        if order >= 2 and self.reconstruction_variables == "xz":
            raise NotImplementedError("reconstruction_variables='xz' (Xing-Zhang "
                                      "scaling) is not on the GPU path")
        if self.positivity_method or self.front_theta_tol is not None:
            raise NotImplementedError("positivity_method / front_theta_tol are "
                                      "not on the GPU path")
        if self.mood and recon != "eta":
            raise NotImplementedError(
                "mood=True needs a reconstruction that supports per-cell "
                "1st-order demotion (reconstruction_variables='eta')")
        if recon == "eta" and nsm.riemann == "rusanov":
            raise NotImplementedError("the eta reconstruction needs a "
                                      "hydrostatic-reconstruction flux "
                                      "(rusanov_hr or hll_hr)")
        cd = self.compute_dt
        if isinstance(cd, Adaptive):
            cd = cd.with_dt_max(nsm.dt_max)
        return order, recon, cd

    def _fill_common(self, cfg, nsm, order, recon, cd):
        m = nsm.model
        cfg.order = order
        cfg.recon = L.RECON[recon]
        cfg.riemann = L.RIEMANN[nsm.riemann]
        cfg.limiter = L.LIMITER[nsm.reconstruction.limiter]
        cfg.g = m.g
        cfg.wet_dry_eps = m.wet_dry_eps
        cfg.eps_wet = -1.0 if self.eps_wet is None else float(self.eps_wet)
        cfg.manning_n = m.manning_n
        cfg.implicit_source = int(self.implicit_source)
        if isinstance(cd, Adaptive):
            cfg.dim_factor, cfg.cfl, cfg.dt_max, cfg.degree = (
                cd.dimension, cd.CFL, cd.dt_max, cd.degree)
        else:
            cfg.dim_factor, cfg.cfl, cfg.dt_max, cfg.degree = 2, 1.0, math.inf, 0
        cfg.t_end = self.time_end
        cfg.dtype = L.ZB_F64 if self.dtype == "float64" else L.ZB_F32
        return cfg

    def _make_cfg(self, mesh, nsm):
        """The libzb config struct for ``mesh`` (Cartesian or triangle)."""
        order, recon, cd = self._scheme(nsm)
        if isinstance(mesh, (TriangleMesh, DeviceTriangleMesh)):
            kinds = nsm.model.bc_kinds()
            if "periodic" in kinds:
                raise NotImplementedError("periodic boundaries on the triangle mesh")
            if nsm.reconstruction.limiter == "venkatakrishnan":
                raise NotImplementedError("Venkatakrishnan on the triangle mesh")
            return self._fill_common(L.ZbTriCfg(), nsm, order, recon, cd)
        cfg = self._fill_common(L.ZbSwe2dCfg(), nsm, order, recon, cd)
        cfg.nx, cfg.ny = mesh.nx, mesh.ny
        cfg.x0, cfg.y0, cfg.dx, cfg.dy = mesh.x0, mesh.y0, mesh.dx, mesh.dy
        for i, k in enumerate(nsm.model.bc_kinds()):
            cfg.bc[i] = L.BC[k]
        return cfg

    # ── setup ─────────────────────────────────────────────────────────────
    def setup_simulation(self, mesh, model):
        """Build the device state and operators (``solver_jax.py:901-988``).
        ``model`` is a :class:`NumericalSystemModel`; ``mesh`` a
        :class:`CartesianMesh` or a :class:`TriangleMesh`.  Returns
        ``(Q, Qaux)`` on the device."""
        import torch
        L.require_cuda()
        self.lib = L.load()
        nsm = model
        self.nsm = nsm
        self.mesh = mesh
        self.cfg = self._make_cfg(mesh, nsm)
        dev = torch.device(self.device or "cuda")
        td = self._torch_dtype()
        if isinstance(mesh, (TriangleMesh, DeviceTriangleMesh)):
            self._mesh_arrays = mesh.device_arrays(
                td, dev, [L.BC[k] for k in nsm.model.bc_kinds()])
            ms = L.ZbTriMesh()
            ms.n_cells, ms.n_faces, ms.n_bf = mesh.n_cells, mesh.n_faces, mesh.n_bf
            for name in L.TRI_MESH_FIELDS:
                setattr(ms, name, self._mesh_arrays[name].data_ptr())
            self._mesh_struct = ms
            self.be = _TriBackend(self.lib, self.cfg, ms)
        else:
            self.be = _CartBackend(self.lib, self.cfg)
        Q = torch.as_tensor(nsm.model.initial_state(mesh), dtype=td, device=dev).contiguous()
        self._ws_bytes = self.be.workspace_bytes()
        self._ws = torch.empty(self._ws_bytes, dtype=torch.uint8, device=dev)
        self._ctrl = torch.zeros(L.CTRL_BYTES, dtype=torch.uint8, device=dev)
        self._mass_part = torch.zeros(self.be.mass_partials(), dtype=torch.float64, device=dev)
        self._n = 0
        self._bed, self._bed_key = None, None
        self._ensure_bed(Q)
        Qaux = self.update_qaux(Q)
        return Q, Qaux

    def _ensure_bed(self, Q):
        """The bed planes the fused float32 eta / HLL-HR steps read in place of
        b's slope (``zb_swe2d_bed_prepare``), prepared again whenever the
        state tensor is another one or was modified from torch since (b is
        never written by the steps, which go through raw pointers)."""
        auto_off = (self.use_bed == "auto" and self.cfg.dtype != L.ZB_F64
                    and self.cfg.limiter != L.LIMITER["venkatakrishnan"])
        if not isinstance(self.be, _CartBackend) or not self.use_bed or auto_off:
            self.cfg.bed = None
            return
        import torch
        nb = int(self.lib.zb_swe2d_bed_bytes(C.byref(self.cfg)))
        if nb == 0:
            self.cfg.bed = None
            return
        key = (Q.data_ptr(), Q._version)
        if self._bed is not None and self._bed_key == key and self.cfg.bed:
            return
        if self._bed is None or self._bed.numel() < nb:
            self._bed = torch.empty(nb, dtype=torch.uint8, device=Q.device)
        L.check(self.lib.zb_swe2d_bed_prepare(C.byref(self.cfg), L.ptr(Q), L.ptr(self._bed),
                                              C.c_size_t(nb), self._s()), "bed_prepare")
        self.cfg.bed = self._bed.data_ptr()
        self._bed_key = key

    # ── operators ─────────────────────────────────────────────────────────
    def _s(self):
        return L.stream_ptr()

    def update_qaux(self, Q):
        """KP ``hinv`` plus the LSQ derivative rows (``solver_jax.py:284-369``)."""
        import torch
        Qaux = torch.empty((7, Q.shape[1]), dtype=Q.dtype, device=Q.device)
        L.check(self.be.aux(L.ptr(Q), L.ptr(Qaux), self._s()), "aux")
        return Qaux

    def read_ctrl(self):
        """Copy the device control block to the host (synchronises)."""
        raw = self._ctrl.cpu().numpy().tobytes()
        return L.ZbCtrl.from_buffer_copy(raw)

    def compute_timestep(self, Q, Qaux=None, parameters=None, time=0.0):
        """dt of the state (``solver_jax.py:1222-1236``): the adaptive CFL law
        over faces, capped by ``dt_max`` and by ``time_end - time``."""
        if isinstance(self.compute_dt, Constant):
            return min(self.compute_dt.dt, self.time_end - time)
        L.check(self.be.dt(C.byref(self.cfg), L.ptr(Q), L.ptr(self._ws),
                           C.c_size_t(self._ws_bytes), L.ptr(self._ctrl), float(time),
                           self._s()), "dt")
        return float(self.read_ctrl().dt)

    def _stage(self, cfg, Qk, Q0, Qo, alpha, beta, dt, hinv=None, fo=None, tr=None):
        L.check(self.be.stage(
            C.byref(cfg), L.ptr(Qk), L.ptr(Q0) if Q0 is not None else None, L.ptr(Qo),
            float(alpha), float(beta), float(dt),
            L.ptr(hinv) if hinv is not None else None,
            L.ptr(fo) if fo is not None else None, L.ptr(tr) if tr is not None else None,
            L.ptr(self._ws), C.c_size_t(self._ws_bytes), L.ptr(self._ctrl), self._s()),
            "stage")

    def _advance(self, Q, dt, force_o1=None, trouble=None):
        """Hyperbolic sub-step with a host dt: SSP-RK2 in Shu-Osher form
        (alpha = 0.5 is exact: scaling by 1/2 commutes with rounding, so it is
        bit-identical to 0.5 (Q0 + Q2)) or Euler.  Optional per-cell MOOD mask
        and troubled-mask output (C bytes)."""
        import torch
        Qn = Q.clone()
        if self.cfg.order >= 2:
            Q1 = torch.empty_like(Q)
            Q1[0].copy_(Q[0])
            self._stage(self.cfg, Q, None, Q1, 0.0, 1.0, dt, fo=force_o1)
            self._stage(self.cfg, Q1, Q, Qn, 0.5, 1.0, dt, fo=force_o1, tr=trouble)
        else:
            self._stage(self.cfg, Q, None, Qn, 0.0, 1.0, dt, fo=force_o1, tr=trouble)
        return Qn

    def step(self, dt, time, Q, Qaux, parameters=None):
        """One explicit step with a host dt (``solver_jax.py:1095-1131``):
        SSP-RK2 (order 2) or Euler (order 1); with ``mood`` the candidate's
        troubled cells (h < 0 or non-finite) are demoted to first order and
        the step is re-run (``solver_jax.py:1055-1071``); then the source as
        RK1 with the step's input aux.  Returns a new state tensor."""
        import torch
        dt = float(dt)
        if self.mood:
            mask = torch.zeros(Q.shape[1], dtype=torch.uint8, device=Q.device)
            Qn = self._advance(Q, dt, trouble=mask)
            if bool(mask.any()):
                Qn = self._advance(Q, dt, force_o1=mask)
        else:
            Qn = self._advance(Q, dt)
        if self.cfg.manning_n != 0.0:
            hinv0 = Qaux[6].contiguous()
            L.check(self.be.source(L.ptr(Qn), L.ptr(hinv0), dt, self._s()), "source")
        return Qn

    def post_step(self, time, dt, Q, Qold, Qaux, parameters=None):
        """``update_q`` (identity: the SWE declares no ``update_variables``)
        and ``update_qaux`` (``solver_jax.py:1133-1172``)."""
        return Q, self.update_qaux(Q)

    def mass(self, Q):
        """``sum h |cell|`` in float64 on the device."""
        L.check(self.be.mass(L.ptr(Q), L.ptr(self._mass_part), L.ptr(self._ctrl),
                             self._s()), "mass")
        return float(self.read_ctrl().mass)

    # ── device-resident march ─────────────────────────────────────────────
    def init_march(self, Q, t0=0.0):
        """Reset the control block for a march from ``t0``."""
        self._ensure_bed(Q)
        L.check(self.be.init(L.ptr(Q), L.ptr(self._ctrl), float(t0), self._s()), "init")
        self._n = 0

    def launch_steps(self, Q, n):
        """Queue ``n`` fused steps (no host sync).  The step index modulo 3
        selects the control-block slots."""
        self._ensure_bed(Q)
        ws, wsb = L.ptr(self._ws), C.c_size_t(self._ws_bytes)
        ctrl, st, qp = L.ptr(self._ctrl), self._s(), L.ptr(Q)
        for _ in range(n):
            rc = self.be.step(qp, ws, wsb, ctrl, self._n % 3, st)
            if rc != L.ZB_OK:
                L.check(rc, "step")
            self._n += 1

    def _raise_dt(self, Q, t):
        if isinstance(self.mesh, CartesianMesh):
            from ..diagnostics import worst_face
            where = worst_face(self, Q)
        else:
            where = ""
        raise FloatingPointError(
            f"dt became non-finite or non-positive at t = {t} (iteration "
            f"{self._n}) -- FATAL. {where}")

    def run_simulation(self, Q, Qaux, write_output=False, parameters=None,
                       max_steps=10 ** 7):
        """March to ``time_end`` (``solver_jax.py:1238-1352``).

        Without MOOD the loop is device-resident: fused steps are queued in
        growing batches and the host only polls the control block; after
        ``time_end`` a queued step takes dt = 0 and leaves the state unchanged.
        With MOOD, or in a subclass that overrides ``step`` (the Chorin
        projection), the host drives ``compute_timestep`` / ``step`` /
        ``post_step`` per step as the reference's ``_advance`` does (the MOOD
        redo decision needs the troubled mask; a subclass's step is not the
        fused kernel).  The state is returned with its aux.

        ``write_output``: snapshots to ``output_path`` as the reference writes
        them -- snapshot 0 before the first step, snapshot ``i`` after the
        first step whose time reaches ``i * time_end / (output_snapshots -
        1)``, at most one per step -- through an asynchronous
        :class:`~zoomy_b200.snapshots.SnapshotWriter` (the march pays a
        device-to-device copy per snapshot).  Near an output time the
        device-resident loop queues single steps so that it stops on the same
        step as the reference.  Before the first snapshot the mesh and the
        run's settings go to the same output (``solver_jax.py:1267-1283``
        writes them there before its loop; see :mod:`zoomy_b200.snapshots`
        for the layout)."""
        writer = None
        if write_output:
            if self.output_path is None:
                raise ValueError("write_output needs the solver's output_path")
            from ..snapshots import SnapshotWriter
            writer = SnapshotWriter(self.output_path)
            writer.write_mesh(self.output_mesh())
            writer.write_settings(self.output_settings())
        try:
            return self._march(Q, Qaux, writer, max_steps)
        finally:
            if writer is not None:
                writer.close()

    def output_mesh(self):
        """The mesh as host arrays for the output: the cell centres ``(2, C)``
        in cell order for every mesh; the grid shape, origin and spacing of a
        Cartesian mesh; the vertices and triangles of a triangle mesh."""
        m = self.mesh
        out = {"cell_centers": np.asarray(m.cell_centers(), dtype=np.float64)}
        if isinstance(m, CartesianMesh):
            out["shape"] = np.array([m.nx, m.ny], dtype=np.int64)
            out["origin"] = np.array([m.x0, m.y0], dtype=np.float64)
            out["spacing"] = np.array([m.dx, m.dy], dtype=np.float64)
        else:
            out["vertices"] = np.asarray(m.vertices, dtype=np.float64)
            out["triangles"] = np.asarray(m.triangles, dtype=np.int64)
        return out

    def output_settings(self):
        """The run's settings as a JSON-serialisable dict: solver, time
        stepping, scheme, boundary conditions, precision and output."""
        cfg = self.cfg
        cd = self.compute_dt
        step = ({"kind": "adaptive", "cfl": cd.CFL, "dimension": cd.dimension,
                 "degree": cd.degree} if isinstance(cd, Adaptive)
                else {"kind": "constant", "dt": getattr(cd, "dt", None)})
        return {
            "solver": type(self).__name__,
            "time_end": self.time_end,
            "compute_dt": step,
            "reconstruction": {"order": int(cfg.order),
                               "variables": self.reconstruction_variables,
                               "limiter": [k for k, v in L.LIMITER.items()
                                           if v == cfg.limiter][0]},
            "riemann": [k for k, v in L.RIEMANN.items() if v == cfg.riemann][0],
            "boundary_conditions": list(self.nsm.model.bc_kinds()),
            "mood": self.mood,
            "eps_wet": self.eps_wet,
            "implicit_source": self.implicit_source,
            "manning_n": float(cfg.manning_n),
            "dtype": self.dtype,
            "mesh": {"kind": type(self.mesh).__name__, "cells": int(self.mesh.n_cells)},
            "output": {"path": self.output_path, "snapshots": self.output_snapshots},
        }

    def _march(self, Q, Qaux, writer, max_steps):
        from ..snapshots import snapshot_times
        stamps = snapshot_times(self.time_end, self.output_snapshots) if writer else []
        i_snap = 0

        def snap(t, Qs, As=None):
            nonlocal i_snap
            writer.save(i_snap, t, Qs, As if As is not None else self.update_qaux(Qs))
            i_snap += 1

        if writer is not None:
            snap(0.0, Q, Qaux)
        if self.mood or type(self).step is not HyperbolicSolver.step:
            t, n = 0.0, 0
            while t < self.time_end:
                dt = self.compute_timestep(Q, Qaux, time=t)
                if not (math.isfinite(dt) and dt > 0.0):
                    self._n = n
                    self._raise_dt(Q, t)
                Qn = self.step(dt, t, Q, Qaux)
                Q, Qaux = self.post_step(t + dt, dt, Qn, Q, Qaux)
                t += dt
                n += 1
                if i_snap < len(stamps) and t >= stamps[i_snap]:
                    snap(t, Q, Qaux)
                if n >= max_steps:
                    raise FloatingPointError(f"march exceeded max_steps = {max_steps}")
            self.time, self.steps_taken = t, n
            return Q, Qaux
        self.init_march(Q, 0.0)
        batch = 1
        while True:
            self.launch_steps(Q, batch)
            c = self.read_ctrl()
            t = c.t[self._n % 3]
            if c.status & L.ZB_ST_DT_INVALID:
                self._raise_dt(Q, t)
            if i_snap < len(stamps) and t >= stamps[i_snap]:
                snap(t, Q)
            if t >= self.time_end:
                break
            if self._n >= max_steps:
                raise FloatingPointError(f"march exceeded max_steps = {max_steps}")
            batch = min(batch * 2, 64)
            if i_snap < len(stamps) and c.dt > 0.0 and stamps[i_snap] - t <= 4.0 * batch * c.dt:
                batch = 1
        self.time = t
        self.steps_taken = int(c.steps)
        return Q, self.update_qaux(Q)

    def solve(self, mesh, model, write_output=False):
        """``setup_simulation`` then ``run_simulation`` (``solver_jax.py:1356-1368``)."""
        Q, Qaux = self.setup_simulation(mesh, model)
        return self.run_simulation(Q, Qaux, write_output=write_output)

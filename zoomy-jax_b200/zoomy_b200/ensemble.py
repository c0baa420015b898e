"""Batched ensemble of independent 2-D SWE instances in shared launches.

Each instance is its own Cartesian grid (own size, spacing, Manning
coefficient, CFL dt and control block).  All instances' states live in one
device array; persistent libzb kernels walk one work list of every
instance's strip items (interior, boundary-column and boundary-row bodies,
one launch each) and the tiles of grids narrower than four cells, so a fixed
set of four launches advances every instance by one stage, whatever the
number of instances.  The launch shape -- strip CTAs per SM and, per size
class of instance, the row-chunk heights of the column-EDGE and interior
items -- is picked by an autotuner that times the candidates on the actual
ensemble (coordinate descent from the untuned shape); the steps can be
captured into a CUDA graph and replayed.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _lib as L

# size classes of instances by side (the last class takes every larger one)
CLASS_MAX_SIDE = (128, 256, 1 << 30)
CTAS_CANDIDATES = (2, 3, 4)
EDGE_ROWS_CANDIDATES = (8, 16, 24, 32)
INTERIOR_ROWS_CANDIDATES = (32, 64, 128, 256)


class Ensemble:
    """``sides`` cells per side of each (unit-square) instance; per-instance
    ``manning`` coefficients; common scheme: eta-MUSCL + HR-HLL, SSP-RK2,
    walls, CFL ``cfl`` with the 2-D law."""

    def __init__(self, sides, manning, dtype="float32", cfl=0.45, wet_dry_eps=1e-6,
                 eps_wet=1e-6, limiter="minmod", bc="wall", t_end=math.inf, g=9.81,
                 device="cuda"):
        self.sides = np.asarray(sides, dtype=np.int64)
        self.manning = np.asarray(manning, dtype=np.float64)
        if len(self.sides) != len(self.manning) or len(self.sides) < 1:
            raise ValueError("sides and manning must have the same non-zero length")
        self.n_inst = len(self.sides)
        self.dtype = dtype
        self.device = device
        c = L.ZbSwe2dCfg()
        c.order, c.recon, c.riemann = 2, L.RECON["eta"], L.RIEMANN["hll_hr"]
        c.limiter = L.LIMITER[limiter]
        for i in range(4):
            c.bc[i] = L.BC[bc]
        c.g, c.wet_dry_eps, c.eps_wet = g, wet_dry_eps, eps_wet
        c.implicit_source, c.dim_factor, c.cfl = 0, 2, cfl
        c.dt_max, c.t_end, c.degree = math.inf, t_end, 0
        c.dtype = L.ZB_F64 if dtype == "float64" else L.ZB_F32
        c.nx = c.ny = 3
        c.dx = c.dy = 1.0
        self.cfg = c
        cells = self.sides ** 2
        self.q_off = np.concatenate([[0], np.cumsum(4 * cells)[:-1]])
        self.ws_off = np.concatenate([[0], np.cumsum(3 * cells)[:-1]])
        self.cells = cells
        inst = (L.ZbEnsInstance * self.n_inst)()
        for i, n in enumerate(self.sides):
            inst[i].nx = inst[i].ny = int(n)
            inst[i].dx = inst[i].dy = 1.0 / int(n)
            inst[i].q_offset = int(self.q_off[i])
            inst[i].ws_offset = int(self.ws_off[i])
            inst[i].manning_n = float(self.manning[i])
            inst[i].t_end = float(t_end)
        self.inst = inst
        self.tile_x = 16
        self.grid = 0
        t = L.ZbEnsTuning()
        t.tile_x = self.tile_x
        t.ctas_per_sm = 2 if dtype == "float64" else 4
        t.n_classes = len(CLASS_MAX_SIDE)
        for k, side in enumerate(CLASS_MAX_SIDE):
            t.class_max_side[k] = side
            t.edge_rows[k] = 32
            t.interior_rows[k] = 64
        self.tuning = t
        self._n = 0

    @property
    def total_cells(self):
        return int(self.cells.sum())

    def setup(self, states):
        """Upload the per-instance ``(4, n*n)`` host states into one device
        array and build the instance table for the current tile height."""
        import torch
        L.require_cuda()
        self.lib = L.load()
        td = torch.float64 if self.dtype == "float64" else torch.float32
        flat = np.concatenate([np.asarray(s, dtype=np.float64).reshape(-1) for s in states])
        if flat.size != 4 * self.total_cells:
            raise ValueError("states do not match the instance sizes")
        self.Q = torch.as_tensor(flat, dtype=td, device=self.device)
        self.W = torch.empty(3 * self.total_cells, dtype=td, device=self.device)
        self.ctrls = torch.zeros(self.n_inst * L.CTRL_BYTES, dtype=torch.uint8,
                                 device=self.device)
        self._build_table()
        return self.Q

    def _build_table(self):
        import torch
        t = C.byref(self.tuning)
        nb = self.lib.zb_ens_table_bytes_tuned(C.byref(self.cfg), self.inst, self.n_inst, t)
        if nb == 0:
            raise L.ZbError("unsupported ensemble configuration")
        self.table = torch.empty(nb, dtype=torch.uint8, device=self.device)
        n_items = C.c_int(0)
        L.check(self.lib.zb_ens_prepare_tuned(C.byref(self.cfg), self.inst, self.n_inst, t,
                                              L.ptr(self.table), C.c_size_t(nb),
                                              C.byref(n_items)),
                "zb_ens_prepare_tuned")
        self.n_items = n_items.value

    def class_sizes(self):
        """(instances, cells) per size class."""
        out = []
        lo = 0
        for side in CLASS_MAX_SIDE:
            m = (self.sides > lo) & (self.sides <= side)
            out.append((int(m.sum()), int(self.cells[m].sum())))
            lo = side
        return out

    def instance(self, i):
        """Device view ``(4, n*n)`` of instance ``i``'s state."""
        n = int(self.cells[i])
        o = int(self.q_off[i])
        return self.Q[o:o + 4 * n].view(4, n)

    def init(self, t0=0.0):
        L.check(self.lib.zb_ens_init(C.byref(self.cfg), L.ptr(self.table), self.n_inst,
                                     L.ptr(self.Q), L.ptr(self.ctrls), 0, float(t0),
                                     L.stream_ptr()), "zb_ens_init")
        self._n = 0

    def launch_part(self, part, phase=None):
        ph = self._n % 3 if phase is None else phase
        rc = self.lib.zb_ens_step_part_tuned(C.byref(self.cfg), L.ptr(self.table), self.n_inst,
                                             self.n_items, C.byref(self.tuning), self.grid,
                                             L.ptr(self.Q), L.ptr(self.W), L.ptr(self.ctrls), ph,
                                             part, L.stream_ptr())
        if rc != L.ZB_OK:
            L.check(rc, "zb_ens_step_part_tuned")

    def launch_steps(self, n):
        for _ in range(n):
            self.launch_part(-1)
            self._n += 1

    def ctrl(self, i):
        raw = self.ctrls[i * L.CTRL_BYTES:(i + 1) * L.CTRL_BYTES].cpu().numpy().tobytes()
        return L.ZbCtrl.from_buffer_copy(raw)

    def status_any(self):
        """OR of every instance's status word (host sync)."""
        raw = self.ctrls.view(self.n_inst, L.CTRL_BYTES).cpu().numpy()
        st = raw[:, 64:68].copy().view(np.uint32).reshape(-1)
        return int(np.bitwise_or.reduce(st))

    # ── autotuner ─────────────────────────────────────────────────────────
    def shape(self):
        """The current launch shape as a plain dict."""
        t = self.tuning
        return {"ctas_per_sm": int(t.ctas_per_sm),
                "edge_rows": [int(t.edge_rows[k]) for k in range(t.n_classes)],
                "interior_rows": [int(t.interior_rows[k]) for k in range(t.n_classes)],
                "class_max_side": [int(t.class_max_side[k]) for k in range(t.n_classes)]}

    def _time_shape(self, saved_q, steps):
        import torch
        self._build_table()
        self.Q.copy_(saved_q)
        self.init()
        self.launch_steps(2)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        self.launch_steps(steps)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def autotune(self, steps=8):
        """Coordinate descent over the launch shape from the untuned one:
        strip CTAs per SM, then per populated size class the column-EDGE and
        the interior chunk heights; each candidate is timed over ``steps``
        steps (after two untimed ones) on a scratch copy of the state and
        replaces the incumbent only when it is faster.  Returns ``{candidate:
        ms_per_step}`` for every candidate timed and keeps the best shape
        (``self.tuned_shape``, ``self.tuned_ms``) for the steps that follow."""
        saved_q = self.Q.clone()
        t = self.tuning
        results = {}
        best = self._time_shape(saved_q, steps)
        results["untuned"] = best

        def trial(key, set_, undo):
            nonlocal best
            set_()
            ms = self._time_shape(saved_q, steps)
            results[key] = ms
            if ms < best:
                best = ms
            else:
                undo()

        for cps in CTAS_CANDIDATES:
            if cps == t.ctas_per_sm or (self.dtype == "float64" and cps > 2):
                continue
            old = t.ctas_per_sm
            trial(f"ctas_per_sm={cps}", lambda v=cps: setattr(t, "ctas_per_sm", v),
                  lambda v=old: setattr(t, "ctas_per_sm", v))
        for k, (n_inst, _) in enumerate(self.class_sizes()):
            if n_inst == 0:
                continue
            for rows in EDGE_ROWS_CANDIDATES:
                if rows == t.edge_rows[k]:
                    continue
                old = t.edge_rows[k]
                trial(f"class{k}.edge_rows={rows}",
                      lambda v=rows, k=k: t.edge_rows.__setitem__(k, v),
                      lambda v=old, k=k: t.edge_rows.__setitem__(k, v))
            for rows in INTERIOR_ROWS_CANDIDATES:
                if rows == t.interior_rows[k]:
                    continue
                old = t.interior_rows[k]
                trial(f"class{k}.interior_rows={rows}",
                      lambda v=rows, k=k: t.interior_rows.__setitem__(k, v),
                      lambda v=old, k=k: t.interior_rows.__setitem__(k, v))
        self._build_table()
        self.Q.copy_(saved_q)
        self.init()
        self.tuned = results
        self.tuned_shape = self.shape()
        self.tuned_ms = best
        return results

    # ── CUDA graph ────────────────────────────────────────────────────────
    def capture(self, steps=3):
        """Capture ``steps`` consecutive steps (a multiple of 3 keeps the
        control-block phases aligned) into a CUDA graph starting at the
        current step index; ``replay()`` advances by ``steps`` steps."""
        import torch
        if steps % 3:
            raise ValueError("capture a multiple of 3 steps")
        start = self._n
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                for k in range(steps):
                    self.launch_part(-1, (start + k) % 3)
        torch.cuda.current_stream().wait_stream(s)
        self._graph, self._graph_steps = g, steps
        return g

    def replay(self, times=1):
        for _ in range(times):
            self._graph.replay()
            self._n += self._graph_steps

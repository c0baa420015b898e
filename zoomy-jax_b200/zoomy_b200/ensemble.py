"""Batched ensemble of independent 2-D SWE instances in shared launches.

Each instance is its own Cartesian grid (own size, spacing, Manning
coefficient, CFL dt and control block).  All instances' states live in one
device array; persistent libzb kernels walk one work list of every
instance's strip items (interior, boundary-column and boundary-row bodies,
one launch each) and the tiles of grids narrower than four cells, so a fixed
set of four launches advances every instance by one stage, whatever the
number of instances.  The tile height and the persistent grid size of the
tile fallback are picked by a small autotuner that times the candidates on
the actual ensemble; the steps can be captured into a CUDA graph and
replayed.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _lib as L

TILE_CANDIDATES = (8, 16)


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
        self._build_table(self.tile_x)
        return self.Q

    def _build_table(self, tile_x):
        import torch
        nb = self.lib.zb_ens_table_bytes(C.byref(self.cfg), self.inst, self.n_inst, tile_x)
        if nb == 0:
            raise L.ZbError("unsupported ensemble configuration")
        self.table = torch.empty(nb, dtype=torch.uint8, device=self.device)
        n_items = C.c_int(0)
        L.check(self.lib.zb_ens_prepare(C.byref(self.cfg), self.inst, self.n_inst, tile_x,
                                        L.ptr(self.table), C.c_size_t(nb), C.byref(n_items)),
                "zb_ens_prepare")
        self.n_items = n_items.value
        self.tile_x = tile_x

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
        rc = self.lib.zb_ens_step_part(C.byref(self.cfg), L.ptr(self.table), self.n_inst,
                                       self.n_items, self.tile_x, self.grid, L.ptr(self.Q),
                                       L.ptr(self.W), L.ptr(self.ctrls), ph, part,
                                       L.stream_ptr())
        if rc != L.ZB_OK:
            L.check(rc, "zb_ens_step_part")

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
    def autotune(self, steps=6, grids=(0,), tiles=TILE_CANDIDATES):
        """Time ``steps`` steps for every (tile height, persistent grid)
        candidate on a scratch copy of the state and keep the fastest.
        Returns ``{(tile, grid): ms_per_step}``."""
        import torch
        saved_q = self.Q.clone()
        results = {}
        for tile in tiles:
            self._build_table(tile)
            for grid in grids:
                self.grid = grid
                self.Q.copy_(saved_q)
                self.init()
                self.launch_steps(2)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                self.launch_steps(steps)
                e1.record()
                torch.cuda.synchronize()
                results[(tile, grid)] = e0.elapsed_time(e1) / steps
        best = min(results, key=results.get)
        self._build_table(best[0])
        self.grid = best[1]
        self.Q.copy_(saved_q)
        self.init()
        self.tuned = results
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

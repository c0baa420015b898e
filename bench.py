"""Benchmark of the 2-D shallow-water finite-volume step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--dtype fp32|fp64]
                    [--n 2048] [--impl ours|reference]

Workload (one "step" = one SSP-RK2 step of the whole grid): 2048 x 2048
Cartesian cells on the unit square, eta (b, h + b, u) MUSCL with the minmod
limiter, hydrostatic-reconstruction HLL faces, SSP-RK2, wet/dry threshold
1e-6 (dry-cell demotion) with KP hinv at 1e-6, wall boundaries, bathymetry =
16 seeded Gaussian bumps (amplitude U[0, 0.8], width U[0.02, 0.1]), circular
dam break (level 2 inside r = 0.2, 1 outside, plus 1e-3 seeded noise;
h = max(level - b, 0)), u = v = 0, CFL 0.45 with the d = 2 law.  Synthetic,
seeded inputs stand in for the reference's test cases.

Under torchrun (N > 1) every rank runs its own replica of the grid (the path
has no data-path collective: replicas only); NCCL carries only the barrier
and the max-over-ranks of the timing.

--impl reference times the CPU restatement of the path (the reference itself
cannot be installed: it needs jax and zoomy_core, absent here) on the host's
cores: one process per core, each stepping a 256 x 256 sample of the same
workload; rank 0 only.

At N = 1 the same JSON line also reports the other configurations: "fp64"
(the same 2048^2 step with a float64 state), "chorin"
(1024^2 Chorin steps at a 1e-8 pressure residual, plain multigrid FCG against
the learned U-Net smoother), "ensemble" (512 uneven instances, boundary and
interior strip launches per stage), "triangles" (about 4M Delaunay triangles,
500 steps, with the GPU mesh preparation) and "snapshots" (the 2048^2 march
with asynchronous snapshot output); --no-extra skips them, --legs picks a
subset.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "zoomy-jax_b200"))

METRIC = "cell-updates/s per B200 (2-D SWE SSP-RK2 step)"
UNIT = "cell-updates/s"
CPU_SAMPLE_N = 256


def workload_state(n, seed=0):
    """Host float64 (4, n*n) initial state of the 2048^2 configuration."""
    from zoomy_b200.workloads import dam_break_2048
    return dam_break_2048(n, seed)


def workload_desc(n):
    return (f"2-D SWE {n}x{n} unit square: eta-MUSCL minmod + hydrostatic "
            f"reconstruction + HLL, SSP-RK2, wet/dry 1e-6, walls, 16 seeded "
            f"Gaussian bumps, circular dam break + 1e-3 noise, CFL 0.45")


# ── CPU leg (oracle restatement) ─────────────────────────────────────────────
def _cpu_worker(args):
    """One process: oracle SSP-RK2 steps on an n x n sample; returns the
    per-step wall times.  Single-threaded BLAS/NumPy."""
    n, warmup, steps, seed = args
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "zoomy-jax_b200"))
    from oracle import mesh as OM
    from oracle import swe as OS
    m = OM.create_2d(0.0, 1.0, 0.0, 1.0, n, n)
    Q = workload_state(n, seed)
    params = OS.Params(wet_dry_eps=1e-6)
    scheme = OS.Scheme(order=2, limiter="minmod", recon="eta", riemann="hll_hr",
                       eps_wet=1e-6, cfl=0.45,
                       bc={t: "wall" for t in ("left", "right", "bottom", "top")})
    kind = OS.bc_kinds(m, scheme)
    times = []
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        dt = OS.compute_dt(m, Q, params, scheme)
        Q = OS.step(m, Q, dt, params, scheme, kind)
        t1 = time.perf_counter()
        if it >= warmup:
            times.append(t1 - t0)
    return times


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_sample_side(total_steps, budget_s=120.0):
    """Side of the per-core sample that lets `total_steps` oracle steps fit
    `budget_s`: one 128^2 step is timed here (single-threaded NumPy, as in
    the workers) and the cost scaled by the cell count; clamped to [32, 256]
    and rounded to a multiple of 8."""
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ.setdefault(k, "1")
    sys.path.insert(0, str(ROOT))
    from oracle import mesh as OM
    from oracle import swe as OS
    n0 = 128
    m = OM.create_2d(0.0, 1.0, 0.0, 1.0, n0, n0)
    Q = workload_state(n0, 0)
    params = OS.Params(wet_dry_eps=1e-6)
    scheme = OS.Scheme(order=2, limiter="minmod", recon="eta", riemann="hll_hr",
                       eps_wet=1e-6, cfl=0.45,
                       bc={t: "wall" for t in ("left", "right", "bottom", "top")})
    kind = OS.bc_kinds(m, scheme)
    t0 = time.perf_counter()
    OS.step(m, Q, OS.compute_dt(m, Q, params, scheme), params, scheme, kind)
    per_cell = (time.perf_counter() - t0) / (n0 * n0)
    cells = budget_s / max(1, total_steps) / per_cell
    side = int(math.sqrt(max(cells, 1.0))) // 8 * 8
    return max(32, min(CPU_SAMPLE_N, side))


def run_cpu(warmup, steps, n=CPU_SAMPLE_N, procs=None):
    """All host cores, one oracle process each (spawn context).  Returns
    (cell-updates/s, cores, per-step seconds, sample text)."""
    import multiprocessing as mp
    procs = procs or min(cpu_cores(), 128)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [(n, warmup, steps, 100 + r) for r in range(procs)])
    # aggregate: all processes step concurrently; a step of the job = one step
    # of every process, bounded by the slowest
    per_step = [max(r[k] for r in res) for k in range(steps)]
    mean_step = sum(per_step) / len(per_step)
    value = procs * n * n / mean_step
    sample = (f"{procs} independent {n}x{n} replicas of the workload (one per "
              f"core), {warmup} warm-up + {steps} timed SSP-RK2 steps each, "
              f"float64 NumPy oracle")
    return value, procs, mean_step, sample


# ── clocks ──────────────────────────────────────────────────────────────────
# A child process polls NVML (query only: SM clock, its maximum and the active
# clock-event reasons) every millisecond and prints one line per sample with a
# CLOCK_MONOTONIC stamp; the parent marks the timed region on the same clock.
# A separate process keeps the polling off the launching thread's interpreter.
_NVML_POLLER = r"""
import sys, time
import pynvml as N
N.nvmlInit()
key = sys.argv[1]
h = (N.nvmlDeviceGetHandleByUUID(key) if key.startswith("GPU-")
     else N.nvmlDeviceGetHandleByPciBusId(key))
reasons = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
    N.nvmlDeviceGetCurrentClocksThrottleReasons
mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
out = sys.stdout
while True:
    t = time.monotonic()
    sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
    r = reasons(h)
    out.write(f"{t:.6f} {sm} {mx} {r}\n")
    out.flush()
    time.sleep(0.001)
"""

# NVML clock-event reason bits (nvml.h)
_REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}


class ClockSampler:
    """SM clocks and throttle reasons DURING the timed region.

    ``start()`` launches the NVML poller for the torch device ``index`` (found
    by UUID, else by PCI bus id) and waits for its first sample; ``mark()``
    stamps the start and the end of the timed region; ``stop()`` ends the
    poller.  ``summary()`` reports the samples inside the region; a region too
    short to hold one (20 steps of 0.2 ms) reports the nearest sample on each
    side and says so.  Without NVML it falls back to ``nvidia-smi -lms 50``
    over the whole bracket."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, path=None):
        self.index = index
        self.path = path
        self.proc = None
        self.kind = None
        self.samples = []       # (t, sm, max, reasons bitmask)
        self.smi_lines = []
        self.window = [None, None]

    def _device_key(self):
        import torch
        p = torch.cuda.get_device_properties(self.index)
        u = str(getattr(p, "uuid", "") or "")
        if u:
            return u if u.startswith("GPU-") else "GPU-" + u
        return f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"

    def start(self):
        try:
            import pynvml  # noqa: F401
            key = self._device_key()
            self.proc = subprocess.Popen([sys.executable, "-c", _NVML_POLLER, key],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True, bufsize=1)
            import select
            ready, _, _ = select.select([self.proc.stdout], [], [], 20.0)
            first = self.proc.stdout.readline() if ready else ""
            if first.strip():
                self.kind = "nvml"
                self._lines = [first]
                return self
            self.proc.kill()
            self.proc.wait()
        except Exception:
            self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.kind = "nvidia-smi"
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def mark(self, which):
        self.window[0 if which == "start" else 1] = time.monotonic()

    def stop(self):
        if self.proc is None:
            return
        time.sleep(0.01)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        if self.kind == "nvml":
            for ln in self._lines + out.splitlines():
                f = ln.split()
                if len(f) == 4:
                    try:
                        self.samples.append((float(f[0]), float(f[1]), float(f[2]), int(f[3])))
                    except ValueError:
                        pass
            if self.path:
                pathlib.Path(self.path).write_text(
                    "t_monotonic,sm_mhz,sm_max_mhz,reasons\n" +
                    "".join(f"{t:.6f},{a:.0f},{b:.0f},{r:#x}\n" for t, a, b, r in self.samples))
        else:
            self.smi_lines = [ln for ln in out.splitlines() if ln.strip()]
            if self.path:
                pathlib.Path(self.path).write_text("\n".join(self.smi_lines) + "\n")

    def __enter__(self):
        self.start()
        self.mark("start")
        return self

    def __exit__(self, *exc):
        self.mark("end")
        self.stop()

    def summary(self):
        if self.kind == "nvml" and self.samples:
            t0, t1 = self.window
            inside = [s for s in self.samples if t0 is not None and t0 <= s[0] <= (t1 or t0)]
            where = "inside the timed region"
            if not inside:
                before = [s for s in self.samples if s[0] < t0]
                after = [s for s in self.samples if s[0] > (t1 or t0)]
                inside = before[-1:] + after[:1]
                where = ("the nearest sample on each side of the timed region "
                         f"({(t1 - t0) * 1e3:.1f} ms, shorter than the 1 ms poll)")
            reasons = sorted({nm for _, _, _, r in inside for nm, b in _REASON_BITS.items()
                              if r & b})
            return {"sm_mhz": statistics.median(s[1] for s in inside),
                    "sm_max_mhz": inside[-1][2], "reasons": reasons,
                    "samples": len(inside), "source": "NVML, " + where}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.smi_lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


# ── GPU leg ──────────────────────────────────────────────────────────────────
def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def max_over_ranks(seconds, world, device=None):
    """The slowest rank's time (the whole job finishes when it does); the
    identity on one rank.  The collective is the only one of the timing path
    and every rank calls it in the same order."""
    if world <= 1:
        return float(seconds)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(cells_per_rank, steps, seconds_max, world):
    """Cell-updates/s of the whole job: every rank advances its own replica
    of ``cells_per_rank`` cells by ``steps`` steps (weak scaling)."""
    return world * cells_per_rank * steps / seconds_max


def run_gpu(args, rank, world, local_rank, dtype_key=None, with_e2e=True):
    import ctypes as C
    import numpy as np
    import torch
    import zoomy_b200 as zb
    from zoomy_b200 import _lib as L
    from zoomy_b200.fvm.solver import HyperbolicSolver

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.n
    C_cells = n * n
    dtype_key = dtype_key or args.dtype
    dtype = "float32" if dtype_key == "fp32" else "float64"
    es = 4 if dtype == "float32" else 8
    Q_host = workload_state(n, seed=0)
    model = zb.ShallowWater2D(wet_dry_eps=1e-6, initial_conditions=Q_host,
                              boundary_conditions={t: "wall" for t in
                                                   ("left", "right", "bottom", "top")})
    nsm = zb.NumericalSystemModel.from_system_model(
        model, zb.ReconstructionSpec(2, "minmod"), "hll_hr")
    mesh = zb.create_2d((0.0, 1.0, 0.0, 1.0), n, n)
    solver = HyperbolicSolver(time_end=math.inf,
                              compute_dt=zb.timestepping.adaptive(0.45, 2),
                              reconstruction_variables="eta", free_surface_h_index=1,
                              eps_wet=1e-6, dtype=dtype, device=f"cuda:{local_rank}")
    Q, Qaux = solver.setup_simulation(mesh, nsm)
    lib = solver.lib
    cfg = C.byref(solver.cfg)
    ws, wsb = L.ptr(solver._ws), C.c_size_t(solver._ws_bytes)
    ctrl = L.ptr(solver._ctrl)
    stream = torch.cuda.current_stream(dev)
    sp = L.stream_ptr(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def part(k, which):
        rc = lib.zb_swe2d_step_part(cfg, L.ptr(Q), ws, wsb, ctrl, k % 3, which, sp)
        if rc != 0:
            L.check(rc, "zb_swe2d_step_part")

    clock_path = None
    if args.clock_log:
        clock_path = args.clock_log if world <= 1 else f"{args.clock_log}.rank{rank}"
    clk = ClockSampler(local_rank, path=clock_path).start()
    # warm-up
    solver.init_march(Q, 0.0)
    for k in range(args.warmup):
        part(k, 0)
        part(k, 1)
    torch.cuda.synchronize(dev)
    k0 = args.warmup

    # timed region: K steps, L2 flushed before each, events around each stage
    # (a stage = the interior strip launch and the EDGE strip launch beside it
    # on the library's second stream, joined back before the stage's end event)
    K = args.steps
    launches_per_step = 4
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
    barrier()
    torch.cuda.synchronize(dev)
    wall0 = time.perf_counter()
    clk.mark("start")
    for k in range(K):
        flush.zero_()
        ev[k][0].record(stream)
        part(k0 + k, 0)
        ev[k][1].record(stream)
        part(k0 + k, 1)
        ev[k][2].record(stream)
    torch.cuda.synchronize(dev)
    clk.mark("end")
    clk.stop()
    barrier()
    wall = time.perf_counter() - wall0
    st1 = [ev[k][0].elapsed_time(ev[k][1]) * 1e-3 for k in range(K)]
    st2 = [ev[k][1].elapsed_time(ev[k][2]) * 1e-3 for k in range(K)]
    step_s = sum(st1) + sum(st2)
    c = solver.read_ctrl()
    status_ok = c.status == 0
    tmax = max_over_ranks(step_s, world, dev)
    value = whole_job_rate(C_cells, K, tmax, world)

    # roofline of the dominant kernel (stage 2: reads Q1 h/qx/qy + b + Q0
    # h/qx/qy = 7 planes, writes 3 planes), algorithmic bytes per launch
    hbm_peak, peak_kind = peaks()
    mean2 = sum(st2) / K
    mean1 = sum(st1) / K
    bytes2 = 10 * C_cells * es
    bytes1 = 7 * C_cells * es
    achieved = bytes2 / mean2 / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak,
            "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
            "traffic": None,
            "kernel": ("swe2d_strip_kernel<MODE_STEP2>: the interior launch and the boundary "
                       "launch (column-EDGE and EDGE items) side by side on two streams, "
                       "timed together (stage 2)"),
            "algorithmic_bytes_per_launch": bytes2,
            "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "stage1": {"ms": round(mean1 * 1e3, 4),
                       "achieved": round(bytes1 / mean1 / 1e9, 1),
                       "algorithmic_bytes_per_launch": bytes1},
            "stage2_ms": round(mean2 * 1e3, 4),
            "step_bytes_per_cell_update": 17 * es,
            "step_achieved": round(17 * es * C_cells * K / step_s / 1e9, 1)}
    traffic_file = ROOT / "profiles" / f"traffic_{dtype_key}.json"
    if traffic_file.exists():
        try:
            roof["traffic"] = json.loads(traffic_file.read_text()).get("bytes_per_launch")
        except ValueError:
            pass

    out = {"value": value, "ms_per_step": tmax / K * 1e3, "roofline": roof,
           "clocks": clk.summary(), "gpu_launches": launches_per_step * K,
           "status_ok": status_ok, "sim_time": float(c.t[(k0 + K) % 3]), "wall_s": wall}
    if not with_e2e:
        return out
    # e2e through the public C ABI with host buffers: upload the state from
    # pinned host memory, K fused steps each followed by a device->host read
    # of the step's control block (dt, time, status) that the host checks,
    # then the state back to pinned host memory
    td = torch.float32 if dtype == "float32" else torch.float64
    host_in = torch.as_tensor(Q_host, dtype=td).contiguous().pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    # a ring of pinned control-block buffers: the host checks step k's block
    # while steps k + 1 .. k + lag run (every step's result is read back and
    # checked, lag steps behind, as a driver that overlaps its checks with the
    # device would)
    lag = max(1, int(args.e2e_lag))
    ring = lag + 1
    ctrl_host = [torch.empty(L.CTRL_BYTES, dtype=torch.uint8).pin_memory() for _ in range(ring)]
    ctrl_ev = [torch.cuda.Event() for _ in range(ring)]
    Qd = torch.empty_like(Q)

    def check_ctrl(buf):
        cc = L.ZbCtrl.from_buffer_copy(buf.numpy().tobytes())
        if cc.status & L.ZB_ST_DT_INVALID:
            raise FloatingPointError("dt invalid during the e2e run")

    def e2e_pass(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        Qd.copy_(host_in, non_blocking=True)
        if solver.cfg.bed:
            # the bed planes of the uploaded state (the solver reads them for
            # this scheme and precision), inside the timed region
            L.check(lib.zb_swe2d_bed_prepare(cfg, L.ptr(Qd), solver.cfg.bed,
                                             C.c_size_t(solver._bed.numel()), sp),
                    "bed_prepare")
        lib.zb_swe2d_init(cfg, L.ptr(Qd), ctrl, 0, 0.0, sp)
        for k in range(steps):
            rc = lib.zb_swe2d_step(cfg, L.ptr(Qd), ws, wsb, ctrl, k % 3, sp)
            L.check(rc, "zb_swe2d_step")
            ctrl_host[k % ring].copy_(solver._ctrl, non_blocking=True)
            ctrl_ev[k % ring].record(stream)
            if k >= lag:
                ctrl_ev[(k - lag) % ring].synchronize()
                check_ctrl(ctrl_host[(k - lag) % ring])
        for j in range(max(0, steps - lag), steps):
            ctrl_ev[j % ring].synchronize()
            check_ctrl(ctrl_host[j % ring])
        host_out.copy_(Qd, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0, e1

    # warm-up pass (untimed, W steps): the first transfers into freshly pinned
    # host buffers pay their one-time mapping (a first 67 MB download took
    # 5.4 ms against 1.2 ms afterwards)
    barrier()
    torch.cuda.synchronize(dev)
    e2e_pass(max(1, args.warmup))
    barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = e2e_pass(K)
    e2e_s = max_over_ranks(e0.elapsed_time(e1) * 1e-3, world, dev)
    state_bytes = 4 * C_cells * es
    e2e = {"value": whole_job_rate(C_cells, K, e2e_s, world), "unit": UNIT,
           "h2d_bytes_per_step": state_bytes // K,
           "d2h_bytes_per_step": L.CTRL_BYTES + state_bytes // K,
           "how": ("public C ABI (zb_swe2d_init/zb_swe2d_step) with pinned host "
                   "buffers: state upload, K steps each followed by a D2H read of the "
                   f"step's control block that the host checks while the next {lag} "
                   "step(s) run, state download; after one untimed warm-up pass of W steps "
                   "through the same pinned buffers")}
    out["e2e"] = e2e
    return out


def _ev_ms(fn, reps):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def poisson_solve_bytes(cells, iterations, levels):
    """Algorithmic bytes of one multigrid-FCG pressure solve on ``cells`` fine
    cells: what the kernels must stream per cell.  Per FCG iteration (float64
    vectors, float64 level-0 face coefficients): q = A p with the p.q and p.r
    dots reads p, r, cx, cy and writes q (40 B); x += a p, r -= a q reads x,
    p, r, q and writes x, r and the float32 copy of r (52 B); z.q reads the
    V-cycle's float32 z and q (12 B); p = z - b p reads z (float32) and p and
    writes p (20 B); the V-cycle (float32) per level reads f, cx, cy, dg and
    writes x and a quarter-size coarse right-hand side on the way down (21 B),
    reads f, cx, cy, dg, x and the quarter-size correction and writes x on the
    way up (25 B), over levels shrinking 4x (46 B x 4/3).  The start is one
    residual (x, b, cx, cy read; r, r32 written: 44 B), one V-cycle and p = z
    (12 B)."""
    vcycle = 46.0 * (1.0 - 0.25 ** levels) / 0.75
    per_it = 40 + 52 + 12 + 20 + vcycle
    start = 44 + vcycle + 12
    return int(cells * (start + iterations * per_it))


def run_chorin(local_rank, n=1024, steps=10, warmup=3, train_steps=2000, use_graph=True):
    """The non-hydrostatic configuration: Chorin steps (hyperbolic Euler ->
    pressure Poisson to 1e-8 -> corrector) on an n x n grid, plain multigrid
    FCG against the learned U-Net post-smoother (trained here on the GPU by
    the project's kernels on 10k solver-generated patches; training is
    outside the timed region and reported)."""
    import torch
    import zoomy_b200 as zb
    from zoomy_b200.fvm.chorin import ChorinSolver, elliptic_accept
    from zoomy_b200.learned import LearnedSmoother, SmootherTrainer, solver_training_set
    from zoomy_b200.workloads import cartesian_centers, circular_dam_state
    tags = ("left", "right", "bottom", "top")
    dev = f"cuda:{local_rank}"

    def make(precond, smoother=None):
        state = circular_dam_state(cartesian_centers(n), seed=0)
        model = zb.ShallowWater2D(boundary_conditions={t: "wall" for t in tags},
                                  initial_conditions=state)
        nsm = zb.NumericalSystemModel.from_system_model(
            model, zb.ReconstructionSpec(2, "minmod"), "hll_hr")
        sol = ChorinSolver(pressure_tol=1e-8, pressure_maxit=200, precond=precond,
                           smoother=smoother, compute_dt=zb.timestepping.adaptive(0.45, 2),
                           reconstruction_variables="eta", free_surface_h_index=1,
                           eps_wet=1e-6, dtype="float32", device=dev, use_graph=use_graph)
        Q, _ = sol.setup_simulation(zb.create_2d((0.0, 1.0, 0.0, 1.0), n, n), nsm)
        return sol, Q

    def measure(precond, smoother=None):
        sol, Q = make(precond, smoother)
        dt = sol.compute_timestep(Q)
        Qw, _ = sol.run_jit_steps(dt, warmup, Q)
        sol._max_rel.zero_()
        sol._iters.zero_()
        state = {"Q": Q}

        def one():
            state["Q"] = sol.chorin_cycle(dt, 0.0, state["Q"], sync=False)
        torch.cuda.synchronize()
        ms = _ev_ms(one, steps)
        rel = float(sol._max_rel.item())
        its = float(sol._iters.item()) / steps
        out = {"ms_per_step": round(ms, 4), "fcg_iterations_per_solve": its,
               "max_rel_residual": rel, "gate_ok": rel <= elliptic_accept(1e-8)}
        # the pressure solve alone (the last step's right-hand side, from x = 0)
        P = sol.poisson

        def solve():
            P.x.zero_()
            P.launch(sol.precond, sol.smoother, sol.pressure_tol, sol.pressure_maxit)
        solve()
        torch.cuda.synchronize()
        ms_solve = _ev_ms(solve, steps)
        it_solve = int(P.scal[8].item())
        out["solve_ms"] = round(ms_solve, 4)
        out["solve_iterations"] = it_solve
        if precond == "mg":
            b_alg = poisson_solve_bytes(n * n, it_solve, P.n_levels)
            hbm_peak, peak_kind = peaks()
            ach = b_alg / (ms_solve * 1e-3) / 1e9
            out["roofline"] = {"bound": "hbm", "achieved": round(ach, 1), "peak": hbm_peak,
                               "unit": "GB/s", "frac": round(ach / hbm_peak, 4),
                               "algorithmic_bytes_per_solve": b_alg,
                               "peak_kind": peak_kind,
                               "what": "one pressure solve (FCG start + iterations), "
                                       "bytes per poisson_solve_bytes()"}
        return out

    out = {"grid": [n, n], "tol": 1e-8, "steps": steps, "warmup": warmup,
           "step": "hyperbolic Euler (eta-MUSCL + HR-HLL) + pressure FCG + corrector, fp32 "
                   "state, fp64 Krylov / fp32 V-cycle(2,2), exact coarsest solve",
           "plain_mg": measure("mg")}
    t0 = time.perf_counter()
    data = solver_training_set(n_grid=256, seeds=(1, 2, 3, 4), steps=3, patch=32, count=10000,
                               targets=False, device=dev)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    for key, (c1, c2) in (("learned", (24, 48)), ("learned_small", (8, 16))):
        sm = LearnedSmoother(c1, c2, seed=0, device=dev)
        tr = SmootherTrainer(sm, batch=64, n=32, lr=3e-3)
        t0 = time.perf_counter()
        hist = tr.fit(data, steps=train_steps, log_every=max(1, train_steps // 2))
        torch.cuda.synchronize()
        t_train = time.perf_counter() - t0
        r = measure("learned", sm)
        r.update({"network": f"U-Net c1={c1} c2={c2}, {sm.n_params} params, bf16 weights, "
                             f"tcgen05 convolutions, fp32 accumulation",
                  "train_s": round(t_train, 2), "train_steps": train_steps,
                  "train_loss": [round(v, 4) for _, v in hist],
                  "training_set": f"{data.count} 32x32 patches from 256^2 solver runs "
                                  f"({round(t_data, 2)} s to generate)",
                  "speed_vs_plain": round(out["plain_mg"]["ms_per_step"] / r["ms_per_step"], 3)})
        out[key] = r
    return out


def run_triangles(local_rank, n_side=1415, steps=500, warmup=3, host_prep=True):
    """The unstructured configuration: a Delaunay triangulation of seeded
    jittered points (about 2 n_side^2 = 4.0M triangles, int32 connectivity),
    eta least-squares MUSCL with the Barth-Jespersen limiter, HR-HLL,
    SSP-RK2, Manning n = 0.03 (point-implicit), dry-cell demotion below
    1 mm, Gaussian-random-field bathymetry with ~10 % dry islands, float32
    state with float64 mass sums;
    `steps` steps after `warmup`, timed with CUDA events.  Mesh generation
    (scipy Delaunay on the host) is outside; the mesh preparation (faces,
    geometry, least-squares stencils, device arrays) runs on the GPU and is
    timed beside the host builder it replaces."""
    import torch
    import zoomy_b200 as zb
    from zoomy_b200 import _lib as L
    from zoomy_b200.fvm.solver import HyperbolicSolver
    from zoomy_b200.trimesh import DeviceTriangleMesh, TriangleMesh, lattice_triangulation
    from zoomy_b200.workloads import grf_dam_state
    t0 = time.perf_counter()
    P, T = lattice_triangulation(n_side, seed=0)
    t_gen = time.perf_counter() - t0
    kinds = [L.BC["wall"]] * 4
    dev = torch.device(f"cuda:{local_rank}")
    # the second of two preparations is timed: the first also pays the CUDA
    # caching allocator's first requests for these sizes
    for _ in range(2):
        mesh = None
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        mesh = DeviceTriangleMesh(P, T, device=dev)
        mesh.device_arrays(torch.float32, dev, kinds)
        torch.cuda.synchronize(dev)
        t_prep_gpu = time.perf_counter() - t0
    t_prep_host = None
    if host_prep:
        t0 = time.perf_counter()
        hm = TriangleMesh.from_points(P, T)
        hm.device_arrays(torch.float32, dev, kinds)
        torch.cuda.synchronize(dev)
        t_prep_host = time.perf_counter() - t0
        del hm
    state = grf_dam_state(mesh.cell_centers(), seed=0)
    model = zb.ShallowWater2D(manning_n=0.03, boundary_conditions={t: "wall" for t in
                                                                  ("left", "right", "bottom",
                                                                   "top")},
                              initial_conditions=state)
    nsm = zb.NumericalSystemModel.from_system_model(
        model, zb.ReconstructionSpec(2, "barth_jespersen"), "hll_hr")
    # Manning friction as the point-implicit local solve (the IMEX source):
    # explicit friction is unstable in the shallow cells around the islands.
    # Cells shallower than 1 mm are demoted to first order: at 1e-6 the float32
    # second-order scheme leaves rounding-level negative depths (-6e-8) at the
    # island shores within two steps
    solver = HyperbolicSolver(time_end=math.inf, compute_dt=zb.timestepping.adaptive(0.45, 2),
                              reconstruction_variables="eta", free_surface_h_index=1,
                              eps_wet=1e-3, dtype="float32", implicit_source=True,
                              device=f"cuda:{local_rank}")
    Q, _ = solver.setup_simulation(mesh, nsm)
    m0 = solver.mass(Q)
    solver.init_march(Q)
    solver.launch_steps(Q, warmup)
    torch.cuda.synchronize()
    ms = _ev_ms(lambda: solver.launch_steps(Q, steps), 1) / steps
    c = solver.read_ctrl()
    m1 = solver.mass(Q)
    cells = int(mesh.n_cells)
    hbm_peak, _ = peaks()
    # algorithmic bytes per float32 cell-update of the unstructured SSP-RK2
    # step: per stage the state (16 B read, 12 B written), cell statics
    # (volume, 3 neighbour indices, 2x3 least-squares weights: 40 B) and 1.5
    # faces of statics (2 indices, normal, length: 30 B); plus the Q0 read
    achieved = cells / (ms * 1e-3) * 208 / 1e9
    return {"cells": cells, "faces": int(mesh.n_faces), "steps": steps,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak,
                         "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                         "bytes_per_cell_update": 208},
            "ms_per_step": round(ms, 4), "value": cells / (ms * 1e-3),
            "unit": "cell-updates/s", "kernels_per_step": 6, "device_copies_per_step": 1,
            "mass_rel_change": abs(m1 - m0) / m0, "status_ok": c.status == 0,
            "dry_fraction_initial": float((state[1] <= 0).mean()),
            "mesh_generation_s": round(t_gen, 1),
            "mesh_prep": {"gpu_ms": round(t_prep_gpu * 1e3, 2),
                          "host_s": None if t_prep_host is None else round(t_prep_host, 2),
                          "how": ("DeviceTriangleMesh (zb_trimesh_match + zb_trimesh_fill, "
                                  "wall clock incl. one synchronisation) vs TriangleMesh."
                                  "from_points + device_arrays (NumPy, upload included)")}}


def run_snapshots(local_rank, n=2048, steps=200, snapshots=5):
    """Snapshot output while marching: the 2048^2 float32 workload, `steps`
    fused steps queued without host synchronisation, against the same steps
    with `snapshots` snapshots (state + 7 aux rows each) handed to the
    asynchronous writer at even intervals; wall clock from the first launch
    to the last file closed.  Files go to a temporary directory."""
    import math as _m
    import tempfile
    import torch
    import zoomy_b200 as zb
    from zoomy_b200.fvm.solver import HyperbolicSolver
    from zoomy_b200.snapshots import SnapshotWriter
    dev = torch.device("cuda", local_rank)
    Q_host = workload_state(n, seed=0)
    model = zb.ShallowWater2D(wet_dry_eps=1e-6, initial_conditions=Q_host,
                              boundary_conditions={t: "wall" for t in
                                                   ("left", "right", "bottom", "top")})
    nsm = zb.NumericalSystemModel.from_system_model(
        model, zb.ReconstructionSpec(2, "minmod"), "hll_hr")
    solver = HyperbolicSolver(time_end=_m.inf, compute_dt=zb.timestepping.adaptive(0.45, 2),
                              reconstruction_variables="eta", free_surface_h_index=1,
                              eps_wet=1e-6, dtype="float32", device=f"cuda:{local_rank}")
    Q, _ = solver.setup_simulation(zb.create_2d((0.0, 1.0, 0.0, 1.0), n, n), nsm)
    Q0 = Q.clone()
    every = max(1, steps // snapshots)

    def march(writer):
        Q.copy_(Q0)
        solver.init_march(Q)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        k = 0
        for i in range(steps):
            solver.launch_steps(Q, 1)
            if writer is not None and (i + 1) % every == 0 and k < snapshots:
                writer.save(k, float(i + 1), Q, solver.update_qaux(Q))
                k += 1
        if writer is not None:
            writer.close()
        torch.cuda.synchronize(dev)
        return time.perf_counter() - t0

    march(None)                                  # warm-up
    t_plain = march(None)
    with tempfile.TemporaryDirectory() as d:
        t_snap = march(SnapshotWriter(os.path.join(d, "run.h5")))
    per_snap = 4 * n * n * 4 + 7 * n * n * 4
    return {"grid": [n, n], "steps": steps, "snapshots": snapshots,
            "bytes_per_snapshot": per_snap,
            "march_s": round(t_plain, 4), "march_with_snapshots_s": round(t_snap, 4),
            "overhead_per_snapshot_ms": round((t_snap - t_plain) / snapshots * 1e3, 2),
            "how": ("wall clock of the march, steps queued without host synchronisation; "
                    "snapshots staged device-to-device, copied to a pinned ring on a side "
                    "stream and written by a writer thread (.npy files: no HDF5 library "
                    "in the image); includes closing the writer")}


def run_ensemble(local_rank, steps=2000):
    """The batched configuration: 512 uneven SWE instances (sides log-uniform
    in [64, 512]) advanced together: per stage persistent launches over every
    instance's column-EDGE and EDGE strip items beside one over the interior
    items, and the tile fallback for grids narrower than four cells (unused
    here): four launches per stage, replayed from a CUDA graph of 30 steps.
    The launch shape (strip CTAs per SM, column-EDGE and interior chunk
    heights per size class of instance) is autotuned first on the ensemble
    itself, and the tuned shape is the one timed."""
    import torch
    from zoomy_b200.ensemble import Ensemble
    from zoomy_b200.workloads import ensemble_512, ensemble_state
    sides, heights, manning = ensemble_512(seed=0)
    ens = Ensemble(sides, manning, dtype="float32", device=f"cuda:{local_rank}")
    ens.setup([ensemble_state(int(k), h) for k, h in zip(sides, heights)])
    tuned = ens.autotune(steps=8)
    ens.init()
    chunk = 30
    ens.capture(chunk)
    ens.init()
    ens.replay(1)
    torch.cuda.synchronize()
    reps = max(1, steps // chunk)
    ms = _ev_ms(lambda: ens.replay(1), reps)
    cells = int(ens.total_cells)
    hbm_peak, _ = peaks()
    achieved = cells * chunk / (ms * 1e-3) * 68 / 1e9     # 17 fp32 planes per cell-update
    return {"instances": int(len(sides)), "cells": cells, "steps": reps * chunk,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak,
                         "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                         "bytes_per_cell_update": 68},
            "ms_per_step": round(ms / chunk, 4),
            "value": cells * chunk / (ms * 1e-3), "unit": "cell-updates/s",
            "launches_per_step": 8,
            "autotune_ms_per_step": {k: round(v, 4) for k, v in tuned.items()},
            "launch_shape": ens.tuned_shape,
            "class_instances_cells": ens.class_sizes(),
            "status_ok": ens.status_any() == 0}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--dtype", choices=("fp32", "fp64"), default="fp32")
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--clock-log", default=None,
                    help="also write the raw nvidia-smi clock samples of the timed region "
                         "to this CSV (the JSON line always carries their summary)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the Chorin and ensemble legs")
    ap.add_argument("--legs", default="swe,fp64,chorin,ensemble,triangles,snapshots",
                    help="comma-separated legs to run (profiling runs pick one)")
    ap.add_argument("--train-steps", type=int, default=2000)
    ap.add_argument("--chorin-steps", type=int, default=10)
    ap.add_argument("--tri-steps", type=int, default=500)
    ap.add_argument("--tri-side", type=int, default=1415,
                    help="lattice side of the triangle mesh (2 side^2 triangles; profiling "
                         "captures use a smaller mesh)")
    ap.add_argument("--tri-host-prep", type=int, default=1,
                    help="also time the host mesh builder in the triangles leg (0: skip)")
    ap.add_argument("--e2e-lag", type=int, default=2,
                    help="steps the e2e host loop runs ahead of the control-block check "
                         "(every step's block is still read and checked)")
    ap.add_argument("--chorin-no-graph", action="store_true",
                    help="drive the pressure iterations from the host (for profilers, which "
                         "do not list kernels inside conditional graph nodes)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": workload_desc(args.n), "grid": [args.n, args.n],
              "global_batch": world * args.n * args.n, "seq_len": None,
              "parallelism": f"replicas x{world}",
              "l2": "flushed between timed steps (256 MiB write, outside the events)",
              "bc": "wall", "seed": 0}

    if args.impl == "reference":
        if rank != 0:
            return
        # all W + K steps, each on a per-core sample sized so that the run
        # ends within about two minutes
        side = reference_sample_side(args.warmup + args.steps)
        value, cores, mean_step, sample = run_cpu(args.warmup, args.steps, n=side)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": mean_step * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config, "impl": "reference",
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores,
                                 "kind": "port", "sample": sample},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "note": ("the reference (jax + zoomy_core) cannot be installed here; "
                         "this arm times the float64 oracle restatement of its path")}
        print(json.dumps(line), flush=True)
        return

    cpu = None
    if rank == 0 and not args.no_cpu:
        # before any CUDA call: spawn-context pool of oracle processes
        v, cores, mean_step, sample = run_cpu(1, args.cpu_steps)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": sample}

    legs = set(args.legs.split(","))
    if "swe" not in legs:
        # a single extra leg (profiling): rank 0 only, its own JSON line
        if rank != 0:
            return
        import torch
        torch.cuda.set_device(local_rank)
        line = {"legs": sorted(legs)}
        if "chorin" in legs:
            line["chorin"] = run_chorin(local_rank, steps=args.chorin_steps,
                                        train_steps=args.train_steps,
                                        use_graph=not args.chorin_no_graph)
        if "ensemble" in legs:
            line["ensemble"] = run_ensemble(local_rank)
        if "triangles" in legs:
            line["triangles"] = run_triangles(local_rank, n_side=args.tri_side, steps=args.tri_steps,
                                              host_prep=bool(args.tri_host_prep))
        if "snapshots" in legs:
            line["snapshots"] = run_snapshots(local_rank)
        print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    res = run_gpu(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return
    extra = {}
    # the extra legs are single-GPU configurations: measured at N = 1 only, so
    # a scaling run holds its N GPUs for the replicated SWE leg alone
    if not args.no_extra and world == 1:
        if "fp64" in legs and args.dtype == "fp32":
            # the same 2048^2 configuration with a float64 state (its other run)
            r64 = run_gpu(args, rank, world, local_rank, dtype_key="fp64", with_e2e=False)
            extra["fp64"] = {"value": r64["value"], "unit": UNIT,
                             "ms_per_step": r64["ms_per_step"], "steps": args.steps,
                             "roofline": r64["roofline"], "clocks": r64["clocks"],
                             "gpu_launches": r64["gpu_launches"],
                             "status_ok": r64["status_ok"]}
        if "chorin" in legs:
            extra["chorin"] = run_chorin(local_rank, steps=args.chorin_steps,
                                         train_steps=args.train_steps)
        if "ensemble" in legs:
            extra["ensemble"] = run_ensemble(local_rank)
        if "triangles" in legs:
            extra["triangles"] = run_triangles(local_rank, n_side=args.tri_side, steps=args.tri_steps,
                                               host_prep=bool(args.tri_host_prep))
        if "snapshots" in legs:
            extra["snapshots"] = run_snapshots(local_rank)
    line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": res["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.dtype == "fp32" else "f64",
            "data": "synthetic", "config": config, "roofline": res["roofline"],
            "cpu_baseline": cpu, "e2e": res["e2e"], "clocks": res["clocks"],
            "gpu_launches": res["gpu_launches"], "status_ok": res["status_ok"],
            "sim_time": res["sim_time"]}
    line.update(extra)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()

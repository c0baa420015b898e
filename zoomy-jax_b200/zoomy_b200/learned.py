"""Learned multigrid smoother: a bf16 U-Net trained and run by libzb kernels.

Counterpart of the reference's learned V-cycle smoother
(``zoomy_jax/gnn_blueprint/vcycle_structured_gnn.py`` :42-71 init, :74-122
apply; ``graph_mp_multibranch.py`` :9-16 the tanh layer) and of its Adam
training loop (``train_vcycle_structured_poisson.py`` :168-306).  The reference
trains a graph message-passing smoother on dense matrices of a 32^2 grid and
uses the V-cycle only as a GMRES initial guess; here the smoother is a
convolutional U-Net with bf16 weights and float32 accumulation that replaces
the level-0 red-black sweeps of the pressure V-cycle inside flexible CG
(``ZB_PRECOND_LEARNED``), trained on the GPU by the project's own forward,
backward and Adam kernels on right-hand sides and residuals the Chorin solver
generates.

Layer layout (``[Cout][Cin][3][3]`` each, concatenated; biases float32):
``e1 2->c1, e2 c1->c1, m1 c1->c2, m2 c2->c2, o1 c2+c1->c1, out c1->1``.
"""
from __future__ import annotations

import ctypes as C
import math

from . import _lib as L

CHANNELS = ((8, 16), (16, 16), (16, 32), (24, 48))


def layer_shapes(c1, c2):
    return [(2, c1), (c1, c1), (c1, c2), (c2, c2), (c1 + c2, c1), (c1, 1)]


def param_counts(c1, c2):
    lib = L.load()
    nw, nb = C.c_size_t(), C.c_size_t()
    total = lib.zb_unet_param_count(c1, c2, C.byref(nw), C.byref(nb))
    if total == 0:
        raise ValueError(f"unsupported U-Net channels ({c1}, {c2}); one of {CHANNELS}")
    return nw.value, nb.value


class LearnedSmoother:
    """Weights of the U-Net smoother on the device (float32 master, bf16
    copy used by every forward) and the ``zb_smoother`` descriptors the
    pressure V-cycle takes, one activation workspace per grid size."""

    def __init__(self, c1=24, c2=48, cmax=2.0, seed=0, device=None):
        import torch
        L.require_cuda()
        self.lib = L.load()
        self.c1, self.c2, self.cmax = int(c1), int(c2), float(cmax)
        self.nw, self.nb = param_counts(self.c1, self.c2)
        self.device = torch.device(device or "cuda")
        g = torch.Generator().manual_seed(int(seed))
        ws, bs = [], []
        shapes = layer_shapes(self.c1, self.c2)
        for k, (ci, co) in enumerate(shapes):
            # tanh layers: Xavier-normal; the output layer starts small so the
            # untrained smoother is a gentle correction
            std = math.sqrt(2.0 / (9 * ci + 9 * co)) * (0.1 if k == len(shapes) - 1 else 1.0)
            ws.append(torch.randn(co * ci * 9, generator=g) * std)
            bs.append(torch.zeros(co))
        self.w = torch.cat(ws).to(self.device, torch.float32).contiguous()
        self.b = torch.cat(bs).to(self.device, torch.float32).contiguous()
        self.w_bf16 = self.w.to(torch.bfloat16).contiguous()
        self._structs = {}

    @property
    def n_params(self):
        return self.nw + self.nb

    def refresh(self):
        """Re-round the bf16 copy from the float32 master (after a load)."""
        self.w_bf16.copy_(self.w.to(self.w_bf16.dtype))

    def struct(self, nx, ny):
        """The ``zb_smoother`` descriptor for an ``nx x ny`` grid."""
        import torch
        key = (int(nx), int(ny))
        hit = self._structs.get(key)
        if hit is not None:
            return hit[0]
        nbytes = self.lib.zb_smoother_workspace_bytes(self.c1, self.c2, nx, ny)
        if nbytes == 0:
            raise ValueError(f"the smoother needs even grid sides, got {nx} x {ny}")
        act = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        s = L.ZbSmoother(self.c1, self.c2, self.w_bf16.data_ptr(), self.b.data_ptr(),
                         self.cmax, act.data_ptr(), nbytes, nx, ny)
        self._structs[key] = (s, act)
        return s

    def apply(self, nx, ny, f, cx, cy, dx, x=None, out=None):
        """``x + S(f - A x)`` on one ``nx x ny`` grid (float32 device
        tensors: f and x of ``nx*ny``, cx ``(nx+1)*ny``, cy ``nx*(ny+1)``;
        ``x=None`` starts from zero)."""
        import torch
        out = torch.empty_like(f) if out is None else out
        r = torch.empty_like(f)
        L.check(self.lib.zb_smoother_apply(
            C.byref(self.struct(nx, ny)), L.ptr(f), L.ptr(x) if x is not None else None,
            L.ptr(out), L.ptr(cx), L.ptr(cy), L.ptr(r), nx, ny, float(dx), int(x is None),
            L.stream_ptr()), "smoother_apply")
        return out

    def state_dict(self):
        return {"c1": self.c1, "c2": self.c2, "cmax": self.cmax,
                "w": self.w.detach().cpu(), "b": self.b.detach().cpu()}

    def load_state_dict(self, sd):
        if (int(sd["c1"]), int(sd["c2"])) != (self.c1, self.c2):
            raise ValueError("channel mismatch")
        self.w.copy_(sd["w"].to(self.w))
        self.b.copy_(sd["b"].to(self.b))
        self.cmax = float(sd["cmax"])
        for s, _ in self._structs.values():
            s.cmax = self.cmax
        self.refresh()

    def save(self, path):
        import torch
        torch.save(self.state_dict(), path)

    @classmethod
    def load(cls, path, device=None):
        import torch
        sd = torch.load(path, map_location="cpu")
        obj = cls(sd["c1"], sd["c2"], sd["cmax"], device=device)
        obj.load_state_dict(sd)
        return obj


class SmootherTrainer:
    """Adam training of a :class:`LearnedSmoother` on batches of ``n x n``
    patches by the libzb kernels (forward, backward, Adam); the loss is the
    residual left after one smoother application,
    ``mean_b |r_b - A_b S(r_b)|^2 / |r_b|^2`` (Dirichlet walls on the patch).
    The reference's loop (``train_vcycle_structured_poisson.py`` :266-306)
    uses Adam with lr 6e-3 on an MSE to the exact solution."""

    def __init__(self, smoother, batch=64, n=32, lr=3e-3):
        import torch
        self.sm = smoother
        self.lib = smoother.lib
        self.batch, self.n, self.lr = int(batch), int(n), float(lr)
        dev = smoother.device
        nbytes = self.lib.zb_unet_train_workspace_bytes(smoother.c1, smoother.c2, self.batch,
                                                        self.n)
        if nbytes == 0:
            raise ValueError("unsupported training shape (batch 1..512, even n >= 4)")
        z = lambda k: torch.zeros(k, dtype=torch.float32, device=dev)  # noqa: E731
        self.m_w, self.v_w, self.g_w = z(smoother.nw), z(smoother.nw), z(smoother.nw)
        self.m_b, self.v_b, self.g_b = z(smoother.nb), z(smoother.nb), z(smoother.nb)
        self.b_shadow = torch.zeros(smoother.nb, dtype=torch.bfloat16, device=dev)
        self.act = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float64, device=dev)
        self.t = L.ZbUnetTrainer(
            smoother.c1, smoother.c2, self.batch, self.n, smoother.cmax,
            smoother.w.data_ptr(), smoother.b.data_ptr(), self.m_w.data_ptr(),
            self.v_w.data_ptr(), self.m_b.data_ptr(), self.v_b.data_ptr(),
            self.g_w.data_ptr(), self.g_b.data_ptr(), smoother.w_bf16.data_ptr(),
            self.b_shadow.data_ptr(), self.act.data_ptr())
        self.step_count = 0

    def _check(self, r, cx, cy):
        B, n = self.batch, self.n
        if r.numel() != B * n * n or cx.numel() != B * (n + 1) * n or \
                cy.numel() != B * n * (n + 1):
            raise ValueError("batch shapes do not match the trainer")
        for t in (r, cx, cy):
            if t.dtype.itemsize != 4 or not t.is_contiguous():
                raise ValueError("patches must be contiguous float32")

    def forward(self, r, cx, cy, dx):
        """``S(r)`` for a batch (``(B, n, n)`` float32)."""
        import torch
        self._check(r, cx, cy)
        y = torch.empty_like(r)
        L.check(self.lib.zb_unet_forward(C.byref(self.t), L.ptr(r), L.ptr(cx), L.ptr(cy),
                                         float(dx), L.ptr(y), L.stream_ptr()), "unet_forward")
        return y

    def loss_and_grad(self, r, cx, cy, dx, target=None):
        """Loss (device float64 tensor) and gradients into ``g_w``, ``g_b``:
        the residual loss, or with ``target`` (the exact errors ``e``,
        ``A e = r``) the energy-norm loss."""
        self._check(r, cx, cy)
        if target is not None and (target.shape != r.shape or not target.is_contiguous()):
            raise ValueError("target must match r")
        L.check(self.lib.zb_unet_backward(C.byref(self.t), L.ptr(r),
                                          L.ptr(target) if target is not None else None,
                                          L.ptr(cx), L.ptr(cy), float(dx), L.ptr(self.loss),
                                          L.stream_ptr()), "unet_backward")
        return self.loss

    def step(self, r, cx, cy, dx, lr=None, target=None):
        """One Adam step on a batch; returns the batch loss (device tensor,
        before the update)."""
        loss = self.loss_and_grad(r, cx, cy, dx, target)
        self.step_count += 1
        L.check(self.lib.zb_unet_adam(C.byref(self.t), float(self.lr if lr is None else lr),
                                      self.step_count, L.stream_ptr()), "unet_adam")
        return loss

    def fit(self, patches, steps=2000, seed=0, lr_final=None, log_every=0):
        """Train on a :class:`PatchSet` for ``steps`` Adam steps with random
        batches (cosine decay to ``lr_final``).  Returns the loss history
        (host floats every ``log_every`` steps, one sync each)."""
        import torch
        g = torch.Generator(device=patches.r.device).manual_seed(int(seed))
        lr0 = self.lr
        lr1 = lr0 * 0.1 if lr_final is None else float(lr_final)
        hist = []
        for s in range(int(steps)):
            idx = torch.randint(0, patches.count, (self.batch,), generator=g,
                                device=patches.r.device)
            r, cx, cy = patches.batch(idx)
            e = patches.e[idx].contiguous() if patches.e is not None else None
            lr = lr1 + 0.5 * (lr0 - lr1) * (1.0 + math.cos(math.pi * s / max(1, steps)))
            loss = self.step(r, cx, cy, patches.dx, lr=lr, target=e)
            if log_every and (s % log_every == 0 or s == steps - 1):
                hist.append((s, float(loss.item())))
        return hist


class PatchSet:
    """Training patches on the device: residual/right-hand-side patches
    ``r (N, n, n)`` with their face coefficients ``cx (N, n+1, n)``,
    ``cy (N, n, n+1)``, optionally the exact errors ``e (N, n, n)`` that solve
    ``A e = r`` on the whole grid, all float32, grid spacing ``dx``."""

    def __init__(self, r, cx, cy, dx, e=None):
        self.r, self.cx, self.cy, self.dx, self.e = r, cx, cy, float(dx), e
        self.count = r.shape[0]

    def batch(self, idx):
        return (self.r[idx].contiguous(), self.cx[idx].contiguous(), self.cy[idx].contiguous())

    @staticmethod
    def cut(fields, cx, cy, nx, ny, n, count, generator, targets=None, min_rms=0.0):
        """Random ``n x n`` patches of the grid fields ``fields (K, nx*ny)``
        (and of ``targets``, same shape) with the matching windows of
        ``cx ((nx+1)*ny)``, ``cy (nx*(ny+1))``.  Patches whose RMS is below
        ``min_rms`` times the RMS of their source field are dropped (patches
        without signal teach nothing).  Returns ``(r, cx, cy, e or None)``."""
        import torch
        dev = fields.device
        K = fields.shape[0]
        k = torch.randint(0, K, (count,), generator=generator, device=dev)
        i0 = torch.randint(0, nx - n + 1, (count,), generator=generator, device=dev)
        j0 = torch.randint(0, ny - n + 1, (count,), generator=generator, device=dev)
        a = torch.arange(n, device=dev)
        a1 = torch.arange(n + 1, device=dev)
        ii = i0[:, None, None] + a[None, :, None]
        jj = j0[:, None, None] + a[None, None, :]
        F = fields.view(K, nx, ny)
        r = F[k[:, None, None], ii, jj]
        CX = cx.view(nx + 1, ny)
        CY = cy.view(nx, ny + 1)
        pcx = CX[i0[:, None, None] + a1[None, :, None], jj[:, :1, :].expand(-1, n + 1, -1)]
        pcy = CY[ii[:, :, :1].expand(-1, -1, n + 1), j0[:, None, None] + a1[None, None, :]]
        e = targets.view(K, nx, ny)[k[:, None, None], ii, jj] if targets is not None else None
        keep = None
        if min_rms > 0.0:
            src = fields.float().pow(2).mean(dim=1).sqrt()
            rms = r.float().pow(2).mean(dim=(1, 2)).sqrt()
            keep = rms > min_rms * src[k]
        out = [r.float(), pcx.float(), pcy.float(), e.float() if e is not None else None]
        if keep is not None:
            out = [t[keep] if t is not None else None for t in out]
        return tuple(t.contiguous() if t is not None else None for t in out)


def solver_training_set(n_grid=256, seeds=(1, 2, 3, 4), steps=3, patch=32, count=10000,
                        tol=1e-8, seed=0, device=None, targets=True):
    """Training patches generated by the solver itself: short seeded Chorin
    marches (dam break over Gaussian bumps, ``n_grid^2``, plain multigrid
    preconditioner) whose pressure solves are re-run step by step to record
    the residual each V-cycle leaves, ``r' = r - A M r`` -- the input of the
    learned post-smoother -- and, with ``targets``, the exact error behind it
    (``A e' = r'`` solved to 1e-10), the output it should produce.  Returns a
    :class:`PatchSet` of ``count`` random ``patch x patch`` windows with
    signal, with their face coefficients."""
    import torch
    import zoomy_b200 as zb
    from .fvm.chorin import ChorinSolver
    from .workloads import cartesian_centers, circular_dam_state
    tags = ("left", "right", "bottom", "top")
    snaps = []
    for s in seeds:
        state = circular_dam_state(cartesian_centers(n_grid), seed=int(s))
        model = zb.ShallowWater2D(boundary_conditions={t: "wall" for t in tags},
                                  initial_conditions=state)
        nsm = zb.NumericalSystemModel.from_system_model(model, zb.ReconstructionSpec(2, "minmod"),
                                                        "hll_hr")
        sol = ChorinSolver(pressure_tol=tol, precond="mg",
                           compute_dt=zb.timestepping.adaptive(0.45, 2),
                           reconstruction_variables="eta", free_surface_h_index=1, eps_wet=1e-6,
                           dtype="float32", device=device)
        Q, _ = sol.setup_simulation(zb.create_2d((0.0, 1.0, 0.0, 1.0), n_grid, n_grid), nsm)
        dt = sol.compute_timestep(Q)
        for k in range(int(steps)):
            Qs = sol._hyperbolic_stage(dt, k * dt, Q)
            P = sol.poisson
            P.setup(Qs[1])
            P.rhs(Qs, dt)
            post = []
            P.solve_stepwise(None, tol=tol, maxit=100, precond="mg", record_post=post)
            F = torch.stack(post)
            E = None
            if targets:
                errs = []
                for rp in post:
                    x, _, _ = P.solve(rp.double(), tol=1e-10, maxit=100, precond="mg")
                    errs.append(x.float().clone())
                E = torch.stack(errs)
            snaps.append((F, E, P.cx32.clone(), P.cy32.clone()))
            # march on with the proper pressure of this step
            P.setup(Qs[1])
            P.rhs(Qs, dt)
            P.solve(None, tol=tol, maxit=100, precond="mg")
            Q = sol._step_corrector(Qs, dt)
    g = torch.Generator(device=snaps[0][0].device).manual_seed(int(seed))
    per = -(-2 * int(count) // len(snaps))
    parts = [PatchSet.cut(F, cx, cy, n_grid, n_grid, patch, per, g, targets=E, min_rms=1e-2)
             for F, E, cx, cy in snaps]
    r = torch.cat([p[0] for p in parts])
    perm = torch.randperm(r.shape[0], generator=g, device=r.device)[:int(count)]
    cat = lambda i: torch.cat([p[i] for p in parts])[perm].contiguous()  # noqa: E731
    return PatchSet(cat(0), cat(1), cat(2), 1.0 / n_grid, e=cat(3) if targets else None)

"""Unstructured triangle mesh of the SWE path (host preparation, device upload).

The reference converts zoomy_core's ``LSQMesh`` into ``MeshJAX`` arrays
(``zoomy_jax/mesh/mesh.py:123-264``) and derives the runtime index sets in
``prepare_mesh`` (``zoomy_jax/fvm/solver2/context.py:99-163``).  Here the
same information is built once on the host with vectorised NumPy and uploaded
as int32 connectivity plus SoA geometry:

* faces: owner ``A``, neighbour ``B`` (``-1 - bf`` on a boundary face), unit
  normal out of ``A``, length, offsets face-centre minus cell-centre for both
  sides, the per-face inradius ``min(r_A, r_B)`` of the CFL law;
* cells: the three faces (``2 f + side``), inverse area, and the
  least-squares gradient stencil = the three face neighbours or boundary
  ghosts at ``2 (x_f - x_c)``; a ghost counts for derivative direction ``d``
  only if its normal has a component along ``d``.

Cells are renumbered in Morton order of their centroids so that face gathers
touch nearby memory.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

TAGS = ("left", "right", "bottom", "top")


def _morton(points, bits=16):
    p = np.asarray(points, dtype=np.float64)
    lo, hi = p.min(axis=0), p.max(axis=0)
    q = ((p - lo) / np.maximum(hi - lo, 1e-300) * ((1 << bits) - 1)).astype(np.uint64)

    def spread(v):
        v = v & np.uint64(0xFFFF)
        for s, m in ((8, 0x00FF00FF), (4, 0x0F0F0F0F), (2, 0x33333333), (1, 0x55555555)):
            v = (v | (v << np.uint64(s))) & np.uint64(m)
        return v
    return np.argsort(spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1)), kind="stable")


@dataclass
class TriangleMesh:
    vertices: np.ndarray
    triangles: np.ndarray
    cell_area: np.ndarray
    cell_center: np.ndarray
    cell_inradius: np.ndarray
    face_cells: np.ndarray       # (2, F) int64, B = -1 on boundary
    face_normal: np.ndarray      # (2, F)
    face_len: np.ndarray
    face_center: np.ndarray      # (F, 2)
    cell_faces: np.ndarray       # (C, 3) faces of each cell, increasing
    bf: np.ndarray               # boundary face ids
    bf_tag: np.ndarray           # 0..3 = left, right, bottom, top
    lsq_idx: np.ndarray          # (C, 3): neighbour cell or -1 - bf number
    lsq_w: np.ndarray            # (2, C, 3)
    dimension: int = 2
    extra: dict = field(default_factory=dict)

    @property
    def n_cells(self):
        return len(self.triangles)

    n_inner_cells = n_cells

    @property
    def n_faces(self):
        return self.face_cells.shape[1]

    @property
    def n_bf(self):
        return len(self.bf)

    def cell_centers(self):
        return self.cell_center.T.copy()

    # ── construction ─────────────────────────────────────────────────────
    @staticmethod
    def create(n_side, jitter=0.3, seed=0, domain=(0.0, 1.0, 0.0, 1.0)):
        """Delaunay triangulation of an ``n_side x n_side`` lattice with
        interior points jittered by U[-jitter, jitter] spacings (seeded);
        about ``2 n_side^2`` triangles."""
        P, T = lattice_triangulation(n_side, jitter, seed, domain)
        return TriangleMesh.from_points(P, T)

    @staticmethod
    def from_points(P, T):
        """Mesh from vertices ``(n, 2)`` and triangles ``(C, 3)`` (cell order
        kept; triangles re-oriented counter-clockwise)."""
        P = np.asarray(P, dtype=np.float64)
        T = np.asarray(T, dtype=np.int64).copy()
        a, b, c = P[T[:, 0]], P[T[:, 1]], P[T[:, 2]]
        cross = (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0])
        flip = cross < 0
        T[flip, 1], T[flip, 2] = T[flip, 2].copy(), T[flip, 1].copy()
        area = 0.5 * np.abs(cross)
        cen = (P[T[:, 0]] + P[T[:, 1]] + P[T[:, 2]]) / 3.0
        C = len(T)
        e = np.concatenate([T[:, [0, 1]], T[:, [1, 2]], T[:, [2, 0]]])
        own = np.tile(np.arange(C), 3)
        k = np.sort(e, axis=1)
        key = k[:, 0] * (len(P) + 1) + k[:, 1]
        order = np.argsort(key, kind="stable")
        ks = key[order]
        first = np.ones(len(ks), dtype=bool)
        first[1:] = ks[1:] != ks[:-1]
        fid = np.cumsum(first) - 1
        F = int(fid[-1]) + 1
        fc = np.full((2, F), -1, dtype=np.int64)
        fv = np.zeros((F, 2), dtype=np.int64)
        fc[0, fid[first]] = own[order[first]]
        fv[fid[first]] = e[order[first]]
        fc[1, fid[~first]] = own[order[~first]]
        va, vb = P[fv[:, 0]], P[fv[:, 1]]
        t = vb - va
        L = np.hypot(t[:, 0], t[:, 1])
        nrm = np.stack([t[:, 1], -t[:, 0]]) / L
        fcen = 0.5 * (va + vb)
        per = np.bincount(fc[0], weights=L, minlength=C)
        inb = fc[1] >= 0
        per += np.bincount(fc[1][inb], weights=L[inb], minlength=C)
        inr = 2.0 * area / per
        bf = np.nonzero(~inb)[0]
        nb = nrm[:, bf]
        tag = np.where(nb[0] < -0.5, 0, np.where(nb[0] > 0.5, 1, np.where(nb[1] < 0, 2, 3)))
        # cell -> faces (increasing face id)
        cc = np.concatenate([fc[0], fc[1][inb]])
        ff = np.concatenate([np.arange(F), np.arange(F)[inb]])
        o = np.lexsort((ff, cc))
        cell_faces = ff[o].reshape(C, 3)
        m = TriangleMesh(P, T, area, cen, inr, fc, nrm, L, fcen, cell_faces, bf,
                         tag.astype(np.int64), None, None)
        m._build_lsq()
        return m

    def _build_lsq(self):
        C = self.n_cells
        cf = self.cell_faces
        fc = self.face_cells[:, cf]                       # (2, C, 3)
        cells = np.arange(C)[:, None]
        other = np.where(fc[0] == cells, fc[1], fc[0])
        bnum = np.full(self.n_faces, -1, dtype=np.int64)
        bnum[self.bf] = np.arange(len(self.bf))
        ghost = other < 0
        xc = self.cell_center
        off = np.where(ghost[..., None], 2.0 * (self.face_center[cf] - xc[:, None, :]),
                       xc[np.maximum(other, 0)] - xc[:, None, :])
        nrm = self.face_normal[:, cf]
        W = np.zeros((2, C, 3))
        for d in range(2):
            use = (~ghost) | (np.abs(nrm[d]) > 1e-12)
            M = off * use[..., None]
            inv = np.linalg.inv(np.einsum("cki,ckj->cij", M, M))
            W[d] = np.einsum("cj,ckj->ck", inv[:, d, :], M)
        self.lsq_idx = np.where(ghost, -(bnum[cf] + 1), other)
        self.lsq_w = W

    # ── device upload ────────────────────────────────────────────────────
    def device_arrays(self, dtype, device, bc_kinds):
        """SoA device arrays the kernels read; ``bc_kinds`` = per-tag kind
        codes (left, right, bottom, top).  Returns a dict of torch tensors."""
        import torch
        C, F = self.n_cells, self.n_faces
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.int32, device=device)
        fl = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=device)
        cf = self.cell_faces
        xc = self.cell_center
        r = self.face_center[cf] - xc[:, None, :]                  # (C, 3, 2)
        side = (self.face_cells[1, cf] == np.arange(C)[:, None]).astype(np.int64)
        fc = self.face_cells
        A = fc[0]
        B = fc[1]
        bnum = np.full(F, -1, dtype=np.int64)
        bnum[self.bf] = np.arange(len(self.bf))
        Bcode = np.where(B >= 0, B, -(bnum + 1))
        rA = self.face_center - xc[A]
        rB = np.where((B >= 0)[:, None], self.face_center - xc[np.maximum(B, 0)], rA)
        inr_f = np.minimum(self.cell_inradius[A], self.cell_inradius[np.where(B >= 0, B, A)])
        kinds = np.asarray(bc_kinds, dtype=np.int64)[self.bf_tag]
        return {
            "lsq_idx": i32(self.lsq_idx.T), "lsq_wx": fl(self.lsq_w[0].T),
            "lsq_wy": fl(self.lsq_w[1].T), "cf_rx": fl(r[:, :, 0].T), "cf_ry": fl(r[:, :, 1].T),
            "cell_face": i32((2 * cf + side).T), "cell_inv_area": fl(1.0 / self.cell_area),
            "face_a": i32(A), "face_b": i32(Bcode), "face_nx": fl(self.face_normal[0]),
            "face_ny": fl(self.face_normal[1]), "face_len": fl(self.face_len),
            "face_rax": fl(rA[:, 0]), "face_ray": fl(rA[:, 1]),
            "face_rbx": fl(rB[:, 0]), "face_rby": fl(rB[:, 1]),
            "face_inr": torch.as_tensor(inr_f, dtype=torch.float64, device=device),
            "bf_kind": i32(kinds), "bf_nx": fl(self.face_normal[0, self.bf]),
            "bf_ny": fl(self.face_normal[1, self.bf]),
        }


def lattice_triangulation(n_side, jitter=0.3, seed=0, domain=(0.0, 1.0, 0.0, 1.0)):
    """Vertices and Morton-ordered triangles of the Delaunay triangulation of
    an ``n_side x n_side`` lattice with interior points jittered by
    U[-jitter, jitter] spacings (seeded) -- the mesh generation that
    :meth:`TriangleMesh.create` and :meth:`DeviceTriangleMesh.create` share."""
    from scipy.spatial import Delaunay
    rng = np.random.default_rng(seed)
    x0, x1, y0, y1 = domain
    hx, hy = (x1 - x0) / (n_side - 1), (y1 - y0) / (n_side - 1)
    gx, gy = np.meshgrid(np.linspace(x0, x1, n_side), np.linspace(y0, y1, n_side),
                         indexing="ij")
    P = np.stack([gx.reshape(-1), gy.reshape(-1)], axis=1)
    jit = rng.uniform(-jitter, jitter, size=P.shape) * np.array([hx, hy])
    jit[np.isclose(P[:, 0], x0) | np.isclose(P[:, 0], x1), 0] = 0.0
    jit[np.isclose(P[:, 1], y0) | np.isclose(P[:, 1], y1), 1] = 0.0
    P = P + jit
    T = Delaunay(P).simplices.astype(np.int64)
    cen = P[T].mean(axis=1)
    return P, T[_morton(cen)]


class DeviceTriangleMesh:
    """Triangle mesh whose faces, geometry and least-squares stencils are
    prepared on the GPU (``zb_trimesh_match`` / ``zb_trimesh_fill``) from
    vertices and triangles: the host conversion of zoomy_core's ``LSQMesh``
    into ``MeshJAX`` arrays (``zoomy_jax/mesh/mesh.py:123-264``) and
    ``prepare_mesh``'s index sets (``zoomy_jax/fvm/solver2/context.py:99-163``)
    as device kernels.  The solver sees the interface of
    :class:`TriangleMesh` (``n_cells``, ``n_faces``, ``n_bf``,
    ``cell_centers()``, ``cell_inradius``, ``device_arrays()``); faces are
    numbered by (owner cell, local edge), the owner of a shared edge being
    the lower cell index, so face-indexed arrays differ from the host
    builder's by that renumbering only."""

    dimension = 2

    def __init__(self, P, T, device="cuda"):
        import ctypes as C
        import torch
        from . import _lib as L
        L.require_cuda()
        self.lib = L.load()
        self.vertices = np.ascontiguousarray(P, dtype=np.float64)
        self.triangles = np.ascontiguousarray(T, dtype=np.int32)
        if self.vertices.ndim != 2 or self.vertices.shape[1] != 2:
            raise ValueError("vertices must be (n, 2)")
        if self.triangles.ndim != 2 or self.triangles.shape[1] != 3:
            raise ValueError("triangles must be (C, 3)")
        dev = torch.device(device)
        self._P = torch.as_tensor(self.vertices, device=dev)
        self._T = torch.as_tensor(self.triangles, device=dev)
        n = len(self.triangles)
        nb = self.lib.zb_trimesh_scratch_bytes(n)
        if nb == 0:
            raise L.ZbError("too many triangles for int32 half-edge numbers")
        self._scratch = torch.empty(nb, dtype=torch.uint8, device=dev)
        self._scratch_bytes = nb
        nf, nbf = C.c_int32(0), C.c_int32(0)
        L.check(self.lib.zb_trimesh_match(L.ptr(self._P), len(self.vertices), L.ptr(self._T),
                                          n, L.ptr(self._scratch), C.c_size_t(nb),
                                          C.byref(nf), C.byref(nbf), L.stream_ptr()),
                "zb_trimesh_match")
        self.n_faces, self.n_bf = nf.value, nbf.value
        self._geo = None
        self._arrays = {}

    @staticmethod
    def create(n_side, jitter=0.3, seed=0, domain=(0.0, 1.0, 0.0, 1.0), device="cuda"):
        """The lattice triangulation of :meth:`TriangleMesh.create`, prepared
        on the GPU."""
        P, T = lattice_triangulation(n_side, jitter, seed, domain)
        return DeviceTriangleMesh(P, T, device)

    @property
    def n_cells(self):
        return len(self.triangles)

    n_inner_cells = n_cells

    def _host_geometry(self):
        # centroid (vertex order after the counter-clockwise flip, as the
        # device kernels and TriangleMesh.from_points take it) and inradius
        if self._geo is None:
            P, T = self.vertices, self.triangles.astype(np.int64)
            a, b, c = P[T[:, 0]], P[T[:, 1]], P[T[:, 2]]
            cross = (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0])
            flip = cross < 0
            b2 = np.where(flip[:, None], c, b)
            c2 = np.where(flip[:, None], b, c)
            area = 0.5 * np.abs(cross)
            per = (np.hypot(*(b2 - a).T) + np.hypot(*(c2 - b2).T) + np.hypot(*(a - c2).T))
            self._geo = ((a + b2 + c2) / 3.0, area, 2.0 * area / per)
        return self._geo

    @property
    def cell_center(self):
        return self._host_geometry()[0]

    @property
    def cell_area(self):
        return self._host_geometry()[1]

    @property
    def cell_inradius(self):
        return self._host_geometry()[2]

    def cell_centers(self):
        return self.cell_center.T.copy()

    def device_arrays(self, dtype, device, bc_kinds):
        """Allocate the SoA device arrays the kernels read and fill them on the
        GPU; ``bc_kinds`` = kind codes of the left, right, bottom and top
        sides.  Returns a dict of torch tensors (the keys of
        :meth:`TriangleMesh.device_arrays`)."""
        import ctypes as C
        import torch
        from . import _lib as L
        dev = torch.device(device)
        if dtype not in (torch.float32, torch.float64):
            raise ValueError("dtype must be torch.float32 or torch.float64")
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        key = (dtype, str(dev), tuple(int(k) for k in bc_kinds))
        if key in self._arrays:
            return self._arrays[key]
        n, F, nbf = self.n_cells, self.n_faces, self.n_bf
        i32 = lambda *sh: torch.empty(sh, dtype=torch.int32, device=dev)  # noqa: E731
        fl = lambda *sh: torch.empty(sh, dtype=dtype, device=dev)  # noqa: E731
        d = {"lsq_idx": i32(3, n), "lsq_wx": fl(3, n), "lsq_wy": fl(3, n),
             "cf_rx": fl(3, n), "cf_ry": fl(3, n), "cell_face": i32(3, n),
             "cell_inv_area": fl(n), "face_a": i32(F), "face_b": i32(F), "face_nx": fl(F),
             "face_ny": fl(F), "face_len": fl(F), "face_rax": fl(F), "face_ray": fl(F),
             "face_rbx": fl(F), "face_rby": fl(F),
             "face_inr": torch.empty(F, dtype=torch.float64, device=dev),
             "bf_kind": i32(max(nbf, 1)), "bf_nx": fl(max(nbf, 1)), "bf_ny": fl(max(nbf, 1))}
        ms = L.ZbTriMesh()
        ms.n_cells, ms.n_faces, ms.n_bf = n, F, nbf
        for name in L.TRI_MESH_FIELDS:
            setattr(ms, name, d[name].data_ptr())
        kinds = (C.c_int32 * 4)(*[int(k) for k in bc_kinds])
        code = L.ZB_F32 if dtype == torch.float32 else L.ZB_F64
        L.check(self.lib.zb_trimesh_fill(L.ptr(self._P), n, kinds, code, L.ptr(self._scratch),
                                         C.c_size_t(self._scratch_bytes), C.byref(ms),
                                         L.stream_ptr()), "zb_trimesh_fill")
        self._arrays[key] = d
        return d


def create_tri(n_side, jitter=0.3, seed=0, domain=(0.0, 1.0, 0.0, 1.0)):
    return TriangleMesh.create(n_side, jitter, seed, domain)

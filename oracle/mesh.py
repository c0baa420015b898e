"""Face-based meshes for the oracle -- TEST INFRASTRUCTURE ONLY (see package doc).

A ``Mesh`` carries exactly the arrays the reference's runtime mesh view holds
(``zoomy_jax/fvm/solver2/context.py:38-73``, ``MeshRT``; the source container is
``zoomy_jax/mesh/mesh.py:123-169``, ``MeshJAX``):

* ``face_cells (2, F)``: owner, neighbour; ``-1`` neighbour on boundary faces.
* ``face_normals (dim, F)``: unit normal, outward from the owner.
* ``face_volumes (F,)``, ``face_centers (F, dim)``.
* ``cell_volumes (C,)``, ``cell_centers (C, dim)``, ``cell_inradius (C,)``.
* boundary faces ``bf (n_bf,)`` with owner cell ``bf_cell``, side tag
  ``bf_tag`` and periodic partner ``bf_partner`` (``-1`` if not periodic).
* the least-squares gradient stencil (``lsq_*``), see ``_lsq_weights``.

Cell numbering of the Cartesian builder is ``i * ny + j`` (``y`` fastest),
which is the numbering of the reference's ``LSQMesh.create_2d`` (pinned by the
golden ``swe_2d``: the x-fastest numbering misses it by 4.8e-2, this one
matches to 1.8e-16).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

TAGS_1D = ("left", "right")
TAGS_2D = ("left", "right", "bottom", "top")


@dataclass
class Mesh:
    dim: int
    n_cells: int
    n_faces: int
    face_cells: np.ndarray
    face_normals: np.ndarray
    face_volumes: np.ndarray
    face_centers: np.ndarray
    cell_volumes: np.ndarray
    cell_centers: np.ndarray
    cell_inradius: np.ndarray
    bf: np.ndarray
    bf_cell: np.ndarray
    bf_tag: np.ndarray
    tag_names: tuple
    bf_partner: np.ndarray = None
    # cell -> faces (incl. boundary), CSR
    cf_ptr: np.ndarray = None
    cf_idx: np.ndarray = None
    # LSQ stencil (CSR); lsq_idx >= 0: neighbour cell, < 0: ghost of boundary
    # face number (-idx - 1) (index into ``bf``); lsq_w (dim, nnz)
    lsq_ptr: np.ndarray = None
    lsq_idx: np.ndarray = None
    lsq_w: np.ndarray = None
    # structured metadata (Cartesian builder only)
    shape: tuple = None
    spacing: tuple = None
    origin: tuple = None
    extra: dict = field(default_factory=dict)

    # -- derived index sets (reference: context.py:104-119) -----------------
    @property
    def interior(self):
        return np.nonzero(self.face_cells[1] >= 0)[0]

    @property
    def iA(self):
        return self.face_cells[0]

    @property
    def iB_or_owner(self):
        """Neighbour of every face, the OWNER on boundary faces
        (``zoomy_jax/fvm/solver2/context.py:111-117``)."""
        nb = self.face_cells[1].copy()
        m = nb < 0
        nb[m] = self.face_cells[0][m]
        return nb

    @property
    def inradius_f(self):
        """Per-face min inradius of the two adjacent cells
        (``zoomy_jax/fvm/solver_jax.py:971-973``; owner on both sides at a
        boundary face, ``context.py:119-120``)."""
        ir = self.cell_inradius
        return np.minimum(ir[self.face_cells[0]], ir[self.iB_or_owner])

    def set_periodic(self, pairs):
        """Map boundary faces of tag ``a`` onto the facing cell of tag ``b``.

        After ``resolve_periodic_bcs`` the reference stores the PARTNER cell in
        ``boundary_face_cells`` (``zoomy_jax/fvm/solver2/context.py:122-125``).
        Here the partner sits in ``bf_partner``; only the Cartesian and 1-D
        builders know the geometry to pair faces.
        """
        pairfn = self.extra.get("periodic_partner")
        if pairfn is None:
            raise NotImplementedError("periodic pairing needs a structured mesh")
        self.bf_partner = np.full(len(self.bf), -1, dtype=np.int64)
        for a, b in pairs:
            ta = self.tag_names.index(a)
            for k in np.nonzero(self.bf_tag == ta)[0]:
                self.bf_partner[k] = pairfn(k, b)


def _csr_from_lists(lists):
    ptr = np.zeros(len(lists) + 1, dtype=np.int64)
    ptr[1:] = np.cumsum([len(x) for x in lists])
    idx = np.concatenate([np.asarray(x, dtype=np.int64) for x in lists]) \
        if ptr[-1] > 0 else np.zeros(0, np.int64)
    return ptr, idx


def _lsq_weights(mesh, nbr_lists):
    """Least-squares gradient weights, one set per derivative direction.

    The reference evaluates ``grad u_i = scale * A_i^T [u_nbr - u_i ; u_bf -
    u_i]`` (``zoomy_jax/fvm/reconstruction_jax.py:433-522``,
    ``zoomy_jax/mesh/mesh.py:74-120``) with the pseudo-inverse ``A_i`` built by
    zoomy_core's ``LSQMesh``.  Pinned here against the golden derivative aux
    rows of ``swe_2d`` (max error 1.6e-15) and ``parity``/``stoker_wet``:

    * degree-1 unweighted least squares over the stencil;
    * Cartesian 2-D stencil = the 8 cells of the 3x3 block, 1-D = the two face
      neighbours;
    * a boundary face contributes a ghost point at ``2 (x_face - x_cell)``
      (the docstring at ``reconstruction_jax.py:436-464``), and only to the
      derivative directions its normal has a component in (at a corner cell
      the x-derivative sees only the left/right ghost and the y-derivative
      only the bottom/top one -- the single rule that reproduces all four
      corners of the golden).
    """
    dim = mesh.dim
    C = mesh.n_cells
    cell_bfs = [[] for _ in range(C)]
    for k, c in enumerate(mesh.bf_cell):
        cell_bfs[int(c)].append(k)
    lists, wts = [], []
    xc = mesh.cell_centers
    fcen = mesh.face_centers
    nrm = mesh.face_normals
    for i in range(C):
        nb = list(nbr_lists[i])
        gh = cell_bfs[i]
        P = [xc[j] - xc[i] for j in nb]
        Pg = [2.0 * (fcen[mesh.bf[k]] - xc[i]) for k in gh]
        w = np.zeros((dim, len(nb) + len(gh)))
        for d in range(dim):
            use = [abs(nrm[d, mesh.bf[k]]) > 1e-12 for k in gh]
            pts = P + [p for p, u in zip(Pg, use) if u]
            M = np.asarray(pts, dtype=np.float64).reshape(-1, dim)
            pinv = np.linalg.pinv(M)          # (dim, n_pts)
            row = pinv[d]
            w[d, :len(nb)] = row[:len(nb)]
            gi = len(nb)
            for jj, u in enumerate(use):
                if u:
                    w[d, len(nb) + jj] = row[gi]
                    gi += 1
        lists.append(nb + [-(k + 1) for k in gh])
        wts.append(w)
    mesh.lsq_ptr, mesh.lsq_idx = _csr_from_lists(lists)
    mesh.lsq_w = np.concatenate(wts, axis=1) if wts else np.zeros((dim, 0))


def _cell_faces(mesh):
    """Cell -> faces CSR (faces in increasing face number per cell)."""
    fc = mesh.face_cells
    F = mesh.n_faces
    c = np.concatenate([fc[0], fc[1]])
    f = np.concatenate([np.arange(F), np.arange(F)])
    keep = c >= 0
    c, f = c[keep], f[keep]
    order = np.lexsort((f, c))
    mesh.cf_idx = f[order].astype(np.int64)
    counts = np.bincount(c, minlength=mesh.n_cells)
    mesh.cf_ptr = np.zeros(mesh.n_cells + 1, dtype=np.int64)
    mesh.cf_ptr[1:] = np.cumsum(counts)


def create_1d(x0, x1, n):
    """Uniform 1-D mesh on ``[x0, x1]`` (reference: ``LSQMesh.create_1d``)."""
    dx = (x1 - x0) / n
    xc = x0 + (np.arange(n) + 0.5) * dx
    F = n + 1
    fcells = np.full((2, F), -1, dtype=np.int64)
    fcells[0, 1:n] = np.arange(n - 1)
    fcells[1, 1:n] = np.arange(1, n)
    fcells[0, 0] = 0
    fcells[0, n] = n - 1
    nrm = np.ones((1, F))
    nrm[0, 0] = -1.0
    fcen = (x0 + np.arange(F) * dx).reshape(F, 1)
    m = Mesh(dim=1, n_cells=n, n_faces=F, face_cells=fcells,
             face_normals=nrm, face_volumes=np.ones(F),
             face_centers=fcen, cell_volumes=np.full(n, dx),
             cell_centers=xc.reshape(n, 1), cell_inradius=np.full(n, dx / 2),
             bf=np.array([0, n]), bf_cell=np.array([0, n - 1]),
             bf_tag=np.array([0, 1]), tag_names=TAGS_1D,
             shape=(n,), spacing=(dx,), origin=(x0,))
    m.bf_partner = np.full(2, -1, dtype=np.int64)
    m.extra["periodic_partner"] = lambda k, b: (n - 1 if k == 0 else 0)
    # interior cells: the two face neighbours; an end cell, which has only one,
    # takes the next cell beyond it as well (one-sided pair + its boundary
    # ghost) -- pinned by the derivative rows of the reference's bc_wall,
    # bc_periodic and bc_inflow goldens (tests/runtime/test_bc_runtime.py).
    nbrs = [[j for j in (i - 1, i + 1) if 0 <= j < n] for i in range(n)]
    if n >= 3:
        nbrs[0] = [1, 2]
        nbrs[n - 1] = [n - 2, n - 3]
    _lsq_weights(m, nbrs)
    _cell_faces(m)
    return m


def cart_faces(nx, ny):
    """Face numbering of the Cartesian builder: x-faces ``(i, j)``,
    ``i = 0..nx``, first (index ``i * ny + j``), then y-faces ``(i, j)``,
    ``j = 0..ny`` (index ``(nx + 1) * ny + i * (ny + 1) + j``)."""
    nfx = (nx + 1) * ny
    nfy = nx * (ny + 1)
    return nfx, nfy


def create_2d(x0, x1, y0, y1, nx, ny):
    """Uniform Cartesian mesh (reference: ``LSQMesh.create_2d(domain=(x0, x1,
    y0, y1), nx, ny)``, ``tests/runtime/test_swe_2d.py:34``).  Cell ``(i, j)``
    is number ``i * ny + j``."""
    dx = (x1 - x0) / nx
    dy = (y1 - y0) / ny
    C = nx * ny
    nfx, nfy = cart_faces(nx, ny)
    F = nfx + nfy
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    cid = (ii * ny + jj).reshape(-1)
    xc = np.stack([x0 + (ii.reshape(-1) + 0.5) * dx,
                   y0 + (jj.reshape(-1) + 0.5) * dy], axis=1)
    fcells = np.full((2, F), -1, dtype=np.int64)
    nrm = np.zeros((2, F))
    fvol = np.zeros(F)
    fcen = np.zeros((F, 2))
    # x-faces
    fi, fj = np.meshgrid(np.arange(nx + 1), np.arange(ny), indexing="ij")
    fi = fi.reshape(-1)
    fj = fj.reshape(-1)
    fx = fi * ny + fj
    left = fi - 1
    right = fi
    own = np.where(fi == 0, right, left)
    nb = np.where((fi == 0) | (fi == nx), -1, right)
    fcells[0, fx] = own * ny + fj
    fcells[1, fx] = np.where(nb >= 0, nb * ny + fj, -1)
    nrm[0, fx] = np.where(fi == 0, -1.0, 1.0)
    fvol[fx] = dy
    fcen[fx, 0] = x0 + fi * dx
    fcen[fx, 1] = y0 + (fj + 0.5) * dy
    # y-faces
    gi, gj = np.meshgrid(np.arange(nx), np.arange(ny + 1), indexing="ij")
    gi = gi.reshape(-1)
    gj = gj.reshape(-1)
    fy = nfx + gi * (ny + 1) + gj
    own = np.where(gj == 0, gj, gj - 1)
    nb = np.where((gj == 0) | (gj == ny), -1, gj)
    fcells[0, fy] = gi * ny + own
    fcells[1, fy] = np.where(nb >= 0, gi * ny + nb, -1)
    nrm[1, fy] = np.where(gj == 0, -1.0, 1.0)
    fvol[fy] = dx
    fcen[fy, 0] = x0 + (gi + 0.5) * dx
    fcen[fy, 1] = y0 + gj * dy
    bmask = fcells[1] < 0
    bf = np.nonzero(bmask)[0]
    tag = np.zeros(len(bf), dtype=np.int64)
    isx = bf < nfx
    tag[isx & (nrm[0, bf] < 0)] = 0
    tag[isx & (nrm[0, bf] > 0)] = 1
    tag[~isx & (nrm[1, bf] < 0)] = 2
    tag[~isx & (nrm[1, bf] > 0)] = 3
    inr = np.full(C, dx * dy / (dx + dy))   # 2 * area / perimeter
    m = Mesh(dim=2, n_cells=C, n_faces=F, face_cells=fcells,
             face_normals=nrm, face_volumes=fvol, face_centers=fcen,
             cell_volumes=np.full(C, dx * dy), cell_centers=xc,
             cell_inradius=inr, bf=bf, bf_cell=fcells[0, bf], bf_tag=tag,
             tag_names=TAGS_2D, shape=(nx, ny), spacing=(dx, dy),
             origin=(x0, y0))
    m.bf_partner = np.full(len(bf), -1, dtype=np.int64)

    def partner(k, _b):
        c = int(m.bf_cell[k])
        i, j = divmod(c, ny)
        t = TAGS_2D[int(m.bf_tag[k])]
        if t == "left":
            return (nx - 1) * ny + j
        if t == "right":
            return j
        if t == "bottom":
            return i * ny + ny - 1
        return i * ny
    m.extra["periodic_partner"] = partner
    _cart_lsq(m)
    _cell_faces(m)
    return m


def _cart_lsq(m):
    """Vectorised ``_lsq_weights`` for the Cartesian mesh: a padded stencil
    of 10 slots per cell (the 3x3 block in row-major (a, b) order, then the
    ghost of the x-boundary face, then the ghost of the y-boundary face); a
    missing slot points at the cell itself with weight 0.  Cells fall into 9
    classes (first / interior / last row and column) that share weights."""
    nx, ny = m.shape
    dx, dy = m.spacing
    C = nx * ny
    ii, jj = np.divmod(np.arange(C), ny)
    ci = np.where(ii == 0, 0, np.where(ii == nx - 1, 2, 1))
    cj = np.where(jj == 0, 0, np.where(jj == ny - 1, 2, 1))
    # bf number of each cell's boundary faces
    nfx, _ = cart_faces(nx, ny)
    bnum = np.full(m.n_faces, -1, dtype=np.int64)
    bnum[m.bf] = np.arange(len(m.bf))
    fxl = ii * ny + jj                      # x-face (i, j) is the left face
    fxr = (ii + 1) * ny + jj
    fyb = nfx + ii * (ny + 1) + jj
    fyt = nfx + ii * (ny + 1) + jj + 1
    gx = np.where(ii == 0, bnum[fxl], np.where(ii == nx - 1, bnum[fxr], -1))
    gy = np.where(jj == 0, bnum[fyb], np.where(jj == ny - 1, bnum[fyt], -1))
    offs = [(a, b) for a in (-1, 0, 1) for b in (-1, 0, 1) if a or b]
    idx = np.zeros((C, 10), dtype=np.int64)
    W = np.zeros((2, C, 10))
    for k, (a, b) in enumerate(offs):
        ni, nj = ii + a, jj + b
        ok = (ni >= 0) & (ni < nx) & (nj >= 0) & (nj < ny)
        idx[:, k] = np.where(ok, ni * ny + nj, np.arange(C))
    idx[:, 8] = np.where(gx >= 0, -(gx + 1), np.arange(C))
    idx[:, 9] = np.where(gy >= 0, -(gy + 1), np.arange(C))
    for a_cls in range(3):
        for b_cls in range(3):
            sel = (ci == a_cls) & (cj == b_cls)
            if not sel.any():
                continue
            r = np.nonzero(sel)[0][0]
            i0, j0 = ii[r], jj[r]
            pts, slots = [], []
            for k, (a, b) in enumerate(offs):
                if 0 <= i0 + a < nx and 0 <= j0 + b < ny:
                    pts.append((a * dx, b * dy))
                    slots.append(k)
            for d in range(2):
                P = list(pts)
                S = list(slots)
                if d == 0 and gx[r] >= 0:
                    P.append((2.0 * (0.5 * dx) * (-1 if i0 == 0 else 1), 0.0))
                    S.append(8)
                if d == 1 and gy[r] >= 0:
                    P.append((0.0, 2.0 * (0.5 * dy) * (-1 if j0 == 0 else 1)))
                    S.append(9)
                row = np.linalg.pinv(np.asarray(P))[d]
                w = np.zeros(10)
                w[S] = row
                W[d, sel] = w
    m.lsq_ptr = np.arange(0, 10 * C + 1, 10, dtype=np.int64)
    m.lsq_idx = idx.reshape(-1)
    m.lsq_w = W.reshape(2, -1)


def morton_order(points, bits=16):
    """Z-order (Morton) permutation of 2-D points, used to renumber the
    unstructured mesh so that face gathers hit nearby cells."""
    p = np.asarray(points, dtype=np.float64)
    lo = p.min(axis=0)
    hi = p.max(axis=0)
    q = ((p - lo) / np.maximum(hi - lo, 1e-300) * ((1 << bits) - 1)).astype(np.uint64)

    def spread(v):
        v = v & np.uint64(0xFFFF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF)
        v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F)
        v = (v | (v << np.uint64(2))) & np.uint64(0x33333333)
        v = (v | (v << np.uint64(1))) & np.uint64(0x55555555)
        return v
    key = spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1))
    return np.argsort(key, kind="stable")


def create_tri(n_side, jitter=0.3, seed=0, domain=(0.0, 1.0, 0.0, 1.0),
               build_lsq=True):
    """Delaunay triangulation of seeded jittered lattice points.

    ``n_side x n_side`` lattice points on the domain, interior points jittered
    by ``jitter * spacing`` (boundary points stay on the boundary), giving about
    ``2 n_side^2`` triangles, renumbered in Morton order of their centroids.
    """
    from scipy.spatial import Delaunay
    rng = np.random.default_rng(seed)
    x0, x1, y0, y1 = domain
    hx = (x1 - x0) / (n_side - 1)
    hy = (y1 - y0) / (n_side - 1)
    gx, gy = np.meshgrid(np.linspace(x0, x1, n_side),
                         np.linspace(y0, y1, n_side), indexing="ij")
    P = np.stack([gx.reshape(-1), gy.reshape(-1)], axis=1)
    jit = rng.uniform(-jitter, jitter, size=P.shape) * np.array([hx, hy])
    onx = (np.isclose(P[:, 0], x0) | np.isclose(P[:, 0], x1))
    ony = (np.isclose(P[:, 1], y0) | np.isclose(P[:, 1], y1))
    jit[onx, 0] = 0.0
    jit[ony, 1] = 0.0
    P = P + jit
    T = Delaunay(P).simplices.astype(np.int64)
    cen = (P[T[:, 0]] + P[T[:, 1]] + P[T[:, 2]]) / 3.0
    T = T[morton_order(cen)]
    return tri_from_points(P, T, build_lsq=build_lsq)


def tri_from_points(P, T, build_lsq=True):
    """Face-based triangle mesh from vertices ``P (n, 2)`` and triangles
    ``T (C, 3)``, keeping the given cell order.  Faces are numbered by sorted
    vertex pair; the owner is the first triangle listing the edge, the normal
    points out of it; the boundary tag follows the outward normal
    (left/right/bottom/top for |n_x| > 0.5 / otherwise)."""
    P = np.asarray(P, dtype=np.float64)
    T = np.asarray(T, dtype=np.int64).copy()
    a, b, c = P[T[:, 0]], P[T[:, 1]], P[T[:, 2]]
    cross = (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0])
    neg = cross < 0
    T[neg, 1], T[neg, 2] = T[neg, 2].copy(), T[neg, 1].copy()
    area = 0.5 * np.abs(cross)
    cen = (P[T[:, 0]] + P[T[:, 1]] + P[T[:, 2]]) / 3.0
    C = len(T)
    e = np.concatenate([T[:, [0, 1]], T[:, [1, 2]], T[:, [2, 0]]], axis=0)
    owner = np.concatenate([np.arange(C)] * 3)
    key = np.sort(e, axis=1)
    k1 = key[:, 0] * (len(P) + 1) + key[:, 1]
    order = np.argsort(k1, kind="stable")
    k1s = k1[order]
    first = np.ones(len(k1s), dtype=bool)
    first[1:] = k1s[1:] != k1s[:-1]
    fid_sorted = np.cumsum(first) - 1
    F = int(fid_sorted[-1] + 1)
    fcells = np.full((2, F), -1, dtype=np.int64)
    fverts = np.zeros((F, 2), dtype=np.int64)
    # first occurrence = owner (its directed ccw edge gives the outward normal)
    occ_first = order[first]
    fcells[0, fid_sorted[first]] = owner[occ_first]
    fverts[fid_sorted[first]] = e[occ_first]
    second = ~first
    fcells[1, fid_sorted[second]] = owner[order[second]]
    va = P[fverts[:, 0]]
    vb = P[fverts[:, 1]]
    t = vb - va
    L = np.sqrt((t ** 2).sum(axis=1))
    # ccw triangle: outward normal of directed edge (a->b) is (t_y, -t_x)
    nrm = np.stack([t[:, 1], -t[:, 0]], axis=0) / L
    fcen = 0.5 * (va + vb)
    # perimeter per cell
    per = np.zeros(C)
    np.add.at(per, fcells[0], L)
    m1 = fcells[1] >= 0
    np.add.at(per, fcells[1][m1], L[m1])
    inr = 2.0 * area / per
    bf = np.nonzero(fcells[1] < 0)[0]
    tag = np.zeros(len(bf), dtype=np.int64)
    nb_ = nrm[:, bf]
    tag[nb_[0] < -0.5] = 0
    tag[nb_[0] > 0.5] = 1
    tag[(np.abs(nb_[0]) <= 0.5) & (nb_[1] < 0)] = 2
    tag[(np.abs(nb_[0]) <= 0.5) & (nb_[1] > 0)] = 3
    m = Mesh(dim=2, n_cells=C, n_faces=F, face_cells=fcells,
             face_normals=nrm, face_volumes=L, face_centers=fcen,
             cell_volumes=area, cell_centers=cen, cell_inradius=inr,
             bf=bf, bf_cell=fcells[0, bf], bf_tag=tag, tag_names=TAGS_2D)
    m.bf_partner = np.full(len(bf), -1, dtype=np.int64)
    m.extra["vertices"] = P
    m.extra["triangles"] = T
    _cell_faces(m)
    if build_lsq:
        build_tri_lsq(m)
    return m


def build_tri_lsq(m):
    """Vectorised LSQ weights for the triangle stencil (face neighbours plus
    boundary ghosts; every ghost counts in both directions because triangle
    boundary normals are general -- for axis-aligned boundary faces the
    direction rule of ``_lsq_weights`` would drop it from one direction, and
    that rule is applied here too)."""
    C = m.n_cells
    dim = 2
    # per cell: 3 faces -> neighbour or ghost
    cf = m.cf_idx.reshape(C, 3)
    fc = m.face_cells[:, cf]                 # (2, C, 3)
    cells = np.arange(C)[:, None]
    other = np.where(fc[0] == cells, fc[1], fc[0])   # -1 at boundary
    bnum = np.full(m.n_faces, -1, dtype=np.int64)
    bnum[m.bf] = np.arange(len(m.bf))
    isg = other < 0
    xc = m.cell_centers
    off = np.where(isg[..., None],
                   2.0 * (m.face_centers[cf] - xc[:, None, :]),
                   xc[np.maximum(other, 0)] - xc[:, None, :])   # (C, 3, 2)
    nrm = m.face_normals[:, cf]              # (2, C, 3)
    W = np.zeros((dim, C, 3))
    for d in range(dim):
        use = (~isg) | (np.abs(nrm[d]) > 1e-12)
        M = off * use[..., None]
        MtM = np.einsum("cki,ckj->cij", M, M)
        inv = np.linalg.inv(MtM)
        W[d] = np.einsum("cj,ckj->ck", inv[:, d, :], M)
    idx = np.where(isg, -(bnum[cf] + 1), other)
    m.lsq_ptr = np.arange(0, 3 * C + 1, 3, dtype=np.int64)
    m.lsq_idx = idx.reshape(-1)
    m.lsq_w = W.reshape(dim, -1)

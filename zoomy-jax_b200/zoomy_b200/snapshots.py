"""Asynchronous snapshot output of a march.

The reference writes snapshot ``i`` of a run to an HDF5 file as the group
``fields/iteration_i`` holding ``time``, ``Q`` and ``Qaux``
(``zoomy_jax/misc/io.py:12-81``), from an ordered host callback inside its
time loop: the loop waits for each write.  Here a snapshot costs the march one
device-to-device copy of the state (and of its aux rows) into a staging slot
on the launching stream; the copy to pinned host memory runs on a side stream
and a writer thread writes the file, so the steps that follow overlap the
transfer and the disk.  A ring of ``slots`` staging slots bounds the memory; a
snapshot that finds every slot still in flight waits for the oldest.

The file format: with ``h5py`` importable, the reference's own layout in
``path`` (an existing group of the same name is replaced, as the reference's
default ``overwrite=True`` does); without it (this image has no HDF5 library),
the same group paths as NumPy files: ``<root>/fields/iteration_<i>/time.npy``,
``Q.npy``, ``Qaux.npy`` with ``<root>`` = ``path`` minus a ``.h5`` suffix.

Beside the snapshots a run writes its mesh and its settings, as the reference
does before its time loop (``zoomy_jax/fvm/solver_jax.py:1267-1283``:
``mesh.write_to_hdf5`` and ``io.save_settings``).  Those two writers belong to
zoomy_core, which is not part of the reference tree, so their layouts here are
this package's own: the mesh arrays in the group ``mesh`` (HDF5) or as
``<root>/mesh/<name>.npy``, the settings as JSON (the file attribute
``settings`` in HDF5, ``<root>/settings.json`` otherwise).
"""
from __future__ import annotations

import json
import os
import queue
import threading

import numpy as np

try:  # pragma: no cover - the image has no h5py; kept for hosts that do
    import h5py as _h5py
except ImportError:  # pragma: no cover
    _h5py = None


def snapshot_times(time_end, snapshots):
    """Output times of a run: snapshot ``i`` is written after the first step
    whose time reaches ``i * time_end / max(snapshots - 1, 1)``
    (``zoomy_jax/fvm/solver_jax.py``: ``dt_snapshot``, ``time_stamp``)."""
    dt = time_end / max(snapshots - 1, 1)
    return [i * dt for i in range(snapshots)]


def read_snapshots(path):
    """Snapshots written by :class:`SnapshotWriter` as ``{i: (time, Q,
    Qaux or None)}`` (either file format)."""
    out = {}
    if _h5py is not None and os.path.isfile(path):  # pragma: no cover
        with _h5py.File(path, "r") as f:
            for name, g in f["fields"].items():
                i = int(name.split("_")[1])
                out[i] = (float(g["time"][()]), g["Q"][()],
                          g["Qaux"][()] if "Qaux" in g else None)
        return out
    root = os.path.join(_npy_root(path), "fields")
    if not os.path.isdir(root):
        return out
    for name in os.listdir(root):
        if not name.startswith("iteration_"):
            continue
        d = os.path.join(root, name)
        aux = os.path.join(d, "Qaux.npy")
        out[int(name.split("_")[1])] = (float(np.load(os.path.join(d, "time.npy"))),
                                        np.load(os.path.join(d, "Q.npy")),
                                        np.load(aux) if os.path.exists(aux) else None)
    return out


def read_mesh(path):
    """The mesh arrays :meth:`SnapshotWriter.write_mesh` wrote (``{}`` if none)."""
    if _h5py is not None and os.path.isfile(path):  # pragma: no cover
        with _h5py.File(path, "r") as f:
            return {k: v[()] for k, v in f["mesh"].items()} if "mesh" in f else {}
    d = os.path.join(_npy_root(path), "mesh")
    if not os.path.isdir(d):
        return {}
    return {f[:-4]: np.load(os.path.join(d, f)) for f in os.listdir(d) if f.endswith(".npy")}


def read_settings(path):
    """The settings :meth:`SnapshotWriter.write_settings` wrote (``{}`` if none)."""
    if _h5py is not None and os.path.isfile(path):  # pragma: no cover
        with _h5py.File(path, "r") as f:
            return json.loads(f.attrs["settings"]) if "settings" in f.attrs else {}
    p = os.path.join(_npy_root(path), "settings.json")
    if not os.path.isfile(p):
        return {}
    with open(p) as fh:
        return json.load(fh)


def _npy_root(path):
    p = str(path)
    return p[:-3] if p.endswith(".h5") else p


class SnapshotWriter:
    """Writes snapshots of device (or host) state arrays without stalling the
    launching stream on the transfer or the disk.  Use as a context manager or
    call :meth:`close`, which waits for every queued snapshot and re-raises a
    writer error."""

    def __init__(self, path, slots=2, fmt=None):
        self.path = str(path)
        self.format = fmt or ("hdf5" if _h5py is not None else "npy")
        if self.format == "hdf5" and _h5py is None:
            raise ImportError("h5py is not installed: use fmt='npy'")
        if slots < 1:
            raise ValueError("slots must be >= 1")
        self.n_slots = slots
        self._slots = [None] * slots
        self._free = queue.Queue()
        for k in range(slots):
            self._free.put(k)
        self._todo = queue.Queue()
        self._error = None
        self._side = None
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        self.written = 0

    # ── staging ───────────────────────────────────────────────────────────
    def _slot(self, k, Q, Qaux):
        import torch
        s = self._slots[k]
        shape_aux = None if Qaux is None else tuple(Qaux.shape)
        if (s is None or s["shape"] != tuple(Q.shape) or s["dtype"] != Q.dtype
                or s["shape_aux"] != shape_aux or s["device"] != Q.device):
            cuda = Q.is_cuda
            s = {"shape": tuple(Q.shape), "dtype": Q.dtype, "shape_aux": shape_aux,
                 "device": Q.device, "cuda": cuda,
                 "dq": torch.empty_like(Q) if cuda else None,
                 "da": (torch.empty_like(Qaux) if (cuda and Qaux is not None) else None),
                 "hq": torch.empty(Q.shape, dtype=Q.dtype, pin_memory=cuda),
                 "ha": (torch.empty(Qaux.shape, dtype=Qaux.dtype, pin_memory=cuda)
                        if Qaux is not None else None),
                 "ev": torch.cuda.Event() if cuda else None}
            self._slots[k] = s
        return s

    def save(self, i_snapshot, time, Q, Qaux=None, stream=None):
        """Queue snapshot ``i_snapshot`` of ``Q`` (and ``Qaux``) at ``time``.
        The state is read in order on ``stream`` (default: the current
        stream), so the caller may launch the next step right away."""
        import torch
        self._check()
        k = self._free.get()
        s = self._slot(k, Q, Qaux)
        if s["cuda"]:
            cur = stream if stream is not None else torch.cuda.current_stream(Q.device)
            if self._side is None:
                self._side = torch.cuda.Stream(device=Q.device)
            with torch.cuda.stream(cur):
                s["dq"].copy_(Q, non_blocking=True)
                if Qaux is not None:
                    s["da"].copy_(Qaux, non_blocking=True)
            staged = torch.cuda.Event()
            staged.record(cur)
            with torch.cuda.stream(self._side):
                self._side.wait_event(staged)
                s["hq"].copy_(s["dq"], non_blocking=True)
                if Qaux is not None:
                    s["ha"].copy_(s["da"], non_blocking=True)
                s["ev"].record(self._side)
        else:
            s["hq"].copy_(Q)
            if Qaux is not None:
                s["ha"].copy_(Qaux)
        self._todo.put(("snapshot", k, int(i_snapshot), float(time), Qaux is not None))

    def write_mesh(self, arrays):
        """Queue the run's mesh: ``{name: host array}``, written once, in
        order with the snapshots, by the writer thread."""
        self._check()
        self._todo.put(("mesh", {k: np.asarray(v) for k, v in arrays.items()}))

    def write_settings(self, settings):
        """Queue the run's settings (a JSON-serialisable dict)."""
        self._check()
        self._todo.put(("settings", json.dumps(settings, sort_keys=True)))

    # ── the writer thread ─────────────────────────────────────────────────
    def _run(self):
        while True:
            item = self._todo.get()
            if item is None:
                return
            if item[0] != "snapshot":
                try:
                    self._write_meta(item[0], item[1])
                except BaseException as e:  # noqa: BLE001 - handed to the caller
                    self._error = e
                continue
            _, k, i, t, has_aux = item
            try:
                s = self._slots[k]
                if s["ev"] is not None:
                    s["ev"].synchronize()
                q = s["hq"].numpy()
                a = s["ha"].numpy() if has_aux else None
                self._write(i, t, q, a)
                self.written += 1
            except BaseException as e:  # noqa: BLE001 - handed to the caller
                self._error = e
            finally:
                self._free.put(k)

    def _write(self, i, t, q, a):
        name = f"iteration_{i}"
        if self.format == "hdf5":  # pragma: no cover - needs h5py
            with _h5py.File(self.path, "a") as f:
                fields = f.require_group("fields")
                if name in fields:
                    del fields[name]
                g = fields.create_group(name)
                g.create_dataset("time", data=t, dtype=float)
                g.create_dataset("Q", data=q)
                if a is not None:
                    g.create_dataset("Qaux", data=a)
            return
        d = os.path.join(_npy_root(self.path), "fields", name)
        os.makedirs(d, exist_ok=True)
        for f in ("time.npy", "Q.npy", "Qaux.npy"):
            if os.path.exists(os.path.join(d, f)):
                os.remove(os.path.join(d, f))
        np.save(os.path.join(d, "time.npy"), np.float64(t))
        np.save(os.path.join(d, "Q.npy"), q)
        if a is not None:
            np.save(os.path.join(d, "Qaux.npy"), a)

    def _write_meta(self, kind, payload):
        if self.format == "hdf5":  # pragma: no cover - needs h5py
            with _h5py.File(self.path, "a") as f:
                if kind == "settings":
                    f.attrs["settings"] = payload
                    return
                if "mesh" in f:
                    del f["mesh"]
                g = f.create_group("mesh")
                for name, a in payload.items():
                    g.create_dataset(name, data=a)
            return
        root = _npy_root(self.path)
        os.makedirs(root, exist_ok=True)
        if kind == "settings":
            with open(os.path.join(root, "settings.json"), "w") as fh:
                fh.write(payload)
            return
        d = os.path.join(root, "mesh")
        os.makedirs(d, exist_ok=True)
        for f in os.listdir(d):
            if f.endswith(".npy"):
                os.remove(os.path.join(d, f))
        for name, a in payload.items():
            np.save(os.path.join(d, name + ".npy"), a)

    def _check(self):
        if self._error is not None:
            e, self._error = self._error, None
            raise e

    def close(self):
        """Wait for every queued snapshot, stop the writer, re-raise its
        error if it had one."""
        if self._thread.is_alive():
            self._todo.put(None)
            self._thread.join()
        self._check()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

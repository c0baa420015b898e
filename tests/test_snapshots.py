"""The asynchronous snapshot writer on host arrays (no GPU): the reference's
group layout fields/iteration_<i>/{time, Q, Qaux} (as NumPy files where h5py
is absent), the output times, a one-slot ring that makes every snapshot wait
for the previous write, replacement of an existing iteration, and a write
error re-raised at close."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from zoomy_b200.snapshots import (SnapshotWriter, read_mesh, read_settings,  # noqa: E402
                                  read_snapshots, snapshot_times)


def test_output_times_follow_the_reference():
    assert snapshot_times(1.0, 5) == [0.0, 0.25, 0.5, 0.75, 1.0]
    assert snapshot_times(2.0, 1) == [0.0]
    assert snapshot_times(3.0, 2) == [0.0, 3.0]


def test_snapshots_round_trip_through_a_one_slot_ring(tmp_path):
    path = str(tmp_path / "run.h5")
    rng = np.random.default_rng(0)
    states = [rng.standard_normal((4, 37)) for _ in range(4)]
    auxes = [rng.standard_normal((7, 37)) for _ in range(4)]
    with SnapshotWriter(path, slots=1, fmt="npy") as w:
        for i, (q, a) in enumerate(zip(states, auxes)):
            w.save(i, 0.5 * i, torch.as_tensor(q), torch.as_tensor(a) if i % 2 == 0 else None)
    assert w.written == 4
    got = read_snapshots(path)
    assert sorted(got) == [0, 1, 2, 3]
    for i in range(4):
        t, q, a = got[i]
        assert t == 0.5 * i
        assert np.array_equal(q, states[i])
        if i % 2 == 0:
            assert np.array_equal(a, auxes[i])
        else:
            assert a is None
    assert os.path.isdir(str(tmp_path / "run" / "fields" / "iteration_3"))


def test_an_iteration_written_again_is_replaced(tmp_path):
    path = str(tmp_path / "out.h5")
    with SnapshotWriter(path, fmt="npy") as w:
        w.save(0, 0.0, torch.zeros(4, 5), torch.ones(7, 5))
    with SnapshotWriter(path, fmt="npy") as w:
        w.save(0, 1.5, torch.ones(4, 5))
    t, q, a = read_snapshots(path)[0]
    assert t == 1.5 and np.all(q == 1.0) and a is None


def test_a_write_error_is_raised_at_close(tmp_path):
    blocker = tmp_path / "file"
    blocker.write_text("x")
    w = SnapshotWriter(str(blocker / "run.h5"), fmt="npy")   # a directory under a file
    w.save(0, 0.0, torch.zeros(4, 3))
    with pytest.raises(OSError):
        w.close()


def test_mesh_and_settings_round_trip(tmp_path):
    """The run's mesh arrays and settings go through the writer thread in
    order with the snapshots; written again, they are replaced."""
    path = str(tmp_path / "run.h5")
    mesh = {"cell_centers": np.arange(12.0).reshape(2, 6), "shape": np.array([2, 3])}
    with SnapshotWriter(path, fmt="npy") as w:
        w.write_mesh(mesh)
        w.write_settings({"time_end": 0.5, "riemann": "hll_hr", "bc": ["wall"] * 4})
        w.save(0, 0.0, torch.zeros(4, 6))
    got = read_mesh(path)
    assert sorted(got) == ["cell_centers", "shape"]
    assert np.array_equal(got["cell_centers"], mesh["cell_centers"])
    assert read_settings(path) == {"time_end": 0.5, "riemann": "hll_hr", "bc": ["wall"] * 4}
    with SnapshotWriter(path, fmt="npy") as w:
        w.write_mesh({"vertices": np.zeros((3, 2))})
        w.write_settings({"time_end": 1.0})
    assert sorted(read_mesh(path)) == ["vertices"]
    assert read_settings(path) == {"time_end": 1.0}
    assert read_mesh(str(tmp_path / "none.h5")) == {} and read_settings(str(tmp_path / "x")) == {}


def test_a_settings_error_is_raised_at_close(tmp_path):
    w = SnapshotWriter(str(tmp_path / "run.h5"), fmt="npy")
    w.write_settings({"fine": 1})
    w.close()
    w = SnapshotWriter(str(tmp_path / "run2.h5"), fmt="npy")
    with pytest.raises(TypeError):
        w.write_settings({"not serialisable": object()})
    w.close()

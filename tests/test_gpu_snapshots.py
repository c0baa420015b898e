"""Snapshot output of a device-resident march against a step-by-step march.

run_simulation(write_output=True) queues fused steps in batches, drops to
single steps near each output time and hands snapshots to the asynchronous
writer; the reference writes snapshot i after the first step whose time
reaches i * time_end / (snapshots - 1).  The same march driven one step at a
time from the host, recording the state at those steps, gives the expected
snapshots: the same times and the same bits."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import zoomy_b200 as zb  # noqa: E402
from zoomy_b200.fvm.solver import HyperbolicSolver  # noqa: E402
from zoomy_b200.snapshots import read_mesh, read_settings, read_snapshots, snapshot_times  # noqa: E402
from zoomy_b200.workloads import circular_dam_state  # noqa: E402

TAGS = ("left", "right", "bottom", "top")


def make(path, t_end, snapshots):
    mesh = zb.create_2d((0.0, 1.0, 0.0, 1.0), 64, 48)
    Q0 = circular_dam_state(mesh.cell_centers(), seed=2)
    model = zb.ShallowWater2D(boundary_conditions={t: "wall" for t in TAGS},
                              initial_conditions=Q0)
    nsm = zb.NumericalSystemModel.from_system_model(
        model, zb.ReconstructionSpec(2, "minmod"), "hll_hr")
    solver = HyperbolicSolver(time_end=t_end, compute_dt=zb.timestepping.adaptive(0.45, 2),
                              reconstruction_variables="eta", free_surface_h_index=1,
                              eps_wet=1e-6, dtype="float64", output_path=path,
                              output_snapshots=snapshots)
    Q, Qaux = solver.setup_simulation(mesh, nsm)
    return solver, Q, Qaux


def test_snapshots_match_a_step_by_step_march(tmp_path):
    t_end, n_snap = 0.02, 5
    path = str(tmp_path / "run.h5")
    solver, Q, Qaux = make(path, t_end, n_snap)
    Qf, Af = solver.run_simulation(Q.clone(), Qaux, write_output=True)
    got = read_snapshots(path)
    assert sorted(got) == list(range(n_snap))

    # the same march one step at a time
    ref, Q2 = {}, Q.clone()
    stamps = snapshot_times(t_end, n_snap)
    ref[0] = (0.0, Q.cpu().numpy(), Qaux.cpu().numpy())
    solver.init_march(Q2, 0.0)
    i = 1
    for _ in range(100000):
        solver.launch_steps(Q2, 1)
        t = solver.read_ctrl().t[solver._n % 3]
        if i < n_snap and t >= stamps[i]:
            ref[i] = (t, Q2.cpu().numpy(), solver.update_qaux(Q2).cpu().numpy())
            i += 1
        if t >= t_end:
            break
    assert i == n_snap
    for k in range(n_snap):
        assert got[k][0] == ref[k][0], k
        assert got[k][0] >= stamps[k]
        assert np.array_equal(got[k][1], ref[k][1]), k
        assert np.array_equal(got[k][2], ref[k][2]), k
    assert np.array_equal(got[n_snap - 1][1], Qf.cpu().numpy())
    assert math.isclose(solver.time, t_end, rel_tol=0, abs_tol=1e-15)
    # the mesh and the settings written beside the snapshots
    mesh = read_mesh(path)
    assert np.array_equal(mesh["cell_centers"], solver.mesh.cell_centers())
    assert mesh["shape"].tolist() == [64, 48]
    st = read_settings(path)
    assert st["time_end"] == t_end and st["riemann"] == "hll_hr"
    assert st["compute_dt"]["cfl"] == 0.45 and st["output"]["snapshots"] == n_snap
    assert st["boundary_conditions"] == ["wall"] * 4 and st["dtype"] == "float64"

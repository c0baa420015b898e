"""GPU tests of the batched ensemble (one persistent launch per stage).

Every instance must evolve exactly as the same grid run alone through the
single-grid fused step (itself pinned to the oracle at 1e-12 per step): float64
agreement <= 1e-13 relative L-infinity after 5 steps, independent of the tile
height; CUDA-graph replay equals direct launches; the 512-instance
configuration runs with every instance's mass conserved (float64 sums).
"""
import math

import numpy as np
import pytest

from oracle import mesh as OM
from oracle import swe as OS

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import zoomy_b200 as zb  # noqa: E402
from zoomy_b200 import _lib as L  # noqa: E402
from zoomy_b200.ensemble import Ensemble  # noqa: E402
from zoomy_b200.fvm.solver import HyperbolicSolver  # noqa: E402
from zoomy_b200.workloads import ensemble_512, ensemble_state  # noqa: E402

TAGS = ("left", "right", "bottom", "top")
SIDES = [37, 40, 48, 53, 64, 70, 77, 81, 90, 96, 100, 33]


def single_run(n, height, manning, steps, dtype):
    model = zb.ShallowWater2D(wet_dry_eps=1e-6, manning_n=manning,
                              boundary_conditions={t: "wall" for t in TAGS},
                              initial_conditions=ensemble_state(n, height))
    nsm = zb.NumericalSystemModel.from_system_model(
        model, zb.ReconstructionSpec(2, "minmod"), "hll_hr")
    s = HyperbolicSolver(time_end=math.inf, compute_dt=zb.timestepping.adaptive(0.45, 2),
                         reconstruction_variables="eta", free_surface_h_index=1,
                         eps_wet=1e-6, dtype=dtype)
    Q, _ = s.setup_simulation(zb.create_2d((0, 1, 0, 1), n, n), nsm)
    s.init_march(Q)
    s.launch_steps(Q, steps)
    return Q.double().cpu().numpy(), s.read_ctrl()


def make_ens(sides, dtype, tile):
    rng = np.random.default_rng(3)
    heights = rng.uniform(1.1, 3.0, len(sides))
    manning = rng.uniform(0.01, 0.05, len(sides))
    ens = Ensemble(sides, manning, dtype=dtype)
    ens.tile_x = ens.tuning.tile_x = tile
    ens.setup([ensemble_state(n, h) for n, h in zip(sides, heights)])
    return ens, heights, manning


@pytest.mark.parametrize("tile", [8, 16])
def test_ensemble_matches_single_grids(tile):
    ens, heights, manning = make_ens(SIDES, "float64", tile)
    ens.init()
    ens.launch_steps(5)
    assert ens.status_any() == 0
    for i, n in enumerate(SIDES):
        ref, c = single_run(n, heights[i], manning[i], 5, "float64")
        got = ens.instance(i).cpu().numpy()
        scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-300
        assert (np.abs(got - ref) / scale).max() <= 1e-13, f"instance {i} (n={n})"
        ci = ens.ctrl(i)
        assert ci.t[5 % 3] == pytest.approx(c.t[5 % 3], rel=1e-14)


def test_float32_ensemble_matches_single_grids():
    """float32 runs the boundary strips' inner rows in the paired column-EDGE
    body (32-row chunks in the ensemble's lists, 8-row chunks in a single
    grid's): every instance -- a grid too small for strips (tile fallback),
    grids without inner rows or middle strips, grids with one and several
    middle strips -- agrees with the same grid run alone after 5 steps (the
    two kernels may contract a few products differently: 1e-5 relative)."""
    sides = [3, 4, 5, 6, 29, 30, 31, 57, 58, 60, 85]
    ens, heights, manning = make_ens(sides, "float32", 16)
    ens.init()
    ens.launch_steps(5)
    assert ens.status_any() == 0
    for i, n in enumerate(sides):
        ref, c = single_run(n, heights[i], manning[i], 5, "float32")
        got = ens.instance(i).double().cpu().numpy()
        scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-30
        assert (np.abs(got - ref) / scale).max() <= 1e-5, f"instance {i} (n={n})"
        assert ens.ctrl(i).t[5 % 3] == pytest.approx(c.t[5 % 3], rel=1e-5)


def test_ensemble_instance_matches_oracle_per_step():
    ens, heights, manning = make_ens([40, 56], "float64", 16)
    ens.init()
    om = OM.create_2d(0.0, 1.0, 0.0, 1.0, 56, 56)
    scheme = OS.Scheme(order=2, recon="eta", riemann="hll_hr", eps_wet=1e-6, cfl=0.45,
                       bc={t: "wall" for t in TAGS})
    params = OS.Params(wet_dry_eps=1e-6, manning_n=float(manning[1]))
    for it in range(3):
        q = ens.instance(1).cpu().numpy().copy()
        ens.launch_steps(1)
        c = ens.ctrl(1)
        assert c.dt == pytest.approx(OS.compute_dt(om, q, params, scheme), rel=1e-14)
        ref = OS.step(om, q, c.dt, params, scheme)
        got = ens.instance(1).cpu().numpy()
        scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-300
        assert (np.abs(got - ref) / scale).max() <= 1e-12


def test_ensemble_result_does_not_depend_on_the_launch_shape():
    """Small column-EDGE and interior chunks, one strip CTA per SM and three
    size classes with different chunk heights: every instance still evolves
    as the same grid run alone (float64, 1e-13)."""
    ens, heights, manning = make_ens(SIDES, "float64", 16)
    t = ens.tuning
    t.ctas_per_sm = 1
    t.n_classes = 3
    for k, (side, e, r) in enumerate(((48, 8, 16), (80, 16, 24), (1 << 30, 4, 8))):
        t.class_max_side[k], t.edge_rows[k], t.interior_rows[k] = side, e, r
    ens._build_table()
    ens.init()
    ens.launch_steps(5)
    assert ens.status_any() == 0
    for i, n in enumerate(SIDES):
        ref, c = single_run(n, heights[i], manning[i], 5, "float64")
        got = ens.instance(i).cpu().numpy()
        scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-300
        assert (np.abs(got - ref) / scale).max() <= 1e-13, f"instance {i} (n={n})"


def test_graph_replay_equals_direct_launches_and_autotune():
    ens, *_ = make_ens(SIDES, "float32", 16)
    res = ens.autotune(steps=3)
    # the untuned shape, the other strip CTA counts and the chunk heights of
    # a populated size class were timed; the kept shape is the fastest
    assert "untuned" in res and "ctas_per_sm=2" in res and "ctas_per_sm=3" in res
    assert any(k.startswith("class0.edge_rows=") for k in res)
    assert any(k.startswith("class0.interior_rows=") for k in res)
    assert ens.tuned_ms == min(res.values())
    q0 = ens.Q.clone()
    ens.init()
    ens.launch_steps(6)
    direct = ens.Q.clone()
    ens.Q.copy_(q0)
    ens.init()
    ens.capture(3)
    ens.Q.copy_(q0)      # capture recorded, did not run; start again from q0
    ens.init()
    ens.replay(2)
    torch.cuda.synchronize()
    assert torch.equal(ens.Q, direct)
    assert ens.status_any() == 0


def test_512_instance_configuration():
    sides, heights, manning = ensemble_512(seed=0)
    assert len(sides) == 512 and sides.min() >= 64 and sides.max() <= 512
    ens = Ensemble(sides, manning, dtype="float32")
    ens.setup([ensemble_state(int(n), h) for n, h in zip(sides, heights)])
    m0 = [float(ens.instance(i)[1].double().sum()) / int(n) ** 2 for i, n in enumerate(sides)]
    ens.init()
    ens.capture(3)
    ens.init()
    ens.replay(4)
    torch.cuda.synchronize()
    assert ens.status_any() == 0
    for i, n in enumerate(sides):
        m1 = float(ens.instance(i)[1].double().sum()) / int(n) ** 2
        assert abs(m1 - m0[i]) / m0[i] <= 1e-5
    assert ens.ctrl(0).steps == 12

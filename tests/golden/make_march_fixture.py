"""Generate the float64 oracle march that the float32 GPU march is checked against.

``python tests/golden/make_march_fixture.py`` marches the noisy circular dam
break over 16 seeded Gaussian bumps (the 2048^2 configuration's scheme: eta
least-squares MUSCL with the minmod clip, HLL with hydrostatic
reconstruction, SSP-RK2, walls, CFL 0.45, dry-cell demotion below 1e-6) on a
256^2 grid of the unit square for 1000 steps through the float64 oracle
(about 12 minutes on one core) and writes ``march_256_1000.npz``: the
initial-state seed, the final time and the final ``h, q_x, q_y`` rounded to
float32 (the float32 comparison's tolerance is four orders above that
rounding).
"""
import pathlib
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
for p in (ROOT, ROOT / "tests", ROOT / "zoomy-jax_b200"):
    sys.path.insert(0, str(p))

from cases import circular_dam_state  # noqa: E402
from oracle import mesh as OM  # noqa: E402
from oracle import swe as OS  # noqa: E402

N, STEPS, SEED = 256, 1000, 7
TAGS = ("left", "right", "bottom", "top")


def main():
    om = OM.create_2d(0.0, 1.0, 0.0, 1.0, N, N)
    Q0 = circular_dam_state(om.cell_centers.T, seed=SEED)
    scheme = OS.Scheme(order=2, recon="eta", riemann="hll_hr", limiter="minmod",
                       cfl=0.45, bc={t: "wall" for t in TAGS}, eps_wet=1e-6)
    t0 = time.time()
    Q, _, t, steps = OS.march(om, Q0, OS.Params(), scheme, n_steps=STEPS)
    dst = pathlib.Path(__file__).with_name("march_256_1000.npz")
    np.savez_compressed(dst, n=N, steps=STEPS, seed=SEED, t=t,
                        Q=Q[1:].astype(np.float32))
    print(f"{steps} steps to t = {t:.9f} in {time.time() - t0:.0f} s; wrote {dst}")


if __name__ == "__main__":
    main()

"""Copy the reference's golden end states used to pin the oracle.

Usage: ``ZB_REFERENCE_DIR=<zoomy-jax checkout> python tests/golden/make_golden.py``
(or pass the checkout as the first argument).  Reads
``tests/refs/<name>.npz`` of that checkout and writes the ``Q``/``Qaux``
arrays into ``tests/golden/reference_goldens.npz`` as ``<name>__Q`` and
``<name>__Qaux``.  The cases and the runs that produced them (all float64,
adaptive CFL 0.9):

* ``parity``      1-D Stoker, 50 cells on [0, 10], t_end 0.5, extrapolation
                  (reference ``tests/runtime/test_parity_numpy_jax.py``)
* ``stoker_wet``  1-D Stoker, 100 cells, t_end 1.0 (``test_swe_stoker_wet.py``)
* ``ritter_dry``  1-D Ritter, 100 cells, t_end 1.0 (``test_swe_ritter_dry.py``)
* ``wb_lake``     1-D lake at rest over a Gaussian bump, 100 cells, t_end 1.0,
                  walls, positive nonconservative Rusanov
                  (``test_wb_lake_at_rest.py``)
* ``swe_2d``      2-D Gaussian pulse, 32x32 on [-1, 1]^2, t_end 0.1,
                  extrapolation (``test_swe_2d.py``)
* ``bc_wall``, ``bc_periodic``: 1-D tilted free surface, 40 cells on [0, 1],
                  t_end 0.2, walls / periodic (``test_bc_runtime.py:19-37``)
* ``stoker_wet_o2_small``, ``ritter_dry_o2_small``: the order-2 twins
  (20 cells, 2 steps) -- kept to document the restated order-2 path.
"""
import os
import pathlib
import sys

import numpy as np

CASES = ("parity", "stoker_wet", "ritter_dry", "wb_lake", "swe_2d",
         "bc_wall", "bc_periodic", "stoker_wet_o2_small", "ritter_dry_o2_small")


def main(argv):
    src = argv[1] if len(argv) > 1 else os.environ.get("ZB_REFERENCE_DIR")
    if not src:
        raise SystemExit("give the zoomy-jax checkout as an argument or in "
                         "ZB_REFERENCE_DIR")
    ref = pathlib.Path(src)
    out = {}
    for name in CASES:
        d = np.load(ref / "tests" / "refs" / f"{name}.npz")
        out[f"{name}__Q"] = d["Q"]
        out[f"{name}__Qaux"] = d["Qaux"]
    dst = pathlib.Path(__file__).with_name("reference_goldens.npz")
    np.savez_compressed(dst, **out)
    print(f"wrote {dst} ({dst.stat().st_size} bytes)")


if __name__ == "__main__":
    main(sys.argv)

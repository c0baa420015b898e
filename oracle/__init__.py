"""CPU oracle for the zoomy-b200 finite-volume path -- TEST INFRASTRUCTURE ONLY.

This package is the checker, never the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The CUDA library never routes through it
and the host package refuses to run without the CUDA extension.

Contents
--------
``mesh``     face-based meshes (1-D, Cartesian 2-D, Delaunay triangles) with
             the least-squares gradient stencil.
``swe``      float64 NumPy restatement of zoomy_jax's explicit shallow-water
             step: BC ghosts, LSQ-MUSCL and the emitted-W (b, eta, u)
             reconstruction with its limiters, Rusanov / HLL face fluxes with
             hydrostatic reconstruction, the flux-divergence scatter, the CFL dt
             reduction, SSP-RK2, MOOD and Manning friction.
``poisson``  the variable-coefficient pressure Poisson operator of the Chorin
             projection, geometric multigrid, (flexible) CG, and the learned
             smoother network in float64.

Parity pin
----------
The reference (ZoomyLab/zoomy-jax) cannot run here: ``jax`` and its symbolic
model layer ``zoomy_core`` (``>=0.1.14``, no lock file) are absent.  The
oracle is pinned against the reference's own golden end states
(``tests/refs/*.npz`` in the reference, copied into ``tests/golden/`` by
``tests/golden/make_golden.py``):

* first-order Rusanov march, CFL law, KP ``hinv`` and LSQ derivative rows:
  reproduced to round-off (1-D ``parity``/``stoker_wet``/``ritter_dry``,
  2-D ``swe_2d``);
* second-order paths (LSQ-MUSCL, emitted-W hydrostatic reconstruction, HLL):
  restated from ``reconstruction_jax.py`` and from the published methods the
  absent ``zoomy_core`` implements (HLL: Harten, Lax & van Leer 1983 with
  Davis wave speeds; hydrostatic reconstruction: Audusse, Bouchut, Bristeau,
  Klein & Perthame 2004) -- parity for these is restated, not pinned.
"""

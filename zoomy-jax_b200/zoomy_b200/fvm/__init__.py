"""Finite-volume solvers: ``solver.HyperbolicSolver`` and ``solver2``'s
``MarchSolver`` with its named blocks."""

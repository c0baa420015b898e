"""Shared case builders for the tests (initial conditions as the reference's
``tests/cases.py`` states them, plus the seeded 2-D configurations)."""
import numpy as np

ETA_L, ETA_R, DAM_X = 0.005, 0.001, 5.0


def stoker_ic(x):
    return np.array([0.0, ETA_L if float(x) < DAM_X else ETA_R, 0.0])


def ritter_ic(x):
    return np.array([0.0, ETA_L if float(x) < DAM_X else 0.0, 0.0])


def lake_at_rest_ic(x):
    b = 0.1 * np.exp(-((float(x) - 5.0) ** 2) / 0.5)
    return np.array([b, 0.3 - b, 0.0])


def gaussian_pulse_2d(x):
    r2 = float(x[0]) ** 2 + float(x[1]) ** 2
    return np.array([0.0, 0.5 + 0.05 * np.exp(-r2 / 0.2), 0.0, 0.0])


from zoomy_b200.workloads import bumps, circular_dam_state  # noqa: E402,F401


def tilted_ic(x):
    """The reference's tilted free surface on [0, 1] (its ``tests/cases.py``
    ``tilted_ic``), the initial state of the BC goldens."""
    return np.array([0.0, 0.5 + 0.05 * (float(x) - 0.5), 0.0])

"""The reference suite's cases, restated for this package.

Each golden case is the model, IC and settings of one test in the reference
(tests/test_swe_stoker_wet.py, test_swe_ritter_dry.py, test_wb_lake_at_rest.py,
test_swe_2d.py, test_parity_numpy.py, test_parallel_two_ranks.py), with the IC
functions of tests/cases.py:195-227 and the CFL law of tests/conftest.py:37
(c_cfl = 0.9 in 1-D and 2-D; the dimension divisor does the rest).
"""
import numpy as np

from zoomy_amrex_b200.models import SWE, initial_state
from zoomy_amrex_b200.settings import config_from_settings, grid

CFL_1D, CFL_2D = 0.9, 0.9


def stoker_ic(x):
    """Wet dam break: h = 0.005 left of x = 5, 0.001 right of it; [b, h, hu]."""
    h = np.where(x[0] < 5.0, 0.005, 0.001)
    z = np.zeros_like(h)
    return np.array([z, h, z])


def ritter_ic(x):
    """Dry dam break: h = 0.005 left of x = 5, dry right of it."""
    h = np.where(x[0] < 5.0, 0.005, 0.0)
    z = np.zeros_like(h)
    return np.array([z, h, z])


def lake_at_rest_ic(x):
    """Still water over a Gaussian bump: eta = 1, u = 0."""
    b = 0.2 * np.exp(-((x[0] - 5.0) ** 2))
    return np.array([b, 1.0 - b, np.zeros_like(b)])


def gaussian_pulse_2d(x):
    h = 1.0 + 0.1 * np.exp(-((x[0]) ** 2 + (x[1]) ** 2) / 0.05)
    z = np.zeros_like(h)
    return np.array([z, h, z, z])


_1D = {"dimension": 1, "domain": [0.0, 10.0], "spatial_order": 1, "output_snapshots": 1,
       "max_level": 0}

# name -> (model, settings); golden file tests/golden/<name>.npz
GOLDEN_CASES = {
    "stoker_wet": (SWE(1, "swashes", stoker_ic), dict(_1D, n_cells=100, time_end=1.0, cfl=CFL_1D)),
    "ritter_dry": (SWE(1, "swashes", ritter_ic), dict(_1D, n_cells=100, time_end=1.0, cfl=CFL_1D)),
    "wb_lake": (SWE(1, "wall", lake_at_rest_ic),
                dict(_1D, n_cells=100, time_end=1.0, cfl=CFL_1D, well_balanced=True)),
    "swe_2d": (SWE(2, "extrapolation", gaussian_pulse_2d),
               {"dimension": 2, "domain": [-1.0, 1.0, -1.0, 1.0], "n_cells": [32, 32],
                "spatial_order": 1, "time_end": 0.1, "cfl": CFL_2D}),
    "parity_numpy_n100": (SWE(1, "swashes", stoker_ic),
                          dict(_1D, n_cells=100, time_end=0.5, cfl=CFL_1D)),
    "parity_numpy_n200": (SWE(1, "swashes", stoker_ic),
                          dict(_1D, n_cells=200, time_end=0.5, cfl=CFL_1D)),
    "parallel_2rank": (SWE(1, "swashes", stoker_ic),
                       dict(_1D, n_cells=128, time_end=0.5, cfl=CFL_1D)),
}


def setup(model, settings):
    """(cfg, Q0, aux0) for a model + settings pair."""
    cfg = config_from_settings(model, settings)
    _, nx, ny, lo, hi = grid(settings)
    Q0, A0 = initial_state(model, nx, ny, lo, hi)
    return cfg, Q0, A0


def golden_setup(name):
    model, settings = GOLDEN_CASES[name]
    return setup(model, settings)

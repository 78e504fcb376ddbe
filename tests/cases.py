"""The reference suite's cases, restated for this package.

Each golden case is the model, IC and settings of one test in the reference
(tests/test_swe_stoker_wet.py, test_swe_ritter_dry.py, test_wb_lake_at_rest.py,
test_swe_2d.py, test_parity_numpy.py, test_parallel_two_ranks.py), with the IC
functions of tests/cases.py:195-227 and the CFL law of tests/conftest.py:37
(c_cfl = 0.9 in 1-D and 2-D; the dimension divisor does the rest).
"""
import numpy as np

from zoomy_amrex_b200.models import SME, SWE, initial_state
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


# ---------------------------------------------------------------------------
# Parity cases beyond the goldens: order 2, wet/dry, walls and mixed sides,
# implicit and explicit Manning friction, odd grid sizes (1-D and 2-D).

def _bumps(x, seed, n=6, lo=0.0, hi=10.0, amp=(0.2, 1.2), width=(0.5, 2.0)):
    rng = np.random.default_rng(seed)
    b = np.zeros(x.shape[1])
    for _ in range(n):
        cx, cy = rng.uniform(lo, hi, 2)
        a, w = rng.uniform(*amp), rng.uniform(*width)
        b += a * np.exp(-((x[0] - cx) ** 2 + (x[1] - cy) ** 2) / (2 * w * w))
    return b


def wetdry_ic(seed, eta0=1.0, hump=0.3, moving=False):
    def ic(x):
        b = _bumps(x, seed)
        rng = np.random.default_rng(seed + 1)
        cx, cy = rng.uniform(2, 8, 2)
        eta = eta0 + hump * np.exp(-((x[0] - cx) ** 2 + (x[1] - cy) ** 2) / 2.0)
        h = np.maximum(eta - b, 0.0)
        hu = h * rng.uniform(-0.1, 0.1, h.shape) if moving else np.zeros_like(h)
        hv = h * rng.uniform(-0.1, 0.1, h.shape) if moving else np.zeros_like(h)
        return np.array([b, h, hu, hv])
    return ic


def dambreak_2d(x):
    h = np.where(x[0] < 0.5, 2.0, 1.0)
    z = np.zeros_like(h)
    return np.array([z, h, z, z])


CASES_2D = {
    # config 1: 100x100 dam break, order 2, cfl 0.45 (Exec/inputs), extrapolation, t=0.1
    "dambreak_o2": (SWE(2, "extrapolation", None),
                    dict(dimension=2, domain=[0, 1, 0, 1], n_cells=[100, 100], spatial_order=2,
                         cfl=0.45, time_end=0.1, dtmax=0.1)),
    "dambreak_o2_clamp": (SWE(2, "extrapolation", None),
                          dict(dimension=2, domain=[0, 1, 0, 1], n_cells=[100, 100], spatial_order=2,
                               cfl=0.45, time_end=0.1, dtmax=0.1, clamp_positivity=True)),
    "wetdry_wb_manning_o2": (SWE(2, "wall", wetdry_ic(3), parameters={"n_m": 0.03}),
                             dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[48, 40],
                                  spatial_order=2, cfl=0.9, time_end=1e30, max_step=40,
                                  well_balanced=True, implicit_source=True)),
    "wetdry_moving_o2_mixed_bc": (SWE(2, {"West": "wall", "East": "extrapolation", "South": "extrapolation",
                                          "North": "wall"}, wetdry_ic(5, moving=True),
                                      parameters={"n_m": 0.05}),
                                  dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[33, 17],
                                       spatial_order=2, cfl=0.9, time_end=1e30, max_step=30,
                                       well_balanced=True, implicit_source=True)),
    "wetdry_o1_impl": (SWE(2, "wall", wetdry_ic(7, moving=True), parameters={"n_m": 0.03}),
                       dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[37, 29], spatial_order=1,
                            cfl=0.9, time_end=1e30, max_step=25, well_balanced=True,
                            implicit_source=True)),
    "tiny_7x5_o2": (SWE(2, "wall", wetdry_ic(11, moving=True)),
                    dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[7, 5], spatial_order=2,
                         cfl=0.9, time_end=1e30, max_step=20, well_balanced=True)),
    "strip_65x2_o2": (SWE(2, "extrapolation", wetdry_ic(13, moving=True)),
                      dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[65, 2], spatial_order=2,
                           cfl=0.9, time_end=1e30, max_step=10)),
}


def ritter_o2(x):
    h = np.where(x[0] < 5.0, 0.005, 0.0)
    z = np.zeros_like(h)
    return np.array([z, h, z])


def bump_1d(x):
    b = 0.3 * np.exp(-((x[0] - 4.0) ** 2)) + 0.8 * np.exp(-((x[0] - 7.0) ** 2) * 4)
    h = np.maximum(0.9 - b, 0.0)
    return np.array([b, h, 0.02 * h])


CASES_1D = {
    "ritter_o2": (SWE(1, "swashes", ritter_o2),
                  dict(dimension=1, domain=[0, 10], n_cells=129, spatial_order=2, cfl=0.9, time_end=2.0)),
    "bump_wall_wb_impl_o2": (SWE(1, "wall", bump_1d, parameters={"n_m": 0.04}),
                             dict(dimension=1, domain=[0, 10], n_cells=200, spatial_order=2, cfl=0.9,
                                  time_end=1e30, max_step=60, well_balanced=True, implicit_source=True)),
    "bump_o1_explicit_manning": (SWE(1, {"West": "wall", "East": "extrapolation"}, bump_1d,
                                     parameters={"n_m": 0.04}),
                                 dict(dimension=1, domain=[0, 10], n_cells=301, spatial_order=1,
                                      cfl=0.9, time_end=1e30, max_step=40, well_balanced=True)),
}


def config2_strip_setup(steps: int = 20, rows: int = 64):
    """A strip of the benchmark's 4096^2 level: rows 0..rows-1 of its fields
    (16 seeded Gaussian bumps, eta = 1 m + 0.3 m hump, Manning n = 0.03),
    walls on all four sides of the strip, ``steps`` SSP-RK2 steps."""
    from zoomy_amrex_b200.workloads import BUMP_DOMAIN, bump_workload_config, bump_workload_fields
    n = 4096
    Q0, A0 = bump_workload_fields(n, rows=slice(0, rows))
    cfg = bump_workload_config(n, ny=rows, y_extent=BUMP_DOMAIN * rows / n)
    cfg.max_step = steps
    return cfg, Q0, A0


# ---------------------------------------------------------------------------
# Shallow-moment level-2 cases (csrc/models/sme.H): moments seeded as
# h U(-0.05, 0.05) m/s. The reference driver's well-balancing rescales only
# the mean momenta at a face (make_rhs.H:91-94), not the moments, so a
# well-balanced case starts at rest in the mean (a moving one with moments
# near wet/dry fronts is unstable under the reference scheme).

def sme_ic(seed, u0=0.0, dim=2):
    def ic(x):
        rng = np.random.default_rng(seed + 2)
        if dim == 2:
            b = _bumps(x, seed)
            cx, cy = rng.uniform(2, 8, 2)
            eta = 1.0 + 0.3 * np.exp(-((x[0] - cx) ** 2 + (x[1] - cy) ** 2) / 2.0)
        else:
            b = 0.3 * np.exp(-((x[0] - 4.0) ** 2)) + 0.8 * np.exp(-((x[0] - 7.0) ** 2) * 4)
            eta = 0.9 + 0.2 * np.exp(-((x[0] - 2.0) ** 2))
        h = np.maximum(eta - b, 0.0)
        nm = 4 if dim == 2 else 2
        mom = [h * rng.uniform(-0.05, 0.05, h.shape) for _ in range(nm)]
        if dim == 2:
            return np.array([b, h, u0 * h, -0.5 * u0 * h, *mom])
        return np.array([b, h, u0 * h, *mom])
    return ic


CASES_SME = {
    "sme2d_wetdry_wb_impl_o2": (SME(level=2, dimension=3, bc="wall", initial_conditions=sme_ic(3)),
                                dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[48, 40], spatial_order=2,
                                     cfl=0.45, time_end=1e30, max_step=40, well_balanced=True,
                                     implicit_source=True)),
    "sme2d_moving_mixed_bc_o2": (SME(level=2, dimension=3,
                                     bc={"West": "wall", "East": "extrapolation", "South": "extrapolation",
                                         "North": "wall"},
                                     initial_conditions=sme_ic(5, u0=0.1)),
                                 dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[33, 17], spatial_order=2,
                                      cfl=0.45, time_end=1e30, max_step=30, implicit_source=True)),
    "sme2d_o1_impl_wb": (SME(level=2, dimension=3, bc="wall", initial_conditions=sme_ic(7)),
                         dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[37, 29], spatial_order=1,
                              cfl=0.45, time_end=1e30, max_step=25, well_balanced=True, implicit_source=True)),
    "sme2d_tiny_7x5_o2": (SME(level=2, dimension=3, bc="wall", initial_conditions=sme_ic(11, u0=0.05)),
                          dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[7, 5], spatial_order=2,
                               cfl=0.45, time_end=1e30, max_step=20, implicit_source=True)),
    "sme1d_wb_impl_o2": (SME(level=2, dimension=2, bc="wall", initial_conditions=sme_ic(13, dim=1)),
                         dict(dimension=1, domain=[0, 10], n_cells=200, spatial_order=2, cfl=0.45,
                              time_end=1e30, max_step=60, well_balanced=True, implicit_source=True)),
}


def sme_strip_setup(steps: int = 20, rows: int = 32, n: int = 2048):
    """A strip of the shallow-moment benchmark level (n^2 over [0,50]^2 m):
    rows 0..rows-1 of its fields, walls on the strip's four sides."""
    from zoomy_amrex_b200.workloads import SME_DOMAIN, sme_workload_config, sme_workload_fields
    Q0, A0 = sme_workload_fields(n, rows=slice(0, rows))
    cfg = sme_workload_config(n, ny=rows, y_extent=SME_DOMAIN * rows / n)
    cfg.max_step = steps
    return cfg, Q0, A0

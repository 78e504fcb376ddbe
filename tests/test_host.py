"""Host-side checks that need no GPU: the C ABI library loads and exports
every declared entry point, configuration validation, and the settings /
model / initial-condition semantics taken from the reference's Python side."""
import ctypes as C
import pathlib
import re

import numpy as np
import pytest

from zoomy_amrex_b200 import _lib
from zoomy_amrex_b200._abi import (MODELS, ZFV_MODEL_SWE1D, ZFV_MODEL_SWE2D, make_config, zfv_config,
                                   zfv_status)
from zoomy_amrex_b200.models import SME, SWE, default_fields, initial_state
from zoomy_amrex_b200.settings import config_from_settings, grid
from zoomy_amrex_b200.solvers import HyperbolicSolver

HEADER = pathlib.Path(__file__).resolve().parent.parent / "include" / "zoomy_fv.h"


@pytest.fixture(scope="module")
def lib():
    from zoomy_amrex_b200.build import build
    build()
    return _lib.lib()


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zfv_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.SYMBOLS) == set(names)


def test_struct_layouts_match(lib):
    assert lib.zfv_sizeof_config() == C.sizeof(zfv_config)
    assert lib.zfv_sizeof_status() == C.sizeof(zfv_status) == 64


def test_model_info(lib):
    for mid, info in MODELS.items():
        nq, na, npar, dim = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        assert lib.zfv_model_info(mid, C.byref(nq), C.byref(na), C.byref(npar), C.byref(dim)) == 0
        assert (nq.value, na.value, npar.value, dim.value) == (info["n_q"], info["n_aux"],
                                                                info["n_params"], info["dimension"])
    assert lib.zfv_model_info(99, None, None, None, None) != 0


@pytest.mark.parametrize("mutate, msg", [
    (lambda c: setattr(c, "model", 42), "unknown model"),
    (lambda c: setattr(c, "spatial_order", 3), "spatial_order"),
    (lambda c: setattr(c, "n_params", 2), "parameters"),
    (lambda c: setattr(c, "nx", 0), "bad grid"),
    (lambda c: c.bc_tag.__setitem__(1, 7), "not declared"),
    (lambda c: setattr(c, "cfl_dimension", 0), "march constants"),
])
def test_create_rejects_bad_config(lib, mutate, msg):
    cfg = make_config(ZFV_MODEL_SWE2D, 8, 8, (0, 0), (1, 1))
    mutate(cfg)
    h = C.c_void_p()
    rc = lib.zfv_create(C.byref(cfg), C.byref(h))
    assert rc != 0 and not h.value
    assert msg in lib.zfv_last_error().decode()


def test_grid_must_cover_the_ghost_layers(lib):
    cfg = make_config(ZFV_MODEL_SWE2D, 65, 1, (0, 0), (1, 1), spatial_order=2)
    h = C.c_void_p()
    assert lib.zfv_create(C.byref(cfg), C.byref(h)) != 0
    assert "at least 2 cells" in lib.zfv_last_error().decode()


def test_one_d_model_needs_single_row(lib):
    cfg = make_config(ZFV_MODEL_SWE1D, 8, 2, (0, 0), (1, 1))
    h = C.c_void_p()
    assert lib.zfv_create(C.byref(cfg), C.byref(h)) != 0


def test_settings_semantics():
    """run_case.py:75-84 grid, build.py:55-120 defaults, _constants.py CFL law."""
    m = SWE(1, "wall")
    s = {"dimension": 1, "domain": [0.0, 10.0], "n_cells": 100, "time_end": 1.0, "spatial_order": 2}
    dim, nx, ny, lo, hi = grid(s)
    assert (dim, nx, ny) == (1, 100, 1) and lo == (0.0, 0.0) and hi == (10.0, 0.1)
    cfg = config_from_settings(m, s)
    assert cfg.dtmax == 1.0 and cfg.dtmin == 1e-7 and cfg.max_step == -1
    assert cfg.cfl == 0.45 and cfg.cfl_dimension == 1 and cfg.cfl_degree_factor == 3
    assert list(cfg.bc_tag) == [1, 1, 0, 0]
    assert cfg.clamp_positivity == 0 and cfg.implicit_source == 0 and cfg.positivity_mood == 0
    cfg2 = config_from_settings(SWE(2, {"West": "wall", "East": "extrapolation"}),
                                {"dimension": 2, "domain": [0, 1, 0, 2], "n_cells": [4, 8],
                                 "max_step": 3, "dtmax": 0.5, "params": {"n_m": 0.03}})
    assert list(cfg2.bc_tag) == [1, 0, 0, 0] and cfg2.max_step == 3 and cfg2.dtmax == 0.5
    assert cfg2.params[3] == 0.03 and cfg2.cfl_dimension == 2 and cfg2.cfl_degree_factor == 1


def test_unknown_bc_and_param_are_errors():
    with pytest.raises(ValueError):
        SWE(2, "periodic").side_kinds()
    with pytest.raises(ValueError):
        SWE(1, {"North": "wall"}).side_kinds()
    with pytest.raises(KeyError):
        make_config(ZFV_MODEL_SWE2D, 4, 4, (0, 0), (1, 1), params={"nu": 1.0})
    with pytest.raises(ValueError):
        make_config(ZFV_MODEL_SWE2D, 4, 4, (0, 0), (1, 1), bc=("West",) * 4)


def test_sme_level0_dimension_convention():
    from zoomy_amrex_b200._abi import ZFV_MODEL_SME1D_L2, ZFV_MODEL_SME2D_L2
    assert SME(level=0, dimension=3).dimension == 2
    assert SME(level=0, dimension=2).dimension == 1
    assert SME(level=2, dimension=3).model_id == ZFV_MODEL_SME2D_L2
    assert SME(level=2, dimension=2).model_id == ZFV_MODEL_SME1D_L2
    assert SME(level=2).state_names() == ["b", "h", "hu", "hv", "halpha_1", "halpha_2", "hbeta_1", "hbeta_2"]
    for level in (1, 3):
        with pytest.raises(NotImplementedError):
            SME(level=level)


def test_default_fields_are_init_solution():
    """init_solution.cpp:78-116 on state and aux (ZoomyAmr.cpp:174-175)."""
    Q, A = initial_state(SWE(2, "wall"), 6, 3, (-1.0, 0.0), (1.0, 1.0))
    assert np.array_equal(Q[1, 0], [2, 2, 2, 1, 1, 1]) and not Q[[0, 2, 3]].any()
    assert np.array_equal(A[1, 2], [2, 2, 2, 1, 1, 1]) and not A[[0, 2, 3, 4, 5, 6]].any()
    assert not default_fields(1, 4, 4, (0, 0), (1, 1)).any()


def test_hyperbolic_solver_validation():
    with pytest.raises(ValueError):
        HyperbolicSolver(CFL=1.5)
    with pytest.raises(ValueError):
        HyperbolicSolver(order=3)
    with pytest.raises(ValueError):
        HyperbolicSolver(positivity="clamp")
    s = HyperbolicSolver(CFL=0.45, order=2)._legacy_settings(
        {"domain": [0, 1, 0, 1], "n_cells": [10, 10]}, {"time_end": 0.2})
    assert s["dimension"] == 2 and s["time_end"] == 0.2 and s["n_cells"] == [10, 10]


def test_amr_patches_tile_the_blocks():
    """group_patches covers every refined block exactly once with rectangles
    no larger than the side limit (the AMR kernels' map offsets rely on it)."""
    import numpy as np
    from zoomy_amrex_b200.amr import group_patches
    rng = np.random.default_rng(5)
    for trial in range(20):
        mask = rng.random((24, 40)) < rng.uniform(0.2, 0.9)
        blocks = [(int(x), int(y)) for y, x in zip(*np.nonzero(mask))]
        side = int(rng.integers(1, 9))
        rects = group_patches(blocks, side)
        cover = np.zeros_like(mask, dtype=int)
        for bx, by, nbx, nby in rects:
            assert 1 <= nbx <= side and 1 <= nby <= side
            cover[by:by + nby, bx:bx + nbx] += 1
        assert np.array_equal(cover, mask.astype(int))


def test_run_case_rejects_fluxes_not_built():
    """A non-default Riemann solver is refused before any device work."""
    import pytest
    from zoomy_amrex_b200.models import SWE
    from zoomy_amrex_b200.run_case import run_case
    with pytest.raises(NotImplementedError, match="NonconservativeRusanov"):
        run_case(SWE(2, "wall", None), dict(dimension=2, domain=[0, 1, 0, 1], n_cells=[8, 8],
                                            riemann="PositiveNonconservativeHLL"), return_result=True)


def _record_many(args):
    from zoomy_amrex_b200.autotune import record
    path, k = args
    shapes = [(4, 8, 2, 3)] * 13
    for i in range(40):
        record(4, "fp32", 4096.0 * 4096.0, (k + i) % 13, {0: 1.0 + k, 1: 2.0}, shapes, path=path)
    return k


def _record_own_key(args):
    from zoomy_amrex_b200.autotune import record
    path, k = args
    shapes = [(4, 8, 2, 3)] * 13
    for i in range(20):
        record(4 + k, "fp32", 4096.0 * 4096.0, i % 13, {0: 1.0}, shapes, path=path)
    return k


def test_autotune_concurrent_writers_keep_every_key(tmp_path):
    """Processes tuning different keys at the same time all keep their entry
    (the read-modify-write runs under a lock)."""
    import json
    import multiprocessing as mp
    path = tmp_path / "autotune.json"
    with mp.get_context("spawn").Pool(4) as pool:
        pool.map(_record_own_key, [(path, k) for k in range(4)])
    data = json.loads(path.read_text())
    assert sorted(data) == sorted(f"n_q={4 + k}/fp32/large" for k in range(4))


def test_autotune_cache_survives_concurrent_writers(tmp_path):
    """One process per GPU tunes and records at the same time: every write
    succeeds and the cache stays a complete JSON document."""
    import json
    import multiprocessing as mp
    from zoomy_amrex_b200.autotune import cached_variant
    path = tmp_path / "autotune.json"
    with mp.get_context("spawn").Pool(4) as pool:
        assert sorted(pool.map(_record_many, [(path, k) for k in range(4)])) == [0, 1, 2, 3]
    data = json.loads(path.read_text())
    assert list(data) == ["n_q=4/fp32/large"]
    assert cached_variant(4, "fp32", 4096.0 * 4096.0, path=path) in range(13)
    assert not list(tmp_path.glob("*.tmp"))

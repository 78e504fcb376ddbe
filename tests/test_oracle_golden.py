"""The CPU oracle against the reference's golden data and assertions.

The reference suite compares each run to tests/refs/<name>.npz with
np.allclose (tests/refs.py:301-312) and asserts physical properties per test;
both are applied here to the oracle, which the GPU path is then checked
against. The oracle is also checked bitwise against the reference's own
make_rhs.H (oracle/_ref) on the same driver.
"""
import numpy as np
import pytest

from cases import GOLDEN_CASES, golden_setup

GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"


def golden(name):
    return np.load(GOLDEN / f"{name}.npz")


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
@pytest.mark.parametrize("face_based", [True, False])
def test_oracle_matches_reference_golden(oracle, name, face_based):
    cfg, Q0, A0 = golden_setup(name)
    Q, A, n, t, log, _ = oracle.run(cfg, Q0, A0, face_based=face_based)
    g = golden(name)
    assert np.allclose(Q, g["Q"]), f"{name}.Q: max|diff| {np.abs(Q - g['Q']).max():.3e}"
    assert np.allclose(A, g["Qaux"]), f"{name}.Qaux: max|diff| {np.abs(A - g['Qaux']).max():.3e}"
    # far tighter than allclose: the restated model is fitted to the last bits
    assert np.abs(Q - g["Q"]).max() <= 2e-15 * max(1.0, np.abs(g["Q"]).max())
    assert t == cfg.time_end


def test_stoker_properties(oracle):    # tests/test_swe_stoker_wet.py:36-41
    Q, _, _, _, _, _ = oracle.run(*golden_setup("stoker_wet"))
    assert np.isfinite(Q).all() and Q[1].min() > 0.0 and np.abs(Q[2]).max() > 0.0


def test_ritter_properties(oracle):    # tests/test_swe_ritter_dry.py
    Q, _, _, _, _, _ = oracle.run(*golden_setup("ritter_dry"))
    assert np.isfinite(Q).all() and Q[1].min() >= 0.0 and Q[1].max() > 0.0


def test_lake_at_rest_properties(oracle):   # tests/test_wb_lake_at_rest.py:94-103
    Q, _, _, _, _, _ = oracle.run(*golden_setup("wb_lake"))
    eta = Q[0] + Q[1]
    u = Q[2] / np.maximum(Q[1], 1e-300)
    assert np.abs(eta - eta.mean()).max() < 1e-12
    assert np.abs(u).max() < 1e-12


def test_swe_2d_properties(oracle):     # tests/test_swe_2d.py:145-151
    Q, _, _, _, _, _ = oracle.run(*golden_setup("swe_2d"))
    assert np.isfinite(Q).all() and Q[1].min() > 0.0
    assert np.abs(Q[2]).max() > 0.0 and np.abs(Q[3]).max() > 0.0


def test_exact_goldens_are_bitwise(oracle):
    """Where the oracle reproduces the reference bit for bit, keep it that way."""
    for name in ("ritter_dry", "parity_numpy_n100", "parallel_2rank"):
        Q, A, _, _, _, _ = oracle.run(*golden_setup(name))
        g = golden(name)
        assert np.array_equal(Q, g["Q"]) and np.array_equal(A, g["Qaux"]), name


def test_decomposition_free_two_rank_golden(oracle):
    """test_parallel_two_ranks.py:283-296: 1 rank == 2 ranks bitwise; the
    2-rank golden is reproduced exactly by the single-box oracle."""
    Q, A, _, _, _, _ = oracle.run(*golden_setup("parallel_2rank"))
    g = golden("parallel_2rank")
    assert np.abs(Q - g["Q"]).max() == 0.0 and np.abs(A - g["Qaux"]).max() == 0.0


def _all_parity_setups():
    from cases import CASES_1D, CASES_2D, CASES_SME, config2_strip_setup, setup, sme_strip_setup
    out = {f"golden/{n}": (lambda n=n: golden_setup(n)) for n in sorted(GOLDEN_CASES)}
    out.update({f"2d/{n}": (lambda n=n: setup(*CASES_2D[n])) for n in sorted(CASES_2D)})
    out.update({f"1d/{n}": (lambda n=n: setup(*CASES_1D[n])) for n in sorted(CASES_1D)})
    out["config2_strip_4096x64_20steps"] = lambda: config2_strip_setup(steps=20)
    out.update({f"sme/{n}": (lambda n=n: setup(*CASES_SME[n])) for n in sorted(CASES_SME)})
    out["sme_strip_2048x32_10steps"] = lambda: sme_strip_setup(steps=10)
    return out


PARITY_SETUPS = _all_parity_setups()


@pytest.mark.parametrize("name", sorted(PARITY_SETUPS))
def test_oracle_equals_reference_make_rhs(oracle, ref_oracle, name):
    """The restated make_rhs.H is bitwise the reference's make_rhs.H on every
    case the GPU parity tests use: the goldens (order 1), order-2 MUSCL,
    Audusse well-balancing over wet/dry bumps, point-implicit and explicit
    Manning friction, walls and mixed sides, 1-D and 2-D, and a strip of the
    benchmark level itself — so the GPU's bitwise parity with either oracle
    is parity with the reference's own make_rhs.H arithmetic
    (make_rhs.H:31-131, 154-163, 429-509)."""
    cfg, Q0, A0 = PARITY_SETUPS[name]()
    a = oracle.run(cfg, Q0, A0)
    b = ref_oracle.run(cfg, Q0, A0)
    assert a[2] == b[2] and a[3] == b[3], "step count / final time differ"
    assert np.isfinite(a[0]).all(), "the case should stay finite"
    assert np.array_equal(a[0], b[0], equal_nan=True), f"state max diff {np.nanmax(np.abs(a[0] - b[0])):.3e}"
    assert np.array_equal(a[1], b[1], equal_nan=True)
    assert np.array_equal(a[4][:, :2], b[4][:, :2]), "dt / time sequences differ"


def test_oracle_implicit_global_solves_backward_euler(oracle):
    """The oracle's implicit_global path solves q = q_exp + dt S(q) per cell:
    without a source term it equals the point-implicit path bitwise; with
    Manning friction it differs from the one linearised step by O(dt^2)."""
    from zoomy_amrex_b200._abi import ZFV_MODEL_SWE2D, make_config
    nx, ny = 24, 20
    x = (np.arange(nx) + 0.5) / nx * 5.0
    X, Y = np.meshgrid(x, (np.arange(ny) + 0.5) / ny * 5.0)
    h = 1.0 + 0.2 * np.exp(-((X - 2.5) ** 2 + (Y - 2.0) ** 2))
    Q0 = np.array([0 * h, h, 0.5 * h, -0.2 * h])
    A0 = np.zeros((7, ny, nx))
    out = {}
    for n_m in (0.0, 0.05):
        for glob in (False, True):
            cfg = make_config(ZFV_MODEL_SWE2D, nx, ny, (0, 0), (5, 5), spatial_order=2, implicit_source=True,
                              implicit_global=glob, cfl=0.45, time_end=1e30, max_step=6,
                              params={"n_m": n_m})
            out[(n_m, glob)] = oracle.run(cfg, Q0, A0)[0]
    assert np.array_equal(out[(0.0, False)], out[(0.0, True)])
    d = np.abs(out[(0.05, True)] - out[(0.05, False)]).max()
    assert 0.0 < d < 1e-4

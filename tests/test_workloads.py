"""The seeded synthetic workload generators (CPU only)."""
import numpy as np

from zoomy_amrex_b200._abi import ZFV_PREC_FP32
from zoomy_amrex_b200.workloads import dam_break_ensemble, fp64_twin


def test_ensemble_is_seeded_and_in_range():
    a = dam_break_ensemble(64, seed=11)
    b = dam_break_ensemble(64, seed=11)
    sides = []
    for (ca, qa, aa), (cb, qb, ab) in zip(a, b):
        assert (ca.nx, ca.ny) == (cb.nx, cb.ny)
        assert np.array_equal(qa, qb) and np.array_equal(aa, ab)
        assert 32 <= ca.nx <= 512 and 32 <= ca.ny <= 512
        assert ca.precision == ZFV_PREC_FP32 and fp64_twin(ca).precision == 0
        assert qa.shape == (4, ca.ny, ca.nx) and (qa[1] >= 0).all()
        eta = qa[0] + qa[1]
        left = eta[:, : ca.nx // 2][qa[1][:, : ca.nx // 2] > 0]
        assert 1.2 <= left.min() + 1e-12 and left.max() <= 3.0 + 1e-12
        sides += [ca.nx, ca.ny]
    # log-uniform: about half of the sides below the geometric mean 128
    assert 0.3 < np.mean(np.array(sides) < 128) < 0.7

"""oracle/torch_swe.py (the tensor restatement autograd is taken of) against the oracle."""
import numpy as np
import pytest
import torch

from oracle import torch_swe as T
from zoomy_amrex_b200._abi import ZFV_MODEL_SWE2D, make_config
from test_adjoint_cpu import wet_state


@pytest.mark.parametrize("wb", [True, False])
def test_torch_restatement_matches_oracle(oracle, wb):
    nx, ny = 20, 16
    Q0 = wet_state(nx, ny, 2, dry=True)
    A0 = np.zeros((7, ny, nx))
    A0[6] = T.hinv(torch.from_numpy(Q0[1]), 1e-24).numpy()
    cfg = make_config(ZFV_MODEL_SWE2D, nx, ny, (0, 0), (1, 1), spatial_order=2, well_balanced=wb,
                      implicit_source=True, bc=("wall", "extrapolation", "wall", "wall"),
                      params={"n_m": 0.03}, cfl=0.45, time_end=1e30, max_step=10)
    Qo, _, n, _, log, _ = oracle.run(cfg, Q0, A0)
    p = dict(g=9.81, ex=0.0, ey=0.0, h_floor=1e-6, eps=1e-24)
    Qt, dts = T.run(torch.from_numpy(Q0), torch.from_numpy(A0[6]), 0.03, 10, p, 1 / nx, 1 / ny, (1, 0, 1, 1), wb=wb)
    assert n == 10
    # the same IEEE operations in the same order: bit for bit
    assert np.array_equal(Qt.numpy(), Qo)
    assert np.array_equal(np.array([float(d) for d in dts]), log[:, 0])


def test_torch_restatement_bitwise_on_the_benchmark_fields(oracle):
    """The benchmark's wet/dry bump fields at 128^2 (Manning implicit, WB,
    walls), 30 steps: bit for bit the oracle, so autograd of the restatement
    takes the same minmod / max / wet-dry branches as the CUDA forward."""
    from zoomy_amrex_b200.workloads import bump_workload_config, bump_workload_fields
    m = 128
    Q0, A0 = bump_workload_fields(m)
    cfg = bump_workload_config(m)
    cfg.max_step = 30
    Qo, _, n, _, log, _ = oracle.run(cfg, Q0, A0)
    p = dict(g=9.81, ex=0.0, ey=0.0, h_floor=1e-6, eps=1e-24)
    Qt, dts = T.run(torch.from_numpy(Q0), torch.from_numpy(A0[6]), torch.tensor(0.03, dtype=torch.float64), 30,
                    p, 100.0 / m, 100.0 / m, (1, 1, 1, 1), checkpoint=True)
    assert n == 30 and np.array_equal(Qt.numpy(), Qo)
    assert np.array_equal(np.array([float(d) for d in dts]), log[:, 0])

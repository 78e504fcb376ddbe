"""Known answers for the shallow-moment model through the CPU oracle.

A spatially uniform state (flat bed, extrapolation sides) has no flux
differences and no fluctuations, so each SSP-RK2 stage reduces to the
point-implicit friction step q -> (I - dt J)^{-1} q (the Navier-slip
friction is linear in the momenta at fixed depth, S = J q) and a step to
q -> (q + (I - dt J)^{-2} q) / 2. With J taken from the symbolic derivation
(tests/sme_sympy.py) this checks the model's source and Jacobian, the
reference's 8 x 8 elimination (make_rhs.H:429-509, through oracle/_ref where
built) and the stage/Heun driver together.
"""
import numpy as np
import pytest

from zoomy_amrex_b200._abi import ZFV_MODEL_SME1D_L2, ZFV_MODEL_SME2D_L2, make_config


@pytest.fixture(scope="module")
def impl(parity_oracle):
    return parity_oracle


@pytest.mark.parametrize("dim", [1, 2])
def test_uniform_state_friction_decay(impl, dim):
    from sme_sympy import numeric
    nx, ny = (12, 1) if dim == 1 else (8, 6)
    q0 = np.array([0.0, 1.3, 0.2, -0.1, 0.04, -0.03, 0.02, 0.01]) if dim == 2 else \
        np.array([0.0, 1.3, 0.2, 0.04, -0.03])
    n = len(q0)
    Q0 = np.ascontiguousarray(np.broadcast_to(q0[:, None, None], (n, ny, nx)))
    A0 = np.zeros((1, ny, nx))
    nu, lam = 2e-2, 0.05
    model = ZFV_MODEL_SME2D_L2 if dim == 2 else ZFV_MODEL_SME1D_L2
    cfg = make_config(model, nx, ny, (0, 0), (1.0, 1.0 if dim == 2 else 1.0 / nx), spatial_order=2,
                      implicit_source=True, cfl=0.45, time_end=1e30, max_step=25,
                      params={"nu": nu, "lambda": lam})
    Q, A, steps, t, log, _ = impl.run(cfg, Q0, A0)
    assert steps == 25
    # every cell stays the same
    assert np.array_equal(Q, np.broadcast_to(Q[:, :1, :1], Q.shape))
    J = np.asarray(numeric(2, dim)["dSdq"](q0, (9.81, 0.0, 0.0, nu, lam)), float)
    q = q0.copy()
    for k in range(steps):
        M = np.linalg.inv(np.eye(n) - log[k, 0] * J)
        q = 0.5 * (q + M @ (M @ q))
    np.testing.assert_allclose(Q[:, 0, 0], q, rtol=1e-12, atol=1e-15)
    # friction dissipates the depth-integrated kinetic energy
    # h/2 (u^2 + sum_j alpha_j^2/(2j+1)) (per velocity component)
    def energy(v):
        h = v[1]
        vel = v[2:] / h
        w = np.array(([1.0] * dim) + [1 / 3, 1 / 5] * dim)
        return 0.5 * h * (w * vel * vel).sum()
    assert energy(Q[:, 0, 0]) < energy(q0)


def test_lake_at_rest_stays_at_rest(impl):
    """Still water over a bump, fully wet, no moments, well-balanced, order 2:
    the momenta and moments stay at round-off level (every moment source and
    product is proportional to a velocity)."""
    from cases import setup
    from zoomy_amrex_b200.models import SME

    def ic(x):
        b = 0.4 * np.exp(-((x[0] - 5.0) ** 2 + (x[1] - 5.0) ** 2) / 3.0)
        h = 1.0 - b
        z = np.zeros_like(h)
        return np.array([b, h, z, z, z, z, z, z])
    model = SME(level=2, dimension=3, bc="wall", initial_conditions=ic)
    s = dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[30, 30], spatial_order=2, cfl=0.45, time_end=1e30,
             max_step=50, well_balanced=True, implicit_source=True)
    cfg, Q0, A0 = setup(model, s)
    Q, _, _, _, _, _ = impl.run(cfg, Q0, A0)
    assert np.abs(Q[2:4]).max() < 1e-13 and np.abs(Q[4:]).max() < 1e-14

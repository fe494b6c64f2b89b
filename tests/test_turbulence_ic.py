"""The decaying-turbulence workload ("turb"): properties of its initial state,
built by the shared problem header, through the CPU restatement (which the
reference's fixtures turb_16 / turb_32 pin bit for bit).

On a uniform grid of more than 8 points per axis the 128 Fourier modes
(1 <= |k| <= 4) are orthogonal, so the sampled field has exactly the rms Mach
number the mode amplitudes were scaled to (5 at sound speed 1) and zero mean
momentum; the field is B = (B_x, 0, 0) with beta = 2 p / B^2 = 0.1 and the
pressure is uniform, p = 1 / gamma.
"""
import numpy as np
import pytest

GAMMA = 5 / 3


@pytest.fixture(scope="module")
def state():
    from oracle.kr_oracle import OracleMesh
    m = OracleMesh(True, (2, 1, 1), (8, 16, 16), GAMMA)
    m.init_problem("turb", 4)
    return m.get_state()


def test_rms_mach_and_zero_mean(state):
    u, _ = state
    rho = u[..., 0]
    v = u[..., 2:5] / rho[..., None]
    assert np.allclose(rho, 1.0)
    assert abs(np.sqrt((v ** 2).sum(-1).mean()) - 5.0) <= 1e-12
    assert np.abs(u[..., 2:5].mean(axis=(0, 1, 2, 3))).max() <= 1e-12


def test_pressure_and_beta(state):
    u, bf = state
    v2 = ((u[..., 2:5] / u[..., :1]) ** 2).sum(-1)
    b2 = (u[..., 5:8] ** 2).sum(-1)
    p = (u[..., 1] - 0.5 * u[..., 0] * v2 - 0.5 * b2) * (GAMMA - 1)
    np.testing.assert_allclose(p, 1 / GAMMA, rtol=1e-12)
    np.testing.assert_allclose(2 * p / b2, 0.1, rtol=1e-12)
    assert np.all(u[..., 6:8] == 0)


def test_seed_changes_phases_only():
    from oracle.kr_oracle import OracleMesh
    out = []
    for seed in (4, 5):
        m = OracleMesh(True, (1, 1, 1), (16, 16, 16), GAMMA)
        m.init_problem("turb", seed)
        u, _ = m.get_state()
        v = u[..., 2:5] / u[..., :1]
        out.append(v)
        assert abs(np.sqrt((v ** 2).sum(-1).mean()) - 5.0) <= 1e-12
    assert np.abs(out[0] - out[1]).max() > 1.0

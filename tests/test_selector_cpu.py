"""The CPU restatement of the selector MLP (oracle/kr_mlp_ref.py) is itself
checked here: analytic gradient vs central finite differences, and the bf16
rounding helper."""
import numpy as np

from oracle import kr_mlp_ref as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(64, M.N_IN))
    y = (rng.random(64) > 0.4).astype(float)
    w = rng.normal(scale=0.3, size=M.N_PARAM)
    loss, g = M.loss_grad(X, y, w, wneg=3.0)
    for k in rng.choice(M.N_PARAM, 60, replace=False):
        e = np.zeros(M.N_PARAM)
        e[k] = 1e-6
        num = (M.loss_grad(X, y, w + e, 3.0)[0] - M.loss_grad(X, y, w - e, 3.0)[0]) / 2e-6
        assert abs(num - g[k]) <= 1e-6 * max(1.0, abs(num)), (k, num, g[k])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.001953125, 3.14159265, -2.5e-3], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0      # 1 + 2^-8 is a tie: to even
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)

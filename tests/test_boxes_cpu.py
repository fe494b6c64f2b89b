"""Batched independent boxes without a GPU: the seeded box parameters (shared
problem header, through the library's kr_box_params) and the configuration
checks of KR_FLAG_BOXES contexts, which run before any device call."""
import numpy as np
import pytest

from kratos_b200 import KratosError


def test_box_parameters_in_range():
    from kratos_b200.boxes import box_params
    from oracle.kr_oracle import box_n
    gam = 5 / 3
    ps = [box_params(5, b, gam) for b in range(1024)]
    sizes = np.array([p["n"] for p in ps])
    assert set(sizes.tolist()) == {16, 24, 32, 48, 64}
    assert np.bincount(np.searchsorted([16, 24, 32, 48, 64], sizes)).min() > 150   # ~205 each
    for b, p in enumerate(ps[:64]):
        assert p["n"] == box_n(5, b)
    for p in ps:
        assert 0.5 <= p["rho"] < 2 and 0.1 <= p["pre"] < 10 and 0.05 <= p["beta"] < 10
        cs = np.sqrt(gam * p["pre"] / p["rho"])
        assert 0.1 - 1e-12 <= p["amp"] / cs < 2
        b2 = sum(x * x for x in p["b"])
        assert abs(2 * p["pre"] / b2 - p["beta"]) <= 1e-12 * p["beta"]


@pytest.mark.parametrize("kw,msg", [
    (dict(mhd=False), "KR_FLAG_BOXES needs MHD"),
    (dict(nb=(4, 2, 1)), "KR_FLAG_BOXES needs"),
    (dict(kinds=("out", "out", "per", "per", "per", "per")), "KR_FLAG_BOXES needs"),
    (dict(n_ranks=2, rank=0), "KR_FLAG_BOXES needs"),
])
def test_boxes_context_rejects(kw, msg):
    from kratos_b200 import Dynamics
    from kratos_b200._lib import KR_FLAG_BOXES
    mhd = kw.pop("mhd", True)
    nb = kw.pop("nb", (4, 1, 1))
    with pytest.raises(KratosError, match=msg):
        Dynamics(mhd, nb, (16, 16, 16), flags=KR_FLAG_BOXES, **kw)

"""Static mesh refinement without a GPU: the refined-mesh checks of the C ABI
that run before any device call, and the oracle's refined step on properties
that do not depend on the reference fixtures."""
import numpy as np
import pytest

from kratos_b200 import KratosError

REG = [(1, (0.3, 0.1, 0.1), (0.45, 0.4, 0.4))]


def _refined(mhd=False, nb=(2, 2, 2), n=(8, 8, 8), regions=REG, **kw):
    from kratos_b200 import Dynamics
    return Dynamics(mhd, nb, n, regions=regions, **kw)


@pytest.mark.parametrize("kw,msg", [
    (dict(mhd=True, riemann=2), "uniform meshes"),
    (dict(n_ranks=2, rank=0), "one rank"),
    (dict(flags=2), "one rank"),
    (dict(n=(8, 6, 9)), "even number of cells"),
    (dict(regions=[(1, (0.3, 0.1, 0.1), (1.5, 0.4, 0.4))]), "Incorrect SMR region"),
    (dict(regions=[(7, (0.3, 0.1, 0.1), (0.4, 0.4, 0.4))]), "refinement level out of range"),
])
def test_refined_context_rejects(kw, msg):
    with pytest.raises(KratosError, match=msg):
        _refined(**kw)


def test_oracle_refined_step_conserves():
    """The flux correction makes the refined step conservative: on a periodic
    mesh with two level jumps the volume-weighted totals stay constant."""
    from oracle.kr_oracle import OracleMesh
    m = OracleMesh(False, (2, 2, 2), (8, 8, 8), 1.4,
                   regions=[(1, (0.3, 0.3, 0.3), (0.7, 0.45, 0.6)), (2, (0.4, 0.35, 0.4), (0.45, 0.4, 0.45))])
    assert m.level.max() == 2
    vol = np.array([np.prod([m.dx(b, a) for a in range(3)]) for b in range(m.nblk)])
    m.init_problem("shock", 4)
    u0, _ = m.get_state()
    m.step(12)
    u1, _ = m.get_state()
    t0 = np.einsum("b,bzyxk->k", vol, u0)
    t1 = np.einsum("b,bzyxk->k", vol, u1)
    assert abs(t1[0] - t0[0]) <= 1e-13 * t0[0]
    assert abs(t1[1] - t0[1]) <= 1e-13 * t0[1]
    assert np.all(np.abs(t1[2:] - t0[2:]) <= 1e-13 * t0[1])
    # the shock moved across the level jumps
    assert np.abs(u1 - u0).max() > 1e-2


def test_oracle_refined_leaves_cover_the_domain():
    """Every point of the domain lies in exactly one leaf: leaf volumes add up
    to the domain and no two leaves overlap."""
    from oracle.kr_oracle import OracleMesh
    m = OracleMesh(False, (3, 2, 2), (8, 8, 8), 1.4, kinds=("ref", "out", "per", "per", "fre", "fre"),
                   regions=[(2, (0.05, 0.9, 0.1), (0.1, 0.95, 0.2)), (1, (0.5, 0.2, 0.6), (0.7, 0.3, 0.9))])
    top = m.level.max()
    assert top == 2
    fine = np.zeros((2 << top, 2 << top, 3 << top), dtype=int)   # z, y, x at the top level
    for b in range(m.nblk):
        s = 1 << (top - m.level[b])
        x, y, z = m.reg[b] * s
        fine[z:z + s, y:y + s, x:x + s] += 1
    assert np.all(fine == 1)

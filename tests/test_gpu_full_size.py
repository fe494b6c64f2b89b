"""The benchmark configurations at their full sizes, through properties that do
not depend on a fixture: |div B| at FP64 roundoff, exact conservation on
periodic meshes, and the mixed-precision and learned steps within 1e-4
relative L1 density of the FP64 step (the stated tolerance of the headline
metric).

* 256^3 Orszag-Tang MHD in 64 blocks of 64^3, 50 steps (the headline mesh);
* decaying turbulence (rms Mach 5, beta 0.1) on 128^3 in 8 blocks of 64^3;
* 256 boxes of the batched-box workload (seed 5; 16^3 to 64^3), each on its
  own dt, 10 steps.
Fixture-pinned parity at small sizes is in test_gpu_parity.py,
test_gpu_selector.py and test_gpu_boxes.py.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GAMMA = 5 / 3


def rel_l1(a, b):
    return np.abs(a - b).sum() / np.abs(b).sum()


def _trained_selector():
    from kratos_b200 import Dynamics
    from kratos_b200 import selector as S

    def mk():
        d = Dynamics(True, (2, 2, 2), (32, 32, 32), gamma=GAMMA, precision=1)
        d.init_problem("ot", 2)
        return d
    w, _ = S.build_selector([mk], steps=4, stride=8, epochs=20)
    return w, S.DEFAULT_THRESHOLD


def _totals(u):
    """Mass, energy and momentum summed on the host, each component as one
    contiguous array so that numpy sums pairwise (~1e-15 relative over 10^7
    cells; a row-by-row reduction along a strided axis, or the device's
    atomic totals, carry up to ~N eps)."""
    return np.array([np.ascontiguousarray(u[..., k]).sum() for k in range(5)])


def _run(mesh, workload, steps, **kw):
    """(rho, div B before, div B after, totals before, totals after)."""
    from kratos_b200 import Dynamics
    nb, n = mesh
    sel = kw.pop("selector", None)
    d = Dynamics(True, nb, n, gamma=GAMMA, **kw)
    try:
        d.init_problem(workload, 2 if workload == "ot" else 4)
        if sel is not None:
            d.set_selector(*sel)
        div0, _ = d.diagnostics()
        tot0 = _totals(d.get_state()[0])
        d.step(steps)
        div1, _ = d.diagnostics()
        assert d.status() == 0
        u, _ = d.get_state()
        return u[..., 0].copy(), div0, div1, tot0, _totals(u)
    finally:
        d.close()


def _check_invariants(div0, div1, tot0, tot1):
    assert div0 <= 1e-12 and div1 <= 1e-12, (div0, div1)
    assert abs(tot1[0] - tot0[0]) <= 1e-12 * abs(tot0[0])       # mass
    assert abs(tot1[1] - tot0[1]) <= 1e-12 * abs(tot0[1])       # energy
    assert np.all(np.abs(tot1[2:] - tot0[2:]) <= 1e-12 * abs(tot0[1]))


def test_headline_mesh_fp64_mixed_learned():
    """256^3 OT, 64 blocks of 64^3, 50 steps: the three modes of the metric."""
    mesh, steps = ((4, 4, 4), (64, 64, 64)), 50
    rho64, *inv = _run(mesh, "ot", steps, precision=2)
    _check_invariants(*inv)
    rho32, *inv = _run(mesh, "ot", steps, precision=1)
    _check_invariants(*inv)
    e_mixed = rel_l1(rho32, rho64)
    sel = _trained_selector()
    rhol, *inv = _run(mesh, "ot", steps, precision=1, riemann=2, sel_period=16, selector=sel)
    _check_invariants(*inv)
    e_learn = rel_l1(rhol, rho64)
    print("256^3 OT, 50 steps: rel L1 density vs FP64: mixed %.2e, learned %.2e" % (e_mixed, e_learn))
    assert e_mixed <= 1e-4 and e_learn <= 1e-4


def test_turbulence_128_mixed_and_learned():
    mesh, steps = ((2, 2, 2), (64, 64, 64)), 20
    rho64, *inv = _run(mesh, "turb", steps, precision=2)
    _check_invariants(*inv)
    rho32, *inv = _run(mesh, "turb", steps, precision=1)
    _check_invariants(*inv)
    sel = _trained_selector()
    rhol, *inv = _run(mesh, "turb", steps, precision=1, riemann=2, sel_period=16, selector=sel)
    _check_invariants(*inv)
    e_mixed, e_learn = rel_l1(rho32, rho64), rel_l1(rhol, rho64)
    print("128^3 turbulence, 20 steps: rel L1 density vs FP64: mixed %.2e, learned %.2e" % (e_mixed, e_learn))
    assert e_mixed <= 1e-4 and e_learn <= 1e-4


def test_box_batch_256_boxes():
    from kratos_b200.boxes import BoxBatch
    steps = 10
    out = {}
    for prec in (2, 1):
        bb = BoxBatch(5, 256, precision=prec)
        try:
            before = {n: (d.diagnostics()[0], _totals(d.get_state()[0]))
                      for n, (d, _) in bb.groups.items()}
            bb.step(steps)
            assert bb.status() == 0
            for n, (d, _) in bb.groups.items():
                div1, _ = d.diagnostics()
                _check_invariants(before[n][0], div1, before[n][1], _totals(d.get_state()[0]))
            t, _ = bb.times()
            assert np.all(t > 0)
            out[prec] = ({b: u[..., 0].copy() for b, (u, _) in bb.states().items()}, t)
        finally:
            bb.close()
    # every box advanced on its own dt; mixed within 1e-4 of FP64 box by box
    assert len(set(np.round(out[2][1], 10))) > 200
    worst = max(rel_l1(out[1][0][b], out[2][0][b]) for b in out[2][0])
    print("256 boxes, 10 steps: worst box rel L1 density mixed vs FP64 %.2e" % worst)
    assert worst <= 1e-4

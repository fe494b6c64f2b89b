"""Statically refined hydro meshes on the GPU, through the C ABI
(kr_ctx_create_refined), against the original Kratos solver's refined runs
(golden fixtures smr_*) and the CPU restatement.

Tolerances as for the uniform FP64 step: relative L1 per conserved field
(momentum components against the momentum vector's L1 norm) <= 1e-11 after
the fixtures' 4-5 steps (fused multiply-adds on the device),
<= 1e-10 for the longer oracle runs; the mixed step (FP32 reconstruction,
Riemann solver and ghost words, FP64 state) within 1e-4 relative L1 density.
The size-independent checks: the flux correction makes the refined step
conservative (periodic mesh: total mass, energy and momentum kept to
rounding), and a refinement region over a uniform state leaves it uniform.
"""
import numpy as np
import pytest

import golden_io as G

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-11
TOL_FP64_LONG = 1e-10
TOL_MIXED = 1e-4


def rel_l1(a, b):
    den = np.abs(b).sum()
    return np.abs(a - b).sum() / (den if den > 0 else 1.0)


def _dyn(meta, precision=2, **kw):
    from kratos_b200 import Dynamics
    kinds, w_fix, b_fix = G.boundary(meta)
    return Dynamics(False, meta["nb"], meta["n"], gamma=meta["gamma"], cfl=meta["cfl"],
                    precision=precision, kinds=kinds, w_fix=w_fix, regions=G.regions(meta), **kw)


@pytest.mark.parametrize("name", G.SMR_CASES)
def test_refined_step_matches_reference(name):
    meta, g = G.load(name)
    d = _dyn(meta)
    assert np.array_equal(d.level, g["level"]) and np.array_equal(d.reg, g["reg"])
    d.init_problem("shock", meta["seed"])
    if "u0" in g:
        u0, _ = d.get_state()
        assert np.array_equal(u0, g["u0"])
    d.step(meta["steps"])
    u, _ = d.get_state()
    tm = d.time()
    assert d.status() == 0
    assert abs(tm["t"] - meta["t"]) <= 1e-12 * meta["t"]
    assert abs(tm["dt_last"] - meta["dt"]) <= 1e-12 * meta["dt"]
    for k, e in enumerate(G.field_errors(u, g["u1"])):
        assert e <= TOL_FP64, "field %d rel L1 %.3e" % (k, e)


REGIONS = [(1, (0.1, 0.6, 0.2), (0.4, 0.9, 0.3)), (2, (0.55, 0.2, 0.7), (0.6, 0.25, 0.75))]


@pytest.mark.parametrize("kinds", [("per",) * 6, ("ref", "out", "fre", "fixd", "per", "per")])
def test_refined_step_matches_oracle(kinds):
    from kratos_b200 import Dynamics
    from oracle.kr_oracle import OracleMesh
    nb, n = (2, 2, 2), (8, 8, 16)
    w_fix = (1.0, 1.0, 0.3, 0.0, 0.0)
    m = OracleMesh(False, nb, n, 1.4, kinds=kinds, w_fix=w_fix, regions=REGIONS)
    d = Dynamics(False, nb, n, gamma=1.4, kinds=kinds, w_fix=w_fix, regions=REGIONS)
    assert np.array_equal(d.level, m.level) and np.array_equal(d.reg, m.reg)
    assert d.level.max() == 2
    m.init_problem("shock", 21)
    d.init_problem("shock", 21)
    m.step(12)
    d.step(12)
    u_ref, _ = m.get_state()
    u, _ = d.get_state()
    assert d.time()["t"] == pytest.approx(m.t, rel=1e-12)
    for k, e in enumerate(G.field_errors(u, u_ref)):
        assert e <= TOL_FP64_LONG, "field %d rel L1 %.3e" % (k, e)


def test_refined_mixed_precision_against_oracle():
    from kratos_b200 import Dynamics
    from oracle.kr_oracle import OracleMesh
    meta, g = G.load("smr_shock")
    d = _dyn(meta, precision=1)
    d.init_problem("shock", meta["seed"])
    d.step(meta["steps"])
    u, _ = d.get_state()
    assert rel_l1(u[..., 0], g["u1"][..., 0]) <= TOL_MIXED


@pytest.mark.parametrize("precision", [2, 1])
def test_refined_step_conserves(precision):
    """Periodic refined mesh: the fine fluxes replace the coarse ones on every
    level jump, so the volume-weighted totals stay constant to rounding."""
    from kratos_b200 import Dynamics
    d = Dynamics(False, (4, 4, 4), (16, 16, 16), gamma=1.4, precision=precision,
                 regions=[(1, (0.3, 0.3, 0.3), (0.7, 0.45, 0.6)), (2, (0.4, 0.35, 0.4), (0.5, 0.4, 0.5))])
    assert d.level.max() == 2
    d.init_problem("shock", 8)
    _, tot0 = d.diagnostics()
    d.step(40)
    _, tot1 = d.diagnostics()
    assert d.status() == 0
    assert abs(tot1[0] - tot0[0]) <= 1e-12 * abs(tot0[0])      # mass
    assert abs(tot1[1] - tot0[1]) <= 1e-12 * abs(tot0[1])      # energy
    for k in (2, 3, 4):                                        # momentum (starts at 0)
        assert abs(tot1[k] - tot0[k]) <= 1e-12 * abs(tot0[1])


def test_uniform_state_stays_uniform_across_levels():
    """A constant state on a refined mesh: restriction, prolongation (zero
    slopes) and the corrected update reproduce it exactly at every level."""
    from kratos_b200 import Dynamics
    d = Dynamics(False, (2, 2, 2), (8, 8, 8), gamma=1.4,
                 regions=[(2, (0.3, 0.3, 0.3), (0.35, 0.35, 0.35))])
    u = np.zeros(d.u_shape)
    u[..., 0] = 1.25
    u[..., 1] = 2.5
    u[..., 2] = 0.5
    d.set_state(u)
    d.step(5)
    out, _ = d.get_state()
    np.testing.assert_allclose(out, u, rtol=1e-13, atol=1e-13)


def test_refined_mixed_precision_with_sides_against_reference():
    """The mixed step on the refined fixture with reflecting / outflow / free
    sides and ragged blocks, against the reference's FP64 run."""
    meta, g = G.load("smr_bc")
    d = _dyn(meta, precision=1)
    d.init_problem("shock", meta["seed"])
    d.step(meta["steps"])
    u, _ = d.get_state()
    assert d.status() == 0
    assert rel_l1(u[..., 0], g["u1"][..., 0]) <= TOL_MIXED

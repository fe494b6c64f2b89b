"""CUDA step against the original Kratos solver (golden fixtures) and the CPU
restatement of it, through the C ABI.

Tolerances (FP64 step): the device arithmetic follows the reference expression
by expression but fuses multiply-adds, so agreement is to rounding, not to the
bit.  Stated bound: relative L1 per conserved field and per face-B component
<= 1e-11 after the fixtures' 3-10 steps, <= 1e-10 after config 1's 20 shock
steps (limiter switches amplify rounding there); initial states are bit-exact
(host-built from the same header).  Mixed step (FP32 reconstruction / Riemann,
FP64 state): relative L1 density error vs the FP64 oracle <= 1e-4 (the
north-star bound); |div B| <= 1e-12 in both modes.
"""
import numpy as np
import pytest

import golden_io as G

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-11
TOL_FP64_LONG = 1e-10


def _dyn(meta, precision=2, riemann=0):
    from kratos_b200 import Dynamics
    extra = meta.get("dynamics", {})
    kinds, w_fix, b_fix = G.boundary(meta)
    return Dynamics(meta["workload"] in G.MHD_WORKLOADS, meta["nb"], meta["n"], gamma=meta["gamma"],
                    cfl=meta["cfl"], tmp_floor=float(extra.get("tmp_floor", 1e-9)),
                    precision=precision, riemann=riemann, kinds=kinds, w_fix=w_fix, b_fix=b_fix)


def rel_l1(a, b):
    den = np.abs(b).sum()
    return np.abs(a - b).sum() / (den if den > 0 else 1.0)


@pytest.mark.parametrize("name", ["shock_16", "ot_16"])
def test_initial_state_bit_exact(name):
    meta, g = G.load(name)
    d = _dyn(meta)
    d.init_problem(meta["workload"], meta["seed"])
    u, bf = d.get_state()
    assert np.array_equal(u[..., :5], g["u0"][..., :5])
    if d.mhd:
        mask = G.face_mask(meta["n"])
        assert np.array_equal(G.owned_bf(bf, meta["n"])[:, mask], g["bf0"][:, mask])
        # u slots 5..7 hold the face-averaged B, which is what the reference
        # pgen writes there initially
        np.testing.assert_array_equal(u[..., 5:], g["u0"][..., 5:])


@pytest.mark.parametrize("name", ["shock_16", "ot_16", "ot_ragged", "shock_floor",
                                  "shock_bc", "shock_fixd", "ot_bc_out", "ot_bc_fre", "ot_bc_fix",
                                  "turb_16"])
def test_fp64_step_matches_reference(name):
    meta, g = G.load(name)
    d = _dyn(meta)
    d.init_problem(meta["workload"], meta["seed"])
    d.step(meta["steps"])
    u, bf = d.get_state()
    tm = d.time()
    assert d.status() == 0
    assert abs(tm["t"] - meta["t"]) <= 1e-12 * meta["t"]
    assert abs(tm["dt_last"] - meta["dt"]) <= 1e-12 * meta["dt"]
    for k in range(5):
        e = rel_l1(u[..., k], g["u1"][..., k])
        assert e <= TOL_FP64, "field %d rel L1 %.3e" % (k, e)
    if d.mhd:
        own = G.owned_bf(bf, meta["n"])
        mask = G.face_mask(meta["n"])
        for c in range(3):
            m = mask[..., c]
            e = rel_l1(own[..., c][:, m], g["bf1"][..., c][:, m])
            assert e <= TOL_FP64, "bf %d rel L1 %.3e" % (c, e)


def _bf_errors(bf, ref_own, n):
    """Relative L1 per face-B component over the owned faces, against the L1
    norm of the whole field (B_z starts at zero in the OT workload)."""
    own, mask = G.owned_bf(bf, n), G.face_mask(n)
    den = sum(np.abs(ref_own[..., c][:, mask[..., c]]).sum() for c in range(3))
    return [np.abs(own[..., c][:, mask[..., c]] - ref_own[..., c][:, mask[..., c]]).sum() / den
            for c in range(3)]


def test_mhd_reflecting_sides():
    """Reflecting MHD walls put mirror-image states on the two sides of the
    wall face, where HLLD's branches (the contact-speed sign, the f_tiny
    switches) sit at their thresholds, so rounding alone moves the result.
    Measured: the oracle built with fused multiply-add differs from the one
    without it (the reference's own arithmetic, bit-exact with the fixture) by
    3.6e-6 relative L1 in density after one step and 2.7e-5 after four, and
    the device's no-FMA build lands as far away as its fused build (its
    arithmetic is restructured, so its roundings differ either way).  The
    device step (FP64) is therefore held, field by field, to 3x the FMA
    oracle's own distance from the fixture, with mass conserved exactly and
    div B at roundoff; the same bound with the FMA oracle replaced by the
    fixture itself is 0, so a kernel error of that size would fail."""
    from oracle.kr_oracle import OracleMesh
    meta, g = G.load("ot_bc_ref")
    kinds, w_fix, b_fix = G.boundary(meta)
    n = meta["n"]
    o = OracleMesh(True, meta["nb"], n, meta["gamma"], kinds=kinds, w_fix=w_fix, b_fix=b_fix,
                   variant="fma")
    o.init_problem("ot", meta["seed"])
    o.step(meta["steps"])
    uf, bff = o.get_state()
    spread_u = G.field_errors(uf, g["u1"])
    spread_b = _bf_errors(bff, g["bf1"], n)
    assert max(spread_u) > 1e-8, "rounding must move this case (else hold it to 1e-11)"
    d = _dyn(meta)
    d.init_problem("ot", meta["seed"])
    div0, tot0 = d.diagnostics()
    d.step(meta["steps"])
    u, bf = d.get_state()
    div1, tot1 = d.diagnostics()
    assert abs(d.time()["t"] - meta["t"]) <= 1e-5 * meta["t"]
    for k, (e, sp) in enumerate(zip(G.field_errors(u, g["u1"]), spread_u)):
        assert e <= max(TOL_FP64, 3 * sp), "field %d: %.2e vs FMA spread %.2e" % (k, e, sp)
    for c, (e, sp) in enumerate(zip(_bf_errors(bf, g["bf1"], n), spread_b)):
        assert e <= max(TOL_FP64, 3 * sp), "bf %d: %.2e vs FMA spread %.2e" % (c, e, sp)
    assert div1 <= 1e-12
    assert abs(tot1[0] - tot0[0]) <= 1e-12 * abs(tot0[0])    # walls pass no mass


def test_mhd_static_fixed_sides():
    """Fixed MHD sides holding a static medium (vel0 = 0, ot_bc_fix0): the
    fluxes on the ghost lines between identical static ghost states carry a
    mass flux that is rounding residue, and the edge EMF's upwind switch
    (mhd/integrator/integrator.h:268-300) takes its branch from that residue's
    sign; the reference's residues are -1.4e-17, 2.1e-17 and 0 along x, y, z on
    this state (tests/test_oracle_golden.py), the device's restructured HLLD
    leaves others.  With an inflowing medium the same sides match the
    reference to 1e-11 (ot_bc_fix, above); here the device step is held to
    1e-4 relative L1 per conserved field and 1e-3 on face B (measured 1e-5
    and 4e-4 after the 4 steps), with mass conservation and div B exact."""
    meta, g = G.load("ot_bc_fix0")
    d = _dyn(meta)
    d.init_problem("ot", meta["seed"])
    div0, _ = d.diagnostics()
    d.step(meta["steps"])
    u, bf = d.get_state()
    div1, _ = d.diagnostics()
    assert d.status() == 0
    for k, e in enumerate(G.field_errors(u, g["u1"])):
        assert e <= 1e-4, "field %d: %.2e" % (k, e)
    for c, e in enumerate(_bf_errors(bf, g["bf1"], meta["n"])):
        assert e <= 1e-3, "bf %d: %.2e" % (c, e)
    assert div1 <= 1e-12


@pytest.mark.parametrize("name", ["shock_c1", "ot_64", "turb_32"])
def test_fp64_full_size_checksums(name):
    """Configs at full block size (turb_32: the turbulence workload on 16^3
    blocks): checksum-of-fields against the reference."""
    meta, g = G.load(name)
    d = _dyn(meta)
    d.init_problem(meta["workload"], meta["seed"])
    u0, _ = d.get_state()
    assert np.array_equal(G.checksums(u0[..., :5]), g["u0_sum"][:, :5])
    d.step(meta["steps"])
    u, bf = d.get_state()
    s = G.checksums(u[..., :5])
    ref = g["u1_sum"][:, :5]
    # sums of |u| and extrema to 1e-11 relative; signed sums (momenta ~ 0) absolute
    np.testing.assert_allclose(s[1:], ref[1:], rtol=TOL_FP64, atol=0)
    scale = ref[1]
    assert np.all(np.abs(s[0] - ref[0]) <= TOL_FP64 * scale)
    assert abs(d.time()["t"] - meta["t"]) <= 1e-12 * meta["t"]


def test_fp64_headline_mesh_against_reference():
    """The headline MHD configuration at its full size -- 256^3 Orszag-Tang,
    64 blocks of 64^3, seed 2, 50 steps -- against the reference's own CPU run
    of the same mesh (ot_256: per-field checksums and two sampled z-planes of
    the final state).  FP64 step, 1e-10 relative (50 steps of fused rounding
    through HLLD's branch switches), time to 1e-12."""
    import sys
    import os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_golden import sampled_planes
    meta, g = G.load("ot_256")
    d = _dyn(meta)
    d.init_problem(meta["workload"], meta["seed"])
    u0, _ = d.get_state()
    assert np.array_equal(G.checksums(u0[..., :5]), g["u0_sum"][:, :5])
    d.step(meta["steps"])
    u, bf = d.get_state()
    assert d.status() == 0
    s = G.checksums(u[..., :5])
    ref = g["u1_sum"][:, :5]
    np.testing.assert_allclose(s[1:], ref[1:], rtol=TOL_FP64_LONG, atol=0)
    assert np.all(np.abs(s[0] - ref[0]) <= TOL_FP64_LONG * ref[1])
    planes = sampled_planes(u, meta["nb"], meta["n"])
    for k, e in enumerate(G.field_errors(planes[..., :5], g["u1_planes"][..., :5])):
        assert e <= TOL_FP64_LONG, "plane field %d rel L1 %.2e" % (k, e)
    n = meta["n"]
    sb = G.face_checksums(bf, n)
    np.testing.assert_allclose(sb[1:], g["bf1_sum"][1:], rtol=TOL_FP64_LONG, atol=0)
    assert abs(d.time()["t"] - meta["t"]) <= 1e-12 * meta["t"]
    assert abs(d.time()["dt_last"] - meta["dt"]) <= 1e-12 * meta["dt"]


def test_fp64_against_oracle_c1_shape():
    """C1's mesh (64^3 in 8 blocks of 32^3), 20 steps, field by field."""
    from oracle.kr_oracle import OracleMesh
    meta, _ = G.load("shock_c1")
    d = _dyn(meta)
    d.init_problem("shock", meta["seed"])
    d.step(meta["steps"])
    u, _ = d.get_state()
    o = OracleMesh(False, meta["nb"], meta["n"], meta["gamma"])
    o.init_problem("shock", meta["seed"])
    o.step(meta["steps"])
    uo, _ = o.get_state()
    for k in range(5):
        assert rel_l1(u[..., k], uo[..., k]) <= TOL_FP64_LONG


def test_mhd_invariants_fp64():
    """div B at roundoff and conservation of mass, momentum and energy."""
    from kratos_b200 import Dynamics
    d = Dynamics(True, (2, 2, 2), (16, 16, 16), gamma=5 / 3)
    d.init_problem("ot", 7)
    div0, tot0 = d.diagnostics()
    d.step(10)
    div1, tot1 = d.diagnostics()
    assert div0 <= 1e-12 and div1 <= 1e-12, (div0, div1)
    assert abs(tot1[0] - tot0[0]) <= 1e-12 * abs(tot0[0])   # atomic summation order
    assert abs(tot1[1] - tot0[1]) <= 1e-12 * abs(tot0[1])
    assert np.all(np.abs(tot1[2:] - tot0[2:]) <= 1e-12 * abs(tot0[1]))


def test_mixed_precision_error_bound():
    """FP32 reconstruction + Riemann with FP64 state: density within 1e-4
    relative L1 of the FP64 oracle; div B at FP64 roundoff."""
    from oracle.kr_oracle import OracleMesh
    meta, _ = G.load("ot_64")
    d = _dyn(meta, precision=1)
    d.init_problem("ot", meta["seed"])
    d.step(meta["steps"])
    u, _ = d.get_state()
    div, _ = d.diagnostics()
    o = OracleMesh(True, meta["nb"], meta["n"], meta["gamma"])
    o.init_problem("ot", meta["seed"])
    o.step(meta["steps"])
    uo, _ = o.get_state()
    e = rel_l1(u[..., 0], uo[..., 0])
    assert e <= 1e-4, e
    assert div <= 1e-12


def test_status_word_starts_clean_and_steps_counted():
    from kratos_b200 import Dynamics
    d = Dynamics(False, (1, 1, 1), (8, 8, 8), gamma=1.4)
    d.init_problem("shock", 1)
    d.step(3)
    tm = d.time()
    assert tm["n_steps"] == 3 and d.status() == 0
    assert d.launches_per_step() == 12      # 2 x (c2p, 3 flux sweeps, update) + begin, end

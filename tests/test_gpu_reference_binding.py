"""The engine as a drop-in dynamics module of the ORIGINAL Kratos code.

oracle/_ref/kratos_ref_b200 is the reference's own sources (its mesh, cycle,
block data, boundary keeper, snapshot writer and main), built for the CPU by
oracle/Makefile.ref, with the problem generator's dynamics modules derived from
kratos_b200::b200_t< dynamics::mhd_t / hydro_t >
(kratos_b200/reference_binding/b200_dynamics.h): the reference's module class
whose step() runs on the B200 engine through the C ABI.  Run on the golden
fixtures' parameter files, its snapshots match the reference's own runs to the
FP64 parity bound (1e-11 relative L1 per conserved field and face-B
component), with the reference's cycle taking the engine's dt (time to 1e-12).
"""
import os
import sys

import numpy as np
import pytest

import golden_io as G

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "kratos_ref_b200")
TOL = 1e-11


@pytest.mark.parametrize("name", ["ot_16", "shock_16", "ot_bc_out", "ot_bc_fix"])
def test_reference_cycle_with_b200_module_matches_reference(name):
    if not os.path.exists(EXE):
        pytest.fail("%s is not built (make -f oracle/Makefile.ref REF=<kratos tree> b200)" % EXE)
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as MG
    from kratos_b200.snapshot import to_lex_arrays
    case = [c for c in MG.CASES if c[0] == name][0]
    _, problem, nb, n, steps, seed, gamma, extra, _ = case
    s0, s1 = MG.run_snapshots(EXE, problem, nb, n, steps, seed, gamma, extra)
    meta, g = G.load(name)
    u1, bf1 = to_lex_arrays(s1, nb)
    assert int(s1.array("cycle", "i")[0]) == steps - 1
    assert abs(float(s1.array("time")[0]) - meta["t"]) <= 1e-12 * meta["t"]
    for k, e in enumerate(G.field_errors(u1[..., :5], g["u1"][..., :5])):
        assert e <= TOL, "field %d rel L1 %.3e" % (k, e)
    if bf1 is not None:
        own, mask = G.owned_bf(bf1, n), G.face_mask(n)
        for c in range(3):
            m = mask[..., c]
            ref = g["bf1"][..., c][:, m]
            assert np.abs(own[..., c][:, m] - ref).sum() / np.abs(ref).sum() <= TOL, c

"""Batched independent periodic MHD boxes on the GPU (KR_FLAG_BOXES contexts,
kratos_b200/boxes.py) against the original Kratos solver run on each box alone.

The batch holds boxes 0..7 of seed 5 (edge lengths 64, 24, 48, 32, 64, 16, 24,
64), grouped into one context per edge length; every box advances on its own
CFL dt.  Fixtures: box 5 (16^3, final fields), boxes 1 (24^3) and 3 (32^3)
(checksums), 5 steps each.  Tolerances as for the uniform FP64 step: relative
L1 <= 1e-11 per conserved field and face-B component, checksums to 1e-11, each
box's own time and last dt to 1e-12; mixed precision within 1e-4 relative L1
density of the FP64 batch, div B at roundoff in both.
"""
import numpy as np
import pytest

import golden_io as G

pytestmark = pytest.mark.gpu

TOL = 1e-11


def rel_l1(a, b):
    return np.abs(a - b).sum() / np.abs(b).sum()


@pytest.fixture(scope="module")
def fp64_batch():
    from kratos_b200.boxes import BoxBatch
    bb = BoxBatch(5, 8)
    bb.step(5)
    yield bb
    bb.close()


@pytest.mark.parametrize("name", sorted(G.BOX_CASES))
def test_batched_box_matches_reference(fp64_batch, name):
    meta, g = G.load(name)
    box = G.BOX_CASES[name]
    bb = fp64_batch
    assert bb.sizes[box] == meta["n"][0]
    assert bb.status() == 0
    u, bf = bb.get_state(box)
    t, dl = bb.times()
    assert abs(t[box] - meta["t"]) <= 1e-12 * meta["t"]
    assert abs(dl[box] - meta["dt"]) <= 1e-12 * meta["dt"]
    if "u1" in g:
        for k, e in enumerate(G.field_errors(u, g["u1"])):
            assert e <= TOL, "field %d rel L1 %.3e" % (k, e)
        own = G.owned_bf(bf, meta["n"])
        mask = G.face_mask(meta["n"])
        for c in range(3):
            m = mask[..., c]
            assert rel_l1(own[..., c][:, m], g["bf1"][..., c][:, m]) <= TOL
    s = G.checksums(u[..., :5])
    ref = g["u1_sum"][:, :5]
    np.testing.assert_allclose(s[1:], ref[1:], rtol=TOL, atol=0)
    assert np.all(np.abs(s[0] - ref[0]) <= TOL * ref[1])


def test_boxes_keep_their_own_dt(fp64_batch):
    """Boxes of one context advance on different dt (independent CFL)."""
    t, dl = fp64_batch.times()
    d, ids = fp64_batch.groups[64]
    assert len(ids) == 3
    assert len(set(np.round(t[ids] / t[ids].max(), 12))) == 3
    assert np.all(t > 0)


def test_batched_box_matches_oracle(fp64_batch):
    """A 48^3 box of the batch against the CPU restatement run on it alone."""
    from oracle.kr_oracle import OracleMesh
    o = OracleMesh(True, (1, 1, 1), (48, 48, 48), 5 / 3)
    o.init_box(5, 2)
    o.step(5)
    uo, _ = o.get_state()
    u, _ = fp64_batch.get_state(2)
    for k, e in enumerate(G.field_errors(u, uo)):
        assert e <= 1e-10, (k, e)


def test_mixed_batch_error_bound(fp64_batch):
    from kratos_b200.boxes import BoxBatch
    mb = BoxBatch(5, 8, precision=1)
    mb.step(5)
    assert mb.status() == 0
    st64 = fp64_batch.states()
    for b, (u, _) in mb.states().items():
        assert rel_l1(u[..., 0], st64[b][0][..., 0]) <= 1e-4, b
    for d, _ in list(mb.groups.values()) + list(fp64_batch.groups.values()):
        div, _ = d.diagnostics()
        assert div <= 1e-12
    mb.close()


@pytest.mark.parametrize("kw", [dict(precision=2), dict(precision=1),
                                dict(precision=1, riemann=2, sel_period=2)])
def test_batched_launch_matches_per_group_launches(kw):
    """One launch per kernel kind over the work list of every group's CTA
    tiles (kr_batch) runs the per-group launches' tiles with the same device
    functions, compiled into other kernels, where the compiler may fuse
    multiply-adds differently: with the default grid, one CTA per item, and a
    grid of one wave, the boxes' states, times and dt agree with the per-group
    steps to the rounding of the step's arithmetic (FP64: 1e-12 relative;
    mixed and learned: 1e-6, the learned mode's HLLE choices within 1% of the
    faces).  Measured: bit for bit in FP64 and the learned mode, rounding-level
    differences in the mixed mode."""
    from kratos_b200.boxes import BoxBatch
    from kratos_b200 import selector as S
    w = S.init_params(5) if kw.get("riemann") == 2 else None
    ref = BoxBatch(5, 24, **kw)
    if w is not None:
        ref.set_selector(w, -1.0)
    ref.step(4)
    st_ref = ref.states()
    t_ref, dl_ref = ref.times()
    for grid in (None, 0, 1):
        bb = BoxBatch(5, 24, batched=True, **kw)
        assert bb.launches_per_step() == (20 if w is not None else 14)   # stage 0's update fused with c2p
        if grid is not None:
            g = bb.grid()
            bb.set_grid({k: (0 if grid == 0 else 148) for k in g})
        if w is not None:
            bb.set_selector(w, -1.0)
        bb.step(4)
        assert bb.status() == 0
        st = bb.states()
        t, dl = bb.times()
        tol = 1e-12 if kw["precision"] == 2 else 1e-6
        worst = max(rel_l1(st[b][0][..., 0], st_ref[b][0][..., 0]) for b in st_ref)
        exact = all(np.array_equal(st[b][0], st_ref[b][0]) and np.array_equal(st[b][1], st_ref[b][1])
                    for b in st_ref)
        print("batched vs per-group, %r grid %r: bit-identical %s, worst box rel L1 density %.2e, "
              "max |dt| rel %.2e" % (kw, grid, exact, worst, np.abs(dl / dl_ref - 1).max()))
        assert np.allclose(t, t_ref, rtol=tol, atol=0) and np.allclose(dl, dl_ref, rtol=tol, atol=0)
        assert worst <= tol
        for b in st_ref:
            assert rel_l1(st[b][1], st_ref[b][1]) <= tol, b
        if w is not None:
            f0, c0 = ref.selector_stats()
            f1, c1 = bb.selector_stats()
            assert f0 == f1 and abs(c1 - c0) <= 0.01 * f0
        bb.close()
    ref.close()


def test_batch_autotune_caches_and_keeps_state(tmp_path):
    """Autotuning times candidate grids on a copy of the state: the boxes'
    state and times are unchanged by it; the choice is appended to the cache
    file under the batch's key and read back by the next call."""
    from kratos_b200.boxes import BATCH_KINDS, BoxBatch
    cache = str(tmp_path / "tune.txt")
    bb = BoxBatch(5, 16, batched=True, precision=1)
    bb.step(2)
    before = bb.states()
    t0, _ = bb.times()
    grid, cached = bb.autotune(cache)
    assert not cached and set(grid) == set(BATCH_KINDS)
    after = bb.states()
    t1, _ = bb.times()
    assert np.array_equal(t0, t1)
    for b in before:
        assert np.array_equal(before[b][0], after[b][0])
    text = open(cache).read()
    assert text.count("kr_batch v2") == 1 and "prec1" in text
    grid2, cached2 = bb.autotune(cache)
    assert cached2 and grid2 == grid
    bb.step(2)
    assert bb.status() == 0
    bb.close()

"""Learned HLLE/HLLD face selector on the GPU.

* the hand-written FP32 training kernels' loss and gradient against the float64
  CPU restatement (oracle/kr_mlp_ref.py): relative error <= 1e-4;
* the BF16 tensor-core inference path against the same network with bf16
  roundings restated on the CPU;
* training on faces logged from the method's own runs separates safe from
  unsafe faces;
* the learned mixed step stays within 1e-4 relative L1 density of the FP64
  oracle with div B at roundoff, and its gain over the method without it: it
  sends a share of faces to HLLE (whole warps of 32 faces, each passed by the
  network) while its error stays far below the all-HLLE step's.
"""
import numpy as np
import pytest

from oracle import kr_mlp_ref as M

pytestmark = pytest.mark.gpu


def _data(n=3000, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 16)).astype(np.float32)
    y = (X[:, 0] * 0.7 - X[:, 3] + 0.2 * X[:, 9] ** 2 > 0.1).astype(np.float32)
    return X, y


def test_training_gradient_matches_cpu_oracle():
    from kratos_b200 import selector as S
    X, y = _data()
    w = S.init_params(3) * 1.0
    loss, g = S.grad(X, y, w, wneg=2.5)
    lo, go = M.loss_grad(X, y, w, wneg=2.5)
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    scale = np.abs(go).max()
    np.testing.assert_allclose(g, go, rtol=1e-3, atol=1e-4 * scale)
    assert np.abs(g - go).max() <= 1e-4 * scale


def test_bf16_inference_matches_restated_rounding():
    from kratos_b200 import selector as S
    X, y = _data(1000, 1)
    w, _ = S.train(X, y, epochs=5, batch=256, lr=3e-3, wneg=1.0)
    z = S.infer(X, w)
    zo = M.forward_bf16(X, w)
    zf, _ = M.forward(X, w)
    # bf16 roundings of inputs, weights and activations: agreement to ~1e-2
    assert np.abs(z - zo).max() <= 2e-2 * (1 + np.abs(zo).max())
    assert np.corrcoef(z, zf)[0, 1] > 0.999


def test_training_separates_synthetic_classes():
    from kratos_b200 import selector as S
    X, y = _data(20000, 2)
    w, loss = S.train(X, y, epochs=30, batch=1024, lr=3e-3, wneg=1.0)
    z = S.infer(X, w)
    acc = ((z > 0) == (y > 0.5)).mean()
    assert acc > 0.95, acc
    assert loss < 0.2


def _ot(nb=(2, 2, 2), n=(32, 32, 32), **kw):
    from kratos_b200 import Dynamics
    d = Dynamics(True, nb, n, gamma=5 / 3, **kw)
    d.init_problem("ot", 2)
    return d


def _trained_ot():
    from kratos_b200 import selector as S
    w, _ = S.build_selector([lambda: _ot(n=(16, 16, 16), precision=1)], steps=4, stride=4, tol=3e-4, epochs=25)
    return w


def test_learned_step_error_and_gain():
    from kratos_b200 import selector as S
    from oracle.kr_oracle import OracleMesh
    # training data: faces logged from the method's own mixed steps
    w, info = S.build_selector([lambda: _ot(n=(16, 16, 16), precision=1),
                                lambda: _ot(precision=1)], steps=4, stride=4, tol=3e-4, epochs=25)
    assert info["samples"] > 10000
    steps = 10
    o = OracleMesh(True, (2, 2, 2), (32, 32, 32), 5 / 3)
    o.init_problem("ot", 2)
    o.step(steps)
    ref, _ = o.get_state()

    def run(riemann, thr=None, **kw):
        d = _ot(precision=1, riemann=riemann, **kw)
        if thr is not None:
            d.set_selector(w, thr)
        d.step(steps)
        u, _ = d.get_state()
        div, _ = d.diagnostics()
        stats = d.selector_stats() if thr is not None else None
        e = np.abs(u[..., 0] - ref[..., 0]).sum() / np.abs(ref[..., 0]).sum()
        return e, div, stats

    e_hlld, _, _ = run(0)
    e_hlle, _, _ = run(1)
    # a warp's own faces go to HLLE only when all of them pass the logit
    # threshold, so the threshold sits below the per-face default; faces that
    # a neighbour block computes too follow their own logit
    thr = -3.0
    e_learn, div, (faces, cheap) = run(2, thr=thr)
    frac = cheap / faces
    print("rel L1 density: hlld %.2e  hlle %.2e  learned %.2e (HLLE on %.1f%% of faces)"
          % (e_hlld, e_hlle, e_learn, 100 * frac))
    assert e_learn <= 1e-4
    assert div <= 1e-12
    # the network must select: a share of the faces on HLLE, at well under
    # the all-HLLE step's error
    assert frac > 0.05, frac
    assert e_learn < 0.5 * e_hlle
    # choices kept for 4 steps between evaluations of the network
    e_p4, div4, (faces4, cheap4) = run(2, thr=thr, sel_period=4)
    print("sel_period 4: rel L1 density %.2e (HLLE on %.1f%% of faces)" % (e_p4, 100 * cheap4 / faces4))
    assert e_p4 <= 1e-4 and div4 <= 1e-12


def test_gradient_and_training_are_reproducible():
    """The gradient kernel writes one row of partial sums per CTA, added in a
    fixed order: the mean gradient and a training run give the same bits every
    time (float atomics would not)."""
    from kratos_b200 import selector as S
    X, y = _data(30000, seed=7)
    w0 = S.init_params(3)
    l1, g1 = S.grad(X, y, w0, wneg=4.0)
    l2, g2 = S.grad(X, y, w0, wneg=4.0)
    assert np.array_equal(g1, g2)
    wa, _ = S.train(X, y, w=w0, epochs=3, batch=4096)
    wb, _ = S.train(X, y, w=w0, epochs=3, batch=4096)
    assert np.array_equal(wa, wb)
    assert not np.array_equal(wa, w0)


def test_learned_step_on_turbulence():
    """The learned step on the decaying-turbulence workload (rms Mach 5,
    beta 0.1; 2^3 blocks of 16^3), with a network trained on the method's own
    turbulence steps: within 1e-4 relative L1 density of the FP64 oracle, div B
    at roundoff, and no less accurate than the all-HLLE step."""
    from kratos_b200 import Dynamics
    from kratos_b200 import selector as S
    from oracle.kr_oracle import OracleMesh

    def mk(**kw):
        d = Dynamics(True, (2, 2, 2), (16, 16, 16), gamma=5 / 3, **kw)
        d.init_problem("turb", 4)
        return d

    w, info = S.build_selector([lambda: mk(precision=1)], steps=4, stride=2, tol=3e-4, epochs=25)
    assert info["samples"] > 10000
    steps = 6
    o = OracleMesh(True, (2, 2, 2), (16, 16, 16), 5 / 3)
    o.init_problem("turb", 4)
    o.step(steps)
    ref, _ = o.get_state()

    def run(riemann, thr=None):
        d = mk(precision=1, riemann=riemann)
        if thr is not None:
            d.set_selector(w, thr)
        d.step(steps)
        u, _ = d.get_state()
        div, _ = d.diagnostics()
        assert d.status() == 0
        stats = d.selector_stats() if thr is not None else None
        return np.abs(u[..., 0] - ref[..., 0]).sum() / np.abs(ref[..., 0]).sum(), div, stats

    e_hlld, _, _ = run(0)
    e_hlle, _, _ = run(1)
    e_learn, div, (faces, cheap) = run(2, thr=S.DEFAULT_THRESHOLD)
    print("turbulence rel L1 density: hlld %.2e  hlle %.2e  learned %.2e (HLLE on %.1f%% of faces)"
          % (e_hlld, e_hlle, e_learn, 100 * cheap / faces))
    assert e_hlld <= 1e-4 and e_learn <= 1e-4
    assert div <= 1e-12
    assert e_learn <= e_hlle


def test_learned_step_conserves():
    """Periodic multi-block mesh: the learned step keeps mass, energy and
    momentum to rounding.  A face that two blocks compute (block sides, and the
    transverse ghost lines of the edge EMFs) must get the same solver in both,
    whatever the rest of its warp chose; totals summed on the host pairwise.
    64^3 blocks, so that warps away from the block sides can take HLLE."""
    from kratos_b200 import Dynamics
    w = _trained_ot()
    d = Dynamics(True, (2, 1, 1), (64, 64, 64), gamma=5 / 3, precision=1, riemann=2, sel_period=4)
    d.init_problem("ot", 2)
    d.set_selector(w, -3.0)

    def tot():
        u, _ = d.get_state()
        return np.array([np.ascontiguousarray(u[..., k]).sum() for k in range(5)])
    t0 = tot()
    d.step(12)
    t1 = tot()
    faces, cheap = d.selector_stats()
    print("learned conservation run: HLLE on %.1f%% of faces" % (100 * cheap / faces))
    assert cheap / faces > 0.05, "the network must send faces (shared ones included) to HLLE"
    assert d.status() == 0
    assert abs(t1[0] - t0[0]) <= 1e-12 * abs(t0[0])
    assert abs(t1[1] - t0[1]) <= 1e-12 * abs(t0[1])
    assert np.all(np.abs(t1[2:] - t0[2:]) <= 1e-12 * abs(t0[1]))

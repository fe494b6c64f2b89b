"""The allocation-free entry point kr_c2p_dt_noalloc, through the C ABI.

Some callers cannot allocate device memory (their host framework owns the memory
pool, or allocation is not allowed where they run).  kr_c2p_dt_noalloc serves
them: it converts one block's conserved state to primitives and reduces the CFL
dt using only a fixed scratch array inside the library.  The tests check, on two
calls in a row, that its dt equals the dt the regular engine (kr_ctx_create +
kr_step) computes for the same state and that its primitives match a plain
formula of that state; that with the pressure floor active (a state that the
floor heals in about half the cells) its primitives and dt match the oracle's
cons->prim; and that a warmed-up call changes neither torch's allocated bytes
nor the device's free memory.  The tests allocate their buffers with torch; the
entry point allocates nothing.  This file is collected last so a failure here
cannot hide other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _prims(u, gamma):
    rho = u[..., 0]
    v = u[..., 2:5] / rho[..., None]
    ek = 0.5 * (u[..., 2:5] ** 2).sum(-1) / rho
    em = 0.5 * (u[..., 5:8] ** 2).sum(-1) if u.shape[-1] == 8 else 0.0
    p = (u[..., 1] - ek - em) * (gamma - 1)
    return rho, p, v


@pytest.mark.parametrize("mhd", [True, False])
def test_noalloc_matches_engine_on_two_calls(mhd):
    import torch
    from kratos_b200 import Dynamics
    from kratos_b200 import _lib as L
    n = (32, 24, 16)
    gamma = 5.0 / 3.0 if mhd else 1.4
    name = "ot" if mhd else "shock"
    d = Dynamics(mhd, (1, 1, 1), n, gamma=gamma)
    d.init_problem(name, 5)
    u_aos, bf_aos = d.get_state()                    # [1, n2, n1, n0, nw], [1, ..., 3]
    d.step(1)                                         # first step: dt = CFL minimum
    dt_engine = d.time()["dt_last"]
    cfg = d.cfg
    dev = torch.device("cuda:0")
    u_soa = torch.from_numpy(np.ascontiguousarray(np.moveaxis(u_aos[0, ..., :5], -1, 0))).to(dev)
    bf_soa = (torch.from_numpy(np.ascontiguousarray(np.moveaxis(bf_aos[0], -1, 0))).to(dev)
              if mhd else None)
    nw = 8 if mhd else 5
    w = torch.zeros((nw, n[2] + 4, n[1] + 4, n[0] + 4), dtype=torch.float64, device=dev)
    dt = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    lib = L.lib()
    for call in range(2):
        w.zero_()
        dt.fill_(-1.0)
        rc = lib.kr_c2p_dt_noalloc(ctypes.byref(cfg), ctypes.c_void_p(u_soa.data_ptr()),
                                   ctypes.c_void_p(bf_soa.data_ptr() if mhd else 0),
                                   ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(dt.data_ptr()),
                                   ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.kr_last_error(None)
        torch.cuda.synchronize()
        assert float(dt.item()) == pytest.approx(dt_engine, rel=1e-13, abs=0), call
        wi = w[:, 2:-2, 2:-2, 2:-2].cpu().numpy()
        rho, p, v = _prims(u_aos[0], gamma)
        np.testing.assert_allclose(wi[0], rho, rtol=1e-13, atol=0)
        np.testing.assert_allclose(wi[1], p, rtol=1e-11, atol=1e-14)
        for a in range(3):
            np.testing.assert_allclose(wi[2 + a], v[..., a], rtol=1e-12, atol=1e-15)
        if mhd:
            np.testing.assert_allclose(wi[5:8], np.moveaxis(u_aos[0, ..., 5:8], -1, 0), rtol=0, atol=0)


def test_noalloc_rejects_oversized_block():
    from kratos_b200 import _lib as L
    lib = L.lib()
    cfg = L.kr_cfg()
    lib.kr_cfg_default(ctypes.byref(cfg))
    cfg.n[0] = cfg.n[1] = cfg.n[2] = 256                # 16.7 M cells > 4,194,304
    rc = lib.kr_c2p_dt_noalloc(ctypes.byref(cfg), ctypes.c_void_p(8), None,
                               ctypes.c_void_p(8), ctypes.c_void_p(8), None)
    assert rc == -2
    assert b"exceeds the scratch limit" in lib.kr_last_error(None)


def _noalloc(lib, cfg, u_soa, bf_soa, w, dt, stream):
    return lib.kr_c2p_dt_noalloc(ctypes.byref(cfg), ctypes.c_void_p(u_soa.data_ptr()),
                                 ctypes.c_void_p(bf_soa.data_ptr() if bf_soa is not None else 0),
                                 ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(dt.data_ptr()),
                                 ctypes.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("mhd", [True, False])
def test_noalloc_floors_match_oracle(mhd):
    """Density and pressure floors: the primitives and dt agree with the
    oracle's cons->prim (floors applied to w) to rounding; u is left as given."""
    import torch
    from kratos_b200 import _lib as L
    from kratos_b200.engine import make_cfg
    from oracle.kr_oracle import OracleMesh
    n = (16, 8, 8)
    gamma = 5.0 / 3.0 if mhd else 1.4
    name = "ot" if mhd else "shock"
    # tmp_floor = 1 (as the shock_floor fixture): p < rho on part of the mesh
    o = OracleMesh(mhd, (1, 1, 1), n, gamma, d_floor=1e-9, t_floor=1.0)
    o.init_problem(name, 4)
    u0, bf0 = o.get_state()
    rng = np.random.default_rng(7)
    u0[0, ..., 0][rng.random(u0.shape[1:4]) < 0.05] = 1e-12       # density below the floor too
    o.set_state(u0, bf0)
    w_ref, dt_ref = o.c2p_dt()
    cfg = make_cfg(mhd, (1, 1, 1), n, gamma=gamma, rho_floor=1e-9, tmp_floor=1.0)
    dev = torch.device("cuda:0")
    u_soa = torch.from_numpy(np.ascontiguousarray(np.moveaxis(u0[0, ..., :5], -1, 0))).to(dev)
    bf_soa = torch.from_numpy(np.ascontiguousarray(np.moveaxis(bf0[0], -1, 0))).to(dev) if mhd else None
    u_before = u_soa.clone()
    nw = 8 if mhd else 5
    w = torch.zeros((nw, n[2] + 4, n[1] + 4, n[0] + 4), dtype=torch.float64, device=dev)
    dt = torch.zeros(1, dtype=torch.float64, device=dev)
    lib = L.lib()
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        w.zero_()
        assert _noalloc(lib, cfg, u_soa, bf_soa, w, dt, stream) == 0, lib.kr_last_error(None)
        torch.cuda.synchronize()
        wi = np.moveaxis(w[:, 2:-2, 2:-2, 2:-2].cpu().numpy(), 0, -1)
        healed = w_ref[0, ..., 1] <= 1.0 * w_ref[0, ..., 0] * (1 + 1e-15)
        assert healed.mean() > 0.2, "the floor must be active in this case"
        np.testing.assert_allclose(wi, w_ref[0], rtol=1e-12, atol=1e-14)
        assert float(dt.item()) == pytest.approx(float(dt_ref[0]), rel=1e-13, abs=0), call
    assert torch.equal(u_soa, u_before), "u is read only"


def test_noalloc_allocates_nothing():
    """After a first (set-up) call, further calls leave torch's allocated bytes
    and the device's free memory unchanged."""
    import torch
    from kratos_b200 import Dynamics
    from kratos_b200 import _lib as L
    n = (32, 32, 32)
    d = Dynamics(True, (1, 1, 1), n, gamma=5.0 / 3.0)
    d.init_problem("ot", 3)
    u_aos, bf_aos = d.get_state()
    dev = torch.device("cuda:0")
    u_soa = torch.from_numpy(np.ascontiguousarray(np.moveaxis(u_aos[0, ..., :5], -1, 0))).to(dev)
    bf_soa = torch.from_numpy(np.ascontiguousarray(np.moveaxis(bf_aos[0], -1, 0))).to(dev)
    w = torch.zeros((8, n[2] + 4, n[1] + 4, n[0] + 4), dtype=torch.float64, device=dev)
    dt = torch.zeros(1, dtype=torch.float64, device=dev)
    lib = L.lib()
    stream = torch.cuda.current_stream(dev)
    assert _noalloc(lib, d.cfg, u_soa, bf_soa, w, dt, stream) == 0
    torch.cuda.synchronize()
    alloc0, free0 = torch.cuda.memory_allocated(dev), torch.cuda.mem_get_info(dev)[0]
    for _ in range(5):
        assert _noalloc(lib, d.cfg, u_soa, bf_soa, w, dt, stream) == 0
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated(dev) == alloc0
    assert torch.cuda.mem_get_info(dev)[0] == free0

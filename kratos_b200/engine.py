"""Python handle on the device engine (tests, bench and scripting).

A `Dynamics` object owns one kr_ctx: the device state of a uniform block mesh
and the captured step.  Arrays exchanged with it use the reference's per-block
layouts in lexicographic block order (see include/kratos_b200.h).
"""
import ctypes

import numpy as np

from . import _lib as L

FLT_MAX = float(np.finfo(np.float32).max)


class KratosError(RuntimeError):
    pass


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def make_cfg(mhd, nb, n, gamma=1.66667, cfl=0.3, precision=2, riemann=0,
             x_min=(0, 0, 0), x_max=(1, 1, 1), rho_floor=1e-9, tmp_floor=1e-9,
             dt_init=0.0, dt_expand=2.0, device=0, flags=0,
             kinds=("per",) * 6, w_fix=(0, 0, 0, 0, 0), b_fix=(0, 0, 0), n_ranks=1, rank=0,
             sel_period=1, integrator=0):
    """A kr_cfg (include/kratos_b200.h) from keyword arguments."""
    lib = L.lib()
    c = L.kr_cfg()
    lib.kr_cfg_default(ctypes.byref(c))
    c.mhd, c.precision, c.riemann = int(mhd), int(precision), int(riemann)
    for a in range(3):
        c.nb[a], c.n[a] = int(nb[a]), int(n[a])
        c.x_min[a], c.x_max[a] = float(x_min[a]), float(x_max[a])
    c.gamma, c.cfl = float(gamma), float(cfl)
    c.rho_floor, c.tmp_floor = float(rho_floor), float(tmp_floor)
    c.dt_init, c.dt_expand, c.device = float(dt_init), float(dt_expand), int(device)
    c.flags = int(flags)              # KR_FLAG_HALO_ALL, KR_FLAG_BOXES
    c.n_ranks, c.rank = int(n_ranks), int(rank)
    c.sel_period = int(sel_period)
    c.integrator = int(integrator)    # KR_INTEGRATOR_RK2 (the reference's), KR_INTEGRATOR_VL2
    for k in range(6):
        c.bc[k] = L.BC_KINDS[kinds[k]]
    for k in range(5):
        c.w_fix[k] = float(w_fix[k])
    for k in range(3):
        c.b_fix[k] = float(b_fix[k])
    return c


def shard_owner(cfg):
    """Owner rank of every global block, and the number of cfg.rank's blocks."""
    nglob = cfg.nb[0] * cfg.nb[1] * cfg.nb[2]
    owner = np.empty(nglob, np.int32)
    k = L.lib().kr_shard_owner(ctypes.byref(cfg), _ptr(owner))
    if k < 0:
        raise KratosError(L.lib().kr_last_error(None).decode())
    return owner, k


def halo_counts(cfg):
    """Per-stage halo words of cfg.rank with every peer: (send, recv), each
    [n_ranks, 2] = (primitive words, face-B words)."""
    r = max(1, cfg.n_ranks)
    snd, rcv = np.zeros((r, 2), np.int64), np.zeros((r, 2), np.int64)
    if L.lib().kr_halo_counts(ctypes.byref(cfg), _ptr(snd), _ptr(rcv)) != 0:
        raise KratosError(L.lib().kr_last_error(None).decode())
    return snd, rcv


def _nccl_host():
    """Point the engine at the libnccl.so.2 that torch links (the nvidia-nccl
    wheel), without importing torch: a process holds one NCCL, and torch
    needs its own version's symbols when it is imported later."""
    import importlib.util
    import os
    if os.environ.get("KRATOS_B200_NCCL"):
        return
    try:
        spec = importlib.util.find_spec("nvidia.nccl")
    except (ImportError, ValueError):
        spec = None
    for d in (spec.submodule_search_locations if spec else []) or []:
        cand = os.path.join(d, "lib", "libnccl.so.2")
        if os.path.exists(cand):
            os.environ["KRATOS_B200_NCCL"] = cand
            return


def comm_unique_id():
    """128-byte NCCL unique id (ncclGetUniqueId), to be shared with every rank."""
    _nccl_host()
    buf = (ctypes.c_ubyte * 128)()
    if L.lib().kr_comm_unique_id(buf) != 0:
        raise KratosError(L.lib().kr_last_error(None).decode())
    return bytes(buf)


def group_step(dyns, n_steps=1):
    """Step the n_ranks shard contexts of one mesh together from this process
    (one device; the exchange is device copies, synchronous)."""
    arr = (ctypes.c_void_p * len(dyns))(*[d._h for d in dyns])
    if L.lib().kr_group_step(arr, len(dyns), int(n_steps)) != 0:
        raise KratosError(L.lib().kr_last_error(None).decode())


class Dynamics:
    """One engine context.  With n_ranks > 1 it holds rank `rank`'s share of
    the nb[0] x nb[1] x nb[2] blocks (`gid`, ascending global ids) and needs a
    communicator (`comm_init`) or `group_step` to advance.  `regions`, a list of
    (level, x_min, x_max) as [refine_region*] sections give them, makes a
    statically refined hydro mesh: its blocks are the tree's leaves, level by
    level (`level`, `reg`: each block's level and logical position)."""

    def __init__(self, mhd, nb, n, regions=(), **kw):
        lib = L.lib()
        c = make_cfg(mhd, nb, n, **kw)
        self.cfg = c
        if regions:
            rg = (L.kr_region * len(regions))()
            for k, (lvl, lo, hi) in enumerate(regions):
                rg[k].level = int(lvl)
                for a in range(3):
                    rg[k].x_min[a], rg[k].x_max[a] = float(lo[a]), float(hi[a])
            self._h = lib.kr_ctx_create_refined(ctypes.byref(c), len(regions), rg)
        else:
            self._h = lib.kr_ctx_create(ctypes.byref(c))
        if not self._h:
            raise KratosError(lib.kr_last_error(None).decode())
        self.mhd = bool(mhd)
        self.nb, self.n = tuple(int(x) for x in nb), tuple(int(x) for x in n)
        self.nblk = lib.kr_shard_blocks(self._h, None)
        gid = np.empty(self.nblk, np.int32)
        lib.kr_shard_blocks(self._h, _ptr(gid))
        self.gid = gid
        self.level = np.empty(self.nblk, np.int32)
        self.reg = np.empty((self.nblk, 3), np.int32)
        lib.kr_block_info(self._h, _ptr(self.level), _ptr(self.reg))
        self.nw = 8 if mhd else 5

    def comm_init(self, uid):
        _nccl_host()
        buf = (ctypes.c_ubyte * 128).from_buffer_copy(uid)
        self._check(L.lib().kr_comm_init(self._h, buf), "kr_comm_init")

    # ------------------------------------------------------------------ admin
    def close(self):
        if getattr(self, "_h", None):
            L.lib().kr_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _check(self, rc, what):
        if rc != 0:
            raise KratosError("%s: %s" % (what, L.lib().kr_last_error(self._h).decode()))

    @property
    def u_shape(self):
        n = self.n
        return (self.nblk, n[2], n[1], n[0], self.nw)

    @property
    def bf_shape(self):
        n = self.n
        return (self.nblk, n[2] + 5, n[1] + 5, n[0] + 5, 3)

    @property
    def n_cells(self):
        return self.nblk * self.n[0] * self.n[1] * self.n[2]

    # ------------------------------------------------------------------ state
    def set_stream(self, stream_handle):
        self._check(L.lib().kr_set_stream(self._h, ctypes.c_void_p(stream_handle)), "kr_set_stream")

    def init_problem(self, name, seed):
        self._check(L.lib().kr_init_problem(self._h, name.encode(), int(seed)), "kr_init_problem")

    def init_boxes(self, seed, box_ids):
        """Block b becomes box box_ids[b] of the seeded batch (a context made
        with flags=KR_FLAG_BOXES, or a periodic one-block MHD mesh)."""
        ids = np.ascontiguousarray(box_ids, dtype=np.int32).reshape(self.nblk)
        self._check(L.lib().kr_init_boxes(self._h, int(seed), _ptr(ids)), "kr_init_boxes")

    def init_box(self, seed, box):
        """One box on a periodic one-block MHD mesh."""
        self.init_boxes(seed, [box])

    def box_times(self):
        """Per block: time, last dt and steps (independent boxes: each its own)."""
        t, dl = np.empty(self.nblk), np.empty(self.nblk)
        ns = np.empty(self.nblk, np.int64)
        self._check(L.lib().kr_box_times(self._h, _ptr(t), _ptr(dl), _ptr(ns)), "kr_box_times")
        return t, dl, ns

    def set_state(self, u, bf=None):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.u_shape)
        if self.mhd:
            bf = np.ascontiguousarray(bf, dtype=np.float64).reshape(self.bf_shape)
        self._check(L.lib().kr_set_state(self._h, _ptr(u), _ptr(bf) if self.mhd else None),
                    "kr_set_state")

    def get_state(self, u=None, bf=None):
        u = np.empty(self.u_shape) if u is None else u
        if self.mhd:
            bf = np.empty(self.bf_shape) if bf is None else bf
        self._check(L.lib().kr_get_state(self._h, _ptr(u), _ptr(bf) if self.mhd else None),
                    "kr_get_state")
        return u, (bf if self.mhd else None)

    def state_bytes(self):
        b = self.nblk * self.n[0] * self.n[1] * self.n[2] * self.nw * 8
        if self.mhd:
            b += self.nblk * (self.n[0] + 5) * (self.n[1] + 5) * (self.n[2] + 5) * 3 * 8
        return b

    # ------------------------------------------------------------------- time
    def step(self, n_steps=1):
        self._check(L.lib().kr_step(self._h, int(n_steps)), "kr_step")

    def time(self):
        t, dl, db = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        ns = ctypes.c_longlong()
        self._check(L.lib().kr_get_time(self._h, ctypes.byref(t), ctypes.byref(dl),
                                        ctypes.byref(db), ctypes.byref(ns)), "kr_get_time")
        return {"t": t.value, "dt_last": dl.value, "dt_bound": db.value, "n_steps": ns.value}

    def set_time(self, t, dt_bound):
        self._check(L.lib().kr_set_time(self._h, float(t), float(dt_bound)), "kr_set_time")

    def status(self):
        s = L.lib().kr_status(self._h)
        if s < 0:
            raise KratosError("kr_status: " + L.lib().kr_last_error(self._h).decode())
        return s

    def launches_per_step(self):
        return L.lib().kr_launches_per_step(self._h)

    KERNEL_KINDS = ("c2p", "ghost", "flux_z", "flux_y", "flux_x", "emf", "update")

    def profile_step(self):
        """One eager step with CUDA events per kernel: {kind: ms}."""
        ms = (ctypes.c_double * 7)()
        self._check(L.lib().kr_profile_step(self._h, 7, ms), "kr_profile_step")
        return dict(zip(self.KERNEL_KINDS, ms[:]))

    def set_selector(self, params, threshold=0.0):
        import numpy as _np
        w = _np.ascontiguousarray(params, _np.float32)
        self._check(L.lib().kr_set_selector(self._h, ctypes.c_void_p(w.ctypes.data), float(threshold)),
                    "kr_set_selector")

    def selector_stats(self, reset=False):
        f, c = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(L.lib().kr_selector_stats(self._h, ctypes.byref(f), ctypes.byref(c), int(reset)),
                    "kr_selector_stats")
        return f.value, c.value

    def diagnostics(self):
        dv = ctypes.c_double()
        tot = (ctypes.c_double * 5)()
        self._check(L.lib().kr_diagnostics(self._h, ctypes.byref(dv), tot), "kr_diagnostics")
        return dv.value, np.array(tot[:])

"""ctypes front end of the CPU restatement of the step (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker; the product never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# "" : the restatement as the reference's CPU build computes it (no fused
#      multiply-add); "fma": the same source with fused multiply-add, to
#      measure how far rounding alone moves a case
_LIB_PATHS = {"": os.path.join(_HERE, "ref_cpu", "libkr_oracle.so"),
              "fma": os.path.join(_HERE, "ref_cpu", "libkr_oracle_fma.so")}


class _Cfg(ctypes.Structure):
    _fields_ = [
        ("mhd", ctypes.c_int),
        ("nb", ctypes.c_int * 3),
        ("n", ctypes.c_int * 3),
        ("x_min", ctypes.c_double * 3),
        ("x_max", ctypes.c_double * 3),
        ("gamma", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("d_floor", ctypes.c_double),
        ("t_floor", ctypes.c_double),
        ("dt_expand", ctypes.c_double),
        ("n_threads", ctypes.c_int),
        ("bc", ctypes.c_int * 6),
        ("w_fix", ctypes.c_double * 5),
        ("b_fix", ctypes.c_double * 3),
        ("integrator", ctypes.c_int),
    ]


class _Region(ctypes.Structure):
    _fields_ = [
        ("level", ctypes.c_int),
        ("x_min", ctypes.c_double * 3),
        ("x_max", ctypes.c_double * 3),
    ]


BC_KINDS = {"per": 0, "out": 1, "ref": 2, "fre": 3, "fixd": 4}


_libs = {}


def build():
    subprocess.check_call(["make", "-s", "-f", os.path.join(_HERE, "Makefile")])


def lib(variant=""):
    if variant not in _libs:
        path = _LIB_PATHS[variant]
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        L.kro_create.restype = ctypes.c_void_p
        L.kro_create.argtypes = [ctypes.POINTER(_Cfg)]
        L.kro_create_tree.restype = ctypes.c_void_p
        L.kro_create_tree.argtypes = [ctypes.POINTER(_Cfg), ctypes.c_int, ctypes.POINTER(_Region)]
        L.kro_nblk.restype = ctypes.c_int
        L.kro_nblk.argtypes = [ctypes.c_void_p]
        ip = ctypes.POINTER(ctypes.c_int)
        L.kro_block_info.argtypes = [ctypes.c_void_p, ip, ip]
        L.kro_destroy.argtypes = [ctypes.c_void_p]
        L.kro_set_state.argtypes = [ctypes.c_void_p, dp, dp]
        L.kro_get_state.argtypes = [ctypes.c_void_p, dp, dp]
        L.kro_c2p_dt.argtypes = [ctypes.c_void_p, dp, dp]
        L.kro_step.restype = ctypes.c_int
        L.kro_step.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, dp, dp]
        for f in ("kro_x_cc", "kro_x_fc"):
            getattr(L, f).restype = ctypes.c_double
            getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.kro_dx.restype = ctypes.c_double
        L.kro_dx.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.kro_hllc.argtypes = [dp, dp, ctypes.c_int, ctypes.c_double, dp]
        L.kro_hlld.argtypes = [dp, dp, ctypes.c_int, ctypes.c_double, dp]
        L.kro_plm.argtypes = [dp, dp, dp]
        L.kro_init_problem.restype = ctypes.c_int
        L.kro_init_problem.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_ulonglong]
        L.kro_init_box.restype = ctypes.c_int
        L.kro_init_box.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_int]
        L.kro_box_n.restype = ctypes.c_int
        L.kro_box_n.argtypes = [ctypes.c_ulonglong, ctypes.c_int]
        _libs[variant] = L
    return _libs[variant]


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


FLT_MAX = float(np.finfo(np.float32).max)


class OracleMesh:
    """Mesh of nb root blocks of n cells, state in block order: level by level,
    lexicographic (x fastest) inside a level (a uniform mesh is one level).
    u: [nblk, n2, n1, n0, nw]; bf: [nblk, n2+5, n1+5, n0+5, 3] (face lattice
    with 2 ghost layers).  `regions`: static refinement, a list of
    (level, x_min, x_max) as the [refine_region*] sections give them."""

    def __init__(self, mhd, nb, n, gamma, cfl=0.3, x_min=(0, 0, 0), x_max=(1, 1, 1),
                 d_floor=1e-9, t_floor=1e-9, dt_expand=2.0, dt_init=0.0, n_threads=0,
                 kinds=("per",) * 6, w_fix=(0, 0, 0, 0, 0), b_fix=(0, 0, 0), regions=(), variant="",
                 integrator=0):
        c = _Cfg()
        c.mhd = int(mhd)
        for a in range(3):
            c.nb[a], c.n[a] = int(nb[a]), int(n[a])
            c.x_min[a], c.x_max[a] = float(x_min[a]), float(x_max[a])
        c.gamma, c.cfl, c.d_floor, c.t_floor = float(gamma), float(cfl), float(d_floor), float(t_floor)
        c.dt_expand, c.n_threads = float(dt_expand), int(n_threads)
        c.integrator = int(integrator)            # 0 Heun RK2, 1 VL2
        for k in range(6):
            c.bc[k] = BC_KINDS[kinds[k]]
        for k in range(5):
            c.w_fix[k] = float(w_fix[k])
        for k in range(3):
            c.b_fix[k] = float(b_fix[k])
        self.cfg = c
        self.mhd = bool(mhd)
        self.nb, self.n = tuple(nb), tuple(n)
        self.nw = 8 if mhd else 5
        rg = (_Region * max(1, len(regions)))()
        for k, (lvl, lo, hi) in enumerate(regions):
            rg[k].level = int(lvl)
            for a in range(3):
                rg[k].x_min[a], rg[k].x_max[a] = float(lo[a]), float(hi[a])
        self._L = lib(variant)
        self._h = self._L.kro_create_tree(ctypes.byref(c), len(regions), rg)
        if not self._h:
            raise ValueError("oracle: kro_create_tree failed")
        self.nblk = self._L.kro_nblk(self._h)
        self.level = np.zeros(self.nblk, dtype=np.int32)
        self.reg = np.zeros((self.nblk, 3), dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        self._L.kro_block_info(self._h, self.level.ctypes.data_as(ip), self.reg.ctypes.data_as(ip))
        self.t = 0.0
        # cycle.cpp:163-166: an unset dt_init starts the device dt at FLT_MAX / 10
        self.dt_bound = dt_init if dt_init >= np.finfo(np.float32).tiny else FLT_MAX / 10
        self.dt_last = 0.0

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.kro_destroy(self._h)
            self._h = None

    @property
    def u_shape(self):
        n = self.n
        return (self.nblk, n[2], n[1], n[0], self.nw)

    @property
    def bf_shape(self):
        n = self.n
        return (self.nblk, n[2] + 5, n[1] + 5, n[0] + 5, 3)

    def set_state(self, u, bf=None):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.u_shape)
        if self.mhd:
            bf = np.ascontiguousarray(bf, dtype=np.float64).reshape(self.bf_shape)
            self._L.kro_set_state(self._h, _p(u), _p(bf))
        else:
            self._L.kro_set_state(self._h, _p(u), None)

    def get_state(self):
        u = np.empty(self.u_shape)
        if self.mhd:
            bf = np.empty(self.bf_shape)
            self._L.kro_get_state(self._h, _p(u), _p(bf))
            return u, bf
        self._L.kro_get_state(self._h, _p(u), None)
        return u, None

    def step(self, n_steps=1):
        t = ctypes.c_double(self.t)
        db = ctypes.c_double(self.dt_bound)
        dl = ctypes.c_double(0.0)
        rc = self._L.kro_step(self._h, int(n_steps), ctypes.byref(t), ctypes.byref(db), ctypes.byref(dl))
        if rc == -2:
            raise NotImplementedError("oracle: a refined MHD mesh steps on periodic domains only")
        if rc != 0:
            raise FloatingPointError("oracle step produced a non-finite dt")
        self.t, self.dt_bound, self.dt_last = t.value, db.value, dl.value

    def c2p_dt(self):
        """cons -> prim (floors applied, healing the conserved state) and each
        block's CFL dt of the current state, without stepping
        (hydro/eos/adiabatic.h:159-258, mhd/eos/adiabatic.h:84-234).
        Returns (w [nblk, n2, n1, n0, nw], dt [nblk])."""
        w = np.empty(self.u_shape)
        dt = np.empty(self.nblk)
        self._L.kro_c2p_dt(self._h, _p(w), _p(dt))
        return w, dt

    def init_problem(self, name, seed):
        if self._L.kro_init_problem(self._h, name.encode(), int(seed)) != 0:
            raise ValueError("unknown problem %r for this mesh" % name)

    def init_box(self, seed, box):
        """Box `box` of a batch of independent periodic MHD boxes."""
        if self._L.kro_init_box(self._h, int(seed), int(box)) != 0:
            raise ValueError("box workloads need an MHD mesh")

    def x_cc(self, block, axis, i):
        return self._L.kro_x_cc(self._h, block, axis, i)

    def dx(self, block, axis):
        return self._L.kro_dx(self._h, block, axis)


def hllc(ql, qr, axis, gamma):
    ql = np.ascontiguousarray(ql, dtype=np.float64)
    qr = np.ascontiguousarray(qr, dtype=np.float64)
    f = np.empty(5)
    lib().kro_hllc(_p(ql), _p(qr), int(axis), float(gamma), _p(f))
    return f


def hlld(ql, qr, axis, gamma):
    ql = np.ascontiguousarray(ql, dtype=np.float64)
    qr = np.ascontiguousarray(qr, dtype=np.float64)
    f = np.empty(8)
    lib().kro_hlld(_p(ql), _p(qr), int(axis), float(gamma), _p(f))
    return f


def box_n(seed, box):
    """Edge length in cells of box `box` of a batch (problems.h kr_box_params)."""
    return lib().kro_box_n(int(seed), int(box))

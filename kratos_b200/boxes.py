"""Batched independent periodic MHD boxes: a seeded batch of boxes with edge
lengths from {16, 24, 32, 48, 64} cells, random density, pressure, velocity
amplitude, field orientation and plasma beta (kratos_b200/csrc/problems.h
kr_box_params), each advancing on its own CFL dt.

The original Kratos solver runs each box as its own one-block periodic mesh
(one process per box).  Here the boxes of one edge length are the blocks of one
context made with KR_FLAG_BOXES: every block is periodic onto itself and keeps
its own dt and time, so one captured graph steps all boxes of that size, and
the contexts of the five sizes run on their own streams.  A box advanced here
matches the same box run alone (tests/test_gpu_boxes.py).
"""
import ctypes

import numpy as np

from . import _lib as L
from .engine import Dynamics, KratosError


# launch kinds of the batched step, in kr_batch_get_grid's order
BATCH_KINDS = ("c2p0", "c2p1", "flux", "eval", "emf", "upd1", "upd2", "updc2p")


def box_params(seed, box, gamma=5 / 3):
    """Parameters of box `box` of the batch `seed`."""
    out = (ctypes.c_double * 8)()
    if L.lib().kr_box_params(int(seed), int(box), float(gamma), out) != 0:
        raise KratosError("kr_box_params: bad box index %r" % (box,))
    return {"n": int(out[0]), "rho": out[1], "pre": out[2], "amp": out[3], "beta": out[4],
            "b": (out[5], out[6], out[7])}


class BoxBatch:
    """Boxes 0..n_boxes-1 of the batch `seed`, grouped by edge length.

    Keyword arguments go to each group's Dynamics (precision, riemann, cfl,
    device, ...).  `groups` maps an edge length to (Dynamics, box indices in
    block order).  batched=True steps all groups through one kr_batch: one
    launch per kernel kind over every box (a work list of the groups' CTA
    tiles), one CUDA graph per step on the first group's stream."""

    def __init__(self, seed, n_boxes, gamma=5 / 3, batched=False, **kw):
        if n_boxes < 1:
            raise ValueError("need at least one box")
        self.seed, self.n_boxes, self.gamma = int(seed), int(n_boxes), float(gamma)
        sizes = np.array([box_params(seed, b, gamma)["n"] for b in range(n_boxes)])
        self.sizes = sizes
        self.groups = {}
        self.where = {}
        flags = kw.pop("flags", 0) | L.KR_FLAG_BOXES
        try:
            for n in sorted(set(sizes.tolist())):
                ids = np.flatnonzero(sizes == n).astype(np.int32)
                d = Dynamics(True, (len(ids), 1, 1), (n, n, n), gamma=gamma, flags=flags, **kw)
                self.groups[n] = (d, ids)
                for k, b in enumerate(ids):
                    self.where[int(b)] = (n, k)
                d.init_boxes(seed, ids)
            self._batch = None
            if batched:
                hs = (ctypes.c_void_p * len(self.groups))(*[d._h for d, _ in self.groups.values()])
                self._batch = L.lib().kr_batch_create(hs, len(self.groups))
                if not self._batch:
                    raise KratosError(L.lib().kr_batch_last_error(None).decode())
        except Exception:
            self.close()
            raise

    @property
    def n_cells(self):
        return int(sum(int(n) ** 3 for n in self.sizes))

    def _bcheck(self, rc, what):
        if rc < 0:
            raise KratosError("%s: %s" % (what, L.lib().kr_batch_last_error(self._batch).decode()))
        return rc

    def step(self, n_steps=1):
        """Advance every box n_steps of its own dt (enqueued on each group's
        stream, or on the first group's with batched=True; get_state / times
        wait for them)."""
        if self._batch:
            self._bcheck(L.lib().kr_batch_step(self._batch, int(n_steps)), "kr_batch_step")
            return
        for d, _ in self.groups.values():
            d.step(n_steps)

    @property
    def stream_groups(self):
        """The groups whose streams carry the work: all of them, or the first
        with batched=True."""
        g = list(self.groups.values())
        return g[:1] if self._batch else g

    def launches_per_step(self):
        if self._batch:
            return L.lib().kr_batch_launches_per_step(self._batch)
        return sum(d.launches_per_step() for d, _ in self.groups.values())

    def grid(self):
        """CTAs of each launch kind of the batched step (0: one per work item)."""
        g = (ctypes.c_int * len(BATCH_KINDS))()
        self._bcheck(L.lib().kr_batch_get_grid(self._batch, g), "kr_batch_get_grid")
        return dict(zip(BATCH_KINDS, list(g)))

    def set_grid(self, grid):
        g = (ctypes.c_int * len(BATCH_KINDS))(*[int(grid[k]) for k in BATCH_KINDS])
        self._bcheck(L.lib().kr_batch_set_grid(self._batch, g), "kr_batch_set_grid")

    def profile_step(self):
        """One step eagerly with CUDA events around every launch: milliseconds
        per launch kind (batched), or per group and kind (kr_profile_step)."""
        if self._batch:
            ms = (ctypes.c_double * len(BATCH_KINDS))()
            self._bcheck(L.lib().kr_batch_profile_step(self._batch, len(BATCH_KINDS), ms), "kr_batch_profile_step")
            return dict(zip(BATCH_KINDS, list(ms)))
        return {n: d.profile_step() for n, (d, _) in self.groups.items()}

    def autotune(self, cache_path=None):
        """Pick each launch kind's CTA count by timing (kr_batch_autotune), or
        reuse the choice cached in `cache_path` for this device and batch.
        Returns (grid, cached)."""
        g = (ctypes.c_int * len(BATCH_KINDS))()
        rc = self._bcheck(L.lib().kr_batch_autotune(self._batch, cache_path.encode() if cache_path else None, g),
                          "kr_batch_autotune")
        return dict(zip(BATCH_KINDS, list(g))), rc == 1

    def set_selector(self, params, threshold):
        """Learned mode (riemann = KR_RIEMANN_LEARNED): the same network and
        threshold for every size group."""
        for d, _ in self.groups.values():
            d.set_selector(params, threshold)

    def selector_stats(self, reset=False):
        """Faces evaluated and faces given HLLE, summed over the groups."""
        f = c = 0
        for d, _ in self.groups.values():
            a, b = d.selector_stats(reset)
            f, c = f + a, c + b
        return f, c

    def status(self):
        return max(d.status() for d, _ in self.groups.values())

    def times(self):
        """Per box (index order): time, last dt."""
        t, dl = np.empty(self.n_boxes), np.empty(self.n_boxes)
        for d, ids in self.groups.values():
            tg, dg, _ = d.box_times()
            t[ids], dl[ids] = tg, dg
        return t, dl

    def get_state(self, box):
        """(u, bf) of one box, in the layout of a one-block mesh."""
        n, k = self.where[int(box)]
        d = self.groups[n][0]
        u, bf = d.get_state()
        return u[k:k + 1], bf[k:k + 1]

    def states(self):
        """{box: (u, bf)} of every box (one download per group)."""
        out = {}
        for d, ids in self.groups.values():
            u, bf = d.get_state()
            for k, b in enumerate(ids):
                out[int(b)] = (u[k:k + 1], bf[k:k + 1])
        return out

    def close(self):
        if getattr(self, "_batch", None):
            L.lib().kr_batch_destroy(self._batch)
            self._batch = None
        for d, _ in self.groups.values():
            d.close()
        self.groups = {}

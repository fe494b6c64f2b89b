"""Learned HLLE/HLLD face selector: sample collection, GPU training, install.

The network and its training kernels live in the engine (kr_learn.cu); this
module only moves arrays across the C ABI:

    X, gap = collect(dyn, steps, stride)     # faces logged from ordinary steps
    y = (gap < tol).astype(float32)          # 1 = HLLE within tolerance
    w = train(X, y)                           # Adam on the GPU, project kernels
    dyn.set_selector(w, threshold)            # used when riemann = LEARNED
"""
import ctypes

import numpy as np

from . import _lib as L

N_IN = 16
N_PARAM = 16 * 32 + 32 + 32 * 32 + 32 + 32 + 1


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _err():
    return L.lib().kr_learn_last_error().decode()


def init_params(seed=0):
    w = np.empty(N_PARAM, np.float32)
    L.lib().kr_mlp_init(_p(w), int(seed))
    return w


def grad(X, y, w, wneg=1.0, device=0):
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    g = np.empty(N_PARAM, np.float32)
    loss = ctypes.c_double()
    rc = L.lib().kr_mlp_grad(_p(X), _p(y), len(y), _p(w), float(wneg), _p(g), ctypes.byref(loss), device)
    if rc:
        raise RuntimeError(_err())
    return loss.value, g


def train(X, y, w=None, epochs=20, batch=4096, lr=3e-3, wneg=4.0, seed=0, device=0):
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    w = init_params(seed) if w is None else np.array(w, np.float32)
    loss = ctypes.c_double()
    rc = L.lib().kr_mlp_train(_p(X), _p(y), len(y), _p(w), int(epochs), int(batch), float(lr),
                              float(wneg), ctypes.byref(loss), device)
    if rc:
        raise RuntimeError(_err())
    return w, loss.value


def infer(X, w, device=0):
    X = np.ascontiguousarray(X, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    out = np.empty(len(X), np.float32)
    if L.lib().kr_mlp_infer(_p(X), len(X), _p(w), _p(out), device):
        raise RuntimeError(_err())
    return out


def collect(dyn, steps, stride=64, seed=0, max_samples=1 << 21):
    """Faces sampled from `steps` ordinary steps (a hash of the face picks one
    in `stride`).  The device appends them in whatever order its threads get
    there; they come back in a canonical order (sorted by a hash of their
    bytes), so the same run gives the same training data.  Raises if the
    samples would overflow `max_samples`: which ones were kept would then
    depend on that order too."""
    out = np.empty((max_samples, N_IN + 1), np.float32)
    n = ctypes.c_longlong()
    rc = L.lib().kr_selector_collect(dyn._h, int(steps), int(stride), int(seed), int(max_samples),
                                     _p(out), ctypes.byref(n))
    dyn._check(rc, "kr_selector_collect")
    if n.value >= max_samples:
        raise ValueError("selector sampling reached %d samples; use a larger stride" % max_samples)
    out = out[:n.value]
    words = out.view(np.uint32).astype(np.uint64)
    h = np.zeros(len(out), np.uint64)
    with np.errstate(over="ignore"):
        for j in range(words.shape[1]):
            h = (h ^ words[:, j]) * np.uint64(0x100000001B3)
    out = out[np.argsort(h, kind="stable")]
    return out[:, :N_IN].copy(), out[:, N_IN].copy()


def shuffle(X, y, seed=0):
    idx = np.random.default_rng(seed).permutation(len(y))
    return X[idx], y[idx]


# Defaults: a gap tolerance of 3e-4 for the labels, and a logit threshold of 2.
# A warp of 32 faces goes to HLLE only when all of its faces pass the threshold
# and none of them is also computed by a neighbouring block; on the 256^3 OT
# mesh (64 blocks of 64^3) that is 8.9% of the faces, at 3.4e-6 relative L1
# density error vs the FP64 step after 23 steps (all-HLLE: 5e-5).
DEFAULT_TOL = 3e-4
DEFAULT_THRESHOLD = 2.0


def build_selector(dyn_factory, steps=4, stride=16, tol=DEFAULT_TOL, epochs=30, seed=0, device=0):
    """Collect faces from runs of the given workloads, label them with the gap
    tolerance and train.  dyn_factory: iterable of callables returning a
    Dynamics object with its initial state set.  Returns (params, info)."""
    Xs, gs = [], []
    for make in dyn_factory:
        d = make()
        X, g = collect(d, steps, stride, seed)
        Xs.append(X)
        gs.append(g)
        d.close()
    X = np.concatenate(Xs)
    gap = np.concatenate(gs)
    y = (gap < tol).astype(np.float32)
    X, y = shuffle(X, y, seed)
    w, loss = train(X, y, epochs=epochs, seed=seed, device=device)
    return w, {"samples": int(len(y)), "safe_fraction": float(y.mean()), "loss": loss, "tol": tol}

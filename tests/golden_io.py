"""Loading of the golden fixtures made by tests/golden/make_golden.py."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["shock_16", "ot_16", "ot_ragged", "shock_floor", "shock_c1", "ot_64",
         "shock_bc", "shock_fixd", "ot_bc_out", "ot_bc_ref", "ot_bc_fre", "ot_bc_fix", "ot_bc_fix0",
         "smr_shock", "smr_bc", "smr_3lvl", "smr_ot", "smr_ot3", "smr_ot_slab", "smr_blast", "smr_ot_bc", "smr_ot_fix",
         "turb_16", "turb_32", "box_5", "box_1", "box_3"]
# MHD workloads
MHD_WORKLOADS = ("ot", "turb", "box", "blast")
# single boxes of the batched-box workload (seed 5): the box index of each
BOX_CASES = {"box_5": 5, "box_1": 1, "box_3": 3}
# statically refined MHD fixtures (two and three levels; the blast's mesh from
# the gradient criterion, kratos_b200/amr.py)
MHD_SMR_CASES = ["smr_ot", "smr_ot3", "smr_ot_slab", "smr_blast", "smr_ot_bc", "smr_ot_fix"]
# statically refined fixtures (blocks in tree order, with level / reg arrays)
SMR_CASES = ["smr_shock", "smr_bc", "smr_3lvl"]


def boundary(meta):
    """(kinds per side, fixed primitive state, fixed B) of a fixture;
    periodic when unset."""
    extra = meta.get("dynamics", {})
    kinds = extra.get("kinds", "per per per per per per").split()
    init = extra.get("init", {})
    w_fix = [float(init.get("rho0", 0)), float(init.get("pre0", 0))] + \
        [float(x) for x in init.get("vel0", "0 0 0").split()]
    b_fix = [float(x) for x in init.get("b0", "0 0 0").split()]
    return kinds, w_fix, b_fix


def regions(meta):
    """Static refinement regions of a fixture: [(level, x_min, x_max)]."""
    return [(int(l), tuple(lo), tuple(hi)) for l, lo, hi in meta.get("dynamics", {}).get("regions", [])]


def field_errors(u, ref):
    """Relative L1 error per conserved field (0..4); the momentum components
    against the L1 norm of the whole momentum vector (a transverse component
    that only seeded noise drives is near zero, and its own norm would turn
    rounding into a large relative number)."""
    mom = np.abs(ref[..., 2:5]).sum()
    out = []
    for k in range(5):
        den = mom if k >= 2 else np.abs(ref[..., k]).sum()
        out.append(np.abs(u[..., k] - ref[..., k]).sum() / den)
    return out


def init(mesh, meta):
    """Initial state of a fixture's workload on a mesh (oracle or device)."""
    if meta["workload"] == "box":
        mesh.init_box(meta["seed"], meta["dynamics"]["box"])
    else:
        mesh.init_problem(meta["workload"], meta["seed"])


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    return meta, {k: z[k] for k in z.files if k != "meta"}


def checksums(a):
    a = a.reshape(-1, a.shape[-1])
    return np.stack([a.sum(0), np.abs(a).sum(0), a.min(0), a.max(0)])


def owned_bf(bf, n):
    """Owned face-lattice box [nblk, n2+1, n1+1, n0+1, 3] of a full bf array
    [nblk, n2+5, n1+5, n0+5, 3] (2 ghost layers)."""
    return bf[:, 2:3 + n[2], 2:3 + n[1], 2:3 + n[0], :]


def face_mask(n):
    """Boolean mask over the owned box marking faces a block owns:
    component c at index 0..n along c and 0..n-1 along the other axes."""
    m = np.zeros((n[2] + 1, n[1] + 1, n[0] + 1, 3), bool)
    for c in range(3):
        sl = [slice(0, n[2]), slice(0, n[1]), slice(0, n[0])]
        sl[2 - c] = slice(0, n[c] + 1)
        m[tuple(sl) + (c,)] = True
    return m


def face_checksums(bf, n):
    """Checksums [4, 3] (sum, sum of |.|, min, max per component) of the faces
    each block owns, as tests/golden/make_golden.py stores them."""
    own = owned_bf(bf, n)
    out = np.zeros((4, 3))
    for c in range(3):
        sl = [slice(None), slice(0, n[2]), slice(0, n[1]), slice(0, n[0])]
        sl[3 - c] = slice(0, n[c] + 1)
        v = own[tuple(sl) + (c,)].ravel()
        out[:, c] = [v.sum(), np.abs(v).sum(), v.min(), v.max()]
    return out

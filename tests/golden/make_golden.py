"""Generate the golden fixtures of the hydro / MHD step from the original Kratos
solver.

The reference is compiled for the CPU from its own sources (its ARCH=HIPCPU
path, PRECISION=2) by oracle/Makefile.ref into oracle/_ref/kratos_ref, with the
problem generator oracle/pgen/kr_ref_pgen.cpp.  This script runs it on a few
small seeded workloads, reads the snapshots it writes (initial and final) and
stores them under tests/golden/ as compressed .npz files:

    u0, u1      conserved state before / after the run, [nblk, n2, n1, n0, nw]
                in lexicographic block order (x fastest); refined meshes in
                tree order (level, then lexicographic) with
    level, reg  each block's level and logical position at that level
    bf0, bf1    MHD face field, owned lattice box [nblk, n2+1, n1+1, n0+1, 3]
    meta        JSON: workload, mesh, physics, steps, final time and dt
Large cases keep only checksums (per-component sum, sum of |.|, min, max).

Usage:  make -f oracle/Makefile.ref REF=<kratos tree> -j8
        python tests/golden/make_golden.py
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from kratos_b200.snapshot import Snapshot, block_ids, to_lex_arrays, to_tree_arrays  # noqa: E402
from kratos_b200.amr import gradient_regions  # noqa: E402

REF_BIN = os.environ.get("KR_REF_BIN", os.path.join(ROOT, "oracle", "_ref", "kratos_ref"))

CASES = [
    # name, problem, nb, n, steps, seed, gamma, extra dynamics keys, keep fields
    # keep: "full" (initial and final fields), "final" (final fields), "sums",
    # or "planes" (sums plus two sampled planes of the final state, below)
    ("shock_16", "shock", (2, 2, 2), (8, 8, 8), 5, 1, 1.4, {}, "full"),
    ("ot_16", "ot", (2, 2, 2), (8, 8, 8), 5, 2, 1.6666666666666667, {}, "full"),
    ("ot_ragged", "ot", (3, 2, 1), (8, 8, 8), 4, 3, 1.6666666666666667, {}, "final"),
    ("shock_floor", "shock", (2, 2, 2), (8, 8, 8), 3, 4, 1.4, {"tmp_floor": "1.0"}, "final"),
    ("shock_c1", "shock", (2, 2, 2), (32, 32, 32), 20, 1, 1.4, {}, "sums"),
    ("ot_64", "ot", (2, 2, 2), (32, 32, 32), 10, 2, 1.6666666666666667, {}, "sums"),
    # the headline MHD mesh at its full size: 256^3, 64 blocks of 64^3, seed 2,
    # 50 steps (about 20 minutes of the reference's CPU path on 8 cores)
    ("ot_256", "ot", (4, 4, 4), (64, 64, 64), 50, 2, 1.6666666666666667, {}, "planes"),
    # physical boundaries (hydro/boundary/phys_functors.h): reflect, outflow, free,
    # fixed (Dirichlet inflow from [init]); "kinds" lists x-, x+, y-, y+, z-, z+
    ("shock_bc", "shock", (2, 2, 2), (8, 8, 8), 5, 5, 1.4,
     {"kinds": "ref out fre out per per"}, "final"),
    ("shock_fixd", "shock", (2, 2, 1), (8, 8, 8), 4, 6, 1.4,
     {"kinds": "fixd out ref ref per per", "init": {"rho0": "1.0", "pre0": "1.0", "vel0": "0.5 0 0"}},
     "final"),
    # MHD physical boundaries (mhd/boundary/phys.h, phys_functors.h), one
    # non-periodic axis per case; out / fre sides also take the high-side
    # boundary-plane edge EMF (mhd/integrator/integrator.h:329-382)
    # (the MHD boundary kernel needs >= 2 n_gh threads per CTA; it has no
    # barrier, so the CPU build runs them one after another)
    ("ot_bc_out", "ot", (2, 2, 1), (8, 8, 8), 4, 7, 1.6666666666666667,
     {"kinds": "out out per per per per", "bnd_thread_limit": "4"}, "final"),
    ("ot_bc_ref", "ot", (2, 2, 1), (8, 8, 8), 4, 8, 1.6666666666666667,
     {"kinds": "per per ref ref per per", "bnd_thread_limit": "4"}, "final"),
    ("ot_bc_fre", "ot", (2, 1, 2), (8, 8, 8), 4, 9, 1.6666666666666667,
     {"kinds": "per per per per fre out", "bnd_thread_limit": "4"}, "final"),
    # fixed MHD sides (the reference built without g++'s loop optimisations
    # that exploit fixed_t::hydro's read past w_fix, oracle/Makefile.ref):
    # an inflowing medium, and a static one (vel0 = 0), where the ghost lines'
    # fluxes between identical states carry a mass flux that is rounding
    # residue and the edge EMF's upwind switch reads its sign
    ("ot_bc_fix", "ot", (2, 1, 2), (8, 8, 8), 4, 9, 1.6666666666666667,
     {"kinds": "per per per per fixd fixd", "bnd_thread_limit": "4",
      "init": {"rho0": "0.2", "pre0": "0.15", "vel0": "0.3 -0.2 0.1", "b0": "0.1 0.05 0.2"}}, "final"),
    ("ot_bc_fix0", "ot", (2, 1, 2), (8, 8, 8), 4, 9, 1.6666666666666667,
     {"kinds": "per per per per fixd fixd", "bnd_thread_limit": "4",
      "init": {"rho0": "0.2", "pre0": "0.15", "vel0": "0 0 0", "b0": "0.1 0.05 0.2"}}, "final"),
    # decaying supersonic MHD turbulence (the initial field of the 512^3
    # turbulence workload, at small size): rms Mach 5, beta 0.1
    ("turb_16", "turb", (2, 2, 2), (8, 8, 8), 5, 4, 1.6666666666666667, {}, "final"),
    ("turb_32", "turb", (2, 2, 2), (16, 16, 16), 6, 4, 1.6666666666666667, {}, "sums"),
    # single boxes of the batched independent-box workload (seed 5; box 5 is
    # 16^3, box 1 24^3, box 3 32^3): each box is its own periodic one-block mesh
    ("box_5", "box", (1, 1, 1), (16, 16, 16), 5, 5, 1.6666666666666667, {"box": 5}, "final"),
    ("box_1", "box", (1, 1, 1), (24, 24, 24), 5, 5, 1.6666666666666667, {"box": 1}, "sums"),
    ("box_3", "box", (1, 1, 1), (32, 32, 32), 5, 5, 1.6666666666666667, {"box": 3}, "sums"),
    # static mesh refinement, hydro ([refine_region*] sections: level, x_min,
    # x_max); blocks are stored in tree order (level, then z, y, x) with their
    # levels and logical positions
    ("smr_shock", "shock", (2, 2, 2), (8, 8, 8), 5, 3, 1.4,
     {"regions": [(1, (0.3, 0.1, 0.1), (0.45, 0.4, 0.4))]}, "full"),
    # refined blocks on physical sides, ragged blocks, two regions
    ("smr_bc", "shock", (3, 2, 1), (8, 16, 8), 4, 11, 1.4,
     {"kinds": "ref out fre out per per",
      "regions": [(1, (0.05, 0.05, 0.2), (0.2, 0.3, 0.6)), (1, (0.7, 0.8, 0.1), (0.9, 0.95, 0.2))]},
     "final"),
    # static refinement, MHD (Orszag-Tang): the reference's face-B restriction /
    # Toth-Roe prolongation and EMF correction across the level jump
    ("smr_ot", "ot", (2, 2, 2), (8, 8, 8), 4, 2, 1.6666666666666667,
     {"regions": [(1, (0.3, 0.1, 0.1), (0.45, 0.4, 0.4))], "bnd_thread_limit": "4"}, "final"),
    # MHD on three levels (a level-2 point region inside a level-1 one)
    ("smr_ot3", "ot", (1, 1, 1), (8, 8, 8), 4, 13, 1.6666666666666667,
     {"regions": [(2, (0.3, 0.3, 0.3), (0.3, 0.3, 0.3))], "bnd_thread_limit": "4"}, "final"),
    # MHD, a level-1 slab across four root blocks: coarse blocks that meet
    # the refined region only along an edge or at a vertex
    ("smr_ot_slab", "ot", (2, 2, 2), (8, 8, 8), 4, 14, 1.6666666666666667,
     {"regions": [(1, (0.3, 0.3, 0.2), (0.7, 0.45, 0.6))], "bnd_thread_limit": "4"}, "sums"),
    # the magnetized blast on a mesh that the gradient criterion refines at
    # t = 0 (kratos_b200/amr.py; 2^3 roots of 8^3, two levels, 120 blocks)
    ("smr_blast", "blast", (2, 2, 2), (8, 8, 8), 4, 15, 1.6666666666666667,
     {"regions": gradient_regions((2, 2, 2), (8, 8, 8), 2), "bnd_thread_limit": "4"}, "sums"),
    # refined MHD with physical sides: outflow / free along x, reflecting along
    # y, the level-1 region touching the x- and y- sides
    ("smr_ot_bc", "ot", (2, 2, 2), (8, 8, 8), 4, 16, 1.6666666666666667,
     {"kinds": "out fre ref ref per per", "bnd_thread_limit": "4",
      "regions": [(1, (0.05, 0.05, 0.3), (0.2, 0.2, 0.6))]}, "final"),
    # refined MHD with fixed (inflowing) z sides, the region touching both
    ("smr_ot_fix", "ot", (2, 1, 2), (8, 8, 8), 4, 17, 1.6666666666666667,
     {"kinds": "per per per per fixd fixd", "bnd_thread_limit": "4",
      "init": {"rho0": "0.2", "pre0": "0.15", "vel0": "0.3 -0.2 0.1", "b0": "0.1 0.05 0.2"},
      "regions": [(1, (0.55, 0.3, 0.05), (0.7, 0.6, 0.95))]}, "final"),
    # three levels (a level-2 region inside a level-1 one)
    ("smr_3lvl", "shock", (1, 1, 1), (8, 8, 8), 4, 12, 1.4,
     {"regions": [(2, (0.3, 0.3, 0.3), (0.3, 0.3, 0.3))]}, "final"),
]


def par_text(problem, nb, n, steps, seed, gamma, extra, prefix):
    ng = [nb[a] * n[a] for a in range(3)]
    dyn = {"gamma": repr(gamma), "cfl": "0.3", "thread_limit": "1", "bnd_thread_limit": "1"}
    extra = dict(extra)
    kinds = extra.pop("kinds", "per per per per per per")
    init = extra.pop("init", {})
    regions = extra.pop("regions", [])
    box = extra.pop("box", None)
    dyn.update(extra)
    lines = [
        "[problem]", "name = %s" % problem, "seed = %d" % seed] + \
        (["box = %d" % box] if box is not None else []) + [
        "",
        "[mesh]", "x_min = 0 0 0", "x_max = 1 1 1",
        "n_cell_global = %d %d %d" % tuple(ng), "n_cell_block = %d %d %d" % tuple(n), "",
        "[cycle]", "prefix_output = %s" % prefix, "n_cycle_lim = %d" % (steps - 1),
        "final_output = 1", "n_display_freq = 1000000", "",
        "[dynamics]"] + ["%s = %s" % kv for kv in dyn.items()] + [
        "", "[boundary]", "kinds = %s" % kinds, ""]
    if init:
        lines += ["[init]"] + ["%s = %s" % kv for kv in init.items()] + [""]
    for k, (level, lo, hi) in enumerate(regions):
        lines += ["[refine_region_%04d]" % k, "level = %d" % level,
                  "x_min = %r %r %r" % tuple(lo), "x_max = %r %r %r" % tuple(hi), ""]
    return "\n".join(lines)


def checksums(a):
    a = a.reshape(-1, a.shape[-1])
    return np.stack([a.sum(0), np.abs(a).sum(0), a.min(0), a.max(0)])


def owned_bf(bf, n):
    return bf[:, 2:3 + n[2], 2:3 + n[1], 2:3 + n[0], :].copy()


def face_checksums(bf, n):
    """Checksums [4, 3] of the faces each block owns (component c at 0..n
    along c and 0..n-1 along the other axes; the rest of the owned box holds
    ghost slots whose fill is a convention of each code)."""
    own = owned_bf(bf, n)
    out = np.zeros((4, 3))
    for c in range(3):
        sl = [slice(None), slice(0, n[2]), slice(0, n[1]), slice(0, n[0])]
        sl[3 - c] = slice(0, n[c] + 1)
        v = own[tuple(sl) + (c,)].ravel()
        out[:, c] = [v.sum(), np.abs(v).sum(), v.min(), v.max()]
    return out


PLANE_STRIDE = 8


def sampled_planes(u, nb, n):
    """Two z-planes of the global cell grid (global z = 0 and the middle one),
    every PLANE_STRIDE-th cell along x and y: [2, ny, nx, nw]."""
    nblk, n2, n1, n0, nw = u.shape
    g = u.reshape(nb[2], nb[1], nb[0], n2, n1, n0, nw).transpose(0, 3, 1, 4, 2, 5, 6)
    g = g.reshape(nb[2] * n2, nb[1] * n1, nb[0] * n0, nw)
    zs = [0, g.shape[0] // 2]
    return np.stack([g[z, ::PLANE_STRIDE, ::PLANE_STRIDE, :] for z in zs])


def block_ids_in_order(snap, nb, refined):
    """The reference's global id of each block, in the fixture's block order
    (lexicographic, or tree order for a refined mesh)."""
    rows = []
    for bid in block_ids(snap):
        lv = int(snap.array("block_%d|level" % bid, "i")[0])
        il = snap.array("block_%d|i_logic" % bid, "i").astype(int)
        key = (lv, int(il[2]), int(il[1]), int(il[0])) if refined else \
            (0, int(il[2]), int(il[1]), int(il[0]))
        rows.append((key, bid))
    rows.sort()
    return np.array([bid for _, bid in rows], np.int64)


def run_snapshots(exe, problem, nb, n, steps, seed, gamma, extra, env=None):
    """Run a Kratos executable on a case; its initial and final snapshots."""
    with tempfile.TemporaryDirectory() as tmp:
        prefix = os.path.join(tmp, "snap")
        par = os.path.join(tmp, "case.par")
        with open(par, "w") as f:
            f.write(par_text(problem, nb, n, steps, seed, gamma, extra, prefix))
        subprocess.check_call([exe, par], cwd=tmp, stdout=subprocess.DEVNULL,
                              env=dict(os.environ, **(env or {})))
        return Snapshot.read(prefix + "_00000.bin"), Snapshot.read(prefix + "_00001.bin")


def run_case(name, problem, nb, n, steps, seed, gamma, extra, keep):
    s0, s1 = run_snapshots(REF_BIN, problem, nb, n, steps, seed, gamma, extra)
    if extra.get("regions"):
        level, reg, u0, bf0 = to_tree_arrays(s0)
        level1, reg1, u1, bf1 = to_tree_arrays(s1)
        assert np.array_equal(level, level1) and np.array_equal(reg, reg1)
    else:
        u0, bf0 = to_lex_arrays(s0, nb)
        u1, bf1 = to_lex_arrays(s1, nb)
    if int(s1.array("cycle", "i")[0]) != steps - 1 or not float(s1.array("time")[0]) > 0:
        raise RuntimeError("%s: the reference run stopped early" % name)
    meta = {
        "workload": problem, "seed": seed, "gamma": gamma, "nb": list(nb), "n": list(n),
        "steps": steps, "cfl": 0.3, "dynamics": extra,
        "t": float(s1.array("time")[0]), "dt": float(s1.array("dt")[0]),
        "cycle": int(s1.array("cycle", "i")[0]),
    }
    out = {"meta": np.array(json.dumps(meta))}
    if extra.get("regions"):
        out["level"], out["reg"] = level, reg
    out["ids"] = block_ids_in_order(s0, nb, bool(extra.get("regions")))
    if keep == "full":
        out["u0"] = u0
        if bf0 is not None:
            out["bf0"] = owned_bf(bf0, n)
    if keep in ("full", "final"):
        out["u1"] = u1
        if bf1 is not None:
            out["bf1"] = owned_bf(bf1, n)
    if keep == "planes":
        out["u1_planes"] = sampled_planes(u1, nb, n)
    out["u0_sum"], out["u1_sum"] = checksums(u0), checksums(u1)
    if bf0 is not None:
        out["bf0_sum"] = face_checksums(bf0, n)
        out["bf1_sum"] = face_checksums(bf1, n)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("%-12s t=%.6e  %7.1f kB" % (name, meta["t"], os.path.getsize(path) / 1e3))


def main():
    if not os.path.exists(REF_BIN):
        sys.exit("build the reference first: make -f oracle/Makefile.ref REF=<kratos tree>")
    only = set(sys.argv[1:])
    for c in CASES:
        if not only or c[0] in only:
            run_case(*c)


if __name__ == "__main__":
    main()

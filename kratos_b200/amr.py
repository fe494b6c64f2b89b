"""Static refinement chosen at t = 0 by a gradient criterion (no reference
counterpart: the reference's mesh refinement is static, from [refine_region*]
boxes read at start-up, meshgen.cpp:111-163, and it has no criterion).

The criterion flags a block when one of its cells has
    max over axes of ( |rho_+ - rho_-| / (2 rho) + |p_+ - p_-| / (2 p) ) > theta
(central differences of the initial state at that block's resolution, its
neighbours across the block sides included).  Starting from the root blocks,
the children of every flagged block are examined one level down, to
`levels` refinement levels.  The result is exported the way the reference
reads refinement: one point region per flagged block, at the next level and
at the centre of the block's first child, so that inserting it refines the
block; the block tree's 2:1 balance adds the neighbours both codes need
(tree.cpp:139-232).  `par_sections` writes the regions as [refine_region_NNNN]
sections of a Kratos parameter file, so the original code builds the same
tree.
"""
import numpy as np


def blast_state(x, centre):
    """(rho, p) of the magnetized blast workload at cell centres x [..., 3]
    (kratos_b200/csrc/problems.h kr_blast_pre)."""
    r2 = np.zeros(x.shape[:-1])
    for a in range(3):
        r2 = r2 + (x[..., a] - centre[a]) * (x[..., a] - centre[a])
    return np.ones_like(r2), np.where(r2 < 0.01, 100.0, 0.1)


def _flag(state, x_min, x_max, nb, n, level, reg, theta, centre):
    lim = np.array(nb) << level
    h = (np.array(x_max, float) - np.array(x_min, float)) / lim / np.array(n)
    axes = [np.array(x_min[a], float) + (reg[a] * n[a] + np.arange(-1, n[a] + 1) + 0.5) * h[a]
            for a in range(3)]
    # periodic domain: wrap the halo cells
    for a in range(3):
        span = x_max[a] - x_min[a]
        axes[a] = np.where(axes[a] < x_min[a], axes[a] + span, axes[a])
        axes[a] = np.where(axes[a] >= x_max[a], axes[a] - span, axes[a])
    x = np.stack(np.meshgrid(axes[0], axes[1], axes[2], indexing="ij"), axis=-1)
    rho, p = state(x, centre)
    crit = np.zeros(tuple(n))
    inner = (slice(1, -1),) * 3
    for a in range(3):
        lo = [slice(1, -1)] * 3
        hi = [slice(1, -1)] * 3
        lo[a] = slice(0, -2)
        hi[a] = slice(2, None)
        g = (np.abs(rho[tuple(hi)] - rho[tuple(lo)]) / (2 * rho[inner])
             + np.abs(p[tuple(hi)] - p[tuple(lo)]) / (2 * p[inner]))
        crit = np.maximum(crit, g)
    return bool((crit > theta).any())


def gradient_regions(nb, n, levels, theta=0.5, state=blast_state, x_min=(0, 0, 0), x_max=(1, 1, 1)):
    """Refinement regions [(level, x_lo, x_hi)] of the gradient criterion on
    the initial state `state(x, centre) -> (rho, p)` of a periodic domain."""
    centre = [(x_min[a] + x_max[a]) / 2 for a in range(3)]
    cand = [(0, (i, j, k)) for k in range(nb[2]) for j in range(nb[1]) for i in range(nb[0])]
    regions = []
    for level in range(levels):
        flagged = [reg for lv, reg in cand if _flag(state, x_min, x_max, nb, n, lv, reg, theta, centre)]
        cand = []
        for reg in flagged:
            child = [2 * r for r in reg]
            h = [(x_max[a] - x_min[a]) / (nb[a] << (level + 1)) for a in range(3)]
            pt = tuple(x_min[a] + (child[a] + 0.5) * h[a] for a in range(3))
            regions.append((level + 1, pt, pt))
            for d in np.ndindex(2, 2, 2):
                cand.append((level + 1, tuple(child[a] + d[a] for a in range(3))))
    return regions


def par_sections(regions):
    """[refine_region_NNNN] sections for a Kratos parameter file."""
    lines = []
    for k, (level, lo, hi) in enumerate(regions):
        lines += ["[refine_region_%04d]" % k, "level = %d" % level,
                  "x_min = %r %r %r" % tuple(lo), "x_max = %r %r %r" % tuple(hi), ""]
    return "\n".join(lines)

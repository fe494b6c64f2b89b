"""The magnetized blast on a criterion-refined MHD mesh: root 128^3 in 16^3
blocks, three refinement levels picked at t = 0 by kratos_b200.amr's gradient
criterion, periodic, PLM + HLLD + CT, Heun RK2.

    python -m kratos_b200.blast --steps 3 --precision 1

steps the mesh and prints its time, status, launches per step and the per-kind
kernel times of one profiled step (kr_profile_step)."""
import argparse
import json

from .amr import gradient_regions
from .engine import Dynamics

NB, N, LEVELS = (8, 8, 8), (16, 16, 16), 3


def blast_mesh(precision=1, device=0, nb=NB, n=N, levels=LEVELS):
    regions = gradient_regions(nb, n, levels)
    return Dynamics(True, nb, n, gamma=5 / 3, precision=precision, device=device, regions=regions), regions


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--precision", type=int, default=1, help="2 FP64, 1 mixed")
    p.add_argument("--seed", type=int, default=15)
    args = p.parse_args(argv)
    d, regions = blast_mesh(args.precision)
    d.init_problem("blast", args.seed)
    d.step(args.steps)
    out = {"t": d.time()["t"], "status": d.status(), "blocks": d.nblk, "cells": d.n_cells,
           "regions": len(regions), "launches_per_step": d.launches_per_step(),
           "kernels_ms_per_step": d.profile_step()}
    print(json.dumps(out))
    d.close()


if __name__ == "__main__":
    main()

"""A mesh sharded over torch.distributed ranks, one process per GPU.

The blocks are split between the ranks by the engine (kr_shard_owner: recursive
coordinate bisection of the block grid); each rank's context exchanges its
halo with the others through NCCL inside the step's CUDA graph and reduces dt
over all ranks (kr_comm_init).  torch.distributed is only the plumbing here:
it checks that every rank derived the same exchange plan, and hands the NCCL
unique id from rank 0 to the others.
"""
import numpy as np
import torch.distributed as dist

from .engine import Dynamics, KratosError, comm_unique_id, halo_counts, make_cfg


def check_plan(cfg, group=None):
    """Raise on every rank unless the words each rank will send to each peer
    equal what that peer expects to receive (same mesh, same partition)."""
    snd, rcv = halo_counts(cfg)
    world = dist.get_world_size(group)
    mesh = (tuple(cfg.nb), tuple(cfg.n), cfg.mhd, cfg.precision, cfg.riemann, tuple(cfg.bc),
            cfg.flags, cfg.n_ranks, tuple(cfg.x_min), tuple(cfg.x_max))
    plans = [None] * world
    dist.all_gather_object(plans, (int(cfg.rank), snd.tolist(), rcv.tolist(), mesh), group=group)
    bad = ["rank %d built a different mesh than rank 0" % p
           for p in range(world) if plans[p][3] != plans[0][3]]
    for p in range(world):
        rp, sp, _, _ = plans[p]
        if rp != p or len(sp) != world:
            bad.append("rank %d reports rank %d of %d" % (p, rp, len(sp)))
            continue
        for q in range(world):
            if list(sp[q]) != list(plans[q][2][p]):
                bad.append("rank %d sends %s words to %d, which expects %s"
                           % (p, sp[q], q, plans[q][2][p]))
    if bad:
        raise KratosError("halo plans disagree: " + "; ".join(bad[:4]))
    return np.array([plans[p][1] for p in range(world)], np.int64)


def sharded_dynamics(mhd, nb, n, group=None, **kw):
    """This rank's share of an nb[0] x nb[1] x nb[2]-block mesh with a
    communicator attached; `kw` as for Dynamics (device: this rank's GPU)."""
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    cfg = make_cfg(mhd, nb, n, n_ranks=world, rank=rank, **kw)
    check_plan(cfg, group)
    d = Dynamics(mhd, nb, n, n_ranks=world, rank=rank, **kw)
    uid = [comm_unique_id() if rank == 0 else None]
    src = dist.get_global_rank(group, 0) if group is not None else 0
    dist.broadcast_object_list(uid, src=src, group=group)
    d.comm_init(uid[0])
    return d

"""Sharding of the block mesh over ranks, on the CPU (no device needed):
the block partition (kr_shard_owner), the per-stage halo plan (kr_halo_counts)
and the torch.distributed handshake that checks the plans agree before any
NCCL call (kratos_b200.shard.check_plan), run as world-size-2 gloo ranks."""
import os

import numpy as np
import pytest

from kratos_b200.engine import KratosError, halo_counts, make_cfg, shard_owner


def _cfg(nb, ranks, rank=0, mhd=True, n=(8, 8, 8), **kw):
    return make_cfg(mhd, nb, n, n_ranks=ranks, rank=rank, **kw)


@pytest.mark.parametrize("nb,ranks", [((4, 4, 4), 8), ((4, 4, 8), 2), ((4, 8, 8), 4), ((8, 8, 8), 8),
                                      ((12, 4, 4), 3), ((3, 2, 1), 2), ((5, 3, 2), 4), ((2, 2, 2), 8),
                                      ((1, 1, 1), 1)])
def test_partition_is_boxes_covering_the_mesh(nb, ranks):
    owner, k0 = shard_owner(_cfg(nb, ranks))
    o = owner.reshape(nb[2], nb[1], nb[0])
    assert set(np.unique(o)) == set(range(ranks))
    assert k0 == int((owner == 0).sum())
    sizes = []
    for r in range(ranks):
        z, y, x = np.nonzero(o == r)
        box = (z.max() - z.min() + 1) * (y.max() - y.min() + 1) * (x.max() - x.min() + 1)
        assert box == len(z), "rank %d does not own a box" % r
        sizes.append(len(z))
        assert shard_owner(_cfg(nb, ranks, rank=r))[1] == len(z)
    total = nb[0] * nb[1] * nb[2]
    if total % ranks == 0 and all(x & (x - 1) == 0 for x in nb) and ranks & (ranks - 1) == 0:
        assert sizes == [total // ranks] * ranks


def test_weak_scaling_meshes_give_equal_cubes():
    """The meshes bench.py uses for 2, 4, 8 GPUs: 4x4x4 blocks per rank."""
    for nb, ranks in (((4, 4, 8), 2), ((4, 8, 8), 4), ((8, 8, 8), 8)):
        o = shard_owner(_cfg(nb, ranks))[0].reshape(nb[2], nb[1], nb[0])
        for r in range(ranks):
            z, y, x = np.nonzero(o == r)
            assert (np.ptp(z) + 1, np.ptp(y) + 1, np.ptp(x) + 1) == (4, 4, 4)


def test_too_many_ranks_is_an_error():
    with pytest.raises(KratosError):
        shard_owner(_cfg((1, 1, 1), 2))
    with pytest.raises(KratosError):
        shard_owner(_cfg((2, 1, 1), 2, rank=2))


@pytest.mark.parametrize("mhd,kinds", [(True, ("per",) * 6), (False, ("per",) * 6),
                                       (False, ("ref", "out", "per", "per", "fre", "fixd"))])
@pytest.mark.parametrize("nb,ranks", [((2, 2, 2), 2), ((4, 2, 2), 4), ((3, 2, 1), 3), ((2, 2, 2), 8)])
def test_halo_plans_pair_up(mhd, kinds, nb, ranks):
    """What rank p sends to q is what q expects from p; nothing to oneself."""
    plans = [halo_counts(_cfg(nb, ranks, r, mhd=mhd, kinds=kinds)) for r in range(ranks)]
    for p in range(ranks):
        assert not plans[p][0][p].any() and not plans[p][1][p].any()
        for q in range(ranks):
            assert np.array_equal(plans[p][0][q], plans[q][1][p])
        if not mhd:
            assert not plans[p][0][:, 1].any()


def test_halo_words_two_blocks_along_x():
    """nb = 2 x 1 x 1, 8^3 MHD, periodic: every ghost direction with an x
    component reads the other block -- 2 x (8+2+2)^2 cells x 11 words per x
    side -- plus the two face-B strips of the x faces, 2 x (9 x 8) words each."""
    snd, rcv = halo_counts(_cfg((2, 1, 1), 2, 0))
    assert tuple(rcv[1]) == (2 * 2 * 12 * 12 * 11, 2 * 2 * 9 * 8)
    assert tuple(snd[1]) == tuple(rcv[1])


def test_halo_all_routes_every_neighbour_copy():
    """KR_FLAG_HALO_ALL on one unsharded block: the whole ghost shell and all
    six face-B strip pairs go through the exchange, to and from oneself."""
    n = (8, 6, 4)
    snd, rcv = halo_counts(_cfg((1, 1, 1), 1, 0, n=n, flags=2))
    shell = (n[0] + 4) * (n[1] + 4) * (n[2] + 4) - n[0] * n[1] * n[2]
    strips = sum(2 * (n[c] + 1) * (n[(c + 1) % 3] + n[(c + 2) % 3]) for c in range(3))
    assert tuple(snd[0]) == tuple(rcv[0]) == (shell * 11, strips)


# ------------------------------------------------------------ gloo, 2 ranks
def _worker(rank, world, port, results):
    import torch.distributed as dist
    from kratos_b200.shard import check_plan
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = {}
        cfg = _cfg((4, 2, 2), world, rank)
        out["sends"] = check_plan(cfg).tolist()
        # a rank that built a different mesh: every rank must refuse
        bad = _cfg((4, 2, 2) if rank == 0 else (2, 4, 2), world, rank)
        try:
            check_plan(bad)
            out["mismatch"] = "accepted"
        except KratosError as e:
            out["mismatch"] = str(e)
        # a planted error in one rank's exchange plan (same mesh)
        import kratos_b200.shard as S
        if rank == 1:
            real = S.halo_counts

            def planted(c):
                snd, rcv = real(c)
                rcv[0, 0] += 1
                return snd, rcv
            S.halo_counts = planted
        try:
            check_plan(cfg)
            out["planted"] = "accepted"
        except KratosError as e:
            out["planted"] = str(e)
        results[rank] = out
    finally:
        dist.destroy_process_group()


def test_plan_handshake_over_gloo():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mgr = mp.get_context("spawn").Manager()
    results = mgr.dict()
    mp.spawn(_worker, args=(2, port, results), nprocs=2, join=True)
    r0, r1 = results[0], results[1]
    assert r0["sends"] == r1["sends"]
    s = np.array(r0["sends"])            # [rank][peer][2]
    assert s[0, 1, 0] > 0 and s[1, 0, 0] == s[0, 1, 0]
    assert "different mesh" in r0["mismatch"] and "different mesh" in r1["mismatch"]
    assert "rank 0 sends" in r0["planted"] and "rank 0 sends" in r1["planted"]

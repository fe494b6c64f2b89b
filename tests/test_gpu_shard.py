"""Sharded meshes on one GPU, through the C ABI.

Every sharded state must equal the unsharded step bit for bit: the halo
exchange copies exactly the values the same-rank ghost fill copies, and dt is
the same global minimum.  Three routes cover the exchange:
  * kr_group_step: the n_ranks contexts of one mesh in this process, the
    exchange as device copies between them (partition, per-rank geometry,
    initial state, physical sides and the pairing of send / receive plans);
  * KR_FLAG_HALO_ALL on one context: every neighbour copy goes through pack,
    exchange and unpack inside the captured step graph;
  * the same with an NCCL communicator of one rank: the exchange is NCCL
    send / receive (to itself) and the dt all-reduce, captured in the graph.
"""
import numpy as np
import pytest

import golden_io as G

pytestmark = pytest.mark.gpu


def _own(bf, n):
    """Owned faces of a face-B array: its ghost slots hold whatever the last
    fill left (pushed by the last update on the same rank, unpacked at the
    last stage start across ranks), which is not part of the state."""
    return G.owned_bf(bf, n)[:, G.face_mask(n)]

SHOCK_BC = ("ref", "out", "fre", "out", "per", "per")


def _pair(mhd, nb, n, steps, workload, seed, ranks, precision=2, kinds=("per",) * 6, **kw):
    from kratos_b200 import Dynamics
    from kratos_b200.engine import group_step
    gamma = 5 / 3 if mhd else 1.4
    ref = Dynamics(mhd, nb, n, gamma=gamma, precision=precision, kinds=kinds, **kw)
    ref.init_problem(workload, seed)
    ref.step(steps)
    shards = [Dynamics(mhd, nb, n, gamma=gamma, precision=precision, kinds=kinds,
                       n_ranks=ranks, rank=r, **kw) for r in range(ranks)]
    for d in shards:
        d.init_problem(workload, seed)
    group_step(shards, steps)
    return ref, shards


def _assemble(shards, ref):
    u = np.full(ref.u_shape, np.nan)
    bf = np.full(ref.bf_shape, np.nan) if ref.mhd else None
    seen = []
    for d in shards:
        ud, bd = d.get_state()
        u[d.gid] = ud
        if ref.mhd:
            bf[d.gid] = bd
        seen += list(d.gid)
    assert sorted(seen) == list(range(ref.nblk))
    return u, bf


@pytest.mark.parametrize("precision", [2, 1])
@pytest.mark.parametrize("mhd,nb,ranks,kinds", [
    (True, (4, 2, 2), 2, ("per",) * 6),
    (True, (3, 2, 2), 3, ("per",) * 6),
    (True, (2, 2, 2), 8, ("per",) * 6),          # every block alone on its rank
    (False, (4, 2, 2), 4, SHOCK_BC),
    (False, (3, 2, 1), 2, ("fixd", "out", "ref", "ref", "per", "per")),
    (True, (2, 2, 2), 4, ("out", "fre", "per", "per", "ref", "fixd")),
])
def test_group_step_equals_unsharded(mhd, nb, ranks, kinds, precision):
    n = (8, 8, 8)
    extra = {"w_fix": (1.0, 1.0, 0.5, 0.0, 0.0)} if "fixd" in kinds else {}
    if "fixd" in kinds and mhd:
        extra["b_fix"] = (0.1, 0.05, 0.2)
    ref, shards = _pair(mhd, nb, n, 3, "ot" if mhd else "shock", 5, ranks, precision, kinds, **extra)
    u_ref, bf_ref = ref.get_state()
    u, bf = _assemble(shards, ref)
    assert np.array_equal(u, u_ref)
    if mhd:
        assert np.array_equal(_own(bf, n), _own(bf_ref, n))
    t_ref = ref.time()
    for d in shards:
        t = d.time()
        assert t["t"] == t_ref["t"] and t["dt_last"] == t_ref["dt_last"] and t["n_steps"] == 3
        assert d.status() == 0


def test_group_initial_state_and_ragged_blocks():
    """Non-cubic blocks and a rank count that does not divide the blocks."""
    ref, shards = _pair(True, (3, 2, 1), (12, 8, 4), 2, "ot", 9, 4)
    u, bf = _assemble(shards, ref)
    u_ref, bf_ref = ref.get_state()
    assert np.array_equal(u, u_ref) and np.array_equal(_own(bf, (12, 8, 4)), _own(bf_ref, (12, 8, 4)))


@pytest.mark.parametrize("precision", [2, 1])
@pytest.mark.parametrize("mhd", [True, False])
def test_halo_all_flag_is_bit_exact(mhd, precision):
    from kratos_b200 import Dynamics
    out = []
    for flags in (0, 2):
        d = Dynamics(mhd, (2, 2, 1), (8, 8, 8), gamma=5 / 3 if mhd else 1.4, precision=precision,
                     flags=flags, kinds=("per",) * 6 if mhd else SHOCK_BC)
        d.init_problem("ot" if mhd else "shock", 4)
        d.step(3)
        out.append((d.get_state(), d.time(), d.launches_per_step()))
    (a, ta, la), (b, tb, lb) = out
    assert np.array_equal(a[0], b[0])
    if mhd:
        assert np.array_equal(_own(a[1], (8, 8, 8)), _own(b[1], (8, 8, 8)))
    assert ta["t"] == tb["t"] and lb == la + 4


def test_nccl_exchange_one_rank():
    """The NCCL transport (grouped send / receive to itself, all-reduce of dt)
    captured in the step graph gives the same state as the plain step."""
    from kratos_b200 import Dynamics
    from kratos_b200.engine import comm_unique_id
    out = []
    for route in ("plain", "nccl"):
        d = Dynamics(True, (2, 2, 2), (8, 8, 8), gamma=5 / 3, flags=2 if route == "nccl" else 0)
        if route == "nccl":
            d.comm_init(comm_unique_id())
        d.init_problem("ot", 6)
        d.step(3)
        out.append((d.get_state(), d.time()))
        d.close()
    (a, ta), (b, tb) = out
    assert np.array_equal(a[0], b[0]) and np.array_equal(_own(a[1], (8, 8, 8)), _own(b[1], (8, 8, 8)))
    assert ta["t"] == tb["t"]


def test_sharded_context_needs_a_communicator():
    from kratos_b200 import Dynamics, KratosError
    d = Dynamics(True, (2, 1, 1), (8, 8, 8), gamma=5 / 3, n_ranks=2, rank=1)
    assert list(d.gid) == [1]
    with pytest.raises(KratosError, match="communicator"):
        d.step(1)

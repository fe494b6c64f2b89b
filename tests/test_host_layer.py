"""The C++ host layer (kratos_b200/host): a problem generator written for the
original Kratos -- oracle/pgen/kr_ref_pgen.cpp, the same source the reference
solver is built with for the golden fixtures -- compiles unchanged against the
host headers, and the executable reproduces the reference's snapshots.

CPU: the pgen builds and links; the parameter-file parser follows the
reference's rules (input.cpp:70-108: '#' comments, [section], trimmed
key = value, later files override); without a device the executable fails
loudly through the engine's error path.
GPU: the executable run on the golden fixtures' parameter files writes
snapshots whose initial state is bit-exact and whose final state agrees with
the reference to the FP64 tolerance of the parity tests; a restart from a
snapshot continues exactly like the engine does from the same time and dt.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import golden_io as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
PGEN = os.path.join(ROOT, "oracle", "pgen", "kr_ref_pgen.cpp")

TOL_FP64 = 1e-11

PARSER_PGEN = r"""
#include <iostream>
#include "user/probgen.h"
namespace prob
{
void run( int argc, char * argv[  ] )
{
    input args;
    cmd( argc, argv, args );
    const auto v = args.get< type::coord2_t >( "mesh", "x_max" );
    std::vector< std::string > kinds;
    args( "boundary", "kinds", kinds );
    std::cout << "n=" << args.get< int >( "cycle", "n_cycle_lim" )
              << " g=" << args.get< double >( "dynamics", "gamma" )
              << " x=" << v[ 0 ] << "," << v[ 1 ] << "," << v[ 2 ]
              << " k=" << kinds.size(  ) << ":" << kinds.back(  )
              << " p=" << args.get< std::string >( "cycle", "prefix_output", "test" )
              << " d=" << args.get< double >( "cycle", "dt_output", 7.5 )
              << " f=" << args.found( "cycle", "final_output" ) << std::endl;
}
}
"""


@pytest.fixture(scope="module")
def host_exe(tmp_path_factory):
    from kratos_b200.build import build_host
    out = str(tmp_path_factory.mktemp("host") / "kratos.x")
    build_host([PGEN], out)
    return out


def test_reference_pgen_builds_against_host_layer(host_exe):
    assert os.access(host_exe, os.X_OK)


def test_parameter_parser(tmp_path):
    from kratos_b200.build import build_host
    src = tmp_path / "parse.cpp"
    src.write_text(PARSER_PGEN)
    exe = build_host([str(src)], str(tmp_path / "parse.x"))
    a = tmp_path / "a.par"
    a.write_text("# leading comment\n[mesh]\n  x_max =  1 2 3   # trailing\n"
                 "[cycle]\nn_cycle_lim = 4\nprefix_output = snap\nfinal_output = 1\n"
                 "[dynamics]\ngamma = 1.4\n[boundary]\nkinds = per per out out ref fixd\n")
    b = tmp_path / "b.par"
    b.write_text("[cycle]\nn_cycle_lim=9\n\n[dynamics]\n gamma = 1.5 = ignored\n")
    out = subprocess.check_output([exe, str(a), str(b)], text=True)
    line = out.strip().splitlines()[-1]
    assert line == "n=9 g=1.5 x=1,2,3 k=6:fixd p=snap d=7.5 f=1", line


def test_executable_fails_loudly_without_device(host_exe, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import make_golden as M
    par = tmp_path / "ot.par"
    par.write_text(M.par_text("ot", (1, 1, 1), (8, 8, 8), 1, 1, 5 / 3, {}, str(tmp_path / "s")))
    r = subprocess.run([host_exe, str(par)], capture_output=True, text=True)
    assert r.returncode != 0
    assert "kratos_b200:" in r.stderr
    assert not (tmp_path / "s_00000.bin").exists()


def _run_case(exe, tmp, name):
    import make_golden as M
    from kratos_b200.snapshot import Snapshot, to_lex_arrays, to_tree_arrays
    c = [x for x in M.CASES if x[0] == name][0]
    _, problem, nb, n, steps, seed, gamma, extra, _ = c
    prefix = os.path.join(tmp, name)
    par = os.path.join(tmp, name + ".par")
    with open(par, "w") as f:
        f.write(M.par_text(problem, nb, n, steps, seed, gamma, extra, prefix))
    subprocess.check_call([exe, par], cwd=tmp, stdout=subprocess.DEVNULL)
    s0 = Snapshot.read(prefix + "_00000.bin")
    s1 = Snapshot.read(prefix + "_00001.bin")
    if extra.get("regions"):                 # refined: blocks in tree order
        return s0, s1, to_tree_arrays(s0)[2:], to_tree_arrays(s1)[2:]
    return s0, s1, to_lex_arrays(s0, nb), to_lex_arrays(s1, nb)


def rel_l1(a, b):
    den = np.abs(b).sum()
    return np.abs(a - b).sum() / (den if den > 0 else 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["shock_16", "ot_16", "shock_bc", "shock_fixd", "smr_shock", "smr_bc"])
def test_executable_snapshots_match_reference(host_exe, tmp_path, name):
    meta, g = G.load(name)
    s0, s1, (u0, bf0), (u1, bf1) = _run_case(host_exe, str(tmp_path), name)
    assert float(s1.array("time")[0]) == pytest.approx(meta["t"], rel=1e-12)
    assert float(s1.array("dt")[0]) == pytest.approx(meta["dt"], rel=1e-12)
    assert int(s1.array("cycle", "i")[0]) == meta["cycle"]
    assert int(s1.array("i_out", "i")[0]) == 2
    if "u0" in g:
        assert np.array_equal(u0[..., :5], g["u0"][..., :5])
    for k, e in enumerate(G.field_errors(u1, g["u1"])):
        assert e <= TOL_FP64, "field %d rel L1 %.3e" % (k, e)
    if bf1 is not None:
        n = meta["n"]
        own, mask = G.owned_bf(bf1, n), G.face_mask(n)
        if "bf0" in g:
            assert np.array_equal(G.owned_bf(bf0, n)[:, mask], g["bf0"][:, mask])
        for c in range(3):
            m = mask[..., c]
            e = rel_l1(own[..., c][:, m], g["bf1"][..., c][:, m])
            assert e <= TOL_FP64, "bf %d rel L1 %.3e" % (c, e)


@pytest.mark.gpu
def test_restart_from_snapshot(host_exe, tmp_path):
    """Run 2 steps, restart from the final snapshot for 3 more (the stored
    cycle index is repeated by the reference's loop, cycle.cpp:167-169), and
    compare with the engine continued from the same time and dt bound."""
    import make_golden as M
    from kratos_b200 import Dynamics
    from kratos_b200.snapshot import Snapshot, to_lex_arrays
    nb, n = (2, 2, 2), (8, 8, 8)
    prefix = str(tmp_path / "r")
    par = tmp_path / "r.par"
    par.write_text(M.par_text("ot", nb, n, 2, 5, 5 / 3, {}, prefix))
    subprocess.check_call([host_exe, str(par)], cwd=str(tmp_path), stdout=subprocess.DEVNULL)
    s1 = Snapshot.read(prefix + "_00001.bin")
    # renumber the blocks (the reference numbers them along a Hilbert curve):
    # a restart matches blocks by i_logic, not by id
    ren = Snapshot()
    for k in s1.keys():
        nk = k
        if k.startswith("block_"):
            bid, rest = k[6:].split("|", 1)
            nk = "block_%d|%s" % (7 - int(bid), rest)
        ren.data[nk], ren.unit[nk] = s1.data[k], s1.unit[k]
    ren.write(str(tmp_path / "renamed.bin"))
    over = tmp_path / "more.par"
    over.write_text("[cycle]\nn_cycle_lim = 3\n")
    subprocess.check_call([host_exe, str(tmp_path / "renamed.bin"), str(over)], cwd=str(tmp_path),
                          stdout=subprocess.DEVNULL)
    s3 = Snapshot.read(prefix + "_00002.bin")
    assert int(s3.array("cycle", "i")[0]) == 3
    u3, bf3 = to_lex_arrays(s3, nb)

    d = Dynamics(True, nb, n, gamma=5 / 3)
    d.init_problem("ot", 5)
    d.step(2)
    tm = d.time()
    assert tm["t"] == float(s1.array("time")[0])
    d.set_time(tm["t"], tm["dt_last"])
    d.step(3)
    u, bf = d.get_state()
    assert np.array_equal(u3[..., :5], u[..., :5])
    assert np.array_equal(G.owned_bf(bf3, n), G.owned_bf(bf, n))


@pytest.mark.gpu
def test_refined_restart_from_reference_snapshot(host_exe, tmp_path):
    """A refined mesh restarts from a snapshot whose blocks carry the
    reference's own numbering: blocks are matched by level and i_logic, and
    the continued run equals the engine stepped straight through."""
    import make_golden as M
    from kratos_b200 import Dynamics
    from kratos_b200.snapshot import Snapshot, to_tree_arrays
    regions = [(1, (0.3, 0.1, 0.1), (0.45, 0.4, 0.4))]
    nb, n = (2, 2, 2), (8, 8, 8)
    prefix = str(tmp_path / "r")
    par = tmp_path / "r.par"
    par.write_text(M.par_text("shock", nb, n, 2, 7, 1.4, {"regions": regions}, prefix))
    subprocess.check_call([host_exe, str(par)], cwd=str(tmp_path), stdout=subprocess.DEVNULL)
    s1 = Snapshot.read(prefix + "_00001.bin")
    ren = Snapshot()                          # reverse the block ids
    nblk = len(to_tree_arrays(s1)[0])
    for k in s1.keys():
        nk = k
        if k.startswith("block_"):
            bid, rest = k[6:].split("|", 1)
            nk = "block_%d|%s" % (nblk - 1 - int(bid), rest)
        ren.data[nk], ren.unit[nk] = s1.data[k], s1.unit[k]
    ren.write(str(tmp_path / "renamed.bin"))
    over = tmp_path / "more.par"
    over.write_text("[cycle]\nn_cycle_lim = 3\n")
    subprocess.check_call([host_exe, str(tmp_path / "renamed.bin"), str(over)], cwd=str(tmp_path),
                          stdout=subprocess.DEVNULL)
    lvl, reg, u3, _ = to_tree_arrays(Snapshot.read(prefix + "_00002.bin"))

    d = Dynamics(False, nb, n, gamma=1.4, regions=regions)
    assert np.array_equal(lvl, d.level) and np.array_equal(reg, d.reg)
    d.init_problem("shock", 7)
    d.step(2)
    tm = d.time()
    d.set_time(tm["t"], tm["dt_last"])
    d.step(3)
    u, _ = d.get_state()
    assert np.array_equal(u3, u)


def test_hilbert_numbering_matches_reference_snapshots():
    """The block ids the host layer writes follow the reference's Hilbert-curve
    order (meshgen.cpp:188-243): the Python restatement (kratos_b200.snapshot,
    the same walk as host.cpp's) against the ids in the reference's own
    snapshots -- uniform, ragged and refined meshes up to three levels."""
    from kratos_b200.snapshot import hilbert_ids
    for name in ["ot_16", "ot_ragged", "smr_shock", "smr_bc", "smr_3lvl", "smr_ot"]:
        meta, g = G.load(name)
        if "level" in g:
            lvl, reg = g["level"], g["reg"]
        else:
            nb = meta["nb"]
            idx = np.arange(nb[0] * nb[1] * nb[2])
            lvl = np.zeros(len(idx), int)
            reg = np.stack([idx % nb[0], (idx // nb[0]) % nb[1], idx // (nb[0] * nb[1])], 1)
        ids, _ = hilbert_ids(lvl, reg, meta["nb"])
        assert sorted(ids) == list(range(len(ids)))
        if "ids" in g:
            assert np.array_equal(ids, g["ids"]), name


def _tree(blob):
    """mesh_tree entry decoded: [(key, id_l, id_g, rank, mask)], n_dim,
    reg_max, periodic (the padding bytes after each node's mask are whatever
    the writer's memory held, so the comparison is by field)."""
    import struct
    (count,) = struct.unpack_from("<Q", blob, 0)
    nodes = [struct.unpack_from("<4i3i?", blob, 8 + 32 * k) for k in range(count)]
    tail = 8 + 32 * count
    return nodes, struct.unpack_from("<4i", blob, tail), tuple(blob[tail + 16:tail + 19])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ot_16", "smr_shock"])
def test_reference_restarts_from_host_layer_snapshot(host_exe, tmp_path, name):
    """The snapshot format is a two-way boundary: the host layer writes the
    serialized block tree (mesh_tree, mesh/tree/tree.cpp:11-20) and names its
    blocks by the reference's Hilbert ids, so the ORIGINAL Kratos code
    (oracle/_ref/kratos_ref) restarts from it.  3 steps on the GPU, then the
    reference continues to the fixture's 5 (its loop repeats the stored cycle,
    so n_cycle_lim = 3) and matches the reference's own 5-step run to the FP64
    parity bound; the mesh_tree entry equals the reference's own field by
    field."""
    import make_golden as M
    from kratos_b200.snapshot import Snapshot, to_lex_arrays, to_tree_arrays
    ref = os.path.join(ROOT, "oracle", "_ref", "kratos_ref")
    if not os.path.exists(ref):
        pytest.fail("%s is not built (make -f oracle/Makefile.ref REF=<kratos tree>)" % ref)
    c = [x for x in M.CASES if x[0] == name][0]
    _, problem, nb, n, steps, seed, gamma, extra, _ = c
    prefix = str(tmp_path / "h")
    par = tmp_path / "h.par"
    par.write_text(M.par_text(problem, nb, n, 3, seed, gamma, extra, prefix))
    subprocess.check_call([host_exe, str(par)], cwd=str(tmp_path), stdout=subprocess.DEVNULL)
    # the reference's own snapshot of the same mesh, for the tree bytes
    s_ref, _ = M.run_snapshots(ref, problem, nb, n, 1, seed, gamma, extra)
    s_host = Snapshot.read(prefix + "_00000.bin")
    assert _tree(s_host.data["mesh_tree"]) == _tree(s_ref.data["mesh_tree"])
    over = tmp_path / "more.par"
    over.write_text("[cycle]\nn_cycle_lim = 3\nprefix_output = %s\n" % str(tmp_path / "r"))
    subprocess.check_call([ref, prefix + "_00001.bin", str(over)], cwd=str(tmp_path), stdout=subprocess.DEVNULL)
    s = Snapshot.read(str(tmp_path / "r_00002.bin"))
    meta, g = G.load(name)
    assert int(s.array("cycle", "i")[0]) == 3
    assert abs(float(s.array("time")[0]) - meta["t"]) <= 1e-12 * meta["t"]
    u = to_tree_arrays(s)[2] if extra.get("regions") else to_lex_arrays(s, nb)[0]
    for k, e in enumerate(G.field_errors(u[..., :5], g["u1"][..., :5])):
        assert e <= TOL_FP64, "field %d rel L1 %.3e" % (k, e)

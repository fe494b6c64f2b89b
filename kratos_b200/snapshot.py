"""Reader and writer for Kratos binary snapshots.

Format (reference: src/io/binary/binary_io_base.cpp:101-118 save_header,
binary_io_types.h:58-78 b_info_t, utilities/data_transfer/serialize.h):
    char   (is_little_endian | sizeof(size_t))
    size_t header_size
    size_t n_entries, then per entry:
        size_t key_len, key bytes, size_t size, char unit_size, size_t offset
    bulk: entry data at header_size + offset
Entries are sorted by key (std::map order) and laid out in that order.
"""
import struct
from typing import Dict, Tuple

import numpy as np


class Snapshot:
    def __init__(self):
        self.data: Dict[str, bytes] = {}
        self.unit: Dict[str, int] = {}

    # ------------------------------------------------------------------ read
    @classmethod
    def read(cls, path: str) -> "Snapshot":
        snap = cls()
        with open(path, "rb") as f:
            raw = f.read()
        sst = raw[0]
        if not (sst & 1):
            raise ValueError("big-endian snapshots are not supported")
        if (sst & ~1) != 8:
            raise ValueError("snapshot written with sizeof(size_t) != 8")
        header_size, n = struct.unpack_from("<QQ", raw, 1)
        pos = 17
        for _ in range(n):
            (klen,) = struct.unpack_from("<Q", raw, pos)
            pos += 8
            key = raw[pos:pos + klen].decode("ascii")
            pos += klen
            size, usize, off = struct.unpack_from("<QbQ", raw, pos)
            pos += 17
            snap.data[key] = raw[header_size + off: header_size + off + size]
            snap.unit[key] = usize
        if pos != header_size:
            raise ValueError("inconsistent snapshot header")
        return snap

    # ----------------------------------------------------------------- write
    def write(self, path: str) -> None:
        keys = sorted(self.data)
        hdr = bytearray(struct.pack("<Q", len(keys)))
        off = 0
        for k in keys:
            kb = k.encode("ascii")
            size = len(self.data[k])
            hdr += struct.pack("<Q", len(kb)) + kb + struct.pack("<QbQ", size, self.unit[k], off)
            off += size
        header_size = 1 + 8 + len(hdr)
        with open(path, "wb") as f:
            f.write(bytes([1 | 8]))
            f.write(struct.pack("<Q", header_size))
            f.write(hdr)
            for k in keys:
                f.write(self.data[k])

    # --------------------------------------------------------------- access
    def keys(self):
        return self.data.keys()

    def array(self, key: str, kind: str = "f") -> np.ndarray:
        return np.frombuffer(self.data[key], dtype="<%s%d" % (kind, self.unit[key]))

    def put(self, key: str, arr, unit: int = None) -> None:
        a = np.ascontiguousarray(arr)
        self.data[key] = a.tobytes()
        self.unit[key] = int(unit if unit is not None else a.dtype.itemsize)

    def field(self, block: int, prefix: str) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(data[n_step?, z, y, x, n_int], n_cell, n_gh) of a dat_3d_t entry
        such as prefix='hydro_cons_' or 'field_bf_' (dat_3d.h:117-126)."""
        base = "block_%d|%s" % (block, prefix)
        n_int = int(self.array(base + "n_int", "i")[0])
        n_cell = self.array(base + "n_cell", "i").astype(int)
        n_gh = self.array(base + "n_gh", "i").astype(int)
        f = self.array(base + "field", "f")
        return f.reshape(n_cell[2], n_cell[1], n_cell[0], n_int), n_cell, n_gh


def block_ids(snap: Snapshot):
    """Block ids present in a snapshot, sorted."""
    ids = set()
    for k in snap.keys():
        if k.startswith("block_"):
            ids.add(int(k.split("|")[0][6:]))
    return sorted(ids)


def to_lex_arrays(snap: Snapshot, nb):
    """Gather the per-block conserved field (and face field, if present) of a
    single-level snapshot into arrays in lexicographic block order (x fastest):
    u [nblk, n2, n1, n0, n_int], bf [nblk, n2+5, n1+5, n0+5, 3] or None.
    Block positions come from the `i_logic` entry (block.cpp:18-39)."""
    nblk = nb[0] * nb[1] * nb[2]
    u_out, bf_out = [None] * nblk, [None] * nblk
    for bid in block_ids(snap):
        il = snap.array("block_%d|i_logic" % bid, "i")
        lex = int(il[0] + nb[0] * (il[1] + nb[1] * il[2]))
        u, _, _ = snap.field(bid, "hydro_cons_")
        u_out[lex] = u
        if ("block_%d|field_bf_field" % bid) in snap.data:
            bf, _, _ = snap.field(bid, "field_bf_")
            bf_out[lex] = bf
    u = np.stack(u_out)
    bf = np.stack(bf_out) if bf_out[0] is not None else None
    return u, bf


def to_tree_arrays(snap: Snapshot):
    """Gather a (possibly refined) snapshot's blocks in tree order: level by
    level, lexicographic (x fastest) inside a level, from each block's `level`
    and `i_logic` entries.  Returns (level [nblk], reg [nblk, 3], u, bf or None)
    with u and bf shaped as in to_lex_arrays."""
    rows = []
    for bid in block_ids(snap):
        lv = int(snap.array("block_%d|level" % bid, "i")[0])
        il = snap.array("block_%d|i_logic" % bid, "i").astype(int)
        rows.append(((lv, int(il[2]), int(il[1]), int(il[0])), bid))
    rows.sort()
    level = np.array([r[0][0] for r in rows], dtype=np.int32)
    reg = np.array([[r[0][3], r[0][2], r[0][1]] for r in rows], dtype=np.int32).reshape(-1, 3)
    u = np.stack([snap.field(bid, "hydro_cons_")[0] for _, bid in rows])
    bf = None
    if rows and ("block_%d|field_bf_field" % rows[0][1]) in snap.data:
        bf = np.stack([snap.field(bid, "field_bf_")[0] for _, bid in rows])
    return level, reg, u, bf


# ---------------------------------------------------------------- block ids
# The reference numbers blocks along a Hilbert curve (meshgen.cpp:188-243
# dist_fractal), drawn by an L-system turtle (utilities/l_system/l_system.cpp):
# the 3-D rule below, 'F' a unit step along the turtle's x axis, the other
# symbols quarter turns (+ - about z, & ^ about y, > < about x) composed on the
# right.  A refined node is replaced by its children in the order of the same
# curve one level down, placed where the curve's bounding box meets the node's
# children.  Restated here (turns as integer rotation matrices) so that a
# snapshot names its blocks block_<id> as the reference would on restart.
_HILBERT_3D = "^<XF^<XFX-F^>>XFX&F+>>XFX-F>X->"


def _turn(axis, sgn):
    m = np.eye(3, dtype=np.int64)
    a1, a2 = (axis + 1) % 3, (axis + 2) % 3
    m[a1, a1] = m[a2, a2] = 0
    m[a2, a1] = sgn
    m[a1, a2] = -sgn
    return m


_TURNS = {"+": _turn(2, 1), "-": _turn(2, -1), "&": _turn(1, 1), "^": _turn(1, -1),
          ">": _turn(0, 1), "<": _turn(0, -1)}


def hilbert_ids(levels, regs, nb):
    """Global block ids (the reference's id_g) of the blocks of a 3-D mesh:
    levels[b], regs[b] (logical position at that level), nb root blocks per
    axis.  Returns (ids [nblk], tree) with tree the refined (masked) nodes as
    a set of (level, x0, x1, x2)."""
    leaves = {(int(l), *map(int, r)): b for b, (l, r) in enumerate(zip(levels, regs))}
    masked = set()
    for (l, x0, x1, x2) in leaves:
        x = [x0, x1, x2]
        for up in range(l, 0, -1):
            x = [(v if v > 0 else v - 1) // 2 if v < 0 else v // 2 for v in x]
            masked.add((up - 1, *x))
    n_base = max(nb) - 1
    l_base = 0
    while n_base > 1:
        n_base >>= 1
        l_base += 1
    l_base += 1 if max(nb) > 1 else 1
    ids = np.full(len(levels), -1, np.int64)
    state = {"lim": l_base, "reg": False, "next": 0}
    nodes = []

    def rule_ref(x, l):
        key = (l - l_base, *x)
        if key in masked:
            return True
        if key in leaves:
            ids[leaves[key]] = state["next"]
            state["next"] += 1
        return False

    def step(t):
        if t["l"] >= state["lim"]:
            refine(t)
            return
        for ch in _HILBERT_3D:
            if ch == "X":
                t["l"] += 1
                step(t)
                t["l"] -= 1
            elif ch == "F":
                t["x"] = [t["x"][a] + int(t["m"][a, 0]) for a in range(3)]
            else:
                t["m"] = t["m"] @ _TURNS[ch]

    def refine(t):
        if state["reg"] or not rule_ref(t["x"], t["l"]):
            nodes.append(list(t["x"]))
            return
        start = len(nodes)
        state["reg"] = True
        state["lim"] += 1
        dry = {"l": t["l"], "x": [0, 0, 0], "m": t["m"].copy()}
        step(dry)
        dx = [0, 0, 0]
        for p in nodes[start:]:
            dx = [min(dx[a], p[a]) for a in range(3)]
        del nodes[start:]
        sub = {"l": t["l"], "x": [2 * t["x"][a] - dx[a] for a in range(3)], "m": t["m"].copy()}
        state["reg"] = False
        step(sub)
        state["lim"] -= 1

    step({"l": 0, "x": [0, 0, 0], "m": np.eye(3, dtype=np.int64)})
    return ids, masked

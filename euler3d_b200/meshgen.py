"""Seeded synthetic workloads for the euler3D residual/update path.

The reference solver reads SU2-dialect block files plus a ``.top`` topology file
and a positional input deck.  This module writes exactly those three formats so
that the reference CPU solver and this package consume the same inputs.

File formats follow the reference readers:

* block file: ``ConcreteBlockBuilder::preReadMyBlock`` / ``readMyBlock``
  (BlockBuilder/src/ConcreteBlockBuilder.cpp:22-225, :227-495): ``NDIME=``, blank,
  ``NPOIN=`` + coordinates without index, blank, ``NELEM=`` + ``10 a b c d`` rows,
  blank, ``NMARK=`` + per marker ``MARKER_TAG=``/``MARKER_ELEMS=`` + ``5 a b c`` rows.
  Physical markers (WALL/FARFIELD/SYMMETRY) precede CONNEXION markers because the
  reference only applies the first ``n_real_boundaries`` markers
  (ConcreteBlockBuilder.cpp:107-108,143-149; Updater.cpp:84-87).
* topology file: ``CompleteMesh::getBlockFileName`` / ``InitializeMyBlocks``
  (DataStructure/src/CompleteMesh.cpp:45-76, :170-292).
* input deck: ``Interface::readInputFile`` (Solver/src/Interface.cpp:14-237).

The bump channel is the unit box split into n^3 hexahedra, each cut into six
tetrahedra along its main diagonal (Kuhn / Freudenthal split, conforming between
neighbours).  The lower wall y=0 carries a Gaussian bump
h(x) = height * exp(-(x-0.5)^2 / (2 sigma^2)); nodes move as y <- y + h(x)(1-y).
Multi-block cases cut the box into x-slabs of whole hexahedron layers.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

# Six tetrahedra of the Kuhn split of a unit cube: corner bit pattern
# (bit0 = +x, bit1 = +y, bit2 = +z).  Each tetrahedron walks from corner 0 to
# corner 7 adding one axis at a time, one tetrahedron per axis permutation.
_KUHN_TETS = np.array(
    [
        [0, 1, 3, 7],  # x, y, z
        [0, 1, 5, 7],  # x, z, y
        [0, 2, 3, 7],  # y, x, z
        [0, 2, 6, 7],  # y, z, x
        [0, 4, 5, 7],  # z, x, y
        [0, 4, 6, 7],  # z, y, x
    ],
    dtype=np.int64,
)
# Tetrahedron faces as local node triples (any fixed choice works: the face
# builder only compares node sets; orientation is fixed later by geometry).
_TET_FACES = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]], dtype=np.int64)


@dataclass
class BumpChannel:
    """A tetrahedral bump channel: global nodes, tetrahedra and hex layout."""

    n: int
    nodes: np.ndarray  # (P, 3) float64
    tets: np.ndarray  # (E, 4) int64, global node ids
    hex_i: np.ndarray  # (E,) x-layer index of the parent hexahedron
    node_ijk: np.ndarray  # (P, 3) integer lattice coordinates


def bump_channel(n: int, height: float = 0.05, sigma: float = 0.1, ytop: float = 1.0) -> BumpChannel:
    """Build the n x n x n hexahedron box [0,1] x [0,ytop] x [0,1] split into 6 n^3 tetrahedra."""
    m = n + 1
    ii, jj, kk = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    # node id = i + m*(j + m*k)  (x fastest)
    ijk = np.stack([ii.transpose(2, 1, 0).ravel(), jj.transpose(2, 1, 0).ravel(),
                    kk.transpose(2, 1, 0).ravel()], axis=1).astype(np.int64)
    x = ijk[:, 0] / n
    y = ijk[:, 1] / n
    z = ijk[:, 2] / n
    if ytop != 1.0:
        y = y * ytop
    h = height * np.exp(-((x - 0.5) ** 2) / (2.0 * sigma * sigma))
    y = y + h * (1.0 - y / ytop)
    nodes = np.stack([x, y, z], axis=1)

    hi, hj, hk = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    hi = hi.transpose(2, 1, 0).ravel()
    hj = hj.transpose(2, 1, 0).ravel()
    hk = hk.transpose(2, 1, 0).ravel()  # hex id = i + n*(j + n*k)
    base = hi + m * (hj + m * hk)
    corner = np.array([(b & 1) + m * (((b >> 1) & 1) + m * ((b >> 2) & 1)) for b in range(8)],
                      dtype=np.int64)
    hex_nodes = base[:, None] + corner[None, :]  # (H, 8)
    tets = hex_nodes[:, _KUHN_TETS].reshape(-1, 4)  # 6 tets per hex, hex-major
    hex_i = np.repeat(hi, 6)
    return BumpChannel(n=n, nodes=nodes, tets=tets, hex_i=hex_i, node_ijk=ijk)


@dataclass
class BlockMesh:
    """One SU2 block: local nodes, cells and ordered boundary markers."""

    nodes: np.ndarray  # (P_b, 3)
    tets: np.ndarray  # (E_b, 4) local node ids
    markers: list = field(default_factory=list)  # [(tag, (k,3) local node ids)]
    # CONNEXION bookkeeping: per connexion marker (origin block, origin local cell ids)
    connexions: list = field(default_factory=list)
    global_cell: np.ndarray | None = None  # (E_b,) global tet ids

    @property
    def n_real(self) -> int:
        return int(self.tets.shape[0])

    @property
    def n_physical_ghosts(self) -> int:
        return int(sum(len(f) for t, f in self.markers if t != "CONNEXION"))


def slab_blocks(mesh: BumpChannel, n_blocks: int = 1, sides: str = "farfield") -> list[BlockMesh]:
    """Cut the channel into ``n_blocks`` x-slabs of whole hexahedron layers.

    Every block lists WALL (y=0) then FARFIELD (other outer sides) then one
    CONNEXION marker per neighbouring slab (lower x first).  With
    ``sides="symmetry"`` the z=0 and z=1 planes form a SYMMETRY marker (after
    FARFIELD) instead of being farfield, and with ``sides="channel"`` the top
    plane joins them: the inlet and outlet are then the only farfield faces.
    Farfield faces the flow runs along switch between the inflow and outflow
    states with the sign of u.n, which keeps the residual from dropping below
    a few orders; a channel has none.  Ghost elements of a
    marker follow ascending (owner cell, local face).  The connexion origin ids
    are the neighbour block's local cell ids across each interface face, in the
    same order, which is what the topology file records.
    """
    n = mesh.n
    if n % n_blocks != 0:
        raise ValueError(f"{n} hexahedron layers do not split into {n_blocks} equal slabs")
    layers = n // n_blocks
    ijk = mesh.node_ijk.astype(np.int32)
    n_tets = mesh.tets.shape[0]
    faces = mesh.tets[:, _TET_FACES].reshape(-1, 3)  # (4E, 3) ordered by tet, local face
    owner = np.repeat(np.arange(n_tets), 4)

    def plane(axis):
        v = ijk[faces, axis]  # (4E, 3)
        lo = v.min(axis=1)
        return np.where(lo == v.max(axis=1), lo, -1)

    px, py, pz = plane(0), plane(1), plane(2)
    if sides not in ("farfield", "symmetry", "channel"):
        raise ValueError(f"sides must be 'farfield', 'symmetry' or 'channel', not {sides!r}")
    wall = py == 0
    zside = (pz == 0) | (pz == n)
    top = py == n
    far = (px == 0) | (px == n)
    if sides == "farfield":
        far = far | top | zside
        sym = np.zeros_like(far)
    elif sides == "symmetry":
        far = far | top
        sym = zside & ~far
    else:
        sym = (zside | top) & ~far
    iface = (px > 0) & (px < n) & (px % layers == 0)
    keep = np.nonzero(wall | far | sym | iface)[0]  # small: only faces on planes of interest
    faces, owner = faces[keep], owner[keep]
    wall, far, sym, iface, px = wall[keep], far[keep], sym[keep], iface[keep], px[keep]

    tet_block = mesh.hex_i // layers
    local_id = np.empty(n_tets, dtype=np.int64)
    for b in range(n_blocks):
        sel = np.nonzero(tet_block == b)[0]
        local_id[sel] = np.arange(sel.size)
    fblock = tet_block[owner]

    # pair interface faces: each sorted node triple occurs once on either side
    ii = np.nonzero(iface)[0]
    key = np.sort(faces[ii], axis=1).astype(np.int64)
    P = np.int64(mesh.nodes.shape[0] + 1)
    packed = (key[:, 0] * P + key[:, 1]) * P + key[:, 2]
    order = np.argsort(packed, kind="stable")
    if ii.size:
        ps = packed[order]
        if not (ii.size % 2 == 0 and np.all(ps[0::2] == ps[1::2])):
            raise RuntimeError("slab interface faces do not pair up")
    mate = np.empty(ii.size, dtype=np.int64)
    mate[order[0::2]] = order[1::2]
    mate[order[1::2]] = order[0::2]
    mate_owner = np.full(faces.shape[0], -1, dtype=np.int64)
    mate_owner[ii] = owner[ii[mate]]

    blocks = []
    for b in range(n_blocks):
        cells = np.nonzero(tet_block == b)[0]
        used = np.unique(mesh.tets[cells].ravel())
        g2l = -np.ones(mesh.nodes.shape[0], dtype=np.int64)
        g2l[used] = np.arange(used.size)
        blk = BlockMesh(nodes=mesh.nodes[used], tets=g2l[mesh.tets[cells]], global_cell=cells)
        in_b = fblock == b
        blk.markers.append(("WALL", g2l[faces[in_b & wall]]))
        blk.markers.append(("FARFIELD", g2l[faces[in_b & far]]))
        if sides != "farfield":
            blk.markers.append(("SYMMETRY", g2l[faces[in_b & sym]]))
        for nb, pl in ((b - 1, b * layers), (b + 1, (b + 1) * layers)):
            if nb < 0 or nb >= n_blocks:
                continue
            mine = np.nonzero(in_b & iface & (px == pl))[0]
            blk.markers.append(("CONNEXION", g2l[faces[mine]]))
            blk.connexions.append((nb, local_id[mate_owner[mine]]))
        blocks.append(blk)
    return blocks


def _fast_int_rows(prefix: str, arr: np.ndarray) -> str:
    # vectorised integer formatting: far faster than per-row % for millions of rows
    strs = [arr[:, c].astype(str) for c in range(arr.shape[1])]
    out = strs[0]
    for s in strs[1:]:
        out = np.char.add(np.char.add(out, " "), s)
    if prefix:
        out = np.char.add(prefix, out)
    return "\n".join(out.tolist()) + "\n"


def _fmt_coords(nodes: np.ndarray) -> str:
    # %.17g round-trips every double exactly through sscanf("%lf")
    return "".join("%.17g %.17g %.17g\n" % (a, b, c) for a, b, c in nodes.tolist())


def write_su2(path: str, blk: BlockMesh) -> None:
    """Write one block in the SU2 dialect the reference reader accepts."""
    parts = ["NDIME= 3\n", "\n", f"NPOIN= {blk.nodes.shape[0]}\n", _fmt_coords(blk.nodes), "\n",
             f"NELEM= {blk.tets.shape[0]}\n", _fast_int_rows("10 ", blk.tets), "\n",
             f"NMARK= {len(blk.markers)}\n"]
    for tag, faces in blk.markers:
        parts.append(f"MARKER_TAG= {tag}\n")
        parts.append(f"MARKER_ELEMS= {faces.shape[0]}\n")
        parts.append(_fast_int_rows("5 ", faces) if faces.shape[0] else "")
    with open(path, "w") as f:
        f.write("".join(parts))


def write_topology(path: str, block_files: list[str], blocks: list[BlockMesh]) -> None:
    """Write the ``.top`` topology in the layout CompleteMesh.cpp:170-292 reads."""
    lines = [f"NBLOCK= {len(blocks)}"]
    lines += list(block_files)
    for b, blk in enumerate(blocks):
        lines.append(f"Block= {b}")
        lines.append(f"GhostCount= {blk.n_real + blk.n_physical_ghosts}")
        lines.append(f"Nconnexion= {len(blk.connexions)}")
        for origin_block, origin_cells in blk.connexions:
            lines.append(f"Nmark= {origin_block}")
            lines.append(f"Nelems= {origin_cells.size}")
            lines.extend(str(int(c)) for c in origin_cells)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


@dataclass
class Deck:
    """The positional input deck fields (Solver/src/Interface.cpp:35-198)."""

    topology: str
    cfl: float = 1.5
    gamma: float = 1.4
    aoa_deg: float = 0.0
    stages: int = 5
    mach: float = 0.5
    cmac: float = 1.0
    max_iter: int = 500
    criterion: float = -15.0
    smoothing: int = 0
    flux: str = "roe"
    order: int = 1
    gradient: str = "leastsquares"
    limiter: str = "venkatakrishnan"
    omega: float = 2.16e-16
    k: float = 5.0


def write_deck(path: str, d: Deck) -> None:
    """Write a deck with the same 32-line layout as the reference's input files."""
    txt = (
        "MESH\n"
        "topologyfilename\n"
        f"{d.topology}\n"
        "INPUT\n"
        "cfl gamma angleattackdeg\n"
        f"{d.cfl!r} {d.gamma!r} {d.aoa_deg!r}\n"
        "rkstage mach cmac\n"
        f"{d.stages} {d.mach!r} {d.cmac!r}\n"
        "nbitermax convcriterion\n"
        f"{d.max_iter} {d.criterion!r}\n"
        "residual smoothing (0-no 1-yes)\n"
        f"{d.smoothing}\n"
        "fluxscheme schemeorder\n"
        f"{d.flux} {d.order}\n"
        "gradient limiter\n"
        f"{d.gradient} {d.limiter}\n"
        "omega k\n"
        f"{d.omega!r} {d.k!r}\n"
        "EXECUTABLE (0-no 1-yes)\n"
        "build execute\n"
        "0 1\n"
        "OUTPUT (0-no 1-yes)\n"
        "clalpha cdalpha cmalpha\n"
        "0 0 0\n"
        "coefficientsconv cdconv cmconv residualconv\n"
        "1 1 1 1\n"
        "cpxc machcontour cpcontour\n"
        "0 0 0\n"
        "slicecp\n"
        "0\n"
        "axis xcoord ycoord zcoord\n"
        "x 1.00 1.00 1.00\n"
    )
    with open(path, "w") as f:
        f.write(txt)


def hex_channel(n: int, nz: int = 1, height: float = 0.05, sigma: float = 0.1) -> BlockMesh:
    """A 2.5-D hexahedron channel: n x n x nz hexes (SU2 type 12), WALL at y=0,
    SYMMETRY at z=0 and z=1, FARFIELD elsewhere.  Exercises quadrilateral
    faces and symmetry ghosts (the reference's NACA test mesh has the same
    marker mix)."""
    m = n + 1
    ii, jj, kk = np.meshgrid(np.arange(m), np.arange(m), np.arange(nz + 1), indexing="ij")
    ijk = np.stack([ii.transpose(2, 1, 0).ravel(), jj.transpose(2, 1, 0).ravel(),
                    kk.transpose(2, 1, 0).ravel()], axis=1).astype(np.int64)
    x = ijk[:, 0] / n
    y = ijk[:, 1] / n
    z = ijk[:, 2] / nz
    h = height * np.exp(-((x - 0.5) ** 2) / (2.0 * sigma * sigma))
    nodes = np.stack([x, y + h * (1.0 - y), z], axis=1)

    def nid(i, j, k):
        return i + m * (j + m * k)

    hi, hj, hk = np.meshgrid(np.arange(n), np.arange(n), np.arange(nz), indexing="ij")
    hi, hj, hk = (a.transpose(2, 1, 0).ravel() for a in (hi, hj, hk))
    # SU2 hexahedron order: bottom quad (z-) counter-clockwise, then top quad
    hexes = np.stack([nid(hi, hj, hk), nid(hi + 1, hj, hk), nid(hi + 1, hj + 1, hk), nid(hi, hj + 1, hk),
                      nid(hi, hj, hk + 1), nid(hi + 1, hj, hk + 1), nid(hi + 1, hj + 1, hk + 1),
                      nid(hi, hj + 1, hk + 1)], axis=1)
    wall = [(nid(i, 0, k), nid(i + 1, 0, k), nid(i + 1, 0, k + 1), nid(i, 0, k + 1))
            for k in range(nz) for i in range(n)]
    sym = [(nid(i, j, kz), nid(i + 1, j, kz), nid(i + 1, j + 1, kz), nid(i, j + 1, kz))
           for kz in (0, nz) for j in range(n) for i in range(n)]
    far = [(nid(i, n, k), nid(i + 1, n, k), nid(i + 1, n, k + 1), nid(i, n, k + 1)) for k in range(nz) for i in range(n)]
    far += [(nid(ie, j, k), nid(ie, j + 1, k), nid(ie, j + 1, k + 1), nid(ie, j, k + 1))
            for ie in (0, n) for k in range(nz) for j in range(n)]
    blk = BlockMesh(nodes=nodes, tets=hexes)
    blk.markers = [("WALL", np.array(wall)), ("SYMMETRY", np.array(sym)), ("FARFIELD", np.array(far))]
    return blk


def write_su2_hex(path: str, blk: BlockMesh) -> None:
    """Like write_su2 for hexahedra (type 12) with quadrilateral markers (type 9)."""
    parts = ["NDIME= 3\n", "\n", f"NPOIN= {blk.nodes.shape[0]}\n", _fmt_coords(blk.nodes), "\n",
             f"NELEM= {blk.tets.shape[0]}\n", _fast_int_rows("12 ", blk.tets), "\n",
             f"NMARK= {len(blk.markers)}\n"]
    for tag, faces in blk.markers:
        parts.append(f"MARKER_TAG= {tag}\n")
        parts.append(f"MARKER_ELEMS= {faces.shape[0]}\n")
        parts.append(_fast_int_rows("9 ", faces) if faces.shape[0] else "")
    with open(path, "w") as f:
        f.write("".join(parts))


def write_hex_case(directory: str, n: int, nz: int = 1, prefix: str = "hexchan", deck: Deck | None = None) -> str:
    """Single-block hexahedron channel case; returns the deck path."""
    os.makedirs(directory, exist_ok=True)
    blk = hex_channel(n, nz)
    write_su2_hex(os.path.join(directory, prefix + ".su2"), blk)
    write_topology(os.path.join(directory, prefix + ".top"), [prefix + ".su2"], [blk])
    d = deck or Deck(topology=prefix + ".top")
    d.topology = prefix + ".top"
    deck_path = os.path.join(directory, prefix + ".deck")
    write_deck(deck_path, d)
    os.makedirs(os.path.join(directory, "bin"), exist_ok=True)
    return deck_path


def write_case(directory: str, n: int, n_blocks: int = 1, prefix: str = "bump",
               deck: Deck | None = None, height: float = 0.05, sigma: float = 0.1, sides: str = "farfield",
               ytop: float = 1.0) -> str:
    """Generate a bump-channel case in ``directory``; return the deck path.

    File names inside the topology and deck are relative, so the case runs
    from ``directory`` as the working directory (the reference opens them
    relative to its CWD).
    """
    os.makedirs(directory, exist_ok=True)
    mesh = bump_channel(n, height=height, sigma=sigma, ytop=ytop)
    blocks = slab_blocks(mesh, n_blocks, sides)
    files = []
    for b, blk in enumerate(blocks):
        name = f"{prefix}_B{b}.su2" if n_blocks > 1 else f"{prefix}.su2"
        write_su2(os.path.join(directory, name), blk)
        files.append(name)
    top = f"{prefix}.top"
    write_topology(os.path.join(directory, top), files, blocks)
    d = deck or Deck(topology=top)
    d.topology = top
    deck_path = os.path.join(directory, f"{prefix}.deck")
    write_deck(deck_path, d)
    os.makedirs(os.path.join(directory, "bin"), exist_ok=True)
    return deck_path

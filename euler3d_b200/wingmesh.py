"""Synthetic swept trapezoidal wing in a tetrahedral farfield box.

The wing: NACA 4-digit symmetric section (the published thickness
polynomial, closed trailing edge), thickness ratio 12 %, leading-edge sweep
30 deg, taper 0.56, root chord 1, semi-span 1.5, no twist; chord along +x,
thickness along +y (the reference's lift axis), span along +z with the root
in the symmetry plane z = 0.  The box [-4, 6] x [-5, 5] x [0, 4] is farfield
except its z = 0 face (SYMMETRY).

The tetrahedra are the Delaunay triangulation (scipy's Qhull) of a seeded,
wall-graded point cloud: points on the wing surface (cosine-clustered
chordwise), geometric layers along the surface normals, volume points whose
distance to the wing is log-uniform, and points on the box faces.  Tetrahedra
whose centroid lies inside the wing are removed; the faces they leave exposed
form the WALL marker.

Cells are split into x-slab topology blocks of equal cell count, and each
block's cells (and nodes) are ordered along a Morton (Z-order) curve of their
centroids, so that neighbouring cells sit close in memory; the reference
reads cells in file order, so the order is part of the mesh, not a solver
change.  Everything goes through the reference's file formats (SU2 blocks,
.top topology, deck).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

from . import meshgen as mg

_TET_FACES = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]], dtype=np.int64)


@dataclass
class WingSpec:
    root_chord: float = 1.0
    taper: float = 0.56
    sweep_deg: float = 30.0
    semi_span: float = 1.5
    thickness: float = 0.12
    box: tuple = (-4.0, 6.0, -5.0, 5.0, 0.0, 4.0)


def naca_half_thickness(s: np.ndarray, t: float, closed: bool = True) -> np.ndarray:
    """NACA 4-digit thickness distribution, chord 1: the closed trailing-edge
    variant (last coefficient 0.1036) or the published one (0.1015, a blunt
    trailing edge 0.021 t thick)."""
    s = np.clip(s, 0.0, 1.0)
    a4 = 0.1036 if closed else 0.1015
    return 5.0 * t * (0.2969 * np.sqrt(s) - 0.1260 * s - 0.3516 * s ** 2 + 0.2843 * s ** 3 - a4 * s ** 4)


def _le_chord(w: WingSpec, z):
    eta = np.clip(z / w.semi_span, 0.0, 1.0)
    return z * np.tan(np.radians(w.sweep_deg)), w.root_chord * (1.0 - (1.0 - w.taper) * eta)


def inside_wing(w: WingSpec, p: np.ndarray) -> np.ndarray:
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    xle, c = _le_chord(w, z)
    s = (x - xle) / c
    ok = (z >= 0.0) & (z <= w.semi_span) & (s >= 0.0) & (s <= 1.0)
    return ok & (np.abs(y) < c * naca_half_thickness(s, w.thickness))


def _surface(w: WingSpec, s: np.ndarray, eta: np.ndarray, upper: np.ndarray) -> np.ndarray:
    z = eta * w.semi_span
    xle, c = _le_chord(w, z)
    y = c * naca_half_thickness(s, w.thickness)
    return np.stack([xle + s * c, np.where(upper, y, -y), z], axis=1)


def _normals(w: WingSpec, s, eta, up):
    h = 1e-5
    ds = _surface(w, np.clip(s + h, 0, 1), eta, up) - _surface(w, np.clip(s - h, 0, 1), eta, up)
    de = _surface(w, s, np.clip(eta + h, 0, 1), up) - _surface(w, s, np.clip(eta - h, 0, 1), up)
    nrm = np.cross(ds, de)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True) + 1e-300
    return nrm * np.where((nrm[:, 1] > 0) == up, 1.0, -1.0)[:, None]  # outward: away from the chord plane


def _jittered_grid(rng, ns: int, ne: int, s_lo=0.0):
    """Chordwise cosine-clustered x spanwise uniform grid, jittered by a quarter cell."""
    i = (np.arange(ns) + 0.5 + rng.uniform(-0.25, 0.25, (ne, ns))) / ns
    s = s_lo + (1.0 - s_lo) * 0.5 * (1.0 - np.cos(np.pi * i))
    e = (np.arange(ne)[:, None] + rng.uniform(-0.25, 0.25, (ne, ns))) / max(ne - 1, 1)
    return s.ravel(), np.clip(e, 0.0, 1.0).ravel()


def point_cloud(w: WingSpec, n_points: int, seed: int) -> np.ndarray:
    """Seeded wall-graded points: a jittered surface grid on both sides of the
    wing (spacing h), layers along the surface normals at offsets 0.5 h x 1.2^k
    whose in-layer spacing grows with the offset (near-isotropic cells), volume
    points at log-uniform distance from the wing, and jittered grids on the box
    faces."""
    rng = np.random.default_rng(seed)
    x0, x1, y0, y1, z0, z1 = w.box
    c_avg = w.root_chord * (1.0 + w.taper) / 2.0
    n_side = int(0.03 * n_points)  # surface points per side
    ne = max(4, int(np.sqrt(n_side * w.semi_span / c_avg)))
    ns = max(4, n_side // ne)
    hs = c_avg / ns * 1.2
    pts = []
    for up in (True, False):
        s_, e_ = _jittered_grid(rng, ns, ne)
        pts.append(_surface(w, s_, e_, np.full(s_.size, up)))
    # tip cap: points on the z = semi-span plane inside the section
    nc = max(4, ns // 2)
    s_, f_ = _jittered_grid(rng, nc, max(3, int(0.12 * ns)))
    cap = _surface(w, s_, np.ones(s_.size), np.ones(s_.size, bool))
    cap[:, 1] *= 2.0 * f_ - 1.0
    pts.append(cap)
    # normal layers
    d, k = 0.5 * hs, 0
    budget = int(0.30 * n_points)
    while d < 0.25 and budget > 0:
        hk = max(hs, 0.9 * d)
        nsk, nek = max(4, int(ns * hs / hk)), max(4, int(ne * hs / hk))
        for up in (True, False):
            s_, e_ = _jittered_grid(rng, nsk, nek, s_lo=1e-4)
            u_ = np.full(s_.size, up)
            pts.append(_surface(w, s_, e_, u_) + _normals(w, s_, e_, u_) * (d * rng.uniform(0.9, 1.1, s_.size))[:, None])
            budget -= s_.size
        d *= 1.2
        k += 1
    n_face = int(0.004 * n_points)
    n_vol = max(0, n_points - sum(p.shape[0] for p in pts) - 6 * n_face - 8)
    # volume: log-uniform distance from a random surface point, random direction
    base = _surface(w, 0.5 * (1.0 - np.cos(np.pi * rng.uniform(0, 1, n_vol))), rng.uniform(0, 1, n_vol),
                    rng.uniform(0, 1, n_vol) < 0.5)
    r = np.exp(rng.uniform(np.log(0.25), np.log(8.0), n_vol))
    dv = rng.normal(size=(n_vol, 3))
    dv /= np.linalg.norm(dv, axis=1, keepdims=True)
    pts.append(base + dv * r[:, None])
    # box faces (jittered grids) and corners
    m = max(4, int(np.sqrt(n_face)))
    for axis, lo, hi in ((0, x0, x1), (1, y0, y1), (2, z0, z1)):
        other = [a for a in range(3) if a != axis]
        los, his = [w.box[2 * a] for a in other], [w.box[2 * a + 1] for a in other]
        g = (np.arange(m)[:, None] + 0.5 + rng.uniform(-0.3, 0.3, (m, m))) / m
        g2 = (np.arange(m)[None, :] + 0.5 + rng.uniform(-0.3, 0.3, (m, m))) / m
        for val in (lo, hi):
            q = np.zeros((m * m, 3))
            q[:, axis] = val
            q[:, other[0]] = los[0] + (his[0] - los[0]) * g.ravel()
            q[:, other[1]] = los[1] + (his[1] - los[1]) * g2.ravel()
            pts.append(q)
    pts.append(np.array([[a, b, c] for a in (x0, x1) for b in (y0, y1) for c in (z0, z1)], dtype=float))
    n_wall = sum(p.shape[0] for p in pts[:3])
    pts = np.concatenate(pts)
    keep = (pts[:, 0] >= x0) & (pts[:, 0] <= x1) & (pts[:, 1] >= y0) & (pts[:, 1] <= y1) & (pts[:, 2] >= z0) & \
           (pts[:, 2] <= z1)
    # off-wall points must lie outside the wing; points on the wall stay
    off = np.ones(pts.shape[0], bool)
    off[n_wall:] = ~inside_wing(w, pts[n_wall:])
    return np.unique(pts[keep & off], axis=0)


def _morton(p: np.ndarray, lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    q = ((p - lo) / np.maximum(hi - lo, 1e-300) * 1023.999).astype(np.uint64)
    code = np.zeros(p.shape[0], dtype=np.uint64)
    for bit in range(10):
        for a in range(3):
            code |= ((q[:, a] >> np.uint64(bit)) & np.uint64(1)) << np.uint64(3 * bit + a)
    return code


def wing_mesh(w: WingSpec, n_points: int, seed: int = 5):
    """Nodes and tetrahedra of the wing domain (interior tetrahedra removed)."""
    from scipy.spatial import Delaunay

    pts = point_cloud(w, n_points, seed)
    tri = Delaunay(pts)
    tets = tri.simplices.astype(np.int64)
    cen = pts[tets].mean(axis=1)
    tets = tets[~inside_wing(w, cen)]
    vol = np.einsum("ij,ij->i", np.cross(pts[tets[:, 1]] - pts[tets[:, 0]], pts[tets[:, 2]] - pts[tets[:, 0]]),
                    pts[tets[:, 3]] - pts[tets[:, 0]])
    if np.any(vol == 0.0):  # slivers next to the wall stay (removing one would open a hole)
        raise RuntimeError("the triangulation has flat tetrahedra; change the seed or the point count")
    return pts, tets


def _box_kinds(w: WingSpec, pts: np.ndarray):
    """Boundary faces of the Delaunay box: SYMMETRY on z = 0, FARFIELD on the
    other box faces, WALL for the rest (the faces the removed tets exposed)."""
    x0, x1, y0, y1, z0, z1 = w.box

    def kinds(fnodes: np.ndarray):
        fx = pts[fnodes]  # (faces, 3 nodes, 3)
        on = {}
        for name, axis, val in (("x0", 0, x0), ("x1", 0, x1), ("y0", 1, y0), ("y1", 1, y1), ("z0", 2, z0),
                                ("z1", 2, z1)):
            on[name] = np.all(fx[:, :, axis] == val, axis=1)
        sym = on["z0"]
        far = ~sym & (on["x0"] | on["x1"] | on["y0"] | on["y1"] | on["z1"])
        return sym, far
    return kinds


def split_blocks(w: WingSpec, pts: np.ndarray, tets: np.ndarray, n_blocks: int, kinds=None) -> list[mg.BlockMesh]:
    """x-slab blocks of equal cell count, Morton-ordered cells, markers
    WALL, FARFIELD, SYMMETRY, then one CONNEXION per neighbouring block.
    ``kinds(face_nodes) -> (symmetry, farfield)`` labels the boundary faces
    (the rest are WALL); by default the faces of the Delaunay box."""
    kinds = kinds or _box_kinds(w, pts)
    cen = pts[tets].mean(axis=1)
    order = np.argsort(cen[:, 0], kind="stable")
    blk_of = np.empty(tets.shape[0], dtype=np.int64)
    blk_of[order] = (np.arange(tets.shape[0]) * n_blocks) // tets.shape[0]
    # Morton order inside each block
    code = _morton(cen, pts.min(axis=0), pts.max(axis=0))
    perm = np.lexsort((code, blk_of))
    tets, blk_of = tets[perm], blk_of[perm]
    local = np.empty(tets.shape[0], dtype=np.int64)
    starts = np.searchsorted(blk_of, np.arange(n_blocks + 1))
    for b in range(n_blocks):
        local[starts[b]:starts[b + 1]] = np.arange(starts[b + 1] - starts[b])
    faces = tets[:, _TET_FACES].reshape(-1, 3)
    owner = np.repeat(np.arange(tets.shape[0]), 4)
    key = np.sort(faces, axis=1)
    P = np.int64(pts.shape[0] + 1)
    packed = (key[:, 0] * P + key[:, 1]) * P + key[:, 2]
    srt = np.argsort(packed, kind="stable")
    ps = packed[srt]
    same_next = np.zeros(ps.size, bool)
    same_next[:-1] = ps[:-1] == ps[1:]
    pair_first = np.nonzero(same_next)[0]
    mate = np.full(faces.shape[0], -1, dtype=np.int64)
    mate[srt[pair_first]] = srt[pair_first + 1]
    mate[srt[pair_first + 1]] = srt[pair_first]
    bnd = mate < 0
    bidx = np.nonzero(bnd)[0]
    sym = np.zeros(faces.shape[0], bool)
    far = np.zeros(faces.shape[0], bool)
    wall = np.zeros(faces.shape[0], bool)
    sym[bidx], far[bidx] = kinds(faces[bidx])
    far[bidx] &= ~sym[bidx]
    wall[bidx] = ~sym[bidx] & ~far[bidx]
    fblock = blk_of[owner]
    mblock = np.where(mate >= 0, blk_of[owner[np.maximum(mate, 0)]], -1)
    iface = (mate >= 0) & (mblock != fblock)
    blocks = []
    for b in range(n_blocks):
        cells = np.arange(starts[b], starts[b + 1])
        # nodes in first-use order of the Morton-ordered cells
        u, first = np.unique(tets[cells].ravel(), return_index=True)
        used = u[np.argsort(first, kind="stable")]
        g2l = -np.ones(pts.shape[0], dtype=np.int64)
        g2l[used] = np.arange(used.size)
        blk = mg.BlockMesh(nodes=pts[used], tets=g2l[tets[cells]], global_cell=cells)
        in_b = fblock == b
        blk.markers.append(("WALL", g2l[faces[in_b & wall]]))
        blk.markers.append(("FARFIELD", g2l[faces[in_b & far]]))
        blk.markers.append(("SYMMETRY", g2l[faces[in_b & sym]]))
        for nb in range(n_blocks):
            if nb == b:
                continue
            mine = np.nonzero(in_b & iface & (mblock == nb))[0]
            if mine.size == 0:
                continue
            blk.markers.append(("CONNEXION", g2l[faces[mine]]))
            blk.connexions.append((nb, local[owner[mate[mine]]]))
        blocks.append(blk)
    return blocks


def write_wing_case(directory: str, n_points: int, n_blocks: int = 16, seed: int = 5, prefix: str = "wing",
                    deck: mg.Deck | None = None, spec: WingSpec | None = None) -> tuple[str, dict]:
    """Generate, split and write the wing case; returns (deck path, summary)."""
    w = spec or WingSpec()
    os.makedirs(directory, exist_ok=True)
    pts, tets = wing_mesh(w, n_points, seed)
    blocks = split_blocks(w, pts, tets, n_blocks)
    files = []
    for b, blk in enumerate(blocks):
        name = f"{prefix}_B{b}.su2"
        mg.write_su2(os.path.join(directory, name), blk)
        files.append(name)
    top = f"{prefix}.top"
    mg.write_topology(os.path.join(directory, top), files, blocks)
    d = deck or mg.Deck(topology=top)
    d.topology = top
    path = os.path.join(directory, f"{prefix}.deck")
    mg.write_deck(path, d)
    os.makedirs(os.path.join(directory, "bin"), exist_ok=True)
    counts = {t: int(sum(f.shape[0] for blk in blocks for tg, f in blk.markers if tg == t))
              for t in ("WALL", "FARFIELD", "SYMMETRY", "CONNEXION")}
    return path, {"points": int(pts.shape[0]), "tets": int(tets.shape[0]), "blocks": n_blocks, **counts}


# ---------------------------------------------------------------- body-fitted
# The same wing meshed with a boundary-conforming structured grid.  In every
# spanwise station an O-grid wraps the section: node i sits at angle
# theta = 2 pi (i + 1/2) / ni from the trailing edge (upper surface for
# i < ni / 2) at chord fraction s = 1 - sin(theta / 2), clustered at the
# leading edge; the section is the published NACA thickness polynomial with
# its blunt trailing edge, whose base is the face between nodes ni - 1 and 0.
# Ring j = 0 is the wall, ring j = nj a wind-tunnel rectangle reached along
# rays from the section's mid-chord, with geometric growth from a first layer
# about as thick as the steps around the section.  Stations k cluster toward
# the tip, where the thickness falls to zero over a rounded cap; from the tip
# station outward the section is a slit: the lower node i and the upper node
# ni - 1 - i of ring j = 0 are one node, so the cells above and below share
# faces, and the two cells around the slit's leading and trailing edges
# become prisms.  With tip_round = 0 and no stations beyond the tip, the wing
# spans the tunnel instead (its tip section on the far SYMMETRY plane).
# Each hexahedron splits into the 6 Kuhn tetrahedra around its
# (0,0,0)-(1,1,1) diagonal, in i-mirrored local coordinates for the lower half
# (i >= ni / 2): every shared face, the slit's included, then gets the same
# diagonal from both sides, so the tetrahedra are conforming; the tetrahedra
# of a collapsed edge (two corners one node) have no volume and are left out.
@dataclass
class TunnelSpec:
    x0: float = -6.0   # inlet plane (FARFIELD)
    x1: float = 8.0    # outlet plane (FARFIELD)
    h: float = 6.0     # y = -h and y = +h planes (SYMMETRY)
    z1: float = 4.0    # far spanwise plane (SYMMETRY); z = 0 is the root's SYMMETRY plane
    wall_spacing: float | None = None  # first cell height off the wall (root chords); None: 2 / ni, about the
    #                                    mean step around the section, so the cells at the wall are near cubes
    tip_round: float = 0.06      # span over which the thickness falls to zero (elliptic cap); 0: no tip


def _stretch(n: int, first: float, length: float) -> np.ndarray:
    """n + 1 monotone offsets 0..length, the first step `first`, geometric growth."""
    if first * n >= length:
        return np.linspace(0.0, length, n + 1)
    lo, hi = 1.0 + 1e-12, 2.0
    while first * (hi ** n - 1) / (hi - 1) < length:
        hi *= 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if first * (r ** n - 1) / (r - 1) < length:
            lo = r
        else:
            hi = r
    r = 0.5 * (lo + hi)
    d = first * r ** np.arange(n)
    x = np.concatenate([[0.0], np.cumsum(d)])
    return x * (length / x[-1])


def _stations(w: WingSpec, t: TunnelSpec, nk_wing: int, nk_out: int) -> np.ndarray:
    b = w.semi_span
    if nk_out == 0:  # the wing spans the tunnel (its far plane at the tip section)
        return np.linspace(0.0, b, nk_wing + 1)
    zw = b * np.sin(0.5 * np.pi * np.arange(nk_wing + 1) / nk_wing)
    zw[-1] = b
    zo = b + _stretch(nk_out, zw[-1] - zw[-2], t.z1 - b)
    return np.concatenate([zw, zo[1:]])


def _thickness_factor(w: WingSpec, t: TunnelSpec, z: np.ndarray) -> np.ndarray:
    if t.tip_round <= 0.0:  # the wing spans the tunnel: no tip
        return np.ones_like(z)
    zr = w.semi_span - t.tip_round
    u = np.clip((z - zr) / t.tip_round, 0.0, 1.0)
    return np.where(z >= w.semi_span, 0.0, np.sqrt(np.maximum(0.0, 1.0 - u * u)))


def _ray_to_box(cx: float, theta: np.ndarray, t: TunnelSpec) -> np.ndarray:
    """Where rays from (cx, 0) at angle theta meet the rectangle [x0,x1] x [-h,h]."""
    c, s = np.cos(theta), np.sin(theta)
    with np.errstate(divide="ignore"):
        tx = np.where(c > 0, (t.x1 - cx) / c, np.where(c < 0, (t.x0 - cx) / c, np.inf))
        ty = np.where(s != 0, t.h / np.abs(s), np.inf)
    r = np.minimum(tx, ty)
    x, y = cx + r * c, r * s
    x = np.where(tx <= ty, np.where(c > 0, t.x1, t.x0), x)  # exactly on the planes
    y = np.where(ty <= tx, np.sign(s) * t.h, y)
    return np.stack([x, y], axis=1)


_MIRROR = np.array([b ^ 1 for b in range(8)])  # corner (a, b, c) -> (1 - a, b, c)


def body_fitted_wing(w: WingSpec, ni: int, nj: int, nk_wing: int, nk_out: int, t: TunnelSpec | None = None):
    """Nodes, tetrahedra and boundary-face labeller of the body-fitted mesh."""
    t = t or TunnelSpec()
    if ni % 2:
        raise ValueError("ni must be even (the leading edge is node ni / 2)")
    z = _stations(w, t, nk_wing, nk_out)
    nk = z.size - 1
    theta = 2.0 * np.pi * (np.arange(ni) + 0.5) / ni
    # chord fraction: clustered at the leading edge (s ~ (pi - theta)^2), even
    # steps at the blunt trailing edge (whose base is the face from node ni - 1
    # to node 0)
    s_c = 1.0 - np.sin(0.5 * theta)
    upper = np.arange(ni) < ni // 2
    first = t.wall_spacing if t.wall_spacing is not None else 2.0 * w.root_chord / ni
    g = _stretch(nj, first / 6.0, 1.0)  # ray fraction; first step ~ `first` on a 6-chord ray
    X = np.empty((ni, nj + 1, nk + 1, 3))
    for k in range(nk + 1):
        xle, c = _le_chord(w, np.array([min(z[k], w.semi_span)]))
        xle, c = float(xle[0]), float(c[0])
        yt = c * naca_half_thickness(s_c, w.thickness, closed=False) * _thickness_factor(w, t, np.array([z[k]]))[0]
        inner = np.stack([xle + s_c * c, np.where(upper, yt, -yt)], axis=1)
        outer = _ray_to_box(xle + 0.5 * c, theta, t)
        X[:, :, k, 0:2] = inner[:, None, :] + g[None, :, None] * (outer - inner)[:, None, :]
        X[:, :, k, 2] = z[k]
    # node ids with the slit identified: from the tip station outward, the
    # lower-surface node i of ring j = 0 is the upper node ni - 1 - i
    kt = nk_wing
    nid = np.arange(ni * (nj + 1) * (nk + 1)).reshape(ni, nj + 1, nk + 1)
    if nk_out > 0:
        low = np.arange(ni // 2, ni)
        ks = np.arange(kt, nk + 1)[None, :]
        nid[low[:, None], 0, ks] = nid[(ni - 1 - low)[:, None], 0, ks]
    used, inv = np.unique(nid.ravel(), return_inverse=True)
    pts = X.reshape(-1, 3)[used]
    nid = inv.reshape(nid.shape)
    # hexahedra (i, j, k) -> 8 corners, bit 0: i + 1, bit 1: j + 1, bit 2: k + 1
    hi, hj, hk = np.meshgrid(np.arange(ni), np.arange(nj), np.arange(nk), indexing="ij")
    hi, hj, hk = hi.ravel(), hj.ravel(), hk.ravel()
    corners = np.stack([nid[(hi + (b & 1)) % ni, hj + ((b >> 1) & 1), hk + ((b >> 2) & 1)] for b in range(8)], axis=1)
    lower = hi >= ni // 2
    corners[lower] = corners[lower][:, _MIRROR]
    tets = corners[:, mg._KUHN_TETS].reshape(-1, 4)
    st = np.sort(tets, axis=1)
    tets = tets[np.all(st[:, 1:] != st[:, :-1], axis=1)]  # collapsed edges: no volume

    # node flags for the boundary labels: 1 on the inlet or outlet plane,
    # 4 on z = 0, 8 on the far spanwise plane, 16 on the outer ring
    ring = np.zeros(nid.shape, np.int8)
    ox = X[:, nj, :, 0]
    ring[:, nj, :] |= np.where((ox == t.x0) | (ox == t.x1), 17, 16).astype(np.int8)
    ring[:, :, 0] |= 4
    ring[:, :, nk] |= 8
    flag = np.zeros(pts.shape[0], np.int8)
    np.bitwise_or.at(flag, nid.ravel(), ring.ravel())

    def kinds(fnodes: np.ndarray):
        """SYMMETRY: the z = 0 and far spanwise planes and the tunnel's y = -h
        and y = +h sides; FARFIELD: the inlet and outlet planes, and the ring
        faces that cut a corner of the tunnel between one of them and a side."""
        f = flag[fnodes]
        zsym = np.all((f & 4) != 0, axis=1) | np.all((f & 8) != 0, axis=1)
        on_ring = np.all((f & 16) != 0, axis=1) & ~zsym
        inout = np.any((f & 1) != 0, axis=1)
        return zsym | (on_ring & ~inout), on_ring & inout

    return pts, tets, kinds


def write_body_fitted_wing_case(directory: str, ni: int, nj: int, nk_wing: int, nk_out: int, n_blocks: int = 16,
                                prefix: str = "wing", deck: mg.Deck | None = None, spec: WingSpec | None = None,
                                tunnel: TunnelSpec | None = None) -> tuple[str, dict]:
    """Generate, split and write the body-fitted wing case; returns (deck path, summary)."""
    w = spec or WingSpec()
    os.makedirs(directory, exist_ok=True)
    pts, tets, kinds = body_fitted_wing(w, ni, nj, nk_wing, nk_out, tunnel)
    blocks = split_blocks(w, pts, tets, n_blocks, kinds)
    files = []
    for b, blk in enumerate(blocks):
        name = f"{prefix}_B{b}.su2"
        mg.write_su2(os.path.join(directory, name), blk)
        files.append(name)
    top = f"{prefix}.top"
    mg.write_topology(os.path.join(directory, top), files, blocks)
    d = deck or mg.Deck(topology=top)
    d.topology = top
    path = os.path.join(directory, f"{prefix}.deck")
    mg.write_deck(path, d)
    os.makedirs(os.path.join(directory, "bin"), exist_ok=True)
    counts = {tg: int(sum(f.shape[0] for blk in blocks for t_, f in blk.markers if t_ == tg))
              for tg in ("WALL", "FARFIELD", "SYMMETRY", "CONNEXION")}
    return path, {"points": int(pts.shape[0]), "tets": int(tets.shape[0]), "blocks": n_blocks, **counts}

"""Host-side case ingest against the reference (CPU only).

The SU2 reader, face builder, connectivity and metrics of libe3d.so must give
exactly the reference's arrays (Block/Cell/Face members as dumped by the
compiled reference in tests/golden).
"""
import os

import numpy as np
import pytest
from conftest import Golden, golden_names, same

from euler3d_b200 import meshgen as mg
from euler3d_b200._lib import E3DError
from euler3d_b200.api import Case

PAIRS = [("face_cells", "face_cells"), ("face_nodes", "face_nodes"), ("face_normal", "face_normal"),
         ("face_area", "face_area"), ("face_center", "face_center"), ("r_left", "r_left"), ("r_right", "r_right"),
         ("cell_faces", "cell_faces"), ("cell_cells", "cell_cells"), ("cell_volume", "cell_volume"),
         ("cell_center", "cell_center"), ("ls_weights", "ls_weights"), ("marker_cells", "marker_cells"),
         ("marker_kind", "marker_kind"), ("marker_size", "marker_size"), ("wall_faces", "wall_faces")]


@pytest.mark.parametrize("name", golden_names())
def test_geometry_bitwise(name, tmp_path):
    g = Golden(name)
    case = Case(g.write_case(str(tmp_path)))
    assert case.n_blocks == g.n_blocks
    for b in range(g.n_blocks):
        cnt = g[f"init.b{b}.counts"]
        info = case.block_info(b)
        assert (info.n_real, info.n_all, info.n_faces, info.n_real_boundaries) == tuple(cnt[:4])
        assert info.n_wall_faces == cnt[5]
        for mine, ref in PAIRS:
            a = case.get(b, mine)
            r = g[f"init.b{b}.{ref}"]
            assert same(a, r), f"block {b} {mine}"
            if a.dtype == np.float64:  # bit patterns too, not only values
                assert np.array_equal(a.view(np.uint64), r.view(np.uint64)), f"block {b} {mine} bits"


def test_deck_fields(tmp_path):
    d = mg.Deck(topology="", cfl=0.75, gamma=1.3, aoa_deg=2.5, stages=4, mach=0.85, cmac=2.0, max_iter=77,
                criterion=-9.0, flux="ausm", order=2, gradient="greengauss", limiter="barthjespersen",
                omega=1e-3, k=3.0)
    c = Case(mg.write_case(str(tmp_path), 2, 1, deck=d))
    i = c.deck
    assert (i.cfl, i.gamma, i.aoa_deg, i.stages, i.mach, i.cmac, i.max_iter, i.criterion) == \
        (0.75, 1.3, 2.5, 4, 0.85, 2.0, 77, -9.0)
    assert (i.flux, i.order, i.gradient, i.limiter, i.omega, i.k) == (1, 2, 0, 0, 1e-3, 3.0)


def test_deck_reads_like_the_reference(tmp_path):
    # The reference reads the omega/k line with `>>`: "2.16-16" is omega 2.16, k -16
    # (seen in the reference's input_test1 deck).
    deck = mg.write_case(str(tmp_path), 2, 1)
    txt = open(deck).read().replace(f"{2.16e-16!r} 5.0", "2.16-16")
    open(deck, "w").write(txt)
    i = Case(deck).deck
    assert (i.omega, i.k) == (2.16, -16.0)


def test_selection_strings_like_reference(tmp_path):
    # any gradient other than "leastsquares" is Green-Gauss; any limiter other than
    # "venkatakrishnan" is Barth-Jespersen (SecondOrder.cpp:50-61)
    d = mg.Deck(topology="", order=2, gradient="foo", limiter="bar")
    i = Case(mg.write_case(str(tmp_path), 2, 1, deck=d)).deck
    assert (i.gradient, i.limiter) == (0, 0)


def _corrupt(path, old, new):
    s = open(path).read()
    assert old in s
    open(path, "w").write(s.replace(old, new, 1))


def test_missing_block_file(tmp_path):
    deck = mg.write_case(str(tmp_path), 2, 2)
    os.remove(os.path.join(tmp_path, "bump_B1.su2"))
    with pytest.raises(E3DError) as e:
        Case(deck)
    assert e.value.code == -2


def test_missing_deck(tmp_path):
    with pytest.raises(E3DError) as e:
        Case(str(tmp_path / "nope.deck"))
    assert e.value.code == -2


def test_pyramid_rejected(tmp_path):
    deck = mg.write_case(str(tmp_path), 2, 1)
    su2 = os.path.join(tmp_path, "bump.su2")
    lines = open(su2).read().split("\n")
    i = next(k for k, l in enumerate(lines) if l.startswith("10 "))
    lines[i] = "14 " + lines[i][3:] + " 0"
    open(su2, "w").write("\n".join(lines))
    with pytest.raises(E3DError) as e:
        Case(deck)
    assert e.value.code == -3 and "pyramid" in str(e.value)


def test_unknown_marker_rejected(tmp_path):
    deck = mg.write_case(str(tmp_path), 2, 1)
    _corrupt(os.path.join(tmp_path, "bump.su2"), "MARKER_TAG= FARFIELD", "MARKER_TAG= INLET")
    with pytest.raises(E3DError) as e:
        Case(deck)
    assert e.value.code == -3


def test_boundary_element_without_face(tmp_path):
    deck = mg.write_case(str(tmp_path), 2, 1)
    su2 = os.path.join(tmp_path, "bump.su2")
    lines = open(su2).read().split("\n")
    i = next(k for k, l in enumerate(lines) if l.startswith("5 "))
    lines[i] = "5 0 1 26"  # nodes that form no tetrahedron face
    open(su2, "w").write("\n".join(lines))
    with pytest.raises(E3DError) as e:
        Case(deck)
    assert e.value.code == -4


def test_open_boundary_face(tmp_path):
    deck = mg.write_case(str(tmp_path), 2, 1)
    su2 = os.path.join(tmp_path, "bump.su2")
    s = open(su2).read()
    # drop the last farfield element: one boundary face has no ghost cell
    head, tail = s.rsplit("MARKER_ELEMS= ", 1)
    n = int(tail.split("\n", 1)[0])
    rows = tail.split("\n")[1:1 + n]
    open(su2, "w").write(head + f"MARKER_ELEMS= {n - 1}\n" + "\n".join(rows[:-1]) + "\n")
    with pytest.raises(E3DError) as e:
        Case(deck)
    assert e.value.code == -4


def test_topology_out_of_range(tmp_path):
    deck = mg.write_case(str(tmp_path), 2, 2)
    top = os.path.join(tmp_path, "bump.top")
    lines = open(top).read().split("\n")
    i = lines.index("Nelems= 8")
    lines[i + 1] = "999999"
    open(top, "w").write("\n".join(lines))
    with pytest.raises(E3DError) as e:
        Case(deck)
    assert e.value.code == -4


def test_truncated_su2(tmp_path):
    deck = mg.write_case(str(tmp_path), 2, 1)
    su2 = os.path.join(tmp_path, "bump.su2")
    s = open(su2).read()
    open(su2, "w").write(s[: len(s) // 2])
    with pytest.raises(E3DError) as e:
        Case(deck)
    assert e.value.code in (-3, -4)

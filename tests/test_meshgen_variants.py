"""Synthetic mesh generators beyond the bump channel of the default workload:
the channel side variants and the Delaunay swept wing.  Host only."""
import numpy as np
import pytest

from euler3d_b200 import api
from euler3d_b200 import meshgen as mg
from euler3d_b200 import wingmesh as wm


@pytest.mark.parametrize("sides", ["farfield", "symmetry", "channel"])
def test_channel_side_variants_load(tmp_path, sides):
    deck = mg.write_case(str(tmp_path), 6, 2, deck=mg.Deck(topology=""), sides=sides)
    case = api.Case(deck)
    tags = {"farfield": {"WALL", "FARFIELD", "CONNEXION"}, "symmetry": {"WALL", "FARFIELD", "SYMMETRY", "CONNEXION"},
            "channel": {"WALL", "FARFIELD", "SYMMETRY", "CONNEXION"}}[sides]
    blocks = mg.slab_blocks(mg.bump_channel(6), 2, sides)
    assert {t for t, _ in blocks[0].markers} == tags
    n_bnd = sum(f.shape[0] for t, f in blocks[0].markers if t != "CONNEXION")
    n_bnd += sum(f.shape[0] for t, f in blocks[1].markers if t != "CONNEXION")
    assert n_bnd == 2 * 6 * 6 * 6  # six faces of the box, 2 triangles per square, 36 squares each
    assert case.n_blocks == 2


def test_channel_default_is_unchanged():
    """sides="farfield" and ytop=1 reproduce the configuration-1 mesh exactly."""
    a = mg.bump_channel(5)
    b = mg.bump_channel(5, ytop=1.0)
    assert np.array_equal(a.nodes, b.nodes)


def test_wing_case_is_closed_and_well_posed(tmp_path):
    deck = mg.Deck(topology="", order=2, flux="ausm", gradient="leastsquares", limiter="barthjespersen")
    path, summ = wm.write_wing_case(str(tmp_path), 6000, n_blocks=3, seed=5, deck=deck)
    assert summ["WALL"] > 0 and summ["FARFIELD"] > 0 and summ["SYMMETRY"] > 0
    case = api.Case(path)  # every cell closed, every boundary face on a marker (else E3D_ERR_MESH)
    assert case.n_blocks == 3
    n = [case.block_info(b).n_real for b in range(3)]
    assert max(n) - min(n) <= 1 and sum(n) == summ["tets"]
    for b in range(3):
        assert np.all(np.isfinite(case.get(b, "ls_weights")))
        assert np.all(case.get(b, "cell_volume")[:n[b]] > 0)
    # the same seed gives the same mesh
    path2, summ2 = wm.write_wing_case(str(tmp_path / "again"), 6000, n_blocks=3, seed=5, deck=deck)
    assert summ == summ2
    assert open(tmp_path / "wing_B1.su2").read() == open(tmp_path / "again" / "wing_B1.su2").read()


def test_wing_geometry():
    w = wm.WingSpec()
    t = wm.naca_half_thickness(np.linspace(0, 1, 1001), 0.12)
    assert abs(2 * t.max() - 0.12) < 1e-3 and abs(t[-1]) < 1e-12 and t[0] == 0
    root_mid = np.array([[0.3, 0.0, 0.0], [0.3, 0.1, 0.0], [2.0, 0.0, 0.5]])
    assert list(wm.inside_wing(w, root_mid)) == [True, False, False]
    # swept leading edge: at mid-span the section starts at z tan(30 deg)
    z = 0.75
    assert wm.inside_wing(w, np.array([[z * np.tan(np.radians(30)) + 0.05, 0.0, z]]))[0]
    assert not wm.inside_wing(w, np.array([[z * np.tan(np.radians(30)) - 0.01, 0.0, z]]))[0]


@pytest.mark.parametrize("ni,nj,nkw,nko", [(16, 4, 6, 2), (32, 8, 12, 4)])
def test_body_fitted_wing_is_conforming(ni, nj, nkw, nko):
    """The structured wing: every triangle is shared by at most two tets (the
    slit beyond the tip included), no tet is flat, the wall is exactly the
    wing surface (2 triangles per surface quad, one fewer at each of the two
    collapsed tip edges), and the domain is the tunnel minus the wing."""
    w, t = wm.WingSpec(), wm.TunnelSpec()
    pts, tets, kinds = wm.body_fitted_wing(w, ni, nj, nkw, nko)
    p = pts[tets]
    vol = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0]) / 6
    assert np.all(np.abs(vol) > 0)
    faces = np.sort(tets[:, [[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]]].reshape(-1, 3), axis=1)
    u, c = np.unique(faces, axis=0, return_counts=True)
    assert set(np.unique(c)) == {1, 2}
    bnd = u[c == 1]
    sym, far = kinds(bnd)
    wall = ~sym & ~far
    assert wall.sum() == 2 * ni * nkw - 2
    wp = pts[bnd[wall]]
    assert wp[:, :, 2].max() <= w.semi_span and np.all(wm.inside_wing(w, wp.mean(axis=1) * [1, 0, 1]))
    fp = pts[bnd[far]]
    assert np.all(np.isin(fp[:, :, 0], [t.x0, t.x1]).any(axis=1))  # inlet, outlet and their corner cuts
    box = (t.x1 - t.x0) * 2 * t.h * t.z1  # less the wing and the tunnel corners the outer ring cuts off
    assert box * 0.9 < np.abs(vol).sum() < box


def test_body_fitted_wing_case_loads(tmp_path):
    deck = mg.Deck(topology="", order=2, flux="ausm", gradient="leastsquares", limiter="venkatakrishnan", mach=0.8,
                   aoa_deg=3.0)
    path, summ = wm.write_body_fitted_wing_case(str(tmp_path), 24, 6, 8, 3, n_blocks=3, deck=deck)
    case = api.Case(path)  # closed cells, every boundary face on a marker
    n = [case.block_info(b).n_real for b in range(3)]
    assert sum(n) == summ["tets"] and max(n) - min(n) <= 1
    for b in range(3):
        assert np.all(np.isfinite(case.get(b, "ls_weights")))
        assert np.all(case.get(b, "cell_volume")[:n[b]] > 0)
    assert sum(case.block_info(b).n_wall_faces for b in range(3)) == summ["WALL"] == 2 * 24 * 8 - 2

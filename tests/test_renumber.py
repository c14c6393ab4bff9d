"""Cell renumbering on the host (CPU only): every mode gives a permutation of
a block's real cells, reverse Cuthill-McKee narrows the adjacency bandwidth
of a shuffled mesh, and the Z-order follows the cell centres.  The GPU tests
(tests/test_parity_gpu.py) show the FP64 results are bit for bit the same in
every order."""
import numpy as np
import pytest
from conftest import Golden

from euler3d_b200 import meshgen as mg
from euler3d_b200.api import Case


def _bandwidth(case, b, order):
    """largest |position(c) - position(neighbour)| over real-cell pairs"""
    pos = np.empty_like(order)
    pos[order] = np.arange(order.size)
    ptr = case.get(b, "cell_face_ptr")
    nbr = case.get(b, "cell_cells")
    n = order.size
    own = np.repeat(np.arange(n), np.diff(ptr[:n + 1]))
    other = nbr[:ptr[n]]
    keep = other < n
    return int(np.max(np.abs(pos[own[keep]] - pos[other[keep]])))


@pytest.mark.parametrize("mode", ["none", "rcm", "morton", "shuffle", "none+boundary_last", "morton+boundary_last"])
def test_orders_are_permutations(mode, tmp_path):
    case = Case(mg.write_case(str(tmp_path), 6, 2))
    for b in range(case.n_blocks):
        o = case.cell_order(b, mode)
        assert np.array_equal(np.sort(o), np.arange(case.block_info(b).n_real))
        if mode == "none":
            assert np.array_equal(o, np.arange(o.size))
    # deterministic
    assert np.array_equal(case.cell_order(1, mode), case.cell_order(1, mode))


@pytest.mark.parametrize("base", ["none", "morton"])
def test_boundary_last_groups_cells_with_ghost_neighbours(base, tmp_path):
    """Cells with a ghost neighbour (boundary or connexion face) come last in
    their block; each group keeps the base order."""
    case = Case(mg.write_case(str(tmp_path), 6, 3))
    for b in range(case.n_blocks):
        n = case.block_info(b).n_real
        ptr = case.get(b, "cell_face_ptr")
        nbr = case.get(b, "cell_cells")
        own = np.repeat(np.arange(n), np.diff(ptr[:n + 1]))
        boundary = np.zeros(n, bool)
        boundary[own[nbr[:ptr[n]] >= n]] = True
        o = case.cell_order(b, base + "+boundary_last")
        k = int(np.count_nonzero(~boundary))
        assert 0 < k < n
        assert not boundary[o[:k]].any() and boundary[o[k:]].all()
        ref = case.cell_order(b, base)
        assert np.array_equal(o[:k], ref[~boundary[ref]]) and np.array_equal(o[k:], ref[boundary[ref]])


def test_rcm_restores_locality_of_a_shuffled_order(tmp_path):
    case = Case(mg.write_case(str(tmp_path), 10, 1))
    n = case.block_info(0).n_real
    shuffled = _bandwidth(case, 0, case.cell_order(0, "shuffle"))
    rcm = _bandwidth(case, 0, case.cell_order(0, "rcm"))
    assert shuffled > n // 2
    assert rcm < n // 10, (rcm, n)


def test_morton_follows_the_cell_centres(tmp_path):
    case = Case(mg.write_case(str(tmp_path), 8, 1))
    o = case.cell_order(0, "morton")
    cen = case.get(0, "cell_center").reshape(-1, 3)[: o.size]
    # consecutive cells in Z-order are close: mean step well below the box size
    steps = np.linalg.norm(np.diff(cen[o], axis=0), axis=1)
    assert np.mean(steps) < 0.1


def test_rcm_on_hexahedra_and_reference_mesh(tmp_path):
    g = Golden("ref_naca_o1_roe")
    case = Case(g.write_case(str(tmp_path)))
    o = case.cell_order(0, "rcm")
    assert np.array_equal(np.sort(o), np.arange(case.block_info(0).n_real))


def test_unknown_mode_is_an_argument_error(tmp_path):
    from euler3d_b200 import _lib as L

    case = Case(mg.write_case(str(tmp_path), 2, 1))
    out = np.empty(case.block_info(0).n_real, dtype=np.int32)
    assert L.lib().e3d_case_cell_order(case._h, 0, 7, L.ptr(out), out.size) == -1
    assert b"renumbering" in L.lib().e3d_last_error()
    with pytest.raises(KeyError):
        case.cell_order(0, "hilbert")

"""Full-size workloads against the reference solver, plus size-independent properties.

* bump20_o1_roe_500: the 20^3 x 6 (48,000-tet) bump channel, first-order Roe,
  500 iterations of the reference CPU solver.
* bump80b16_o2_ls_venk_roe_3: the 80^3 x 6 (3,072,000-tet) bump channel in 16
  slab blocks, least squares + Venkatakrishnan + Roe, 3 reference iterations.

FP64 bar: Cl/Cd identical to the reference (bit for bit), residual norms within
1e-12 relative (summation order).  FP32 bar (from the target): Cl/Cd within
1e-4 relative of the FP64 reference after the 500 iterations of the small
workload; transient iterations of the large one within 5e-3 of the Cl scale.
"""
import os

import numpy as np
import pytest
from conftest import Golden, max_rel, same

from euler3d_b200 import api
from euler3d_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _solver(name, tmp_path, precision):
    g = Golden(name)
    case = api.Case(g.write_case(str(tmp_path)))
    return g, case, api.Solver(case, precision=precision)


def test_bump20_fp64_500_iterations(tmp_path):
    g, case, s = _solver("bump20_o1_roe_500", tmp_path, "fp64")
    s.iterate(500)
    h = s.history()
    for col in ("cl", "cd", "cmx", "cmy", "cmz"):
        assert same(h[col], g.hist(col)), col
    for q, col in enumerate(("rms_ro", "rms_uu", "rms_vv", "rms_ww", "rms_pp")):
        assert max_rel(h["rms"][:, q], g.hist(col)) < 1e-12, col
    assert np.max(np.abs(h["conv"][:, 0] - g.hist("ro_conv"))) < 1e-11


def test_bump20_fp32_500_iterations(tmp_path):
    g, case, s = _solver("bump20_o1_roe_500", tmp_path, "fp32")
    s.iterate(500)
    h = s.history()
    for col in ("cl", "cd"):
        ref = g.hist(col)[-1]
        assert abs(h[col][-1] - ref) / abs(ref) < 1e-4, (col, h[col][-1], ref)
    # the density-drop history within 1e-3 decades over the whole run
    assert np.max(np.abs(h["conv"][:, 0] - g.hist("ro_conv"))) < 1e-3


def test_bump80_16_blocks_fp64(tmp_path):
    g, case, s = _solver("bump80b16_o2_ls_venk_roe_3", tmp_path, "fp64")
    s.iterate(3)
    h = s.history()
    for col in ("cl", "cd", "cmx", "cmy", "cmz"):
        assert same(h[col], g.hist(col)), col
    for q, col in enumerate(("rms_ro", "rms_uu", "rms_vv", "rms_ww", "rms_pp")):
        assert max_rel(h["rms"][:, q], g.hist(col)) < 1e-12, col


def test_bump80_16_blocks_fp32(tmp_path):
    g, case, s = _solver("bump80b16_o2_ls_venk_roe_3", tmp_path, "fp32")
    s.iterate(3)
    h = s.history()
    for col in ("cl", "cd"):
        scale = max(np.max(np.abs(g.hist(col))), 1e-2)
        assert np.max(np.abs(h[col] - g.hist(col))) / scale < 5e-3, col
    assert max_rel(h["rms"][:, 0], g.hist("rms_ro")) < 1e-2


@pytest.mark.parametrize("order,flux", [(1, "roe"), (2, "roe"), (2, "ausm")])
def test_freestream_preserved(tmp_path, order, flux):
    """Uniform flow with farfield boundaries only: every closed cell's area
    vectors sum to zero, so the residual vanishes to rounding and the state
    stays at freestream (40^3 x 6 = 384,000 tets, 4 blocks)."""
    deck = mg.write_case(str(tmp_path), 40, 4, deck=mg.Deck(topology="", order=order, flux=flux, mach=0.6,
                                                            aoa_deg=2.0, gradient="leastsquares",
                                                            limiter="venkatakrishnan"))
    for b in range(4):
        p = os.path.join(tmp_path, f"bump_B{b}.su2")
        s = open(p).read().replace("MARKER_TAG= WALL", "MARKER_TAG= FARFIELD")
        open(p, "w").write(s)
    case = api.Case(deck)
    for precision, tol in (("fp64", 1e-12), ("fp32", 1e-5)):
        s = api.Solver(case, precision=precision)
        s.iterate(3)
        for b in range(4):
            p = s.get(b, "prim").reshape(5, -1)
            free = np.array([1.0, 0.6 * np.sqrt(1.4) * np.cos(np.radians(2.0)),
                             0.6 * np.sqrt(1.4) * np.sin(np.radians(2.0)), 0.0, 1.0])
            assert np.max(np.abs(p - free[:, None])) < tol, (precision, b)


def test_least_squares_exact_on_linear_fields(tmp_path):
    """The least-squares gradient reproduces a linear field exactly (to
    rounding) in every cell whose neighbours are all real cells."""
    deck = mg.write_case(str(tmp_path), 12, 1, deck=mg.Deck(topology="", order=2))
    case = api.Case(deck)
    s = api.Solver(case, precision="fp64")
    info = case.block_info(0)
    cc = case.get(0, "cell_center").reshape(-1, 3)
    A = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0], [7.0, 8.0, 9.0], [10.0, 11.0, 12.0], [13.0, 14.0, 15.0]])
    base = np.array([5.0, 1.0, 2.0, 3.0, 7.0])
    prim = (base[:, None] + A @ cc.T)
    s.set(0, "prim", prim.ravel())
    api.LeastSquares().computeGradients(api.Block(s, 0))
    grad = s.get(0, "grad").reshape(5, info.n_all, 3)
    ptr = case.get(0, "cell_face_ptr")
    nbr = case.get(0, "cell_cells")
    interior = [c for c in range(info.n_real) if np.all(nbr[ptr[c]:ptr[c + 1]] < info.n_real)]
    assert len(interior) > info.n_real // 2
    for q in range(5):
        err = np.abs(grad[q, interior, :] - A[q][None, :])
        assert np.max(err) < 1e-9 * np.max(np.abs(A[q])), q

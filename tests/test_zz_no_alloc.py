"""The non-allocating residual-norm entry point (e3d_residual_norms_noalloc).

Callers that cannot allocate device memory (a host that owns every device byte
through its own pool, a time-stepping loop that must not allocate) get the
per-block sums of (Rc - Rd)^2 from this entry point, whose scratch is a static
device array.  Its output must equal what the existing entry point,
e3d_flow_data, reports for the same residuals, within the tolerance the other
norm tests use (relative 1e-12), on two calls in a row (the scratch keeps the
previous call's contents, so a second call shows that nothing stale leaks).

This file is collected last on purpose: a failure here leaves every other test
already run.  It allocates its own device buffers with torch (the test may
allocate; the entry point under test does not).
"""
import ctypes as C

import numpy as np
import pytest
from conftest import Golden, max_rel

from euler3d_b200 import _lib as L
from euler3d_b200 import api
from euler3d_b200 import meshgen as mg

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the residual-norm tolerance of tests/test_parity_gpu.py


def _residuals_on_device(solver, case):
    import torch

    nb = case.n_blocks
    n_real = [case.block_info(b).n_real for b in range(nb)]
    rc = np.concatenate([solver.get(b, "conv_res").reshape(5, -1) for b in range(nb)], axis=1)
    rd = np.concatenate([solver.get(b, "diss_res").reshape(5, -1) for b in range(nb)], axis=1)
    off = np.concatenate([[0], np.cumsum(n_real)]).astype(np.int32)
    dev = torch.device("cuda", 0)
    t_rc = torch.from_numpy(np.ascontiguousarray(rc)).to(dev)
    t_rd = torch.from_numpy(np.ascontiguousarray(rd)).to(dev)
    t_off = torch.from_numpy(off).to(dev)
    t_out = torch.full((nb * 5,), float("nan"), dtype=torch.float64, device=dev)
    return t_rc, t_rd, t_off, t_out, int(off[-1]), max(n_real)


def _call(t_rc, t_rd, t_off, t_out, n, max_cells):
    import torch

    nb = t_off.numel() - 1
    rc = L.lib().e3d_residual_norms_noalloc(C.c_void_p(t_rc.data_ptr()), C.c_void_p(t_rd.data_ptr()), n, nb,
                                            C.c_void_p(t_off.data_ptr()), max_cells, C.c_void_p(t_out.data_ptr()),
                                            None)
    L.check(rc)
    torch.cuda.synchronize()
    return t_out.cpu().numpy().reshape(nb, 5).copy()


def _check_case(solver, case):
    solver.iterate(3)
    ref = solver.flow_data()[:, :5]  # existing entry point: per-block sums of (Rc-Rd)^2
    t_rc, t_rd, t_off, t_out, n, max_cells = _residuals_on_device(solver, case)
    first = _call(t_rc, t_rd, t_off, t_out, n, max_cells)
    # a call with a different chunk layout in between: a larger max_block_cells
    # puts each block's partial sums at other scratch indices, so a second call
    # with the first layout would read stale partials if any were left unwritten
    wide = _call(t_rc, t_rd, t_off, t_out, n, max_cells + 3 * 4096)
    second = _call(t_rc, t_rd, t_off, t_out, n, max_cells)
    assert max_rel(first, ref) <= RTOL
    assert max_rel(wide, ref) <= RTOL
    assert max_rel(second, ref) <= RTOL


def test_noalloc_norms_match_flow_data_golden_case(tmp_path):
    g = Golden("t4_o2_ls_venk_roe_b2")  # two blocks, one partial sum each
    case = api.Case(g.write_case(str(tmp_path)))
    _check_case(api.Solver(case, precision="fp64", device=0), case)


def test_noalloc_norms_match_flow_data_several_chunks(tmp_path):
    # 16^3 x 6 tets in 4 slabs: 6,144 cells per block, two 4,096-cell chunks each
    deck = mg.write_case(str(tmp_path), 16, 4, deck=mg.Deck(topology="", order=2, mach=0.7, aoa_deg=1.25))
    case = api.Case(deck)
    _check_case(api.Solver(case, precision="fp64", device=0), case)


def test_noalloc_understated_block_size_gives_nan(tmp_path):
    # max_block_cells below the real size: the host cannot see the device
    # offsets, so the blocks the grid does not cover come back NaN (never a
    # silently truncated sum); blocks that fit stay exact
    deck = mg.write_case(str(tmp_path), 16, 4, deck=mg.Deck(topology="", order=2, mach=0.7, aoa_deg=1.25))
    case = api.Case(deck)
    solver = api.Solver(case, precision="fp64", device=0)
    solver.iterate(2)
    ref = solver.flow_data()[:, :5]
    t_rc, t_rd, t_off, t_out, n, max_cells = _residuals_on_device(solver, case)
    assert max_cells > 4096  # every block needs two chunks
    got = _call(t_rc, t_rd, t_off, t_out, n, 4096)
    assert np.all(np.isnan(got))
    again = _call(t_rc, t_rd, t_off, t_out, n, max_cells)
    assert max_rel(again, ref) <= RTOL


def test_noalloc_rejects_sizes_beyond_the_scratch():
    # rejected on the host before anything is launched; no pointer is touched
    nb = 3
    too_many = 4096 * (8192 // nb + 1)
    rc = L.lib().e3d_residual_norms_noalloc(C.c_void_p(16), C.c_void_p(16), too_many, nb, C.c_void_p(16), too_many,
                                            C.c_void_p(16), None)
    assert rc == -9
    assert b"static scratch" in L.lib().e3d_last_error()
    # a max_block_cells near INT_MAX is rejected too (its chunk count is formed in 64 bits)
    rc = L.lib().e3d_residual_norms_noalloc(C.c_void_p(16), C.c_void_p(16), 1, 1, C.c_void_p(16), 2**31 - 1,
                                            C.c_void_p(16), None)
    assert rc == -9

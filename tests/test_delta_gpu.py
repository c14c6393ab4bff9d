"""FP32 iterations in difference form (e3d_solver_set_precision E3D_FP32_DELTA).

The form exists to take a batched FP32 solve past the FP32 floor: the state is
an FP64 base plus FP32 differences, the base residual is evaluated in FP64 at
every rebase and the per-stage residual adds the change of the fluxes since
the base, computed in a form whose rounding scales with that change.  Bar:
from an FP32 state stopped at its floor, the difference form reaches a
10-order drop, and its converged Cl/Cd equal those of the FP64 solve from the
same start within 1e-9 relative (both converge to the same discrete
solution; only their rounding differs), in about the same number of
iterations.
"""
import numpy as np
import pytest

from euler3d_b200 import _lib as L
from euler3d_b200 import api
from euler3d_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _channel(tmp_path, name, n, mach, aoa, order=1, flux="ausm", blocks=1):
    d = mg.Deck(topology="", mach=mach, aoa_deg=aoa, stages=5, cfl=1.5, order=order, flux=flux,
                gradient="greengauss", limiter="barthjespersen")
    return api.Case(mg.write_case(str(tmp_path / name), n, blocks, prefix=name, deck=d, sides="channel"))


def _first_below(conv, level):
    hit = np.nonzero(conv <= level)[0]
    return int(hit[0]) + 1 if hit.size else None


def _solve(cases, finish, crit):
    b = api.Batch(cases, precision="fp32", hist_capacity=4096)
    b.solve_batch(30000, -4.5, iters_per_launch=50)  # FP32 to near its floor
    api.set_precision(b, finish)
    b.solve_batch(60000, crit, iters_per_launch=50)
    hs = [b.case_history(c) for c in range(len(cases))]
    return b, hs


def test_difference_form_passes_the_fp32_floor_to_the_fp64_solution(tmp_path):
    # the second case has 3 blocks: halo ghosts rebased from their origin cells
    cases = [_channel(tmp_path, "a", 8, 0.5, 2.0), _channel(tmp_path, "b", 9, 0.72, -1.0, blocks=3)]
    bd, hd = _solve(cases, "fp32-delta", -10.0)
    bf, hf = _solve(cases, "fp64-fma", -10.0)
    for c in range(len(cases)):
        nd, nf = _first_below(hd[c]["conv"][:, 0], -10.0), _first_below(hf[c]["conv"][:, 0], -10.0)
        assert nd is not None and nf is not None
        assert abs(nd - nf) <= 0.01 * nf
        for col in ("cl", "cd"):
            assert abs(hd[c][col][-1] - hf[c][col][-1]) <= 1e-9 * max(abs(hf[c][col][-1]), 1e-2), col
    # the full state is readable in difference form and equals the FP64 solve's
    # converged state to the same accuracy
    for blk in range(bd.n_blocks):
        case, local = (cases[0], 0) if blk == 0 else (cases[1], blk - 1)
        nr, na = case.block_info(local).n_real, case.block_info(local).n_all
        pd = bd.get(blk, "prim").reshape(5, na)[:, :nr]
        pf = bf.get(blk, "prim").reshape(5, na)[:, :nr]
        assert np.max(np.abs(pd - pf) / np.abs(pf).clip(1e-2)) < 1e-8
    bd.close()
    bf.close()


def test_difference_form_rejects_other_schemes_and_calls(tmp_path):
    roe = _channel(tmp_path, "roe", 6, 0.5, 1.0, flux="roe")
    b = api.Batch([roe], precision="fp32")
    b.solve_batch(2, -1e300, iters_per_launch=1)
    with pytest.raises(L.E3DError) as e:
        api.set_precision(b, "fp32-delta")
    assert e.value.code == -1
    b.close()
    case = _channel(tmp_path, "au", 6, 0.5, 1.0)
    s = api.Solver(case, precision="fp64")
    with pytest.raises(L.E3DError) as e:
        api.set_precision(s, "fp32-delta")  # needs an FP32 solver
    assert e.value.code == -7
    s.close()
    b = api.Batch([case], precision="fp32")
    b.solve_batch(2, -1e300, iters_per_launch=1)
    api.set_precision(b, "fp32-delta")
    with pytest.raises(L.E3DError) as e:
        b.iterate(1)  # only batch solves run in difference form
    assert e.value.code == -7
    b.solve_batch(5, -1e300, iters_per_launch=2)
    api.set_precision(b, "fp64")  # leaves the form: the FP64 state carries on
    b.iterate(1)
    assert len(b.case_history(0)["conv"]) == 6
    b.close()

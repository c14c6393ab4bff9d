"""Batches of cases (Mach / alpha sweeps on meshes of uneven size).

A batch holds every block of every case in one device arena, each case with its
own freestream.  The bar is the reference run on each case alone (the
batch_polar3 fixture, uneven meshes and freestreams) and, for more schemes,
the single-case solver: in FP64 every case of a batch must follow, bit for
bit, the primitives and Cl/Cd of the same case solved alone, through both
batch paths (the per-pass graph of e3d_iterate and the persistent cooperative
kernel of e3d_batch_solve).  Residual norms are
summed per tile in the persistent kernel, so they match within 1e-12.
"""
import numpy as np
import pytest
from conftest import max_rel, same

from euler3d_b200 import api
from euler3d_b200 import meshgen as mg
from euler3d_b200._lib import E3DError

pytestmark = pytest.mark.gpu

# (cells per side, blocks, Mach, alpha): uneven sizes, different freestreams
SWEEP = [(6, 1, 0.5, 0.0), (10, 2, 0.75, 2.5), (5, 1, 0.3, -1.5), (9, 3, 0.6, 5.0)]
O2_AUSM = dict(order=2, flux="ausm", gradient="greengauss", limiter="barthjespersen", stages=5, cfl=1.5)
O2_ROE = dict(order=2, flux="roe", gradient="leastsquares", limiter="venkatakrishnan", stages=4, cfl=1.2)
O1_ROE = dict(order=1, flux="roe", stages=5, cfl=1.5)
NEVER = -1e300


def _cases(tmp_path, opts, sweep=SWEEP):
    out = []
    for i, (n, nb, mach, aoa) in enumerate(sweep):
        d = mg.Deck(topology="", mach=mach, aoa_deg=aoa, **opts)
        out.append(api.Case(mg.write_case(str(tmp_path / f"c{i}"), n, nb, prefix=f"c{i}", deck=d)))
    return out


def _prims(solver, first_block, n_blocks):
    return [solver.get(first_block + b, "prim") for b in range(n_blocks)]


def _single(case, precision, iters):
    s = api.Solver(case, precision=precision)
    s.iterate(iters)
    return s


def _check_case(batch, c, first_block, single, hist=None, rms_tol=1e-12):
    for a, b in zip(_prims(batch, first_block, single.case.n_blocks), _prims(single, 0, single.case.n_blocks)):
        assert same(a, b)
    h = hist if hist is not None else batch.case_history(c)
    r = single.history()
    assert len(h["cl"]) == len(r["cl"])
    for col in ("cl", "cd"):
        assert same(h[col], r[col]), (c, col)
    assert max_rel(h["rms"], r["rms"]) < rms_tol


@pytest.mark.parametrize("opts", [O2_AUSM, O2_ROE, O1_ROE], ids=["o2_gg_bj_ausm", "o2_ls_venk_roe", "o1_roe"])
def test_batch_graph_path_matches_single_cases_fp64(tmp_path, opts):
    cases = _cases(tmp_path, opts)
    batch = api.Batch(cases, precision="fp64")
    batch.iterate(6)
    fb = 0
    for c, case in enumerate(cases):
        _check_case(batch, c, fb, _single(case, "fp64", 6))
        fb += case.n_blocks


@pytest.mark.parametrize("form", ["persistent", "per-pass"])
@pytest.mark.parametrize("opts", [O2_AUSM, O2_ROE, O1_ROE], ids=["o2_gg_bj_ausm", "o2_ls_venk_roe", "o1_roe"])
def test_batch_persistent_matches_single_cases_fp64(tmp_path, monkeypatch, opts, form):
    monkeypatch.setenv("E3D_BATCH_FORM", form)
    cases = _cases(tmp_path, opts)
    batch = api.Batch(cases, precision="fp64")
    done, ms = batch.solve_batch(12, NEVER, iters_per_launch=5)
    assert list(done) == [12] * len(cases) and ms > 0
    t = batch.tuning()
    assert t["tile_cells"] in (128, 256, 512) and t["mode"] == form
    fb = 0
    for c, case in enumerate(cases):
        _check_case(batch, c, fb, _single(case, "fp64", 12))
        fb += case.n_blocks


@pytest.mark.parametrize("form", ["persistent", "per-pass", "graph"])
def test_batch_matches_the_reference_run_case_by_case(tmp_path, monkeypatch, form):
    """Uneven meshes and freestreams in one batch, against the reference run
    on each case alone (tests/golden/batch_polar3.npz): every block's
    primitives after the first and the last iteration bit for bit, Cl/Cd
    identical, residual norms within 1e-12 (summation order)."""
    import json
    import os
    import sys

    from conftest import GOLDEN

    sys.path.insert(0, GOLDEN)
    import make_batch_golden as mbg

    z = np.load(os.path.join(GOLDEN, mbg.NAME + ".npz"))
    meta = json.loads(str(z["meta"]))
    cases = [api.Case(mbg.write_case(str(tmp_path / f"c{i}"), i)) for i in range(len(meta["cases"]))]
    batch = api.Batch(cases, precision="fp64")
    n = meta["iters"]
    if form == "graph":  # e3d_iterate on a batch: every case advances together
        batch.iterate(1)
    else:
        monkeypatch.setenv("E3D_BATCH_FORM", form)
        batch.solve_batch(1, NEVER, iters_per_launch=1)
    fb = 0
    for c, case in enumerate(cases):
        for b in range(case.n_blocks):
            assert same(batch.get(fb + b, "prim"), z[f"c{c}.iter1.b{b}.prim"]), (c, b)
        fb += case.n_blocks
    if form == "graph":
        batch.iterate(n - 1)
    else:
        batch.solve_batch(n, NEVER, iters_per_launch=3)
    fb = 0
    for c, case in enumerate(cases):
        for b in range(case.n_blocks):
            assert same(batch.get(fb + b, "prim"), z[f"c{c}.iter{n}.b{b}.prim"]), (c, b)
        h = batch.case_history(c)
        for col in ("cl", "cd"):
            assert same(h[col], z[f"c{c}.hist.{col}"]), (c, col)
        assert max_rel(h["rms"][:, 0], z[f"c{c}.hist.rms_ro"]) < 1e-12
        fb += case.n_blocks


@pytest.mark.parametrize("form", ["persistent", "per-pass"])
def test_batch_freezes_converged_cases_fp64(tmp_path, monkeypatch, form):
    """A case leaves the work list after the launch in which it reached the
    criterion; its state is then the single-case state of that many iterations."""
    monkeypatch.setenv("E3D_BATCH_FORM", form)
    cases = _cases(tmp_path, O1_ROE)
    K, ipl = 40, 4
    singles = [_single(c, "fp64", K) for c in cases]
    conv = [s.history()["conv"][:, 0] for s in singles]
    # a criterion every case but the slowest reaches within K iterations
    best = sorted(float(np.min(c)) for c in conv)
    crit = 0.5 * (best[-2] + best[-1])
    need = [int(np.argmax(c <= crit)) + 1 if np.any(c <= crit) else K for c in conv]
    assert min(need) < K and max(need) == K
    batch = api.Batch(cases, precision="fp64")
    done, _ = batch.solve_batch(K, crit, iters_per_launch=ipl)
    assert list(done) == need
    fb = 0
    for c, case in enumerate(cases):
        ran = min(K, -(-need[c] // ipl) * ipl)
        h = batch.case_history(c)
        assert len(h["cl"]) == ran
        _check_case(batch, c, fb, _single(case, "fp64", ran), hist=h)
        fb += case.n_blocks


@pytest.mark.parametrize("form", ["persistent", "per-pass"])
def test_batch_fp32_persistent_tracks_fp32_graph(tmp_path, monkeypatch, form):
    monkeypatch.setenv("E3D_BATCH_FORM", form)
    cases = _cases(tmp_path, O2_AUSM)
    a = api.Batch(cases, precision="fp32")
    a.solve_batch(20, NEVER, iters_per_launch=10)
    b = api.Batch(cases, precision="fp32")
    b.iterate(20)
    for blk in range(a.n_blocks):
        pa, pb = a.get(blk, "prim"), b.get(blk, "prim")
        assert np.max(np.abs(pa - pb) / np.maximum(np.abs(pb), 1e-3)) < 1e-5
    for c in range(len(cases)):
        ha, hb = a.case_history(c), b.case_history(c)
        assert abs(ha["cl"][-1] - hb["cl"][-1]) < 1e-5 * max(1.0, abs(hb["cl"][-1]))


O1_AUSM = dict(order=1, flux="ausm", stages=5, cfl=1.5)


@pytest.mark.parametrize("scheme", ["o2_roe", "o1_ausm"])
@pytest.mark.parametrize("form", ["persistent", "per-pass"])
def test_batch_fp64_fma_tracks_the_bitwise_batch(tmp_path, monkeypatch, form, scheme):
    """The FP64 batch kernels built with fused multiply-add solve the same
    equations: after 12 iterations every state within 1e-9.  First-order
    AUSM there also forms each cell's side quantities once per cell.
    Channel cases: a farfield face the flow runs along switches branch on the
    sign of u.n, which last-bit differences may flip."""
    monkeypatch.setenv("E3D_BATCH_FORM", form)
    cases = []
    for i, (n, nb, mach, aoa) in enumerate(SWEEP):
        d = mg.Deck(topology="", mach=mach, aoa_deg=aoa, **(O2_ROE if scheme == "o2_roe" else O1_AUSM))
        cases.append(api.Case(mg.write_case(str(tmp_path / f"k{i}"), n, nb, prefix=f"k{i}", deck=d,
                                            sides="channel")))
    a = api.Batch(cases, precision="fp64")
    a.solve_batch(12, NEVER, iters_per_launch=6)
    b = api.Batch(cases, precision="fp64")
    api.set_precision(b, "fp64-fma")
    b.solve_batch(12, NEVER, iters_per_launch=6)
    assert b.tuning()["mode"] == form
    for blk in range(a.n_blocks):
        pa, pb = a.get(blk, "prim"), b.get(blk, "prim")
        assert max_rel(pb, pa, floor=1e-3) < 1e-9
    for c in range(len(cases)):
        assert abs(a.case_history(c)["cl"][-1] - b.case_history(c)["cl"][-1]) < 1e-9


def test_batch_fp32_against_fp64_single(tmp_path):
    """FP32 batch within the FP32 variant's bar of each FP64 single case."""
    cases = _cases(tmp_path, O1_ROE, sweep=SWEEP[:2])
    batch = api.Batch(cases, precision="fp32")
    batch.solve_batch(200, NEVER, iters_per_launch=50)
    for c, case in enumerate(cases):
        ref = _single(case, "fp64", 200).history()
        h = batch.case_history(c)
        scale = max(abs(ref["cl"][-1]), abs(ref["cd"][-1]), 1e-3)
        for col in ("cl", "cd"):
            assert abs(h[col][-1] - ref[col][-1]) < 5e-3 * scale, (c, col)


def test_autotune_is_cached_per_size_bucket(tmp_path):
    cases = _cases(tmp_path, O1_ROE, sweep=SWEEP[:3])
    a = api.Batch(cases, precision="fp32")
    a.solve_batch(3, NEVER, iters_per_launch=3)
    b = api.Batch(cases, precision="fp32")
    b.solve_batch(3, NEVER, iters_per_launch=3)
    ta, tb = a.tuning(), b.tuning()
    assert tb["from_cache"] and (ta["tile_cells"], ta["grid"]) == (tb["tile_cells"], tb["grid"])
    # tuning never changes the solution
    for blk in range(a.n_blocks):
        assert same(a.get(blk, "prim"), b.get(blk, "prim"))


def test_batch_rejects_mixed_settings_and_hex_meshes(tmp_path):
    c0 = _cases(tmp_path / "a", O1_ROE, sweep=SWEEP[:1])[0]
    c1 = _cases(tmp_path / "b", O2_AUSM, sweep=SWEEP[:1])[0]
    with pytest.raises(E3DError):
        api.Batch([c0, c1], precision="fp32")
    hx = api.Case(mg.write_hex_case(str(tmp_path / "hex"), 4, deck=mg.Deck(topology="", **O1_ROE)))
    b = api.Batch([hx], precision="fp32")
    with pytest.raises(E3DError):
        b.solve_batch(2, NEVER)
    b.iterate(2)  # the per-pass path covers mixed-element meshes


def test_stalled_case_leaves_the_work_list(tmp_path):
    """A case whose residual stops falling (first-order Roe on the bump box with
    farfield side faces stalls near 2-4 orders) leaves the batch after the stall
    window; a channel case beside it keeps going to the criterion."""
    d1 = mg.Deck(topology="", mach=0.5, aoa_deg=2.0, **O1_ROE)
    stall = api.Case(mg.write_case(str(tmp_path / "s"), 6, 1, prefix="s", deck=d1, sides="farfield"))
    d2 = mg.Deck(topology="", mach=0.5, aoa_deg=2.0, **O1_ROE)
    conv = api.Case(mg.write_case(str(tmp_path / "c"), 6, 1, prefix="c", deck=d2, sides="channel"))
    b = api.Batch([stall, conv], precision="fp64", hist_capacity=8192)
    done, _ = b.solve_batch(30000, -7.0, iters_per_launch=100, stall_window=1500)
    hs, hc = b.case_history(0)["conv"][:, 0], b.case_history(1)["conv"][:, 0]
    assert hc.min() <= -7.0 and done[1] == int(np.argmax(hc <= -7.0)) + 1
    assert hs.min() > -7.0 and len(hs) < 30000
    # the stalled case stopped within one launch of the first window without a new minimum
    best = np.minimum.accumulate(hs)
    assert best[-1] > best[-1501] - 0.05


def test_non_finite_case_leaves_the_batch(tmp_path):
    """A case whose state turns non-finite (here: a negative density planted on
    the host) is dropped with iters_done = -1; the other cases are unaffected
    and match their single-case solves bit for bit."""
    cases = _cases(tmp_path, O1_ROE, sweep=SWEEP[:3])
    batch = api.Batch(cases, precision="fp64")
    prim = batch.get(0, "prim")
    prim[0] = -1.0  # density of cell 0 of case 0
    batch.set(0, "prim", prim)
    done, _ = batch.solve_batch(8, NEVER, iters_per_launch=4)
    assert done[0] == -1 and list(done[1:]) == [8, 8]
    fb = cases[0].n_blocks
    for c, case in enumerate(cases[1:], start=1):
        _check_case(batch, c, fb, _single(case, "fp64", 8))
        fb += case.n_blocks
    done2, _ = batch.solve_batch(12, NEVER, iters_per_launch=4)
    assert done2[0] == -1 and list(done2[1:]) == [12, 12]
    # a batch with no case left reports the failure
    solo = api.Batch(cases[:1], precision="fp64")
    p0 = solo.get(0, "prim")
    p0[0] = -1.0
    solo.set(0, "prim", p0)
    with pytest.raises(E3DError):
        solo.solve_batch(4, NEVER, iters_per_launch=2)

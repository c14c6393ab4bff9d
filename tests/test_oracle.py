"""Pins the C restatement oracle to the reference (CPU only).

The oracle runs on the reference's own geometry (golden dumps) and must give
the reference's arrays exactly after every RK stage, and its history over all
golden iterations.  Once pinned, GPU tests may use it on inputs the goldens do
not cover (larger meshes, perturbed states).
"""
import ctypes as C
import os

import numpy as np
import pytest
from conftest import Golden, golden_names, max_rel, same
from oracle_c import OracleBlock, OracleCase, case_oracle, lib, params_from_deck

from euler3d_b200.api import Case

RK = {1: ([1.0], [1.0]), 2: ([0.6, 1.0], [1.0, 0.0]), 3: ([0.6, 0.6, 1.0], [1.0, 0.0, 0.0]),
      4: ([0.25, 1.0 / 3.0, 0.5, 1.0], [1.0, 0.5, 0.0, 0.0]),
      5: ([0.2742, 0.2067, 0.5020, 0.5142, 1.0], [1.0, 0.0, 0.56, 0.0, 0.44])}


def _golden_case(g):
    p = params_from_deck(g.meta["deck"])
    blocks = [OracleBlock.from_golden(g, b) for b in range(g.n_blocks)]
    return blocks, p


@pytest.mark.parametrize("name", golden_names())
def test_oracle_stage_by_stage(name):
    g = Golden(name)
    blocks, p = _golden_case(g)
    oc = OracleCase(blocks, p)
    L = lib()
    alpha, beta = RK[p.stages]
    for b, blk in enumerate(blocks):
        # state after the initial halo = the reference's init dump
        blk.prim[:] = g[f"init.b{b}.prim"]
        s = C.byref(oc.arr[b])
        L.e3d_oracle_save_w0(s, C.byref(p))
        L.e3d_oracle_spectral_radius(s, C.byref(p))
        L.e3d_oracle_timestep(s, C.byref(p))
        for st in range(p.stages):
            if p.order == 2:
                L.e3d_oracle_gradients(s, p.gradient)
                L.e3d_oracle_limiters(s, p.limiter, C.c_double(p.omega), C.c_double(p.k))
            L.e3d_oracle_flux_conv(s, C.byref(p))
            L.e3d_oracle_flux_diss(s, C.byref(p), C.c_double(beta[st]))
            pre = f"it0.s{st}.res.b{b}."
            nr, na = blk.n_real, blk.n_all
            for k in ("conv_res", "diss_res", "w0"):
                assert same(getattr(blk, k).reshape(5, na)[:, :nr], g[pre + k].reshape(5, na)[:, :nr]), (b, st, k)
            for k in ("grad", "limiter", "dt", "spectral_radius"):
                assert same(getattr(blk, k), g[pre + k]), (b, st, k)
            L.e3d_oracle_update_internal(s, C.byref(p), C.c_double(alpha[st]))
            L.e3d_oracle_update_boundary(s, C.byref(p))
            assert same(blk.prim, g[f"it0.s{st}.upd.b{b}.prim"]), (b, st, "prim")


@pytest.mark.parametrize("name", golden_names())
def test_oracle_history(name, tmp_path):
    """Whole iterations on the host library's geometry (itself pinned bitwise to
    the reference) against the reference's history and final state."""
    g = Golden(name)
    deck = g.write_case(str(tmp_path))
    case = Case(deck)
    oc = case_oracle(case, os.path.join(tmp_path, os.path.basename(deck).rsplit(".", 1)[0] + ".top"))
    n = len(g.hist("iter"))
    h = oc.iterate(n)
    assert same(h[:, 0], g.hist("rms_ro"))  # same summation order as the reference: exact
    assert same(h[:, 5], g.hist("cl")) and same(h[:, 6], g.hist("cd"))
    assert same(h[:, 10], g.hist("ro_conv"))
    for b, blk in enumerate(oc.blocks):
        assert same(blk.prim, g[f"iter{n}.b{b}.prim"]), b


def test_oracle_catches_a_planted_error():
    """A mistake planted in the oracle's input (one face normal flipped) must
    show up as a mismatch: the comparison is not vacuous."""
    g = Golden("t3_o1_roe")
    blocks, p = _golden_case(g)
    blocks[0].a["face_normal"][3:6] *= -1.0
    oc = OracleCase(blocks, p)
    h = oc.iterate(2)
    assert not same(h[:, 5], g.hist("cl")[:2]) or not same(h[:, 0], g.hist("rms_ro")[:2])


def test_oracle_large_history_prefix():
    """The 48,000-cell bump channel: first 10 of the reference's 500 iterations."""
    g = Golden("bump20_o1_roe_500")
    import tempfile

    with tempfile.TemporaryDirectory() as td:
        deck = g.write_case(td)
        case = Case(deck)
        oc = case_oracle(case, os.path.join(td, "bump.top"))
        h = oc.iterate(10)
    assert max_rel(h[:, 0], g.hist("rms_ro")[:10]) == 0.0
    assert same(h[:, 5], g.hist("cl")[:10])

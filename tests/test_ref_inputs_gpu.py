"""GPU parity on the reference's own shipped meshes (NACA0012 hexahedra and
12 blocks of the ONERA M6 160-block partition).

The fixtures (tests/golden/ref_*.npz, made by the compiled reference, see
tests/golden/make_ref_inputs.py) hold SHA-256 hashes of the reference's arrays
instead of the arrays: bitwise equality of every compared array is equality
of its hash (signed zeros hashed as +0).  Bars as for the generated meshes:
the FP64 path reproduces every reference array after every RK stage and after
whole iterations; residual norms agree within 1e-12 relative (a tree
reduction on the device against the reference's sequential sums); Cl/Cd are
identical; the FP32 variant stays within the bounds derived from the model of
the FP32 build (tests/golden/fp32_bounds.json).
"""
import json
import os

import numpy as np
import pytest
from conftest import GOLDEN, Golden, array_hash, max_rel, ref_golden_names

from euler3d_b200 import api

pytestmark = pytest.mark.gpu

RMS_RTOL = 1e-12  # reduction order only


def _open(name, tmp_path, precision="fp64", **kw):
    g = Golden(name)
    case = api.Case(g.write_case(str(tmp_path)))
    return g, case, api.Solver(case, precision=precision, **kw)


@pytest.mark.parametrize("name", ref_golden_names())
def test_strategy_calls_stage_by_stage_on_reference_meshes(name, tmp_path):
    """One kernel per reference method, every array after every RK stage of
    the first iteration, block by block."""
    g, case, s = _open(name, tmp_path)
    rsol = api.ReferenceSolver(s)
    rk = rsol.runge_kutta_
    api.halo(s)
    for b in range(g.n_blocks):
        blk = api.Block(s, b)
        n_real = case.block_info(b).n_real
        assert array_hash(s.get(b, "prim")) == g.hash(f"init.b{b}.prim"), (b, "init")
        api.save_w0(blk)
        rsol.timestep_.computeSpectralRadius(blk)
        rsol.timestep_.computeTimestep(blk)
        for st in range(g.stages):
            rk.residual_calculator_.current_stage_ = st
            rk.residual_calculator_.computeResidual(blk)
            pre = f"it0.s{st}.res.b{b}."
            assert array_hash(s.get(b, "w0").reshape(5, n_real)) == g.hash(pre + "w0"), (b, st, "w0")
            assert array_hash(s.get(b, "dt")) == g.hash(pre + "dt"), (b, st, "dt")
            assert array_hash(s.get(b, "spectral_radius")) == g.hash(pre + "spectral_radius"), (b, st, "srad")
            if g.spec["deck"]["order"] == 2:
                assert array_hash(s.get(b, "grad")) == g.hash(pre + "grad"), (b, st, "grad")
                assert array_hash(s.get(b, "limiter")) == g.hash(pre + "limiter"), (b, st, "limiter")
            for k in ("conv_res", "diss_res"):
                assert array_hash(s.get(b, k).reshape(5, n_real)) == g.hash(pre + k), (b, st, k)
            rk.updater_.current_stage_ = st
            rk.updater_.updateInternalBlock(blk)
            rk.updater_.updateBoundary(blk)
            assert array_hash(s.get(b, "prim")) == g.hash(f"it0.s{st}.upd.b{b}.prim"), (b, st, "prim")


@pytest.mark.parametrize("name", ref_golden_names())
def test_fused_fp64_on_reference_meshes(name, tmp_path):
    """Fused stage kernels under a CUDA graph: the reference's arrays after
    iteration 1 and after the last iteration, and its whole history."""
    g, case, s = _open(name, tmp_path)
    s.iterate(1)
    for b in range(g.n_blocks):
        n_real = case.block_info(b).n_real
        assert array_hash(s.get(b, "prim")) == g.hash(f"iter1.b{b}.prim"), b
        for k in ("conv_res", "diss_res"):
            assert array_hash(s.get(b, k).reshape(5, n_real)) == g.hash(f"iter1.b{b}.{k}"), (b, k)
    n = len(g.hist("iter"))
    s.iterate(n - 1)
    h = s.history()
    for b in range(g.n_blocks):
        assert array_hash(s.get(b, "prim")) == g.hash(f"iter{n}.b{b}.prim"), b
    for q, col in enumerate(("rms_ro", "rms_uu", "rms_vv", "rms_ww", "rms_pp")):
        assert max_rel(h["rms"][:, q], g.hist(col)) < RMS_RTOL, col
    for col in ("cl", "cd", "cmx", "cmy", "cmz"):
        assert np.array_equal(h[col], g.hist(col)), col


@pytest.mark.parametrize("renumber", ["none", "rcm", "morton"])
@pytest.mark.parametrize("name", ["ref_naca_o2_gg_bj_ausm", "ref_onera_o2_ls_venk_roe"])
def test_fused_fp64_renumbered_on_reference_meshes(name, renumber, tmp_path):
    """Renumbered device order on the reference's meshes: the same arrays."""
    g, case, s = _open(name, tmp_path, renumber=renumber)
    n = len(g.hist("iter"))
    s.iterate(n)
    h = s.history()
    for b in range(g.n_blocks):
        assert array_hash(s.get(b, "prim")) == g.hash(f"iter{n}.b{b}.prim"), b
    for col in ("cl", "cd"):
        assert np.array_equal(h[col], g.hist(col)), col


@pytest.mark.parametrize("name", ref_golden_names())
def test_fp32_variant_on_reference_meshes(name, tmp_path):
    """The FP32 variant against the reference history (bounds derived per
    iteration from the FP32 model) and its final state against the FP64 path's,
    which is first checked to be the reference's."""
    bounds = json.load(open(os.path.join(GOLDEN, "fp32_bounds.json")))["fixtures"][name]
    g, case, s64 = _open(name, tmp_path / "a")
    n = len(g.hist("iter"))
    s64.iterate(n)
    ref = []
    for b in range(g.n_blocks):
        ref.append(s64.get(b, "prim").reshape(5, -1))
        assert array_hash(ref[-1]) == g.hash(f"iter{n}.b{b}.prim"), b
    _, _, s = _open(name, tmp_path / "b", precision="fp32")
    s.iterate(n)
    h = s.history()
    dev = np.abs(h["rms"][:, 0] - g.hist("rms_ro")) / np.abs(g.hist("rms_ro"))
    assert np.all(dev <= np.array(bounds["rms"])), ("rms", dev.max())
    for col in ("cl", "cd"):
        scale = max(np.max(np.abs(g.hist(col))), 1e-2)
        dev = np.abs(h[col] - g.hist(col)) / scale
        assert np.all(dev <= np.array(bounds[col])), (col, dev.max())
    st = max(float(np.max(np.abs(s.get(b, "prim").reshape(5, -1) - r) / np.maximum(np.abs(r), 1.0)))
             for b, r in enumerate(ref))
    assert st <= bounds["state"], ("state", st, bounds["state"])

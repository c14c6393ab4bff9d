"""The FP32 variant's parity bounds and the FP32 model they come from (CPU only).

tests/golden/fp32_bounds.json holds, per golden fixture and per iteration, the
bounds the GPU FP32 parity test applies.  They are derived, not chosen:
tests/golden/make_fp32_bounds.py runs the oracle built with float working
precision (oracle/libe3d_oracle32.so) under 16 rounding realisations and takes
twice the largest deviation from the reference.  These tests check that the
committed file is exactly what the model gives, and that the model is a real
FP32 model: it departs from the FP64 oracle by FP32 rounding, not more, on a
smooth case, and its seeds differ from one another.
"""
import json
import os
import sys

import numpy as np
import pytest
from conftest import GOLDEN, Golden, golden_names, ref_golden_names

sys.path.insert(0, GOLDEN)
import make_fp32_bounds as mb  # noqa: E402


def _committed():
    with open(mb.OUT) as f:
        return json.load(f)


# all seeds of the reference-mesh fixtures take minutes: the exact regeneration
# covers the generated meshes, and the reference-mesh bounds are checked
# against seed 0 and one perturbed seed
FAST = golden_names()
SLOW = ref_golden_names()


def test_bounds_cover_every_fixture():
    c = _committed()
    assert sorted(c["fixtures"]) == sorted(golden_names() + ref_golden_names())
    assert (c["seeds"], c["factor"], c["floor"]) == (mb.SEEDS, mb.FACTOR, mb.FLOOR)
    for name, b in c["fixtures"].items():
        n = len(Golden(name).hist("iter"))
        assert len(b["rms"]) == len(b["cl"]) == len(b["cd"]) == n, name


@pytest.mark.parametrize("name", FAST)
def test_bounds_are_what_the_model_gives(name):
    got = mb.compute([name])["fixtures"][name]
    want = _committed()["fixtures"][name]
    for k in ("rms", "cl", "cd"):
        assert np.array_equal(np.array(got[k]), np.array(want[k])), k
    assert got["state"] == want["state"]


@pytest.mark.parametrize("name", SLOW)
def test_bounds_hold_the_model_seeds(name):
    want = _committed()["fixtures"][name]
    for r in mb.fixture_deviations(name, (0, 3)):
        for k in ("rms", "cl", "cd"):
            assert np.all(mb.FACTOR * r[k] <= np.array(want[k])), k
        assert mb.FACTOR * r["state"] <= want["state"]


def test_model_is_fp32_and_seeds_differ():
    # first-order hexahedra: smooth, no switch near; the model departs from
    # the reference by FP32 rounding (well above FP64 rounding, well below 1e-4)
    rows = mb.fixture_deviations("h5_o1_ausm", range(3))
    for r in rows:
        assert 1e-8 < np.max(r["rms"]) < 1e-4
        assert 1e-9 < r["state"] < 1e-5
    assert not np.array_equal(rows[0]["rms"], rows[1]["rms"])
    assert not np.array_equal(rows[1]["rms"], rows[2]["rms"])


def test_fp64_oracle_ignores_the_seed(tmp_path):
    # the seed only perturbs the FP32 model: the FP64 library stays the reference
    from oracle_c import case_oracle, lib

    from euler3d_b200.api import Case

    g = Golden("t3_o1_roe")
    deck = g.write_case(str(tmp_path))
    case = Case(deck)
    oc = case_oracle(case, os.path.join(str(tmp_path), os.path.basename(deck).rsplit(".", 1)[0] + ".top"))
    lib().e3d_oracle_set_noise(5)
    try:
        h = oc.iterate(len(g.hist("iter")))
    finally:
        lib().e3d_oracle_set_noise(0)
    assert np.array_equal(h[:, 5], g.hist("cl"))
    assert np.array_equal(oc.blocks[0].prim, g[f"iter{len(g.hist('iter'))}.b0.prim"])

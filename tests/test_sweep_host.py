"""Host side of the polar sweeps (euler3d_b200/sweep.py): seeded case lists,
case files written by a spawn pool, and the iteration count to a drop.  Host
only."""
import os

import numpy as np

from euler3d_b200 import api
from euler3d_b200 import sweep as sw

SCHEME = dict(order=2, flux="ausm", gradient="greengauss", limiter="barthjespersen", omega=2.16e-16)


def test_polar_specs_are_seeded_and_in_range():
    a = sw.polar_specs(3, 64)
    b = sw.polar_specs(3, 64)
    assert a == b and len(a) == 64
    assert sw.polar_specs(4, 64) != a
    assert all(25 <= s.n <= 60 and 0.3 <= s.mach <= 0.8 and -2.0 <= s.aoa_deg <= 6.0 for s in a)
    assert len({s.name for s in a}) == 64


def test_pool_writes_the_same_files_as_a_serial_write(tmp_path):
    specs = sw.polar_specs(7, 3, n_range=(3, 4))
    pooled = sw.write_cases(str(tmp_path / "pool"), specs, SCHEME, processes=2)
    serial = sw.write_cases(str(tmp_path / "serial"), specs, SCHEME, processes=1)
    assert [os.path.basename(p) for p in pooled] == [os.path.basename(p) for p in serial]
    for p, q in zip(pooled, serial):
        d_p, d_q = os.path.dirname(p), os.path.dirname(q)
        assert sorted(os.listdir(d_p)) == sorted(os.listdir(d_q))
        files = [n for n in os.listdir(d_p) if os.path.isfile(os.path.join(d_p, n))]
        assert any(n.endswith(".su2") for n in files) and any(n.endswith(".top") for n in files)
        for name in files:
            assert open(os.path.join(d_p, name), "rb").read() == open(os.path.join(d_q, name), "rb").read()
    for spec, deck in zip(specs, pooled):
        case = api.Case(deck)  # the reference's formats round-trip through the host reader
        assert case.n_blocks == 1 and case.block_info(0).n_real == 6 * spec.n ** 3
        assert abs(case.deck.mach - spec.mach) < 1e-12 and abs(case.deck.aoa_deg - spec.aoa_deg) < 1e-12


def test_first_below_counts_iterations_like_the_stop_test():
    conv = np.array([0.0, -1.0, -3.0, -8.0, -7.5, -9.0])
    assert sw._first_below(conv, -8.0) == 4  # the 4th iteration is the first at or below -8
    assert sw._first_below(conv, -9.0) == 6
    assert sw._first_below(conv, -10.0) is None


class _FakeBatch:
    """Stands in for api.Batch on a host without a GPU: records the solve calls."""

    def __init__(self, cases, precision="fp32", hist_capacity=4096):
        self.cases, self.precision, self.calls = cases, precision, []

    def solve_batch(self, max_iter, criterion, iters_per_launch=10, stall_window=0):
        self.calls.append((self.precision, criterion))
        return np.zeros(len(self.cases), dtype=np.int32), 1.0

    def tuning(self):
        return {"mode": "per-pass"}

    def case_history(self, c):
        return {"conv": np.array([[0.0] * 5, [-9.0] * 5]), "cl": np.array([0.1, 0.1]), "cd": np.array([0.01, 0.01])}

    def close(self):
        pass


def _fake_set_precision(supports_delta, code=-1):
    from euler3d_b200 import _lib as L

    def set_precision(b, precision):
        if precision == "fp32-delta" and not supports_delta:
            raise L.E3DError(code, "the difference form covers first-order AUSM")
        b.precision = precision

    return set_precision


def test_finishing_form_is_the_difference_form_where_the_scheme_has_one(monkeypatch):
    monkeypatch.setattr(sw.api, "Batch", _FakeBatch)
    monkeypatch.setattr(sw.api, "set_precision", _fake_set_precision(True))
    r = sw.solve_batched(["a", "b"], -8.0, 100)
    assert [p["precision"] for p in r["phases"]] == ["fp32", "switch", "fp32-delta"]
    monkeypatch.setattr(sw.api, "set_precision", _fake_set_precision(False))
    r = sw.solve_batched(["a", "b"], -8.0, 100)
    assert [p["precision"] for p in r["phases"]] == ["fp32", "switch", "fp64-fma"]
    r = sw.solve_batched(["a"], -8.0, 100, fp64="fp64")  # an explicit form is used as given
    assert r["phases"][-1]["precision"] == "fp64"
    r = sw.solve_batched(["a"], -8.0, 100, switch_at=None)  # FP64 from the start
    assert [p["precision"] for p in r["phases"]] == ["fp64"]


def test_finishing_form_selection_passes_other_errors_on(monkeypatch):
    from euler3d_b200 import _lib as L

    monkeypatch.setattr(sw.api, "Batch", _FakeBatch)
    monkeypatch.setattr(sw.api, "set_precision", _fake_set_precision(False, code=-5))
    try:
        sw.solve_batched(["a"], -8.0, 100)
    except L.E3DError as e:
        assert e.code == -5
    else:
        raise AssertionError("a CUDA error from the switch must not fall back silently")

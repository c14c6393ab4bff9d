"""The solver's output files against the reference program's.

tests/golden/output_files.json holds the text the unmodified reference program
wrote for two small cases (tests/golden/make_output_golden.py):
./bin/Convergence.dat, ./bin/AerodynamicCoefficients.dat
(OutputTecplot.cpp:413-470) and its "Iter: ..." lines
(PostProcessing.cpp:263-266); one case stops at its iteration limit, the other
on the density criterion (PostProcessing.cpp:77).

On the CPU the fixture is pinned to the C oracle: the oracle's history,
printed the way a default C++ stream prints a double (six significant digits,
%g), gives the same text.  On the GPU, e3d_solve must write the same files.
"""
import json
import os
import subprocess
import sys

import pytest
from conftest import GOLDEN, REPO

from euler3d_b200.api import Case

sys.path.insert(0, GOLDEN)
import make_output_golden as mog  # noqa: E402

EXE = os.path.join(REPO, "euler3d_b200", "e3d_solve")
FIX = json.load(open(os.path.join(GOLDEN, "output_files.json")))
NAMES = sorted(FIX["outputs"])


def _g(x: float) -> str:
    return "%g" % x


def test_fixture_covers_both_stop_rules():
    assert set(NAMES) == set(mog.CASES) == {"iter_limit", "criterion"}
    for name in NAMES:
        n, nb, fields = mog.CASES[name]
        assert FIX["cases"][name] == [n, nb, fields]
    lim = FIX["outputs"]["iter_limit"]["iter_lines"]
    assert len(lim) == mog.CASES["iter_limit"][2]["max_iter"]
    crit = FIX["outputs"]["criterion"]["iter_lines"]
    assert len(crit) < mog.CASES["criterion"][2]["max_iter"]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_prints_the_reference_files(name, tmp_path):
    from oracle_c import case_oracle

    deck = mog.write_case(str(tmp_path), name)
    case = Case(deck)
    oc = case_oracle(case, os.path.join(str(tmp_path), f"{name}.top"))
    out = FIX["outputs"][name]
    n = len(out["iter_lines"])
    h = oc.iterate(n)
    conv = ["Iteration Cl Cd Cmx Cmy Cmz Density_Convergence Uu_Convergence Vv_Convergence Ww_Convergence "
            "Pressure_Convergence "]
    lines = []
    for i, r in enumerate(h):
        conv.append(" ".join([str(i)] + [_g(v) for v in r[5:10]] + [_g(v) for v in r[10:15]]))
        lines.append(f"Iter: {i} Convergence Ro: {_g(r[10])} cl: {_g(r[5])} cd: {_g(r[6])}")
    assert lines == out["iter_lines"]
    assert "\n".join(conv) + "\n" == out["files"]["Convergence.dat"]
    crit = case.deck.criterion
    stops = [i for i, r in enumerate(h) if i + 1 == case.deck.max_iter or r[10] <= crit]
    assert stops == [n - 1]
    ac = "Angle of attack Cl Cd Cmx Cmy Cmz\n" + " ".join(
        [_g(case.deck.aoa_deg)] + [_g(v) for v in h[-1, 5:10]]) + "\n"
    assert ac == out["files"]["AerodynamicCoefficients.dat"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_e3d_solve_writes_the_reference_files(name, tmp_path):
    deck = mog.write_case(str(tmp_path), name)
    r = subprocess.run([EXE, os.path.basename(deck)], cwd=str(tmp_path), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = FIX["outputs"][name]
    assert [ln for ln in r.stdout.splitlines() if ln.startswith("Iter: ")] == out["iter_lines"]
    for f, text in out["files"].items():
        with open(os.path.join(str(tmp_path), "bin", f)) as fh:
            assert fh.read() == text, f

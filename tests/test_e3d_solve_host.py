"""Host-side behaviour of the e3d_solve program, the counterpart of the
reference's main.cpp: argument errors, an unreadable case (exit 42, as the
reference exits on file errors), and no GPU.  Host only."""
import os
import subprocess

import pytest
import torch
from conftest import REPO

from euler3d_b200 import meshgen as mg

EXE = os.path.join(REPO, "euler3d_b200", "e3d_solve")
pytestmark = pytest.mark.skipif(not os.path.exists(EXE), reason="e3d_solve not built")


def _run(args, cwd):
    return subprocess.run([EXE] + args, cwd=cwd, capture_output=True, text=True, timeout=60)


def test_no_input_file(tmp_path):
    r = _run([], tmp_path)
    assert r.returncode == 255 and "ERROR: No input file" in r.stdout


@pytest.mark.parametrize("args", [["--bogus"], ["--check-every", "0"], ["--check-every", "-3"],
                                  ["--check-every", "x"]])
def test_bad_options(tmp_path, args):
    r = _run(["case.deck"] + args, tmp_path)
    assert r.returncode == 2, (args, r.stdout, r.stderr)


def test_unreadable_case(tmp_path):
    r = _run(["missing.deck"], tmp_path)
    assert r.returncode == 42 and "reading the case" in r.stderr


@pytest.mark.skipif(torch.cuda.is_available(), reason="a GPU is present")
def test_no_gpu(tmp_path):
    deck = mg.write_case(str(tmp_path), 3, 1, deck=mg.Deck(topology=""))
    r = _run([os.path.basename(deck)], tmp_path)
    assert r.returncode == 42 and "creating the solver" in r.stderr and "cuda" in r.stderr.lower()

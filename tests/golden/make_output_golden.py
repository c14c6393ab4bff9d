"""Golden fixture for the solver's output files: the text the unmodified
reference program writes for two small cases.

Test infrastructure.  The reference program (main.cpp) prints one
"Iter: ..." line per outer iteration and writes ./bin/Convergence.dat (one
line per iteration) and, when the stop test fires, ./bin/AerodynamicCoefficients.dat
(OutputTecplot.cpp:413-470; PostProcessing.cpp:59-83, 263-294).  e3d_solve
writes the same files from the same FP64 numbers, so their text must be
identical.  This script runs the reference program built by `make -C oracle`
(oracle/_ref/euler3D, serial, its own quadratic face search; the meshes are
small) and stores the texts:

    make -C oracle
    python tests/golden/make_output_golden.py

Cases: one that stops at its iteration limit (2 slab blocks, second order,
least squares + Venkatakrishnan + Roe) and one that stops on the density
criterion (1 block, first-order AUSM).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from euler3d_b200 import meshgen as mg  # noqa: E402

PROGRAM = os.path.join(REPO, "oracle", "_ref", "euler3D")
NAME = "output_files"
# name -> (hexahedra per side, blocks, deck fields)
CASES = {
    "iter_limit": (4, 2, dict(mach=0.6, aoa_deg=1.5, order=2, flux="roe", gradient="leastsquares",
                              limiter="venkatakrishnan", k=5.0, max_iter=25, criterion=-15.0)),
    "criterion": (3, 1, dict(mach=0.5, aoa_deg=2.0, order=1, flux="ausm", max_iter=400, criterion=-1.0)),
}


def write_case(directory: str, name: str) -> str:
    n, nb, fields = CASES[name]
    return mg.write_case(directory, n, nb, prefix=name, deck=mg.Deck(topology="", **fields))


def iter_lines(stdout: str) -> list[str]:
    return [ln for ln in stdout.splitlines() if ln.startswith("Iter: ")]


def main() -> None:
    if not os.path.exists(PROGRAM):
        sys.exit(f"{PROGRAM} missing: run `make -C oracle` first")
    out = {}
    for name in CASES:
        with tempfile.TemporaryDirectory() as td:
            deck = write_case(td, name)
            r = subprocess.run([PROGRAM, os.path.basename(deck)], cwd=td, capture_output=True, text=True,
                               check=True)
            files = {}
            for f in ("Convergence.dat", "AerodynamicCoefficients.dat"):
                with open(os.path.join(td, "bin", f)) as fh:
                    files[f] = fh.read()
            out[name] = dict(files=files, iter_lines=iter_lines(r.stdout))
            print(f"{name}: {len(out[name]['iter_lines'])} iterations")
    path = os.path.join(HERE, NAME + ".json")
    with open(path, "w") as fh:
        json.dump(dict(cases={k: [v[0], v[1], v[2]] for k, v in CASES.items()}, outputs=out), fh, indent=1)
    print(path)


if __name__ == "__main__":
    main()

"""Golden fixture for batches: uneven meshes and freestreams, each case run
alone by the compiled reference.

Test infrastructure.  A batch (e3d_batch_create) advances several cases in one
device arena; its FP64 result for every case must be the reference's for that
case run on its own.  The GPU batch tests compare with this fixture directly,
not only with the single-case GPU path.

    make -C oracle                          # oracle/_ref/e3d_refdriver
    python tests/golden/make_batch_golden.py

Cases (config-3-style scheme: AUSM + Green-Gauss + Barth-Jespersen, second
order, 5 stages, CFL 1.5): bump channels of 3^3 x 6, 6^3 x 6 in 2 slab blocks
and 4^3 x 6 tetrahedra, at Mach 0.35 / 0.62 / 0.78 and alpha -1.5 / 2.5 / 5.
For each case the fixture holds the reference's history and the primitives
of every block after iteration 1 and iteration ITERS.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(HERE))

from euler3d_b200 import meshgen as mg  # noqa: E402
from refdump import read_dump  # noqa: E402

DRIVER = os.path.join(REPO, "oracle", "_ref", "e3d_refdriver")
NAME = "batch_polar3"
ITERS = 8
SCHEME = dict(order=2, flux="ausm", gradient="greengauss", limiter="barthjespersen", omega=2.16e-16, stages=5,
              cfl=1.5)
# (hexahedra per side, blocks, Mach, alpha)
CASES = [(3, 1, 0.35, -1.5), (6, 2, 0.62, 2.5), (4, 1, 0.78, 5.0)]


def write_case(directory: str, i: int) -> str:
    n, nb, mach, aoa = CASES[i]
    deck = mg.Deck(topology="", mach=mach, aoa_deg=aoa, **SCHEME)
    return mg.write_case(directory, n, nb, prefix=f"c{i}", deck=deck)


def main() -> None:
    if not os.path.exists(DRIVER):
        sys.exit(f"{DRIVER} missing: run `make -C oracle` first")
    out = {}
    for i, (n, nb, _, _) in enumerate(CASES):
        with tempfile.TemporaryDirectory() as td:
            deck = write_case(td, i)
            dump = os.path.join(td, "dump")
            os.makedirs(dump)
            subprocess.run([DRIVER, deck, "--iters", str(ITERS), "--history", os.path.join(td, "hist.csv"),
                            "--quiet", "--dump-dir", dump, "--dump-every", "1"], cwd=td, capture_output=True,
                           check=True)
            hist = np.genfromtxt(os.path.join(td, "hist.csv"), delimiter=",", names=True)
            for col in hist.dtype.names:
                out[f"c{i}.hist.{col}"] = np.asarray(hist[col], dtype=np.float64)
            for it in (1, ITERS):
                d = read_dump(os.path.join(dump, f"iter{it}.bin"))
                for b in range(nb):
                    out[f"c{i}.iter{it}.b{b}.prim"] = d[f"b{b}.prim"]
    meta = dict(name=NAME, cases=CASES, scheme=SCHEME, iters=ITERS)
    out["meta"] = np.array(json.dumps(meta))
    path = os.path.join(HERE, NAME + ".npz")
    np.savez_compressed(path, **out)
    print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()

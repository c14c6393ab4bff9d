"""Derive the FP32 variant's error bounds from a model of the FP32 build.

Test infrastructure.  The FP32 variant (FP32 fluxes, gradients, limiters and
storage; FP64 conservative update, carried W and reductions) cannot reproduce
the FP64 reference bit for bit, so its parity test needs a bound per quantity.
The bounds here are not round numbers: they come from the oracle built a
second time with float working precision (oracle/libe3d_oracle32.so, see the
header of oracle/e3d_oracle.c), which rounds where the FP32 kernels round.

For every golden fixture (generated meshes and the reference's own) the model
runs the fixture's iterations SEEDS times:
seed 0 with every value rounded to nearest, seeds 1.. with each face flux left
as computed or moved one FP32 unit up or down by a seeded hash (what another
evaluation order, contraction or approximate division gives on the GPU).
Against the reference's FP64 history it records, per iteration,

    rms    |rho-residual norm - reference| / reference
    cl, cd |value - reference| / max(max |reference|, 1e-2)

and, after the last iteration, the largest |state - reference| /
max(|reference|, 1) over every cell and variable.  The bound of each is
FACTOR x the largest deviation over the seeds, and at least FLOOR.  The model
reproduces the B200 FP32 run closely (the LS + Barth-Jespersen + AUSM fixture:
density-residual deviation 1.03e-2 in the model, 1.033e-2 measured), and the
seeds show where a fixture sits at a discrete switch (a farfield face whose
u.n is zero in freestream takes the inflow or the outflow branch by rounding):
there the spread, and so the bound, widens after the switch.

    python tests/golden/make_fp32_bounds.py     # rewrites tests/golden/fp32_bounds.json

tests/test_fp32_bounds.py checks that the committed file is what this script
computes; the GPU parity test reads it.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
sys.path.insert(0, os.path.dirname(TESTS))
sys.path.insert(0, TESTS)

SEEDS = 16
FACTOR = 2.0
FLOOR = 2e-6
OUT = os.path.join(HERE, "fp32_bounds.json")


def deviations(g, hist: np.ndarray, blocks, ref_prims) -> dict:
    """Per-iteration rms/cl/cd deviations and the final state deviation
    (ref_prims: the reference's final primitives of each block)."""
    out = {}
    ref = g.hist("rms_ro")
    out["rms"] = np.abs(hist[:, 0] - ref) / np.abs(ref)
    for j, col in ((5, "cl"), (6, "cd")):
        scale = max(float(np.max(np.abs(g.hist(col)))), 1e-2)
        out[col] = np.abs(hist[:, j] - g.hist(col)) / scale
    st = 0.0
    for blk, r in zip(blocks, ref_prims):
        p = blk.prim.reshape(5, -1)
        r = r.reshape(5, -1)
        st = max(st, float(np.max(np.abs(p - r) / np.maximum(np.abs(r), 1.0))))
    out["state"] = st
    return out


def topology_path(g, deck: str) -> str:
    if "input" in g.spec:  # a reference-input fixture
        import make_ref_inputs

        return os.path.join(os.path.dirname(deck), make_ref_inputs.INPUTS[g.spec["input"]][1])
    return os.path.join(os.path.dirname(deck), os.path.basename(deck).rsplit(".", 1)[0] + ".top")


def fixture_deviations(name: str, seeds) -> list[dict]:
    from conftest import Golden, array_hash
    from oracle_c import case_oracle

    from euler3d_b200.api import Case

    g = Golden(name)
    rows = []
    with tempfile.TemporaryDirectory() as td:
        deck = g.write_case(td)
        case = Case(deck)
        top = topology_path(g, deck)
        n = len(g.hist("iter"))
        if "input" in g.spec:
            # reference-input fixtures store hashes, not arrays: the reference's
            # final state is the FP64 oracle's, checked against the hashes
            oc = case_oracle(case, top)
            oc.iterate(n)
            ref = [blk.prim.copy() for blk in oc.blocks]
            for b, r in enumerate(ref):
                assert array_hash(r) == g.hash(f"iter{n}.b{b}.prim"), (name, b)
        else:
            ref = [g[f"iter{n}.b{b}.prim"] for b in range(g.n_blocks)]
        for seed in seeds:
            oc = case_oracle(case, top, fp32=True, noise_seed=seed)
            hist = oc.iterate(n)
            rows.append(deviations(g, hist, oc.blocks, ref))
        case.close()
    return rows


def bounds_from(rows: list[dict]) -> dict:
    out = {}
    for k in ("rms", "cl", "cd"):
        m = np.max(np.stack([r[k] for r in rows]), axis=0)
        out[k] = [float(x) for x in np.maximum(FACTOR * m, FLOOR)]
    out["state"] = float(max(FACTOR * max(r["state"] for r in rows), FLOOR))
    return out


def compute(names=None) -> dict:
    from conftest import golden_names, ref_golden_names

    names = names or golden_names() + ref_golden_names()
    res = {"seeds": SEEDS, "factor": FACTOR, "floor": FLOOR, "fixtures": {}}
    for name in names:
        res["fixtures"][name] = bounds_from(fixture_deviations(name, range(SEEDS)))
    return res


def main() -> None:
    res = compute()
    with open(OUT, "w") as f:
        json.dump(res, f, indent=1)
    for name, b in res["fixtures"].items():
        print(f"{name:24s} rms <= {max(b['rms']):.2e}  cl <= {max(b['cl']):.2e}  cd <= {max(b['cd']):.2e}  "
              f"state <= {b['state']:.2e}")


if __name__ == "__main__":
    main()

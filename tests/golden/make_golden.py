"""Generate golden fixtures by running the compiled reference solver.

Test infrastructure.  Run here, where the reference sources exist:

    make -C oracle            # builds oracle/_ref/e3d_refdriver from the reference sources
    python tests/golden/make_golden.py [--only NAME] [--large]

For every case in CASES the bump-channel (or hexahedron channel) generator
writes the SU2 blocks, topology and deck; the reference's own solver objects
(oracle/_ref/e3d_refdriver, see oracle/refdriver/driver.cpp) run the case and
dump their arrays; the arrays needed by the tests are saved to
tests/golden/<name>.npz together with the generator parameters and a SHA-256 of
the generated files (so a test can detect generator drift).
"""
from __future__ import annotations

import argparse
import dataclasses
import hashlib
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
OMEGA = 2.16e-16  # the omega of the reference's shipped decks

# name -> generator + deck + run lengths
CASES = {
    "t3_o1_roe": dict(kind="tet", n=3, blocks=1, deck=dict(order=1, flux="roe", mach=0.5, aoa_deg=0.0),
                      iters=30, dump_iters=[1, 30]),
    "t3_o1_ausm_b3": dict(kind="tet", n=3, blocks=3, deck=dict(order=1, flux="ausm", mach=0.6, aoa_deg=2.0),
                          iters=30, dump_iters=[1, 30]),
    "t3_o1_roe_m15": dict(kind="tet", n=3, blocks=1, deck=dict(order=1, flux="roe", mach=1.5, aoa_deg=4.0),
                          iters=20, dump_iters=[1, 20]),
    "t4_o2_ls_venk_roe_b2": dict(kind="tet", n=4, blocks=2,
                                 deck=dict(order=2, flux="roe", gradient="leastsquares", limiter="venkatakrishnan",
                                           k=5.0, omega=OMEGA, mach=0.7, aoa_deg=1.25),
                                 iters=20, dump_iters=[1, 20]),
    "t3_o2_gg_bj_ausm": dict(kind="tet", n=3, blocks=1,
                             deck=dict(order=2, flux="ausm", gradient="greengauss", limiter="barthjespersen",
                                       omega=OMEGA, mach=0.6, aoa_deg=3.0),
                             iters=20, dump_iters=[1, 20]),
    "t3_o2_ls_bj_roe": dict(kind="tet", n=3, blocks=1,
                            deck=dict(order=2, flux="roe", gradient="leastsquares", limiter="barthjespersen",
                                      omega=OMEGA, mach=0.5, aoa_deg=-2.0),
                            iters=20, dump_iters=[1, 20]),
    "t3_o2_gg_venk_ausm_b3": dict(kind="tet", n=3, blocks=3,
                                  deck=dict(order=2, flux="ausm", gradient="greengauss", limiter="venkatakrishnan",
                                            k=5.0, omega=OMEGA, mach=0.8, aoa_deg=6.0),
                                  iters=20, dump_iters=[1, 20]),
    "t3_o2_ls_venk_roe_rk4": dict(kind="tet", n=3, blocks=1,
                                  deck=dict(order=2, flux="roe", gradient="leastsquares", limiter="venkatakrishnan",
                                            k=5.0, omega=OMEGA, mach=0.5, aoa_deg=1.0, stages=4, cfl=1.0),
                                  iters=20, dump_iters=[1, 20]),
    # the other four flux x gradient x limiter pairings, so all eight are pinned
    "t3_o2_gg_bj_roe": dict(kind="tet", n=3, blocks=1,
                            deck=dict(order=2, flux="roe", gradient="greengauss", limiter="barthjespersen",
                                      omega=OMEGA, mach=0.5, aoa_deg=2.0),
                            iters=20, dump_iters=[1, 20]),
    "t4_o2_gg_venk_roe_b2": dict(kind="tet", n=4, blocks=2,
                                 deck=dict(order=2, flux="roe", gradient="greengauss", limiter="venkatakrishnan",
                                           k=5.0, omega=OMEGA, mach=0.6, aoa_deg=1.0),
                                 iters=20, dump_iters=[1, 20]),
    "t3_o2_ls_bj_ausm": dict(kind="tet", n=3, blocks=1,
                             deck=dict(order=2, flux="ausm", gradient="leastsquares", limiter="barthjespersen",
                                       omega=OMEGA, mach=0.6, aoa_deg=3.0),
                             iters=20, dump_iters=[1, 20]),
    "t3_o2_ls_venk_ausm": dict(kind="tet", n=3, blocks=1,
                               deck=dict(order=2, flux="ausm", gradient="leastsquares", limiter="venkatakrishnan",
                                         k=5.0, omega=OMEGA, mach=0.6, aoa_deg=3.0),
                               iters=20, dump_iters=[1, 20]),
    "h5_o2_ls_venk_roe": dict(kind="hex", n=5, nz=1,
                              deck=dict(order=2, flux="roe", gradient="leastsquares", limiter="venkatakrishnan",
                                        k=5.0, omega=OMEGA, mach=0.6, aoa_deg=3.0, cfl=0.5),
                              iters=20, dump_iters=[1, 20]),
    "h5_o1_ausm": dict(kind="hex", n=5, nz=2, deck=dict(order=1, flux="ausm", mach=0.6, aoa_deg=3.0, cfl=0.5),
                       iters=20, dump_iters=[1, 20]),
    # residual smoothing: only the first smoothed residual is comparable (the
    # reference's dissipative w-momentum start value is never set)
    "irs_t3_o1_roe_b2": dict(kind="tet", n=4, blocks=2, deck=dict(order=1, flux="roe", mach=0.5, aoa_deg=2.0,
                                                                  smoothing=1),
                             iters=1, dump_iters=[1]),
}
# Full-size history goldens (minutes of reference CPU time): --large
LARGE = {
    # the 20^3 x 6 bump channel, first-order Roe, 500 iterations (the small plain-method workload)
    "bump20_o1_roe_500": dict(kind="tet", n=20, blocks=1, deck=dict(order=1, flux="roe", mach=0.5, aoa_deg=0.0),
                              iters=500, dump_iters=[], history_only=True),
    # the 80^3 x 6 bump channel in 16 slabs, LS + Venkatakrishnan + Roe (second-order workload), 3 iterations
    "bump80b16_o2_ls_venk_roe_3": dict(kind="tet", n=80, blocks=16,
                                       deck=dict(order=2, flux="roe", gradient="leastsquares",
                                                 limiter="venkatakrishnan", k=5.0, omega=OMEGA, mach=0.7,
                                                 aoa_deg=1.25),
                                       iters=3, dump_iters=[], history_only=True),
}

STATE_KEYS = ("prim", "conv_res", "diss_res", "w0", "limiter", "grad", "dt", "spectral_radius")
GEO_KEYS = ("counts", "face_cells", "face_nodes", "face_normal", "face_area", "face_center", "r_left", "r_right",
            "cell_nfaces", "cell_faces", "cell_cells", "cell_volume", "cell_center", "ls_weights", "marker_kind",
            "marker_size", "marker_cells", "wall_faces")


def write(spec: dict, directory: str) -> str:
    deck = mg.Deck(topology="", **spec["deck"])
    if spec["kind"] == "hex":
        return mg.write_hex_case(directory, spec["n"], spec.get("nz", 1), deck=deck)
    return mg.write_case(directory, spec["n"], spec.get("blocks", 1), deck=deck)


def files_sha(directory: str) -> str:
    h = hashlib.sha256()
    for name in sorted(os.listdir(directory)):
        p = os.path.join(directory, name)
        if os.path.isfile(p) and name.rsplit(".", 1)[-1] in ("su2", "top", "deck"):
            h.update(name.encode())
            with open(p, "rb") as f:
                h.update(f.read())
    return h.hexdigest()


def make(name: str, spec: dict) -> None:
    with tempfile.TemporaryDirectory() as td:
        deck = write(spec, td)
        dump = os.path.join(td, "dump")
        os.makedirs(dump)
        cmd = [DRIVER, deck, "--iters", str(spec["iters"]), "--history", os.path.join(td, "hist.csv"), "--quiet"]
        if not spec.get("history_only"):
            cmd += ["--dump-dir", dump, "--dump-init", "--dump-stages", "--dump-every", "1"]
        res = subprocess.run(cmd, cwd=td, capture_output=True, text=True, check=True)
        run = json.loads(res.stdout.strip().splitlines()[-1])
        out: dict[str, np.ndarray] = {}
        hist = np.genfromtxt(os.path.join(td, "hist.csv"), delimiter=",", names=True)
        for col in hist.dtype.names:
            out["hist." + col] = np.asarray(hist[col], dtype=np.float64)
        if not spec.get("history_only"):
            init = read_dump(os.path.join(dump, "init.bin"))
            nb = spec.get("blocks", 1)
            for b in range(nb):
                for k in GEO_KEYS + STATE_KEYS:
                    out[f"init.b{b}.{k}"] = init[f"b{b}.{k}"]
                for s in range(spec["deck"].get("stages", 5)):
                    for phase in ("res", "upd"):
                        d = read_dump(os.path.join(dump, f"it0_b{b}_s{s}_{phase}.bin"))
                        for k in STATE_KEYS:
                            out[f"it0.s{s}.{phase}.b{b}.{k}"] = d[f"b{b}.{k}"]
            for it in spec["dump_iters"]:
                d = read_dump(os.path.join(dump, f"iter{it}.bin"))
                for key, val in d.items():
                    out[f"iter{it}.{key}"] = val
        meta = dict(name=name, spec=spec, deck=dataclasses.asdict(mg.Deck(topology="", **spec["deck"])),
                    sha256=files_sha(td), reference_run=run)
        out["meta"] = np.array(json.dumps(meta))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        size = os.path.getsize(os.path.join(HERE, name + ".npz"))
        print(f"{name}: {run['cells']} cells x {run['iters']} iterations, {size/1024:.0f} KiB")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=None)
    ap.add_argument("--large", action="store_true")
    a = ap.parse_args()
    if not os.path.exists(DRIVER):
        sys.exit(f"{DRIVER} missing: run `make -C oracle` first")
    cases = dict(LARGE) if a.large else dict(CASES)
    for name, spec in cases.items():
        if a.only and a.only != name:
            continue
        make(name, spec)


if __name__ == "__main__":
    main()

"""Golden fixtures on the reference's own shipped meshes.

Test infrastructure.  The other goldens run meshes from this project's
generators; these run the files the reference ships, so the drop-in is checked
on reference-written SU2, real CONNEXION topology and cell orders this project
did not choose.  Run here, where the reference checkout and its compiled
driver exist:

    make -C oracle                        # oracle/_ref/e3d_refdriver
    python tests/golden/make_ref_inputs.py [--only NAME]

Inputs (tests/golden/ref_inputs/<input>.tar.xz, made once from the reference
files by this script; nothing at test time reads the reference checkout):

* naca0012_coarse: Meshes/naca0012_coarse.su2 verbatim (4,446 hexahedra, one
  layer in z: WALL airfoil, FARFIELD, two SYMMETRY planes), with a one-block
  topology file.  The reference's own decks for it (input_test1,
  input_testg2) name the SU2 file where the deck wants a topology file, or
  give omega as "2.16-16"; the decks here follow the survey's NACA runs
  (M 0.6, alpha 3, CFL 0.5).
* onera_m6_160b_sub12: 12 connected blocks of Meshes/oneraM6_160B (blocks
  41 40 56 55 53 46 45 42 44 43 58 59, 43,408 tetrahedra at the wing root:
  WALL and SYMMETRY faces and 64 CONNEXION markers between the 12).  Each
  block file is the reference's, except that a CONNEXION marker whose origin
  block is not among the 12 becomes a FARFIELD marker, moved before the
  remaining CONNEXION markers (the reference applies boundary conditions to
  the first n_real_boundaries markers only); the topology file keeps the
  reference's ghost-to-origin-cell lists of the kept connexions, with blocks
  renumbered 0..11.  The 120-block partition (input_onera120) is not usable:
  every one of its block files declares more markers (NMARK) than it holds,
  and the unmodified reference program ends with a segmentation fault while
  building block 0's faces (the host library rejects the file with
  E3D_ERR_FORMAT).
* wing_body_fitted_16x4x8: not a reference file: the body-fitted swept wing
  of the large configuration (euler3d_b200.wingmesh) at a small size, packed
  the same way so that its fixture does not depend on the generator staying
  unchanged.

For every case in CASES the compiled reference driver (oracle/_ref/
e3d_refdriver, the reference's own solver objects) runs the deck; the fixture
tests/golden/<name>.npz stores the history of every iteration and, instead of
the arrays (megabytes per stage), the SHA-256 of every array the GPU tests
compare: each RK stage of the first iteration (w0, dt, spectral radius,
gradients, limiters, residuals, primitives) and the primitives and residuals
after iterations 1 and N, plus the geometry arrays after ingest.  Signed zeros
are hashed as +0.
"""
from __future__ import annotations

import argparse
import dataclasses
import hashlib
import io
import json
import lzma
import os
import subprocess
import sys
import tarfile
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(HERE))

INPUTS_DIR = os.path.join(HERE, "ref_inputs")
DRIVER = os.path.join(REPO, "oracle", "_ref", "e3d_refdriver")
REFERENCE = os.environ.get("E3D_REFERENCE", os.path.join(os.path.dirname(REPO), "reference"))
OMEGA = 2.16e-16

ONERA_BLOCKS = [41, 40, 56, 55, 53, 46, 45, 42, 44, 43, 58, 59]

CASES = {
    "ref_naca_o1_roe": dict(input="naca0012_coarse", iters=20,
                            deck=dict(order=1, flux="roe", mach=0.6, aoa_deg=3.0, cfl=0.5)),
    "ref_naca_o2_gg_bj_ausm": dict(input="naca0012_coarse", iters=20,
                                   deck=dict(order=2, flux="ausm", gradient="greengauss", limiter="barthjespersen",
                                             omega=OMEGA, mach=0.6, aoa_deg=3.0, cfl=0.5)),
    "ref_naca_o2_ls_bj_ausm": dict(input="naca0012_coarse", iters=20,
                                   deck=dict(order=2, flux="ausm", gradient="leastsquares", limiter="barthjespersen",
                                             omega=OMEGA, mach=0.6, aoa_deg=3.0, cfl=0.5)),
    "ref_naca_o2_gg_venk_roe": dict(input="naca0012_coarse", iters=20,
                                    deck=dict(order=2, flux="roe", gradient="greengauss", limiter="venkatakrishnan",
                                              k=5.0, omega=OMEGA, mach=0.6, aoa_deg=3.0, cfl=0.5)),
    # input_onera160's scheme (Roe first order, M 0.65, alpha 4.25, CFL 1.5)
    "ref_onera_o1_roe": dict(input="onera_m6_160b_sub12", iters=10,
                             deck=dict(order=1, flux="roe", gradient="leastsquares", limiter="venkatakrishnan",
                                       k=5.0, omega=OMEGA, mach=0.65, aoa_deg=4.25, cfl=1.5)),
    # input_onera120's scheme (LS + Venkatakrishnan + Roe second order, M 0.8, alpha 1.25, CFL 1.5)
    "ref_onera_o2_ls_venk_roe": dict(input="onera_m6_160b_sub12", iters=5,
                                     deck=dict(order=2, flux="roe", gradient="leastsquares",
                                               limiter="venkatakrishnan", k=5.0, omega=OMEGA, mach=0.8,
                                               aoa_deg=1.25, cfl=1.5)),
    # the swept-wing configuration's scheme (AUSM + LS + Venkatakrishnan, M 0.8, alpha 3) on the
    # body-fitted wing mesh
    "ref_wingbf_o2_ls_venk_ausm": dict(input="wing_body_fitted_16x4x8", iters=20,
                                       deck=dict(order=2, flux="ausm", gradient="leastsquares",
                                                 limiter="venkatakrishnan", k=5.0, omega=OMEGA, mach=0.8,
                                                 aoa_deg=3.0, cfl=1.5)),
}

STAGE_KEYS = ("w0", "dt", "spectral_radius", "grad", "limiter", "conv_res", "diss_res")
GEO_KEYS = ("face_cells", "face_nodes", "face_normal", "face_area", "face_center", "r_left", "r_right", "cell_faces",
            "cell_cells", "cell_volume", "cell_center", "ls_weights", "marker_cells", "marker_kind", "marker_size",
            "wall_faces")


def array_hash(a: np.ndarray) -> str:
    """SHA-256 of an array's values (float64 or int32, little endian; -0.0 as +0.0)."""
    a = np.asarray(a)
    if a.dtype.kind == "f":
        a = np.ascontiguousarray(a, dtype="<f8") + 0.0
    else:
        a = np.ascontiguousarray(a, dtype="<i4")
    return hashlib.sha256(a.tobytes()).hexdigest()


def compared(key: str, a: np.ndarray, n_real: int, n_all: int) -> np.ndarray:
    """The part of a dumped array the tests read back from the solver:
    w0 and the residuals over real cells ([5][n_real]); the rest whole."""
    if key in ("w0", "conv_res", "diss_res"):
        return a.reshape(5, n_all)[:, :n_real]
    return a


# ----------------------------------------------------------------------------- inputs
def _su2_sections(text: str):
    """(header lines up to NMARK, [(tag, element lines)]) of an SU2 block file."""
    lines = text.split("\n")
    i = next(k for k, l in enumerate(lines) if l.startswith("NMARK="))
    head = lines[:i]
    marks = []
    k = i + 1
    while k < len(lines):
        if lines[k].startswith("MARKER_TAG="):
            tag = lines[k].split()[1]
            n = int(lines[k + 1].split()[1])
            marks.append((tag, lines[k + 2:k + 2 + n]))
            k += 2 + n
        else:
            k += 1
    return head, marks


def _write_su2(head, marks) -> str:
    out = list(head) + [f"NMARK= {len(marks)}"]
    for tag, elems in marks:
        out += [f"MARKER_TAG= {tag}", f"MARKER_ELEMS= {len(elems)}"] + list(elems)
    return "\n".join(out) + "\n"


def _read_topology(path: str):
    return _read_topology_text(open(path).read())


def _read_topology_text(text: str):
    """(block count, file lines, {block: (GhostCount, [(origin, cell lines)])})."""
    lines = text.split("\n")
    nb = int(lines[0].split()[1])
    pos = 1 + nb
    entries = {}
    while pos < len(lines) and lines[pos].strip():
        idx = int(lines[pos].split()[1])
        gc = int(lines[pos + 1].split()[1])
        m = int(lines[pos + 2].split()[1])
        pos += 3
        conns = []
        for _ in range(m):
            origin = int(lines[pos].split()[1])
            k = int(lines[pos + 1].split()[1])
            conns.append((origin, lines[pos + 2:pos + 2 + k]))
            pos += 2 + k
        entries[idx] = (gc, conns)
    return nb, lines[1:1 + nb], entries


def naca_files() -> dict[str, bytes]:
    su2 = open(os.path.join(REFERENCE, "Meshes", "naca0012_coarse.su2"), "rb").read()
    head, marks = _su2_sections(su2.decode())
    n_real = int(next(l for l in head if l.startswith("NELEM=")).split()[1])
    ghosts = sum(len(e) for t, e in marks if t != "CONNEXION")
    top = f"NBLOCK= 1\nnaca0012_coarse.su2\nBlock= 0\nGhostCount= {n_real + ghosts}\nNconnexion= 0\n"
    return {"naca0012_coarse.su2": su2, "naca0012_coarse.top": top.encode()}


def onera_files() -> dict[str, bytes]:
    root = os.path.join(REFERENCE, "Meshes", "oneraM6_160B")
    nb, _, entries = _read_topology(os.path.join(root, "oneraM6_160B.top"))
    new_id = {b: j for j, b in enumerate(ONERA_BLOCKS)}
    files = {}
    top = [f"NBLOCK= {len(ONERA_BLOCKS)}"] + [f"onera_sub_{j}.su2" for j in range(len(ONERA_BLOCKS))]
    for j, b in enumerate(ONERA_BLOCKS):
        head, marks = _su2_sections(open(os.path.join(root, f"oneraM6_160B{b}.su2")).read())
        gc, conns = entries[b]
        phys = [m for m in marks if m[0] != "CONNEXION"]
        cmarks = [m for m in marks if m[0] == "CONNEXION"]
        assert len(cmarks) == len(conns) and all(len(m[1]) == len(c[1]) for m, c in zip(cmarks, conns)), b
        n_real = int(next(l for l in head if l.startswith("NELEM=")).split()[1])
        assert gc == n_real + sum(len(m[1]) for m in phys), b
        lost = [("FARFIELD", m[1]) for m, c in zip(cmarks, conns) if c[0] not in new_id]
        kept = [(m, c) for m, c in zip(cmarks, conns) if c[0] in new_id]
        files[f"onera_sub_{j}.su2"] = _write_su2(head, phys + lost + [m for m, _ in kept]).encode()
        top += [f"Block= {j}", f"GhostCount= {n_real + sum(len(m[1]) for m in phys + lost)}",
                f"Nconnexion= {len(kept)}"]
        for _, (origin, cells) in kept:
            top += [f"Nmark= {new_id[origin]}", f"Nelems= {len(cells)}"] + list(cells)
    files["onera_sub.top"] = ("\n".join(top) + "\n").encode()
    return files


def wing_files() -> dict[str, bytes]:
    """The body-fitted swept wing of the large configuration at a small size
    (euler3d_b200.wingmesh: O-grid sections, rounded tip, slit beyond it,
    tunnel box), 16 x 4 x (6 + 2) hexahedra split into tetrahedra, 2 blocks."""
    from euler3d_b200 import wingmesh as wm

    with tempfile.TemporaryDirectory() as td:
        wm.write_body_fitted_wing_case(td, 16, 4, 6, 2, n_blocks=2, prefix="wing")
        return {f: open(os.path.join(td, f), "rb").read() for f in sorted(os.listdir(td))
                if f.endswith((".su2", ".top"))}


INPUTS = {"naca0012_coarse": (naca_files, "naca0012_coarse.top"),
          "onera_m6_160b_sub12": (onera_files, "onera_sub.top"),
          "wing_body_fitted_16x4x8": (wing_files, "wing.top")}


def pack(files: dict[str, bytes]) -> bytes:
    """A deterministic tar.xz of the case files (sorted, no times or owners)."""
    buf = io.BytesIO()
    with tarfile.open(fileobj=buf, mode="w", format=tarfile.USTAR_FORMAT) as tf:
        for name in sorted(files):
            ti = tarfile.TarInfo(name)
            ti.size = len(files[name])
            ti.mode = 0o644
            tf.addfile(ti, io.BytesIO(files[name]))
    return lzma.compress(buf.getvalue(), preset=9 | lzma.PRESET_EXTREME)


def unpack(input_name: str, directory: str) -> str:
    """Writes the input's case files into directory; returns the topology name."""
    with tarfile.open(os.path.join(INPUTS_DIR, input_name + ".tar.xz"), mode="r:xz") as tf:
        tf.extractall(directory, filter="data")
    return INPUTS[input_name][1]


def write_case(spec: dict, directory: str) -> str:
    """Case files plus the deck of one fixture; returns the deck path."""
    from euler3d_b200 import meshgen as mg

    os.makedirs(directory, exist_ok=True)
    top = unpack(spec["input"], directory)
    deck = mg.Deck(topology=top, **spec["deck"])
    path = os.path.join(directory, "case.deck")
    mg.write_deck(path, deck)
    os.makedirs(os.path.join(directory, "bin"), exist_ok=True)
    return path


def files_sha(directory: str) -> str:
    h = hashlib.sha256()
    for name in sorted(os.listdir(directory)):
        p = os.path.join(directory, name)
        if os.path.isfile(p) and name.rsplit(".", 1)[-1] in ("su2", "top", "deck"):
            h.update(name.encode())
            with open(p, "rb") as f:
                h.update(f.read())
    return h.hexdigest()


# ----------------------------------------------------------------------------- fixtures
def make(name: str, spec: dict) -> None:
    from refdump import read_dump

    from euler3d_b200 import meshgen as mg

    with tempfile.TemporaryDirectory() as td:
        deck = write_case(spec, td)
        dump = os.path.join(td, "dump")
        os.makedirs(dump)
        n = spec["iters"]
        cmd = [DRIVER, deck, "--iters", str(n), "--history", os.path.join(td, "hist.csv"), "--quiet",
               "--dump-dir", dump, "--dump-init", "--dump-stages", "--dump-every", "1"]
        res = subprocess.run(cmd, cwd=td, capture_output=True, text=True, check=True)
        run = json.loads(res.stdout.strip().splitlines()[-1])
        out: dict[str, np.ndarray] = {}
        hist = np.genfromtxt(os.path.join(td, "hist.csv"), delimiter=",", names=True)
        for col in hist.dtype.names:
            out["hist." + col] = np.asarray(hist[col], dtype=np.float64)
        init = read_dump(os.path.join(dump, "init.bin"))
        nb = sum(1 for k in init if k.endswith(".counts"))
        counts = np.stack([init[f"b{b}.counts"] for b in range(nb)])
        out["counts"] = counts
        hashes = {}
        for b in range(nb):
            n_real, n_all = int(counts[b, 0]), int(counts[b, 1])
            for k in GEO_KEYS:
                hashes[f"init.b{b}.{k}"] = array_hash(init[f"b{b}.{k}"])
            hashes[f"init.b{b}.prim"] = array_hash(init[f"b{b}.prim"])
            for s in range(spec["deck"].get("stages", 5)):
                d = read_dump(os.path.join(dump, f"it0_b{b}_s{s}_res.bin"))
                for k in STAGE_KEYS:
                    hashes[f"it0.s{s}.res.b{b}.{k}"] = array_hash(compared(k, d[f"b{b}.{k}"], n_real, n_all))
                d = read_dump(os.path.join(dump, f"it0_b{b}_s{s}_upd.bin"))
                hashes[f"it0.s{s}.upd.b{b}.prim"] = array_hash(d[f"b{b}.prim"])
        for it in sorted({1, n}):
            d = read_dump(os.path.join(dump, f"iter{it}.bin"))
            for b in range(nb):
                n_real, n_all = int(counts[b, 0]), int(counts[b, 1])
                for k in ("prim", "conv_res", "diss_res"):
                    hashes[f"iter{it}.b{b}.{k}"] = array_hash(compared(k, d[f"b{b}.{k}"], n_real, n_all))
        meta = dict(name=name, spec=spec, deck=dataclasses.asdict(mg.Deck(topology="", **spec["deck"])),
                    sha256=files_sha(td), reference_run=run, blocks=nb, hashes=hashes)
        out["meta"] = np.array(json.dumps(meta))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        size = os.path.getsize(os.path.join(HERE, name + ".npz"))
        print(f"{name}: {run['cells']} cells x {run['iters']} iterations, {nb} blocks, {size / 1024:.0f} KiB")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=None)
    ap.add_argument("--inputs-only", action="store_true")
    a = ap.parse_args()
    os.makedirs(INPUTS_DIR, exist_ok=True)
    for name, (fn, _) in INPUTS.items():
        path = os.path.join(INPUTS_DIR, name + ".tar.xz")
        data = pack(fn())
        with open(path, "wb") as f:
            f.write(data)
        print(f"{path}: {len(data) / 1024:.0f} KiB")
    if a.inputs_only:
        return
    if not os.path.exists(DRIVER):
        sys.exit(f"{DRIVER} missing: run `make -C oracle` first")
    for name, spec in CASES.items():
        if a.only and a.only != name:
            continue
        make(name, spec)


if __name__ == "__main__":
    main()

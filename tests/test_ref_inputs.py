"""The reference's own shipped meshes on the host side (CPU only).

Fixtures tests/golden/ref_*.npz were made by the compiled reference on the
NACA0012 hexahedron mesh and on 12 blocks of the ONERA M6 160-block
partition (tests/golden/make_ref_inputs.py).  Here: the packed inputs are
intact; the host library's ingest (SU2 reader, face builder, connectivity,
metrics) gives the reference's geometry bit for bit on them; and the C oracle
reproduces the reference's history and final state on them, which pins the
oracle on reference-written meshes too.
"""
import os
import sys

import numpy as np
import pytest
from conftest import GOLDEN, Golden, array_hash, ref_golden_names, same

from euler3d_b200.api import Case

sys.path.insert(0, GOLDEN)
import make_ref_inputs as mri  # noqa: E402

GEO = ("face_cells", "face_nodes", "face_normal", "face_area", "face_center", "r_left", "r_right", "cell_faces",
       "cell_cells", "cell_volume", "cell_center", "ls_weights", "marker_cells", "marker_kind", "marker_size",
       "wall_faces")


def _first_per_input():
    seen, out = set(), []
    for n in ref_golden_names():
        inp = Golden(n).spec["input"]
        if inp not in seen:
            seen.add(inp)
            out.append(n)
    return out


def test_every_reference_input_has_fixtures():
    assert {Golden(n).spec["input"] for n in ref_golden_names()} == set(mri.INPUTS)
    assert len(ref_golden_names()) == len(mri.CASES)


@pytest.mark.parametrize("name", _first_per_input())
def test_geometry_bitwise_on_reference_meshes(name, tmp_path):
    g = Golden(name)
    case = Case(g.write_case(str(tmp_path)))  # also checks the unpacked files' SHA-256
    assert case.n_blocks == g.n_blocks
    counts = g["counts"]
    for b in range(g.n_blocks):
        info = case.block_info(b)
        assert (info.n_real, info.n_all, info.n_faces, info.n_real_boundaries) == tuple(counts[b, :4]), b
        assert info.n_wall_faces == counts[b, 5]
        for k in GEO:
            assert array_hash(case.get(b, k)) == g.hash(f"init.b{b}.{k}"), (b, k)


@pytest.mark.parametrize("name", ref_golden_names())
def test_oracle_on_reference_meshes(name, tmp_path):
    from oracle_c import case_oracle

    g = Golden(name)
    deck = g.write_case(str(tmp_path))
    case = Case(deck)
    oc = case_oracle(case, os.path.join(str(tmp_path), mri.INPUTS[g.spec["input"]][1]))
    n = len(g.hist("iter"))
    h = oc.iterate(1)
    for b, blk in enumerate(oc.blocks):
        assert array_hash(blk.prim) == g.hash(f"iter1.b{b}.prim"), b
    h = np.vstack([h, oc.iterate(n - 1)]) if n > 1 else h
    assert same(h[:, 0], g.hist("rms_ro"))  # the reference's summation order: exact
    assert same(h[:, 5], g.hist("cl")) and same(h[:, 6], g.hist("cd"))
    for b, blk in enumerate(oc.blocks):
        assert array_hash(blk.prim) == g.hash(f"iter{n}.b{b}.prim"), b


def test_onera_subset_keeps_reference_topology(tmp_path):
    """In the packed ONERA subset every block lists its physical markers
    first, and each kept CONNEXION marker matches its topology list in size."""
    top = mri.unpack("onera_m6_160b_sub12", str(tmp_path))
    nb, files, entries = mri._read_topology(os.path.join(str(tmp_path), top))
    assert nb == len(mri.ONERA_BLOCKS) and sum(len(c) for _, c in entries.values()) == 64
    for j in range(nb):
        head, marks = mri._su2_sections(open(os.path.join(str(tmp_path), files[j].strip())).read())
        kinds = [t for t, _ in marks]
        first_conn = kinds.index("CONNEXION") if "CONNEXION" in kinds else len(kinds)
        assert all(k == "CONNEXION" for k in kinds[first_conn:]), j
        assert [len(e) for t, e in marks if t == "CONNEXION"] == [len(c) for _, c in entries[j][1]], j

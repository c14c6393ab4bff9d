"""Shared test helpers: the gpu marker, golden fixtures and case regeneration."""
from __future__ import annotations

import glob
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden_names(small_only: bool = True) -> list[str]:
    """Fixtures on generated meshes with their arrays stored (ref_* and the
    batch fixture batch_* excluded)."""
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
    names = [n for n in names if not n.startswith(("ref_", "batch_"))]
    if small_only:
        # bump*: full-size histories; irs*: residual smoothing, whose reference run
        # reads an unset array after the first smoothing (dedicated tests)
        names = [n for n in names if not n.startswith(("bump", "irs"))]
    return names


def ref_golden_names() -> list[str]:
    """Fixtures on the reference's own shipped meshes (array hashes, no arrays)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "ref_*.npz")))


class Golden:
    def __init__(self, name: str):
        self.name = name
        self.z = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.meta = json.loads(str(self.z["meta"]))
        self.spec = self.meta["spec"]

    def __getitem__(self, k):
        return self.z[k]

    def has(self, k):
        return k in self.z.files

    @property
    def n_blocks(self):
        return self.meta.get("blocks", self.spec.get("blocks", 1))

    @property
    def stages(self):
        return self.spec["deck"].get("stages", 5)

    def write_case(self, directory: str) -> str:
        """Regenerate the case files; fails if the generator output drifted."""
        sys.path.insert(0, GOLDEN)
        if "input" in self.spec:  # the reference's own meshes, unpacked from tests/golden/ref_inputs
            import make_ref_inputs  # noqa: E402

            deck = make_ref_inputs.write_case(self.spec, directory)
            assert make_ref_inputs.files_sha(directory) == self.meta["sha256"], "reference input files changed"
            return deck
        import make_golden  # noqa: E402

        deck = make_golden.write(self.spec, directory)
        assert make_golden.files_sha(directory) == self.meta["sha256"], "mesh generator output changed"
        return deck

    def hash(self, key: str) -> str:
        """SHA-256 of a reference array (ref_* fixtures; see make_ref_inputs.array_hash)."""
        return self.meta["hashes"][key]

    def hist(self, col: str) -> np.ndarray:
        return self.z["hist." + col]


@pytest.fixture(scope="session")
def golden():
    return Golden


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def same(a: np.ndarray, b: np.ndarray) -> bool:
    """Exact equality of every value (signed zeros compare equal; NaN never)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return a.shape == b.shape and bool(np.all(a == b))


def array_hash(a: np.ndarray) -> str:
    sys.path.insert(0, GOLDEN)
    import make_ref_inputs  # noqa: E402

    return make_ref_inputs.array_hash(a)


def max_rel(a: np.ndarray, b: np.ndarray, floor: float = 1e-300) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.abs(a - b)
    s = np.maximum(np.abs(b), floor)
    return float(np.max(d / s)) if d.size else 0.0

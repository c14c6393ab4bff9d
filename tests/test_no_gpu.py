"""Without a GPU the product fails loudly: every object that would run the path
(single case, batch, surrogate) and smoke() raise E3D_ERR_CUDA, and nothing
falls back to a CPU implementation.  Host only; skipped where a GPU is present."""
import pytest
import torch

from euler3d_b200 import api
from euler3d_b200 import meshgen as mg
from euler3d_b200._lib import ERRORS, E3DError

E3D_ERR_CUDA = next(k for k, v in ERRORS.items() if v == "E3D_ERR_CUDA")

pytestmark = pytest.mark.skipif(torch.cuda.is_available(), reason="a GPU is present")


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    d = tmp_path_factory.mktemp("nogpu")
    return api.Case(mg.write_case(str(d), 3, 1, deck=mg.Deck(topology="")))


@pytest.mark.parametrize("make", [lambda c: api.Solver(c, precision="fp64"),
                                  lambda c: api.Solver(c, precision="fp32"),
                                  lambda c: api.Batch([c], precision="fp32"),
                                  lambda c: api.Surrogate(seed=1, gamma=1.4)],
                         ids=["solver-fp64", "solver-fp32", "batch", "surrogate"])
def test_path_objects_raise(case, make):
    with pytest.raises(E3DError) as e:
        make(case)
    assert e.value.code == E3D_ERR_CUDA


def test_smoke_raises():
    import __graft_entry__ as g
    with pytest.raises(E3DError) as e:
        g.smoke()
    assert e.value.code == E3D_ERR_CUDA

"""The reference's own outer loop and post-processing with the B200 strategies
plugged in through include/e3d_reference_adapters.hpp (oracle/_ref/e3d_hybrid).

The reference computes norms, Cl/Cd and the convergence drop on its host
arrays after the GPU has advanced each block; the result must be the reference's
own history, value for value.  This is the C++ drop-in demonstration: the
adapters subclass the reference's FluxScheme / Gradient / Limiter interfaces.
"""
import os
import subprocess

import numpy as np
import pytest
from conftest import REPO, Golden, same

pytestmark = pytest.mark.gpu

HYBRID = os.path.join(REPO, "oracle", "_ref", "e3d_hybrid")


@pytest.mark.skipif(not os.path.exists(HYBRID), reason="e3d_hybrid not built (reference sources absent at build)")
@pytest.mark.parametrize("name", ["t4_o2_ls_venk_roe_b2", "t3_o2_gg_bj_ausm", "t3_o1_roe", "h5_o2_ls_venk_roe",
                                  "t3_o2_gg_venk_ausm_b3"])
def test_reference_loop_with_gpu_strategies(name, tmp_path):
    g = Golden(name)
    deck = g.write_case(str(tmp_path))
    n = len(g.hist("iter"))
    hist = os.path.join(tmp_path, "h.csv")
    subprocess.run([HYBRID, os.path.basename(deck), "--iters", str(n), "--history", hist], cwd=tmp_path,
                   check=True, capture_output=True, timeout=600)
    h = np.genfromtxt(hist, delimiter=",", names=True)
    for col in ("cl", "cd", "cmx", "cmy", "cmz", "rms_ro", "ro_conv"):
        assert same(h[col], g.hist(col)), col

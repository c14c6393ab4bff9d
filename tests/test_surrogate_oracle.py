"""The surrogate's CPU oracle pinned on its own: BF16 rounding against torch's
conversion, and the analytic gradient against central finite differences."""
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as mo  # noqa: E402


def _random_params(rng, scale=0.3):
    p = np.zeros(mo.N_PARAM)
    W1, b1, W2, b2, W3, b3, W4, b4 = (slice(mo.OFF_W1, mo.OFF_B1), slice(mo.OFF_B1, mo.OFF_W2),
                                      slice(mo.OFF_W2, mo.OFF_B2), slice(mo.OFF_B2, mo.OFF_W3),
                                      slice(mo.OFF_W3, mo.OFF_B3), slice(mo.OFF_B3, mo.OFF_W4),
                                      slice(mo.OFF_W4, mo.OFF_B4), slice(mo.OFF_B4, mo.N_PARAM))
    w1 = rng.normal(0, scale, (mo.H, mo.IN))
    w1[:, mo.N_IN:] = 0
    p[W1] = w1.ravel()
    for s in (W2, W3):
        p[s] = rng.normal(0, scale / np.sqrt(8), s.stop - s.start)
    w4 = rng.normal(0, scale / 4, (mo.OUT, mo.H))
    w4[mo.N_OUT:] = 0
    p[W4] = w4.ravel()
    for s in (b1, b2, b3):
        p[s] = rng.normal(0, 0.1, s.stop - s.start)
    p[b4][:mo.N_OUT] = rng.normal(0, 0.1, mo.N_OUT)
    return p


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(0, 1, 20000), rng.normal(0, 1e-3, 1000), rng.normal(0, 1e4, 1000)])
    # exact ties: the 16 low bits 0x8000
    ties = (rng.integers(0, 2**31, 2000, dtype=np.uint64) & 0x7FFF0000 | 0x8000).astype(np.uint32).view(np.float32)
    ties = ties[np.isfinite(ties)]
    x = np.concatenate([x.astype(np.float32), ties, -ties])
    ours = mo.bf16(x)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32))


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = _random_params(rng)
    x = np.zeros((48, mo.IN))
    x[:, :mo.N_IN] = rng.normal(0, 1, (48, mo.N_IN))
    t = rng.normal(0, 1, (48, mo.N_OUT))
    _, g = mo.loss_and_grad(p, x, t, bf=False)
    w1_used = (mo.OFF_W1 + np.arange(mo.H)[:, None] * mo.IN + np.arange(mo.N_IN)[None, :]).ravel()
    pools = [w1_used] + [np.arange(a, b) for a, b in
                         ((mo.OFF_B1, mo.OFF_W2), (mo.OFF_W2, mo.OFF_B2), (mo.OFF_B2, mo.OFF_W3),
                          (mo.OFF_W3, mo.OFF_B3), (mo.OFF_B3, mo.OFF_W4), (mo.OFF_W4, mo.OFF_W4 + mo.N_OUT * mo.H),
                          (mo.OFF_B4, mo.OFF_B4 + mo.N_OUT))]
    idx = np.concatenate([rng.choice(pool, min(8, pool.size), replace=False) for pool in pools])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss_and_grad(pp, x, t, bf=False)[0] - mo.loss_and_grad(pm, x, t, bf=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, np.max(np.abs(g))), (i, fd, g[i])
    # padding parameters carry no gradient
    w1 = g[mo.OFF_W1:mo.OFF_B1].reshape(mo.H, mo.IN)
    assert np.all(w1[:, mo.N_IN:] == 0)
    assert np.all(g[mo.OFF_W4:mo.OFF_B4].reshape(mo.OUT, mo.H)[mo.N_OUT:] == 0)


def test_bf16_mode_stays_close_to_fp64():
    rng = np.random.default_rng(2)
    p = _random_params(rng)
    x = np.zeros((64, mo.IN))
    x[:, :mo.N_IN] = rng.normal(0, 1, (64, mo.N_IN))
    t = rng.normal(0, 1, (64, mo.N_OUT))
    l64, g64 = mo.loss_and_grad(p, x, t, bf=False)
    lbf, gbf = mo.loss_and_grad(p, mo.bf16(x.astype(np.float32)).astype(np.float64), t, bf=True)
    assert abs(lbf - l64) < 2e-2 * l64
    assert np.linalg.norm(gbf - g64) < 5e-2 * np.linalg.norm(g64)

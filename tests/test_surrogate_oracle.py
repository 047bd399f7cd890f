"""CPU checks of the surrogate network's oracle (oracle/oracle_surrogate.py).

The network is the learned part of the scatter surrogate; it has no
counterpart in the reference project, so its oracle is pinned by its own
mathematics: the fp64 gradient must match central finite differences of the
fp64 loss, and the bf16-rounded variant (the arithmetic the tensor cores do)
must stay close to the fp64 one.
"""
import numpy as np

import oracle_surrogate as osr

SHAPE = dict(n_crystals=7, layers=3, width=16, freqs=3, emb=8)
GRID = (5, 4, 3)


def _batch(seed=0, B=9, ncol=12):
    rng = np.random.default_rng(seed)
    N = SHAPE["n_crystals"]
    vox = rng.integers(0, int(np.prod(GRID)), B)
    col = rng.integers(0, ncol, B)
    rho = rng.normal(size=(N, ncol)).astype(np.float32)
    wgt = rng.uniform(0.1, 2.0, size=(N, ncol)).astype(np.float32)
    return vox, col, rho, wgt


def test_fp64_gradient_matches_finite_differences():
    p, offs, shapes = osr.init_params(seed=3, **SHAPE)
    p = p.astype(np.float64)
    vox, col, rho, wgt = _batch()
    _, g = osr.loss_grad(p, offs, shapes, GRID, SHAPE["freqs"], vox, col, rho, wgt, round_bf16=False)
    rng = np.random.default_rng(1)
    # every block, a few coordinates each
    for o, s in zip(offs, shapes):
        for i in rng.choice(int(np.prod(s)), min(4, int(np.prod(s))), replace=False):
            k = o + int(i)
            h = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[k] += h
            pm[k] -= h
            lp, _ = osr.loss_grad(pp, offs, shapes, GRID, SHAPE["freqs"], vox, col, rho, wgt, round_bf16=False)
            lm, _ = osr.loss_grad(pm, offs, shapes, GRID, SHAPE["freqs"], vox, col, rho, wgt, round_bf16=False)
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])


def test_bf16_variant_is_close_to_fp64():
    p, offs, shapes = osr.init_params(seed=4, **SHAPE)
    vox, col, rho, wgt = _batch(seed=2)
    l64, g64 = osr.loss_grad(p, offs, shapes, GRID, SHAPE["freqs"], vox, col, rho, wgt, round_bf16=False)
    l16, g16 = osr.loss_grad(p, offs, shapes, GRID, SHAPE["freqs"], vox, col, rho, wgt, round_bf16=True)
    assert abs(l16 - l64) <= 2e-2 * abs(l64)
    assert np.linalg.norm(g16 - g64) <= 3e-2 * np.linalg.norm(g64)


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0, 3.0e38], dtype=np.float32)
    y = osr.bf16(x)
    assert y[0] == 1.0 and y[1] == 1.0          # halfway: ties to even
    assert y[2] == 1.0 + 2 ** -7                 # above halfway rounds up
    assert y[3] == -2.5 and y[4] == 0.0


def test_adam_matches_closed_form_first_step():
    w = np.array([1.0, -2.0])
    g = np.array([0.5, -0.25])
    w1, m, v = osr.adam(w, g, np.zeros(2), np.zeros(2), 1, 0.1)
    # the first bias-corrected step is lr * sign(g) (up to eps)
    np.testing.assert_allclose(w1, w - 0.1 * np.sign(g), rtol=0, atol=1e-6)

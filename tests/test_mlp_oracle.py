"""The network checker's own gradient against finite differences (CPU)."""
import numpy as np

import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    params = np.concatenate([rng.normal(0, 0.3, M.NPARAM), rng.normal(0, 1, M.F), np.ones(M.F)])
    rows = np.concatenate([rng.normal(0, 1, (32, M.F)), rng.normal(0, 1, (32, M.O))], axis=1)
    loss, g = M.loss_and_grad(params, rows)
    idx = rng.choice(M.NPARAM, 40, replace=False)
    h = 1e-6
    for k in idx:
        p1, p2 = params.copy(), params.copy()
        p1[k] += h
        p2[k] -= h
        fd = (M.loss_and_grad(p1, rows)[0] - M.loss_and_grad(p2, rows)[0]) / (2 * h)
        assert abs(fd - g[k]) < 1e-7 + 1e-5 * abs(fd)


def test_bf16_rounding_and_emulated_gradient():
    # round to nearest even at 8 significant bits
    assert M.bf(np.array([1.0]))[0] == 1.0
    assert M.bf(np.array([1.0 + 2.0 ** -8]))[0] == 1.0                 # tie to even
    assert M.bf(np.array([1.0 + 3 * 2.0 ** -8]))[0] == 1.0 + 2.0 ** -6  # tie to even (up)
    assert M.bf(np.array([1.0 + 2.0 ** -7]))[0] == 1.0 + 2.0 ** -7      # exact
    rng = np.random.default_rng(2)
    params = np.concatenate([rng.normal(0, 0.3, M.NPARAM), rng.normal(0, 1, M.F), np.ones(M.F)])
    rows = np.concatenate([rng.normal(0, 1, (256, M.F)), rng.normal(0, 1, (256, M.O))], axis=1)
    _, g = M.loss_and_grad(params, rows)
    _, gb = M.loss_and_grad(params, rows, bf16=True)
    # the BF16 operands move the gradient by well under a percent
    assert np.linalg.norm(gb - g) / np.linalg.norm(g) < 1e-2

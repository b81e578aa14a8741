"""Dipole-guess network: GPU forward/backward against the CPU checker, and
what the trained network gains over the first-order start."""
import numpy as np
import pytest

import mlp_oracle as M
from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _pw(seed=3):
    return systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=seed,
                                     n_steps=10)


def test_forward_and_gradient_match_cpu():
    ens = engine.GpuEnsemble(_pw())
    ens.mlp_init(capacity_frames=4, seed=7)
    ens.compute_forces(L.TERM_IND_SHORT)
    feats = ens.mlp_features()
    assert np.all(np.isfinite(feats))
    rng = np.random.default_rng(1)
    params = ens.mlp_params()
    # a non-trivial normalisation
    params[M.NPARAM:M.NPARAM + M.F] = feats.mean(0)
    params[M.NPARAM + M.F:] = 1.0 / (feats.std(0) + 1e-3)
    ens.mlp_params(set_to=params)
    y = ens.mlp_eval(feats)
    y_ref, _ = M.forward(params, feats)
    assert np.max(np.abs(y - y_ref)) < 1e-4 * (1 + np.abs(y_ref).max())
    rows = np.concatenate([feats[:512], rng.normal(0, 1, (512, 3)).astype(np.float32)], axis=1)
    g = ens.mlp_gradient(rows)
    _, g_ref = M.loss_and_grad(params, rows)
    rel = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    print("gradient rel err", rel)
    assert rel < 1e-4


def test_learned_guess_cuts_iterations():
    s = _pw(seed=5)
    ens = engine.GpuEnsemble(s)
    ens.set_solver(tol=2.0819e-8, max_iter=500, guess=L.GUESS_DIRECT)
    lf = engine.LFIntegrator(ens)
    lf.start()
    lf.run(2)                      # the guess starts from the last two solves
    ens.mlp_init(capacity_frames=40, seed=3)
    for _ in range(40):            # training frames from the solver itself
        lf.run(2)
        ens.compute_forces(L.TERM_IND_SHORT)
        ens.mlp_collect()
    loss = ens.mlp_train(epochs=30, batch=2048, lr=2e-3)
    print("final loss", loss)
    lf.run(5)
    ens.compute_forces(L.TERM_IND_SHORT)
    it_direct, _ = ens.solver_stats()
    p_direct = ens.polarization()["p"]
    ens.set_solver(tol=2.0819e-8, max_iter=500, guess=L.GUESS_LEARNED)
    ens.compute_forces(L.TERM_IND_SHORT)
    it_learned, _ = ens.solver_stats()
    p_learned = ens.polarization()["p"]
    print("iterations direct", it_direct, "learned", it_learned)
    # same tolerance from either start
    assert np.sqrt(np.mean((p_learned - p_direct) ** 2)) < 1e-7
    assert it_learned < it_direct

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
    # tensor-core forward (BF16 operands, FP32 sums) against the checker with
    # the same operands rounded to BF16, and against plain FP64
    y = ens.mlp_eval(feats)
    y_bf, _ = M.forward(params, feats, bf16=True)
    y_64, _ = M.forward(params, feats)
    scale = 1 + np.abs(y_64).max()
    print("forward err vs bf16 checker", np.max(np.abs(y - y_bf)) / scale, "vs fp64", np.max(np.abs(y - y_64)) / scale)
    assert np.max(np.abs(y - y_bf)) < 2e-3 * scale
    assert np.max(np.abs(y - y_64)) < 3e-2 * scale
    rows = np.concatenate([feats[:512], rng.normal(0, 1, (512, 3)).astype(np.float32)], axis=1)
    g = ens.mlp_gradient(rows)
    _, g_bf = M.loss_and_grad(params, rows, bf16=True)
    _, g_64 = M.loss_and_grad(params, rows)
    rel_bf = np.linalg.norm(g - g_bf) / np.linalg.norm(g_bf)
    rel_64 = np.linalg.norm(g - g_64) / np.linalg.norm(g_64)
    print("gradient rel err vs bf16 checker", rel_bf, "vs fp64", rel_64)
    assert rel_bf < 5e-3
    assert rel_64 < 3e-2
    # per parameter group, so that no block of the gradient hides in the norm
    k = 0
    for name, shp in M.SIZES:
        m = int(np.prod(shp))
        gg, rr = g[k:k + m], g_bf[k:k + m]
        assert np.linalg.norm(gg - rr) <= 1e-2 * np.linalg.norm(rr) + 1e-7, name
        k += m


def _iters(ens, lf, guess, steps=10):
    ens.set_solver(tol=2.0819e-8, max_iter=500, guess=guess)
    lf.run(3)
    its, first = [], []
    for _ in range(steps):
        lf.run(1)
        its.append(ens.solver_stats()[0])
        first.append(ens.solver_trace()[0])
    return float(np.mean(its)), float(np.exp(np.mean(np.log(first))))


def test_learned_guess_beats_the_same_guess_without_network():
    # the benchmark's 4096-molecule water: the network corrects the
    # second-order extrapolation (its base); switched off, the same
    # extrapolation (and the first-order guess) is the method without it
    s = systems.polarizable_water(nmol=4096, kmax=18, seed=1)
    ens = engine.GpuEnsemble(s, precision="mixed")
    ens.set_solver(tol=2.0819e-8, max_iter=500, guess=L.GUESS_FIRST_ORDER)
    lf = engine.LFIntegrator(ens)
    lf.start()
    lf.run(1500)
    it_fo, r_fo = _iters(ens, lf, L.GUESS_FIRST_ORDER)
    it_x2, r_x2 = _iters(ens, lf, L.GUESS_EXTRAP2)
    ens.mlp_init(capacity_frames=40, seed=1)
    ens.mlp_set_base(2)
    for _ in range(40):            # training frames from the solver itself
        lf.run(5)
        ens.compute_forces(L.TERM_IND_SHORT)
        ens.mlp_collect()
    loss = ens.mlp_train(epochs=30, batch=16384, lr=2e-3)
    it_ml, r_ml = _iters(ens, lf, L.GUESS_LEARNED)
    print("iterations first-order", it_fo, "extrap2", it_x2, "learned", it_ml, "loss", loss)
    print("first update RMS", r_fo, r_x2, r_ml)
    # the start is closer and the solve shorter than with the network off
    assert r_ml < 0.95 * r_x2 and r_ml < 0.95 * r_fo
    assert it_ml < min(it_fo, it_x2)
    # the same tolerance from either start, at one configuration
    ens.compute_forces(L.TERM_IND_SHORT)
    p_learned = ens.polarization()["p"]
    ens.set_solver(tol=2.0819e-8, max_iter=500, guess=L.GUESS_DIRECT)
    ens.compute_forces(L.TERM_IND_SHORT)
    p_direct = ens.polarization()["p"]
    assert np.sqrt(np.mean((p_learned - p_direct) ** 2)) < 1e-7
    ens.close()


def test_learned_guess_small_system_converges_to_same_dipoles():
    s = _pw(seed=5)
    ens = engine.GpuEnsemble(s)
    ens.set_solver(tol=2.0819e-8, max_iter=500, guess=L.GUESS_DIRECT)
    lf = engine.LFIntegrator(ens)
    lf.start()
    lf.run(2)                      # the guess starts from the last two solves
    ens.mlp_init(capacity_frames=40, seed=3)
    for _ in range(40):
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
    assert np.sqrt(np.mean((p_learned - p_direct) ** 2)) < 1e-7
    assert it_learned < it_direct


@pytest.mark.parametrize("rows", [1, 127, 130, 1000])
def test_tensor_paths_agree(rows):
    # tcgen05 128-row tiles (the default) and the warp-level mma.sync tiles,
    # on ragged row counts: the same BF16 operands, FP32 sums in another
    # order, so the two agree far inside the BF16 checker's bound
    ens = engine.GpuEnsemble(_pw())
    ens.mlp_init(capacity_frames=4, seed=11)
    ens.compute_forces(L.TERM_IND_SHORT)
    feats = ens.mlp_features()
    params = ens.mlp_params()
    params[M.NPARAM:M.NPARAM + M.F] = feats.mean(0)
    params[M.NPARAM + M.F:] = 1.0 / (feats.std(0) + 1e-3)
    ens.mlp_params(set_to=params)
    x = np.ascontiguousarray(np.resize(feats, (rows, feats.shape[1])))
    y_tc = ens.mlp_eval(x)
    ens.mlp_set_tensor_path(0)
    y_ws = ens.mlp_eval(x)
    ens.mlp_set_tensor_path(1)
    y_bf, _ = M.forward(params, x, bf16=True)
    scale = 1 + np.abs(y_bf).max()
    print("tcgen05 vs mma.sync", np.max(np.abs(y_tc - y_ws)) / scale, "vs bf16 checker",
          np.max(np.abs(y_tc - y_bf)) / scale)
    assert np.max(np.abs(y_tc - y_ws)) < 2e-3 * scale
    assert np.max(np.abs(y_tc - y_bf)) < 2e-3 * scale
    with pytest.raises(L.SmdError):
        ens.mlp_set_tensor_path(2)
    ens.close()


def test_learned_guess_same_on_both_tensor_paths():
    s = _pw(seed=9)
    ens = engine.GpuEnsemble(s)
    ens.set_solver(tol=2.0819e-8, max_iter=500, guess=L.GUESS_DIRECT)
    lf = engine.LFIntegrator(ens)
    lf.start()
    lf.run(2)
    ens.mlp_init(capacity_frames=20, seed=5)
    for _ in range(20):
        lf.run(2)
        ens.compute_forces(L.TERM_IND_SHORT)
        ens.mlp_collect()
    ens.mlp_train(epochs=10, batch=2048, lr=2e-3)
    lf.run(3)
    ens.set_solver(tol=2.0819e-8, max_iter=500, guess=L.GUESS_LEARNED)
    out = {}
    for path in (1, 0):
        ens.mlp_set_tensor_path(path)
        ens.compute_forces(L.TERM_IND_SHORT)
        out[path] = (ens.solver_trace()[0], ens.solver_stats()[0], ens.polarization()["p"])
    print("first update", out[1][0], out[0][0], "iterations", out[1][1], out[0][1])
    assert abs(out[1][0] - out[0][0]) <= 1e-2 * out[0][0]
    assert abs(out[1][1] - out[0][1]) <= 1
    assert np.sqrt(np.mean((out[1][2] - out[0][2]) ** 2)) < 1e-7
    ens.close()

"""Batched replicas: one CUDA graph per step advancing replicas of uneven
size, seed and strain rate must give each replica exactly the trajectory it
has when run on its own, and the autotuner must pick a valid shape."""
import numpy as np
import pytest

from swinmd_b200 import engine, systems

pytestmark = pytest.mark.gpu


def _replicas():
    reps = systems.replica_set(count=5, n_min=500, n_max=2000, rate_max_star=1.0, seed=7, n_steps=50)
    out = []
    for s in reps:
        e = engine.GpuEnsemble(s, precision="mixed")
        nh = engine.NHIntegrator(e)
        nh.start()
        out.append((s, e, nh))
    return out


def test_batch_matches_single_runs():
    alone = _replicas()
    for _, e, nh in alone:
        nh.run(30)
    together = _replicas()
    batch = engine.ReplicaBatch([e for _, e, _ in together])
    ms = batch.run(30)
    assert ms > 0
    for (s, ea, na), (_, eb, nb) in zip(alone, together):
        a, b = ea.state(), eb.state()
        assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["vel"], b["vel"])
        oa, ob = na.observables(), nb.observables()
        assert oa.step == ob.step == 30
        assert oa.e_potential == ob.e_potential
    batch.close()


def test_autotune_and_run():
    reps = _replicas()
    batch = engine.ReplicaBatch([e for _, e, _ in reps])
    tpp = batch.autotune(reps=5)
    assert all(t in (1, 2, 4, 8, 16, 32) for t in tpp)
    batch.run(20)
    for s, e, nh in reps:
        o = nh.observables()
        assert o.step == 20 and np.isfinite(o.e_potential)
        # mixed-precision forces of each replica against FP64
        f32, _, _ = e.compute_forces()
        e.set_precision("fp64")
        f64, _, _ = e.compute_forces()
        e.set_precision("mixed")
        assert np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum()) < 1e-6
    batch.close()


def test_water_batch_matches_single_runs():
    # LJ + Ewald water replicas (SHAKE, leap-frog Nose-Hoover) in one graph
    # give each replica its own trajectory
    reps = systems.water_replica_set(count=3, n_min=300, n_max=900, seed=4, n_steps=20)

    def build():
        out = []
        for s in reps:
            e = engine.GpuEnsemble(s, precision="mixed")
            lf = engine.LFIntegrator(e)
            lf.start()
            out.append((e, lf))
        return out

    alone = build()
    for _, lf in alone:
        lf.run(10)
    together = build()
    batch = engine.ReplicaBatch([e for e, _ in together])
    batch.run(10)
    for (ea, la), (eb, lb) in zip(alone, together):
        a, b = ea.state(), eb.state()
        assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["vel"], b["vel"])
        assert la.observables().e_potential == lb.observables().e_potential
    batch.close()
    for e, _ in alone + together:
        e.close()


def test_sheared_water_batch_matches_single_runs():
    # flexible LJ + Ewald water replicas with their own strain rates (SLLOD,
    # the sheared cell's k list) and Nose-Hoover chains in one graph
    reps = systems.water_replica_set(count=3, n_min=300, n_max=900, seed=6, n_steps=20, flexible=True,
                                     rate_max_star=4.0)
    assert len({s.config.rate for s in reps}) == 3 and min(s.config.rate for s in reps) > 0

    def build():
        out = []
        for s in reps:
            e = engine.GpuEnsemble(s, precision="mixed")
            nh = engine.NHIntegrator(e)
            nh.start()
            out.append((e, nh))
        return out

    alone = build()
    for _, nh in alone:
        nh.run(20)
    together = build()
    batch = engine.ReplicaBatch([e for e, _ in together])
    batch.run(20)
    for (ea, la), (eb, lb) in zip(alone, together):
        a, b = ea.state(), eb.state()
        assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["vel"], b["vel"])
        oa, ob = la.observables(), lb.observables()
        assert oa.e_potential == ob.e_potential
        assert oa.shear_offset == ob.shear_offset and oa.shear_offset > 0
    batch.close()
    for e, _ in alone + together:
        e.close()

"""Observables on the device: the RDF histogram against the reference's own
RDF::sampling of the same configuration (bit-exact counts), its
normalisation as RDF::write_result, and the running averages of the step
observables against the per-step values."""
import numpy as np
import pytest

from conftest import golden
from swinmd_b200 import engine, systems

pytestmark = pytest.mark.gpu


def _lj():
    s = systems.lj_fluid(ncell=5, jitter_star=0.05, seed=3, n_steps=20)
    s.config.long_correct = True
    return s


def _spce():
    return systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=20)


@pytest.mark.parametrize("make,name", [(_lj, "lj500"), (_spce, "spce512")])
def test_rdf_counts_match_reference(make, name):
    g = golden(name)
    s = make()
    ens = engine.GpuEnsemble(s)
    nb = int(g["rdf_nbins"][0])
    ens.rdf_setup(nb)
    ens.rdf_sample()
    r, rdf, hist, cnt = ens.rdf()
    assert cnt == 1
    ref = g["rdf_hist"].reshape(hist.shape)
    assert np.array_equal(hist.astype(np.float64), ref)
    # RDF::write_result's normalisation of the same counts
    maxr = float(g["rdf_maxr"][0])
    dr = maxr / nb
    vol = ens.box ** 3
    npt = g["rdf_numpertype"]
    rr = np.arange(nb) * dr + 0.5 * dr
    assert np.allclose(r, rr, rtol=0, atol=1e-15)
    col = 0
    for t1 in range(len(npt)):
        for t2 in range(t1, len(npt)):
            expect = 0.5 * (ref[t1, t2] + ref[t2, t1]) / (4 * np.pi * dr / vol) / (rr ** 2 * npt[t1] * npt[t2])
            assert np.allclose(rdf[col], expect, rtol=1e-13, atol=0)
            col += 1
    ens.close()


def test_rdf_accumulates_samples():
    s = _lj()
    ens = engine.GpuEnsemble(s)
    lf = engine.LFIntegrator(ens)
    lf.start()
    ens.rdf_setup(100)
    total = np.zeros((1, 1, 100))
    for _ in range(3):
        lf.run(5)
        ens.rdf_sample()
    r, rdf, hist, cnt = ens.rdf()
    assert cnt == 3
    # every sample counts every pair below the cutoff once in each order
    n = s.n_atoms
    assert 0 < hist.sum() <= 3 * n * (n - 1)
    ens.close()


def test_running_averages():
    s = _spce()
    ens = engine.GpuEnsemble(s)
    lf = engine.LFIntegrator(ens, series_capacity=64)
    lf.start()
    lf.run(20)
    a = ens.averages()
    ser = lf.series()
    assert a.samples == 20
    assert np.isclose(a.e_potential, ser[:, 0].mean(), rtol=1e-12)
    assert np.isclose(a.ke_atom, ser[:, 1].mean(), rtol=1e-12)
    assert np.isclose(a.atom_stress[0], ser[:, 4].mean(), rtol=1e-10)
    assert np.isclose(a.e_total, (ser[:, 0] + ser[:, 1]).mean(), rtol=1e-12)
    # the last step's tensors enter the means like every other step
    o = lf.observables()
    ens.reset_averages()
    lf.run(1)
    a1 = ens.averages()
    o1 = lf.observables()
    assert a1.samples == 1
    assert np.allclose(np.array(a1.atom_pressure), np.array(o1.atom_pressure), rtol=1e-14)
    assert np.isclose(a1.mol_stress[1], 0.5 * (o1.mol_pressure[1] + o1.mol_pressure[3]), rtol=1e-12)
    ens.close()


def test_checkpoint_restart_continues_the_run(tmp_path):
    # 10 steps, checkpoint, a new context restarted from the files, 10 more
    # steps: the trajectory of 20 uninterrupted steps (the restart rebuilds
    # the pair list, so only the order of the per-thread sums differs)
    s = _spce()
    ref = engine.GpuEnsemble(s)
    lf = engine.LFIntegrator(ref)
    lf.start()
    lf.run(10)
    lf.write_state(str(tmp_path / "state.out"), str(tmp_path / "vtMinus.out"))
    real10 = ref.real_positions()
    lf.run(10)
    st_ref = ref.state()
    e2 = engine.GpuEnsemble(s)
    lf2 = engine.LFIntegrator(e2)
    lf2.restart(str(tmp_path / "state.out"), str(tmp_path / "vtMinus.out"))
    lf2.run(10)
    st = e2.state()
    assert np.allclose(st["pos"], st_ref["pos"], rtol=0, atol=1e-10)
    assert np.allclose(st["vel"], st_ref["vel"], rtol=0, atol=1e-8)
    # real positions continue from the checkpoint's (unwrapped: no jumps of a box)
    real = e2.real_positions()
    assert np.max(np.abs(real - real10)) < 0.5 * e2.box
    # the restarted real positions equal the uninterrupted run's
    assert np.allclose(real, ref.real_positions(), rtol=0, atol=1e-10)
    ref.close()
    e2.close()

"""LJ fluid on the GPU against the reference's own results (golden fixture
made by running SwinMD's LJForce / LFIntegrator, tests/golden/make_golden.py)."""
import numpy as np
import pytest

from conftest import golden
from swinmd_b200 import engine, systems

pytestmark = pytest.mark.gpu


def _sys():
    s = systems.lj_fluid(ncell=5, jitter_star=0.05, seed=3, n_steps=20)
    s.config.long_correct = True
    return s


def rms_rel(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


@pytest.mark.parametrize("tpp", [1, 4, 8, 32])
def test_pair_set_matches_reference(tpp):
    g = golden("lj500")
    ens = engine.GpuEnsemble(_sys(), threads_per_site=tpp)
    pairs = ens.pairs()
    pairs = pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]
    assert pairs.shape == g["pairs"].shape
    assert np.array_equal(pairs, g["pairs"])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_lj_forces_energy_virial(precision, tol):
    g = golden("lj500")
    ens = engine.GpuEnsemble(_sys(), precision=precision)
    lj = engine.LJForce(ens)
    lj.compute()
    ref_f = g["f_lj_force"].reshape(-1, 3)
    err = rms_rel(lj.force, ref_f)
    print(precision, "rms rel force err", err)
    assert err < tol
    e_ref = g["f_lj_energy"][0]
    assert abs(lj.energy - e_ref) / abs(e_ref) < max(tol, 1e-12)
    vir = lj.get_virial()
    ref_w = g["f_lj_virial"]
    assert np.max(np.abs(vir - ref_w)) < max(tol, 1e-11) * np.linalg.norm(ref_w)


def test_lj_deterministic():
    ens = engine.GpuEnsemble(_sys(), precision="mixed")
    a = ens.compute_forces()
    b = ens.compute_forces()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


def test_leapfrog_nose_hoover_trajectory():
    g = golden("lj500")
    ens = engine.GpuEnsemble(_sys())
    lf = engine.LFIntegrator(ens, series_capacity=64)
    lf.start()
    st = ens.state()
    assert np.allclose(st["vtminus"].reshape(-1), g["r_start_vtminus"], rtol=0, atol=1e-12)
    lf.run(20)
    ser = lf.series()
    # potential energy, temperature and zeta of every step
    assert np.allclose(ser[:, 0], g["r_step_epot"], rtol=1e-10)
    assert np.allclose(ser[:, 2], g["r_step_atomtemp"], rtol=1e-10)
    assert np.allclose(ser[:, 3], g["r_step_zeta"], rtol=1e-8, atol=1e-14)
    st = ens.state()
    assert np.allclose(st["pos"].reshape(-1), g["r_final_pos"], rtol=0, atol=1e-10)
    assert np.allclose(st["vel"].reshape(-1), g["r_final_vel"], rtol=0, atol=1e-9)
    o = lf.observables()
    assert o.step == 20
    assert o.list_updates == int(g["r_step_nupdates"][-1])   # numUpdates: rebuilds of the run
    p_ref = g["r_step_atompressure"].reshape(-1, 9)[-1]
    assert np.allclose(np.array(o.atom_pressure), p_ref, rtol=1e-8, atol=1e-6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_upload_within_skin_keeps_the_list(precision):
    """Uploading positions that moved less than half the skin since the last
    rebuild keeps the pair list (the displacement test decides, as in a step):
    a run interrupted by a download and upload of the same positions matches
    an uninterrupted one bit for bit, with no extra rebuild."""
    runs = []
    for upload in (False, True):
        ens = engine.GpuEnsemble(_sys(), precision=precision)
        lf = engine.LFIntegrator(ens)
        lf.start()
        lf.run(10)
        if upload:
            ens.upload_positions(ens.state()["pos"])
        lf.run(10)
        runs.append((ens.state()["pos"].copy(), lf.observables().list_updates))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]

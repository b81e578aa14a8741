"""Rigid SPC/E water (LJ on O + Ewald + SHAKE) on the GPU against the
reference's own LJForce / EwaldForce / LFIntegrator::shake results."""
import numpy as np
import pytest

from conftest import golden
from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def _spce():
    return systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=20)


def test_water_pair_set_excludes_intramolecular():
    g = golden("spce512")
    ens = engine.GpuEnsemble(_spce())
    p = ens.pairs()
    p = p[np.lexsort((p[:, 1], p[:, 0]))]
    assert np.array_equal(p, g["pairs"])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 2e-6)])
def test_water_forces(precision, tol):
    g = golden("spce512")
    ens = engine.GpuEnsemble(_spce(), precision=precision)
    f, e, w = ens.compute_forces(L.TERM_VDW)
    assert rms_rel(f, g["f_lj_force"].reshape(-1, 3)) < tol
    assert abs(e[L.E_VDW] - g["f_lj_energy"][0]) < tol * abs(g["f_lj_energy"][0])
    f, e, w = ens.compute_forces(L.TERM_EWALD_REAL)
    err = rms_rel(f, g["f_ewald_short_force"].reshape(-1, 3))
    print(precision, "ewald real", err)
    assert err < 5 * tol
    ref_e = g["f_ewald_short_energy"]
    assert abs(e[L.E_REAL] - ref_e[1]) < tol * abs(ref_e[1])
    assert abs(e[L.E_CORRECT] - ref_e[3]) < 1e-10 * abs(ref_e[3])
    assert abs(e[L.E_MOLCORRECT] - ref_e[4]) < 1e-9 * abs(ref_e[4])
    f, e, w = ens.compute_forces(L.TERM_EWALD_LONG)
    err = rms_rel(f, g["f_ewald_long_force"].reshape(-1, 3))
    print(precision, "ewald long", err)
    assert err < 5 * tol
    assert abs(e[L.E_LONG] - g["f_ewald_long_energy"][2]) < tol * abs(g["f_ewald_long_energy"][2])


def test_water_shake_trajectory():
    g = golden("spce512")
    s = _spce()
    ens = engine.GpuEnsemble(s)
    lf = engine.LFIntegrator(ens, series_capacity=32)
    lf.start()
    lf.run(19)
    # the reciprocal virial's ZZ component at the configuration whose forces
    # the 20th step uses: the reference leaves it out of its pressures
    # (EwaldForce::compute_long copies longVirial components 0..7 only,
    # src/forces/EwaldForce.cpp:194-195); the GPU step includes it
    _, _, w_long = ens.compute_forces(L.TERM_EWALD_LONG)
    lf.run(1)
    ser = lf.series()
    print(np.max(np.abs(ser[:, 0] / g["r_step_epot"] - 1)))
    assert np.allclose(ser[:, 0], g["r_step_epot"], rtol=1e-7)
    assert np.allclose(ser[:, 2], g["r_step_atomtemp"], rtol=1e-7)
    st = ens.state()
    assert np.allclose(st["pos"].reshape(-1), g["r_final_pos"], rtol=0, atol=1e-8)
    # constraint lengths hold to the SHAKE tolerance
    p = st["pos"].reshape(-1, 3, 3)
    d01 = np.linalg.norm(p[:, 0] - p[:, 1], axis=1)
    d12 = np.linalg.norm(p[:, 1] - p[:, 2], axis=1)
    assert np.max(np.abs(d01 ** 2 / 0.01 - 1)) < 3e-8
    assert np.max(np.abs(d12 ** 2 / 0.01 - 1)) < 3e-8
    o = lf.observables()
    assert o.list_updates == int(g["r_step_nupdates"][-1])
    vol = s.box[0] ** 3
    for ours, key in ((o.atom_pressure, "r_step_atompressure"), (o.mol_pressure, "r_step_molpressure")):
        p = np.array(ours)
        p_ref = g[key].reshape(-1, 9)[-1].copy()
        print(key, p - p_ref)
        assert np.allclose(p[:8], p_ref[:8], rtol=1e-8, atol=1e-6)
        assert abs(p[8] - w_long[8] / vol - p_ref[8]) < 1e-6 * abs(p_ref[8])

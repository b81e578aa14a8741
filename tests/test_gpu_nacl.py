"""NaCl melt on the GPU: Mie 14-7 + Ewald against the reference's own
MieForce / EwaldForce results, Born-Mayer-Huggins against the oracle."""
import numpy as np
import pytest

import oracle
from conftest import golden
from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def _mie():
    return systems.nacl_melt(ncell=10, potential="mie", kmax=6, seed=5)


def test_nacl_pair_set():
    g = golden("nacl1000_mie")
    ens = engine.GpuEnsemble(_mie())
    p = ens.pairs()
    p = p[np.lexsort((p[:, 1], p[:, 0]))]
    assert np.array_equal(p, g["pairs"])
    assert ens.ewald_nk() == int(g["f_ewald_nk"][0])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_nacl_mie_ewald_forces(precision, tol):
    g = golden("nacl1000_mie")
    ens = engine.GpuEnsemble(_mie(), precision=precision)
    f_vdw, e_vdw, w_vdw = ens.compute_forces(L.TERM_VDW)
    err = rms_rel(f_vdw, g["m_mie_force"].reshape(-1, 3))
    print(precision, "mie", err)
    assert err < tol
    assert abs(e_vdw[L.E_VDW] - g["m_mie_energy"][0]) < tol * abs(g["m_mie_energy"][0])
    f_re, e_re, _ = ens.compute_forces(L.TERM_EWALD_REAL)
    err = rms_rel(f_re, g["f_ewald_short_force"].reshape(-1, 3))
    print(precision, "ewald real", err)
    assert err < tol * 5
    assert abs(e_re[L.E_REAL] - g["f_ewald_short_energy"][1]) < tol * abs(g["f_ewald_short_energy"][1])
    assert abs(e_re[L.E_CORRECT] - g["f_ewald_short_energy"][3]) < 1e-9 * abs(g["f_ewald_short_energy"][3])
    f_lo, e_lo, w_lo = ens.compute_forces(L.TERM_EWALD_LONG)
    err = rms_rel(f_lo, g["f_ewald_long_force"].reshape(-1, 3))
    print(precision, "ewald long", err)
    assert err < tol * 5
    assert abs(e_lo[L.E_LONG] - g["f_ewald_long_energy"][2]) < tol * abs(g["f_ewald_long_energy"][2])
    ref_lw = g["f_ewald_long_longvirial"]
    assert np.max(np.abs(w_lo[:8] - ref_lw[:8])) < 1e-6 * np.abs(ref_lw).max() + 1e-6
    # total force of all terms
    f_all, _, _ = ens.compute_forces(L.TERM_ALL)
    ref_all = (g["m_mie_force"] + g["f_ewald_short_force"] + g["f_ewald_long_force"]).reshape(-1, 3)
    err = rms_rel(f_all, ref_all)
    print(precision, "total", err)
    assert err < tol * 5


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 2e-6)])
def test_nacl_bmh_against_oracle(precision, tol):
    s = systems.nacl_melt(ncell=10, potential="bmh", kmax=6, seed=7)
    ens = engine.GpuEnsemble(s, precision=precision)
    box = ens.box
    pairs = oracle.pairlist(s, s.pos, box)
    f_ref, e_ref, w_ref = oracle.vdw(s, s.pos, box, pairs)
    f, e, w = ens.compute_forces(L.TERM_VDW)
    err = rms_rel(f, f_ref)
    print(precision, "bmh", err)
    assert err < tol
    assert abs(e[L.E_VDW] - e_ref) < tol * abs(e_ref)
    assert np.max(np.abs(w - w_ref)) < tol * np.abs(w_ref).max()

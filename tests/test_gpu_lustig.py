"""Lustig's volume derivatives of the LJ energy (Ensemble::myLustig.ljUlus,
ljdUlus, ljd2Ulus) against the reference's LJForce::compute with
computeLustig on: atoms (r_ij . r_ij) and rigid water under constraints
(r_ij . R_ij with the molecules' centres)."""
import numpy as np
import pytest

from conftest import golden
from swinmd_b200 import engine, systems

pytestmark = pytest.mark.gpu


def _lj():
    s = systems.lj_fluid(ncell=5, jitter_star=0.05, seed=3)
    s.config.long_correct = True
    s.config.lustig = True
    return s


def _spce():
    s = systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11)
    s.config.lustig = True
    return s


def test_lustig_lj_atoms():
    g = golden("lj500_lustig")
    ens = engine.GpuEnsemble(_lj())
    out = ens.lustig_lj()
    print(out, g["f_lustig_lj"])
    assert np.allclose(out, g["f_lustig_lj"], rtol=1e-10, atol=0)
    ens.close()


def test_lustig_lj_rigid_water():
    # the reference fills the molecules' centres in during a step: its second
    # step's values belong to the positions its first step left
    g = golden("spce512_lustig")
    ens = engine.GpuEnsemble(_spce())
    ens.upload_positions(g["r_step_after1_pos"].reshape(-1, 3))
    out = ens.lustig_lj()
    ref = g["r_step_lustig"].reshape(-1, 3)[1]
    print(out, ref)
    assert np.allclose(out, ref, rtol=1e-10, atol=0)
    ens.close()


# ---------------------------------------------------------------------------
# every field of Ensemble::myLustig against the reference's second step of a
# two-step run (tests/golden/make_golden.py, cases *_lustig): the GPU
# evaluates the positions the reference's first step left
# ---------------------------------------------------------------------------
def _compare(ens, g, rtol=1e-8, atol_rel=1e-11):
    from swinmd_b200 import _lib as L
    ens.upload_positions(g["r_step_after1_pos"].reshape(-1, 3))
    got = ens.lustig()
    ref = g["r_step_lustig_all"].reshape(-1, len(L.LUSTIG_FIELDS))[1]
    scale = np.abs(ref).max()
    bad = []
    for name, r in zip(L.LUSTIG_FIELDS, ref):
        if name == "virialcorrect":
            # formed by LFIntegrator after the position update (this step's
            # forces against the next positions): not a field of one
            # configuration, and returned as 0
            assert got[name] == 0.0
            continue
        v = got[name]
        ok = abs(v - r) <= rtol * abs(r) + atol_rel * scale
        print(f"{name:20s} {v: .12e} {r: .12e} {'' if ok else 'MISMATCH'}")
        if not ok:
            bad.append(name)
    assert not bad, bad
    # the integrator's Lustig virial from these fields
    mv = engine.lustig_molvirt(got, float(np.prod(g["box"])))
    ref_mv = g["r_step_molvirt"][1]
    print("molVirt", mv, ref_mv)
    assert abs(mv - ref_mv) <= rtol * abs(ref_mv) + 1e-9 * scale


def test_lustig_all_ions():
    # point charges and LJ on ions, surface term (no constraints)
    s = systems.nacl_melt(ncell=10, potential="lj", kmax=6, seed=5, n_steps=2)
    s.config.lustig = True
    s.config.surface_correct = True
    ens = engine.GpuEnsemble(s)
    _compare(ens, golden("nacl1000_lustig"))
    ens.close()


def test_lustig_all_flexible_water():
    # bonds, angles and the intramolecular Ewald correction's forces
    s = systems.spce_flexible(nmol=216, seed=4, n_steps=2)
    s.config.lustig = True
    s.config.surface_correct = True
    s.config.thermostat = "NoseHoover"
    ens = engine.GpuEnsemble(s)
    _compare(ens, golden("spcf216_lustig"))
    ens.close()


def test_lustig_all_rigid_water():
    # constraints: r_ij . R_ij and the reciprocal centre-of-mass sums
    ens = engine.GpuEnsemble(_spce())
    _compare(ens, golden("spce512_lustig"))
    ens.close()


def test_lustig_all_polarisable_water():
    s = systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3, n_steps=2)
    s.config.lustig = True
    s.config.surface_correct = True
    ens = engine.GpuEnsemble(s)
    ens.set_solver(tol=1e-13, max_iter=1000)
    _compare(ens, golden("polwater216_lustig"), rtol=1e-7)
    ens.close()


def test_lustig_all_reference_case(tmp_path):
    # the reference's own flexible polarisable case (bonds, Urey-Bradley,
    # buffered 14-7, multipoles, induction, surface terms)
    g = golden("ref_test_nvt")
    for key, fn in (("case_config", "config.txt"), ("case_sysdata", "sysData.in"), ("case_coords", "coordinate.in")):
        (tmp_path / fn).write_text(str(g[key]))
    s = systems.read_reference_case(str(tmp_path))
    ens = engine.GpuEnsemble(s)
    ens.set_solver(tol=1e-13, max_iter=1000)
    _compare(ens, golden("ref_test_lustig"), rtol=1e-7)
    ens.close()


def test_lustig_all_wolf():
    # the Wolf sum with the O charges on WolfForce's displaced sites
    s = systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=2)
    s.config.compute_ewald, s.config.compute_wolf, s.config.alpha = False, True, 2.0
    s.config.lustig = True
    ens = engine.GpuEnsemble(s)
    _compare(ens, golden("spce512_wolf_lustig"))
    ens.close()

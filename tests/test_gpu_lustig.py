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

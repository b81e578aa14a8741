"""SAAP pair potential (SAAPForce) against the reference's own evaluation
with its built-in three-type table, in FP64 and in the mixed path."""
import numpy as np
import pytest

from conftest import golden, rms_rel
from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 2e-5)])
def test_saap_matches_reference(precision, tol):
    g = golden("saap500")
    s = systems.three_type_fluid(ncell=5, seed=3)
    ens = engine.GpuEnsemble(s, precision=precision)
    ens.set_saap(g["s_saap_params"].reshape(-1, 6))
    f, e, w = ens.compute_forces(L.TERM_VDW)
    err = rms_rel(f, g["s_saap_force"].reshape(-1, 3))
    e_ref = g["s_saap_energy"][L.E_VDW]
    print(precision, "force", err, "energy", e[L.E_VDW], e_ref)
    assert err < tol
    assert abs(e[L.E_VDW] - e_ref) < tol * abs(e_ref)
    assert np.allclose(w, g["s_saap_virial"], rtol=0, atol=tol * np.abs(g["s_saap_virial"]).max())
    ens.close()

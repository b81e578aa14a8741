"""The AMOEBA damping branch of the induced real space (dampAMOEBA,
Induction.cpp:1051-1079) on the GPU against the reference's own run of
polwater216 with the flag on (fixture polwater216_amoeba): energy and forces
(with the torques carried onto the sites) of the induced short-range term, in FP64 and in the mixed path."""
import numpy as np
import pytest

from conftest import golden
from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _sys():
    s = systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3, n_steps=10)
    s.config.damp_amoeba = True
    return s


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("mixed", 2e-6)])
def test_amoeba_induced_real_space_matches_reference(precision, tol):
    g = golden("polwater216_amoeba")
    s = _sys()
    s.pos = g["pos"].copy()
    ens = engine.GpuEnsemble(s, precision=precision)
    ens.set_solver(tol=1e-13, max_iter=3000, guess=L.GUESS_DIRECT)
    f, e, w = ens.compute_forces(L.TERM_IND_SHORT)
    p = ens.polarization()["p"]
    ref_p = g["f_ind_P"].reshape(-1, 3)
    print("dipoles", np.abs(p - ref_p).max() / np.abs(ref_p).max())
    e_ref = g["f_ind_short_energy"]
    f_ref = g["f_ind_short_force"].reshape(-1, 3)
    ferr = np.sqrt(np.sum((f - f_ref) ** 2) / np.sum(f_ref ** 2))
    print(precision, "energy", e[L.E_POL_REAL], e_ref[6], "force rms rel", ferr)
    assert abs(e[L.E_POL_REAL] - e_ref[6]) < tol * abs(e_ref[6])
    assert ferr < 10 * tol
    # Thole damping differs: the flag reaches the kernels
    ens.lib.smd_set_induction_damping(ens.ctx, 0)
    _, e0, _ = ens.compute_forces(L.TERM_IND_SHORT)
    assert abs(e0[L.E_POL_REAL] - golden("polwater216")["f_ind_short_energy"][6]) < 1e3 * tol * abs(e_ref[6])
    ens.close()

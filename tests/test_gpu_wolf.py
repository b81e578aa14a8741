"""Wolf summation of the charges (WolfForce) against the reference's own
evaluation: water whose O charges sit on the displaced site (a second pass
of the charge term) and an ionic melt (the charge term fused into the pair
pass), in FP64 and in the mixed path."""
import numpy as np
import pytest

from conftest import golden, rms_rel
from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _spce():
    s = systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11)
    s.config.compute_ewald, s.config.compute_wolf, s.config.alpha = False, True, 2.0
    return s


def _nacl():
    s = systems.nacl_melt(ncell=10, potential="mie", kmax=6, seed=5)
    s.config.compute_ewald, s.config.compute_wolf, s.config.alpha = False, True, 2.5
    return s


@pytest.mark.parametrize("make,name", [(_spce, "spce512_wolf"), (_nacl, "nacl1000_wolf")])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 2e-6)])
def test_wolf_matches_reference(make, name, precision, tol):
    g = golden(name)
    ens = engine.GpuEnsemble(make(), precision=precision)
    f, e, w = ens.compute_forces(L.TERM_WOLF)
    ref_f = g["f_wolf_force"].reshape(-1, 3)
    err = rms_rel(f, ref_f)
    e_ref = g["f_wolf_energy"][L.E_REAL]
    print(name, precision, "force", err, "energy", e[L.E_REAL], e_ref)
    assert err < tol
    assert abs(e[L.E_REAL] - e_ref) < max(tol, 1e-12) * abs(e_ref)
    # the reference's virial of the term (Ensemble::virial -= sum f r)
    # (off-diagonal entries cancel: the bound is relative to the tensor's size)
    assert np.allclose(w, g["f_wolf_virial"], rtol=0, atol=max(tol, 1e-10) * np.abs(g["f_wolf_virial"]).max())
    ens.close()


def test_wolf_runs_in_the_step():
    # the step graph carries the Wolf term: a short run conserves nothing in
    # particular, but it must run and match a run built the same way
    runs = []
    for _ in range(2):
        ens = engine.GpuEnsemble(_spce())
        lf = engine.LFIntegrator(ens)
        lf.start()
        lf.run(5)
        runs.append(ens.state()["pos"])
        ens.close()
    assert np.array_equal(runs[0], runs[1])

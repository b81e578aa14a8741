"""The Force-plugin entry point used the way the reference's integrator calls
its force objects: one call per term on the same positions
(LFIntegrator::run, src/integrators/LFIntegrator.cpp:387-458).  The dipoles
are solved once per configuration (Induction::compute_long uses what
Induction::compute solved), and the pair list is kept while every site
stays within half the skin of its last build."""
import numpy as np
import pytest

from conftest import rms_rel
from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _pw():
    return systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3,
                                     n_steps=10)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dipoles_solved_once_per_configuration(precision):
    # from the previous dipoles a second solve would start converged and end
    # after one or two iterations with slightly different dipoles: the
    # long-range call must reuse the short-range call's solve instead
    ens = engine.GpuEnsemble(_pw(), precision=precision)
    ens.set_solver(tol=2.0819e-8, max_iter=500, guess=L.GUESS_PREVIOUS)
    ens.compute_forces(L.TERM_IND_SHORT)
    it1 = ens.solver_stats()
    p1 = ens.polarization()["p"]
    assert it1[0] > 3
    ens.compute_forces(L.TERM_IND_LONG)
    assert ens.solver_stats() == it1
    assert np.array_equal(ens.polarization()["p"], p1)
    # a new configuration is solved again (from the previous dipoles)
    s = ens.system
    ens.upload_positions(s.pos + 1e-4)
    ens.compute_forces(L.TERM_IND_LONG)
    it2 = ens.solver_stats()
    assert it2 != it1
    assert not np.array_equal(ens.polarization()["p"], p1)
    ens.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_terms_one_by_one_equal_one_call(precision):
    # the reference's call sequence (each term on its own, the solve shared)
    # gives the forces of one full evaluation
    ens = engine.GpuEnsemble(_pw(), precision=precision)
    ens.set_solver(tol=1e-12, max_iter=1000)
    f_all, e_all, w_all = ens.compute_forces()
    ens.upload_positions(ens.system.pos)   # a new configuration version, same positions
    f_sum = np.zeros_like(f_all)
    for term in (L.TERM_VDW, L.TERM_MP_SHORT, L.TERM_MP_LONG, L.TERM_IND_SHORT, L.TERM_IND_LONG):
        f, _, _ = ens.compute_forces(term)
        f_sum += f
    err = rms_rel(f_sum, f_all)
    print(precision, err)
    # (a full evaluation forms both reciprocal terms in one combined pass)
    assert err < (1e-10 if precision == "fp64" else 3e-7)
    ens.close()


def test_kept_list_gives_the_rebuilt_list_forces():
    # positions moved by less than half the skin keep the list; the forces
    # equal those of a fresh context whose list is built at these positions
    s = systems.lj_fluid(ncell=5, jitter_star=0.05, seed=3)
    ens = engine.GpuEnsemble(s)
    ens.compute_forces()
    rng = np.random.default_rng(0)
    moved = s.pos + rng.uniform(-0.01, 0.01, s.pos.shape) * s.config.cut_buffer
    ens.upload_positions(moved)
    f_kept, e_kept, _ = ens.compute_forces()
    fresh = engine.GpuEnsemble(s.replace(pos=moved))
    f_new, e_new, _ = fresh.compute_forces()
    assert rms_rel(f_kept, f_new) < 1e-13
    assert abs(e_kept[L.E_VDW] - e_new[L.E_VDW]) < 1e-12 * abs(e_new[L.E_VDW])
    # the pair set of the current positions is still available
    a = ens.pairs()
    b = fresh.pairs()
    a = a[np.lexsort((a[:, 1], a[:, 0]))]
    b = b[np.lexsort((b[:, 1], b[:, 0]))]
    assert np.array_equal(a, b)
    ens.close()
    fresh.close()


def test_force_call_between_steps_leaves_the_run_unchanged():
    # smd_compute_forces between smd_run calls (a sampling point) changes
    # nothing of the trajectory or of the next steps' observables
    def run(probe):
        s = systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=20)
        e = engine.GpuEnsemble(s)
        lf = engine.LFIntegrator(e, series_capacity=16)
        lf.start()
        lf.run(5)
        if probe:
            e.compute_forces(L.TERM_EWALD_LONG)
            e.compute_forces()
        lf.run(5)
        out = (lf.series().copy(), e.state()["pos"].copy(), np.array(lf.observables().atom_pressure))
        e.close()
        return out
    a, b = run(False), run(True)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2], b[2])

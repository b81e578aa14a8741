"""Polarisable multipole water (buffered 14-7 + permanent multipoles +
Thole induction, rigid H O H) on the GPU against the reference's own
BuffvdWForce / Multipole / Induction / LFIntegrator results."""
import numpy as np
import pytest

from conftest import golden
from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def _pw():
    return systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3,
                                     n_steps=10)


@pytest.fixture(scope="module")
def ens():
    e = engine.GpuEnsemble(_pw())
    e.set_solver(tol=1e-13, max_iter=1000)
    return e


def test_frames_and_pairs(ens):
    g = golden("polwater216")
    ens.compute_forces(L.TERM_MP_SHORT)
    pol = ens.polarization()
    assert np.allclose(pol["mu"].reshape(-1), g["f_mp_dip"], rtol=0, atol=1e-14)
    assert np.allclose(pol["quad"].reshape(-1), g["f_mp_quad"], rtol=0, atol=1e-14)
    p = ens.pairs()
    p = p[np.lexsort((p[:, 1], p[:, 0]))]
    assert np.array_equal(p, g["pairs"])


def test_buffered_14_7(ens):
    g = golden("polwater216")
    f, e, w = ens.compute_forces(L.TERM_VDW)
    err = rms_rel(f, g["f_buff_force"].reshape(-1, 3))
    print("buff", err, e[L.E_VDW], g["f_buff_energy"][0])
    assert err < 1e-10
    assert abs(e[L.E_VDW] - g["f_buff_energy"][0]) < 1e-9 * abs(g["f_buff_energy"][0])


def test_multipole_short_and_long(ens):
    g = golden("polwater216")
    f, e, w = ens.compute_forces(L.TERM_MP_SHORT)
    ref = g["f_mp_short_energy"]
    print("mp energies", e[:6], ref[:6])
    err = rms_rel(f, g["f_mp_short_force"].reshape(-1, 3))
    print("mp short force", err)
    assert abs(e[L.E_REAL] - ref[1]) < 1e-9 * abs(ref[1])
    assert abs(e[L.E_CORRECT] - ref[3]) < 1e-9 * abs(ref[3])
    assert abs(e[L.E_MOLCORRECT] - ref[4]) < 1e-9 * abs(ref[4])
    assert err < 1e-9
    f, e, w = ens.compute_forces(L.TERM_MP_LONG)
    err = rms_rel(f, g["f_mp_long_force"].reshape(-1, 3))
    print("mp long force", err, e[L.E_LONG], g["f_mp_long_energy"][2])
    assert abs(e[L.E_LONG] - g["f_mp_long_energy"][2]) < 1e-9 * abs(g["f_mp_long_energy"][2])
    assert err < 1e-9


def test_induction(ens):
    g = golden("polwater216")
    f, e, w = ens.compute_forces(L.TERM_IND_SHORT)
    pol = ens.polarization()
    it, rms = ens.solver_stats()
    e0_err = rms_rel(pol["e0"].reshape(-1), g["f_ind_E0"])
    p_err = rms_rel(pol["p"].reshape(-1), g["f_ind_P"])
    print("E0", e0_err, "P", p_err, "iters", it, rms)
    assert e0_err < 1e-12
    assert p_err < 1e-9
    ref = g["f_ind_short_energy"]
    print("ind energies", e[6:10], ref[6:11])
    err = rms_rel(f, g["f_ind_short_force"].reshape(-1, 3))
    print("ind short force", err)
    assert abs(e[L.E_POL_REAL] - ref[6]) < 1e-8 * abs(ref[6])
    assert abs(e[L.E_POL_SELF] - ref[8]) < 1e-8 * abs(ref[8])
    assert abs(e[L.E_POL_INTRA] - ref[9]) < 1e-8 * abs(ref[9])
    assert err < 1e-8
    f, e, w = ens.compute_forces(L.TERM_IND_LONG)
    err = rms_rel(f, g["f_ind_long_force"].reshape(-1, 3))
    print("ind long force", err, e[L.E_POL_LONG], g["f_ind_long_energy"][7])
    assert abs(e[L.E_POL_LONG] - g["f_ind_long_energy"][7]) < 1e-8 * abs(g["f_ind_long_energy"][7])
    assert err < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_preconditioners(precision):
    # the diagonal and the molecule-block preconditioner converge to the same
    # dipoles (the reference's, in FP64); the blocks take fewer iterations at
    # both the tight and the working tolerance
    g = golden("polwater216")
    its = {}
    for pc in (L.PRECOND_SITE, L.PRECOND_MOLECULE):
        e = engine.GpuEnsemble(_pw(), precision=precision)
        for tol in (1e-13, 2.0819e-8):
            e.set_solver(tol=tol, max_iter=1000, precond=pc)
            e.compute_forces(L.TERM_IND_SHORT)
            its[pc, tol] = e.solver_stats()[0]
            if tol == 1e-13:
                p = e.polarization()["p"].reshape(-1)
                err = rms_rel(p, g["f_ind_P"])
                print(precision, pc, "p err", err)
                assert err < (1e-9 if precision == "fp64" else 1e-6)
        e.close()
    print(its)
    for tol in (1e-13, 2.0819e-8):
        assert its[L.PRECOND_MOLECULE, tol] < its[L.PRECOND_SITE, tol]


@pytest.mark.parametrize("term,fkey,ekey,eidx", [
    (L.TERM_VDW, "f_buff_force", "f_buff_energy", (L.E_VDW, 0)),
    (L.TERM_MP_SHORT, "f_mp_short_force", "f_mp_short_energy", (L.E_REAL, 1)),
    (L.TERM_MP_LONG, "f_mp_long_force", "f_mp_long_energy", (L.E_LONG, 2)),
    (L.TERM_IND_SHORT, "f_ind_short_force", "f_ind_short_energy", (L.E_POL_REAL, 6)),
    (L.TERM_IND_LONG, "f_ind_long_force", "f_ind_long_energy", (L.E_POL_LONG, 7)),
])
def test_mixed_terms_against_reference(term, fkey, ekey, eidx):
    # the mixed path (FP32 pair and multipole algebra on exact-fraction
    # displacements, FP32 reciprocal phases, FP32 dipole solve rows) against
    # the reference's FP64 results: RMS relative force error below 1e-6
    g = golden("polwater216")
    e = engine.GpuEnsemble(_pw(), precision="mixed")
    e.set_solver(tol=1e-13, max_iter=1000)
    f, en, _ = e.compute_forces(term)
    err = rms_rel(f, g[fkey].reshape(-1, 3))
    ref = g[ekey][eidx[1]]
    print(fkey, err, en[eidx[0]], ref)
    assert err < 1e-6
    assert abs(en[eidx[0]] - ref) < 1e-6 * abs(ref)
    e.close()


def test_mixed_full_evaluation():
    # a full mixed evaluation runs the multipole and the induced real space
    # as one fused pass after the dipole solve: it equals the sum of the
    # single-term evaluations (separate passes) and the reference's total
    g = golden("polwater216")
    e = engine.GpuEnsemble(_pw(), precision="mixed")
    e.set_solver(tol=1e-13, max_iter=1000)
    f_all, en_all, w_all = e.compute_forces()
    f_sum = np.zeros_like(f_all)
    en = {}
    for term in (L.TERM_VDW, L.TERM_MP_SHORT, L.TERM_MP_LONG, L.TERM_IND_SHORT, L.TERM_IND_LONG):
        f, en[term], _ = e.compute_forces(term)
        f_sum += f
    # the fused pass does the same pair arithmetic as the two separate ones
    for slot, term in ((L.E_REAL, L.TERM_MP_SHORT), (L.E_POL_REAL, L.TERM_IND_SHORT)):
        assert abs(en_all[slot] - en[term][slot]) < 1e-10 * abs(en[term][slot])
    # a full evaluation takes the reciprocal terms from one combined pass
    # (six structure factors, one force pass), the single-term calls from
    # separate FP32 passes: the totals agree to FP32 rounding
    print("full vs terms", rms_rel(f_all, f_sum))
    assert rms_rel(f_all, f_sum) < 3e-7
    ref = sum(g[k].reshape(-1, 3) for k in ("f_buff_force", "f_mp_short_force", "f_mp_long_force",
                                            "f_ind_short_force", "f_ind_long_force"))
    err = rms_rel(f_all, ref)
    print("mixed total vs reference", err)
    assert err < 1e-6
    assert abs(en_all[L.E_REAL] - g["f_mp_short_energy"][1]) < 1e-6 * abs(g["f_mp_short_energy"][1])
    assert abs(en_all[L.E_POL_REAL] - g["f_ind_short_energy"][6]) < 1e-6 * abs(g["f_ind_short_energy"][6])
    e.close()


def _mixed_run(steps):
    e = engine.GpuEnsemble(_pw(), precision="mixed")
    e.set_solver(tol=1e-10, max_iter=1000)
    lf = engine.LFIntegrator(e, series_capacity=16)
    lf.start()
    lf.run(steps)
    ser, st = lf.series(), e.state()
    e.close()
    return ser, st


def test_mixed_step():
    # the mixed step (FP64 buffered 14-7, fused real space after the solve,
    # column reciprocal passes): integer atomics make every sum independent
    # of thread order, so two runs are bitwise equal, and the energies follow
    # the reference's trajectory
    g = golden("polwater216")
    ser1, st1 = _mixed_run(10)
    ser2, st2 = _mixed_run(10)
    assert np.array_equal(st1["pos"], st2["pos"])
    assert np.array_equal(st1["vel"], st2["vel"])
    assert np.array_equal(ser1, ser2)
    print(ser1[:, 0], g["r_step_epot"])
    assert np.allclose(ser1[:, 0], g["r_step_epot"], rtol=2e-6)
    assert np.allclose(ser1[:, 2], g["r_step_atomtemp"], rtol=2e-6)


def test_polar_trajectory():
    g = golden("polwater216")
    e = engine.GpuEnsemble(_pw())
    e.set_solver(tol=1e-13, max_iter=1000)
    lf = engine.LFIntegrator(e, series_capacity=16)
    lf.start()
    lf.run(10)
    ser = lf.series()
    print(ser[:, 0], g["r_step_epot"])
    assert np.allclose(ser[:, 0], g["r_step_epot"], rtol=1e-7)
    assert np.allclose(ser[:, 2], g["r_step_atomtemp"], rtol=1e-7)
    st = e.state()
    assert np.allclose(st["pos"].reshape(-1), g["r_final_pos"], rtol=0, atol=1e-9)


@pytest.mark.parametrize("reference_forms", [False, True])
def test_fp64_forms_against_reference(reference_forms):
    # the FP64 path by its default algorithms (column reciprocal passes with
    # exact 64-bit phases, product-form 14-7) and by the reference's own forms
    # (one sine/cosine per (site, k), pow()) both give the reference's forces
    g = golden("polwater216")
    e = engine.GpuEnsemble(_pw())
    e.set_reference_forms(reference_forms)
    e.set_solver(tol=1e-13, max_iter=1000)
    for term, key in ((L.TERM_VDW, "f_buff_force"), (L.TERM_MP_LONG, "f_mp_long_force"),
                      (L.TERM_IND_LONG, "f_ind_long_force")):
        f, _, _ = e.compute_forces(term)
        err = rms_rel(f, g[key].reshape(-1, 3))
        print(reference_forms, key, err)
        assert err < 1e-10
    f_all, _, _ = e.compute_forces()
    ref = sum(g[k].reshape(-1, 3) for k in ("f_buff_force", "f_mp_short_force", "f_mp_long_force",
                                            "f_ind_short_force", "f_ind_long_force"))
    assert rms_rel(f_all, ref) < 1e-9
    e.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("nmol,kmax", [(216, 7), (4096, 18)])
def test_pipelined_solve_matches_single_reduction(nmol, kmax, precision):
    """The pipelined PCG (one grid barrier per iteration) and the
    single-reduction form solve the same system at the working dipole
    tolerance: the same iterations within one, forces within the tolerance's
    own effect, both well inside the 1e-6 bound."""
    if nmol == 216:
        s = systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3)
    else:
        s = systems.polarizable_water(nmol=nmol, kmax=kmax, seed=1)
    ens = engine.GpuEnsemble(s, precision=precision)
    out = {}
    for pipe in (False, True):
        ens.set_solver_pipelined(2 if pipe else 0)
        ens.set_solver(tol=2.0819e-8, max_iter=500)
        f, e, _ = ens.compute_forces()
        out[pipe] = (f, e, ens.solver_stats()[0])
    print(out[False][2], out[True][2], rms_rel(out[True][0], out[False][0]))
    assert abs(out[True][2] - out[False][2]) <= 1
    assert rms_rel(out[True][0], out[False][0]) < 2e-7
    ens.close()

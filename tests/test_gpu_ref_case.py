"""The reference's own shipped case (its test/ directory: 500 flexible
polarisable waters with AMOEBA bonds and angles, a Urey-Bradley H-H term,
buffered 14-7, permanent multipoles, induced dipoles and surface-dipole
corrections), read from its input files by systems.read_reference_case and
run at constant volume, against the reference's own results for the same
inputs (tests/golden/make_golden.py, case ref_test_nvt)."""
import os

import numpy as np
import pytest

from conftest import golden, rms_rel
from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu

TERMS = ((L.TERM_VDW, "f_buff", L.E_VDW, 0), (L.TERM_MP_SHORT, "f_mp_short", L.E_REAL, 1),
         (L.TERM_MP_LONG, "f_mp_long", L.E_LONG, 2), (L.TERM_IND_SHORT, "f_ind_short", L.E_POL_REAL, 6),
         (L.TERM_IND_LONG, "f_ind_long", L.E_POL_LONG, 7), (L.TERM_BOND, "f_bond", L.E_BOND, 11),
         (L.TERM_ANGLE, "f_angle", L.E_ANGLE, 12), (L.TERM_UB, "f_ub", L.E_UB, 13))


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    g = golden("ref_test_nvt")
    d = tmp_path_factory.mktemp("ref_test_nvt")
    for key, fn in (("case_config", "config.txt"), ("case_sysdata", "sysData.in"), ("case_coords", "coordinate.in")):
        (d / fn).write_text(str(g[key]))
    s = systems.read_reference_case(str(d))
    assert np.array_equal(s.pos, g["pos"])
    return s, g


def test_pairs_and_velocities(case):
    s, g = case
    ens = engine.GpuEnsemble(s)
    p = ens.pairs()
    p = p[np.lexsort((p[:, 1], p[:, 0]))]
    assert np.array_equal(p, g["pairs"])
    assert np.allclose(engine.init_velocity(s).reshape(-1), g["f_init_vel"], rtol=0, atol=1e-12)
    ens.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_terms(case, precision, tol):
    s, g = case
    ens = engine.GpuEnsemble(s, precision=precision)
    ens.set_solver(tol=1e-13, max_iter=2000)
    f_tot = np.zeros((ens.n, 3))
    for term, key, slot, eidx in TERMS:
        f, e, w = ens.compute_forces(term)
        f_tot += f
        err = rms_rel(f, g[key + "_force"])
        ref_e = g[key + "_energy"]
        print(precision, key, err, e[slot], ref_e[eidx])
        assert err < (2 * tol if term in (L.TERM_MP_LONG, L.TERM_IND_LONG) else tol)
        assert abs(e[slot] - ref_e[eidx]) < tol * abs(ref_e[eidx])
        if term == L.TERM_MP_SHORT:     # the multipole surface term
            assert abs(e[L.E_SURF] - ref_e[5]) < 1e-9 * abs(ref_e[5])
        if term == L.TERM_IND_SHORT:    # the induced-dipole surface term
            assert abs(e[L.E_POL_SURF] - ref_e[10]) < max(tol, 1e-8) * abs(ref_e[10])
        if precision == "fp64":
            # the virial with the reference's sign and component order: the
            # short-range terms' Ensemble::virial, the reciprocal terms'
            # Ensemble::longVirial (components 0..7, as their compute_long
            # copies them)
            if term in (L.TERM_MP_LONG, L.TERM_IND_LONG):
                ref_w, ours = g[key + "_longvirial"][:8], w[:8]
            else:
                ref_w, ours = g[key + "_virial"], w
            print(key, "virial", np.max(np.abs(ours - ref_w)))
            assert np.max(np.abs(ours - ref_w)) < 1e-8 * max(1.0, np.max(np.abs(ref_w)))
    ref = sum(g[k + "_force"] for _, k, _, _ in TERMS)
    err = rms_rel(f_tot, ref)
    print(precision, "total", err)
    assert err < tol
    ens.close()


def test_trajectory(case):
    s, g = case
    ens = engine.GpuEnsemble(s)
    ens.set_solver(tol=1e-13, max_iter=2000)
    lf = engine.LFIntegrator(ens, series_capacity=16)
    lf.start()
    lf.run(10)
    ser = lf.series()
    print(ser[:, 0] - g["r_step_epot"])
    assert np.allclose(ser[:, 0], g["r_step_epot"], rtol=1e-8)
    assert np.allclose(ser[:, 2], g["r_step_atomtemp"], rtol=1e-8)
    st = ens.state()
    assert np.allclose(st["pos"].reshape(-1), g["r_final_pos"], rtol=0, atol=1e-9)
    assert np.allclose(st["vel"].reshape(-1), g["r_final_vel"], rtol=0, atol=1e-7)
    ens.close()

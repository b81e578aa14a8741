"""Failure paths of the C ABI: each one is made on the host side (an
iteration cap, a non-finite upload, a compressed cluster, a solve block that
never arrives at its barrier, whose waits are bounded) and must come back as
its status code with the context still usable.  Nothing here faults, traps
or hangs the GPU: every device-side wait has a time limit and every list
write is bounds-checked."""
import numpy as np
import pytest

from conftest import rms_rel
from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _pw():
    return systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3,
                                     n_steps=10)


def _status(fn):
    try:
        fn()
    except L.SmdError as ex:
        return ex.code, str(ex)
    return L.SMD_OK, ""


def test_dipole_iteration_cap():
    """A solve stopped by its iteration cap returns SMD_ERR_CG; a cap equal to
    the iterations the solve needs converges and returns SMD_OK."""
    ens = engine.GpuEnsemble(_pw())
    ens.set_solver(tol=2.0819e-8, max_iter=500)
    f_ok, _, _ = ens.compute_forces(L.TERM_IND_SHORT)
    need = ens.solver_stats()[0]
    assert need > 2
    ens.set_solver(tol=2.0819e-8, max_iter=need)
    code, _ = _status(lambda: ens.compute_forces(L.TERM_IND_SHORT))
    assert code == L.SMD_OK
    assert ens.solver_stats()[0] == need
    ens.set_solver(tol=2.0819e-8, max_iter=need - 1)
    code, msg = _status(lambda: ens.compute_forces(L.TERM_IND_SHORT))
    assert code == L.SMD_ERR_CG, msg
    ens.set_solver(tol=2.0819e-8, max_iter=1)
    code, msg = _status(lambda: ens.compute_forces(L.TERM_IND_SHORT))
    assert code == L.SMD_ERR_CG and "converge" in msg
    # the context stays usable
    ens.set_solver(tol=2.0819e-8, max_iter=500)
    f, _, _ = ens.compute_forces(L.TERM_IND_SHORT)
    assert np.array_equal(f, f_ok)
    ens.close()


def test_barrier_wait_runs_out():
    """One block of the dipole solve never arrives at the grid barrier: the
    others give up after the (1 ms) wait limit, the call returns
    SMD_ERR_TIMEOUT, and the next solve without the hook gives the normal
    result."""
    ens = engine.GpuEnsemble(_pw())
    ens.set_solver(tol=2.0819e-8, max_iter=500)
    f_ok, _, _ = ens.compute_forces(L.TERM_IND_SHORT)
    ens._chk(ens.lib.smd_set_wait_limit(ens.ctx, 1e-3))
    ens._chk(ens.lib.smd_test_skip_arrival(ens.ctx, 1))
    code, msg = _status(lambda: ens.compute_forces(L.TERM_IND_SHORT))
    assert code == L.SMD_ERR_TIMEOUT, msg
    assert "barrier" in msg
    ens._chk(ens.lib.smd_test_skip_arrival(ens.ctx, -1))
    ens._chk(ens.lib.smd_set_wait_limit(ens.ctx, 1.0))
    f, _, _ = ens.compute_forces(L.TERM_IND_SHORT)
    assert rms_rel(f, f_ok) < 1e-12
    # the hook refuses blocks the solve does not have
    code, _ = _status(lambda: ens._chk(ens.lib.smd_test_skip_arrival(ens.ctx, 1 << 20)))
    assert code == L.SMD_ERR_ARG
    ens.close()


def test_shake_iteration_cap():
    s = systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=20)
    s.config.max_count = 1
    ens = engine.GpuEnsemble(s)
    lf = engine.LFIntegrator(ens)
    lf.start()
    code, msg = _status(lambda: lf.run(2))
    assert code == L.SMD_ERR_SHAKE, msg
    ens.close()


def test_non_finite_upload():
    s = systems.lj_fluid(ncell=5, jitter_star=0.05, seed=3)
    ens = engine.GpuEnsemble(s)
    f0, _, _ = ens.compute_forces()
    bad = s.pos.copy()
    bad[17, 1] = np.nan
    code, msg = _status(lambda: ens.upload_positions(bad))
    assert code == L.SMD_ERR_NAN and "17" in msg
    v = np.zeros((s.n_atoms, 3))
    v[3, 0] = np.inf
    code, _ = _status(lambda: ens.upload_velocities(v))
    assert code == L.SMD_ERR_NAN
    # the state is unchanged
    f1, _, _ = ens.compute_forces()
    assert np.array_equal(f0, f1)
    ens.close()


def test_list_overflow():
    """A cluster compressed to 0.6 of its spacing holds 4.6x the neighbours
    the list was sized for: SMD_ERR_LIST_OVERFLOW (every write past a row's
    end is skipped), and the original positions evaluate normally again."""
    s = systems.lj_fluid(ncell=5, jitter_star=0.05, seed=3)
    ens = engine.GpuEnsemble(s)
    f0, _, _ = ens.compute_forces()
    code, msg = _status(lambda: (ens.upload_positions(s.pos * 0.6), ens.compute_forces()))
    assert code == L.SMD_ERR_LIST_OVERFLOW, msg
    ens.upload_positions(s.pos)
    f1, _, _ = ens.compute_forces()
    assert rms_rel(f1, f0) < 1e-12
    ens.close()

"""The reference's NpT run (NHIntegrator: Nose-Hoover chain plus the
isotropic MTK barostat driven by the Lustig virial pressure) on the GPU
chain integrator, step by step against the reference's own run of the same
system (lj500_npt: 25 steps of 4 fs near the state's pressure), and the
barostat's cell-grid guard."""
import ctypes

import numpy as np
import pytest

from conftest import golden
from swinmd_b200 import engine, systems
from swinmd_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _lj_npt(ncell=5, pressure=-240.0, baros=1.0, cells=True, tail=True):
    s = systems.lj_fluid(ncell=ncell, jitter_star=0.05, seed=3, n_steps=25)
    c = s.config
    c.long_correct = tail
    c.ensemble, c.pressure, c.baros_const, c.coupl_const = 1, pressure, baros, 0.5
    c.lustig = True
    c.timestep = 0.004
    c.use_cell_list = cells
    return s


def test_npt_trajectory_matches_reference():
    g = golden("lj500_npt")
    ens = engine.GpuEnsemble(_lj_npt())
    nh = engine.NHIntegrator(ens)
    nh.start()
    rows = []
    for _ in range(25):
        nh.run(1)
        o = nh.observables()
        vlog, molvirt, vol = nh.barostat_state()
        rows.append([o.e_potential, o.ke_atom, o.t_atom, vol, nh.box()[0], vlog, molvirt,
                     2.0 * o.ke_atom / (3.0 * vol) - molvirt, *nh.chain_state()])
    r = np.array(rows)
    print("volume", r[[0, -1], 3], g["nh_volume"][[0, -1]])
    assert np.allclose(r[:, 3], g["nh_volume"], rtol=1e-11, atol=0)
    assert np.allclose(r[:, 4], g["nh_boxl"], rtol=1e-11, atol=0)
    assert np.allclose(r[:, 0], g["nh_epot"], rtol=1e-9, atol=0)
    assert np.allclose(r[:, 1], g["nh_ekin"], rtol=1e-9, atol=0)
    assert np.allclose(r[:, 2], g["nh_atomtemp"], rtol=1e-9, atol=0)
    assert np.allclose(r[:, 5], g["nh_vlog"], rtol=1e-7, atol=1e-12)
    assert np.allclose(r[:, 6], g["nh_molvirt"], rtol=1e-9, atol=0)
    assert np.allclose(r[:, 7], g["nh_molpt"], rtol=1e-8, atol=0)
    assert np.allclose(r[:, 8:12].reshape(-1), g["nh_vnh"], rtol=1e-7, atol=1e-12)
    st = ens.state()
    assert np.allclose(st["pos"].reshape(-1), g["nh_final_pos"], rtol=0, atol=1e-9)
    assert np.allclose(st["vel"].reshape(-1), g["nh_final_vel"], rtol=0, atol=1e-8)
    ens.close()


def test_npt_tail_correction_follows_the_volume():
    # with the tail correction the energy and molVirt carry E = K / V and
    # dU/dV = -2 E / V of the current volume (LJForce::long_range_correct)
    s = _lj_npt(tail=True)
    e0, _ = engine.lj_long_range_correction(s)
    v0 = systems.reference_box(s) ** 3
    runs = []
    for tail in (True, False):
        ens = engine.GpuEnsemble(_lj_npt(tail=tail))
        nh = engine.NHIntegrator(ens)
        nh.start()
        nh.run(1)   # the first step's drift does not depend on the forces
        o = nh.observables()
        runs.append((o.e_potential, nh.barostat_state()))
        ens.close()
    (ea, (_, mva, vol)), (eb, (_, mvb, _)) = runs
    e_lrc = e0 * v0 / vol
    assert abs((ea - eb) - e_lrc) < 1e-9 * abs(e_lrc)
    assert abs((mva - mvb) - (-2.0 * e_lrc / vol)) < 1e-9 * abs(e_lrc / vol)


def test_npt_cell_grid_matches_all_pairs():
    # 4000 atoms: the cell grid (laid out 10 % small, scaled with the box)
    # and the all-pairs build give the same pair set, so the same run
    runs = []
    for cells in (True, False):
        ens = engine.GpuEnsemble(_lj_npt(ncell=10, pressure=200.0, baros=0.5, cells=cells))
        nh = engine.NHIntegrator(ens)
        nh.start()
        nh.run(40)
        runs.append((ens.state()["pos"], nh.box()[0], nh.observables().list_updates))
        ens.close()
    (p1, b1, u1), (p2, b2, u2) = runs
    print("box", b1, b2, "list updates", u1, u2)
    # the list orders differ, so the per-site sums round differently
    assert abs(b1 - b2) < 1e-12 * b1
    assert np.allclose(p1, p2, rtol=0, atol=1e-9)


def test_barostat_guard_and_refusals():
    # a box squeezed past what the cell grid covers stops the run with
    # SMD_ERR_BOX (the kernels only ever clamp a cell index: no fault)
    # (2000 MPa pulls the edges in by 10 % within a few tens of steps,
    # before the compressed fluid's repulsion could stop it)
    ens = engine.GpuEnsemble(_lj_npt(ncell=10, pressure=2000.0, baros=1.0))
    nh = engine.NHIntegrator(ens)
    nh.start()
    code = ens.lib.smd_run(ens.ctx, 200)
    print("box after the guard", nh.box()[0])
    assert code == L.SMD_ERR_BOX, code
    ens.close()
    # mixed precision and the leap-frog integrator are refused under NpT
    ens = engine.GpuEnsemble(_lj_npt(), precision="mixed")
    nh = engine.NHIntegrator(ens)
    assert ens.lib.smd_integrator_start(ens.ctx) == L.SMD_ERR_ARG
    ens.close()
    ens = engine.GpuEnsemble(_lj_npt())
    with pytest.raises(NotImplementedError):
        engine.LFIntegrator(ens)
    ens.close()

"""Nose-Hoover chain velocity-Verlet integrator and SLLOD shear with
Lees-Edwards images on the GPU against the FP64 restatement in
oracle/smd_oracle.c (or_lj_nhc_md).  The reference has no constant-volume
chain integrator and no SLLOD code, so these rows are checked against the
restatement only."""
import numpy as np
import pytest

import oracle
from swinmd_b200 import engine, systems

pytestmark = pytest.mark.gpu

AR_TAU = systems.AR_TAU


def _sys(rate_star=0.0, ncell=5, steps=40):
    s = systems.lj_fluid(ncell=ncell, jitter_star=0.05, seed=3, n_steps=steps, strain_rate_star=rate_star)
    s.config.long_correct = False
    return s


def rel(a, b):
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300))


@pytest.mark.parametrize("rate_star", [0.0, 1.0])
def test_chain_trajectory_matches_oracle(rate_star):
    s = _sys(rate_star)
    ens = engine.GpuEnsemble(s, precision="fp64")
    st0 = ens.state()
    nh = engine.NHIntegrator(ens, series_capacity=64)
    nh.start()
    nsteps = 40
    nh.run(nsteps)
    ser = nh.series()
    st = ens.state()
    ref = oracle.lj_nhc_md(s, st0["pos"], st0["vel"], s.box, nsteps,
                           strain_rate=s.config.rate if rate_star else 0.0)
    # per-step potential energy, temperature, first chain velocity, P_xy
    assert rel(ser[:, 0], ref["epot"]) < 1e-9
    assert rel(ser[:, 2], ref["temp"]) < 1e-9
    assert rel(ser[:, 3], ref["vnh0"]) < 1e-8
    assert rel(ser[:, 4], ref["pxy"]) < 1e-7
    assert rel(st["vel"], ref["vel"]) < 1e-8
    d = st["pos"] - ref["pos"]
    L = np.array(s.box)
    d -= L * np.round(d / L)
    assert np.max(np.abs(d)) < 1e-9
    o = nh.observables()
    if rate_star:
        # the shear stress of a sheared LJ liquid is negative (P_xy < 0)
        assert np.mean(ref["pxy"][nsteps // 2:]) < 0
        assert ref["delta"][-1] > 0
        assert abs(o.shear_offset - ref["delta"][-1]) < 1e-12
        assert o.list_updates >= 1


def test_sheared_forces_mixed_vs_fp64():
    s = _sys(1.0)
    ens = engine.GpuEnsemble(s, precision="fp64")
    nh = engine.NHIntegrator(ens)
    nh.start()
    nh.run(60)   # moves the Lees-Edwards offset well away from zero
    f64, e64, w64 = ens.compute_forces()
    ens.set_precision("mixed")
    f32, e32, w32 = ens.compute_forces()
    err = float(np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum()))
    print("sheared mixed rms rel force err", err)
    assert err < 1e-6
    assert abs(e32[0] - e64[0]) < 1e-6 * abs(e64[0])


def test_sheared_pair_set_with_cells():
    # 4000 atoms: the cell search (5 cells per edge) with the Lees-Edwards
    # window must find the same pairs as the all-pairs search
    s = _sys(1.0, ncell=10)
    ens = engine.GpuEnsemble(s, precision="fp64")
    nh = engine.NHIntegrator(ens)
    nh.start()
    nh.run(30)
    f_cells, e_cells, _ = ens.compute_forces()
    st = ens.state()
    delta = nh.observables().shear_offset
    assert delta > 0
    # all-pairs forces at the same configuration and offset from the oracle
    f_ref, e_ref = oracle.lj_le_forces(s, st["pos"], s.box, delta)
    assert rel(f_cells, f_ref) < 1e-10
    assert abs(e_cells[0] - e_ref) < 1e-10 * abs(e_ref)

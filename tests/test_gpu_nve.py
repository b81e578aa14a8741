"""Energy conservation as the reference has it: the polarisable water run
without thermostat (NVE) from the reference's start, 80 steps, against the
reference's own per-step potential and kinetic energies.  The model's total
energy is not conserved (it rises by about 1.6e6 kJ/mol/ns at 216
molecules from this start, in the reference as here), so the test pins the
curve, not a flat line: the GPU run must gain the energy the reference
gains, step by step."""
import numpy as np
import pytest

from conftest import golden
from swinmd_b200 import engine, systems

pytestmark = pytest.mark.gpu


def _pw_nve():
    s = systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3, n_steps=80)
    s.config.thermostat = "None"
    return s


def test_nve_energy_curve_matches_reference():
    g = golden("polwater216_nve")
    e = engine.GpuEnsemble(_pw_nve())
    e.set_solver(tol=1e-13, max_iter=1000)
    lf = engine.LFIntegrator(e, series_capacity=128)
    lf.start()
    lf.run(80)
    ser = lf.series()
    u_ref, k_ref = g["r_step_epot"], g["r_step_ekin"]
    # the first 40 steps to the reference's precision, the rest within the
    # divergence of two chaotic trajectories after 80 steps
    assert np.allclose(ser[:40, 0], u_ref[:40], rtol=1e-7)
    assert np.allclose(ser[:40, 1], k_ref[:40], rtol=1e-7)
    h, h_ref = ser[:, 0] + ser[:, 1], u_ref + k_ref
    assert np.max(np.abs(h - h_ref)) < 1e-3 * np.max(np.abs(h_ref))
    # the thermostat is off: zeta stays zero
    assert np.all(ser[:, 3] == 0.0)
    # the energy gained over the run, as the reference gains it
    gain, gain_ref = h[-1] - h[20], h_ref[-1] - h_ref[20]
    assert abs(gain - gain_ref) < 0.02 * abs(gain_ref)
    e.close()

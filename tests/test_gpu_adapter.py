"""The drop-in boundary in C++: the reference's own LFIntegrator (leap-frog,
Nose-Hoover, SHAKE, pressure, all on the host) driving the GPU force object
of swinmd_b200/adapter/swinmd_gpu.h through the C ABI (every non-bonded
term, reciprocal space included, on the GPU), on the rigid SPC/E water and
on the polarisable multipole water.  The binary (oracle/_ref/adapter_run) is
the reference's sources plus the adapter, built by oracle/Makefile; its
trajectory must be the one the unmodified reference produced for the same
case."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden
from swinmd_b200 import systems

pytestmark = pytest.mark.gpu

EXE = os.path.join(ROOT, "oracle", "_ref", "adapter_run")


def _run(tmp_path, nsteps, precision="fp64", system=None):
    import refdump
    assert os.path.exists(EXE), "oracle/_ref/adapter_run is not built (make -C oracle)"
    s = system or systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=20)
    systems.write_reference_case(s, str(tmp_path))
    args = [EXE, str(nsteps), "out.txt"] + (["mixed"] if precision == "mixed" else [])
    r = subprocess.run(args, cwd=str(tmp_path), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return refdump.read_records(os.path.join(str(tmp_path), "out.txt"))


def test_reference_integrator_with_gpu_forces(tmp_path):
    g = golden("spce512")
    out = _run(tmp_path, 20)
    print(np.max(np.abs(out["step_epot"] / g["r_step_epot"] - 1)))
    assert np.allclose(out["step_epot"], g["r_step_epot"], rtol=1e-8)
    assert np.allclose(out["step_atomtemp"], g["r_step_atomtemp"], rtol=1e-8)
    assert np.allclose(out["step_zeta"], g["r_step_zeta"], rtol=1e-7, atol=1e-12)
    assert np.array_equal(out["step_nupdates"], g["r_step_nupdates"])
    # all nine components: the adapter copies the reciprocal virial as
    # EwaldForce::compute_long does (components 0..7)
    assert np.allclose(out["step_atompressure"], g["r_step_atompressure"], rtol=1e-7, atol=1e-6)
    # the Lustig pressure LFIntegrator reports (LFIntegrator.cpp:731-741)
    # from the myLustig fields the GPU object filled; from the second step,
    # as the reference's first step reads molecular centres no step has set
    print(out["step_molpt"] - g["r_step_molpt"])
    assert np.allclose(out["step_molpt"][1:], g["r_step_molpt"][1:], rtol=1e-7, atol=1e-6)
    assert np.allclose(out["final_pos"], g["r_final_pos"], rtol=0, atol=1e-8)
    assert np.allclose(out["final_vel"], g["r_final_vel"], rtol=0, atol=1e-6)


def test_reference_integrator_with_mixed_gpu_forces(tmp_path):
    # the mixed path under the reference's integrator: the trajectory follows
    # the FP64 reference within the mixed path's force error
    g = golden("spce512")
    out = _run(tmp_path, 20, "mixed")
    assert np.allclose(out["step_epot"], g["r_step_epot"], rtol=2e-6)
    assert np.allclose(out["final_pos"], g["r_final_pos"], rtol=0, atol=1e-6)


def test_reference_integrator_with_gpu_polarisable_water(tmp_path):
    # buffered 14-7, permanent multipoles and induced dipoles (solved on the
    # GPU far below the reference's own stopping point) under the
    # reference's integrator with SHAKE
    g = golden("polwater216")
    s = systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3, n_steps=10)
    out = _run(tmp_path, 10, system=s)
    print(np.max(np.abs(out["step_epot"] / g["r_step_epot"] - 1)))
    assert np.allclose(out["step_epot"], g["r_step_epot"], rtol=1e-7)
    assert np.allclose(out["step_atomtemp"], g["r_step_atomtemp"], rtol=1e-7)
    print(out["step_molpt"] - g["r_step_molpt"])
    assert np.allclose(out["step_molpt"][1:], g["r_step_molpt"][1:], rtol=1e-6, atol=1e-5)
    assert np.allclose(out["final_pos"], g["r_final_pos"], rtol=0, atol=1e-9)

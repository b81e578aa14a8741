"""SLLOD planar shear with the point-charge Ewald sum: flexible SPC/E-like
water (bonds, angle, LJ on O, Ewald) under Lees-Edwards images, whose
reciprocal sum runs over the sheared cell's k list, rebuilt on the device
every evaluation.  Checked against the FP64 restatement
(or_flex_le_forces / or_flex_nhc_md in oracle/smd_oracle.c): the reference
has no shear, so parity is unpinned; the restatement's sheared lattice sum
is pinned by its properties in tests/test_oracle_shear.py."""
import numpy as np
import pytest

import oracle
from swinmd_b200 import _lib as L
from swinmd_b200 import engine, systems

pytestmark = pytest.mark.gpu

RATE = 5.0   # 1/ps: moves the offset by about 0.1 nm in 40 steps of 0.5 fs


def _sys(rate=RATE, nmol=343):
    """The seeded waters sit on a grid whose outer layer keeps clear of the
    box faces; shifted in y by a part of the grid spacing and wrapped by
    their centres, some molecules straddle the y faces, so that sites stick
    out of the box (the case the sheared images must get right)."""
    s = systems.spce_flexible(nmol=nmol, seed=2, strain_rate=rate)
    L = s.box[1]
    a = L / int(np.ceil(nmol ** (1.0 / 3.0) - 1e-9))
    pos = s.pos.reshape(-1, 3, 3) + np.array([0.0, 0.45 * a, 0.0])
    m = np.array([1.008, 15.9994, 1.008])
    com = (pos * m[None, :, None]).sum(1) / m.sum()
    pos += (com - L * np.floor(com / L + 0.5) - com)[:, None, :]
    s.pos = pos.reshape(-1, 3)
    return s


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def rel(a, b):
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_zero_offset_equals_the_unsheared_path(precision):
    out = []
    for rate in (0.0, RATE):
        s = _sys(rate)
        ens = engine.GpuEnsemble(s, precision=precision)
        engine.NHIntegrator(ens).start()   # the offset is zero before the first step
        out.append(ens.compute_forces() + (ens.ewald_nk(),))
    (f0, e0, w0, nk0), (f1, e1, w1, nk1) = out
    assert nk0 == nk1
    assert rms_rel(f1, f0) < 1e-13
    np.testing.assert_allclose(e1, e0, rtol=1e-13, atol=1e-10)
    np.testing.assert_allclose(w1, w0, rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_sheared_forces_match_oracle(precision, tol):
    s = _sys()
    ens = engine.GpuEnsemble(s, precision="fp64")
    nh = engine.NHIntegrator(ens)
    nh.start()
    nh.run(40)
    delta = nh.observables().shear_offset
    assert delta > 0.05
    ens.set_precision(precision)
    f, e, w = ens.compute_forces()
    st = ens.state()
    # molecules are wrapped whole, so some sites stick out of the box in y:
    # the FP32 path must take them to their Lees-Edwards image
    assert (np.abs(st["pos"][:, 1]) >= 0.5 * s.box[1]).any()
    ref = oracle.flex_le_forces(s, st["pos"], s.box[0], delta)
    assert ens.ewald_nk() == ref["nk"]
    err = rms_rel(f, ref["force"])
    print(precision, "sheared water rms rel force err", err)
    assert err < tol
    for idx, key in ((L.E_VDW, "vdw"), (L.E_REAL, "real"), (L.E_LONG, "long"), (L.E_MOLCORRECT, "intra"),
                     (L.E_BOND, "bond"), (L.E_ANGLE, "angle")):
        assert abs(e[idx] - ref[key]) < tol * abs(ref[key]) + 1e-9, key
    assert np.max(np.abs(w - ref["virial"])) < 10 * tol * np.abs(ref["virial"]).max()
    # the reciprocal term alone (sheared k set, FP32 phases on the mixed path)
    fl, el, _ = ens.compute_forces(L.TERM_EWALD_LONG)
    rl = oracle.ewald_recip_le(s, st["pos"], s.box[0], delta)
    assert rms_rel(fl, rl["force"]) < 10 * tol
    assert abs(el[L.E_LONG] - rl["energy"]) < tol * abs(rl["energy"])


def test_sheared_trajectory_matches_oracle():
    s = _sys(nmol=216)
    ens = engine.GpuEnsemble(s, precision="fp64")
    st0 = ens.state()
    nh = engine.NHIntegrator(ens, series_capacity=64)
    nh.start()
    _, e0, _ = ens.compute_forces()
    e_self = e0[L.E_CORRECT]
    nsteps = 40
    nh.run(nsteps)
    ser = nh.series()
    st = ens.state()
    ref = oracle.flex_nhc_md(s, st0["pos"], st0["vel"], s.box, nsteps, strain_rate=s.config.rate)
    assert rel(ser[:, 0] - e_self, ref["epot"]) < 1e-9
    assert rel(ser[:, 2], ref["temp"]) < 1e-9
    assert rel(ser[:, 3], ref["vnh0"]) < 1e-8
    assert rel(ser[:, 4], ref["pxy"]) < 1e-7
    assert rel(st["vel"], ref["vel"]) < 1e-8
    d = st["pos"] - ref["pos"]
    box = np.array(s.box)
    d -= box * np.round(d / box)
    assert np.max(np.abs(d)) < 1e-9
    assert abs(nh.observables().shear_offset - ref["delta"][-1]) < 1e-12
    assert ref["delta"][-1] > 0.05


def test_shear_refuses_multipoles():
    s = systems.polarizable_water(nmol=64, kmax=4, seed=1)
    s.config.constraint = 0   # flexible: the chain integrator's own requirement
    s.config.test_mode, s.config.rate = 2, 1.0
    ens = engine.GpuEnsemble(s, precision="fp64")
    with pytest.raises(L.SmdError):
        engine.NHIntegrator(ens)

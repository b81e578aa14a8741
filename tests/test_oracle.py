"""The CPU restatement (oracle/smd_oracle.c) pinned against the reference's
own outputs (golden fixtures made by running SwinMD's C++)."""
import numpy as np

import oracle
from conftest import golden
from swinmd_b200 import engine, systems


def _lj500():
    s = systems.lj_fluid(ncell=5, jitter_star=0.05, seed=3, n_steps=20)
    s.config.long_correct = True
    return s


def test_oracle_pairlist_matches_reference():
    g = golden("lj500")
    s = _lj500()
    p = oracle.pairlist(s, s.pos, float(g["box"][0]))
    p = p[np.lexsort((p[:, 1], p[:, 0]))]
    assert np.array_equal(p, g["pairs"])


def test_oracle_lj_matches_reference():
    g = golden("lj500")
    s = _lj500()
    e_lrc, v_lrc = engine.lj_long_range_correction(s)
    f, e, w = oracle.lj(s, s.pos, float(g["box"][0]), g["pairs"], e_lrc, v_lrc)
    assert np.allclose(f.reshape(-1), g["f_lj_force"], rtol=0, atol=1e-11)
    assert abs(e - g["f_lj_energy"][0]) < 1e-9 * abs(e)
    assert np.allclose(w, g["f_lj_virial"], rtol=1e-12, atol=1e-9)


def test_oracle_lj_md_matches_reference():
    g = golden("lj500")
    s = _lj500()
    e_lrc, v_lrc = engine.lj_long_range_correction(s)
    v0 = engine.init_velocity(s)
    assert np.array_equal(v0.reshape(-1), g["f_init_vel"])
    r = oracle.lj_md(s, s.pos, v0, float(g["box"][0]), 20, e_lrc, v_lrc)
    assert np.allclose(r["epot"], g["r_step_epot"], rtol=1e-12)
    assert np.allclose(r["temp"], g["r_step_atomtemp"], rtol=1e-12)
    assert np.allclose(r["zeta"], g["r_step_zeta"], rtol=1e-9, atol=1e-15)
    assert np.allclose(r["pos"].reshape(-1), g["r_final_pos"], rtol=0, atol=1e-12)

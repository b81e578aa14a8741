"""Checkpoint files in the reference's formats, on the CPU: a state.out and
vtMinus.out round trip exactly, and the reference's own reader layout
(title, count, rows) is what is written."""
import numpy as np

from swinmd_b200 import checkpoint


def test_state_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    pos, real, vel = rng.normal(size=(3, 7, 3))
    scal = rng.normal(size=32)
    p = tmp_path / "state.out"
    checkpoint.write_state(str(p), 42, pos, real, vel, scal, (2.5, 2.5, 2.5))
    step, p2, r2, v2, s2, box = checkpoint.read_state(str(p))
    assert step == 42 and box == (2.5, 2.5, 2.5)
    assert np.array_equal(p2, pos) and np.array_equal(r2, real) and np.array_equal(v2, vel)
    assert np.array_equal(s2, scal)
    lines = p.read_text().splitlines()
    # Integrator::write_state's layout: title, count, rows per section
    assert lines[0] == "Coordinate at step: 42" and lines[1] == "7"
    assert lines[9].startswith("Real positions at step: 42") and lines[10] == "7"
    assert lines[18].startswith("velocity at steps: 42")


def test_vtminus_round_trip(tmp_path):
    v = np.random.default_rng(1).normal(size=(5, 3))
    p = tmp_path / "vtMinus.out"
    checkpoint.write_vtminus(str(p), 100, v)
    assert p.read_text().splitlines()[0] == "vtMinus100"
    assert np.array_equal(checkpoint.read_vtminus(str(p)), v)

"""Checkpoint and restart files in the reference's formats.

``state.out`` (``Integrator::write_state``, src/Integrator.cpp:275-302):
a title line and the atom count, then one ``x y z`` line per atom, for the
positions, the real (unwrapped) positions and the velocities in turn.  The
reference reads the same layout back as ``state.in`` when a run does not
start new (``Ensemble::set_configuration``, src/Ensemble.cpp:303-317).
``vtMinus.out`` (``LFIntegrator::write_vtMinus``,
src/integrators/LFIntegrator.cpp:2030-2050): a title line, the atom count
and the half-step velocities, read back as ``vtMinus.in``
(``LFIntegrator::read_vtMinus``, :2052-2092).

The numbers are written with 17 significant digits (the reference writes
the stream default of 6), so a restart continues the trajectory exactly.
After the three sections this writer adds two lines the reference's reader
never reaches: the integrator's scalars (the Nose-Hoover zeta and its
half-step value, and the rest of smd_get_integrator_state) and the box.
"""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np


def _block(title: str, a: np.ndarray) -> str:
    rows = "\n".join(f"{float(x)!r} {float(y)!r} {float(z)!r}" for x, y, z in np.asarray(a).reshape(-1, 3))
    return f"{title}\n{len(np.asarray(a).reshape(-1, 3))}\n{rows}\n"


def write_state(path: str, step: int, pos: np.ndarray, real: np.ndarray, vel: np.ndarray,
                integrator_state: Optional[np.ndarray] = None, box: Optional[Tuple[float, float, float]] = None):
    text = _block(f"Coordinate at step: {step}", pos) + _block(f"Real positions at step: {step}", real) + \
        _block(f"velocity at steps: {step}", vel) + "\n"
    if integrator_state is not None:
        text += "Integrator state: " + " ".join(repr(float(v)) for v in integrator_state) + "\n"
    if box is not None:
        text += "Box: " + " ".join(repr(float(v)) for v in box) + "\n"
    with open(path, "w") as f:
        f.write(text)


def _read_block(lines, k):
    n = int(lines[k + 1].split()[0])
    a = np.array([[float(v) for v in lines[k + 2 + i].split()[:3]] for i in range(n)])
    return a, k + 2 + n


def read_state(path: str):
    """Returns (step, pos, real, vel, integrator_state or None, box or None)."""
    with open(path) as f:
        lines = f.read().splitlines()
    step = int(lines[0].split(":")[-1])
    pos, k = _read_block(lines, 0)
    real, k = _read_block(lines, k)
    vel, k = _read_block(lines, k)
    state = box = None
    for ln in lines[k:]:
        if ln.startswith("Integrator state:"):
            state = np.array([float(v) for v in ln.split(":", 1)[1].split()])
        elif ln.startswith("Box:"):
            box = tuple(float(v) for v in ln.split(":", 1)[1].split())
    return step, pos, real, vel, state, box


def write_vtminus(path: str, step: int, vtminus: np.ndarray):
    with open(path, "w") as f:
        f.write(_block(f"vtMinus{step}", vtminus) + "\n")


def read_vtminus(path: str) -> np.ndarray:
    with open(path) as f:
        lines = f.read().splitlines()
    a, _ = _read_block(lines, 0)
    return a

"""Generates the golden fixtures under tests/golden/ by running the reference.

Each fixture is one small seeded system from ``swinmd_b200.systems`` written
in the reference's input formats, run through the reference's own C++ code
(``oracle/_ref/ref_dump``, built by ``make -C oracle`` from the reference
sources) and saved with its inputs as a compressed .npz.  The GPU tests and
the CPU oracle are checked against these files; the reference itself is not
needed to run the tests.

    make -C oracle && python tests/golden/make_golden.py [case ...]
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from swinmd_b200 import systems  # noqa: E402
import refdump  # noqa: E402


def lj500():
    s = systems.lj_fluid(ncell=5, jitter_star=0.05, seed=3, n_steps=20)
    s.config.long_correct = True
    return s, [("forces",), ("run", 20)]


def nacl1000_mie():
    s = systems.nacl_melt(ncell=10, potential="mie", kmax=6, seed=5)
    return s, [("forces",), ("mie",)]


def spce512():
    s = systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=20)
    return s, [("forces",), ("run", 20)]


def polwater216():
    s = systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3,
                                  n_steps=10)
    return s, [("forces",), ("run", 10)]


CASES = {"lj500": lj500, "nacl1000_mie": nacl1000_mie, "spce512": spce512,
         "polwater216": polwater216}


def pack(name, s, results):
    out = {
        "box": np.array(results["forces"]["box"]),
        "pos": s.pos.astype(np.float64),
        "atom_type": s.atom_type.astype(np.int32),
        "mol_id": s.mol_id.astype(np.int32),
    }
    f = results["forces"]
    for k, v in f.items():
        if k in ("pairs",):
            p = v.astype(np.int32).reshape(-1, 2)
            p = p[np.lexsort((p[:, 1], p[:, 0]))]
            out["pairs"] = p
        elif k in ("mass", "scaled_charge", "type", "molid", "init_pos"):
            continue
        else:
            out["f_" + k] = v
    if "mie" in results:
        for k, v in results["mie"].items():
            if k.startswith("mie_"):
                out["m_" + k] = v
    if "run" in results:
        for k, v in results["run"].items():
            if k.startswith(("step_", "final_", "start_")):
                out["r_" + k] = v
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


def main(names):
    for name in names:
        s, modes = CASES[name]()
        with tempfile.TemporaryDirectory() as d:
            systems.write_reference_case(s, d)
            results = {}
            for m in modes:
                results[m[0]] = refdump.run_ref(d, *m, out=f"{m[0]}.txt")
        pack(name, s, results)
        print(name, "ok")


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES))

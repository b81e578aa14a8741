"""Generates the golden fixtures under tests/golden/ by running the reference.

Each fixture is one small seeded system from ``swinmd_b200.systems`` written
in the reference's input formats, run through the reference's own C++ code
(``oracle/_ref/ref_dump``, built by ``make -C oracle`` from the reference
sources) and saved with its inputs as a compressed .npz.  The GPU tests and
the CPU oracle are checked against these files; the reference itself is not
needed to run the tests.

    make -C oracle && python tests/golden/make_golden.py [case ...]

With no case names it makes the small cases; ``all`` adds the full-size
benchmark configurations (polwater4096 needs about 12 GB of memory and a
few minutes of one core).
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))

from swinmd_b200 import systems  # noqa: E402
import refdump  # noqa: E402
from conftest import pair_digest  # noqa: E402


def lj500():
    s = systems.lj_fluid(ncell=5, jitter_star=0.05, seed=3, n_steps=20)
    s.config.long_correct = True
    return s, [("forces",), ("run", 20), ("rdf",)]


def nacl1000_mie():
    s = systems.nacl_melt(ncell=10, potential="mie", kmax=6, seed=5)
    return s, [("forces",), ("mie",)]


def spce512():
    s = systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=20)
    return s, [("forces",), ("run", 20), ("rdf",)]


def polwater216():
    s = systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3,
                                  n_steps=10)
    return s, [("forces",), ("run", 10)]


def polwater216_amoeba():
    # the induced real space damped as Tinker's AMOEBA (dampAMOEBA,
    # Induction.cpp:1051-1079): the same configuration as polwater216
    s, _ = polwater216()
    s.config.damp_amoeba = True
    return s, [("forces",)]


def lj500_npt():
    # NHIntegrator's NpT run (chain + isotropic barostat, Lustig virial
    # pressure) near the state's own pressure; 25 steps of 4 fs keep every
    # atom within half the skin of the start's list, which the reference's
    # NpT loop never rebuilds.  The tail correction is recomputed at every
    # step's volume (with the checker build's zero start of its accumulator)
    s = systems.lj_fluid(ncell=5, jitter_star=0.05, seed=3, n_steps=25)
    c = s.config
    c.long_correct = True
    c.ensemble, c.pressure, c.baros_const, c.coupl_const = 1, -240.0, 1.0, 0.5
    c.lustig = True
    c.timestep = 0.004
    return s, [("forces",), ("nhrun", 25)]


def spce512_wolf():
    # Wolf summation instead of Ewald; the O charge of every "WAT" molecule
    # sits on WolfForce's displaced site
    s = systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11)
    s.config.compute_ewald, s.config.compute_wolf, s.config.alpha = False, True, 2.0
    return s, [("forces",)]


def nacl1000_wolf():
    # ions (no displaced sites): the charge term fused into the pair pass
    s = systems.nacl_melt(ncell=10, potential="mie", kmax=6, seed=5)
    s.config.compute_ewald, s.config.compute_wolf, s.config.alpha = False, True, 2.5
    return s, [("forces",)]


def lj500_lustig():
    # Lustig's volume derivatives of the LJ energy (LJForce.cpp:136-250)
    s, _ = lj500()
    s.config.lustig = True
    return s, [("forces",)]


def spce512_lustig():
    # the same with constraints: r_ij . R_ij with the molecules' centres,
    # which the reference fills in during a step; so from a run: the second
    # step's values at the positions the first step left
    s = systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=2)
    s.config.lustig = True
    return s, [("forces",), ("run", 2)]


# Every field of Ensemble::myLustig (Ensemble.h:77-108) as the reference's
# force terms write it during a step: two steps of LFIntegrator, the second
# step's values belonging to the positions (and molecular centres) the first
# step left.  One case per branch of the terms' derivative code: atoms
# (no constraints), flexible molecules (intramolecular forces, bonds),
# rigid molecules (r_ij . R_ij, the reciprocal centre-of-mass terms), the
# polarisable model and the reference's own flexible polarisable case.
def nacl1000_lustig():
    # point charges + LJ on ions, surface term on (EwaldForce, LJForce)
    s = systems.nacl_melt(ncell=10, potential="lj", kmax=6, seed=5, n_steps=2)
    s.config.lustig = True
    s.config.surface_correct = True
    return s, [("forces",), ("run", 2)]


def spcf216_lustig():
    # flexible SPC/E-like water: harmonic bonds and angle, Ewald with the
    # intramolecular correction's forces
    s = systems.spce_flexible(nmol=216, seed=4, n_steps=2)
    s.config.lustig = True
    s.config.surface_correct = True
    s.config.thermostat = "NoseHoover"
    return s, [("forces",), ("run", 2)]


def polwater216_lustig():
    # rigid polarisable multipole water with the surface terms
    s = systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3,
                                  n_steps=2)
    s.config.lustig = True
    s.config.surface_correct = True
    return s, [("forces",), ("run", 2)]


def spce512_wolf_lustig():
    # the Wolf sum with displaced O charge sites (WolfForce, realDeriv with
    # the molecules' centres)
    s = systems.spce_water(nmol=512, box=2.4953, cutoff=0.9, kmax=6, seed=11, n_steps=2)
    s.config.compute_ewald, s.config.compute_wolf, s.config.alpha = False, True, 2.0
    s.config.lustig = True
    return s, [("forces",), ("run", 2)]


def ref_test_lustig():
    # the reference's shipped flexible polarisable case (bonds, angles,
    # Urey-Bradley, buffered 14-7, multipoles, induction, surface terms)
    s, _ = ref_test_nvt()
    s.config.n_steps = 2
    s.config.lustig = True
    return s, [("forces",), ("run", 2)]


def saap500():
    # SAAPForce with the reference's own three-type table
    s = systems.three_type_fluid(ncell=5, seed=3)
    return s, [("forces",), ("saap",)]


def polwater216_nve():
    # the same water without thermostat: energy conservation of the model as
    # the reference integrates it (its total energy rises: the GPU run must
    # follow the same curve, not a conserved one)
    s = systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3,
                                  n_steps=80)
    s.config.thermostat = "None"
    return s, [("forces",), ("run", 80)]


# Full-size cases: the configurations the benchmark runs.  Their pair sets
# are stored as a count and a SHA-256 of the sorted (i < j) int32 pairs
# instead of the pairs themselves, which would take megabytes.
def lj4000():
    s = systems.lj_fluid(ncell=10, seed=1, n_steps=20)
    s.config.long_correct = True
    return s, [("forces",), ("run", 20)]


def lj4000_jitter():
    # the benchmark lattice starts as a perfect FCC crystal, whose forces
    # vanish by symmetry: the full-size force check uses the same lattice with
    # every atom displaced by up to 0.05 sigma
    s = systems.lj_fluid(ncell=10, jitter_star=0.05, seed=1)
    s.config.long_correct = True
    return s, [("forces",)]


def nacl8000_mie():
    s = systems.nacl_melt(ncell=20, potential="mie", kmax=10, seed=1)
    return s, [("forces",), ("mie",)]


def spce2160():
    s = systems.spce_water(nmol=2160, box=4.03, cutoff=1.0, kmax=9, seed=1, n_steps=20)
    return s, [("forces",), ("run", 20)]


def polwater4096():
    # the benchmark's polarisable water (|n| < 18); one force evaluation with
    # the reference's dipoles solved to its own tolerance (|r| < 1e-14)
    s = systems.polarizable_water(nmol=4096, kmax=18, seed=1)
    return s, [("forces",)]


def ref_test_nvt():
    # the reference's own shipped case (test/: 500 flexible polarisable
    # waters, AMOEBA bonds and angles, Urey-Bradley, buffered 14-7,
    # multipoles, induction, surface corrections), read from its input files
    # and run at constant volume (ensembleStatus 0) instead of NPT
    src = os.path.join(os.environ.get("SWINMD_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference"), "test")
    s = systems.read_reference_case(src, name="ref_test_nvt")
    s.config.ensemble = 0
    s.config.n_steps = 10
    return s, [("forces",), ("run", 10)]


CASES = {"lj500": lj500, "lj500_npt": lj500_npt, "nacl1000_mie": nacl1000_mie, "spce512": spce512,
         "polwater216": polwater216, "polwater216_amoeba": polwater216_amoeba, "spce512_wolf": spce512_wolf, "saap500": saap500,
         "lj500_lustig": lj500_lustig, "spce512_lustig": spce512_lustig, "nacl1000_wolf": nacl1000_wolf, "polwater216_nve": polwater216_nve, "ref_test_nvt": ref_test_nvt,
         "nacl1000_lustig": nacl1000_lustig, "spcf216_lustig": spcf216_lustig,
         "polwater216_lustig": polwater216_lustig, "ref_test_lustig": ref_test_lustig,
         "spce512_wolf_lustig": spce512_wolf_lustig}
LARGE = {"lj4000": lj4000, "lj4000_jitter": lj4000_jitter, "nacl8000_mie": nacl8000_mie, "spce2160": spce2160,
         "polwater4096": polwater4096}


def pack(name, s, results, large=False):
    out = {
        "box": np.array(results["forces"]["box"]),
        "pos": s.pos.astype(np.float64),
        "atom_type": s.atom_type.astype(np.int32),
        "mol_id": s.mol_id.astype(np.int32),
    }
    f = results["forces"]
    for k, v in f.items():
        if k in ("pairs",):
            if large:
                cnt, dig = pair_digest(v.reshape(-1, 2))
                out["pair_count"] = np.array(cnt, np.int64)
                out["pair_sha256"] = np.array(dig)
                continue
            p = v.astype(np.int32).reshape(-1, 2)
            p = p[np.lexsort((p[:, 1], p[:, 0]))]
            out["pairs"] = p
        elif k in ("mass", "scaled_charge", "type", "molid", "init_pos"):
            continue
        elif large and k in ("ind_E0", "init_vel", "mp_quad", "mp_dip"):
            continue
        else:
            out["f_" + k] = v
    if "mie" in results:
        for k, v in results["mie"].items():
            if k.startswith("mie_"):
                out["m_" + k] = v
    if "saap" in results:
        for k, v in results["saap"].items():
            if k.startswith("saap_"):
                out["s_" + k] = v
    if "nhrun" in results:
        for k, v in results["nhrun"].items():
            if k.startswith("nh_"):
                out[k] = v
    if "rdf" in results:
        for k, v in results["rdf"].items():
            if k.startswith("rdf_"):
                out[k] = v
    if "run" in results:
        for k, v in results["run"].items():
            if k.startswith(("step_", "final_", "start_")):
                # full-size runs keep the per-step series, the final state and
                # the small records (energies, virials)
                if large and v.size > 64 and k not in ("final_pos", "final_vel"):
                    continue
                out["r_" + k] = v
    if name == "ref_test_nvt":
        # the case itself as this project's writers emit it, so that the GPU
        # test can rebuild the System without the reference's files
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            systems.write_reference_case(s, d)
            for fn, key in (("config.txt", "case_config"), ("sysData.in", "case_sysdata"),
                            ("coordinate.in", "case_coords")):
                out[key] = np.array(open(os.path.join(d, fn)).read())
    if name.endswith("_lustig"):
        out = {k: v for k, v in out.items() if not k.startswith(("f_", "r_")) or
               k in ("f_lustig_lj", "f_lj_energy", "r_step_lustig", "r_step_lustig_all",
                     "r_step_molvirt", "r_step_molpt", "r_step_after1_pos", "r_step_epot",
                     "r_start_vtminus")}
        out.pop("pairs", None)
    if name.startswith("saap"):
        out = {k: v for k, v in out.items() if not k.startswith("f_")}
        out.pop("pairs", None)
    if name.endswith("_wolf"):  # (the Wolf Lustig case ends in _lustig)
        out = {k: v for k, v in out.items() if not k.startswith("f_") or k.startswith("f_wolf_")}
        out.pop("pairs", None)
    if name.endswith("_amoeba"):
        # the induced terms only: the rest is polwater216's
        out = {k: v for k, v in out.items() if not k.startswith("f_") or k.startswith(("f_ind_", "f_mp_dip", "f_mp_quad"))}
        out.pop("pairs", None)
    if name.endswith(("_nve", "_npt")):
        # the trajectory only: the forces of the start are polwater216's
        out = {k: v for k, v in out.items() if not k.startswith("f_") and k != "pairs"}
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


def main(names):
    for name in names:
        s, modes = {**CASES, **LARGE}[name]()
        with tempfile.TemporaryDirectory() as d:
            systems.write_reference_case(s, d)
            results = {}
            for m in modes:
                results[m[0]] = refdump.run_ref(d, *m, out=f"{m[0]}.txt")
        pack(name, s, results, large=name in LARGE)
        print(name, "ok")


if __name__ == "__main__":
    args = sys.argv[1:] or list(CASES)
    if args == ["all"]:
        args = list(CASES) + list(LARGE)
    main(args)

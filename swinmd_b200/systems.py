"""Synthetic systems and the reference's input-file formats.

A :class:`System` holds one simulation set-up the way SwinMD's input files
describe it: the per-type parameter table and topology of ``sysData.in``
(parsed by ``Parameters::read_sys_data``, src/Parameters.cpp:76-380), the
coordinates of the coordinate file (``Ensemble::read_coordinate``,
src/Ensemble.cpp:630-667) and the positional run configuration of
``config.txt`` (``SimConfiguration::read_config_file``,
src/SimConfiguration.cpp:695-932).  Units are the reference's: nm, ps, amu,
kJ/mol, e, K (src/NEMD_defs.h:97-108).

The generators build the benchmark systems from seeds (an FCC Lennard-Jones
fluid, a rock-salt NaCl melt, rigid 3-site water, polarisable multipole
water); :func:`write_reference_case` writes any of them in the reference's
formats so the same system can be fed to SwinMD itself.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional, Tuple

import numpy as np

BOLTZMAN = 0.0083145112          # kJ/mol/K          src/NEMD_defs.h:108
SQRTCOULOMBCONSTANT = 11.78708976  # sqrt(kJ nm/mol)/e src/NEMD_defs.h:97
COULOMBS = 138.93548501          # kJ nm/mol/e^2     src/NEMD_defs.h:98


@dataclasses.dataclass
class AtomType:
    """One row of the ``!AtomParams`` section (src/Parameters.cpp:108-140)."""
    mass: float
    charge: float
    eps: float
    sigma: float
    dip: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    quad: Tuple[float, float, float, float, float, float] = (0.0,) * 6  # xx xy xz yy yz zz
    polar: float = 0.0
    name: str = "X"
    long_name: str = "Atom"


@dataclasses.dataclass
class Config:
    """The fields of ``config.txt`` this path reads, with the reference's
    meaning (src/SimConfiguration.cpp:695-932)."""
    seed: int = 1
    timestep: float = 0.001          # ps
    n_steps: int = 10
    long_steps: int = 1              # longElectTsFrequency
    integrator: int = 2              # 0 Gear, 1 VV, 2 leap-frog, 3 NH chain
    ensemble: int = 0                # 0 NVT, 1 NPT
    temperature: float = 300.0       # K
    pressure: float = 0.101
    atom_thermo: bool = True         # 1: atomic thermostat, else molecular
    coupl_const: float = 0.5         # ps, Nose-Hoover tau
    thermostat: str = "NoseHoover"
    baros_const: float = 0.5
    test_mode: int = 0               # 0 equilibrium, 2 shear
    rate: float = 0.0                # strain rate (1/ps)
    cutoff: float = 1.0              # nm
    cutoff_ew: float = 1.0
    cut_buffer: float = 0.1
    density: float = 0.0             # sites per nm^3 (0: from coordinates)
    use_cell_list: bool = True
    constraint: int = 0              # 0 none, 1 Gaussian, 2 SHAKE
    tolerance: float = 1e-8
    max_count: int = 1000            # SHAKE iteration cap / bending type
    long_correct: bool = False
    switch_on: bool = True           # LJ energy shift at the cutoff
    switch_dist: float = 0.9
    compute_coulomb: bool = False
    compute_ewald: bool = False
    surface_correct: bool = False
    compute_wolf: bool = False
    alpha: float = 3.0               # Ewald alpha, 1/nm
    k_cutoff: float = 15.0           # |k| cutoff, 1/nm
    compute_multipole: bool = False
    compute_induction: bool = False
    compute_torques: bool = True
    damp_induction: bool = True
    induction_min: bool = True
    damp_amoeba: bool = False
    cutoff_ind: float = 0.9
    a_damping: float = 0.39
    compute_buff: bool = False
    n_buff: int = 14
    m_buff: int = 7
    delta_buff: float = 0.07
    gamma_buff: float = 0.12
    h_factor: float = 0.91
    compute_mie: bool = False
    n_mie: float = 12
    m_mie: float = 6
    lustig: bool = False


@dataclasses.dataclass
class System:
    name: str
    pos: np.ndarray                  # (N, 3) nm
    box: Tuple[float, float, float]
    atom_types: List[AtomType]
    atom_type: np.ndarray            # (N,) int32
    mol_id: np.ndarray               # (N,) int32
    mol_type_names: List[Tuple[str, int]]  # (name, atoms per molecule)
    mol_type: np.ndarray             # (nmol,) int32
    config: Config
    bonds: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 3), np.int32))   # a1 a2 type
    angles: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 4), np.int32))  # a1 a2 a3 type
    bond_params: List[Tuple[int, int, float, float]] = dataclasses.field(default_factory=list)  # t1 t2 r0 k
    angle_params: List[Tuple[int, int, int, float, float]] = dataclasses.field(default_factory=list)  # t1 t2 t3 deg k
    # pair-potential tables that the reference's input files cannot carry
    bmh: Optional[Dict[str, np.ndarray]] = None

    @property
    def n_atoms(self) -> int:
        return int(self.pos.shape[0])

    @property
    def n_mols(self) -> int:
        return int(self.mol_type.shape[0])

    def masses(self) -> np.ndarray:
        return np.array([self.atom_types[t].mass for t in self.atom_type], np.float64)

    def scaled_charges(self) -> np.ndarray:
        """``Atom::scaledCharge`` = charge * SQRTCOULOMBCONSTANT
        (src/Ensemble.cpp:183)."""
        return np.array([self.atom_types[t].charge * SQRTCOULOMBCONSTANT
                         for t in self.atom_type], np.float64)

    def lj_table(self) -> Tuple[np.ndarray, np.ndarray]:
        """Lorentz-Berthelot table storing sigma^2 and 4 eps
        (``Parameters::set_lj_param``, src/Parameters.cpp:1360-1372)."""
        nt = len(self.atom_types)
        s2 = np.zeros((nt, nt))
        e4 = np.zeros((nt, nt))
        for i, a in enumerate(self.atom_types):
            for j, b in enumerate(self.atom_types):
                sig = (a.sigma + b.sigma) / 2
                eps = math.sqrt(a.eps * b.eps)
                s2[i, j] = sig * sig
                e4[i, j] = 4.0 * eps
        return s2, e4

    def exclusion_table(self) -> List[List[int]]:
        """1-2 and 1-3 partners of every atom, ascending, as
        ``Ensemble::build_exclusion_table`` builds them
        (src/Ensemble.cpp:323-367)."""
        sets = [set() for _ in range(self.n_atoms)]
        for a1, a2, _ in self.bonds:
            sets[a1].add(int(a2)); sets[a2].add(int(a1))
        for a1, _, a3, _ in self.angles:
            sets[a1].add(int(a3)); sets[a3].add(int(a1))
        return [sorted(s) for s in sets]

    def replace(self, **kw) -> "System":
        return dataclasses.replace(self, **kw)


# ---------------------------------------------------------------------------
# reference file writers
# ---------------------------------------------------------------------------

def _tf(b: bool) -> str:
    return "t" if b else "f"


def write_config(cfg: Config, path: str, sysdata="sysData.in", coords="coordinate.in") -> None:
    """Writes ``config.txt`` in the positional layout that
    ``SimConfiguration::read_config_file`` expects (one field group per line,
    rest of the line ignored)."""
    c = cfg
    g = lambda x: repr(float(x))
    lines = [
        f"{sysdata}\t{coords}\t// input files",
        "result.out\trestart.out\tdump.out\t// outputs",
        "f\ttrajectory.out\t// trajectory",
        f"t\t{c.seed}\tf\tvelocity.in\t// isNewStart seed readVelocity",
        f"{g(c.timestep)}\t{c.n_steps}\t0\t// timeStep numSteps startSteps",
        f"1\t{c.long_steps}\t// nonbond / long frequencies",
        "10\t10\t10\t// avg print backup",
        f"{c.integrator}\t// integrator type",
        f"{c.ensemble}\t{g(c.temperature)}\t{g(c.pressure)}\t{1 if c.atom_thermo else 2}\t"
        f"{g(c.coupl_const)}\t{c.thermostat}\t{g(c.baros_const)}\t// ensemble",
        f"{c.test_mode}\t{g(c.rate)}\t// testMode rate",
        f"{g(c.cutoff)}\t{g(c.cutoff_ew)}\t{g(c.k_cutoff)}\t{g(c.cut_buffer)}\t// cutoffs",
        f"{g(c.density)}\t// density",
        "1.0\t1.0\t1.0\t// box",
        f"{_tf(c.use_cell_list)}\t1.5\t// cell list",
    ]
    if c.constraint == 2:
        lines.append(f"2\t{g(c.tolerance)}\t{c.max_count}\t// SHAKE")
    else:
        lines.append(f"{c.constraint}\t{g(c.tolerance)}\t{c.max_count}\t0.01\t// constraint")
    lines += [
        "f\t0.0\t0.0\t// UB",
        f"{_tf(c.long_correct)}\t{_tf(c.switch_on)}\t{g(c.switch_dist)}\t// lrc switch",
        f"{_tf(c.compute_coulomb)}\t{_tf(c.compute_ewald)}\t{_tf(c.surface_correct)}\t"
        f"{_tf(c.compute_wolf)}\t{g(c.alpha)}\t{g(c.k_cutoff)}\t// electrostatics",
        f"{_tf(c.compute_multipole)}\t{_tf(c.compute_induction)}\t{_tf(c.compute_torques)}\t"
        f"{_tf(c.damp_induction)}\t{_tf(c.induction_min)}\t{_tf(c.damp_amoeba)}\t"
        f"{g(c.cutoff_ind)}\t{g(c.a_damping)}\t// multipole",
        f"{_tf(c.compute_buff)}\t{c.n_buff}\t{c.m_buff}\t{g(c.delta_buff)}\t"
        f"{g(c.gamma_buff)}\t{g(c.h_factor)}\t// buffered 14-7",
        f"{_tf(c.compute_mie)}\t{g(c.n_mie)}\t{g(c.m_mie)}\t// Mie",
        "f\tf\t// ext forces",
        "30000\t20\t// sampling",
        "f\t0\t0\t// TTCF",
        "f\t400\t// RDF",
        "f\tmsd.xyz\t// MSD",
        "f\tvacf.out\t// VACF",
        f"{_tf(c.lustig)}\t// Lustig",
    ]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_sysdata(s: System, path: str) -> None:
    """Writes ``sysData.in`` in the sectioned layout of
    ``Parameters::read_sys_data`` (src/Parameters.cpp:76-380)."""
    g = lambda x: repr(float(x))
    L = ["!sysData file", "!Size_of_system",
         f"{s.n_mols}\t{len(s.mol_type_names)}\t! molecules, molecule types",
         f"{s.n_atoms}\t{len(s.atom_types)}\t! atoms, atom types",
         f"{len(s.bonds)}\t{len(s.bond_params)}\t! bonds",
         f"{len(s.angles)}\t{len(s.angle_params)}\t! angles",
         "0\t0\t! dihedrals", "0\t0\t! impropers", "",
         "!AtomParams", "!typeID Mass Charge Epsilon Sigma dip quad polar typeName atomName"]
    for i, a in enumerate(s.atom_types):
        vals = [a.mass, a.charge, a.eps, a.sigma, *a.dip, *a.quad, a.polar]
        L.append(f"{i}\t" + "\t".join(g(v) for v in vals) + f"\t{a.name}\t{a.long_name}")
    L += ["", "!BondParams", "!bondTypeID atomType1 atomType2 length forceConstant"]
    for i, (t1, t2, r0, k) in enumerate(s.bond_params):
        L.append(f"{i}\t{t1}\t{t2}\t{g(r0)}\t{g(k)}")
    L += ["", "!AngleParams", "!angTypeID aType1 aType2 aType3 degree K"]
    for i, (t1, t2, t3, deg, k) in enumerate(s.angle_params):
        L.append(f"{i}\t{t1}\t{t2}\t{t3}\t{g(deg)}\t{g(k)}")
    L += ["", "!DihedralParams", "!TypeID", "", "!ImproperParams", "!TypeID", "",
          "!MolTypes", "!molTypeID numOfAtoms molNames"]
    for i, (nm, na) in enumerate(s.mol_type_names):
        L.append(f"{i}\t{na}\t{nm}")
    L += ["", "!Atoms", "!atomID atomType molID molType"]
    for i in range(s.n_atoms):
        m = int(s.mol_id[i])
        L.append(f"{i}\t{int(s.atom_type[i])}\t{m}\t{int(s.mol_type[m])}")
    L += ["", "!Bonds", "!bondID atom1 atom2 bondType"]
    for i, (a1, a2, t) in enumerate(s.bonds):
        L.append(f"{i}\t{a1}\t{a2}\t{t}")
    L += ["", "!Angles", "!angleID atom1 atom2 atom3 angleType"]
    for i, (a1, a2, a3, t) in enumerate(s.angles):
        L.append(f"{i}\t{a1}\t{a2}\t{a3}\t{t}")
    L += ["", "!Dihedrals", "!dihedralID", "", "!Impropers", "!ImproperID"]
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def write_coordinates(pos: np.ndarray, path: str) -> None:
    """Coordinate file: atom count, then one ``x y z`` line per atom."""
    with open(path, "w") as f:
        f.write(f"{pos.shape[0]}\n")
        for x, y, z in pos:
            f.write(f"{float(x)!r} {float(y)!r} {float(z)!r}\n")


def write_reference_case(s: System, directory: str) -> None:
    os.makedirs(directory, exist_ok=True)
    cfg = dataclasses.replace(s.config, density=s.n_atoms / (s.box[0] * s.box[1] * s.box[2]))
    write_config(cfg, os.path.join(directory, "config.txt"))
    write_sysdata(s, os.path.join(directory, "sysData.in"))
    write_coordinates(s.pos, os.path.join(directory, "coordinate.in"))


def reference_box(s: System) -> float:
    """The cubic box edge the reference derives from the written density
    (``Ensemble::compute_bound_box``, src/Ensemble.cpp:399-406)."""
    dens = s.n_atoms / (s.box[0] * s.box[1] * s.box[2])
    return (s.n_atoms / dens) ** (1.0 / 3.0)


# ---------------------------------------------------------------------------
# generators
# ---------------------------------------------------------------------------

# argon reduced units for the Lennard-Jones fluid
AR_SIGMA = 0.3405                 # nm
AR_EPS = 119.8 * BOLTZMAN         # kJ/mol
AR_MASS = 39.948                  # amu
AR_TAU = AR_SIGMA * math.sqrt(AR_MASS / AR_EPS)  # ps


def _wrap(pos: np.ndarray, L: float) -> np.ndarray:
    return pos - L * np.floor(pos / L + 0.5)


def lj_fluid(ncell: int = 10, rho_star: float = 0.8442, t_star: float = 0.722,
             rc_star: float = 2.5, skin_star: float = 0.3, dt_star: float = 0.005,
             tau_star: float = 0.5, seed: int = 1, jitter_star: float = 0.0,
             n_steps: int = 10000, strain_rate_star: float = 0.0) -> System:
    """FCC Lennard-Jones fluid, ``4*ncell^3`` atoms at reduced density
    ``rho_star``, argon units (sigma 0.3405 nm, eps/kB 119.8 K)."""
    n = 4 * ncell ** 3
    L = (n / rho_star) ** (1.0 / 3.0) * AR_SIGMA
    a = L / ncell
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(ncell), np.arange(ncell), np.arange(ncell),
                             indexing="ij"), -1).reshape(-1, 3)
    pos = ((g[:, None, :] + basis[None, :, :] + 0.25) * a).reshape(-1, 3) - L / 2
    if jitter_star > 0:
        rng = np.random.default_rng(seed)
        pos = pos + rng.uniform(-jitter_star, jitter_star, pos.shape) * AR_SIGMA
    pos = _wrap(pos, L)
    cfg = Config(seed=seed, timestep=dt_star * AR_TAU, n_steps=n_steps,
                 temperature=t_star * 119.8, coupl_const=tau_star * AR_TAU,
                 cutoff=rc_star * AR_SIGMA, cutoff_ew=rc_star * AR_SIGMA,
                 cut_buffer=skin_star * AR_SIGMA, switch_on=True,
                 switch_dist=rc_star * AR_SIGMA,
                 test_mode=2 if strain_rate_star else 0,
                 rate=strain_rate_star / AR_TAU)
    return System(name=f"lj{n}", pos=pos, box=(L, L, L),
                  atom_types=[AtomType(AR_MASS, 0.0, AR_EPS, AR_SIGMA, name="Ar", long_name="Argon")],
                  atom_type=np.zeros(n, np.int32), mol_id=np.arange(n, dtype=np.int32),
                  mol_type_names=[("AR", 1)], mol_type=np.zeros(n, np.int32), config=cfg)

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
    max_count: int = 1000            # SHAKE iteration cap (constraint 2)
    bend_type: int = 1               # bond/angle form without constraints: 1 harmonic, 2 AMOEBA
    compute_ub: bool = False         # harmonic Urey-Bradley H-H term
    kl_ub: float = 0.0               # its force constant (kJ/mol/nm^2)
    l0_ub: float = 0.0               # its ideal distance (nm)
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
        lines.append(f"{c.constraint}\t{g(c.tolerance)}\t{c.bend_type}\t0.01\t// constraint, bending type")
    lines += [
        f"{_tf(c.compute_ub)}\t{g(c.kl_ub)}\t{g(c.l0_ub)}\t// UB",
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


def _tf_read(tok: str) -> bool:
    return tok.strip().lower().startswith("t")


def read_config(path: str) -> Tuple[Config, str, str]:
    """Reads the fields of ``config.txt`` this path uses, in the positional
    layout ``SimConfiguration::read_config_file`` parses
    (src/SimConfiguration.cpp:695-932): one field group per line, the rest of
    a line ignored.  Returns the Config and the sysData / coordinate file
    names."""
    with open(path) as f:
        rows = [ln.split("//")[0].split() for ln in f]
    rows = [r for r in rows if r]
    c = Config()
    sysdata, coords = rows[0][0], rows[0][1]
    c.seed = int(rows[3][1])
    c.timestep, c.n_steps = float(rows[4][0]), int(rows[4][1])
    c.long_steps = int(rows[5][1])
    c.integrator = int(rows[7][0])
    r = rows[8]
    c.ensemble, c.temperature, c.pressure = int(r[0]), float(r[1]), float(r[2])
    c.atom_thermo = int(r[3]) == 1
    c.coupl_const, c.thermostat, c.baros_const = float(r[4]), r[5], float(r[6])
    c.test_mode, c.rate = int(rows[9][0]), float(rows[9][1])
    r = rows[10]
    c.cutoff, c.cutoff_ew, c.k_cutoff, c.cut_buffer = float(r[0]), float(r[1]), float(r[2]), float(r[3])
    c.density = float(rows[11][0])
    c.use_cell_list = _tf_read(rows[13][0])
    r = rows[14]
    c.constraint, c.tolerance = int(r[0]), float(r[1])
    if c.constraint == 2:
        c.max_count = int(r[2])
    else:
        c.bend_type = int(r[2])
    r = rows[15]
    c.compute_ub, c.kl_ub, c.l0_ub = _tf_read(r[0]), float(r[1]), float(r[2])
    r = rows[16]
    c.long_correct, c.switch_on, c.switch_dist = _tf_read(r[0]), _tf_read(r[1]), float(r[2])
    r = rows[17]
    c.compute_coulomb, c.compute_ewald, c.surface_correct, c.compute_wolf = (_tf_read(x) for x in r[:4])
    c.alpha, c.k_cutoff = float(r[4]), float(r[5])
    r = rows[18]
    (c.compute_multipole, c.compute_induction, c.compute_torques, c.damp_induction, c.induction_min,
     c.damp_amoeba) = (_tf_read(x) for x in r[:6])
    c.cutoff_ind, c.a_damping = float(r[6]), float(r[7])
    r = rows[19]
    c.compute_buff, c.n_buff, c.m_buff = _tf_read(r[0]), int(r[1]), int(r[2])
    c.delta_buff, c.gamma_buff, c.h_factor = float(r[3]), float(r[4]), float(r[5])
    r = rows[20]
    c.compute_mie, c.n_mie, c.m_mie = _tf_read(r[0]), float(r[1]), float(r[2])
    c.lustig = _tf_read(rows[-1][0])
    return c, sysdata, coords


_SYSDATA_SECTIONS = {"Size_of_system", "AtomParams", "BondParams", "AngleParams", "DihedralParams",
                     "ImproperParams", "MolTypes", "Atoms", "Bonds", "Angles", "Dihedrals", "Impropers"}


def read_sysdata(path: str):
    """Reads ``sysData.in`` (``Parameters::read_sys_data``,
    src/Parameters.cpp:76-380): atom types, bond and angle parameters,
    molecule types and the topology sections."""
    with open(path) as f:
        lines = [ln.split("!")[0].strip() if not ln.lstrip().startswith("!") else ln.strip() for ln in f]
    sec, data = None, {}
    counts = []
    for ln in lines:
        if not ln:
            continue
        if ln.startswith("!"):
            head = ln[1:].split()[0] if len(ln) > 1 else ""
            if head in _SYSDATA_SECTIONS:
                sec = head
                data.setdefault(sec, [])
            continue
        if sec == "Size_of_system":
            counts.append([int(x) for x in ln.split()[:2]])
        elif sec is not None:
            data[sec].append(ln.split())
    types = []
    for r in data.get("AtomParams", []):
        # typeID, mass, charge, epsilon, sigma, dipole (3), quadrupole (6),
        # polarisability, type name, atom name
        v = [float(x) for x in r[1:15]]
        types.append(AtomType(mass=v[0], charge=v[1], eps=v[2], sigma=v[3], dip=tuple(v[4:7]),
                              quad=tuple(v[7:13]), polar=v[13], name=r[15] if len(r) > 15 else "X",
                              long_name=r[16] if len(r) > 16 else "Atom"))
    bond_params = [(int(r[1]), int(r[2]), float(r[3]), float(r[4])) for r in data.get("BondParams", [])]
    angle_params = [(int(r[1]), int(r[2]), int(r[3]), float(r[4]), float(r[5])) for r in data.get("AngleParams", [])]
    mol_types = [(r[2], int(r[1])) for r in data.get("MolTypes", [])]
    atoms = np.array([[int(x) for x in r[:4]] for r in data.get("Atoms", [])], np.int64)
    bonds = np.array([[int(x) for x in r[1:4]] for r in data.get("Bonds", [])], np.int32).reshape(-1, 3)
    angles = np.array([[int(x) for x in r[1:5]] for r in data.get("Angles", [])], np.int32).reshape(-1, 4)
    return types, bond_params, angle_params, mol_types, atoms, bonds, angles


def read_reference_case(directory: str, name: str = "case") -> System:
    """A System from a directory of the reference's own input files
    (config.txt, its sysData file and coordinate file), so that an existing
    SwinMD case runs on the GPU path as it is.  The cubic box follows from
    the configured site density as in ``Ensemble::compute_bound_box``
    (src/Ensemble.cpp:399-406)."""
    cfg, sysdata, coords = read_config(os.path.join(directory, "config.txt"))
    types, bp, ap, mt, atoms, bonds, angles = read_sysdata(os.path.join(directory, sysdata))
    with open(os.path.join(directory, coords)) as f:
        n = int(f.readline().split()[0])
        pos = np.array([[float(x) for x in f.readline().split()[:3]] for _ in range(n)])
    box = (n / cfg.density) ** (1.0 / 3.0)
    mol_id = atoms[:, 2].astype(np.int32)
    nmol = int(mol_id.max()) + 1
    mol_type = np.zeros(nmol, np.int32)
    mol_type[mol_id] = atoms[:, 3]
    return System(name=name, pos=pos, box=(box, box, box), atom_types=types,
                  atom_type=atoms[:, 1].astype(np.int32), mol_id=mol_id, mol_type_names=mt,
                  mol_type=mol_type, config=cfg, bonds=bonds, angles=angles, bond_params=bp,
                  angle_params=ap)


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


# Tosi-Fumi (1964) Born-Mayer-Huggins parameters for NaCl, converted to
# kJ/mol and nm: phi = A exp(-r/rho) - C r^-6 - D r^-8 with
# A = A_ij b exp((s_i + s_j)/rho), b = 0.338e-19 J, rho = 0.317 A.
_TF_B = 0.338e-19 * 6.02214076e23 / 1000.0
_TF_RHO = 0.0317
_TF_S = {"Na": 0.117, "Cl": 0.1585}
_TF_A = {("Na", "Na"): 1.25, ("Na", "Cl"): 1.00, ("Cl", "Cl"): 0.75}
_TF_C = {("Na", "Na"): 1.68, ("Na", "Cl"): 11.2, ("Cl", "Cl"): 116.0}   # 1e-79 J m^6
_TF_D = {("Na", "Na"): 0.8, ("Na", "Cl"): 13.9, ("Cl", "Cl"): 233.0}    # 1e-99 J m^8


def nacl_bmh_tables():
    names = ["Na", "Cl"]
    A = np.zeros((2, 2)); C = np.zeros((2, 2)); D = np.zeros((2, 2))
    for i, a in enumerate(names):
        for j, b in enumerate(names):
            key = (a, b) if (a, b) in _TF_A else (b, a)
            A[i, j] = _TF_A[key] * _TF_B * math.exp((_TF_S[a] + _TF_S[b]) / _TF_RHO)
            C[i, j] = _TF_C[key] * 6.02214076e-5
            D[i, j] = _TF_D[key] * 6.02214076e-7
    return {"A": A, "rho": np.full((2, 2), _TF_RHO), "C": C, "D": D}


def three_type_fluid(ncell: int = 5, seed: int = 3) -> System:
    """The jittered LJ lattice with its atoms cycled over three types of
    equal parameters (O, C, B): a system for pair potentials whose tables
    are written for three types, such as the reference's SAAP table."""
    s = lj_fluid(ncell=ncell, jitter_star=0.05, seed=seed)
    base = s.atom_types[0]
    s.atom_types = [AtomType(base.mass, 0.0, base.eps, base.sigma, name=nm, long_name=nm) for nm in ("O", "C", "B")]
    s.atom_type = (np.arange(s.n_atoms) % 3).astype(np.int32)
    s.name = f"tri{s.n_atoms}"
    return s


def nacl_melt(ncell: int = 20, density_gcc: float = 1.55, temperature: float = 1200.0,
              seed: int = 1, jitter: float = 0.02, cutoff: float = 1.1, skin: float = 0.1,
              alpha: float = 2.8, kmax: int = 10, potential: str = "bmh",
              dt: float = 0.001, n_steps: int = 1000) -> System:
    """Rock-salt NaCl with ``ncell^3`` ions (ncell even), +-1 e, at the given
    mass density, each ion displaced uniformly by up to ``jitter`` nm from its
    lattice site (seeded).  potential: "bmh" (Tosi-Fumi Born-Mayer-Huggins) or
    "mie" (Mie 14-7 with Joung-Cheatham-like sigma/eps through the LJ table,
    as the reference's MieForce reads it).  Ewald with |n| < kmax."""
    assert ncell % 2 == 0
    n = ncell ** 3
    m_na, m_cl = 22.98977, 35.453
    mass_g = (n // 2) * (m_na + m_cl) / 6.02214076e23
    L = (mass_g / density_gcc) ** (1.0 / 3.0) * 1e7  # cm -> nm
    a = L / ncell
    g = np.stack(np.meshgrid(np.arange(ncell), np.arange(ncell), np.arange(ncell),
                             indexing="ij"), -1).reshape(-1, 3)
    typ = (g.sum(1) % 2).astype(np.int32)   # 0 Na, 1 Cl alternate
    rng = np.random.default_rng(seed)
    pos = (g + 0.5) * a - L / 2 + rng.uniform(-jitter, jitter, (n, 3))
    pos = _wrap(pos, L)
    # |k| cutoff strictly between kmax-1 and kmax shells: n^2 < kmax^2
    kcut = 2 * math.pi * math.sqrt(kmax * kmax - 0.5) / L
    cfg = Config(seed=seed, timestep=dt, n_steps=n_steps, temperature=temperature,
                 coupl_const=0.5, cutoff=cutoff, cutoff_ew=cutoff, cut_buffer=skin,
                 compute_ewald=True, alpha=alpha, k_cutoff=kcut, switch_on=True,
                 switch_dist=cutoff - 0.1, compute_mie=(potential == "mie"), n_mie=14, m_mie=7)
    types = [AtomType(m_na, 1.0, 0.3658, 0.2439, name="Na", long_name="Sodium"),
             AtomType(m_cl, -1.0, 0.1489, 0.4478, name="Cl", long_name="Chloride")]
    s = System(name=f"nacl{n}", pos=pos, box=(L, L, L), atom_types=types, atom_type=typ,
               mol_id=np.arange(n, dtype=np.int32), mol_type_names=[("ION", 1)],
               mol_type=np.zeros(n, np.int32), config=cfg)
    if potential == "bmh":
        s.bmh = nacl_bmh_tables()
    return s


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def _place_waters(nmol, L, r_oh, theta_deg, rng, masses, min_dist=0.2):
    """Molecule centres on a cubic grid (first nmol of g^3 points), random
    orientations (seeded), re-drawn while any site of a molecule comes
    closer than min_dist to a site of an already placed molecule."""
    g = int(math.ceil(nmol ** (1.0 / 3.0) - 1e-9))
    a = L / g
    th = math.radians(theta_deg)
    # H O H in the molecule frame, centre of mass at the origin
    body = np.array([[r_oh * math.sin(th / 2), r_oh * math.cos(th / 2), 0.0],
                     [0.0, 0.0, 0.0],
                     [-r_oh * math.sin(th / 2), r_oh * math.cos(th / 2), 0.0]])
    com = (masses[:, None] * body).sum(0) / masses.sum()
    body -= com
    idx = np.stack(np.meshgrid(np.arange(g), np.arange(g), np.arange(g), indexing="ij"), -1).reshape(-1, 3)
    order = rng.permutation(len(idx))[:nmol]
    cells = idx[np.sort(order)]
    centres = (cells + 0.5) * a - L / 2
    # molecules outside the 27 surrounding grid points sit two or more grid
    # spacings away, so with every site within R of its centre they never
    # come within min_dist: only the placed neighbours are tested
    R = float(np.sqrt((body ** 2).sum(1)).max())
    near = 2.0 * a - 2.0 * R >= min_dist
    owner = {}
    pos = np.zeros((nmol, 3, 3))
    for m in range(nmol):
        if near:
            ci = cells[m]
            prev_ids = [owner[key] for key in
                        {tuple((ci + (dx, dy, dz)) % g) for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)}
                        if key in owner]
        for _ in range(200):
            cand = centres[m] + body @ _random_rotation(rng).T
            if m == 0:
                break
            prev = pos[sorted(prev_ids)].reshape(-1, 3) if near else pos[:m].reshape(-1, 3)
            if len(prev) == 0:
                break
            d = cand[:, None, :] - prev[None, :, :]
            d -= L * np.round(d / L)
            if np.sqrt((d ** 2).sum(-1)).min() >= min_dist:
                break
        pos[m] = cand
        owner[tuple(cells[m])] = m
    return pos.reshape(-1, 3)


def spce_water(nmol: int = 2160, box: float = 4.03, seed: int = 1, temperature: float = 298.0,
               cutoff: float = 1.0, skin: float = 0.1, alpha: float = 3.1, kmax: int = 9,
               dt: float = 0.002, tol: float = 1e-8, n_steps: int = 1000) -> System:
    """Rigid SPC/E-like water: H O H sites (molecule name WAT so the
    reference applies its 3-site SHAKE), q_O = -0.8476 e, r_OH = 0.1 nm,
    HOH = 109.47 deg, LJ on O only (sigma 0.3166 nm, eps 0.650 kJ/mol),
    Ewald with |n| < kmax, SHAKE, Nose-Hoover."""
    rng = np.random.default_rng(seed)
    m_h, m_o = 1.008, 15.9994
    pos = _place_waters(nmol, box, 0.1, 109.47, rng, np.array([m_h, m_o, m_h]))
    pos = _wrap(pos, box)
    n = 3 * nmol
    typ = np.tile(np.array([0, 1, 0], np.int32), nmol)
    mol = np.repeat(np.arange(nmol, dtype=np.int32), 3)
    bonds = np.array([[3 * m + a, 3 * m + b, 0] for m in range(nmol) for a, b in ((0, 1), (1, 2))], np.int32)
    angles = np.array([[3 * m, 3 * m + 1, 3 * m + 2, 0] for m in range(nmol)], np.int32)
    kcut = 2 * math.pi * math.sqrt(kmax * kmax - 0.5) / box
    cfg = Config(seed=seed, timestep=dt, n_steps=n_steps, temperature=temperature, coupl_const=0.5,
                 cutoff=cutoff, cutoff_ew=cutoff, cut_buffer=skin, compute_ewald=True, alpha=alpha,
                 k_cutoff=kcut, switch_on=True, switch_dist=cutoff, constraint=2, tolerance=tol,
                 max_count=1000, long_correct=True)
    types = [AtomType(m_h, 0.4238, 0.0, 0.1, name="H", long_name="Hydrogen"),
             AtomType(m_o, -0.8476, 0.650, 0.3166, name="O", long_name="Oxygen")]
    return System(name=f"spce{nmol}", pos=pos, box=(box, box, box), atom_types=types,
                  atom_type=typ, mol_id=mol, mol_type_names=[("WAT", 3)],
                  mol_type=np.zeros(nmol, np.int32), config=cfg, bonds=bonds, angles=angles,
                  bond_params=[(0, 1, 0.1, 345000.0)], angle_params=[(0, 1, 0, 109.47, 383.0)])


def spce_flexible(nmol: int = 343, box: float = None, seed: int = 1, temperature: float = 298.0,
                  cutoff: float = 0.9, skin: float = 0.1, alpha: float = 3.1, kmax: int = None,
                  dt: float = 0.0005, tau: float = 0.1, strain_rate: float = 0.0,
                  n_steps: int = 1000) -> System:
    """Flexible SPC/E-like water for the chain integrator: the charges, LJ
    and geometry of ``spce_water`` held by harmonic O-H bonds
    (k = 345000 kJ/mol/nm^2) and a harmonic H-O-H angle (383 kJ/mol/rad^2)
    instead of constraints, at the 2160-molecule case's density, |n| < kmax
    (default: 9 scaled with the box), each molecule whole around its centre
    of mass, and SLLOD planar Couette shear at ``strain_rate`` (1/ps)."""
    if box is None:
        box = 4.03 * (nmol / 2160.0) ** (1.0 / 3.0)
    if kmax is None:
        kmax = max(4, int(round(9 * box / 4.03)))
    s = spce_water(nmol=nmol, box=box, seed=seed, temperature=temperature, cutoff=cutoff, skin=skin,
                   alpha=alpha, kmax=kmax, dt=dt, n_steps=n_steps)
    # whole molecules: each H next to its O, then the molecule shifted by
    # the image of its centre of mass
    pos = s.pos.reshape(nmol, 3, 3).copy()
    pos -= box * np.round((pos - pos[:, 1:2, :]) / box)
    mass = np.array([1.008, 15.9994, 1.008])
    com = (pos * mass[None, :, None]).sum(1) / mass.sum()
    pos = pos + (_wrap(com, box) - com)[:, None, :]
    c = s.config
    c.constraint = 0
    c.bend_type = 1
    c.thermostat = "NoseHoover"
    c.coupl_const = tau
    c.long_correct = False
    c.test_mode = 2 if strain_rate else 0
    c.rate = strain_rate
    return s.replace(name=f"spcf{nmol}", pos=pos.reshape(-1, 3))


def polarizable_water(nmol: int = 4096, density_gcc: float = 0.997, seed: int = 1,
                      temperature: float = 298.0, cutoff: float = 0.9, skin: float = 0.1,
                      switch: float = 0.8, alpha: float = 3.5, kmax: int = 20, dt: float = 0.001,
                      tol: float = 1e-8, a_damping: float = 0.39, n_steps: int = 1000) -> System:
    """Rigid polarisable multipole water with the site parameters of the
    reference's shipped test model (charges, local-frame dipoles and
    traceless quadrupoles, isotropic polarisabilities, buffered 14-7 on O and
    H with the H sites pulled towards O by 0.91): H O H sites, molecule name
    WAT, SHAKE on r_OH = 0.09572 nm and HOH = 108.5 deg, Ewald for the
    multipoles with |n| < kmax, Thole-damped induction solved each step."""
    rng = np.random.default_rng(seed)
    m_h, m_o = 1.008, 15.999
    mass_g = nmol * (2 * m_h + m_o) / 6.02214076e23
    box = (mass_g / density_gcc) ** (1.0 / 3.0) * 1e7
    pos = _place_waters(nmol, box, 0.09572, 108.5, rng, np.array([m_h, m_o, m_h]), min_dist=0.18)
    pos = _wrap(pos, box)
    typ = np.tile(np.array([0, 1, 0], np.int32), nmol)
    mol = np.repeat(np.arange(nmol, dtype=np.int32), 3)
    bonds = np.array([[3 * m + a, 3 * m + b, 0] for m in range(nmol) for a, b in ((0, 1), (1, 2))], np.int32)
    angles = np.array([[3 * m, 3 * m + 1, 3 * m + 2, 0] for m in range(nmol)], np.int32)
    kcut = 2 * math.pi * math.sqrt(kmax * kmax - 0.5) / box
    cfg = Config(seed=seed, timestep=dt, n_steps=n_steps, temperature=temperature, coupl_const=0.5,
                 cutoff=cutoff, cutoff_ew=cutoff, cut_buffer=skin, compute_ewald=False,
                 alpha=alpha, k_cutoff=kcut, switch_on=True, switch_dist=switch, constraint=2,
                 tolerance=tol, max_count=1000, long_correct=True, compute_multipole=True,
                 compute_induction=True, compute_torques=True, damp_induction=True,
                 induction_min=True, damp_amoeba=False, cutoff_ind=cutoff, a_damping=a_damping,
                 compute_buff=True, n_buff=14, m_buff=7, delta_buff=0.07, gamma_buff=0.12,
                 h_factor=0.91)
    types = [AtomType(m_h, 0.25983, 0.0565245, 0.2655, dip=(-0.002042095, 0.0, -0.003078753),
                      quad=(-0.0001028545, 0.0, -5.684578967e-06, -0.000300723, 0.0, 0.0004035771),
                      polar=0.000496, name="H", long_name="Hydrogen"),
             AtomType(m_o, -0.51966, 0.46057, 0.3405, dip=(0.0, 0.0, 0.0075561214),
                      quad=(0.0010620922, 0.0, 0.0, -0.00117077124, 0.0, 0.000108679),
                      polar=0.000837, name="O", long_name="Oxygen")]
    return System(name=f"polwater{nmol}", pos=pos, box=(box, box, box), atom_types=types,
                  atom_type=typ, mol_id=mol, mol_type_names=[("WAT", 3)],
                  mol_type=np.zeros(nmol, np.int32), config=cfg, bonds=bonds, angles=angles,
                  bond_params=[(0, 1, 0.09572, 221743.52)], angle_params=[(0, 1, 0, 108.5, 142.56735)])


def constraint_lengths(s: System) -> np.ndarray:
    """Squared constraint lengths per molecule for the cyclic 3-site SHAKE
    (LFIntegrator::initialise, src/integrators/LFIntegrator.cpp:156-167):
    bond 0-1, bond 1-2, and the 0..2 distance from the two bonds and the
    angle (Parameters::get_bond_length(a1,a2,a3), src/Parameters.h:219-226)."""
    (t1, t2, r0, _), = s.bond_params[:1]
    out = np.zeros((s.n_mols, 3))
    theta = s.angle_params[0][3] * 2 * math.pi / 360.0
    l1 = l2 = r0
    l3 = math.sqrt(l1 * l1 + l2 * l2 - 2 * l1 * l2 * math.cos(theta))
    out[:, 0] = l1 * l1
    out[:, 1] = l2 * l2
    out[:, 2] = l3 * l3
    return out


# time unit of the water model's LJ reduced units: sigma_O sqrt(m_water / eps_O) (ps)
WATER_TAU = 0.3166 * math.sqrt(18.0154 / 0.650)


def water_replica_set(count: int = 64, n_min: int = 500, n_max: int = 8000, seed: int = 1,
                      n_steps: int = 5000, flexible: bool = False, rate_max_star: float = 0.2) -> list:
    """Independent SPC/E-like waters (LJ on O + Ewald) for batched runs:
    molecule counts log-uniform in [n_min, n_max], boxes at the density of
    the 2160-molecule case (4.03 nm), |n| < kmax with kmax scaled with the
    box from 9 at 4.03 nm, rc 1.0 nm, one seed each.  Rigid (default): SHAKE
    and the leap-frog Nose-Hoover thermostat at zero shear.  flexible: bonds
    and angle (``spce_flexible``, dt 0.5 fs), each with its own strain rate
    uniform in [0, rate_max_star] reduced units (1 / WATER_TAU) for SLLOD and
    its own Nose-Hoover chain."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        box = 4.03 * (n / 2160.0) ** (1.0 / 3.0)
        kmax = max(5, int(round(9 * box / 4.03)))
        if flexible:
            rate = float(rng.uniform(0.0, rate_max_star)) / WATER_TAU
            out.append(spce_flexible(nmol=n, box=box, cutoff=1.0, kmax=kmax, seed=seed * 1000 + r,
                                     strain_rate=rate, n_steps=n_steps))
        else:
            out.append(spce_water(nmol=n, box=box, cutoff=1.0, kmax=kmax, seed=seed * 1000 + r,
                                  n_steps=n_steps))
    return out


def replica_set(count: int = 64, n_min: int = 500, n_max: int = 8000, rate_max_star: float = 0.2,
                seed: int = 1, n_steps: int = 5000) -> list:
    """Independent Lennard-Jones fluids for batched runs: sizes log-uniform
    in [n_min, n_max] atoms (rounded to the nearest FCC 4 ncell^3, ncell >= 5),
    strain rates uniform in [0, rate_max_star] (reduced units), one seed each."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(count):
        n = math.exp(rng.uniform(math.log(n_min), math.log(n_max)))
        ncell = max(5, int(round((n / 4.0) ** (1.0 / 3.0))))
        rate = float(rng.uniform(0.0, rate_max_star))
        s = lj_fluid(ncell=ncell, seed=seed * 1000 + r, jitter_star=0.02, n_steps=n_steps,
                     strain_rate_star=rate)
        s.config.long_correct = False
        out.append(s)
    return out

"""Host side of the B200 path, mirroring the reference's plugin interface.

``GpuEnsemble`` plays the part of SwinMD's ``Ensemble`` (src/Ensemble.h):
it owns one system's topology, box, pair list and state on the GPU.  The
force classes mirror ``Force`` subclasses (src/Force.h:30-72): ``compute()``
evaluates the term and leaves its energy and virial in the object, and
``compute_long()`` does the reciprocal part where the reference has one.
``LFIntegrator`` mirrors the leap-frog integrator's ``start()``/``run(n)``
(src/integrators/LFIntegrator.cpp).  Every call goes through the C ABI of
``libswinmd_b200.so``; nothing here computes forces or moves atoms.
"""
from __future__ import annotations

import ctypes
import math
from typing import Dict, Optional

import numpy as np

from . import _lib as L
from .systems import BOLTZMAN, System, reference_box


# ---------------------------------------------------------------------------
# reference set-up arithmetic (host, once per run)
# ---------------------------------------------------------------------------

class _RefLCG:
    """``Ensemble::drand`` (src/Ensemble.cpp:1851-1864): 20-bit LCG whose state
    is a function-level static seeded once from the config seed."""

    def __init__(self, seed: float):
        self.s = int(seed) & 0xFFFFFFFF

    def drand(self) -> float:
        self.s = (self.s * 1029 + 221591) % 1048576
        return float(self.s) / 1048576

    def gauss(self) -> float:
        """``Ensemble::gauss`` (src/Ensemble.cpp:1826-1849): sum of 12 uniforms
        mapped through an odd polynomial (Allen & Tildesley's GAUSS)."""
        a1, a3, a5, a7, a9 = 3.949846138, 0.252408784, 0.076542912, 0.008355968, 0.029899776
        s = 0.0
        for _ in range(12):
            s += self.drand()
        r = (s - 6.0) / 4.0
        r2 = r * r
        return ((((a9 * r2 + a7) * r2 + a5) * r2 + a3) * r2 + a1) * r


def init_velocity(s: System) -> np.ndarray:
    """``Ensemble::init_velocity`` (src/Ensemble.cpp:1752-1823): Gaussian
    momenta from the seeded LCG, zero total momentum, scaled to T."""
    c = s.config
    rng = _RefLCG(c.seed)
    nb, na = len(s.bonds), len(s.angles)
    if c.atom_thermo:
        n = s.n_atoms
        ndf = 3 * n - nb - na - 3 if c.constraint else 3 * n - 3
        mass = s.masses()
    else:
        n = s.n_mols
        ndf = 3 * n - 3
        mass = np.zeros(n)
        np.add.at(mass, s.mol_id, s.masses())
    p = np.zeros((n, 3))
    for i in range(n):
        p[i, 0] = rng.gauss()
        p[i, 1] = rng.gauss()
        p[i, 2] = rng.gauss()
    avg = [0.0, 0.0, 0.0]
    for i in range(n):
        for d in range(3):
            avg[d] += p[i, d]
    avg = [a / n for a in avg]
    tavg = 0.0
    for i in range(n):
        for d in range(3):
            p[i, d] -= avg[d]
        x, y, z = p[i]
        tavg += (x * x + y * y + z * z) / mass[i]
    tavg /= (ndf * BOLTZMAN)
    scale = math.sqrt(c.temperature / tavg)
    if c.atom_thermo:
        mom = scale * p
        return mom / mass[:, None]
    v = np.zeros((s.n_atoms, 3))
    for m in range(n):
        vm = (scale * p[m]) / mass[m]
        v[s.mol_id == m] = vm
    return v


def lj_long_range_correction(s: System) -> tuple:
    """``LJForce::long_range_correct`` (src/forces/LJForce.cpp:260-337):
    energy and virial corrections of the dispersion tail."""
    s2, e4 = s.lj_table()
    nt = len(s.atom_types)
    counts = np.bincount(s.atom_type, minlength=nt)
    rc = s.config.cutoff
    vol = reference_box(s) ** 3
    csix, npair, nexcl = 0.0, 0, 0
    for i in range(nt):
        for j in range(i, nt):
            sig6 = s2[i, j] ** 3
            nij = int(counts[i] * counts[j]) if i != j else int(counts[i] * (counts[i] - 1) * 0.5)
            csix += nij * e4[i, j] * sig6
            npair += nij
    excl = s.exclusion_table()
    for i in range(s.n_atoms):
        for j in excl[i]:
            if j >= i:
                sig6 = s2[s.atom_type[i], s.atom_type[j]] ** 3
                csix -= e4[s.atom_type[i], s.atom_type[j]] * sig6
                nexcl += 1
    csix = 0.0 if npair - nexcl <= 0 else csix / (npair - nexcl)
    n = s.n_atoms
    e_lrc = -2.0 * math.pi * n * n * (1.0 / vol) * csix / (3.0 * rc ** 3)
    return e_lrc, -2.0 * e_lrc


def buff_table(s: System) -> np.ndarray:
    """Pair parameters of the buffered 14-7 term as
    ``BuffvdWForce::set_buff_param`` mixes them (src/forces/BuffvdWForce.cpp:
    392-433): cubic-mean sigma, HHG epsilon; pairs with a zero epsilon get
    sigma 1e-7 and epsilon 0.  Returns [nt, nt, 2] = (sigma, eps)."""
    nt = len(s.atom_types)
    out = np.zeros((nt, nt, 2))
    for i, a in enumerate(s.atom_types):
        for j, b in enumerate(s.atom_types):
            if a.eps == 0 or b.eps == 0:
                out[i, j] = (0.0000001, 0.0)
                continue
            si2, sj2 = a.sigma * a.sigma, b.sigma * b.sigma
            es = math.sqrt(a.eps) + math.sqrt(b.eps)
            out[i, j, 0] = (si2 * a.sigma + sj2 * b.sigma) / (si2 + sj2)
            out[i, j, 1] = (4.0 * a.eps * b.eps) / (es * es)
    return out


def buff_taper(rc: float, sd: float) -> np.ndarray:
    """Coefficients c0..c5 of the 5th-order taper in r
    (BuffvdWForce.cpp:60-73)."""
    rc2, sd2 = rc * rc, sd * sd
    off = rc - sd
    den = off ** 5
    return np.array([rc * rc2 * (rc2 - 5.0 * rc * sd + 10.0 * sd2) / den,
                     -30.0 * rc2 * sd2 / den,
                     30.0 * (rc2 * sd + rc * sd2) / den,
                     -10.0 * (rc2 + 4.0 * rc * sd + sd2) / den,
                     15.0 * (rc + sd) / den,
                     -6.0 / den])


def _buff_pot(r, sigma, eps, n, m, delta, gamma):
    """BuffvdWForce::potFunc (BuffvdWForce.cpp:435-463) on an array of r."""
    if eps == 0:
        return np.zeros_like(r), np.zeros_like(r)
    inv = 1.0 / sigma
    rho = r * inv
    rho_m, rho_m1 = rho ** m, rho ** (m - 1.0)
    nm = n - m
    par1 = (1.0 + delta) / (rho + delta)
    par2 = (1.0 + gamma) / (rho_m + gamma)
    p1 = par1 ** nm
    e = eps * p1 * (par2 - 2.0)
    f = -eps * nm * p1 * (par2 - 2.0) * inv / (rho + delta) - eps * p1 * par2 * m * rho_m1 * inv / (rho_m + gamma)
    return e, f


def buff_long_range_correction(s: System, box: float) -> tuple:
    """``BuffvdWForce::long_range_correct`` (BuffvdWForce.cpp:468-601): the
    trapezoid rule with 2^20 intervals of r^2 U(r) and r^3 U'(r) from the
    cutoff to 5000 nm, averaged over type pairs.  Returns (e_lrc, v_lrc)."""
    c = s.config
    tab = buff_table(s)
    nt = len(s.atom_types)
    counts = np.bincount(s.atom_type, minlength=nt)
    rc = c.cutoff
    vol = box ** 3
    level = 20
    h = (5000.0 - rc) / 2.0 ** level
    k = np.arange(1, 2 ** level, dtype=np.float64)
    r_in = rc + k * h
    U = P = 0.0
    npair = 0
    for i in range(nt):
        for j in range(i, nt):
            nij = int(counts[i] * counts[j]) if i != j else int(counts[i] * (counts[i] - 1) * 0.5)
            npair += nij
            sig, eps = tab[i, j]
            e0, f0 = _buff_pot(np.array([rc]), sig, eps, c.n_buff, c.m_buff, c.delta_buff, c.gamma_buff)
            e1, f1 = _buff_pot(np.array([5000.0]), sig, eps, c.n_buff, c.m_buff, c.delta_buff, c.gamma_buff)
            ei, fi = _buff_pot(r_in, sig, eps, c.n_buff, c.m_buff, c.delta_buff, c.gamma_buff)
            sumU = 0.5 * h * rc * rc * e0[0] + float(np.sum(h * r_in * r_in * ei)) + \
                0.5 * h * 5000.0 ** 2 * e1[0]
            sumP = 0.5 * h * rc * rc * rc * f0[0] + float(np.sum(h * r_in * r_in * r_in * fi)) + \
                0.5 * h * 5000.0 ** 3 * f1[0]
            U += nij * sumU
            P += nij * sumP
    if npair <= 0:
        return 0.0, 0.0
    U /= npair
    P /= npair
    N = s.n_atoms
    e_lrc = 2.0 * math.pi * N * N / vol * U
    dU = 2.0 * math.pi * N * N / (vol * vol) * P / 3.0
    return e_lrc, dU * vol


# ---------------------------------------------------------------------------
# the GPU system
# ---------------------------------------------------------------------------

# R_OP / F_Length of WolfForce.h:38, 45, 51 (0.505783 Bohr in nm)
WOLF_R_OP_NM = 0.505783 / (1.0e-9 / 5.29189379e-11)


def lustig_molvirt(fields: dict, volume: float, tb_energy: float = 0.0) -> float:
    """The Lustig virial of LFIntegrator::run (molVirt,
    src/integrators/LFIntegrator.cpp:731-734) from the fields of
    GpuEnsemble.lustig(); the pressure it reports is then
    2 K / 3V - molVirt with K the molecular kinetic energy under
    constraints and the atomic one otherwise (:736-741)."""
    f = fields
    V = volume
    return (f["ljdUlus"] + f["inducDeriv"] - 3.0 * tb_energy / V + f["surfDeriv"] + f["molDeriv"]
            + f["surfPolDeriv"] + f["molPolDeriv"]
            + (f["longDeriv"] + f["realDeriv"] + f["ubDeriv"] + f["BondDeriv"] + f["longPolDeriv"]
               + f["realPolDeriv"] + f["selfPolDeriv"]) / (3.0 * V))


def refuse_unsupported(c) -> None:
    """Raises for configuration options the GPU path does not compute, so a
    caller never gets different physics with a success status: Wolf with
    another electrostatic method."""
    if c.compute_ub and c.constraint:
        # Integrator::initialise refuses the same combination (src/Integrator.cpp:178-187)
        raise NotImplementedError("a flexible Urey-Bradley term with constraints")
    if c.compute_wolf and (c.compute_ewald or c.compute_multipole):
        # the reference stops on more than one electrostatic method
        # (LFIntegrator.cpp:1027, 1058)
        raise NotImplementedError("Wolf together with Ewald or multipoles")


def refuse_unsupported_molecules(s: System) -> None:
    """Raises for molecule kinds whose special cases the GPU path does not
    carry: "MCY" (its O charge moved to a dummy site in Ewald, Multipole and
    Induction, e.g. EwaldForce.cpp:99-125, Multipole.cpp:143-160), "BBV" (its
    own Coulomb damping and SHAKE, Multipole.cpp:639, LFIntegrator::shakeBBV)
    and "CO2" (LFIntegrator::shakeCFR)."""
    names = {nm for nm, _ in s.mol_type_names}
    bad = sorted(names & {"MCY", "BBV", "CO2"})
    if bad:
        raise NotImplementedError(f"molecule kinds {bad} are not built on the GPU path")


class GpuEnsemble:
    """One system on one GPU behind the C ABI (the role of ``Ensemble``)."""

    def __init__(self, system: System, precision: str = "fp64", device: int = 0,
                 threads_per_site: int = 0, velocities: Optional[np.ndarray] = None,
                 box: Optional[float] = None):
        self.lib = L.load()
        self.system = s = system
        self.n = s.n_atoms
        refuse_unsupported(s.config)
        refuse_unsupported_molecules(s)
        ctx = ctypes.c_void_p()
        code = self.lib.smd_create(device, ctypes.byref(ctx))
        if code != L.SMD_OK:
            raise L.SmdError(code, "smd_create failed (no CUDA device?)")
        self.ctx = ctx
        c = s.config
        self.box = box if box is not None else reference_box(s)
        types = np.ascontiguousarray(s.atom_type, np.int32)
        mol = np.ascontiguousarray(s.mol_id, np.int32)
        self.mass = s.masses()
        self.charge = s.scaled_charges()
        self._chk(self.lib.smd_set_topology(ctx, self.n, len(s.atom_types), L.iptr(types),
                                            L.iptr(mol), L.dptr(self.mass), L.dptr(self.charge)))
        excl = s.exclusion_table()
        off = np.zeros(self.n + 1, np.int32)
        off[1:] = np.cumsum([len(e) for e in excl])
        flat = np.array([j for e in excl for j in e] or [0], np.int32)
        self._chk(self.lib.smd_set_exclusions(ctx, L.iptr(off), L.iptr(flat)))
        self._chk(self.lib.smd_set_box(ctx, self.box, self.box, self.box))
        self._chk(self.lib.smd_set_pairlist(ctx, c.cutoff, c.cut_buffer, int(c.use_cell_list)))
        self._setup_vdw()
        if c.compute_ewald:
            self._chk(self.lib.smd_set_ewald(ctx, c.alpha, c.k_cutoff, c.cutoff))
        elif c.compute_wolf:
            # WolfForce: the type-1 site of a "WAT" molecule carries its charge
            # R_OP (in Bohr, WolfForce.h:38) along the bisector
            names = [s.mol_type_names[t][0] for t in s.mol_type]
            msite = np.ascontiguousarray([1 if names[s.mol_id[i]] == "WAT" and s.atom_type[i] == 1 else 0
                                          for i in range(s.n_atoms)], np.int32)
            self._chk(self.lib.smd_set_wolf(ctx, c.alpha, c.cutoff, L.iptr(msite), WOLF_R_OP_NM))
        if c.constraint == 2:
            from .systems import constraint_lengths
            cl = np.ascontiguousarray(constraint_lengths(s).reshape(-1))
            self._chk(self.lib.smd_set_constraints(ctx, L.dptr(cl)))
        if c.compute_buff:
            tab = np.ascontiguousarray(buff_table(s).reshape(-1))
            tap = buff_taper(c.cutoff, c.switch_dist)
            e_lrc, v_lrc = buff_long_range_correction(s, self.box) if c.long_correct else (0.0, 0.0)
            self._chk(self.lib.smd_set_buff(ctx, L.dptr(tab), float(c.n_buff), float(c.m_buff),
                                            c.delta_buff, c.gamma_buff, c.h_factor, int(c.switch_on),
                                            c.switch_dist, L.dptr(tap), e_lrc, v_lrc))
        if c.compute_multipole:
            mp = np.ascontiguousarray([[*t.dip, *t.quad] for t in s.atom_types], np.float64).reshape(-1)
            pol = np.ascontiguousarray([t.polar for t in s.atom_types], np.float64)
            self._chk(self.lib.smd_set_multipole(ctx, L.dptr(mp), L.dptr(pol), c.alpha, c.k_cutoff,
                                                 c.cutoff_ew, int(c.compute_induction), c.cutoff_ind,
                                                 c.a_damping))
            # Config dampAmoeba (Induction.cpp:52): Tinker's damping form
            self._chk(self.lib.smd_set_induction_damping(ctx, int(bool(c.damp_amoeba))))
        # bonded terms of flexible molecules (Integrator::initialise,
        # src/Integrator.cpp:163-190): bonds and angles without constraints,
        # Urey-Bradley when configured
        flexible = c.constraint == 0 and (len(s.bonds) or len(s.angles))
        if flexible or c.compute_ub:
            nb = len(s.bonds) if c.constraint == 0 else 0
            na = len(s.angles) if c.constraint == 0 else 0
            bonds = np.ascontiguousarray(np.asarray(s.bonds, np.int32).reshape(-1, 3)[:nb].reshape(-1)) \
                if nb else np.zeros(3, np.int32)
            angles = np.ascontiguousarray(np.asarray(s.angles, np.int32).reshape(-1, 4)[:na].reshape(-1)) \
                if na else np.zeros(4, np.int32)
            bp = np.ascontiguousarray([[r0, k] for (_, _, r0, k) in s.bond_params] or [[0.0, 0.0]], np.float64)
            ap = np.ascontiguousarray([[deg * 2 * math.pi / 360.0, k] for (_, _, _, deg, k) in s.angle_params]
                                      or [[0.0, 0.0]], np.float64)
            self._chk(self.lib.smd_set_bonded(ctx, nb, L.iptr(bonds), max(1, len(s.bond_params)),
                                              L.dptr(bp.reshape(-1)), na, L.iptr(angles),
                                              max(1, len(s.angle_params)), L.dptr(ap.reshape(-1)),
                                              int(c.bend_type), int(c.compute_ub), c.kl_ub, c.l0_ub))
        if c.surface_correct:
            self._chk(self.lib.smd_set_surface_correct(ctx, 1))
        self.set_precision(precision)
        if threads_per_site:
            self._chk(self.lib.smd_set_tuning(ctx, threads_per_site))
        self.upload_positions(np.asarray(s.pos, np.float64))
        v = velocities if velocities is not None else init_velocity(s)
        self.upload_velocities(v)

    # -- plumbing -------------------------------------------------------
    def _chk(self, code):
        L.check(self.ctx, code)

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.smd_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_reference_forms(self, on: bool):
        """FP64 path: the reference's pow() and per-(site, k) sine forms
        instead of the product form and the column passes."""
        self._chk(self.lib.smd_set_reference_forms(self.ctx, int(bool(on))))

    def lustig_lj(self) -> np.ndarray:
        """(U, dU/dV, d2U/dV2) of the LJ term at the current positions
        (Ensemble::myLustig.ljUlus, ljdUlus, ljd2Ulus)."""
        out = np.zeros(3)
        self._chk(self.lib.smd_lustig_lj(self.ctx, L.dptr(out)))
        return out

    def lustig(self) -> dict:
        """Every field of Ensemble::myLustig at the current configuration
        (FP64), keyed by the reference's field names."""
        out = np.zeros(len(L.LUSTIG_FIELDS))
        self._chk(self.lib.smd_lustig(self.ctx, L.dptr(out)))
        return dict(zip(L.LUSTIG_FIELDS, out.tolist()))

    def set_saap(self, table: np.ndarray, switch_on: bool = False, switch_dist: float = 0.0):
        """The SAAP pair potential as the vdW term (SAAPForce): table rows
        (a0 .. a5) per type pair, ntypes^2 of them."""
        t = np.ascontiguousarray(table, np.float64).reshape(-1)
        nt = len(self.system.atom_types)
        if t.size != 6 * nt * nt:
            raise ValueError(f"set_saap: {nt * nt} rows of 6 parameters expected")
        self._chk(self.lib.smd_set_saap(self.ctx, L.dptr(t), int(switch_on), float(switch_dist) ** 2))

    def set_precision(self, precision: str):
        self.precision = precision
        self._chk(self.lib.smd_set_precision(self.ctx, L.PREC_MIXED if precision == "mixed" else L.PREC_FP64))

    def _setup_vdw(self):
        s, c = self.system, self.system.config
        nt = len(s.atom_types)
        par = np.zeros((nt, nt, 4))
        kind = L.VDW_NONE
        e_lrc = v_lrc = 0.0
        if s.bmh is not None:
            kind = L.VDW_BMH
            par[..., 0] = s.bmh["A"]
            par[..., 1] = 1.0 / s.bmh["rho"]
            par[..., 2] = s.bmh["C"]
            par[..., 3] = s.bmh["D"]
        elif c.compute_mie:
            # MieForce: sigma = sqrt(sigma^2), eps = 4eps/4, Cn (MieForce.cpp:26-35,122-124)
            kind = L.VDW_MIE
            s2, e4 = s.lj_table()
            n_, m_ = float(c.n_mie), float(c.m_mie)
            cn = (n_ / (n_ - m_)) * math.pow(n_ / m_, m_ / (n_ - m_))
            par[..., 0] = np.sqrt(s2)
            par[..., 1] = cn * 0.25 * e4
            par[..., 2] = n_
            par[..., 3] = m_
        elif not c.compute_buff:
            kind = L.VDW_LJ
            s2, e4 = s.lj_table()
            par[..., 0] = s2
            par[..., 1] = e4
            if c.long_correct:
                e_lrc, v_lrc = lj_long_range_correction(s)
        self.vdw_kind = kind
        p = np.ascontiguousarray(par.reshape(-1))
        self._chk(self.lib.smd_set_vdw(self.ctx, kind, L.dptr(p), int(c.switch_on),
                                       c.switch_dist ** 2, e_lrc, v_lrc))

    # -- state ----------------------------------------------------------
    def upload_positions(self, pos: np.ndarray):
        p = np.ascontiguousarray(pos, np.float64).reshape(-1)
        self._chk(self.lib.smd_upload_positions(self.ctx, L.dptr(p)))

    def upload_velocities(self, vel: np.ndarray, vtminus: Optional[np.ndarray] = None):
        v = np.ascontiguousarray(vel, np.float64).reshape(-1)
        vm = None if vtminus is None else np.ascontiguousarray(vtminus, np.float64).reshape(-1)
        self._chk(self.lib.smd_upload_velocities(self.ctx, L.dptr(v), L.dptr(vm)))

    def state(self) -> Dict[str, np.ndarray]:
        pos = np.zeros(3 * self.n); vel = np.zeros(3 * self.n); vtm = np.zeros(3 * self.n)
        self._chk(self.lib.smd_download_state(self.ctx, L.dptr(pos), L.dptr(vel), L.dptr(vtm)))
        return {"pos": pos.reshape(-1, 3), "vel": vel.reshape(-1, 3), "vtminus": vtm.reshape(-1, 3)}

    # -- forces ---------------------------------------------------------
    def real_positions(self) -> np.ndarray:
        """Unwrapped positions (Atom::realPos): the stored positions plus the
        box shifts the integrator applied to each molecule."""
        real = np.zeros(3 * self.n)
        self._chk(self.lib.smd_download_real_positions(self.ctx, L.dptr(real)))
        return real.reshape(self.n, 3)

    def compute_forces(self, terms: int = L.TERM_ALL):
        f = np.zeros(3 * self.n)
        e = np.zeros(L.E_COUNT)
        w = np.zeros(9)
        self._chk(self.lib.smd_compute_forces(self.ctx, terms, L.dptr(f), L.dptr(e), L.dptr(w)))
        return f.reshape(-1, 3), e, w

    def compute_forces_noalloc(self, terms: int = L.TERM_ALL):
        """compute_forces through the entry point that allocates no device
        memory (static scratch of 65536 sites)."""
        f = np.zeros(3 * self.n)
        e = np.zeros(L.E_COUNT)
        w = np.zeros(9)
        self._chk(self.lib.smd_compute_forces_noalloc(self.ctx, terms, L.dptr(f), L.dptr(e), L.dptr(w)))
        return f.reshape(-1, 3), e, w

    def pairs(self) -> np.ndarray:
        cnt = ctypes.c_int64()
        self._chk(self.lib.smd_get_pairs(self.ctx, None, 0, ctypes.byref(cnt)))
        out = np.zeros(2 * cnt.value, np.int32)
        self._chk(self.lib.smd_get_pairs(self.ctx, L.iptr(out), cnt.value, ctypes.byref(cnt)))
        return out.reshape(-1, 2)

    def ewald_nk(self) -> int:
        nk = ctypes.c_int()
        self._chk(self.lib.smd_ewald_nk(self.ctx, ctypes.byref(nk)))
        return nk.value

    def set_solver_pipelined(self, mode: int):
        """Solve with molecule blocks at tolerances >= 1e-9 e nm: the
        pipelined PCG (one grid barrier per iteration) in the mixed path
        (mode 1, the default), in both precisions (2), or never (0: the
        single-reduction form)."""
        self._chk(self.lib.smd_set_solver_pipelined(self.ctx, int(mode)))

    def mlp_set_tensor_path(self, path: int):
        """Network inference and evaluation on tcgen05 128-row tiles (1, the
        default) or warp-level mma.sync tiles (0)."""
        self._chk(self.lib.smd_mlp_set_tensor_path(self.ctx, int(path)))

    def set_solver(self, tol: float = 2.0819e-8, max_iter: int = 500, guess: int = L.GUESS_DIRECT,
                   precond: int = None):
        """Dipole solve settings; precond (L.PRECOND_SITE / L.PRECOND_MOLECULE,
        default molecule blocks) is left unchanged when None."""
        self._chk(self.lib.smd_set_solver(self.ctx, tol, max_iter, guess))
        if precond is not None:
            self._chk(self.lib.smd_set_preconditioner(self.ctx, precond))

    def solver_stats(self):
        it = ctypes.c_int()
        rms = ctypes.c_double()
        self._chk(self.lib.smd_solver_stats(self.ctx, ctypes.byref(it), ctypes.byref(rms)))
        return it.value, rms.value

    def solver_trace(self) -> np.ndarray:
        """RMS dipole change of each iteration of the last solve."""
        out = np.zeros(64)
        cnt = ctypes.c_int()
        self._chk(self.lib.smd_solver_trace(self.ctx, L.dptr(out), 64, ctypes.byref(cnt)))
        return out[:min(cnt.value, 64)]

    def polarization(self):
        n = self.n
        mu, q, e0, p = np.zeros(3 * n), np.zeros(6 * n), np.zeros(3 * n), np.zeros(3 * n)
        self._chk(self.lib.smd_get_polarization(self.ctx, L.dptr(mu), L.dptr(q), L.dptr(e0), L.dptr(p)))
        return {"mu": mu.reshape(-1, 3), "quad": q.reshape(-1, 6), "e0": e0.reshape(-1, 3),
                "p": p.reshape(-1, 3)}

    def set_induced(self, p: np.ndarray):
        pp = np.ascontiguousarray(p, np.float64).reshape(-1)
        self._chk(self.lib.smd_set_induced(self.ctx, L.dptr(pp)))

    # -- observables on the device -------------------------------------------
    def rdf_setup(self, nbins: int):
        """RDF histogram of nbins bins up to the smallest half box edge
        (``RDF``, src/observables/RDF.cpp)."""
        self._chk(self.lib.smd_rdf_setup(self.ctx, int(nbins)))
        self.rdf_nbins = int(nbins)

    def rdf_sample(self):
        """Adds the current configuration (``RDF::sampling``)."""
        self._chk(self.lib.smd_rdf_sample(self.ctx))

    def rdf(self):
        """(r, g, hist, samples): bin centres, the normalised RDF of each
        type pair t1 <= t2 (``RDF::write_result``) and the raw counts."""
        nt = len(self.system.atom_types)
        nb = self.rdf_nbins
        hist = np.zeros(nt * nt * nb, np.uint64)
        g = np.zeros(nt * (nt + 1) // 2 * nb)
        r = np.zeros(nb)
        cnt = ctypes.c_int64()
        self._chk(self.lib.smd_rdf_get(self.ctx, hist.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                       L.dptr(g), L.dptr(r), ctypes.byref(cnt)))
        return r, g.reshape(-1, nb), hist.reshape(nt, nt, nb), cnt.value

    def averages(self) -> L.Averages:
        """Means of the step observables since the integrator start or the
        last reset (``Ensemble::accumulate``)."""
        a = L.Averages()
        self._chk(self.lib.smd_get_averages(self.ctx, ctypes.byref(a)))
        return a

    def reset_averages(self):
        self._chk(self.lib.smd_averages_reset(self.ctx))

    # -- learned initial guess of the induced dipoles ------------------------
    def mlp_init(self, capacity_frames: int, seed: int = 1):
        self._chk(self.lib.smd_mlp_init(self.ctx, capacity_frames, seed))

    def mlp_set_base(self, order: int):
        """Order (1-3) of the extrapolated guess the network corrects."""
        self._chk(self.lib.smd_mlp_set_base(self.ctx, int(order)))

    def mlp_collect(self):
        self._chk(self.lib.smd_mlp_collect(self.ctx))

    def mlp_train(self, epochs: int, batch: int = 4096, lr: float = 1e-3, seed: int = 1) -> float:
        loss = ctypes.c_double()
        self._chk(self.lib.smd_mlp_train(self.ctx, epochs, batch, lr, seed, ctypes.byref(loss)))
        return loss.value

    def mlp_params(self, set_to: Optional[np.ndarray] = None) -> np.ndarray:
        cnt = ctypes.c_int()
        self._chk(self.lib.smd_mlp_params(self.ctx, None, None, ctypes.byref(cnt)))
        out = np.zeros(cnt.value, np.float32)
        s = None if set_to is None else np.ascontiguousarray(set_to, np.float32)
        self._chk(self.lib.smd_mlp_params(self.ctx, L.fptr(out), L.fptr(s), ctypes.byref(cnt)))
        return out

    def mlp_dims(self):
        """(inputs per site, weights) of the network."""
        f, p = ctypes.c_int(), ctypes.c_int()
        self._chk(self.lib.smd_mlp_dims(ctypes.byref(f), ctypes.byref(p)))
        return f.value, p.value

    def mlp_eval(self, feats: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(feats, np.float32)
        if x.ndim != 2 or x.shape[1] != self.mlp_dims()[0]:
            raise ValueError(f"mlp_eval: rows of {self.mlp_dims()[0]} features expected")
        y = np.zeros((x.shape[0], 3), np.float32)
        self._chk(self.lib.smd_mlp_eval(self.ctx, L.fptr(x), x.shape[0], L.fptr(y)))
        return y

    def mlp_gradient(self, rows: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(rows, np.float32)
        nf, npar = self.mlp_dims()
        if r.ndim != 2 or r.shape[1] != nf + 3:
            raise ValueError(f"mlp_gradient: rows of {nf} features and 3 targets expected")
        g = np.zeros(npar, np.float32)
        self._chk(self.lib.smd_mlp_gradient(self.ctx, L.fptr(r), r.shape[0], L.fptr(g)))
        return g

    def mlp_features(self) -> np.ndarray:
        f = np.zeros((self.n, self.mlp_dims()[0]), np.float32)
        self._chk(self.lib.smd_mlp_features(self.ctx, L.fptr(f)))
        return f


# ---------------------------------------------------------------------------
# Force plugin mirrors (Force::compute / compute_long)
# ---------------------------------------------------------------------------

class GpuForce:
    """Base of the force mirrors: after ``compute()`` the object holds
    ``force`` (this term's contribution to Atom::force), ``energy`` and
    ``virial`` (its contribution to Ensemble::virial, row-major 3x3)."""
    terms = 0
    energy_index = L.E_VDW

    def __init__(self, ensemble: GpuEnsemble):
        self.ens = ensemble
        self.force = None
        self.energy = 0.0
        self.energies = None
        self.virial = np.zeros(9)

    def compute(self):
        self.force, self.energies, self.virial = self.ens.compute_forces(self.terms)
        self.energy = float(self.energies[self.energy_index])

    def get_energy(self):
        return self.energy

    def get_virial(self):
        return self.virial.copy()


class LJForce(GpuForce):
    """``LJForce::compute`` (src/forces/LJForce.cpp:58-255); also serves the
    Mie and BMH kinds the ensemble was configured with."""
    terms = L.TERM_VDW
    energy_index = L.E_VDW


class EwaldForce(GpuForce):
    """``EwaldForce::compute`` (real space + self/charged energies,
    src/forces/EwaldForce.cpp:127-172) and ``compute_long`` (reciprocal,
    :174-196)."""
    terms = L.TERM_EWALD_REAL
    energy_index = L.E_REAL

    def compute_long(self):
        f, e, w = self.ens.compute_forces(L.TERM_EWALD_LONG)
        self.long_force, self.long_energy, self.long_virial = f, float(e[L.E_LONG]), w
        return f


# ---------------------------------------------------------------------------
# integrator mirror
# ---------------------------------------------------------------------------

class LFIntegrator:
    """``LFIntegrator`` (src/integrators/LFIntegrator.cpp): ``start()`` is
    LFIntegrator::start (F(0), vtMinus), ``run(n)`` advances n steps."""

    thermostat_kind = None   # set by subclasses; None: from the configuration

    def __init__(self, ensemble: GpuEnsemble, series_capacity: int = 0):
        self.ens = ensemble
        s, c = ensemble.system, ensemble.system.config
        p = L.IntegratorParams()
        p.timestep = c.timestep
        p.temperature = c.temperature
        p.coupl_const = c.coupl_const
        p.thermostat = L.THERMO_NOSE_HOOVER if c.thermostat == "NoseHoover" else L.THERMO_NONE
        if self.thermostat_kind is not None:
            p.thermostat = self.thermostat_kind
        p.atom_thermo = int(c.atom_thermo)
        p.constraint = int(c.constraint)
        p.long_steps = int(c.long_steps)
        p.shake_tol = c.tolerance
        p.shake_max_iter = int(c.max_count)
        # degrees of freedom (Integrator.cpp:22-27)
        p.mol_ndf = 3 * s.n_mols - 3
        p.atom_ndf = 6 * s.n_mols - 3 if c.constraint else 3 * s.n_atoms - 3
        p.strain_rate = c.rate if c.test_mode == 2 else 0.0
        self.params = p
        L.check(ensemble.ctx, ensemble.lib.smd_set_integrator(ensemble.ctx, ctypes.byref(p)))
        if series_capacity:
            L.check(ensemble.ctx, ensemble.lib.smd_set_series_capacity(ensemble.ctx, series_capacity))
        self.series_capacity = series_capacity
        # the NpT ensemble (ensemble 1): the barostat of NHIntegrator; the
        # leap-frog integrator's own NpT branch is not built
        npt = int(c.ensemble) == 1
        if npt and p.thermostat != L.THERMO_NH_CHAIN:
            raise NotImplementedError("NpT runs with the chain integrator (NHIntegrator) only")
        L.check(ensemble.ctx, ensemble.lib.smd_set_barostat(ensemble.ctx, float(c.pressure),
                                                            float(c.baros_const), int(npt)))

    def start(self):
        L.check(self.ens.ctx, self.ens.lib.smd_integrator_start(self.ens.ctx))

    def run(self, nsteps: int):
        L.check(self.ens.ctx, self.ens.lib.smd_run(self.ens.ctx, int(nsteps)))

    def run_timed(self, nsteps: int) -> float:
        """run(n) returning the device time in ms (CUDA events)."""
        ms = ctypes.c_double()
        L.check(self.ens.ctx, self.ens.lib.smd_run_timed(self.ens.ctx, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def observables(self) -> L.Observables:
        o = L.Observables()
        L.check(self.ens.ctx, self.ens.lib.smd_get_observables(self.ens.ctx, ctypes.byref(o)))
        return o

    # -- checkpoint and restart (Integrator::write_state, LFIntegrator::write_vtMinus)
    def write_state(self, path: str, vtminus_path: Optional[str] = None):
        """Writes state.out (positions, real positions, velocities, the
        integrator's scalars and the box) and, when given, vtMinus.out."""
        from . import checkpoint
        e = self.ens
        st = e.state()
        real = e.real_positions()
        scal = np.zeros(32)
        L.check(e.ctx, e.lib.smd_get_integrator_state(e.ctx, L.dptr(scal)))
        step = int(self.observables().step)
        checkpoint.write_state(path, step, st["pos"], real, st["vel"], scal, (e.box, e.box, e.box))
        if vtminus_path:
            checkpoint.write_vtminus(vtminus_path, step, st["vtminus"])

    def restart(self, path: str, vtminus_path: Optional[str] = None):
        """Continues from state.in (and vtMinus.in): the run that does not
        start new (Ensemble::set_configuration, src/Ensemble.cpp:303-317;
        LFIntegrator::read_vtMinus).  Without vtMinus.in the half-step
        velocities are the on-step ones, as the reference takes them."""
        from . import checkpoint
        e = self.ens
        _, pos, real, vel, scal, _ = checkpoint.read_state(path)
        vtm = checkpoint.read_vtminus(vtminus_path) if vtminus_path else None
        e.upload_positions(pos)
        L.check(e.ctx, e.lib.smd_upload_real_positions(e.ctx, L.dptr(np.ascontiguousarray(real.reshape(-1)))))
        e.upload_velocities(vel, vtm)
        L.check(e.ctx, e.lib.smd_integrator_resume(e.ctx))
        if scal is not None:
            L.check(e.ctx, e.lib.smd_set_integrator_state(e.ctx, L.dptr(np.ascontiguousarray(scal))))

    def series(self) -> np.ndarray:
        out = np.zeros(5 * max(self.series_capacity, 1))
        cnt = ctypes.c_int()
        L.check(self.ens.ctx, self.ens.lib.smd_get_series(self.ens.ctx, L.dptr(out),
                                                          self.series_capacity, ctypes.byref(cnt)))
        return out[:5 * cnt.value].reshape(-1, 5)


class NHIntegrator(LFIntegrator):
    """Velocity-Verlet integrator with the 4-link Nose-Hoover chain of
    ``NHIntegrator::chain`` (src/integrators/NHIntegrator.cpp:1814-1912):
    with the isotropic barostat of the reference's NpT run when the
    configuration asks for ensemble 1 (``NHIntegrator::run``, :276-694), at
    constant volume otherwise, and SLLOD planar Couette shear with
    Lees-Edwards images when the configuration asks for it (testMode 2,
    ``rate``).  ``start()`` computes F(0) and the chain's starting kinetic
    energy."""

    thermostat_kind = L.THERMO_NH_CHAIN

    def box(self):
        """Current box edges (nm)."""
        out = np.zeros(3)
        L.check(self.ens.ctx, self.ens.lib.smd_get_box(self.ens.ctx, L.dptr(out)))
        return out

    def barostat_state(self):
        """(vlog, molVirt, volume) after the last step."""
        scal = np.zeros(32)
        L.check(self.ens.ctx, self.ens.lib.smd_get_integrator_state(self.ens.ctx, L.dptr(scal)))
        return float(scal[17]), float(scal[18]), float(scal[21])

    def chain_state(self):
        """The four chain velocities vnh after the last step."""
        scal = np.zeros(32)
        L.check(self.ens.ctx, self.ens.lib.smd_get_integrator_state(self.ens.ctx, L.dptr(scal)))
        return scal[8:12].copy()


class BuffvdWForce(GpuForce):
    """``BuffvdWForce::compute`` (src/forces/BuffvdWForce.cpp:93-343)."""
    terms = L.TERM_VDW
    energy_index = L.E_VDW


class Multipole(GpuForce):
    """``Multipole::compute`` (self + real + intramolecular,
    src/forces/Multipole.cpp:163-205) and ``compute_long`` (:207-222)."""
    terms = L.TERM_MP_SHORT
    energy_index = L.E_REAL

    def compute_long(self):
        f, e, w = self.ens.compute_forces(L.TERM_MP_LONG)
        self.long_force, self.long_energy, self.long_virial = f, float(e[L.E_LONG]), w
        return f


class Induction(GpuForce):
    """``Induction::compute`` (dipole solve, self, real, intramolecular,
    src/forces/Induction.cpp:486-565) and ``compute_long`` (:567-590)."""
    terms = L.TERM_IND_SHORT
    energy_index = L.E_POL_REAL

    def compute_long(self):
        f, e, w = self.ens.compute_forces(L.TERM_IND_LONG)
        self.long_force, self.long_energy, self.long_virial = f, float(e[L.E_POL_LONG]), w
        return f


class WolfForce(GpuForce):
    """``WolfForce::compute`` (src/forces/WolfForce.cpp:100-260): the charges'
    damped, shifted real-space sum (energy into realEnergy)."""
    terms = L.TERM_WOLF
    energy_index = L.E_REAL


class SAAPForce(GpuForce):
    """``SAAPForce::compute`` (src/forces/SAAPForce.cpp:54-230), once the
    ensemble carries a SAAP table (``GpuEnsemble.set_saap``)."""
    terms = L.TERM_VDW
    energy_index = L.E_VDW


class BondForce(GpuForce):
    """``BondForce::compute`` (src/forces/BondForce.cpp:37-110)."""
    terms = L.TERM_BOND
    energy_index = L.E_BOND


class AngleForce(GpuForce):
    """``AngleForce::compute`` (src/forces/AngleForce.cpp:34-130)."""
    terms = L.TERM_ANGLE
    energy_index = L.E_ANGLE


class UreyBradleyForce(GpuForce):
    """``UreyBradleyForce::compute`` (src/forces/UreyBradleyForce.cpp:39-100)."""
    terms = L.TERM_UB
    energy_index = L.E_UB


class ReplicaBatch:
    """Independent replicas (``GpuEnsemble`` objects with their integrators
    started) advanced by one CUDA graph per step (``smd_batch_*``)."""

    def __init__(self, ensembles):
        self.lib = L.load()
        self.ensembles = list(ensembles)
        arr = (ctypes.c_void_p * len(self.ensembles))(*[e.ctx for e in self.ensembles])
        b = ctypes.c_void_p()
        code = self.lib.smd_batch_create(arr, len(self.ensembles), ctypes.byref(b))
        if code != L.SMD_OK:
            raise L.SmdError(code, "smd_batch_create failed")
        self.b = b

    def _chk(self, code):
        if code != L.SMD_OK:
            raise L.SmdError(code, (self.lib.smd_batch_last_error(self.b) or b"").decode())

    def autotune(self, reps: int = 20) -> np.ndarray:
        """Threads per site chosen for each replica's pair kernel."""
        out = np.zeros(len(self.ensembles), np.int32)
        self._chk(self.lib.smd_batch_autotune(self.b, int(reps), L.iptr(out)))
        return out

    def run(self, nsteps: int) -> float:
        """Advances every replica by nsteps; returns the device time (ms)."""
        ms = ctypes.c_double()
        self._chk(self.lib.smd_batch_run(self.b, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def close(self):
        if self.b:
            self.lib.smd_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""ctypes binding of the CPU restatement in oracle/smd_oracle.c.

Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's CPU
baseline call it as the checker; the product never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int32)


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "smd_oracle.c")
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
            subprocess.run(["make", "-C", HERE, "-s", "lib"], check=True)
        _lib = ctypes.CDLL(LIB)
        _lib.or_pairlist.restype = ctypes.c_int64
        _lib.or_pairlist.argtypes = [ctypes.c_int, _D, _D, ctypes.c_double, _I, _I, _I, ctypes.c_int64]
        _lib.or_lj.restype = ctypes.c_double
        _lib.or_lj.argtypes = [ctypes.c_int, _D, _I, _I, _D, ctypes.c_int, _D, _D, ctypes.c_double,
                               ctypes.c_int, ctypes.c_double, ctypes.c_double, _I, ctypes.c_int64, _D, _D]
        _lib.or_lj_md.restype = ctypes.c_int
        _lib.or_lj_md.argtypes = [ctypes.c_int, _D, _D, _D, _D, _I, _I, _D, ctypes.c_int, _D, _D,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_int, _D, _D, _D]
        _lib.or_lj_nhc_md.restype = ctypes.c_int
        _lib.or_lj_nhc_md.argtypes = [ctypes.c_int, _D, _D, _D, _I, _D, ctypes.c_int, _D, _D,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                      _D, _D, _D, _D, _D]
        _lib.or_lj_le_forces.restype = ctypes.c_double
        _lib.or_lj_le_forces.argtypes = [ctypes.c_int, _D, _I, _D, ctypes.c_double, ctypes.c_int, _D, _D,
                                         ctypes.c_double, ctypes.c_int, _D, _D]
        _lib.or_ewald_real.restype = ctypes.c_double
        _lib.or_ewald_real.argtypes = [ctypes.c_int, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                                       _I, ctypes.c_int64, _D, _D]
        _lib.or_ewald_recip.restype = ctypes.c_double
        _lib.or_ewald_recip.argtypes = [ctypes.c_int, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                                        _D, _D, ctypes.POINTER(ctypes.c_int)]
        _lib.or_vdw.restype = ctypes.c_double
        _lib.or_vdw.argtypes = [ctypes.c_int, ctypes.c_int, _D, _I, _I, _D, ctypes.c_int, _D,
                                ctypes.c_double, ctypes.c_int, ctypes.c_double, _I, ctypes.c_int64,
                                _D, _D]
    return _lib


def d(a):
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(_D)


def i32(a):
    return np.ascontiguousarray(a, np.int32).ctypes.data_as(_I)


def _excl_csr(system):
    ex = system.exclusion_table()
    off = np.zeros(system.n_atoms + 1, np.int32)
    off[1:] = np.cumsum([len(e) for e in ex])
    flat = np.array([j for e in ex for j in e] or [0], np.int32)
    return off, flat


def pairlist(system, pos, box):
    c = system.config
    rl = c.cutoff + c.cut_buffer
    L = np.array([box] * 3, np.float64)
    off, flat = _excl_csr(system)
    pos = np.ascontiguousarray(pos, np.float64)
    n = system.n_atoms
    cap = n * 600
    out = np.zeros(2 * cap, np.int32)
    k = lib().or_pairlist(n, d(pos), d(L), rl * rl, i32(off), i32(flat), i32(out), cap)
    assert k <= cap
    return out[:2 * k].reshape(-1, 2)


def lj(system, pos, box, pairs, e_lrc=0.0, v_lrc=0.0):
    s2, e4 = system.lj_table()
    L = np.array([box] * 3, np.float64)
    f = np.zeros(3 * system.n_atoms)
    w = np.zeros(9)
    pairs = np.ascontiguousarray(pairs, np.int32)
    e = lib().or_lj(system.n_atoms, d(pos), i32(system.atom_type), i32(system.mol_id), d(L),
                    len(system.atom_types), d(s2), d(e4), system.config.cutoff,
                    int(system.config.switch_on), e_lrc, v_lrc, i32(pairs), len(pairs),
                    f.ctypes.data_as(_D), w.ctypes.data_as(_D))
    return f.reshape(-1, 3), e, w


def lj_md(system, pos, vel, box, nsteps, e_lrc=0.0, v_lrc=0.0):
    c = system.config
    s2, e4 = system.lj_table()
    L = np.array([box] * 3, np.float64)
    pos = np.array(pos, np.float64).reshape(-1).copy()
    vel = np.array(vel, np.float64).reshape(-1).copy()
    vtm = np.zeros_like(vel)
    ep, tt, zz = np.zeros(nsteps), np.zeros(nsteps), np.zeros(nsteps)
    r = lib().or_lj_md(system.n_atoms, pos.ctypes.data_as(_D), vel.ctypes.data_as(_D),
                       vtm.ctypes.data_as(_D), d(system.masses()), i32(system.atom_type),
                       i32(system.mol_id), d(L), len(system.atom_types), d(s2), d(e4), c.cutoff,
                       c.cut_buffer, int(c.switch_on), e_lrc, v_lrc, c.timestep, c.temperature,
                       c.coupl_const, nsteps, ep.ctypes.data_as(_D), tt.ctypes.data_as(_D),
                       zz.ctypes.data_as(_D))
    assert r == 0, r
    return {"pos": pos.reshape(-1, 3), "vel": vel.reshape(-1, 3), "vtminus": vtm.reshape(-1, 3),
            "epot": ep, "temp": tt, "zeta": zz}


def lj_nhc_md(system, pos, vel, box, nsteps, strain_rate=0.0, ndf=None):
    """Nose-Hoover chain velocity-Verlet MD (optionally SLLOD + Lees-Edwards)
    of a Lennard-Jones system; see or_lj_nhc_md in smd_oracle.c."""
    c = system.config
    s2, e4 = system.lj_table()
    L = np.array(box if np.ndim(box) else [box] * 3, np.float64)
    pos = np.array(pos, np.float64).reshape(-1).copy()
    vel = np.array(vel, np.float64).reshape(-1).copy()
    out = [np.zeros(nsteps) for _ in range(5)]
    ndf = 3 * system.n_atoms - 3 if ndf is None else ndf
    r = lib().or_lj_nhc_md(system.n_atoms, pos.ctypes.data_as(_D), vel.ctypes.data_as(_D),
                           d(system.masses()), i32(system.atom_type), d(L), len(system.atom_types), d(s2),
                           d(e4), c.cutoff, int(c.switch_on), c.timestep, c.temperature, c.coupl_const,
                           strain_rate, ndf, nsteps, *[o.ctypes.data_as(_D) for o in out])
    assert r == 0, r
    return {"pos": pos.reshape(-1, 3), "vel": vel.reshape(-1, 3), "epot": out[0], "temp": out[1],
            "vnh0": out[2], "pxy": out[3], "delta": out[4]}


def lj_le_forces(system, pos, box, delta):
    """LJ forces and energy with Lees-Edwards images at offset delta."""
    c = system.config
    s2, e4 = system.lj_table()
    L = np.array(box if np.ndim(box) else [box] * 3, np.float64)
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
    f = np.zeros(3 * system.n_atoms)
    w = np.zeros(9)
    e = lib().or_lj_le_forces(system.n_atoms, pos.ctypes.data_as(_D), i32(system.atom_type), d(L), delta,
                              len(system.atom_types), d(s2), d(e4), c.cutoff, int(c.switch_on),
                              f.ctypes.data_as(_D), w.ctypes.data_as(_D))
    return f.reshape(-1, 3), e


def ewald(system, pos, box, pairs):
    c = system.config
    L = np.array([box] * 3, np.float64)
    q = system.scaled_charges()
    n = system.n_atoms
    f = np.zeros(3 * n)
    w = np.zeros(9)
    pairs = np.ascontiguousarray(pairs, np.int32)
    er = lib().or_ewald_real(n, d(pos), d(q), d(L), c.alpha, c.cutoff, i32(pairs), len(pairs),
                             f.ctypes.data_as(_D), w.ctypes.data_as(_D))
    fl = np.zeros(3 * n)
    wl = np.zeros(9)
    nk = ctypes.c_int()
    el = lib().or_ewald_recip(n, d(pos), d(q), d(L), c.alpha, c.k_cutoff, fl.ctypes.data_as(_D),
                              wl.ctypes.data_as(_D), ctypes.byref(nk))
    return {"real_force": f.reshape(-1, 3), "real_energy": er, "real_virial": w,
            "long_force": fl.reshape(-1, 3), "long_energy": el, "long_virial": wl, "nk": nk.value}


def vdw_table(system):
    """The per-type-pair table the pair term uses (kind, params[nt, nt, 4])."""
    import math
    c = system.config
    nt = len(system.atom_types)
    par = np.zeros((nt, nt, 4))
    if system.bmh is not None:
        b = system.bmh
        par[..., 0], par[..., 1], par[..., 2], par[..., 3] = b["A"], 1.0 / b["rho"], b["C"], b["D"]
        return 3, par
    s2, e4 = system.lj_table()
    n_, m_ = float(c.n_mie), float(c.m_mie)
    cn = (n_ / (n_ - m_)) * math.pow(n_ / m_, m_ / (n_ - m_))
    par[..., 0], par[..., 1], par[..., 2], par[..., 3] = np.sqrt(s2), cn * 0.25 * e4, n_, m_
    return 2, par


def vdw(system, pos, box, pairs):
    c = system.config
    kind, par = vdw_table(system)
    L = np.array([box] * 3, np.float64)
    n = system.n_atoms
    f = np.zeros(3 * n)
    w = np.zeros(9)
    pairs = np.ascontiguousarray(pairs, np.int32)
    e = lib().or_vdw(kind, n, d(pos), i32(system.atom_type), i32(system.mol_id), d(L),
                     len(system.atom_types), d(par), c.cutoff, int(c.switch_on), c.switch_dist ** 2,
                     i32(pairs), len(pairs), f.ctypes.data_as(_D), w.ctypes.data_as(_D))
    return f.reshape(-1, 3), e, w


def water_md(system, pos, vel, box, nsteps):
    from swinmd_b200.systems import constraint_lengths
    import math
    c = system.config
    lb = lib()
    lb.or_water_md.restype = ctypes.c_int
    lb.or_water_md.argtypes = [ctypes.c_int, _D, _D, _D, _I, _I, _D, _D, ctypes.c_int, _D, _D,
                               ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                               ctypes.c_double, ctypes.c_double, _I, _I, _D, ctypes.c_double,
                               ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                               ctypes.c_int, _D, _D, _D]
    s2, e4 = system.lj_table()
    L = np.array([box] * 3, np.float64)
    q = system.scaled_charges()
    e_self = -float((q * q).sum()) * c.alpha / math.sqrt(math.pi)
    off, flat = _excl_csr(system)
    pos = np.array(pos, np.float64).reshape(-1).copy()
    vel = np.array(vel, np.float64).reshape(-1).copy()
    ep, tt, zz = np.zeros(nsteps), np.zeros(nsteps), np.zeros(nsteps)
    cl = constraint_lengths(system)[0].copy()
    r = lb.or_water_md(system.n_mols, pos.ctypes.data_as(_D), vel.ctypes.data_as(_D),
                       d(system.masses()), i32(system.atom_type), i32(system.mol_id), d(q), d(L),
                       len(system.atom_types), d(s2), d(e4), c.cutoff, c.cut_buffer, int(c.switch_on),
                       c.alpha, c.k_cutoff, e_self, i32(off), i32(flat), d(cl), c.tolerance,
                       int(c.max_count), c.timestep, c.temperature, c.coupl_const, nsteps,
                       ep.ctypes.data_as(_D), tt.ctypes.data_as(_D), zz.ctypes.data_as(_D))
    assert r == 0, r
    return {"pos": pos.reshape(-1, 3), "vel": vel.reshape(-1, 3), "epot": ep, "temp": tt, "zeta": zz}


def _bonded_tables(system):
    """bonds [nb][3], (r0, k) per bond type; angles [na][4], (t0 rad, k) per type."""
    import math
    bonds = np.ascontiguousarray(system.bonds, np.int32).reshape(-1, 3)
    angles = np.ascontiguousarray(system.angles, np.int32).reshape(-1, 4)
    bpar = np.array([[r0, k] for (_, _, r0, k) in system.bond_params] or [[0.0, 0.0]], np.float64)
    apar = np.array([[math.radians(t0), k] for (_, _, _, t0, k) in system.angle_params] or [[0.0, 0.0]],
                    np.float64)
    return bonds, bpar, angles, apar


def _flex_args(system, box):
    c = system.config
    s2, e4 = system.lj_table()
    L = np.array(box if np.ndim(box) else [box] * 3, np.float64)
    q = system.scaled_charges()
    off, flat = _excl_csr(system)
    bonds, bpar, angles, apar = _bonded_tables(system)
    ns = system.mol_type_names[0][1]
    return c, s2, e4, L, q, off, flat, bonds, bpar, angles, apar, ns


def flex_le_forces(system, pos, box, delta):
    """Forces, per-term energies and virial of a flexible point-charge model
    (LJ, Ewald real / sheared reciprocal / intramolecular, bonds, angles)
    with Lees-Edwards images at offset delta; see or_flex_le_forces."""
    lb = lib()
    lb.or_flex_le_forces.restype = None
    lb.or_flex_le_forces.argtypes = [ctypes.c_int, ctypes.c_int, _D, _I, _I, _D, _D, ctypes.c_double,
                                     ctypes.c_int, _D, _D, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, _I, _I, ctypes.c_int, _I, _D, ctypes.c_int, _I, _D,
                                     _D, _D, _D]
    c, s2, e4, L, q, off, flat, bonds, bpar, angles, apar, ns = _flex_args(system, box)
    n = system.n_atoms
    f = np.zeros(3 * n)
    w = np.zeros(9)
    e = np.zeros(7)
    lb.or_flex_le_forces(n, ns, d(pos), i32(system.atom_type), i32(system.mol_id), d(q), d(L), float(delta),
                         len(system.atom_types), d(s2), d(e4), c.cutoff, int(c.switch_on), c.alpha, c.k_cutoff,
                         i32(off), i32(flat), len(bonds), i32(bonds), d(bpar), len(angles), i32(angles), d(apar),
                         f.ctypes.data_as(_D), w.ctypes.data_as(_D), e.ctypes.data_as(_D))
    return {"force": f.reshape(-1, 3), "virial": w, "vdw": e[0], "real": e[1], "long": e[2], "intra": e[3],
            "bond": e[4], "angle": e[5], "nk": int(e[6])}


def ewald_recip_le(system, pos, box, delta, alpha=None, kcut=None):
    """Reciprocal Ewald energy, forces and long virial in the sheared cell."""
    lb = lib()
    lb.or_ewald_recip_le.restype = ctypes.c_double
    lb.or_ewald_recip_le.argtypes = [ctypes.c_int, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, _D, _D, ctypes.POINTER(ctypes.c_int)]
    c = system.config
    L = np.array(box if np.ndim(box) else [box] * 3, np.float64)
    n = system.n_atoms
    f = np.zeros(3 * n)
    w = np.zeros(9)
    nk = ctypes.c_int()
    e = lb.or_ewald_recip_le(n, d(pos), d(system.scaled_charges()), d(L), float(delta),
                             c.alpha if alpha is None else alpha, c.k_cutoff if kcut is None else kcut,
                             f.ctypes.data_as(_D), w.ctypes.data_as(_D), ctypes.byref(nk))
    return {"energy": e, "force": f.reshape(-1, 3), "virial": w, "nk": nk.value}


def ewald_real_le(system, pos, box, delta, alpha=None, rc=None):
    lb = lib()
    lb.or_ewald_real_le.restype = ctypes.c_double
    lb.or_ewald_real_le.argtypes = [ctypes.c_int, _D, _D, _I, _D, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, _D, _D]
    c = system.config
    L = np.array(box if np.ndim(box) else [box] * 3, np.float64)
    n = system.n_atoms
    f = np.zeros(3 * n)
    w = np.zeros(9)
    e = lb.or_ewald_real_le(n, d(pos), d(system.scaled_charges()), i32(system.mol_id), d(L), float(delta),
                            c.alpha if alpha is None else alpha, c.cutoff if rc is None else rc,
                            f.ctypes.data_as(_D), w.ctypes.data_as(_D))
    return {"energy": e, "force": f.reshape(-1, 3), "virial": w}


def flex_nhc_md(system, pos, vel, box, nsteps, strain_rate=0.0, ndf=None):
    """Chain / SLLOD velocity-Verlet MD of a flexible point-charge model with
    molecules wrapped by their centres; see or_flex_nhc_md."""
    lb = lib()
    lb.or_flex_nhc_md.restype = ctypes.c_int
    lb.or_flex_nhc_md.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, _I, _I, _D, _D, ctypes.c_int, _D, _D,
                                  ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double, _I, _I,
                                  ctypes.c_int, _I, _D, ctypes.c_int, _I, _D, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D]
    c, s2, e4, L, q, off, flat, bonds, bpar, angles, apar, ns = _flex_args(system, box)
    n = system.n_atoms
    pos = np.array(pos, np.float64).reshape(-1).copy()
    vel = np.array(vel, np.float64).reshape(-1).copy()
    out = [np.zeros(nsteps) for _ in range(5)]
    ndf = 3 * n - 3 if ndf is None else ndf
    r = lb.or_flex_nhc_md(n, ns, pos.ctypes.data_as(_D), vel.ctypes.data_as(_D), d(system.masses()),
                          i32(system.atom_type), i32(system.mol_id), d(q), d(L), len(system.atom_types), d(s2),
                          d(e4), c.cutoff, int(c.switch_on), c.alpha, c.k_cutoff, i32(off), i32(flat),
                          len(bonds), i32(bonds), d(bpar), len(angles), i32(angles), d(apar), c.timestep,
                          c.temperature, c.coupl_const, strain_rate, ndf, nsteps,
                          *[o.ctypes.data_as(_D) for o in out])
    assert r == 0, r
    return {"pos": pos.reshape(-1, 3), "vel": vel.reshape(-1, 3), "epot": out[0], "temp": out[1],
            "vnh0": out[2], "pxy": out[3], "delta": out[4]}

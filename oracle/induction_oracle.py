"""Restatement of the reference's polarisable multipole model: lab-frame
multipoles, the multipole Ewald real-space energy, and the induced-dipole
system (permanent field and dense matrix).  Test infrastructure: only
tests/ use it, as the checker.

Induction::compute builds A p = E0 over all 3N dipole components
(src/forces/Induction.cpp):

* diagonal 3 x 3 blocks 1 / max(polmin, alpha_i) I, polmin = 1e-8
  (:193, :218-256);
* for every pair i < j whose minimum-image distance is within cutoffInd
  (:258-292), intramolecular pairs included (the exclusion test at :371
  only guards the permanent-field terms), the off-diagonal blocks
  A_ij = A_ji = -T_ij with the Thole-damped dipole tensor (:295-343)
      u^3 = r^3 / sqrt(alpha_i alpha_j),  e = exp(-a u^3),
      l3 = 1 - e,  l5 = 1 - (1 + a u^3) e,
      T_ij = 3 l5 r r^T / r^5 - l3 I / r^3   (r = r_i - r_j);
  the undamped tensor when damping is off.

The reference solves it by unpreconditioned CG; here numpy's dense solve
gives the exact solution of the same system.
"""
import numpy as np

POLMIN = 1e-8


def min_image(d, box):
    return d - box * np.round(d / box)


def induction_matrix(pos, polar, box, a, cutoff, damp=True):
    """A (3N x 3N) for sites at pos (N x 3, nm), polarisabilities polar (N,
    nm^3), orthorhombic box (3,), Thole parameter a and cutoffInd (nm)."""
    pos = np.asarray(pos, np.float64)
    box = np.asarray(box, np.float64)
    n = len(pos)
    al = np.maximum(POLMIN, np.asarray(polar, np.float64))
    A = np.zeros((3 * n, 3 * n))
    for i in range(n):
        A[3 * i:3 * i + 3, 3 * i:3 * i + 3] = np.eye(3) / al[i]
        if i + 1 == n:
            continue
        j = np.arange(i + 1, n)
        r = min_image(pos[i] - pos[j], box)
        r2 = np.einsum("ij,ij->i", r, r)
        keep = r2 <= cutoff * cutoff
        j, r, r2 = j[keep], r[keep], r2[keep]
        rr = np.sqrt(r2)
        r_3 = 1.0 / (r2 * rr)
        r_5 = r_3 / r2
        if damp:
            u3 = r2 * rr / np.sqrt(al[i] * al[j])
            e = np.exp(-a * u3)
            l3 = 1.0 - e
            l5 = 1.0 - (1.0 + a * u3) * e
        else:
            l3 = np.ones_like(rr)
            l5 = np.ones_like(rr)
        T = (3.0 * (l5 * r_5))[:, None, None] * r[:, :, None] * r[:, None, :]
        T -= (l3 * r_3)[:, None, None] * np.eye(3)[None]
        for k, jj in enumerate(j):
            A[3 * i:3 * i + 3, 3 * jj:3 * jj + 3] = -T[k]
            A[3 * jj:3 * jj + 3, 3 * i:3 * i + 3] = -T[k]
    return A


def lab_multipoles(pos, mol_id, dip_local, quad_local):
    """Lab-frame dipoles (N x 3) and quadrupoles (N x 6, xx xy xz yy yz zz)
    of H O H molecules (sites in that order within each molecule), from
    each site's local-frame values (Local2Global::FrameofReference,
    src/utils/Local2Global.cpp): an H site takes w along O - H and the lab x
    axis (lab y when |w.x| > 0.866) as its second vector; O takes w along
    the sum of the unit O->H vectors and the unit O->H2 vector; then
    u = s - (s.w) w normalised, v = w x u, mu = [u v w] mu_local and
    Q = [u v w] Q_local [u v w]^T / 3.  Positions are used as given (whole
    molecules), as the reference does."""
    pos = np.asarray(pos, np.float64)
    mol = np.asarray(mol_id)
    dl = np.asarray(dip_local, np.float64).reshape(-1, 3)
    QL = quad_matrix(quad_local)
    n = len(pos)
    mu = np.zeros((n, 3))
    Q6 = np.zeros((n, 6))

    def unit(v):
        return v / np.linalg.norm(v)

    for m in np.unique(mol):
        h1, o, h2 = np.flatnonzero(mol == m)
        p1 = [pos[o] - pos[h1], unit(pos[h1] - pos[o]) + unit(pos[h2] - pos[o]), pos[o] - pos[h2]]
        ex, ey = np.array([1.0, 0.0, 0.0]), np.array([0.0, 1.0, 0.0])
        p2 = [ey if abs(p1[0][0] / np.linalg.norm(p1[0])) > 0.8660 else ex, unit(pos[h2] - pos[o]),
              ey if abs(p1[2][0] / np.linalg.norm(p1[2])) > 0.8660 else ex]
        for k, i in enumerate((h1, o, h2)):
            w = unit(p1[k])
            ss = p2[k] - (p2[k] @ w) * w
            u = unit(ss)
            v = np.cross(w, u)
            R = np.stack([u, v, w], axis=1)
            mu[i] = R @ dl[i]
            G = R @ QL[i] @ R.T / 3.0
            Q6[i] = [G[0, 0], G[0, 1], G[0, 2], G[1, 1], G[1, 2], G[2, 2]]
    return mu, Q6


def quad_matrix(q6):
    """3 x 3 quadrupoles from the six components xx xy xz yy yz zz (N x 6)."""
    q6 = np.asarray(q6, np.float64).reshape(-1, 6)
    Q = np.empty((len(q6), 3, 3))
    for (r, c), k in {(0, 0): 0, (0, 1): 1, (0, 2): 2, (1, 1): 3, (1, 2): 4, (2, 2): 5}.items():
        Q[:, r, c] = q6[:, k]
        Q[:, c, r] = q6[:, k]
    return Q


def permanent_field(pos, q, dip, quad, polar, box, a, cutoff, mol_id):
    """E0 (N x 3): the Thole-damped field of the other molecules' charges,
    dipoles and quadrupoles (lab frame) at every site, pairs within
    cutoffInd, sites of one molecule excluded from each other
    (Induction.cpp:371-431, the b_i / b_j terms):
        b_i = q_j l3 r / r^3 + 3 l5 r (r.mu_j) / r^5 - l3 mu_j / r^3
              + 15 l7 (r.Q_j.r) r / r^7 - 6 l5 Q_j r / r^5 - 3 l5 tr(Q_j) r / r^5
    with r = r_i - r_j, b_j the same with i, j swapped (r -> -r) and
    l7 = 1 - (1 + a u^3 + 3 (a u^3)^2 / 5) e."""
    pos = np.asarray(pos, np.float64)
    box = np.asarray(box, np.float64)
    q = np.asarray(q, np.float64)
    mu = np.asarray(dip, np.float64).reshape(-1, 3)
    Q = quad_matrix(quad)
    mol = np.asarray(mol_id)
    n = len(pos)
    al = np.maximum(POLMIN, np.asarray(polar, np.float64))
    E = np.zeros((n, 3))
    trQ = np.trace(Q, axis1=1, axis2=2)
    for i in range(n - 1):
        j = np.arange(i + 1, n)
        r = min_image(pos[i] - pos[j], box)
        r2 = np.einsum("ij,ij->i", r, r)
        keep = (r2 <= cutoff * cutoff) & (mol[j] != mol[i])
        j, r, r2 = j[keep], r[keep], r2[keep]
        if len(j) == 0:
            continue
        rr = np.sqrt(r2)
        r_3 = 1.0 / (r2 * rr)
        r_5 = r_3 / r2
        r_7 = r_5 / r2
        au3 = a * r2 * rr / np.sqrt(al[i] * al[j])
        e = np.exp(-au3)
        l3 = 1.0 - e
        l5 = 1.0 - (1.0 + au3) * e
        l7 = 1.0 - (1.0 + au3 + 0.6 * au3 * au3) * e
        Qj_r = np.einsum("kab,kb->ka", Q[j], r)
        Qi_r = Q[i] @ r.T
        rQjr = np.einsum("ka,ka->k", r, Qj_r)
        rQir = np.einsum("ka,ak->k", r, Qi_r)
        r_muj = np.einsum("ka,ka->k", r, mu[j])
        r_mui = r @ mu[i]
        bi = ((q[j] * l3 * r_3)[:, None] * r + (3.0 * l5 * r_5 * r_muj)[:, None] * r
              - (l3 * r_3)[:, None] * mu[j] + (15.0 * l7 * r_7 * rQjr)[:, None] * r
              - (6.0 * l5 * r_5)[:, None] * Qj_r - (3.0 * l5 * r_5 * trQ[j])[:, None] * r)
        bj = (-(q[i] * l3 * r_3)[:, None] * r + (3.0 * l5 * r_5 * r_mui)[:, None] * r
              - (l3 * r_3)[:, None] * mu[i] - (15.0 * l7 * r_7 * rQir)[:, None] * r
              + (6.0 * l5 * r_5)[:, None] * Qi_r.T + (3.0 * l5 * r_5 * trQ[i])[:, None] * r)
        E[i] += bi.sum(axis=0)
        np.add.at(E, j, bj)
    return E


COULOMBS = 138.93548501   # 1 / (4 pi eps0) in kJ mol^-1 nm e^-2 (src/NEMD_defs.h:104)


def multipole_real_energy(pos, q, dip, quad, box, alpha, cutoff, mol_id):
    """Ewald real-space energy of charges, dipoles and quadrupoles
    (Multipole::compute, src/forces/Multipole.cpp:540-653): for every pair of
    sites of different molecules within the real-space cutoff,
    COULOMBS * sum_n G_n B_n with r = r_i - r_j,
        B_0 = erfc(alpha r) / r,
        B_n = ((2n - 1) B_{n-1} + (2 alpha^2)^n e^{-alpha^2 r^2} / (alpha sqrt(pi))) / r^2
              (with the reference's signs: B1 = (-B0 - c e)/r^2, B2 = (-3 B1 + 2 c a^2 e)/r^2, ...)
        G_0 = q_i q_j
        G_1 = q_j mu_i.r - q_i mu_j.r - mu_i.mu_j + q_j tr Q_i + q_i tr Q_j
        G_2 = q_j r.Q_i.r + q_i r.Q_j.r - (mu_i.r)(mu_j.r) - (mu_j.r) tr Q_i + (mu_i.r) tr Q_j
              - 2 mu_j.Q_i r + 2 mu_i.Q_j r + tr Q_i tr Q_j + 2 Q_i:Q_j
        G_3 = (mu_i.r) r.Q_j.r - (mu_j.r) r.Q_i.r + tr Q_i r.Q_j.r + tr Q_j r.Q_i.r
              + 4 (Q_i r).(Q_j r)
        G_4 = (r.Q_i.r)(r.Q_j.r)."""
    from scipy.special import erfc
    pos = np.asarray(pos, np.float64)
    box = np.asarray(box, np.float64)
    q = np.asarray(q, np.float64)
    mu = np.asarray(dip, np.float64).reshape(-1, 3)
    Q = quad_matrix(quad)
    trQ = np.trace(Q, axis1=1, axis2=2)
    mol = np.asarray(mol_id)
    n = len(pos)
    a2 = alpha * alpha
    c = 2.0 * alpha / np.sqrt(np.pi)
    energy = 0.0
    for i in range(n - 1):
        j = np.arange(i + 1, n)
        r = min_image(pos[i] - pos[j], box)
        r2 = np.einsum("ij,ij->i", r, r)
        keep = (r2 < cutoff * cutoff) & (mol[j] != mol[i])
        j, r, r2 = j[keep], r[keep], r2[keep]
        if len(j) == 0:
            continue
        rr = np.sqrt(r2)
        ex = np.exp(-a2 * r2)
        B0 = erfc(alpha * rr) / rr
        B1 = (-B0 - c * ex) / r2
        B2 = (-3 * B1 + 2 * c * a2 * ex) / r2
        B3 = (-5 * B2 - 4 * c * a2 * a2 * ex) / r2
        B4 = (-7 * B3 + 8 * c * a2 * a2 * a2 * ex) / r2
        G0, G1, G2, G3, G4 = _pair_invariants(q, mu, Q, trQ, i, j, r)
        energy += float(np.sum(G0 * B0 + G1 * B1 + G2 * B2 + G3 * B3 + G4 * B4))
    return energy * COULOMBS


def multipole_recip_energy(pos, q, dip, quad, box, alpha, kcut):
    """Ewald reciprocal energy of charges, dipoles and quadrupoles
    (Multipole::reciprocal_term, src/forces/Multipole.cpp:245-293 for the k
    half-space, :1054-1131 for the sums):
        k = 2 pi (nx / Lx, ny / Ly, nz / Lz), nx >= 0, k^2 < kcut^2, one of each +-k pair,
        C = sum_i (q_i - k.Q_i.k) cos(k.r_i),  S = sum_i (q_i - k.Q_i.k) sin(k.r_i),
        M_c = sum_i (mu_i.k) cos(k.r_i),       M_s = sum_i (mu_i.k) sin(k.r_i),
        E = COULOMBS (4 pi / V) sum_k e^{-k^2 / (4 alpha^2)} / k^2
            (C^2 + S^2 + 2 (S M_c - C M_s) + M_c^2 + M_s^2)."""
    pos = np.asarray(pos, np.float64)
    box = np.asarray(box, np.float64)
    q = np.asarray(q, np.float64)
    mu = np.asarray(dip, np.float64).reshape(-1, 3)
    Q = quad_matrix(quad)
    C, S, Mc, Ms, Pc, Ps, coef = _recip_sums(pos, q, mu, Q, None, box, alpha, kcut)
    return float(np.sum(coef * (C * C + S * S + 2 * (S * Mc - C * Ms) + Mc * Mc + Ms * Ms))) * COULOMBS


def _recip_sums(pos, q, mu, Q, p, box, alpha, kcut):
    """Structure sums over the reference's k half-space (see
    multipole_recip_energy) and the coefficients 4 pi / V e^{-k^2/(4 alpha^2)} / k^2;
    Pc, Ps are those of the dipoles p (None: zeros)."""
    nmax = [int(kcut * L / (2 * np.pi)) for L in box]
    v = 2 * np.pi / box
    ks = []
    for nx in range(0, nmax[0] + 1):
        for ny in range(0 if nx == 0 else -nmax[1], nmax[1] + 1):
            for nz in range(1 if nx == 0 and ny == 0 else -nmax[2], nmax[2] + 1):
                k = np.array([nx, ny, nz]) * v
                if k @ k < kcut * kcut:
                    ks.append(k)
    ks = np.array(ks)
    k2 = np.einsum("ka,ka->k", ks, ks)
    ph = pos @ ks.T                                    # N x K
    w = q[:, None] - np.einsum("ka,iab,kb->ik", ks, Q, ks)
    m = mu @ ks.T
    cs, sn = np.cos(ph), np.sin(ph)
    C, S = (w * cs).sum(0), (w * sn).sum(0)
    Mc, Ms = (m * cs).sum(0), (m * sn).sum(0)
    if p is None:
        Pc = Ps = np.zeros_like(C)
    else:
        pk = np.asarray(p, np.float64).reshape(-1, 3) @ ks.T
        Pc, Ps = (pk * cs).sum(0), (pk * sn).sum(0)
    coef = 4 * np.pi / np.prod(box) * np.exp(-k2 / (4 * alpha * alpha)) / k2
    return C, S, Mc, Ms, Pc, Ps, coef


def induced_recip_energy(pos, q, dip, quad, p, box, alpha, kcut):
    """The reference's longPolEnergy: the reciprocal energy between the
    induced dipoles and the permanent multipoles,
        COULOMBS sum_k coef_k [(S P_c - C P_s) + (P_c M_c + P_s M_s)]
    with the sums of multipole_recip_energy and P_c, P_s those of p.k."""
    pos = np.asarray(pos, np.float64)
    box = np.asarray(box, np.float64)
    C, S, Mc, Ms, Pc, Ps, coef = _recip_sums(pos, np.asarray(q, np.float64),
                                             np.asarray(dip, np.float64).reshape(-1, 3), quad_matrix(quad), p,
                                             box, alpha, kcut)
    return float(np.sum(coef * ((S * Pc - C * Ps) + (Pc * Mc + Ps * Ms)))) * COULOMBS


def _pair_invariants(q, mu, Q, trQ, i, j, r):
    """G_0..G_4 of site i with sites j (arrays), r = r_i - r_j (the same
    invariants as in multipole_real_energy)."""
    Qi_r = (Q[i] @ r.T).T
    Qj_r = np.einsum("kab,kb->ka", Q[j], r)
    rQir = np.einsum("ka,ka->k", r, Qi_r)
    rQjr = np.einsum("ka,ka->k", r, Qj_r)
    mir = r @ mu[i]
    mjr = np.einsum("ka,ka->k", r, mu[j])
    G0 = q[i] * q[j]
    G1 = q[j] * mir - q[i] * mjr - mu[j] @ mu[i] + q[j] * trQ[i] + q[i] * trQ[j]
    G2 = (q[j] * rQir + q[i] * rQjr - mir * mjr - mjr * trQ[i] + mir * trQ[j]
          - 2 * np.einsum("ka,ka->k", mu[j], Qi_r) + 2 * (Qj_r @ mu[i]) + trQ[i] * trQ[j]
          + 2 * np.einsum("ab,kab->k", Q[i], Q[j]))
    G3 = mir * rQjr - mjr * rQir + trQ[i] * rQjr + trQ[j] * rQir + 4 * np.einsum("ka,ka->k", Qi_r, Qj_r)
    G4 = rQir * rQjr
    return G0, G1, G2, G3, G4


def multipole_correct_energies(pos, q, dip, quad, box, alpha, mol_id):
    """The reference's correctEnergy and molCorrectEnergy of the multipoles
    (Multipole::self_correct, src/forces/Multipole.cpp:338-386, the net
    charge term at :104, and the intramolecular correction set at :1689):
        self = -1/2 COULOMBS sum_i [q^2 c + (mu.mu - 2 q tr Q) 2 c alpha^2 / 3
                                    + ((tr Q)^2 + 2 Q:Q) 4 c alpha^4 / 5],  c = 2 alpha / sqrt(pi)
        charged = -pi (sum q)^2 / (2 V alpha^2)
        intra = -COULOMBS sum over site pairs of one molecule of sum_n G_n D_n
    with D_0 = erf(alpha r) / r and the upward recursion of the B_n with the
    signs of erf (D_1 = (-D_0 + c e^{-alpha^2 r^2}) / r^2, ...)."""
    from scipy.special import erf
    pos = np.asarray(pos, np.float64)
    box = np.asarray(box, np.float64)
    q = np.asarray(q, np.float64)
    mu = np.asarray(dip, np.float64).reshape(-1, 3)
    Q = quad_matrix(quad)
    trQ = np.trace(Q, axis1=1, axis2=2)
    QQ = np.einsum("iab,iab->i", Q, Q)
    a2 = alpha * alpha
    c = 2.0 * alpha / np.sqrt(np.pi)
    selfterm = (q * q * c + (np.einsum("ia,ia->i", mu, mu) - 2 * q * trQ) * 2 * c * a2 / 3
                + (trQ * trQ + 2 * QQ) * 4 * c * a2 * a2 / 5)
    e_self = float(np.sum(-0.5 * selfterm * COULOMBS))
    e_charged = -np.pi * q.sum() ** 2 / (2.0 * np.prod(box) * a2)
    mol = np.asarray(mol_id)
    intra = 0.0
    for m in np.unique(mol):
        sites = np.flatnonzero(mol == m)
        for k, i in enumerate(sites[:-1]):
            j = sites[k + 1:]
            r = min_image(pos[i] - pos[j], box)
            r2 = np.einsum("ka,ka->k", r, r)
            rr = np.sqrt(r2)
            ex = np.exp(-a2 * r2)
            D0 = erf(alpha * rr) / rr
            D1 = (-D0 + c * ex) / r2
            D2 = (-3 * D1 - 2 * c * a2 * ex) / r2
            D3 = (-5 * D2 + 4 * c * a2 * a2 * ex) / r2
            D4 = (-7 * D3 - 8 * c * a2 * a2 * a2 * ex) / r2
            G0, G1, G2, G3, G4 = _pair_invariants(q, mu, Q, trQ, i, j, r)
            intra += float(np.sum(G0 * D0 + G1 * D1 + G2 * D2 + G3 * D3 + G4 * D4))
    return e_self + e_charged, -intra * COULOMBS


def induced_correct_energies(pos, q, dip, quad, p, box, alpha, mol_id):
    """The reference's correctPolEnergy and molCorrectPolEnergy: the induced
    dipoles' Ewald self term -COULOMBS sum_i (mu_i.p_i) c alpha^2 / 3 and the
    intramolecular correction -1/2 COULOMBS sum over site pairs of one
    molecule of (G1_i + G1_j) D_1 + (G2_i + G2_j) D_2 + (G3_i + G3_j) D_3,
    with the permanent-induced invariants (r = r_i - r_j)
        G1_i = -q_i p_j.r - mu_i.p_j
        G2_i = -(mu_i.r)(p_j.r) - 2 p_j.Q_i r - (p_j.r) tr Q_i
        G3_i = -(p_j.r)(r.Q_i.r)
    and G*_j the same with i, j swapped (r -> -r), D_n as in
    multipole_correct_energies."""
    from scipy.special import erf
    pos = np.asarray(pos, np.float64)
    box = np.asarray(box, np.float64)
    q = np.asarray(q, np.float64)
    mu = np.asarray(dip, np.float64).reshape(-1, 3)
    pp = np.asarray(p, np.float64).reshape(-1, 3)
    Q = quad_matrix(quad)
    trQ = np.trace(Q, axis1=1, axis2=2)
    a2 = alpha * alpha
    c = 2.0 * alpha / np.sqrt(np.pi)
    e_self = float(np.sum(-np.einsum("ia,ia->i", mu, pp) * c * a2 / 3 * COULOMBS))
    mol = np.asarray(mol_id)
    intra = 0.0
    for m in np.unique(mol):
        sites = np.flatnonzero(mol == m)
        for k, i in enumerate(sites[:-1]):
            for j in sites[k + 1:]:
                r = min_image(pos[i] - pos[j], box)
                r2 = r @ r
                rr = np.sqrt(r2)
                ex = np.exp(-a2 * r2)
                D0 = erf(alpha * rr) / rr
                D1 = (-D0 + c * ex) / r2
                D2 = (-3 * D1 - 2 * c * a2 * ex) / r2
                D3 = (-5 * D2 + 4 * c * a2 * a2 * ex) / r2
                pjr, pir = pp[j] @ r, pp[i] @ (-r)
                G1i = -q[i] * pjr - mu[i] @ pp[j]
                G2i = -(mu[i] @ r) * pjr - 2.0 * (pp[j] @ (Q[i] @ r)) - pjr * trQ[i]
                G3i = -pjr * (r @ Q[i] @ r)
                G1j = -q[j] * pir - mu[j] @ pp[i]
                G2j = -(mu[j] @ (-r)) * pir - 2.0 * (pp[i] @ (Q[j] @ (-r))) - pir * trQ[j]
                G3j = -pir * (r @ Q[j] @ r)
                intra += (G1i + G1j) * D1 + (G2i + G2j) * D2 + (G3i + G3j) * D3
    return e_self, -0.5 * intra * COULOMBS


def induced_real_energy(pos, q, dip, quad, p, polar, box, alpha, a, cutoff, mol_id, amoeba=False):
    """The reference's realPolEnergy (Induction.cpp:985-1075, Thole damping
    applied to the Ewald B_n, not the AMOEBA form): for every pair of sites
    of different molecules within the real-space cutoff
        1/2 COULOMBS [(G1_i + G1_j) B1d + (G2_i + G2_j) B2d + (G3_i + G3_j) B3d]
    with the invariants of induced_correct_energies, u^3 = r^3 / sqrt(a_i a_j),
    e = exp(-a u^3), l3 = 1 - e, g3 = 3 a u^3 e / r^2, g5 = 3 (a u^3)^2 e / r^2,
        B1d = B1 l3,  B2d = B2 l3 + B1 g3,  B3d = B3 l3 + 2 B2 g3 + B1 (g3 - 3 g5) / r^2
    and the erfc-based B_n of multipole_real_energy.

    amoeba=True is the reference's dampAMOEBA branch (Induction.cpp:1051-1084,
    Tinker's form): pairs of one molecule (excluded, s = 0) are summed too,
    and with l5 = 1 - (1 + a u^3) e, l7 = 1 - (1 + a u^3 + 3 (a u^3)^2 / 5) e,
        B1d = B1 + (1 - s l3) / r^3,  B2d = B2 - 3 (1 - s l5) / r^5,
        B3d = B3 + 15 (1 - s l7) / r^7."""
    from scipy.special import erfc
    pos = np.asarray(pos, np.float64)
    box = np.asarray(box, np.float64)
    q = np.asarray(q, np.float64)
    mu = np.asarray(dip, np.float64).reshape(-1, 3)
    pp = np.asarray(p, np.float64).reshape(-1, 3)
    al = np.asarray(polar, np.float64)
    Q = quad_matrix(quad)
    trQ = np.trace(Q, axis1=1, axis2=2)
    mol = np.asarray(mol_id)
    n = len(pos)
    a2 = alpha * alpha
    c = 2.0 * alpha / np.sqrt(np.pi)
    energy = 0.0
    for i in range(n - 1):
        j = np.arange(i + 1, n)
        r = min_image(pos[i] - pos[j], box)
        r2 = np.einsum("ij,ij->i", r, r)
        keep = r2 < cutoff * cutoff
        if not amoeba:
            keep &= mol[j] != mol[i]
        j, r, r2 = j[keep], r[keep], r2[keep]
        sc = (mol[j] != mol[i]).astype(np.float64)
        if len(j) == 0:
            continue
        rr = np.sqrt(r2)
        ex = np.exp(-a2 * r2)
        B0 = erfc(alpha * rr) / rr
        B1 = (-B0 - c * ex) / r2
        B2 = (-3 * B1 + 2 * c * a2 * ex) / r2
        B3 = (-5 * B2 - 4 * c * a2 * a2 * ex) / r2
        au3 = a * r2 * rr / np.sqrt(al[i] * al[j])
        e = np.exp(-au3)
        l3 = 1.0 - e
        g3 = 3.0 * au3 * e / r2
        g5 = 3.0 * au3 * au3 * e / r2
        if amoeba:
            l5 = 1.0 - (1.0 + au3) * e
            l7 = 1.0 - (1.0 + au3 + 0.6 * au3 * au3) * e
            ir3 = 1.0 / (r2 * rr)
            B1d = B1 + (1.0 - sc * l3) * ir3
            B2d = B2 - (1.0 - sc * l5) * 3.0 * ir3 / r2
            B3d = B3 + (1.0 - sc * l7) * 15.0 * ir3 / (r2 * r2)
        else:
            B1d = B1 * l3
            B2d = B2 * l3 + B1 * g3
            B3d = B3 * l3 + 2.0 * B2 * g3 + B1 * (g3 - 3.0 * g5) / r2
        Qi_r = (Q[i] @ r.T).T
        Qj_r = np.einsum("kab,kb->ka", Q[j], r)
        rQir = np.einsum("ka,ka->k", r, Qi_r)
        rQjr = np.einsum("ka,ka->k", r, Qj_r)
        pjr = np.einsum("ka,ka->k", pp[j], r)
        pir = -(r @ pp[i])
        G1i = -q[i] * pjr - pp[j] @ mu[i]
        G2i = -(r @ mu[i]) * pjr - 2.0 * np.einsum("ka,ka->k", pp[j], Qi_r) - pjr * trQ[i]
        G3i = -pjr * rQir
        G1j = -q[j] * pir - mu[j] @ pp[i]
        G2j = -(-np.einsum("ka,ka->k", mu[j], r)) * pir + 2.0 * (Qj_r @ pp[i]) - pir * trQ[j]
        G3j = -pir * rQjr
        energy += float(np.sum((G1i + G1j) * B1d + (G2i + G2j) * B2d + (G3i + G3j) * B3d))
    return 0.5 * energy * COULOMBS


def solve_dipoles(pos, polar, box, a, cutoff, e0, damp=True):
    """Induced dipoles p (N x 3) with A p = E0 (e0: N x 3 or 3N, site-major)."""
    A = induction_matrix(pos, polar, box, a, cutoff, damp)
    return np.linalg.solve(A, np.asarray(e0, np.float64).reshape(-1)).reshape(-1, 3)

"""The restatement of the reference's induced-dipole system against the
reference's own results (golden fixture polwater216): its permanent field
from the reference's lab-frame multipoles, and its converged dipoles; and the
molecule-block preconditioner of the CUDA solve restated on that matrix (CPU
only)."""
import numpy as np

from conftest import golden
import induction_oracle
from swinmd_b200 import systems

TOL = 2.0819e-8   # 1e-6 D in e nm: RMS change of the dipoles at which the solve stops


def _case():
    g = golden("polwater216")
    s = systems.polarizable_water(nmol=216, cutoff=0.9, switch=0.8, alpha=3.5, kmax=7, seed=3, n_steps=10)
    polar = np.array([s.atom_types[t].polar for t in g["atom_type"]])
    return g, s, polar


def rms_rel(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def test_dense_solve_matches_reference_dipoles():
    g, s, polar = _case()
    p = induction_oracle.solve_dipoles(g["pos"], polar, g["box"], s.config.a_damping, s.config.cutoff_ind,
                                       g["f_ind_E0"])
    err = rms_rel(p.reshape(-1), g["f_ind_P"])
    print("rms rel error vs reference dipoles", err)
    assert err < 1e-10


def test_permanent_field_matches_reference():
    """E0 from the fixture's positions and the reference's own lab-frame
    multipoles, then the dipoles from that field."""
    g, s, polar = _case()
    q = np.array([s.atom_types[t].charge for t in g["atom_type"]])
    e0 = induction_oracle.permanent_field(g["pos"], q, g["f_mp_dip"], g["f_mp_quad"], polar, g["box"],
                                          s.config.a_damping, s.config.cutoff_ind, g["mol_id"])
    err = rms_rel(e0.reshape(-1), g["f_ind_E0"])
    print("rms rel error vs reference E0", err)
    assert err < 1e-12
    p = induction_oracle.solve_dipoles(g["pos"], polar, g["box"], s.config.a_damping, s.config.cutoff_ind, e0)
    assert rms_rel(p.reshape(-1), g["f_ind_P"]) < 1e-10


def test_chain_from_positions_matches_reference():
    """Positions -> lab-frame multipoles -> permanent field -> dipoles, every
    stage against the reference's own output."""
    g, s, polar = _case()
    t = g["atom_type"]
    dl = np.array([s.atom_types[k].dip for k in t])
    ql = np.array([s.atom_types[k].quad for k in t])
    q = np.array([s.atom_types[k].charge for k in t])
    mu, quad = induction_oracle.lab_multipoles(g["pos"], g["mol_id"], dl, ql)
    assert np.allclose(mu.reshape(-1), g["f_mp_dip"], rtol=0, atol=1e-15)
    assert np.allclose(quad.reshape(-1), g["f_mp_quad"], rtol=0, atol=1e-15)
    e0 = induction_oracle.permanent_field(g["pos"], q, mu, quad, polar, g["box"], s.config.a_damping,
                                          s.config.cutoff_ind, g["mol_id"])
    assert rms_rel(e0.reshape(-1), g["f_ind_E0"]) < 1e-12
    p = induction_oracle.solve_dipoles(g["pos"], polar, g["box"], s.config.a_damping, s.config.cutoff_ind, e0)
    assert rms_rel(p.reshape(-1), g["f_ind_P"]) < 1e-10


def test_multipole_real_energy_matches_reference():
    """Ewald real-space energy of the permanent multipoles (sum G_n B_n over
    pairs of different molecules) against the reference's realEnergy."""
    g, s, polar = _case()
    q = np.array([s.atom_types[k].charge for k in g["atom_type"]])
    e = induction_oracle.multipole_real_energy(g["pos"], q, g["f_mp_dip"], g["f_mp_quad"], g["box"],
                                               s.config.alpha, s.config.cutoff_ew, g["mol_id"])
    ref = g["f_mp_short_energy"][1]
    print("real-space energy", e, ref)
    assert abs(e - ref) < 1e-12 * abs(ref)


def test_multipole_recip_energy_matches_reference():
    """Ewald reciprocal energy of the permanent multipoles over the
    reference's k half-space against its longEnergy."""
    g, s, polar = _case()
    q = np.array([s.atom_types[k].charge for k in g["atom_type"]])
    e = induction_oracle.multipole_recip_energy(g["pos"], q, g["f_mp_dip"], g["f_mp_quad"], g["box"],
                                                s.config.alpha, s.config.k_cutoff)
    ref = g["f_mp_long_energy"][2]
    print("reciprocal energy", e, ref)
    assert abs(e - ref) < 1e-12 * abs(ref)


def test_multipole_correct_energies_match_reference():
    """Self (+ net charge) and intramolecular corrections of the multipoles
    against the reference's correctEnergy and molCorrectEnergy."""
    g, s, polar = _case()
    q = np.array([s.atom_types[k].charge for k in g["atom_type"]])
    e_corr, e_intra = induction_oracle.multipole_correct_energies(g["pos"], q, g["f_mp_dip"], g["f_mp_quad"],
                                                                  g["box"], s.config.alpha, g["mol_id"])
    ref = g["f_mp_short_energy"]
    assert abs(e_corr - ref[3]) < 1e-12 * abs(ref[3])
    assert abs(e_intra - ref[4]) < 1e-12 * abs(ref[4])


def test_induced_correct_energies_match_reference():
    """Induced dipoles' self and intramolecular corrections (from the
    reference's converged dipoles) against its correctPolEnergy and
    molCorrectPolEnergy."""
    g, s, polar = _case()
    q = np.array([s.atom_types[k].charge for k in g["atom_type"]])
    e_self, e_intra = induction_oracle.induced_correct_energies(g["pos"], q, g["f_mp_dip"], g["f_mp_quad"],
                                                                g["f_ind_P"], g["box"], s.config.alpha, g["mol_id"])
    ref = g["f_ind_short_energy"]
    assert abs(e_self - ref[8]) < 1e-12 * abs(ref[8])
    assert abs(e_intra - ref[9]) < 1e-12 * abs(ref[9])


def test_induced_real_energy_amoeba_matches_reference():
    """The dampAMOEBA branch (fixture polwater216_amoeba: the same
    configuration and dipoles, the induced real space damped as Tinker's)."""
    g0, s, polar = _case()
    g = golden("polwater216_amoeba")
    assert np.array_equal(g["f_ind_P"], g0["f_ind_P"])
    q = np.array([s.atom_types[k].charge for k in g["atom_type"]])
    e = induction_oracle.induced_real_energy(g["pos"], q, g["f_mp_dip"], g["f_mp_quad"], g["f_ind_P"], polar,
                                             g["box"], s.config.alpha, s.config.a_damping, s.config.cutoff_ew,
                                             g["mol_id"], amoeba=True)
    ref = g["f_ind_short_energy"][6]
    print(e, ref, g0["f_ind_short_energy"][6])
    assert abs(e - ref) < 1e-12 * abs(ref)


def test_induced_real_energy_matches_reference():
    """Thole-damped Ewald real-space energy of the induced dipoles (from the
    reference's converged dipoles) against its realPolEnergy."""
    g, s, polar = _case()
    q = np.array([s.atom_types[k].charge for k in g["atom_type"]])
    e = induction_oracle.induced_real_energy(g["pos"], q, g["f_mp_dip"], g["f_mp_quad"], g["f_ind_P"], polar,
                                             g["box"], s.config.alpha, s.config.a_damping, s.config.cutoff_ew,
                                             g["mol_id"])
    ref = g["f_ind_short_energy"][6]
    assert abs(e - ref) < 1e-12 * abs(ref)


def test_induced_recip_energy_matches_reference():
    """Reciprocal energy between the induced dipoles (the reference's
    converged ones) and the permanent multipoles against its longPolEnergy."""
    g, s, polar = _case()
    q = np.array([s.atom_types[k].charge for k in g["atom_type"]])
    e = induction_oracle.induced_recip_energy(g["pos"], q, g["f_mp_dip"], g["f_mp_quad"], g["f_ind_P"],
                                              g["box"], s.config.alpha, s.config.k_cutoff)
    ref = g["f_ind_long_energy"][7]
    assert abs(e - ref) < 1e-12 * abs(ref)


def pcg(A, b, apply_m, x0, tol, max_iter=200):
    """Preconditioned CG stopping when the RMS step of x drops below tol
    (the CUDA solve's test); returns x and the iteration count."""
    x = x0.copy()
    r = b - A @ x
    z = apply_m(r)
    p = z.copy()
    rz = r @ z
    for it in range(1, max_iter + 1):
        Ap = A @ p
        alpha = rz / (p @ Ap)
        x += alpha * p
        if np.sqrt(np.mean((alpha * p) ** 2)) < tol:
            return x, it
        r -= alpha * Ap
        z = apply_m(r)
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x, max_iter


def test_molecule_blocks_cut_iterations():
    g, s, polar = _case()
    A = induction_oracle.induction_matrix(g["pos"], polar, g["box"], s.config.a_damping, s.config.cutoff_ind)
    b = np.asarray(g["f_ind_E0"], np.float64)
    exact = np.linalg.solve(A, b)
    al = np.repeat(np.maximum(induction_oracle.POLMIN, polar), 3)
    # each molecule's own block of A (its sites' 1/alpha and mutual couplings), inverted
    mol = np.asarray(g["mol_id"])
    blocks = []
    for m in np.unique(mol):
        idx = np.concatenate([np.arange(3 * i, 3 * i + 3) for i in np.flatnonzero(mol == m)])
        blocks.append((idx, np.linalg.inv(A[np.ix_(idx, idx)])))

    def m_site(r):
        return al * r

    def m_mol(r):
        out = np.empty_like(r)
        for idx, inv in blocks:
            out[idx] = inv @ r[idx]
        return out

    x_site, it_site = pcg(A, b, m_site, m_site(b), TOL)
    x_mol, it_mol = pcg(A, b, m_mol, m_mol(b), TOL)
    print("iterations: site", it_site, "molecule blocks", it_mol)
    for x in (x_site, x_mol):
        assert np.sqrt(np.mean((x - exact) ** 2)) < 10 * TOL
    assert it_mol < it_site

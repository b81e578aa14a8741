"""The oracle's point-charge Ewald sums in the Lees-Edwards cell (CPU).

The reference has no shear, so nothing of its own output pins these sums.
They are checked here by properties of the lattice sum instead: at zero
offset they are the reference-pinned unsheared sums; the half-space k set of
the sheared lattice equals a brute-force enumeration with the unreduced
offset; the total Coulomb energy does not depend on the splitting parameter;
the forces are the energy's derivatives."""
import math

import numpy as np
import pytest

import oracle as O
from swinmd_b200 import systems


def _sys(nmol=27, **kw):
    return systems.spce_flexible(nmol=nmol, seed=5, **kw)


def test_zero_offset_is_the_unsheared_sum():
    s = _sys()
    L = s.box[0]
    a = O.ewald_recip_le(s, s.pos, L, 0.0)
    b = O.ewald(s, s.pos, L, O.pairlist(s, s.pos, L))
    assert a["nk"] == b["nk"]
    assert a["energy"] == pytest.approx(b["long_energy"], rel=1e-13)
    np.testing.assert_allclose(a["force"], b["long_force"], rtol=0, atol=1e-10 * np.abs(b["long_force"]).max())
    np.testing.assert_allclose(a["virial"], b["long_virial"], rtol=0, atol=1e-10 * np.abs(b["long_virial"]).max())


def _brute_recip(s, delta):
    """Every n of a wide cube, k(n) = 2 pi (nx/Lx, (ny - nx d/Lx)/Ly, nz/Lz)
    with the offset as given (not reduced), half space, |k| < kcut."""
    c = s.config
    L = s.box[0]
    q = s.scaled_charges()
    pos = s.pos
    t = delta / L
    nm = int(c.k_cutoff * L / (2 * math.pi))
    M = nm + int(math.ceil(abs(t) * nm)) + 2
    r = np.arange(-M, M + 1)
    nx, ny, nz = np.meshgrid(np.arange(0, nm + 1), r, r, indexing="ij")
    nx, ny, nz = nx.ravel(), ny.ravel(), nz.ravel()
    half = (nx > 0) | ((nx == 0) & (ny > 0)) | ((nx == 0) & (ny == 0) & (nz > 0))
    k = 2 * math.pi * np.stack([nx / L, (ny - nx * t) / L, nz / L], 1)
    k2 = (k ** 2).sum(1)
    sel = half & (k2 < c.k_cutoff ** 2)
    k, k2 = k[sel], k2[sel]
    ph = pos @ k.T
    S = (q[:, None] * np.exp(1j * ph)).sum(0)
    V = L ** 3
    e = (4 * math.pi / V * np.exp(-k2 / (4 * c.alpha ** 2)) / k2 * np.abs(S) ** 2).sum()
    return e, int(sel.sum())


@pytest.mark.parametrize("frac", [0.23, 0.5, 0.71, 1.37])
def test_sheared_k_set_matches_brute_force(frac):
    s = _sys()
    L = s.box[0]
    a = O.ewald_recip_le(s, s.pos, L, frac * L)
    e, nk = _brute_recip(s, frac * L)
    assert a["nk"] == nk
    assert a["energy"] == pytest.approx(e, rel=1e-11)


def test_offset_by_a_box_edge_is_the_same_lattice():
    s = _sys()
    L = s.box[0]
    a = O.ewald_recip_le(s, s.pos, L, 0.31 * L)
    b = O.ewald_recip_le(s, s.pos, L, 1.31 * L)
    assert a["nk"] == b["nk"]
    assert a["energy"] == pytest.approx(b["energy"], rel=1e-12)


def _coulomb_total(s, delta, alpha, rc, kcut):
    c = s.config
    c.alpha, c.cutoff, c.k_cutoff = alpha, rc, kcut
    t = O.flex_le_forces(s, s.pos, s.box[0], delta)
    q = s.scaled_charges()
    e_self = -alpha / math.sqrt(math.pi) * float((q * q).sum())
    return t["real"] + t["long"] + t["intra"] + e_self


def test_total_coulomb_energy_is_independent_of_alpha_under_shear():
    s = _sys()
    L = s.box[0]
    rc = 0.5 * L - 1e-9
    e = []
    for alpha in (10.0, 12.0):
        kcut = 2 * alpha * math.sqrt(math.log(1e11))
        e.append(_coulomb_total(s, 0.37 * L, alpha, rc, kcut))
    assert e[0] == pytest.approx(e[1], rel=2e-8)
    # and the sheared energy differs from the unsheared one: the test sees the shear
    kcut = 2 * 10.0 * math.sqrt(math.log(1e11))
    e0 = _coulomb_total(s, 0.0, 10.0, rc, kcut)
    assert abs(e0 - e[0]) > 1e-3 * abs(e0)


def test_sheared_forces_are_energy_derivatives():
    s = _sys(nmol=8)
    L = s.box[0]
    delta = 0.42 * L
    base = O.flex_le_forces(s, s.pos, L, delta)
    tot = lambda t: t["vdw"] + t["real"] + t["long"] + t["intra"] + t["bond"] + t["angle"]
    h = 1e-6
    for i in (0, 4, 10):
        for d in range(3):
            p = s.pos.copy()
            p[i, d] += h
            ep = tot(O.flex_le_forces(s, p, L, delta))
            p[i, d] -= 2 * h
            em = tot(O.flex_le_forces(s, p, L, delta))
            assert -(ep - em) / (2 * h) == pytest.approx(base["force"][i, d], rel=2e-5, abs=2e-3)

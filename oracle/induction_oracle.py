"""Dense restatement of the reference's induced-dipole system (test
infrastructure: only tests/ use it, as the checker).

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


def solve_dipoles(pos, polar, box, a, cutoff, e0, damp=True):
    """Induced dipoles p (N x 3) with A p = E0 (e0: N x 3 or 3N, site-major)."""
    A = induction_matrix(pos, polar, box, a, cutoff, damp)
    return np.linalg.solve(A, np.asarray(e0, np.float64).reshape(-1)).reshape(-1, 3)

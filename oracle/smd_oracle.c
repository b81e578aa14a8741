/* smd_oracle.c — CPU restatement of the SwinMD force/integration path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this
 * file; tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it
 * as the checker of the CUDA path.  It restates, in plain C and FP64, the
 * reference's algorithms for the functions the CUDA path replaces; each
 * function cites the reference lines it follows.  It is pinned against the
 * reference's own outputs (tests/golden/*.npz, made by running the
 * reference's C++ through oracle/_ref/ref_dump) by tests/test_oracle.py.
 *
 * Conventions: positions/forces are n x 3 row-major doubles (nm, kJ/mol/nm),
 * r_ij = r_j - r_i, f_i += f_ij, the returned virial is the contribution to
 * Ensemble::virial (= -sum f_ij (x) r_ij, row-major).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159265358979323846
#define OR_SQRT_PI 1.7724538509055160273
#define OR_KB 0.0083145112

/* Ensemble::apply_pbc (src/Ensemble.h:319-334) */
static void pbc(double *d, const double *L) {
    for (int k = 0; k < 3; k++) {
        double h = L[k] / 2.0;
        while (d[k] >= h) d[k] -= L[k];
        while (d[k] < -h) d[k] += L[k];
    }
}

static int excluded(int i, int j, const int32_t *off, const int32_t *ex) {
    for (int e = off[i]; e < off[i + 1]; e++)
        if (ex[e] == j) return 1;
    return 0;
}

/* Ensemble::build_pairlist (src/Ensemble.cpp:492-525): all i < j not in the
 * exclusion table with |pbc(r_j - r_i)|^2 < (rc + skin)^2.  Writes pairs as
 * (i, j) into out (capacity cap pairs); returns the number of pairs. */
int64_t or_pairlist(int n, const double *pos, const double *L, double rl2, const int32_t *off,
                    const int32_t *ex, int32_t *out, int64_t cap) {
    int64_t k = 0;
    for (int i = 0; i < n - 1; i++)
        for (int j = i + 1; j < n; j++) {
            if (excluded(i, j, off, ex)) continue;
            double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                           pos[3 * j + 2] - pos[3 * i + 2]};
            pbc(d, L);
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (r2 < rl2) {
                if (k < cap) { out[2 * k] = i; out[2 * k + 1] = j; }
                k++;
            }
        }
    return k;
}

static void vir_add(double *w, const double *f, const double *r) {
    /* local virial[XY] += f.y * r.x (LJForce.cpp:206-214), stored negated */
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) w[3 * a + b] -= f[b] * r[a];
}

/* LJForce::compute (src/forces/LJForce.cpp:58-255) over a given pair list:
 * same-molecule pairs skipped, r*r <= rc^2 with r = |r_ij|, energy shifted
 * by U(rc) when shift != 0, long-range correction e_lrc / v_lrc added. */
double or_lj(int n, const double *pos, const int32_t *type, const int32_t *mol, const double *L,
             int nt, const double *sig2, const double *eps4, double rc, int shift, double e_lrc,
             double v_lrc, const int32_t *pairs, int64_t np, double *f, double *w) {
    double rc2 = rc * rc, rcut_2 = 1.0 / rc2, energy = 0.0;
    memset(f, 0, sizeof(double) * 3 * n);
    memset(w, 0, sizeof(double) * 9);
    for (int64_t p = 0; p < np; p++) {
        int i = pairs[2 * p], j = pairs[2 * p + 1];
        if (mol[i] == mol[j]) continue;
        double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                       pos[3 * j + 2] - pos[3 * i + 2]};
        pbc(d, L);
        double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double rij2 = r * r;
        if (rij2 > rc2) continue;
        int t = type[i] * nt + type[j];
        double r_1 = 1.0 / r, rij_2 = r_1 * r_1;
        double sr2 = sig2[t] * rij_2, sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
        double e = eps4[t] * (sr12 - sr6);
        double fs = (sr12 + sr12 - sr6) * 6 * eps4[t] * rij_2;
        if (shift) {
            double c2 = sig2[t] * rcut_2, c6 = c2 * c2 * c2;
            e -= eps4[t] * (c6 * c6 - c6);
        }
        energy += e;
        double fij[3] = {-fs * d[0], -fs * d[1], -fs * d[2]};
        for (int k = 0; k < 3; k++) { f[3 * i + k] += fij[k]; f[3 * j + k] -= fij[k]; }
        vir_add(w, fij, d);
    }
    w[0] -= v_lrc; w[4] -= v_lrc; w[8] -= v_lrc;
    return energy + e_lrc;
}

/* Leap-frog Nose-Hoover MD of a Lennard-Jones system: LFIntegrator::start
 * (LFIntegrator.cpp:1172-1173) then nsteps of LFIntegrator::run
 * (:278-941) with the unconstrained update (:588-642), zeta update
 * (:688-722), COM drift removal (:359-379), molecule wrap (:897-912) and
 * brute-force list rebuild when a displacement exceeds skin/2.
 * Monatomic molecules (mol[i] == i) only.  out_epot/out_temp/out_zeta:
 * per-step potential energy (at the step's start), atomic temperature and
 * zeta.  pos/vel are updated in place; vtm receives v(t - dt/2). */
int or_lj_md(int n, double *pos, double *vel, double *vtm, const double *mass,
             const int32_t *type, const int32_t *mol, const double *L, int nt, const double *sig2,
             const double *eps4, double rc, double skin, int shift, double e_lrc, double v_lrc,
             double dt, double T, double tau, int nsteps, double *out_epot, double *out_temp,
             double *out_zeta) {
    int64_t cap = (int64_t)n * 400;
    int32_t *pairs = (int32_t *)malloc(sizeof(int32_t) * 2 * cap);
    int32_t *off = (int32_t *)calloc(n + 1, sizeof(int32_t));
    double *f = (double *)malloc(sizeof(double) * 3 * n);
    double *disp = (double *)calloc(3 * n, sizeof(double));
    double w[9];
    double rl = rc + skin, rl2 = rl * rl, drmax = skin * skin / 4.0;
    int64_t np = or_pairlist(n, pos, L, rl2, off, NULL, pairs, cap);
    if (np > cap) return -1;
    or_lj(n, pos, type, mol, L, nt, sig2, eps4, rc, shift, e_lrc, v_lrc, pairs, np, f, w);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) vtm[3 * i + k] = vel[3 * i + k] - 0.5 * dt * (1.0 / mass[i]) * f[3 * i + k];
    int ndf = 3 * n - 3;
    double fnh = 0, fnhmi = 0, mtot = 0;
    for (int i = 0; i < n; i++) mtot += mass[i];
    for (int s = 0; s < nsteps; s++) {
        int upd = 0;
        for (int i = 0; i < n && !upd; i++)
            if (disp[3 * i] * disp[3 * i] + disp[3 * i + 1] * disp[3 * i + 1] + disp[3 * i + 2] * disp[3 * i + 2] > drmax) upd = 1;
        if (upd) {
            memset(disp, 0, sizeof(double) * 3 * n);
            np = or_pairlist(n, pos, L, rl2, off, NULL, pairs, cap);
            if (np > cap) return -1;
        }
        double vom[3] = {0, 0, 0};
        for (int i = 0; i < n; i++)
            for (int k = 0; k < 3; k++) vom[k] += vtm[3 * i + k] * mass[i];
        for (int k = 0; k < 3; k++) vom[k] /= mtot;
        if (fabs(vom[0]) > 1e-11 || fabs(vom[1]) > 1e-11 || fabs(vom[2]) > 1e-11)
            for (int i = 0; i < n; i++)
                for (int k = 0; k < 3; k++) { vtm[3 * i + k] -= vom[k]; vel[3 * i + k] -= vom[k]; }
        out_epot[s] = or_lj(n, pos, type, mol, L, nt, sig2, eps4, rc, shift, e_lrc, v_lrc, pairs, np, f, w);
        double ke = 0;
        for (int i = 0; i < n; i++) {
            double mr = 1.0 / mass[i], vp[3], *v = &vel[3 * i], *vm = &vtm[3 * i];
            double velcheck = 1.0;
            int cnt = 0;
            while (velcheck > 1e-10 && cnt < 11) {
                for (int k = 0; k < 3; k++) vp[k] = vm[k] + dt * (mr * f[3 * i + k] - fnh * v[k]);
                double dd = 0;
                for (int k = 0; k < 3; k++) {
                    double nv = (vp[k] + vm[k]) * 0.5;
                    dd += (nv - v[k]) * (nv - v[k]);
                    v[k] = nv;
                }
                velcheck = sqrt(dd);
                cnt++;
            }
            if (cnt == 10) return -2;
            for (int k = 0; k < 3; k++) {
                double dr = dt * vp[k];
                pos[3 * i + k] += dr;
                disp[3 * i + k] += dr;
                v[k] = (vp[k] + vm[k]) * 0.5;
                vm[k] = vp[k];
            }
            ke += (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * mass[i];
            /* monatomic molecule: wrap the atom into the box */
            double c[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]}, o[3] = {c[0], c[1], c[2]};
            pbc(c, L);
            for (int k = 0; k < 3; k++) pos[3 * i + k] += c[k] - o[k];
        }
        double qq = ndf * OR_KB * T * tau * tau;
        double fnhpl = fnhmi + dt * (1.0 / qq) * (ke - ndf * OR_KB * T);
        fnh = 0.5 * (fnhpl + fnhmi);
        fnhmi = fnhpl;
        out_temp[s] = ke / (ndf * OR_KB);
        out_zeta[s] = fnh;
    }
    free(pairs); free(off); free(f); free(disp);
    return 0;
}

/* Ewald real-space term (EwaldForce::real_term, src/forces/EwaldForce.cpp:
 * 296-527) over a pair list: q_i q_j erfc(a r)/r for r^2 < rc^2 (scaled
 * charges), all listed pairs.  Returns the real-space energy. */
double or_ewald_real(int n, const double *pos, const double *q, const double *L, double alpha,
                     double rc, const int32_t *pairs, int64_t np, double *f, double *w) {
    double rc2 = rc * rc, a2 = alpha * alpha, a2pi = 2.0 * alpha / OR_SQRT_PI, energy = 0;
    for (int64_t p = 0; p < np; p++) {
        int i = pairs[2 * p], j = pairs[2 * p + 1];
        double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                       pos[3 * j + 2] - pos[3 * i + 2]};
        pbc(d, L);
        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        if (!(r2 < rc2)) continue;
        double qij = q[i] * q[j], r = sqrt(r2);
        double e = erfc(alpha * r) / r;
        double fs = (e + a2pi * exp(-a2 * r2)) / r2;
        energy += qij * e;
        double fij[3] = {-qij * fs * d[0], -qij * fs * d[1], -qij * fs * d[2]};
        for (int k = 0; k < 3; k++) { f[3 * i + k] += fij[k]; f[3 * j + k] -= fij[k]; }
        vir_add(w, fij, d);
    }
    return energy;
}

/* Ewald reciprocal term (EwaldForce::set_up + reciprocal_term,
 * src/forces/EwaldForce.cpp:198-257, 529-698): half-space k set with
 * k^2 < kcut^2.  Adds forces into f, the long virial into w (all nine
 * components), returns the energy; *nk receives the k count. */
double or_ewald_recip(int n, const double *pos, const double *q, const double *L, double alpha,
                      double kcut, double *f, double *w, int *nk_out) {
    double kc2 = kcut * kcut, aR4 = 1.0 / (4.0 * alpha * alpha);
    int nmax[3];
    for (int d = 0; d < 3; d++) nmax[d] = (int)(kcut * L[d] / (2 * OR_PI));
    double v[3] = {2.0 * OR_PI / L[0], 2.0 * OR_PI / L[1], 2.0 * OR_PI / L[2]};
    double vol = L[0] * L[1] * L[2], pi4V = 4.0 * OR_PI * (1.0 / vol), pi8V = 2.0 * pi4V;
    double *sc = (double *)malloc(sizeof(double) * 2 * n), pe = 0;
    int nk = 0;
    for (int nx = 0; nx <= nmax[0]; nx++)
        for (int ny = (nx == 0 ? 0 : -nmax[1]); ny <= nmax[1]; ny++)
            for (int nz = ((nx == 0 && ny == 0) ? 1 : -nmax[2]); nz <= nmax[2]; nz++) {
                double k[3] = {nx * v[0], ny * v[1], nz * v[2]};
                double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                if (!(k2 < kc2)) continue;
                nk++;
                double expK = exp(-k2 * aR4) / k2, ss = 0, cs = 0;
                for (int i = 0; i < n; i++) {
                    double a = pos[3 * i] * k[0] + pos[3 * i + 1] * k[1] + pos[3 * i + 2] * k[2];
                    sc[2 * i] = q[i] * sin(a);
                    sc[2 * i + 1] = q[i] * cos(a);
                    ss += sc[2 * i];
                    cs += sc[2 * i + 1];
                }
                double e = pi4V * expK * (ss * ss + cs * cs);
                pe += e;
                double coeff = 2.0 * (aR4 + 1.0 / k2);
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) w[3 * a + b] += (a == b ? e : 0.0) - e * coeff * k[a] * k[b];
                double b = pi8V * expK;
                for (int i = 0; i < n; i++) {
                    double val = b * (sc[2 * i] * cs - sc[2 * i + 1] * ss);
                    for (int d = 0; d < 3; d++) f[3 * i + d] += k[d] * val;
                }
            }
    free(sc);
    if (nk_out) *nk_out = nk;
    return pe;
}

/* Mie n-m and Born-Mayer-Huggins pair terms over a pair list, with the
 * 5th-order switch of MieForce::compute (src/forces/MieForce.cpp:89-196,
 * switch constants :26-46) applied between sqrt(rs2) and rc when sw != 0.
 * kind 2 (Mie): par = {sigma, Cn*eps, n, m} per type pair, as MieForce
 * derives them from the LJ table (:26-35, :122-124).
 * kind 3 (BMH, no reference code): par = {A, 1/rho, C, D},
 * U = A exp(-r/rho) - C r^-6 - D r^-8.
 * Same-molecule pairs are skipped (:111).  Returns the energy. */
double or_vdw(int kind, int n, const double *pos, const int32_t *type, const int32_t *mol,
              const double *L, int nt, const double *par, double rc, int sw, double rs2,
              const int32_t *pairs, int64_t np, double *f, double *w) {
    double rc2 = rc * rc, energy = 0;
    double c1 = 0, c2 = 0, c3 = 0;
    if (sw && rc2 > rs2) {
        c1 = 1.0 / (rc2 - rs2);
        c1 = c1 * c1 * c1;
        c2 = rc2 - 3.0 * rs2;
        c3 = 4 * c1;
    }
    memset(f, 0, sizeof(double) * 3 * n);
    memset(w, 0, sizeof(double) * 9);
    for (int64_t p = 0; p < np; p++) {
        int i = pairs[2 * p], j = pairs[2 * p + 1];
        if (mol[i] == mol[j]) continue;
        double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                       pos[3 * j + 2] - pos[3 * i + 2]};
        pbc(d, L);
        double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double rij2 = r * r;
        if (rij2 > rc2) continue;
        const double *q = &par[4 * (type[i] * nt + type[j])];
        double r_1 = 1.0 / r, rij_2 = r_1 * r_1, e, fs;
        if (kind == 2) {
            double s = q[0] * r_1, srn = pow(s, q[2]), srm = pow(s, q[3]);
            e = q[1] * (srn - srm);
            fs = q[1] * (q[2] * srn - q[3] * srm) * rij_2;
        } else {
            double ex = q[0] * exp(-r * q[1]), r6 = rij_2 * rij_2 * rij_2, r8 = r6 * rij_2;
            e = ex - q[2] * r6 - q[3] * r8;
            fs = ex * q[1] * r_1 - 6.0 * q[2] * r8 - 8.0 * q[3] * r8 * rij_2;
        }
        if (sw && rij2 > rs2) {
            double c = rc2 - rij2, c4 = c * (2 * rij2 + c2);
            double sv = c * c4 * c1, dsv = c3 * (c * c - c4);
            fs = fs * sv - e * dsv;
            e *= sv;
        }
        energy += e;
        double fij[3] = {-fs * d[0], -fs * d[1], -fs * d[2]};
        for (int k = 0; k < 3; k++) { f[3 * i + k] += fij[k]; f[3 * j + k] -= fij[k]; }
        vir_add(w, fij, d);
    }
    return energy;
}

/* EwaldForce::intraMolCorrect energy (src/forces/EwaldForce.cpp:709-813) for
 * molecules of consecutive sites (ns per molecule): -sum over excluded
 * intramolecular pairs of q_i q_j erf(a r)/r.  Forces only when !constrained
 * (the reference applies none under constraints). */
double or_ewald_intra(int nmol, int ns, const double *pos, const double *q, const double *L,
                      double alpha, const int32_t *off, const int32_t *ex, int constrained,
                      double *f) {
    double en = 0, a2 = alpha * alpha, a2pi = 2.0 * alpha / OR_SQRT_PI;
    for (int m = 0; m < nmol; m++)
        for (int a = 0; a < ns; a++)
            for (int b = a + 1; b < ns; b++) {
                int i = m * ns + a, j = m * ns + b;
                if (!excluded(i, j, off, ex)) continue;
                double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                               pos[3 * j + 2] - pos[3 * i + 2]};
                pbc(d, L);
                double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], r = sqrt(r2);
                double qij = q[i] * q[j], e = erf(alpha * r) / r;
                en += qij * e;
                if (!constrained) {
                    double dudr = e - a2pi * exp(-a2 * r2);
                    for (int k = 0; k < 3; k++) {
                        double fij = qij * dudr / r2 * d[k];
                        f[3 * i + k] += fij;
                        f[3 * j + k] -= fij;
                    }
                }
            }
    return -en;
}

/* Rigid 3-site water MD: LJ (LJForce) + Ewald (real, reciprocal, intra
 * energy, self) forces, then LFIntegrator::shake (LFIntegrator.cpp:1678-1827,
 * NVT branch with the Nose-Hoover term -zeta P_mol/ns) for every molecule
 * and the step's molecular bookkeeping and zeta update (:646-722), molecule
 * wrap (:897-912), drift removal (:359-379) and list rebuild (:307-341).
 * Molecules are consecutive triples (H O H); clen2[3] the squared
 * constraint distances.  out_*: per-step potential energy, temperature. */
int or_water_md(int nmol, double *pos, double *vel, const double *mass, const int32_t *type,
                const int32_t *mol, const double *q, const double *L, int nt, const double *sig2,
                const double *eps4, double rc, double skin, int shift, double alpha, double kcut,
                double e_self, const int32_t *off, const int32_t *ex, const double *clen2,
                double tol, int maxcount, double dt, double T, double tau, int nsteps,
                double *out_epot, double *out_temp, double *out_zeta) {
    int n = 3 * nmol;
    int64_t cap = (int64_t)n * 600;
    int32_t *pairs = (int32_t *)malloc(sizeof(int32_t) * 2 * cap);
    double *f = (double *)malloc(sizeof(double) * 3 * n), *f2 = (double *)malloc(sizeof(double) * 3 * n);
    double *vtm = (double *)malloc(sizeof(double) * 3 * n);
    double *disp = (double *)calloc(3 * n, sizeof(double));
    double *P = (double *)calloc(3 * nmol, sizeof(double));
    double w[9];
    double rl = rc + skin, rl2 = rl * rl, drmax = skin * skin / 4.0;
    int64_t np = or_pairlist(n, pos, L, rl2, off, ex, pairs, cap);
    if (np > cap) return -1;
#define OR_FORCES(E)                                                                          \
    do {                                                                                      \
        double e_ = or_lj(n, pos, type, mol, L, nt, sig2, eps4, rc, shift, 0.0, 0.0, pairs, np, f, w); \
        memset(w, 0, sizeof(w));                                                              \
        e_ += or_ewald_real(n, pos, q, L, alpha, rc, pairs, np, f, w);                        \
        e_ += or_ewald_intra(nmol, 3, pos, q, L, alpha, off, ex, 1, f);                       \
        e_ += or_ewald_recip(n, pos, q, L, alpha, kcut, f, w, NULL) + e_self;                 \
        E = e_;                                                                               \
    } while (0)
    double e0;
    OR_FORCES(e0);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) vtm[3 * i + k] = vel[3 * i + k] - 0.5 * dt * (1.0 / mass[i]) * f[3 * i + k];
    int ndf = 6 * nmol - 3;
    double fnh = 0, fnhmi = 0, mtot = 0;
    for (int i = 0; i < n; i++) mtot += mass[i];
    for (int s = 0; s < nsteps; s++) {
        int upd = 0;
        for (int i = 0; i < n && !upd; i++)
            if (disp[3 * i] * disp[3 * i] + disp[3 * i + 1] * disp[3 * i + 1] + disp[3 * i + 2] * disp[3 * i + 2] > drmax) upd = 1;
        if (upd) {
            memset(disp, 0, sizeof(double) * 3 * n);
            np = or_pairlist(n, pos, L, rl2, off, ex, pairs, cap);
        }
        double vom[3] = {0, 0, 0};
        for (int i = 0; i < n; i++)
            for (int k = 0; k < 3; k++) vom[k] += vtm[3 * i + k] * mass[i];
        for (int k = 0; k < 3; k++) vom[k] /= mtot;
        if (fabs(vom[0]) > 1e-11 || fabs(vom[1]) > 1e-11 || fabs(vom[2]) > 1e-11)
            for (int i = 0; i < n; i++)
                for (int k = 0; k < 3; k++) { vtm[3 * i + k] -= vom[k]; vel[3 * i + k] -= vom[k]; }
        OR_FORCES(out_epot[s]);
        double ke = 0;
        for (int m = 0; m < nmol; m++) {
            double ro[3][3], rn[3][3], mr[3];
            for (int a = 0; a < 3; a++) {
                int i = 3 * m + a;
                mr[a] = 1.0 / mass[i];
                for (int k = 0; k < 3; k++) {
                    double vp = vtm[3 * i + k] + dt * mr[a] * (f[3 * i + k] - fnh * P[3 * m + k] / 3);
                    ro[a][k] = pos[3 * i + k];
                    rn[a][k] = ro[a][k] + dt * vp;
                }
            }
            int count = 0, done = 0;
            while (!done && count < maxcount) {
                done = 1;
                for (int b = 0; b < 3; b++) {
                    int nx = (b + 1) % 3;
                    double dn[3] = {rn[b][0] - rn[nx][0], rn[b][1] - rn[nx][1], rn[b][2] - rn[nx][2]};
                    pbc(dn, L);
                    double r2 = dn[0] * dn[0] + dn[1] * dn[1] + dn[2] * dn[2];
                    double diff = clen2[b] - r2;
                    if (fabs(diff) > clen2[b] * 2 * tol) {
                        double dold[3] = {ro[b][0] - ro[nx][0], ro[b][1] - ro[nx][1], ro[b][2] - ro[nx][2]};
                        pbc(dold, L);
                        double rr = dold[0] * dn[0] + dold[1] * dn[1] + dold[2] * dn[2];
                        if (rr < clen2[b] * tol) return -3;
                        double factor = diff / (2 * rr * (mr[b] + mr[nx]));
                        for (int k = 0; k < 3; k++) {
                            rn[b][k] += factor * dold[k] * mr[b];
                            rn[nx][k] -= factor * dold[k] * mr[nx];
                        }
                        done = 0;
                    }
                }
                count++;
            }
            if (!done) return -4;
            double Pm[3] = {0, 0, 0}, com[3] = {0, 0, 0}, M = 0;
            for (int a = 0; a < 3; a++) {
                int i = 3 * m + a;
                for (int k = 0; k < 3; k++) {
                    double dr = rn[a][k] - pos[3 * i + k];
                    pos[3 * i + k] += dr;
                    disp[3 * i + k] += dr;
                    double vp = dr / dt;
                    vel[3 * i + k] = (vp + vtm[3 * i + k]) * 0.5;
                    vtm[3 * i + k] = vp;
                    Pm[k] += vel[3 * i + k] * mass[i];
                    com[k] += mass[i] * pos[3 * i + k];
                }
                M += mass[i];
                ke += (vel[3 * i] * vel[3 * i] + vel[3 * i + 1] * vel[3 * i + 1] + vel[3 * i + 2] * vel[3 * i + 2]) * mass[i];
            }
            for (int k = 0; k < 3; k++) { P[3 * m + k] = Pm[k]; com[k] /= M; }
            double c[3] = {com[0], com[1], com[2]};
            pbc(c, L);
            for (int a = 0; a < 3; a++)
                for (int k = 0; k < 3; k++) pos[3 * (3 * m + a) + k] += c[k] - com[k];
        }
        double qq = ndf * OR_KB * T * tau * tau;
        double fnhpl = fnhmi + dt * (1.0 / qq) * (ke - ndf * OR_KB * T);
        fnh = 0.5 * (fnhpl + fnhmi);
        fnhmi = fnhpl;
        out_temp[s] = ke / (ndf * OR_KB);
        out_zeta[s] = fnh;
    }
#undef OR_FORCES
    free(pairs); free(f); free(f2); free(vtm); free(disp); free(P);
    return 0;
}

/* ------------------------------------------------------------------------
 * Nose-Hoover chain (NVT) velocity-Verlet MD of a Lennard-Jones system,
 * optionally under SLLOD planar Couette shear with Lees-Edwards images.
 *
 * The chain restates NHIntegrator::chain (src/integrators/NHIntegrator.cpp:
 * 1814-1912): 4 links, nc = 5 multiple steps, 3 Suzuki-Yoshida weights,
 * Q_0 = Nf kT tau^2, Q_k = kT tau^2 (:113-119).  The reference's integrator
 * couples a barostat in every step (vlog, glog, box rescaling); this NVT
 * restatement drops that degree of freedom (vlog = 0, Nf kT in the first
 * link's force).  Step order as NHIntegrator::run (:380-408, :628-644):
 * chain half step, half kick, drift, forces, half kick, chain half step.
 *
 * SLLOD (no reference code; Evans and Morriss, "Statistical Mechanics of
 * Nonequilibrium Liquids", ch. 6): peculiar velocities v, flow u = (g y,0,0);
 *   dr/dt = v + g y e_x,   dv/dt = F/m - g v_y e_x - zeta v.
 * The streaming and the -g v_y e_x term are each integrated exactly over
 * their sub-steps: around every half kick v_x -= g (dt/2) v_y; the drift is
 * x += dt v_x + g dt (y + dt v_y / 2), y += dt v_y, z += dt v_z.
 * Lees-Edwards: the image one box up is shifted by delta = g Ly t (mod Lx)
 * in x; minimum image takes y first (shifting x by -/+ delta per crossing),
 * then x and z.  All pairs within rc are found by a direct O(N^2) search.
 * Outputs per step: potential energy after the step's forces, atomic
 * temperature 2 KE / (Nf kB), first chain velocity, pressure tensor xy
 * component (sum m v_x v_y + W_xy)/V with W_ab = -sum r_a f_b, and delta.
 * Parity unpinned: the reference has neither a constant-volume chain
 * integrator nor SLLOD, so nothing of the reference's own output checks this
 * function.
 * ---------------------------------------------------------------------- */
static void pbc_le(double *d, const double *L, double delta) {
    double hy = L[1] / 2.0, hx = L[0] / 2.0, hz = L[2] / 2.0;
    while (d[1] >= hy) { d[1] -= L[1]; d[0] -= delta; }
    while (d[1] < -hy) { d[1] += L[1]; d[0] += delta; }
    while (d[0] >= hx) d[0] -= L[0];
    while (d[0] < -hx) d[0] += L[0];
    while (d[2] >= hz) d[2] -= L[2];
    while (d[2] < -hz) d[2] += L[2];
}

static double lj_le_forces(int n, const double *pos, const int32_t *type, const double *L, double delta,
                           int nt, const double *sig2, const double *eps4, double rc, int shift,
                           double *f, double *w) {
    double rc2 = rc * rc, rcut_2 = 1.0 / rc2, energy = 0.0;
    memset(f, 0, sizeof(double) * 3 * n);
    memset(w, 0, sizeof(double) * 9);
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                           pos[3 * j + 2] - pos[3 * i + 2]};
            pbc_le(d, L, delta);
            double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            double rij2 = r * r;
            if (rij2 > rc2) continue;
            int t = type[i] * nt + type[j];
            double r_1 = 1.0 / r, rij_2 = r_1 * r_1;
            double sr2 = sig2[t] * rij_2, sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
            double e = eps4[t] * (sr12 - sr6);
            double fs = (sr12 + sr12 - sr6) * 6 * eps4[t] * rij_2;
            if (shift) {
                double c2 = sig2[t] * rcut_2, c6 = c2 * c2 * c2;
                e -= eps4[t] * (c6 * c6 - c6);
            }
            energy += e;
            double fij[3] = {-fs * d[0], -fs * d[1], -fs * d[2]};
            for (int k = 0; k < 3; k++) { f[3 * i + k] += fij[k]; f[3 * j + k] -= fij[k]; }
            vir_add(w, fij, d);
        }
    return energy;
}

static double nhc_half(double *vnh, const double *qnh, double ekin, double kT, double nf, double dt) {
    const double w0 = 1.0 / (2.0 - pow(2.0, 1.0 / 3.0));
    const double wj[3] = {w0, 1.0 - 2.0 * w0, w0};
    const int nc = 5;
    double scale = 1.0, gnh[4];
    for (int i = 0; i < nc; i++)
        for (int j = 0; j < 3; j++) {
            double dts = wj[j] * dt / nc, dts2 = 0.5 * dts, dts4 = 0.25 * dts, dts8 = 0.125 * dts, ex;
            gnh[3] = (qnh[2] * vnh[2] * vnh[2] - kT) / qnh[3];
            vnh[3] += gnh[3] * dts4;
            gnh[2] = (qnh[1] * vnh[1] * vnh[1] - kT) / qnh[2];
            ex = exp(-vnh[3] * dts8);
            vnh[2] = ex * (vnh[2] * ex + gnh[2] * dts4);
            gnh[1] = (qnh[0] * vnh[0] * vnh[0] - kT) / qnh[1];
            ex = exp(-vnh[2] * dts8);
            vnh[1] = ex * (vnh[1] * ex + gnh[1] * dts4);
            gnh[0] = (2.0 * ekin - nf * kT) / qnh[0];
            ex = exp(-vnh[1] * dts8);
            vnh[0] = ex * (vnh[0] * ex + gnh[0] * dts4);
            ex = exp(-vnh[0] * dts2);
            scale *= ex;
            ekin = ekin * ex * ex;
            gnh[0] = (2.0 * ekin - nf * kT) / qnh[0];
            ex = exp(-vnh[1] * dts8);
            vnh[0] = ex * (vnh[0] * ex + gnh[0] * dts4);
            gnh[1] = (qnh[0] * vnh[0] * vnh[0] - kT) / qnh[1];
            ex = exp(-vnh[2] * dts8);
            vnh[1] = ex * (vnh[1] * ex + gnh[1] * dts4);
            gnh[2] = (qnh[1] * vnh[1] * vnh[1] - kT) / qnh[2];
            ex = exp(-vnh[3] * dts8);
            vnh[2] = ex * (vnh[2] * ex + gnh[2] * dts4);
            gnh[3] = (qnh[2] * vnh[2] * vnh[2] - kT) / qnh[3];
            vnh[3] += gnh[3] * dts4;
        }
    return scale;
}

int or_lj_nhc_md(int n, double *pos, double *vel, const double *mass, const int32_t *type, const double *L,
                 int nt, const double *sig2, const double *eps4, double rc, int shift, double dt, double T,
                 double tau, double gamma, int ndf, int nsteps, double *out_epot, double *out_temp,
                 double *out_vnh0, double *out_pxy, double *out_delta) {
    double *f = (double *)malloc(sizeof(double) * 3 * n);
    double w[9];
    const double kT = OR_KB * T, nf = (double)ndf, vol = L[0] * L[1] * L[2];
    double qnh[4], vnh[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; k++) qnh[k] = kT * tau * tau;
    qnh[0] *= nf;
    double delta = 0.0;
    lj_le_forces(n, pos, type, L, delta, nt, sig2, eps4, rc, shift, f, w);
    for (int s = 0; s < nsteps; s++) {
        double ekin = 0;
        for (int i = 0; i < n; i++)
            ekin += 0.5 * mass[i] * (vel[3 * i] * vel[3 * i] + vel[3 * i + 1] * vel[3 * i + 1] + vel[3 * i + 2] * vel[3 * i + 2]);
        double sc = nhc_half(vnh, qnh, ekin, kT, nf, dt);
        delta = fmod(delta + gamma * L[1] * dt, L[0]);
        if (delta < 0) delta += L[0];
        for (int i = 0; i < n; i++) {
            double *v = &vel[3 * i], *r = &pos[3 * i], mr = 1.0 / mass[i];
            for (int k = 0; k < 3; k++) v[k] *= sc;
            v[0] -= gamma * 0.5 * dt * v[1];
            for (int k = 0; k < 3; k++) v[k] += 0.5 * dt * mr * f[3 * i + k];
            r[0] += dt * v[0] + gamma * dt * (r[1] + 0.5 * dt * v[1]);
            r[1] += dt * v[1];
            r[2] += dt * v[2];
            /* Lees-Edwards wrap (y first), then x and z */
            if (r[1] >= L[1] / 2.0) { r[1] -= L[1]; r[0] -= delta; }
            else if (r[1] < -L[1] / 2.0) { r[1] += L[1]; r[0] += delta; }
            while (r[0] >= L[0] / 2.0) r[0] -= L[0];
            while (r[0] < -L[0] / 2.0) r[0] += L[0];
            while (r[2] >= L[2] / 2.0) r[2] -= L[2];
            while (r[2] < -L[2] / 2.0) r[2] += L[2];
        }
        out_epot[s] = lj_le_forces(n, pos, type, L, delta, nt, sig2, eps4, rc, shift, f, w);
        ekin = 0;
        double kxy = 0;
        for (int i = 0; i < n; i++) {
            double *v = &vel[3 * i], mr = 1.0 / mass[i];
            for (int k = 0; k < 3; k++) v[k] += 0.5 * dt * mr * f[3 * i + k];
            v[0] -= gamma * 0.5 * dt * v[1];
            ekin += 0.5 * mass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        }
        sc = nhc_half(vnh, qnh, ekin, kT, nf, dt);
        ekin = 0;
        for (int i = 0; i < n; i++) {
            double *v = &vel[3 * i];
            for (int k = 0; k < 3; k++) v[k] *= sc;
            ekin += 0.5 * mass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            kxy += mass[i] * v[0] * v[1];
        }
        out_temp[s] = 2.0 * ekin / (nf * OR_KB);
        out_vnh0[s] = vnh[0];
        out_pxy[s] = (kxy + w[1]) / vol;
        out_delta[s] = delta;
    }
    free(f);
    return 0;
}

/* Lees-Edwards LJ forces of a configuration at offset delta (all pairs). */
double or_lj_le_forces(int n, const double *pos, const int32_t *type, const double *L, double delta, int nt,
                       const double *sig2, const double *eps4, double rc, int shift, double *f, double *w) {
    return lj_le_forces(n, pos, type, L, delta, nt, sig2, eps4, rc, shift, f, w);
}

/* ----------------------------------------------------------------------
 * Point-charge Ewald sums in the Lees-Edwards (sliding brick) cell, and
 * the chain/SLLOD MD of flexible point-charge molecules that uses them.
 * No reference code: the reference has no shear.  The images of the box
 * under planar Couette shear with offset d are the lattice a1 = (Lx, 0, 0),
 * a2 = (d, Ly, 0), a3 = (0, 0, Lz); its reciprocal vectors give
 * k(n) = 2 pi (nx / Lx, (ny - nx d / Lx) / Ly, nz / Lz).  The reciprocal
 * sum is the reference's (EwaldForce::set_up + reciprocal_term,
 * src/forces/EwaldForce.cpp:198-257, 529-698) over the half space of n with
 * |k| < kcut for that lattice; d and d + Lx describe the same lattice, so
 * d is first reduced to [-Lx/2, Lx/2].  Parity unpinned: checked by the
 * properties of the lattice sum (independence of alpha, of d -> d + Lx, the
 * unsheared sum at d = 0, forces as the energy's derivative).
 * ---------------------------------------------------------------------- */
double or_ewald_recip_le(int n, const double *pos, const double *q, const double *L, double delta,
                         double alpha, double kcut, double *f, double *w, int *nk_out) {
    double kc2 = kcut * kcut, aR4 = 1.0 / (4.0 * alpha * alpha);
    double dd = delta - L[0] * floor(delta / L[0] + 0.5), t = dd / L[0];
    int nmax[3];
    for (int d = 0; d < 3; d++) nmax[d] = (int)(kcut * L[d] / (2 * OR_PI));
    int nyr = nmax[1] + nmax[0] + 1;   /* |ny - nx t| < kcut Ly / 2 pi for every |t| <= 1/2 */
    double vol = L[0] * L[1] * L[2], pi4V = 4.0 * OR_PI * (1.0 / vol), pi8V = 2.0 * pi4V;
    double *sc = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1)), pe = 0;
    int nk = 0;
    for (int nx = 0; nx <= nmax[0]; nx++)
        for (int ny = -nyr; ny <= nyr; ny++)
            for (int nz = -nmax[2]; nz <= nmax[2]; nz++) {
                if (!(nx > 0 || (nx == 0 && ny > 0) || (nx == 0 && ny == 0 && nz > 0))) continue;
                double k[3] = {2.0 * OR_PI * nx / L[0], 2.0 * OR_PI * (ny - nx * t) / L[1],
                               2.0 * OR_PI * nz / L[2]};
                double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                if (!(k2 < kc2)) continue;
                nk++;
                double expK = exp(-k2 * aR4) / k2, ss = 0, cs = 0;
                for (int i = 0; i < n; i++) {
                    double a = pos[3 * i] * k[0] + pos[3 * i + 1] * k[1] + pos[3 * i + 2] * k[2];
                    sc[2 * i] = q[i] * sin(a);
                    sc[2 * i + 1] = q[i] * cos(a);
                    ss += sc[2 * i];
                    cs += sc[2 * i + 1];
                }
                double e = pi4V * expK * (ss * ss + cs * cs);
                pe += e;
                double coeff = 2.0 * (aR4 + 1.0 / k2);
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) w[3 * a + b] += (a == b ? e : 0.0) - e * coeff * k[a] * k[b];
                double b = pi8V * expK;
                for (int i = 0; i < n; i++) {
                    double val = b * (sc[2 * i] * cs - sc[2 * i + 1] * ss);
                    for (int d = 0; d < 3; d++) f[3 * i + d] += k[d] * val;
                }
            }
    free(sc);
    if (nk_out) *nk_out = nk;
    return pe;
}

/* Ewald real space with Lees-Edwards images: q_i q_j erfc(a r)/r over all
 * pairs of different molecules within rc (EwaldForce::real_term,
 * EwaldForce.cpp:296-527, whose pair list holds no same-molecule pair of a
 * water).  Adds forces and the virial, returns the energy. */
double or_ewald_real_le(int n, const double *pos, const double *q, const int32_t *mol, const double *L,
                        double delta, double alpha, double rc, double *f, double *w) {
    double rc2 = rc * rc, a2 = alpha * alpha, a2pi = 2.0 * alpha / OR_SQRT_PI, energy = 0;
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            if (mol[i] == mol[j]) continue;
            double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                           pos[3 * j + 2] - pos[3 * i + 2]};
            pbc_le(d, L, delta);
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (!(r2 < rc2)) continue;
            double qij = q[i] * q[j], r = sqrt(r2);
            double e = erfc(alpha * r) / r;
            double fs = (e + a2pi * exp(-a2 * r2)) / r2;
            energy += qij * e;
            double fij[3] = {-qij * fs * d[0], -qij * fs * d[1], -qij * fs * d[2]};
            for (int k = 0; k < 3; k++) { f[3 * i + k] += fij[k]; f[3 * j + k] -= fij[k]; }
            vir_add(w, fij, d);
        }
    return energy;
}

/* Harmonic bonds and angles (BondForce::compute, BondForce.cpp:37-110;
 * AngleForce::compute, AngleForce.cpp:34-130): U = k/2 (r - r0)^2 and
 * k/2 (t - t0)^2 (t0 in radians), cos t clamped at -0.9999999.  Each class
 * adds f_a r_b of its own vectors (r12 = r1 - r2; r2 - r1 and r2 - r3 for
 * the angle) to a local virial that it subtracts from Ensemble::virial,
 * which is what w receives.  bonds: [nb][3] (a1 a2 type), bpar [type][2]
 * (r0, k); angles: [na][4] (a1 apex a3 type), apar [type][2] (t0, k). */
void or_bonded(int nb, const int32_t *bonds, const double *bpar, int na, const int32_t *angles,
               const double *apar, const double *pos, const double *L, double *f, double *w,
               double *e_bond, double *e_angle) {
    double eb = 0, ea = 0;
    for (int b = 0; b < nb; b++) {
        int i = bonds[3 * b], j = bonds[3 * b + 1], t = bonds[3 * b + 2];
        double x[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
        pbc(x, L);
        double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]), dr = r - bpar[2 * t], k = bpar[2 * t + 1];
        eb += 0.5 * k * dr * dr;
        double s = -k * dr / r;
        for (int p = 0; p < 3; p++) {
            f[3 * i + p] += s * x[p];
            f[3 * j + p] -= s * x[p];
            for (int c = 0; c < 3; c++) w[3 * p + c] -= s * x[p] * x[c];
        }
    }
    for (int a = 0; a < na; a++) {
        int i1 = angles[4 * a], i2 = angles[4 * a + 1], i3 = angles[4 * a + 2], t = angles[4 * a + 3];
        double r12[3], r32[3];
        for (int p = 0; p < 3; p++) {
            r12[p] = pos[3 * i2 + p] - pos[3 * i1 + p];
            r32[p] = pos[3 * i2 + p] - pos[3 * i3 + p];
        }
        pbc(r12, L);
        pbc(r32, L);
        double d12r = 1.0 / sqrt(r12[0] * r12[0] + r12[1] * r12[1] + r12[2] * r12[2]);
        double d32r = 1.0 / sqrt(r32[0] * r32[0] + r32[1] * r32[1] + r32[2] * r32[2]);
        double cs = (r12[0] * r32[0] + r12[1] * r32[1] + r12[2] * r32[2]) * d12r * d32r;
        if (cs < -0.9999999) cs = -0.9999999;
        double isn = 1.0 / sqrt(1.0 - cs * cs), diff = acos(cs) - apar[2 * t], k = apar[2 * t + 1];
        ea += 0.5 * k * diff * diff;
        double v = k * diff;
        for (int p = 0; p < 3; p++) {
            double u12 = r12[p] * d12r, u32 = r32[p] * d32r;
            double f1 = v * d12r * isn * (u12 * cs - r32[p] * d32r);
            double f3 = v * d32r * isn * (u32 * cs - r12[p] * d12r);
            f[3 * i1 + p] += f1;
            f[3 * i2 + p] -= f1 + f3;
            f[3 * i3 + p] += f3;
            for (int c = 0; c < 3; c++) w[3 * p + c] -= f1 * r12[c] + f3 * r32[c];
        }
    }
    *e_bond = eb;
    *e_angle = ea;
}

/* All terms of a flexible point-charge model at offset delta: LJ (shifted at
 * rc when shift, every pair of different molecules), Ewald real space,
 * reciprocal space in the sheared cell, the intramolecular erf correction
 * with its forces (molecules of ns consecutive sites, excluded pairs from
 * off/ex), bonds and angles.  e[7] = {vdw, real, long, intra, bond, angle,
 * k count}; f and w are overwritten; w holds Ensemble::virial + longVirial. */
void or_flex_le_forces(int n, int ns, const double *pos, const int32_t *type, const int32_t *mol,
                       const double *q, const double *L, double delta, int nt, const double *sig2,
                       const double *eps4, double rc, int shift, double alpha, double kcut,
                       const int32_t *off, const int32_t *ex, int nb, const int32_t *bonds, const double *bpar,
                       int na, const int32_t *angles, const double *apar, double *f, double *w, double *e) {
    double *ft = (double *)malloc(sizeof(double) * 3 * n), wt[9];
    int nk = 0;
    e[0] = lj_le_forces(n, pos, type, L, delta, nt, sig2, eps4, rc, shift, f, w);
    e[1] = or_ewald_real_le(n, pos, q, mol, L, delta, alpha, rc, f, w);
    memset(ft, 0, sizeof(double) * 3 * n);
    memset(wt, 0, sizeof(wt));
    e[2] = or_ewald_recip_le(n, pos, q, L, delta, alpha, kcut, ft, wt, &nk);
    for (int k = 0; k < 3 * n; k++) f[k] += ft[k];
    for (int k = 0; k < 9; k++) w[k] += wt[k];
    e[3] = or_ewald_intra(n / ns, ns, pos, q, L, alpha, off, ex, 0, f);
    or_bonded(nb, bonds, bpar, na, angles, apar, pos, L, f, w, &e[4], &e[5]);
    e[6] = nk;
    free(ft);
}

/* The chain / SLLOD velocity-Verlet of or_lj_nhc_md for flexible molecules
 * with the forces of or_flex_le_forces, each molecule wrapped by its centre
 * of mass (y first, moving x by -/+ delta under shear; then x and z).
 * Outputs per step: the sum of the force terms' energies, 2 KE / (Nf kB),
 * the first chain velocity, P_xy = (sum m v_x v_y + W_xy) / V and delta. */
int or_flex_nhc_md(int n, int ns, double *pos, double *vel, const double *mass, const int32_t *type,
                   const int32_t *mol, const double *q, const double *L, int nt, const double *sig2,
                   const double *eps4, double rc, int shift, double alpha, double kcut, const int32_t *off,
                   const int32_t *ex, int nb, const int32_t *bonds, const double *bpar, int na,
                   const int32_t *angles, const double *apar, double dt, double T, double tau, double gamma,
                   int ndf, int nsteps, double *out_epot, double *out_temp, double *out_vnh0, double *out_pxy,
                   double *out_delta) {
    double *f = (double *)malloc(sizeof(double) * 3 * n);
    double w[9], e[7];
    const double kT = OR_KB * T, nf = (double)ndf, vol = L[0] * L[1] * L[2];
    double qnh[4], vnh[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; k++) qnh[k] = kT * tau * tau;
    qnh[0] *= nf;
    double delta = 0.0;
    const int nmol = n / ns;
    or_flex_le_forces(n, ns, pos, type, mol, q, L, delta, nt, sig2, eps4, rc, shift, alpha, kcut, off, ex, nb,
                      bonds, bpar, na, angles, apar, f, w, e);
    for (int s = 0; s < nsteps; s++) {
        double ekin = 0;
        for (int i = 0; i < n; i++)
            ekin += 0.5 * mass[i] * (vel[3 * i] * vel[3 * i] + vel[3 * i + 1] * vel[3 * i + 1] + vel[3 * i + 2] * vel[3 * i + 2]);
        double sc = nhc_half(vnh, qnh, ekin, kT, nf, dt);
        delta = fmod(delta + gamma * L[1] * dt, L[0]);
        if (delta < 0) delta += L[0];
        for (int i = 0; i < n; i++) {
            double *v = &vel[3 * i], *r = &pos[3 * i], mr = 1.0 / mass[i];
            for (int k = 0; k < 3; k++) v[k] *= sc;
            v[0] -= gamma * 0.5 * dt * v[1];
            for (int k = 0; k < 3; k++) v[k] += 0.5 * dt * mr * f[3 * i + k];
            r[0] += dt * v[0] + gamma * dt * (r[1] + 0.5 * dt * v[1]);
            r[1] += dt * v[1];
            r[2] += dt * v[2];
        }
        for (int m = 0; m < nmol; m++) {
            double c[3] = {0, 0, 0}, M = 0, sh[3] = {0, 0, 0};
            for (int a = 0; a < ns; a++) {
                int i = m * ns + a;
                for (int k = 0; k < 3; k++) c[k] += mass[i] * pos[3 * i + k];
                M += mass[i];
            }
            for (int k = 0; k < 3; k++) c[k] /= M;
            if (c[1] >= L[1] / 2.0) { sh[1] = -L[1]; sh[0] = -delta; }
            else if (c[1] < -L[1] / 2.0) { sh[1] = L[1]; sh[0] = delta; }
            if (gamma == 0.0) sh[0] = 0.0;
            double cx = c[0] + sh[0], cz = c[2];
            while (cx >= L[0] / 2.0) cx -= L[0];
            while (cx < -L[0] / 2.0) cx += L[0];
            while (cz >= L[2] / 2.0) cz -= L[2];
            while (cz < -L[2] / 2.0) cz += L[2];
            sh[0] = cx - c[0];
            sh[2] = cz - c[2];
            for (int a = 0; a < ns; a++)
                for (int k = 0; k < 3; k++) pos[3 * (m * ns + a) + k] += sh[k];
        }
        or_flex_le_forces(n, ns, pos, type, mol, q, L, delta, nt, sig2, eps4, rc, shift, alpha, kcut, off, ex,
                          nb, bonds, bpar, na, angles, apar, f, w, e);
        out_epot[s] = e[0] + e[1] + e[2] + e[3] + e[4] + e[5];
        ekin = 0;
        double kxy = 0;
        for (int i = 0; i < n; i++) {
            double *v = &vel[3 * i], mr = 1.0 / mass[i];
            for (int k = 0; k < 3; k++) v[k] += 0.5 * dt * mr * f[3 * i + k];
            v[0] -= gamma * 0.5 * dt * v[1];
            ekin += 0.5 * mass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        }
        sc = nhc_half(vnh, qnh, ekin, kT, nf, dt);
        ekin = 0;
        for (int i = 0; i < n; i++) {
            double *v = &vel[3 * i];
            for (int k = 0; k < 3; k++) v[k] *= sc;
            ekin += 0.5 * mass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            kxy += mass[i] * v[0] * v[1];
        }
        out_temp[s] = 2.0 * ekin / (nf * OR_KB);
        out_vnh0[s] = vnh[0];
        out_pxy[s] = (kxy + w[1]) / vol;
        out_delta[s] = delta;
    }
    free(f);
    return 0;
}
